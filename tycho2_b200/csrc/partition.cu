// One partition of a multi-partition mesh: the incoming psi on faces toward
// other partitions (psiBound), and the exchange of those values between
// partitions (the reference's CommSides).
//
// Reference semantics:
//   Transport::populateLocalPsiBound  src/Transport.cc:740-776 -- a face
//       whose neighbour is another partition reads psiBound(g, fv, a, side)
//   Util::sweepLocal                  src/Util.cc:138-145
//   CommSides::CommSides / commSides  src/CommSides.cc:48-240 -- toward each
//       neighbouring partition, every (cell, face, angle) with the face
//       outgoing sends psi at the face's vertices in face-vertex order; the
//       receiver stores it at psiBound(g, fv, angle, its side of that face)
//   SweeperPBJ::sweep                 src/SweeperPBJ.cc:168-211 (L1 change of psi)
//
// The values live in ghost psi rows (set up in Sweeper::init): the sweep
// kernels read them as ordinary upwind rows.
#include "sweeper.hpp"

#include <cstring>
#include <unordered_map>

#include "devmem.hpp"
#include "status.hpp"

namespace tycho {

#define TY_CUDA(expr)                                                                  \
    do {                                                                               \
        cudaError_t e_ = (expr);                                                       \
        if (e_ != cudaSuccess) {                                                       \
            err = std::string(#expr) + ": " + cudaGetErrorString(e_);                  \
            return e_ == cudaErrorMemoryAllocation ? kErrOom : kErrCuda;               \
        }                                                                              \
    } while (0)

#define TY_CHECK(expr)                  \
    do {                                \
        int s_ = (expr);                \
        if (s_ != kOk) return s_;       \
    } while (0)

namespace {

constexpr uint64_t kSkip = ~0ull;

// Packet k ([3][G] values) to ghost row idx[k] (identity when idx is null;
// kSkip: not a direction of this sweeper), in FP64 and, when g32 is set,
// FP32.  One thread per value.
__global__ void ghost_write_kernel(const double *__restrict__ src, const uint64_t *__restrict__ idx, uint64_t n,
                                   uint32_t G, double *__restrict__ g64, float *__restrict__ g32)
{
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t per = 3ull * G;
    if (i >= n * per) return;
    const uint64_t k = i / per, e = i - k * per;
    const uint64_t row = idx ? idx[k] : k;
    if (row == kSkip) return;
    const uint64_t v = e / G, g = e - v * G;
    const uint64_t o = row * 4 * G + v * G + g;
    const double x = src[i];
    g64[o] = x;
    if (g32) g32[o] = (float)x;
}

// Packet k from psi row row[k] at the face's cell vertices (vtx[k], 2 bits
// per face vertex).  One thread per value.
template <typename Real>
__global__ void side_pack_kernel(const Real *__restrict__ psi, const uint64_t *__restrict__ row,
                                 const uint32_t *__restrict__ vtx, uint64_t n, uint32_t G,
                                 double *__restrict__ dst)
{
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t per = 3ull * G;
    if (i >= n * per) return;
    const uint64_t k = i / per, e = i - k * per;
    const uint32_t v = (uint32_t)(e / G), g = (uint32_t)(e - (uint64_t)v * G);
    const uint32_t cv = (vtx[k] >> (2 * v)) & 3u;
    dst[i] = (double)psi[row[k] * 4 * G + (uint64_t)cv * G + g];
}

// L1 of a - b and of a (per-block partials, summed on the host in block
// order), then b = a.
__global__ void l1_change_kernel(const double *__restrict__ a, double *__restrict__ b, uint64_t n,
                                 double *__restrict__ part)
{
    __shared__ double sd[256], sn[256];
    double d = 0.0, m = 0.0;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const double x = a[i];
        d += fabs(x - b[i]);
        m += fabs(x);
        b[i] = x;
    }
    sd[threadIdx.x] = d;
    sn[threadIdx.x] = m;
    __syncthreads();
    for (unsigned s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            sd[threadIdx.x] += sd[threadIdx.x + s];
            sn[threadIdx.x] += sn[threadIdx.x + s];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = sd[0];
        part[2 * blockIdx.x + 1] = sn[0];
    }
}

unsigned blocks_for(uint64_t n, unsigned bs) { return (unsigned)((n + bs - 1) / bs); }

// Orders `s` after the work queued so far on `from`.
cudaError_t follow(cudaStream_t s, cudaStream_t from)
{
    if (s == from) return cudaSuccess;
    cudaEvent_t ev;
    cudaError_t e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    if (e != cudaSuccess) return e;
    e = cudaEventRecord(ev, from);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(s, ev, 0);
    cudaEventDestroy(ev);
    return e;
}

}  // namespace

double *Sweeper::ghost64() const
{
    return static_cast<double *>(d_psi_) + psi_size();
}

float *Sweeper::ghost32() const
{
    if (!fp32_) return nullptr;
    return static_cast<float *>(d_psi_) + 2 * (nc_ + n_bound_) * (uint64_t)A_ * 4 * G_;
}

int Sweeper::set_psi_bound(const double *psi_bound, std::string &err)
{
    if (!psi_bound) { err = "psi_bound is required"; return kErrArg; }
    TY_CUDA(cudaSetDevice(device_));
    if (!n_bound_) return kOk;  // no face toward another partition reads it
    // this sweeper's directions of each bound side, contiguous in the layout
    const uint64_t per_side = (uint64_t)A_ * 3 * G_;
    std::vector<double> packed(n_bound_ * per_side);
    for (uint64_t b = 0; b < n_bound_; ++b)
        std::memcpy(&packed[b * per_side],
                    psi_bound + ((bound_side_[b] * (uint64_t)n_angles_full_ + angle_begin_) * 3) * G_,
                    sizeof(double) * per_side);
    double *d = nullptr;
    TY_CUDA(dev_malloc(&d, sizeof(double) * packed.size(), stream_));
    cudaError_t e = cudaMemcpyAsync(d, packed.data(), sizeof(double) * packed.size(), cudaMemcpyHostToDevice, stream_);
    const uint64_t n = n_bound_ * (uint64_t)A_;
    if (e == cudaSuccess) {
        ghost_write_kernel<<<blocks_for(n * 3 * G_, 256), 256, 0, stream_>>>(d, nullptr, n, (uint32_t)G_,
                                                                              ghost64(), ghost32());
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
    dev_free(d, stream_);
    TY_CUDA(e);
    return kOk;
}

int Sweeper::get_psi_bound(double *psi_bound, std::string &err)
{
    if (!psi_bound) { err = "psi_bound is required"; return kErrArg; }
    TY_CUDA(cudaSetDevice(device_));
    const uint64_t ns = tables_->n_sides;
    std::memset(psi_bound, 0, sizeof(double) * ns * n_angles_full_ * 3 * G_);
    if (!n_bound_) return kOk;
    const uint64_t row = 4ull * G_;
    std::vector<double> g(n_bound_ * (uint64_t)A_ * row);
    TY_CUDA(cudaMemcpyAsync(g.data(), ghost64(), sizeof(double) * g.size(), cudaMemcpyDeviceToHost, stream_));
    TY_CUDA(cudaStreamSynchronize(stream_));
    for (uint64_t b = 0; b < n_bound_; ++b)
        for (int a = 0; a < A_; ++a)
            std::memcpy(psi_bound + ((bound_side_[b] * (uint64_t)n_angles_full_ + angle_begin_ + a) * 3) * G_,
                        &g[(b * A_ + a) * row], sizeof(double) * 3 * G_);
    return kOk;
}

// The packets toward partition q in the reference's order: cells, faces,
// directions (src/CommSides.cc:68-95); the face vertices in fv order
// (faceToCellVrtx, src/CommSides.cc:160-164).
int Sweeper::side_link_build(uint64_t q, SideLink *&l, std::string &err)
{
    const MeshTables &t = *tables_;
    if (q == t.partition || (t.n_partitions && q >= t.n_partitions)) {
        err = "not a neighbouring partition: " + std::to_string(q);
        return kErrArg;
    }
    l = &links_[q];
    if (l->built) return kOk;
    std::vector<uint64_t> rows;
    std::vector<uint32_t> vtx;
    l->n_recv = 0;
    if (!t.adj_rank.empty())
        for (uint64_t c = 0; c < nc_; ++c)
            for (int f = 0; f < 4; ++f) {
                if (t.adj_cell[c * 4 + f] != kNone || t.adj_rank[c * 4 + f] != q) continue;
                uint32_t fv = 0;
                for (int k = 0; k < 3; ++k) fv |= (uint32_t)(t.face_to_cell[(c * 4 + f) * 3 + k] & 3u) << (2 * k);
                const uint64_t gside = t.side_gid[t.side[c * 4 + f]];
                for (int a = 0; a < A_; ++a) {
                    if (omega_dot_n(quad_, a, &t.normal[(c * 4 + f) * 3]) > 0) {
                        l->send_gside.push_back(gside);
                        l->send_angle.push_back((uint32_t)(angle_begin_ + a));
                        rows.push_back(c * (uint64_t)A_ + a);
                        vtx.push_back(fv);
                    } else {
                        ++l->n_recv;
                    }
                }
            }
    if (!rows.empty()) {
        TY_CUDA(dev_malloc(&l->d_send_row, sizeof(uint64_t) * rows.size(), stream_));
        TY_CUDA(dev_malloc(&l->d_send_vtx, sizeof(uint32_t) * vtx.size(), stream_));
        TY_CUDA(cudaMemcpyAsync(l->d_send_row, rows.data(), sizeof(uint64_t) * rows.size(), cudaMemcpyHostToDevice,
                                stream_));
        TY_CUDA(cudaMemcpyAsync(l->d_send_vtx, vtx.data(), sizeof(uint32_t) * vtx.size(), cudaMemcpyHostToDevice,
                                stream_));
        TY_CUDA(cudaStreamSynchronize(stream_));
    }
    l->built = true;
    return kOk;
}

int Sweeper::side_counts(uint64_t q, uint64_t &n_send, uint64_t &n_recv, std::string &err)
{
    TY_CUDA(cudaSetDevice(device_));
    SideLink *l = nullptr;
    TY_CHECK(side_link_build(q, l, err));
    n_send = l->send_gside.size();
    n_recv = l->n_recv;
    return kOk;
}

int Sweeper::side_send_list(uint64_t q, uint64_t *gside, uint32_t *angle, std::string &err)
{
    TY_CUDA(cudaSetDevice(device_));
    SideLink *l = nullptr;
    TY_CHECK(side_link_build(q, l, err));
    if (gside) std::memcpy(gside, l->send_gside.data(), sizeof(uint64_t) * l->send_gside.size());
    if (angle) std::memcpy(angle, l->send_angle.data(), sizeof(uint32_t) * l->send_angle.size());
    return kOk;
}

int Sweeper::side_pack(uint64_t q, double *dst, cudaStream_t s, bool sync, std::string &err)
{
    TY_CUDA(cudaSetDevice(device_));
    SideLink *l = nullptr;
    TY_CHECK(side_link_build(q, l, err));
    const uint64_t n = l->send_gside.size();
    if (!n) return kOk;
    if (!dst) { err = "dst is required"; return kErrArg; }
    // the resident psi: the last sweep's precision
    TY_CUDA(follow(stream_, s));
    const unsigned grid = blocks_for(n * 3 * G_, 256);
    if (last_psi_prec_ == 1)
        side_pack_kernel<float><<<grid, 256, 0, stream_>>>(static_cast<const float *>(d_psi_), l->d_send_row,
                                                            l->d_send_vtx, n, (uint32_t)G_, dst);
    else
        side_pack_kernel<double><<<grid, 256, 0, stream_>>>(static_cast<const double *>(d_psi_), l->d_send_row,
                                                             l->d_send_vtx, n, (uint32_t)G_, dst);
    TY_CUDA(cudaGetLastError());
    TY_CUDA(follow(s, stream_));
    if (sync) TY_CUDA(cudaStreamSynchronize(stream_));
    return kOk;
}

int Sweeper::side_link(uint64_t q, uint64_t n, const uint64_t *gside, const uint32_t *angle, std::string &err)
{
    TY_CUDA(cudaSetDevice(device_));
    SideLink *l = nullptr;
    TY_CHECK(side_link_build(q, l, err));
    if (n && (!gside || !angle)) { err = "gside and angle are required"; return kErrArg; }
    const MeshTables &t = *tables_;
    // global side id -> this partition's side (TychoMesh::getGLSide)
    std::unordered_map<uint64_t, uint64_t> gl;
    gl.reserve(n_bound_ * 2);
    for (uint64_t b = 0; b < n_bound_; ++b) gl.emplace(t.side_gid[bound_side_[b]], b);
    std::vector<uint64_t> ghost(n);
    for (uint64_t k = 0; k < n; ++k) {
        auto it = gl.find(gside[k]);
        if (it == gl.end()) {
            err = "packet for global side " + std::to_string(gside[k]) + ", which faces no other partition here";
            return kErrArg;
        }
        if (angle[k] >= (uint32_t)n_angles_full_) { err = "packet angle out of range"; return kErrArg; }
        const int64_t a = (int64_t)angle[k] - angle_begin_;
        ghost[k] = a >= 0 && a < A_ ? it->second * (uint64_t)A_ + (uint64_t)a : kSkip;
    }
    dev_free(l->d_recv_ghost, stream_);
    l->d_recv_ghost = nullptr;
    l->n_link = n;
    if (n) {
        TY_CUDA(dev_malloc(&l->d_recv_ghost, sizeof(uint64_t) * n, stream_));
        TY_CUDA(cudaMemcpyAsync(l->d_recv_ghost, ghost.data(), sizeof(uint64_t) * n, cudaMemcpyHostToDevice, stream_));
        TY_CUDA(cudaStreamSynchronize(stream_));
    }
    return kOk;
}

int Sweeper::side_unpack(uint64_t q, const double *src, cudaStream_t s, bool sync, std::string &err)
{
    TY_CUDA(cudaSetDevice(device_));
    auto it = links_.find(q);
    if (it == links_.end() || !it->second.built) {
        err = "no link with partition " + std::to_string(q) + " (tycho_sweeper_side_link first)";
        return kErrMissing;
    }
    SideLink &l = it->second;
    if (!l.n_link) return kOk;
    if (!src) { err = "src is required"; return kErrArg; }
    TY_CUDA(follow(stream_, s));
    ghost_write_kernel<<<blocks_for(l.n_link * 3 * G_, 256), 256, 0, stream_>>>(
        src, l.d_recv_ghost, l.n_link, (uint32_t)G_, ghost64(), ghost32());
    TY_CUDA(cudaGetLastError());
    TY_CUDA(follow(s, stream_));
    if (sync) TY_CUDA(cudaStreamSynchronize(stream_));
    return kOk;
}

int Sweeper::psi_change(double &diff, double &norm, std::string &err)
{
    TY_CUDA(cudaSetDevice(device_));
    if (last_psi_prec_ == 1) { err = "the resident psi is an FP32 sweep's"; return kErrArg; }
    const uint64_t n = psi_size();
    if (!d_psi_prev_) {
        TY_CUDA(dev_malloc(&d_psi_prev_, sizeof(double) * std::max<uint64_t>(n, 1), stream_));
        TY_CUDA(cudaMemsetAsync(d_psi_prev_, 0, sizeof(double) * n, stream_));
    }
    constexpr unsigned kBlocks = 592, kThreads = 256;
    double *part = nullptr;
    TY_CUDA(dev_malloc(&part, sizeof(double) * 2 * kBlocks, stream_));
    l1_change_kernel<<<kBlocks, kThreads, 0, stream_>>>(static_cast<const double *>(d_psi_), d_psi_prev_, n, part);
    cudaError_t e = cudaGetLastError();
    std::vector<double> h(2 * kBlocks);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h.data(), part, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, stream_);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
    dev_free(part, stream_);
    TY_CUDA(e);
    diff = norm = 0.0;
    for (unsigned b = 0; b < kBlocks; ++b) {
        diff += h[2 * b];
        norm += h[2 * b + 1];
    }
    return kOk;
}

}  // namespace tycho
