// Streaming kernels around the wavefront sweep, and deterministic vector
// kernels for the outer solvers.  This translation unit is compiled with
// -fmad=false: the FP64 wavefront kernel, the per-item face terms, the
// scalar flux and the scattering source keep the reference's rounding.
#include "device_ops.hpp"

#include <cstring>
#include "devmem.hpp"
#include "sweep_kernels.cuh"
#include "sweep_tiles.cuh"
#include "sweep_records.cuh"
#include "stream_ops.cuh"

namespace tycho {

template cudaError_t launch_level<double>(int, const LevelArgs &, uint64_t, uint64_t, cudaStream_t);
template cudaError_t launch_dataflow<double>(int, const LevelArgs &, const DataflowArgs &, unsigned, cudaStream_t);
template cudaError_t dataflow_blocks_per_sm<double>(int, int *);
template cudaError_t launch_level_tile<double>(int, const LevelArgs &, uint64_t, uint64_t, cudaStream_t);
template cudaError_t launch_dataflow_tile<double>(int, const LevelArgs &, const DataflowArgs &, unsigned, cudaStream_t);
template cudaError_t tile_dataflow_blocks_per_sm<double>(int, int *);
template cudaError_t launch_item_records<double>(const LevelArgs &, uint64_t, void *, cudaStream_t);
template cudaError_t launch_level_record<double>(int, const LevelArgs &, const void *, uint64_t, uint64_t, cudaStream_t);
template cudaError_t launch_dataflow_record<double>(int, const LevelArgs &, const void *, const DataflowArgs &, unsigned,
                                               cudaStream_t);
template cudaError_t record_dataflow_blocks_per_sm<double>(int, int, int *);
template cudaError_t launch_persist_record<double>(int, const LevelArgs &, const void *, const uint64_t *, uint32_t,
                                                   unsigned long long *, const DataflowArgs &, unsigned, cudaStream_t);
template cudaError_t record_persist_blocks_per_sm<double>(int, int, int *);
template cudaError_t launch_direct_subset<double>(const LevelArgs &, const void *, const uint32_t *, uint64_t, uint64_t,
                                                   cudaStream_t);
template cudaError_t launch_direct_level<double>(int, const LevelArgs &, const void *, uint64_t, uint64_t, cudaStream_t,
                                                  bool);
template cudaError_t launch_compact_records<double>(const LevelArgs &, uint64_t, void *, cudaStream_t);
template cudaError_t launch_direct_dataflow<double>(const LevelArgs &, const void *, bool, const DataflowArgs &,
                                                     unsigned, cudaStream_t);
template cudaError_t direct_dataflow_blocks_per_sm<double>(int, bool, int *);

namespace {

__global__ void item_abar_kernel(const uint32_t *__restrict__ items, uint64_t n, uint32_t A,
                                 const double *__restrict__ normal, const double *__restrict__ area,
                                 const double *__restrict__ omega, double4 *abar64, float4 *abar32)
{
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t ca = items[i];
    if (ca == kSentinel) {  // level padding: never read by the sweep
        abar64[i] = make_double4(0.0, 0.0, 0.0, 0.0);
        if (abar32) abar32[i] = make_float4(0.f, 0.f, 0.f, 0.f);
        return;
    }
    const uint32_t c = ca / A, a = ca - c * A;
    const double xi = omega[a], eta = omega[A + a], mu = omega[2 * A + a];
    double ab[4];
#pragma unroll
    for (int f = 0; f < 4; ++f) {
        const double *nrm = normal + ((size_t)c * 4 + f) * 3;
        // TychoMesh.cc:219-221 then Transport.cc:694-701
        const double odn = xi * nrm[0] + eta * nrm[1] + mu * nrm[2];
        ab[f] = area[(size_t)c * 4 + f] * odn;
    }
    abar64[i] = make_double4(ab[0], ab[1], ab[2], ab[3]);
    if (abar32) abar32[i] = make_float4((float)ab[0], (float)ab[1], (float)ab[2], (float)ab[3]);
}

template <typename Real>
__global__ void psi_to_phi_kernel(const Real *__restrict__ psi, const double *__restrict__ w,
                                  double *__restrict__ phi, uint64_t nc, uint32_t A, uint32_t G)
{
    // 8..15 groups: one element per thread (a warp's 32 elements share one
    // 128-byte line per angle); fewer or more: four elements per thread, 16
    // bytes per angle, eight angles in flight (measured on the 64^3 G=16
    // pass: 11.6 -> 10.9 ms FP32, 18.9 -> 17.2 ms FP64; at G=8 the element
    // form is as fast)
    if (G >= 8 && G < 16) {
        const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
        if (i >= nc * 4 * G) return;
        phi[i] = psi_to_phi_elem(psi, w, i, A, G);
        return;
    }
    const uint64_t i = 4 * ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x);
    if (i >= nc * 4 * G) return;
    double s[4];
    psi_to_phi_quad(psi, w, i, A, G, s);
    reinterpret_cast<double2 *>(phi + i)[0] = make_double2(s[0], s[1]);
    reinterpret_cast<double2 *>(phi + i)[1] = make_double2(s[2], s[3]);
}

// One thread per (cell, group): the group's four vertex elements (groups
// fastest, so a warp writes runs of G consecutive elements per vertex).
__global__ void scatter_source_kernel(const double *__restrict__ phi, const double *__restrict__ q,
                                      const double *__restrict__ sigma_s,
                                      const double *__restrict__ scat, double *__restrict__ iso,
                                      float *__restrict__ iso32, uint64_t nc, uint32_t G)
{
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nc * G) return;
    const uint64_t c = t < (1ull << 32) ? (uint64_t)((uint32_t)t / G) : t / G;
    const uint32_t g = (uint32_t)(t - c * G);
    double s[4];
    scatter_cell_group(phi, q, sigma_s, scat, c, g, G, s);
    const uint64_t base = c * 4 * G + g;
#pragma unroll
    for (int v = 0; v < 4; ++v) iso[base + v * G] = s[v];
    if (iso32) {
#pragma unroll
        for (int v = 0; v < 4; ++v) iso32[base + v * G] = (float)s[v];
    }
}

template <int K>
__global__ void __launch_bounds__(256)
multi_dot_kernel(const double *__restrict__ w, const double *__restrict__ V, size_t ld, int k,
                 int j0, uint64_t n, double *__restrict__ partials)
{
    double acc[K];
#pragma unroll
    for (int j = 0; j < K; ++j) acc[j] = 0.0;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const double wi = w[i];
#pragma unroll
        for (int j = 0; j < K; ++j)
            if (j0 + j < k) acc[j] = __fma_rn(wi, V[(size_t)(j0 + j) * ld + i], acc[j]);
    }
    __shared__ double sh[8][K];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int j = 0; j < K; ++j) {
        const double v = warp_sum(acc[j]);
        if (lane == 0) sh[warp][j] = v;
    }
    __syncthreads();
    if (threadIdx.x < K && j0 + (int)threadIdx.x < k) {
        double s = 0.0;
        for (int q = 0; q < 8; ++q) s += sh[q][threadIdx.x];
        partials[(size_t)blockIdx.x * 64 + j0 + threadIdx.x] = s;
    }
}

// The same inner products on 16-byte pairs (n even, 16-byte aligned
// vectors): each thread issues U x (K + 1) pair loads before its FMAs, so
// that the few-vector passes of an Arnoldi step keep enough loads in
// flight to stream at HBM rate.  Per thread: the pairs it visits in
// grid-stride order, the first element of each pair before the second.
template <int K, int U>
__global__ void __launch_bounds__(256)
multi_dot2_kernel(const double2 *__restrict__ w, const double2 *__restrict__ V, size_t ld2, int k, int j0,
                  uint64_t n2, double *__restrict__ partials)
{
    double acc[K];
#pragma unroll
    for (int j = 0; j < K; ++j) acc[j] = 0.0;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i0 = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i0 < n2; i0 += stride * U) {
        double2 wv[U], v[U][K];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const uint64_t i = i0 + u * stride;
            if (i < n2) {
                wv[u] = w[i];
#pragma unroll
                for (int j = 0; j < K; ++j)
                    if (j0 + j < k) v[u][j] = V[(size_t)(j0 + j) * ld2 + i];
            }
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            if (i0 + u * stride >= n2) break;
#pragma unroll
            for (int j = 0; j < K; ++j)
                if (j0 + j < k) {
                    acc[j] = __fma_rn(wv[u].x, v[u][j].x, acc[j]);
                    acc[j] = __fma_rn(wv[u].y, v[u][j].y, acc[j]);
                }
        }
    }
    __shared__ double sh[8][K];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int j = 0; j < K; ++j) {
        const double v = warp_sum(acc[j]);
        if (lane == 0) sh[warp][j] = v;
    }
    __syncthreads();
    if (threadIdx.x < K && j0 + (int)threadIdx.x < k) {
        double s = 0.0;
        for (int q = 0; q < 8; ++q) s += sh[q][threadIdx.x];
        partials[(size_t)blockIdx.x * 64 + j0 + threadIdx.x] = s;
    }
}

__global__ void l1_kernel(const double *__restrict__ x, const double *__restrict__ y, uint64_t n,
                          double *__restrict__ partials)
{
    double d = 0.0, m = 0.0;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const double xi = x[i];
        d += fabs(y ? xi - y[i] : xi);
        m += fabs(xi);
    }
    __shared__ double sh[8][2];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    d = warp_sum(d);
    m = warp_sum(m);
    if (lane == 0) { sh[warp][0] = d; sh[warp][1] = m; }
    __syncthreads();
    if (threadIdx.x < 2) {
        double s = 0.0;
        for (int q = 0; q < 8; ++q) s += sh[q][threadIdx.x];
        partials[(size_t)blockIdx.x * 64 + threadIdx.x] = s;
    }
}

__global__ void reduce_partials_kernel(const double *__restrict__ partials, int nblocks, int k,
                                       double *__restrict__ out)
{
    const int j = threadIdx.x;
    if (j >= k) return;
    double s = 0.0;
    for (int b = 0; b < nblocks; ++b) s += partials[(size_t)b * 64 + j];
    out[j] = s;
}

// w /= sqrt(*sq) (left as is when the norm is 0); *norm_out = sqrt(*sq).
__global__ void scale_by_norm_kernel(double *__restrict__ w, uint64_t n, const double *__restrict__ sq,
                                     double *__restrict__ norm_out)
{
    const double hn = sqrt(*sq);
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0 && norm_out) *norm_out = hn;
    if (i >= n || !(hn > 0.0)) return;
    w[i] = w[i] * (1.0 / hn);
}

__global__ void multi_axpy_kernel(double *__restrict__ w, const double *__restrict__ V, size_t ld,
                                  const double *__restrict__ h, int k, uint64_t n)
{
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double s = w[i];
    for (int j = 0; j < k; ++j) s = __fma_rn(-h[j], V[(size_t)j * ld + i], s);
    w[i] = s;
}

// The same update on 16-byte pairs, eight basis vectors' loads issued
// before their FMAs (the same operations in the same order per element).
__global__ void multi_axpy2_kernel(double2 *__restrict__ w, const double2 *__restrict__ V, size_t ld2,
                                   const double *__restrict__ h, int k, uint64_t n2)
{
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n2) return;
    double2 s = w[i];
    for (int j0 = 0; j0 < k; j0 += 8) {
        double2 v[8];
#pragma unroll
        for (int j = 0; j < 8; ++j)
            if (j0 + j < k) v[j] = V[(size_t)(j0 + j) * ld2 + i];
#pragma unroll
        for (int j = 0; j < 8; ++j)
            if (j0 + j < k) {
                const double hj = h[j0 + j];
                s.x = __fma_rn(-hj, v[j].x, s.x);
                s.y = __fma_rn(-hj, v[j].y, s.y);
            }
    }
    w[i] = s;
}

__global__ void axpby_kernel(double alpha, const double *__restrict__ x, double beta,
                             double *__restrict__ y, uint64_t n)
{
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] = __fma_rn(alpha, x[i], beta * y[i]);
}

__global__ void sub_from_kernel(const double *__restrict__ x, double *__restrict__ y, uint64_t n)
{
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] = x[i] - y[i];
}

__global__ void bump_epoch_kernel(uint32_t *epoch)
{
    const uint32_t v = *epoch + 1u;
    *epoch = v == 0u ? 1u : v;
}

inline unsigned blocks_for(uint64_t n, unsigned t = 256) { return (unsigned)((n + t - 1) / t); }

}  // namespace

cudaError_t launch_item_abar(const uint32_t *items, uint64_t n, uint32_t A, const double *normal,
                             const double *area, const double *omega, double4 *abar64,
                             float4 *abar32, cudaStream_t s)
{
    if (n == 0) return cudaSuccess;
    item_abar_kernel<<<blocks_for(n), 256, 0, s>>>(items, n, A, normal, area, omega, abar64, abar32);
    return cudaGetLastError();
}

cudaError_t launch_psi_to_phi(const void *psi, bool psi_fp32, const double *w, double *phi,
                              uint64_t nc, uint32_t A, uint32_t G, cudaStream_t s)
{
    const uint64_t n = nc * 4 * G;
    if (n == 0) return cudaSuccess;
    // one thread per element for 8..15 groups, else per four elements
    const unsigned grid = G >= 8 && G < 16 ? blocks_for(n) : blocks_for(n / 4);
    if (psi_fp32)
        psi_to_phi_kernel<float><<<grid, 256, 0, s>>>((const float *)psi, w, phi, nc, A, G);
    else
        psi_to_phi_kernel<double><<<grid, 256, 0, s>>>((const double *)psi, w, phi, nc, A, G);
    return cudaGetLastError();
}

cudaError_t launch_scatter_source(const double *phi_in, const double *q_fixed, const double *sigma_s,
                                  const double *scatter, double *iso, float *iso32, uint64_t nc,
                                  uint32_t G, cudaStream_t s)
{
    const uint64_t n = nc * G;
    if (n == 0) return cudaSuccess;
    scatter_source_kernel<<<blocks_for(n), 256, 0, s>>>(phi_in, q_fixed, sigma_s, scatter, iso, iso32, nc, G);
    return cudaGetLastError();
}

cudaError_t launch_bump_epoch(uint32_t *epoch, cudaStream_t s)
{
    bump_epoch_kernel<<<1, 1, 0, s>>>(epoch);
    return cudaGetLastError();
}

cudaError_t reducer_init(Reducer &r, cudaStream_t s)
{
    cudaError_t e = dev_malloc(&r.partials, sizeof(double) * std::max(kReduceBlocks, kDotBlocks) * 64, s);
    if (e == cudaSuccess) e = dev_malloc(&r.result, sizeof(double) * kReduceSlots, s);
    if (e == cudaSuccess) e = cudaMallocHost(&r.host, sizeof(double) * kReduceSlots);
    if (e == cudaSuccess) std::memset(r.host, 0, sizeof(double) * kReduceSlots);
    return e;
}

void reducer_free(Reducer &r, cudaStream_t s)
{
    dev_free(r.partials, s);
    dev_free(r.result, s);
    if (r.host) cudaFreeHost(r.host);
    r = Reducer();
}

// k inner products <w, V_j> into per-block partials: pairs of doubles when
// the vectors allow it, in passes of at most 8 basis vectors.
static int launch_multi_dot(const double *w, const double *V, size_t ld, int k, uint64_t n, double *partials,
                            cudaStream_t s)
{
    const bool pairs = n % 2 == 0 && ld % 2 == 0 && (reinterpret_cast<uintptr_t>(w) & 15u) == 0 &&
                       (reinterpret_cast<uintptr_t>(V) & 15u) == 0;
    if (!pairs) {
        for (int j0 = 0; j0 < k; j0 += 16)
            multi_dot_kernel<16><<<kReduceBlocks, 256, 0, s>>>(w, V, ld, k, j0, n, partials);
        return kReduceBlocks;
    }
    const double2 *w2 = reinterpret_cast<const double2 *>(w);
    const double2 *V2 = reinterpret_cast<const double2 *>(V);
    for (int j0 = 0; j0 < k;) {
        const int rem = k - j0;
        if (rem <= 2) {
            multi_dot2_kernel<2, 4><<<kDotBlocks, 256, 0, s>>>(w2, V2, ld / 2, k, j0, n / 2, partials);
            j0 += 2;
        } else if (rem <= 4) {
            multi_dot2_kernel<4, 2><<<kDotBlocks, 256, 0, s>>>(w2, V2, ld / 2, k, j0, n / 2, partials);
            j0 += 4;
        } else {
            multi_dot2_kernel<8, 1><<<kDotBlocks, 256, 0, s>>>(w2, V2, ld / 2, k, j0, n / 2, partials);
            j0 += 8;
        }
    }
    return kDotBlocks;
}

cudaError_t multi_dot_dev(const double *w, const double *V, size_t ld, int k, uint64_t n, Reducer &r, double *dst,
                          cudaStream_t s)
{
    if (k < 1 || k > 64) return cudaErrorInvalidValue;
    const int nb = launch_multi_dot(w, V, ld, k, n, r.partials, s);
    reduce_partials_kernel<<<1, 64, 0, s>>>(r.partials, nb, k, dst);
    return cudaGetLastError();
}

cudaError_t l1_pair_dev(const double *x, const double *y, uint64_t n, Reducer &r, double *dst, cudaStream_t s)
{
    l1_kernel<<<kReduceBlocks, 256, 0, s>>>(x, y, n, r.partials);
    reduce_partials_kernel<<<1, 64, 0, s>>>(r.partials, kReduceBlocks, 2, dst);
    return cudaGetLastError();
}

cudaError_t scale_by_norm(double *w, uint64_t n, const double *sq, double *norm_out, cudaStream_t s)
{
    scale_by_norm_kernel<<<blocks_for(std::max<uint64_t>(n, 1)), 256, 0, s>>>(w, n, sq, norm_out);
    return cudaGetLastError();
}

cudaError_t multi_dot(const double *w, const double *V, size_t ld, int k, uint64_t n, Reducer &r,
                      cudaStream_t s)
{
    if (k < 1 || k > 64) return cudaErrorInvalidValue;
    const int nb = launch_multi_dot(w, V, ld, k, n, r.partials, s);
    reduce_partials_kernel<<<1, 64, 0, s>>>(r.partials, nb, k, r.result);
    cudaError_t e = cudaMemcpyAsync(r.host, r.result, sizeof(double) * k, cudaMemcpyDeviceToHost, s);
    if (e != cudaSuccess) return e;
    return cudaStreamSynchronize(s);
}

cudaError_t l1_pair(const double *x, const double *y, uint64_t n, Reducer &r, cudaStream_t s)
{
    l1_kernel<<<kReduceBlocks, 256, 0, s>>>(x, y, n, r.partials);
    reduce_partials_kernel<<<1, 64, 0, s>>>(r.partials, kReduceBlocks, 2, r.result);
    cudaError_t e = cudaMemcpyAsync(r.host, r.result, sizeof(double) * 2, cudaMemcpyDeviceToHost, s);
    if (e != cudaSuccess) return e;
    return cudaStreamSynchronize(s);
}

cudaError_t multi_axpy(double *w, const double *V, size_t ld, const double *h, int k, uint64_t n,
                       cudaStream_t s)
{
    if (n == 0 || k == 0) return cudaSuccess;
    if (n % 2 == 0 && ld % 2 == 0 && (reinterpret_cast<uintptr_t>(w) & 15u) == 0 &&
        (reinterpret_cast<uintptr_t>(V) & 15u) == 0)
        multi_axpy2_kernel<<<blocks_for(n / 2), 256, 0, s>>>(reinterpret_cast<double2 *>(w),
                                                             reinterpret_cast<const double2 *>(V), ld / 2, h, k,
                                                             n / 2);
    else
        multi_axpy_kernel<<<blocks_for(n), 256, 0, s>>>(w, V, ld, h, k, n);
    return cudaGetLastError();
}

cudaError_t axpby(double alpha, const double *x, double beta, double *y, uint64_t n, cudaStream_t s)
{
    if (n == 0) return cudaSuccess;
    axpby_kernel<<<blocks_for(n), 256, 0, s>>>(alpha, x, beta, y, n);
    return cudaGetLastError();
}

cudaError_t sub_from(const double *x, double *y, uint64_t n, cudaStream_t s)
{
    if (n == 0) return cudaSuccess;
    sub_from_kernel<<<blocks_for(n), 256, 0, s>>>(x, y, n);
    return cudaGetLastError();
}

}  // namespace tycho
