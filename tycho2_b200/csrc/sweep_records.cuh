// Record variant of the wavefront update: the group-independent part of
// every (cell, angle) item -- face terms, LU factors of the 4x4 matrix, the
// rows of its upwind neighbours -- depends only on the mesh, the quadrature
// and sigma_t, so it is computed once per cross-section set
// (item_record_kernel) into a level-ordered array of fixed-size records and
// reused by every sweep.  A sweep then streams the records, the upwind psi
// rows and the source, and does only the per-group arithmetic.
//
// Global record (R = Real; 128 B for float, 256 B for double):
//   f[0..3]   t1[f] = A_f / 12  (t2 = 2 t1 exactly: scaling by 2 commutes
//                                with rounding; t1 < 0 marks an upwind face)
//   f[4..20]  vs20 r0 u01 u02 u03 l1 l2 l3 r1 u12 u13 a21 a31 r2 u23 b32 c33
//   u[0..6]   c, c*A + a, nmap, row[f] = nb*A + a of the neighbour across face
//             f (kNoRow on the boundary)
// A padding item has c == kSentinel.
//
// A warp takes IPW consecutive items; lane i < IPW copies record i into a
// field-major (structure-of-arrays) tile in shared memory, so that lanes
// reading one field of different items hit different banks.  The warp then
// walks the IPW*G (item, group) pairs, pair p = lane + 32k -> item p / G,
// group p % G, UNROLL pairs per lane at a time with all their loads issued
// before any arithmetic.
//
// Level schedule kernels use programmatic dependent launch: a level lets the
// next one be scheduled at once, stages its records (which do not depend on
// psi), then waits on the previous level (griddepcontrol.wait: completion and
// visibility of the prerequisite grid) before it reads upwind psi.
#pragma once

#include "sweep_kernels.cuh"

namespace tycho {

constexpr uint32_t kNoRow = 0xFFFFFFFFu;

template <typename Real>
struct alignas(16) ItemRecord {
    Real f[21];
    uint32_t u[7];
    uint32_t pad[(sizeof(Real) == 8 ? 64 : 32) - 21 * (sizeof(Real) / 4) - 7];
};
static_assert(sizeof(ItemRecord<float>) == 128, "float record is one 128-byte line");
static_assert(sizeof(ItemRecord<double>) == 256, "double record is two 128-byte lines");

template <typename Real>
__global__ void item_record_kernel(const LevelArgs p, uint64_t n, ItemRecord<Real> *out)
{
    const uint64_t it = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (it >= n) return;
    const uint32_t ca = p.items[it];
    ItemRecord<Real> r;
    if (ca == kSentinel) {
        for (int i = 0; i < 21; ++i) r.f[i] = Real(0);
        r.u[0] = kSentinel; r.u[1] = 0; r.u[2] = 0;
        for (int f = 0; f < 4; ++f) r.u[3 + f] = kNoRow;
    } else {
        ItemFactor<Real> F;
        item_setup(p, it, ca, F);
        for (int f = 0; f < 4; ++f) r.f[f] = F.t1[f];
        r.f[4] = F.vs20; r.f[5] = F.r0; r.f[6] = F.u01; r.f[7] = F.u02; r.f[8] = F.u03;
        r.f[9] = F.l1; r.f[10] = F.l2; r.f[11] = F.l3; r.f[12] = F.r1; r.f[13] = F.u12;
        r.f[14] = F.u13; r.f[15] = F.a21; r.f[16] = F.a31; r.f[17] = F.r2; r.f[18] = F.u23;
        r.f[19] = F.b32; r.f[20] = F.c33;
        r.u[0] = F.c; r.u[1] = ca; r.u[2] = F.nmap;
        for (int f = 0; f < 4; ++f) r.u[3 + f] = F.adj[f] < 0 ? kNoRow : (uint32_t)F.adj[f] * p.A + F.a;
    }
    for (unsigned i = 0; i < sizeof(r.pad) / 4; ++i) r.pad[i] = 0;
    out[it] = r;
}

// Field-major tile of IPW records in shared memory.
template <typename Real, int IPW>
struct RecordTile {
    Real f[21][IPW];
    uint32_t u[7][IPW];
};

template <typename Real, int IPW>
__device__ __forceinline__ void tile_fill(RecordTile<Real, IPW> &T, const ItemRecord<Real> *__restrict__ src,
                                          uint32_t lane, bool valid)
{
    if (lane >= (uint32_t)IPW) return;
    if (!valid) { T.u[0][lane] = kSentinel; return; }
    constexpr int N = (21 * sizeof(Real) + 28 + 15) / 16;  // 16-byte chunks holding f[] and u[]
    uint4 v[N];
    const uint4 *s = reinterpret_cast<const uint4 *>(src);
#pragma unroll
    for (int i = 0; i < N; ++i) v[i] = __ldg(s + i);
    const Real *fr = reinterpret_cast<const Real *>(v);
    const uint32_t *ur = reinterpret_cast<const uint32_t *>(reinterpret_cast<const char *>(v) + 21 * sizeof(Real));
#pragma unroll
    for (int k = 0; k < 21; ++k) T.f[k][lane] = fr[k];
#pragma unroll
    for (int k = 0; k < 7; ++k) T.u[k][lane] = ur[k];
}

template <typename Real, bool L2_ONLY>
__device__ __forceinline__ Real load_psi(const Real *p)
{
    if (L2_ONLY) return __ldcg(p);
    return *p;
}

// All the inputs of one (item, group) pair, loaded before any arithmetic.
template <typename Real>
struct PairIn {
    Real q[4];
    Real pn[4][3];  // [face][the three cell vertices j != f, increasing]
};

template <typename Real, int IPW, bool L2_ONLY>
__device__ __forceinline__ void pair_load(const LevelArgs &p, const RecordTile<Real, IPW> &T, uint32_t i,
                                          uint32_t g, PairIn<Real> &in)
{
    const uint32_t G = p.G;
    const size_t rowG = (size_t)4 * G;
    const uint32_t c = T.u[0][i];
    const Real *__restrict__ psi = reinterpret_cast<const Real *>(p.psi);
    const Real *__restrict__ iso = reinterpret_cast<const Real *>(p.iso);
    if (p.qang) {
        const double *qa = p.qang + (size_t)T.u[1][i] * rowG + g;
        const Real *ic = iso ? iso + (size_t)c * rowG + g : nullptr;
#pragma unroll
        for (int v = 0; v < 4; ++v) in.q[v] = ic ? (Real)qa[v * G] + ic[v * G] : (Real)qa[v * G];
    } else if (iso) {
        const Real *ic = iso + (size_t)c * rowG + g;
#pragma unroll
        for (int v = 0; v < 4; ++v) in.q[v] = ic[v * G];
    } else {
#pragma unroll
        for (int v = 0; v < 4; ++v) in.q[v] = Real(0);
    }
    const uint32_t nmap = T.u[2][i];
#pragma unroll
    for (int f = 0; f < 4; ++f) {
        const uint32_t row = T.u[3 + f][i];
        const bool live = T.f[f][i] < Real(0) && row != kNoRow;
        const Real *nrow = psi + (size_t)(live ? row : 0u) * rowG + g;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const int j = k < f ? k : k + 1;
            const uint32_t nv = (nmap >> ((f * 4 + j) * 2)) & 3u;
            in.pn[f][k] = live ? load_psi<Real, L2_ONLY>(nrow + nv * G) : Real(0);
        }
    }
}

template <typename Real, int IPW>
__device__ __forceinline__ void pair_solve_store(const LevelArgs &p, const RecordTile<Real, IPW> &T, uint32_t i,
                                                 uint32_t g, const PairIn<Real> &in)
{
    const Real *q = in.q;
    const Real vs20 = T.f[4][i];
    Real b[4];
    b[0] = vs20 * (Real(2) * q[0] + q[1] + q[2] + q[3]);
    b[1] = vs20 * (q[0] + Real(2) * q[1] + q[2] + q[3]);
    b[2] = vs20 * (q[0] + q[1] + Real(2) * q[2] + q[3]);
    b[3] = vs20 * (q[0] + q[1] + q[2] + Real(2) * q[3]);
    // Upwind faces in increasing order; for face f, rows i != f in increasing
    // order, each subtracting its three terms j != f in increasing order.
#pragma unroll
    for (int f = 0; f < 4; ++f) {
        const Real t1 = T.f[f][i];
        if (t1 < Real(0)) {
            const Real t2 = Real(2) * t1;
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                if (r == f) continue;
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    const int j = k < f ? k : k + 1;
                    b[r] -= (r == j ? t2 : t1) * in.pn[f][k];
                }
            }
        }
    }
    b[0] = b[0] * T.f[5][i];
    b[1] = b[1] - b[0] * T.f[9][i];
    b[2] = b[2] - b[0] * T.f[10][i];
    b[3] = b[3] - b[0] * T.f[11][i];
    b[1] = b[1] * T.f[12][i];
    b[2] = b[2] - b[1] * T.f[15][i];
    b[3] = b[3] - b[1] * T.f[16][i];
    b[2] = b[2] * T.f[17][i];
    b[3] = b[3] - b[2] * T.f[19][i];
    b[3] = div_ref(b[3], T.f[20][i]);
    b[2] = b[2] - T.f[18][i] * b[3];
    b[1] = b[1] - T.f[14][i] * b[3] - T.f[13][i] * b[2];
    b[0] = b[0] - T.f[8][i] * b[3] - T.f[7][i] * b[2] - T.f[6][i] * b[1];
    Real *__restrict__ out = reinterpret_cast<Real *>(p.psi) + (size_t)T.u[1][i] * 4 * p.G + g;
#pragma unroll
    for (int v = 0; v < 4; ++v) out[v * p.G] = b[v];
}

template <typename Real, int IPW, int UNROLL, bool L2_ONLY>
__device__ __forceinline__ void record_pairs(const LevelArgs &p, const RecordTile<Real, IPW> &T, uint32_t lane)
{
    const uint32_t G = p.G, npairs = (uint32_t)IPW * G;
    for (uint32_t q0 = lane; q0 < npairs; q0 += 32u * UNROLL) {
        PairIn<Real> in[UNROLL];
        uint32_t item[UNROLL], grp[UNROLL];
        bool live[UNROLL];
#pragma unroll
        for (int u = 0; u < UNROLL; ++u) {
            const uint32_t q = q0 + 32u * u;
            const uint32_t it = G == 1u ? q : __umulhi(q, p.gmagic);
            item[u] = it < (uint32_t)IPW ? it : 0u;
            grp[u] = q - it * G;
            live[u] = q < npairs && T.u[0][item[u]] != kSentinel;
            if (live[u]) pair_load<Real, IPW, L2_ONLY>(p, T, item[u], grp[u], in[u]);
        }
#pragma unroll
        for (int u = 0; u < UNROLL; ++u)
            if (live[u]) pair_solve_store(p, T, item[u], grp[u], in[u]);
    }
}

__device__ __forceinline__ void pdl_launch_dependents()
{
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

__device__ __forceinline__ void pdl_wait_prerequisites()
{
    asm volatile("griddepcontrol.wait;" ::: "memory");
}

// Level schedule: 4 warps per block, IPW items per warp.
template <typename Real, int IPW, int UNROLL>
__global__ void __launch_bounds__(128)
sweep_record_level_kernel(const LevelArgs p, const ItemRecord<Real> *__restrict__ rec, const uint64_t begin,
                          const uint64_t end)
{
    __shared__ RecordTile<Real, IPW> tiles[4];
    pdl_launch_dependents();
    const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
    const uint64_t base = begin + ((uint64_t)blockIdx.x * 4 + w) * IPW;
    const bool any = base < end;
    if (any) tile_fill<Real, IPW>(tiles[w], rec + base + lane, lane, true);
    pdl_wait_prerequisites();
    if (!any) return;
    __syncwarp();
    record_pairs<Real, IPW, UNROLL, false>(p, tiles[w], lane);
}

// Dataflow schedule: persistent warps take IPW-item chunks round-robin; lane
// i < IPW stages record i and waits for its upwind items, the warp sweeps the
// chunk's pairs, fences, and lane i publishes item i's epoch.
template <typename Real, int IPW, int UNROLL>
__global__ void __launch_bounds__(128)
sweep_record_dataflow_kernel(const LevelArgs p, const ItemRecord<Real> *__restrict__ rec, const DataflowArgs df)
{
    __shared__ RecordTile<Real, IPW> tiles[4];
    const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
    const uint64_t warp = (uint64_t)blockIdx.x * 4 + w;
    const uint64_t nwarps = (uint64_t)gridDim.x * 4;
    const uint64_t nchunks = df.n_items / IPW;
    const uint32_t epoch = *df.epoch;
    RecordTile<Real, IPW> &T = tiles[w];
    for (uint64_t chunk = warp; chunk < nchunks; chunk += nwarps) {
        if (*(volatile const uint32_t *)df.abort) break;
        tile_fill<Real, IPW>(T, rec + chunk * IPW + lane, lane, true);
        bool ok = false;
        uint32_t ca = 0;
        if (lane < (uint32_t)IPW && T.u[0][lane] != kSentinel) {
            ok = true;
            ca = T.u[1][lane];
#pragma unroll
            for (int f = 0; f < 4; ++f) {
                const uint32_t row = T.u[3 + f][lane];
                if (ok && T.f[f][lane] < Real(0) && row != kNoRow) ok = wait_done(df, epoch, row, ca, f);
            }
            if (!ok) T.u[0][lane] = kSentinel;
        }
        __syncwarp();
        record_pairs<Real, IPW, UNROLL, true>(p, T, lane);
        __threadfence();
        __syncwarp();
        if (ok) st_release_gpu(df.done + ca, epoch);
    }
}

template <typename Real>
cudaError_t launch_item_records(const LevelArgs &p, uint64_t n, void *out, cudaStream_t s)
{
    if (n == 0) return cudaSuccess;
    item_record_kernel<Real><<<(unsigned)((n + 127) / 128), 128, 0, s>>>(p, n, (ItemRecord<Real> *)out);
    return cudaGetLastError();
}

template <typename Real, int IPW>
static cudaError_t launch_level_record_ipw(const LevelArgs &p, const ItemRecord<Real> *r, uint64_t begin,
                                           uint64_t end, cudaStream_t s)
{
    const uint64_t warps = (end - begin + IPW - 1) / IPW;
    const unsigned blocks = (unsigned)((warps + 3) / 4);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(blocks);
    cfg.blockDim = dim3(128);
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    constexpr int U = IPW == 32 ? 4 : 2;
    return cudaLaunchKernelEx(&cfg, sweep_record_level_kernel<Real, IPW, U>, p, r, begin, end);
}

// knob = items per warp (8, 16 or 32).
template <typename Real>
cudaError_t launch_level_record(int ipw, const LevelArgs &p, const void *rec, uint64_t begin, uint64_t end,
                                cudaStream_t s)
{
    if (end <= begin) return cudaSuccess;
    const ItemRecord<Real> *r = (const ItemRecord<Real> *)rec;
    switch (ipw) {
    case 8: return launch_level_record_ipw<Real, 8>(p, r, begin, end, s);
    case 16: return launch_level_record_ipw<Real, 16>(p, r, begin, end, s);
    case 32: return launch_level_record_ipw<Real, 32>(p, r, begin, end, s);
    default: return cudaErrorInvalidValue;
    }
}

template <typename Real>
static const void *record_dataflow_fn(int ipw)
{
    switch (ipw) {
    case 8: return (const void *)sweep_record_dataflow_kernel<Real, 8, 2>;
    case 16: return (const void *)sweep_record_dataflow_kernel<Real, 16, 2>;
    case 32: return (const void *)sweep_record_dataflow_kernel<Real, 32, 4>;
    default: return nullptr;
    }
}

template <typename Real>
cudaError_t record_dataflow_blocks_per_sm(int ipw, int *blocks)
{
    const void *fn = record_dataflow_fn<Real>(ipw);
    if (!fn) return cudaErrorInvalidValue;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks, fn, 128, 0);
}

template <typename Real>
cudaError_t launch_dataflow_record(int ipw, const LevelArgs &p, const void *rec, const DataflowArgs &df,
                                   unsigned grid, cudaStream_t s)
{
    const void *fn = record_dataflow_fn<Real>(ipw);
    if (!fn || grid == 0) return cudaErrorInvalidValue;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(128);
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    const ItemRecord<Real> *r = (const ItemRecord<Real> *)rec;
    void *args[] = {(void *)&p, (void *)&r, (void *)&df};
    return cudaLaunchKernelExC(&cfg, fn, args);
}

}  // namespace tycho
