// Record variant of the wavefront update: the group-independent part of
// every (cell, angle) item -- face terms, LU factors of the 4x4 matrix, the
// cell's neighbours -- depends only on the mesh, the quadrature and sigma_t,
// so it is computed once per cross-section set (item_record_kernel) into a
// level-ordered array of fixed-size records and reused by every sweep.  A
// sweep then only streams the records, the upwind psi rows and the source.
//
// Record layout (R = Real; 32 words for float, 32 doubles for double):
//   [0..3]  t1[f] = A_f / 12          (t2 = 2 t1 exactly: scaling by 2 commutes
//                                      with rounding)
//   [4..20] vs20 r0 u01 u02 u03 l1 l2 l3 r1 u12 u13 a21 a31 r2 u23 b32 c33
//   then, as 32-bit words from byte 21*sizeof(R): c, a, nmap, adj[4]
// A padding item has c == kSentinel.
//
// Pairs are processed UNROLL at a time: all their loads are issued before
// any of them is consumed, so a lane keeps UNROLL*(4 + up to 9) loads in
// flight instead of one pair's.
#pragma once

#include "sweep_kernels.cuh"

namespace tycho {

template <typename Real>
struct alignas(16) ItemRecord {
    Real f[21];
    uint32_t c, a, nmap;
    int adj[4];
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
        r.c = kSentinel; r.a = 0; r.nmap = 0;
        for (int f = 0; f < 4; ++f) r.adj[f] = -1;
    } else {
        ItemFactor<Real> F;
        item_setup(p, it, ca, F);
        for (int f = 0; f < 4; ++f) r.f[f] = F.t1[f];
        r.f[4] = F.vs20; r.f[5] = F.r0; r.f[6] = F.u01; r.f[7] = F.u02; r.f[8] = F.u03;
        r.f[9] = F.l1; r.f[10] = F.l2; r.f[11] = F.l3; r.f[12] = F.r1; r.f[13] = F.u12;
        r.f[14] = F.u13; r.f[15] = F.a21; r.f[16] = F.a31; r.f[17] = F.r2; r.f[18] = F.u23;
        r.f[19] = F.b32; r.f[20] = F.c33;
        r.c = F.c; r.a = F.a; r.nmap = F.nmap;
        for (int f = 0; f < 4; ++f) r.adj[f] = F.adj[f];
    }
    for (unsigned i = 0; i < sizeof(r.pad) / 4; ++i) r.pad[i] = 0;
    out[it] = r;
}

// Inputs of one (item, group) pair, loaded before any arithmetic.
template <typename Real>
struct PairIn {
    Real q[4];
    Real pn[4][4];  // [face][cell vertex]
};

template <typename Real, bool L2_ONLY>
__device__ __forceinline__ void pair_load(const LevelArgs &p, const ItemRecord<Real> &R, uint32_t g,
                                          PairIn<Real> &in)
{
    const uint32_t A = p.A, G = p.G;
    const size_t rowG = (size_t)4 * G;
    const Real *__restrict__ psi = reinterpret_cast<const Real *>(p.psi);
    const Real *__restrict__ iso = reinterpret_cast<const Real *>(p.iso);
    const size_t ca = (size_t)R.c * A + R.a;
    if (p.qang) {
        const double *qa = p.qang + ca * rowG;
        const Real *ic = iso ? iso + (size_t)R.c * rowG : nullptr;
#pragma unroll
        for (int v = 0; v < 4; ++v) in.q[v] = ic ? (Real)qa[v * G + g] + ic[v * G + g] : (Real)qa[v * G + g];
    } else if (iso) {
        const Real *ic = iso + (size_t)R.c * rowG;
#pragma unroll
        for (int v = 0; v < 4; ++v) in.q[v] = ic[v * G + g];
    } else {
#pragma unroll
        for (int v = 0; v < 4; ++v) in.q[v] = Real(0);
    }
#pragma unroll
    for (int f = 0; f < 4; ++f) {
        const int nb = R.adj[f];
        const bool up = R.f[f] < Real(0);
        const Real *nrow = psi + ((size_t)(nb < 0 ? 0 : nb) * A + R.a) * rowG + g;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            in.pn[f][j] = Real(0);
            if (j == f) continue;
            const uint32_t nv = (R.nmap >> ((f * 4 + j) * 2)) & 3u;
            if (up && nb >= 0) in.pn[f][j] = load_upwind<Real, L2_ONLY>(nrow + nv * G);
        }
    }
}

template <typename Real>
__device__ __forceinline__ void pair_solve_store(const LevelArgs &p, const ItemRecord<Real> &R, uint32_t g,
                                                 const PairIn<Real> &in)
{
    const Real *F = R.f;
    const Real *q = in.q;
    Real b[4];
    b[0] = F[4] * (Real(2) * q[0] + q[1] + q[2] + q[3]);
    b[1] = F[4] * (q[0] + Real(2) * q[1] + q[2] + q[3]);
    b[2] = F[4] * (q[0] + q[1] + Real(2) * q[2] + q[3]);
    b[3] = F[4] * (q[0] + q[1] + q[2] + Real(2) * q[3]);
#pragma unroll
    for (int f = 0; f < 4; ++f) {
        if (F[f] < Real(0)) {
            const Real t1 = F[f], t2 = Real(2) * F[f];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                if (i == f) continue;
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    if (j == f) continue;
                    b[i] -= (i == j ? t2 : t1) * in.pn[f][j];
                }
            }
        }
    }
    b[0] = b[0] * F[5];
    b[1] = b[1] - b[0] * F[9];
    b[2] = b[2] - b[0] * F[10];
    b[3] = b[3] - b[0] * F[11];
    b[1] = b[1] * F[12];
    b[2] = b[2] - b[1] * F[15];
    b[3] = b[3] - b[1] * F[16];
    b[2] = b[2] * F[17];
    b[3] = b[3] - b[2] * F[19];
    b[3] = div_ref(b[3], F[20]);
    b[2] = b[2] - F[18] * b[3];
    b[1] = b[1] - F[14] * b[3] - F[13] * b[2];
    b[0] = b[0] - F[8] * b[3] - F[7] * b[2] - F[6] * b[1];
    const size_t ca = (size_t)R.c * p.A + R.a;
    Real *__restrict__ out = reinterpret_cast<Real *>(p.psi) + ca * 4 * p.G;
#pragma unroll
    for (int v = 0; v < 4; ++v) out[v * p.G + g] = b[v];
}

// Copies one record into shared memory with independent 16-byte loads.
template <typename Real>
__device__ __forceinline__ void record_copy(ItemRecord<Real> &dst, const ItemRecord<Real> *__restrict__ src)
{
    constexpr int N = sizeof(ItemRecord<Real>) / 16;
    uint4 v[N];
    const uint4 *s = reinterpret_cast<const uint4 *>(src);
#pragma unroll
    for (int i = 0; i < N; ++i) v[i] = __ldg(s + i);
    uint4 *d = reinterpret_cast<uint4 *>(&dst);
#pragma unroll
    for (int i = 0; i < N; ++i) d[i] = v[i];
}

// Phase 2 over a 32-item tile held in shared memory, UNROLL pairs at a time.
template <typename Real, int UNROLL, bool L2_ONLY>
__device__ __forceinline__ void record_pairs(const LevelArgs &p, const ItemRecord<Real> *tile, uint32_t lane)
{
    const uint32_t G = p.G, npairs = 32u * G;
    for (uint32_t q0 = lane; q0 < npairs; q0 += 32u * UNROLL) {
        PairIn<Real> in[UNROLL];
        uint32_t item[UNROLL], grp[UNROLL];
        bool live[UNROLL];
#pragma unroll
        for (int u = 0; u < UNROLL; ++u) {
            const uint32_t q = q0 + 32u * u;
            item[u] = G == 1u ? q : __umulhi(q, p.gmagic);
            grp[u] = q - item[u] * G;
            live[u] = q < npairs && tile[item[u] < 32u ? item[u] : 0].c != kSentinel;
            if (live[u]) pair_load<Real, L2_ONLY>(p, tile[item[u]], grp[u], in[u]);
        }
#pragma unroll
        for (int u = 0; u < UNROLL; ++u)
            if (live[u]) pair_solve_store(p, tile[item[u]], grp[u], in[u]);
    }
}

// Level schedule: one warp per 32-item chunk of the level.
template <typename Real, int WPB, int UNROLL>
__global__ void __launch_bounds__(WPB * 32)
sweep_record_level_kernel(const LevelArgs p, const ItemRecord<Real> *__restrict__ rec, const uint64_t begin,
                          const uint64_t end)
{
    __shared__ ItemRecord<Real> tiles[WPB][32];
    const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
    const uint64_t base = begin + ((uint64_t)blockIdx.x * WPB + w) * 32u;
    if (base >= end) return;
    record_copy(tiles[w][lane], rec + base + lane);
    __syncwarp();
    record_pairs<Real, UNROLL, false>(p, tiles[w], lane);
}

// Dataflow schedule: persistent warps take 32-item chunks round-robin; lane
// i stages record i and waits for its upwind items, the warp sweeps the
// tile's pairs, fences, and lane i publishes item i's epoch.
template <typename Real, int WPB, int UNROLL>
__global__ void __launch_bounds__(WPB * 32)
sweep_record_dataflow_kernel(const LevelArgs p, const ItemRecord<Real> *__restrict__ rec, const DataflowArgs df)
{
    __shared__ ItemRecord<Real> tiles[WPB][32];
    const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
    const uint64_t warp = (uint64_t)blockIdx.x * WPB + w;
    const uint64_t nwarps = (uint64_t)gridDim.x * WPB;
    const uint64_t nchunks = df.n_items / 32u;
    const uint32_t epoch = *df.epoch;
    for (uint64_t chunk = warp; chunk < nchunks; chunk += nwarps) {
        if (*(volatile const uint32_t *)df.abort) break;
        ItemRecord<Real> &r = tiles[w][lane];
        record_copy(r, rec + chunk * 32u + lane);
        bool ok = r.c != kSentinel;
        const uint32_t ca = ok ? r.c * p.A + r.a : 0u;
#pragma unroll
        for (int f = 0; f < 4; ++f)
            if (ok && r.f[f] < Real(0) && r.adj[f] >= 0)
                ok = wait_done(df, epoch, (uint32_t)r.adj[f] * p.A + r.a, ca, f);
        if (!ok) r.c = kSentinel;
        __syncwarp();
        record_pairs<Real, UNROLL, true>(p, tiles[w], lane);
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

template <typename Real>
cudaError_t launch_level_record(int wpb, const LevelArgs &p, const void *rec, uint64_t begin, uint64_t end,
                                cudaStream_t s)
{
    const uint64_t warps = (end - begin + 31) / 32;
    if (warps == 0) return cudaSuccess;
    const unsigned blocks = (unsigned)((warps + wpb - 1) / wpb);
    const ItemRecord<Real> *r = (const ItemRecord<Real> *)rec;
    switch (wpb) {
    case 1: sweep_record_level_kernel<Real, 1, 4><<<blocks, 32, 0, s>>>(p, r, begin, end); break;
    case 2: sweep_record_level_kernel<Real, 2, 4><<<blocks, 64, 0, s>>>(p, r, begin, end); break;
    case 4: sweep_record_level_kernel<Real, 4, 2><<<blocks, 128, 0, s>>>(p, r, begin, end); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

template <typename Real>
static const void *record_dataflow_fn(int wpb)
{
    switch (wpb) {
    case 1: return (const void *)sweep_record_dataflow_kernel<Real, 1, 4>;
    case 2: return (const void *)sweep_record_dataflow_kernel<Real, 2, 4>;
    case 4: return (const void *)sweep_record_dataflow_kernel<Real, 4, 2>;
    default: return nullptr;
    }
}

template <typename Real>
cudaError_t record_dataflow_blocks_per_sm(int wpb, int *blocks)
{
    const void *fn = record_dataflow_fn<Real>(wpb);
    if (!fn) return cudaErrorInvalidValue;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks, fn, wpb * 32, 0);
}

template <typename Real>
cudaError_t launch_dataflow_record(int wpb, const LevelArgs &p, const void *rec, const DataflowArgs &df,
                                   unsigned grid, cudaStream_t s)
{
    const void *fn = record_dataflow_fn<Real>(wpb);
    if (!fn || grid == 0) return cudaErrorInvalidValue;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(wpb * 32);
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
