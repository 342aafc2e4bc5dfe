// Warp-tile variant of the wavefront update (1, 2 or 4 warps per block).
//
// A warp owns a tile of 32 level-contiguous (cell, angle) items.
//   Phase 1: lane i assembles and LU-factors item i's 4x4 matrix once (no
//            per-group or per-lane redundancy) into shared memory; in the
//            dataflow schedule it first waits for item i's upwind items.
//   Phase 2: the warp walks the tile's 32*G (item, group) pairs, pair
//            p = lane + 32k -> item p / G, group p % G, so neighbouring lanes
//            handle neighbouring groups of one item and every load of an
//            upwind vertex row or of the source row is one contiguous run.
//   Phase 3 (dataflow): fence, then lane i publishes item i's epoch.
// The arithmetic per (item, group) is item_groups' (the reference's order),
// so the FP64 instantiation stays bit-identical to the reference.
#pragma once

#include "sweep_kernels.cuh"

namespace tycho {

// Per-item record in shared memory: the factor plus what phase 2 indexes.
template <typename Real>
struct TileItem {
    Real t1[4], t2[4];
    Real vs20, r0, u01, u02, u03, l1, l2, l3, r1, u12, u13, a21, a31, r2, u23, b32, c33;
    uint32_t c, a, nmap, up;  // up: bit f set when face f is upwind (A_f < 0)
    int adj[4];
};

template <typename Real>
__device__ __forceinline__ void tile_store(TileItem<Real> &T, const ItemFactor<Real> &F, bool valid)
{
#pragma unroll
    for (int f = 0; f < 4; ++f) {
        T.t1[f] = F.t1[f];
        T.t2[f] = F.t2[f];
        T.adj[f] = F.adj[f];
    }
    T.vs20 = F.vs20; T.r0 = F.r0; T.u01 = F.u01; T.u02 = F.u02; T.u03 = F.u03;
    T.l1 = F.l1; T.l2 = F.l2; T.l3 = F.l3; T.r1 = F.r1; T.u12 = F.u12; T.u13 = F.u13;
    T.a21 = F.a21; T.a31 = F.a31; T.r2 = F.r2; T.u23 = F.u23; T.b32 = F.b32; T.c33 = F.c33;
    T.c = valid ? F.c : kSentinel;
    T.a = F.a;
    T.nmap = F.nmap;
    uint32_t up = 0;
#pragma unroll
    for (int f = 0; f < 4; ++f)
        if (F.ab[f] < Real(0)) up |= 1u << f;
    T.up = up;
}

// One (item, group) update from the shared-memory record.
template <typename Real, bool L2_ONLY>
__device__ __forceinline__ void tile_pair(const LevelArgs &p, const TileItem<Real> &T, uint32_t g)
{
    const uint32_t A = p.A, G = p.G;
    const size_t rowG = (size_t)4 * G;
    const size_t ca = (size_t)T.c * A + T.a;
    const Real *__restrict__ psi_in = reinterpret_cast<const Real *>(p.psi);
    Real *__restrict__ psi_out = reinterpret_cast<Real *>(p.psi) + ca * rowG;
    const Real *__restrict__ iso = reinterpret_cast<const Real *>(p.iso);
    Real q[4];
    if (p.qang) {
        const double *qa = p.qang + ca * rowG;
        const Real *ic = iso ? iso + (size_t)T.c * rowG : nullptr;
#pragma unroll
        for (int v = 0; v < 4; ++v) q[v] = ic ? (Real)qa[v * G + g] + ic[v * G + g] : (Real)qa[v * G + g];
    } else if (iso) {
        const Real *ic = iso + (size_t)T.c * rowG;
#pragma unroll
        for (int v = 0; v < 4; ++v) q[v] = ic[v * G + g];
    } else {
#pragma unroll
        for (int v = 0; v < 4; ++v) q[v] = Real(0);
    }
    Real b[4];
    b[0] = T.vs20 * (Real(2) * q[0] + q[1] + q[2] + q[3]);
    b[1] = T.vs20 * (q[0] + Real(2) * q[1] + q[2] + q[3]);
    b[2] = T.vs20 * (q[0] + q[1] + Real(2) * q[2] + q[3]);
    b[3] = T.vs20 * (q[0] + q[1] + q[2] + Real(2) * q[3]);
#pragma unroll
    for (int f = 0; f < 4; ++f) {
        if (T.up >> f & 1u) {
            Real pn[4];
            const int nb = T.adj[f];
            const Real *nrow = psi_in + ((size_t)(nb < 0 ? 0 : nb) * A + T.a) * rowG + g;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                if (j == f) { pn[j] = Real(0); continue; }
                const uint32_t nv = (T.nmap >> ((f * 4 + j) * 2)) & 3u;
                pn[j] = nb >= 0 ? load_upwind<Real, L2_ONLY>(nrow + nv * G) : Real(0);
            }
            const Real t1 = T.t1[f], t2 = T.t2[f];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                if (i == f) continue;
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    if (j == f) continue;
                    b[i] -= (i == j ? t2 : t1) * pn[j];
                }
            }
        }
    }
    b[0] = b[0] * T.r0;
    b[1] = b[1] - b[0] * T.l1;
    b[2] = b[2] - b[0] * T.l2;
    b[3] = b[3] - b[0] * T.l3;
    b[1] = b[1] * T.r1;
    b[2] = b[2] - b[1] * T.a21;
    b[3] = b[3] - b[1] * T.a31;
    b[2] = b[2] * T.r2;
    b[3] = b[3] - b[2] * T.b32;
    b[3] = div_ref(b[3], T.c33);
    b[2] = b[2] - T.u23 * b[3];
    b[1] = b[1] - T.u13 * b[3] - T.u12 * b[2];
    b[0] = b[0] - T.u03 * b[3] - T.u02 * b[2] - T.u01 * b[1];
#pragma unroll
    for (int v = 0; v < 4; ++v) psi_out[v * G + g] = b[v];
}

// Phase 2 for the whole tile.  gmagic = ceil(2^32 / G) (exact p / G for
// p < 32*64); G == 1 maps pair p to item p.
template <typename Real, bool L2_ONLY>
__device__ __forceinline__ void tile_pairs(const LevelArgs &p, const TileItem<Real> *tile, uint32_t lane)
{
    const uint32_t G = p.G, npairs = 32u * G;
    for (uint32_t q = lane; q < npairs; q += 32u) {
        const uint32_t i = G == 1u ? q : __umulhi(q, p.gmagic);
        const uint32_t g = q - i * G;
        const TileItem<Real> &T = tile[i];
        if (T.c != kSentinel) tile_pair<Real, L2_ONLY>(p, T, g);
    }
}

template <typename Real, int WPB>
__global__ void __launch_bounds__(WPB * 32)
sweep_tile_level_kernel(const LevelArgs p, const uint64_t begin, const uint64_t end)
{
    __shared__ TileItem<Real> tiles[WPB][32];
    const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
    const uint64_t base = begin + ((uint64_t)blockIdx.x * WPB + w) * 32u;
    if (base >= end) return;  // whole warp
    const uint64_t it = base + lane;
    const uint32_t ca = __ldg(p.items + it);
    ItemFactor<Real> F;
    if (ca != kSentinel) item_setup(p, it, ca, F);
    tile_store(tiles[w][lane], F, ca != kSentinel);
    __syncwarp();
    tile_pairs<Real, false>(p, tiles[w], lane);
}

template <typename Real, int WPB>
__global__ void __launch_bounds__(WPB * 32)
sweep_tile_dataflow_kernel(const LevelArgs p, const DataflowArgs df)
{
    __shared__ TileItem<Real> tiles[WPB][32];
    const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
    const uint64_t warp = (uint64_t)blockIdx.x * WPB + w;
    const uint64_t nwarps = (uint64_t)gridDim.x * WPB;
    const uint64_t nchunks = df.n_items / 32u;
    const uint32_t epoch = *df.epoch;
    for (uint64_t chunk = warp; chunk < nchunks; chunk += nwarps) {
        if (*(volatile const uint32_t *)df.abort) break;
        const uint64_t it = chunk * 32u + lane;
        const uint32_t ca = __ldg(p.items + it);
        bool ok = ca != kSentinel;
        ItemFactor<Real> F;
        if (ok) {
            item_setup(p, it, ca, F);
#pragma unroll
            for (int f = 0; f < 4; ++f)
                if (ok && F.ab[f] < Real(0) && F.adj[f] >= 0)
                    ok = wait_done(df, epoch, (uint32_t)F.adj[f] * p.A + F.a, ca, f);
        }
        tile_store(tiles[w][lane], F, ok);
        __syncwarp();
        tile_pairs<Real, true>(p, tiles[w], lane);
        __threadfence();
        __syncwarp();
        if (ok) st_release_gpu(df.done + ca, epoch);
    }
}

template <typename Real>
cudaError_t launch_level_tile(int wpb, const LevelArgs &p, uint64_t begin, uint64_t end, cudaStream_t s)
{
    const uint64_t warps = (end - begin + 31) / 32;
    if (warps == 0) return cudaSuccess;
    const unsigned blocks = (unsigned)((warps + wpb - 1) / wpb);
    switch (wpb) {
    case 1: sweep_tile_level_kernel<Real, 1><<<blocks, 32, 0, s>>>(p, begin, end); break;
    case 2: sweep_tile_level_kernel<Real, 2><<<blocks, 64, 0, s>>>(p, begin, end); break;
    case 4: sweep_tile_level_kernel<Real, 4><<<blocks, 128, 0, s>>>(p, begin, end); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

template <typename Real>
static const void *tile_dataflow_fn(int wpb)
{
    switch (wpb) {
    case 1: return (const void *)sweep_tile_dataflow_kernel<Real, 1>;
    case 2: return (const void *)sweep_tile_dataflow_kernel<Real, 2>;
    case 4: return (const void *)sweep_tile_dataflow_kernel<Real, 4>;
    default: return nullptr;
    }
}

template <typename Real>
cudaError_t tile_dataflow_blocks_per_sm(int wpb, int *blocks)
{
    const void *fn = tile_dataflow_fn<Real>(wpb);
    if (!fn) return cudaErrorInvalidValue;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks, fn, wpb * 32, 0);
}

template <typename Real>
cudaError_t launch_dataflow_tile(int wpb, const LevelArgs &p, const DataflowArgs &df, unsigned grid,
                                 cudaStream_t s)
{
    const void *fn = tile_dataflow_fn<Real>(wpb);
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
    void *args[] = {(void *)&p, (void *)&df};
    return cudaLaunchKernelExC(&cfg, fn, args);
}

}  // namespace tycho
