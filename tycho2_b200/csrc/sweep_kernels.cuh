// Wavefront kernels of the DG SN sweep (sm_100a).
//
// Every (cell, angle) item updates all energy groups of that pair.  Per item
// the 4x4 streaming+collision matrix depends only on (cell, angle) -- the
// reference rebuilds and re-eliminates it for every group
// (src/Transport.cc:687-733) -- so here it is assembled and LU-factored once
// in registers and the G right-hand sides are pushed through the same
// elimination.  The arithmetic, including the order of every addition, is the
// reference's (calcSource :57-72, calcVolumeIntegrals :78-103,
// calcOutgoingFlux :109-168, calcIncomingFlux :174-271, gaussElim4 NoPivot
// :338-410), so the FP64 instantiation, compiled without FMA contraction, is
// bit-identical to the reference's CPU sweep.  The FP32 instantiation runs the
// same steps in single precision for the mixed-precision solver.
//
// TPI threads cooperate on one item; thread `sub` handles groups sub,
// sub+TPI, ...  so the TPI lanes' loads of one upwind vertex row are
// contiguous (TPI*sizeof(Real) >= 32 B fills a DRAM sector).
//
// Two schedules drive the same item update:
//   sweep_level_kernel     one launch per wavefront level (level-synchronous);
//   sweep_dataflow_kernel  one persistent cooperative launch per sweep: warps
//                          take level-ordered 32-item chunks round-robin and
//                          wait, with a bounded spin, only for the upwind items
//                          they read, through per-item completion epochs.
#pragma once

#include <cstdint>
#include <type_traits>
#include <cuda_runtime.h>

#include "launch.hpp"

namespace tycho {

template <typename Real> struct Vec4Of;
template <> struct Vec4Of<double> { using type = double4; };
template <> struct Vec4Of<float> { using type = float4; };

constexpr uint32_t kSentinel = 0xFFFFFFFFu;  // padding item of a level

// The group-independent part of one item's update.  NoPivot keeps its
// factors in the named fields; the other solvers in f16 (+ perm).
template <typename Real>
struct ItemFactor {
    uint32_t c, a;
    int adj[4];
    uint32_t nmap;
    Real ab[4], t1[4], t2[4], vs20;
    Real r0, u01, u02, u03, l1, l2, l3, r1, u12, u13, a21, a31, r2, u23, b32, c33;
    Real f16[16];
    uint32_t perm;  // Original: b row i comes from row (perm >> 2i) & 3
};

// FP64 keeps the reference's IEEE divisions (bit-identical results); FP32,
// checked by tolerance, uses the hardware's approximate reciprocal (about 1
// ulp; the pivots are far inside its range), which keeps the chain of the
// per-item factorization short.
template <typename Real>
__device__ __forceinline__ Real div_ref(Real x, Real y)
{
    if constexpr (std::is_same<Real, float>::value) return __fdividef(x, y);
    else return x / y;
}

template <typename Real>
__device__ __forceinline__ Real over12(Real x)
{
    if constexpr (std::is_same<Real, float>::value) return x * (1.0f / 12.0f);
    else return x / 12.0;
}

// recip (nullable): the NoPivot pivots' reciprocals 1/M00, 1/a11, 1/b22,
// computed by this function before (the FP64 compact records carry them),
// used instead of dividing again.
template <typename Real>
__device__ __forceinline__ void item_lu(ItemFactor<Real> &F, Real d1, Real d2, const bool (&out)[4],
                                        uint32_t kind = kSolveNoPivot, const Real *recip = nullptr);

template <typename Real>
__device__ __forceinline__ void item_setup(const LevelArgs &p, uint64_t it, uint32_t ca, ItemFactor<Real> &F)
{
    using R4 = typename Vec4Of<Real>::type;
    F.c = ca / p.A;
    F.a = ca - F.c * p.A;
    const R4 ab4 = reinterpret_cast<const R4 *>(p.abar)[it];
    F.ab[0] = ab4.x; F.ab[1] = ab4.y; F.ab[2] = ab4.z; F.ab[3] = ab4.w;
    const int4 adj4 = __ldg(p.adj + F.c);
    F.adj[0] = adj4.x; F.adj[1] = adj4.y; F.adj[2] = adj4.z; F.adj[3] = adj4.w;
    F.nmap = __ldg(p.nbrmap + F.c);
    const Real *ck = reinterpret_cast<const Real *>(p.cellk) + 3 * (size_t)F.c;
    F.vs20 = ck[0];
    const Real d1 = ck[1], d2 = ck[2];

    // Face terms A_f/12 and 2 A_f/12 with A_f = area * omega.n.
    bool out[4];
#pragma unroll
    for (int f = 0; f < 4; ++f) {
        F.t1[f] = over12(F.ab[f]);
        F.t2[f] = over12(Real(2) * F.ab[f]);
        out[f] = F.ab[f] > Real(0);
    }
    item_lu(F, d1, d2, out, p.solver);
}

template <typename Real>
__device__ __forceinline__ Real abs_real(Real x)
{
    return x < Real(0) ? -x : x;
}

// gaussElim4 Original (src/Transport.cc:284-337): column by column, the row
// of largest |entry| becomes the pivot row, the pivot is replaced by its
// reciprocal, the column below is scaled by it, and the next column is
// updated Crout-style.  Leaves the factored matrix in A (row major) and the
// row order of b in perm.
template <typename Real>
__device__ __forceinline__ void factor_original(Real (&A)[4][4], uint32_t &perm)
{
    uint32_t idx = 0u | (1u << 2) | (2u << 4) | (3u << 6);
    for (int column = 0; column < 3; ++column) {
        int rowmax = column;
        Real colmax = abs_real(A[column][column]);
        for (int row = column + 1; row < 4; ++row) {
            const Real t = abs_real(A[row][column]);
            if (t > colmax) {
                rowmax = row;
                colmax = t;
            }
        }
        if (rowmax != column) {
            for (int c2 = 0; c2 < 4; ++c2) {
                const Real t = A[rowmax][c2];
                A[rowmax][c2] = A[column][c2];
                A[column][c2] = t;
            }
            const uint32_t ir = (idx >> (2 * rowmax)) & 3u, ic = (idx >> (2 * column)) & 3u;
            idx &= ~((3u << (2 * rowmax)) | (3u << (2 * column)));
            idx |= (ic << (2 * rowmax)) | (ir << (2 * column));
        }
        A[column][column] = div_ref(Real(1), A[column][column]);
        for (int row = column + 1; row < 4; ++row) A[row][column] *= A[column][column];
        for (int c2 = 0; c2 <= column; ++c2)
            for (int row = c2 + 1; row < 4; ++row) A[row][column + 1] -= A[row][c2] * A[c2][column + 1];
    }
    A[3][3] = div_ref(Real(1), A[3][3]);
    perm = idx;
}

// gaussElim4 CramerGlu (src/Transport.cc:414-557): inv[4a + b] is the
// (b, a) cofactor, (-1)^(a+b) times the minor without row b and column a,
// expanded along its first column over its rows in increasing order, each
// row's 2x2 minor as m[r][c0] m[r'][c1] m[r''][c2] - m[r][c0] m[r'][c2]
// m[r''][c1]; products and the six terms left to right (the reference's
// expressions); then det = row 0 . column 0 of inv, inv *= 1/det.
template <typename Real>
__device__ __forceinline__ void factor_cramer_glu(const Real (&A)[4][4], Real (&inv)[16])
{
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int bb = 0; bb < 4; ++bb) {
            int rows[3], cols[3];
            int nr = 0, ncl = 0;
#pragma unroll
            for (int r = 0; r < 4; ++r)
                if (r != bb) rows[nr++] = r;
#pragma unroll
            for (int c = 0; c < 4; ++c)
                if (c != a) cols[ncl++] = c;
            const bool neg = ((a + bb) & 1) != 0;
            Real acc = Real(0);
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const int r = rows[k], r1 = rows[k == 0 ? 1 : 0], r2 = rows[k == 2 ? 1 : 2];
                const bool plus = neg == ((k & 1) != 0);
                const Real t1 = A[r][cols[0]] * A[r1][cols[1]] * A[r2][cols[2]];
                const Real t2 = A[r][cols[0]] * A[r1][cols[2]] * A[r2][cols[1]];
                if (k == 0) acc = plus ? t1 : -t1;
                else acc = plus ? acc + t1 : acc - t1;
                acc = plus ? acc - t2 : acc + t2;
            }
            inv[4 * a + bb] = acc;
        }
    Real det = A[0][0] * inv[0] + A[0][1] * inv[4] + A[0][2] * inv[8] + A[0][3] * inv[12];
    det = div_ref(Real(1), det);
#pragma unroll
    for (int i = 0; i < 16; ++i) inv[i] = inv[i] * det;
}

// gaussElim4 CramerIntel (src/Transport.cc:559-677): the scalar form of
// Intel's SSE 4x4 inverse (application note "Streaming SIMD Extensions -
// Inverse of 4x4 Matrix").  src = A column major; for each half, products of
// pairs of two src rows (tmp), then every cofactor as the sum of three
// (tmp x src) products minus the sum of three more, in the (tmp, src) order
// of the tables; det = src row 0 . dst, dst *= 1/det.
__constant__ const unsigned char kIntelCof[16][6][2] = {
    {{0, 5}, {3, 6}, {4, 7}, {1, 5}, {2, 6}, {5, 7}},       {{1, 4}, {6, 6}, {9, 7}, {0, 4}, {7, 6}, {8, 7}},
    {{2, 4}, {7, 5}, {10, 7}, {3, 4}, {6, 5}, {11, 7}},     {{5, 4}, {8, 5}, {11, 6}, {4, 4}, {9, 5}, {10, 6}},
    {{1, 1}, {2, 2}, {5, 3}, {0, 1}, {3, 2}, {4, 3}},       {{0, 0}, {7, 2}, {8, 3}, {1, 0}, {6, 2}, {9, 3}},
    {{3, 0}, {6, 1}, {11, 3}, {2, 0}, {7, 1}, {10, 3}},     {{4, 0}, {9, 1}, {10, 2}, {5, 0}, {8, 1}, {11, 2}},
    {{0, 13}, {3, 14}, {4, 15}, {1, 13}, {2, 14}, {5, 15}}, {{1, 12}, {6, 14}, {9, 15}, {0, 12}, {7, 14}, {8, 15}},
    {{2, 12}, {7, 13}, {10, 15}, {3, 12}, {6, 13}, {11, 15}}, {{5, 12}, {8, 13}, {11, 14}, {4, 12}, {9, 13}, {10, 14}},
    {{2, 10}, {5, 11}, {1, 9}, {4, 11}, {0, 9}, {3, 10}},   {{8, 11}, {0, 8}, {7, 10}, {6, 10}, {9, 11}, {1, 8}},
    {{6, 9}, {11, 11}, {3, 8}, {10, 11}, {2, 8}, {7, 9}},   {{10, 10}, {4, 8}, {9, 9}, {8, 9}, {11, 10}, {5, 8}}};

template <typename Real>
__device__ __forceinline__ void factor_cramer_intel(const Real (&A)[4][4], Real (&dst)[16])
{
    constexpr int pairs[6][2] = {{2, 3}, {1, 3}, {1, 2}, {0, 3}, {0, 2}, {0, 1}};
    Real src[16], tmp[12];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) src[i + 4 * j] = A[i][j];
#pragma unroll
    for (int half = 0; half < 2; ++half) {
        const int lo = half ? 0 : 8, hi = half ? 4 : 12;
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            tmp[2 * k] = src[lo + pairs[k][0]] * src[hi + pairs[k][1]];
            tmp[2 * k + 1] = src[lo + pairs[k][1]] * src[hi + pairs[k][0]];
        }
#pragma unroll
        for (int j = 8 * half; j < 8 * half + 8; ++j) {
            const Real plus = tmp[kIntelCof[j][0][0]] * src[kIntelCof[j][0][1]] +
                              tmp[kIntelCof[j][1][0]] * src[kIntelCof[j][1][1]] +
                              tmp[kIntelCof[j][2][0]] * src[kIntelCof[j][2][1]];
            const Real minus = tmp[kIntelCof[j][3][0]] * src[kIntelCof[j][3][1]] +
                               tmp[kIntelCof[j][4][0]] * src[kIntelCof[j][4][1]] +
                               tmp[kIntelCof[j][5][0]] * src[kIntelCof[j][5][1]];
            dst[j] = plus - minus;
        }
    }
    Real det = src[0] * dst[0] + src[1] * dst[1] + src[2] * dst[2] + src[3] * dst[3];
    det = div_ref(Real(1), det);
#pragma unroll
    for (int j = 0; j < 16; ++j) dst[j] *= det;
}

// The 16 per-item numbers of a solver as stored in a record (f[5..20]).
template <typename Real>
__device__ __forceinline__ void factor16(const ItemFactor<Real> &F, uint32_t kind, Real (&out)[16])
{
    if (kind == kSolveNoPivot) {
        out[0] = F.r0; out[1] = F.u01; out[2] = F.u02; out[3] = F.u03; out[4] = F.l1; out[5] = F.l2;
        out[6] = F.l3; out[7] = F.r1; out[8] = F.u12; out[9] = F.u13; out[10] = F.a21; out[11] = F.a31;
        out[12] = F.r2; out[13] = F.u23; out[14] = F.b32; out[15] = F.c33;
    } else {
#pragma unroll
        for (int i = 0; i < 16; ++i) out[i] = F.f16[i];
    }
}

// The matrix of one (cell, angle) item from its face terms t1, t2 and the
// volume terms d1 = sigma_t V/20, d2 = 2 sigma_t V/20 (out[f]: face f is
// outgoing), and its LU factors.
template <typename Real>
__device__ __forceinline__ void item_lu(ItemFactor<Real> &F, Real d1, Real d2, const bool (&out)[4], uint32_t kind,
                                        const Real *recip)
{
    // Streaming + collision (volume integrals), then outgoing-face terms in
    // increasing face order.
    Real M[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) M[i][j] = F.t1[i] + (i == j ? d2 : d1);
#pragma unroll
    for (int f = 0; f < 4; ++f) {
        if (out[f]) {
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j)
                    if (i != f && j != f) M[i][j] += (i == j ? F.t2[f] : F.t1[f]);
        }
    }
    F.perm = 0u | (1u << 2) | (2u << 4) | (3u << 6);
    if (kind == kSolveOriginal) {
        factor_original(M, F.perm);
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) F.f16[4 * i + j] = M[i][j];
        return;
    }
    if (kind == kSolveCramerGlu) {
        factor_cramer_glu(M, F.f16);
        return;
    }
    if (kind == kSolveCramerIntel) {
        factor_cramer_intel(M, F.f16);
        return;
    }
    // LU without pivoting: the elimination steps of gaussElim4 NoPivot that
    // touch only the matrix.
    F.r0 = recip ? recip[0] : div_ref(Real(1), M[0][0]);
    F.u01 = M[0][1] * F.r0; F.u02 = M[0][2] * F.r0; F.u03 = M[0][3] * F.r0;
    F.l1 = M[1][0]; F.l2 = M[2][0]; F.l3 = M[3][0];
    const Real a11 = M[1][1] - F.u01 * F.l1, a12 = M[1][2] - F.u02 * F.l1, a13 = M[1][3] - F.u03 * F.l1;
    const Real a21 = M[2][1] - F.u01 * F.l2, a22 = M[2][2] - F.u02 * F.l2, a23 = M[2][3] - F.u03 * F.l2;
    const Real a31 = M[3][1] - F.u01 * F.l3, a32 = M[3][2] - F.u02 * F.l3, a33 = M[3][3] - F.u03 * F.l3;
    F.a21 = a21; F.a31 = a31;
    F.r1 = recip ? recip[1] : div_ref(Real(1), a11);
    F.u12 = a12 * F.r1; F.u13 = a13 * F.r1;
    const Real b22 = a22 - F.u12 * a21, b23 = a23 - F.u13 * a21;
    F.b32 = a32 - F.u12 * a31;
    const Real b33 = a33 - F.u13 * a31;
    F.r2 = recip ? recip[2] : div_ref(Real(1), b22);
    F.u23 = b23 * F.r2;
    F.c33 = b33 - F.u23 * F.b32;
}

// Loads an upwind psi value; L2_ONLY bypasses L1, which another SM's recent
// write may have left stale (the dataflow schedule reads values written in
// the same launch).
template <typename Real, bool L2_ONLY>
__device__ __forceinline__ Real load_upwind(const Real *p)
{
    if (L2_ONLY) return __ldcg(p);
    return *p;
}

template <typename Real, int TPI, bool L2_ONLY>
__device__ __forceinline__ void item_groups(const LevelArgs &p, uint32_t ca, int sub, const ItemFactor<Real> &F)
{
    const uint32_t A = p.A, G = p.G;
    const size_t rowG = (size_t)4 * G;
    const Real *__restrict__ psi_in = reinterpret_cast<const Real *>(p.psi);
    Real *__restrict__ psi_out = reinterpret_cast<Real *>(p.psi) + (size_t)ca * rowG;
    const Real *__restrict__ iso = reinterpret_cast<const Real *>(p.iso);
    const Real *iso_c = iso ? iso + (size_t)F.c * rowG : nullptr;
    const double *qang_ca = p.qang ? p.qang + (size_t)ca * rowG : nullptr;

    for (uint32_t g = sub; g < G; g += TPI) {
        Real q[4];
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            if (qang_ca && iso_c) q[v] = (Real)qang_ca[v * G + g] + iso_c[v * G + g];
            else if (qang_ca) q[v] = (Real)qang_ca[v * G + g];
            else if (iso_c) q[v] = iso_c[v * G + g];
            else q[v] = Real(0);
        }
        Real b[4];
        b[0] = F.vs20 * (Real(2) * q[0] + q[1] + q[2] + q[3]);
        b[1] = F.vs20 * (q[0] + Real(2) * q[1] + q[2] + q[3]);
        b[2] = F.vs20 * (q[0] + q[1] + Real(2) * q[2] + q[3]);
        b[3] = F.vs20 * (q[0] + q[1] + q[2] + Real(2) * q[3]);
        // Upwind faces, increasing face order; vacuum (0) on the boundary.
#pragma unroll
        for (int f = 0; f < 4; ++f) {
            if (F.ab[f] < Real(0)) {
                Real pn[4];
                const int nb = F.adj[f];
                const Real *nrow = psi_in + ((size_t)(nb < 0 ? 0 : nb) * A + F.a) * rowG + g;
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    if (j == f) { pn[j] = Real(0); continue; }
                    const uint32_t nv = (F.nmap >> ((f * 4 + j) * 2)) & 3u;
                    pn[j] = nb >= 0 ? load_upwind<Real, L2_ONLY>(nrow + nv * G) : Real(0);
                }
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    if (i == f) continue;
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        if (j == f) continue;
                        b[i] -= (i == j ? F.t2[f] : F.t1[f]) * pn[j];
                    }
                }
            }
        }
        // The right-hand-side steps of gaussElim4 NoPivot.
        b[0] = b[0] * F.r0;
        b[1] = b[1] - b[0] * F.l1;
        b[2] = b[2] - b[0] * F.l2;
        b[3] = b[3] - b[0] * F.l3;
        b[1] = b[1] * F.r1;
        b[2] = b[2] - b[1] * F.a21;
        b[3] = b[3] - b[1] * F.a31;
        b[2] = b[2] * F.r2;
        b[3] = b[3] - b[2] * F.b32;
        b[3] = div_ref(b[3], F.c33);
        b[2] = b[2] - F.u23 * b[3];
        b[1] = b[1] - F.u13 * b[3] - F.u12 * b[2];
        b[0] = b[0] - F.u03 * b[3] - F.u02 * b[2] - F.u01 * b[1];
#pragma unroll
        for (int v = 0; v < 4; ++v) psi_out[v * G + g] = b[v];
    }
}

template <typename Real, int TPI>
__global__ void __launch_bounds__(256)
sweep_level_kernel(const LevelArgs p, const uint64_t begin, const uint64_t end)
{
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t it = begin + t / TPI;
    if (it >= end) return;
    const uint32_t ca = __ldg(p.items + it);
    if (ca == kSentinel) return;
    ItemFactor<Real> F;
    item_setup(p, it, ca, F);
    item_groups<Real, TPI, false>(p, ca, (int)(t % TPI), F);
}

__device__ __forceinline__ uint32_t ld_acquire_gpu(const uint32_t *p)
{
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release_gpu(uint32_t *p, uint32_t v)
{
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Waits until done[idx] == epoch.  Gives up after df.spin_limit polls: records
// the item and face in df.err (first failure wins), raises df.abort, and
// returns false; every warp then drains without computing.
__device__ __forceinline__ bool wait_done(const DataflowArgs &df, uint32_t epoch, uint32_t idx,
                                          uint32_t ca, int f)
{
    const uint32_t *flag = df.done + idx;
    if (ld_acquire_gpu(flag) == epoch) return true;
    unsigned backoff = 32;
    for (uint32_t spin = 0; spin < df.spin_limit; ++spin) {
        if (*(volatile const uint32_t *)df.abort) return false;
        __nanosleep(backoff);
        if (backoff < 1024) backoff <<= 1;
        if (ld_acquire_gpu(flag) == epoch) return true;
    }
    if (atomicCAS(df.err, 0u, (uint32_t)kErrTimeoutCode) == 0u) {
        df.err[1] = ca;
        df.err[2] = (uint32_t)f;
    }
    atomicExch(df.abort, 1u);
    return false;
}

// One persistent launch per sweep.  Items are padded per level to multiples
// of 32, so a warp's 32/TPI-item chunk never spans two levels: an item only
// waits for items of lower levels, which belong to chunks of lower index.
// Warps take chunks round-robin in increasing order and every warp is
// resident (cooperative launch), so the lowest unfinished chunk can always
// make progress.
template <typename Real, int TPI>
__global__ void __launch_bounds__(256)
sweep_dataflow_kernel(const LevelArgs p, const DataflowArgs df)
{
    constexpr uint32_t IPW = 32 / TPI;  // items per warp chunk
    const uint32_t lane = threadIdx.x & 31u;
    const int sub = (int)(lane % TPI);
    const uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    const uint64_t nchunks = df.n_items / IPW;
    const uint32_t epoch = *df.epoch;
    for (uint64_t chunk = warp; chunk < nchunks; chunk += nwarps) {
        if (*(volatile const uint32_t *)df.abort) break;
        const uint64_t it = chunk * IPW + lane / TPI;
        const uint32_t ca = __ldg(p.items + it);
        bool ok = true;
        if (ca != kSentinel) {
            ItemFactor<Real> F;
            item_setup(p, it, ca, F);
#pragma unroll
            for (int f = 0; f < 4; ++f)
                if (ok && F.ab[f] < Real(0) && F.adj[f] >= 0)
                    ok = wait_done(df, epoch, (uint32_t)F.adj[f] * p.A + F.a, ca, f);
            if (ok) item_groups<Real, TPI, true>(p, ca, sub, F);
        }
        __threadfence();
        __syncwarp();
        if (ca != kSentinel && sub == 0 && ok) st_release_gpu(df.done + ca, epoch);
    }
}

// Launches one level with TPI chosen at run time.
template <typename Real>
cudaError_t launch_level(int tpi, const LevelArgs &p, uint64_t begin, uint64_t end, cudaStream_t s)
{
    const uint64_t threads = (end - begin) * (uint64_t)tpi;
    const unsigned blocks = (unsigned)((threads + 255) / 256);
    if (blocks == 0) return cudaSuccess;
    switch (tpi) {
    case 1: sweep_level_kernel<Real, 1><<<blocks, 256, 0, s>>>(p, begin, end); break;
    case 2: sweep_level_kernel<Real, 2><<<blocks, 256, 0, s>>>(p, begin, end); break;
    case 4: sweep_level_kernel<Real, 4><<<blocks, 256, 0, s>>>(p, begin, end); break;
    case 8: sweep_level_kernel<Real, 8><<<blocks, 256, 0, s>>>(p, begin, end); break;
    case 16: sweep_level_kernel<Real, 16><<<blocks, 256, 0, s>>>(p, begin, end); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

template <typename Real>
static const void *dataflow_fn(int tpi)
{
    switch (tpi) {
    case 1: return (const void *)sweep_dataflow_kernel<Real, 1>;
    case 2: return (const void *)sweep_dataflow_kernel<Real, 2>;
    case 4: return (const void *)sweep_dataflow_kernel<Real, 4>;
    case 8: return (const void *)sweep_dataflow_kernel<Real, 8>;
    case 16: return (const void *)sweep_dataflow_kernel<Real, 16>;
    default: return nullptr;
    }
}

template <typename Real>
cudaError_t dataflow_blocks_per_sm(int tpi, int *blocks)
{
    const void *fn = dataflow_fn<Real>(tpi);
    if (!fn) return cudaErrorInvalidValue;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks, fn, 256, 0);
}

template <typename Real>
cudaError_t launch_dataflow(int tpi, const LevelArgs &p, const DataflowArgs &df, unsigned grid, cudaStream_t s)
{
    const void *fn = dataflow_fn<Real>(tpi);
    if (!fn || grid == 0) return cudaErrorInvalidValue;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(256);
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
