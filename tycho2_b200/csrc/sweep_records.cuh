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
//             f (kNoRow on the boundary); the word after u[6] holds the
//             row order of the Original solver
// f[5..20] are the 16 numbers of the 4x4 solver (GaussElim): the NoPivot
// factors below, Original's factored matrix, or the Cramer inverses.
// A padding item has c == kSentinel.
//
// A warp takes IPW consecutive items; lane i < IPW copies record i into a
// field-major (structure-of-arrays) tile in shared memory, so that lanes
// reading one field of different items hit different banks.  The warp then
// walks the IPW*G (item, group) pairs in tasks of VG consecutive groups
// (vector loads and stores of psi rows), task t = lane + 32k -> item
// t / (G/VG), several tasks per lane at a time with all their loads issued
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
    for (unsigned i = 0; i < sizeof(r.pad) / 4; ++i) r.pad[i] = 0;
    if (ca == kSentinel) {
        for (int i = 0; i < 21; ++i) r.f[i] = Real(0);
        r.u[0] = kSentinel; r.u[1] = 0; r.u[2] = 0;
        for (int f = 0; f < 4; ++f) r.u[3 + f] = kNoRow;
    } else {
        ItemFactor<Real> F;
        item_setup(p, it, ca, F);
        for (int f = 0; f < 4; ++f) r.f[f] = F.t1[f];
        r.f[4] = F.vs20;
        Real f16[16];
        factor16(F, p.solver, f16);
        for (int i = 0; i < 16; ++i) r.f[5 + i] = f16[i];
        r.u[0] = F.c; r.u[1] = ca; r.u[2] = F.nmap;
        for (int f = 0; f < 4; ++f) r.u[3 + f] = F.adj[f] < 0 ? kNoRow : (uint32_t)F.adj[f] * p.A + F.a;
        r.pad[0] = F.perm;  // the Original solver's row order, right after u[]
    }
    out[it] = r;
}

// Compact record (64 B float, 112 B double): the inputs of the item's matrix
// instead of its factors -- t1[f] = A_f/12 (f[0..3]), vs20 = V/20 (f[4]),
// d1 = sigma_t V/20 (f[5]), d2 = 2 sigma_t V/20 (f[6]) -- and the same
// topology words as ItemRecord.  The loader rebuilds the LU factors with
// item_lu (the arithmetic of item_setup: t2 = 2 t1 exactly, a face is
// outgoing iff t1 > 0), so FP64 results stay bit-identical.  The FP64 record
// also carries the NoPivot pivots' reciprocals (f[7..9], computed by the
// same item_lu when the record is built): an IEEE FP64 division is a long
// dependent sequence, and three of them per task sat on the rebuild's chain.
template <typename Real>
constexpr int kCompactF = sizeof(Real) == 8 ? 10 : 7;

template <typename Real>
struct alignas(16) CompactRecord {
    Real f[kCompactF<Real>];
    uint32_t u[7];
    uint32_t pad[(sizeof(Real) == 8 ? 28 : 16) - kCompactF<Real> * (sizeof(Real) / 4) - 7];
};
static_assert(sizeof(CompactRecord<float>) == 64, "float compact record is 64 bytes");
static_assert(sizeof(CompactRecord<double>) == 112, "double compact record is 112 bytes");

template <typename Real>
__global__ void compact_record_kernel(const LevelArgs p, uint64_t n, CompactRecord<Real> *out)
{
    const uint64_t it = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (it >= n) return;
    const uint32_t ca = p.items[it];
    CompactRecord<Real> r;
    if (ca == kSentinel) {
        for (int i = 0; i < kCompactF<Real>; ++i) r.f[i] = Real(0);
        r.u[0] = kSentinel; r.u[1] = 0; r.u[2] = 0;
        for (int f = 0; f < 4; ++f) r.u[3 + f] = kNoRow;
    } else {
        ItemFactor<Real> F;
        item_setup(p, it, ca, F);
        const Real *ck = reinterpret_cast<const Real *>(p.cellk) + 3 * (size_t)F.c;
        for (int f = 0; f < 4; ++f) r.f[f] = F.t1[f];
        r.f[4] = F.vs20;
        r.f[5] = ck[1];
        r.f[6] = ck[2];
        if constexpr (kCompactF<Real> == 10) {
            const bool np = p.solver == kSolveNoPivot;  // the other solvers factor without them
            r.f[7] = np ? F.r0 : Real(0);
            r.f[8] = np ? F.r1 : Real(0);
            r.f[9] = np ? F.r2 : Real(0);
        }
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
    uint32_t u[8][IPW];  // u[7]: the Original solver's row order
};

template <typename Real, int IPW>
__device__ __forceinline__ void tile_fill(RecordTile<Real, IPW> &T, const ItemRecord<Real> *__restrict__ src,
                                          uint32_t lane, bool valid)
{
    if (lane >= (uint32_t)IPW) return;
    if (!valid) { T.u[0][lane] = kSentinel; return; }
    constexpr int N = (21 * sizeof(Real) + 32 + 15) / 16;  // 16-byte chunks holding f[], u[] and the row order
    uint4 v[N];
    const uint4 *s = reinterpret_cast<const uint4 *>(src);
#pragma unroll
    for (int i = 0; i < N; ++i) v[i] = __ldg(s + i);
    const Real *fr = reinterpret_cast<const Real *>(v);
    const uint32_t *ur = reinterpret_cast<const uint32_t *>(reinterpret_cast<const char *>(v) + 21 * sizeof(Real));
#pragma unroll
    for (int k = 0; k < 21; ++k) T.f[k][lane] = fr[k];
#pragma unroll
    for (int k = 0; k < 8; ++k) T.u[k][lane] = ur[k];
}

// VG consecutive groups of one psi/phi row move as one vector access (the
// group index is fastest in both layouts; the host picks VG dividing G).
template <typename Real, int VG> struct GVec;
template <> struct GVec<float, 1> { using T = float; };
template <> struct GVec<float, 2> { using T = float2; };
template <> struct GVec<float, 4> { using T = float4; };
template <> struct GVec<double, 1> { using T = double; };
template <> struct GVec<double, 2> { using T = double2; };

__device__ __forceinline__ void gv_unpack(float v, float (&o)[1]) { o[0] = v; }
__device__ __forceinline__ void gv_unpack(float2 v, float (&o)[2]) { o[0] = v.x; o[1] = v.y; }
__device__ __forceinline__ void gv_unpack(float4 v, float (&o)[4]) { o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w; }
__device__ __forceinline__ void gv_unpack(double v, double (&o)[1]) { o[0] = v; }
__device__ __forceinline__ void gv_unpack(double2 v, double (&o)[2]) { o[0] = v.x; o[1] = v.y; }
__device__ __forceinline__ void gv_store(float *p, const float (&o)[1]) { *p = o[0]; }
__device__ __forceinline__ void gv_store(float *p, const float (&o)[2]) { *reinterpret_cast<float2 *>(p) = make_float2(o[0], o[1]); }
__device__ __forceinline__ void gv_store(float *p, const float (&o)[4])
{
    *reinterpret_cast<float4 *>(p) = make_float4(o[0], o[1], o[2], o[3]);
}
__device__ __forceinline__ void gv_store(double *p, const double (&o)[1]) { *p = o[0]; }
__device__ __forceinline__ void gv_store(double *p, const double (&o)[2]) { *reinterpret_cast<double2 *>(p) = make_double2(o[0], o[1]); }

// L2_ONLY: upwind rows written by other SMs during this launch (dataflow and
// persistent schedules) are read around L1.
template <typename Real, int VG, bool L2_ONLY>
__device__ __forceinline__ void gv_load(const Real *p, Real (&o)[VG])
{
    using V = typename GVec<Real, VG>::T;
    const V *vp = reinterpret_cast<const V *>(p);
    if constexpr (L2_ONLY) gv_unpack(__ldcg(vp), o);
    else gv_unpack(*vp, o);
}

// Read access to one item's record: item i of a shared-memory tile, or a
// record held in registers (the direct variant).
template <typename Real, int IPW>
struct TileView {
    const RecordTile<Real, IPW> &T;
    uint32_t i;
    __device__ __forceinline__ Real f(int k) const { return T.f[k][i]; }
    __device__ __forceinline__ uint32_t u(int k) const { return T.u[k][i]; }
};

template <typename Real>
struct RegRecord {
    Real fv[21];
    uint32_t uv[8];  // uv[7]: the Original solver's row order
    __device__ __forceinline__ Real f(int k) const { return fv[k]; }
    __device__ __forceinline__ uint32_t u(int k) const { return uv[k]; }
};

// One record from global memory straight into registers (read-only path).
// kind: the solver the caller applies; only Original needs the row-order
// word after u[] (NoPivot callers pass the constant and skip its load).
template <typename Real>
__device__ __forceinline__ void load_record(const ItemRecord<Real> *__restrict__ src, RegRecord<Real> &r,
                                            uint32_t kind = kSolveNoPivot)
{
    constexpr int N = (21 * sizeof(Real) + 28 + 15) / 16;  // f[] and u[]
    uint4 v[N + 1];
    const uint4 *s = reinterpret_cast<const uint4 *>(src);
#pragma unroll
    for (int i = 0; i < N; ++i) v[i] = __ldg(s + i);
    const bool order = kind == kSolveOriginal;
    constexpr int tail = (21 * sizeof(Real) + 28) / 16;  // the chunk holding the row order
    if (order && tail == N) v[N] = __ldg(s + N);
    const Real *fr = reinterpret_cast<const Real *>(v);
    const uint32_t *ur = reinterpret_cast<const uint32_t *>(reinterpret_cast<const char *>(v) + 21 * sizeof(Real));
#pragma unroll
    for (int k = 0; k < 21; ++k) r.fv[k] = fr[k];
#pragma unroll
    for (int k = 0; k < 7; ++k) r.uv[k] = ur[k];
    r.uv[7] = order ? ur[7] : 0u;
}

// A compact record into registers, with the factors rebuilt.
template <typename Real>
__device__ __forceinline__ void load_record(const CompactRecord<Real> *__restrict__ src, RegRecord<Real> &r,
                                            uint32_t kind = kSolveNoPivot)
{
    constexpr int N = sizeof(CompactRecord<Real>) / 16;
    uint4 v[N];
    const uint4 *s = reinterpret_cast<const uint4 *>(src);
#pragma unroll
    for (int i = 0; i < N; ++i) v[i] = __ldg(s + i);
    const Real *fr = reinterpret_cast<const Real *>(v);
    const uint32_t *ur =
        reinterpret_cast<const uint32_t *>(reinterpret_cast<const char *>(v) + kCompactF<Real> * sizeof(Real));
#pragma unroll
    for (int k = 0; k < 7; ++k) r.uv[k] = ur[k];
    r.uv[7] = 0;
    if (r.uv[0] == kSentinel) return;
    ItemFactor<Real> F;
    bool out[4];
#pragma unroll
    for (int f = 0; f < 4; ++f) {
        F.t1[f] = fr[f];
        F.t2[f] = Real(2) * fr[f];
        out[f] = fr[f] > Real(0);
    }
    if constexpr (kCompactF<Real> == 10) item_lu(F, fr[5], fr[6], out, kind, kind == kSolveNoPivot ? fr + 7 : nullptr);
    else item_lu(F, fr[5], fr[6], out, kind);
#pragma unroll
    for (int f = 0; f < 4; ++f) r.fv[f] = F.t1[f];
    r.fv[4] = fr[4];
    Real f16[16];
    factor16(F, kind, f16);
#pragma unroll
    for (int i = 0; i < 16; ++i) r.fv[5 + i] = f16[i];
    r.uv[7] = F.perm;
}

// A compact record into registers without its factors: the face terms
// (fv[0..3]), the volume source factor (fv[4]), the volume terms d1, d2 in
// fv[5], fv[6] (FP64: the three NoPivot reciprocals in fv[7..9]) and the
// integer words; compact_factor_nopivot rebuilds the NoPivot LU later, once
// the task's upwind loads are in flight.
template <typename Real>
__device__ __forceinline__ void load_compact_raw(const CompactRecord<Real> *__restrict__ src, RegRecord<Real> &r)
{
    constexpr int N = sizeof(CompactRecord<Real>) / 16;
    uint4 v[N];
    const uint4 *s = reinterpret_cast<const uint4 *>(src);
#pragma unroll
    for (int i = 0; i < N; ++i) v[i] = __ldg(s + i);
    const Real *fr = reinterpret_cast<const Real *>(v);
    const uint32_t *ur =
        reinterpret_cast<const uint32_t *>(reinterpret_cast<const char *>(v) + kCompactF<Real> * sizeof(Real));
#pragma unroll
    for (int k = 0; k < 7; ++k) r.uv[k] = ur[k];
    r.uv[7] = 0;
#pragma unroll
    for (int k = 0; k < kCompactF<Real>; ++k) r.fv[k] = fr[k];
}

template <typename Real>
__device__ __forceinline__ void compact_factor_nopivot(RegRecord<Real> &r)
{
    ItemFactor<Real> F;
    bool out[4];
#pragma unroll
    for (int f = 0; f < 4; ++f) {
        F.t1[f] = r.fv[f];
        F.t2[f] = Real(2) * r.fv[f];
        out[f] = r.fv[f] > Real(0);
    }
    Real recip[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) recip[k] = kCompactF<Real> == 10 ? r.fv[7 + k] : Real(0);
    item_lu(F, r.fv[5], r.fv[6], out, (uint32_t)kSolveNoPivot, kCompactF<Real> == 10 ? recip : nullptr);
    Real f16[16];
    factor16(F, (uint32_t)kSolveNoPivot, f16);
#pragma unroll
    for (int i = 0; i < 16; ++i) r.fv[5 + i] = f16[i];
}

// All the inputs of one (item, VG groups) task, loaded before any arithmetic.
template <typename Real, int VG>
struct PairIn {
    Real q[4][VG];
    Real pn[4][3][VG];  // [face][the three cell vertices j != f, increasing][group]
};

// Source of one task (fixed angular source, FP64 only, plus the isotropic
// total source; either may be absent).
template <typename Real, int VG, typename View>
__device__ __forceinline__ void pair_load_source(const LevelArgs &p, const View &R, uint32_t g, PairIn<Real, VG> &in)
{
    const uint32_t G = p.G;
    const uint32_t rowG = 4u * G;  // G <= 64: 32-bit operands, one widening multiply per address
    const uint32_t c = R.u(0);
    const Real *__restrict__ iso = reinterpret_cast<const Real *>(p.iso);
    if (p.qang) {
        const double *qa = p.qang + (uint64_t)R.u(1) * rowG + g;
        const Real *ic = iso ? iso + (uint64_t)c * rowG + g : nullptr;
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            Real icv[VG];
            if (ic) gv_load<Real, VG, false>(ic + v * G, icv);
#pragma unroll
            for (int k = 0; k < VG; ++k) in.q[v][k] = ic ? (Real)qa[v * G + k] + icv[k] : (Real)qa[v * G + k];
        }
    } else if (iso) {
        const Real *ic = iso + (uint64_t)c * rowG + g;
#pragma unroll
        for (int v = 0; v < 4; ++v) gv_load<Real, VG, false>(ic + v * G, in.q[v]);
    } else {
#pragma unroll
        for (int v = 0; v < 4; ++v)
#pragma unroll
            for (int k = 0; k < VG; ++k) in.q[v][k] = Real(0);
    }
}

// Upwind values of one task: for each incoming interior face, the
// neighbour's psi at the three face vertices.
template <typename Real, int VG, bool L2_ONLY, typename View>
__device__ __forceinline__ void pair_load_upwind(const LevelArgs &p, const View &R, uint32_t g, PairIn<Real, VG> &in)
{
    const uint32_t G = p.G;
    const uint32_t rowG = 4u * G;  // G <= 64: 32-bit operands, one widening multiply per address
    const Real *__restrict__ psi = reinterpret_cast<const Real *>(p.psi);
    const uint32_t nmap = R.u(2);
#pragma unroll
    for (int f = 0; f < 4; ++f) {
        const uint32_t row = R.u(3 + f);
        const bool live = R.f(f) < Real(0) && row != kNoRow;
        const Real *nrow = psi + (uint64_t)(live ? row : 0u) * rowG + g;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const int j = k < f ? k : k + 1;
            const uint32_t nv = (nmap >> ((f * 4 + j) * 2)) & 3u;
            if (live) {
                gv_load<Real, VG, L2_ONLY>(nrow + nv * G, in.pn[f][k]);
            } else {
#pragma unroll
                for (int e = 0; e < VG; ++e) in.pn[f][k][e] = Real(0);
            }
        }
    }
}

template <typename Real, int IPW, int VG, bool L2_ONLY>
__device__ __forceinline__ void pair_load(const LevelArgs &p, const RecordTile<Real, IPW> &T, uint32_t i,
                                          uint32_t g, PairIn<Real, VG> &in)
{
    const TileView<Real, IPW> R{T, i};
    pair_load_source<Real, VG>(p, R, g, in);
    pair_load_upwind<Real, VG, L2_ONLY>(p, R, g, in);
}

// The right-hand-side steps of the record's 4x4 solver on one group, in the
// reference's order: NoPivot's elimination and back substitution, Original's
// row order then forward and backward substitution with the factored matrix
// (its diagonal holds reciprocals), Cramer's x = inv b summed left to right.
template <typename Real, bool ANY, typename View>
__device__ __forceinline__ void solve_apply(uint32_t kind, const View &R, Real (&b)[4])
{
    if (!ANY || kind == kSolveNoPivot) {
        b[0] = b[0] * R.f(5);
        b[1] = b[1] - b[0] * R.f(9);
        b[2] = b[2] - b[0] * R.f(10);
        b[3] = b[3] - b[0] * R.f(11);
        b[1] = b[1] * R.f(12);
        b[2] = b[2] - b[1] * R.f(15);
        b[3] = b[3] - b[1] * R.f(16);
        b[2] = b[2] * R.f(17);
        b[3] = b[3] - b[2] * R.f(19);
        b[3] = div_ref(b[3], R.f(20));
        b[2] = b[2] - R.f(18) * b[3];
        b[1] = b[1] - R.f(14) * b[3] - R.f(13) * b[2];
        b[0] = b[0] - R.f(8) * b[3] - R.f(7) * b[2] - R.f(6) * b[1];
    } else if (kind == kSolveOriginal) {
        const uint32_t perm = R.u(7);
        Real x[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const uint32_t src = (perm >> (2 * i)) & 3u;
            x[i] = src == 0 ? b[0] : src == 1 ? b[1] : src == 2 ? b[2] : b[3];
        }
#pragma unroll
        for (int column = 0; column < 3; ++column)
#pragma unroll
            for (int row = column + 1; row < 4; ++row) x[row] -= R.f(5 + 4 * row + column) * x[column];
#pragma unroll
        for (int column = 3; column >= 0; --column) {
            x[column] *= R.f(5 + 5 * column);
#pragma unroll
            for (int row = column - 1; row >= 0; --row) x[row] -= R.f(5 + 4 * row + column) * x[column];
        }
#pragma unroll
        for (int i = 0; i < 4; ++i) b[i] = x[i];
    } else {
        Real x[4];
#pragma unroll
        for (int r = 0; r < 4; ++r)
            x[r] = R.f(5 + 4 * r) * b[0] + R.f(6 + 4 * r) * b[1] + R.f(7 + 4 * r) * b[2] + R.f(8 + 4 * r) * b[3];
#pragma unroll
        for (int i = 0; i < 4; ++i) b[i] = x[i];
    }
}

// The per-group arithmetic of one task, group by group in the reference's
// operation order (the factors are read once per task).
template <typename Real, int VG, typename View, bool ANY = false>
__device__ __forceinline__ void pair_solve_store_v(const LevelArgs &p, const View &R, uint32_t g,
                                                   const PairIn<Real, VG> &in)
{
    Real res[4][VG];
#pragma unroll
    for (int e = 0; e < VG; ++e) {
        const Real q[4] = {in.q[0][e], in.q[1][e], in.q[2][e], in.q[3][e]};
        const Real vs20 = R.f(4);
        Real b[4];
        b[0] = vs20 * (Real(2) * q[0] + q[1] + q[2] + q[3]);
        b[1] = vs20 * (q[0] + Real(2) * q[1] + q[2] + q[3]);
        b[2] = vs20 * (q[0] + q[1] + Real(2) * q[2] + q[3]);
        b[3] = vs20 * (q[0] + q[1] + q[2] + Real(2) * q[3]);
        // Upwind faces in increasing order; for face f, rows r != f in
        // increasing order, each subtracting its three terms j != f in
        // increasing order.
#pragma unroll
        for (int f = 0; f < 4; ++f) {
            const Real t1 = R.f(f);
            if (t1 < Real(0)) {
                const Real t2 = Real(2) * t1;
#pragma unroll
                for (int r = 0; r < 4; ++r) {
                    if (r == f) continue;
#pragma unroll
                    for (int k = 0; k < 3; ++k) {
                        const int j = k < f ? k : k + 1;
                        b[r] -= (r == j ? t2 : t1) * in.pn[f][k][e];
                    }
                }
            }
        }
        solve_apply<Real, ANY>(p.solver, R, b);
#pragma unroll
        for (int v = 0; v < 4; ++v) res[v][e] = b[v];
    }
    Real *__restrict__ out = reinterpret_cast<Real *>(p.psi) + (uint64_t)R.u(1) * (4u * p.G) + g;
#pragma unroll
    for (int v = 0; v < 4; ++v) gv_store(out + v * p.G, res[v]);
}

// FP32 with an even group vector: the same arithmetic on pairs of groups
// with Blackwell's packed FP32x2 add / multiply / fused multiply-add (half
// the arithmetic instructions).  The source sum is reassociated as
// vs20 * ((q0 + q1) + (q2 + q3) + q_v); FP32 results are checked by
// tolerance, the FP64 path above keeps the reference's order.
// The volume source term of the right-hand side, V/20 (sum_j q_j + q_v), in
// place of the sources (packed FP32x2): it does not depend on the previous
// level, so the direct kernel forms it before waiting for that level.
template <int VG, typename View>
__device__ __forceinline__ void pair_source_rhs_f32x2(const View &R, PairIn<float, VG> &in)
{
    const float vs = R.f(4);
    const float2 vs2 = make_float2(vs, vs);
#pragma unroll
    for (int e = 0; e < VG; e += 2) {
        float2 q[4];
#pragma unroll
        for (int v = 0; v < 4; ++v) q[v] = make_float2(in.q[v][e], in.q[v][e + 1]);
        const float2 s = __fadd2_rn(__fadd2_rn(q[0], q[1]), __fadd2_rn(q[2], q[3]));
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            const float2 b = __fmul2_rn(vs2, __fadd2_rn(s, q[v]));
            in.q[v][e] = b.x;
            in.q[v][e + 1] = b.y;
        }
    }
}

// PRE: in.q already holds the volume source term (pair_source_rhs_f32x2).
template <int VG, typename View, bool PRE = false>
__device__ __forceinline__ void pair_solve_store_f32x2(const LevelArgs &p, const View &R, uint32_t g,
                                                       const PairIn<float, VG> &in)
{
    static_assert(VG % 2 == 0, "pairs of groups");
    float res[4][VG];
    const float vs = R.f(4);
    const float2 vs2 = make_float2(vs, vs);
#pragma unroll
    for (int e = 0; e < VG; e += 2) {
        float2 q[4];
#pragma unroll
        for (int v = 0; v < 4; ++v) q[v] = make_float2(in.q[v][e], in.q[v][e + 1]);
        float2 b[4];
        if constexpr (PRE) {
#pragma unroll
            for (int v = 0; v < 4; ++v) b[v] = q[v];
        } else {
            const float2 s = __fadd2_rn(__fadd2_rn(q[0], q[1]), __fadd2_rn(q[2], q[3]));
#pragma unroll
            for (int v = 0; v < 4; ++v) b[v] = __fmul2_rn(vs2, __fadd2_rn(s, q[v]));
        }
#pragma unroll
        for (int f = 0; f < 4; ++f) {
            const float t1 = R.f(f);
            if (t1 < 0.0f) {
                const float2 m1 = make_float2(-t1, -t1), m2 = make_float2(-2.0f * t1, -2.0f * t1);
#pragma unroll
                for (int r = 0; r < 4; ++r) {
                    if (r == f) continue;
#pragma unroll
                    for (int k = 0; k < 3; ++k) {
                        const int j = k < f ? k : k + 1;
                        const float2 pn = make_float2(in.pn[f][k][e], in.pn[f][k][e + 1]);
                        b[r] = __ffma2_rn(r == j ? m2 : m1, pn, b[r]);
                    }
                }
            }
        }
        auto sp = [](float x) { return make_float2(x, x); };
        b[0] = __fmul2_rn(b[0], sp(R.f(5)));
        b[1] = __ffma2_rn(sp(-R.f(9)), b[0], b[1]);
        b[2] = __ffma2_rn(sp(-R.f(10)), b[0], b[2]);
        b[3] = __ffma2_rn(sp(-R.f(11)), b[0], b[3]);
        b[1] = __fmul2_rn(b[1], sp(R.f(12)));
        b[2] = __ffma2_rn(sp(-R.f(15)), b[1], b[2]);
        b[3] = __ffma2_rn(sp(-R.f(16)), b[1], b[3]);
        b[2] = __fmul2_rn(b[2], sp(R.f(17)));
        b[3] = __ffma2_rn(sp(-R.f(19)), b[2], b[3]);
        b[3] = __fmul2_rn(b[3], sp(__fdividef(1.0f, R.f(20))));
        b[2] = __ffma2_rn(sp(-R.f(18)), b[3], b[2]);
        b[1] = __ffma2_rn(sp(-R.f(13)), b[2], __ffma2_rn(sp(-R.f(14)), b[3], b[1]));
        b[0] = __ffma2_rn(sp(-R.f(6)), b[1], __ffma2_rn(sp(-R.f(7)), b[2], __ffma2_rn(sp(-R.f(8)), b[3], b[0])));
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            res[v][e] = b[v].x;
            res[v][e + 1] = b[v].y;
        }
    }
    float *__restrict__ out = reinterpret_cast<float *>(p.psi) + (uint64_t)R.u(1) * (4u * p.G) + g;
#pragma unroll
    for (int v = 0; v < 4; ++v) gv_store(out + v * p.G, res[v]);
}

// The arithmetic of one task: packed FP32x2 where it applies.  ANY: the
// record may hold any of the four solvers (p.solver); otherwise NoPivot.
template <typename Real, int VG, typename View, bool ANY = false>
__device__ __forceinline__ void pair_solve_store_any(const LevelArgs &p, const View &R, uint32_t g,
                                                     const PairIn<Real, VG> &in)
{
    if constexpr (std::is_same<Real, float>::value && VG % 2 == 0 && !ANY) pair_solve_store_f32x2<VG>(p, R, g, in);
    else pair_solve_store_v<Real, VG, View, ANY>(p, R, g, in);
}

// FP32: a tet has at most three faces with omega.n < 0, so the upwind rows
// of a task fit three slots (the item's interior upwind faces in increasing
// face order) instead of four face-indexed ones: 3*3*VG loaded values live
// at once instead of 4*3*VG.  Slot s keeps the neighbour's psi at the face's
// three vertices j != f in increasing j.  Summation order differs from the
// face-indexed form (FP32 is checked by tolerance).
template <int VG>
struct SlotIn {
    float p[3][3][VG];
    uint32_t faces;  // slot s's face in bits 2s, 2s+1
    uint32_t count;  // occupied slots
};

template <int VG, typename View>
__device__ __forceinline__ void slot_load_upwind(const LevelArgs &p, const View &R, uint32_t g, SlotIn<VG> &in)
{
    const float *__restrict__ psi = reinterpret_cast<const float *>(p.psi);
    const uint32_t G = p.G, rowG = 4u * G, nmap = R.u(2);
    uint32_t live = 0;
#pragma unroll
    for (int f = 0; f < 4; ++f)
        if (R.f(f) < 0.0f && R.u(3 + f) != kNoRow) live |= 1u << f;
    uint32_t faces = 0, count = 0;
#pragma unroll
    for (int s = 0; s < 3; ++s) {
        const bool has = live != 0u;
        const uint32_t f = has ? (uint32_t)(__ffs(live) - 1) : 0u;
        live &= live - 1u;
        faces |= f << (2 * s);
        count += has ? 1u : 0u;
        const uint32_t row = f == 0u ? R.u(3) : f == 1u ? R.u(4) : f == 2u ? R.u(5) : R.u(6);
        const float *nrow = psi + (uint64_t)(has ? row : 0u) * rowG + g;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const uint32_t j = (uint32_t)k < f ? (uint32_t)k : (uint32_t)k + 1u;
            const uint32_t nv = (nmap >> ((f * 4u + j) * 2u)) & 3u;
            if (has) {
                gv_load<float, VG, false>(nrow + nv * G, in.p[s][k]);
            } else {
#pragma unroll
                for (int e = 0; e < VG; ++e) in.p[s][k][e] = 0.0f;
            }
        }
    }
    in.faces = faces;
    in.count = count;
}

// The solve of a slotted task (packed FP32x2; in.q holds the volume source
// term): for an upwind face f with A_f/12 = t, row r != f loses t (S + p_r),
// S the sum of the face's three vertex values and p_r the value at vertex r.
template <int VG, typename View>
__device__ __forceinline__ void slot_solve_store_f32x2(const LevelArgs &p, const View &R, uint32_t g,
                                                       const float (&q)[4][VG], const SlotIn<VG> &in)
{
    static_assert(VG % 2 == 0, "pairs of groups");
    float c[3][4];  // per slot and row: -t, or 0 on the face's own row and for an empty slot
#pragma unroll
    for (int s = 0; s < 3; ++s) {
        const uint32_t f = (in.faces >> (2 * s)) & 3u;
        const float t = (uint32_t)s < in.count ? (f == 0u ? R.f(0) : f == 1u ? R.f(1) : f == 2u ? R.f(2) : R.f(3))
                                               : 0.0f;
#pragma unroll
        for (int r = 0; r < 4; ++r) c[s][r] = f == (uint32_t)r ? 0.0f : -t;
    }
    float res[4][VG];
#pragma unroll
    for (int e = 0; e < VG; e += 2) {
        float2 b[4];
#pragma unroll
        for (int v = 0; v < 4; ++v) b[v] = make_float2(q[v][e], q[v][e + 1]);
#pragma unroll
        for (int s = 0; s < 3; ++s) {
            const uint32_t f = (in.faces >> (2 * s)) & 3u;
            float2 pk[3];
#pragma unroll
            for (int k = 0; k < 3; ++k) pk[k] = make_float2(in.p[s][k][e], in.p[s][k][e + 1]);
            const float2 S = __fadd2_rn(__fadd2_rn(pk[0], pk[1]), pk[2]);
            // vertex r is k = r (r < f) or k = r - 1 (r > f)
            const float2 p0 = pk[0];
            const float2 p1 = f > 1u ? pk[1] : pk[0];
            const float2 p2 = f > 2u ? pk[2] : pk[1];
            const float2 p3 = pk[2];
            b[0] = __ffma2_rn(make_float2(c[s][0], c[s][0]), __fadd2_rn(S, p0), b[0]);
            b[1] = __ffma2_rn(make_float2(c[s][1], c[s][1]), __fadd2_rn(S, p1), b[1]);
            b[2] = __ffma2_rn(make_float2(c[s][2], c[s][2]), __fadd2_rn(S, p2), b[2]);
            b[3] = __ffma2_rn(make_float2(c[s][3], c[s][3]), __fadd2_rn(S, p3), b[3]);
        }
        auto sp = [](float x) { return make_float2(x, x); };
        b[0] = __fmul2_rn(b[0], sp(R.f(5)));
        b[1] = __ffma2_rn(sp(-R.f(9)), b[0], b[1]);
        b[2] = __ffma2_rn(sp(-R.f(10)), b[0], b[2]);
        b[3] = __ffma2_rn(sp(-R.f(11)), b[0], b[3]);
        b[1] = __fmul2_rn(b[1], sp(R.f(12)));
        b[2] = __ffma2_rn(sp(-R.f(15)), b[1], b[2]);
        b[3] = __ffma2_rn(sp(-R.f(16)), b[1], b[3]);
        b[2] = __fmul2_rn(b[2], sp(R.f(17)));
        b[3] = __ffma2_rn(sp(-R.f(19)), b[2], b[3]);
        b[3] = __fmul2_rn(b[3], sp(__fdividef(1.0f, R.f(20))));
        b[2] = __ffma2_rn(sp(-R.f(18)), b[3], b[2]);
        b[1] = __ffma2_rn(sp(-R.f(13)), b[2], __ffma2_rn(sp(-R.f(14)), b[3], b[1]));
        b[0] = __ffma2_rn(sp(-R.f(6)), b[1], __ffma2_rn(sp(-R.f(7)), b[2], __ffma2_rn(sp(-R.f(8)), b[3], b[0])));
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            res[v][e] = b[v].x;
            res[v][e + 1] = b[v].y;
        }
    }
    float *__restrict__ out = reinterpret_cast<float *>(p.psi) + (uint64_t)R.u(1) * (4u * p.G) + g;
#pragma unroll
    for (int v = 0; v < 4; ++v) gv_store(out + v * p.G, res[v]);
}

// Whether a task's arithmetic runs packed FP32x2 (and can form its volume
// source term before the wait).
template <typename Real, int VG, bool ANY>
constexpr bool kPairedF32 = std::is_same<Real, float>::value && VG % 2 == 0 && !ANY;

template <typename Real, int IPW, int VG>
__device__ __forceinline__ void pair_solve_store(const LevelArgs &p, const RecordTile<Real, IPW> &T, uint32_t i,
                                                 uint32_t g, const PairIn<Real, VG> &in)
{
    pair_solve_store_v<Real, VG>(p, TileView<Real, IPW>{T, i}, g, in);
}

// Tasks per lane in flight: fewer as the vector width grows (registers).
template <typename Real, int IPW, int VG>
__host__ __device__ constexpr int record_unroll()
{
    return VG == 1 ? (IPW == 32 ? 4 : 2) : (VG == 2 && sizeof(Real) == 4 ? 2 : 1);
}

// The warp walks the IPW * (G / VG) tasks of a tile: task t -> item
// t / (G / VG), groups VG * (t % (G / VG)) and the next VG - 1.
template <typename Real, int IPW, int VG, bool L2_ONLY>
__device__ __forceinline__ void record_pairs(const LevelArgs &p, const RecordTile<Real, IPW> &T, uint32_t lane)
{
    constexpr int UNROLL = record_unroll<Real, IPW, VG>();
    const uint32_t gpv = p.G / VG, ntask = (uint32_t)IPW * gpv;
    for (uint32_t q0 = lane; q0 < ntask; q0 += 32u * UNROLL) {
        PairIn<Real, VG> in[UNROLL];
        uint32_t item[UNROLL], grp[UNROLL];
        bool live[UNROLL];
#pragma unroll
        for (int u = 0; u < UNROLL; ++u) {
            const uint32_t q = q0 + 32u * u;
            const uint32_t it = gpv == 1u ? q : __umulhi(q, p.vmagic);
            item[u] = it < (uint32_t)IPW ? it : 0u;
            grp[u] = (q - it * gpv) * VG;
            live[u] = q < ntask && T.u[0][item[u]] != kSentinel;
            if (live[u]) pair_load<Real, IPW, VG, L2_ONLY>(p, T, item[u], grp[u], in[u]);
        }
#pragma unroll
        for (int u = 0; u < UNROLL; ++u)
            if (live[u]) pair_solve_store<Real, IPW, VG>(p, T, item[u], grp[u], in[u]);
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
template <typename Real, int IPW, int VG>
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
    record_pairs<Real, IPW, VG, false>(p, tiles[w], lane);
}

// Record prefetch of a deep launch (PF kernels): the task half a resident
// wave ahead (blocks of BS threads, MINB per SM) starts in a later wave,
// after this level's first blocks are gone; its record is prefetched into
// L2 now, so that its own record load (the head of its dependent chain)
// hits L2 instead of HBM.  The gpv tasks of an item share its 32-byte
// sectors.
template <typename Rec, int BS, int MINB>
__device__ __forceinline__ void prefetch_record_ahead(const Rec *__restrict__ rec, uint32_t t, uint32_t gpv,
                                                      uint32_t vmagic, uint64_t begin, uint64_t end)
{
    uint32_t nsm;
    asm("mov.u32 %0, %%nsmid;" : "=r"(nsm));
    const uint32_t t2 = t + nsm * (uint32_t)(MINB * BS / 2);
    const uint32_t itl2 = gpv == 1u ? t2 : __umulhi(t2, vmagic);
    const uint64_t it2 = begin + itl2;
    if (it2 < end) {
        const char *r2 = reinterpret_cast<const char *>(rec + it2);
        for (uint32_t sct = t2 - itl2 * gpv; sct * 32u < sizeof(Rec); sct += gpv)
            asm volatile("prefetch.global.L2 [%0];" ::"l"(r2 + sct * 32u));
    }
}

// Direct variant (level schedule only): one thread per (item, VG groups)
// task with the item's record loaded straight into registers -- the lanes of
// one item read the same 128/256 bytes and L1 serves the repeats -- and its
// source loaded before the wait on the previous level; only the upwind rows
// are read after it.  No shared memory.  Tasks of a level: item t / (G/VG),
// groups VG * (t % (G/VG)) and on (the host keeps a level's task count
// below 2^26 so that the multiply-high division is exact).
template <typename Real, int VG, int BS, typename Rec, int MINB = 1, bool ANY = false, bool PF = false>
__global__ void __launch_bounds__(BS, MINB)
sweep_direct_level_kernel(const LevelArgs p, const Rec *__restrict__ rec, const uint64_t begin, const uint64_t end)
{
    pdl_launch_dependents();
    const uint32_t gpv = p.G / VG;
    const uint32_t t = blockIdx.x * (uint32_t)BS + threadIdx.x;
    const uint32_t itl = gpv == 1u ? t : __umulhi(t, p.vmagic);
    const uint32_t g = (t - itl * gpv) * VG;
    const uint64_t it = begin + itl;
    bool live = it < end;
    RegRecord<Real> R;
    PairIn<Real, VG> in;
    // Compact NoPivot records without a register cap (MINB 1): the LU is
    // rebuilt after the upwind loads are issued, in their latency.  Under a
    // cap the four face-indexed upwind rows leave it no registers there and
    // it stays before the wait (FP64 at 102 registers measured 5% slower
    // the other way).
    constexpr bool kLate = std::is_same<Rec, CompactRecord<Real>>::value && !ANY && MINB == 1;
    if constexpr (PF) prefetch_record_ahead<Rec, BS, MINB>(rec, t, gpv, p.vmagic, begin, end);
    if (live) {
        if constexpr (kLate) load_compact_raw(rec + it, R);
        else load_record(rec + it, R, ANY ? p.solver : (uint32_t)kSolveNoPivot);
        live = R.u(0) != kSentinel;
    }
    if (live) {
        pair_load_source<Real, VG>(p, R, g, in);
        if constexpr (kPairedF32<Real, VG, ANY>) pair_source_rhs_f32x2<VG>(R, in);
    }
    pdl_wait_prerequisites();
    if (!live) return;
    pair_load_upwind<Real, VG, false>(p, R, g, in);
    if constexpr (kLate) compact_factor_nopivot(R);
    if constexpr (kPairedF32<Real, VG, ANY>) pair_solve_store_f32x2<VG, RegRecord<Real>, true>(p, R, g, in);
    else pair_solve_store_any<Real, VG, RegRecord<Real>, ANY>(p, R, g, in);
}

// The FP32 direct kernel with slotted upwind rows (even vector widths).
// PF: the launch is several resident waves deep (record prefetch, below).
template <int VG, int BS, typename Rec, int MINB, bool PF = false>
__global__ void __launch_bounds__(BS, MINB)
sweep_direct_slot_kernel(const LevelArgs p, const Rec *__restrict__ rec, const uint64_t begin, const uint64_t end)
{
    pdl_launch_dependents();
    const uint32_t gpv = p.G / VG;
    const uint32_t t = blockIdx.x * (uint32_t)BS + threadIdx.x;
    const uint32_t itl = gpv == 1u ? t : __umulhi(t, p.vmagic);
    const uint32_t g = (t - itl * gpv) * VG;
    const uint64_t it = begin + itl;
    bool live = it < end;
    RegRecord<float> R;
    PairIn<float, VG> in;  // sources only
    // Compact records: the LU is rebuilt after the upwind loads are issued,
    // in their latency, not before the wait on the previous level -- except
    // at 14 blocks per SM (73 registers), where that order spills more and
    // measured slower.
    constexpr bool kLate = std::is_same<Rec, CompactRecord<float>>::value && MINB <= 12;
    if constexpr (PF) prefetch_record_ahead<Rec, BS, MINB>(rec, t, gpv, p.vmagic, begin, end);
    if (live) {
        if constexpr (kLate) load_compact_raw(rec + it, R);
        else load_record(rec + it, R, (uint32_t)kSolveNoPivot);
        live = R.u(0) != kSentinel;
    }
    if (live) {
        pair_load_source<float, VG>(p, R, g, in);
        pair_source_rhs_f32x2<VG>(R, in);
    }
    pdl_wait_prerequisites();
    if (!live) return;
    SlotIn<VG> sl;
    slot_load_upwind<VG>(p, R, g, sl);
    if constexpr (kLate) compact_factor_nopivot(R);
    slot_solve_store_f32x2<VG>(p, R, g, in.q, sl);
}

// Direct variant, two group vectors per task: the task covers 2*VG groups
// of one item (vector width 8 in FP32, 4 in FP64), swept as two halves that
// share the record (one load, one LU rebuild for compact records) and whose
// sources are both read before the wait; half the threads of the one-vector
// kernel for the same level.
template <typename Real, int VG, int BS, typename Rec>
__global__ void __launch_bounds__(BS)
sweep_direct2_level_kernel(const LevelArgs p, const Rec *__restrict__ rec, const uint64_t begin, const uint64_t end)
{
    pdl_launch_dependents();
    const uint32_t gpv = p.G / (2 * VG);
    const uint32_t t = blockIdx.x * (uint32_t)BS + threadIdx.x;
    const uint32_t itl = gpv == 1u ? t : __umulhi(t, p.vmagic);
    const uint32_t g = (t - itl * gpv) * (2 * VG);
    const uint64_t it = begin + itl;
    bool live = it < end;
    RegRecord<Real> R;
    PairIn<Real, VG> in0, in1;
    if (live) {
        load_record(rec + it, R);
        live = R.u(0) != kSentinel;
    }
    if (live) {
        pair_load_source<Real, VG>(p, R, g, in0);
        pair_load_source<Real, VG>(p, R, g + VG, in1);
    }
    pdl_wait_prerequisites();
    if (!live) return;
    pair_load_upwind<Real, VG, false>(p, R, g, in0);
    pair_solve_store_any<Real, VG>(p, R, g, in0);
    pair_load_upwind<Real, VG, false>(p, R, g + VG, in1);
    pair_solve_store_any<Real, VG>(p, R, g + VG, in1);
}

// Wait on one completion flag: back-to-back polls first (one poll is an L2
// round trip), then polls 64 ns apart; gives up after df.spin_limit polls
// (records the item and face, raises abort) so that no wait can hang.
__device__ __forceinline__ uint32_t ld_relaxed_gpu(const uint32_t *p)
{
    uint32_t v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Polls with relaxed loads (no L1 invalidation per poll); the caller follows
// its last successful wait with one fence.acq_rel.gpu, which with the
// observed release forms the acquire pattern of the PTX memory model.
__device__ __forceinline__ bool wait_flag_tight(const DataflowArgs &df, uint32_t epoch, const uint32_t *flag,
                                                uint32_t ca, int f)
{
    for (uint32_t spin = 0; spin < df.spin_limit; ++spin) {
        if (ld_relaxed_gpu(flag) == epoch) return true;
        if ((spin & 31u) == 31u && *(volatile const uint32_t *)df.abort) return false;
        if (spin >= 128) __nanosleep(64);
    }
    if (atomicCAS(df.err, 0u, (uint32_t)kErrTimeoutCode) == 0u) {
        df.err[1] = ca;
        df.err[2] = (uint32_t)f;
    }
    atomicExch(df.abort, 1u);
    return false;
}

// Direct dataflow: one cooperative launch per sweep; warps take chunks of 32
// (item, group vector) tasks in level order, round-robin; a lane loads its
// record and source, waits for the completion flags of its upwind tasks (the
// same group vector of the neighbour's item, flag index = row * (G/VG) + gv),
// sweeps its groups and releases its own flag.  G/VG must be a power of two
// up to 32, so a chunk is 32/(G/VG) whole items and never spans two levels
// (levels hold multiples of 32 items).  Deadlock freedom as for the other
// dataflow kernels: tasks wait only on lower levels, warps visit chunks in
// increasing order, every warp is resident.
template <typename Real, int VG, typename Rec>
__global__ void __launch_bounds__(128)
sweep_direct_dataflow_kernel(const LevelArgs p, const Rec *__restrict__ rec, const DataflowArgs df)
{
    const uint32_t gpv = p.G / VG;
    const uint32_t lg = 31u - __clz(gpv);  // log2(gpv)
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t warp = (uint64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const uint64_t nwarps = (uint64_t)gridDim.x * (blockDim.x >> 5);
    const uint64_t ipc = 32u >> lg;  // items per chunk
    const uint64_t nchunks = df.n_items / ipc;
    const uint32_t epoch = *df.epoch;
    const uint32_t gv = lane & (gpv - 1u), g = gv * VG;
    for (uint64_t ch = warp; ch < nchunks; ch += nwarps) {
        if (*(volatile const uint32_t *)df.abort) break;
        const uint64_t it = ch * ipc + (lane >> lg);
        RegRecord<Real> R;
        load_record(rec + it, R);
        if (R.u(0) == kSentinel) continue;
        PairIn<Real, VG> in;
        pair_load_source<Real, VG>(p, R, g, in);
        bool ok = true;
#pragma unroll
        for (int f = 0; f < 4; ++f) {
            const uint32_t row = R.u(3 + f);
            if (ok && R.f(f) < Real(0) && row != kNoRow)
                ok = wait_flag_tight(df, epoch, df.done + (size_t)row * gpv + gv, R.u(1), f);
        }
        if (!ok) continue;
        asm volatile("fence.acq_rel.gpu;" ::: "memory");
        pair_load_upwind<Real, VG, true>(p, R, g, in);
        pair_solve_store_any<Real, VG>(p, R, g, in);
        st_release_gpu(df.done + (size_t)R.u(1) * gpv + gv, epoch);  // orders this thread's psi stores first
    }
}

// Dataflow schedule: persistent warps take IPW-item chunks round-robin; lane
// i < IPW stages record i and waits for its upwind items, the warp sweeps the
// chunk's pairs, fences, and lane i publishes item i's epoch.
template <typename Real, int IPW, int VG>
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
        record_pairs<Real, IPW, VG, true>(p, T, lane);
        __threadfence();
        __syncwarp();
        if (ok) st_release_gpu(df.done + ca, epoch);
    }
}

// Block-level barrier across the whole (co-resident) grid with a bounded
// wait: thread 0 of every block adds one arrival to *count and waits until
// it reaches `target`; gives up after spin_limit polls (records the level in
// err, raises abort) so that no wait can hang the device.
__device__ __forceinline__ bool grid_barrier(unsigned long long *count, unsigned long long target,
                                             const DataflowArgs &df, uint32_t level)
{
    __shared__ int ok_s;
    __syncthreads();  // the block's psi stores happen before thread 0's fence
    if (threadIdx.x == 0) {
        int ok = 1;
        __threadfence();
        atomicAdd(count, 1ull);
        unsigned backoff = 32;
        uint32_t spin = 0;
        for (;;) {
            unsigned long long v;
            asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(count) : "memory");
            if (v >= target) break;
            if (*(volatile const uint32_t *)df.abort || ++spin > df.spin_limit) {
                if (atomicCAS(df.err, 0u, (uint32_t)kErrTimeoutCode) == 0u) {
                    df.err[1] = level;
                    df.err[2] = 4u;  // face 4: a level barrier, not an upwind face
                }
                atomicExch(df.abort, 1u);
                ok = 0;
                break;
            }
            __nanosleep(backoff);
            if (backoff < 256) backoff <<= 1;
        }
        __threadfence();
        ok_s = ok;
    }
    __syncthreads();
    return ok_s != 0;
}

// Persistent levels: one cooperative launch per sweep; all warps take the
// chunks of level L (warp w: chunks w, w + W, ...), then every block meets at
// a barrier before level L+1.  The records of a warp's first chunk of the
// next level are staged before the barrier (they do not depend on psi).
template <typename Real, int IPW, int VG>
__global__ void __launch_bounds__(128)
sweep_record_persist_kernel(const LevelArgs p, const ItemRecord<Real> *__restrict__ rec,
                            const uint64_t *__restrict__ level_off, const uint32_t n_levels,
                            unsigned long long *barrier, const DataflowArgs df)
{
    __shared__ RecordTile<Real, IPW> tiles[4][2];
    const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
    const uint64_t warp = (uint64_t)blockIdx.x * 4 + w;
    const uint64_t nwarps = (uint64_t)gridDim.x * 4;
    int cur = 0;
    // stage the first chunk of level 0
    if (warp * IPW < level_off[1] - level_off[0]) tile_fill<Real, IPW>(tiles[w][cur], rec + level_off[0] + warp * IPW + lane, lane, true);
    for (uint32_t L = 0; L < n_levels; ++L) {
        const uint64_t b = level_off[L], nch = (level_off[L + 1] - b) / IPW;
        for (uint64_t ch = warp, k = 0; ch < nch; ch += nwarps, ++k) {
            if (k > 0) tile_fill<Real, IPW>(tiles[w][cur], rec + b + ch * IPW + lane, lane, true);
            __syncwarp();
            record_pairs<Real, IPW, VG, true>(p, tiles[w][cur], lane);
            __syncwarp();
        }
        if (L + 1 < n_levels) {
            const uint64_t nb = level_off[L + 1];
            if (warp * IPW < level_off[L + 2] - nb)
                tile_fill<Real, IPW>(tiles[w][cur ^ 1], rec + nb + warp * IPW + lane, lane, true);
            if (!grid_barrier(barrier, (unsigned long long)(L + 1) * gridDim.x, df, L)) return;
            cur ^= 1;
        }
    }
}

// Kernel selection by items per warp and group vector width.  The double
// variants stop at VG = 2 (one 16-byte access); two 32-item double tiles per
// warp (persistent levels) exceed static shared memory.
template <typename Real, int IPW, int VG>
struct LevelK {
    static const void *fn() { return (const void *)sweep_record_level_kernel<Real, IPW, VG>; }
};
template <typename Real, int IPW, int VG>
struct DataflowK {
    static const void *fn() { return (const void *)sweep_record_dataflow_kernel<Real, IPW, VG>; }
};
template <typename Real, int IPW, int VG>
struct PersistK {
    static const void *fn()
    {
        if constexpr (sizeof(Real) == 8 && IPW == 32) return nullptr;
        else return (const void *)sweep_record_persist_kernel<Real, IPW, VG>;
    }
};

template <typename Real, template <typename, int, int> class K, int IPW>
static const void *record_fn_vg(int vg)
{
    switch (vg) {
    case 1: return K<Real, IPW, 1>::fn();
    case 2: return K<Real, IPW, 2>::fn();
    case 4:
        if constexpr (sizeof(Real) == 4) return K<Real, IPW, 4>::fn();
        else return nullptr;
    default: return nullptr;
    }
}

template <typename Real, template <typename, int, int> class K>
static const void *record_fn(int ipw, int vg)
{
    switch (ipw) {
    case 8: return record_fn_vg<Real, K, 8>(vg);
    case 16: return record_fn_vg<Real, K, 16>(vg);
    case 32: return record_fn_vg<Real, K, 32>(vg);
    default: return nullptr;
    }
}

template <typename Real>
cudaError_t record_persist_blocks_per_sm(int ipw, int vg, int *blocks)
{
    const void *fn = record_fn<Real, PersistK>(ipw, vg);
    if (!fn) return cudaErrorInvalidValue;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks, fn, 128, 0);
}

template <typename Real>
cudaError_t launch_persist_record(int ipw, const LevelArgs &p, const void *rec, const uint64_t *level_off,
                                  uint32_t n_levels, unsigned long long *barrier, const DataflowArgs &df,
                                  unsigned grid, cudaStream_t s)
{
    const void *fn = record_fn<Real, PersistK>(ipw, (int)p.vg);
    if (!fn || grid == 0) return cudaErrorInvalidValue;
    cudaError_t e = cudaMemsetAsync(barrier, 0, sizeof(unsigned long long), s);
    if (e != cudaSuccess) return e;
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
    void *args[] = {(void *)&p, (void *)&r, (void *)&level_off, (void *)&n_levels, (void *)&barrier, (void *)&df};
    return cudaLaunchKernelExC(&cfg, fn, args);
}

template <typename Real>
cudaError_t launch_item_records(const LevelArgs &p, uint64_t n, void *out, cudaStream_t s)
{
    if (n == 0) return cudaSuccess;
    item_record_kernel<Real><<<(unsigned)((n + 127) / 128), 128, 0, s>>>(p, n, (ItemRecord<Real> *)out);
    return cudaGetLastError();
}

template <typename Real, int BS, typename Rec, int MINB>
static const void *direct_fn_vg(int vg, bool pf = false)
{
    if constexpr (MINB == 10) {  // -96: the record prefetch of deep launches
        if (pf && vg == 1) return (const void *)sweep_direct_level_kernel<Real, 1, BS, Rec, MINB, false, true>;
        if (pf && vg == 2) return (const void *)sweep_direct_level_kernel<Real, 2, BS, Rec, MINB, false, true>;
        if constexpr (sizeof(Real) == 4)
            if (pf && vg == 4) return (const void *)sweep_direct_level_kernel<Real, 4, BS, Rec, MINB, false, true>;
    }
    switch (vg) {
    case 8:  // two 4-group halves per task (FP32)
        if constexpr (sizeof(Real) == 4 && MINB == 1) return (const void *)sweep_direct2_level_kernel<Real, 4, BS, Rec>;
        else return nullptr;
    case 1: return (const void *)sweep_direct_level_kernel<Real, 1, BS, Rec, MINB>;
    case 2: return (const void *)sweep_direct_level_kernel<Real, 2, BS, Rec, MINB>;
    case 4:
        if constexpr (sizeof(Real) == 4) return (const void *)sweep_direct_level_kernel<Real, 4, BS, Rec, MINB>;
        else if constexpr (MINB == 1) return (const void *)sweep_direct2_level_kernel<Real, 2, BS, Rec>;  // FP64 halves
        else return nullptr;
    default: return nullptr;
    }
}

template <typename Real, typename Rec>
static const void *direct_any_fn(int vg)
{
    switch (vg) {
    case 1: return (const void *)sweep_direct_level_kernel<Real, 1, 128, Rec, 1, true>;
    case 2: return (const void *)sweep_direct_level_kernel<Real, 2, 128, Rec, 1, true>;
    case 4:
        if constexpr (sizeof(Real) == 4) return (const void *)sweep_direct_level_kernel<Real, 4, 128, Rec, 1, true>;
        else return nullptr;
    default: return nullptr;
    }
}

template <typename Real, typename Rec, int BS, int MINB>
static const void *direct_slot_fn(int vg, bool pf)
{
    if constexpr (sizeof(Real) == 4) {
        if (vg == 2)
            return pf ? (const void *)sweep_direct_slot_kernel<2, BS, Rec, MINB, true>
                      : (const void *)sweep_direct_slot_kernel<2, BS, Rec, MINB>;
        if (vg == 4)
            return pf ? (const void *)sweep_direct_slot_kernel<4, BS, Rec, MINB, true>
                      : (const void *)sweep_direct_slot_kernel<4, BS, Rec, MINB>;
    }
    return nullptr;
}

template <typename Real, typename Rec>
static const void *direct_fn(int knob, int vg, uint32_t solver, bool pf = false)
{
    // Original and the Cramer solvers: one 128-thread kernel per vector width
    if (solver != kSolveNoPivot) return knob == 128 ? direct_any_fn<Real, Rec>(vg) : nullptr;
    switch (knob) {
    // slotted upwind rows: 64 threads with <= 102 / 85 / 73 registers
    case -196: return direct_slot_fn<Real, Rec, 64, 10>(vg, pf);
    case -180: return direct_slot_fn<Real, Rec, 64, 12>(vg, pf);
    case -172: return direct_slot_fn<Real, Rec, 64, 14>(vg, pf);
    case 64: return direct_fn_vg<Real, 64, Rec, 1>(vg);
    case 128: return direct_fn_vg<Real, 128, Rec, 1>(vg);
    case 256: return direct_fn_vg<Real, 256, Rec, 1>(vg);
    case -64: return direct_fn_vg<Real, 64, Rec, 16>(vg);   // <= 64 registers
    case -96: return direct_fn_vg<Real, 64, Rec, 10>(vg, pf);  // <= 102 registers
    case -80: return direct_fn_vg<Real, 64, Rec, 12>(vg);   // <= 85 registers
    case -128: return direct_fn_vg<Real, 128, Rec, 8>(vg);  // <= 64 registers
    default: return nullptr;
    }
}

// Direct variant: knob = threads per block (64, 128 or 256; -64 / -128: the
// same with registers capped at 64 so that more blocks are resident; -96 /
// -80: 64 threads with at most 102 / 85 registers, 10 / 12 blocks per SM;
// -196 / -180 / -172: the FP32 kernel with slotted upwind rows, 64 threads
// with at most 102 / 85 / 73 registers); compact picks the compact record
// format.
// Streaming multiprocessors of the current device (cached per device).
inline int device_sm_count()
{
    static int cache[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 0;
    if (!cache[dev]) {
        int n = 0;
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
        cache[dev] = n;
    }
    return cache[dev];
}

inline int direct_block_threads(int knob)
{
    switch (knob) {
    case -96: case -80: case -196: case -180: case -172: return 64;
    default: return knob < 0 ? -knob : knob;
    }
}

template <typename Real>
cudaError_t launch_direct_level(int knob, const LevelArgs &p, const void *rec, uint64_t begin, uint64_t end,
                                cudaStream_t s, bool compact)
{
    const int bs = direct_block_threads(knob);
    if (end <= begin) return cudaSuccess;
    const uint64_t tasks = (end - begin) * (p.G / p.vg);
    if (tasks >= (1ull << 26)) return cudaErrorInvalidValue;
    // Slotted kernels (10 / 12 / 14 blocks per SM) and -96 (10): the record
    // prefetch half a resident wave ahead in launches at least two waves deep.
    const int pf_blocks = knob == -196 || knob == -96 ? 10 : knob == -180 ? 12 : knob == -172 ? 14 : 0;
    const uint64_t sms = (uint64_t)device_sm_count();
    const bool pf = pf_blocks && sms && tasks >= sms * pf_blocks * bs * 2;
    const void *fn = compact ? direct_fn<Real, CompactRecord<Real>>(knob, (int)p.vg, p.solver, pf)
                             : direct_fn<Real, ItemRecord<Real>>(knob, (int)p.vg, p.solver, pf);
    if (!fn) return cudaErrorInvalidValue;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)((tasks + bs - 1) / bs));
    cfg.blockDim = dim3(bs);
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    const void *r = rec;
    void *args[] = {(void *)&p, (void *)&r, (void *)&begin, (void *)&end};
    return cudaLaunchKernelExC(&cfg, fn, args);
}

// The direct kernel over a list of schedule positions instead of a
// contiguous range: the items of one level that belong to a chunk of angles,
// for the drop-in sweep that overlaps its host copies with the sweep chunk by
// chunk.  Compact records, NoPivot, 64 threads with at most 102 registers;
// the same per-item arithmetic as the level kernels.
template <typename Real, int VG>
__global__ void __launch_bounds__(64, 10)
sweep_direct_subset_kernel(const LevelArgs p, const CompactRecord<Real> *__restrict__ rec,
                           const uint32_t *__restrict__ pos, const uint64_t begin, const uint64_t end)
{
    pdl_launch_dependents();
    const uint32_t gpv = p.G / VG;
    const uint32_t t = blockIdx.x * 64u + threadIdx.x;
    const uint32_t itl = gpv == 1u ? t : __umulhi(t, p.vmagic);
    const uint32_t g = (t - itl * gpv) * VG;
    const uint64_t k = begin + itl;
    bool live = k < end;
    RegRecord<Real> R;
    PairIn<Real, VG> in;
    if (live) {
        load_record(rec + pos[k], R, (uint32_t)kSolveNoPivot);
        live = R.u(0) != kSentinel;
    }
    if (live) pair_load_source<Real, VG>(p, R, g, in);
    pdl_wait_prerequisites();
    if (!live) return;
    pair_load_upwind<Real, VG, false>(p, R, g, in);
    pair_solve_store_any<Real, VG>(p, R, g, in);
}

// Positions pos[begin, end) of compact records `rec` (p.vg 1 or 2).
template <typename Real>
cudaError_t launch_direct_subset(const LevelArgs &p, const void *rec, const uint32_t *pos, uint64_t begin,
                                 uint64_t end, cudaStream_t s)
{
    if (end <= begin) return cudaSuccess;
    if (p.solver != kSolveNoPivot) return cudaErrorInvalidValue;
    const uint64_t tasks = (end - begin) * (p.G / p.vg);
    if (tasks >= (1ull << 26)) return cudaErrorInvalidValue;
    const void *fn = p.vg == 1   ? (const void *)sweep_direct_subset_kernel<Real, 1>
                     : p.vg == 2 ? (const void *)sweep_direct_subset_kernel<Real, 2>
                                 : nullptr;
    if (!fn) return cudaErrorInvalidValue;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)((tasks + 63) / 64));
    cfg.blockDim = dim3(64);
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    void *args[] = {(void *)&p, (void *)&rec, (void *)&pos, (void *)&begin, (void *)&end};
    return cudaLaunchKernelExC(&cfg, fn, args);
}

template <typename Real, typename Rec>
static const void *direct_dataflow_fn(int vg)
{
    switch (vg) {
    case 1: return (const void *)sweep_direct_dataflow_kernel<Real, 1, Rec>;
    case 2: return (const void *)sweep_direct_dataflow_kernel<Real, 2, Rec>;
    case 4:
        if constexpr (sizeof(Real) == 4) return (const void *)sweep_direct_dataflow_kernel<Real, 4, Rec>;
        else return nullptr;
    default: return nullptr;
    }
}

template <typename Real>
cudaError_t direct_dataflow_blocks_per_sm(int vg, bool compact, int *blocks)
{
    const void *fn = compact ? direct_dataflow_fn<Real, CompactRecord<Real>>(vg)
                             : direct_dataflow_fn<Real, ItemRecord<Real>>(vg);
    if (!fn) return cudaErrorInvalidValue;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks, fn, 128, 0);
}

// df.done must hold n_cells * A * (G / vg) flags; G / vg a power of two <= 32.
template <typename Real>
cudaError_t launch_direct_dataflow(const LevelArgs &p, const void *rec, bool compact, const DataflowArgs &df,
                                   unsigned grid, cudaStream_t s)
{
    const uint32_t gpv = p.G / p.vg;
    if (grid == 0 || gpv == 0 || gpv > 32 || (gpv & (gpv - 1)) != 0) return cudaErrorInvalidValue;
    const void *fn = compact ? direct_dataflow_fn<Real, CompactRecord<Real>>((int)p.vg)
                             : direct_dataflow_fn<Real, ItemRecord<Real>>((int)p.vg);
    if (!fn) return cudaErrorInvalidValue;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(128);
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    const void *r = rec;
    void *args[] = {(void *)&p, (void *)&r, (void *)&df};
    return cudaLaunchKernelExC(&cfg, fn, args);
}

template <typename Real>
cudaError_t launch_compact_records(const LevelArgs &p, uint64_t n, void *out, cudaStream_t s)
{
    if (n == 0) return cudaSuccess;
    compact_record_kernel<Real><<<(unsigned)((n + 127) / 128), 128, 0, s>>>(p, n, (CompactRecord<Real> *)out);
    return cudaGetLastError();
}

// knob = items per warp (8, 16 or 32); one launch over items [begin, end).
template <typename Real>
cudaError_t launch_level_record(int ipw, const LevelArgs &p, const void *rec, uint64_t begin, uint64_t end,
                                cudaStream_t s)
{
    if (end <= begin) return cudaSuccess;
    const void *fn = record_fn<Real, LevelK>(ipw, (int)p.vg);
    if (!fn) return cudaErrorInvalidValue;
    const uint64_t warps = (end - begin + ipw - 1) / ipw;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)((warps + 3) / 4));
    cfg.blockDim = dim3(128);
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    const ItemRecord<Real> *r = (const ItemRecord<Real> *)rec;
    void *args[] = {(void *)&p, (void *)&r, (void *)&begin, (void *)&end};
    return cudaLaunchKernelExC(&cfg, fn, args);
}

template <typename Real>
cudaError_t record_dataflow_blocks_per_sm(int ipw, int vg, int *blocks)
{
    const void *fn = record_fn<Real, DataflowK>(ipw, vg);
    if (!fn) return cudaErrorInvalidValue;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks, fn, 128, 0);
}

template <typename Real>
cudaError_t launch_dataflow_record(int ipw, const LevelArgs &p, const void *rec, const DataflowArgs &df,
                                   unsigned grid, cudaStream_t s)
{
    const void *fn = record_fn<Real, DataflowK>(ipw, (int)p.vg);
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
