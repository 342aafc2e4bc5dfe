// Wavefront kernels of the DG SN sweep (sm_100a).
//
// One launch updates every (cell, angle) item of one wavefront level, for all
// energy groups.  Per item the 4x4 streaming+collision matrix depends only on
// (cell, angle) -- the reference rebuilds and re-eliminates it for every group
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
// sub+TPI, ...  so a warp's loads of one upwind vertex row are contiguous.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "launch.hpp"

namespace tycho {

template <typename Real> struct Vec4Of;
template <> struct Vec4Of<double> { using type = double4; };
template <> struct Vec4Of<float> { using type = float4; };



template <typename Real, int TPI>
__global__ void __launch_bounds__(256)
sweep_level_kernel(const LevelArgs p, const uint64_t begin, const uint64_t end)
{
    using R4 = typename Vec4Of<Real>::type;
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t it = begin + t / TPI;
    if (it >= end) return;
    const int sub = (int)(t % TPI);

    const uint32_t A = p.A, G = p.G;
    const uint32_t ca = __ldg(p.items + it);
    const uint32_t c = ca / A;
    const uint32_t a = ca - c * A;
    const R4 ab4 = reinterpret_cast<const R4 *>(p.abar)[it];
    const Real ab[4] = {ab4.x, ab4.y, ab4.z, ab4.w};
    const int4 adj4 = __ldg(p.adj + c);
    const int adj[4] = {adj4.x, adj4.y, adj4.z, adj4.w};
    const uint32_t nmap = __ldg(p.nbrmap + c);
    const Real *ck = reinterpret_cast<const Real *>(p.cellk) + 3 * (size_t)c;
    const Real vs20 = ck[0], d1 = ck[1], d2 = ck[2];

    // Face terms A_f/12 and 2 A_f/12 with A_f = area * omega.n.
    Real t1[4], t2[4];
#pragma unroll
    for (int f = 0; f < 4; ++f) {
        t1[f] = ab[f] / Real(12);
        t2[f] = Real(2) * ab[f] / Real(12);
    }
    // Streaming + collision (volume integrals), then outgoing-face terms in
    // increasing face order.
    Real M[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) M[i][j] = t1[i] + (i == j ? d2 : d1);
#pragma unroll
    for (int f = 0; f < 4; ++f) {
        if (ab[f] > Real(0)) {
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j)
                    if (i != f && j != f) M[i][j] += (i == j ? t2[f] : t1[f]);
        }
    }
    // LU without pivoting: the elimination steps of gaussElim4 NoPivot that
    // touch only the matrix.
    const Real r0 = Real(1) / M[0][0];
    const Real u01 = M[0][1] * r0, u02 = M[0][2] * r0, u03 = M[0][3] * r0;
    const Real l1 = M[1][0], l2 = M[2][0], l3 = M[3][0];
    const Real a11 = M[1][1] - u01 * l1, a12 = M[1][2] - u02 * l1, a13 = M[1][3] - u03 * l1;
    const Real a21 = M[2][1] - u01 * l2, a22 = M[2][2] - u02 * l2, a23 = M[2][3] - u03 * l2;
    const Real a31 = M[3][1] - u01 * l3, a32 = M[3][2] - u02 * l3, a33 = M[3][3] - u03 * l3;
    const Real r1 = Real(1) / a11;
    const Real u12 = a12 * r1, u13 = a13 * r1;
    const Real b22 = a22 - u12 * a21, b23 = a23 - u13 * a21;
    const Real b32 = a32 - u12 * a31, b33 = a33 - u13 * a31;
    const Real r2 = Real(1) / b22;
    const Real u23 = b23 * r2;
    const Real c33 = b33 - u23 * b32;

    const size_t rowG = (size_t)4 * G;
    const Real *__restrict__ psi_in = reinterpret_cast<const Real *>(p.psi);
    Real *__restrict__ psi_out = reinterpret_cast<Real *>(p.psi) + (size_t)ca * rowG;
    const Real *__restrict__ iso = reinterpret_cast<const Real *>(p.iso);
    const Real *iso_c = iso ? iso + (size_t)c * rowG : nullptr;
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
        b[0] = vs20 * (Real(2) * q[0] + q[1] + q[2] + q[3]);
        b[1] = vs20 * (q[0] + Real(2) * q[1] + q[2] + q[3]);
        b[2] = vs20 * (q[0] + q[1] + Real(2) * q[2] + q[3]);
        b[3] = vs20 * (q[0] + q[1] + q[2] + Real(2) * q[3]);
        // Upwind faces, increasing face order; vacuum (0) on the boundary.
#pragma unroll
        for (int f = 0; f < 4; ++f) {
            if (ab[f] < Real(0)) {
                Real pn[4];
                const int nb = adj[f];
                const Real *nrow = psi_in + ((size_t)(nb < 0 ? 0 : nb) * A + a) * rowG + g;
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    if (j == f) { pn[j] = Real(0); continue; }
                    const uint32_t nv = (nmap >> ((f * 4 + j) * 2)) & 3u;
                    pn[j] = nb >= 0 ? nrow[nv * G] : Real(0);
                }
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    if (i == f) continue;
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        if (j == f) continue;
                        b[i] -= (i == j ? t2[f] : t1[f]) * pn[j];
                    }
                }
            }
        }
        // The right-hand-side steps of gaussElim4 NoPivot.
        b[0] = b[0] * r0;
        b[1] = b[1] - b[0] * l1;
        b[2] = b[2] - b[0] * l2;
        b[3] = b[3] - b[0] * l3;
        b[1] = b[1] * r1;
        b[2] = b[2] - b[1] * a21;
        b[3] = b[3] - b[1] * a31;
        b[2] = b[2] * r2;
        b[3] = b[3] - b[2] * b32;
        b[3] = b[3] / c33;
        b[2] = b[2] - u23 * b[3];
        b[1] = b[1] - u13 * b[3] - u12 * b[2];
        b[0] = b[0] - u03 * b[3] - u02 * b[2] - u01 * b[1];
#pragma unroll
        for (int v = 0; v < 4; ++v) psi_out[v * G + g] = b[v];
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

}  // namespace tycho
