// Element arithmetic of the streaming passes around the sweep, shared by the
// single-instance kernels (device_ops.cu) and the batched ones (batch_ops.cu)
// so that a batch member computes bit for bit what it computes alone.  Both
// translation units are compiled with -fmad=false.
#pragma once

#include <cstdint>

namespace tycho {

constexpr double kFourPi = 4.0 * 3.14159265358979323846;

// Isotropic total source of phi element i = (c*4 + v)*G + g:
//   [q_i +] sum_g' sigma_s[c] * scat[g][g'] / (4 pi) * phi_(c,v,g')
// (within-group when scat is null: Util.cc:126-128).  phi == nullptr gives
// q_i (or 0).
__device__ __forceinline__ double scatter_elem(const double *__restrict__ phi, const double *__restrict__ q,
                                               const double *__restrict__ sigma_s,
                                               const double *__restrict__ scat, uint64_t i, uint32_t G)
{
    const uint64_t c = i / ((uint64_t)4 * G);
    double s;
    if (phi) {
        if (!scat) {
            s = sigma_s[c] / kFourPi * phi[i];
        } else {
            const uint32_t g = (uint32_t)(i % G);
            const double *pv = phi + (i - g);
            s = 0.0;
            for (uint32_t gp = 0; gp < G; ++gp) {
                const double k = scat[g * G + gp];
                if (k == 0.0) continue;
                s += sigma_s[c] * k / kFourPi * pv[gp];
            }
        }
        if (q) s = q[i] + s;
    } else {
        s = q ? q[i] : 0.0;
    }
    return s;
}

// The four vertex elements (c, v, g), v = 0..3, of the total isotropic
// source, with the arithmetic of scatter_elem term by term (the same
// coefficient sigma_s[c] * k / 4pi, the same summation order over g'), so
// the results are bit-identical; the coefficient is formed once for the four
// vertices instead of once per element.
__device__ __forceinline__ void scatter_cell_group(const double *__restrict__ phi, const double *__restrict__ q,
                                                   const double *__restrict__ sigma_s,
                                                   const double *__restrict__ scat, uint64_t c, uint32_t g,
                                                   uint32_t G, double (&s)[4])
{
    const uint64_t base = c * 4 * G;
    if (phi) {
        if (!scat) {
            const double k = sigma_s[c] / kFourPi;
#pragma unroll
            for (int v = 0; v < 4; ++v) s[v] = k * phi[base + v * G + g];
        } else {
#pragma unroll
            for (int v = 0; v < 4; ++v) s[v] = 0.0;
            for (uint32_t gp = 0; gp < G; ++gp) {
                const double k = scat[g * G + gp];
                if (k == 0.0) continue;
                const double kc = sigma_s[c] * k / kFourPi;
#pragma unroll
                for (int v = 0; v < 4; ++v) s[v] += kc * phi[base + v * G + gp];
            }
        }
        if (q) {
#pragma unroll
            for (int v = 0; v < 4; ++v) s[v] = q[base + v * G + g] + s[v];
        }
    } else {
#pragma unroll
        for (int v = 0; v < 4; ++v) s[v] = q ? q[base + v * G + g] : 0.0;
    }
}

// Scalar flux of phi element i: sum_a w_a psi(c,a,v,g), angles in increasing
// order, FP64 accumulation (Util::psiToPhi, Util.cc:85-97).
template <typename Real>
__device__ __forceinline__ double psi_to_phi_elem(const Real *__restrict__ psi, const double *__restrict__ w,
                                                  uint64_t i, uint32_t A, uint32_t G)
{
    const uint64_t row = (uint64_t)4 * G;
    const uint64_t c = i / row;
    const uint64_t vg = i - c * row;
    const Real *p = psi + c * A * row + vg;
    double s = 0.0;
    for (uint32_t a = 0; a < A; ++a) s += (double)p[(size_t)a * row] * w[a];
    return s;
}

// The same sum with eight angles' loads issued before their products are
// added (in the same order, so the same bits): for grid-stride loops over
// many elements per thread (the batched passes), which would otherwise
// wait one load latency per angle.
template <typename Real>
__device__ __forceinline__ double psi_to_phi_elem8(const Real *__restrict__ psi, const double *__restrict__ w,
                                                   uint64_t i, uint32_t A, uint32_t G)
{
    const uint64_t row = (uint64_t)4 * G;
    const uint64_t c = i / row;
    const uint64_t vg = i - c * row;
    const Real *p = psi + c * A * row + vg;
    double s = 0.0;
    uint32_t a = 0;
    for (; a + 8 <= A; a += 8) {
        Real v[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) v[k] = p[(size_t)(a + k) * row];
#pragma unroll
        for (int k = 0; k < 8; ++k) s += (double)v[k] * w[a + k];
    }
    for (; a < A; ++a) s += (double)p[(size_t)a * row] * w[a];
    return s;
}

// The same for the four elements i .. i+3 (i a multiple of 4: they lie in one
// cell's row and are contiguous in psi for every angle): one 16-byte (FP32)
// or two 16-byte (FP64) loads per angle, eight angles in flight, and for
// each element the same products and sums in the same order as
// psi_to_phi_elem.
template <typename Real>
__device__ __forceinline__ void psi_to_phi_quad(const Real *__restrict__ psi, const double *__restrict__ w,
                                                uint64_t i, uint32_t A, uint32_t G, double (&s)[4])
{
    const uint64_t row = (uint64_t)4 * G;
    const uint64_t c = i / row;
    const Real *p = psi + c * A * row + (i - c * row);
    s[0] = s[1] = s[2] = s[3] = 0.0;
    uint32_t a = 0;
    for (; a + 8 <= A; a += 8) {
        Real v[8][4];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const Real *q = p + (size_t)(a + k) * row;
            if constexpr (sizeof(Real) == 4) {
                const float4 t = *reinterpret_cast<const float4 *>(q);
                v[k][0] = t.x; v[k][1] = t.y; v[k][2] = t.z; v[k][3] = t.w;
            } else {
                const double2 t0 = reinterpret_cast<const double2 *>(q)[0];
                const double2 t1 = reinterpret_cast<const double2 *>(q)[1];
                v[k][0] = t0.x; v[k][1] = t0.y; v[k][2] = t1.x; v[k][3] = t1.y;
            }
        }
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const double wa = w[a + k];
#pragma unroll
            for (int e = 0; e < 4; ++e) s[e] += (double)v[k][e] * wa;
        }
    }
    for (; a < A; ++a) {
        const Real *q = p + (size_t)a * row;
#pragma unroll
        for (int e = 0; e < 4; ++e) s[e] += (double)q[e] * w[a];
    }
}

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

}  // namespace tycho
