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

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

}  // namespace tycho
