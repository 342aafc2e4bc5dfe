// Host wrappers of the sweep's streaming kernels and of the deterministic
// vector kernels used by the outer solvers.  All take an explicit stream.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "launch.hpp"

namespace tycho {

// Per item: A_f = area(c,f) * omega.n(a,c,f) in FP64 with the reference's
// operation order; optionally an FP32 copy.
cudaError_t launch_item_abar(const uint32_t *items, uint64_t n, uint32_t A, const double *normal,
                             const double *area, const double *omega /* xi,eta,mu: 3*A */,
                             double4 *abar64, float4 *abar32, cudaStream_t s);

// phi(c,v,g) = sum_a w_a psi(c,a,v,g), angles in increasing order, FP64 sum.
cudaError_t launch_psi_to_phi(const void *psi, bool psi_fp32, const double *w, double *phi,
                              uint64_t nc, uint32_t A, uint32_t G, cudaStream_t s);

// iso = [q_fixed +] S phi_in, FP64; iso32 (nullable) gets an FP32 copy.
// phi_in == nullptr: iso = q_fixed (or 0).  scatter == nullptr: within-group.
cudaError_t launch_scatter_source(const double *phi_in, const double *q_fixed, const double *sigma_s,
                                  const double *scatter, double *iso, float *iso32, uint64_t nc,
                                  uint32_t G, cudaStream_t s);

// epoch = epoch + 1, skipping 0 (the value a fresh completion array holds).
cudaError_t launch_bump_epoch(uint32_t *epoch, cudaStream_t s);

// Deterministic reductions: a fixed grid writes per-block partials that one
// block sums in a fixed order, so results do not depend on scheduling.
constexpr int kReduceBlocks = 592;  // 4 per SM on 148 SMs
constexpr int kDotBlocks = 444;     // inner products on pairs: 3 per SM (74-80 registers)
constexpr int kReduceSlots = 256;   // result / host doubles
struct Reducer {
    double *partials = nullptr;  // kReduceBlocks * 64
    double *result = nullptr;    // kReduceSlots device doubles
    double *host = nullptr;      // kReduceSlots page-locked host doubles
};
// Device buffers from the stream-ordered pool on stream s; the host copy of
// the results is ordinary host memory (each reduction synchronizes s before
// reading it).
cudaError_t reducer_init(Reducer &r, cudaStream_t s);
void reducer_free(Reducer &r, cudaStream_t s);

// result[j] = <w, V_j> for j < k (V_j = V + j*ld), k <= 64; host copy in r.host.
cudaError_t multi_dot(const double *w, const double *V, size_t ld, int k, uint64_t n, Reducer &r,
                      cudaStream_t s);
// result[0] = sum |x - y| (y may be null), result[1] = sum |x|.
cudaError_t l1_pair(const double *x, const double *y, uint64_t n, Reducer &r, cudaStream_t s);
// The same reductions into device memory dst (dst[j], j < k; dst[0..1]),
// without a copy to the host or a synchronization: usable in a captured
// graph (the same partial sums in the same order, so the same results).
cudaError_t multi_dot_dev(const double *w, const double *V, size_t ld, int k, uint64_t n, Reducer &r, double *dst,
                          cudaStream_t s);
cudaError_t l1_pair_dev(const double *x, const double *y, uint64_t n, Reducer &r, double *dst, cudaStream_t s);
// w /= sqrt(*sq) unless it is 0; *norm_out (nullable) = sqrt(*sq).
cudaError_t scale_by_norm(double *w, uint64_t n, const double *sq, double *norm_out, cudaStream_t s);
// w -= sum_j h[j] V_j (h on device), j < k.
cudaError_t multi_axpy(double *w, const double *V, size_t ld, const double *h, int k, uint64_t n,
                       cudaStream_t s);
// y = alpha * x + beta * y
cudaError_t axpby(double alpha, const double *x, double beta, double *y, uint64_t n, cudaStream_t s);
// y = x - y
cudaError_t sub_from(const double *x, double *y, uint64_t n, cudaStream_t s);

}  // namespace tycho
