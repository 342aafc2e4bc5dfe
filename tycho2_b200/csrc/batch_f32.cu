// FP32 level kernel of the batched sweep (FMA contraction on: checked by
// tolerance, like sweep_f32.cu).
#include "batch_kernels.cuh"

namespace tycho {

cudaError_t batch_level_launch(const void *fn, const BatchSlot *slots, const BatchPlan &pl, uint32_t level,
                               const BatchCuts &cut, cudaStream_t s);

template <>
cudaError_t launch_batch_level<float>(int ipw, const BatchSlot *slots, const BatchPlan &pl, uint32_t level,
                                      const BatchCuts &cut, bool any_solver, cudaStream_t s)
{
    const void *fn = ipw == 0    ? (any_solver ? (const void *)batch_direct_level_kernel<float, true>
                                               : (const void *)batch_direct_level_kernel<float, false>)
                     : ipw == 8  ? (const void *)batch_level_kernel<float, 8>
                     : ipw == 16 ? (const void *)batch_level_kernel<float, 16>
                     : ipw == 32 ? (const void *)batch_level_kernel<float, 32>
                                 : nullptr;
    if (!fn) return cudaErrorInvalidValue;
    return batch_level_launch(fn, slots, pl, level, cut, s);
}

template <>
cudaError_t launch_batch_persist<float>(const BatchSlot *slots, const BatchPlan &pl, const BatchPersistArgs &a,
                                        bool any_solver, cudaStream_t s)
{
    return any_solver ? batch_persist_launch<float, true, 1>(slots, pl, a, s)
                      : batch_persist_launch<float, false, 4>(slots, pl, a, s);
}

}  // namespace tycho
