// FP32 instantiation of the wavefront kernel (mixed-precision sweeps).
// Compiled with FMA contraction on: this path is checked against the FP64
// sweep by tolerance, not bit for bit.
#include "sweep_kernels.cuh"
#include "sweep_tiles.cuh"
#include "sweep_records.cuh"

namespace tycho {

template cudaError_t launch_level<float>(int, const LevelArgs &, uint64_t, uint64_t, cudaStream_t);
template cudaError_t launch_dataflow<float>(int, const LevelArgs &, const DataflowArgs &, unsigned, cudaStream_t);
template cudaError_t dataflow_blocks_per_sm<float>(int, int *);
template cudaError_t launch_level_tile<float>(int, const LevelArgs &, uint64_t, uint64_t, cudaStream_t);
template cudaError_t launch_dataflow_tile<float>(int, const LevelArgs &, const DataflowArgs &, unsigned, cudaStream_t);
template cudaError_t tile_dataflow_blocks_per_sm<float>(int, int *);
template cudaError_t launch_item_records<float>(const LevelArgs &, uint64_t, void *, cudaStream_t);
template cudaError_t launch_level_record<float>(int, const LevelArgs &, const void *, uint64_t, uint64_t, cudaStream_t);
template cudaError_t launch_dataflow_record<float>(int, const LevelArgs &, const void *, const DataflowArgs &, unsigned,
                                               cudaStream_t);
template cudaError_t record_dataflow_blocks_per_sm<float>(int, int, int *);
template cudaError_t launch_persist_record<float>(int, const LevelArgs &, const void *, const uint64_t *, uint32_t,
                                                  unsigned long long *, const DataflowArgs &, unsigned, cudaStream_t);
template cudaError_t record_persist_blocks_per_sm<float>(int, int, int *);
template cudaError_t launch_direct_level<float>(int, const LevelArgs &, const void *, uint64_t, uint64_t, cudaStream_t,
                                                  bool);
template cudaError_t launch_compact_records<float>(const LevelArgs &, uint64_t, void *, cudaStream_t);
template cudaError_t launch_direct_dataflow<float>(const LevelArgs &, const void *, bool, const DataflowArgs &,
                                                     unsigned, cudaStream_t);
template cudaError_t direct_dataflow_blocks_per_sm<float>(int, bool, int *);

}  // namespace tycho
