// radik_engine_bf16.cu -- bf16 instantiations of the selection engine
// (split per value type so the three compile in parallel).
#include "radik_engine.cuh"

namespace radik {

cudaError_t launch_engine_bf16(const EngineParams& p, int grid, cudaStream_t stream, bool coop) {
  return (p.flags & kFlagWithScale) ? launch_typed<kBF16, true>(p, grid, stream, coop)
                                    : launch_typed<kBF16, false>(p, grid, stream, coop);
}

cudaError_t launch_short_bf16(const EngineParams& p, int grid, cudaStream_t stream) {
  return (p.flags & kFlagWithScale) ? launch_short_typed<kBF16, true>(p, grid, stream)
                                    : launch_short_typed<kBF16, false>(p, grid, stream);
}

cudaError_t occupancy_bf16(uint32_t flags, int* per_sm) {
  return (flags & kFlagWithScale) ? engine_occupancy<kBF16, true>(per_sm) : engine_occupancy<kBF16, false>(per_sm);
}

}  // namespace radik
