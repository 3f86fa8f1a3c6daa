// radik_engine_f32.cu -- f32 instantiations of the selection engine
// (split per value type so the three compile in parallel).
#include "radik_engine.cuh"

namespace radik {

cudaError_t launch_engine_f32(const EngineParams& p, int grid, cudaStream_t stream, bool coop) {
  return (p.flags & kFlagWithScale) ? launch_typed<kF32, true>(p, grid, stream, coop)
                                    : launch_typed<kF32, false>(p, grid, stream, coop);
}

cudaError_t launch_short_f32(const EngineParams& p, int grid, cudaStream_t stream) {
  return (p.flags & kFlagWithScale) ? launch_short_typed<kF32, true>(p, grid, stream)
                                    : launch_short_typed<kF32, false>(p, grid, stream);
}

cudaError_t occupancy_f32(uint32_t flags, int* per_sm) {
  return (flags & kFlagWithScale) ? engine_occupancy<kF32, true>(per_sm) : engine_occupancy<kF32, false>(per_sm);
}

}  // namespace radik
