// Dense 8D ENO/Lax-Friedrichs stage, fast variant: the shared stage kernel
// (world8d_stage.cuh) with reciprocal spacings and multiply-add contraction.
#include "world8d_stage.cuh"

namespace pe {

cudaError_t world8_stage_fast(const World8Grid &g, const World8Stage &s,
                              cudaStream_t stream) {
  return w8::launch_stage<true>(g, s, stream);
}

}  // namespace pe
