// Batched relative 5D solves with the exact cell update (double local
// arithmetic in the reference executable's order, relative5d_exact.cuh):
// every solve of a batch reproduces the reference executable bit for bit.
// This file is compiled with -fmad=false.
#include "relative5d_batch_impl.cuh"
#include "relative5d_exact.cuh"

namespace pe {
namespace {

struct ExactCell {
  template <int BLEND>
  __device__ static void update(const Rel5Grid &g, const Rel5Stage &s, int ix, int iy, int ip,
                                int iv, int ie, int64_t j, double &ca, double &cu, bool &bad) {
    exact::cell_update<2, BLEND>(g, s, ix, iy, ip, iv, ie, j, ca, cu, bad);
  }
};

}  // namespace

int rel5_batch_grid_exact() { return batch_impl::grid_size<ExactCell>(); }

cudaError_t rel5_batch_run_exact(const Rel5BatchArgs &args, int grid, cudaStream_t stream) {
  return batch_impl::launch<ExactCell>(args, grid, stream);
}

}  // namespace pe
