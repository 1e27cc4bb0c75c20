// Instantiation of the 2D propagator kernels for T=float, EXACT=false.
#include "fd2d_kernels.cuh"

namespace rsgpu {
cudaError_t launch_step_2d_f32f(int cfg, int physics, int half, bool adj, const void *args, const void *coefs,
                                 int grid, cudaStream_t st)
{
    return launch_2d_t<float, false>(cfg, physics, half, adj, args, coefs, grid, st);
}
}  // namespace rsgpu
