// Instantiation of the 2D propagator kernels for T=double, EXACT=true.
#include "fd2d_kernels.cuh"

namespace rsgpu {
cudaError_t launch_step_2d_f64(int cfg, int physics, int half, bool adj, const void *args, const void *coefs,
                                 int grid, cudaStream_t st)
{
    return launch_2d_t<double, true>(cfg, physics, half, adj, args, coefs, grid, st);
}
}  // namespace rsgpu
