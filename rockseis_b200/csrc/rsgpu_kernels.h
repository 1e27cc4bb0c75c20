// Launch wrappers exported by the CUDA translation units to the host runtime.
#pragma once
#include <cuda_runtime.h>
#include <cstddef>

namespace rsgpu {

enum { PHYS_A2D = 0, PHYS_E2D = 1, PHYS_A3D = 2, PHYS_E3D = 3 };
enum { PREC_F32_EXACT = 0, PREC_F32_FAST = 1, PREC_F64 = 2 };
// Tile shapes of the 2D kernels: TX x TZ outputs per CTA, RZ rows per thread.
enum { TILECFG_64x32 = 0, TILECFG_64x64 = 1, TILECFG_32x32 = 2, TILECFG_128x32 = 3, TILECFG_32x16 = 4,
       TILECFG_COUNT_2D = 5 };
struct TileShape { int tx, tz; };
inline TileShape tile_shape_2d(int cfg)
{
    switch (cfg) {
    case TILECFG_64x32: return {64, 32};
    case TILECFG_64x64: return {64, 64};
    case TILECFG_32x32: return {32, 32};
    case TILECFG_128x32: return {128, 32};
    default: return {32, 16};
    }
}

// One half-step (half = 0 velocity, 1 stress) of every tile in args.
cudaError_t launch_step_2d(int prec, int cfg, int physics, int half, bool adj, const void *args, const void *coefs,
                           int grid, cudaStream_t st);
// Source injection followed by receiver recording, one CTA per shot.
cudaError_t launch_injrec_2d(int prec, const void *shots, const void *plans, int nshots, double dt, int it_base,
                             const int *it_dev, cudaStream_t st);
cudaError_t launch_advance(int *it_dev, int by, cudaStream_t st);
size_t coefset_bytes(int prec);
int coef_row_stride();

}  // namespace rsgpu
