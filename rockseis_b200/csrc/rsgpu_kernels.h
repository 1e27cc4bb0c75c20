// Launch wrappers exported by the CUDA translation units to the host runtime.
#pragma once
#include <cuda_runtime.h>
#include <cstddef>

namespace rsgpu {

enum { PHYS_A2D = 0, PHYS_E2D = 1, PHYS_A3D = 2, PHYS_E3D = 3 };
enum { PREC_F32_EXACT = 0, PREC_F32_FAST = 1, PREC_F64 = 2 };
// Tile shapes of the 2D kernels: TX x TZ outputs per CTA, RZ rows per thread,
// MINB resident CTAs per SM requested from the register allocator.  The table
// (tile_shape_2d and the kernel instantiations) is generated by build.py.
struct TileShape { int tx, tz, rz, minb; };
TileShape tile_shape_2d(int cfg);
int tile_count_2d();
enum { TILECFG_64x32 = 0, TILECFG_32x16 = 3, TILECFG_DEFAULT = 6, TILECFG_E2D = 9 };

// One half-step (half = 0 velocity, 1 stress) of every tile in args.
// maps: per shot NMAP2D CUtensorMaps of the halo-loaded fields; err: device error word.
// flags: LAUNCH_ADJ (adjoint kernels), LAUNCH_INL (acoustic: the kernels whose
// reduced-order edge stencils are inlined; faster when the batch's tiles fit about
// one wave, slower for large batches; the elastic kernels always inline them)
enum { LAUNCH_ADJ = 1, LAUNCH_INL = 2 };
cudaError_t launch_step_2d(int prec, int cfg, int physics, int half, int flags, const void *args, const void *coefs,
                           const void *maps, int *err, int grid, cudaStream_t st);
constexpr int NMAP2D = 5;
// Kernel instantiation table (generated at build time): variant "f32x" (exact),
// "f32f" (fast), "f64"; nullptr if the tile config is not built for the variant.
using Launch2DFn = cudaError_t (*)(int physics, int half, int flags, const void *args, const void *coefs,
                                   const void *maps, int *err, int grid, cudaStream_t st);
Launch2DFn launch_2d_table(const char *variant, int cfg);
// Source injection followed by receiver recording, one CTA per shot.
cudaError_t launch_injrec_2d(int prec, const void *shots, const void *plans, int nshots, double dt, int it_base,
                             const int *it_dev, cudaStream_t st);
cudaError_t launch_advance(int *it_dev, int by, cudaStream_t st);
cudaError_t launch_set_counter(int *it_dev, int value, cudaStream_t st);
cudaError_t launch_wait_for_nothing(int *err, cudaStream_t st);
// Fused z-marching 2D step (fd2d_fused.cuh): velocity, stress and injection of one
// time step plus the recording of the previous one, in one launch over all shots.
// args: Zm2DArgs<T>; ctl: device control words (step counter, error word, gate,
// first step of the run, two work counters); cur: the wavefield copy read.
int zm_strip_width();
size_t zm_args_bytes(int prec);
cudaError_t launch_zm_step_2d(int prec, int physics, const void *args, const void *coefs, int *ctl, int cur,
                              int it_base, int use_dev_it, int nitems, cudaStream_t st);
cudaError_t launch_zm_record_2d(int prec, const void *args, const int *ctl, int cur, int step, cudaStream_t st);
// ctl[0] = ctl[3] = it0: the step counter of graph replays and the first step of a run
cudaError_t launch_zm_set_run(int *ctl, int it0, cudaStream_t st);
// CTAs of the fused step resident on the current device at once
int zm_resident_ctas(int prec, int physics);
size_t coefset_bytes(int prec);
int coef_row_stride();
// Column-marching elastic 2D half-steps (fd2d_march.cu): FAST arithmetic, forward
// propagation; half 0 = velocity, 1 = stress; args: March2DArgs.
struct March2DArgs;
cudaError_t launch_march_2d(int half, const March2DArgs &args, int nitems, cudaStream_t st);
int march_resident_ctas();   // CTAs of the slower half-step resident per SM (0 = query failed)
int march_smem_bytes();

}  // namespace rsgpu
