// Dispatch of the 2D half-step kernels by precision, and the small per-step
// kernels (source injection / receiver recording, step counter).
#include "fd2d_kernels.cuh"

namespace rsgpu {

static_assert(NMAP2D == NMAP, "tensor-map slots per shot");

cudaError_t launch_step_2d(int prec, int cfg, int physics, int half, int flags, const void *args, const void *coefs,
                           const void *maps, int *err, int grid, cudaStream_t st)
{
    const char *v = prec == PREC_F32_EXACT ? "f32x" : prec == PREC_F32_FAST ? "f32f" : "f64";
    Launch2DFn fn = launch_2d_table(v, cfg);
    if (!fn) return cudaErrorInvalidValue;
    return fn(physics, half, flags, args, coefs, maps, err, grid, st);
}

cudaError_t launch_injrec_2d(int prec, const void *shots, const void *plans, int nshots, double dt, int it_base,
                             const int *it_dev, cudaStream_t st)
{
    if (prec == PREC_F64)
        inject_record_2d<double, MODE_IEEE><<<nshots, 256, 0, st>>>((const Shot2D<double> *)shots,
                                                                    (const InjRec<double> *)plans, dt, it_base, it_dev);
    else if (prec == PREC_F32_EXACT)
        inject_record_2d<float, MODE_IEEE><<<nshots, 256, 0, st>>>((const Shot2D<float> *)shots,
                                                                   (const InjRec<float> *)plans, (float)dt, it_base, it_dev);
    else
        inject_record_2d<float, MODE_FAST><<<nshots, 256, 0, st>>>((const Shot2D<float> *)shots,
                                                                   (const InjRec<float> *)plans, (float)dt, it_base, it_dev);
    return cudaGetLastError();
}

cudaError_t launch_advance(int *it_dev, int by, cudaStream_t st)
{
    advance_counter<<<1, 32, 0, st>>>(it_dev, by);
    return cudaGetLastError();
}

cudaError_t launch_set_counter(int *it_dev, int value, cudaStream_t st)
{
    set_counter<<<1, 32, 0, st>>>(it_dev, value);
    return cudaGetLastError();
}

// Failure-detection self test: one CTA waits on a shared-memory barrier that
// expects one arrival that never comes.  The bounded wait gives up after its
// wall-clock limit, records RSGPU_ERR_TIMEOUT in the error word and the kernel
// returns normally, leaving the context usable.
static __global__ void wait_for_nothing(int *err)
{
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) mbar_init(&bar, 1);
    __syncthreads();
    mbar_wait_bounded(&bar, 0, err);
}

cudaError_t launch_wait_for_nothing(int *err, cudaStream_t st)
{
    wait_for_nothing<<<1, 32, 0, st>>>(err);
    return cudaGetLastError();
}

size_t coefset_bytes(int prec) { return prec == PREC_F64 ? sizeof(CoefSet<double>) : sizeof(CoefSet<float>); }
int coef_row_stride() { return CROW; }

}  // namespace rsgpu
