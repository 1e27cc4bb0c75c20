// Instantiations and launchers of the fused z-marching 2D step (fd2d_fused.cuh).
#include "fd2d_fused.cuh"

namespace rsgpu {
namespace {

template <typename K>
cudaError_t prepare(K kernel, size_t smem, int *ctas_per_sm)
{
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int b = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kernel, ZM_NT, smem);
    if (e != cudaSuccess) return e;
    *ctas_per_sm = b > 0 ? b : 1;
    return cudaSuccess;
}

int sm_count()
{
    int dev = 0, n = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
        cudaGetLastError();
        return 1;
    }
    return n > 0 ? n : 1;
}

// Resident CTAs per SM requested from the register allocator, per physics: the
// elastic step holds ~80 KB of rings (two CTAs per SM), the acoustic one ~43 KB.
template <typename T, int PHYS> struct ZmMinB { static constexpr int v = sizeof(T) == 8 ? 1 : (PHYS == PHYS_E2D ? 2 : 4); };

template <typename T, int MODE, int PHYS>
int resident()
{
    using G = ZmGeo<T, PHYS, ZM_TX>;
    auto k = zm_step_2d<T, MODE, PHYS, ZM_TX, ZmMinB<T, PHYS>::v>;
    int per_sm = 0;
    if (prepare(k, G::bytes, &per_sm) != cudaSuccess) {
        cudaGetLastError();
        return sm_count();
    }
    return per_sm * sm_count();
}

__global__ void zm_set_run(int *ctl, int it0)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) { ctl[0] = it0; ctl[3] = it0; }
}

template <typename T, int MODE, int PHYS>
cudaError_t step(const void *args, const void *coefs, int *ctl, int cur, int it_base, int use_dev_it, int nitems,
                 cudaStream_t st)
{
    using G = ZmGeo<T, PHYS, ZM_TX>;
    auto k = zm_step_2d<T, MODE, PHYS, ZM_TX, ZmMinB<T, PHYS>::v>;
    static int per_sm = 0;
    static const cudaError_t e = prepare(k, G::bytes, &per_sm);
    if (e != cudaSuccess) return e;
    static const int resident_ctas = per_sm * sm_count();
    const int grid = nitems < resident_ctas ? nitems : resident_ctas;
    k<<<grid, ZM_NT, G::bytes, st>>>(*reinterpret_cast<const Zm2DArgs<T> *>(args), (const CoefSet<T> *)coefs, ctl, cur,
                                     it_base, use_dev_it);
    return cudaGetLastError();
}

template <typename T, int MODE>
cudaError_t record(const void *args, const int *ctl, int cur, int step_, cudaStream_t st)
{
    const Zm2DArgs<T> &a = *reinterpret_cast<const Zm2DArgs<T> *>(args);
    if (a.nrecs == 0) return cudaSuccess;
    const int grid = (a.nrecs + 255) / 256;
    zm_record_2d<T, MODE><<<grid, 256, 0, st>>>(a, ctl, cur, step_);
    return cudaGetLastError();
}

}  // namespace

int zm_strip_width() { return ZM_TX; }

cudaError_t launch_zm_set_run(int *ctl, int it0, cudaStream_t st)
{
    zm_set_run<<<1, 32, 0, st>>>(ctl, it0);
    return cudaGetLastError();
}

int zm_resident_ctas(int prec, int physics)
{
    if (physics == PHYS_E2D) {
        if (prec == PREC_F64) return resident<double, MODE_IEEE, PHYS_E2D>();
        if (prec == PREC_F32_EXACT) return resident<float, MODE_IEEE, PHYS_E2D>();
        return resident<float, MODE_FAST, PHYS_E2D>();
    }
    if (prec == PREC_F64) return resident<double, MODE_IEEE, PHYS_A2D>();
    if (prec == PREC_F32_EXACT) return resident<float, MODE_IEEE, PHYS_A2D>();
    return resident<float, MODE_FAST, PHYS_A2D>();
}

size_t zm_args_bytes(int prec) { return prec == PREC_F64 ? sizeof(Zm2DArgs<double>) : sizeof(Zm2DArgs<float>); }

cudaError_t launch_zm_step_2d(int prec, int physics, const void *args, const void *coefs, int *ctl, int cur,
                              int it_base, int use_dev_it, int nitems, cudaStream_t st)
{
    if (physics == PHYS_E2D) {
        if (prec == PREC_F64) return step<double, MODE_IEEE, PHYS_E2D>(args, coefs, ctl, cur, it_base, use_dev_it, nitems, st);
        if (prec == PREC_F32_EXACT) return step<float, MODE_IEEE, PHYS_E2D>(args, coefs, ctl, cur, it_base, use_dev_it, nitems, st);
        return step<float, MODE_FAST, PHYS_E2D>(args, coefs, ctl, cur, it_base, use_dev_it, nitems, st);
    }
    if (physics == PHYS_A2D) {
        if (prec == PREC_F64) return step<double, MODE_IEEE, PHYS_A2D>(args, coefs, ctl, cur, it_base, use_dev_it, nitems, st);
        if (prec == PREC_F32_EXACT) return step<float, MODE_IEEE, PHYS_A2D>(args, coefs, ctl, cur, it_base, use_dev_it, nitems, st);
        return step<float, MODE_FAST, PHYS_A2D>(args, coefs, ctl, cur, it_base, use_dev_it, nitems, st);
    }
    return cudaErrorInvalidValue;
}

cudaError_t launch_zm_record_2d(int prec, const void *args, const int *ctl, int cur, int step_, cudaStream_t st)
{
    if (prec == PREC_F64) return record<double, MODE_IEEE>(args, ctl, cur, step_, st);
    if (prec == PREC_F32_EXACT) return record<float, MODE_IEEE>(args, ctl, cur, step_, st);
    return record<float, MODE_FAST>(args, ctl, cur, step_, st);
}

}  // namespace rsgpu
