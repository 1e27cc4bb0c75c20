// Trace resampling in time (Interp<T>::interp, lib/interp.cpp:38-186): every
// output sample of every trace is one thread.  The index arithmetic and the
// LINEAR / BSPLINE weights follow the reference's mixed float/double C++
// expressions operation by operation (explicitly rounded), so those modes are
// bit-identical to the reference; SINC evaluates sin in double and rounds to the
// element type like the reference, whose libm sin may differ from CUDA's in the
// last bit of the double, which the rounding to float almost always hides.
#include <cstdint>
#include <vector>
#include <cuda_runtime.h>
#include "rsgpu.h"
#include "rsgpu_host.h"

namespace rsgpu {
namespace {

constexpr double kPi = 3.14159265358979323846;

template <typename T> struct R;
template <> struct R<float> {
    static __device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
    static __device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
    static __device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
    static __device__ __forceinline__ float div(float a, float b) { return __fdiv_rn(a, b); }
    static __device__ __forceinline__ float of(double a) { return __double2float_rn(a); }
    static __device__ __forceinline__ float of_long(long v) { return __ll2float_rn(v); }
};
template <> struct R<double> {
    static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
    static __device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
    static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
    static __device__ __forceinline__ double div(double a, double b) { return __ddiv_rn(a, b); }
    static __device__ __forceinline__ double of(double a) { return a; }
    static __device__ __forceinline__ double of_long(long v) { return __ll2double_rn(v); }
};

// (1.0-d)*m0 + d*m1: the first product in double, the second in T (lib/interp.cpp:67-74)
template <typename T>
__device__ T lin(const T *m, T d)
{
    const double a = __dmul_rn(__dsub_rn(1.0, (double)d), (double)m[0]);
    return R<T>::of(__dadd_rn(a, (double)R<T>::mul(d, m[1])));
}

// cubic B-spline weights in double, stored in T, then the T-typed weighted sum
// (lib/interp.cpp:76-93)
template <typename T>
__device__ T bspline(const T *m, T d)
{
    const T xp = R<T>::of(__dadd_rn((double)d, 1.0));
    const T om = R<T>::of(__dsub_rn(1.0, (double)d));
    const double xp_ = xp, om_ = om, d_ = d;
    double t = __dadd_rn(__dmul_rn(-(1.0 / 6.0), xp_), 1.0);
    t = __dsub_rn(__dmul_rn(t, xp_), 2.0);
    const T a0 = R<T>::of(__dadd_rn(__dmul_rn(t, xp_), 4.0 / 3.0));
    const T a1 = R<T>::of(__dadd_rn(__dmul_rn(__dmul_rn(__dsub_rn(__dmul_rn(0.5, d_), 1.0), d_), d_), 2.0 / 3.0));
    const T a2 = R<T>::of(__dadd_rn(__dmul_rn(__dmul_rn(__dsub_rn(__dmul_rn(0.5, om_), 1.0), om_), om_), 2.0 / 3.0));
    const T a3 = R<T>::of(__dsub_rn(__dsub_rn(__dsub_rn(1.0, (double)a0), (double)a1), (double)a2));
    T s = R<T>::add(R<T>::mul(a0, m[0]), R<T>::mul(a1, m[1]));
    s = R<T>::add(s, R<T>::mul(a2, m[2]));
    return R<T>::add(s, R<T>::mul(a3, m[3]));
}

// sin(pi x)/(pi x) of a T argument, 1 at 0 (lib/interp.cpp:99-106)
template <typename T>
__device__ T sinc(T x)
{
    if (x == T(0)) return T(1);
    const double px = __dmul_rn(kPi, (double)x);
    return R<T>::of(__ddiv_rn(sin(px), px));
}

// six-tap windowed sinc (lib/interp.cpp:109-119)
template <typename T>
__device__ T sinc6(const T *m, T d)
{
    T acc = T(0);
    for (int i = 0; i < 6; i++) {
        const double u = __dadd_rn(2.0 - i, (double)d);
        const T w1 = sinc(R<T>::of(u)), w2 = sinc(R<T>::of(__ddiv_rn(u, 3.0)));
        acc = R<T>::add(acc, R<T>::mul(R<T>::mul(m[i], w1), w2));
    }
    return acc;
}

template <typename T>
__global__ void __launch_bounds__(256) interp_traces(int mode, int pad, int ntr, long n1, T o1, T d1, const T *in,
                                                     long n2, T o2, T d2, T *out)
{
    const long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= (long)ntr * n2) return;
    const long tr = k / n2, j = k % n2;
    const T val = R<T>::add(o2, R<T>::mul(R<T>::of_long(j), d2));
    const T q = R<T>::div(R<T>::sub(val, o1), d1);
    const long i0 = (long)q - (pad - 1);          // truncation toward zero, as the C++ cast
    T r = T(0);
    if (i0 >= 0 && i0 + 2 * pad - 1 <= n1 - 1) {
        const T x0 = R<T>::add(o1, R<T>::mul(R<T>::of_long(i0 + (pad - 1)), d1));
        const T d = R<T>::div(R<T>::sub(val, x0), d1);
        const T *m = in + tr * n1 + i0;
        r = mode == RSGPU_INTERP_LINEAR ? lin(m, d) : mode == RSGPU_INTERP_BSPLINE ? bspline(m, d) : sinc6(m, d);
    }
    out[k] = r;
}

template <typename T>
rsgpu_status run(int mode, int ntr, int n1, double o1, double d1, const void *in, int n2, double o2, double d2,
                 void *out)
{
    const int pad = mode == RSGPU_INTERP_LINEAR ? 1 : mode == RSGPU_INTERP_BSPLINE ? 2 : 3;
    const size_t bin = sizeof(T) * (size_t)ntr * n1, bout = sizeof(T) * (size_t)ntr * n2;
    T *din = nullptr, *dout = nullptr;
    cudaStream_t st = nullptr;
    cudaError_t e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMallocAsync((void **)&din, bin, st);
    if (e == cudaSuccess) e = cudaMallocAsync((void **)&dout, bout, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(din, in, bin, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        const long n = (long)ntr * n2;
        interp_traces<T><<<(unsigned)((n + 255) / 256), 256, 0, st>>>(mode, pad, ntr, n1, (T)o1, (T)d1, din, n2,
                                                                        (T)o2, (T)d2, dout);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, dout, bout, cudaMemcpyDeviceToHost, st);
    if (din) cudaFreeAsync(din, st);
    if (dout) cudaFreeAsync(dout, st);
    const cudaError_t es = st ? cudaStreamSynchronize(st) : cudaSuccess;
    if (st) cudaStreamDestroy(st);
    if (e == cudaSuccess) e = es;
    if (e == cudaErrorMemoryAllocation) { set_error("interp: out of device memory"); return RSGPU_ERR_NOMEM; }
    if (e != cudaSuccess) { set_error("interp: %s", cudaGetErrorString(e)); return RSGPU_ERR_CUDA; }
    return RSGPU_OK;
}

}  // namespace
}  // namespace rsgpu

extern "C" rsgpu_status rsgpu_interp_traces(int precision, int mode, int ntr, int n1, double o1, double d1,
                                            const void *in, int n2, double o2, double d2, void *out)
{
    using namespace rsgpu;
    if (mode < RSGPU_INTERP_LINEAR || mode > RSGPU_INTERP_SINC) { set_error("bad interpolation mode %d", mode); return RSGPU_ERR_ARG; }
    if (precision < RSGPU_F32_EXACT || precision > RSGPU_F64) { set_error("bad precision %d", precision); return RSGPU_ERR_ARG; }
    if (ntr < 0 || n1 < 0 || n2 < 0 || !(d1 > 0) || !(d2 > 0)) { set_error("bad trace sizes or sampling"); return RSGPU_ERR_ARG; }
    if ((long)ntr * n2 == 0) return RSGPU_OK;
    if (!in || !out) { set_error("null trace array"); return RSGPU_ERR_ARG; }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) {
        cudaGetLastError();
        set_error("no CUDA device");
        return RSGPU_ERR_NODEVICE;
    }
    return precision == RSGPU_F64 ? run<double>(mode, ntr, n1, o1, d1, in, n2, o2, d2, out)
                                  : run<float>(mode, ntr, n1, o1, d1, in, n2, o2, d2, out);
}
