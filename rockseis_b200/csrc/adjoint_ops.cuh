// Explicitly rounded arithmetic shared by the gradient / image kernels.
//
// The reference evaluates its correlation expressions with C's usual arithmetic
// conversions: float operands combine in float, and a double literal (0.5, 2.0,
// 0.25) lifts the rest of the expression to double, rounded back to float on
// assignment.  These helpers spell each such operation out with a rounding
// intrinsic so that nvcc cannot contract or reorder it.
#pragma once
#include <cstring>
#include <cuda_runtime.h>

namespace rsgpu {
namespace {

template <typename T> struct X;   // explicitly rounded operations of the element type
template <> struct X<float> {
    static __device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
    static __device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
    static __device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
    static __device__ __forceinline__ float div(float a, float b) { return __fdiv_rn(a, b); }
    static __device__ __forceinline__ float rnd(double a) { return __double2float_rn(a); }
};
template <> struct X<double> {
    static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
    static __device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
    static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
    static __device__ __forceinline__ double div(double a, double b) { return __ddiv_rn(a, b); }
    static __device__ __forceinline__ double rnd(double a) { return a; }
};

// 0.5 * w * r * dd / h  in double, rounded to T (the reference's mixed-type expression)
template <typename T>
__device__ __forceinline__ double half_term(T w, T r, T dd, double h)
{
    return __ddiv_rn(__dmul_rn(__dmul_rn(__dmul_rn(0.5, (double)w), (double)r), (double)dd), h);
}

// ---------------------------------------------------------------- order statistics of |r|
// The reference's residual clips sort the magnitudes of a shot's residuals and take
// the element at a given index; the magnitude bit patterns order like the
// non-negative values, so a radix select on them finds the same element.
template <typename T> struct Bits;
template <> struct Bits<float> { using U = unsigned int; static constexpr int NB = 32; };
template <> struct Bits<double> { using U = unsigned long long; static constexpr int NB = 64; };

template <typename T> __device__ __forceinline__ T sqrt_rn(T x);
template <> __device__ __forceinline__ float sqrt_rn<float>(float x) { return __fsqrt_rn(x); }
template <> __device__ __forceinline__ double sqrt_rn<double>(double x) { return __dsqrt_rn(x); }

template <typename T>
__device__ __forceinline__ typename Bits<T>::U mag_bits(T x)
{
    using U = typename Bits<T>::U;
    U u;
    memcpy(&u, &x, sizeof u);
    return u & ~((U)1 << (Bits<T>::NB - 1));
}

// Magnitude bit pattern of the k-th smallest |r[i]|, i < n (k < n), found by the
// whole CTA with four (float) or eight (double) 8-bit histogram passes.
template <typename T>
__device__ typename Bits<T>::U kth_mag_bits(const T *r, long n, long k)
{
    using U = typename Bits<T>::U;
    __shared__ unsigned int hist[256];
    __shared__ U prefix_s;
    __shared__ long rank_s;
    __syncthreads();
    if (threadIdx.x == 0) { prefix_s = 0; rank_s = k; }
    U mask = 0;
    for (int shift = Bits<T>::NB - 8; shift >= 0; shift -= 8) {
        for (int b = threadIdx.x; b < 256; b += blockDim.x) hist[b] = 0;
        __syncthreads();
        const U prefix = prefix_s;
        for (long i = threadIdx.x; i < n; i += blockDim.x) {
            const U u = mag_bits(r[i]);
            if ((u & mask) == prefix) atomicAdd(&hist[(unsigned)(u >> shift) & 255u], 1u);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            long rr = rank_s;
            int b = 0;
            while (b < 255 && rr >= (long)hist[b]) { rr -= hist[b]; b++; }
            rank_s = rr;
            prefix_s = prefix | ((U)b << shift);
        }
        mask |= (U)255 << shift;
        __syncthreads();
    }
    const U out = prefix_s;
    __syncthreads();
    return out;
}

template <typename T>
__device__ __forceinline__ T from_bits(typename Bits<T>::U u)
{
    T x;
    memcpy(&x, &u, sizeof x);
    return x;
}

}  // namespace
}  // namespace rsgpu
