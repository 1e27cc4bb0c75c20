// Explicitly rounded arithmetic shared by the gradient / image kernels.
//
// The reference evaluates its correlation expressions with C's usual arithmetic
// conversions: float operands combine in float, and a double literal (0.5, 2.0,
// 0.25) lifts the rest of the expression to double, rounded back to float on
// assignment.  These helpers spell each such operation out with a rounding
// intrinsic so that nvcc cannot contract or reorder it.
#pragma once
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

}  // namespace
}  // namespace rsgpu
