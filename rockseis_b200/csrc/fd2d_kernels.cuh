// 2D staggered-grid finite-difference propagators for sm_100a (kernel templates).
//
// One kernel per half-step (velocity, stress), each covering every shot of a
// batch in one launch: the grid walks a table of (shot, tile) work items, so
// shots with different aperture windows share a launch.  Each CTA stages the
// stencil inputs of its TX x TZ tile plus an 8-cell halo in shared memory with
// TMA (cp.async.bulk.tensor, completion on an mbarrier), while its threads fetch
// the point-wise inputs (velocities, moduli) straight into registers.  Every
// thread then produces a 4(x) x RZ(z) block with the C-PML memory-variable
// update and correction fused into the same pass:
//   - x-derivatives: one 128-bit shared load per 4 taps, scalar arithmetic;
//   - z-derivatives: column pairs, 64-bit shared loads, paired f32x2 arithmetic
//     (FADD2/FMUL2/FFMA2), each lane rounded exactly like a scalar op;
//   - interior tiles keep the 8 coefficients in registers; tiles within `order`
//     cells of an array end use per-point coefficient rows (reduced order).
//
// Arithmetic follows the reference operation by operation (Der::ddx_fw etc. in
// lib/der.cpp:155-540, WavesAcoustic2D/WavesElastic2D::forwardstep* in
// lib/waves.cpp:217-404, 1416-1735, backwardstep* in lib/waves.cpp:1738-2080):
//   MODE_IEEE : every add/sub/mul is a separately rounded IEEE op in the
//               reference's order and the final division is __fdiv_rn;
//   MODE_RCP  : as MODE_IEEE, but x/d is computed as q=x*r, e=fma(-q,d,x),
//               q+=e*r (Markstein's correction with r = RN(1/d)); the host only
//               selects it after checking on the device, for all 2^32 float x,
//               that it returns exactly what IEEE division returns for this d;
//   MODE_FAST : FMA contraction, coefficients pre-divided by the spacing.
#pragma once
#include <cuda.h>
#include <cstdint>
#include <type_traits>
#include "rsgpu.h"
#include "rsgpu_internal.h"
#include "rsgpu_kernels.h"

namespace rsgpu {

enum { MODE_IEEE = 0, MODE_RCP = 1, MODE_FAST = 2 };

// ------------------------------------------------------------------ scalar arithmetic
template <typename T, int MODE> struct Ar;
template <int MODE> struct Ar<float, MODE> {
    static constexpr bool exact = MODE != MODE_FAST;
    static __device__ __forceinline__ float add(float a, float b) { return exact ? __fadd_rn(a, b) : a + b; }
    static __device__ __forceinline__ float sub(float a, float b) { return exact ? __fsub_rn(a, b) : a - b; }
    static __device__ __forceinline__ float mul(float a, float b) { return exact ? __fmul_rn(a, b) : a * b; }
    // a + b*c (product rounded separately in the exact modes)
    static __device__ __forceinline__ float mad(float a, float b, float c)
    {
        return exact ? __fadd_rn(a, __fmul_rn(b, c)) : fmaf(b, c, a);
    }
    // a - b*c
    static __device__ __forceinline__ float msub(float a, float b, float c)
    {
        return exact ? __fsub_rn(a, __fmul_rn(b, c)) : fmaf(-b, c, a);
    }
    static __device__ __forceinline__ float div(float a, float d, float r)
    {
        if (MODE == MODE_IEEE) return __fdiv_rn(a, d);
        const float q = __fmul_rn(a, r);
        const float e = fmaf(-q, d, a);
        return fmaf(e, r, q);
    }
};
template <int MODE> struct Ar<double, MODE> {
    static constexpr bool exact = true;
    static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
    static __device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
    static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
    static __device__ __forceinline__ double mad(double a, double b, double c) { return __dadd_rn(a, __dmul_rn(b, c)); }
    static __device__ __forceinline__ double msub(double a, double b, double c) { return __dsub_rn(a, __dmul_rn(b, c)); }
    static __device__ __forceinline__ double div(double a, double d, double) { return __ddiv_rn(a, d); }
};

// ------------------------------------------------------------------ paired arithmetic (x-neighbour columns)
template <typename T> struct Pair;
template <> struct Pair<float> { using t = float2; };
template <> struct Pair<double> { using t = double2; };

template <typename T, int MODE> struct Ar2;
// Fast mode uses the paired FADD2/FMUL2/FFMA2 instructions; the exact modes
// evaluate the two lanes with separately rounded scalar operations.
template <int MODE> struct Ar2<float, MODE> {
    using P = float2;
    static constexpr bool exact = MODE != MODE_FAST;
    static __device__ __forceinline__ P mk(float a) { return make_float2(a, a); }
    static __device__ __forceinline__ P add(P a, P b)
    {
        return exact ? make_float2(__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y)) : __fadd2_rn(a, b);
    }
    static __device__ __forceinline__ P sub(P a, P b)
    {
        return exact ? make_float2(__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y)) : __fadd2_rn(a, make_float2(-b.x, -b.y));
    }
    static __device__ __forceinline__ P mul(P a, P b)
    {
        return exact ? make_float2(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)) : __fmul2_rn(a, b);
    }
    static __device__ __forceinline__ P acc(P s, P d, P c)
    {
        return exact ? make_float2(__fadd_rn(s.x, __fmul_rn(d.x, c.x)), __fadd_rn(s.y, __fmul_rn(d.y, c.y)))
                     : __ffma2_rn(d, c, s);
    }
    static __device__ __forceinline__ P div(P a, P d, P r)
    {
        return make_float2(Ar<float, MODE>::div(a.x, d.x, r.x), Ar<float, MODE>::div(a.y, d.y, r.y));
    }
};
template <int MODE> struct Ar2<double, MODE> {
    using P = double2;
    static constexpr bool exact = true;
    static __device__ __forceinline__ P mk(double a) { return make_double2(a, a); }
    static __device__ __forceinline__ P add(P a, P b) { return make_double2(__dadd_rn(a.x, b.x), __dadd_rn(a.y, b.y)); }
    static __device__ __forceinline__ P sub(P a, P b) { return make_double2(__dsub_rn(a.x, b.x), __dsub_rn(a.y, b.y)); }
    static __device__ __forceinline__ P mul(P a, P b) { return make_double2(__dmul_rn(a.x, b.x), __dmul_rn(a.y, b.y)); }
    static __device__ __forceinline__ P acc(P s, P d, P c) { return add(s, mul(d, c)); }
    static __device__ __forceinline__ P div(P a, P d, P) { return make_double2(__ddiv_rn(a.x, d.x), __ddiv_rn(a.y, d.y)); }
};

template <typename T> struct Vec4;
template <> struct Vec4<float> { using type = float4; };
template <> struct Vec4<double> { using type = double4; };

template <typename T>
__device__ __forceinline__ void ld4(const T *p, T (&v)[4])
{
    typename Vec4<T>::type q = *reinterpret_cast<const typename Vec4<T>::type *>(p);
    v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
}
__device__ __forceinline__ void ldg4(const float *p, float (&v)[4])
{
    const float4 q = __ldg(reinterpret_cast<const float4 *>(p));
    v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
}
__device__ __forceinline__ void ldg4(const double *p, double (&v)[4])
{
    const double2 a = __ldg(reinterpret_cast<const double2 *>(p)), b = __ldg(reinterpret_cast<const double2 *>(p) + 1);
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}

// Number of coefficient pairs the reference uses at index i of an axis of
// length n (last writer wins in lib/der.cpp's three loops).
__device__ __forceinline__ int kfw(int i, int n, int order)
{
    if (i >= n - 1) return 0;
    if (i >= n - order - 1) return n - 1 - i;
    if (i >= order - 1) return order;
    return i + 1;
}
__device__ __forceinline__ int kbw(int i, int n, int order)
{
    if (i >= n) return 0;   // padding lanes beyond the array (never stored)
    if (i >= n - order) return n - i;
    if (i >= order) return order;
    return i;   // i == 0 gives 0
}

// Coefficient rows in shared memory, row stride 9 so that a warp reading rows
// K = 0..8 touches nine distinct banks.
constexpr int CROW = 9;
template <typename T>
struct CoefSet {
    T cx[9 * CROW];   // x-direction table (pre-divided by dx in fast mode)
    T cz[9 * CROW];
};

// ------------------------------------------------------------------ TMA + mbarrier (bounded waits)
__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_test(uint64_t *bar, uint32_t phase)
{
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok)
                 : "r"(smem_u32(bar)), "r"(phase)
                 : "memory");
    return ok != 0;
}
__device__ __forceinline__ uint64_t global_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// Wait for the barrier phase with a wall-clock limit; on timeout record an
// error code for the host and report failure (the caller then skips its work).
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t phase, int *err)
{
    if (mbar_test(bar, phase)) return true;
    const uint64_t t0 = global_ns();
    while (!mbar_test(bar, phase)) {
        if (global_ns() - t0 > 2000000000ull) {   // 2 s
            if (err) atomicExch(err, RSGPU_ERR_TIMEOUT);
            return false;
        }
        __nanosleep(64);
    }
    return true;
}
// 2D tiled TMA load of a box at element coordinates (x, y) into shared memory.
__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, uint64_t *bar, int x, int y)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];"
        ::"r"(smem_u32(dst)), "l"(map), "r"(smem_u32(bar)), "r"(x), "r"(y)
        : "memory");
}

// ------------------------------------------------------------------ derivative blocks
// x-derivative of a quad of 4 outputs on shared row `srow` (pointer at the
// quad's first halo column).  FW: f[i+k+1]-f[i-k]; BW: f[i+k]-f[i-k-1]
// (lib/der.cpp:183-188, 378-383).  `cu` = uniform coefficients (interior), or
// per-point rows `ce[j]` (edge tiles).
template <typename T, int MODE, bool FW, bool EDGE>
__device__ __forceinline__ void dx_quad(const T *srow, const T (&cu)[NCOEF], const T *const (&ce)[4], T d, T r,
                                        T (&out)[4])
{
    using A = Ar<T, MODE>;
    T v[20];
#pragma unroll
    for (int q = 0; q < 5; q++) {
        T t[4];
        ld4(srow + 4 * q, t);
        v[4 * q] = t[0]; v[4 * q + 1] = t[1]; v[4 * q + 2] = t[2]; v[4 * q + 3] = t[3];
    }
#pragma unroll
    for (int j = 0; j < 4; j++) {
        T acc = T(0);
#pragma unroll
        for (int k = 0; k < NCOEF; k++) {
            const T dl = FW ? A::sub(v[j + 9 + k], v[j + 8 - k]) : A::sub(v[j + 8 + k], v[j + 7 - k]);
            const T c = EDGE ? ce[j][k] : cu[k];
            acc = (k == 0) ? A::mul(dl, c) : A::mad(acc, dl, c);
        }
        out[j] = (MODE == MODE_FAST) ? acc : A::div(acc, d, r);
    }
}

// z-derivatives of a column pair (local columns c, c+1 of the tile, as one
// 64-bit lane pair) for RZ rows starting at tile row zr.  Window of RZ+16 rows.
template <typename T, int MODE, bool FW, bool EDGE, int W, int RZ>
__device__ __forceinline__ void dz_pair(const T *s, int zr, int col, const T (&cu)[NCOEF], const T *const (&ce)[RZ],
                                        T d, T r, typename Pair<T>::t (&out)[RZ])
{
    using A2 = Ar2<T, MODE>;
    using P = typename Pair<T>::t;
    P w[RZ + 16];
#pragma unroll
    for (int q = 0; q < RZ + 16; q++) w[q] = *reinterpret_cast<const P *>(s + (zr + q) * W + col);
    const P d2 = A2::mk(d), r2 = A2::mk(r);
#pragma unroll
    for (int rr = 0; rr < RZ; rr++) {
        P acc;
#pragma unroll
        for (int k = 0; k < NCOEF; k++) {
            const P dl = FW ? A2::sub(w[rr + 9 + k], w[rr + 8 - k]) : A2::sub(w[rr + 8 + k], w[rr + 7 - k]);
            const P c = A2::mk(EDGE ? ce[rr][k] : cu[k]);
            acc = (k == 0) ? A2::mul(dl, c) : A2::acc(acc, dl, c);
        }
        out[rr] = (MODE == MODE_FAST) ? acc : A2::div(acc, d2, r2);
    }
}

// ------------------------------------------------------------------ C-PML helpers
__device__ __forceinline__ int xstrip(int ix, int nxp, int lpml, int &tab_base, int &col)
{
    if (ix < lpml) { tab_base = 0; col = ix; return ix; }
    const int r = ix - (nxp - lpml);
    if (r >= 0 && ix < nxp) { tab_base = 6; col = lpml + r; return r; }
    return -1;
}
__device__ __forceinline__ int zstrip(int iz, int nzp, int lpml, int &tab_base, int &row)
{
    if (iz < lpml) { tab_base = 0; row = iz; return iz; }
    const int r = iz - (nzp - lpml);
    if (r >= 0 && iz < nzp) { tab_base = 6; row = lpml + r; return r; }
    return -1;
}
// psi = B*psi + A*df ;  F -= a*(psi + C*df)   (lib/waves.cpp:252-253)
template <typename T, int MODE>
__device__ __forceinline__ T pml_correct(T F, T a, T df, T *psi, const T *tab, int lp, int base, int idx)
{
    using A = Ar<T, MODE>;
    const T tA = __ldg(tab + (base + PT_A) * lp + idx);
    const T tB = __ldg(tab + (base + PT_B) * lp + idx);
    const T tC = __ldg(tab + (base + PT_C) * lp + idx);
    T p = *psi;
    p = A::mad(A::mul(tB, p), tA, df);
    *psi = p;
    return A::msub(F, a, A::mad(p, tC, df));
}

// ------------------------------------------------------------------ tile bookkeeping
template <typename T, int TX, int TZ, int RZ>
struct Geo2D {
    static constexpr int NTX = TX / 4, NTZ = TZ / RZ, NT = NTX * NTZ;
    static constexpr int W = TX + 2 * GUARD, H = TZ + 2 * GUARD;
    static constexpr int TILE_BYTES = (int)sizeof(T) * W * H;
    static constexpr int TILE_STRIDE = (TILE_BYTES + 127) / 128 * 128;
};

// Shared-memory prologue shared by all 2D kernels: nfield halo'd tiles (TMA),
// the coefficient tables and one mbarrier.
template <typename T, int TX, int TZ, int RZ>
struct Smem2D {
    using G = Geo2D<T, TX, TZ, RZ>;
    __host__ __device__ static constexpr size_t coef_off(int nfield) { return (size_t)nfield * G::TILE_STRIDE; }
    __host__ __device__ static constexpr size_t bar_off(int nfield) { return (coef_off(nfield) + sizeof(CoefSet<T>) + 15) / 16 * 16; }
    __host__ __device__ static constexpr size_t bytes(int nfield) { return bar_off(nfield) + 16; }
};

template <typename T>
__device__ __forceinline__ void load_coefs(CoefSet<T> &s, const CoefSet<T> *g)
{
    const T *src = reinterpret_cast<const T *>(g);
    T *dst = reinterpret_cast<T *>(&s);
    for (int i = threadIdx.x; i < (int)(sizeof(CoefSet<T>) / sizeof(T)); i += blockDim.x) dst[i] = src[i];
}

// Issue the TMA loads of `nmap` halo'd tiles (maps[m_0..]) into consecutive tiles.
template <typename T, int TX, int TZ, int RZ>
__device__ __forceinline__ void tma_stage(unsigned char *sm, uint64_t *bar, const CUtensorMap *maps, const int *which,
                                          int nmap, int x0, int z0)
{
    using G = Geo2D<T, TX, TZ, RZ>;
    if (threadIdx.x == 0) {
        mbar_init(bar, 1);
        mbar_expect_tx(bar, (uint32_t)(nmap * G::TILE_BYTES));
        // element (x0 - GUARD, z0 - GUARD) of the field is element (x0, z0) of the allocation
        for (int m = 0; m < nmap; m++) tma_load_2d(sm + m * G::TILE_STRIDE, maps + which[m], bar, x0, z0);
    }
}

// Per-thread coefficient setup for one derivative direction.
template <typename T, int N>
__device__ __forceinline__ void coef_uniform(const T *tab, int order, T (&cu)[NCOEF])
{
#pragma unroll
    for (int k = 0; k < NCOEF; k++) cu[k] = tab[order * CROW + k];
}

// ------------------------------------------------------------------ acoustic 2D
// Field tensor maps per shot: [0] P, [1] Vx, [2] Vz  (acoustic)
//                             [0] Vx, [1] Vz, [2] Sxx, [3] Szz, [4] Sxz (elastic)
constexpr int NMAP = 5;

// Reduced-order stencil of K pairs at one point (reference rule near the array
// ends): taps read from memory at `stride`, K known only at run time.  Used to
// overwrite the few outputs of an edge tile whose K differs from the order.
// Two forms with the same operations in the same order: a call (stencil_k), and
// an inlined form unrolled over the NCOEF taps with the taps k >= K predicated
// off (stencil_ki), which saves the edge lanes of a warp the call's register
// saves at the price of registers in the caller.  Measured on B200, the inlined
// form is faster in the elastic 2D tile kernels (16-shot batch +11 %) and the
// acoustic 3D kernels (+14 %), slower in the acoustic 2D tile kernels of a
// 64-shot FWI batch (-6 %) and in the elastic 3D kernels (-17 %).
template <typename T, int MODE>
__device__ __noinline__ T stencil_k(const T *center, int stride, int K, const T *c, bool fw, T d, T r)
{
    using A = Ar<T, MODE>;
    if (K == 0) return T(0);
    T acc = A::mul(fw ? A::sub(center[stride], center[0]) : A::sub(center[0], center[-stride]), c[0]);
    for (int k = 1; k < K; k++) {
        const T dl = fw ? A::sub(center[(k + 1) * stride], center[-k * stride])
                        : A::sub(center[k * stride], center[-(k + 1) * stride]);
        acc = A::mad(acc, dl, c[k]);
    }
    return (MODE == MODE_FAST) ? acc : A::div(acc, d, r);
}
template <typename T, int MODE>
__device__ __forceinline__ T stencil_ki(const T *center, int stride, int K, const T *c, bool fw, T d, T r)
{
    using A = Ar<T, MODE>;
    if (K == 0) return T(0);
    T acc = A::mul(fw ? A::sub(center[stride], center[0]) : A::sub(center[0], center[-stride]), c[0]);
#pragma unroll
    for (int k = 1; k < NCOEF; k++) {
        if (k < K) {
            const T dl = fw ? A::sub(center[(k + 1) * stride], center[-k * stride])
                            : A::sub(center[k * stride], center[-(k + 1) * stride]);
            acc = A::mad(acc, dl, c[k]);
        }
    }
    return (MODE == MODE_FAST) ? acc : A::div(acc, d, r);
}
template <bool INL, typename T, int MODE>
__device__ __forceinline__ T stencil_sel(const T *center, int stride, int K, const T *c, bool fw, T d, T r)
{
    return INL ? stencil_ki<T, MODE>(center, stride, K, c, fw, d, r) : stencil_k<T, MODE>(center, stride, K, c, fw, d, r);
}

template <typename T, int MODE, int TX, int TZ, int RZ, bool INL = false>
__device__ __forceinline__ void row_dx(const T *tile, int row, int xq, const CoefSet<T> &cs, const T (&cu)[NCOEF],
                                       bool fw, bool xedge, int gx, int nxp, int order, T d, T r, T (&out)[4])
{
    using G = Geo2D<T, TX, TZ, RZ>;
    const T *ce[4] = {nullptr, nullptr, nullptr, nullptr};
    const T *srow = tile + row * G::W + xq;
    if (fw) dx_quad<T, MODE, true, false>(srow, cu, ce, d, r, out);
    else dx_quad<T, MODE, false, false>(srow, cu, ce, d, r, out);
    if (xedge) {
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int K = fw ? kfw(gx + j, nxp, order) : kbw(gx + j, nxp, order);
            if (K != order) out[j] = stencil_sel<INL, T, MODE>(srow + j + GUARD, 1, K, cs.cx + K * CROW, fw, d, r);
        }
    }
}

// FAST-mode z-derivatives of the thread's 4 columns x RZ rows, streamed: each
// of the RZ+16 window rows is read once as a 128-bit shared load and scattered
// into the RZ accumulators with paired FMAs (c*w+ and -c*w- as separate terms),
// so neither the window nor a difference is held in registers.  Same taps and
// coefficients as dz_pair; only the summation order differs.
template <int W, int RZ, bool FW>
__device__ __forceinline__ void dz_stream_f32(const float *s, int zr, int col, const float (&cu)[NCOEF],
                                              float (&out)[RZ][4])
{
    float2 lo[RZ], hi[RZ];
#pragma unroll
    for (int rr = 0; rr < RZ; rr++) { lo[rr] = make_float2(0.f, 0.f); hi[rr] = lo[rr]; }
#pragma unroll
    for (int q = 0; q < RZ + 16; q++) {
        const float4 w = *reinterpret_cast<const float4 *>(s + (zr + q) * W + col);
        const float2 wl = make_float2(w.x, w.y), wh = make_float2(w.z, w.w);
#pragma unroll
        for (int rr = 0; rr < RZ; rr++) {
            // forward: d = sum_k c_k (w[rr+9+k] - w[rr+8-k]); backward: (w[rr+8+k] - w[rr+7-k])
            const int kp = FW ? q - rr - 9 : q - rr - 8;
            const int km = FW ? rr + 8 - q : rr + 7 - q;
            if (kp >= 0 && kp < NCOEF) {
                const float2 c = make_float2(cu[kp], cu[kp]);
                lo[rr] = __ffma2_rn(wl, c, lo[rr]);
                hi[rr] = __ffma2_rn(wh, c, hi[rr]);
            }
            if (km >= 0 && km < NCOEF) {
                const float2 c = make_float2(-cu[km], -cu[km]);
                lo[rr] = __ffma2_rn(wl, c, lo[rr]);
                hi[rr] = __ffma2_rn(wh, c, hi[rr]);
            }
        }
    }
#pragma unroll
    for (int rr = 0; rr < RZ; rr++) {
        out[rr][0] = lo[rr].x; out[rr][1] = lo[rr].y; out[rr][2] = hi[rr].x; out[rr][3] = hi[rr].y;
    }
}

template <typename T, int MODE, int TX, int TZ, int RZ, bool FW, bool INL = false>
__device__ __forceinline__ void block_dz(const T *tile, int zr, int xq, const CoefSet<T> &cs, const T (&cu)[NCOEF],
                                         bool zedge, int gz, int nzp, int order, T d, T r, T (&out)[RZ][4])
{
    using G = Geo2D<T, TX, TZ, RZ>;
    using P = typename Pair<T>::t;
    if constexpr (MODE == MODE_FAST && std::is_same<T, float>::value) {
        dz_stream_f32<G::W, RZ, FW>(tile, zr, xq + GUARD, cu, out);
    } else {
        const T *ce[RZ];
#pragma unroll
        for (int q = 0; q < RZ; q++) ce[q] = nullptr;
#pragma unroll
        for (int cp = 0; cp < 2; cp++) {
            P o[RZ];
            dz_pair<T, MODE, FW, false, G::W, RZ>(tile, zr, xq + GUARD + 2 * cp, cu, ce, d, r, o);
#pragma unroll
            for (int q = 0; q < RZ; q++) { out[q][2 * cp] = o[q].x; out[q][2 * cp + 1] = o[q].y; }
        }
    }
    if (zedge) {
#pragma unroll
        for (int q = 0; q < RZ; q++) {
            const int K = FW ? kfw(gz + q, nzp, order) : kbw(gz + q, nzp, order);
            if (K != order) {
#pragma unroll
                for (int j = 0; j < 4; j++)
                    out[q][j] = stencil_sel<INL, T, MODE>(tile + (zr + q + GUARD) * G::W + xq + GUARD + j, G::W, K,
                                                          cs.cz + K * CROW, FW, d, r);
            }
        }
    }
}

// Point-wise blocks.  Rows and columns beyond the padded grid (up to the tile
// edge) lie inside the allocation; their parameters are zero, so the update
// leaves the fields there exactly zero, and loads and stores need no bounds
// checks.  `o0` is the element offset of the thread's first output.
template <typename T, int RZ>
__device__ __forceinline__ void load_block(const T *base, int o0, int pitch, T (&v)[RZ][4])
{
#pragma unroll
    for (int q = 0; q < RZ; q++) ldg4(base + o0 + q * pitch, v[q]);
}
template <typename T, int RZ>
__device__ __forceinline__ void load_block_rw(const T *base, int o0, int pitch, T (&v)[RZ][4])
{
#pragma unroll
    for (int q = 0; q < RZ; q++) ld4(base + o0 + q * pitch, v[q]);
}
template <typename T, int RZ>
__device__ __forceinline__ void store_block(T *base, int o0, int pitch, const T (&v)[RZ][4])
{
#pragma unroll
    for (int q = 0; q < RZ; q++)
        *reinterpret_cast<typename Vec4<T>::type *>(base + o0 + q * pitch) = {v[q][0], v[q][1], v[q][2], v[q][3]};
}

// C-PML memory variables of a thread's RZ x 4 block in the x strip and the z strip,
// all loaded before any is stored back, so that the loads are in flight together
// (a load that follows a store to memory the compiler cannot tell apart waits
// behind it: one L2 round trip per point otherwise).  Costs 2 x RZ x 4 registers,
// so only the kernels with room for them (the elastic ones) use it.
template <typename T, int RZ>
struct PmlBlock {
    int xi[4], xb[4], xc[4];     // per column: x strip index (-1: none), table base, psix column
    int zi[RZ], zb[RZ], zr[RZ];  // per row: z strip index (-1: none), table base, psiz row
    bool rowin[RZ], colin[4];
    T px[RZ][4], pz[RZ][4];
    __device__ __forceinline__ bool ux(int q, int j) const { return xi[j] >= 0 && rowin[q]; }
    __device__ __forceinline__ bool uz(int q, int j) const { return zi[q] >= 0 && colin[j]; }
    __device__ __forceinline__ void load(const Shot2D<T> &sh, int lpml, int gx, int gz, const T *psix, const T *psiz,
                                         bool has1, bool has2)
    {
#pragma unroll
        for (int j = 0; j < 4; j++) {
            xi[j] = has1 ? xstrip(gx + j, sh.nxp, lpml, xb[j], xc[j]) : -1;
            colin[j] = gx + j < sh.nxp;
        }
#pragma unroll
        for (int q = 0; q < RZ; q++) {
            zi[q] = has2 ? zstrip(gz + q, sh.nzp, lpml, zb[q], zr[q]) : -1;
            rowin[q] = gz + q < sh.nzp;
        }
#pragma unroll
        for (int q = 0; q < RZ; q++)
#pragma unroll
            for (int j = 0; j < 4; j++) {
                px[q][j] = ux(q, j) ? psix[(gz + q) * 2 * lpml + xc[j]] : T(0);
                pz[q][j] = uz(q, j) ? psiz[zr[q] * sh.nxp + gx + j] : T(0);
            }
    }
    __device__ __forceinline__ void store(const Shot2D<T> &sh, int lpml, int gx, int gz, T *psix, T *psiz) const
    {
#pragma unroll
        for (int q = 0; q < RZ; q++)
#pragma unroll
            for (int j = 0; j < 4; j++) {
                if (ux(q, j)) psix[(gz + q) * 2 * lpml + xc[j]] = px[q][j];
                if (uz(q, j)) psiz[zr[q] * sh.nxp + gx + j] = pz[q][j];
            }
    }
};

// One C-PML memory update with the memory value in a register (pml_correct's
// arithmetic): psi = B*psi + A*df; F -= a*(psi + C*df).
template <typename T, int MODE>
__device__ __forceinline__ T pml_step(T F, T a, T df, T &psi, const T *tab, int lp, int base, int idx)
{
    using A = Ar<T, MODE>;
    const T tA = __ldg(tab + (base + PT_A) * lp + idx);
    const T tB = __ldg(tab + (base + PT_B) * lp + idx);
    const T tC = __ldg(tab + (base + PT_C) * lp + idx);
    psi = A::mad(A::mul(tB, psi), tA, df);
    return A::msub(F, a, A::mad(psi, tC, df));
}

// update_field with the block's C-PML memory gathered first (PmlBlock).
template <typename T, int MODE, int RZ>
__device__ __forceinline__ void update_field_g(T (&F)[RZ][4], const T (&Mo)[RZ][4], const T (&d1)[RZ][4],
                                               const T (&d2)[RZ][4], const Shot2D<T> &sh, const Step2DArgs<T> &a,
                                               int gx, int gz, T *psix, int xb_add, T *psiz, int zb_add, bool const_mod,
                                               bool has1 = true, bool has2 = true)
{
    using A = Ar<T, MODE>;
    PmlBlock<T, RZ> pm;
    pm.load(sh, a.lpml, gx, gz, psix, psiz, has1, has2);
#pragma unroll
    for (int q = 0; q < RZ; q++) {
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const T am = const_mod ? a.dt : A::mul(a.dt, Mo[q][j]);
            if (has1) {
                F[q][j] = A::mad(F[q][j], am, d1[q][j]);
                if (pm.ux(q, j))
                    F[q][j] = pml_step<T, MODE>(F[q][j], am, d1[q][j], pm.px[q][j], a.pml, a.lpml, pm.xb[j] + xb_add,
                                                pm.xi[j]);
            }
            if (has2) {
                F[q][j] = A::mad(F[q][j], am, d2[q][j]);
                if (pm.uz(q, j))
                    F[q][j] = pml_step<T, MODE>(F[q][j], am, d2[q][j], pm.pz[q][j], a.pml, a.lpml, pm.zb[q] + zb_add,
                                                pm.zi[q]);
            }
        }
    }
    pm.store(sh, a.lpml, gx, gz, psix, psiz);
}

// x-part then z-part of one field, a = dt*modulus (lib/waves.cpp:245-307):
//   F += a*d1 ; [x strip] psi = B*psi + A*d1, F -= a*(psi + C*d1) ;
//   F += a*d2 ; [z strip] the same with the z memory variable.
// PML = false for tiles that do not touch a C-PML strip.
template <typename T, int MODE, int RZ, bool PML>
__device__ __forceinline__ void update_field(T (&F)[RZ][4], const T (&Mo)[RZ][4], const T (&d1)[RZ][4],
                                             const T (&d2)[RZ][4], bool has1, bool has2, const Shot2D<T> &sh,
                                             const Step2DArgs<T> &a, int gx, int gz, T *psix, int xb_add, T *psiz,
                                             int zb_add, bool const_mod)
{
    using A = Ar<T, MODE>;
#pragma unroll
    for (int q = 0; q < RZ; q++) {
        const int iz = gz + q;
        int zb = 0, zrow = 0, zi = -1;
        if (PML) zi = zstrip(iz, sh.nzp, a.lpml, zb, zrow);
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const T am = const_mod ? a.dt : A::mul(a.dt, Mo[q][j]);
            if (has1) {
                F[q][j] = A::mad(F[q][j], am, d1[q][j]);
                if (PML) {
                    int xb, xcol;
                    const int xi = (iz < sh.nzp) ? xstrip(gx + j, sh.nxp, a.lpml, xb, xcol) : -1;
                    if (xi >= 0)
                        F[q][j] = pml_correct<T, MODE>(F[q][j], am, d1[q][j], psix + iz * 2 * a.lpml + xcol, a.pml,
                                                       a.lpml, xb + xb_add, xi);
                }
            }
            if (has2) {
                F[q][j] = A::mad(F[q][j], am, d2[q][j]);
                if (PML && zi >= 0 && gx + j < sh.nxp)
                    F[q][j] = pml_correct<T, MODE>(F[q][j], am, d2[q][j], psiz + zrow * sh.nxp + gx + j, a.pml, a.lpml,
                                                   zb + zb_add, zi);
            }
        }
    }
}

template <typename T, int MODE, int RZ>
__device__ __forceinline__ void update_field_any(bool pml, T (&F)[RZ][4], const T (&Mo)[RZ][4], const T (&d1)[RZ][4],
                                                 const T (&d2)[RZ][4], bool has1, bool has2, const Shot2D<T> &sh,
                                                 const Step2DArgs<T> &a, int gx, int gz, T *psix, int xb_add, T *psiz,
                                                 int zb_add, bool const_mod)
{
    if (pml) update_field<T, MODE, RZ, true>(F, Mo, d1, d2, has1, has2, sh, a, gx, gz, psix, xb_add, psiz, zb_add, const_mod);
    else update_field<T, MODE, RZ, false>(F, Mo, d1, d2, has1, has2, sh, a, gx, gz, psix, xb_add, psiz, zb_add, const_mod);
}

// C-PML update of a tile: gathered memory loads (GAT, for tile shapes with the
// registers for them) or the point-by-point form.
template <typename T, int MODE, int RZ, bool GAT>
__device__ __forceinline__ void update_field_sel(bool pml, T (&F)[RZ][4], const T (&Mo)[RZ][4], const T (&d1)[RZ][4],
                                                 const T (&d2)[RZ][4], bool has1, bool has2, const Shot2D<T> &sh,
                                                 const Step2DArgs<T> &a, int gx, int gz, T *psix, int xb_add, T *psiz,
                                                 int zb_add, bool const_mod)
{
    if (GAT && pml) update_field_g<T, MODE, RZ>(F, Mo, d1, d2, sh, a, gx, gz, psix, xb_add, psiz, zb_add, const_mod, has1, has2);
    else update_field_any<T, MODE, RZ>(pml, F, Mo, d1, d2, has1, has2, sh, a, gx, gz, psix, xb_add, psiz, zb_add, const_mod);
}

#define RS_TILE_SETUP()                                                                        \
    using G = Geo2D<T, TX, TZ, RZ>;                                                            \
    const int tx = threadIdx.x % G::NTX, tz = threadIdx.x / G::NTX;                            \
    const int xq = 4 * tx, zr = tz * RZ, gx = tl.x0 + xq, gz = tl.z0 + zr;                     \
    const int o0 = gz * sh.pitch + gx, pitch = sh.pitch;                                       \
    const bool xe = tl.flags & TILE_XEDGE, ze = tl.flags & TILE_ZEDGE;                         \
    const bool pml = tl.flags & (TILE_XPML | TILE_ZPML);                                       \
    T cux[NCOEF], cuz[NCOEF];                                                                  \
    coef_uniform<T, 0>(cs.cx, a.order, cux);                                                   \
    coef_uniform<T, 0>(cs.cz, a.order, cuz);                                                   \
    (void)xe; (void)ze; (void)pml

// Velocity half-step: Vx += dt*Rx*Dx+P (+ x C-PML), Vz += dt*Rz*Dz+P (+ z C-PML)
// (lib/waves.cpp:217-310).
template <typename T, int MODE, int TX, int TZ, int RZ, bool INL, bool GAT>
__device__ __forceinline__ void a2d_velocity_tile(const Step2DArgs<T> &a, const Shot2D<T> &sh, const Tile2D &tl,
                                                  const T *sP, const CoefSet<T> &cs, int *err, uint64_t *bar)
{
    RS_TILE_SETUP();
    T F[RZ][4], M[RZ][4], F2[RZ][4], M2[RZ][4], d[RZ][4];
    load_block_rw<T, RZ>(sh.f[A2_VX], o0, pitch, F);
    load_block<T, RZ>(sh.m[M_RX], o0, pitch, M);
    load_block_rw<T, RZ>(sh.f[A2_VZ], o0, pitch, F2);
    load_block<T, RZ>(sh.m[M_RZ], o0, pitch, M2);
    if (!mbar_wait_bounded(bar, 0, err)) return;
#pragma unroll
    for (int q = 0; q < RZ; q++) row_dx<T, MODE, TX, TZ, RZ, INL>(sP, zr + q + GUARD, xq, cs, cux, true, xe, gx, sh.nxp, a.order, a.dx, a.rdx, d[q]);
    update_field_sel<T, MODE, RZ, GAT>(pml, F, M, d, d, true, false, sh, a, gx, gz, sh.psix[0], 3, sh.psiz[0], 3, false);
    store_block<T, RZ>(sh.f[A2_VX], o0, pitch, F);
#pragma unroll
    for (int q = 0; q < RZ; q++)
#pragma unroll
        for (int j = 0; j < 4; j++) { F[q][j] = F2[q][j]; M[q][j] = M2[q][j]; }
    block_dz<T, MODE, TX, TZ, RZ, true, INL>(sP, zr, xq, cs, cuz, ze, gz, sh.nzp, a.order, a.dz, a.rdz, d);
    update_field_sel<T, MODE, RZ, GAT>(pml, F, M, d, d, false, true, sh, a, gx, gz, sh.psix[0], 3, sh.psiz[0], 3, false);
    store_block<T, RZ>(sh.f[A2_VZ], o0, pitch, F);
}

// Stress half-step: P += dt*L*Dx-Vx (+x C-PML), then P += dt*L*Dz-Vz (+z C-PML)
// (lib/waves.cpp:313-404).
template <typename T, int MODE, int TX, int TZ, int RZ, bool INL, bool GAT>
__device__ __forceinline__ void a2d_stress_tile(const Step2DArgs<T> &a, const Shot2D<T> &sh, const Tile2D &tl,
                                                const T *sVx, const T *sVz, const CoefSet<T> &cs, int *err,
                                                uint64_t *bar)
{
    RS_TILE_SETUP();
    T F[RZ][4], M[RZ][4], d1[RZ][4], d2[RZ][4];
    load_block_rw<T, RZ>(sh.f[A2_P], o0, pitch, F);
    load_block<T, RZ>(sh.m[M_L], o0, pitch, M);
    if (!mbar_wait_bounded(bar, 0, err)) return;
#pragma unroll
    for (int q = 0; q < RZ; q++) row_dx<T, MODE, TX, TZ, RZ, INL>(sVx, zr + q + GUARD, xq, cs, cux, false, xe, gx, sh.nxp, a.order, a.dx, a.rdx, d1[q]);
    block_dz<T, MODE, TX, TZ, RZ, false, INL>(sVz, zr, xq, cs, cuz, ze, gz, sh.nzp, a.order, a.dz, a.rdz, d2);
    update_field_sel<T, MODE, RZ, GAT>(pml, F, M, d1, d2, true, true, sh, a, gx, gz, sh.psix[1], 0, sh.psiz[1], 0, false);
    store_block<T, RZ>(sh.f[A2_P], o0, pitch, F);
}

// ---------------------------------------------------------------- elastic 2D
// Velocity half-step.  Forward (lib/waves.cpp:1416-1566):
//   Vx += dt*Rx*Dx+Sxx [x stag psi0] ; Vx += dt*Rx*Dz-Sxz [z psi0]
//   Vz += dt*Rz*Dx-Sxz [x psi1]      ; Vz += dt*Rz*Dz+Szz [z stag psi1]
// Adjoint (lib/waves.cpp:1738-1913): Sxx -> L2M*Sxx + L*Szz, Sxz -> M*Sxz,
// Szz -> L*Sxx + L2M*Szz (formed in shared memory after the TMA loads).
template <typename T, int MODE, int TX, int TZ, int RZ>
__device__ __forceinline__ void e2d_velocity_tile(const Step2DArgs<T> &a, const Shot2D<T> &sh, const Tile2D &tl,
                                                  const T *sXX, const T *sZZ, const T *sXZ, const CoefSet<T> &cs,
                                                  uint64_t *bar, int *err, uint32_t phase = 0)
{
    RS_TILE_SETUP();
    T F[RZ][4], M[RZ][4], F2[RZ][4], M2[RZ][4], d1[RZ][4], d2[RZ][4];
    // all point-wise inputs of both passes are requested before the first wait
    load_block_rw<T, RZ>(sh.f[E2_VX], o0, pitch, F);
    load_block<T, RZ>(sh.m[M_RX], o0, pitch, M);
    load_block_rw<T, RZ>(sh.f[E2_VZ], o0, pitch, F2);
    load_block<T, RZ>(sh.m[M_RZ], o0, pitch, M2);
    if (bar && !mbar_wait_bounded(bar, phase, err)) return;
#pragma unroll
    for (int q = 0; q < RZ; q++) row_dx<T, MODE, TX, TZ, RZ, true>(sXX, zr + q + GUARD, xq, cs, cux, true, xe, gx, sh.nxp, a.order, a.dx, a.rdx, d1[q]);
    block_dz<T, MODE, TX, TZ, RZ, false, true>(sXZ, zr, xq, cs, cuz, ze, gz, sh.nzp, a.order, a.dz, a.rdz, d2);
    if (pml) update_field_g<T, MODE, RZ>(F, M, d1, d2, sh, a, gx, gz, sh.psix[0], 3, sh.psiz[0], 0, false);
    else update_field<T, MODE, RZ, false>(F, M, d1, d2, true, true, sh, a, gx, gz, sh.psix[0], 3, sh.psiz[0], 0, false);
    store_block<T, RZ>(sh.f[E2_VX], o0, pitch, F);
#pragma unroll
    for (int q = 0; q < RZ; q++)
#pragma unroll
        for (int j = 0; j < 4; j++) { F[q][j] = F2[q][j]; M[q][j] = M2[q][j]; }
#pragma unroll
    for (int q = 0; q < RZ; q++) row_dx<T, MODE, TX, TZ, RZ, true>(sXZ, zr + q + GUARD, xq, cs, cux, false, xe, gx, sh.nxp, a.order, a.dx, a.rdx, d1[q]);
    block_dz<T, MODE, TX, TZ, RZ, true, true>(sZZ, zr, xq, cs, cuz, ze, gz, sh.nzp, a.order, a.dz, a.rdz, d2);
    if (pml) update_field_g<T, MODE, RZ>(F, M, d1, d2, sh, a, gx, gz, sh.psix[1], 0, sh.psiz[1], 3, false);
    else update_field<T, MODE, RZ, false>(F, M, d1, d2, true, true, sh, a, gx, gz, sh.psix[1], 0, sh.psiz[1], 3, false);
    store_block<T, RZ>(sh.f[E2_VZ], o0, pitch, F);
}

// Normal stresses of the elastic stress half-step (lib/waves.cpp:1596-1674):
//   d1 = Dx-Vx: Sxx += dt*L2M*d1, Szz += dt*L*d1, one x memory update for both;
//   d2 = Dz-Vz: Sxx += dt*L*d2,   Szz += dt*L2M*d2, one z memory update;
//   free surface: Szz = 0 on row lpml.
// Adjoint (lib/waves.cpp:1939-2018): Sxx += dt*d1, Szz += dt*d2 with their own memories.
template <typename T, int MODE, int RZ, bool PML, bool ADJ>
__device__ __forceinline__ void update_normal(T (&sxx)[RZ][4], T (&szz)[RZ][4], const T (&l)[RZ][4],
                                              const T (&l2m)[RZ][4], const T (&d1)[RZ][4], const T (&d2)[RZ][4],
                                              const Shot2D<T> &sh, const Step2DArgs<T> &a, int gx, int gz)
{
    using A = Ar<T, MODE>;
    PmlBlock<T, RZ> pm;
    if (PML) pm.load(sh, a.lpml, gx, gz, sh.psix[2], sh.psiz[2], true, true);
#pragma unroll
    for (int q = 0; q < RZ; q++) {
        const bool fsrow = sh.fs && gz + q == a.lpml;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            if (!ADJ) {
                const T a2 = A::mul(a.dt, l2m[q][j]), a1 = A::mul(a.dt, l[q][j]);
                sxx[q][j] = A::mad(sxx[q][j], a2, d1[q][j]);
                szz[q][j] = A::mad(szz[q][j], a1, d1[q][j]);
                if (PML && pm.ux(q, j)) {
                    const int xb = pm.xb[j], xi = pm.xi[j];
                    const T tA = __ldg(a.pml + (xb + PT_A) * a.lpml + xi), tB = __ldg(a.pml + (xb + PT_B) * a.lpml + xi),
                            tC = __ldg(a.pml + (xb + PT_C) * a.lpml + xi);
                    const T p = A::mad(A::mul(tB, pm.px[q][j]), tA, d1[q][j]);
                    pm.px[q][j] = p;
                    const T cq = A::mad(p, tC, d1[q][j]);
                    sxx[q][j] = A::msub(sxx[q][j], a2, cq);
                    szz[q][j] = A::msub(szz[q][j], a1, cq);
                }
                sxx[q][j] = A::mad(sxx[q][j], a1, d2[q][j]);
                szz[q][j] = A::mad(szz[q][j], a2, d2[q][j]);
                if (PML && pm.uz(q, j)) {
                    const int zb = pm.zb[q], zi = pm.zi[q];
                    const T tA = __ldg(a.pml + (zb + PT_A) * a.lpml + zi), tB = __ldg(a.pml + (zb + PT_B) * a.lpml + zi),
                            tC = __ldg(a.pml + (zb + PT_C) * a.lpml + zi);
                    const T p = A::mad(A::mul(tB, pm.pz[q][j]), tA, d2[q][j]);
                    pm.pz[q][j] = p;
                    const T cq = A::mad(p, tC, d2[q][j]);
                    sxx[q][j] = A::msub(sxx[q][j], a1, cq);
                    szz[q][j] = A::msub(szz[q][j], a2, cq);
                }
            } else {
                sxx[q][j] = A::mad(sxx[q][j], a.dt, d1[q][j]);
                if (PML && pm.ux(q, j))
                    sxx[q][j] = pml_step<T, MODE>(sxx[q][j], a.dt, d1[q][j], pm.px[q][j], a.pml, a.lpml, pm.xb[j],
                                                  pm.xi[j]);
                szz[q][j] = A::mad(szz[q][j], a.dt, d2[q][j]);
                if (PML && pm.uz(q, j))
                    szz[q][j] = pml_step<T, MODE>(szz[q][j], a.dt, d2[q][j], pm.pz[q][j], a.pml, a.lpml, pm.zb[q],
                                                  pm.zi[q]);
            }
            if (fsrow) szz[q][j] = T(0);
        }
    }
    if (PML) pm.store(sh, a.lpml, gx, gz, sh.psix[2], sh.psiz[2]);
}

// Stress half-step.  Forward (lib/waves.cpp:1571-1735): normal stresses as
// above, then Sxz += dt*M*Dx+Vz [x stag psi3] ; Sxz += dt*M*Dz+Vx [z stag psi3].
// Adjoint (lib/waves.cpp:1916-2080): Sxz without the modulus.
template <typename T, int MODE, int TX, int TZ, int RZ, bool ADJ>
__device__ __forceinline__ void e2d_stress_tile(const Step2DArgs<T> &a, const Shot2D<T> &sh, const Tile2D &tl,
                                                const T *sVx, const T *sVz, const CoefSet<T> &cs, uint64_t *bar,
                                                int *err, uint32_t phase = 0)
{
    RS_TILE_SETUP();
    T d1[RZ][4], d2[RZ][4], sxx[RZ][4], szz[RZ][4];
    {
        T l[RZ][4], l2m[RZ][4];
        load_block_rw<T, RZ>(sh.f[E2_SXX], o0, pitch, sxx);
        load_block_rw<T, RZ>(sh.f[E2_SZZ], o0, pitch, szz);
        if (!ADJ) {
            load_block<T, RZ>(sh.m[M_L], o0, pitch, l);
            load_block<T, RZ>(sh.m[M_L2M], o0, pitch, l2m);
        }
        // warm the shear-stress inputs of the second pass into L1/L2 meanwhile
#pragma unroll
        for (int q = 0; q < RZ; q++) {
            asm volatile("prefetch.global.L2 [%0];" ::"l"(sh.f[E2_SXZ] + o0 + q * pitch));
            if (!ADJ) asm volatile("prefetch.global.L2 [%0];" ::"l"(sh.m[M_M] + o0 + q * pitch));
        }
        if (bar && !mbar_wait_bounded(bar, phase, err)) return;
#pragma unroll
        for (int q = 0; q < RZ; q++) row_dx<T, MODE, TX, TZ, RZ, true>(sVx, zr + q + GUARD, xq, cs, cux, false, xe, gx, sh.nxp, a.order, a.dx, a.rdx, d1[q]);
        block_dz<T, MODE, TX, TZ, RZ, false, true>(sVz, zr, xq, cs, cuz, ze, gz, sh.nzp, a.order, a.dz, a.rdz, d2);
        if (pml) update_normal<T, MODE, RZ, true, ADJ>(sxx, szz, l, l2m, d1, d2, sh, a, gx, gz);
        else update_normal<T, MODE, RZ, false, ADJ>(sxx, szz, l, l2m, d1, d2, sh, a, gx, gz);
    }
    {
        // the shear inputs are requested before the normal stresses are stored: a
        // load that follows a store to memory the compiler cannot tell apart waits
        // behind it
        T F[RZ][4], M[RZ][4];
        load_block_rw<T, RZ>(sh.f[E2_SXZ], o0, pitch, F);
        if (!ADJ) load_block<T, RZ>(sh.m[M_M], o0, pitch, M);
        store_block<T, RZ>(sh.f[E2_SXX], o0, pitch, sxx);
        store_block<T, RZ>(sh.f[E2_SZZ], o0, pitch, szz);
#pragma unroll
        for (int q = 0; q < RZ; q++) row_dx<T, MODE, TX, TZ, RZ, true>(sVz, zr + q + GUARD, xq, cs, cux, true, xe, gx, sh.nxp, a.order, a.dx, a.rdx, d1[q]);
        block_dz<T, MODE, TX, TZ, RZ, true, true>(sVx, zr, xq, cs, cuz, ze, gz, sh.nzp, a.order, a.dz, a.rdz, d2);
        if (pml) update_field_g<T, MODE, RZ>(F, M, d1, d2, sh, a, gx, gz, sh.psix[3], 3, sh.psiz[3], 3, ADJ);
        else update_field<T, MODE, RZ, false>(F, M, d1, d2, true, true, sh, a, gx, gz, sh.psix[3], 3, sh.psiz[3], 3, ADJ);
        store_block<T, RZ>(sh.f[E2_SXZ], o0, pitch, F);
    }
}

// ------------------------------------------------------------------ kernels

template <typename T, int MODE, int TX, int TZ, int RZ, int MINB, bool INL>
__global__ void __launch_bounds__(Geo2D<T, TX, TZ, RZ>::NT, MINB)
a2d_velocity(Step2DArgs<T> a, const CoefSet<T> *coefs, const CUtensorMap *maps, int *err)
{
    using S = Smem2D<T, TX, TZ, RZ>;
    extern __shared__ __align__(128) unsigned char sm[];
    CoefSet<T> &cs = *reinterpret_cast<CoefSet<T> *>(sm + S::coef_off(1));
    uint64_t *bar = reinterpret_cast<uint64_t *>(sm + S::bar_off(1));
    const Tile2D tl = a.tiles[blockIdx.x];
    const Shot2D<T> &sh = a.shots[tl.shot];
    const int which[1] = {tl.shot * NMAP + A2_P};
    tma_stage<T, TX, TZ, RZ>(sm, bar, maps, which, 1, tl.x0, tl.z0);
    load_coefs(cs, coefs);
    __syncthreads();
    const T *sP = reinterpret_cast<const T *>(sm);
    a2d_velocity_tile<T, MODE, TX, TZ, RZ, INL, (65536 / (Geo2D<T, TX, TZ, RZ>::NT * MINB) >= 128)>(a, sh, tl, sP, cs, err, bar);
}

template <typename T, int MODE, int TX, int TZ, int RZ, int MINB, bool INL>
__global__ void __launch_bounds__(Geo2D<T, TX, TZ, RZ>::NT, MINB)
a2d_stress(Step2DArgs<T> a, const CoefSet<T> *coefs, const CUtensorMap *maps, int *err)
{
    using G = Geo2D<T, TX, TZ, RZ>;
    using S = Smem2D<T, TX, TZ, RZ>;
    extern __shared__ __align__(128) unsigned char sm[];
    CoefSet<T> &cs = *reinterpret_cast<CoefSet<T> *>(sm + S::coef_off(2));
    uint64_t *bar = reinterpret_cast<uint64_t *>(sm + S::bar_off(2));
    const Tile2D tl = a.tiles[blockIdx.x];
    const Shot2D<T> &sh = a.shots[tl.shot];
    const int which[2] = {tl.shot * NMAP + A2_VX, tl.shot * NMAP + A2_VZ};
    tma_stage<T, TX, TZ, RZ>(sm, bar, maps, which, 2, tl.x0, tl.z0);
    load_coefs(cs, coefs);
    __syncthreads();
    const T *sVx = reinterpret_cast<const T *>(sm), *sVz = reinterpret_cast<const T *>(sm + G::TILE_STRIDE);
    a2d_stress_tile<T, MODE, TX, TZ, RZ, INL, (65536 / (Geo2D<T, TX, TZ, RZ>::NT * MINB) >= 128)>(a, sh, tl, sVx, sVz, cs, err, bar);
}

// Adjoint work arrays in place: wrk1 = L2M*Sxx + L*Szz, wrk3 = L*Sxx + L2M*Szz,
// wrk2 = M*Sxz (lib/waves.cpp:1774, 1812, 1885), over the whole halo'd tile.
template <typename T, int MODE, int TX, int TZ, int RZ>
__device__ __forceinline__ void adjoint_work(T *sXX, T *sZZ, T *sXZ, const Shot2D<T> &sh, int x0, int z0)
{
    using G = Geo2D<T, TX, TZ, RZ>;
    using A = Ar<T, MODE>;
    const long off0 = (long)(z0 - GUARD) * sh.pitch + (x0 - GUARD);
    for (int q = threadIdx.x; q < G::W * G::H; q += G::NT) {
        const int rr = q / G::W, c = q - rr * G::W;
        const long o = off0 + (long)rr * sh.pitch + c;
        const T sxx = sXX[q], szz = sZZ[q], l = sh.m[M_L][o], l2m = sh.m[M_L2M][o], m = sh.m[M_M][o];
        sXX[q] = A::add(A::mul(l2m, sxx), A::mul(l, szz));
        sZZ[q] = A::add(A::mul(l, sxx), A::mul(l2m, szz));
        sXZ[q] = A::mul(m, sXZ[q]);
    }
}

template <typename T, int MODE, int TX, int TZ, int RZ, int MINB, bool ADJ>
__global__ void __launch_bounds__(Geo2D<T, TX, TZ, RZ>::NT, MINB)
e2d_velocity(Step2DArgs<T> a, const CoefSet<T> *coefs, const CUtensorMap *maps, int *err)
{
    using G = Geo2D<T, TX, TZ, RZ>;
    using S = Smem2D<T, TX, TZ, RZ>;
    extern __shared__ __align__(128) unsigned char sm[];
    CoefSet<T> &cs = *reinterpret_cast<CoefSet<T> *>(sm + S::coef_off(3));
    uint64_t *bar = reinterpret_cast<uint64_t *>(sm + S::bar_off(3));
    const Tile2D tl = a.tiles[blockIdx.x];
    const Shot2D<T> &sh = a.shots[tl.shot];
    const int which[3] = {tl.shot * NMAP + E2_SXX, tl.shot * NMAP + E2_SZZ, tl.shot * NMAP + E2_SXZ};
    tma_stage<T, TX, TZ, RZ>(sm, bar, maps, which, 3, tl.x0, tl.z0);
    load_coefs(cs, coefs);
    __syncthreads();
    T *sXX = reinterpret_cast<T *>(sm), *sZZ = reinterpret_cast<T *>(sm + G::TILE_STRIDE),
      *sXZ = reinterpret_cast<T *>(sm + 2 * G::TILE_STRIDE);
    uint64_t *wbar = bar;
    if (ADJ) {
        // every thread reaches the same barriers whether or not the wait succeeded
        const bool ok = __syncthreads_and(mbar_wait_bounded(bar, 0, err));
        if (!ok) return;
        adjoint_work<T, MODE, TX, TZ, RZ>(sXX, sZZ, sXZ, sh, tl.x0, tl.z0);
        __syncthreads();
        wbar = nullptr;
    }
    e2d_velocity_tile<T, MODE, TX, TZ, RZ>(a, sh, tl, sXX, sZZ, sXZ, cs, wbar, err);
}

template <typename T, int MODE, int TX, int TZ, int RZ, int MINB, bool ADJ>
__global__ void __launch_bounds__(Geo2D<T, TX, TZ, RZ>::NT, MINB)
e2d_stress(Step2DArgs<T> a, const CoefSet<T> *coefs, const CUtensorMap *maps, int *err)
{
    using G = Geo2D<T, TX, TZ, RZ>;
    using S = Smem2D<T, TX, TZ, RZ>;
    extern __shared__ __align__(128) unsigned char sm[];
    CoefSet<T> &cs = *reinterpret_cast<CoefSet<T> *>(sm + S::coef_off(2));
    uint64_t *bar = reinterpret_cast<uint64_t *>(sm + S::bar_off(2));
    const Tile2D tl = a.tiles[blockIdx.x];
    const Shot2D<T> &sh = a.shots[tl.shot];
    const int which[2] = {tl.shot * NMAP + E2_VX, tl.shot * NMAP + E2_VZ};
    tma_stage<T, TX, TZ, RZ>(sm, bar, maps, which, 2, tl.x0, tl.z0);
    load_coefs(cs, coefs);
    __syncthreads();
    const T *sVx = reinterpret_cast<const T *>(sm), *sVz = reinterpret_cast<const T *>(sm + G::TILE_STRIDE);
    e2d_stress_tile<T, MODE, TX, TZ, RZ, ADJ>(a, sh, tl, sVx, sVz, cs, bar, err);
}

// ---------------------------------------------------------------- sources and receivers
// One CTA per shot.  Injection first (lib/waves.cpp:407-497, 2085-2174), then,
// after a CTA barrier, recording (lib/waves.cpp:500-595, 2178-2288) of the same step.
template <typename T, int MODE>
__global__ void inject_record_2d(const Shot2D<T> *shots, const InjRec<T> *plans, T dt, int it_base,
                                 const int *it_dev)
{
    using A = Ar<T, MODE == MODE_FAST ? MODE_FAST : MODE_IEEE>;
    const Shot2D<T> &sh = shots[blockIdx.x];
    const InjRec<T> &pl = plans[blockIdx.x];
    const int it_step = it_base + (it_dev ? *it_dev : 0);
    const int it = pl.rev ? pl.nt - 1 - it_step : it_step;
    for (int set = 0; set < pl.ninjsets; set++) {
        const InjSet<T> &q = pl.inj[set];
        if (q.kind == INJ_NONE) continue;
        if (set > 0) __syncthreads();   // sets that touch the same field add in set order
        for (int j = threadIdx.x; j < q.ninj; j += blockDim.x) {
            const int p = q.pt[j];
            if (q.kind == INJ_E2_P) {
                T sxx = sh.f[E2_SXX][p], szz = sh.f[E2_SZZ][p];
                for (int c = q.start[j]; c < q.start[j + 1]; c++) {
                    const T w = q.wav[(long)q.trace[c] * pl.nt + it];
                    const T s = A::mul(A::mul(A::mul(dt, w), q.wx[c]), q.wz[c]);
                    sxx = A::sub(sxx, s);
                    szz = A::sub(szz, s);
                }
                sh.f[E2_SXX][p] = sxx;
                sh.f[E2_SZZ][p] = szz;
            } else {
                T *F; const T *Mod;
                switch (q.kind) {
                case INJ_A2_P: F = sh.f[A2_P]; Mod = sh.m[M_L]; break;
                case INJ_A2_VX: F = sh.f[A2_VX]; Mod = sh.m[M_RX]; break;
                case INJ_A2_VZ: F = sh.f[A2_VZ]; Mod = sh.m[M_RZ]; break;
                case INJ_E2_VX: F = sh.f[E2_VX]; Mod = sh.m[M_RX]; break;
                default: F = sh.f[E2_VZ]; Mod = sh.m[M_RZ]; break;
                }
                T v = F[p];
                const T dm = A::mul(dt, Mod[p]);
                for (int c = q.start[j]; c < q.start[j + 1]; c++) {
                    const T w = q.wav[(long)q.trace[c] * pl.nt + it];
                    v = A::add(v, A::mul(A::mul(A::mul(dm, w), q.wx[c]), q.wz[c]));
                }
                F[p] = v;
            }
        }
    }
    if (pl.nrecsets == 0 || (pl.rec_gate && *pl.rec_gate == 0)) return;
    __syncthreads();
    for (int set = 0; set < pl.nrecsets; set++) {
        const RecSet<T> &q = pl.rec[set];
        if (q.kind == REC_NONE) continue;
        for (int tr = threadIdx.x; tr < q.nrec; tr += blockDim.x) {
            const int p = q.pt[tr];
            if (p < 0) continue;
            const T wx0 = q.w[4 * tr], wx1 = q.w[4 * tr + 1];
            const T wz0 = q.w[4 * tr + 2], wz1 = q.w[4 * tr + 3];
            const int off[4] = {0, 1, sh.pitch, sh.pitch + 1};
            const T wx[4] = {wx0, wx1, wx0, wx1}, wz[4] = {wz0, wz0, wz1, wz1};
            T *out = q.out + (long)tr * pl.nt + it;
            if (q.kind == REC_E2_P) {
                // (1./2.)*xtri*ytri*F/factor is evaluated in double by the reference and
                // added to the T-typed trace sample (lib/waves.cpp:2238-2239)
                const double fac = (double)q.factor[tr];
                T acc = *out;
#pragma unroll
                for (int c = 0; c < 4; c++) {
                    const double w = __dmul_rn(__dmul_rn(0.5, (double)wx[c]), (double)wz[c]);
                    acc = (T)__dadd_rn((double)acc, __ddiv_rn(__dmul_rn(w, (double)sh.f[E2_SXX][p + off[c]]), fac));
                    acc = (T)__dadd_rn((double)acc, __ddiv_rn(__dmul_rn(w, (double)sh.f[E2_SZZ][p + off[c]]), fac));
                }
                *out = acc;
            } else {
                if (q.kind == REC_E2_PSUM) {
                    T acc = *out;
#pragma unroll
                    for (int c = 0; c < 4; c++)
                        acc = A::add(acc, A::mul(A::mul(wx[c], wz[c]), A::add(sh.f[E2_SXX][p + off[c]], sh.f[E2_SZZ][p + off[c]])));
                    *out = acc;
                    continue;
                }
                const T *F;
                switch (q.kind) {
                case REC_A2_P: F = sh.f[A2_P]; break;
                case REC_A2_VX: F = sh.f[A2_VX]; break;
                case REC_A2_VZ: F = sh.f[A2_VZ]; break;
                case REC_E2_VX: F = sh.f[E2_VX]; break;
                default: F = sh.f[E2_VZ]; break;
                }
                T acc = *out;
#pragma unroll
                for (int c = 0; c < 4; c++) acc = A::add(acc, A::mul(A::mul(wx[c], wz[c]), F[p + off[c]]));
                *out = acc;
            }
        }
    }
}

static __global__ void advance_counter(int *it_dev, int by)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) *it_dev += by;
}

static __global__ void set_counter(int *it_dev, int value)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) *it_dev = value;
}

// ---------------------------------------------------------------- launchers
template <typename K>
static cudaError_t set_smem(K k, size_t bytes)
{
    return cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

template <typename T, int MODE, int TX, int TZ, int RZ, int MINB>
cudaError_t launch_2d_cfg(int physics, int half, int flags, const Step2DArgs<T> &a, const CoefSet<T> *coefs,
                          const CUtensorMap *maps, int *err, int grid, cudaStream_t st)
{
    using G = Geo2D<T, TX, TZ, RZ>;
    using S = Smem2D<T, TX, TZ, RZ>;
    const bool adj = (flags & LAUNCH_ADJ) != 0, inl = (flags & LAUNCH_INL) != 0;
    if (physics == PHYS_A2D) {
        if (half == 0) {
            static const cudaError_t e0 = set_smem(a2d_velocity<T, MODE, TX, TZ, RZ, MINB, false>, S::bytes(1));
            static const cudaError_t e1 = set_smem(a2d_velocity<T, MODE, TX, TZ, RZ, MINB, true>, S::bytes(1));
            if (e0 != cudaSuccess) return e0;
            if (e1 != cudaSuccess) return e1;
            if (inl) a2d_velocity<T, MODE, TX, TZ, RZ, MINB, true><<<grid, G::NT, S::bytes(1), st>>>(a, coefs, maps, err);
            else a2d_velocity<T, MODE, TX, TZ, RZ, MINB, false><<<grid, G::NT, S::bytes(1), st>>>(a, coefs, maps, err);
        } else {
            static const cudaError_t e0 = set_smem(a2d_stress<T, MODE, TX, TZ, RZ, MINB, false>, S::bytes(2));
            static const cudaError_t e1 = set_smem(a2d_stress<T, MODE, TX, TZ, RZ, MINB, true>, S::bytes(2));
            if (e0 != cudaSuccess) return e0;
            if (e1 != cudaSuccess) return e1;
            if (inl) a2d_stress<T, MODE, TX, TZ, RZ, MINB, true><<<grid, G::NT, S::bytes(2), st>>>(a, coefs, maps, err);
            else a2d_stress<T, MODE, TX, TZ, RZ, MINB, false><<<grid, G::NT, S::bytes(2), st>>>(a, coefs, maps, err);
        }
    } else {
        if (half == 0) {
            static const cudaError_t e0 = set_smem(e2d_velocity<T, MODE, TX, TZ, RZ, MINB, false>, S::bytes(3));
            static const cudaError_t e1 = set_smem(e2d_velocity<T, MODE, TX, TZ, RZ, MINB, true>, S::bytes(3));
            if (e0 != cudaSuccess) return e0;
            if (e1 != cudaSuccess) return e1;
            if (adj) e2d_velocity<T, MODE, TX, TZ, RZ, MINB, true><<<grid, G::NT, S::bytes(3), st>>>(a, coefs, maps, err);
            else e2d_velocity<T, MODE, TX, TZ, RZ, MINB, false><<<grid, G::NT, S::bytes(3), st>>>(a, coefs, maps, err);
        } else {
            static const cudaError_t e0 = set_smem(e2d_stress<T, MODE, TX, TZ, RZ, MINB, false>, S::bytes(2));
            static const cudaError_t e1 = set_smem(e2d_stress<T, MODE, TX, TZ, RZ, MINB, true>, S::bytes(2));
            if (e0 != cudaSuccess) return e0;
            if (e1 != cudaSuccess) return e1;
            if (adj) e2d_stress<T, MODE, TX, TZ, RZ, MINB, true><<<grid, G::NT, S::bytes(2), st>>>(a, coefs, maps, err);
            else e2d_stress<T, MODE, TX, TZ, RZ, MINB, false><<<grid, G::NT, S::bytes(2), st>>>(a, coefs, maps, err);
        }
    }
    return cudaGetLastError();
}

}  // namespace rsgpu
