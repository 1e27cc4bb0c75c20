// 2D staggered-grid finite-difference propagators for sm_100a (kernel templates).
//
// One kernel per half-step (velocity, stress), each covering every shot of a
// batch in one launch: the grid walks a table of (shot, tile) work items, so
// shots with different aperture windows share a launch.  Each CTA stages the
// input fields of a TX x TZ tile plus an 8-cell halo in shared memory, then every
// thread produces a 4(x) x RZ(z) block of outputs with the C-PML memory-variable
// update and correction fused into the same pass.
//
// Arithmetic follows the reference operation by operation (Der::ddx_fw etc. in
// lib/der.cpp:155-540, WavesAcoustic2D/WavesElastic2D::forwardstep* in
// lib/waves.cpp:217-404, 1416-1735, backwardstep* in lib/waves.cpp:1738-2080).
// With EXACT=true every add/sub/mul/div is an explicitly rounded IEEE op in the
// reference's order (no FMA contraction), so a float run reproduces the
// reference's float results bit for bit; EXACT=false allows FMA and folds 1/dx
// into the coefficients.
#pragma once
#include "rsgpu_internal.h"
#include "rsgpu_kernels.h"

namespace rsgpu {

// ------------------------------------------------------------------ arithmetic
template <typename T, bool EXACT> struct Ar;
template <> struct Ar<float, true> {
    static __device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
    static __device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
    static __device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
    static __device__ __forceinline__ float div(float a, float b) { return __fdiv_rn(a, b); }
    // a + b*c with the product rounded first
    static __device__ __forceinline__ float mad(float a, float b, float c) { return __fadd_rn(a, __fmul_rn(b, c)); }
};
template <> struct Ar<float, false> {
    static __device__ __forceinline__ float add(float a, float b) { return a + b; }
    static __device__ __forceinline__ float sub(float a, float b) { return a - b; }
    static __device__ __forceinline__ float mul(float a, float b) { return a * b; }
    static __device__ __forceinline__ float div(float a, float b) { return a / b; }
    static __device__ __forceinline__ float mad(float a, float b, float c) { return fmaf(b, c, a); }
};
template <> struct Ar<double, true> {
    static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
    static __device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
    static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
    static __device__ __forceinline__ double div(double a, double b) { return __ddiv_rn(a, b); }
    static __device__ __forceinline__ double mad(double a, double b, double c) { return __dadd_rn(a, __dmul_rn(b, c)); }
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

// Reference order of the stencil for one output (lib/der.cpp:183-188):
//   acc = (f[a0]-f[b0])*c0 ; acc += (f[ak]-f[bk])*ck for k=1..7 ; acc /= d
// In EXACT mode the table holds the raw coefficients (unused taps zero) and
// `d` is the grid spacing.  In fast mode the table is pre-divided by d.
template <typename T, bool EXACT>
__device__ __forceinline__ T stencil(const T (&dlt)[NCOEF], const T *c, T d)
{
    using A = Ar<T, EXACT>;
    T acc = A::mul(dlt[0], c[0]);
#pragma unroll
    for (int k = 1; k < NCOEF; k++) acc = EXACT ? A::add(acc, A::mul(dlt[k], c[k])) : A::mad(acc, dlt[k], c[k]);
    if (EXACT) acc = A::div(acc, d);
    return acc;
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

// Coefficient rows live in shared memory with a row stride of 9 so that a warp
// reading rows K=0..8 touches nine distinct banks.
constexpr int CROW = 9;

template <typename T>
struct CoefSet {
    T cx[9 * CROW];   // x-direction table (pre-divided by dx in fast mode)
    T cz[9 * CROW];
};

// ------------------------------------------------------------------ tile loader
// smem tile: (TZ + 2G) rows x (TX + 2G) cols, origin at (x0 - G, z0 - G).
template <typename T, int TX, int TZ, int NT>
__device__ __forceinline__ void load_tile(T *s, const T *origin, int pitch, int x0, int z0)
{
    constexpr int W = TX + 2 * GUARD, H = TZ + 2 * GUARD, WQ = W / 4;
    const T *base = origin + (long)(z0 - GUARD) * pitch + (x0 - GUARD);
    for (int q = threadIdx.x; q < WQ * H; q += NT) {
        int r = q / WQ, c = (q - r * WQ) * 4;
        typename Vec4<T>::type v = *reinterpret_cast<const typename Vec4<T>::type *>(base + (long)r * pitch + c);
        *reinterpret_cast<typename Vec4<T>::type *>(s + r * W + c) = v;
    }
}

// Elementwise tile of a combination a*F1 + b*F2 (adjoint work arrays, exact order:
// lib/waves.cpp:1774 wrk = L2M*Sxx + L*Szz).
template <typename T, bool EXACT, int TX, int TZ, int NT>
__device__ __forceinline__ void load_tile_comb(T *s, const T *m1, const T *f1, const T *m2, const T *f2,
                                               int pitch, int x0, int z0)
{
    using A = Ar<T, EXACT>;
    constexpr int W = TX + 2 * GUARD, H = TZ + 2 * GUARD;
    long off0 = (long)(z0 - GUARD) * pitch + (x0 - GUARD);
    for (int q = threadIdx.x; q < W * H; q += NT) {
        int r = q / W, c = q - r * W;
        long o = off0 + (long)r * pitch + c;
        T v = A::mul(m1[o], f1[o]);
        if (m2) v = A::add(v, A::mul(m2[o], f2[o]));
        s[r * W + c] = v;
    }
}

// x-derivatives of a quad of 4 outputs on smem row `row` (local x of the quad = xq).
// FW: df[i] uses f[i+k+1]-f[i-k];  BW: f[i+k]-f[i-k-1].
template <typename T, bool EXACT, bool FW, int W>
__device__ __forceinline__ void dx_quad(const T *s, int row, int xq, const T *crow[4], T d, T (&out)[4])
{
    T v[20];
#pragma unroll
    for (int j = 0; j < 5; j++) {
        T q[4];
        ld4(s + row * W + xq + 4 * j, q);
        v[4 * j] = q[0]; v[4 * j + 1] = q[1]; v[4 * j + 2] = q[2]; v[4 * j + 3] = q[3];
    }
#pragma unroll
    for (int j = 0; j < 4; j++) {
        T dl[NCOEF];
#pragma unroll
        for (int k = 0; k < NCOEF; k++)
            dl[k] = FW ? Ar<T, EXACT>::sub(v[j + 9 + k], v[j + 8 - k]) : Ar<T, EXACT>::sub(v[j + 8 + k], v[j + 7 - k]);
        out[j] = stencil<T, EXACT>(dl, crow[j], d);
    }
}

// z-derivatives of the 4 columns of a quad for RZ rows starting at local row zr.
// One column at a time with a scalar window of RZ+16 values keeps the register
// footprint small; the results are returned per (row, column).
template <typename T, bool EXACT, bool FW, int W, int RZ>
__device__ __forceinline__ void dz_block(const T *s, int zr, int xq, const T *crow[RZ], T d, T (&out)[RZ][4])
{
#pragma unroll
    for (int j = 0; j < 4; j++) {
        T w[RZ + 16];
#pragma unroll
        for (int r = 0; r < RZ + 16; r++) w[r] = s[(zr + r) * W + xq + GUARD + j];
#pragma unroll
        for (int r = 0; r < RZ; r++) {
            T dl[NCOEF];
#pragma unroll
            for (int k = 0; k < NCOEF; k++)
                dl[k] = FW ? Ar<T, EXACT>::sub(w[r + 9 + k], w[r + 8 - k]) : Ar<T, EXACT>::sub(w[r + 8 + k], w[r + 7 - k]);
            out[r][j] = stencil<T, EXACT>(dl, crow[r], d);
        }
    }
}

// ------------------------------------------------------------------ PML helpers
// Left/right strip of x: returns table index and psi column, or -1.
__device__ __forceinline__ int xstrip(int ix, int nxp, int lpml, int &tab_base, int &col)
{
    if (ix < lpml) { tab_base = 0; col = ix; return ix; }
    int r = ix - (nxp - lpml);
    if (r >= 0 && ix < nxp) { tab_base = 6; col = lpml + r; return r; }
    return -1;
}
__device__ __forceinline__ int zstrip(int iz, int nzp, int lpml, int &tab_base, int &row)
{
    if (iz < lpml) { tab_base = 0; row = iz; return iz; }
    int r = iz - (nzp - lpml);
    if (r >= 0 && iz < nzp) { tab_base = 6; row = lpml + r; return r; }
    return -1;
}

// One C-PML correction in the reference's order (lib/waves.cpp:252-253):
//   psi = B*psi + A*df ;  F -= a*(psi + C*df)      where a = dt*modulus
template <typename T, bool EXACT>
__device__ __forceinline__ T pml_correct(T F, T a, T df, T *psi, const T *tab, int lp, int base_stag, int idx)
{
    using A = Ar<T, EXACT>;
    const T tA = tab[(base_stag + PT_A) * lp + idx];
    const T tB = tab[(base_stag + PT_B) * lp + idx];
    const T tC = tab[(base_stag + PT_C) * lp + idx];
    T p = *psi;
    p = A::add(A::mul(tB, p), A::mul(tA, df));
    *psi = p;
    return A::sub(F, A::mul(a, A::add(p, A::mul(tC, df))));
}

// ------------------------------------------------------------------ kernels
template <typename T, int TX, int TZ, int RZ>
struct Geo2D {
    static constexpr int NTX = TX / 4, NTZ = TZ / RZ, NT = NTX * NTZ;
    static constexpr int W = TX + 2 * GUARD, H = TZ + 2 * GUARD;
};

// Fill the per-point coefficient row pointers of a quad (x) and block (z).
template <typename T, int RZ>
__device__ __forceinline__ void coef_rows(const CoefSet<T> &cs, bool xedge, bool zedge, bool fwx, bool fwz,
                                          int gx, int gz, int nxp, int nzp, int order,
                                          const T *cx[4], const T *cz[RZ])
{
#pragma unroll
    for (int j = 0; j < 4; j++) {
        int K = xedge ? (fwx ? kfw(gx + j, nxp, order) : kbw(gx + j, nxp, order)) : order;
        cx[j] = cs.cx + K * CROW;
    }
#pragma unroll
    for (int r = 0; r < RZ; r++) {
        int K = zedge ? (fwz ? kfw(gz + r, nzp, order) : kbw(gz + r, nzp, order)) : order;
        cz[r] = cs.cz + K * CROW;
    }
}

template <typename T>
__device__ __forceinline__ void load_coefs(CoefSet<T> &s, const CoefSet<T> &g)
{
    const T *src = reinterpret_cast<const T *>(&g);
    T *dst = reinterpret_cast<T *>(&s);
    for (int i = threadIdx.x; i < (int)(sizeof(CoefSet<T>) / sizeof(T)); i += blockDim.x) dst[i] = src[i];
}

// ---------------------------------------------------------------- acoustic 2D
// Velocity half-step: Vx += dt*Rx*Dx+P (+ x C-PML), Vz += dt*Rz*Dz+P (+ z C-PML).
template <typename T, bool EXACT, int TX, int TZ, int RZ>
__global__ void __launch_bounds__(Geo2D<T, TX, TZ, RZ>::NT)
a2d_velocity(Step2DArgs<T> a, const CoefSet<T> *coefs)
{
    using G = Geo2D<T, TX, TZ, RZ>;
    using A = Ar<T, EXACT>;
    extern __shared__ __align__(16) unsigned char smraw[];
    T *sP = reinterpret_cast<T *>(smraw);
    CoefSet<T> &cs = *reinterpret_cast<CoefSet<T> *>(sP + G::H * G::W);
    load_coefs(cs, *coefs);
    const int tx = threadIdx.x % G::NTX, tz = threadIdx.x / G::NTX;
    for (int t = blockIdx.x; t < a.ntiles; t += gridDim.x) {
        const Tile2D tl = a.tiles[t];
        const Shot2D<T> &sh = a.shots[tl.shot];
        __syncthreads();
        load_tile<T, TX, TZ, G::NT>(sP, sh.f[A2_P], sh.pitch, tl.x0, tl.z0);
        __syncthreads();
        const int xq = 4 * tx, zr = tz * RZ;
        const int gx = tl.x0 + xq, gz = tl.z0 + zr;
        const T *cx[4], *cz[RZ];
        T dfx[RZ][4], dfz[RZ][4];
        coef_rows<T, RZ>(cs, tl.flags & TILE_XEDGE, false, true, true, gx, gz, sh.nxp, sh.nzp, a.order, cx, cz);
#pragma unroll
        for (int r = 0; r < RZ; r++) dx_quad<T, EXACT, true, G::W>(sP, zr + r + GUARD, xq, cx, a.dx, dfx[r]);
        coef_rows<T, RZ>(cs, false, tl.flags & TILE_ZEDGE, true, true, gx, gz, sh.nxp, sh.nzp, a.order, cx, cz);
        dz_block<T, EXACT, true, G::W, RZ>(sP, zr, xq, cz, a.dz, dfz);
#pragma unroll
        for (int r = 0; r < RZ; r++) {
            const int iz = gz + r;
            if (iz >= sh.nzp) break;
            const long o = (long)iz * sh.pitch + gx;
            T vx[4], vz[4], rx[4], rz[4];
            ld4(sh.f[A2_VX] + o, vx); ld4(sh.f[A2_VZ] + o, vz);
            ld4(sh.m[M_RX] + o, rx); ld4(sh.m[M_RZ] + o, rz);
            int zb, zrow; const int zi = (tl.flags & TILE_ZPML) ? zstrip(iz, sh.nzp, a.lpml, zb, zrow) : -1;
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const int ix = gx + j;
                const T ax = A::mul(a.dt, rx[j]);
                vx[j] = A::add(vx[j], A::mul(ax, dfx[r][j]));
                if (tl.flags & TILE_XPML) {
                    int xb, xcol; const int xi = xstrip(ix, sh.nxp, a.lpml, xb, xcol);
                    if (xi >= 0)
                        vx[j] = pml_correct<T, EXACT>(vx[j], ax, dfx[r][j], sh.psix[0] + (long)iz * 2 * a.lpml + xcol,
                                                      a.pml, a.lpml, xb + 3, xi);
                }
                const T az = A::mul(a.dt, rz[j]);
                vz[j] = A::add(vz[j], A::mul(az, dfz[r][j]));
                if (zi >= 0 && ix < sh.nxp)
                    vz[j] = pml_correct<T, EXACT>(vz[j], az, dfz[r][j], sh.psiz[0] + (long)zrow * sh.nxp + ix,
                                                  a.pml, a.lpml, zb + 3, zi);
            }
#pragma unroll
            for (int j = 0; j < 4; j++)
                if (gx + j < sh.nxp) { sh.f[A2_VX][o + j] = vx[j]; sh.f[A2_VZ][o + j] = vz[j]; }
        }
    }
}

// Stress half-step: P += dt*L*Dx-Vx (+x C-PML), then P += dt*L*Dz-Vz (+z C-PML).
template <typename T, bool EXACT, int TX, int TZ, int RZ>
__global__ void __launch_bounds__(Geo2D<T, TX, TZ, RZ>::NT)
a2d_stress(Step2DArgs<T> a, const CoefSet<T> *coefs)
{
    using G = Geo2D<T, TX, TZ, RZ>;
    using A = Ar<T, EXACT>;
    extern __shared__ __align__(16) unsigned char smraw[];
    T *sVx = reinterpret_cast<T *>(smraw);
    T *sVz = sVx + G::H * G::W;
    CoefSet<T> &cs = *reinterpret_cast<CoefSet<T> *>(sVz + G::H * G::W);
    load_coefs(cs, *coefs);
    const int tx = threadIdx.x % G::NTX, tz = threadIdx.x / G::NTX;
    for (int t = blockIdx.x; t < a.ntiles; t += gridDim.x) {
        const Tile2D tl = a.tiles[t];
        const Shot2D<T> &sh = a.shots[tl.shot];
        __syncthreads();
        load_tile<T, TX, TZ, G::NT>(sVx, sh.f[A2_VX], sh.pitch, tl.x0, tl.z0);
        load_tile<T, TX, TZ, G::NT>(sVz, sh.f[A2_VZ], sh.pitch, tl.x0, tl.z0);
        __syncthreads();
        const int xq = 4 * tx, zr = tz * RZ;
        const int gx = tl.x0 + xq, gz = tl.z0 + zr;
        const T *cx[4], *cz[RZ];
        T dfx[RZ][4], dfz[RZ][4];
        coef_rows<T, RZ>(cs, tl.flags & TILE_XEDGE, false, false, false, gx, gz, sh.nxp, sh.nzp, a.order, cx, cz);
#pragma unroll
        for (int r = 0; r < RZ; r++) dx_quad<T, EXACT, false, G::W>(sVx, zr + r + GUARD, xq, cx, a.dx, dfx[r]);
        coef_rows<T, RZ>(cs, false, tl.flags & TILE_ZEDGE, false, false, gx, gz, sh.nxp, sh.nzp, a.order, cx, cz);
        dz_block<T, EXACT, false, G::W, RZ>(sVz, zr, xq, cz, a.dz, dfz);
#pragma unroll
        for (int r = 0; r < RZ; r++) {
            const int iz = gz + r;
            if (iz >= sh.nzp) break;
            const long o = (long)iz * sh.pitch + gx;
            T p[4], l[4];
            ld4(sh.f[A2_P] + o, p); ld4(sh.m[M_L] + o, l);
            int zb, zrow; const int zi = (tl.flags & TILE_ZPML) ? zstrip(iz, sh.nzp, a.lpml, zb, zrow) : -1;
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const int ix = gx + j;
                const T al = A::mul(a.dt, l[j]);
                p[j] = A::add(p[j], A::mul(al, dfx[r][j]));
                if (tl.flags & TILE_XPML) {
                    int xb, xcol; const int xi = xstrip(ix, sh.nxp, a.lpml, xb, xcol);
                    if (xi >= 0)
                        p[j] = pml_correct<T, EXACT>(p[j], al, dfx[r][j], sh.psix[1] + (long)iz * 2 * a.lpml + xcol,
                                                     a.pml, a.lpml, xb, xi);
                }
                p[j] = A::add(p[j], A::mul(al, dfz[r][j]));
                if (zi >= 0 && ix < sh.nxp)
                    p[j] = pml_correct<T, EXACT>(p[j], al, dfz[r][j], sh.psiz[1] + (long)zrow * sh.nxp + ix,
                                                 a.pml, a.lpml, zb, zi);
            }
#pragma unroll
            for (int j = 0; j < 4; j++)
                if (gx + j < sh.nxp) sh.f[A2_P][o + j] = p[j];
        }
    }
}

// ---------------------------------------------------------------- elastic 2D
// Velocity half-step.  Forward (lib/waves.cpp:1416-1566):
//   Vx += dt*Rx*Dx+Sxx [x stag PML psi0] ; Vx += dt*Rx*Dz-Sxz [z PML psi0]
//   Vz += dt*Rz*Dx-Sxz [x PML psi1]      ; Vz += dt*Rz*Dz+Szz [z stag PML psi1]
// Adjoint (lib/waves.cpp:1738-1913): the same with Sxx -> L2M*Sxx + L*Szz,
// Sxz -> M*Sxz, Szz -> L*Sxx + L2M*Szz.
template <typename T, bool EXACT, bool ADJ, int TX, int TZ, int RZ>
__global__ void __launch_bounds__(Geo2D<T, TX, TZ, RZ>::NT)
e2d_velocity(Step2DArgs<T> a, const CoefSet<T> *coefs)
{
    using G = Geo2D<T, TX, TZ, RZ>;
    using A = Ar<T, EXACT>;
    extern __shared__ __align__(16) unsigned char smraw[];
    T *sXX = reinterpret_cast<T *>(smraw);
    T *sZZ = sXX + G::H * G::W;
    T *sXZ = sZZ + G::H * G::W;
    CoefSet<T> &cs = *reinterpret_cast<CoefSet<T> *>(sXZ + G::H * G::W);
    load_coefs(cs, *coefs);
    const int tx = threadIdx.x % G::NTX, tz = threadIdx.x / G::NTX;
    for (int t = blockIdx.x; t < a.ntiles; t += gridDim.x) {
        const Tile2D tl = a.tiles[t];
        const Shot2D<T> &sh = a.shots[tl.shot];
        __syncthreads();
        if (!ADJ) {
            load_tile<T, TX, TZ, G::NT>(sXX, sh.f[E2_SXX], sh.pitch, tl.x0, tl.z0);
            load_tile<T, TX, TZ, G::NT>(sZZ, sh.f[E2_SZZ], sh.pitch, tl.x0, tl.z0);
            load_tile<T, TX, TZ, G::NT>(sXZ, sh.f[E2_SXZ], sh.pitch, tl.x0, tl.z0);
        } else {
            load_tile_comb<T, EXACT, TX, TZ, G::NT>(sXX, sh.m[M_L2M], sh.f[E2_SXX], sh.m[M_L], sh.f[E2_SZZ], sh.pitch, tl.x0, tl.z0);
            load_tile_comb<T, EXACT, TX, TZ, G::NT>(sZZ, sh.m[M_L], sh.f[E2_SXX], sh.m[M_L2M], sh.f[E2_SZZ], sh.pitch, tl.x0, tl.z0);
            load_tile_comb<T, EXACT, TX, TZ, G::NT>(sXZ, sh.m[M_M], sh.f[E2_SXZ], nullptr, nullptr, sh.pitch, tl.x0, tl.z0);
        }
        __syncthreads();
        const int xq = 4 * tx, zr = tz * RZ;
        const int gx = tl.x0 + xq, gz = tl.z0 + zr;
        const bool xe = tl.flags & TILE_XEDGE, ze = tl.flags & TILE_ZEDGE;
        const T *cx[4], *cz[RZ];
        T d1[RZ][4], d2[RZ][4];
        // Vx: Dx+ Sxx and Dz- Sxz
        coef_rows<T, RZ>(cs, xe, ze, true, false, gx, gz, sh.nxp, sh.nzp, a.order, cx, cz);
#pragma unroll
        for (int r = 0; r < RZ; r++) dx_quad<T, EXACT, true, G::W>(sXX, zr + r + GUARD, xq, cx, a.dx, d1[r]);
        dz_block<T, EXACT, false, G::W, RZ>(sXZ, zr, xq, cz, a.dz, d2);
#pragma unroll
        for (int r = 0; r < RZ; r++) {
            const int iz = gz + r;
            if (iz >= sh.nzp) break;
            const long o = (long)iz * sh.pitch + gx;
            T v[4], m[4];
            ld4(sh.f[E2_VX] + o, v); ld4(sh.m[M_RX] + o, m);
            int zb, zrow; const int zi = (tl.flags & TILE_ZPML) ? zstrip(iz, sh.nzp, a.lpml, zb, zrow) : -1;
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const int ix = gx + j;
                const T am = A::mul(a.dt, m[j]);
                v[j] = A::add(v[j], A::mul(am, d1[r][j]));
                if (tl.flags & TILE_XPML) {
                    int xb, xcol; const int xi = xstrip(ix, sh.nxp, a.lpml, xb, xcol);
                    if (xi >= 0)
                        v[j] = pml_correct<T, EXACT>(v[j], am, d1[r][j], sh.psix[0] + (long)iz * 2 * a.lpml + xcol,
                                                     a.pml, a.lpml, xb + 3, xi);
                }
                v[j] = A::add(v[j], A::mul(am, d2[r][j]));
                if (zi >= 0 && ix < sh.nxp)
                    v[j] = pml_correct<T, EXACT>(v[j], am, d2[r][j], sh.psiz[0] + (long)zrow * sh.nxp + ix,
                                                 a.pml, a.lpml, zb, zi);
            }
#pragma unroll
            for (int j = 0; j < 4; j++)
                if (gx + j < sh.nxp) sh.f[E2_VX][o + j] = v[j];
        }
        // Vz: Dx- Sxz and Dz+ Szz
        coef_rows<T, RZ>(cs, xe, ze, false, true, gx, gz, sh.nxp, sh.nzp, a.order, cx, cz);
#pragma unroll
        for (int r = 0; r < RZ; r++) dx_quad<T, EXACT, false, G::W>(sXZ, zr + r + GUARD, xq, cx, a.dx, d1[r]);
        dz_block<T, EXACT, true, G::W, RZ>(sZZ, zr, xq, cz, a.dz, d2);
#pragma unroll
        for (int r = 0; r < RZ; r++) {
            const int iz = gz + r;
            if (iz >= sh.nzp) break;
            const long o = (long)iz * sh.pitch + gx;
            T v[4], m[4];
            ld4(sh.f[E2_VZ] + o, v); ld4(sh.m[M_RZ] + o, m);
            int zb, zrow; const int zi = (tl.flags & TILE_ZPML) ? zstrip(iz, sh.nzp, a.lpml, zb, zrow) : -1;
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const int ix = gx + j;
                const T am = A::mul(a.dt, m[j]);
                v[j] = A::add(v[j], A::mul(am, d1[r][j]));
                if (tl.flags & TILE_XPML) {
                    int xb, xcol; const int xi = xstrip(ix, sh.nxp, a.lpml, xb, xcol);
                    if (xi >= 0)
                        v[j] = pml_correct<T, EXACT>(v[j], am, d1[r][j], sh.psix[1] + (long)iz * 2 * a.lpml + xcol,
                                                     a.pml, a.lpml, xb, xi);
                }
                v[j] = A::add(v[j], A::mul(am, d2[r][j]));
                if (zi >= 0 && ix < sh.nxp)
                    v[j] = pml_correct<T, EXACT>(v[j], am, d2[r][j], sh.psiz[1] + (long)zrow * sh.nxp + ix,
                                                 a.pml, a.lpml, zb + 3, zi);
            }
#pragma unroll
            for (int j = 0; j < 4; j++)
                if (gx + j < sh.nxp) sh.f[E2_VZ][o + j] = v[j];
        }
    }
}

// Stress half-step.  Forward (lib/waves.cpp:1571-1735):
//   d = Dx-Vx: Sxx += dt*L2M*d, Szz += dt*L*d  [x PML psi2] ;
//   d = Dz-Vz: Sxx += dt*L*d,   Szz += dt*L2M*d [z PML psi2] ; free surface Szz=0 ;
//   Sxz += dt*M*Dx+Vz [x stag psi3] ; Sxz += dt*M*Dz+Vx [z stag psi3]
// Adjoint (lib/waves.cpp:1916-2080): Sxx += dt*Dx-Vx, Szz += dt*Dz-Vz, Sxz as
// above without the modulus.
template <typename T, bool EXACT, bool ADJ, int TX, int TZ, int RZ>
__global__ void __launch_bounds__(Geo2D<T, TX, TZ, RZ>::NT)
e2d_stress(Step2DArgs<T> a, const CoefSet<T> *coefs)
{
    using G = Geo2D<T, TX, TZ, RZ>;
    using A = Ar<T, EXACT>;
    extern __shared__ __align__(16) unsigned char smraw[];
    T *sVx = reinterpret_cast<T *>(smraw);
    T *sVz = sVx + G::H * G::W;
    CoefSet<T> &cs = *reinterpret_cast<CoefSet<T> *>(sVz + G::H * G::W);
    load_coefs(cs, *coefs);
    const int tx = threadIdx.x % G::NTX, tz = threadIdx.x / G::NTX;
    for (int t = blockIdx.x; t < a.ntiles; t += gridDim.x) {
        const Tile2D tl = a.tiles[t];
        const Shot2D<T> &sh = a.shots[tl.shot];
        __syncthreads();
        load_tile<T, TX, TZ, G::NT>(sVx, sh.f[E2_VX], sh.pitch, tl.x0, tl.z0);
        load_tile<T, TX, TZ, G::NT>(sVz, sh.f[E2_VZ], sh.pitch, tl.x0, tl.z0);
        __syncthreads();
        const int xq = 4 * tx, zr = tz * RZ;
        const int gx = tl.x0 + xq, gz = tl.z0 + zr;
        const bool xe = tl.flags & TILE_XEDGE, ze = tl.flags & TILE_ZEDGE;
        const T *cx[4], *cz[RZ];
        T d1[RZ][4], d2[RZ][4];
        // normal stresses: Dx- Vx, Dz- Vz
        coef_rows<T, RZ>(cs, xe, ze, false, false, gx, gz, sh.nxp, sh.nzp, a.order, cx, cz);
#pragma unroll
        for (int r = 0; r < RZ; r++) dx_quad<T, EXACT, false, G::W>(sVx, zr + r + GUARD, xq, cx, a.dx, d1[r]);
        dz_block<T, EXACT, false, G::W, RZ>(sVz, zr, xq, cz, a.dz, d2);
#pragma unroll
        for (int r = 0; r < RZ; r++) {
            const int iz = gz + r;
            if (iz >= sh.nzp) break;
            const long o = (long)iz * sh.pitch + gx;
            T sxx[4], szz[4], l[4], l2m[4];
            ld4(sh.f[E2_SXX] + o, sxx); ld4(sh.f[E2_SZZ] + o, szz);
            if (!ADJ) { ld4(sh.m[M_L] + o, l); ld4(sh.m[M_L2M] + o, l2m); }
            int zb, zrow; const int zi = (tl.flags & TILE_ZPML) ? zstrip(iz, sh.nzp, a.lpml, zb, zrow) : -1;
            const bool fsrow = sh.fs && iz == a.lpml;
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const int ix = gx + j;
                int xb = 0, xcol = 0;
                const int xi = (tl.flags & TILE_XPML) ? xstrip(ix, sh.nxp, a.lpml, xb, xcol) : -1;
                if (!ADJ) {
                    const T a2 = A::mul(a.dt, l2m[j]), a1 = A::mul(a.dt, l[j]);
                    sxx[j] = A::add(sxx[j], A::mul(a2, d1[r][j]));
                    szz[j] = A::add(szz[j], A::mul(a1, d1[r][j]));
                    if (xi >= 0) {
                        // one psi update shared by both corrections (lib/waves.cpp:1625-1627)
                        T *ps = sh.psix[2] + (long)iz * 2 * a.lpml + xcol;
                        const T tA = a.pml[(xb + PT_A) * a.lpml + xi], tB = a.pml[(xb + PT_B) * a.lpml + xi],
                                tC = a.pml[(xb + PT_C) * a.lpml + xi];
                        T p = A::add(A::mul(tB, *ps), A::mul(tA, d1[r][j]));
                        *ps = p;
                        const T q = A::add(p, A::mul(tC, d1[r][j]));
                        sxx[j] = A::sub(sxx[j], A::mul(a2, q));
                        szz[j] = A::sub(szz[j], A::mul(a1, q));
                    }
                    sxx[j] = A::add(sxx[j], A::mul(a1, d2[r][j]));
                    szz[j] = A::add(szz[j], A::mul(a2, d2[r][j]));
                    if (zi >= 0 && ix < sh.nxp) {
                        T *ps = sh.psiz[2] + (long)zrow * sh.nxp + ix;
                        const T tA = a.pml[(zb + PT_A) * a.lpml + zi], tB = a.pml[(zb + PT_B) * a.lpml + zi],
                                tC = a.pml[(zb + PT_C) * a.lpml + zi];
                        T p = A::add(A::mul(tB, *ps), A::mul(tA, d2[r][j]));
                        *ps = p;
                        const T q = A::add(p, A::mul(tC, d2[r][j]));
                        sxx[j] = A::sub(sxx[j], A::mul(a1, q));
                        szz[j] = A::sub(szz[j], A::mul(a2, q));
                    }
                } else {
                    sxx[j] = A::add(sxx[j], A::mul(a.dt, d1[r][j]));
                    if (xi >= 0)
                        sxx[j] = pml_correct<T, EXACT>(sxx[j], a.dt, d1[r][j], sh.psix[2] + (long)iz * 2 * a.lpml + xcol,
                                                       a.pml, a.lpml, xb, xi);
                    szz[j] = A::add(szz[j], A::mul(a.dt, d2[r][j]));
                    if (zi >= 0 && ix < sh.nxp)
                        szz[j] = pml_correct<T, EXACT>(szz[j], a.dt, d2[r][j], sh.psiz[2] + (long)zrow * sh.nxp + ix,
                                                       a.pml, a.lpml, zb, zi);
                }
                if (fsrow) szz[j] = T(0);
            }
#pragma unroll
            for (int j = 0; j < 4; j++)
                if (gx + j < sh.nxp) { sh.f[E2_SXX][o + j] = sxx[j]; sh.f[E2_SZZ][o + j] = szz[j]; }
        }
        // shear stress: Dx+ Vz, Dz+ Vx
        coef_rows<T, RZ>(cs, xe, ze, true, true, gx, gz, sh.nxp, sh.nzp, a.order, cx, cz);
#pragma unroll
        for (int r = 0; r < RZ; r++) dx_quad<T, EXACT, true, G::W>(sVz, zr + r + GUARD, xq, cx, a.dx, d1[r]);
        dz_block<T, EXACT, true, G::W, RZ>(sVx, zr, xq, cz, a.dz, d2);
#pragma unroll
        for (int r = 0; r < RZ; r++) {
            const int iz = gz + r;
            if (iz >= sh.nzp) break;
            const long o = (long)iz * sh.pitch + gx;
            T sxz[4], mm[4];
            ld4(sh.f[E2_SXZ] + o, sxz);
            if (!ADJ) ld4(sh.m[M_M] + o, mm);
            int zb, zrow; const int zi = (tl.flags & TILE_ZPML) ? zstrip(iz, sh.nzp, a.lpml, zb, zrow) : -1;
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const int ix = gx + j;
                const T am = ADJ ? a.dt : A::mul(a.dt, mm[j]);
                sxz[j] = A::add(sxz[j], A::mul(am, d1[r][j]));
                if (tl.flags & TILE_XPML) {
                    int xb, xcol; const int xi = xstrip(ix, sh.nxp, a.lpml, xb, xcol);
                    if (xi >= 0)
                        sxz[j] = pml_correct<T, EXACT>(sxz[j], am, d1[r][j], sh.psix[3] + (long)iz * 2 * a.lpml + xcol,
                                                       a.pml, a.lpml, xb + 3, xi);
                }
                sxz[j] = A::add(sxz[j], A::mul(am, d2[r][j]));
                if (zi >= 0 && ix < sh.nxp)
                    sxz[j] = pml_correct<T, EXACT>(sxz[j], am, d2[r][j], sh.psiz[3] + (long)zrow * sh.nxp + ix,
                                                   a.pml, a.lpml, zb + 3, zi);
            }
#pragma unroll
            for (int j = 0; j < 4; j++)
                if (gx + j < sh.nxp) sh.f[E2_SXZ][o + j] = sxz[j];
        }
    }
}

// ---------------------------------------------------------------- sources and receivers
// One CTA per shot.  Injection first (lib/waves.cpp:407-497, 2085-2174), then,
// after a CTA barrier, recording (lib/waves.cpp:500-595, 2178-2288) of the same step.
template <typename T, bool EXACT>
__global__ void inject_record_2d(const Shot2D<T> *shots, const InjRec<T> *plans, T dt, int it_base,
                                 const int *it_dev)
{
    using A = Ar<T, EXACT>;
    const Shot2D<T> &sh = shots[blockIdx.x];
    const InjRec<T> &pl = plans[blockIdx.x];
    const int it = it_base + (it_dev ? *it_dev : 0);
    if (pl.kind_inj != INJ_NONE) {
        for (int q = threadIdx.x; q < pl.ninj; q += blockDim.x) {
            const int p = pl.inj_pt[q];
            switch (pl.kind_inj) {
            case INJ_A2_P: case INJ_A2_VX: case INJ_A2_VZ:
            case INJ_E2_VX: case INJ_E2_VZ: {
                T *F; const T *Mod;
                if (pl.kind_inj == INJ_A2_P) { F = sh.f[A2_P]; Mod = sh.m[M_L]; }
                else if (pl.kind_inj == INJ_A2_VX) { F = sh.f[A2_VX]; Mod = sh.m[M_RX]; }
                else if (pl.kind_inj == INJ_A2_VZ) { F = sh.f[A2_VZ]; Mod = sh.m[M_RZ]; }
                else if (pl.kind_inj == INJ_E2_VX) { F = sh.f[E2_VX]; Mod = sh.m[M_RX]; }
                else { F = sh.f[E2_VZ]; Mod = sh.m[M_RZ]; }
                T v = F[p];
                const T dm = A::mul(dt, Mod[p]);
                for (int c = pl.inj_start[q]; c < pl.inj_start[q + 1]; c++) {
                    const T w = pl.wav[(long)pl.inj_trace[c] * pl.nt + it];
                    v = A::add(v, A::mul(A::mul(A::mul(dm, w), pl.inj_wx[c]), pl.inj_wz[c]));
                }
                F[p] = v;
                break;
            }
            case INJ_E2_P: {
                T sxx = sh.f[E2_SXX][p], szz = sh.f[E2_SZZ][p];
                for (int c = pl.inj_start[q]; c < pl.inj_start[q + 1]; c++) {
                    const T w = pl.wav[(long)pl.inj_trace[c] * pl.nt + it];
                    const T s = A::mul(A::mul(A::mul(dt, w), pl.inj_wx[c]), pl.inj_wz[c]);
                    sxx = A::sub(sxx, s);
                    szz = A::sub(szz, s);
                }
                sh.f[E2_SXX][p] = sxx; sh.f[E2_SZZ][p] = szz;
                break;
            }
            }
        }
    }
    if (pl.kind_rec == REC_NONE) return;
    __syncthreads();
    for (int tr = threadIdx.x; tr < pl.nrec; tr += blockDim.x) {
        const int p = pl.rec_pt[tr];
        if (p < 0) continue;
        const T wx0 = pl.rec_w[4 * tr], wx1 = pl.rec_w[4 * tr + 1];
        const T wz0 = pl.rec_w[4 * tr + 2], wz1 = pl.rec_w[4 * tr + 3];
        const int off[4] = {0, 1, sh.pitch, sh.pitch + 1};
        const T wx[4] = {wx0, wx1, wx0, wx1}, wz[4] = {wz0, wz0, wz1, wz1};
        T *out = pl.rec_out + (long)tr * pl.nt + it;
        if (pl.kind_rec == REC_E2_P) {
            // (1./2.)*xtri*ytri*F/factor is evaluated in double by the reference and
            // added to the T-typed trace sample (lib/waves.cpp:2240-2241)
            const double fac = pl.rec_factor ? (double)pl.rec_factor[tr] : 1.0;
            T acc = *out;
#pragma unroll
            for (int c = 0; c < 4; c++) {
                const double w = __dmul_rn(__dmul_rn(0.5, (double)wx[c]), (double)wz[c]);
                acc = (T)__dadd_rn((double)acc, __ddiv_rn(__dmul_rn(w, (double)sh.f[E2_SXX][p + off[c]]), fac));
                acc = (T)__dadd_rn((double)acc, __ddiv_rn(__dmul_rn(w, (double)sh.f[E2_SZZ][p + off[c]]), fac));
            }
            *out = acc;
        } else {
            const T *F;
            switch (pl.kind_rec) {
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

static __global__ void advance_counter(int *it_dev, int by)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) *it_dev += by;
}

// ---------------------------------------------------------------- launchers
template <typename T, bool EXACT, int TX, int TZ, int RZ>
cudaError_t launch_2d_cfg(int physics, int half, bool adj, const Step2DArgs<T> &a, const CoefSet<T> *coefs,
                                 int grid, cudaStream_t st)
{
    using G = Geo2D<T, TX, TZ, RZ>;
    const size_t tile = sizeof(T) * G::H * G::W;
    const size_t cb = sizeof(CoefSet<T>);
    if (physics == PHYS_A2D) {
        if (half == 0) {
            auto k = a2d_velocity<T, EXACT, TX, TZ, RZ>;
            const size_t smem = tile + cb;
            static const cudaError_t attr = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (attr != cudaSuccess) return attr;
            k<<<grid, G::NT, smem, st>>>(a, coefs);
        } else {
            auto k = a2d_stress<T, EXACT, TX, TZ, RZ>;
            const size_t smem = 2 * tile + cb;
            static const cudaError_t attr = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (attr != cudaSuccess) return attr;
            k<<<grid, G::NT, smem, st>>>(a, coefs);
        }
    } else {
        if (half == 0) {
            const size_t smem = 3 * tile + cb;
            auto k = adj ? e2d_velocity<T, EXACT, true, TX, TZ, RZ> : e2d_velocity<T, EXACT, false, TX, TZ, RZ>;
            static const cudaError_t a0 = cudaFuncSetAttribute(e2d_velocity<T, EXACT, false, TX, TZ, RZ>,
                                                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            static const cudaError_t a1 = cudaFuncSetAttribute(e2d_velocity<T, EXACT, true, TX, TZ, RZ>,
                                                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (a0 != cudaSuccess) return a0;
            if (a1 != cudaSuccess) return a1;
            k<<<grid, G::NT, smem, st>>>(a, coefs);
        } else {
            const size_t smem = 2 * tile + cb;
            auto k = adj ? e2d_stress<T, EXACT, true, TX, TZ, RZ> : e2d_stress<T, EXACT, false, TX, TZ, RZ>;
            static const cudaError_t a0 = cudaFuncSetAttribute(e2d_stress<T, EXACT, false, TX, TZ, RZ>,
                                                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            static const cudaError_t a1 = cudaFuncSetAttribute(e2d_stress<T, EXACT, true, TX, TZ, RZ>,
                                                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (a0 != cudaSuccess) return a0;
            if (a1 != cudaSuccess) return a1;
            k<<<grid, G::NT, smem, st>>>(a, coefs);
        }
    }
    return cudaGetLastError();
}

template <typename T, bool EXACT>
cudaError_t launch_2d_t(int cfg, int physics, int half, bool adj, const void *args, const void *coefs,
                               int grid, cudaStream_t st)
{
    const Step2DArgs<T> &a = *static_cast<const Step2DArgs<T> *>(args);
    const CoefSet<T> *c = static_cast<const CoefSet<T> *>(coefs);
    switch (cfg) {
    case TILECFG_64x32: return launch_2d_cfg<T, EXACT, 64, 32, 4>(physics, half, adj, a, c, grid, st);
    case TILECFG_64x64: return launch_2d_cfg<T, EXACT, 64, 64, 4>(physics, half, adj, a, c, grid, st);
    case TILECFG_32x32: return launch_2d_cfg<T, EXACT, 32, 32, 4>(physics, half, adj, a, c, grid, st);
    case TILECFG_128x32: return launch_2d_cfg<T, EXACT, 128, 32, 4>(physics, half, adj, a, c, grid, st);
    case TILECFG_32x16: return launch_2d_cfg<T, EXACT, 32, 16, 2>(physics, half, adj, a, c, grid, st);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace rsgpu
