// Fused 2D time step for sm_100a: velocity half-step, stress half-step, source
// injection and receiver recording in ONE launch, z-marching.
//
// The reference runs forwardstepVelocity, forwardstepStress, insertSource and
// recordData as separate passes over the grid (lib/waves.cpp:217-595 acoustic,
// 1416-1735 and 2085-2288 elastic).  Here one CTA owns a strip of TX columns of
// one shot and a range of rows [z0, z1), and walks down z in slabs of 8 rows:
//
//   stress ring   old stresses (elastic Sxx, Szz, Sxz; acoustic P) of the strip
//                 plus a 16-column halo on each side, 4 slabs deep, filled by
//                 TMA (cp.async.bulk.tensor, mbarrier completion with a bounded
//                 wait) two slabs ahead of use;
//   velocity      the new velocities of slab i are computed on the strip plus an
//                 8-column halo (the halo is recomputed by both neighbours, so no
//                 CTA waits for another), kept in a 3-slab shared ring and written
//                 to HBM for the owned columns;
//   stress        slab i-1's new stresses follow from the velocity ring (x
//                 derivatives on a row, z derivatives streamed down the ring).
//
// HBM traffic per point and step is then the algorithmic minimum: each field is
// read once and written once, each parameter read once (elastic 60 B, acoustic
// 36 B in FP32) plus the C-PML memory strips; halo re-reads are served by L2.
// Because neighbouring CTAs read each other's columns while the step runs, the
// wavefields and the velocity C-PML memory are double-buffered: step n reads
// copy n&1 and writes the other (Shot2D::f / fb).  The stresses' own C-PML
// memory is only touched by the point's owner and stays in place.
//
// Work items (shot, x0, z0, z1) are handed out through an atomic counter so that
// CTAs finishing early take more; the items are ordered by z band so that the
// CTAs running at one time cover neighbouring strips at the same depth, and
// their halo reads hit L2.
//
// Recording of step n-1 (its state is the copy this launch reads) is done at the
// start of launch n; the last step of a run is recorded by a small record-only
// launch.  Injection of step n is applied by the owner of the target point to the
// copy it writes, after its stores, in the reference's order (sets in order,
// contributions in trace / z-corner / x-corner order).
//
// Arithmetic per point is the per-tile kernels' (fd2d_kernels.cuh): MODE_IEEE
// reproduces the reference's float operations bit for bit, MODE_FAST uses FMA
// and coefficients pre-divided by the spacing.
//
// Measured on B200 (16-shot 801 x 401 elastic batch): DRAM traffic is at the
// algorithmic 60 B per point, but the step issues about as many instructions per
// point as the per-tile kernels (~440) with two CTAs of four warps per SM (the
// rings take 80 KB of shared memory, the block state ~240 registers per thread),
// so it is issue-bound at 15-18 % issue efficiency and runs slower than the
// per-tile kernels; it is selected by launch_mode 3 only.
#pragma once
#include "fd2d_kernels.cuh"

namespace rsgpu {

constexpr int ZM_RB = 8;       // rows per slab
constexpr int ZM_SLOTS = 4;    // stress-ring slabs: i-1, i, i+1 in use, i+2 in flight
constexpr int ZM_VSLOTS = 3;   // velocity-ring slabs: i-2, i-1, i
constexpr int ZM_NT = 128;     // threads: 4 warps = 2 row halves x 64 column pairs
constexpr int ZM_TX = 112;     // owned columns of a strip (velocity: 128 with the halo)

template <typename T, int PHYS, int TX>
struct ZmGeo {
    static constexpr int VW = TX + 16;          // velocity columns (strip + 8-column halo each side)
    static constexpr int SW = TX + 32;          // stress-ring columns (strip + 16 each side)
    static constexpr int NRF = PHYS == PHYS_E2D ? 3 : 1;
    static constexpr int NPV = VW / 2, NPS = TX / 2;
    static constexpr int SLAB = ZM_RB * SW;     // elements of one field's slab in the stress ring
    static constexpr int VSLAB = ZM_RB * VW;
    static constexpr size_t ring_bytes = (size_t)ZM_SLOTS * NRF * SLAB * sizeof(T);
    static constexpr size_t vring_bytes = (size_t)ZM_VSLOTS * 2 * VSLAB * sizeof(T);
    static constexpr size_t coef_off = ring_bytes + vring_bytes;
    static constexpr size_t bar_off = (coef_off + sizeof(CoefSet<T>) + 15) / 16 * 16;
    static constexpr size_t bytes = bar_off + ZM_SLOTS * sizeof(uint64_t) + 16;
    static_assert(TX % 16 == 0 && NPV <= 64, "strip width: multiple of 16, at most 112 columns");
    static_assert(SW <= 256, "TMA box width");
    static_assert((SLAB * sizeof(T)) % 128 == 0 && (VSLAB * sizeof(T)) % 128 == 0, "slab alignment");
};

// ------------------------------------------------------------------ pair derivatives
// x-derivatives of the two outputs at columns c, c+1 of a shared row; `row` points
// at column c-8 (16-byte aligned pairs).  FW: f[i+k+1]-f[i-k]; BW: f[i+k]-f[i-k-1]
// (lib/der.cpp:183-188, 378-383), summed in the reference's order.
template <typename T, int MODE, bool FW>
__device__ __forceinline__ void dx_pair(const T *row, const T (&cu)[NCOEF], T d, T r, T (&out)[2])
{
    using A = Ar<T, MODE>;
    using P = typename Pair<T>::t;
    T v[18];
#pragma unroll
    for (int q = 0; q < 9; q++) {
        const P pr = *reinterpret_cast<const P *>(row + 2 * q);
        v[2 * q] = pr.x;
        v[2 * q + 1] = pr.y;
    }
#pragma unroll
    for (int j = 0; j < 2; j++) {
        T acc = T(0);
#pragma unroll
        for (int k = 0; k < NCOEF; k++) {
            const T dl = FW ? A::sub(v[j + 9 + k], v[j + 8 - k]) : A::sub(v[j + 8 + k], v[j + 7 - k]);
            acc = (k == 0) ? A::mul(dl, cu[k]) : A::mad(acc, dl, cu[k]);
        }
        out[j] = (MODE == MODE_FAST) ? acc : A::div(acc, d, r);
    }
}

// Row W (0..23) of the 24-row window formed by three ring slabs (slab i-1 rows
// 0..7, slab i rows 8..15, slab i+1 rows 16..23).  W is a compile-time constant
// at every call (unrolled loops), so the selection folds.
template <int RS, typename T>
__device__ __forceinline__ const T *ring_row(const T *s0, const T *s1, const T *s2, int W)
{
    return (W < 8 ? s0 : W < 16 ? s1 : s2) + (W & 7) * RS;
}

// z-derivatives of the thread's column pair for the 4 rows 4H..4H+3 of slab i,
// from the window rows 4H..4H+19.  s0/s1/s2 point at the pair in row 0 of slabs
// i-1, i, i+1.  FAST float: each window row is read once and scattered into the
// four accumulators with paired FMAs (c*w+ and -c*w- as separate terms); other
// modes: the reference's order with separately rounded operations.
template <typename T, int MODE, bool FW, int H, int RS>
__device__ __forceinline__ void dz_ring(const T *s0, const T *s1, const T *s2, const T (&cu)[NCOEF], T d, T r,
                                        T (&out)[4][2])
{
    using P = typename Pair<T>::t;
    if constexpr (MODE == MODE_FAST && std::is_same<T, float>::value) {
        float2 acc[4], cp[NCOEF], cn[NCOEF];
#pragma unroll
        for (int k = 0; k < NCOEF; k++) { cp[k] = make_float2(cu[k], cu[k]); cn[k] = make_float2(-cu[k], -cu[k]); }
#pragma unroll
        for (int rr = 0; rr < 4; rr++) acc[rr] = make_float2(0.f, 0.f);
#pragma unroll
        for (int q = 0; q < 20; q++) {
            const float2 w = *reinterpret_cast<const float2 *>(ring_row<RS>(s0, s1, s2, 4 * H + q));
#pragma unroll
            for (int rr = 0; rr < 4; rr++) {
                const int kp = FW ? q - rr - 9 : q - rr - 8;
                const int km = FW ? rr + 8 - q : rr + 7 - q;
                if (kp >= 0 && kp < NCOEF) acc[rr] = __ffma2_rn(w, cp[kp], acc[rr]);
                if (km >= 0 && km < NCOEF) acc[rr] = __ffma2_rn(w, cn[km], acc[rr]);
            }
        }
#pragma unroll
        for (int rr = 0; rr < 4; rr++) { out[rr][0] = acc[rr].x; out[rr][1] = acc[rr].y; }
    } else {
        using A2 = Ar2<T, MODE>;
        P w[20];
#pragma unroll
        for (int q = 0; q < 20; q++) w[q] = *reinterpret_cast<const P *>(ring_row<RS>(s0, s1, s2, 4 * H + q));
        const P d2 = A2::mk(d), r2 = A2::mk(r);
#pragma unroll
        for (int rr = 0; rr < 4; rr++) {
            P acc;
#pragma unroll
            for (int k = 0; k < NCOEF; k++) {
                const P dl = FW ? A2::sub(w[rr + 9 + k], w[rr + 8 - k]) : A2::sub(w[rr + 8 + k], w[rr + 7 - k]);
                const P c = A2::mk(cu[k]);
                acc = (k == 0) ? A2::mul(dl, c) : A2::acc(acc, dl, c);
            }
            const P o = (MODE == MODE_FAST) ? acc : A2::div(acc, d2, r2);
            out[rr][0] = o.x;
            out[rr][1] = o.y;
        }
    }
}

// Reduced-order z stencil of K pairs at window row Wc (reference rule near the
// array ends), reading through the three ring slabs.
template <typename T, int MODE>
__device__ __noinline__ T stencil_k_ring(const T *s0, const T *s1, const T *s2, int rs, int Wc, int K, const T *c,
                                         bool fw, T d, T r)
{
    using A = Ar<T, MODE>;
    auto at = [&](int W) -> T { return (W < 8 ? s0 : W < 16 ? s1 : s2)[(W & 7) * rs]; };
    if (K <= 0) return T(0);
    T acc = A::mul(fw ? A::sub(at(Wc + 1), at(Wc)) : A::sub(at(Wc), at(Wc - 1)), c[0]);
    for (int k = 1; k < K; k++) {
        const T dl = fw ? A::sub(at(Wc + k + 1), at(Wc - k)) : A::sub(at(Wc + k), at(Wc - k - 1));
        acc = A::mad(acc, dl, c[k]);
    }
    return (MODE == MODE_FAST) ? acc : A::div(acc, d, r);
}

// Coefficient pairs at index i of an axis of n cells; `order` (no fix-up) outside the axis.
__device__ __forceinline__ int kfw_in(int i, int n, int order) { return (i < 0 || i >= n) ? order : kfw(i, n, order); }
__device__ __forceinline__ int kbw_in(int i, int n, int order) { return (i < 0 || i >= n) ? order : kbw(i, n, order); }

// z-derivative dispatch on the thread's row half (uniform per warp).
template <typename T, int MODE, bool FW, int RS>
__device__ __forceinline__ void dz_half(int h, const T *s0, const T *s1, const T *s2, const T (&cu)[NCOEF], T d, T r,
                                        T (&out)[4][2])
{
    if (h == 0) dz_ring<T, MODE, FW, 0, RS>(s0, s1, s2, cu, d, r, out);
    else dz_ring<T, MODE, FW, 1, RS>(s0, s1, s2, cu, d, r, out);
}

// ------------------------------------------------------------------ C-PML with double-buffered memory
// psi = B*psi + A*df ; F -= a*(psi + C*df)   (lib/waves.cpp:252-253); the new psi
// is stored only by the point's owner.
template <typename T, int MODE>
__device__ __forceinline__ T pml_pp(T F, T a, T df, const T *psi_in, T *psi_out, bool own, const T *tab, int lp,
                                    int base, int idx)
{
    using A = Ar<T, MODE>;
    const T tA = __ldg(tab + (base + PT_A) * lp + idx);
    const T tB = __ldg(tab + (base + PT_B) * lp + idx);
    const T tC = __ldg(tab + (base + PT_C) * lp + idx);
    const T p = A::mad(A::mul(tB, *psi_in), tA, df);
    if (own) *psi_out = p;
    return A::msub(F, a, A::mad(p, tC, df));
}

// x-strip / z-strip coordinates of point (ix, iz); -1 outside the strips or the grid.
__device__ __forceinline__ int xstrip_in(int ix, int iz, int nxp, int nzp, int lp, int &tb, int &col)
{
    if (iz < 0 || iz >= nzp || ix < 0) return -1;
    return xstrip(ix, nxp, lp, tb, col);
}
__device__ __forceinline__ int zstrip_in(int ix, int iz, int nxp, int nzp, int lp, int &tb, int &row)
{
    if (ix < 0 || ix >= nxp || iz < 0) return -1;
    return zstrip(iz, nzp, lp, tb, row);
}

// Fast update of one field at a 4 x 2 block that touches no C-PML strip, no
// reduced-order stencil and no free-surface row (lib/waves.cpp:245-307 without the
// strip corrections): F += a*d1 ; F += a*d2 with a = dt*modulus.
template <typename T, int MODE>
__device__ __forceinline__ void fast_update(T (&F)[4][2], const T (&Mo)[4][2], const T (&d1)[4][2],
                                            const T (&d2)[4][2], bool has1, bool has2, T dt)
{
    using A = Ar<T, MODE>;
#pragma unroll
    for (int rr = 0; rr < 4; rr++)
#pragma unroll
        for (int j = 0; j < 2; j++) {
            const T am = A::mul(dt, Mo[rr][j]);
            if (has1) F[rr][j] = A::mad(F[rr][j], am, d1[rr][j]);
            if (has2) F[rr][j] = A::mad(F[rr][j], am, d2[rr][j]);
        }
}

// Do the index ranges [a, b] and [lo, hi) meet?
__device__ __forceinline__ bool meets(int a, int b, int lo, int hi) { return a < hi && b >= lo; }

// Does the block of columns [gx, gx+1] x rows [gz0, gz0+3] need the general
// per-point path: a reduced-order stencil near an array end, a C-PML strip point
// or (stress) the free-surface row?
__device__ __forceinline__ bool block_special(int gx, int gz0, int nxp, int nzp, int order, int lp, bool fsrow_check,
                                              bool fs)
{
    const int gx1 = gx + 1, gz1 = gz0 + 3;
    const bool in_x = meets(gx, gx1, 0, nxp), in_z = meets(gz0, gz1, 0, nzp);
    const bool edge = (in_z && (meets(gx, gx1, 0, order) || meets(gx, gx1, nxp - order - 1, nxp))) ||
                      (in_x && (meets(gz0, gz1, 0, order) || meets(gz0, gz1, nzp - order - 1, nzp)));
    const bool pml = (in_z && (meets(gx, gx1, 0, lp) || meets(gx, gx1, nxp - lp, nxp))) ||
                     (in_x && (meets(gz0, gz1, 0, lp) || meets(gz0, gz1, nzp - lp, nzp)));
    return edge || pml || (fsrow_check && fs && meets(gz0, gz1, lp, lp + 1));
}

// What the general per-point path needs to know about one field's update.
template <typename T>
struct ZmPoint {
    const T *xrow;              // x-derivative field: row 0 of the block, column gx-8 (shared memory)
    int xrs;                    // its row stride
    const T *z0, *z1, *z2;      // z-derivative field at column gx, row 0 of slabs i-1, i, i+1
    int zrs;
    int h, gx, gz0;
    bool fw1, fw2;              // forward (staggered) derivatives
    const T *pxi, *pzi;         // C-PML memory read (x strip, z strip)
    T *pxo, *pzo;               // ... and written (by the owner)
    int xb_add, zb_add;         // 3 = staggered C-PML tables
    bool own;
};

// The reference's reduced-order x / z stencils at one point of the block, where the
// coefficient count differs from `order` (lib/der.cpp:155-540).
template <typename T, int MODE>
__device__ __forceinline__ T fix_dx_pt(T d, const ZmPoint<T> &q, int rr, int j, int nxp, const Zm2DArgs<T> &a,
                                       const CoefSet<T> *cs)
{
    const int ix = q.gx + j;
    const int K = q.fw1 ? kfw_in(ix, nxp, a.order) : kbw_in(ix, nxp, a.order);
    if (K == a.order) return d;
    return stencil_k<T, MODE>(q.xrow + rr * q.xrs + 8 + j, 1, K, cs->cx + K * CROW, q.fw1, a.dx, a.rdx);
}
template <typename T, int MODE>
__device__ __forceinline__ T fix_dz_pt(T d, const ZmPoint<T> &q, int rr, int j, int nzp, const Zm2DArgs<T> &a,
                                       const CoefSet<T> *cs)
{
    const int iz = q.gz0 + rr;
    const int K = q.fw2 ? kfw_in(iz, nzp, a.order) : kbw_in(iz, nzp, a.order);
    if (K == a.order) return d;
    return stencil_k_ring<T, MODE>(q.z0 + j, q.z1 + j, q.z2 + j, q.zrs, 4 * q.h + rr + 8, K, cs->cz + K * CROW, q.fw2,
                                   a.dz, a.rdz);
}

// General per-point update of one field (a loop over the block's 8 points, not
// unrolled, so the code stays small): reduced-order derivatives where the
// reference uses them, then F += a*d1 [x strip: psi = B*psi + A*d1,
// F -= a*(psi + C*d1)] ; F += a*d2 [z strip likewise]  (lib/waves.cpp:245-307).
template <typename T, int MODE>
__device__ __noinline__ void general_update(T *F, const T *Mo, const T *d1, const T *d2, bool has1, bool has2,
                                            const ZmPoint<T> &q, const Shot2D<T> &sh, const Zm2DArgs<T> &a,
                                            const CoefSet<T> *cs)
{
    using A = Ar<T, MODE>;
    for (int k = 0; k < 8; k++) {
        const int rr = k >> 1, j = k & 1, ix = q.gx + j, iz = q.gz0 + rr;
        const T am = A::mul(a.dt, Mo[k]);
        if (has1) {
            const T d = fix_dx_pt<T, MODE>(d1[k], q, rr, j, sh.nxp, a, cs);
            F[k] = A::mad(F[k], am, d);
            int xb, xc;
            const int xi = xstrip_in(ix, iz, sh.nxp, sh.nzp, a.lpml, xb, xc);
            if (xi >= 0) {
                const int o = iz * 2 * a.lpml + xc;
                F[k] = pml_pp<T, MODE>(F[k], am, d, q.pxi + o, q.pxo + o, q.own, a.pml, a.lpml, xb + q.xb_add, xi);
            }
        }
        if (has2) {
            const T d = fix_dz_pt<T, MODE>(d2[k], q, rr, j, sh.nzp, a, cs);
            F[k] = A::mad(F[k], am, d);
            int zb, zr;
            const int zi = zstrip_in(ix, iz, sh.nxp, sh.nzp, a.lpml, zb, zr);
            if (zi >= 0) {
                const int o = zr * sh.nxp + ix;
                F[k] = pml_pp<T, MODE>(F[k], am, d, q.pzi + o, q.pzo + o, q.own, a.pml, a.lpml, zb + q.zb_add, zi);
            }
        }
    }
}

// General per-point update of the normal stresses (lib/waves.cpp:1596-1674):
// d1 = Dx-Vx feeds Sxx with L2M and Szz with L and one x memory; d2 = Dz-Vz
// likewise with one z memory; free surface Szz = 0 on row lpml.
template <typename T, int MODE>
__device__ __noinline__ void general_normal(T *sxx, T *szz, const T *l, const T *l2m, const T *d1, const T *d2,
                                            const ZmPoint<T> &q, const Shot2D<T> &sh, const Zm2DArgs<T> &a,
                                            const CoefSet<T> *cs)
{
    using A = Ar<T, MODE>;
    for (int k = 0; k < 8; k++) {
        const int rr = k >> 1, j = k & 1, ix = q.gx + j, iz = q.gz0 + rr;
        const T a2 = A::mul(a.dt, l2m[k]), a1 = A::mul(a.dt, l[k]);
        const T e1 = fix_dx_pt<T, MODE>(d1[k], q, rr, j, sh.nxp, a, cs);
        const T e2 = fix_dz_pt<T, MODE>(d2[k], q, rr, j, sh.nzp, a, cs);
        T xx = A::mad(sxx[k], a2, e1), zz = A::mad(szz[k], a1, e1);
        int xb, xc;
        const int xi = xstrip_in(ix, iz, sh.nxp, sh.nzp, a.lpml, xb, xc);
        if (xi >= 0) {
            T *ps = sh.psix[2] + iz * 2 * a.lpml + xc;
            const T tA = __ldg(a.pml + (xb + PT_A) * a.lpml + xi), tB = __ldg(a.pml + (xb + PT_B) * a.lpml + xi),
                    tC = __ldg(a.pml + (xb + PT_C) * a.lpml + xi);
            const T p = A::mad(A::mul(tB, *ps), tA, e1);
            *ps = p;
            const T cq = A::mad(p, tC, e1);
            xx = A::msub(xx, a2, cq);
            zz = A::msub(zz, a1, cq);
        }
        xx = A::mad(xx, a1, e2);
        zz = A::mad(zz, a2, e2);
        int zb, zr;
        const int zi = zstrip_in(ix, iz, sh.nxp, sh.nzp, a.lpml, zb, zr);
        if (zi >= 0) {
            T *ps = sh.psiz[2] + zr * sh.nxp + ix;
            const T tA = __ldg(a.pml + (zb + PT_A) * a.lpml + zi), tB = __ldg(a.pml + (zb + PT_B) * a.lpml + zi),
                    tC = __ldg(a.pml + (zb + PT_C) * a.lpml + zi);
            const T p = A::mad(A::mul(tB, *ps), tA, e2);
            *ps = p;
            const T cq = A::mad(p, tC, e2);
            xx = A::msub(xx, a1, cq);
            zz = A::msub(zz, a2, cq);
        }
        if (sh.fs && iz == a.lpml) zz = T(0);
        sxx[k] = xx;
        szz[k] = zz;
    }
}

// Register block <-> flat per-point arrays for the general path.
template <typename T>
__device__ __forceinline__ void flat(T *o, const T (&v)[4][2])
{
#pragma unroll
    for (int k = 0; k < 8; k++) o[k] = v[k >> 1][k & 1];
}
template <typename T>
__device__ __forceinline__ void unflat(T (&v)[4][2], const T *o)
{
#pragma unroll
    for (int k = 0; k < 8; k++) v[k >> 1][k & 1] = o[k];
}

// One field's update: the fast path, or the general path through flat arrays.
template <typename T, int MODE>
__device__ __forceinline__ void field_update(bool special, T (&F)[4][2], const T (&Mo)[4][2], const T (&d1)[4][2],
                                             const T (&d2)[4][2], bool has1, bool has2, const ZmPoint<T> &q,
                                             const Shot2D<T> &sh, const Zm2DArgs<T> &a, const CoefSet<T> *cs)
{
    if (!special) {
        fast_update<T, MODE>(F, Mo, d1, d2, has1, has2, a.dt);
        return;
    }
    T f[8], m[8], e1[8], e2[8];
    flat(f, F);
    flat(m, Mo);
    flat(e1, d1);
    flat(e2, d2);
    general_update<T, MODE>(f, m, e1, e2, has1, has2, q, sh, a, cs);
    unflat(F, f);
}

// ------------------------------------------------------------------ point-wise inputs
template <typename T>
struct VelIn { T f1[4][2], f2[4][2], m1[4][2], m2[4][2]; };   // Vx, Vz (old), Rx, Rz
template <typename T, int PHYS>
struct StrIn { T l[4][2], l2m[4][2], m[4][2]; };               // L (acoustic: L only), L2M, M

template <typename T>
__device__ __forceinline__ void ld_pair_rows(const T *base, int o0, int pitch, T (&v)[4][2])
{
    using P = typename Pair<T>::t;
#pragma unroll
    for (int rr = 0; rr < 4; rr++) {
        const P q = *reinterpret_cast<const P *>(base + o0 + rr * pitch);
        v[rr][0] = q.x;
        v[rr][1] = q.y;
    }
}
template <typename T>
__device__ __forceinline__ void ldg_pair_rows(const T *base, int o0, int pitch, T (&v)[4][2])
{
    using P = typename Pair<T>::t;
#pragma unroll
    for (int rr = 0; rr < 4; rr++) {
        const P q = __ldg(reinterpret_cast<const P *>(base + o0 + rr * pitch));
        v[rr][0] = q.x;
        v[rr][1] = q.y;
    }
}
template <typename T>
__device__ __forceinline__ void st_pair_rows(T *base, int o0, int pitch, const T (&v)[4][2])
{
    using P = typename Pair<T>::t;
#pragma unroll
    for (int rr = 0; rr < 4; rr++) {
        P q;
        q.x = v[rr][0];
        q.y = v[rr][1];
        *reinterpret_cast<P *>(base + o0 + rr * pitch) = q;
    }
}

// ------------------------------------------------------------------ injection / recording of one point or trace
// Injection of set q's contributions at its j-th target point into field copy F
// (lib/waves.cpp:407-497, 2085-2174): contributions in the reference's order.
template <typename T, int MODE>
__device__ __forceinline__ void inject_point(T *const *F, const T *const *Mp, const InjSet<T> &q, int j, int it, int nt,
                                             T dt)
{
    using A = Ar<T, MODE == MODE_FAST ? MODE_FAST : MODE_IEEE>;
    const int p = q.pt[j];
    if (q.kind == INJ_E2_P) {
        T sxx = F[E2_SXX][p], szz = F[E2_SZZ][p];
        for (int c = q.start[j]; c < q.start[j + 1]; c++) {
            const T w = q.wav[(long)q.trace[c] * nt + it];
            const T s = A::mul(A::mul(A::mul(dt, w), q.wx[c]), q.wz[c]);
            sxx = A::sub(sxx, s);
            szz = A::sub(szz, s);
        }
        F[E2_SXX][p] = sxx;
        F[E2_SZZ][p] = szz;
        return;
    }
    T *G;
    const T *Mod;
    switch (q.kind) {
    case INJ_A2_P: G = F[A2_P]; Mod = Mp[M_L]; break;
    case INJ_A2_VX: G = F[A2_VX]; Mod = Mp[M_RX]; break;
    case INJ_A2_VZ: G = F[A2_VZ]; Mod = Mp[M_RZ]; break;
    case INJ_E2_VX: G = F[E2_VX]; Mod = Mp[M_RX]; break;
    default: G = F[E2_VZ]; Mod = Mp[M_RZ]; break;
    }
    T v = G[p];
    const T dm = A::mul(dt, Mod[p]);
    for (int c = q.start[j]; c < q.start[j + 1]; c++) {
        const T w = q.wav[(long)q.trace[c] * nt + it];
        v = A::add(v, A::mul(A::mul(A::mul(dm, w), q.wx[c]), q.wz[c]));
    }
    G[p] = v;
}

// Recording of trace tr of set q at sample `it` from field copy F
// (lib/waves.cpp:500-595, 2178-2288), accumulated into the trace.
template <typename T, int MODE>
__device__ __forceinline__ void record_trace(const T *const *F, int pitch, const RecSet<T> &q, int tr, int it, int nt)
{
    using A = Ar<T, MODE == MODE_FAST ? MODE_FAST : MODE_IEEE>;
    const int p = q.pt[tr];
    if (p < 0) return;
    const T wx0 = q.w[4 * tr], wx1 = q.w[4 * tr + 1];
    const T wz0 = q.w[4 * tr + 2], wz1 = q.w[4 * tr + 3];
    const int off[4] = {0, 1, pitch, pitch + 1};
    const T wx[4] = {wx0, wx1, wx0, wx1}, wz[4] = {wz0, wz0, wz1, wz1};
    T *out = q.out + (long)tr * nt + it;
    T acc = *out;
    if (q.kind == REC_E2_P) {
        // (1./2.)*xtri*ytri*F/factor is evaluated in double by the reference and
        // added to the T-typed trace sample (lib/waves.cpp:2238-2239)
        const double fac = (double)q.factor[tr];
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const double w = __dmul_rn(__dmul_rn(0.5, (double)wx[c]), (double)wz[c]);
            acc = (T)__dadd_rn((double)acc, __ddiv_rn(__dmul_rn(w, (double)F[E2_SXX][p + off[c]]), fac));
            acc = (T)__dadd_rn((double)acc, __ddiv_rn(__dmul_rn(w, (double)F[E2_SZZ][p + off[c]]), fac));
        }
    } else if (q.kind == REC_E2_PSUM) {
#pragma unroll
        for (int c = 0; c < 4; c++)
            acc = A::add(acc, A::mul(A::mul(wx[c], wz[c]), A::add(F[E2_SXX][p + off[c]], F[E2_SZZ][p + off[c]])));
    } else {
        const T *G;
        switch (q.kind) {
        case REC_A2_P: G = F[A2_P]; break;
        case REC_A2_VX: G = F[A2_VX]; break;
        case REC_A2_VZ: G = F[A2_VZ]; break;
        case REC_E2_VX: G = F[E2_VX]; break;
        default: G = F[E2_VZ]; break;
        }
#pragma unroll
        for (int c = 0; c < 4; c++) acc = A::add(acc, A::mul(A::mul(wx[c], wz[c]), G[p + off[c]]));
    }
    *out = acc;
}

// ------------------------------------------------------------------ the fused step
// ctl[0]: step counter of graph replays, ctl[1]: error word, ctl[2]: recording
// gate, ctl[3]: first step of the current run (nothing earlier is recorded),
// ctl[4 + c]: work counter of launches that read copy c.
template <typename T, int MODE, int PHYS, int TX>
struct ZmStep {
    using G = ZmGeo<T, PHYS, TX>;
    using A = Ar<T, MODE>;
    static constexpr int SW = G::SW, VW = G::VW, NRF = G::NRF;
    // ring field indices
    static constexpr int R_SXX = 0, R_SZZ = 1, R_SXZ = 2, R_P = 0;

    T *ring, *vring;
    CoefSet<T> *cs;
    uint64_t *bar;
    int tid, h, p;
    unsigned gslab;          // ring slabs issued by this CTA so far (slot = index & 3, parity = (index >> 2) & 1)

    __device__ T *slot_ptr(unsigned g) { return ring + (size_t)(g & 3u) * NRF * G::SLAB; }
    __device__ T *vslot_ptr(int s) { return vring + (size_t)(s % ZM_VSLOTS) * 2 * G::VSLAB; }
    // velocity C-PML memory of copy c
    static __device__ __forceinline__ T *psi_x(const Shot2D<T> &sh, int k, int c) { return c ? sh.psixb[k] : sh.psix[k]; }
    static __device__ __forceinline__ T *psi_z(const Shot2D<T> &sh, int k, int c) { return c ? sh.psizb[k] : sh.psiz[k]; }

    __device__ void issue(const Zm2DArgs<T> &a, const ZmItem &it, int cur, int j, int nslab)
    {
        if (tid != 0 || j >= nslab) return;
        const unsigned g = gslab + (unsigned)j;
        uint64_t *b = &bar[g & 3u];
        // the slot was last read through the generic proxy; order those reads before the async writes
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        mbar_expect_tx(b, (uint32_t)(NRF * G::SLAB * sizeof(T)));
        const CUtensorMap *maps = reinterpret_cast<const CUtensorMap *>(a.maps) + ((size_t)it.shot * 2 + cur) * NRF;
        // field element (x, z) is allocation element (x + GUARD, z + GUARD)
        const int xa = it.x0 - 16 + GUARD, za = it.z0 - 16 + ZM_RB * j + GUARD;
        T *dst = slot_ptr(g);
        for (int f = 0; f < NRF; f++) tma_load_2d(dst + f * G::SLAB, maps + f, b, xa, za);
    }
    __device__ bool wait(int j, int *err)
    {
        const unsigned g = gslab + (unsigned)j;
        return mbar_wait_bounded(&bar[g & 3u], (g >> 2) & 1u, err);
    }

    // velocity point-wise inputs of slab i for the thread's pair
    __device__ void load_vel(VelIn<T> &v, const Shot2D<T> &sh, T *const *Fo, int x0, int z0, int i)
    {
        const int gx = x0 - 8 + 2 * p, gz0 = z0 - 16 + ZM_RB * i + 4 * h;
        const int o0 = gz0 * sh.pitch + gx;
        const int s1 = PHYS == PHYS_E2D ? E2_VX : A2_VX, s2 = PHYS == PHYS_E2D ? E2_VZ : A2_VZ;
        ld_pair_rows(Fo[s1], o0, sh.pitch, v.f1);
        ld_pair_rows(Fo[s2], o0, sh.pitch, v.f2);
        ldg_pair_rows(sh.m[M_RX], o0, sh.pitch, v.m1);
        ldg_pair_rows(sh.m[M_RZ], o0, sh.pitch, v.m2);
    }
    __device__ void load_str(StrIn<T, PHYS> &v, const Shot2D<T> &sh, int x0, int z0, int j)
    {
        const int gx = x0 + 2 * p, gz0 = z0 - 16 + ZM_RB * j + 4 * h;
        const int o0 = gz0 * sh.pitch + gx;
        ldg_pair_rows(sh.m[M_L], o0, sh.pitch, v.l);
        if (PHYS == PHYS_E2D) {
            ldg_pair_rows(sh.m[M_L2M], o0, sh.pitch, v.l2m);
            ldg_pair_rows(sh.m[M_M], o0, sh.pitch, v.m);
        }
    }

    // Per-point context of one field's update for the general path.
    __device__ ZmPoint<T> point(const T *xrow, int xrs, const T *z0, const T *z1, const T *z2, int zrs, int gx, int gz0,
                                bool fw1, bool fw2, const T *pxi, T *pxo, int xb_add, const T *pzi, T *pzo, int zb_add,
                                bool own)
    {
        ZmPoint<T> q;
        q.xrow = xrow; q.xrs = xrs; q.z0 = z0; q.z1 = z1; q.z2 = z2; q.zrs = zrs;
        q.h = h; q.gx = gx; q.gz0 = gz0; q.fw1 = fw1; q.fw2 = fw2;
        q.pxi = pxi; q.pxo = pxo; q.xb_add = xb_add; q.pzi = pzi; q.pzo = pzo; q.zb_add = zb_add; q.own = own;
        return q;
    }

    // ---- velocity of slab i (columns x0-8 .. x0+TX+8)
    __device__ void velocity(const Zm2DArgs<T> &a, const Shot2D<T> &sh, const ZmItem &it, int cur, int i, VelIn<T> &v,
                             T *const *Fn, bool owned_rows)
    {
        const int vc = 2 * p, gx = it.x0 - 8 + vc, gz0 = it.z0 - 16 + ZM_RB * i + 4 * h;
        const T *s0 = slot_ptr(gslab + i - 1), *s1 = slot_ptr(gslab + i), *s2 = slot_ptr(gslab + i + 1);
        const int sc = vc + 8;                         // ring column of the pair
        const bool special = block_special(gx, gz0, sh.nxp, sh.nzp, a.order, a.lpml, false, false);
        const bool own = owned_rows && p >= 4 && p < 4 + G::NPS;
        T cux[NCOEF], cuz[NCOEF];
#pragma unroll
        for (int k = 0; k < NCOEF; k++) { cux[k] = cs->cx[a.order * CROW + k]; cuz[k] = cs->cz[a.order * CROW + k]; }
        const int lo = cur, hi = cur ^ 1;   // psi copies read / written
        T d1[4][2], d2[4][2];
        const T *rowbase = s1 + (4 * h) * SW + sc - 8;   // row 0 of the block, column gx-8, ring field 0
        if constexpr (PHYS == PHYS_E2D) {
            // Vx += dt*Rx*Dx+Sxx [x stag psi0] ; Vx += dt*Rx*Dz-Sxz [z psi0]   (lib/waves.cpp:1416-1490)
            const T *rxz0 = s0 + R_SXZ * G::SLAB + sc, *rxz1 = s1 + R_SXZ * G::SLAB + sc, *rxz2 = s2 + R_SXZ * G::SLAB + sc;
#pragma unroll
            for (int rr = 0; rr < 4; rr++) dx_pair<T, MODE, true>(rowbase + R_SXX * G::SLAB + rr * SW, cux, a.dx, a.rdx, d1[rr]);
            dz_half<T, MODE, false, SW>(h, rxz0, rxz1, rxz2, cuz, a.dz, a.rdz, d2);
            field_update<T, MODE>(special, v.f1, v.m1, d1, d2, true, true,
                                  point(rowbase + R_SXX * G::SLAB, SW, rxz0, rxz1, rxz2, SW, gx, gz0, true, false,
                                        psi_x(sh, 0, lo), psi_x(sh, 0, hi), 3, psi_z(sh, 0, lo), psi_z(sh, 0, hi), 0, own),
                                  sh, a, cs);
            // Vz += dt*Rz*Dx-Sxz [x psi1] ; Vz += dt*Rz*Dz+Szz [z stag psi1]   (lib/waves.cpp:1492-1566)
            const T *rzz0 = s0 + R_SZZ * G::SLAB + sc, *rzz1 = s1 + R_SZZ * G::SLAB + sc, *rzz2 = s2 + R_SZZ * G::SLAB + sc;
#pragma unroll
            for (int rr = 0; rr < 4; rr++) dx_pair<T, MODE, false>(rowbase + R_SXZ * G::SLAB + rr * SW, cux, a.dx, a.rdx, d1[rr]);
            dz_half<T, MODE, true, SW>(h, rzz0, rzz1, rzz2, cuz, a.dz, a.rdz, d2);
            field_update<T, MODE>(special, v.f2, v.m2, d1, d2, true, true,
                                  point(rowbase + R_SXZ * G::SLAB, SW, rzz0, rzz1, rzz2, SW, gx, gz0, false, true,
                                        psi_x(sh, 1, lo), psi_x(sh, 1, hi), 0, psi_z(sh, 1, lo), psi_z(sh, 1, hi), 3, own),
                                  sh, a, cs);
        } else {
            // Vx += dt*Rx*Dx+P [x stag psi0] ; Vz += dt*Rz*Dz+P [z stag psi0]   (lib/waves.cpp:217-310)
            const T *rp0 = s0 + sc, *rp1 = s1 + sc, *rp2 = s2 + sc;
#pragma unroll
            for (int rr = 0; rr < 4; rr++) dx_pair<T, MODE, true>(rowbase + rr * SW, cux, a.dx, a.rdx, d1[rr]);
            dz_half<T, MODE, true, SW>(h, rp0, rp1, rp2, cuz, a.dz, a.rdz, d2);
            const ZmPoint<T> q = point(rowbase, SW, rp0, rp1, rp2, SW, gx, gz0, true, true, psi_x(sh, 0, lo),
                                       psi_x(sh, 0, hi), 3, psi_z(sh, 0, lo), psi_z(sh, 0, hi), 3, own);
            field_update<T, MODE>(special, v.f1, v.m1, d1, d1, true, false, q, sh, a, cs);
            field_update<T, MODE>(special, v.f2, v.m2, d2, d2, false, true, q, sh, a, cs);
        }
        // velocity ring (all columns) and the new copy (owned points)
        T *vs = vslot_ptr(i);
        st_pair_rows(vs, (4 * h) * VW + vc, VW, v.f1);
        st_pair_rows(vs + G::VSLAB, (4 * h) * VW + vc, VW, v.f2);
        if (own) {
            const int o0 = gz0 * sh.pitch + gx;
            st_pair_rows(Fn[PHYS == PHYS_E2D ? E2_VX : A2_VX], o0, sh.pitch, v.f1);
            st_pair_rows(Fn[PHYS == PHYS_E2D ? E2_VZ : A2_VZ], o0, sh.pitch, v.f2);
        }
    }

    // ---- stresses of slab j (owned columns x0 .. x0+TX)
    __device__ void stress(const Zm2DArgs<T> &a, const Shot2D<T> &sh, const ZmItem &it, int j, const StrIn<T, PHYS> &m,
                           T *const *Fn)
    {
        using A = Ar<T, MODE>;
        const int gx = it.x0 + 2 * p, gz0 = it.z0 - 16 + ZM_RB * j + 4 * h;
        const int vc = 2 * p + 8, sc = 2 * p + 16;
        const T *v0 = vslot_ptr(j - 1), *v1 = vslot_ptr(j), *v2 = vslot_ptr(j + 1);
        const T *so = slot_ptr(gslab + j) + (4 * h) * SW + sc;   // old stresses, row 4h of slab j
        const bool special = block_special(gx, gz0, sh.nxp, sh.nzp, a.order, a.lpml, true, sh.fs != 0);
        T cux[NCOEF], cuz[NCOEF];
#pragma unroll
        for (int k = 0; k < NCOEF; k++) { cux[k] = cs->cx[a.order * CROW + k]; cuz[k] = cs->cz[a.order * CROW + k]; }
        const int o0 = gz0 * sh.pitch + gx;
        T d1[4][2], d2[4][2];
        const T *vx0 = v0 + vc, *vx1 = v1 + vc, *vx2 = v2 + vc;                                   // Vx plane
        const T *vz0 = v0 + G::VSLAB + vc, *vz1 = v1 + G::VSLAB + vc, *vz2 = v2 + G::VSLAB + vc;   // Vz plane
        const T *rowx = v1 + (4 * h) * VW + vc - 8, *rowz = rowx + G::VSLAB;   // row 0 of the block, column gx-8
        // d1 = Dx-Vx, d2 = Dz-Vz
#pragma unroll
        for (int rr = 0; rr < 4; rr++) dx_pair<T, MODE, false>(rowx + rr * VW, cux, a.dx, a.rdx, d1[rr]);
        dz_half<T, MODE, false, VW>(h, vz0, vz1, vz2, cuz, a.dz, a.rdz, d2);
        if constexpr (PHYS == PHYS_E2D) {
            T sxx[4][2], szz[4][2];
#pragma unroll
            for (int rr = 0; rr < 4; rr++)
#pragma unroll
                for (int c = 0; c < 2; c++) {
                    sxx[rr][c] = so[R_SXX * G::SLAB + rr * SW + c];
                    szz[rr][c] = so[R_SZZ * G::SLAB + rr * SW + c];
                }
            if (!special) {
                // normal stresses (lib/waves.cpp:1596-1674), no strip, no free surface here
#pragma unroll
                for (int rr = 0; rr < 4; rr++)
#pragma unroll
                    for (int c = 0; c < 2; c++) {
                        const T a2 = A::mul(a.dt, m.l2m[rr][c]), a1 = A::mul(a.dt, m.l[rr][c]);
                        sxx[rr][c] = A::mad(A::mad(sxx[rr][c], a2, d1[rr][c]), a1, d2[rr][c]);
                        szz[rr][c] = A::mad(A::mad(szz[rr][c], a1, d1[rr][c]), a2, d2[rr][c]);
                    }
            } else {
                T fx[8], fz[8], l[8], l2m[8], e1[8], e2[8];
                flat(fx, sxx); flat(fz, szz); flat(l, m.l); flat(l2m, m.l2m); flat(e1, d1); flat(e2, d2);
                const ZmPoint<T> q = point(rowx, VW, vz0, vz1, vz2, VW, gx, gz0, false, false, nullptr, nullptr, 0,
                                           nullptr, nullptr, 0, true);
                general_normal<T, MODE>(fx, fz, l, l2m, e1, e2, q, sh, a, cs);
                unflat(sxx, fx);
                unflat(szz, fz);
            }
            st_pair_rows(Fn[E2_SXX], o0, sh.pitch, sxx);
            st_pair_rows(Fn[E2_SZZ], o0, sh.pitch, szz);
            // Sxz += dt*M*Dx+Vz [x stag psi3] ; Sxz += dt*M*Dz+Vx [z stag psi3]   (lib/waves.cpp:1676-1735)
#pragma unroll
            for (int rr = 0; rr < 4; rr++) dx_pair<T, MODE, true>(rowz + rr * VW, cux, a.dx, a.rdx, d1[rr]);
            dz_half<T, MODE, true, VW>(h, vx0, vx1, vx2, cuz, a.dz, a.rdz, d2);
            T sxz[4][2];
#pragma unroll
            for (int rr = 0; rr < 4; rr++)
#pragma unroll
                for (int c = 0; c < 2; c++) sxz[rr][c] = so[R_SXZ * G::SLAB + rr * SW + c];
            field_update<T, MODE>(special, sxz, m.m, d1, d2, true, true,
                                  point(rowz, VW, vx0, vx1, vx2, VW, gx, gz0, true, true, sh.psix[3], sh.psix[3], 3,
                                        sh.psiz[3], sh.psiz[3], 3, true),
                                  sh, a, cs);
            st_pair_rows(Fn[E2_SXZ], o0, sh.pitch, sxz);
        } else {
            // P += dt*L*Dx-Vx [x psi1] ; P += dt*L*Dz-Vz [z psi1]   (lib/waves.cpp:313-404)
            T pp[4][2];
#pragma unroll
            for (int rr = 0; rr < 4; rr++)
#pragma unroll
                for (int c = 0; c < 2; c++) pp[rr][c] = so[R_P * G::SLAB + rr * SW + c];
            field_update<T, MODE>(special, pp, m.l, d1, d2, true, true,
                                  point(rowx, VW, vz0, vz1, vz2, VW, gx, gz0, false, false, sh.psix[1], sh.psix[1], 0,
                                        sh.psiz[1], sh.psiz[1], 0, true),
                                  sh, a, cs);
            st_pair_rows(Fn[A2_P], o0, sh.pitch, pp);
        }
    }

    // Wait (bounded) for the ring slabs [from, to) this CTA issued, so that no copy
    // is still landing in shared memory when the CTA exits.  Slabs that already
    // completed pass at once.
    __device__ void drain(int from, int to)
    {
        if (tid != 0) return;
        for (int j = from; j < to; j++) wait(j, nullptr);
    }

    // One work item; false if a wait gave up (the CTA then stops).
    __device__ bool item(const Zm2DArgs<T> &a, const ZmItem &it, int cur, int step, int *err)
    {
        const Shot2D<T> &sh = a.shots[it.shot];
        T *const *Fo = cur ? sh.fb : sh.f;
        T *const *Fn = cur ? sh.f : sh.fb;
        const int nown = (it.z1 - it.z0) / ZM_RB, nslab = nown + 4;
        for (int j = 0; j < ZM_SLOTS; j++) issue(a, it, cur, j, nslab);
        VelIn<T> vcur;
        load_vel(vcur, sh, Fo, it.x0, it.z0, 1);
        for (int i = 1; i <= nown + 2; i++) {
            bool ok = i == 1 ? (wait(0, err) && wait(1, err) && wait(2, err)) : wait(i + 1, err);
            if (!__syncthreads_and(ok)) {
                drain(i == 1 ? 0 : i + 1, min(i + 3, nslab));   // slabs up to i+2 were issued
                __syncthreads();
                return false;
            }
            StrIn<T, PHYS> scur;
            const bool do_str = i - 1 >= 2;
            if (do_str && p < G::NPS) load_str(scur, sh, it.x0, it.z0, i - 1);
            if (p < G::NPV) velocity(a, sh, it, cur, i, vcur, Fn, i >= 2 && i <= nown + 1);
            __syncthreads();
            VelIn<T> vnext;
            if (i + 1 <= nown + 2) load_vel(vnext, sh, Fo, it.x0, it.z0, i + 1);
            if (do_str && p < G::NPS) stress(a, sh, it, i - 1, scur, Fn);
            __syncthreads();
            issue(a, it, cur, i + 3, nslab);
            vcur = vnext;
        }
        gslab += (unsigned)nslab;
        // injection of this step into the owned points (sets in order)
        const InjRec<T> &pl = a.plans[it.shot];
        const int itw = pl.rev ? pl.nt - 1 - step : step;
        bool pending = false;   // a point may receive several sets: they add in set order
        for (int s = 0; s < pl.ninjsets; s++) {
            if (it.ie[s + 1] == it.ie[s]) continue;
            if (pending) __syncthreads();
            for (int e = it.ie[s] + tid; e < it.ie[s + 1]; e += ZM_NT)
                inject_point<T, MODE>(Fn, sh.m, pl.inj[s], a.inj[e] & 0xffffff, itw, pl.nt, a.dt);
            pending = true;
        }
        return true;
    }
};

template <typename T, int MODE, int PHYS, int TX, int MINB>
__global__ void __launch_bounds__(ZM_NT, MINB)
zm_step_2d(Zm2DArgs<T> a, const CoefSet<T> *coefs, int *ctl, int cur, int it_base, int use_dev_it)
{
    using G = ZmGeo<T, PHYS, TX>;
    extern __shared__ __align__(128) unsigned char sm[];
    ZmStep<T, MODE, PHYS, TX> z;
    z.ring = reinterpret_cast<T *>(sm);
    z.vring = reinterpret_cast<T *>(sm + G::ring_bytes);
    z.cs = reinterpret_cast<CoefSet<T> *>(sm + G::coef_off);
    z.bar = reinterpret_cast<uint64_t *>(sm + G::bar_off);
    int *s_item = reinterpret_cast<int *>(z.bar + ZM_SLOTS);
    z.tid = threadIdx.x;
    const int w = threadIdx.x >> 5;
    z.h = w >> 1;
    z.p = ((w & 1) << 5) | (threadIdx.x & 31);
    z.gslab = 0;
    int *err = ctl + 1;
    const int step = it_base + (use_dev_it ? ctl[0] : 0);
    // the next launch (which reads the other copy) starts its work counter from zero
    if (blockIdx.x == 0 && threadIdx.x == 0) ctl[4 + (cur ^ 1)] = 0;
    // recording of the previous step, whose state is the copy read here
    if (step > ctl[3] && !(*(volatile int *)err)) {
        for (int g = blockIdx.x * ZM_NT + threadIdx.x; g < a.nrecs; g += gridDim.x * ZM_NT) {
            const int4 r = a.recs[g];
            const Shot2D<T> &sh = a.shots[r.x];
            const InjRec<T> &pl = a.plans[r.x];
            if (pl.rec_gate && *pl.rec_gate == 0) continue;
            const int prev = pl.rev ? pl.nt - 1 - (step - 1) : step - 1;
            record_trace<T, MODE>(cur ? sh.fb : sh.f, sh.pitch, pl.rec[r.y], r.z, prev, pl.nt);
        }
    }
    if (threadIdx.x == 0)
        for (int s = 0; s < ZM_SLOTS; s++) mbar_init(&z.bar[s], 1);
    load_coefs(*z.cs, coefs);
    __syncthreads();
    for (;;) {
        if (threadIdx.x == 0) *s_item = *(volatile int *)err ? a.nitems : atomicAdd(&ctl[4 + cur], 1);
        __syncthreads();
        const int k = *s_item;
        if (k >= a.nitems) break;
        const ZmItem it = a.items[k];
        if (!z.item(a, it, cur, step, err)) break;
        __syncthreads();
    }
}

// Recording only (the last step of a run): the state is in copy `cur`.
template <typename T, int MODE>
__global__ void zm_record_2d(Zm2DArgs<T> a, const int *ctl, int cur, int step)
{
    if (*(volatile const int *)(ctl + 1)) return;
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < a.nrecs; g += gridDim.x * blockDim.x) {
        const int4 r = a.recs[g];
        const Shot2D<T> &sh = a.shots[r.x];
        const InjRec<T> &pl = a.plans[r.x];
        if (pl.rec_gate && *pl.rec_gate == 0) continue;
        const int s = pl.rev ? pl.nt - 1 - step : step;
        record_trace<T, MODE>(cur ? sh.fb : sh.f, sh.pitch, pl.rec[r.y], r.z, s, pl.nt);
    }
}

}  // namespace rsgpu
