// Kernels of the 2D FWI gradient and RTM image drivers:
//   * the gradient correlation of FwiAcoustic2D::crossCorr (lib/fwi.cpp:511-571),
//   * the (extended) image correlation of RtmAcoustic2D::crossCorr (lib/rtm.cpp:191-219),
//   * residuals and misfit of FwiAcoustic2D::computeResiduals / computeMisfit
//     with the DIFFERENCE misfit (lib/fwi.cpp:597-611, 798-806),
//   * checkpoint slot save/restore (the in-core checkpoints of Revolve,
//     lib/revolve.cpp:648-818), optionally as FP16/BF16 with a power-of-two scale
//     per block.
// All of them are memory-bound elementwise passes; one launch covers every shot
// of the batch (blockIdx.z or blockIdx.y selects the shot / block).
//
// Exact mode reproduces the reference's float expression evaluation: C's usual
// arithmetic conversions evaluate `0.5 * a * b * (c - d) / dx` in double when
// a..d are float, and `-2.0 / vp` in double rounded to float; every such operation
// is written out with explicitly rounded intrinsics.
#include <algorithm>
#include <cstring>
#include <cuda_fp16.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "adjoint_ops.cuh"
#include "rsgpu_adjoint.h"
#include "rsgpu_kernels.h"

namespace rsgpu {
namespace {

// ---------------------------------------------------------------- FWI gradient correlation
// vpgrad -= (-2/vp) * Pfw * (dx- Vx_adj + dz- Vz_adj)
// rhograd -= (-1/rho) * Pfw * (same)
// rhograd += 1/2 [ Vx_adj Rx dx+ Pfw ] averaged over the two staggered x-faces (and z)
// srcilum -= (-2/vp) * Pfw * Pfw   (when the shot asks for the source illumination)
// on the interior 1..n-2 of the unpadded window.  G is the accumulator type.
template <typename T, bool EXACT, typename G>
__global__ void __launch_bounds__(256) corr_fwi_a2d(const Corr2D<T> *desc, T dx, T dz)
{
    const Corr2D<T> c = desc[blockIdx.z];
    const int ix = blockIdx.x * blockDim.x + threadIdx.x;
    const int iz = blockIdx.y * blockDim.y + threadIdx.y;
    if (ix < 1 || iz < 1 || ix >= c.nx - 1 || iz >= c.nz - 1) return;
    const long q = (long)(iz + c.lpml) * c.pitch + ix + c.lpml;
    const long u = (long)iz * c.nx + ix;
    const int P = c.pitch;
    const T ws = c.wsp[q], wsl = c.wsp[q - 1], wsr = c.wsp[q + 1], wsu = c.wsp[q - P], wsd = c.wsp[q + P];
    const T wx0 = c.wrx[q], wx1 = c.wrx[q - 1], wz0 = c.wrz[q], wz1 = c.wrz[q - P];
    const T rx0 = c.rx[q], rx1 = c.rx[q - 1], rz0 = c.rz[q], rz1 = c.rz[q - P];
    const T vp = c.vp[u], rho = c.rho[u];
    G *vg = (G *)c.g0 + u;
    G *rg = (G *)c.g1 + u;
    T a, b, uder, il = 0;
    if (EXACT) {
        using O = X<T>;
        const T vpscale = O::rnd(__ddiv_rn(-2.0, (double)vp));
        if (c.ilum) il = O::mul(O::mul(vpscale, ws), ws);
        const T rhoscale1 = O::rnd(__ddiv_rn(-1.0, (double)rho));
        const T mrxx = O::div(O::sub(wx0, wx1), dx);
        const T mrzz = O::div(O::sub(wz0, wz1), dz);
        const T s = O::add(mrxx, mrzz);
        a = O::mul(O::mul(vpscale, ws), s);
        b = O::mul(O::mul(rhoscale1, ws), s);
        const double DX = (double)dx, DZ = (double)dz;
        T ux = O::rnd(__ddiv_rn(__dmul_rn(__dmul_rn(__dmul_rn(0.5, (double)wx0), (double)rx0), (double)O::sub(wsr, ws)), DX));
        ux = O::rnd(__dadd_rn((double)ux,
                              __ddiv_rn(__dmul_rn(__dmul_rn(__dmul_rn(0.5, (double)wx1), (double)rx1), (double)O::sub(ws, wsl)), DX)));
        T uz = O::rnd(__ddiv_rn(__dmul_rn(__dmul_rn(__dmul_rn(0.5, (double)wz0), (double)rz0), (double)O::sub(wsd, ws)), DZ));
        uz = O::rnd(__dadd_rn((double)uz,
                              __ddiv_rn(__dmul_rn(__dmul_rn(__dmul_rn(0.5, (double)wz1), (double)rz1), (double)O::sub(ws, wsu)), DZ)));
        uder = O::add(ux, uz);
    } else {
        const T rdx = T(1) / dx, rdz = T(1) / dz;
        const T s = (wx0 - wx1) * rdx + (wz0 - wz1) * rdz;
        a = (T(-2) / vp) * ws * s;
        b = (T(-1) / rho) * ws * s;
        if (c.ilum) il = (T(-2) / vp) * ws * ws;
        uder = T(0.5) * ((wx0 * rx0 * (wsr - ws) + wx1 * rx1 * (ws - wsl)) * rdx +
                         (wz0 * rz0 * (wsd - ws) + wz1 * rz1 * (ws - wsu)) * rdz);
    }
    if (sizeof(G) == sizeof(T)) {
        // accumulate in the element type, in the reference's order
        using O = X<T>;
        *(T *)vg = EXACT ? O::sub(*(T *)vg, a) : *(T *)vg - a;
        const T r1 = EXACT ? O::sub(*(T *)rg, b) : *(T *)rg - b;
        *(T *)rg = EXACT ? O::add(r1, uder) : r1 + uder;
        if (c.ilum) {
            T *ig = (T *)c.ilum + u;
            *ig = EXACT ? O::sub(*ig, il) : *ig - il;
        }
    } else {
        *vg = __dsub_rn((double)*vg, (double)a);
        *rg = __dadd_rn(__dsub_rn((double)*rg, (double)b), (double)uder);
        if (c.ilum) {
            G *ig = (G *)c.ilum + u;
            *ig = __dsub_rn((double)*ig, (double)il);
        }
    }
}

// ---------------------------------------------------------------- RTM image correlation
// image[ihz][ihx][iz][ix] += Pfw(ix-hx, iz-hz) * Padj(ix+hx, iz+hz) for lags
// hx = ihx - (nhx-1)/2, hz likewise, where both points lie in the window.
template <typename T, bool EXACT, typename G>
__global__ void __launch_bounds__(256) corr_rtm_a2d(const Corr2D<T> *desc, int nhx, int nhz)
{
    const Corr2D<T> c = desc[blockIdx.z];
    const int ix = blockIdx.x * blockDim.x + threadIdx.x;
    const int iz = blockIdx.y * blockDim.y + threadIdx.y;
    if (ix >= c.nx || iz >= c.nz) return;
    const int L = c.lpml, P = c.pitch;
    for (int ihx = 0; ihx < nhx; ihx++) {
        const int hx = -(nhx - 1) / 2 + ihx;
        if (ix - hx < 0 || ix - hx >= c.nx || ix + hx < 0 || ix + hx >= c.nx) continue;
        for (int ihz = 0; ihz < nhz; ihz++) {
            const int hz = -(nhz - 1) / 2 + ihz;
            if (iz - hz < 0 || iz - hz >= c.nz || iz + hz < 0 || iz + hz >= c.nz) continue;
            const T ws = c.wsp[(long)(iz - hz + L) * P + (ix - hx + L)];
            const T wr = c.wrp[(long)(iz + hz + L) * P + (ix + hx + L)];
            G *img = (G *)c.g0 + (((long)ihz * nhx + ihx) * c.nz + iz) * c.nx + ix;
            if (sizeof(G) == sizeof(T)) {
                using O = X<T>;
                *(T *)img = EXACT ? O::add(*(T *)img, O::mul(ws, wr)) : *(T *)img + ws * wr;
            } else {
                *img = __dadd_rn((double)*img, __dmul_rn((double)ws, (double)wr));
            }
        }
    }
}

// 3D: image[ihz][ihy][ihx][iz][iy][ix] += Pfw(x-h) * Padj(x+h) (lib/rtm.cpp:601-637);
// one thread per (x, y) column, marching z.
template <typename T, bool EXACT, typename G>
__global__ void __launch_bounds__(256) corr_rtm_a3d(const Corr3D<T> *desc, int nhx, int nhy, int nhz)
{
    const Corr3D<T> c = desc[blockIdx.z];
    const int ix = blockIdx.x * blockDim.x + threadIdx.x;
    const int iy = blockIdx.y * blockDim.y + threadIdx.y;
    if (ix >= c.nx || iy >= c.ny) return;
    const int L = c.lpml;
    const long long n3 = (long long)c.nx * c.ny * c.nz;
    for (int ihx = 0; ihx < nhx; ihx++) {
        const int hx = -(nhx - 1) / 2 + ihx;
        if (ix - hx < 0 || ix - hx >= c.nx || ix + hx < 0 || ix + hx >= c.nx) continue;
        for (int ihy = 0; ihy < nhy; ihy++) {
            const int hy = -(nhy - 1) / 2 + ihy;
            if (iy - hy < 0 || iy - hy >= c.ny || iy + hy < 0 || iy + hy >= c.ny) continue;
            for (int ihz = 0; ihz < nhz; ihz++) {
                const int hz = -(nhz - 1) / 2 + ihz;
                G *img = (G *)c.img + (((long long)ihz * nhy + ihy) * nhx + ihx) * n3 + (long long)iy * c.nx + ix;
                const T *ws = c.wsp + (long long)(iy - hy + L) * c.pitch + (ix - hx + L);
                const T *wr = c.wrp + (long long)(iy + hy + L) * c.pitch + (ix + hx + L);
                const int z0 = max(hz, -hz), z1 = c.nz - max(hz, -hz);
                for (int iz = z0; iz < z1; iz++) {
                    const T a = ws[(long long)(iz - hz + L) * c.plane], b = wr[(long long)(iz + hz + L) * c.plane];
                    G *o = img + (long long)iz * c.nx * c.ny;
                    if (sizeof(G) == sizeof(T)) {
                        using O = X<T>;
                        *(T *)o = EXACT ? O::add(*(T *)o, O::mul(a, b)) : *(T *)o + a * b;
                    } else {
                        *o = __dadd_rn((double)*o, __dmul_rn((double)a, (double)b));
                    }
                }
            }
        }
    }
}

// ---------------------------------------------------------------- residuals and misfit
// Residual pass: RES_BLOCKS CTAs per shot, each over a contiguous share of the
// shot's samples; with FP64 accumulation each CTA also leaves its partial sum of
// r*r/2 over on-grid traces (fixed-order tree, so the result is reproducible).
constexpr int RES_BLOCKS = 64;

template <typename T, int ACC>
__global__ void __launch_bounds__(256) residual_diff(const Resid2D<T> *desc, double *partials)
{
    const Resid2D<T> d = desc[blockIdx.y];
    const long n = (long)d.nrec * d.nt;
    const long chunk = (n + gridDim.x - 1) / gridDim.x;
    const long k0 = (long)blockIdx.x * chunk, k1 = min(n, k0 + chunk);
    double acc = 0.0;
    for (long k = k0 + threadIdx.x; k < k1; k += blockDim.x) {
        const T r = X<T>::sub(d.mod[k], d.obs[k]);
        d.res[k] = r;
        if (ACC == ACC_F64 && d.rec_pt[k / d.nt] >= 0) acc = fma(0.5 * (double)r, (double)r, acc);
    }
    if (ACC != ACC_F64) return;
    __shared__ double red[256];
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) partials[(long)blockIdx.y * gridDim.x + blockIdx.x] = red[0];
}

// Misfit per shot: ACC_REF sums 0.5*r*r into a T-typed accumulator, traces then
// samples, as the reference does (one thread); ACC_F64 adds the CTA partials in order.
template <typename T, int ACC>
__global__ void __launch_bounds__(32) residual_sum(const Resid2D<T> *desc, const double *partials, double *misfit)
{
    if (threadIdx.x != 0) return;
    const Resid2D<T> d = desc[blockIdx.x];
    if (ACC == ACC_F64) {
        double m = 0.0;
        for (int b = 0; b < RES_BLOCKS; b++) m += partials[(long)blockIdx.x * RES_BLOCKS + b];
        misfit[blockIdx.x] = m;
        return;
    }
    T mis = 0;
    for (int tr = 0; tr < d.nrec; tr++) {
        if (d.rec_pt[tr] < 0) continue;
        const T *r = d.res + (long)tr * d.nt;
        for (int it = 0; it < d.nt; it++) {
            const double rr = (double)r[it];
            mis = X<T>::rnd(__dadd_rn((double)mis, __dmul_rn(__dmul_rn(0.5, rr), rr)));
        }
    }
    misfit[blockIdx.x] = (double)mis;
}

// ---------------------------------------------------------------- CORRELATION misfit
// FwiAcoustic2D::computeMisfit / computeResiduals, CORRELATION (lib/fwi.cpp:617-645,
// 808-849), pressure data.  Per trace, in the element type and the reference's
// order: n1 = sqrt(sum m*m), n2 = sqrt(sum o*o) (zero -> 1), n3 = sum m*o / (n1*n2);
// residual -(o/(n1*n2) - (m/(n1*n1))*n3) for every trace; misfit += -(m*o/(n1*n2))
// over the traces on the grid.  Then the residuals whose magnitude reaches the
// 97th-percentile value of all |residual| samples of the shot (the element at
// index (97*nt*nrec)/100 of the ascending sort) are zeroed (CLIP; the 3D
// driver, FwiAcoustic3D lib/fwi.cpp:1696-1722, has no clip).  The order statistic
// comes from a radix select on the magnitude bit patterns, which order like the
// non-negative values.  One CTA per shot; dynamic shared memory holds n1*n2 of
// every trace.
__device__ __forceinline__ bool finite_f(float v) { return isfinite(v); }
__device__ __forceinline__ bool finite_f(double v) { return isfinite(v); }

template <typename T, int ACC, bool CLIP>
__global__ void __launch_bounds__(256) residual_corr(const Resid2D<T> *desc, double *misfit)
{
    using U = typename Bits<T>::U;
    extern __shared__ __align__(16) unsigned char corr_smem[];
    T *nn = reinterpret_cast<T *>(corr_smem);            // n1*n2 per trace
    const Resid2D<T> d = desc[blockIdx.x];
    const long n = (long)d.nrec * d.nt;
    for (int tr = threadIdx.x; tr < d.nrec; tr += blockDim.x) {
        const T *m = d.mod + (long)tr * d.nt, *o = d.obs + (long)tr * d.nt;
        T n1 = 0, n2 = 0, n3 = 0;
        for (int it = 0; it < d.nt; it++) {
            n1 = X<T>::add(n1, X<T>::mul(m[it], m[it]));
            n2 = X<T>::add(n2, X<T>::mul(o[it], o[it]));
            n3 = X<T>::add(n3, X<T>::mul(m[it], o[it]));
        }
        n1 = sqrt_rn(n1);
        n2 = sqrt_rn(n2);
        if (n1 == T(0)) n1 = T(1);
        if (n2 == T(0)) n2 = T(1);
        const T n12 = X<T>::mul(n1, n2), n11 = X<T>::mul(n1, n1);
        n3 = X<T>::div(n3, n12);
        nn[tr] = n12;
        T *r = d.res + (long)tr * d.nt;
        for (int it = 0; it < d.nt; it++)
            r[it] = -X<T>::sub(X<T>::div(o[it], n12), X<T>::mul(X<T>::div(m[it], n11), n3));
    }
    __syncthreads();
    if (CLIP) {
        const long pos = (long)((97ull * (unsigned long long)d.nt * (unsigned long long)d.nrec) / 100ull);
        const U clip = kth_mag_bits(d.res, n, pos);
        for (long k = threadIdx.x; k < n; k += blockDim.x)
            if (mag_bits(d.res[k]) >= clip) d.res[k] = T(0);
    }
    if (threadIdx.x != 0) return;
    // misfit, traces then samples, on the traces inside the grid
    T mis = 0;
    double mis64 = 0.0;
    for (int tr = 0; tr < d.nrec; tr++) {
        if (d.rec_pt[tr] < 0) continue;
        const T *m = d.mod + (long)tr * d.nt, *o = d.obs + (long)tr * d.nt;
        for (int it = 0; it < d.nt; it++) {
            const T v = -X<T>::div(X<T>::mul(m[it], o[it]), nn[tr]);
            if (ACC == ACC_REF) mis = X<T>::add(mis, v);
            else mis64 += (double)v;
        }
    }
    misfit[blockIdx.x] = ACC == ACC_REF ? (double)mis : mis64;
}

// FwiElastic2D CORRELATION (lib/fwi.cpp:2939-3001, 3309-3426): the acoustic
// per-trace formulas for the P, Ux and Uz components; the misfit adds
// (rp + rx + rz) with non-finite terms zeroed over the traces whose Ux map is on
// the grid.  Clips: x and z share the larger of their 97th-percentile magnitudes
// and a sample whose x residual reaches it loses its x and z residual; P has its
// own; non-finite residuals become zero.  Comparisons are float comparisons, as in
// the reference.  Dynamic shared memory: n1*n2 per component and trace.
template <typename T, int ACC>
__global__ void __launch_bounds__(256) residual_corr_e2d(const Resid2DE<T> *desc, double *misfit)
{
    extern __shared__ __align__(16) unsigned char corr_smem[];
    T *nn = reinterpret_cast<T *>(corr_smem);            // [3][nrec]
    const Resid2DE<T> d = desc[blockIdx.x];
    const long n = (long)d.nrec * d.nt;
    for (int tr = threadIdx.x; tr < d.nrec; tr += blockDim.x)
        for (int c = 0; c < 3; c++) {
            const T *m = d.mod[c] + (long)tr * d.nt, *o = d.obs[c] + (long)tr * d.nt;
            T n1 = 0, n2 = 0, n3 = 0;
            for (int it = 0; it < d.nt; it++) {
                n1 = X<T>::add(n1, X<T>::mul(m[it], m[it]));
                n2 = X<T>::add(n2, X<T>::mul(o[it], o[it]));
                n3 = X<T>::add(n3, X<T>::mul(m[it], o[it]));
            }
            n1 = sqrt_rn(n1);
            n2 = sqrt_rn(n2);
            if (n1 == T(0)) n1 = T(1);
            if (n2 == T(0)) n2 = T(1);
            const T n12 = X<T>::mul(n1, n2), n11 = X<T>::mul(n1, n1);
            n3 = X<T>::div(n3, n12);
            nn[c * d.nrec + tr] = n12;
            T *r = d.res[c] + (long)tr * d.nt;
            for (int it = 0; it < d.nt; it++)
                r[it] = -X<T>::sub(X<T>::div(o[it], n12), X<T>::mul(X<T>::div(m[it], n11), n3));
        }
    __syncthreads();
    const long pos = (long)((97ull * (unsigned long long)d.nt * (unsigned long long)d.nrec) / 100ull);
    T cx = from_bits<T>(kth_mag_bits(d.res[1], n, pos));
    const T cz = from_bits<T>(kth_mag_bits(d.res[2], n, pos));
    if (cz > cx) cx = cz;
    for (long k = threadIdx.x; k < n; k += blockDim.x) {
        T rx = d.res[1][k], rz = d.res[2][k];
        if (fabs(rx) >= cx) { rx = T(0); rz = T(0); }
        if (!finite_f(rx)) rx = T(0);
        if (!finite_f(rz)) rz = T(0);
        d.res[1][k] = rx;
        d.res[2][k] = rz;
    }
    const T cp = from_bits<T>(kth_mag_bits(d.res[0], n, pos));
    for (long k = threadIdx.x; k < n; k += blockDim.x) {
        T rp = d.res[0][k];
        if (fabs(rp) >= cp) rp = T(0);
        if (!finite_f(rp)) rp = T(0);
        d.res[0][k] = rp;
    }
    if (threadIdx.x != 0) return;
    T mis = 0;
    double mis64 = 0.0;
    for (int tr = 0; tr < d.nrec; tr++) {
        if (d.rec_pt_vx[tr] < 0) continue;
        for (int it = 0; it < d.nt; it++) {
            const long j = (long)tr * d.nt + it;
            T r[3];
            for (int c = 0; c < 3; c++) {
                r[c] = -X<T>::div(X<T>::mul(d.mod[c][j], d.obs[c][j]), nn[c * d.nrec + tr]);
                if (!finite_f(r[c])) r[c] = T(0);
            }
            const T s = X<T>::add(X<T>::add(r[0], r[1]), r[2]);
            if (ACC == ACC_REF) mis = X<T>::add(mis, s);
            else mis64 += (double)s;
        }
    }
    misfit[blockIdx.x] = ACC == ACC_REF ? (double)mis : mis64;
}

// ---------------------------------------------------------------- elastic FWI
// FwiElastic2D::crossCorr (lib/fwi.cpp:2591-2775) on the interior 1..n-2:
//   g0 -= (Dx Vx_fw + Dz Vz_fw) (Sxx_bw + Szz_bw)                     (lambda)
//   g1 += 2 (Dx Vx Szz + Dz Vz Sxx) - 1/4 sum of 4 Sxz corner products (mu)
//   g2 -= sum of staggered velocity-stress products                     (rho)
template <typename T, bool EXACT, typename G>
__global__ void __launch_bounds__(256) corr_fwi_e2d(const Corr2DE<T> *desc, T dx, T dz)
{
    const Corr2DE<T> c = desc[blockIdx.z];
    const int ix = blockIdx.x * blockDim.x + threadIdx.x;
    const int iz = blockIdx.y * blockDim.y + threadIdx.y;
    if (ix < 1 || iz < 1 || ix >= c.nx - 1 || iz >= c.nz - 1) return;
    const long q = (long)(iz + c.lpml) * c.pitch + ix + c.lpml;
    const long u = (long)iz * c.nx + ix;
    const int P = c.pitch;
    const T *wsx = c.ws[0], *wsz = c.ws[1], *wsxx = c.ws[2], *wszz = c.ws[3], *wsxz = c.ws[4];
    const T *wrx = c.wr[0], *wrz = c.wr[1], *rsxx = c.wr[2], *rszz = c.wr[3], *rsxz = c.wr[4];
    G *g0 = (G *)c.g[0] + u, *g1 = (G *)c.g[1] + u, *g2 = (G *)c.g[2] + u;
    T a, rh;
    double mu;
    if (EXACT) {
        using O = X<T>;
        const T msxx = O::div(O::sub(wsx[q], wsx[q - 1]), dx);
        const T mszz = O::div(O::sub(wsz[q], wsz[q - P]), dz);
        a = O::mul(O::add(msxx, mszz), O::add(rsxx[q], rszz[q]));
        const T m1 = O::add(O::div(O::sub(wsx[q - 1], wsx[q - 1 - P]), dz), O::div(O::sub(wsz[q - P], wsz[q - 1 - P]), dx));
        const T m2 = O::add(O::div(O::sub(wsx[q], wsx[q - P]), dz), O::div(O::sub(wsz[q + 1 - P], wsz[q - P]), dx));
        const T m3 = O::add(O::div(O::sub(wsx[q - 1 + P], wsx[q - 1]), dz), O::div(O::sub(wsz[q], wsz[q - 1]), dx));
        const T m4 = O::add(O::div(O::sub(wsx[q + P], wsx[q]), dz), O::div(O::sub(wsz[q + 1], wsz[q]), dx));
        const T t1 = O::add(O::mul(msxx, rszz[q]), O::mul(mszz, rsxx[q]));
        const T t2 = O::add(O::add(O::add(O::mul(m1, rsxz[q - 1 - P]), O::mul(m2, rsxz[q - P])), O::mul(m3, rsxz[q - 1])),
                            O::mul(m4, rsxz[q]));
        mu = __dsub_rn(__dmul_rn(2.0, (double)t1), __dmul_rn(0.25, (double)t2));
        const double DX = (double)dx, DZ = (double)dz;
        T ux = O::rnd(half_term(wrx[q], c.rx[q], O::sub(wsxx[q + 1], wsxx[q]), DX));
        ux = O::rnd(__dadd_rn((double)ux, half_term(wrx[q - 1], c.rx[q - 1], O::sub(wsxx[q], wsxx[q - 1]), DX)));
        ux = O::rnd(__dadd_rn((double)ux, half_term(wrx[q], c.rx[q], O::sub(wsxz[q], wsxz[q - P]), DZ)));
        ux = O::rnd(__dadd_rn((double)ux, half_term(wrx[q - 1], c.rx[q - 1], O::sub(wsxz[q - 1], wsxz[q - 1 - P]), DZ)));
        T uz = O::rnd(half_term(wrz[q], c.rz[q], O::sub(wsxz[q], wsxz[q - 1]), DX));
        uz = O::rnd(__dadd_rn((double)uz, half_term(wrz[q - P], c.rz[q - P], O::sub(wsxz[q - P], wsxz[q - 1 - P]), DX)));
        uz = O::rnd(__dadd_rn((double)uz, half_term(wrz[q], c.rz[q], O::sub(wszz[q + P], wszz[q]), DZ)));
        uz = O::rnd(__dadd_rn((double)uz, half_term(wrz[q - P], c.rz[q - P], O::sub(wszz[q], wszz[q - P]), DZ)));
        rh = O::add(ux, uz);
    } else {
        const T rdx = T(1) / dx, rdz = T(1) / dz;
        const T msxx = (wsx[q] - wsx[q - 1]) * rdx, mszz = (wsz[q] - wsz[q - P]) * rdz;
        a = (msxx + mszz) * (rsxx[q] + rszz[q]);
        const T m1 = (wsx[q - 1] - wsx[q - 1 - P]) * rdz + (wsz[q - P] - wsz[q - 1 - P]) * rdx;
        const T m2 = (wsx[q] - wsx[q - P]) * rdz + (wsz[q + 1 - P] - wsz[q - P]) * rdx;
        const T m3 = (wsx[q - 1 + P] - wsx[q - 1]) * rdz + (wsz[q] - wsz[q - 1]) * rdx;
        const T m4 = (wsx[q + P] - wsx[q]) * rdz + (wsz[q + 1] - wsz[q]) * rdx;
        mu = (double)(T(2) * (msxx * rszz[q] + mszz * rsxx[q]) -
                      T(0.25) * (m1 * rsxz[q - 1 - P] + m2 * rsxz[q - P] + m3 * rsxz[q - 1] + m4 * rsxz[q]));
        const T ux = wrx[q] * c.rx[q] * ((wsxx[q + 1] - wsxx[q]) * rdx + (wsxz[q] - wsxz[q - P]) * rdz) +
                     wrx[q - 1] * c.rx[q - 1] * ((wsxx[q] - wsxx[q - 1]) * rdx + (wsxz[q - 1] - wsxz[q - 1 - P]) * rdz);
        const T uz = wrz[q] * c.rz[q] * ((wsxz[q] - wsxz[q - 1]) * rdx + (wszz[q + P] - wszz[q]) * rdz) +
                     wrz[q - P] * c.rz[q - P] * ((wsxz[q - P] - wsxz[q - 1 - P]) * rdx + (wszz[q] - wszz[q - P]) * rdz);
        rh = T(0.5) * (ux + uz);
    }
    if (sizeof(G) == sizeof(T)) {
        using O = X<T>;
        *(T *)g0 = EXACT ? O::sub(*(T *)g0, a) : *(T *)g0 - a;
        *(T *)g1 = O::rnd(__dadd_rn((double)*(T *)g1, mu));
        *(T *)g2 = EXACT ? O::sub(*(T *)g2, rh) : *(T *)g2 - rh;
    } else {
        *g0 = __dsub_rn((double)*g0, (double)a);
        *g1 = __dadd_rn((double)*g1, mu);
        *g2 = __dsub_rn((double)*g2, (double)rh);
    }
}

// FwiAcoustic3D::crossCorr (lib/fwi.cpp:1403-1466) on 1..n-1 of the unpadded
// window, one thread per (x, y) column marching z.  The reference's second z term
// takes the adjoint Vz of the cell at y-1 with Rz of the cell at z-1 (as written
// there); it is reproduced as it is.
template <typename T, bool EXACT, typename G>
__global__ void __launch_bounds__(256) corr_fwi_a3d(const Corr3DF<T> *desc, T dx, T dy, T dz)
{
    const Corr3DF<T> c = desc[blockIdx.z];
    const int ix = blockIdx.x * blockDim.x + threadIdx.x;
    const int iy = blockIdx.y * blockDim.y + threadIdx.y;
    if (ix < 1 || iy < 1 || ix >= c.nx || iy >= c.ny) return;
    const long long P = c.pitch, PL = c.plane;
    const int L = c.lpml;
    for (int iz = 1; iz < c.nz; iz++) {
        const long long q = (long long)(iz + L) * PL + (long long)(iy + L) * P + (ix + L);
        const long long u = ((long long)iz * c.ny + iy) * c.nx + ix;
        const T ws = c.wsp[q];
        G *vg = (G *)c.g0 + u, *rg = (G *)c.g1 + u;
        T a, b, ud;
        if (EXACT) {
            using O = X<T>;
            const T vpscale = O::rnd(__ddiv_rn(-2.0, (double)c.vp[u]));
            const T rhoscale1 = O::rnd(__ddiv_rn(-1.0, (double)c.rho[u]));
            const T mrxx = O::div(O::sub(c.wrx[q], c.wrx[q - 1]), dx);
            const T mryy = O::div(O::sub(c.wry[q], c.wry[q - P]), dy);
            const T mrzz = O::div(O::sub(c.wrz[q], c.wrz[q - PL]), dz);
            const T s = O::add(O::add(mrxx, mryy), mrzz);
            a = O::mul(O::mul(vpscale, ws), s);
            b = O::mul(O::mul(rhoscale1, ws), s);
            const double DX = (double)dx, DY = (double)dy, DZ = (double)dz;
            T ux = O::rnd(half_term(c.wrx[q], c.rx[q], O::sub(c.wsp[q + 1], ws), DX));
            ux = O::rnd(__dadd_rn((double)ux, half_term(c.wrx[q - 1], c.rx[q - 1], O::sub(ws, c.wsp[q - 1]), DX)));
            T uy = O::rnd(half_term(c.wry[q], c.ry[q], O::sub(c.wsp[q + P], ws), DY));
            uy = O::rnd(__dadd_rn((double)uy, half_term(c.wry[q - P], c.ry[q - P], O::sub(ws, c.wsp[q - P]), DY)));
            T uz = O::rnd(half_term(c.wrz[q], c.rz[q], O::sub(c.wsp[q + PL], ws), DZ));
            uz = O::rnd(__dadd_rn((double)uz, half_term(c.wrz[q - P], c.rz[q - PL], O::sub(ws, c.wsp[q - PL]), DZ)));
            ud = O::add(O::add(ux, uy), uz);
        } else {
            const T rdx = T(1) / dx, rdy = T(1) / dy, rdz = T(1) / dz;
            const T s = (c.wrx[q] - c.wrx[q - 1]) * rdx + (c.wry[q] - c.wry[q - P]) * rdy + (c.wrz[q] - c.wrz[q - PL]) * rdz;
            a = (T(-2) / c.vp[u]) * ws * s;
            b = (T(-1) / c.rho[u]) * ws * s;
            ud = T(0.5) * ((c.wrx[q] * c.rx[q] * (c.wsp[q + 1] - ws) + c.wrx[q - 1] * c.rx[q - 1] * (ws - c.wsp[q - 1])) * rdx +
                           (c.wry[q] * c.ry[q] * (c.wsp[q + P] - ws) + c.wry[q - P] * c.ry[q - P] * (ws - c.wsp[q - P])) * rdy +
                           (c.wrz[q] * c.rz[q] * (c.wsp[q + PL] - ws) + c.wrz[q - P] * c.rz[q - PL] * (ws - c.wsp[q - PL])) * rdz);
        }
        if (sizeof(G) == sizeof(T)) {
            using O = X<T>;
            *(T *)vg = EXACT ? O::sub(*(T *)vg, a) : *(T *)vg - a;
            const T r1 = EXACT ? O::sub(*(T *)rg, b) : *(T *)rg - b;
            *(T *)rg = EXACT ? O::add(r1, ud) : r1 + ud;
        } else {
            *vg = __dsub_rn((double)*vg, (double)a);
            *rg = __dadd_rn(__dsub_rn((double)*rg, (double)b), (double)ud);
        }
    }
}

// FwiElastic2D::scaleGrad (lib/fwi.cpp:2778-2849): lambda/mu/rho correlations to
// vp/vs/rho gradients, over the whole window.
template <typename T, typename G>
__global__ void __launch_bounds__(256) scale_grad_e2d(const Corr2DE<T> *desc)
{
    const Corr2DE<T> c = desc[blockIdx.z];
    const int ix = blockIdx.x * blockDim.x + threadIdx.x;
    const int iz = blockIdx.y * blockDim.y + threadIdx.y;
    if (ix >= c.nx || iz >= c.nz) return;
    const long u = (long)iz * c.nx + ix;
    const T vp = c.vp[u], vs = c.vs[u], rho = c.rho[u];
    G *g0 = (G *)c.g[0] + u, *g1 = (G *)c.g[1] + u, *g2 = (G *)c.g[2] + u;
    if (sizeof(G) == sizeof(T)) {
        using O = X<T>;
        const T vpscale = O::rnd(__dmul_rn(__dmul_rn(2.0, (double)rho), (double)vp));
        const T vsscale = O::rnd(__dmul_rn(__dmul_rn(2.0, (double)rho), (double)vs));
        const T rs1 = O::rnd(__dsub_rn((double)O::mul(vp, vp), __dmul_rn(__dmul_rn(2.0, (double)vs), (double)vs)));
        const T rs2 = O::mul(vs, vs);
        const T lambda = *(T *)g0, mu = *(T *)g1, r = *(T *)g2;
        *(T *)g0 = O::mul(vpscale, lambda);
        *(T *)g1 = O::rnd(__dsub_rn((double)O::mul(vsscale, mu), __dmul_rn(__dmul_rn(2.0, (double)vsscale), (double)lambda)));
        *(T *)g2 = O::add(O::add(O::mul(rs1, lambda), O::mul(rs2, mu)), r);
    } else {
        const double dvp = vp, dvs = vs, drho = rho;
        const double vpscale = 2.0 * drho * dvp, vsscale = 2.0 * drho * dvs;
        const double lambda = *g0, mu = *g1, r = *g2;
        *g0 = vpscale * lambda;
        *g1 = vsscale * mu - 2.0 * vsscale * lambda;
        *g2 = (dvp * dvp - 2.0 * dvs * dvs) * lambda + dvs * dvs * mu + r;
    }
}

// FwiElastic2D::computeResiduals / computeMisfit, DIFFERENCE (lib/fwi.cpp:2852-2905, 3227-3290)
template <typename T, int ACC>
__global__ void __launch_bounds__(256) residual_misfit_e2d(const Resid2DE<T> *desc, double *misfit)
{
    const Resid2DE<T> d = desc[blockIdx.x];
    const long n = (long)d.nrec * d.nt;
    for (int k = 0; k < 3; k++)
        for (long j = threadIdx.x; j < n; j += blockDim.x) d.res[k][j] = X<T>::sub(d.mod[k][j], d.obs[k][j]);
    if (ACC == ACC_REF) {
        __syncthreads();
        if (threadIdx.x != 0) return;
        // misfit += 0.5*(rp*rp + rx*rx + rz*rz): squares summed in T, then added in double
        T mis = 0;
        for (int tr = 0; tr < d.nrec; tr++) {
            if (d.rec_pt_vx[tr] < 0) continue;
            for (int it = 0; it < d.nt; it++) {
                const long j = (long)tr * d.nt + it;
                const T rp = d.res[0][j], rx = d.res[1][j], rz = d.res[2][j];
                const T s = X<T>::add(X<T>::add(X<T>::mul(rp, rp), X<T>::mul(rx, rx)), X<T>::mul(rz, rz));
                mis = X<T>::rnd(__dadd_rn((double)mis, __dmul_rn(0.5, (double)s)));
            }
        }
        misfit[blockIdx.x] = (double)mis;
    } else {
        double acc = 0.0;
        for (long j = threadIdx.x; j < n; j += blockDim.x) {
            if (d.rec_pt_vx[j / d.nt] < 0) continue;
            for (int k = 0; k < 3; k++) {
                const double r = (double)X<T>::sub(d.mod[k][j], d.obs[k][j]);
                acc = fma(0.5 * r, r, acc);
            }
        }
        __shared__ double red[256];
        red[threadIdx.x] = acc;
        __syncthreads();
        for (int s = blockDim.x / 2; s > 0; s >>= 1) {
            if ((int)threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
            __syncthreads();
        }
        if (threadIdx.x == 0) misfit[blockIdx.x] = red[0];
    }
}

// ---------------------------------------------------------------- checkpoints
template <typename S> struct Store;
template <> struct Store<__half> {
    static __device__ __forceinline__ __half to(float x) { return __float2half_rn(x); }
    static __device__ __forceinline__ float from(__half h) { return __half2float(h); }
};
template <> struct Store<__nv_bfloat16> {
    static __device__ __forceinline__ __nv_bfloat16 to(float x) { return __float2bfloat16_rn(x); }
    static __device__ __forceinline__ float from(__nv_bfloat16 h) { return __bfloat162float(h); }
};

// Power-of-two scale that maps the block's largest magnitude below 2^15 (exact
// scaling; FP16's largest finite value is 65504).  The exponent is kept at or
// above -126 so that the scale and its reciprocal are both normal floats: a block
// whose largest magnitude is itself subnormal (the numerical tails ahead of a
// wavefront in C-PML memory) would otherwise get a zero scale and an infinite
// reciprocal.
__device__ __forceinline__ float pow2_scale(unsigned maxbits)
{
    const float m = __uint_as_float(maxbits);
    if (!(m > 0.0f) || !isfinite(m)) return 1.0f;
    int e;
    frexpf(m, &e);          // m < 2^e
    return ldexpf(1.0f, max(e - 15, -126));
}

// Element offset of row r of a block (rows of a 3D block run plane by plane).
__device__ __forceinline__ long long seg_row(const CkptSeg &s, int r)
{
    if (s.prow <= 0) return (long long)r * s.pitch;
    const int pl = r / s.prow;
    return pl * s.pstride + (long long)(r - pl * s.prow) * s.pitch;
}

// Checkpoint kernels: one warp per row of a block (rows of a 3D block run plane by
// plane), grid.y = block; lanes walk the row with four independent loads in flight
// before their stores, so the copy is not serialised on load latency.
constexpr int CK_WARPS = 8;       // warps (rows in flight) per CTA

// Applies op(src_index, slot_index) to every element of row r of block s, in
// groups of four per lane.
template <typename F>
__device__ __forceinline__ void ck_row(const CkptSeg &s, int r, int lane, F op)
{
    const long long so = seg_row(s, r), dof = s.dst + (long long)r * s.cols;
    int c = lane;
    for (; c + 96 < s.cols; c += 128) op(so + c, dof + c, 4);
    for (; c < s.cols; c += 32) op(so + c, dof + c, 1);
}

template <typename T>
__global__ void __launch_bounds__(256) ckpt_copy_out(const CkptSeg *segs, T *__restrict__ slot)
{
    const CkptSeg s = segs[blockIdx.y];
    const T *__restrict__ src = (const T *)s.src;
    const int lane = threadIdx.x & 31;
    for (int r = blockIdx.x * CK_WARPS + (threadIdx.x >> 5); r < s.rows; r += gridDim.x * CK_WARPS)
        ck_row(s, r, lane, [&](long long i, long long o, int n) {
            if (n == 4) {
                const T a = src[i], b = src[i + 32], c = src[i + 64], d = src[i + 96];
                slot[o] = a; slot[o + 32] = b; slot[o + 64] = c; slot[o + 96] = d;
            } else {
                slot[o] = src[i];
            }
        });
}

template <typename T>
__global__ void __launch_bounds__(256) ckpt_copy_in(const CkptSeg *segs, const T *__restrict__ slot)
{
    const CkptSeg s = segs[blockIdx.y];
    T *__restrict__ dst = (T *)s.src;
    const int lane = threadIdx.x & 31;
    for (int r = blockIdx.x * CK_WARPS + (threadIdx.x >> 5); r < s.rows; r += gridDim.x * CK_WARPS)
        ck_row(s, r, lane, [&](long long i, long long o, int n) {
            if (n == 4) {
                const T a = slot[o], b = slot[o + 32], c = slot[o + 64], d = slot[o + 96];
                dst[i] = a; dst[i + 32] = b; dst[i + 64] = c; dst[i + 96] = d;
            } else {
                dst[i] = slot[o];
            }
        });
}

template <typename T>
__global__ void __launch_bounds__(256) ckpt_maxabs(const CkptSeg *segs, unsigned *maxbits)
{
    const CkptSeg s = segs[blockIdx.y];
    const T *__restrict__ src = (const T *)s.src;
    const int lane = threadIdx.x & 31;
    float m = 0.0f;
    for (int r = blockIdx.x * CK_WARPS + (threadIdx.x >> 5); r < s.rows; r += gridDim.x * CK_WARPS)
        ck_row(s, r, lane, [&](long long i, long long, int n) {
            if (n == 4) {
                const float a = fabsf((float)src[i]), b = fabsf((float)src[i + 32]);
                const float c = fabsf((float)src[i + 64]), d = fabsf((float)src[i + 96]);
                m = fmaxf(m, fmaxf(fmaxf(a, b), fmaxf(c, d)));
            } else {
                m = fmaxf(m, fabsf((float)src[i]));
            }
        });
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (lane == 0 && m > 0.0f) atomicMax(&maxbits[blockIdx.y], __float_as_uint(m));
}

template <typename T, typename S>
__global__ void __launch_bounds__(256) ckpt_pack(const CkptSeg *segs, S *__restrict__ slot, const unsigned *maxbits,
                                                 float *scales)
{
    const CkptSeg s = segs[blockIdx.y];
    const float scale = pow2_scale(maxbits[blockIdx.y]);
    const float inv = 1.0f / scale;            // exact: a power of two
    if (blockIdx.x == 0 && threadIdx.x == 0) scales[blockIdx.y] = scale;
    const T *__restrict__ src = (const T *)s.src;
    const int lane = threadIdx.x & 31;
    for (int r = blockIdx.x * CK_WARPS + (threadIdx.x >> 5); r < s.rows; r += gridDim.x * CK_WARPS)
        ck_row(s, r, lane, [&](long long i, long long o, int n) {
            if (n == 4) {
                const float a = (float)src[i], b = (float)src[i + 32], c = (float)src[i + 64], d = (float)src[i + 96];
                slot[o] = Store<S>::to(a * inv); slot[o + 32] = Store<S>::to(b * inv);
                slot[o + 64] = Store<S>::to(c * inv); slot[o + 96] = Store<S>::to(d * inv);
            } else {
                slot[o] = Store<S>::to((float)src[i] * inv);
            }
        });
}

template <typename T, typename S>
__global__ void __launch_bounds__(256) ckpt_unpack(const CkptSeg *segs, const S *__restrict__ slot, const float *scales)
{
    const CkptSeg s = segs[blockIdx.y];
    const float scale = scales[blockIdx.y];
    T *__restrict__ dst = (T *)s.src;
    const int lane = threadIdx.x & 31;
    for (int r = blockIdx.x * CK_WARPS + (threadIdx.x >> 5); r < s.rows; r += gridDim.x * CK_WARPS)
        ck_row(s, r, lane, [&](long long i, long long o, int n) {
            if (n == 4) {
                const S a = slot[o], b = slot[o + 32], c = slot[o + 64], d = slot[o + 96];
                dst[i] = (T)(Store<S>::from(a) * scale); dst[i + 32] = (T)(Store<S>::from(b) * scale);
                dst[i + 64] = (T)(Store<S>::from(c) * scale); dst[i + 96] = (T)(Store<S>::from(d) * scale);
            } else {
                dst[i] = (T)(Store<S>::from(slot[o]) * scale);
            }
        });
}

// CTAs per block: enough warps for the tallest block's rows, at most 128 CTAs.
inline dim3 ck_grid(int nseg, int max_rows)
{
    const int bx = std::min(128, std::max(1, (max_rows + CK_WARPS - 1) / CK_WARPS));
    return dim3((unsigned)bx, (unsigned)nseg);
}

template <typename T>
cudaError_t ckpt_save_t(int ck, const CkptSeg *segs, int nseg, int max_rows, void *slot, float *scales,
                        unsigned *maxbits, cudaStream_t st)
{
    const dim3 grid = ck_grid(nseg, max_rows);
    if (ck == CK_NATIVE) {
        ckpt_copy_out<T><<<grid, 256, 0, st>>>(segs, (T *)slot);
        return cudaGetLastError();
    }
    cudaError_t e = cudaMemsetAsync(maxbits, 0, sizeof(unsigned) * nseg, st);
    if (e != cudaSuccess) return e;
    ckpt_maxabs<T><<<grid, 256, 0, st>>>(segs, maxbits);
    if (ck == CK_F16) ckpt_pack<T, __half><<<grid, 256, 0, st>>>(segs, (__half *)slot, maxbits, scales);
    else ckpt_pack<T, __nv_bfloat16><<<grid, 256, 0, st>>>(segs, (__nv_bfloat16 *)slot, maxbits, scales);
    return cudaGetLastError();
}

template <typename T>
cudaError_t ckpt_load_t(int ck, const CkptSeg *segs, int nseg, int max_rows, const void *slot, const float *scales,
                        cudaStream_t st)
{
    const dim3 grid = ck_grid(nseg, max_rows);
    if (ck == CK_NATIVE) ckpt_copy_in<T><<<grid, 256, 0, st>>>(segs, (const T *)slot);
    else if (ck == CK_F16) ckpt_unpack<T, __half><<<grid, 256, 0, st>>>(segs, (const __half *)slot, scales);
    else ckpt_unpack<T, __nv_bfloat16><<<grid, 256, 0, st>>>(segs, (const __nv_bfloat16 *)slot, scales);
    return cudaGetLastError();
}

template <typename T, bool EXACT>
cudaError_t corr_fwi_t(int acc, const void *desc, int nshots, int nxmax, int nzmax, double dx, double dz,
                       cudaStream_t st)
{
    const dim3 block(32, 8), grid((nxmax + 31) / 32, (nzmax + 7) / 8, nshots);
    if (acc == ACC_F64)
        corr_fwi_a2d<T, EXACT, double><<<grid, block, 0, st>>>((const Corr2D<T> *)desc, (T)dx, (T)dz);
    else
        corr_fwi_a2d<T, EXACT, T><<<grid, block, 0, st>>>((const Corr2D<T> *)desc, (T)dx, (T)dz);
    return cudaGetLastError();
}

template <typename T, bool EXACT>
cudaError_t corr_rtm_t(int acc, const void *desc, int nshots, int nxmax, int nzmax, int nhx, int nhz, cudaStream_t st)
{
    const dim3 block(32, 8), grid((nxmax + 31) / 32, (nzmax + 7) / 8, nshots);
    if (acc == ACC_F64) corr_rtm_a2d<T, EXACT, double><<<grid, block, 0, st>>>((const Corr2D<T> *)desc, nhx, nhz);
    else corr_rtm_a2d<T, EXACT, T><<<grid, block, 0, st>>>((const Corr2D<T> *)desc, nhx, nhz);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_corr_fwi_a2d(int prec, int acc, const void *desc, int nshots, int nxmax, int nzmax, double dx,
                                double dz, cudaStream_t st)
{
    if (prec == PREC_F64) return corr_fwi_t<double, true>(acc, desc, nshots, nxmax, nzmax, dx, dz, st);
    if (prec == PREC_F32_EXACT) return corr_fwi_t<float, true>(acc, desc, nshots, nxmax, nzmax, dx, dz, st);
    return corr_fwi_t<float, false>(acc, desc, nshots, nxmax, nzmax, dx, dz, st);
}

cudaError_t launch_corr_rtm_a2d(int prec, int acc, const void *desc, int nshots, int nxmax, int nzmax, int nhx,
                                int nhz, cudaStream_t st)
{
    if (prec == PREC_F64) return corr_rtm_t<double, true>(acc, desc, nshots, nxmax, nzmax, nhx, nhz, st);
    if (prec == PREC_F32_EXACT) return corr_rtm_t<float, true>(acc, desc, nshots, nxmax, nzmax, nhx, nhz, st);
    return corr_rtm_t<float, false>(acc, desc, nshots, nxmax, nzmax, nhx, nhz, st);
}

cudaError_t launch_corr_rtm_a3d(int prec, int acc, const void *desc, int nshots, int nxmax, int nymax, int nhx,
                                int nhy, int nhz, cudaStream_t st)
{
    const dim3 block(32, 8), grid((nxmax + 31) / 32, (nymax + 7) / 8, nshots);
    if (prec == PREC_F64) corr_rtm_a3d<double, true, double><<<grid, block, 0, st>>>((const Corr3D<double> *)desc, nhx, nhy, nhz);
    else if (acc == ACC_F64) {
        if (prec == PREC_F32_EXACT) corr_rtm_a3d<float, true, double><<<grid, block, 0, st>>>((const Corr3D<float> *)desc, nhx, nhy, nhz);
        else corr_rtm_a3d<float, false, double><<<grid, block, 0, st>>>((const Corr3D<float> *)desc, nhx, nhy, nhz);
    } else {
        if (prec == PREC_F32_EXACT) corr_rtm_a3d<float, true, float><<<grid, block, 0, st>>>((const Corr3D<float> *)desc, nhx, nhy, nhz);
        else corr_rtm_a3d<float, false, float><<<grid, block, 0, st>>>((const Corr3D<float> *)desc, nhx, nhy, nhz);
    }
    return cudaGetLastError();
}

cudaError_t launch_corr_fwi_a3d(int prec, int acc, const void *desc, int nshots, int nxmax, int nymax, double dx,
                                double dy, double dz, cudaStream_t st)
{
    const dim3 block(32, 8), grid((nxmax + 31) / 32, (nymax + 7) / 8, nshots);
    if (prec == PREC_F64)
        corr_fwi_a3d<double, true, double><<<grid, block, 0, st>>>((const Corr3DF<double> *)desc, dx, dy, dz);
    else if (prec == PREC_F32_EXACT) {
        if (acc == ACC_F64) corr_fwi_a3d<float, true, double><<<grid, block, 0, st>>>((const Corr3DF<float> *)desc, (float)dx, (float)dy, (float)dz);
        else corr_fwi_a3d<float, true, float><<<grid, block, 0, st>>>((const Corr3DF<float> *)desc, (float)dx, (float)dy, (float)dz);
    } else {
        if (acc == ACC_F64) corr_fwi_a3d<float, false, double><<<grid, block, 0, st>>>((const Corr3DF<float> *)desc, (float)dx, (float)dy, (float)dz);
        else corr_fwi_a3d<float, false, float><<<grid, block, 0, st>>>((const Corr3DF<float> *)desc, (float)dx, (float)dy, (float)dz);
    }
    return cudaGetLastError();
}

template <bool CLIP>
static void launch_corr(int prec, int acc, const void *desc, int nshots, size_t sm, double *misfit, cudaStream_t st)
{
    if (prec == PREC_F64) {
        if (acc == ACC_F64) residual_corr<double, ACC_F64, CLIP><<<nshots, 256, sm, st>>>((const Resid2D<double> *)desc, misfit);
        else residual_corr<double, ACC_REF, CLIP><<<nshots, 256, sm, st>>>((const Resid2D<double> *)desc, misfit);
    } else {
        if (acc == ACC_F64) residual_corr<float, ACC_F64, CLIP><<<nshots, 256, sm, st>>>((const Resid2D<float> *)desc, misfit);
        else residual_corr<float, ACC_REF, CLIP><<<nshots, 256, sm, st>>>((const Resid2D<float> *)desc, misfit);
    }
}

cudaError_t launch_residual_corr(int prec, int acc, const void *desc, int nshots, int nrec_max, double *misfit,
                                 cudaStream_t st, bool clip)
{
    const size_t sm = (size_t)std::max(nrec_max, 1) * (prec == PREC_F64 ? 8 : 4);
    if (clip) launch_corr<true>(prec, acc, desc, nshots, sm, misfit, st);
    else launch_corr<false>(prec, acc, desc, nshots, sm, misfit, st);
    return cudaGetLastError();
}

cudaError_t launch_residual_corr_e2d(int prec, int acc, const void *desc, int nshots, int nrec_max, double *misfit,
                                     cudaStream_t st)
{
    const size_t sm = 3 * (size_t)std::max(nrec_max, 1) * (prec == PREC_F64 ? 8 : 4);
    if (prec == PREC_F64) {
        if (acc == ACC_F64) residual_corr_e2d<double, ACC_F64><<<nshots, 256, sm, st>>>((const Resid2DE<double> *)desc, misfit);
        else residual_corr_e2d<double, ACC_REF><<<nshots, 256, sm, st>>>((const Resid2DE<double> *)desc, misfit);
    } else {
        if (acc == ACC_F64) residual_corr_e2d<float, ACC_F64><<<nshots, 256, sm, st>>>((const Resid2DE<float> *)desc, misfit);
        else residual_corr_e2d<float, ACC_REF><<<nshots, 256, sm, st>>>((const Resid2DE<float> *)desc, misfit);
    }
    return cudaGetLastError();
}

// Image2D::stackImage (lib/image.cpp:348-438) of every shot's window into one global
// image per component: one thread per global point (and lag), the shots added in
// their order, each where its window covers the point.
template <typename G>
__global__ void __launch_bounds__(256) stack_windows(const StackWin *w, int nshots, int ncomp, int nxg, int nzg, int nh,
                                                     G *out0, G *out1, G *out2)
{
    const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long ng = (long long)nxg * nzg;
    if (k >= ng * nh) return;
    const int ih = (int)(k / ng);
    const int iz = (int)((k % ng) / nxg), ix = (int)(k % nxg);
    G *out[3] = {out0, out1, out2};
    for (int c = 0; c < ncomp; c++) {
        G acc = out[c][k];
        for (int i = 0; i < nshots; i++) {
            const StackWin &s = w[i];
            const int lx = ix - s.x0, lz = iz - s.z0;
            if (lx < 0 || lx >= s.nx || lz < 0 || lz >= s.nz) continue;
            const G v = ((const G *)s.g[c])[((long long)ih * s.nz + lz) * s.nx + lx];
            if (sizeof(G) == 4) acc = (G)__fadd_rn((float)acc, (float)v);
            else acc = (G)__dadd_rn((double)acc, (double)v);
        }
        out[c][k] = acc;
    }
}

template <typename T, int ACC>
void residual_t(const void *desc, int nshots, double *misfit, double *partials, cudaStream_t st)
{
    residual_diff<T, ACC><<<dim3(RES_BLOCKS, nshots), 256, 0, st>>>((const Resid2D<T> *)desc, partials);
    residual_sum<T, ACC><<<nshots, 32, 0, st>>>((const Resid2D<T> *)desc, partials, misfit);
}

size_t residual_partials(int nshots) { return (size_t)nshots * RES_BLOCKS; }

cudaError_t launch_stack_windows(int gbytes, const StackWin *w, int nshots, int ncomp, int nxg, int nzg, int nh,
                                 void *out0, void *out1, void *out2, cudaStream_t st)
{
    const long long n = (long long)nxg * nzg * nh;
    const unsigned grid = (unsigned)((n + 255) / 256);
    if (gbytes == 8)
        stack_windows<double><<<grid, 256, 0, st>>>(w, nshots, ncomp, nxg, nzg, nh, (double *)out0, (double *)out1,
                                                     (double *)out2);
    else
        stack_windows<float><<<grid, 256, 0, st>>>(w, nshots, ncomp, nxg, nzg, nh, (float *)out0, (float *)out1,
                                                   (float *)out2);
    return cudaGetLastError();
}

cudaError_t launch_residual(int prec, int acc, const void *desc, int nshots, double *misfit, double *partials,
                            cudaStream_t st)
{
    if (prec == PREC_F64) {
        if (acc == ACC_F64) residual_t<double, ACC_F64>(desc, nshots, misfit, partials, st);
        else residual_t<double, ACC_REF>(desc, nshots, misfit, partials, st);
    } else {
        if (acc == ACC_F64) residual_t<float, ACC_F64>(desc, nshots, misfit, partials, st);
        else residual_t<float, ACC_REF>(desc, nshots, misfit, partials, st);
    }
    return cudaGetLastError();
}

cudaError_t launch_corr_fwi_e2d(int prec, int acc, const void *desc, int nshots, int nxmax, int nzmax, double dx,
                                double dz, cudaStream_t st)
{
    const dim3 block(32, 8), grid((nxmax + 31) / 32, (nzmax + 7) / 8, nshots);
    if (prec == PREC_F64) {
        if (acc == ACC_F64) corr_fwi_e2d<double, true, double><<<grid, block, 0, st>>>((const Corr2DE<double> *)desc, dx, dz);
        else corr_fwi_e2d<double, true, double><<<grid, block, 0, st>>>((const Corr2DE<double> *)desc, dx, dz);
    } else if (prec == PREC_F32_EXACT) {
        if (acc == ACC_F64) corr_fwi_e2d<float, true, double><<<grid, block, 0, st>>>((const Corr2DE<float> *)desc, (float)dx, (float)dz);
        else corr_fwi_e2d<float, true, float><<<grid, block, 0, st>>>((const Corr2DE<float> *)desc, (float)dx, (float)dz);
    } else {
        if (acc == ACC_F64) corr_fwi_e2d<float, false, double><<<grid, block, 0, st>>>((const Corr2DE<float> *)desc, (float)dx, (float)dz);
        else corr_fwi_e2d<float, false, float><<<grid, block, 0, st>>>((const Corr2DE<float> *)desc, (float)dx, (float)dz);
    }
    return cudaGetLastError();
}

cudaError_t launch_scale_grad_e2d(int prec, int acc, const void *desc, int nshots, int nxmax, int nzmax, cudaStream_t st)
{
    const dim3 block(32, 8), grid((nxmax + 31) / 32, (nzmax + 7) / 8, nshots);
    if (prec == PREC_F64) scale_grad_e2d<double, double><<<grid, block, 0, st>>>((const Corr2DE<double> *)desc);
    else if (acc == ACC_F64) scale_grad_e2d<float, double><<<grid, block, 0, st>>>((const Corr2DE<float> *)desc);
    else scale_grad_e2d<float, float><<<grid, block, 0, st>>>((const Corr2DE<float> *)desc);
    return cudaGetLastError();
}

cudaError_t launch_residual_e2d(int prec, int acc, const void *desc, int nshots, double *misfit, cudaStream_t st)
{
    if (prec == PREC_F64) {
        if (acc == ACC_F64) residual_misfit_e2d<double, ACC_F64><<<nshots, 256, 0, st>>>((const Resid2DE<double> *)desc, misfit);
        else residual_misfit_e2d<double, ACC_REF><<<nshots, 256, 0, st>>>((const Resid2DE<double> *)desc, misfit);
    } else {
        if (acc == ACC_F64) residual_misfit_e2d<float, ACC_F64><<<nshots, 256, 0, st>>>((const Resid2DE<float> *)desc, misfit);
        else residual_misfit_e2d<float, ACC_REF><<<nshots, 256, 0, st>>>((const Resid2DE<float> *)desc, misfit);
    }
    return cudaGetLastError();
}

cudaError_t launch_ckpt_save(int prec, int ck, const CkptSeg *segs, int nseg, int max_rows, void *slot, float *scales,
                             unsigned *maxbits, cudaStream_t st)
{
    return prec == PREC_F64 ? ckpt_save_t<double>(ck, segs, nseg, max_rows, slot, scales, maxbits, st)
                            : ckpt_save_t<float>(ck, segs, nseg, max_rows, slot, scales, maxbits, st);
}

cudaError_t launch_ckpt_load(int prec, int ck, const CkptSeg *segs, int nseg, int max_rows, const void *slot,
                             const float *scales, cudaStream_t st)
{
    return prec == PREC_F64 ? ckpt_load_t<double>(ck, segs, nseg, max_rows, slot, scales, st)
                            : ckpt_load_t<float>(ck, segs, nseg, max_rows, slot, scales, st);
}

}  // namespace rsgpu
