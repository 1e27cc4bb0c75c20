// ADAPTIVE_GAUSS / ADAPTIVE_LINEAR / ADAPTIVE_SINGLE misfits and residuals of the FWI
// drivers (FwiAcoustic2D::computeMisfit / computeResiduals, lib/fwi.cpp:646-751,
// 851-1026; FwiAcoustic3D, lib/fwi.cpp:1541-1631, 1725-1842; FwiElastic2D below).
//
// Per trace the reference designs a Wiener shaping filter w that turns the
// observed trace d into the modelled trace u: with R the (whitened) Toeplitz
// autocorrelation matrix of d and c the cross-correlation of d with u, R w = c is
// solved by Levinson recursion.  The misfit penalises filter energy away from zero
// lag, sum (H(t) w(t))^2 / (2 |w|^2), with H a Gaussian (ADAPTIVE_GAUSS, width 1 %
// of the trace, the misfit counted negative) or a ramp clipped at 500 samples
// (ADAPTIVE_LINEAR).  The residual is the adjoint source of that misfit: the
// weighted filter is passed back through the same Toeplitz system and convolved
// with d.  The 2D drivers then zero the residual samples whose magnitude reaches
// the 97th-percentile value of the shot (the same clip as the CORRELATION misfit).
//
// The arithmetic follows the reference operation by operation in the element
// type, with the double-precision sub-expressions that C's usual conversions
// create; sums run in the reference's order:
//   * cross-correlations and the convolution use the index ranges and the
//     summation order of the Seismic Unix conv/xcor routines that the reference
//     carries (Fwi::convolve, Fwi::xcor, lib/fwi.cpp:189-397): every output is an
//     independent sum over the overlap, ascending in the index of the first
//     operand except in the "rolling on" range of the paired loop, which runs
//     descending.  A host walk over the routine's index regions (conv_flags)
//     labels each output, and one lane of the warp computes each output.
//   * the Toeplitz solver is Levinson's recursion as in Fwi::stoep
//     (lib/fwi.cpp:152-187, after Claerbout, FGDP p. 57): the two inner products
//     of each order are sequential sums, computed side by side by lanes 0 and 1;
//     the updates of the prediction filter and of the solution are independent per
//     index and spread over the warp.
// One warp per trace; the per-trace arrays live in a work buffer of 5*nt values.
//
// The elastic gradient (FwiElastic2D, lib/fwi.cpp:3002-3196, 3428-3753) shapes the
// Ux and Uz traces the same way, each with its own filter, clips the two together
// (both lose the samples where |Ux residual| reaches the larger of the two
// 97th-percentile magnitudes) and counts 0.5 (|Hw_x|^2/|w_x|^2 + |Hw_z|^2/|w_z|^2);
// ADAPTIVE_SINGLE joins the Ux and Uz traces end to end (2 nt samples), designs one
// nt-sample filter from the joined traces' correlations, convolves it with the joined
// observed trace and splits the 2 nt outputs into the Ux and Uz residuals (9*nt work
// values per trace: the joined traces are copied in).  The P residual is zero.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <cuda_runtime.h>

#include "adjoint_ops.cuh"
#include "rsgpu_adjoint.h"
#include "rsgpu_kernels.h"

namespace rsgpu {
namespace {

enum : unsigned char { FL_DESC = 1, FL_LEAD = 2, FL_ZERO = 4 };

constexpr double STDEV_FRAC = 0.01;      // Gaussian width as a fraction of nt (fwi.h STDEV)
constexpr double RAMP_MAX = 500;         // ramp clip of ADAPTIVE_LINEAR (fwi.h HMAX)
constexpr double WHITEN = 0.01;          // prewhitening of the autocorrelation (fwi.h PNOISE_ACOUSTIC and PNOISE_ELASTIC)

// Labels the outputs z[ifz .. ifz+lz-1] of z = x (*) y, x on [ifx, ifx+lx-1] and y on
// [ify, ify+ly-1] (lx <= ly), by the region of the Seismic Unix convolution loop that
// writes them: zero outside the overlap; a descending sum (with a leading x*0 term
// in the first output of each pair) for the paired outputs of the rolling-on range;
// an ascending sum everywhere else, with a leading x*0 term in the second output of
// each pair of the rolling-off range.
void conv_flags(int lx, int ifx, int ly, int ify, int lz, int ifz, unsigned char *fl)
{
    const int ilx = ifx + lx - 1, ily = ify + ly - 1, ilz = ifz + lz - 1;
    auto F = [&](int i) -> unsigned char & { return fl[i - ifz]; };
    int i = ifz;
    for (; i <= std::min(ify + ifx - 1, ilz); ++i) F(i) = FL_ZERO;
    // rolling on: a single output first when its overlap has an even number of terms
    if (i < ify + ilx && i <= ilz && (i - ify - ifx) % 2) F(i++) = 0;
    int ih = std::min(ilx + ify - 1, ilz);
    for (; i < ih; i += 2) {
        F(i) = FL_DESC | FL_LEAD;
        F(i + 1) = FL_DESC;
    }
    if (i == ih) F(i++) = 0;
    // full overlap
    ih = std::min(ily + ifx, ilz);
    for (; i < ih; i += 2) F(i) = F(i + 1) = 0;
    if (i == ih) F(i++) = 0;
    // rolling off: a single output first when its overlap has an odd number of terms
    if (i <= ily + ilx && i <= ilz && (ilx - (i - ily)) % 2 == 0) F(i++) = 0;
    ih = std::min(ily + ilx, ilz);
    for (; i < ih; i += 2) {
        F(i) = 0;
        F(i + 1) = FL_LEAD;
    }
    if (i == ih) F(i++) = 0;
    for (; i <= ilz; ++i) F(i) = FL_ZERO;
}

// Output i of x (*) y over the overlap j in [max(ifx, i-ily), min(ilx, i-ify)] in the
// order `fl` names.  REV reads x reversed (x[k] at index ifx+lx-1-k), which turns the
// convolution into the cross-correlation of Fwi::xcor.
template <typename T, bool REV>
__device__ T conv_out(const T *x, int lx, int ifx, const T *y, int ly, int ify, int i, unsigned char fl)
{
    if (fl & FL_ZERO) return T(0);
    const int ilx = ifx + lx - 1, ily = ify + ly - 1;
    auto xv = [&](int j) { return REV ? x[lx - 1 - (j - ifx)] : x[j - ifx]; };
    const int jlo = max(ifx, i - ily), jhi = min(ilx, i - ify);
    T s = T(0);
    if (fl & FL_DESC) {
        if (fl & FL_LEAD) s = X<T>::add(s, X<T>::mul(xv(jhi + 1), T(0)));
        for (int j = jhi; j >= jlo; --j) s = X<T>::add(s, X<T>::mul(xv(j), y[i - j - ify]));
    } else {
        if (fl & FL_LEAD) s = X<T>::add(s, X<T>::mul(xv(jlo - 1), T(0)));
        for (int j = jlo; j <= jhi; ++j) s = X<T>::add(s, X<T>::mul(xv(j), y[i - j - ify]));
    }
    return s;
}

// Levinson recursion for the symmetric Toeplitz system R f = g (R's first column r,
// r[0] != 0); a is the prediction-error filter.  All 32 lanes call it.
template <typename T>
__device__ void toeplitz_solve(int n, const T *r, const T *g, T *f, T *a, int lane)
{
    if (lane == 0) {
        a[0] = T(1);
        f[0] = X<T>::div(g[0], r[0]);
    }
    T v = r[0];
    __syncwarp();
    for (int j = 1; j < n; j++) {
        // lane 0: e = a . r(j..1); lane 1: w = f . r(j..1), both over the previous order
        T s = T(0);
        if (lane < 2) {
            const T *p = lane == 0 ? a : f;
            for (int i = 0; i < j; i++) s = X<T>::add(s, X<T>::mul(p[i], r[j - i]));
            if (lane == 0) a[j] = T(0);
            else f[j] = T(0);
        }
        const T e = __shfl_sync(0xffffffffu, s, 0), w = __shfl_sync(0xffffffffu, s, 1);
        __syncwarp();
        T c = X<T>::div(e, v);
        v = X<T>::sub(v, X<T>::mul(c, e));
        for (int i = lane; i <= j / 2; i += 32) {
            const T ai = a[i], aji = a[j - i];
            const T bot = X<T>::sub(aji, X<T>::mul(c, ai));
            a[i] = X<T>::sub(ai, X<T>::mul(c, aji));
            a[j - i] = bot;
        }
        __syncwarp();
        c = X<T>::div(X<T>::sub(w, g[j]), v);
        for (int i = lane; i <= j; i += 32) f[i] = X<T>::sub(f[i], X<T>::mul(c, a[j - i]));
        __syncwarp();
    }
}

template <typename T>
__device__ __forceinline__ const T *weights(const unsigned char *tab) { return (const T *)tab; }

// One warp per trace: shaping filter, its norm, the residual.
template <typename T, int MODE>
__global__ void __launch_bounds__(128) adaptive_shape(const Resid2D<T> *desc, const unsigned char *tab, int nt)
{
    const int lane = threadIdx.x & 31;
    const Resid2D<T> d = desc[blockIdx.y];
    const int tr = blockIdx.x * 4 + (threadIdx.x >> 5);
    if (tr >= d.nrec) return;
    const T *H = weights<T>(tab);
    const unsigned char *fx = tab + (size_t)nt * sizeof(T), *fc = fx + nt;
    const T *m = d.mod + (long)tr * nt, *o = d.obs + (long)tr * nt;
    T *r = d.work + (long)tr * 5 * nt, *g = r + nt, *f = g + nt, *a = f + nt, *s1 = a + nt;
    // autocorrelation of the observed trace (the matrix) and its correlation with
    // the modelled trace (the right-hand side)
    for (int i = lane; i < nt; i += 32) {
        r[i] = conv_out<T, true>(o, nt, 1 - nt, o, nt, 0, i, fx[i]);
        g[i] = conv_out<T, true>(o, nt, 1 - nt, m, nt, 0, i, fx[i]);
    }
    __syncwarp();
    if (lane == 0) {
        T r0 = r[0];
        if (r0 == T(0)) r0 = T(1);
        r[0] = X<T>::rnd(__dmul_rn((double)r0, 1.0 + WHITEN));
    }
    __syncwarp();
    toeplitz_solve(nt, r, g, f, a, lane);
    T norm = T(0), mis = T(0);
    if (lane == 0) {
        for (int it = 0; it < nt; it++) norm = X<T>::add(norm, X<T>::mul(f[it], f[it]));
        if (norm == T(0)) norm = T(1);
        // the trace's own misfit, in the element type (computeResiduals)
        for (int it = 0; it < nt; it++) {
            const double hs = (double)X<T>::mul(H[it], f[it]);
            mis = X<T>::rnd(__dadd_rn((double)mis, __ddiv_rn(__dmul_rn(__dmul_rn(0.5, hs), hs), (double)norm)));
        }
        d.tnorm[tr] = norm;
    }
    norm = __shfl_sync(0xffffffffu, norm, 0);
    mis = __shfl_sync(0xffffffffu, mis, 0);
    // -(H^2 - 2 misfit) w / |w|^2 (GAUSS) or (H^2 - 2 misfit) w / |w|^2 (LINEAR),
    // pressure data (scaling 1)
    const double sgn = MODE == ADAPT_GAUSS ? -1.0 : 1.0;
    for (int i = lane; i < nt; i += 32) {
        s1[i] = f[i];
        const double t = __dsub_rn((double)X<T>::mul(H[i], H[i]), __dmul_rn(2.0, (double)mis));
        g[i] = X<T>::rnd(__ddiv_rn(__dmul_rn(sgn * t, (double)f[i]), (double)norm));
    }
    __syncwarp();
    toeplitz_solve(nt, r, g, f, a, lane);
    T *res = d.res + (long)tr * nt;
    for (int i = lane; i < nt; i += 32) res[i] = conv_out<T, false>(f, nt, 0, o, nt, 0, i, fc[i]);
}

// One CTA per shot: the 97th-percentile clip (2D) and the misfit over the traces on
// the grid, traces then samples (computeMisfit).
template <typename T, int ACC, int MODE, bool CLIP>
__global__ void __launch_bounds__(256) adaptive_finish(const Resid2D<T> *desc, const unsigned char *tab,
                                                       double *misfit)
{
    using U = typename Bits<T>::U;
    const Resid2D<T> d = desc[blockIdx.x];
    const int nt = d.nt;
    const long n = (long)d.nrec * nt;
    if (CLIP) {
        const long pos = (long)((97ull * (unsigned long long)nt * (unsigned long long)d.nrec) / 100ull);
        const U clip = kth_mag_bits(d.res, n, pos);
        for (long k = threadIdx.x; k < n; k += blockDim.x)
            if (mag_bits(d.res[k]) >= clip) d.res[k] = T(0);
    }
    if (threadIdx.x != 0) return;
    const T *H = weights<T>(tab);
    T mis = T(0);
    double mis64 = 0.0;
    for (int tr = 0; tr < d.nrec; tr++) {
        if (d.rec_pt[tr] < 0) continue;
        const T *w = d.work + (long)tr * 5 * nt + 4L * nt;
        const double norm = (double)d.tnorm[tr];
        for (int it = 0; it < nt; it++) {
            const double hs = (double)X<T>::mul(H[it], w[it]);
            const double term = __ddiv_rn(__dmul_rn(__dmul_rn(0.5, hs), hs), norm);
            if (ACC == ACC_REF)
                mis = X<T>::rnd(MODE == ADAPT_GAUSS ? __dsub_rn((double)mis, term) : __dadd_rn((double)mis, term));
            else
                mis64 = MODE == ADAPT_GAUSS ? mis64 - term : mis64 + term;
        }
    }
    misfit[blockIdx.x] = ACC == ACC_REF ? (double)mis : mis64;
}

// ADAPTIVE_SINGLE, one warp per trace: the Ux and Uz traces joined end to end.
template <typename T>
__global__ void __launch_bounds__(128) adaptive_shape_single(const Resid2DE<T> *desc, const unsigned char *tab, int nt)
{
    const int lane = threadIdx.x & 31;
    const Resid2DE<T> d = desc[blockIdx.y];
    const int tr = blockIdx.x * 4 + (threadIdx.x >> 5);
    if (tr >= d.nrec) return;
    const T *H = weights<T>(tab);
    const unsigned char *fx = tab + (size_t)nt * sizeof(T), *fc = fx + nt;
    const int n2 = 2 * nt;
    T *r = d.work[0] + (long)tr * 9 * nt, *g = r + nt, *f = g + nt, *a = f + nt, *s1 = a + nt;
    T *jo = s1 + nt, *jm = jo + n2;            // joined observed and modelled traces
    const long t0 = (long)tr * nt;
    for (int i = lane; i < nt; i += 32) {
        jo[i] = d.obs[1][t0 + i];
        jo[nt + i] = d.obs[2][t0 + i];
        jm[i] = d.mod[1][t0 + i];
        jm[nt + i] = d.mod[2][t0 + i];
    }
    __syncwarp();
    for (int i = lane; i < nt; i += 32) {
        r[i] = conv_out<T, true>(jo, n2, 1 - n2, jo, n2, 0, i, fx[i]);
        g[i] = conv_out<T, true>(jo, n2, 1 - n2, jm, n2, 0, i, fx[i]);
    }
    __syncwarp();
    if (lane == 0) {
        T r0 = r[0];
        if (r0 == T(0)) r0 = T(1);
        r[0] = X<T>::rnd(__dmul_rn((double)r0, 1.0 + WHITEN));
    }
    __syncwarp();
    toeplitz_solve(nt, r, g, f, a, lane);
    T norm = T(0), mis = T(0);
    if (lane == 0) {
        for (int it = 0; it < nt; it++) norm = X<T>::add(norm, X<T>::mul(f[it], f[it]));
        if (norm == T(0)) norm = T(1);
        for (int it = 0; it < nt; it++) {
            const double hs = (double)X<T>::mul(H[it], f[it]);
            mis = X<T>::rnd(__dadd_rn((double)mis, __ddiv_rn(__dmul_rn(__dmul_rn(0.5, hs), hs), (double)norm)));
        }
        d.tnorm[0][tr] = norm;
    }
    norm = __shfl_sync(0xffffffffu, norm, 0);
    mis = __shfl_sync(0xffffffffu, mis, 0);
    for (int i = lane; i < nt; i += 32) {
        s1[i] = f[i];
        const double t = __dsub_rn((double)X<T>::mul(H[i], H[i]), __dmul_rn(2.0, (double)mis));
        g[i] = X<T>::rnd(__ddiv_rn(__dmul_rn(t, (double)f[i]), (double)norm));
    }
    __syncwarp();
    toeplitz_solve(nt, r, g, f, a, lane);
    for (int i = lane; i < n2; i += 32) {
        const T v = conv_out<T, false>(f, nt, 0, jo, n2, 0, i, fc[i]);
        if (i < nt) d.res[1][t0 + i] = v;
        else d.res[2][t0 + i - nt] = v;
    }
}

// One CTA per shot of the elastic gradient: zero P residual, the joint Ux/Uz clip
// (not for ADAPTIVE_SINGLE), the misfit over the traces whose Ux map is on the grid.
template <typename T, int ACC, int MODE>
__global__ void __launch_bounds__(256) adaptive_finish_e2d(const Resid2DE<T> *desc, const unsigned char *tab,
                                                           double *misfit)
{
    const Resid2DE<T> d = desc[blockIdx.x];
    const int nt = d.nt;
    const long n = (long)d.nrec * nt;
    for (long k = threadIdx.x; k < n; k += blockDim.x) d.res[0][k] = T(0);
    if (MODE != ADAPT_SINGLE) {
        const long pos = (long)((97ull * (unsigned long long)nt * (unsigned long long)d.nrec) / 100ull);
        T cx = from_bits<T>(kth_mag_bits(d.res[1], n, pos));
        const T cz = from_bits<T>(kth_mag_bits(d.res[2], n, pos));
        if (cz > cx) cx = cz;
        for (long k = threadIdx.x; k < n; k += blockDim.x)
            if (fabs(d.res[1][k]) >= cx) {
                d.res[1][k] = T(0);
                d.res[2][k] = T(0);
            }
    }
    if (threadIdx.x != 0) return;
    const T *H = weights<T>(tab);
    const int stride = (int)(MODE == ADAPT_SINGLE ? 9 : 5);
    T mis = T(0);
    double mis64 = 0.0;
    for (int tr = 0; tr < d.nrec; tr++) {
        if (d.rec_pt_vx[tr] < 0) continue;
        const T *wx = d.work[0] + (long)tr * stride * nt + 4L * nt;
        const T nx = d.tnorm[0][tr];
        const T *wz = MODE == ADAPT_SINGLE ? wx : d.work[1] + (long)tr * 5 * nt + 4L * nt;
        const T nz = MODE == ADAPT_SINGLE ? nx : d.tnorm[1][tr];
        for (int it = 0; it < nt; it++) {
            // 0.5*(rx*rx/nx + rz*rz/nz) with the sum in the element type (0.5*(rx*rx/nx) for SINGLE)
            const T rx = X<T>::mul(H[it], wx[it]);
            T sum = X<T>::div(X<T>::mul(rx, rx), nx);
            if (MODE != ADAPT_SINGLE) {
                const T rz = X<T>::mul(H[it], wz[it]);
                sum = X<T>::add(sum, X<T>::div(X<T>::mul(rz, rz), nz));
            }
            const double term = __dmul_rn(0.5, (double)sum);
            if (ACC == ACC_REF)
                mis = X<T>::rnd(MODE == ADAPT_GAUSS ? __dsub_rn((double)mis, term) : __dadd_rn((double)mis, term));
            else
                mis64 = MODE == ADAPT_GAUSS ? mis64 - term : mis64 + term;
        }
    }
    misfit[blockIdx.x] = ACC == ACC_REF ? (double)mis : mis64;
}

template <typename T>
void fill_tables_t(int mode, int nt, unsigned char *tab)
{
    T *H = (T *)tab;
    if (mode == ADAPT_GAUSS) {
        // Fwi::gauss(it, stdev) with stdev = STDEV*nt in T (lib/fwi.cpp:399-406)
        const T stdev = (T)(STDEV_FRAC * (double)nt);
        for (int it = 0; it < nt; it++)
            H[it] = stdev == T(0) ? T(0) : (T)std::exp(-1.0 * (it * it) / (2.0 * (stdev * stdev)));
    } else {
        // Fwi::linear(it, stdev) with stdev = HMAX (lib/fwi.cpp:408-417); also ADAPTIVE_SINGLE
        const T stdev = (T)RAMP_MAX;
        for (int it = 0; it < nt; it++) H[it] = stdev == T(0) ? T(0) : (it < stdev ? (T)it : stdev);
    }
    unsigned char *fx = tab + (size_t)nt * sizeof(T), *fc = fx + nt;
    if (mode == ADAPT_SINGLE) {
        conv_flags(2 * nt, 1 - 2 * nt, 2 * nt, 0, nt, 0, fx);   // xcor(2nt, 0, d, 2nt, 0, y, nt, 0, z)
        conv_flags(nt, 0, 2 * nt, 0, 2 * nt, 0, fc);            // convolve(nt, 0, w, 2nt, 0, d, 2nt, 0, z)
    } else {
        conv_flags(nt, 1 - nt, nt, 0, nt, 0, fx);   // xcor(nt, 0, d, nt, 0, y, nt, 0, z): x reversed
        conv_flags(nt, 0, nt, 0, nt, 0, fc);        // convolve(nt, 0, w, nt, 0, d, nt, 0, z)
    }
}

template <typename T, int ACC, int MODE>
void launch_t(const void *desc, int nshots, int nrec_max, int nt, const void *tables, double *misfit, cudaStream_t st,
              bool clip)
{
    const dim3 grid((unsigned)((nrec_max + 3) / 4), (unsigned)nshots);
    adaptive_shape<T, MODE><<<grid, 128, 0, st>>>((const Resid2D<T> *)desc, (const unsigned char *)tables, nt);
    if (clip)
        adaptive_finish<T, ACC, MODE, true><<<nshots, 256, 0, st>>>((const Resid2D<T> *)desc,
                                                                    (const unsigned char *)tables, misfit);
    else
        adaptive_finish<T, ACC, MODE, false><<<nshots, 256, 0, st>>>((const Resid2D<T> *)desc,
                                                                     (const unsigned char *)tables, misfit);
}

template <typename T, int ACC>
void launch_acc(int mode, const void *desc, int nshots, int nrec_max, int nt, const void *tables, double *misfit,
                cudaStream_t st, bool clip)
{
    if (mode == ADAPT_GAUSS) launch_t<T, ACC, ADAPT_GAUSS>(desc, nshots, nrec_max, nt, tables, misfit, st, clip);
    else launch_t<T, ACC, ADAPT_LINEAR>(desc, nshots, nrec_max, nt, tables, misfit, st, clip);
}

template <typename T, int ACC, int MODE>
void launch_e2d_t(const void *desc, const void *comp, int nshots, int nrec_max, int nt, const void *tables,
                  double *misfit, cudaStream_t st)
{
    const unsigned char *tab = (const unsigned char *)tables;
    if (MODE == ADAPT_SINGLE) {
        const dim3 grid((unsigned)((nrec_max + 3) / 4), (unsigned)nshots);
        adaptive_shape_single<T><<<grid, 128, 0, st>>>((const Resid2DE<T> *)desc, tab, nt);
    } else {
        const dim3 grid((unsigned)((nrec_max + 3) / 4), (unsigned)(2 * nshots));
        adaptive_shape<T, MODE><<<grid, 128, 0, st>>>((const Resid2D<T> *)comp, tab, nt);
    }
    adaptive_finish_e2d<T, ACC, MODE><<<nshots, 256, 0, st>>>((const Resid2DE<T> *)desc, tab, misfit);
}

template <typename T, int ACC>
void launch_e2d_acc(int mode, const void *desc, const void *comp, int nshots, int nrec_max, int nt, const void *tables,
                    double *misfit, cudaStream_t st)
{
    if (mode == ADAPT_GAUSS) launch_e2d_t<T, ACC, ADAPT_GAUSS>(desc, comp, nshots, nrec_max, nt, tables, misfit, st);
    else if (mode == ADAPT_LINEAR) launch_e2d_t<T, ACC, ADAPT_LINEAR>(desc, comp, nshots, nrec_max, nt, tables, misfit, st);
    else launch_e2d_t<T, ACC, ADAPT_SINGLE>(desc, comp, nshots, nrec_max, nt, tables, misfit, st);
}

}  // namespace

size_t adaptive_table_bytes(int prec, int mode, int nt)
{
    return (size_t)nt * (prec == PREC_F64 ? 8 : 4) + (size_t)nt + (size_t)(mode == ADAPT_SINGLE ? 2 : 1) * nt;
}

size_t adaptive_work_values(int mode, int nt)
{
    return (size_t)(mode == ADAPT_SINGLE ? 9 : 5) * nt;
}

cudaError_t launch_residual_adaptive_e2d(int prec, int acc, int mode, const void *desc, const void *comp, int nshots,
                                         int nrec_max, int nt, const void *tables, double *misfit, cudaStream_t st)
{
    if (mode != ADAPT_GAUSS && mode != ADAPT_LINEAR && mode != ADAPT_SINGLE) return cudaErrorInvalidValue;
    if (prec == PREC_F64) {
        if (acc == ACC_F64) launch_e2d_acc<double, ACC_F64>(mode, desc, comp, nshots, nrec_max, nt, tables, misfit, st);
        else launch_e2d_acc<double, ACC_REF>(mode, desc, comp, nshots, nrec_max, nt, tables, misfit, st);
    } else {
        if (acc == ACC_F64) launch_e2d_acc<float, ACC_F64>(mode, desc, comp, nshots, nrec_max, nt, tables, misfit, st);
        else launch_e2d_acc<float, ACC_REF>(mode, desc, comp, nshots, nrec_max, nt, tables, misfit, st);
    }
    return cudaGetLastError();
}

void adaptive_fill_tables(int prec, int mode, int nt, void *host_tables)
{
    if (prec == PREC_F64) fill_tables_t<double>(mode, nt, (unsigned char *)host_tables);
    else fill_tables_t<float>(mode, nt, (unsigned char *)host_tables);
}

cudaError_t launch_residual_adaptive(int prec, int acc, int mode, const void *desc, int nshots, int nrec_max, int nt,
                                     const void *tables, double *misfit, cudaStream_t st, bool clip)
{
    if (mode != ADAPT_GAUSS && mode != ADAPT_LINEAR) return cudaErrorInvalidValue;
    if (prec == PREC_F64) {
        if (acc == ACC_F64) launch_acc<double, ACC_F64>(mode, desc, nshots, nrec_max, nt, tables, misfit, st, clip);
        else launch_acc<double, ACC_REF>(mode, desc, nshots, nrec_max, nt, tables, misfit, st, clip);
    } else {
        if (acc == ACC_F64) launch_acc<float, ACC_F64>(mode, desc, nshots, nrec_max, nt, tables, misfit, st, clip);
        else launch_acc<float, ACC_REF>(mode, desc, nshots, nrec_max, nt, tables, misfit, st, clip);
    }
    return cudaGetLastError();
}

}  // namespace rsgpu
