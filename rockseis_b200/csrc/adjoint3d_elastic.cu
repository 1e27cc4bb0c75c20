// Kernels of the elastic 3D FWI gradient driver:
//   * FwiElastic3D::crossCorr (lib/fwi.cpp:5046-5290): lambda, mu and density
//     correlations of the forward and adjoint wavefields at one adjoint step,
//   * FwiElastic3D::scaleGrad (lib/fwi.cpp:5553-5629): their conversion to vp,
//     vs and density gradients after the last step,
//   * FwiElastic3D::computeResiduals / computeMisfit, DIFFERENCE
//     (lib/fwi.cpp:5901-5935, 5632-5700).
// Memory-bound passes; one launch covers every shot (blockIdx.z selects it).  The
// correlation marches z with one thread per (x, y) column of the unpadded window.
//
// The exact (and FP64) kernel evaluates each point's arithmetic as the reference
// does, operation for operation (see adjoint_ops.cuh): with ACCUM_REFERENCE the three
// gradients are float arrays updated exactly as the reference updates them,
// including the mu correlation's thirteen separate double-rounded subtractions;
// with ACCUM_F64 the same per-step terms are subtracted from double accumulators.
// The FAST kernel sums each gradient's terms in float with multiply-adds and
// subtracts one term per gradient and step.
#include <cuda_runtime.h>

#include "adjoint_ops.cuh"
#include "rsgpu_adjoint.h"
#include "rsgpu_kernels.h"

namespace rsgpu {
namespace {

// Subtract a double term from an accumulator of type G (T: rounded like the
// reference's `grad[k] -= double`; double: exact accumulation of the term).
template <typename T, typename G>
__device__ __forceinline__ void sub_term(G &g, double t)
{
    if (sizeof(G) == sizeof(T)) g = (G)X<T>::rnd(__dsub_rn((double)g, t));
    else g = (G)__dsub_rn((double)g, t);
}

// (a - b)/h1 + (c - d)/h2 in T
template <typename T>
__device__ __forceinline__ T pair_div(T a, T b, T h1, T c, T d, T h2)
{
    using O = X<T>;
    return O::add(O::div(O::sub(a, b), h1), O::div(O::sub(c, d), h2));
}

// `u += 0.5*w*r*dd/h` with u in T
template <typename T>
__device__ __forceinline__ T half_acc(T u, T w, T r, T dd, double h)
{
    return X<T>::rnd(__dadd_rn((double)u, half_term(w, r, dd, h)));
}

template <typename T, typename G>
__global__ void __launch_bounds__(256) corr_fwi_e3d(const Corr3DE<T> *desc, T dx, T dy, T dz)
{
    using O = X<T>;
    const Corr3DE<T> c = desc[blockIdx.z];
    const int ix = blockIdx.x * blockDim.x + threadIdx.x;
    const int iy = blockIdx.y * blockDim.y + threadIdx.y;
    if (ix < 1 || iy < 1 || ix >= c.nx - 1 || iy >= c.ny - 1) return;
    const long long P = c.pitch, PL = c.plane;
    const int L = c.lpml;
    const T *wsx = c.ws[0], *wsy = c.ws[1], *wsz = c.ws[2];
    const T *fsxx = c.ws[3], *fsyy = c.ws[4], *fszz = c.ws[5], *fsyz = c.ws[6], *fsxz = c.ws[7], *fsxy = c.ws[8];
    const T *wrx = c.wr[0], *wry = c.wr[1], *wrz = c.wr[2];
    const T *rsxx = c.wr[3], *rsyy = c.wr[4], *rszz = c.wr[5], *rsyz = c.wr[6], *rsxz = c.wr[7], *rsxy = c.wr[8];
    const double DX = (double)dx, DY = (double)dy, DZ = (double)dz;
    for (int iz = 1; iz < c.nz - 1; iz++) {
        const long long q = (long long)(iz + L) * PL + (long long)(iy + L) * P + (ix + L);
        const long long u = ((long long)iz * c.ny + iy) * c.nx + ix;
        // offsets of the neighbours: x +-1, y +-P, z +-PL
        const long long xm = q - 1, ym = q - P, zm = q - PL;
        const T msxx = O::div(O::sub(wsx[q], wsx[xm]), dx);
        const T msyy = O::div(O::sub(wsy[q], wsy[ym]), dy);
        const T mszz = O::div(O::sub(wsz[q], wsz[zm]), dz);
        const T rxx = rsxx[q], ryy = rsyy[q], rzz = rszz[q];
        // lambda
        const T a = O::mul(O::add(O::add(msxx, msyy), mszz), O::add(O::add(rxx, ryy), rzz));
        // mu: four corner strains of each shear plane times the adjoint shear stress
        const T ryz = rsyz[q], rxz = rsxz[q], rxy = rsxy[q];
        T m[12];
        m[0] = pair_div(wsy[ym], wsy[ym - PL], dz, wsz[zm], wsz[ym - PL], dy);
        m[1] = pair_div(wsy[q], wsy[zm], dz, wsz[zm + P], wsz[zm], dy);
        m[2] = pair_div(wsy[ym + PL], wsy[ym], dz, wsz[q], wsz[ym], dy);
        m[3] = pair_div(wsy[q + PL], wsy[q], dz, wsz[q + P], wsz[q], dy);
        m[4] = pair_div(wsx[xm], wsx[xm - PL], dz, wsz[zm], wsz[xm - PL], dx);
        m[5] = pair_div(wsx[q], wsx[zm], dz, wsz[zm + 1], wsz[zm], dx);
        m[6] = pair_div(wsx[xm + PL], wsx[xm], dz, wsz[q], wsz[xm], dx);
        m[7] = pair_div(wsx[q + PL], wsx[q], dz, wsz[q + 1], wsz[q], dx);
        m[8] = pair_div(wsy[ym], wsy[ym - 1], dx, wsx[xm], wsx[xm - P], dy);
        m[9] = pair_div(wsy[ym + 1], wsy[ym], dx, wsx[q], wsx[ym], dy);
        m[10] = pair_div(wsy[q], wsy[xm], dx, wsx[xm + P], wsx[xm], dy);
        m[11] = pair_div(wsy[q + 1], wsy[q], dx, wsx[q + P], wsx[q], dy);
        // 2 (msxx Sxx + msyy Syy + mszz Szz) in double
        const double two = __dadd_rn(__dadd_rn(__dmul_rn(__dmul_rn(2.0, (double)msxx), (double)rxx),
                                               __dmul_rn(__dmul_rn(2.0, (double)msyy), (double)ryy)),
                                     __dmul_rn(__dmul_rn(2.0, (double)mszz), (double)rzz));
        // density: velocity-weighted stress divergences on the staggered faces
        T ux = O::rnd(half_term(wrx[q], c.rx[q], O::sub(fsxx[q + 1], fsxx[q]), DX));
        ux = half_acc(ux, wrx[xm], c.rx[xm], O::sub(fsxx[q], fsxx[xm]), DX);
        ux = half_acc(ux, wrx[q], c.rx[q], O::sub(fsxy[q], fsxy[ym]), DY);
        ux = half_acc(ux, wrx[xm], c.rx[xm], O::sub(fsxy[xm], fsxy[xm - P]), DY);
        ux = half_acc(ux, wrx[q], c.rx[q], O::sub(fsxz[q], fsxz[zm]), DZ);
        ux = half_acc(ux, wrx[xm], c.rx[xm], O::sub(fsxz[xm], fsxz[xm - PL]), DZ);
        T uy = O::rnd(half_term(wry[q], c.ry[q], O::sub(fsxy[q], fsxy[xm]), DX));
        uy = half_acc(uy, wry[ym], c.ry[ym], O::sub(fsxy[ym], fsxy[ym - 1]), DX);
        uy = half_acc(uy, wry[q], c.ry[q], O::sub(fsyy[q + P], fsyy[q]), DY);
        uy = half_acc(uy, wry[ym], c.ry[ym], O::sub(fsyy[q], fsyy[ym]), DY);
        uy = half_acc(uy, wry[q], c.ry[q], O::sub(fsyz[q], fsyz[zm]), DZ);
        uy = half_acc(uy, wry[ym], c.ry[ym], O::sub(fsyz[ym], fsyz[ym - PL]), DZ);
        // the second term of each pair takes the adjoint Vz of the cell at y-1 with
        // Rz of the cell at z-1, as the reference writes it
        T uz = O::rnd(half_term(wrz[q], c.rz[q], O::sub(fsxz[q], fsxz[xm]), DX));
        uz = half_acc(uz, wrz[ym], c.rz[zm], O::sub(fsxz[zm], fsxz[zm - 1]), DX);
        uz = half_acc(uz, wrz[q], c.rz[q], O::sub(fsyz[q], fsyz[ym]), DY);
        uz = half_acc(uz, wrz[ym], c.rz[zm], O::sub(fsyz[zm], fsyz[zm - P]), DY);
        uz = half_acc(uz, wrz[q], c.rz[q], O::sub(fszz[q + PL], fszz[q]), DZ);
        uz = half_acc(uz, wrz[ym], c.rz[zm], O::sub(fszz[q], fszz[zm]), DZ);
        const T rh = O::add(O::add(ux, uy), uz);

        G *g0 = (G *)c.g[0] + u, *g1 = (G *)c.g[1] + u, *g2 = (G *)c.g[2] + u;
        G v0 = *g0, v1 = *g1, v2 = *g2;
        if (sizeof(G) == sizeof(T)) {
            v0 = (G)O::sub((T)v0, a);
            v2 = (G)O::sub((T)v2, rh);
        } else {
            v0 = (G)__dsub_rn((double)v0, (double)a);
            v2 = (G)__dsub_rn((double)v2, (double)rh);
        }
#pragma unroll
        for (int k = 0; k < 12; k++) {
            const T r = k < 4 ? ryz : k < 8 ? rxz : rxy;
            sub_term<T, G>(v1, __dmul_rn(__dmul_rn(0.25, (double)m[k]), (double)r));
        }
        sub_term<T, G>(v1, two);
        *g0 = v0; *g1 = v1; *g2 = v2;
    }
}

// FAST arithmetic (float, reciprocal spacings, contracted multiply-adds) of the same
// correlation: the three gradients take one summed term per step each.  The z-march
// keeps in registers the values that the next plane reuses (z-1 / z / z+1 of the
// columns whose z-derivatives appear, and the rz of the plane below), so a point
// loads 49 values instead of about 100; x and y neighbours come from L1.
template <typename G>
__global__ void __launch_bounds__(256) corr_fwi_e3d_fast(const Corr3DE<float> *desc, float idx, float idy, float idz)
{
    const Corr3DE<float> c = desc[blockIdx.z];
    const int ix = blockIdx.x * blockDim.x + threadIdx.x;
    const int iy = blockIdx.y * blockDim.y + threadIdx.y;
    if (ix < 1 || iy < 1 || ix >= c.nx - 1 || iy >= c.ny - 1 || c.nz < 3) return;
    const long long P = c.pitch, PL = c.plane;
    const int L = c.lpml;
    const float *__restrict__ wsx = c.ws[0], *__restrict__ wsy = c.ws[1], *__restrict__ wsz = c.ws[2];
    const float *__restrict__ fsxx = c.ws[3], *__restrict__ fsyy = c.ws[4], *__restrict__ fszz = c.ws[5];
    const float *__restrict__ fsyz = c.ws[6], *__restrict__ fsxz = c.ws[7], *__restrict__ fsxy = c.ws[8];
    const float *__restrict__ wrx = c.wr[0], *__restrict__ wry = c.wr[1], *__restrict__ wrz = c.wr[2];
    const float *__restrict__ rsxx = c.wr[3], *__restrict__ rsyy = c.wr[4], *__restrict__ rszz = c.wr[5];
    const float *__restrict__ rsyz = c.wr[6], *__restrict__ rsxz = c.wr[7], *__restrict__ rsxy = c.wr[8];
    const float *__restrict__ rx = c.rx, *__restrict__ ry = c.ry, *__restrict__ rz = c.rz;
    long long q = (long long)(1 + L) * PL + (long long)(iy + L) * P + (ix + L);
    long long u = ((long long)c.ny + iy) * c.nx + ix;
    const long long un = (long long)c.ny * c.nx;
    // values carried from plane to plane: (array, column) at z-1 ("m") and z
    float sx0m = wsx[q - PL], sx0 = wsx[q], sx1m = wsx[q - 1 - PL], sx1 = wsx[q - 1];
    float sy0m = wsy[q - PL], sy0 = wsy[q], sy1m = wsy[q - P - PL], sy1 = wsy[q - P];
    float sz0m = wsz[q - PL], szymm = wsz[q - P - PL], szypm = wsz[q + P - PL];
    float szxmm = wsz[q - 1 - PL], szxpm = wsz[q + 1 - PL];
    float xz0m = fsxz[q - PL], xz1m = fsxz[q - 1 - PL], yz0m = fsyz[q - PL], yz1m = fsyz[q - P - PL];
    float zzm = fszz[q - PL], zz0 = fszz[q], rzm = rz[q - PL];
    for (int iz = 1; iz < c.nz - 1; iz++, q += PL, u += un) {
        const float sx0p = wsx[q + PL], sx1p = wsx[q - 1 + PL], sy0p = wsy[q + PL], sy1p = wsy[q - P + PL];
        const float zzp = fszz[q + PL];
        const float sz0 = wsz[q], szym = wsz[q - P], szyp = wsz[q + P], szxm = wsz[q - 1], szxp = wsz[q + 1];
        const float sxym = wsx[q - P], sxyp = wsx[q + P], sxxmym = wsx[q - 1 - P], sxxmyp = wsx[q - 1 + P];
        const float syxm = wsy[q - 1], syxp = wsy[q + 1], syymxm = wsy[q - P - 1], syymxp = wsy[q - P + 1];
        const float xx0 = fsxx[q], xxp = fsxx[q + 1], xxm = fsxx[q - 1];
        const float xy0 = fsxy[q], xyym = fsxy[q - P], xyxm = fsxy[q - 1], xyxmym = fsxy[q - 1 - P];
        const float xz0 = fsxz[q], xz1 = fsxz[q - 1], yz0 = fsyz[q], yz1 = fsyz[q - P];
        const float yy0 = fsyy[q], yyp = fsyy[q + P], yym = fsyy[q - P];
        const float wq = wrx[q] * rx[q], wm = wrx[q - 1] * rx[q - 1];
        const float vq = wry[q] * ry[q], vm = wry[q - P] * ry[q - P];
        const float rz0 = rz[q];
        const float zq = wrz[q] * rz0, zmm = wrz[q - P] * rzm;
        const float rxx = rsxx[q], ryy = rsyy[q], rzz = rszz[q], ryz = rsyz[q], rxz = rsxz[q], rxy = rsxy[q];

        const float msxx = (sx0 - sx1) * idx, msyy = (sy0 - sy1) * idy, mszz = (sz0 - sz0m) * idz;
        const float a = (msxx + msyy + mszz) * (rxx + ryy + rzz);
        const float myz = ((sy1 - sy1m) * idz + (sz0m - szymm) * idy) + ((sy0 - sy0m) * idz + (szypm - sz0m) * idy) +
                          ((sy1p - sy1) * idz + (sz0 - szym) * idy) + ((sy0p - sy0) * idz + (szyp - sz0) * idy);
        const float mxz = ((sx1 - sx1m) * idz + (sz0m - szxmm) * idx) + ((sx0 - sx0m) * idz + (szxpm - sz0m) * idx) +
                          ((sx1p - sx1) * idz + (sz0 - szxm) * idx) + ((sx0p - sx0) * idz + (szxp - sz0) * idx);
        const float mxy = ((sy1 - syymxm) * idx + (sx1 - sxxmym) * idy) + ((syymxp - sy1) * idx + (sx0 - sxym) * idy) +
                          ((sy0 - syxm) * idx + (sxxmyp - sx1) * idy) + ((syxp - sy0) * idx + (sxyp - sx0) * idy);
        const float mu = 2.0f * (msxx * rxx + msyy * ryy + mszz * rzz) + 0.25f * (myz * ryz + mxz * rxz + mxy * rxy);
        const float ux = wq * ((xxp - xx0) * idx + (xy0 - xyym) * idy + (xz0 - xz0m) * idz) +
                         wm * ((xx0 - xxm) * idx + (xyxm - xyxmym) * idy + (xz1 - xz1m) * idz);
        const float uy = vq * ((xy0 - xyxm) * idx + (yyp - yy0) * idy + (yz0 - yz0m) * idz) +
                         vm * ((xyym - xyxmym) * idx + (yy0 - yym) * idy + (yz1 - yz1m) * idz);
        const float uz = zq * ((xz0 - xz1) * idx + (yz0 - yz1) * idy + (zzp - zz0) * idz) +
                         zmm * ((xz0m - xz1m) * idx + (yz0m - yz1m) * idy + (zz0 - zzm) * idz);
        const float rh = 0.5f * (ux + uy + uz);
        G *g0 = (G *)c.g[0] + u, *g1 = (G *)c.g[1] + u, *g2 = (G *)c.g[2] + u;
        *g0 -= (G)a;
        *g1 -= (G)mu;
        *g2 -= (G)rh;
        sx0m = sx0; sx0 = sx0p; sx1m = sx1; sx1 = sx1p;
        sy0m = sy0; sy0 = sy0p; sy1m = sy1; sy1 = sy1p;
        sz0m = sz0; szymm = szym; szypm = szyp; szxmm = szxm; szxpm = szxp;
        xz0m = xz0; xz1m = xz1; yz0m = yz0; yz1m = yz1;
        zzm = zz0; zz0 = zzp; rzm = rz0;
    }
}

// FwiElastic3D::scaleGrad over the whole window:
//   vp  <- 2 rho vp lambda
//   vs  <- 2 rho vs mu - 2 (2 rho vs) lambda
//   rho <- vp^2 lambda + vs^2 mu + rho
template <typename T, typename G>
__global__ void __launch_bounds__(256) scale_grad_e3d(const Corr3DE<T> *desc)
{
    const Corr3DE<T> c = desc[blockIdx.z];
    const int ix = blockIdx.x * blockDim.x + threadIdx.x;
    const int iy = blockIdx.y * blockDim.y + threadIdx.y;
    if (ix >= c.nx || iy >= c.ny) return;
    for (int iz = 0; iz < c.nz; iz++) {
        const long long u = ((long long)iz * c.ny + iy) * c.nx + ix;
        const T vp = c.vp[u], vs = c.vs[u], rho = c.rho[u];
        G *g0 = (G *)c.g[0] + u, *g1 = (G *)c.g[1] + u, *g2 = (G *)c.g[2] + u;
        if (sizeof(G) == sizeof(T)) {
            using O = X<T>;
            const T vpscale = O::rnd(__dmul_rn(__dmul_rn(2.0, (double)rho), (double)vp));
            const T vsscale = O::rnd(__dmul_rn(__dmul_rn(2.0, (double)rho), (double)vs));
            const T rs1 = O::mul(vp, vp), rs2 = O::mul(vs, vs);
            const T lambda = *(T *)g0, mu = *(T *)g1, r = *(T *)g2;
            *(T *)g0 = O::mul(vpscale, lambda);
            *(T *)g1 = O::rnd(__dsub_rn((double)O::mul(vsscale, mu),
                                        __dmul_rn(__dmul_rn(2.0, (double)vsscale), (double)lambda)));
            *(T *)g2 = O::add(O::add(O::mul(rs1, lambda), O::mul(rs2, mu)), r);
        } else {
            const double dvp = vp, dvs = vs, drho = rho;
            const double vpscale = 2.0 * drho * dvp, vsscale = 2.0 * drho * dvs;
            const double lambda = *g0, mu = *g1, r = *g2;
            *g0 = vpscale * lambda;
            *g1 = vsscale * mu - 2.0 * vsscale * lambda;
            *g2 = dvp * dvp * lambda + dvs * dvs * mu + r;
        }
    }
}

// Residuals r = mod - obs of Ux, Uy, Uz; misfit += 0.5*(rx*rx + ry*ry + rz*rz)
// over every trace (the elastic 3D misfit has no receiver mask), squares summed
// in T and the half added in double to a T accumulator, traces then samples.
template <typename T, int ACC>
__global__ void __launch_bounds__(256) residual_misfit_e3d(const Resid3E<T> *desc, double *misfit)
{
    const Resid3E<T> d = desc[blockIdx.x];
    const long long n = (long long)d.nrec * d.nt;
    for (int k = 0; k < 3; k++)
        for (long long j = threadIdx.x; j < n; j += blockDim.x) d.res[k][j] = X<T>::sub(d.mod[k][j], d.obs[k][j]);
    if (ACC == ACC_REF) {
        __syncthreads();
        if (threadIdx.x != 0) return;
        T mis = 0;
        for (long long j = 0; j < n; j++) {
            const T rx = d.res[0][j], ry = d.res[1][j], rz = d.res[2][j];
            const T s = X<T>::add(X<T>::add(X<T>::mul(rx, rx), X<T>::mul(ry, ry)), X<T>::mul(rz, rz));
            mis = X<T>::rnd(__dadd_rn((double)mis, __dmul_rn(0.5, (double)s)));
        }
        misfit[blockIdx.x] = (double)mis;
    } else {
        double acc = 0.0;
        for (long long j = threadIdx.x; j < n; j += blockDim.x)
            for (int k = 0; k < 3; k++) {
                const double r = (double)X<T>::sub(d.mod[k][j], d.obs[k][j]);
                acc = fma(0.5 * r, r, acc);
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

}  // namespace

cudaError_t launch_corr_fwi_e3d(int prec, int acc, const void *desc, int nshots, int nxmax, int nymax, double dx,
                                double dy, double dz, cudaStream_t st)
{
    const dim3 block(32, 8), grid((nxmax + 31) / 32, (nymax + 7) / 8, nshots);
    if (prec == PREC_F32_FAST) {
        const float ix = (float)(1.0 / dx), iy = (float)(1.0 / dy), iz = (float)(1.0 / dz);
        if (acc == ACC_F64) corr_fwi_e3d_fast<double><<<grid, block, 0, st>>>((const Corr3DE<float> *)desc, ix, iy, iz);
        else corr_fwi_e3d_fast<float><<<grid, block, 0, st>>>((const Corr3DE<float> *)desc, ix, iy, iz);
    } else if (prec == PREC_F64)
        corr_fwi_e3d<double, double><<<grid, block, 0, st>>>((const Corr3DE<double> *)desc, dx, dy, dz);
    else if (acc == ACC_F64)
        corr_fwi_e3d<float, double><<<grid, block, 0, st>>>((const Corr3DE<float> *)desc, (float)dx, (float)dy,
                                                            (float)dz);
    else
        corr_fwi_e3d<float, float><<<grid, block, 0, st>>>((const Corr3DE<float> *)desc, (float)dx, (float)dy,
                                                           (float)dz);
    return cudaGetLastError();
}

cudaError_t launch_scale_grad_e3d(int prec, int acc, const void *desc, int nshots, int nxmax, int nymax,
                                  cudaStream_t st)
{
    const dim3 block(32, 8), grid((nxmax + 31) / 32, (nymax + 7) / 8, nshots);
    if (prec == PREC_F64) scale_grad_e3d<double, double><<<grid, block, 0, st>>>((const Corr3DE<double> *)desc);
    else if (acc == ACC_F64) scale_grad_e3d<float, double><<<grid, block, 0, st>>>((const Corr3DE<float> *)desc);
    else scale_grad_e3d<float, float><<<grid, block, 0, st>>>((const Corr3DE<float> *)desc);
    return cudaGetLastError();
}

cudaError_t launch_residual_e3d(int prec, int acc, const void *desc, int nshots, double *misfit, cudaStream_t st)
{
    if (prec == PREC_F64) {
        if (acc == ACC_F64) residual_misfit_e3d<double, ACC_F64><<<nshots, 256, 0, st>>>((const Resid3E<double> *)desc, misfit);
        else residual_misfit_e3d<double, ACC_REF><<<nshots, 256, 0, st>>>((const Resid3E<double> *)desc, misfit);
    } else {
        if (acc == ACC_F64) residual_misfit_e3d<float, ACC_F64><<<nshots, 256, 0, st>>>((const Resid3E<float> *)desc, misfit);
        else residual_misfit_e3d<float, ACC_REF><<<nshots, 256, 0, st>>>((const Resid3E<float> *)desc, misfit);
    }
    return cudaGetLastError();
}

}  // namespace rsgpu
