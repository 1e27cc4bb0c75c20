// Host-side preprocessing for the C ABI: C-PML tables, model staggering and
// coordinate-to-grid maps.  These restate the reference's host code with the
// same C++ expression types (float products promoted to double where the
// reference writes a double literal), so the arrays they produce are bit-equal
// to the reference's for T = float and T = double.  Callers that already hold
// reference objects pass the reference's own arrays to the plan instead.
#include <cmath>
#include <cstring>
#include <vector>

#include "rsgpu.h"
#include "rsgpu_host.h"

namespace rsgpu {

// Pml<T>::computeABC(sign=1) with Amax=0, Kmax=2, Smax=1200 (lib/pml.cpp:79-126,
// include/pml.h:14-16).  Output order: A,B,C ltf; A,B,C ltf_stag; A,B,C rbb; A,B,C rbb_stag.
template <typename T>
static void pml_tables_t(int L, T dt, T *out)
{
    const T Amax = 0, Kmax = 2, Smax = 1200;
    auto fill = [&](T func, int tab, int i) {
        func = std::pow(func, 3);      // pow(T,int) promotes to double, as in the reference
        T a = Amax * func;
        T k = 1. + (Kmax - 1) * func;
        T s = Smax * func;
        T C = 1.0 - 1.0 / k;
        T B = std::exp(-(a + s / k) * dt);
        T A = (s * (1. - B)) / (k * (k * a + s));
        out[(tab + 0) * L + i] = A;
        out[(tab + 1) * L + i] = B;
        out[(tab + 2) * L + i] = C;
    };
    const int sign = 1;
    for (int i = 0; i < L; i++) {
        fill((T)(L - i) / L, 0, i);
        fill((T)(L - i - sign * 0.5) / L, 3, i);
        fill((T)(i + 1.0) / L, 6, i);
        fill((T)(i + 1.0 + sign * 0.5) / L, 9, i);
    }
}

void pml_tables_host(int lpml, double dt, int prec, void *out)
{
    if (prec == PREC_F64) pml_tables_t<double>(lpml, dt, (double *)out);
    else pml_tables_t<float>(lpml, (float)dt, (float *)out);
}

// ---------------------------------------------------------------- staggering
// Edge-replicating pad (Model::padmodel2d/3d, lib/model.cpp:93-182): every padded
// cell takes the value of the nearest interior cell.
template <typename T>
static void pad3(T *dst, const T *src, int nx, int ny, int nz, int l, bool is3d)
{
    const int nxp = nx + 2 * l, nyp = is3d ? ny + 2 * l : 1, nzp = nz + 2 * l;
    for (int iz = 0; iz < nzp; iz++)
        for (int iy = 0; iy < nyp; iy++)
            for (int ix = 0; ix < nxp; ix++) {
                int sx = std::min(std::max(ix - l, 0), nx - 1);
                int sy = is3d ? std::min(std::max(iy - l, 0), ny - 1) : 0;
                int sz = std::min(std::max(iz - l, 0), nz - 1);
                dst[((size_t)iz * nyp + iy) * nxp + ix] = src[((size_t)sz * (is3d ? ny : 1) + sy) * nx + sx];
            }
}

// Model::staggermodel_x/y/z (lib/model.cpp:185-240): in-place forward average,
// the last cell copies its (already averaged) neighbour.
template <typename T>
static void stagger_axis(T *m, int nx, int ny, int nz, int axis)
{
    auto at = [&](int ix, int iy, int iz) -> T & { return m[((size_t)iz * ny + iy) * nx + ix]; };
    T avg;
    if (axis == 0) {
        for (int iz = 0; iz < nz; iz++)
            for (int iy = 0; iy < ny; iy++) {
                for (int ix = 0; ix < nx - 1; ix++) { avg = (at(ix + 1, iy, iz) + at(ix, iy, iz)) / 2.0; at(ix, iy, iz) = avg; }
                at(nx - 1, iy, iz) = at(nx - 2, iy, iz);
            }
    } else if (axis == 1) {
        for (int iz = 0; iz < nz; iz++)
            for (int ix = 0; ix < nx; ix++) {
                for (int iy = 0; iy < ny - 1; iy++) { avg = (at(ix, iy + 1, iz) + at(ix, iy, iz)) / 2.0; at(ix, iy, iz) = avg; }
                at(ix, ny - 1, iz) = at(ix, ny - 2, iz);
            }
    } else {
        for (int ix = 0; ix < nx; ix++)
            for (int iy = 0; iy < ny; iy++) {
                for (int iz = 0; iz < nz - 1; iz++) { avg = (at(ix, iy, iz + 1) + at(ix, iy, iz)) / 2.0; at(ix, iy, iz) = avg; }
                at(ix, iy, nz - 1) = at(ix, iy, nz - 2);
            }
    }
}

template <typename T>
static int stagger_t(int physics, int nx, int ny, int nz, int l, int fs, const T *vp, const T *vs, const T *rho,
                     T *const *out)
{
    const bool is3d = physics == PHYS_A3D || physics == PHYS_E3D;
    if (!is3d) ny = 1;
    const int nxp = nx + 2 * l, nyp = is3d ? ny + 2 * l : 1, nzp = nz + 2 * l;
    const size_t n = (size_t)nxp * nyp * nzp;
    auto idx = [&](int ix, int iy, int iz) { return ((size_t)iz * nyp + iy) * nxp + ix; };
    auto invert = [&](T *R) {
        for (size_t i = 0; i < n; i++) {
            if (R[i] == 0.0) return -1;
            R[i] = 1.0 / R[i];
        }
        return 0;
    };
    if (physics == PHYS_A2D || physics == PHYS_A3D) {
        // lib/model.cpp:1350-1411 (2D), 1965 (3D): Rx..Rz = 1/avg(rho), L = rho*vp^2
        T *Rx = out[0], *Ry = is3d ? out[1] : nullptr, *Rz = is3d ? out[2] : out[1], *L = is3d ? out[3] : out[2];
        pad3(Rx, rho, nx, ny, nz, l, is3d);
        if (Ry) pad3(Ry, rho, nx, ny, nz, l, is3d);
        pad3(Rz, rho, nx, ny, nz, l, is3d);
        pad3(L, vp, nx, ny, nz, l, is3d);
        for (size_t i = 0; i < n; i++) { T _vp = L[i], _rho = Rx[i]; L[i] = _rho * _vp * _vp; }
        stagger_axis(Rx, nxp, nyp, nzp, 0);
        if (Ry) stagger_axis(Ry, nxp, nyp, nzp, 1);
        stagger_axis(Rz, nxp, nyp, nzp, 2);
        if (invert(Rx) || (Ry && invert(Ry)) || invert(Rz)) return -1;
        if (fs)
            for (int iy = 0; iy < nyp; iy++)
                for (int ix = 0; ix < nxp; ix++) {
                    Rx[idx(ix, iy, l)] *= 2.0;
                    if (Ry) Ry[idx(ix, iy, l)] *= 2.0;
                    L[idx(ix, iy, l)] *= 0.0;
                }
        return 0;
    }
    if (physics == PHYS_E2D) {
        // lib/model.cpp:2720-2802
        T *Rx = out[0], *Rz = out[1], *L = out[2], *L2M = out[3], *M = out[4];
        pad3(Rx, rho, nx, ny, nz, l, false);
        pad3(Rz, rho, nx, ny, nz, l, false);
        pad3(L, vp, nx, ny, nz, l, false);
        pad3(M, vs, nx, ny, nz, l, false);
        for (size_t i = 0; i < n; i++) {
            T _vp = L[i], _vs = M[i], _rho = Rx[i];
            L2M[i] = _rho * _vp * _vp;
            M[i] = _rho * _vs * _vs;
            L[i] = _rho * _vp * _vp - 2.0 * _rho * _vs * _vs;
        }
        if (fs)
            for (int ix = 0; ix < nxp; ix++) { L[idx(ix, 0, l)] = 0.0; L2M[idx(ix, 0, l)] = M[idx(ix, 0, l)]; }
        stagger_axis(Rx, nxp, 1, nzp, 0);
        stagger_axis(Rz, nxp, 1, nzp, 2);
        stagger_axis(M, nxp, 1, nzp, 2);
        stagger_axis(M, nxp, 1, nzp, 0);
        if (invert(Rx) || invert(Rz)) return -1;
        if (fs)
            for (int ix = 0; ix < nxp; ix++) Rx[idx(ix, 0, l)] *= 2.0;
        return 0;
    }
    return stagger_e3d_host(nx, ny, nz, l, fs, vp, vs, rho, out);
}

// ModelElastic3D::staggerModels (lib/model.cpp:3371-3475).  out = Rx, Ry, Rz, L,
// L2M, M_yz, M_xz, M_xy.  Moduli from the padded vp/vs/rho in the reference's
// expression types (2.0 is a double literal there), the free-surface row gets
// L = 0 and L2M = M before staggering, each shear modulus is averaged along its
// two axes, the densities are averaged and inverted, and the free-surface row
// doubles Rx and Ry.
template <typename T>
int stagger_e3d_host(int nx, int ny, int nz, int l, int fs, const T *vp, const T *vs, const T *rho, T *const *out)
{
    const int nxp = nx + 2 * l, nyp = ny + 2 * l, nzp = nz + 2 * l;
    const size_t n = (size_t)nxp * nyp * nzp;
    T *Rx = out[0], *Ry = out[1], *Rz = out[2], *L = out[3], *L2M = out[4], *Myz = out[5], *Mxz = out[6], *Mxy = out[7];
    auto idx = [&](int ix, int iy, int iz) { return ((size_t)iz * nyp + iy) * nxp + ix; };
    pad3(Rx, rho, nx, ny, nz, l, true);
    pad3(Ry, rho, nx, ny, nz, l, true);
    pad3(Rz, rho, nx, ny, nz, l, true);
    pad3(L, vp, nx, ny, nz, l, true);
    pad3(Mxz, vs, nx, ny, nz, l, true);
    for (size_t i = 0; i < n; i++) {
        const T _vp = L[i], _vs = Mxz[i], _rho = Rx[i];
        L2M[i] = _rho * _vp * _vp;
        L[i] = _rho * _vp * _vp - 2.0 * _rho * _vs * _vs;
        Mxz[i] = _rho * _vs * _vs;
        Myz[i] = _rho * _vs * _vs;
        Mxy[i] = _rho * _vs * _vs;
    }
    if (fs)
        for (int ix = 0; ix < nxp; ix++)
            for (int iy = 0; iy < nyp; iy++) {
                L[idx(ix, iy, l)] = 0.0;
                L2M[idx(ix, iy, l)] = Mxz[idx(ix, iy, l)];
            }
    stagger_axis(Rx, nxp, nyp, nzp, 0);
    stagger_axis(Ry, nxp, nyp, nzp, 1);
    stagger_axis(Rz, nxp, nyp, nzp, 2);
    stagger_axis(Mxz, nxp, nyp, nzp, 0);
    stagger_axis(Mxz, nxp, nyp, nzp, 2);
    stagger_axis(Myz, nxp, nyp, nzp, 1);
    stagger_axis(Myz, nxp, nyp, nzp, 2);
    stagger_axis(Mxy, nxp, nyp, nzp, 0);
    stagger_axis(Mxy, nxp, nyp, nzp, 1);
    for (size_t i = 0; i < n; i++) {
        if (Rx[i] == 0.0 || Ry[i] == 0.0 || Rz[i] == 0.0) return -1;
        Rx[i] = 1.0 / Rx[i];
        Ry[i] = 1.0 / Ry[i];
        Rz[i] = 1.0 / Rz[i];
    }
    if (fs)
        for (int ix = 0; ix < nxp; ix++)
            for (int iy = 0; iy < nyp; iy++) {
                Rx[idx(ix, iy, l)] *= 2.0;
                Ry[idx(ix, iy, l)] *= 2.0;
            }
    return 0;
}
template int stagger_e3d_host<float>(int, int, int, int, int, const float *, const float *, const float *, float *const *);
template int stagger_e3d_host<double>(int, int, int, int, int, const double *, const double *, const double *, double *const *);

int stagger_host(int physics, int nx, int ny, int nz, int l, int fs, int prec, const void *vp, const void *vs,
                 const void *rho, void *const *out)
{
    if (prec == PREC_F64)
        return stagger_t<double>(physics, nx, ny, nz, l, fs, (const double *)vp, (const double *)vs,
                                 (const double *)rho, (double *const *)out);
    return stagger_t<float>(physics, nx, ny, nz, l, fs, (const float *)vp, (const float *)vs, (const float *)rho,
                            (float *const *)out);
}

// ---------------------------------------------------------------- maps
// Geometry2D/3D::makeMap with zero pads (lib/geometry.cpp:137-230): index by the
// floor of ((double)coord - o + shift*d)/d with the CLOSE() round-off rules;
// off-grid positions get -1.  `gshift` is the per-axis staggering shift the
// reference's Data2D/3D::makeMap passes for the traced field (-0.5 along x for
// VX, along y for VY, along z for VZ; lib/data.cpp:440-460, 1116-1141).
#define RS_CTHRES 1e-2
static inline bool rs_close(double x, double y, double d) { return std::fabs(x - y) <= d * std::fabs(y); }

template <typename T>
static void make_map_t(int dim, int ntr, const double *coords, const int *n, const double *o, const double *d,
                       const double *gshift, int *map, T *shift)
{
    for (int i = 0; i < ntr; i++) {
        for (int a = 0; a < dim; a++) {
            const double dd = d[a], oo = o[a];
            const double c = coords[(size_t)i * dim + a];
            const T shiftx = gshift ? (T)gshift[a] : (T)0;
            double res = (c - oo + shiftx * dd) / dd;
            int pos = (int)std::floor(res);
            const int padl = 0, padh = 0;
            if (rs_close(res - pos, 1.0, dd * RS_CTHRES) && pos < padl) pos += 1;
            if (rs_close(res - pos, 0.0, dd * RS_CTHRES) && pos >= n[a] - padh) pos -= 1;
            if (pos >= padl && pos < n[a] - padh) {
                map[(size_t)i * dim + a] = pos;
                shift[(size_t)i * dim + a] = ((c - oo + shiftx * dd) / dd) - pos;
            } else {
                map[(size_t)i * dim + a] = -1;
            }
        }
    }
}

void make_map_host(int dim, int prec, int ntr, const double *coords, const int *n, const double *o, const double *d,
                   const double *gshift, int *map, void *shift)
{
    if (prec == PREC_F64) make_map_t<double>(dim, ntr, coords, n, o, d, gshift, map, (double *)shift);
    else make_map_t<float>(dim, ntr, coords, n, o, d, gshift, map, (float *)shift);
}

}  // namespace rsgpu
