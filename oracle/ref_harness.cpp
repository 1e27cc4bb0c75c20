/*
 * ref_harness.cpp -- extern "C" drivers of the unmodified reference library
 * (Der, Pml, staggering, makeMap, Revolve, modelling, FWI gradient).
 * Test infrastructure only; see ref_harness_common.h.
 */
#include "ref_harness_common.h"
#include "fwi.h"
#include "interp.h"

using namespace rockseis;
using namespace refh;

namespace {
/* ---------------------------------------------------------------- Der */
template <typename T>
void der_apply(int nx, int ny, int nz, double dx, double dy, double dz, int order, int which,
               const T *f, T *df)
{
    Der<T> der(nx, ny, nz, (T)dx, (T)dy, (T)dz, order);
    size_t n = (size_t)nx * ny * nz;
    std::vector<T> buf(f, f + n);
    switch (which) {
    case 0: der.ddx_fw(buf.data()); break;
    case 1: der.ddy_fw(buf.data()); break;
    case 2: der.ddz_fw(buf.data()); break;
    case 3: der.ddx_bw(buf.data()); break;
    case 4: der.ddy_bw(buf.data()); break;
    case 5: der.ddz_bw(buf.data()); break;
    }
    std::memcpy(df, der.getDf(), sizeof(T) * n);
}

/* ---------------------------------------------------------------- PML */
template <typename T>
void pml_tables(int lpml, double dt, T *out)
{
    Pml<T> p(lpml, (T)dt);
    p.setSmax(SMAX);
    p.computeABC();
    const T *tabs[12] = {p.A_ltf, p.B_ltf, p.C_ltf, p.A_ltf_stag, p.B_ltf_stag, p.C_ltf_stag,
                         p.A_rbb, p.B_rbb, p.C_rbb, p.A_rbb_stag, p.B_rbb_stag, p.C_rbb_stag};
    for (int k = 0; k < 12; k++) std::memcpy(out + k * lpml, tabs[k], sizeof(T) * lpml);
}

/* ---------------------------------------------------------------- modelling */
template <typename T>
int mod_a2d(const ref_grid *g, const T *vp, const T *rho, int ns, const double *sc, const T *wav,
            int sfield, int nr, const double *gc, int rfield, T *out)
{
    auto model = make_a2d<T>(g, vp, rho);
    auto src = make_data2d<T>(ns, g, sc, sfield, SMAP, model->getGeom(), wav);
    auto rec = make_data2d<T>(nr, g, gc, rfield, GMAP, model->getGeom(), nullptr);
    ModellingAcoustic2D<T> mod(model, src, g->order, 1);
    if (rfield == PRESSURE) mod.setRecP(rec);
    else if (rfield == VX) mod.setRecVx(rec);
    else mod.setRecVz(rec);
    int r = mod.run();
    std::memcpy(out, rec->getData(), sizeof(T) * (size_t)nr * g->nt);
    return r;
}

template <typename T>
int mod_e2d(const ref_grid *g, const T *vp, const T *vs, const T *rho, int ns, const double *sc,
            const T *wav, int sfield, int nr, const double *gc, int rfield, T *out)
{
    auto model = make_e2d<T>(g, vp, vs, rho);
    auto src = make_data2d<T>(ns, g, sc, sfield, SMAP, model->getGeom(), wav);
    auto rec = make_data2d<T>(nr, g, gc, rfield, GMAP, model->getGeom(), nullptr);
    ModellingElastic2D<T> mod(model, src, g->order, 1);
    if (rfield == PRESSURE) mod.setRecP(rec);
    else if (rfield == VX) mod.setRecVx(rec);
    else mod.setRecVz(rec);
    int r = mod.run();
    std::memcpy(out, rec->getData(), sizeof(T) * (size_t)nr * g->nt);
    return r;
}

template <typename T>
int mod_a3d(const ref_grid *g, const T *vp, const T *rho, int ns, const double *sc, const T *wav,
            int sfield, int nr, const double *gc, int rfield, T *out)
{
    auto model = make_a3d<T>(g, vp, rho);
    auto src = make_data3d<T>(ns, g, sc, sfield, SMAP, model->getGeom(), wav);
    auto rec = make_data3d<T>(nr, g, gc, rfield, GMAP, model->getGeom(), nullptr);
    ModellingAcoustic3D<T> mod(model, src, g->order, 1);
    if (rfield == PRESSURE) mod.setRecP(rec);
    else if (rfield == VX) mod.setRecVx(rec);
    else if (rfield == VY) mod.setRecVy(rec);
    else mod.setRecVz(rec);
    int r = mod.run();
    std::memcpy(out, rec->getData(), sizeof(T) * (size_t)nr * g->nt);
    return r;
}

template <typename T>
int mod_e3d(const ref_grid *g, const T *vp, const T *vs, const T *rho, int ns, const double *sc,
            const T *wav, int sfield, int nr, const double *gc, int rfield, T *out)
{
    auto model = make_e3d<T>(g, vp, vs, rho);
    auto src = make_data3d<T>(ns, g, sc, sfield, SMAP, model->getGeom(), wav);
    auto rec = make_data3d<T>(nr, g, gc, rfield, GMAP, model->getGeom(), nullptr);
    ModellingElastic3D<T> mod(model, src, g->order, 1);
    if (rfield == PRESSURE) mod.setRecP(rec);
    else if (rfield == VX) mod.setRecVx(rec);
    else if (rfield == VY) mod.setRecVy(rec);
    else mod.setRecVz(rec);
    int r = mod.run();
    std::memcpy(out, rec->getData(), sizeof(T) * (size_t)nr * g->nt);
    return r;
}

/* ---------------------------------------------------------------- FWI gradient */
template <typename T>
int fwi_a2d(const ref_grid *g, const T *vp, const T *rho, int ns, const double *sc, const T *wav,
            int nr, const double *gc, const T *obs, int ncheck, int misfit_type, T *vpgrad,
            T *rhograd, T *wavgrad, T *datamod, T *datares, double *misfit, T *srcilum = nullptr,
            int full_snapinc = 0, int noreverse = 0)
{
    auto model = make_a2d<T>(g, vp, rho);
    auto src = make_data2d<T>(ns, g, sc, PRESSURE, SMAP, model->getGeom(), wav);
    auto dobs = make_data2d<T>(nr, g, gc, PRESSURE, GMAP, model->getGeom(), obs);
    auto dmod = make_data2d<T>(nr, g, gc, PRESSURE, GMAP, model->getGeom(), nullptr);
    auto dres = make_data2d<T>(nr, g, gc, PRESSURE, GMAP, model->getGeom(), nullptr);
    auto wg = make_data2d<T>(ns, g, sc, PRESSURE, SMAP, model->getGeom(), nullptr);
    auto ivp = std::make_shared<Image2D<T>>(g->nx, g->nz, 1, 1, (T)g->dx, (T)g->dz, (T)g->ox, (T)g->oz);
    auto irho = std::make_shared<Image2D<T>>(g->nx, g->nz, 1, 1, (T)g->dx, (T)g->dz, (T)g->ox, (T)g->oz);
    irho->allocateImage();
    FwiAcoustic2D<T> fwi(model, src, dobs, g->order, full_snapinc > 0 ? full_snapinc : 1);
    fwi.setDatamodP(dmod);
    fwi.setDataresP(dres);
    fwi.setVpgrad(ivp);
    fwi.setRhograd(irho);
    fwi.setWavgrad(wg);
    fwi.setNoreverse(noreverse != 0);
    std::shared_ptr<Image2D<T>> ilum;
    if (srcilum) {
        ilum = std::make_shared<Image2D<T>>(g->nx, g->nz, 1, 1, (T)g->dx, (T)g->dz, (T)g->ox, (T)g->oz);
        fwi.setSrcilum(ilum);
    }
    fwi.setMisfit_type((rs_fwimisfit)misfit_type);
    fwi.setNcheck(ncheck);
    fwi.setIncore(true);
    fwi.setSnapfile(tmpname("fwia2d"));
    int r = full_snapinc > 0 ? fwi.run() : fwi.run_optimal();
    size_t n = (size_t)g->nx * g->nz;
    if (srcilum) std::memcpy(srcilum, ilum->getImagedata(), sizeof(T) * n);
    std::memcpy(vpgrad, ivp->getImagedata(), sizeof(T) * n);
    std::memcpy(rhograd, irho->getImagedata(), sizeof(T) * n);
    std::memcpy(wavgrad, wg->getData(), sizeof(T) * (size_t)ns * g->nt);
    std::memcpy(datamod, dmod->getData(), sizeof(T) * (size_t)nr * g->nt);
    std::memcpy(datares, dres->getData(), sizeof(T) * (size_t)nr * g->nt);
    *misfit = (double)fwi.getMisfit();
    return r;
}

/* FwiElastic2D::run_optimal (lib/fwi.cpp:3937-4143) with P, Ux (VX) and Uz (VZ) data, or, with
 * full_snapinc > 0, FwiElastic2D::run (lib/fwi.cpp:3774-3934): Vx/Vz snapshots every snapinc steps. */
template <typename T>
int fwi_e2d(const ref_grid *g, const T *vp, const T *vs, const T *rho, int ns, const double *sc, const T *wav,
            int sfield, int nr, const double *gc, const T *obsp, const T *obsx, const T *obsz, int ncheck, T *vpgrad,
            T *vsgrad, T *rhograd, T *wavgrad, T *mods, T *ress, double *misfit, int misfit_type = 0,
            int full_snapinc = 0)
{
    auto model = make_e2d<T>(g, vp, vs, rho);
    auto geom = model->getGeom();
    auto src = make_data2d<T>(ns, g, sc, sfield, SMAP, geom, wav);
    auto dp = make_data2d<T>(nr, g, gc, PRESSURE, GMAP, geom, obsp);
    auto dx = make_data2d<T>(nr, g, gc, VX, GMAP, geom, obsx);
    auto dz = make_data2d<T>(nr, g, gc, VZ, GMAP, geom, obsz);
    const int fields[3] = {PRESSURE, VX, VZ};
    std::shared_ptr<Data2D<T>> dm[3], dr[3];
    for (int k = 0; k < 3; k++) {
        dm[k] = make_data2d<T>(nr, g, gc, fields[k], GMAP, geom, nullptr);
        dr[k] = make_data2d<T>(nr, g, gc, fields[k], GMAP, geom, nullptr);
    }
    auto wg = make_data2d<T>(ns, g, sc, sfield, SMAP, geom, nullptr);
    std::shared_ptr<Image2D<T>> img[3];
    for (int k = 0; k < 3; k++) {
        img[k] = std::make_shared<Image2D<T>>(g->nx, g->nz, 1, 1, (T)g->dx, (T)g->dz, (T)g->ox, (T)g->oz);
        img[k]->allocateImage();
    }
    FwiElastic2D<T> fwi(model, src, dp, dx, dz, g->order, full_snapinc > 0 ? full_snapinc : 1);
    fwi.setDatamodP(dm[0]); fwi.setDatamodUx(dm[1]); fwi.setDatamodUz(dm[2]);
    fwi.setDataresP(dr[0]); fwi.setDataresUx(dr[1]); fwi.setDataresUz(dr[2]);
    fwi.setVpgrad(img[0]); fwi.setVsgrad(img[1]); fwi.setRhograd(img[2]);
    fwi.setWavgrad(wg);
    fwi.setMisfit_type((rs_fwimisfit)misfit_type);
    fwi.setNcheck(ncheck);
    fwi.setIncore(true);
    fwi.setSnapfile(tmpname("fwie2d"));
    int r = full_snapinc > 0 ? fwi.run() : fwi.run_optimal();
    size_t n = (size_t)g->nx * g->nz, nd = (size_t)nr * g->nt;
    std::memcpy(vpgrad, img[0]->getImagedata(), sizeof(T) * n);
    std::memcpy(vsgrad, img[1]->getImagedata(), sizeof(T) * n);
    std::memcpy(rhograd, img[2]->getImagedata(), sizeof(T) * n);
    std::memcpy(wavgrad, wg->getData(), sizeof(T) * (size_t)ns * g->nt);
    for (int k = 0; k < 3; k++) {
        std::memcpy(mods + k * nd, dm[k]->getData(), sizeof(T) * nd);
        std::memcpy(ress + k * nd, dr[k]->getData(), sizeof(T) * nd);
    }
    *misfit = (double)fwi.getMisfit();
    return r;
}

/* FwiAcoustic3D::run_optimal (lib/fwi.cpp:1991-2160), DIFFERENCE (0) or CORRELATION (1) misfit. */
template <typename T>
int fwi_a3d(const ref_grid *g, const T *vp, const T *rho, int ns, const double *sc, const T *wav, int nr,
            const double *gc, const T *obs, int ncheck, T *vpgrad, T *rhograd, T *wavgrad, T *datamod, T *datares,
            double *misfit, int misfit_type = 0)
{
    auto model = make_a3d<T>(g, vp, rho);
    auto geom = model->getGeom();
    auto src = make_data3d<T>(ns, g, sc, PRESSURE, SMAP, geom, wav);
    auto dobs = make_data3d<T>(nr, g, gc, PRESSURE, GMAP, geom, obs);
    auto dmod = make_data3d<T>(nr, g, gc, PRESSURE, GMAP, geom, nullptr);
    auto dres = make_data3d<T>(nr, g, gc, PRESSURE, GMAP, geom, nullptr);
    auto wg = make_data3d<T>(ns, g, sc, PRESSURE, SMAP, geom, nullptr);
    auto ivp = std::make_shared<Image3D<T>>(g->nx, g->ny, g->nz, 1, 1, 1, (T)g->dx, (T)g->dy, (T)g->dz, (T)g->ox,
                                            (T)g->oy, (T)g->oz);
    auto irho = std::make_shared<Image3D<T>>(g->nx, g->ny, g->nz, 1, 1, 1, (T)g->dx, (T)g->dy, (T)g->dz, (T)g->ox,
                                             (T)g->oy, (T)g->oz);
    FwiAcoustic3D<T> fwi(model, src, dobs, g->order, 1);
    fwi.setDatamodP(dmod);
    fwi.setDataresP(dres);
    fwi.setVpgrad(ivp);
    fwi.setRhograd(irho);
    fwi.setWavgrad(wg);
    fwi.setMisfit_type((rs_fwimisfit)misfit_type);
    fwi.setNcheck(ncheck);
    fwi.setIncore(true);
    fwi.setSnapfile(tmpname("fwia3d"));
    int r = fwi.run_optimal();
    size_t n = (size_t)g->nx * g->ny * g->nz;
    std::memcpy(vpgrad, ivp->getImagedata(), sizeof(T) * n);
    std::memcpy(rhograd, irho->getImagedata(), sizeof(T) * n);
    std::memcpy(wavgrad, wg->getData(), sizeof(T) * (size_t)ns * g->nt);
    std::memcpy(datamod, dmod->getData(), sizeof(T) * (size_t)nr * g->nt);
    std::memcpy(datares, dres->getData(), sizeof(T) * (size_t)nr * g->nt);
    *misfit = (double)fwi.getMisfit();
    return r;
}

/* FwiElastic3D::run_optimal (lib/fwi.cpp:6770-6990), DIFFERENCE misfit: Ux, Uy and
 * Uz data of nr receivers (one coordinate set for all three), every gradient set. */
template <typename T>
int fwi_e3d(const ref_grid *g, const T *vp, const T *vs, const T *rho, int ns, const double *sc, const T *wav,
            int sfield, int nr, const double *gc, const T *obsx, const T *obsy, const T *obsz, int ncheck,
            T *vpgrad, T *vsgrad, T *rhograd, T *wavgrad, T *mods, T *ress, double *misfit)
{
    auto model = make_e3d<T>(g, vp, vs, rho);
    auto geom = model->getGeom();
    auto src = make_data3d<T>(ns, g, sc, sfield, SMAP, geom, wav);
    auto dx = make_data3d<T>(nr, g, gc, VX, GMAP, geom, obsx);
    auto dy = make_data3d<T>(nr, g, gc, VY, GMAP, geom, obsy);
    auto dz = make_data3d<T>(nr, g, gc, VZ, GMAP, geom, obsz);
    const int fields[3] = {VX, VY, VZ};
    std::shared_ptr<Data3D<T>> dm[3], dr[3];
    for (int k = 0; k < 3; k++) {
        dm[k] = make_data3d<T>(nr, g, gc, fields[k], GMAP, geom, nullptr);
        dr[k] = make_data3d<T>(nr, g, gc, fields[k], GMAP, geom, nullptr);
    }
    auto wg = make_data3d<T>(ns, g, sc, sfield, SMAP, geom, nullptr);
    std::shared_ptr<Image3D<T>> img[3];
    for (int k = 0; k < 3; k++) {
        img[k] = std::make_shared<Image3D<T>>(g->nx, g->ny, g->nz, 1, 1, 1, (T)g->dx, (T)g->dy, (T)g->dz, (T)g->ox,
                                              (T)g->oy, (T)g->oz);
        img[k]->allocateImage();
    }
    FwiElastic3D<T> fwi(model, src, dx, dy, dz, g->order, 1);
    fwi.setDatamodUx(dm[0]); fwi.setDatamodUy(dm[1]); fwi.setDatamodUz(dm[2]);
    fwi.setDataresUx(dr[0]); fwi.setDataresUy(dr[1]); fwi.setDataresUz(dr[2]);
    fwi.setVpgrad(img[0]); fwi.setVsgrad(img[1]); fwi.setRhograd(img[2]);
    fwi.setWavgrad(wg);
    fwi.setMisfit_type(DIFFERENCE);
    fwi.setNcheck(ncheck);
    fwi.setIncore(true);
    fwi.setSnapfile(tmpname("fwie3d"));
    int r = fwi.run_optimal();
    size_t n = (size_t)g->nx * g->ny * g->nz, nd = (size_t)nr * g->nt;
    std::memcpy(vpgrad, img[0]->getImagedata(), sizeof(T) * n);
    std::memcpy(vsgrad, img[1]->getImagedata(), sizeof(T) * n);
    std::memcpy(rhograd, img[2]->getImagedata(), sizeof(T) * n);
    std::memcpy(wavgrad, wg->getData(), sizeof(T) * (size_t)ns * g->nt);
    for (int k = 0; k < 3; k++) {
        std::memcpy(mods + k * nd, dm[k]->getData(), sizeof(T) * nd);
        std::memcpy(ress + k * nd, dr[k]->getData(), sizeof(T) * nd);
    }
    *misfit = (double)fwi.getMisfit();
    return r;
}

/* nsteps of forwardstepVelocity / forwardstepStress / insertSource on a fresh
 * wavefield, state copied out field by field (step-level parity). */
template <typename T>
int steps_e2d(const ref_grid *g, const T *vp, const T *vs, const T *rho, int ns, const double *sc, const T *wav,
              int sfield, int nsteps, int adjoint, T *state)
{
    auto model = make_e2d<T>(g, vp, vs, rho);
    auto src = make_data2d<T>(ns, g, sc, sfield, SMAP, model->getGeom(), wav);
    auto waves = std::make_shared<WavesElastic2D<T>>(model, g->nt, (T)g->dt, (T)0.0);
    auto der = std::make_shared<Der<T>>(waves->getNx_pml(), 1, waves->getNz_pml(), waves->getDx(), 1.0,
                                        waves->getDz(), g->order);
    waves->getPml()->setSmax(SMAX);
    waves->getPml()->computeABC();
    size_t n = (size_t)waves->getNx_pml() * waves->getNz_pml();
    if (adjoint) {
        T *f[5] = {waves->getVx(), waves->getVz(), waves->getSxx(), waves->getSzz(), waves->getSxz()};
        for (int k = 0; k < 5; k++) std::memcpy(f[k], state + k * n, sizeof(T) * n);
    }
    for (int it = 0; it < nsteps; it++) {
        if (adjoint) {
            waves->backwardstepVelocity(model, der);
            waves->backwardstepStress(model, der);
        } else {
            waves->forwardstepVelocity(model, der);
            waves->forwardstepStress(model, der);
            waves->insertSource(model, src, SMAP, it);
        }
    }
    T *f[5] = {waves->getVx(), waves->getVz(), waves->getSxx(), waves->getSzz(), waves->getSxz()};
    for (int k = 0; k < 5; k++) std::memcpy(state + k * n, f[k], sizeof(T) * n);
    return 1;
}

/* The nine WavesElastic3D fields after nsteps forward steps with source injection
 * (or, with adjoint set, nsteps backwardstep* steps from the given state), in the
 * order Vx, Vy, Vz, Sxx, Syy, Szz, Syz, Sxz, Sxy, each padded [nz][ny][nx]. */
template <typename T>
int steps_e3d(const ref_grid *g, const T *vp, const T *vs, const T *rho, int ns, const double *sc, const T *wav,
              int sfield, int nsteps, int adjoint, T *state)
{
    auto model = make_e3d<T>(g, vp, vs, rho);
    auto src = make_data3d<T>(ns, g, sc, sfield, SMAP, model->getGeom(), wav);
    auto waves = std::make_shared<WavesElastic3D<T>>(model, g->nt, (T)g->dt, (T)0.0);
    auto der = std::make_shared<Der<T>>(waves->getNx_pml(), waves->getNy_pml(), waves->getNz_pml(), waves->getDx(),
                                        waves->getDy(), waves->getDz(), g->order);
    waves->getPml()->setSmax(SMAX);
    waves->getPml()->computeABC();
    size_t n = (size_t)waves->getNx_pml() * waves->getNy_pml() * waves->getNz_pml();
    T *f[9] = {waves->getVx(), waves->getVy(), waves->getVz(), waves->getSxx(), waves->getSyy(),
               waves->getSzz(), waves->getSyz(), waves->getSxz(), waves->getSxy()};
    if (adjoint) {
        waves->setAdjoint();
        for (int k = 0; k < 9; k++) std::memcpy(f[k], state + k * n, sizeof(T) * n);
    }
    for (int it = 0; it < nsteps; it++) {
        if (adjoint) {
            waves->backwardstepVelocity(model, der);
            waves->backwardstepStress(model, der);
        } else {
            waves->forwardstepVelocity(model, der);
            waves->forwardstepStress(model, der);
            waves->insertSource(model, src, SMAP, it);
        }
    }
    for (int k = 0; k < 9; k++) std::memcpy(state + k * n, f[k], sizeof(T) * n);
    return 1;
}

template <typename T>
int steps_a2d(const ref_grid *g, const T *vp, const T *rho, int ns, const double *sc, const T *wav, int sfield,
              int nsteps, T *state)
{
    auto model = make_a2d<T>(g, vp, rho);
    auto src = make_data2d<T>(ns, g, sc, sfield, SMAP, model->getGeom(), wav);
    auto waves = std::make_shared<WavesAcoustic2D<T>>(model, g->nt, (T)g->dt, (T)0.0);
    auto der = std::make_shared<Der<T>>(waves->getNx_pml(), 1, waves->getNz_pml(), waves->getDx(), 1.0,
                                        waves->getDz(), g->order);
    waves->getPml()->setSmax(SMAX);
    waves->getPml()->computeABC();
    for (int it = 0; it < nsteps; it++) {
        waves->forwardstepVelocity(model, der);
        waves->forwardstepStress(model, der);
        waves->insertSource(model, src, SMAP, it);
    }
    size_t n = (size_t)waves->getNx_pml() * waves->getNz_pml();
    T *f[3] = {waves->getP(), waves->getVx(), waves->getVz()};
    for (int k = 0; k < 3; k++) std::memcpy(state + k * n, f[k], sizeof(T) * n);
    return 1;
}

} // namespace

extern "C" {

/* Interp<float>::interp (lib/interp.cpp:123-186) on trace-major float arrays. */
int ref_interp_f(int mode, int ntr, int n1, float o1, float d1, const float *in, int n2, float o2, float d2,
                 float *out)
{
    auto from = std::make_shared<rockseis::Data2D<float>>(ntr, n1, d1, o1);
    auto to = std::make_shared<rockseis::Data2D<float>>(ntr, n2, d2, o2);
    std::memcpy(from->getData(), in, sizeof(float) * (size_t)ntr * n1);
    rockseis::Interp<float> ip((rockseis::rs_interpmode)mode);
    ip.interp(from, to);
    std::memcpy(out, to->getData(), sizeof(float) * (size_t)ntr * n2);
    return 1;
}

int ref_steps_e2d_f(const ref_grid *g, const float *vp, const float *vs, const float *rho, int ns, const double *sc,
                    const float *wav, int sfield, int nsteps, int adjoint, float *state)
{ return steps_e2d<float>(g, vp, vs, rho, ns, sc, wav, sfield, nsteps, adjoint, state); }
int ref_steps_e3d_f(const ref_grid *g, const float *vp, const float *vs, const float *rho, int ns, const double *sc,
                    const float *wav, int sfield, int nsteps, int adjoint, float *state)
{ return steps_e3d<float>(g, vp, vs, rho, ns, sc, wav, sfield, nsteps, adjoint, state); }
int ref_steps_a2d_f(const ref_grid *g, const float *vp, const float *rho, int ns, const double *sc,
                    const float *wav, int sfield, int nsteps, float *state)
{ return steps_a2d<float>(g, vp, rho, ns, sc, wav, sfield, nsteps, state); }

/* which: 0 ddx_fw 1 ddy_fw 2 ddz_fw 3 ddx_bw 4 ddy_bw 5 ddz_bw  (lib/der.cpp:155-540) */
void ref_der_f(int nx, int ny, int nz, double dx, double dy, double dz, int order, int which,
               const float *f, float *df)
{ der_apply<float>(nx, ny, nz, dx, dy, dz, order, which, f, df); }
void ref_der_d(int nx, int ny, int nz, double dx, double dy, double dz, int order, int which,
               const double *f, double *df)
{ der_apply<double>(nx, ny, nz, dx, dy, dz, order, which, f, df); }

/* 12 tables of lpml: A,B,C ltf; A,B,C ltf_stag; A,B,C rbb; A,B,C rbb_stag (lib/pml.cpp:79-126) */
void ref_pml_tables_f(int lpml, double dt, float *out) { pml_tables<float>(lpml, dt, out); }
void ref_pml_tables_d(int lpml, double dt, double *out) { pml_tables<double>(lpml, dt, out); }

/* Staggered padded parameters (lib/model.cpp:1350-1411, 2720-2802). */
void ref_stagger_a2d_f(const ref_grid *g, const float *vp, const float *rho, float *Rx, float *Rz, float *L)
{
    auto m = make_a2d<float>(g, vp, rho);
    size_t n = (size_t)(g->nx + 2 * g->lpml) * (g->nz + 2 * g->lpml);
    std::memcpy(Rx, m->getRx(), 4 * n);
    std::memcpy(Rz, m->getRz(), 4 * n);
    std::memcpy(L, m->getL(), 4 * n);
}
void ref_stagger_e2d_f(const ref_grid *g, const float *vp, const float *vs, const float *rho,
                       float *Rx, float *Rz, float *L, float *L2M, float *M)
{
    auto m = make_e2d<float>(g, vp, vs, rho);
    size_t n = (size_t)(g->nx + 2 * g->lpml) * (g->nz + 2 * g->lpml);
    std::memcpy(Rx, m->getRx(), 4 * n);
    std::memcpy(Rz, m->getRz(), 4 * n);
    std::memcpy(L, m->getL(), 4 * n);
    std::memcpy(L2M, m->getL2M(), 4 * n);
    std::memcpy(M, m->getM(), 4 * n);
}
void ref_stagger_a3d_f(const ref_grid *g, const float *vp, const float *rho, float *Rx, float *Ry,
                       float *Rz, float *L)
{
    auto m = make_a3d<float>(g, vp, rho);
    size_t n = (size_t)(g->nx + 2 * g->lpml) * (g->ny + 2 * g->lpml) * (g->nz + 2 * g->lpml);
    std::memcpy(Rx, m->getRx(), 4 * n);
    std::memcpy(Ry, m->getRy(), 4 * n);
    std::memcpy(Rz, m->getRz(), 4 * n);
    std::memcpy(L, m->getL(), 4 * n);
}
void ref_stagger_e3d_f(const ref_grid *g, const float *vp, const float *vs, const float *rho,
                       float *Rx, float *Ry, float *Rz, float *L, float *L2M, float *M_yz,
                       float *M_xz, float *M_xy)
{
    auto m = make_e3d<float>(g, vp, vs, rho);
    size_t n = (size_t)(g->nx + 2 * g->lpml) * (g->ny + 2 * g->lpml) * (g->nz + 2 * g->lpml);
    std::memcpy(Rx, m->getRx(), 4 * n);
    std::memcpy(Ry, m->getRy(), 4 * n);
    std::memcpy(Rz, m->getRz(), 4 * n);
    std::memcpy(L, m->getL(), 4 * n);
    std::memcpy(L2M, m->getL2M(), 4 * n);
    std::memcpy(M_yz, m->getM_yz(), 4 * n);
    std::memcpy(M_xz, m->getM_xz(), 4 * n);
    std::memcpy(M_xy, m->getM_xy(), 4 * n);
}

/* Geometry2D::makeMap (lib/geometry.cpp:137-230), T=float coordinates. */
void ref_makemap2d_field_f(const ref_grid *g, int ntr, const double *coords, int which, int field, int *map,
                           float *shift)
{
    auto m = std::make_shared<ModelAcoustic2D<float>>(g->nx, g->nz, g->lpml, (float)g->dx, (float)g->dz,
                                                      (float)g->ox, (float)g->oz, g->fs != 0);
    auto d = make_data2d<float>(ntr, g, coords, field, which != 0, m->getGeom(), nullptr);
    Point2D<int> *mp = which ? d->getGeom()->getGmap() : d->getGeom()->getSmap();
    Point2D<float> *sh = which ? d->getGeom()->getGshift() : d->getGeom()->getSshift();
    for (int i = 0; i < ntr; i++) {
        map[2 * i] = mp[i].x; map[2 * i + 1] = mp[i].y;
        shift[2 * i] = sh[i].x; shift[2 * i + 1] = sh[i].y;
    }
}
void ref_makemap2d_f(const ref_grid *g, int ntr, const double *coords, int which, int *map, float *shift)
{
    ref_makemap2d_field_f(g, ntr, coords, which, PRESSURE, map, shift);
}
void ref_makemap3d_field_f(const ref_grid *g, int ntr, const double *coords, int which, int field, int *map,
                           float *shift)
{
    auto m = std::make_shared<ModelAcoustic3D<float>>(g->nx, g->ny, g->nz, g->lpml, (float)g->dx,
                                                      (float)g->dy, (float)g->dz, (float)g->ox,
                                                      (float)g->oy, (float)g->oz, g->fs != 0);
    auto d = make_data3d<float>(ntr, g, coords, field, which != 0, m->getGeom(), nullptr);
    Point3D<int> *mp = which ? d->getGeom()->getGmap() : d->getGeom()->getSmap();
    Point3D<float> *sh = which ? d->getGeom()->getGshift() : d->getGeom()->getSshift();
    for (int i = 0; i < ntr; i++) {
        map[3 * i] = mp[i].x; map[3 * i + 1] = mp[i].y; map[3 * i + 2] = mp[i].z;
        shift[3 * i] = sh[i].x; shift[3 * i + 1] = sh[i].y; shift[3 * i + 2] = sh[i].z;
    }
}
void ref_makemap3d_f(const ref_grid *g, int ntr, const double *coords, int which, int *map, float *shift)
{
    ref_makemap3d_field_f(g, ntr, coords, which, PRESSURE, map, shift);
}

/* Revolve::revolve action trace (lib/revolve.cpp:150-305).  Returns the number of
 * actions written (action code, capo after the call), or -1 if max is exceeded. */
int ref_revolve_trace(int nt, int ncheck, int *actions, int *capos, int *checks, int max)
{
    Revolve<float> r(nt, ncheck, true);
    int k = 0;
    revolve_action a;
    do {
        a = r.revolve();
        if (k >= max) return -1;
        actions[k] = (int)a;
        capos[k] = r.getCapo();
        checks[k] = r.getCheck();
        k++;
    } while (a != terminate && a != error);
    return k;
}
int ref_revolve_numforw(int nt, int ncheck)
{
    Revolve<float> r(nt, ncheck, true);
    return r.numforw(nt, ncheck);
}
int ref_revolve_adjust(int nt)
{
    Revolve<float> r(nt, 2, true);
    return r.adjust(nt);
}

int ref_mod_a2d_f(const ref_grid *g, const float *vp, const float *rho, int ns, const double *sc,
                  const float *wav, int sfield, int nr, const double *gc, int rfield, float *out)
{ return mod_a2d<float>(g, vp, rho, ns, sc, wav, sfield, nr, gc, rfield, out); }
int ref_mod_a2d_d(const ref_grid *g, const double *vp, const double *rho, int ns, const double *sc,
                  const double *wav, int sfield, int nr, const double *gc, int rfield, double *out)
{ return mod_a2d<double>(g, vp, rho, ns, sc, wav, sfield, nr, gc, rfield, out); }

int ref_mod_e2d_f(const ref_grid *g, const float *vp, const float *vs, const float *rho, int ns,
                  const double *sc, const float *wav, int sfield, int nr, const double *gc, int rfield,
                  float *out)
{ return mod_e2d<float>(g, vp, vs, rho, ns, sc, wav, sfield, nr, gc, rfield, out); }
int ref_mod_e2d_d(const ref_grid *g, const double *vp, const double *vs, const double *rho, int ns,
                  const double *sc, const double *wav, int sfield, int nr, const double *gc, int rfield,
                  double *out)
{ return mod_e2d<double>(g, vp, vs, rho, ns, sc, wav, sfield, nr, gc, rfield, out); }

int ref_mod_a3d_f(const ref_grid *g, const float *vp, const float *rho, int ns, const double *sc,
                  const float *wav, int sfield, int nr, const double *gc, int rfield, float *out)
{ return mod_a3d<float>(g, vp, rho, ns, sc, wav, sfield, nr, gc, rfield, out); }

int ref_mod_e3d_f(const ref_grid *g, const float *vp, const float *vs, const float *rho, int ns,
                  const double *sc, const float *wav, int sfield, int nr, const double *gc, int rfield,
                  float *out)
{ return mod_e3d<float>(g, vp, vs, rho, ns, sc, wav, sfield, nr, gc, rfield, out); }

int ref_fwi_a3d_f(const ref_grid *g, const float *vp, const float *rho, int ns, const double *sc, const float *wav,
                  int nr, const double *gc, const float *obs, int ncheck, float *vpgrad, float *rhograd,
                  float *wavgrad, float *datamod, float *datares, double *misfit)
{
    return fwi_a3d<float>(g, vp, rho, ns, sc, wav, nr, gc, obs, ncheck, vpgrad, rhograd, wavgrad, datamod, datares,
                          misfit);
}
int ref_fwi_a3d_corr_f(const ref_grid *g, const float *vp, const float *rho, int ns, const double *sc,
                       const float *wav, int nr, const double *gc, const float *obs, int ncheck, float *vpgrad,
                       float *rhograd, float *wavgrad, float *datamod, float *datares, double *misfit)
{
    return fwi_a3d<float>(g, vp, rho, ns, sc, wav, nr, gc, obs, ncheck, vpgrad, rhograd, wavgrad, datamod, datares,
                          misfit, 1);
}
/* FwiAcoustic3D::run_optimal with any rs_fwimisfit value (ADAPTIVE_GAUSS = 2, ADAPTIVE_LINEAR = 3). */
int ref_fwi_a3d_misfit_f(const ref_grid *g, const float *vp, const float *rho, int ns, const double *sc,
                         const float *wav, int nr, const double *gc, const float *obs, int ncheck, float *vpgrad,
                         float *rhograd, float *wavgrad, float *datamod, float *datares, double *misfit,
                         int misfit_type)
{
    return fwi_a3d<float>(g, vp, rho, ns, sc, wav, nr, gc, obs, ncheck, vpgrad, rhograd, wavgrad, datamod, datares,
                          misfit, misfit_type);
}
/* Model::getLocalsize2d / getLocalsize3d (lib/model.cpp:272-470): the aperture window of
 * ntr traces whose source and receiver coordinates are both given (x,z or x,y,z per
 * trace); map = 0 (SMAP) or 1 (GMAP). */
void ref_localsize2d_f(const ref_grid *g, int ntr, const double *sc, const double *gc, double aperture, int map,
                       long long *start, long long *size)
{
    ModelAcoustic2D<float> m(g->nx, g->nz, g->lpml, (float)g->dx, (float)g->dz, (float)g->ox, (float)g->oz,
                             g->fs != 0);
    auto d = std::make_shared<Data2D<float>>(ntr, 1, 1.0f, 0.0f);
    auto geo = d->getGeom();
    for (int i = 0; i < ntr; i++) {
        geo->getScoords()[i].x = (float)sc[2 * i];
        geo->getScoords()[i].y = (float)sc[2 * i + 1];
        geo->getGcoords()[i].x = (float)gc[2 * i];
        geo->getGcoords()[i].y = (float)gc[2 * i + 1];
    }
    off_t st = 0;
    size_t sz = 0;
    m.getLocalsize2d(d, (float)aperture, map != 0, &st, &sz);
    *start = (long long)st;
    *size = (long long)sz;
}
void ref_localsize3d_f(const ref_grid *g, int ntr, const double *sc, const double *gc, double apx, double apy,
                       int map, long long *out)
{
    ModelAcoustic3D<float> m(g->nx, g->ny, g->nz, g->lpml, (float)g->dx, (float)g->dy, (float)g->dz, (float)g->ox,
                             (float)g->oy, (float)g->oz, g->fs != 0);
    auto d = std::make_shared<Data3D<float>>(ntr, 1, 1.0f, 0.0f);
    auto geo = d->getGeom();
    for (int i = 0; i < ntr; i++) {
        Point3D<float> *s = geo->getScoords(), *r = geo->getGcoords();
        s[i].x = (float)sc[3 * i]; s[i].y = (float)sc[3 * i + 1]; s[i].z = (float)sc[3 * i + 2];
        r[i].x = (float)gc[3 * i]; r[i].y = (float)gc[3 * i + 1]; r[i].z = (float)gc[3 * i + 2];
    }
    off_t sx = 0, sy = 0;
    size_t nx = 0, ny = 0;
    m.getLocalsize3d(d, (float)apx, (float)apy, map != 0, &sx, &nx, &sy, &ny);
    out[0] = (long long)sx; out[1] = (long long)nx; out[2] = (long long)sy; out[3] = (long long)ny;
}
int ref_fwi_e3d_f(const ref_grid *g, const float *vp, const float *vs, const float *rho, int ns, const double *sc,
                  const float *wav, int sfield, int nr, const double *gc, const float *obsx, const float *obsy,
                  const float *obsz, int ncheck, float *vpgrad, float *vsgrad, float *rhograd, float *wavgrad,
                  float *mods, float *ress, double *misfit)
{
    return fwi_e3d<float>(g, vp, vs, rho, ns, sc, wav, sfield, nr, gc, obsx, obsy, obsz, ncheck, vpgrad, vsgrad,
                          rhograd, wavgrad, mods, ress, misfit);
}
int ref_fwi_e2d_f(const ref_grid *g, const float *vp, const float *vs, const float *rho, int ns, const double *sc,
                  const float *wav, int sfield, int nr, const double *gc, const float *obsp, const float *obsx,
                  const float *obsz, int ncheck, float *vpgrad, float *vsgrad, float *rhograd, float *wavgrad,
                  float *mods, float *ress, double *misfit)
{
    return fwi_e2d<float>(g, vp, vs, rho, ns, sc, wav, sfield, nr, gc, obsp, obsx, obsz, ncheck, vpgrad, vsgrad,
                          rhograd, wavgrad, mods, ress, misfit);
}
int ref_fwi_e2d_corr_f(const ref_grid *g, const float *vp, const float *vs, const float *rho, int ns,
                       const double *sc, const float *wav, int sfield, int nr, const double *gc, const float *obsp,
                       const float *obsx, const float *obsz, int ncheck, float *vpgrad, float *vsgrad, float *rhograd,
                       float *wavgrad, float *mods, float *ress, double *misfit)
{
    return fwi_e2d<float>(g, vp, vs, rho, ns, sc, wav, sfield, nr, gc, obsp, obsx, obsz, ncheck, vpgrad, vsgrad,
                          rhograd, wavgrad, mods, ress, misfit, 1);
}
/* FwiElastic2D::run (lib/fwi.cpp:3774-3934): full Vx/Vz snapshots every snapinc steps. */
int ref_fwi_e2d_full_f(const ref_grid *g, const float *vp, const float *vs, const float *rho, int ns,
                       const double *sc, const float *wav, int sfield, int nr, const double *gc, const float *obsp,
                       const float *obsx, const float *obsz, int snapinc, float *vpgrad, float *vsgrad,
                       float *rhograd, float *wavgrad, float *mods, float *ress, double *misfit)
{
    return fwi_e2d<float>(g, vp, vs, rho, ns, sc, wav, sfield, nr, gc, obsp, obsx, obsz, 0, vpgrad, vsgrad,
                          rhograd, wavgrad, mods, ress, misfit, 0, snapinc);
}
/* FwiElastic2D::run_optimal with any rs_fwimisfit value (ADAPTIVE_GAUSS = 2, ADAPTIVE_LINEAR = 3,
 * ADAPTIVE_SINGLE = 4). */
int ref_fwi_e2d_misfit_f(const ref_grid *g, const float *vp, const float *vs, const float *rho, int ns,
                         const double *sc, const float *wav, int sfield, int nr, const double *gc, const float *obsp,
                         const float *obsx, const float *obsz, int ncheck, float *vpgrad, float *vsgrad,
                         float *rhograd, float *wavgrad, float *mods, float *ress, double *misfit, int misfit_type)
{
    return fwi_e2d<float>(g, vp, vs, rho, ns, sc, wav, sfield, nr, gc, obsp, obsx, obsz, ncheck, vpgrad, vsgrad,
                          rhograd, wavgrad, mods, ress, misfit, misfit_type);
}
int ref_fwi_a2d_f(const ref_grid *g, const float *vp, const float *rho, int ns, const double *sc,
                  const float *wav, int nr, const double *gc, const float *obs, int ncheck,
                  int misfit_type, float *vpgrad, float *rhograd, float *wavgrad, float *datamod,
                  float *datares, double *misfit)
{ return fwi_a2d<float>(g, vp, rho, ns, sc, wav, nr, gc, obs, ncheck, misfit_type, vpgrad, rhograd,
                        wavgrad, datamod, datares, misfit); }
/* FwiAcoustic2D::run (lib/fwi.cpp:1030-1156): full snapshots every snapinc steps. */
int ref_fwi_a2d_full_f(const ref_grid *g, const float *vp, const float *rho, int ns, const double *sc,
                       const float *wav, int nr, const double *gc, const float *obs, int snapinc, int noreverse,
                       int misfit_type, float *vpgrad, float *rhograd, float *wavgrad, float *datamod,
                       float *datares, double *misfit)
{ return fwi_a2d<float>(g, vp, rho, ns, sc, wav, nr, gc, obs, 0, misfit_type, vpgrad, rhograd, wavgrad, datamod,
                        datares, misfit, nullptr, snapinc, noreverse); }
int ref_fwi_a2d_ilum_f(const ref_grid *g, const float *vp, const float *rho, int ns, const double *sc,
                       const float *wav, int nr, const double *gc, const float *obs, int ncheck,
                       int misfit_type, float *vpgrad, float *rhograd, float *wavgrad, float *datamod,
                       float *datares, double *misfit, float *srcilum)
{ return fwi_a2d<float>(g, vp, rho, ns, sc, wav, nr, gc, obs, ncheck, misfit_type, vpgrad, rhograd,
                        wavgrad, datamod, datares, misfit, srcilum); }
int ref_fwi_a2d_d(const ref_grid *g, const double *vp, const double *rho, int ns, const double *sc,
                  const double *wav, int nr, const double *gc, const double *obs, int ncheck,
                  int misfit_type, double *vpgrad, double *rhograd, double *wavgrad, double *datamod,
                  double *datares, double *misfit)
{ return fwi_a2d<double>(g, vp, rho, ns, sc, wav, nr, gc, obs, ncheck, misfit_type, vpgrad, rhograd,
                         wavgrad, datamod, datares, misfit); }

} // extern "C"
