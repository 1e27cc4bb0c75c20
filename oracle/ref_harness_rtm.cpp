/*
 * ref_harness_rtm.cpp -- extern "C" driver of the unmodified reference RTM
 * classes.  A separate translation unit because the reference's fwi.h and
 * rtm.h both declare rs_snapmethod.  Test infrastructure only.
 */
#include "ref_harness_common.h"
#include "rtm.h"

using namespace rockseis;
using namespace refh;

namespace {
/* ---------------------------------------------------------------- RTM image */
template <typename T>
int rtm_a2d(const ref_grid *g, const T *vp, const T *rho, int ns, const double *sc, const T *wav,
            int nr, const double *gc, const T *data, int ncheck, int nhx, int nhz, T *image)
{
    auto model = make_a2d<T>(g, vp, rho);
    auto src = make_data2d<T>(ns, g, sc, PRESSURE, SMAP, model->getGeom(), wav);
    auto drec = make_data2d<T>(nr, g, gc, PRESSURE, GMAP, model->getGeom(), data);
    auto img = std::make_shared<Image2D<T>>(g->nx, g->nz, nhx, nhz, (T)g->dx, (T)g->dz, (T)g->ox, (T)g->oz);
    RtmAcoustic2D<T> rtm(model, img, src, drec, g->order, 1);
    rtm.setNcheck(ncheck);
    rtm.setIncore(true);
    rtm.setSnapfile(tmpname("rtma2d"));
    int r = rtm.run_optimal();
    std::memcpy(image, img->getImagedata(), sizeof(T) * (size_t)g->nx * g->nz * nhx * nhz);
    return r;
}

/* RtmAcoustic3D::run_optimal (lib/rtm.cpp:735-859); image [nhz][nhy][nhx][nz][ny][nx].
 * With full_snapinc > 0, RtmAcoustic3D::run (lib/rtm.cpp:640-733) with snapshots every
 * full_snapinc steps. */
template <typename T>
int rtm_a3d(const ref_grid *g, const T *vp, const T *rho, int ns, const double *sc, const T *wav,
            int nr, const double *gc, const T *data, int ncheck, int nhx, int nhy, int nhz, T *image,
            int full_snapinc = 0)
{
    auto model = make_a3d<T>(g, vp, rho);
    auto src = make_data3d<T>(ns, g, sc, PRESSURE, SMAP, model->getGeom(), wav);
    auto drec = make_data3d<T>(nr, g, gc, PRESSURE, GMAP, model->getGeom(), data);
    auto img = std::make_shared<Image3D<T>>(g->nx, g->ny, g->nz, nhx, nhy, nhz, (T)g->dx, (T)g->dy, (T)g->dz,
                                            (T)g->ox, (T)g->oy, (T)g->oz);
    RtmAcoustic3D<T> rtm(model, img, src, drec, g->order, full_snapinc > 0 ? full_snapinc : 1);
    rtm.setNcheck(ncheck);
    rtm.setIncore(true);
    rtm.setSnapfile(tmpname("rtma3d"));
    int r = full_snapinc > 0 ? rtm.run() : rtm.run_optimal();
    std::memcpy(image, img->getImagedata(), sizeof(T) * (size_t)g->nx * g->ny * g->nz * nhx * nhy * nhz);
    return r;
}

} // namespace

extern "C" {
int ref_rtm_a3d_f(const ref_grid *g, const float *vp, const float *rho, int ns, const double *sc,
                  const float *wav, int nr, const double *gc, const float *data, int ncheck, int nhx, int nhy,
                  int nhz, float *image)
{ return rtm_a3d<float>(g, vp, rho, ns, sc, wav, nr, gc, data, ncheck, nhx, nhy, nhz, image); }
int ref_rtm_a3d_full_f(const ref_grid *g, const float *vp, const float *rho, int ns, const double *sc,
                       const float *wav, int nr, const double *gc, const float *data, int snapinc, int nhx, int nhy,
                       int nhz, float *image)
{ return rtm_a3d<float>(g, vp, rho, ns, sc, wav, nr, gc, data, 0, nhx, nhy, nhz, image, snapinc); }

int ref_rtm_a2d_f(const ref_grid *g, const float *vp, const float *rho, int ns, const double *sc,
                  const float *wav, int nr, const double *gc, const float *data, int ncheck, int nhx,
                  int nhz, float *image)
{ return rtm_a2d<float>(g, vp, rho, ns, sc, wav, nr, gc, data, ncheck, nhx, nhz, image); }

/* RtmAcoustic2D::run (lib/rtm.cpp:222-326): full snapshots every snapinc steps; with
 * `edges`, RtmAcoustic2D::run_edge (lib/rtm.cpp:328-421): only the wavefield's edges are
 * saved and the source wavefield is re-propagated from them. */
static int rtm_a2d_snap(const ref_grid *g, const float *vp, const float *rho, int ns, const double *sc,
                        const float *wav, int nr, const double *gc, const float *data, int snapinc, int nhx,
                        int nhz, float *image, bool edges)
{
    auto model = make_a2d<float>(g, vp, rho);
    auto src = make_data2d<float>(ns, g, sc, PRESSURE, SMAP, model->getGeom(), wav);
    auto drec = make_data2d<float>(nr, g, gc, PRESSURE, GMAP, model->getGeom(), data);
    auto img = std::make_shared<Image2D<float>>(g->nx, g->nz, nhx, nhz, (float)g->dx, (float)g->dz, (float)g->ox,
                                                (float)g->oz);
    RtmAcoustic2D<float> rtm(model, img, src, drec, g->order, snapinc);
    rtm.setSnapfile(tmpname("rtma2dfull"));
    int r = edges ? rtm.run_edge() : rtm.run();
    std::memcpy(image, img->getImagedata(), sizeof(float) * (size_t)g->nx * g->nz * nhx * nhz);
    return r;
}

int ref_rtm_a2d_full_f(const ref_grid *g, const float *vp, const float *rho, int ns, const double *sc,
                       const float *wav, int nr, const double *gc, const float *data, int snapinc, int nhx,
                       int nhz, float *image)
{ return rtm_a2d_snap(g, vp, rho, ns, sc, wav, nr, gc, data, snapinc, nhx, nhz, image, false); }
int ref_rtm_a2d_edge_f(const ref_grid *g, const float *vp, const float *rho, int ns, const double *sc,
                       const float *wav, int nr, const double *gc, const float *data, int snapinc, int nhx,
                       int nhz, float *image)
{ return rtm_a2d_snap(g, vp, rho, ns, sc, wav, nr, gc, data, snapinc, nhx, nhz, image, true); }

} // extern "C"
