#pragma once
/*
 * ref_harness_common.h -- in-process driver for the UNMODIFIED RockSeis reference
 * library (lib/*.cpp compiled from the read-only reference tree by
 * oracle/Makefile into oracle/_ref/librsref.so).
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the pin for the oracle and for the
 * CUDA path: it builds the reference's own objects (ModelAcoustic2D, Data2D,
 * WavesAcoustic2D, Der, Revolve, FwiAcoustic2D, RtmAcoustic2D, ...) from plain
 * arrays and calls the reference's public methods, so the numbers that come
 * back are the reference's numbers.  Nothing under rockseis_b200/ links it.
 *
 * Every entry point is extern "C" with plain pointers so pytest can call it
 * through ctypes.  `_f` = reference built with T=float, `_d` = T=double.
 * Input layouts follow the reference: grids x fastest (I2D = iz*nx+ix,
 * I3D = iz*nx*ny + iy*nx + ix), traces trace-major (data[it + itr*nt]).
 * Coordinates are passed as doubles (x,z) in 2D or (x,y,z) in 3D and cast to T.
 */
#include <cstring>
#include <memory>
#include <string>
#include <vector>
#include <unistd.h>

#include "der.h"
#include "pml.h"
#include "waves.h"
#include "model.h"
#include "data.h"
#include "geometry.h"
#include "image.h"
#include "modelling.h"
#include "revolve.h"

using namespace rockseis;

extern "C" {
typedef struct {
    int nx, ny, nz;      /* unpadded model size (ny = 1 in 2D) */
    int lpml, order, fs;
    double dx, dy, dz, ox, oy, oz;
    double dt;
    int nt;
} ref_grid;
}

namespace refh {

inline std::string tmpname(const char *tag)
{
    char buf[256];
    snprintf(buf, sizeof buf, "/tmp/rsref_%s_%d", tag, (int)getpid());
    return std::string(buf);
}

template <typename T>
std::shared_ptr<ModelAcoustic2D<T>> make_a2d(const ref_grid *g, const T *vp, const T *rho)
{
    auto m = std::make_shared<ModelAcoustic2D<T>>(g->nx, g->nz, g->lpml, (T)g->dx, (T)g->dz,
                                                  (T)g->ox, (T)g->oz, g->fs != 0);
    m->createModel();
    std::memcpy(m->getVp(), vp, sizeof(T) * g->nx * g->nz);
    std::memcpy(m->getR(), rho, sizeof(T) * g->nx * g->nz);
    m->staggerModels();
    return m;
}

template <typename T>
std::shared_ptr<ModelElastic2D<T>> make_e2d(const ref_grid *g, const T *vp, const T *vs, const T *rho)
{
    auto m = std::make_shared<ModelElastic2D<T>>(g->nx, g->nz, g->lpml, (T)g->dx, (T)g->dz,
                                                 (T)g->ox, (T)g->oz, g->fs != 0);
    m->createModel();
    std::memcpy(m->getVp(), vp, sizeof(T) * g->nx * g->nz);
    std::memcpy(m->getVs(), vs, sizeof(T) * g->nx * g->nz);
    std::memcpy(m->getR(), rho, sizeof(T) * g->nx * g->nz);
    m->staggerModels();
    return m;
}

template <typename T>
std::shared_ptr<ModelAcoustic3D<T>> make_a3d(const ref_grid *g, const T *vp, const T *rho)
{
    auto m = std::make_shared<ModelAcoustic3D<T>>(g->nx, g->ny, g->nz, g->lpml, (T)g->dx, (T)g->dy,
                                                  (T)g->dz, (T)g->ox, (T)g->oy, (T)g->oz, g->fs != 0);
    m->createModel();
    size_t n = (size_t)g->nx * g->ny * g->nz;
    std::memcpy(m->getVp(), vp, sizeof(T) * n);
    std::memcpy(m->getR(), rho, sizeof(T) * n);
    m->staggerModels();
    return m;
}

template <typename T>
std::shared_ptr<ModelElastic3D<T>> make_e3d(const ref_grid *g, const T *vp, const T *vs, const T *rho)
{
    auto m = std::make_shared<ModelElastic3D<T>>(g->nx, g->ny, g->nz, g->lpml, (T)g->dx, (T)g->dy,
                                                 (T)g->dz, (T)g->ox, (T)g->oy, (T)g->oz, g->fs != 0);
    m->createModel();
    size_t n = (size_t)g->nx * g->ny * g->nz;
    std::memcpy(m->getVp(), vp, sizeof(T) * n);
    std::memcpy(m->getVs(), vs, sizeof(T) * n);
    std::memcpy(m->getR(), rho, sizeof(T) * n);
    m->staggerModels();
    return m;
}

/* A 2D trace set: source coords go into scoords, receiver coords into gcoords.
 * which = SMAP builds the source map, GMAP the receiver map. */
template <typename T>
std::shared_ptr<Data2D<T>> make_data2d(int ntr, const ref_grid *g, const double *coords, int field,
                                       bool which, std::shared_ptr<Geometry<T>> mgeom, const T *trace_data)
{
    auto d = std::make_shared<Data2D<T>>(ntr, g->nt, (T)g->dt, (T)0.0);
    auto geo = d->getGeom();
    for (int i = 0; i < ntr; i++) {
        if (which == SMAP) {
            geo->getScoords()[i].x = (T)coords[2 * i];
            geo->getScoords()[i].y = (T)coords[2 * i + 1];
        } else {
            geo->getGcoords()[i].x = (T)coords[2 * i];
            geo->getGcoords()[i].y = (T)coords[2 * i + 1];
        }
    }
    d->setField((rs_field)field);
    if (trace_data) std::memcpy(d->getData(), trace_data, sizeof(T) * (size_t)ntr * g->nt);
    d->makeMap(mgeom, which);
    return d;
}

template <typename T>
std::shared_ptr<Data3D<T>> make_data3d(int ntr, const ref_grid *g, const double *coords, int field,
                                       bool which, std::shared_ptr<Geometry<T>> mgeom, const T *trace_data)
{
    auto d = std::make_shared<Data3D<T>>(ntr, g->nt, (T)g->dt, (T)0.0);
    auto geo = d->getGeom();
    for (int i = 0; i < ntr; i++) {
        Point3D<T> *c = (which == SMAP) ? geo->getScoords() : geo->getGcoords();
        c[i].x = (T)coords[3 * i];
        c[i].y = (T)coords[3 * i + 1];
        c[i].z = (T)coords[3 * i + 2];
    }
    d->setField((rs_field)field);
    if (trace_data) std::memcpy(d->getData(), trace_data, sizeof(T) * (size_t)ntr * g->nt);
    d->makeMap(mgeom, which);
    return d;
}

} // namespace refh
