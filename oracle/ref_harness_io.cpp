/*
 * ref_harness_io.cpp -- extern "C" drivers of the unmodified reference's file and
 * sort classes (Data2D/Data3D::write and read, ModelAcoustic2D::writeVp, Sort maps
 * and gathers) for the shot-gather I/O parity tests.  Test infrastructure only.
 */
#include "ref_harness_common.h"
#include "sort.h"

using namespace rockseis;

namespace {

template <typename T>
int data_write(const char *path, int dim, int nt, double dt, double ot, int ntrace, const T *sc, const T *gc,
               const T *data)
{
    if (dim == 2) {
        auto d = std::make_shared<Data2D<T>>(ntrace, nt, (T)dt, (T)ot);
        Point2D<T> *s = d->getGeom()->getScoords(), *g = d->getGeom()->getGcoords();
        for (int i = 0; i < ntrace; i++) {
            s[i].x = sc[2 * i]; s[i].y = sc[2 * i + 1];
            g[i].x = gc[2 * i]; g[i].y = gc[2 * i + 1];
        }
        std::memcpy(d->getData(), data, sizeof(T) * (size_t)nt * ntrace);
        d->setFile(path);
        return d->write() == FILE_OK ? 1 : 0;
    }
    auto d = std::make_shared<Data3D<T>>(ntrace, nt, (T)dt, (T)ot);
    Point3D<T> *s = d->getGeom()->getScoords(), *g = d->getGeom()->getGcoords();
    for (int i = 0; i < ntrace; i++) {
        s[i].x = sc[3 * i]; s[i].y = sc[3 * i + 1]; s[i].z = sc[3 * i + 2];
        g[i].x = gc[3 * i]; g[i].y = gc[3 * i + 1]; g[i].z = gc[3 * i + 2];
    }
    std::memcpy(d->getData(), data, sizeof(T) * (size_t)nt * ntrace);
    d->setFile(path);
    return d->write() == FILE_OK ? 1 : 0;
}

template <typename T>
int data_read2d(const char *path, int nt, int ntrace, T *sc, T *gc, T *data)
{
    auto d = std::make_shared<Data2D<T>>(ntrace, nt, (T)1, (T)0);
    d->setFile(path);
    if (d->read() != FILE_OK) return 0;
    Point2D<T> *s = d->getGeom()->getScoords(), *g = d->getGeom()->getGcoords();
    for (int i = 0; i < ntrace; i++) {
        sc[2 * i] = s[i].x; sc[2 * i + 1] = s[i].y;
        gc[2 * i] = g[i].x; gc[2 * i + 1] = g[i].y;
    }
    std::memcpy(data, d->getData(), sizeof(T) * (size_t)nt * ntrace);
    return 1;
}

/* Sort::createShotmap / createReceivermap / createCMPmap, then get2DGather(number) or
 * get3DGather(number); returns the gather's trace count (0 on failure), *ngathers
 * the map's size. */
template <typename T>
int sort_gather(const char *path, int dim, int key, double dx, double dy, int order, int number, int reciprocity,
                long long *ngathers, T *sc, T *gc, T *data, int maxtr)
{
    Sort<T> s;
    s.setReciprocity(reciprocity != 0);
    bool ok = key == 0 ? s.createShotmap(path, order) : key == 1 ? s.createReceivermap(path, order)
                                                                 : s.createCMPmap(path, (T)dx, (T)dy, order);
    if (!ok) return 0;
    *ngathers = (long long)s.getNensemb();
    if (number < 0) return 0;
    if (dim == 2) {
        auto g = s.get2DGather((size_t)number);
        const int n = g->getNtrace(), nt = g->getNt();
        if (n > maxtr) return -n;
        Point2D<T> *ps = g->getGeom()->getScoords(), *pg = g->getGeom()->getGcoords();
        for (int i = 0; i < n; i++) {
            sc[2 * i] = ps[i].x; sc[2 * i + 1] = ps[i].y;
            gc[2 * i] = pg[i].x; gc[2 * i + 1] = pg[i].y;
        }
        std::memcpy(data, g->getData(), sizeof(T) * (size_t)n * nt);
        return n;
    }
    auto g = s.get3DGather((size_t)number);
    const int n = g->getNtrace(), nt = g->getNt();
    if (n > maxtr) return -n;
    Point3D<T> *ps = g->getGeom()->getScoords(), *pg = g->getGeom()->getGcoords();
    for (int i = 0; i < n; i++) {
        sc[3 * i] = ps[i].x; sc[3 * i + 1] = ps[i].y; sc[3 * i + 2] = ps[i].z;
        gc[3 * i] = pg[i].x; gc[3 * i + 1] = pg[i].y; gc[3 * i + 2] = pg[i].z;
    }
    std::memcpy(data, g->getData(), sizeof(T) * (size_t)n * nt);
    return n;
}

/* Sort::createEmptydataset(out, n1, d1, o1), then put2DGather of gather `number`
 * with the given samples (the gather's own coordinates from the survey). */
template <typename T>
int sort_put2d(const char *survey, const char *out, int number, int n1, double d1, double o1, const T *data)
{
    Sort<T> s;
    if (!s.createShotmap(survey, 0)) return 0;
    s.createEmptydataset(out, (size_t)n1, (T)d1, (T)o1);
    auto g = s.get2DGather((size_t)number);
    const int n = g->getNtrace();
    auto o = std::make_shared<Data2D<T>>(n, n1, (T)d1, (T)o1);
    Point2D<T> *ps = g->getGeom()->getScoords(), *pg = g->getGeom()->getGcoords();
    Point2D<T> *qs = o->getGeom()->getScoords(), *qg = o->getGeom()->getGcoords();
    for (int i = 0; i < n; i++) { qs[i] = ps[i]; qg[i] = pg[i]; }
    std::memcpy(o->getData(), data, sizeof(T) * (size_t)n * n1);
    o->setFile(out);
    s.put2DGather(o, (size_t)number);
    return n;
}

}  // namespace

extern "C" {
int ref_data_write_f(const char *path, int dim, int nt, double dt, double ot, int ntrace, const float *sc,
                     const float *gc, const float *data)
{ return data_write<float>(path, dim, nt, dt, ot, ntrace, sc, gc, data); }
int ref_data_write_d(const char *path, int dim, int nt, double dt, double ot, int ntrace, const double *sc,
                     const double *gc, const double *data)
{ return data_write<double>(path, dim, nt, dt, ot, ntrace, sc, gc, data); }
int ref_data_read2d_f(const char *path, int nt, int ntrace, float *sc, float *gc, float *data)
{ return data_read2d<float>(path, nt, ntrace, sc, gc, data); }

/* ModelAcoustic2D::writeVp of an nx x nz float model. */
int ref_model_write_f(const char *path, int nx, int nz, double dx, double dz, double ox, double oz, const float *vp)
{
    auto m = std::make_shared<ModelAcoustic2D<float>>(nx, nz, 0, (float)dx, (float)dz, (float)ox, (float)oz, false);
    m->createModel();
    std::memcpy(m->getVp(), vp, sizeof(float) * (size_t)nx * nz);
    m->setVpfile(path);
    m->writeVp();
    return 1;
}

int ref_sort_gather_f(const char *path, int dim, int key, double dx, double dy, int order, int number,
                      int reciprocity, long long *ngathers, float *sc, float *gc, float *data, int maxtr)
{ return sort_gather<float>(path, dim, key, dx, dy, order, number, reciprocity, ngathers, sc, gc, data, maxtr); }
int ref_sort_gather_d(const char *path, int dim, int key, double dx, double dy, int order, int number,
                      int reciprocity, long long *ngathers, double *sc, double *gc, double *data, int maxtr)
{ return sort_gather<double>(path, dim, key, dx, dy, order, number, reciprocity, ngathers, sc, gc, data, maxtr); }
int ref_sort_put2d_f(const char *survey, const char *out, int number, int n1, double d1, double o1,
                     const float *data)
{ return sort_put2d<float>(survey, out, number, n1, d1, o1, data); }
}  // extern "C"
