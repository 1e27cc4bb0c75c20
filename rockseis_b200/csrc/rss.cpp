// Shot-gather files and gather sorting around the propagator: the reference's
// .rss container (File::writeHeader / readHeader, lib/file.cpp:184-250), the
// Data2D/Data3D trace layout (Data2D::write / read, lib/data.cpp:463-635;
// Data3D::write, :1265-1320), model files (ModelAcoustic2D::writeVp,
// lib/model.cpp:1283-1313) and Sort (lib/sort.cpp:132-1055): the ensemble map by
// source, receiver or CMP position, gather reads and writes through it, and the
// gather queue with its NOT_STARTED / RUNNING / FINISHED / FAILED states that the
// MPI drivers hand out (a failed gather goes back to the queue).
//
// File layout (native byte order, as the reference writes it): the 5-byte magic
// "R0CKS"; data_format, header_format, type (int32); Nheader, Ndims (size_t); then
// N[9] (size_t), D[9] (double), O[9] (double); then, per trace, Nheader header
// values of header_format bytes followed by N1 samples of data_format bytes.
// Trace headers are the source and receiver coordinates: (sx, sz, gx, gz) in 2D,
// (sx, sy, sz, gx, gy, gz) in 3D.  Reads and writes go through one contiguous
// buffer per call (a single read or write of the whole trace range).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "rsgpu.h"
#include "rsgpu_host.h"

#define ST(call)                                 \
    do {                                         \
        rsgpu_status st_ = (call);               \
        if (st_ != RSGPU_OK) return st_;         \
    } while (0)

namespace rsgpu {
namespace {

constexpr char RSS_MAGIC[5] = {'R', '0', 'C', 'K', 'S'};
constexpr int RSS_MAXDIMS = 9;
constexpr long RSS_HEADER_BYTES = 5 + 3 * 4 + 2 * 8 + RSS_MAXDIMS * (8 + 8 + 8);

struct FileCloser {
    void operator()(FILE *f) const { if (f) fclose(f); }
};
using FilePtr = std::unique_ptr<FILE, FileCloser>;

rsgpu_status write_header(FILE *f, const rsgpu_rss_header &h)
{
    unsigned long long nh = (unsigned long long)h.nheader, nd = (unsigned long long)h.ndims;
    unsigned long long n[RSS_MAXDIMS];
    for (int i = 0; i < RSS_MAXDIMS; i++) n[i] = (unsigned long long)h.n[i];
    bool ok = fseek(f, 0, SEEK_SET) == 0;
    ok = ok && fwrite(RSS_MAGIC, 1, 5, f) == 5;
    ok = ok && fwrite(&h.data_format, 4, 1, f) == 1 && fwrite(&h.header_format, 4, 1, f) == 1 &&
         fwrite(&h.type, 4, 1, f) == 1;
    ok = ok && fwrite(&nh, 8, 1, f) == 1 && fwrite(&nd, 8, 1, f) == 1;
    ok = ok && fwrite(n, 8, RSS_MAXDIMS, f) == RSS_MAXDIMS && fwrite(h.d, 8, RSS_MAXDIMS, f) == RSS_MAXDIMS &&
         fwrite(h.o, 8, RSS_MAXDIMS, f) == RSS_MAXDIMS;
    if (!ok) { set_error("writing the file header failed"); return RSGPU_ERR_ARG; }
    return RSGPU_OK;
}

rsgpu_status read_header(FILE *f, const char *path, rsgpu_rss_header &h)
{
    char magic[5];
    unsigned long long nh = 0, nd = 0, n[RSS_MAXDIMS];
    bool ok = fseek(f, 0, SEEK_SET) == 0 && fread(magic, 1, 5, f) == 5;
    if (!ok || std::memcmp(magic, RSS_MAGIC, 5) != 0) { set_error("%s is not an rss file", path); return RSGPU_ERR_ARG; }
    ok = fread(&h.data_format, 4, 1, f) == 1 && fread(&h.header_format, 4, 1, f) == 1 && fread(&h.type, 4, 1, f) == 1;
    ok = ok && fread(&nh, 8, 1, f) == 1 && fread(&nd, 8, 1, f) == 1;
    ok = ok && fread(n, 8, RSS_MAXDIMS, f) == RSS_MAXDIMS && fread(h.d, 8, RSS_MAXDIMS, f) == RSS_MAXDIMS &&
         fread(h.o, 8, RSS_MAXDIMS, f) == RSS_MAXDIMS;
    if (!ok) { set_error("%s: truncated header", path); return RSGPU_ERR_ARG; }
    h.nheader = (long long)nh;
    h.ndims = (long long)nd;
    for (int i = 0; i < RSS_MAXDIMS; i++) h.n[i] = (long long)n[i];
    return RSGPU_OK;
}

int esize_of(int precision) { return precision == RSGPU_F64 ? 8 : 4; }

// Header of a Data2D/Data3D trace file as Data2D::write / Data3D::write set it.
rsgpu_rss_header trace_header(int dim, int es, long long nt, double dt, double ot, long long ntrace)
{
    rsgpu_rss_header h{};
    h.data_format = es;
    h.header_format = es;
    h.type = dim == 3 ? RSGPU_RSS_DATA3D : RSGPU_RSS_DATA2D;
    h.nheader = dim == 3 ? 6 : 4;
    h.ndims = 1;                 // the reference's File never raises it from its initial 1
    // the containers hold dt and ot in the sample type
    const double dts = es == 4 ? (double)(float)dt : dt, ots = es == 4 ? (double)(float)ot : ot;
    h.n[0] = nt;
    h.d[0] = dts;
    h.o[0] = dim == 3 ? 0.0 : ots;   // Data3D::write stores a zero time origin
    h.n[1] = ntrace;
    h.d[1] = 1.0;
    h.o[1] = 0.0;
    return h;
}

// CMP bin snapping of Sort::createSort: t = position / d in double, rounded to
// float (the reference stores it in a float, or hands it to rintf), then
// rintf(t) * d with d in the element type.
double snap_bin(double x, double d, int elem_bytes)
{
    if (elem_bytes == 4) {
        const float df = (float)d;
        return (double)(rintf((float)(x / (double)df)) * df);
    }
    return (double)rintf((float)(x / d)) * d;
}

FilePtr open_file(const char *path, const char *mode)
{
    return FilePtr(path ? std::fopen(path, mode) : nullptr);
}

}  // namespace

// ---------------------------------------------------------------- Sort
struct SortPosition {
    double x, offx, y, offy, z, offz, foff;
    size_t ind;
};

}  // namespace rsgpu

using namespace rsgpu;

struct rsgpu_sort {
    std::string file;
    int dim = 2, es = 4, key = RSGPU_SORT_SOURCE;
    long long nt = 0, ntrace = 0;
    double dt = 0, ot = 0;
    std::vector<long long> i0, n;   // per gather: first position in `order`, trace count
    std::vector<int> status;        // RSGPU_GATHER_*
    std::vector<long long> order;   // file trace index of each sorted position
};

extern "C" {

rsgpu_status rsgpu_rss_read_header(const char *path, rsgpu_rss_header *h)
{
    if (!path || !h) { set_error("null path or header"); return RSGPU_ERR_ARG; }
    FilePtr f = open_file(path, "rb");
    if (!f) { set_error("cannot open %s", path); return RSGPU_ERR_ARG; }
    return read_header(f.get(), path, *h);
}

rsgpu_status rsgpu_rss_write_traces(const char *path, int precision, int dim, long long nt, double dt, double ot,
                                    long long ntrace, const void *scoords, const void *gcoords, const void *data)
{
    if (!path || (dim != 2 && dim != 3) || nt < 1 || ntrace < 0 || (ntrace > 0 && (!scoords || !gcoords || !data))) {
        set_error("rss write: bad arguments");
        return RSGPU_ERR_ARG;
    }
    const int es = esize_of(precision), nc = dim;
    FilePtr f = open_file(path, "wb");
    if (!f) { set_error("cannot create %s", path); return RSGPU_ERR_ARG; }
    ST(write_header(f.get(), trace_header(dim, es, nt, dt, ot, ntrace)));
    const size_t rec = (size_t)(2 * nc + nt) * es;
    std::vector<unsigned char> buf(rec * (size_t)ntrace);
    for (long long t = 0; t < ntrace; t++) {
        unsigned char *p = buf.data() + rec * (size_t)t;
        std::memcpy(p, (const unsigned char *)scoords + (size_t)t * nc * es, (size_t)nc * es);
        std::memcpy(p + (size_t)nc * es, (const unsigned char *)gcoords + (size_t)t * nc * es, (size_t)nc * es);
        std::memcpy(p + (size_t)2 * nc * es, (const unsigned char *)data + (size_t)t * nt * es, (size_t)nt * es);
    }
    if (!buf.empty() && fwrite(buf.data(), 1, buf.size(), f.get()) != buf.size()) {
        set_error("writing %s failed", path);
        return RSGPU_ERR_ARG;
    }
    return RSGPU_OK;
}

rsgpu_status rsgpu_rss_read_traces(const char *path, int precision, long long first, long long count, void *scoords,
                                   void *gcoords, void *data)
{
    if (!path || first < 0 || count < 0) { set_error("rss read: bad arguments"); return RSGPU_ERR_ARG; }
    FilePtr f = open_file(path, "rb");
    if (!f) { set_error("cannot open %s", path); return RSGPU_ERR_ARG; }
    rsgpu_rss_header h{};
    ST(read_header(f.get(), path, h));
    const int es = esize_of(precision);
    if ((h.type != RSGPU_RSS_DATA2D && h.type != RSGPU_RSS_DATA3D) || h.data_format != es || h.header_format != es) {
        set_error("%s: not a Data2D/Data3D file of %d-byte samples", path, es);
        return RSGPU_ERR_ARG;
    }
    const int nc = h.type == RSGPU_RSS_DATA3D ? 3 : 2;
    if (h.nheader != 2 * nc || first + count > h.n[1]) {
        set_error("%s: traces [%lld, %lld) outside the %lld in the file", path, first, first + count, h.n[1]);
        return RSGPU_ERR_ARG;
    }
    const long long nt = h.n[0];
    const size_t rec = (size_t)(2 * nc + nt) * es;
    std::vector<unsigned char> buf(rec * (size_t)count);
    if (fseek(f.get(), RSS_HEADER_BYTES + (long)(rec * (size_t)first), SEEK_SET) != 0 ||
        (!buf.empty() && fread(buf.data(), 1, buf.size(), f.get()) != buf.size())) {
        set_error("%s: short read", path);
        return RSGPU_ERR_ARG;
    }
    for (long long t = 0; t < count; t++) {
        const unsigned char *p = buf.data() + rec * (size_t)t;
        if (scoords) std::memcpy((unsigned char *)scoords + (size_t)t * nc * es, p, (size_t)nc * es);
        if (gcoords) std::memcpy((unsigned char *)gcoords + (size_t)t * nc * es, p + (size_t)nc * es, (size_t)nc * es);
        if (data) std::memcpy((unsigned char *)data + (size_t)t * nt * es, p + (size_t)2 * nc * es, (size_t)nt * es);
    }
    return RSGPU_OK;
}

rsgpu_status rsgpu_rss_write_model(const char *path, int precision, int nx, int ny, int nz, double dx, double dy,
                                   double dz, double ox, double oy, double oz, const void *values)
{
    if (!path || nx < 1 || nz < 1 || ny < 0 || !values) { set_error("rss model write: bad arguments"); return RSGPU_ERR_ARG; }
    rsgpu_rss_header h{};
    h.data_format = esize_of(precision);
    h.header_format = -1;           // never set for model files
    h.type = RSGPU_RSS_REGULAR;
    h.ndims = 1;
    h.n[0] = nx; h.d[0] = dx; h.o[0] = ox;
    if (ny > 0) { h.n[1] = ny; h.d[1] = dy; h.o[1] = oy; }
    else h.n[1] = 1;             // a 2D model file records one y sample (d = o = 0)
    h.n[2] = nz; h.d[2] = dz; h.o[2] = oz;
    FilePtr f = open_file(path, "wb");
    if (!f) { set_error("cannot create %s", path); return RSGPU_ERR_ARG; }
    ST(write_header(f.get(), h));
    const size_t n = (size_t)nx * (ny > 0 ? ny : 1) * nz * h.data_format;
    if (fwrite(values, 1, n, f.get()) != n) { set_error("writing %s failed", path); return RSGPU_ERR_ARG; }
    return RSGPU_OK;
}

rsgpu_status rsgpu_rss_read_model(const char *path, int precision, long long count, void *values)
{
    if (!path || count < 0 || !values) { set_error("rss model read: bad arguments"); return RSGPU_ERR_ARG; }
    FilePtr f = open_file(path, "rb");
    if (!f) { set_error("cannot open %s", path); return RSGPU_ERR_ARG; }
    rsgpu_rss_header h{};
    ST(read_header(f.get(), path, h));
    const int es = esize_of(precision);
    if (h.data_format != es) { set_error("%s holds %d-byte values, not %d", path, h.data_format, es); return RSGPU_ERR_ARG; }
    long long total = 1;
    for (int i = 0; i < RSS_MAXDIMS; i++) total *= h.n[i] > 0 ? h.n[i] : 1;
    if (count > total) { set_error("%s holds %lld values, %lld asked for", path, total, count); return RSGPU_ERR_ARG; }
    if (fseek(f.get(), RSS_HEADER_BYTES, SEEK_SET) != 0 || fread(values, es, (size_t)count, f.get()) != (size_t)count) {
        set_error("%s: short read", path);
        return RSGPU_ERR_ARG;
    }
    return RSGPU_OK;
}

// Sort::createSort (lib/sort.cpp:132-399): trace positions by key, ordered by
// (x, y, z, trace) for order 0, (y, x, z, trace) for 1 and (z, x, y, trace) for 2
// -- the trace index makes the order total, so the offsets the reference compares
// after it never decide --, then runs of equal (x, y, z) become gathers.  CMP
// positions are the source-receiver midpoints snapped to dx (and dy) with rintf.
rsgpu_status rsgpu_sort_create(const char *path, int key, double dx, double dy, int order, rsgpu_sort **out)
{
    if (!path || !out || key < RSGPU_SORT_SOURCE || key > RSGPU_SORT_CMP) { set_error("sort: bad arguments"); return RSGPU_ERR_ARG; }
    *out = nullptr;
    FilePtr f = open_file(path, "rb");
    if (!f) { set_error("cannot open %s", path); return RSGPU_ERR_ARG; }
    rsgpu_rss_header h{};
    ST(read_header(f.get(), path, h));
    if (h.type != RSGPU_RSS_DATA2D && h.type != RSGPU_RSS_DATA3D) {
        set_error("sort: %s is neither a Data2D nor a Data3D file", path);
        return RSGPU_ERR_ARG;
    }
    if (h.header_format != 4 && h.header_format != 8) { set_error("sort: header format %d not supported", h.header_format); return RSGPU_ERR_ARG; }
    const bool d3 = h.type == RSGPU_RSS_DATA3D;
    const long long n1 = h.n[0], n2 = h.n[1];
    const int nh = (int)h.nheader, hp = h.header_format, dp = h.data_format;
    if (n2 < 1 || nh < (d3 ? 6 : 4)) { set_error("sort: %s holds no traces", path); return RSGPU_ERR_ARG; }
    std::vector<SortPosition> pos((size_t)n2);
    std::vector<unsigned char> hb((size_t)nh * hp);
    for (long long i2 = 0; i2 < n2; i2++) {
        if (fseek(f.get(), RSS_HEADER_BYTES + (long)(i2 * (n1 * dp + (long long)nh * hp)), SEEK_SET) != 0 ||
            fread(hb.data(), 1, hb.size(), f.get()) != hb.size()) {
            set_error("sort: %s: short read", path);
            return RSGPU_ERR_ARG;
        }
        // header values as the reference holds them: float or double
        double b[6];
        for (int k = 0; k < 6 && k < nh; k++) {
            if (hp == 4) { float v; std::memcpy(&v, hb.data() + 4 * k, 4); b[k] = v; }
            else std::memcpy(&b[k], hb.data() + 8 * k, 8);
        }
        SortPosition &p = pos[(size_t)i2];
        // coordinates: 2D (sx, sz, gx, gz) -> x, z; 3D (sx, sy, sz, gx, gy, gz)
        const double sx = b[0], sy = d3 ? b[1] : 0.0, sz = d3 ? b[2] : b[1];
        const double gx = d3 ? b[3] : b[2], gy = d3 ? b[4] : 0.0, gz = d3 ? b[5] : b[3];
        if (key == RSGPU_SORT_SOURCE) {
            p.x = sx; p.y = sy; p.z = sz;
            p.offx = gx - sx; p.offy = gy - sy; p.offz = gz - sz;
        } else if (key == RSGPU_SORT_RECEIVER) {
            p.x = gx; p.y = gy; p.z = gz;
            p.offx = sx - gx; p.offy = sy - gy; p.offz = sz - gz;
        } else {
            // the midpoint in the header's type, snapped to the bins with the bin sizes
            // in the element type
            if (hp == 4) {
                p.x = 0.5 * (double)((float)b[0] + (float)(d3 ? b[3] : b[2]));
                p.y = d3 ? 0.5 * (double)((float)b[1] + (float)b[4]) : 0.0;
            } else {
                p.x = 0.5 * (b[0] + (d3 ? b[3] : b[2]));
                p.y = d3 ? 0.5 * (b[1] + b[4]) : 0.0;
            }
            p.x = snap_bin(p.x, dx, dp);
            p.y = snap_bin(p.y, dy, dp);
            p.z = 0.0;
        }
        p.ind = (size_t)i2;
    }
    // comparisons as the reference's sort_sr_* make them (an unordered pair of keys
    // counts as equal); a stable sort stays within bounds whatever the keys hold
    auto first = [order](const SortPosition &p, int k) {
        const double v[3][3] = {{p.x, p.y, p.z}, {p.y, p.x, p.z}, {p.z, p.x, p.y}};
        return v[order == 1 ? 1 : order == 2 ? 2 : 0][k];
    };
    std::stable_sort(pos.begin(), pos.end(), [&](const SortPosition &a, const SortPosition &b) {
        for (int k = 0; k < 3; k++) {
            const double u = first(a, k), w = first(b, k);
            if (u < w) return true;
            if (u > w) return false;
        }
        return a.ind < b.ind;
    });
    std::unique_ptr<rsgpu_sort> s(new rsgpu_sort());
    s->file = path;
    s->dim = d3 ? 3 : 2;
    s->es = dp;
    s->key = key;
    s->nt = n1;
    s->ntrace = n2;
    s->dt = h.d[0];
    s->ot = h.o[0];
    s->order.resize((size_t)n2);
    for (long long i = 0; i < n2; i++) s->order[(size_t)i] = (long long)pos[(size_t)i].ind;
    long long start = 0;
    for (long long i = 1; i <= n2; i++) {
        if (i == n2 || pos[(size_t)i].x != pos[(size_t)start].x || pos[(size_t)i].y != pos[(size_t)start].y ||
            pos[(size_t)i].z != pos[(size_t)start].z) {
            s->i0.push_back(start);
            s->n.push_back(i - start);
            s->status.push_back(RSGPU_GATHER_NOT_STARTED);
            start = i;
        }
    }
    *out = s.release();
    return RSGPU_OK;
}

void rsgpu_sort_destroy(rsgpu_sort *s) { delete s; }

rsgpu_status rsgpu_sort_info(const rsgpu_sort *s, long long *ngathers, long long *ntraces, long long *nt)
{
    if (!s) { set_error("null sort"); return RSGPU_ERR_ARG; }
    if (ngathers) *ngathers = (long long)s->n.size();
    if (ntraces) *ntraces = s->ntrace;
    if (nt) *nt = s->nt;
    return RSGPU_OK;
}

long long rsgpu_sort_gather_size(const rsgpu_sort *s, long long number)
{
    if (!s || number < 0 || number >= (long long)s->n.size()) return -1;
    return s->n[(size_t)number];
}

// Sort::get2DGather() (lib/sort.cpp:402-472): the first gather not started or failed.
long long rsgpu_sort_next(const rsgpu_sort *s)
{
    if (!s) return -1;
    for (size_t i = 0; i < s->status.size(); i++)
        if (s->status[i] == RSGPU_GATHER_NOT_STARTED || s->status[i] == RSGPU_GATHER_FAILED) return (long long)i;
    return -1;
}

rsgpu_status rsgpu_sort_set_status(rsgpu_sort *s, long long number, int status)
{
    if (!s || number < 0 || number >= (long long)s->status.size() || status < RSGPU_GATHER_FINISHED ||
        status > RSGPU_GATHER_FAILED) {
        set_error("sort: bad gather number or status");
        return RSGPU_ERR_ARG;
    }
    s->status[(size_t)number] = status;
    return RSGPU_OK;
}

int rsgpu_sort_status(const rsgpu_sort *s, long long number)
{
    if (!s || number < 0 || number >= (long long)s->status.size()) return -1;
    return s->status[(size_t)number];
}

// Sort::get2DGather(number) / get3DGather(number) (lib/sort.cpp:474-533, 805-867):
// the gather's traces in sorted order; with reciprocity the source and receiver
// coordinates trade places.  The gather is marked RUNNING.
rsgpu_status rsgpu_sort_read_gather(rsgpu_sort *s, long long number, int reciprocity, void *scoords, void *gcoords,
                                    void *data)
{
    if (!s || number < 0 || number >= (long long)s->n.size()) { set_error("sort: bad gather number"); return RSGPU_ERR_ARG; }
    FilePtr f = open_file(s->file.c_str(), "rb");
    if (!f) { set_error("cannot open %s", s->file.c_str()); return RSGPU_ERR_ARG; }
    const int es = s->es, nc = s->dim;
    const size_t rec = (size_t)(2 * nc + s->nt) * es;
    std::vector<unsigned char> buf(rec);
    for (long long j = 0; j < s->n[(size_t)number]; j++) {
        const long long tr = s->order[(size_t)(s->i0[(size_t)number] + j)];
        if (fseek(f.get(), RSS_HEADER_BYTES + (long)(rec * (size_t)tr), SEEK_SET) != 0 ||
            fread(buf.data(), 1, rec, f.get()) != rec) {
            set_error("sort: %s: short read", s->file.c_str());
            return RSGPU_ERR_ARG;
        }
        unsigned char *sc = (unsigned char *)scoords + (size_t)j * nc * es, *gc = (unsigned char *)gcoords + (size_t)j * nc * es;
        std::memcpy(reciprocity ? gc : sc, buf.data(), (size_t)nc * es);
        std::memcpy(reciprocity ? sc : gc, buf.data() + (size_t)nc * es, (size_t)nc * es);
        std::memcpy((unsigned char *)data + (size_t)j * s->nt * es, buf.data() + (size_t)2 * nc * es,
                    (size_t)s->nt * es);
    }
    s->status[(size_t)number] = RSGPU_GATHER_RUNNING;
    return RSGPU_OK;
}

// Sort::createEmptydataset (lib/sort.cpp:999-1055): an output file with the survey's
// trace headers and n1 zero samples per trace.
rsgpu_status rsgpu_sort_create_output(const rsgpu_sort *s, const char *path, long long n1, double d1, double o1)
{
    if (!s || !path || n1 < 1) { set_error("sort: bad arguments"); return RSGPU_ERR_ARG; }
    FilePtr in = open_file(s->file.c_str(), "rb");
    FilePtr f = open_file(path, "wb");
    if (!in || !f) { set_error("sort: cannot open %s or %s", s->file.c_str(), path); return RSGPU_ERR_ARG; }
    const int es = s->es, nc = s->dim;
    rsgpu_rss_header h = trace_header(s->dim, es, n1, d1, o1, s->ntrace);
    h.o[0] = es == 4 ? (double)(float)o1 : o1;   // the streaming writer keeps the origin it was given
    ST(write_header(f.get(), h));
    const size_t rin = (size_t)(2 * nc + s->nt) * es, rout = (size_t)(2 * nc + n1) * es;
    std::vector<unsigned char> hb((size_t)2 * nc * es), out(rout, 0);
    for (long long t = 0; t < s->ntrace; t++) {
        if (fseek(in.get(), RSS_HEADER_BYTES + (long)(rin * (size_t)t), SEEK_SET) != 0 ||
            fread(hb.data(), 1, hb.size(), in.get()) != hb.size()) {
            set_error("sort: %s: short read", s->file.c_str());
            return RSGPU_ERR_ARG;
        }
        std::memcpy(out.data(), hb.data(), hb.size());
        if (fwrite(out.data(), 1, rout, f.get()) != rout) { set_error("writing %s failed", path); return RSGPU_ERR_ARG; }
    }
    return RSGPU_OK;
}

// Sort::put2DGather(number) / put3DGather (lib/sort.cpp:535-579, 629-677): the
// gather's traces written back to their places in an output file made by
// rsgpu_sort_create_output (n1 samples per trace).
rsgpu_status rsgpu_sort_write_gather(const rsgpu_sort *s, const char *path, long long number, int reciprocity,
                                     long long n1, const void *scoords, const void *gcoords, const void *data)
{
    if (!s || !path || number < 0 || number >= (long long)s->n.size()) { set_error("sort: bad gather number"); return RSGPU_ERR_ARG; }
    FilePtr f = open_file(path, "r+b");
    if (!f) { set_error("cannot open %s", path); return RSGPU_ERR_ARG; }
    rsgpu_rss_header h{};
    ST(read_header(f.get(), path, h));
    if (h.n[0] != n1 || h.data_format != s->es) { set_error("sort: %s does not hold %lld-sample traces", path, n1); return RSGPU_ERR_ARG; }
    const int es = s->es, nc = s->dim;
    const size_t rec = (size_t)(2 * nc + n1) * es;
    std::vector<unsigned char> buf(rec);
    for (long long j = 0; j < s->n[(size_t)number]; j++) {
        const long long tr = s->order[(size_t)(s->i0[(size_t)number] + j)];
        const unsigned char *sc = (const unsigned char *)scoords + (size_t)j * nc * es;
        const unsigned char *gc = (const unsigned char *)gcoords + (size_t)j * nc * es;
        std::memcpy(buf.data(), reciprocity ? gc : sc, (size_t)nc * es);
        std::memcpy(buf.data() + (size_t)nc * es, reciprocity ? sc : gc, (size_t)nc * es);
        std::memcpy(buf.data() + (size_t)2 * nc * es, (const unsigned char *)data + (size_t)j * n1 * es, (size_t)n1 * es);
        if (fseek(f.get(), RSS_HEADER_BYTES + (long)(rec * (size_t)tr), SEEK_SET) != 0 ||
            fwrite(buf.data(), 1, rec, f.get()) != rec) {
            set_error("writing %s failed", path);
            return RSGPU_ERR_ARG;
        }
    }
    return RSGPU_OK;
}

}  // extern "C"
