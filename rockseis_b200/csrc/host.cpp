// Host runtime of librsgpu: the C ABI of include/rsgpu.h.
//
// A plan owns one device arena holding, for every shot of a batch, the pitched
// wavefields, parameters, C-PML memory variables and trace buffers, plus the
// tile table that lets one kernel launch cover all shots.  The time loop is
// replayed from a captured CUDA graph (velocity, stress, inject/record per step).
#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include "rsgpu.h"
#include "rsgpu_host.h"
#include "rsgpu_internal.h"
#include "rsgpu_plan.h"
#include "rsgpu_plan3d.h"

namespace rsgpu {

static thread_local std::string g_err;

void set_error(const char *fmt, ...)
{
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
}

#define CU(call)                                                                          \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess) {                                                          \
            set_error("%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
            return RSGPU_ERR_CUDA;                                                        \
        }                                                                                 \
    } while (0)

static inline size_t rup(size_t a, size_t b) { return (a + b - 1) / b * b; }

// Acoustic batches of at most this many tiles (about one wave of resident CTAs on
// B200: 148 SMs x 6) launch the tile kernels with inlined edge stencils.  Measured:
// one 541x341 shot (187 tiles) 6.2 -> 8.4 Gpts/s; 64 shots of 641x241 (10,752
// tiles) 25.1 -> 23.3 FWI gradients/s, so large batches keep the stencil calls.
static constexpr int INLINE_EDGE_TILES = 888;

// Coefficient rows for each stencil half-length K (lib/der.cpp:3-53).  The values
// are the reference's optimised staggered-grid coefficients; row K holds the K
// pairs used where the reference reduces the order near an array end.  The K=1
// value is a float literal in the reference, hence its float-rounded double.
static const double kCoef[9][8] = {
    {0, 0, 0, 0, 0, 0, 0, 0},
    {(double)1.0029f, 0, 0, 0, 0, 0, 0, 0},
    {1.188401e+0, -7.046382e-2, 0, 0, 0, 0, 0, 0},
    {1.216624e+0, -9.197724e-2, 1.300041e-2, 0, 0, 0, 0, 0},
    {1.230862e+0, -1.034123e-1, 2.011671e-2, -3.245760e-3, 0, 0, 0, 0},
    {1.239407e+0, -1.105315e-1, 2.496329e-2, -5.804879e-3, 9.358680e-4, 0, 0, 0},
    {1.245095e+0, -1.153979e-1, 2.848442e-2, -7.899473e-3, 1.898222e-3, -2.935304e-4, 0, 0},
    {1.249150e+0, -1.189375e-1, 3.116091e-2, -9.623004e-3, 2.812069e-3, -6.655106e-4, 9.728191e-5, 0},
    {1.252186e+0, -1.216289e-1, 3.326513e-2, -1.105777e-2, 3.647865e-3, -1.066144e-3, 2.437491e-4, -3.351959e-5},
};

template <typename T>
static void build_coefs(int prec, double dx, double dz, std::vector<unsigned char> &out)
{
    const int cr = coef_row_stride();
    std::vector<T> c(2 * 9 * cr, T(0));
    for (int K = 0; K <= 8; K++)
        for (int k = 0; k < 8; k++) {
            T v = (T)kCoef[K][k];
            if (prec == PREC_F32_FAST) {
                c[K * cr + k] = (T)((double)v / (double)(T)dx);
                c[9 * cr + K * cr + k] = (T)((double)v / (double)(T)dz);
            } else {
                c[K * cr + k] = v;
                c[9 * cr + K * cr + k] = v;
            }
        }
    out.resize(c.size() * sizeof(T));
    std::memcpy(out.data(), c.data(), out.size());
}

int esize(int prec) { return prec == PREC_F64 ? 8 : 4; }

// cuTensorMapEncodeTiled from the driver, fetched through the runtime so the
// library needs no link-time dependency on libcuda.
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
        else
            cudaGetLastError();
    }
    return fn;
}

// 2D tensor map over a whole pitched field allocation (guard cells included),
// box = tile plus halo.
static bool encode_field_map(CUtensorMap *m, void *base, int prec, int pitch, int rows, int boxw, int boxh)
{
    auto enc = tensor_map_encoder();
    if (!enc) return false;
    const int es = esize(prec);
    cuuint64_t dims[2] = {(cuuint64_t)pitch, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)pitch * es};
    cuuint32_t box[2] = {(cuuint32_t)boxw, (cuuint32_t)boxh};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = enc(m, prec == PREC_F64 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, base,
                     dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

// ---------------------------------------------------------------- device memory pool
static std::mutex g_pool_mu;
static cudaMemPool_t g_pool[64] = {};

static cudaMemPool_t library_pool(cudaError_t *err)
{
    int dev = 0;
    if ((*err = cudaGetDevice(&dev)) != cudaSuccess) return nullptr;
    if (dev < 0 || dev >= 64) { *err = cudaErrorInvalidDevice; return nullptr; }
    std::lock_guard<std::mutex> lk(g_pool_mu);
    if (!g_pool[dev]) {
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t pool = nullptr;
        if ((*err = cudaMemPoolCreate(&pool, &props)) != cudaSuccess) return nullptr;
        cuuint64_t keep = 8ull << 30;
        if ((*err = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep)) != cudaSuccess) {
            cudaMemPoolDestroy(pool);
            return nullptr;
        }
        g_pool[dev] = pool;
    }
    *err = cudaSuccess;
    return g_pool[dev];
}

cudaError_t dev_alloc(void **p, size_t bytes, cudaStream_t st)
{
    cudaError_t e;
    cudaMemPool_t pool = library_pool(&e);
    if (!pool) return e;
    if ((e = cudaMallocFromPoolAsync(p, std::max<size_t>(bytes, 1), pool, st)) != cudaSuccess) {
        *p = nullptr;
        return e;
    }
    return cudaStreamSynchronize(st);
}

void dev_free(void *p, cudaStream_t st)
{
    if (p) cudaFreeAsync(p, st);
}

cudaError_t dev_trim()
{
    cudaError_t e;
    cudaMemPool_t pool = library_pool(&e);
    if (!pool) return e;
    if ((e = cudaDeviceSynchronize()) != cudaSuccess) return e;
    return cudaMemPoolTrimTo(pool, 0);
}

// Shared with other host translation units (no-allocation entry point).
void coef_table_host(int prec, double dx, double dz, std::vector<unsigned char> &out)
{
    if (prec == PREC_F64) build_coefs<double>(prec, dx, dz, out);
    else build_coefs<float>(prec, dx, dz, out);
}
bool encode_field_map_host(void *map, void *base, int prec, int pitch, int rows, int boxw, int boxh)
{
    return encode_field_map(static_cast<CUtensorMap *>(map), base, prec, pitch, rows, boxw, boxh);
}

// ---------------------------------------------------------------- plan
Plan::~Plan()
{
    if (graph_exec) cudaGraphExecDestroy(graph_exec);
    if (zm_graph) cudaGraphExecDestroy(zm_graph);
    dev_free(d_zm, stream);
    dev_free(d_march, stream);
    for (auto &row : tev)
        for (auto &e : row)
            if (e) cudaEventDestroy(e);
    dev_free(arena, stream);
    dev_free(d_meta, stream);
    if (stream && stream != shared_stream) cudaStreamDestroy(stream);
}

rsgpu_status Plan::check_config(const rsgpu_config *c, int ns, const rsgpu_shot *s, bool sets_given)
{
    if (!c || !s || ns < 1) { set_error("null config/shots or nshots < 1"); return RSGPU_ERR_ARG; }
    if (c->physics < 0 || c->physics > 3) { set_error("bad physics %d", c->physics); return RSGPU_ERR_ARG; }
    if (c->physics >= PHYS_A3D) { set_error("3D physics is not built into this plan type"); return RSGPU_ERR_UNSUPPORTED; }
    if (c->precision < 0 || c->precision > 2) { set_error("bad precision %d", c->precision); return RSGPU_ERR_ARG; }
    if (c->lpml < 1 || c->nt < 1 || !(c->dt > 0) || !(c->dx > 0) || !(c->dz > 0)) {
        set_error("lpml, nt, dt, dx, dz must be positive");
        return RSGPU_ERR_ARG;
    }
    const int order = std::min(std::max(c->order, 1), 8);
    for (int i = 0; i < ns; i++) {
        const int nxp = s[i].nx + 2 * c->lpml, nzp = s[i].nz + 2 * c->lpml;
        if (s[i].nx < 1 || s[i].nz < 1) { set_error("shot %d: empty model window", i); return RSGPU_ERR_ARG; }
        // the reference's Der writes out of bounds for an axis of <= order cells
        if (nxp <= order || nzp <= order) { set_error("shot %d: padded grid smaller than stencil", i); return RSGPU_ERR_ARG; }
        for (int k = 0; k < nparams(c->physics); k++)
            if (!s[i].model[k]) { set_error("shot %d: model parameter %d is null", i, k); return RSGPU_ERR_ARG; }
        if (sets_given) continue;   // trace sets are checked by check_sets
        if (s[i].nsrc < 0 || s[i].nrec < 0) { set_error("shot %d: negative trace count", i); return RSGPU_ERR_ARG; }
        if (s[i].nsrc > 0 && (!s[i].smap || !s[i].sshift || !s[i].wavelet)) {
            set_error("shot %d: source arrays missing", i);
            return RSGPU_ERR_ARG;
        }
        if (s[i].nrec > 0 && (!s[i].gmap || !s[i].gshift)) { set_error("shot %d: receiver arrays missing", i); return RSGPU_ERR_ARG; }
        const int sf = s[i].src_field, rf = s[i].rec_field;
        if (sf != RSGPU_PRESSURE && sf != RSGPU_VX && sf != RSGPU_VZ) { set_error("shot %d: bad source field", i); return RSGPU_ERR_ARG; }
        if (s[i].nrec > 0 && rf != RSGPU_PRESSURE && rf != RSGPU_VX && rf != RSGPU_VZ) {
            set_error("shot %d: bad receiver field", i);
            return RSGPU_ERR_ARG;
        }
    }
    return RSGPU_OK;
}

// Build the device arena layout and upload everything.
// Trace sets of one shot as the plan consumes them: the rsgpu_shot's single source
// and receiver set, or the sets an adjoint driver supplies.
static ShotSets sets_of(const rsgpu_shot &s)
{
    ShotSets t;
    t.nsrc = 1;
    t.src[0].n = s.nsrc; t.src[0].map = s.smap; t.src[0].shift = s.sshift; t.src[0].field = s.src_field;
    t.src[0].data = s.wavelet;
    if (s.nrec > 0) {
        t.nrec = 1;
        t.rec[0].n = s.nrec; t.rec[0].map = s.gmap; t.rec[0].shift = s.gshift; t.rec[0].field = s.rec_field;
        t.rec[0].factor = s.rec_factor;
    }
    return t;
}

static rsgpu_status check_sets(int i, const ShotSets &t)
{
    if (t.nsrc < 0 || t.nsrc > MAXSETS || t.nrec < 0 || t.nrec > MAXSETS) { set_error("shot %d: bad trace-set count", i); return RSGPU_ERR_ARG; }
    for (int k = 0; k < t.nsrc; k++) {
        const TraceSet &q = t.src[k];
        if (q.n < 0) { set_error("shot %d: negative trace count", i); return RSGPU_ERR_ARG; }
        if (q.n > 0 && (!q.map || !q.shift || !q.data)) { set_error("shot %d: source arrays missing", i); return RSGPU_ERR_ARG; }
        if (q.field != RSGPU_PRESSURE && q.field != RSGPU_VX && q.field != RSGPU_VZ) { set_error("shot %d: bad source field", i); return RSGPU_ERR_ARG; }
    }
    for (int k = 0; k < t.nrec; k++) {
        const TraceSet &q = t.rec[k];
        if (q.n < 0) { set_error("shot %d: negative trace count", i); return RSGPU_ERR_ARG; }
        if (q.n > 0 && (!q.map || !q.shift)) { set_error("shot %d: receiver arrays missing", i); return RSGPU_ERR_ARG; }
        if (q.field != RSGPU_PRESSURE && q.field != RSGPU_VX && q.field != RSGPU_VZ) { set_error("shot %d: bad receiver field", i); return RSGPU_ERR_ARG; }
    }
    return RSGPU_OK;
}

rsgpu_status Plan::create(const rsgpu_config *c, int ns, const rsgpu_shot *s, const ShotSets *sets_in)
{
    rsgpu_status st = check_config(c, ns, s, sets_in != nullptr);
    if (st != RSGPU_OK) return st;
    std::vector<ShotSets> sets(ns);
    for (int i = 0; i < ns; i++) {
        sets[i] = sets_in ? sets_in[i] : sets_of(s[i]);
        if ((st = check_sets(i, sets[i])) != RSGPU_OK) return st;
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) {
        cudaGetLastError();
        set_error("no CUDA device");
        return RSGPU_ERR_NODEVICE;
    }
    cfg = *c;
    cfg.order = std::min(std::max(c->order, 1), 8);
    prec = c->precision;
    phys = c->physics;
    nshots = ns;
    const int es = esize(prec);
    if (shared_stream) stream = shared_stream;
    else CU(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));

    long tiles32 = 0;   // 32x32 tiles of the batch (the default shape's count)
    for (int i = 0; i < ns; i++)
        tiles32 += (long)((s[i].nx + 2 * c->lpml + 31) / 32) * ((s[i].nz + 2 * c->lpml + 31) / 32);
    tilecfg = (c->tile >= 0 && c->tile < tile_count_2d()) ? c->tile : default_tile(tiles32);
    // the FP64 oracle propagator is built for two tile shapes only
    if (prec == PREC_F64 && tilecfg != TILECFG_64x32 && tilecfg != TILECFG_32x16) tilecfg = TILECFG_64x32;
    const TileShape ts = tile_shape_2d(tilecfg);
    const int lp = cfg.lpml;
    // The fused z-marching step (launch mode 3) serves forward propagation (the
    // forward operator; the acoustic adjoint is the forward operator run in
    // reversed time).  It is bit-identical to the per-tile kernels but measured
    // slower on B200 (it issues as many instructions per point with a third of the
    // resident warps), so the library's choice (mode 0) is the per-tile kernels.
    fused = c->launch_mode == 3 && !adjoint_steps;
    // Launch mode 4: the column-marching half-steps (fd2d_march.cu) for FAST elastic
    // forward propagation; other plans keep the per-tile kernels.
    march = c->launch_mode == 4 && phys == PHYS_E2D && prec == PREC_F32_FAST && !adjoint_steps;
    const int ztx = zm_strip_width();

    // ---- per-shot layout (byte offsets into the arena)
    shots.resize(ns);
    size_t off = 0;
    auto take = [&](size_t bytes) { size_t o = off; off = rup(off + std::max<size_t>(bytes, 1), 256); return o; };
    for (int i = 0; i < ns; i++) {
        ShotLayout &L = shots[i];
        const ShotSets &t = sets[i];
        L.nx = s[i].nx; L.nz = s[i].nz;
        L.nxp = s[i].nx + 2 * lp; L.nzp = s[i].nz + 2 * lp;
        // the fused step reads velocity columns up to 8 past its last strip
        const size_t wide = fused ? std::max(rup(L.nxp, 128), rup(L.nxp, ztx) + 8) : rup(L.nxp, 128);
        L.pitch = (int)rup(GUARD + wide + GUARD, 32);
        L.rows = GUARD + (int)rup(L.nzp, 64) + GUARD;
        const size_t fbytes = (size_t)L.pitch * L.rows * es;
        // state block first (zeroed by reset): wavefields, C-PML memory, traces
        for (int k = 0; k < nfields(phys); k++) L.f[k] = take(fbytes);
        for (int k = 0; k < npsi(phys); k++) L.psix[k] = take((size_t)L.nzp * 2 * lp * es);
        for (int k = 0; k < npsi(phys); k++) L.psiz[k] = take((size_t)2 * lp * L.nxp * es);
        L.psi_end = off;
        L.nrecsets = t.nrec;
        L.nsrcsets = t.nsrc;
        for (int k = 0; k < t.nrec; k++) {
            L.nrecs[k] = t.rec[k].n;
            L.tracesk[k] = take((size_t)t.rec[k].n * cfg.nt * es);
        }
        if (t.nrec == 0) L.tracesk[0] = take(0);
        if (fused) {
            for (int k = 0; k < nfields(phys); k++) L.fb[k] = take(fbytes);
            for (int k = 0; k < (phys == PHYS_E2D ? 2 : 1); k++) {
                L.psixb[k] = take((size_t)L.nzp * 2 * lp * es);
                L.psizb[k] = take((size_t)2 * lp * L.nxp * es);
            }
        }
        L.nrec = t.nrec > 0 ? t.rec[0].n : 0;
        L.traces = L.tracesk[0];
        L.field_begin = L.f[0];
        L.state_end = off;
        // constant inputs
        for (int k = 0; k < nparams(phys); k++) L.m[k] = take(fbytes);
        for (int k = 0; k < t.nsrc; k++) {
            L.nsrcs[k] = t.src[k].n;
            L.wavk[k] = take((size_t)t.src[k].n * cfg.nt * es);
        }
        if (t.nsrc == 0) L.wavk[0] = take(0);
        L.nsrc = t.nsrc > 0 ? t.src[0].n : 0;
        L.wav = L.wavk[0];
    }
    state_end = off;   // everything above is state or data; plan tables follow
    // ---- injection / recording plans, one per trace set
    struct InjPlan { std::vector<int> pt, start, tr; std::vector<double> wx, wz; };
    struct RecPlan { std::vector<int> pt; std::vector<double> w, fac; };
    std::vector<InjPlan> inj((size_t)ns * MAXSETS);
    std::vector<RecPlan> rec((size_t)ns * MAXSETS);
    auto shift_at = [&](const void *p, int k) -> double {
        return prec == PREC_F64 ? ((const double *)p)[k] : (double)((const float *)p)[k];
    };
    auto tri = [&](double sft, double *w) {
        if (prec == PREC_F64) { w[0] = 1 - sft; w[1] = sft; }
        else { w[0] = (float)(1 - (float)sft); w[1] = (float)sft; }
    };
    for (int i = 0; i < ns; i++) {
        const ShotLayout &L = shots[i];
        for (int k = 0; k < sets[i].nsrc; k++) {
            const TraceSet &q = sets[i].src[k];
            InjPlan &P = inj[(size_t)i * MAXSETS + k];
            // contributions in reference loop order: trace, z-corner, x-corner
            std::map<int, std::vector<std::pair<int, std::pair<double, double>>>> per_pt;
            std::vector<int> order_pts;
            for (int t = 0; t < q.n; t++) {
                const int mx = q.map[2 * t], mz = q.map[2 * t + 1];
                if (mx < 0 || mz < 0) continue;
                double xt[2], zt[2];
                tri(shift_at(q.shift, 2 * t), xt);
                tri(shift_at(q.shift, 2 * t + 1), zt);
                for (int i1 = 0; i1 < 2; i1++)
                    for (int i2 = 0; i2 < 2; i2++) {
                        const int ix = lp + mx + i2, iz = lp + mz + i1;
                        if (ix >= L.nxp || iz >= L.nzp) { set_error("shot %d: source %d maps outside the grid", i, t); return RSGPU_ERR_ARG; }
                        const int p = iz * L.pitch + ix;
                        if (!per_pt.count(p)) order_pts.push_back(p);
                        per_pt[p].push_back({t, {xt[i2], zt[i1]}});
                    }
            }
            P.start.push_back(0);
            for (int p : order_pts) {
                P.pt.push_back(p);
                for (auto &cw : per_pt[p]) {
                    P.tr.push_back(cw.first);
                    P.wx.push_back(cw.second.first);
                    P.wz.push_back(cw.second.second);
                }
                P.start.push_back((int)P.tr.size());
            }
        }
        for (int k = 0; k < sets[i].nrec; k++) {
            const TraceSet &q = sets[i].rec[k];
            RecPlan &R = rec[(size_t)i * MAXSETS + k];
            for (int t = 0; t < q.n; t++) {
                const int mx = q.map[2 * t], mz = q.map[2 * t + 1];
                if (mx < 0 || mz < 0) { R.pt.push_back(-1); for (int j = 0; j < 4; j++) R.w.push_back(0); }
                else {
                    if (lp + mx + 1 >= L.nxp || lp + mz + 1 >= L.nzp) { set_error("shot %d: receiver %d maps outside the grid", i, t); return RSGPU_ERR_ARG; }
                    R.pt.push_back((lp + mz) * L.pitch + lp + mx);
                    double w[2];
                    tri(shift_at(q.shift, 2 * t), w);
                    R.w.push_back(w[0]); R.w.push_back(w[1]);
                    tri(shift_at(q.shift, 2 * t + 1), w);
                    R.w.push_back(w[0]); R.w.push_back(w[1]);
                }
                R.fac.push_back(q.factor ? shift_at(q.factor, t) : 1.0);
            }
        }
    }
    // plan tables in the same arena
    struct InjOff { size_t pt, start, tr, wx, wz; };
    struct RecOff { size_t pt, w, fac; };
    std::vector<InjOff> io((size_t)ns * MAXSETS);
    std::vector<RecOff> ro((size_t)ns * MAXSETS);
    for (size_t j = 0; j < io.size(); j++) {
        io[j] = {take(inj[j].pt.size() * 4), take(std::max<size_t>(1, inj[j].start.size()) * 4), take(inj[j].tr.size() * 4),
                 take(inj[j].wx.size() * es), take(inj[j].wz.size() * es)};
        ro[j] = {take(rec[j].pt.size() * 4), take(rec[j].w.size() * es), take(rec[j].fac.size() * es)};
    }
    const size_t o_pml = take((size_t)12 * lp * es);
    rec_pt_offsets.assign((size_t)ns * MAXSETS, 0);
    for (size_t j = 0; j < ro.size(); j++) rec_pt_offsets[j] = ro[j].pt;
    arena_bytes = off;
    if (dev_alloc(&arena, arena_bytes, stream) != cudaSuccess) {
        cudaGetLastError();
        set_error("device allocation of %zu bytes failed", arena_bytes);
        return RSGPU_ERR_NOMEM;
    }
    CU(cudaMemsetAsync(arena, 0, arena_bytes, stream));
    // the plan tables below go up with synchronous copies, which do not wait for the
    // plan's non-blocking stream: let the clearing finish first
    CU(cudaStreamSynchronize(stream));
    char *A = (char *)arena;

    // ---- uploads
    std::vector<unsigned char> hb;
    auto upload_vec_real = [&](size_t o, const std::vector<double> &v) -> rsgpu_status {
        if (v.empty()) return RSGPU_OK;
        hb.resize(v.size() * es);
        for (size_t k = 0; k < v.size(); k++) {
            if (es == 8) ((double *)hb.data())[k] = v[k];
            else ((float *)hb.data())[k] = (float)v[k];
        }
        CU(cudaMemcpy(A + o, hb.data(), hb.size(), cudaMemcpyHostToDevice));
        return RSGPU_OK;
    };
    auto upload_vec_int = [&](size_t o, const std::vector<int> &v) -> rsgpu_status {
        if (v.empty()) return RSGPU_OK;
        CU(cudaMemcpy(A + o, v.data(), v.size() * 4, cudaMemcpyHostToDevice));
        return RSGPU_OK;
    };
    for (int i = 0; i < ns; i++) {
        const ShotLayout &L = shots[i];
        const size_t org = ((size_t)GUARD * L.pitch + GUARD) * es;
        for (int k = 0; k < nparams(phys); k++)
            CU(cudaMemcpy2DAsync(A + L.m[k] + org, (size_t)L.pitch * es, s[i].model[k], (size_t)L.nxp * es,
                                 (size_t)L.nxp * es, L.nzp, cudaMemcpyHostToDevice, stream));
        for (int k = 0; k < sets[i].nsrc; k++)
            if (sets[i].src[k].n > 0)
                CU(cudaMemcpyAsync(A + L.wavk[k], sets[i].src[k].data, (size_t)sets[i].src[k].n * cfg.nt * es,
                                   cudaMemcpyHostToDevice, stream));
        for (int k = 0; k < MAXSETS; k++) {
            const size_t j = (size_t)i * MAXSETS + k;
            if ((st = upload_vec_int(io[j].pt, inj[j].pt)) != RSGPU_OK) return st;
            if ((st = upload_vec_int(io[j].start, inj[j].start)) != RSGPU_OK) return st;
            if ((st = upload_vec_int(io[j].tr, inj[j].tr)) != RSGPU_OK) return st;
            if ((st = upload_vec_real(io[j].wx, inj[j].wx)) != RSGPU_OK) return st;
            if ((st = upload_vec_real(io[j].wz, inj[j].wz)) != RSGPU_OK) return st;
            if ((st = upload_vec_int(ro[j].pt, rec[j].pt)) != RSGPU_OK) return st;
            if ((st = upload_vec_real(ro[j].w, rec[j].w)) != RSGPU_OK) return st;
            if ((st = upload_vec_real(ro[j].fac, rec[j].fac)) != RSGPU_OK) return st;
        }
    }
    {
        std::vector<unsigned char> tab((size_t)12 * lp * es);
        if (c->pml) std::memcpy(tab.data(), c->pml, tab.size());
        else pml_tables_host(lp, cfg.dt, prec, tab.data());
        CU(cudaMemcpy(A + o_pml, tab.data(), tab.size(), cudaMemcpyHostToDevice));
    }
    d_pml = A + o_pml;

    // ---- device metadata: shot descriptors, injection plans, tiles, coefficients, step counter
    const size_t shot_bytes = prec == PREC_F64 ? sizeof(Shot2D<double>) : sizeof(Shot2D<float>);
    const size_t ir_bytes = prec == PREC_F64 ? sizeof(InjRec<double>) : sizeof(InjRec<float>);
    std::vector<Tile2D> tiles;
    for (int i = 0; i < ns; i++) {
        const ShotLayout &L = shots[i];
        for (int z0 = 0; z0 < L.nzp; z0 += ts.tz)
            for (int x0 = 0; x0 < L.nxp; x0 += ts.tx) {
                int fl = 0;
                const int o = cfg.order;
                if (x0 < o || x0 + ts.tx > L.nxp - o - 1) fl |= TILE_XEDGE;
                if (z0 < o || z0 + ts.tz > L.nzp - o - 1) fl |= TILE_ZEDGE;
                if (x0 < lp || x0 + ts.tx > L.nxp - lp) fl |= TILE_XPML;
                if (z0 < lp || z0 + ts.tz > L.nzp - lp) fl |= TILE_ZPML;
                tiles.push_back({i, x0, z0, fl});
            }
    }
    ntiles = (int)tiles.size();
    std::vector<unsigned char> coefs;
    if (prec == PREC_F64) build_coefs<double>(prec, cfg.dx, cfg.dz, coefs);
    else build_coefs<float>(prec, cfg.dx, cfg.dz, coefs);
    const size_t m_shots = 0;
    const size_t m_ir = rup(m_shots + ns * shot_bytes, 256);
    const size_t m_tiles = rup(m_ir + ns * ir_bytes, 256);
    const size_t m_coef = rup(m_tiles + tiles.size() * sizeof(Tile2D), 256);
    const size_t m_maps = rup(m_coef + coefs.size(), 256);
    const size_t m_it = rup(m_maps + (size_t)ns * NMAP2D * sizeof(CUtensorMap), 256);
    const size_t m_end = m_it + 256;
    CU(dev_alloc(&d_meta, m_end, stream));
    d_it = (int *)((char *)d_meta + m_it);
    d_err = d_it + 1;
    d_gate = d_it + 2;
    std::vector<unsigned char> meta(m_end, 0);
    reinterpret_cast<int *>(meta.data() + m_it)[2] = 1;   // recording on
    for (int i = 0; i < ns; i++) {
        const ShotLayout &L = shots[i];
        const size_t org = ((size_t)GUARD * L.pitch + GUARD) * es;
        std::vector<SetOffsets> so(MAXSETS);
        for (int k = 0; k < MAXSETS; k++) {
            const size_t j = (size_t)i * MAXSETS + k;
            so[k] = {io[j].pt, io[j].start, io[j].tr, io[j].wx, io[j].wz, (int)inj[j].pt.size(), ro[j].pt, ro[j].w, ro[j].fac};
        }
        if (prec == PREC_F64) fill_desc<double>(meta.data() + m_shots + i * shot_bytes, meta.data() + m_ir + i * ir_bytes, L, org, so.data(), sets[i]);
        else fill_desc<float>(meta.data() + m_shots + i * shot_bytes, meta.data() + m_ir + i * ir_bytes, L, org, so.data(), sets[i]);
    }
    std::memcpy(meta.data() + m_tiles, tiles.data(), tiles.size() * sizeof(Tile2D));
    std::memcpy(meta.data() + m_coef, coefs.data(), coefs.size());
    for (int i = 0; i < ns; i++) {
        const ShotLayout &L = shots[i];
        for (int k = 0; k < nfields(phys); k++) {
            CUtensorMap *m = reinterpret_cast<CUtensorMap *>(meta.data() + m_maps) + (size_t)i * NMAP2D + k;
            if (!encode_field_map(m, A + L.f[k], prec, L.pitch, L.rows, ts.tx + 2 * GUARD, ts.tz + 2 * GUARD)) {
                set_error("cuTensorMapEncodeTiled failed for shot %d field %d", i, k);
                return RSGPU_ERR_CUDA;
            }
        }
    }
    CU(cudaMemcpy(d_meta, meta.data(), m_end, cudaMemcpyHostToDevice));
    d_shots = (char *)d_meta + m_shots;
    d_injrec = (char *)d_meta + m_ir;
    d_tiles = (char *)d_meta + m_tiles;
    d_coefs = (char *)d_meta + m_coef;
    d_maps = (char *)d_meta + m_maps;
    if (march && (st = setup_march(coefs)) != RSGPU_OK) return st;
    if (fused) {
        std::vector<std::vector<int>> inj_pts(inj.size());
        for (size_t j = 0; j < inj.size(); j++) inj_pts[j] = inj[j].pt;
        if ((st = setup_fused(inj_pts)) != RSGPU_OK) return st;
    }
    CU(cudaStreamSynchronize(stream));
    return RSGPU_OK;
}

static int inj_kind(int phys, int field)
{
    if (phys == PHYS_A2D) return field == RSGPU_PRESSURE ? INJ_A2_P : field == RSGPU_VX ? INJ_A2_VX : INJ_A2_VZ;
    return field == RSGPU_PRESSURE ? INJ_E2_P : field == RSGPU_VX ? INJ_E2_VX : INJ_E2_VZ;
}
static int rec_kind(int phys, int field)
{
    if (phys == PHYS_A2D) return field == RSGPU_PRESSURE ? REC_A2_P : field == RSGPU_VX ? REC_A2_VX : REC_A2_VZ;
    return field == RSGPU_PRESSURE ? REC_E2_P : field == RSGPU_VX ? REC_E2_VX : REC_E2_VZ;
}

template <typename T>
void Plan::fill_desc(unsigned char *sd, unsigned char *irp, const ShotLayout &L, size_t org, const SetOffsets *so,
                     const ShotSets &t)
{
    char *A = (char *)arena;
    Shot2D<T> d{};
    d.nxp = L.nxp; d.nzp = L.nzp; d.pitch = L.pitch; d.lpml = cfg.lpml; d.fs = cfg.fs;
    for (int k = 0; k < nfields(phys); k++) d.f[k] = (T *)(A + L.f[k] + org);
    for (int k = 0; k < nparams(phys); k++) d.m[k] = (const T *)(A + L.m[k] + org);
    for (int k = 0; k < npsi(phys); k++) { d.psix[k] = (T *)(A + L.psix[k]); d.psiz[k] = (T *)(A + L.psiz[k]); }
    if (fused) {
        for (int k = 0; k < nfields(phys); k++) d.fb[k] = (T *)(A + L.fb[k] + org);
        for (int k = 0; k < (phys == PHYS_E2D ? 2 : 1); k++) {
            d.psixb[k] = (T *)(A + L.psixb[k]);
            d.psizb[k] = (T *)(A + L.psizb[k]);
        }
    }
    std::memcpy(sd, &d, sizeof d);
    InjRec<T> r{};
    r.nt = cfg.nt;
    r.rev = reverse_time ? 1 : 0;
    r.rec_gate = gated_recording ? d_gate : nullptr;
    r.ninjsets = t.nsrc;
    for (int k = 0; k < t.nsrc; k++) {
        InjSet<T> &q = r.inj[k];
        q.ninj = so[k].ninj;
        q.kind = q.ninj > 0 ? inj_kind(phys, t.src[k].field) : INJ_NONE;
        q.pt = (const int *)(A + so[k].ipt);
        q.start = (const int *)(A + so[k].istart);
        q.trace = (const int *)(A + so[k].itr);
        q.wx = (const T *)(A + so[k].iwx);
        q.wz = (const T *)(A + so[k].iwz);
        q.wav = (const T *)(A + L.wavk[k]);
    }
    r.nrecsets = t.nrec;
    for (int k = 0; k < t.nrec; k++) {
        RecSet<T> &q = r.rec[k];
        q.nrec = L.nrecs[k];
        q.kind = q.nrec > 0 ? (t.rec[k].psum ? REC_E2_PSUM : rec_kind(phys, t.rec[k].field)) : REC_NONE;
        q.pt = (const int *)(A + so[k].rpt);
        q.w = (const T *)(A + so[k].rw);
        q.factor = (const T *)(A + so[k].rfac);
        q.out = (T *)(A + L.tracesk[k]);
    }
    std::memcpy(irp, &r, sizeof r);
}

int Plan::default_tile(long tiles32) const
{
    // Elastic float plans: 32x16 tiles at eight CTAs per SM, whose 128-register
    // budget holds the inlined reduced-order stencils and the gathered C-PML memory
    // without spills (16-shot 801x401 batch on B200: FAST 34.5 Gpts/s against 27.3
    // for 32x32 tiles at six before the gather, EXACT 16.7 against 15.8).  Acoustic
    // FAST batches of about one wave of tiles (one 541x341 shot): the same shape
    // (9.8 Gpts/s against 8.6); large acoustic batches (the 64-shot FWI: 25.0
    // against 22.5 gradients/s) and all other plans keep 32x32 tiles at six.
    if (phys == PHYS_E2D && prec != PREC_F64) return TILECFG_E2D;
    if (phys == PHYS_A2D && prec == PREC_F32_FAST && tiles32 <= INLINE_EDGE_TILES / 2) return TILECFG_E2D;
    return TILECFG_DEFAULT;
}

rsgpu_status Plan::reset()
{
    for (const auto &L : shots)
        CU(cudaMemsetAsync((char *)arena + L.field_begin, 0, L.state_end - L.field_begin, stream));
    return RSGPU_OK;
}

template <typename T>
static void make_args(void *out, const Plan &p)
{
    Step2DArgs<T> a;
    a.shots = (const Shot2D<T> *)p.d_shots;
    a.tiles = (const Tile2D *)p.d_tiles;
    a.ntiles = p.ntiles;
    a.order = p.cfg.order;
    a.dt = (T)p.cfg.dt; a.dx = (T)p.cfg.dx; a.dz = (T)p.cfg.dz;
    a.rdx = (T)1 / a.dx; a.rdz = (T)1 / a.dz;
    a.pml = (const T *)p.d_pml;
    a.lpml = p.cfg.lpml;
    static_assert(sizeof a <= 128, "argument block");
    std::memcpy(out, &a, sizeof a);
}

rsgpu_status Plan::launch_step(int it_base, const int *it_dev, bool adj, cudaEvent_t *ev)
{
    alignas(16) unsigned char args[128];
    if (prec == PREC_F64) make_args<double>(args, *this);
    else make_args<float>(args, *this);
    const int grid = ntiles;
    // acoustic plans of at most about one wave of tiles: inlined edge stencils (the
    // edge tiles, up to 4.4x slower than interior ones with the stencil calls,
    // otherwise set the time of a launch that has no second wave to hide them)
    const int flags = (adj ? LAUNCH_ADJ : 0) | (phys == PHYS_A2D && ntiles <= INLINE_EDGE_TILES ? LAUNCH_INL : 0);
    const bool mh = march && !adj;
    cudaError_t e;
    // external records so the events become timestamp nodes of a captured graph
    if (ev && (e = cudaEventRecordWithFlags(ev[0], stream, cudaEventRecordExternal)) != cudaSuccess) goto fail;
    if ((e = mh ? launch_march_2d(0, march_args, march_nitems, stream)
                : launch_step_2d(prec, tilecfg, phys, 0, flags, args, d_coefs, d_maps, d_err, grid, stream)) != cudaSuccess)
        goto fail;
    if (ev && (e = cudaEventRecordWithFlags(ev[1], stream, cudaEventRecordExternal)) != cudaSuccess) goto fail;
    if ((e = mh ? launch_march_2d(1, march_args, march_nitems, stream)
                : launch_step_2d(prec, tilecfg, phys, 1, flags, args, d_coefs, d_maps, d_err, grid, stream)) != cudaSuccess)
        goto fail;
    if (ev && (e = cudaEventRecordWithFlags(ev[2], stream, cudaEventRecordExternal)) != cudaSuccess) goto fail;
    if ((e = launch_injrec_2d(prec, d_shots, d_injrec, nshots, cfg.dt, it_base, it_dev, stream)) != cudaSuccess) goto fail;
    launches += 3;
    return RSGPU_OK;
fail:
    set_error("kernel launch failed: %s", cudaGetErrorString(e));
    return RSGPU_ERR_CUDA;
}

rsgpu_status Plan::run(int it0, int nsteps)
{
    if (it0 < 0 || nsteps < 0 || it0 + nsteps > cfg.nt) { set_error("step range [%d,%d) outside [0,%d)", it0, it0 + nsteps, cfg.nt); return RSGPU_ERR_ARG; }
    if (fused && nsteps >= 2) return run_fused(it0, nsteps);
    int done = 0;
    const int G = graph_steps;
    if (use_graph && nsteps >= G) {
        if (!graph_exec) {
            cudaGraph_t g;
            CU(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
            rsgpu_status st = RSGPU_OK;
            for (int s = 0; s < G && st == RSGPU_OK; s++)
                st = launch_step(s, d_it, adjoint_steps, (time_kernels && s < NTIMED) ? tev[s] : nullptr);
            if (st == RSGPU_OK) {
                cudaError_t e = launch_advance(d_it, G, stream);
                if (e != cudaSuccess) { set_error("launch_advance: %s", cudaGetErrorString(e)); st = RSGPU_ERR_CUDA; }
            }
            cudaError_t ce = cudaStreamEndCapture(stream, &g);
            if (st != RSGPU_OK) return st;
            if (ce != cudaSuccess) { set_error("graph capture failed: %s", cudaGetErrorString(ce)); return RSGPU_ERR_CUDA; }
            CU(cudaGraphInstantiate(&graph_exec, g, 0));
            cudaGraphDestroy(g);
            launches -= 3L * G;   // captured launches are counted at replay
        }
        cudaError_t e = launch_set_counter(d_it, it0, stream);
        if (e != cudaSuccess) { set_error("launch_set_counter: %s", cudaGetErrorString(e)); return RSGPU_ERR_CUDA; }
        launches += 1;
        while (nsteps - done >= G) {
            CU(cudaGraphLaunch(graph_exec, stream));
            launches += 3L * G;
            done += G;
        }
    }
    for (; done < nsteps; done++) {
        rsgpu_status st = launch_step(it0 + done, nullptr, adjoint_steps);
        if (st != RSGPU_OK) return st;
    }
    return RSGPU_OK;
}

rsgpu_status Plan::inject_record_only(int it)
{
    if (it < 0 || it >= cfg.nt) { set_error("step %d outside [0,%d)", it, cfg.nt); return RSGPU_ERR_ARG; }
    cudaError_t e = launch_injrec_2d(prec, d_shots, d_injrec, nshots, cfg.dt, it, nullptr, stream);
    if (e != cudaSuccess) { set_error("kernel launch failed: %s", cudaGetErrorString(e)); return RSGPU_ERR_CUDA; }
    launches += 1;
    return RSGPU_OK;
}

rsgpu_status Plan::set_recording(bool on)
{
    if (!gated_recording) { set_error("plan was created without gated recording"); return RSGPU_ERR_STATE; }
    CU(cudaMemsetAsync(d_gate, on ? 1 : 0, sizeof(int), stream));
    return RSGPU_OK;
}

// Device-side error word (bounded waits that gave up); read after a sync.
rsgpu_status Plan::check_device_error()
{
    int e = 0;
    CU(cudaMemcpyAsync(&e, d_err, sizeof(int), cudaMemcpyDeviceToHost, stream));
    CU(cudaStreamSynchronize(stream));
    if (e != 0) {
        set_error("a device-side wait exceeded its time limit (code %d)", e);
        return (rsgpu_status)e;
    }
    return RSGPU_OK;
}

rsgpu_status Plan::enable_timing()
{
    if (time_kernels) return RSGPU_OK;
    for (auto &row : tev)
        for (auto &e : row) CU(cudaEventCreate(&e));
    time_kernels = true;
    if (graph_exec) { cudaGraphExecDestroy(graph_exec); graph_exec = nullptr; }
    if (zm_graph) { cudaGraphExecDestroy(zm_graph); zm_graph = nullptr; }
    return RSGPU_OK;
}

rsgpu_status Plan::kernel_times(float *ms_vel, float *ms_str)
{
    if (fused && zm_graph && time_kernels) {
        // one fused launch per step: its duration, and no separate stress launch
        CU(cudaStreamSynchronize(stream));
        float v = 0;
        for (int s = 0; s < NTIMED; s++) {
            float a;
            CU(cudaEventElapsedTime(&a, tev[s][0], tev[s][1]));
            v += a;
        }
        *ms_vel = v / NTIMED;
        *ms_str = 0;
        return RSGPU_OK;
    }
    if (!time_kernels || !graph_exec) { set_error("kernel timing needs enable_timing() and one graph replay"); return RSGPU_ERR_STATE; }
    CU(cudaStreamSynchronize(stream));
    float v = 0, w = 0;
    for (int s = 0; s < NTIMED; s++) {
        float a, b;
        CU(cudaEventElapsedTime(&a, tev[s][0], tev[s][1]));
        CU(cudaEventElapsedTime(&b, tev[s][1], tev[s][2]));
        v += a; w += b;
    }
    *ms_vel = v / NTIMED;
    *ms_str = w / NTIMED;
    return RSGPU_OK;
}

rsgpu_status Plan::read_traces(int shot, void *host_out, int set)
{
    if (shot < 0 || shot >= nshots) { set_error("bad shot %d", shot); return RSGPU_ERR_ARG; }
    const ShotLayout &L = shots[shot];
    if (set < 0 || set >= std::max(1, L.nrecsets)) { set_error("bad receiver set %d", set); return RSGPU_ERR_ARG; }
    if (L.nrecsets == 0 || L.nrecs[set] == 0) return RSGPU_OK;
    const int es = esize(prec);
    const size_t n = (size_t)L.nrecs[set] * cfg.nt;
    std::vector<unsigned char> tmp(n * es);
    CU(cudaMemcpyAsync(tmp.data(), (char *)arena + L.tracesk[set], n * es, cudaMemcpyDeviceToHost, stream));
    CU(cudaStreamSynchronize(stream));
    if (rsgpu_status st = check_device_error()) return st;
    if (es == 8) { double *o = (double *)host_out; const double *t = (const double *)tmp.data(); for (size_t k = 0; k < n; k++) o[k] += t[k]; }
    else { float *o = (float *)host_out; const float *t = (const float *)tmp.data(); for (size_t k = 0; k < n; k++) o[k] += t[k]; }
    return RSGPU_OK;
}

rsgpu_status Plan::read_field(int shot, int field, void *host_out)
{
    if (shot < 0 || shot >= nshots) { set_error("bad shot %d", shot); return RSGPU_ERR_ARG; }
    int slot = -1;
    if (phys == PHYS_A2D) slot = field == RSGPU_PRESSURE ? A2_P : field == RSGPU_VX ? A2_VX : field == RSGPU_VZ ? A2_VZ : -1;
    else slot = field == RSGPU_VX ? E2_VX : field == RSGPU_VZ ? E2_VZ : field == 4 ? E2_SXX : field == 6 ? E2_SZZ : field == 8 ? E2_SXZ : -1;
    if (slot < 0) { set_error("field %d not held by this physics", field); return RSGPU_ERR_ARG; }
    const ShotLayout &L = shots[shot];
    const int es = esize(prec);
    const size_t org = ((size_t)GUARD * L.pitch + GUARD) * es;
    CU(cudaMemcpy2DAsync(host_out, (size_t)L.nxp * es, (char *)arena + L.f[slot] + org, (size_t)L.pitch * es,
                         (size_t)L.nxp * es, L.nzp, cudaMemcpyDeviceToHost, stream));
    CU(cudaStreamSynchronize(stream));
    return RSGPU_OK;
}

}  // namespace rsgpu

using namespace rsgpu;

struct rsgpu_plan {
    std::unique_ptr<Plan> p;        // 2D physics
    std::unique_ptr<Plan3D> p3;     // 3D physics
};

extern "C" {

int rsgpu_abi_version(void) { return RSGPU_ABI_VERSION; }
const char *rsgpu_last_error(void) { return g_err.c_str(); }
int rsgpu_device_count(void)
{
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) { cudaGetLastError(); return 0; }
    return n;
}

rsgpu_status rsgpu_plan_create(const rsgpu_config *cfg, int nshots, const rsgpu_shot *shots, rsgpu_plan **plan)
{
    if (!plan) { set_error("plan pointer is null"); return RSGPU_ERR_ARG; }
    *plan = nullptr;
    if (!cfg) { set_error("null config"); return RSGPU_ERR_ARG; }
    auto h = std::unique_ptr<rsgpu_plan>(new rsgpu_plan);
    rsgpu_status st;
    if (cfg->physics == RSGPU_ACOUSTIC3D || cfg->physics == RSGPU_ELASTIC3D) {
        h->p3.reset(new Plan3D());
        st = h->p3->create(cfg, nshots, shots);
    } else {
        h->p.reset(new Plan());
        st = h->p->create(cfg, nshots, shots);
    }
    if (st != RSGPU_OK) return st;
    *plan = h.release();
    return RSGPU_OK;
}
rsgpu_status rsgpu_plan_reset(rsgpu_plan *p)
{
    if (!p) { set_error("null plan"); return RSGPU_ERR_ARG; }
    return p->p3 ? p->p3->reset() : p->p->reset();
}
rsgpu_status rsgpu_plan_run(rsgpu_plan *p, int it0, int nsteps)
{
    if (!p) { set_error("null plan"); return RSGPU_ERR_ARG; }
    return p->p3 ? p->p3->run(it0, nsteps) : p->p->run(it0, nsteps);
}
rsgpu_status rsgpu_plan_read_traces(rsgpu_plan *p, int shot, void *out)
{
    if (!p || !out) { set_error("null plan/output"); return RSGPU_ERR_ARG; }
    return p->p3 ? p->p3->read_traces(shot, out) : p->p->read_traces(shot, out);
}
rsgpu_status rsgpu_plan_read_field(rsgpu_plan *p, int shot, int field, void *out)
{
    if (!p || !out) { set_error("null plan/output"); return RSGPU_ERR_ARG; }
    return p->p3 ? p->p3->read_field(shot, field, out) : p->p->read_field(shot, field, out);
}
rsgpu_status rsgpu_plan_sync(rsgpu_plan *p)
{
    if (!p) { set_error("null plan"); return RSGPU_ERR_ARG; }
    cudaError_t e = cudaStreamSynchronize(p->p3 ? p->p3->stream : p->p->stream);
    if (e != cudaSuccess) { set_error("stream sync: %s", cudaGetErrorString(e)); return RSGPU_ERR_CUDA; }
    return p->p3 ? p->p3->check_device_error() : p->p->check_device_error();
}
void *rsgpu_plan_stream(rsgpu_plan *p) { return p ? (void *)(p->p3 ? p->p3->stream : p->p->stream) : nullptr; }
rsgpu_status rsgpu_plan_enable_timing(rsgpu_plan *p)
{
    if (!p) { set_error("null plan"); return RSGPU_ERR_ARG; }
    if (p->p3) { set_error("kernel timing is recorded by 2D plans only"); return RSGPU_ERR_UNSUPPORTED; }
    return p->p->enable_timing();
}
rsgpu_status rsgpu_plan_kernel_times(rsgpu_plan *p, float *ms_velocity, float *ms_stress)
{
    if (!p || !ms_velocity || !ms_stress) { set_error("null argument"); return RSGPU_ERR_ARG; }
    if (p->p3) { set_error("kernel timing is recorded by 2D plans only"); return RSGPU_ERR_UNSUPPORTED; }
    return p->p->kernel_times(ms_velocity, ms_stress);
}
rsgpu_status rsgpu_plan_info(rsgpu_plan *p, int *launch_mode, int *work_items, int *band_rows)
{
    if (!p || !launch_mode || !work_items || !band_rows) { set_error("null argument"); return RSGPU_ERR_ARG; }
    if (p->p3) { set_error("3D plans have no 2D launch mode"); return RSGPU_ERR_UNSUPPORTED; }
    const Plan &q = *p->p;
    *launch_mode = q.fused ? 3 : q.march ? 4 : 2;
    *work_items = q.fused ? q.zm_nitems : q.march ? q.march_nitems : 0;
    *band_rows = q.fused ? q.zm_band : q.march ? q.march_band : 0;
    return RSGPU_OK;
}
long long rsgpu_plan_launch_count(rsgpu_plan *p) { return p ? (p->p3 ? p->p3->launches : p->p->launches) : 0; }
void rsgpu_plan_destroy(rsgpu_plan *p) { delete p; }

rsgpu_status rsgpu_modelling(const rsgpu_config *cfg, int nshots, const rsgpu_shot *shots)
{
    rsgpu_plan *p = nullptr;
    rsgpu_status st = rsgpu_plan_create(cfg, nshots, shots, &p);
    if (st != RSGPU_OK) return st;
    st = rsgpu_plan_run(p, 0, cfg->nt);
    for (int i = 0; st == RSGPU_OK && i < nshots; i++)
        if (shots[i].nrec > 0) {
            if (!shots[i].rec_out) { set_error("shot %d: rec_out is null", i); st = RSGPU_ERR_ARG; break; }
            st = rsgpu_plan_read_traces(p, i, shots[i].rec_out);
        }
    rsgpu_plan_destroy(p);
    return st;
}

rsgpu_status rsgpu_release_cached_memory(void)
{
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) {
        cudaGetLastError();
        set_error("no CUDA device");
        return RSGPU_ERR_NODEVICE;
    }
    cudaError_t e = dev_trim();
    if (e != cudaSuccess) { set_error("releasing the memory pool: %s", cudaGetErrorString(e)); return RSGPU_ERR_CUDA; }
    return RSGPU_OK;
}

rsgpu_status rsgpu_selftest_bounded_wait(void)
{
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) {
        cudaGetLastError();
        set_error("no CUDA device");
        return RSGPU_ERR_NODEVICE;
    }
    int *d_err = nullptr, h_err = 0;
    cudaStream_t st = nullptr;
    CU(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    cudaError_t e = cudaMallocAsync((void **)&d_err, sizeof(int), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_err, 0, sizeof(int), st);
    if (e == cudaSuccess) e = launch_wait_for_nothing(d_err, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h_err, d_err, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (d_err) cudaFreeAsync(d_err, st);
    const cudaError_t es = cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
    if (e == cudaSuccess) e = es;
    if (e != cudaSuccess) { set_error("self test: %s", cudaGetErrorString(e)); return RSGPU_ERR_CUDA; }
    if (h_err == RSGPU_ERR_TIMEOUT) { set_error("a device-side wait exceeded its time limit (self test)"); return RSGPU_ERR_TIMEOUT; }
    set_error("self test: the bounded wait did not report its time-out (code %d)", h_err);
    return RSGPU_ERR_STATE;
}

int rsgpu_tile_count(int precision)
{
    return (precision == PREC_F64) ? TILECFG_32x16 + 1 : tile_count_2d();
}

rsgpu_status rsgpu_tile_shape(int precision, int idx, int *tx, int *tz, int *rows_per_thread, int *ctas_per_sm)
{
    if (!tx || !tz || !rows_per_thread || !ctas_per_sm) { set_error("null argument"); return RSGPU_ERR_ARG; }
    const bool f64 = precision == PREC_F64;
    if (idx < 0 || idx >= tile_count_2d() || (f64 && idx != TILECFG_64x32 && idx != TILECFG_32x16)) {
        set_error("tile shape %d is not built for precision %d", idx, precision);
        return RSGPU_ERR_ARG;
    }
    const TileShape t = tile_shape_2d(idx);
    *tx = t.tx; *tz = t.tz; *rows_per_thread = t.rz; *ctas_per_sm = t.minb;
    return RSGPU_OK;
}

rsgpu_status rsgpu_pml_tables(int lpml, double dt, int precision, void *out12)
{
    if (lpml < 1 || !out12 || precision < 0 || precision > 2) { set_error("bad arguments"); return RSGPU_ERR_ARG; }
    pml_tables_host(lpml, dt, precision, out12);
    return RSGPU_OK;
}

rsgpu_status rsgpu_stagger_model(int physics, int nx, int ny, int nz, int lpml, int fs, int precision,
                                 const void *vp, const void *vs, const void *rho, void *const *out)
{
    if (physics < 0 || physics > 3 || nx < 2 || nz < 2 || lpml < 0 || !vp || !rho || !out) { set_error("bad arguments"); return RSGPU_ERR_ARG; }
    if ((physics == PHYS_E2D || physics == PHYS_E3D) && !vs) { set_error("elastic physics needs vs"); return RSGPU_ERR_ARG; }
    if ((physics == PHYS_A3D || physics == PHYS_E3D) && ny < 2) { set_error("3D physics needs ny >= 2"); return RSGPU_ERR_ARG; }
    int r = stagger_host(physics, nx, ny, nz, lpml, fs, precision, vp, vs, rho, out);
    if (r == -2) { set_error("physics not supported"); return RSGPU_ERR_UNSUPPORTED; }
    if (r != 0) { set_error("staggerModels: Zero density found."); return RSGPU_ERR_ARG; }
    return RSGPU_OK;
}

rsgpu_status rsgpu_make_map(int dim, int precision, int ntr, const double *coords, const int *n, const double *o,
                            const double *d, const double *gshift, int *map, void *shift)
{
    if ((dim != 2 && dim != 3) || ntr < 0 || (ntr > 0 && (!coords || !map || !shift)) || !n || !o || !d) {
        set_error("bad arguments");
        return RSGPU_ERR_ARG;
    }
    make_map_host(dim, precision, ntr, coords, n, o, d, gshift, map, shift);
    return RSGPU_OK;
}

rsgpu_status rsgpu_revolve_trace(int nt, int ncheck, int max, int *actions, int *capos, int *checks, int *n)
{
    if (nt < 1 || !actions || !capos || !checks || !n) { set_error("bad arguments"); return RSGPU_ERR_ARG; }
    RevolveSchedule r(nt, ncheck);
    int k = 0, a;
    do {
        a = r.next();
        if (k >= max) { set_error("action trace longer than %d", max); return RSGPU_ERR_ARG; }
        actions[k] = a; capos[k] = r.capo(); checks[k] = r.check();
        k++;
    } while (a != RSGPU_TERMINATE && a != RSGPU_ERROR);
    *n = k;
    return RSGPU_OK;
}

int rsgpu_revolve_numforw(int nt, int ncheck) { return RevolveSchedule::numforw(nt, ncheck); }

}  // extern "C"
