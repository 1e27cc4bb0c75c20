// FWI gradient and RTM image drivers (host runtime behind rsgpu_fwi_gradient,
// rsgpu_rtm_image and rsgpu_adjoint_*).
//
// The reference's FwiAcoustic2D::run_optimal (lib/fwi.cpp:1159-1332) and
// RtmAcoustic2D::run_optimal (lib/rtm.cpp:423-545) drive a forward and an
// adjoint propagator with a Revolve checkpoint schedule.  Here the same schedule
// (RevolveSchedule, csrc/revolve.cpp) drives two batched plans that share one
// stream:
//   fw : the shots as given; records the modelled data during the first sweep
//   bw : the adjoint wavefield, run forward in reversed time (it' = nt-1-it):
//        its sources are the receivers (residuals or data injected as pressure
//        at GMAP), its receivers the sources (wavelet gradient at SMAP).
// Actions:
//   ADVANCE   fw steps oldcapo..capo-1 (inject, and record until FIRSTURN)
//   TAKESHOT  all shots' wavefields + C-PML memory -> checkpoint slot `check`
//   RESTORE   slot `check` -> fw state
//   FIRSTURN  fw step nt-1 (inject, record); residuals + misfit; bw injection at
//             nt-1 without propagation; correlation at nt-1
//   YOUTURN   bw step at it = capo (propagate, inject, record); correlation of
//             the bw state with the fw state at capo, i.e. the forward state
//             after step capo-1 (the reference's pairing)
// Every correlation launch covers all shots.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <vector>

#include <cuda_runtime.h>

#include "rsgpu.h"
#include "rsgpu_adjoint.h"
#include "rsgpu_adjoint3d.h"
#include "rsgpu_host.h"
#include "rsgpu_internal.h"
#include "rsgpu_plan.h"

namespace rsgpu {

#define CU(call)                                                                          \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess) {                                                          \
            set_error("%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
            return RSGPU_ERR_CUDA;                                                        \
        }                                                                                 \
    } while (0)
#define ST(call)                                 \
    do {                                         \
        rsgpu_status s_ = (call);                \
        if (s_ != RSGPU_OK) return s_;           \
    } while (0)

static inline size_t rup(size_t a, size_t b) { return (a + b - 1) / b * b; }

class Adjoint {
public:
    ~Adjoint();
    rsgpu_status create(const rsgpu_config *c, const rsgpu_adjoint_opts *o, int kind, int ns,
                        const rsgpu_adjoint_shot *s);
    rsgpu_status run();
    rsgpu_status read(int ns, const rsgpu_adjoint_shot *s);
    rsgpu_status stack(int nxg, int nzg, const int *x0, const int *z0, void *const *out);

    int kind = RSGPU_KIND_FWI, phys = PHYS_A2D, nshots = 0, prec = 0, es = 4, acc = ACC_REF, ck = CK_NATIVE;
    int nhx = 1, nhz = 1;
    int ncheck = 0, nslots = 0, nxmax = 0, nzmax = 0;
    // FULL snapshots (FwiAcoustic2D::run, RtmAcoustic2D::run): the forward P interior
    // every snapinc steps, snapnt of them, correlated at adjoint times t with
    // (t - enddiff) % snapinc == 0
    int snapmethod = RSGPU_SNAP_OPTIMAL, snapinc = 1, snapnt = 0, enddiff = 0;
    bool noreverse = false;
    int misfit_type = RSGPU_MISFIT_DIFFERENCE, nrec_max = 0;
    rsgpu_config cfg{};
    std::unique_ptr<Plan> fw, bw;
    cudaStream_t stream = nullptr;
    void *dbuf = nullptr, *ckpt = nullptr;
    size_t slot_elems = 0, ck_es = 4;
    int seg_rows = 1;                       // rows of the tallest checkpoint block
    std::vector<CkptSeg> segs;
    std::vector<size_t> o_vp, o_vs, o_rho, o_obs, o_obsx, o_obsz, o_g0, o_g1, o_g2;
    std::vector<size_t> o_ilum;      // acoustic FWI source illumination (0 = not asked for)
    size_t o_misfit = 0, o_corr = 0, o_res = 0, o_segs = 0, o_scales = 0, o_maxbits = 0;
    size_t o_rpart = 0;                     // residual pass: per-CTA partial misfits
    std::vector<size_t> o_work, o_tnorm;   // ADAPTIVE misfits: per-trace scratch and filter norms
    std::vector<size_t> o_work2, o_tnorm2; // elastic ADAPTIVE_GAUSS / _LINEAR: the Uz filters
    size_t o_comp = 0;                      // elastic ADAPTIVE_GAUSS / _LINEAR: Ux and Uz views per shot
    std::vector<unsigned char> comp;        // host copy of those views until the upload completes
    std::vector<size_t> o_wav0;             // EDGES: the forward plan's source traces, kept aside
    size_t o_atab = 0;                      // ADAPTIVE misfits: weights and summation-order tables
    std::vector<int> nx, nz, nrec, nsrc;
    long long fw_steps = 0, bw_steps = 0, ckpt_bytes = 0, launches = 0;
    bool ran = false;

private:
    rsgpu_status run_full();
    rsgpu_status reset_outputs();
    rsgpu_status residuals();
    rsgpu_status correlate();
    rsgpu_status save(int slot);
    rsgpu_status load(int slot);
    template <typename T>
    void build_desc(std::vector<unsigned char> &corr, std::vector<unsigned char> &res);
    template <typename T>
    void build_desc_e2d(std::vector<unsigned char> &corr, std::vector<unsigned char> &res);
    bool elastic() const { return phys == PHYS_E2D; }
    char *D(size_t o) const { return (char *)dbuf + o; }
};

Adjoint::~Adjoint()
{
    fw.reset();
    bw.reset();
    dev_free(dbuf, stream);
    dev_free(ckpt, stream);
    if (stream) cudaStreamDestroy(stream);
}

static rsgpu_status check_adjoint(const rsgpu_config *c, const rsgpu_adjoint_opts *o, int kind, int ns,
                                  const rsgpu_adjoint_shot *s)
{
    if (!c || !o || !s || ns < 1) { set_error("null config/options/shots or nshots < 1"); return RSGPU_ERR_ARG; }
    if (kind != RSGPU_KIND_FWI && kind != RSGPU_KIND_RTM) { set_error("bad driver kind %d", kind); return RSGPU_ERR_ARG; }
    if (c->physics != RSGPU_ACOUSTIC2D && !(c->physics == RSGPU_ELASTIC2D && kind == RSGPU_KIND_FWI)) {
        set_error("the gradient/image drivers are built for acoustic 2D (FWI, RTM) and elastic 2D (FWI)");
        return RSGPU_ERR_UNSUPPORTED;
    }
    const bool el = c->physics == RSGPU_ELASTIC2D;
    if (o->misfit < RSGPU_MISFIT_DIFFERENCE || o->misfit > RSGPU_MISFIT_ADAPTIVE_SINGLE) {
        set_error("misfit %d: DIFFERENCE, CORRELATION, ADAPTIVE_GAUSS, ADAPTIVE_LINEAR and ADAPTIVE_SINGLE are built",
                  o->misfit);
        return RSGPU_ERR_UNSUPPORTED;
    }
    if (o->misfit == RSGPU_MISFIT_CORRELATION && kind == RSGPU_KIND_FWI) {
        const int lim = 49152 / ((el ? 3 : 1) * (c->precision == RSGPU_F64 ? 8 : 4));
        for (int i = 0; i < ns; i++)
            if (s[i].shot.nrec > lim) {
                set_error("shot %d: the CORRELATION misfit takes at most %d receivers per shot", i, lim);
                return RSGPU_ERR_UNSUPPORTED;
            }
    }
    if (o->ckpt_precision < RSGPU_CKPT_NATIVE || o->ckpt_precision > RSGPU_CKPT_BF16) {
        set_error("bad checkpoint precision %d", o->ckpt_precision);
        return RSGPU_ERR_ARG;
    }
    if (o->accum != RSGPU_ACCUM_REFERENCE && o->accum != RSGPU_ACCUM_F64) { set_error("bad accumulation %d", o->accum); return RSGPU_ERR_ARG; }
    if (o->snapmethod != RSGPU_SNAP_OPTIMAL && o->snapmethod != RSGPU_SNAP_FULL && o->snapmethod != RSGPU_SNAP_EDGES) {
        set_error("bad snapmethod %d", o->snapmethod);
        return RSGPU_ERR_ARG;
    }
    if (o->snapmethod == RSGPU_SNAP_EDGES && kind != RSGPU_KIND_RTM) {
        set_error("EDGES snapshots belong to the acoustic 2D RTM image (RtmAcoustic2D::run_edge)");
        return RSGPU_ERR_UNSUPPORTED;
    }
    if (o->snapmethod != RSGPU_SNAP_OPTIMAL && el) {
        set_error("FULL snapshots are built for the acoustic 2D gradient and image (FwiAcoustic2D::run, RtmAcoustic2D::run)");
        return RSGPU_ERR_UNSUPPORTED;
    }
    if (kind == RSGPU_KIND_RTM && (o->nhx < 1 || o->nhz < 1 || o->nhx % 2 == 0 || o->nhz % 2 == 0)) {
        set_error("nhx and nhz must be odd and positive");
        return RSGPU_ERR_ARG;
    }
    for (int i = 0; i < ns; i++) {
        const rsgpu_shot &sh = s[i].shot;
        if ((!el && sh.src_field != RSGPU_PRESSURE) || (sh.nrec > 0 && sh.rec_field != RSGPU_PRESSURE)) {
            set_error("shot %d: the gradient/image drivers take pressure %s and a pressure receiver set", i,
                      el ? "data" : "sources");
            return RSGPU_ERR_UNSUPPORTED;
        }
        if (el && (!s[i].gmap_vx || !s[i].gmap_vz || !s[i].gshift_vx || !s[i].gshift_vz || !s[i].data_vx ||
                   !s[i].data_vz || !s[i].vs)) {
            set_error("shot %d: elastic FWI needs the Ux and Uz data sets (maps, shifts, data) and vs", i);
            return RSGPU_ERR_ARG;
        }
        if (sh.nsrc < 1 || sh.nrec < 1) { set_error("shot %d: needs sources and receivers", i); return RSGPU_ERR_ARG; }
        if (!s[i].data) { set_error("shot %d: data is null", i); return RSGPU_ERR_ARG; }
        if (kind == RSGPU_KIND_FWI && (!s[i].vp || !s[i].rho)) { set_error("shot %d: vp/rho are null", i); return RSGPU_ERR_ARG; }
        if (s[i].srcilum && (el || kind != RSGPU_KIND_FWI)) {
            set_error("shot %d: source illumination belongs to the acoustic 2D FWI gradient (FwiAcoustic2D::setSrcilum)", i);
            return RSGPU_ERR_ARG;
        }
    }
    return RSGPU_OK;
}

rsgpu_status Adjoint::create(const rsgpu_config *c, const rsgpu_adjoint_opts *o, int k, int ns,
                             const rsgpu_adjoint_shot *s)
{
    ST(check_adjoint(c, o, k, ns, s));
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) {
        cudaGetLastError();
        set_error("no CUDA device");
        return RSGPU_ERR_NODEVICE;
    }
    kind = k;
    cfg = *c;
    nshots = ns;
    prec = c->precision;
    es = esize(prec);
    acc = o->accum == RSGPU_ACCUM_F64 ? ACC_F64 : ACC_REF;
    // FwiAcoustic2D has no ADAPTIVE_SINGLE case: its misfit and residual switches fall
    // through to the DIFFERENCE code (lib/fwi.cpp:737-749, 1015-1026)
    misfit_type = c->physics != RSGPU_ELASTIC2D && o->misfit == RSGPU_MISFIT_ADAPTIVE_SINGLE ? RSGPU_MISFIT_DIFFERENCE
                                                                                              : o->misfit;
    for (int i = 0; i < ns; i++) nrec_max = std::max(nrec_max, s[i].shot.nrec);
    ck = o->ckpt_precision;
    ck_es = ck == CK_NATIVE ? (size_t)es : 2;
    nhx = kind == RSGPU_KIND_RTM ? o->nhx : 1;
    nhz = kind == RSGPU_KIND_RTM ? o->nhz : 1;
    snapmethod = o->snapmethod;
    if (snapmethod != RSGPU_SNAP_OPTIMAL) {
        snapinc = std::max(o->snapinc, 1);
        snapnt = (c->nt - 1) / snapinc + 1;
        enddiff = snap_enddiff(c->nt, c->dt, snapinc, prec);
        noreverse = kind == RSGPU_KIND_FWI && o->noreverse != 0;
    } else {
        RevolveSchedule probe(c->nt, o->ncheck);
        ncheck = probe.snaps();
    }
    CU(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));

    phys = c->physics == RSGPU_ELASTIC2D ? PHYS_E2D : PHYS_A2D;
    // forward plan: the shots as given, recording switched off after FIRSTURN
    std::vector<rsgpu_shot> fs(ns), bs(ns);
    for (int i = 0; i < ns; i++) {
        fs[i] = s[i].shot;
        fs[i].rec_out = nullptr;
        bs[i] = s[i].shot;
        // adjoint plan: receivers become sources, sources become receivers
        bs[i].nsrc = s[i].shot.nrec;
        bs[i].smap = s[i].shot.gmap;
        bs[i].sshift = s[i].shot.gshift;
        bs[i].wavelet = s[i].data;          // RTM: the data; FWI: replaced by the residuals
        bs[i].src_field = RSGPU_PRESSURE;
        bs[i].nrec = kind == RSGPU_KIND_FWI ? s[i].shot.nsrc : 0;
        bs[i].gmap = s[i].shot.smap;
        bs[i].gshift = s[i].shot.sshift;
        bs[i].rec_field = RSGPU_PRESSURE;
        bs[i].rec_factor = nullptr;
        bs[i].rec_out = nullptr;
    }
    // elastic: the forward plan records P, Ux and Uz; the adjoint plan injects the
    // three residuals and records the wavelet gradient at sources inside the
    // interior 1..n-2 (FwiElastic2D::crossCorr records it inside its interior loop)
    std::vector<ShotSets> fsets, bsets;
    std::vector<std::vector<int>> wmaps(ns);
    if (elastic()) {
        fsets.resize(ns);
        bsets.resize(ns);
        for (int i = 0; i < ns; i++) {
            const rsgpu_adjoint_shot &a = s[i];
            ShotSets &F = fsets[i], &B = bsets[i];
            F.nsrc = 1;
            F.src[0] = {a.shot.nsrc, a.shot.smap, a.shot.sshift, a.shot.src_field, a.shot.wavelet, nullptr, false};
            F.nrec = 3;
            F.rec[0] = {a.shot.nrec, a.shot.gmap, a.shot.gshift, RSGPU_PRESSURE, nullptr, nullptr, false};
            F.rec[1] = {a.shot.nrec, a.gmap_vx, a.gshift_vx, RSGPU_VX, nullptr, nullptr, false};
            F.rec[2] = {a.shot.nrec, a.gmap_vz, a.gshift_vz, RSGPU_VZ, nullptr, nullptr, false};
            B.nsrc = 3;
            B.src[0] = {a.shot.nrec, a.shot.gmap, a.shot.gshift, RSGPU_PRESSURE, a.data, nullptr, false};
            B.src[1] = {a.shot.nrec, a.gmap_vx, a.gshift_vx, RSGPU_VX, a.data_vx, nullptr, false};
            B.src[2] = {a.shot.nrec, a.gmap_vz, a.gshift_vz, RSGPU_VZ, a.data_vz, nullptr, false};
            std::vector<int> &wm = wmaps[i];
            wm.assign(a.shot.smap, a.shot.smap + 2 * a.shot.nsrc);
            for (int t = 0; t < a.shot.nsrc; t++)
                if (wm[2 * t] < 1 || wm[2 * t] > a.shot.nx - 2 || wm[2 * t + 1] < 1 || wm[2 * t + 1] > a.shot.nz - 2)
                    wm[2 * t] = wm[2 * t + 1] = -1;
            B.nrec = 1;
            B.rec[0] = {a.shot.nsrc, wm.data(), a.shot.sshift, a.shot.src_field, nullptr, nullptr,
                        a.shot.src_field == RSGPU_PRESSURE};
        }
    }
    fw.reset(new Plan());
    fw->gated_recording = true;
    fw->shared_stream = stream;
    ST(fw->create(c, ns, fs.data(), elastic() ? fsets.data() : nullptr));
    bw.reset(new Plan());
    bw->reverse_time = true;
    bw->adjoint_steps = elastic();
    bw->shared_stream = stream;
    ST(bw->create(c, ns, bs.data(), elastic() ? bsets.data() : nullptr));

    // device buffer: models, data, outputs, descriptors, checkpoint tables
    const size_t gs = acc == ACC_F64 ? 8 : (size_t)es;
    size_t off = 0;
    auto take = [&](size_t bytes) { size_t r = off; off = rup(off + std::max<size_t>(bytes, 1), 256); return r; };
    for (auto *v : {&o_vp, &o_vs, &o_rho, &o_obs, &o_obsx, &o_obsz, &o_g0, &o_g1, &o_g2, &o_ilum}) v->assign(ns, 0);
    nx.resize(ns); nz.resize(ns); nrec.resize(ns); nsrc.resize(ns);
    for (int i = 0; i < ns; i++) {
        nx[i] = s[i].shot.nx; nz[i] = s[i].shot.nz; nrec[i] = s[i].shot.nrec; nsrc[i] = s[i].shot.nsrc;
        nxmax = std::max(nxmax, nx[i]);
        nzmax = std::max(nzmax, nz[i]);
        const size_t n2 = (size_t)nx[i] * nz[i];
        if (kind == RSGPU_KIND_FWI) {
            o_vp[i] = take(n2 * es);
            o_rho[i] = take(n2 * es);
            o_obs[i] = take((size_t)nrec[i] * cfg.nt * es);
            o_g0[i] = take(n2 * gs);
            o_g1[i] = take(n2 * gs);
            if (!elastic() && s[i].srcilum) o_ilum[i] = take(n2 * gs);
            if (elastic()) {
                o_vs[i] = take(n2 * es);
                o_obsx[i] = take((size_t)nrec[i] * cfg.nt * es);
                o_obsz[i] = take((size_t)nrec[i] * cfg.nt * es);
                o_g2[i] = take(n2 * gs);
            }
        } else {
            o_g0[i] = take(n2 * nhx * nhz * gs);
        }
    }
    o_misfit = take(sizeof(double) * ns);
    o_rpart = take(sizeof(double) * residual_partials(ns));
    const bool adaptive = kind == RSGPU_KIND_FWI && (misfit_type == RSGPU_MISFIT_ADAPTIVE_GAUSS ||
                                                     misfit_type == RSGPU_MISFIT_ADAPTIVE_LINEAR ||
                                                     misfit_type == RSGPU_MISFIT_ADAPTIVE_SINGLE);
    o_wav0.assign(ns, 0);
    for (int i = 0; i < ns && snapmethod == RSGPU_SNAP_EDGES; i++)
        o_wav0[i] = take((size_t)fw->shots[i].nsrcs[0] * cfg.nt * es);
    const bool two_filters = adaptive && elastic() && misfit_type != RSGPU_MISFIT_ADAPTIVE_SINGLE;
    for (auto *v : {&o_work, &o_tnorm, &o_work2, &o_tnorm2}) v->assign(ns, 0);
    if (adaptive) {
        for (int i = 0; i < ns; i++) {
            o_work[i] = take(adaptive_work_values(misfit_type, cfg.nt) * nrec[i] * es);
            o_tnorm[i] = take((size_t)nrec[i] * es);
            if (two_filters) {
                o_work2[i] = take(adaptive_work_values(misfit_type, cfg.nt) * nrec[i] * es);
                o_tnorm2[i] = take((size_t)nrec[i] * es);
            }
        }
        o_atab = take(adaptive_table_bytes(prec, misfit_type, cfg.nt));
        if (two_filters) o_comp = take(2 * ns * (prec == PREC_F64 ? sizeof(Resid2D<double>) : sizeof(Resid2D<float>)));
    }
    const size_t corr_bytes = elastic() ? (prec == PREC_F64 ? sizeof(Corr2DE<double>) : sizeof(Corr2DE<float>))
                                        : (prec == PREC_F64 ? sizeof(Corr2D<double>) : sizeof(Corr2D<float>));
    const size_t res_bytes = elastic() ? (prec == PREC_F64 ? sizeof(Resid2DE<double>) : sizeof(Resid2DE<float>))
                                       : (prec == PREC_F64 ? sizeof(Resid2D<double>) : sizeof(Resid2D<float>));
    o_corr = take(corr_bytes * ns);
    o_res = take(res_bytes * ns);
    // checkpoint blocks: per shot the wavefields (interior of the pitched arrays)
    // and the C-PML memory strips
    segs.clear();
    slot_elems = 0;
    nslots = snapmethod != RSGPU_SNAP_OPTIMAL ? snapnt : ncheck;
    for (int i = 0; i < ns; i++) {
        const ShotLayout &L = fw->shots[i];
        const size_t org = ((size_t)GUARD * L.pitch + GUARD) * es;
        auto add = [&](size_t byte_off, int rows, int cols, int pitch) {
            CkptSeg g{};
            g.src = (char *)fw->arena + byte_off;
            g.rows = rows; g.cols = cols; g.pitch = pitch;
            g.dst = (long long)slot_elems;
            slot_elems += (size_t)rows * cols;
            slot_elems = rup(slot_elems, 64);   // keep every block 128-byte aligned in 16-bit slots
            segs.push_back(g);
        };
        if (snapmethod == RSGPU_SNAP_FULL) {
            // Snapshot2D::writeSnap: the nx*nz interior of P (lib/snap.cpp:638-667)
            add(L.f[A2_P] + org + ((size_t)cfg.lpml * L.pitch + cfg.lpml) * es, nz[i], nx[i], L.pitch);
            continue;
        }
        if (snapmethod == RSGPU_SNAP_EDGES) {
            // Snapshot2D::writeEdge (lib/snap.cpp:690-733): P on the columns x = lpml and
            // x = nx+lpml (the first C-PML column) over the interior rows, and on the rows
            // z = lpml and z = nz+lpml over the interior columns
            const size_t p0 = L.f[A2_P] + org, l = (size_t)cfg.lpml;
            add(p0 + (l * L.pitch + l) * es, nz[i], 1, L.pitch);
            add(p0 + (l * L.pitch + nx[i] + l) * es, nz[i], 1, L.pitch);
            add(p0 + (l * L.pitch + l) * es, 1, nx[i], L.pitch);
            add(p0 + ((nz[i] + l) * L.pitch + l) * es, 1, nx[i], L.pitch);
            continue;
        }
        for (int f = 0; f < nfields(phys); f++) add(L.f[f] + org, L.nzp, L.nxp, L.pitch);
        for (int p = 0; p < npsi(phys); p++) add(L.psix[p], L.nzp, 2 * cfg.lpml, 2 * cfg.lpml);
        for (int p = 0; p < npsi(phys); p++) add(L.psiz[p], 2 * cfg.lpml, L.nxp, L.nxp);
    }
    o_segs = take(sizeof(CkptSeg) * segs.size());
    seg_rows = ckpt_max_rows(segs.data(), segs.size());
    o_scales = take(sizeof(float) * segs.size() * nslots);
    o_maxbits = take(sizeof(unsigned) * segs.size());
    if (dev_alloc(&dbuf, off, stream) != cudaSuccess) {
        cudaGetLastError();
        set_error("device allocation of %zu bytes failed", off);
        return RSGPU_ERR_NOMEM;
    }
    const size_t ck_bytes = slot_elems * ck_es * (size_t)nslots;
    if (dev_alloc(&ckpt, ck_bytes, stream) != cudaSuccess) {
        cudaGetLastError();
        set_error("checkpoint allocation of %zu bytes (%d slots) failed", ck_bytes, nslots);
        return RSGPU_ERR_NOMEM;
    }
    CU(cudaMemsetAsync(dbuf, 0, off, stream));
    for (int i = 0; i < ns; i++)
        if (o_wav0[i])
            CU(cudaMemcpyAsync(D(o_wav0[i]), (char *)fw->arena + fw->shots[i].wavk[0],
                               (size_t)fw->shots[i].nsrcs[0] * cfg.nt * es, cudaMemcpyDeviceToDevice, stream));
    for (int i = 0; i < ns && kind == RSGPU_KIND_FWI; i++) {
        const size_t n2 = (size_t)nx[i] * nz[i];
        CU(cudaMemcpyAsync(D(o_vp[i]), s[i].vp, n2 * es, cudaMemcpyHostToDevice, stream));
        CU(cudaMemcpyAsync(D(o_rho[i]), s[i].rho, n2 * es, cudaMemcpyHostToDevice, stream));
        CU(cudaMemcpyAsync(D(o_obs[i]), s[i].data, (size_t)nrec[i] * cfg.nt * es, cudaMemcpyHostToDevice, stream));
        if (elastic()) {
            CU(cudaMemcpyAsync(D(o_vs[i]), s[i].vs, n2 * es, cudaMemcpyHostToDevice, stream));
            CU(cudaMemcpyAsync(D(o_obsx[i]), s[i].data_vx, (size_t)nrec[i] * cfg.nt * es, cudaMemcpyHostToDevice, stream));
            CU(cudaMemcpyAsync(D(o_obsz[i]), s[i].data_vz, (size_t)nrec[i] * cfg.nt * es, cudaMemcpyHostToDevice, stream));
        }
    }
    CU(cudaMemcpyAsync(D(o_segs), segs.data(), sizeof(CkptSeg) * segs.size(), cudaMemcpyHostToDevice, stream));
    std::vector<unsigned char> atab;
    if (adaptive) {
        atab.resize(adaptive_table_bytes(prec, misfit_type, cfg.nt));
        adaptive_fill_tables(prec, misfit_type, cfg.nt, atab.data());
        CU(cudaMemcpyAsync(D(o_atab), atab.data(), atab.size(), cudaMemcpyHostToDevice, stream));
    }
    std::vector<unsigned char> corr(corr_bytes * ns), res(res_bytes * ns);
    comp.clear();
    if (elastic()) {
        if (prec == PREC_F64) build_desc_e2d<double>(corr, res);
        else build_desc_e2d<float>(corr, res);
    } else {
        if (prec == PREC_F64) build_desc<double>(corr, res);
        else build_desc<float>(corr, res);
    }
    CU(cudaMemcpyAsync(D(o_corr), corr.data(), corr.size(), cudaMemcpyHostToDevice, stream));
    CU(cudaMemcpyAsync(D(o_res), res.data(), res.size(), cudaMemcpyHostToDevice, stream));
    if (o_comp) CU(cudaMemcpyAsync(D(o_comp), comp.data(), comp.size(), cudaMemcpyHostToDevice, stream));
    CU(cudaStreamSynchronize(stream));
    return RSGPU_OK;
}

template <typename T>
void Adjoint::build_desc(std::vector<unsigned char> &corr, std::vector<unsigned char> &res)
{
    for (int i = 0; i < nshots; i++) {
        const ShotLayout &F = fw->shots[i], &B = bw->shots[i];
        const size_t org = ((size_t)GUARD * F.pitch + GUARD) * es;
        char *fa = (char *)fw->arena, *ba = (char *)bw->arena;
        Corr2D<T> c{};
        c.wsp = (const T *)(fa + F.f[A2_P] + org);
        c.wrp = (const T *)(ba + B.f[A2_P] + org);
        c.wrx = (const T *)(ba + B.f[A2_VX] + org);
        c.wrz = (const T *)(ba + B.f[A2_VZ] + org);
        c.rx = (const T *)(fa + F.m[M_RX] + org);
        c.rz = (const T *)(fa + F.m[M_RZ] + org);
        c.vp = kind == RSGPU_KIND_FWI ? (const T *)D(o_vp[i]) : nullptr;
        c.rho = kind == RSGPU_KIND_FWI ? (const T *)D(o_rho[i]) : nullptr;
        c.g0 = D(o_g0[i]);
        c.g1 = kind == RSGPU_KIND_FWI ? D(o_g1[i]) : nullptr;
        c.ilum = o_ilum[i] ? D(o_ilum[i]) : nullptr;
        c.nx = nx[i]; c.nz = nz[i]; c.pitch = F.pitch; c.lpml = cfg.lpml;
        std::memcpy(corr.data() + i * sizeof c, &c, sizeof c);
        Resid2D<T> r{};
        if (kind == RSGPU_KIND_FWI) {
            r.mod = (const T *)(fa + F.traces);
            r.obs = (const T *)D(o_obs[i]);
            r.res = (T *)(ba + B.wav);
            // the forward plan's receiver plan marks off-grid receivers with -1
            r.rec_pt = (const int *)(fa + fw->rec_pt_offsets[(size_t)i * MAXSETS]);
            if (o_work[i]) {
                r.work = (T *)D(o_work[i]);
                r.tnorm = (T *)D(o_tnorm[i]);
            }
        }
        r.nrec = nrec[i];
        r.nt = cfg.nt;
        std::memcpy(res.data() + i * sizeof r, &r, sizeof r);
    }
}

template <typename T>
void Adjoint::build_desc_e2d(std::vector<unsigned char> &corr, std::vector<unsigned char> &res)
{
    for (int i = 0; i < nshots; i++) {
        const ShotLayout &F = fw->shots[i], &B = bw->shots[i];
        const size_t org = ((size_t)GUARD * F.pitch + GUARD) * es;
        char *fa = (char *)fw->arena, *ba = (char *)bw->arena;
        Corr2DE<T> c{};
        for (int k = 0; k < 5; k++) {
            c.ws[k] = (const T *)(fa + F.f[k] + org);
            c.wr[k] = (const T *)(ba + B.f[k] + org);
        }
        c.rx = (const T *)(fa + F.m[M_RX] + org);
        c.rz = (const T *)(fa + F.m[M_RZ] + org);
        c.vp = (const T *)D(o_vp[i]);
        c.vs = (const T *)D(o_vs[i]);
        c.rho = (const T *)D(o_rho[i]);
        c.g[0] = D(o_g0[i]);
        c.g[1] = D(o_g1[i]);
        c.g[2] = D(o_g2[i]);
        c.nx = nx[i]; c.nz = nz[i]; c.pitch = F.pitch; c.lpml = cfg.lpml;
        std::memcpy(corr.data() + i * sizeof c, &c, sizeof c);
        Resid2DE<T> r{};
        const size_t obs[3] = {o_obs[i], o_obsx[i], o_obsz[i]};
        for (int k = 0; k < 3; k++) {
            r.mod[k] = (const T *)(fa + F.tracesk[k]);
            r.obs[k] = (const T *)D(obs[k]);
            r.res[k] = (T *)(ba + B.wavk[k]);
        }
        r.rec_pt_vx = (const int *)(fa + fw->rec_pt_offsets[(size_t)i * MAXSETS + 1]);
        r.nrec = nrec[i];
        r.nt = cfg.nt;
        if (o_work[i]) {
            r.work[0] = (T *)D(o_work[i]);
            r.tnorm[0] = (T *)D(o_tnorm[i]);
            r.work[1] = o_work2[i] ? (T *)D(o_work2[i]) : nullptr;
            r.tnorm[1] = o_tnorm2[i] ? (T *)D(o_tnorm2[i]) : nullptr;
        }
        std::memcpy(res.data() + i * sizeof r, &r, sizeof r);
        if (o_comp) {
            // the Ux and Uz traces as two single-component views, shaped like acoustic traces
            comp.resize(2 * nshots * sizeof(Resid2D<T>));
            for (int k = 0; k < 2; k++) {
                Resid2D<T> v{};
                v.mod = r.mod[1 + k];
                v.obs = r.obs[1 + k];
                v.res = r.res[1 + k];
                v.rec_pt = r.rec_pt_vx;
                v.nrec = nrec[i];
                v.nt = cfg.nt;
                v.work = r.work[k];
                v.tnorm = r.tnorm[k];
                std::memcpy(comp.data() + (2 * i + k) * sizeof v, &v, sizeof v);
            }
        }
    }
}

rsgpu_status Adjoint::save(int slot)
{
    if (slot < 0 || slot >= nslots) { set_error("checkpoint slot %d outside [0,%d)", slot, nslots); return RSGPU_ERR_REVOLVE; }
    cudaError_t e = launch_ckpt_save(prec, ck, (const CkptSeg *)D(o_segs), (int)segs.size(), seg_rows,
                                     (char *)ckpt + (size_t)slot * slot_elems * ck_es,
                                     (float *)D(o_scales) + (size_t)slot * segs.size(), (unsigned *)D(o_maxbits), stream);
    if (e != cudaSuccess) { set_error("checkpoint save: %s", cudaGetErrorString(e)); return RSGPU_ERR_CUDA; }
    launches += ck == CK_NATIVE ? 1 : 2;
    ckpt_bytes += (long long)(slot_elems * ck_es);
    return RSGPU_OK;
}

rsgpu_status Adjoint::load(int slot)
{
    if (slot < 0 || slot >= nslots) { set_error("checkpoint slot %d outside [0,%d)", slot, nslots); return RSGPU_ERR_REVOLVE; }
    cudaError_t e = launch_ckpt_load(prec, ck, (const CkptSeg *)D(o_segs), (int)segs.size(), seg_rows,
                                     (const char *)ckpt + (size_t)slot * slot_elems * ck_es,
                                     (const float *)D(o_scales) + (size_t)slot * segs.size(), stream);
    if (e != cudaSuccess) { set_error("checkpoint restore: %s", cudaGetErrorString(e)); return RSGPU_ERR_CUDA; }
    launches += 1;
    ckpt_bytes += (long long)(slot_elems * ck_es);
    return RSGPU_OK;
}

rsgpu_status Adjoint::correlate()
{
    cudaError_t e = elastic() ? launch_corr_fwi_e2d(prec, acc, D(o_corr), nshots, nxmax, nzmax, cfg.dx, cfg.dz, stream)
                    : kind == RSGPU_KIND_FWI
                        ? launch_corr_fwi_a2d(prec, acc, D(o_corr), nshots, nxmax, nzmax, cfg.dx, cfg.dz, stream)
                        : launch_corr_rtm_a2d(prec, acc, D(o_corr), nshots, nxmax, nzmax, nhx, nhz, stream);
    if (e != cudaSuccess) { set_error("correlation launch: %s", cudaGetErrorString(e)); return RSGPU_ERR_CUDA; }
    launches += 1;
    return RSGPU_OK;
}

rsgpu_status Adjoint::reset_outputs()
{
    launches = 0;
    fw_steps = bw_steps = ckpt_bytes = 0;
    ran = false;
    ST(fw->reset());
    ST(bw->reset());
    for (int i = 0; i < nshots; i++) {
        const size_t gs = acc == ACC_F64 ? 8 : (size_t)es;
        const size_t n2 = (size_t)nx[i] * nz[i];
        CU(cudaMemsetAsync(D(o_g0[i]), 0, n2 * (kind == RSGPU_KIND_FWI ? 1 : (size_t)nhx * nhz) * gs, stream));
        if (kind == RSGPU_KIND_FWI) CU(cudaMemsetAsync(D(o_g1[i]), 0, n2 * gs, stream));
        if (elastic()) CU(cudaMemsetAsync(D(o_g2[i]), 0, n2 * gs, stream));
        if (o_ilum[i]) CU(cudaMemsetAsync(D(o_ilum[i]), 0, n2 * gs, stream));
    }
    return RSGPU_OK;
}

// computeMisfit + computeResiduals of every shot: the misfit and the residual
// traces that the adjoint plan injects
rsgpu_status Adjoint::residuals()
{
    const bool corr = misfit_type == RSGPU_MISFIT_CORRELATION;
    if (o_atab) {
        cudaError_t e = elastic() ? launch_residual_adaptive_e2d(prec, acc, misfit_type, D(o_res),
                                                                 o_comp ? D(o_comp) : nullptr, nshots, nrec_max, cfg.nt,
                                                                 D(o_atab), (double *)D(o_misfit), stream)
                                  : launch_residual_adaptive(prec, acc, misfit_type, D(o_res), nshots, nrec_max, cfg.nt,
                                                             D(o_atab), (double *)D(o_misfit), stream, true);
        if (e != cudaSuccess) { set_error("residual launch: %s", cudaGetErrorString(e)); return RSGPU_ERR_CUDA; }
        launches += 2;
        return RSGPU_OK;
    }
    cudaError_t e = elastic()
                    ? (corr ? launch_residual_corr_e2d(prec, acc, D(o_res), nshots, nrec_max, (double *)D(o_misfit), stream)
                            : launch_residual_e2d(prec, acc, D(o_res), nshots, (double *)D(o_misfit), stream))
                    : corr ? launch_residual_corr(prec, acc, D(o_res), nshots, nrec_max, (double *)D(o_misfit), stream, true)
                           : launch_residual(prec, acc, D(o_res), nshots, (double *)D(o_misfit), (double *)D(o_rpart),
                                             stream);
    if (e != cudaSuccess) { set_error("residual launch: %s", cudaGetErrorString(e)); return RSGPU_ERR_CUDA; }
    launches += elastic() || corr ? 1 : 2;
    return RSGPU_OK;
}

// FwiAcoustic2D::run (lib/fwi.cpp:1030-1156) and RtmAcoustic2D::run
// (lib/rtm.cpp:222-326): the forward loop records every step and saves the P
// interior after steps 0, snapinc, 2*snapinc, ...; the adjoint loop steps the
// adjoint wavefield from a zero state and, at the adjoint times t with
// (t - enddiff) % snapinc == 0, correlates it with snapshot (t - enddiff)/snapinc
// (Snapshot2D::readSnap counts the snapshots down from the last one written).
// RtmAcoustic2D::run_edge (lib/rtm.cpp:328-421) saves only P's four edge lines;
// its adjoint loop also steps the forward wavefield again from a zero state,
// without the source (the plan's source traces are zeroed for that pass: adding
// zero leaves every value as it is), and writes the saved edge lines into it at
// those adjoint times before correlating.
// Steps between two saves or two correlations go to the plans as one range.
rsgpu_status Adjoint::run_full()
{
    const int nt = cfg.nt;
    const bool edges = snapmethod == RSGPU_SNAP_EDGES;
    const long long l0 = fw->launches + bw->launches;
    ST(reset_outputs());
    for (int i = 0; i < nshots && edges; i++)
        CU(cudaMemcpyAsync((char *)fw->arena + fw->shots[i].wavk[0], D(o_wav0[i]),
                           (size_t)fw->shots[i].nsrcs[0] * cfg.nt * es, cudaMemcpyDeviceToDevice, stream));
    ST(fw->set_recording(true));
    ST(fw->run(0, 1));
    ST(save(0));
    for (int k = 1; k < snapnt; k++) {
        ST(fw->run((k - 1) * snapinc + 1, snapinc));
        ST(save(k));
    }
    const int done = (snapnt - 1) * snapinc + 1;
    if (done < nt) ST(fw->run(done, nt - done));
    fw_steps = nt;
    ST(fw->set_recording(false));
    if (kind == RSGPU_KIND_FWI) ST(residuals());
    if (edges) {
        ST(fw->reset());
        for (int i = 0; i < nshots; i++)
            CU(cudaMemsetAsync((char *)fw->arena + fw->shots[i].wavk[0], 0,
                               (size_t)fw->shots[i].nsrcs[0] * cfg.nt * es, stream));
    }
    if (!noreverse) {
        // adjoint step index k runs data time t = nt-1-k
        auto aligned = [&](int k) { return ((nt - 1 - k) - enddiff) % snapinc == 0; };
        for (int k = 0; k < nt;) {
            int e = k;
            while (e < nt && !aligned(e)) e++;
            const int n = (e < nt ? e + 1 : nt) - k;
            if (edges) {
                ST(fw->run(k, n));
                fw_steps += n;
            }
            ST(bw->run(k, n));
            bw_steps += n;
            k += n;
            if (e < nt) {
                ST(load(((nt - 1 - e) - enddiff) / snapinc));
                ST(correlate());
            }
        }
    }
    launches += fw->launches + bw->launches - l0;
    CU(cudaStreamSynchronize(stream));
    ST(fw->check_device_error());
    ST(bw->check_device_error());
    ran = true;
    return RSGPU_OK;
}

rsgpu_status Adjoint::run()
{
    if (snapmethod != RSGPU_SNAP_OPTIMAL) return run_full();
    const int nt = cfg.nt;
    const long long l0 = fw->launches + bw->launches;
    ST(reset_outputs());
    ST(fw->set_recording(true));
    RevolveSchedule rev(nt, ncheck);
    for (;;) {
        const int oldcapo = rev.capo();
        const int a = rev.next();
        const int capo = rev.capo();
        if (a == RSGPU_ADVANCE) {
            ST(fw->run(oldcapo, capo - oldcapo));
            fw_steps += capo - oldcapo;
        } else if (a == RSGPU_TAKESHOT) {
            ST(save(rev.check()));
        } else if (a == RSGPU_RESTORE) {
            ST(load(rev.check()));
        } else if (a == RSGPU_FIRSTURN) {
            // the last forward step, then the first adjoint time level (nt-1)
            ST(fw->run(capo, 1));
            fw_steps += 1;
            ST(fw->set_recording(false));
            if (kind == RSGPU_KIND_FWI) ST(residuals());
            ST(bw->inject_record_only(nt - 1 - capo));
            ST(correlate());
        } else if (a == RSGPU_YOUTURN) {
            ST(bw->run(nt - 1 - capo, 1));
            bw_steps += 1;
            ST(correlate());
        } else if (a == RSGPU_TERMINATE) {
            break;
        } else {
            set_error("revolve schedule error (info %d)", rev.info());
            return RSGPU_ERR_REVOLVE;
        }
    }
    if (elastic()) {
        // FwiElastic2D::scaleGrad after the time loop
        cudaError_t e = launch_scale_grad_e2d(prec, acc, D(o_corr), nshots, nxmax, nzmax, stream);
        if (e != cudaSuccess) { set_error("gradient scaling launch: %s", cudaGetErrorString(e)); return RSGPU_ERR_CUDA; }
        launches += 1;
    }
    launches += fw->launches + bw->launches - l0;
    CU(cudaStreamSynchronize(stream));
    ST(fw->check_device_error());
    ST(bw->check_device_error());
    ran = true;
    return RSGPU_OK;
}

template <typename T, typename G>
static void add_into(void *host, const std::vector<unsigned char> &dev, size_t n)
{
    T *o = (T *)host;
    const G *d = (const G *)dev.data();
    for (size_t k = 0; k < n; k++) o[k] = (T)((G)o[k] + d[k]);
}

// Image2D::stackImage of every shot's window into global arrays, on the device: the
// host arrays out[] (element type) are the running global images; they are uploaded,
// every shot's window is added in shot order and the result is written back, so a
// sequence of batches stacks exactly as the reference's shot-by-shot stackImage
// does.  Components: FWI acoustic vpgrad, rhograd; elastic vpgrad, vsgrad, rhograd;
// RTM the image with its lags.
rsgpu_status Adjoint::stack(int nxg, int nzg, const int *x0, const int *z0, void *const *out)
{
    if (!ran) { set_error("no run to stack"); return RSGPU_ERR_STATE; }
    if (nxg < 1 || nzg < 1 || !x0 || !z0 || !out) { set_error("stack: bad arguments"); return RSGPU_ERR_ARG; }
    const int ncomp = kind == RSGPU_KIND_RTM ? 1 : elastic() ? 3 : 2;
    const int nh = kind == RSGPU_KIND_RTM ? nhx * nhz : 1;
    const size_t gs = acc == ACC_F64 ? 8 : (size_t)es;
    std::vector<StackWin> w(nshots);
    for (int i = 0; i < nshots; i++) {
        w[i].g[0] = D(o_g0[i]);
        w[i].g[1] = kind == RSGPU_KIND_FWI ? D(o_g1[i]) : nullptr;
        w[i].g[2] = elastic() ? D(o_g2[i]) : nullptr;
        w[i].nx = nx[i];
        w[i].nz = nz[i];
        w[i].x0 = x0[i];
        w[i].z0 = z0[i];
    }
    const size_t n = (size_t)nxg * nzg * nh;
    void *buf = nullptr;
    const size_t bytes = gs * n * ncomp + sizeof(StackWin) * nshots;
    if (dev_alloc(&buf, bytes, stream) != cudaSuccess) {
        cudaGetLastError();
        set_error("stack: device allocation of %zu bytes failed", bytes);
        return RSGPU_ERR_NOMEM;
    }
    char *b = (char *)buf;
    StackWin *dw = (StackWin *)(b + gs * n * ncomp);
    rsgpu_status st = RSGPU_OK;
    // the running global images in the accumulator type (a missing output stacks from zero)
    std::vector<unsigned char> tmp(gs * n * ncomp, 0);
    for (int c = 0; c < ncomp; c++) {
        if (!out[c]) continue;
        unsigned char *t = tmp.data() + c * gs * n;
        if (gs == (size_t)es) std::memcpy(t, out[c], gs * n);
        else for (size_t k = 0; k < n; k++) ((double *)t)[k] = (double)((const float *)out[c])[k];
    }
    cudaError_t e = cudaMemcpyAsync(b, tmp.data(), gs * n * ncomp, cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dw, w.data(), sizeof(StackWin) * nshots, cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess)
        e = launch_stack_windows((int)gs, dw, nshots, ncomp, nxg, nzg, nh, b, ncomp > 1 ? b + gs * n : nullptr,
                                 ncomp > 2 ? b + 2 * gs * n : nullptr, stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(tmp.data(), b, gs * n * ncomp, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    for (int c = 0; c < ncomp && e == cudaSuccess; c++) {
        if (!out[c]) continue;
        const unsigned char *t = tmp.data() + c * gs * n;
        if (gs == (size_t)es) std::memcpy(out[c], t, gs * n);
        else for (size_t k = 0; k < n; k++) ((float *)out[c])[k] = (float)((const double *)t)[k];
    }
    if (e != cudaSuccess) {
        set_error("stack: %s", cudaGetErrorString(e));
        st = RSGPU_ERR_CUDA;
    }
    cudaStreamSynchronize(stream);
    dev_free(buf, stream);
    return st;
}


rsgpu_status Adjoint::read(int ns, const rsgpu_adjoint_shot *s)
{
    if (!ran) { set_error("no run to read"); return RSGPU_ERR_STATE; }
    if (ns != nshots || !s) { set_error("read expects the %d shots of the batch", nshots); return RSGPU_ERR_ARG; }
    const size_t gs = acc == ACC_F64 ? 8 : (size_t)es;
    std::vector<unsigned char> tmp;
    auto fetch = [&](size_t o, size_t bytes) -> rsgpu_status {
        tmp.resize(bytes);
        CU(cudaMemcpyAsync(tmp.data(), D(o), bytes, cudaMemcpyDeviceToHost, stream));
        CU(cudaStreamSynchronize(stream));
        return RSGPU_OK;
    };
    // accumulate a device array of accumulator type into a host array of the element type
    auto accumulate = [&](void *host, size_t n) {
        if (es == 8) add_into<double, double>(host, tmp, n);
        else if (gs == 8) add_into<float, double>(host, tmp, n);
        else add_into<float, float>(host, tmp, n);
    };
    std::vector<double> mis(nshots, 0.0);
    if (kind == RSGPU_KIND_FWI) {
        CU(cudaMemcpyAsync(mis.data(), D(o_misfit), sizeof(double) * nshots, cudaMemcpyDeviceToHost, stream));
        CU(cudaStreamSynchronize(stream));
    }
    for (int i = 0; i < nshots; i++) {
        const size_t n2 = (size_t)nx[i] * nz[i];
        if (kind == RSGPU_KIND_RTM) {
            if (s[i].image) { ST(fetch(o_g0[i], n2 * nhx * nhz * gs)); accumulate(s[i].image, n2 * nhx * nhz); }
            continue;
        }
        if (s[i].vpgrad) { ST(fetch(o_g0[i], n2 * gs)); accumulate(s[i].vpgrad, n2); }
        if (elastic()) {
            if (s[i].vsgrad) { ST(fetch(o_g1[i], n2 * gs)); accumulate(s[i].vsgrad, n2); }
            if (s[i].rhograd) { ST(fetch(o_g2[i], n2 * gs)); accumulate(s[i].rhograd, n2); }
        } else if (s[i].rhograd) {
            ST(fetch(o_g1[i], n2 * gs));
            accumulate(s[i].rhograd, n2);
        }
        if (o_ilum[i] && s[i].srcilum) { ST(fetch(o_ilum[i], n2 * gs)); accumulate(s[i].srcilum, n2); }
        void *mods[3] = {s[i].shot.rec_out, elastic() ? s[i].datamod_vx : nullptr, elastic() ? s[i].datamod_vz : nullptr};
        void *ress[3] = {s[i].datares, elastic() ? s[i].datares_vx : nullptr, elastic() ? s[i].datares_vz : nullptr};
        for (int k = 0; k < 3; k++) {
            if (mods[k]) ST(fw->read_traces(i, mods[k], k));
            if (!ress[k] || noreverse) continue;   // FwiAcoustic2D::run leaves dataresP unset
            const size_t n = (size_t)nrec[i] * cfg.nt;
            tmp.resize(n * es);
            CU(cudaMemcpyAsync(tmp.data(), (char *)bw->arena + bw->shots[i].wavk[k], n * es, cudaMemcpyDeviceToHost,
                               stream));
            CU(cudaStreamSynchronize(stream));
            if (es == 8) add_into<double, double>(ress[k], tmp, n);
            else add_into<float, float>(ress[k], tmp, n);
        }
        if (s[i].wavgrad && !noreverse) ST(bw->read_traces(i, s[i].wavgrad));
        if (s[i].misfit) {
            // the reference keeps the misfit in T
            if (acc == ACC_REF && es == 4) *s[i].misfit = (double)(float)((float)*s[i].misfit + (float)mis[i]);
            else *s[i].misfit += mis[i];
        }
    }
    return RSGPU_OK;
}

}  // namespace rsgpu

using namespace rsgpu;

struct rsgpu_adjoint {
    std::unique_ptr<Adjoint> a;       // 2D physics
    std::unique_ptr<Adjoint3D> a3;    // 3D physics
};

extern "C" {

rsgpu_status rsgpu_adjoint_create(const rsgpu_config *cfg, const rsgpu_adjoint_opts *opts, int kind, int nshots,
                                  const rsgpu_adjoint_shot *shots, rsgpu_adjoint **adj)
{
    if (!adj) { set_error("handle pointer is null"); return RSGPU_ERR_ARG; }
    *adj = nullptr;
    std::unique_ptr<rsgpu_adjoint> h(new rsgpu_adjoint);
    rsgpu_status st;
    if (cfg && (cfg->physics == RSGPU_ACOUSTIC3D || cfg->physics == RSGPU_ELASTIC3D)) {
        h->a3.reset(new Adjoint3D());
        st = h->a3->create(cfg, opts, kind, nshots, shots);
    } else {
        h->a.reset(new Adjoint());
        st = h->a->create(cfg, opts, kind, nshots, shots);
    }
    if (st != RSGPU_OK) return st;
    *adj = h.release();
    return RSGPU_OK;
}

rsgpu_status rsgpu_adjoint_run(rsgpu_adjoint *adj)
{
    if (!adj) { set_error("null handle"); return RSGPU_ERR_ARG; }
    return adj->a3 ? adj->a3->run() : adj->a->run();
}

rsgpu_status rsgpu_adjoint_read(rsgpu_adjoint *adj, int nshots, const rsgpu_adjoint_shot *shots)
{
    if (!adj) { set_error("null handle"); return RSGPU_ERR_ARG; }
    return adj->a3 ? adj->a3->read(nshots, shots) : adj->a->read(nshots, shots);
}

rsgpu_status rsgpu_adjoint_stack(rsgpu_adjoint *adj, int nxg, int nzg, const int *ix_start, const int *iz_start,
                                 void *out0, void *out1, void *out2)
{
    if (!adj) { set_error("null handle"); return RSGPU_ERR_ARG; }
    if (adj->a3) { set_error("stacking is built for the 2D drivers"); return RSGPU_ERR_UNSUPPORTED; }
    void *out[3] = {out0, out1, out2};
    return adj->a->stack(nxg, nzg, ix_start, iz_start, out);
}

rsgpu_status rsgpu_adjoint_stats(rsgpu_adjoint *adj, long long *fw_steps, long long *bw_steps, long long *ckpt_bytes,
                                 long long *launches)
{
    if (!adj) { set_error("null handle"); return RSGPU_ERR_ARG; }
    if (fw_steps) *fw_steps = adj->a3 ? adj->a3->fw_steps : adj->a->fw_steps;
    if (bw_steps) *bw_steps = adj->a3 ? adj->a3->bw_steps : adj->a->bw_steps;
    if (ckpt_bytes) *ckpt_bytes = adj->a3 ? adj->a3->ckpt_bytes : adj->a->ckpt_bytes;
    if (launches) *launches = adj->a3 ? adj->a3->launches : adj->a->launches;
    return RSGPU_OK;
}

void *rsgpu_adjoint_stream(rsgpu_adjoint *adj)
{
    return adj ? (void *)(adj->a3 ? adj->a3->stream : adj->a->stream) : nullptr;
}
void rsgpu_adjoint_destroy(rsgpu_adjoint *adj) { delete adj; }

static rsgpu_status one_call(const rsgpu_config *cfg, const rsgpu_adjoint_opts *opts, int kind, int nshots,
                             const rsgpu_adjoint_shot *shots)
{
    rsgpu_adjoint *h = nullptr;
    rsgpu_status st = rsgpu_adjoint_create(cfg, opts, kind, nshots, shots, &h);
    if (st == RSGPU_OK) st = rsgpu_adjoint_run(h);
    if (st == RSGPU_OK) st = rsgpu_adjoint_read(h, nshots, shots);
    rsgpu_adjoint_destroy(h);
    return st;
}

rsgpu_status rsgpu_fwi_gradient(const rsgpu_config *cfg, const rsgpu_adjoint_opts *opts, int nshots,
                                const rsgpu_adjoint_shot *shots)
{
    return one_call(cfg, opts, RSGPU_KIND_FWI, nshots, shots);
}

rsgpu_status rsgpu_rtm_image(const rsgpu_config *cfg, const rsgpu_adjoint_opts *opts, int nshots,
                             const rsgpu_adjoint_shot *shots)
{
    return one_call(cfg, opts, RSGPU_KIND_RTM, nshots, shots);
}

}  // extern "C"
