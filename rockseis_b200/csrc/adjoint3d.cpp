// RTM image and FWI gradient drivers for 3D shots (host runtime behind
// rsgpu_rtm_image, rsgpu_fwi_gradient and rsgpu_adjoint_* for RSGPU_ACOUSTIC3D and,
// FWI only, RSGPU_ELASTIC3D).
//
// The reference's RtmAcoustic3D::run_optimal (lib/rtm.cpp:735-859) runs the same
// Revolve-driven loop as the 2D drivers (FwiAcoustic3D::run_optimal,
// lib/fwi.cpp:1991-2160, likewise): a forward propagator checkpointed in
// `ncheck` slots, an adjoint propagator fed with the recorded data, and a
// correlation of both pressures at every adjoint time level.  Here the forward and
// adjoint wavefields of all shots are two batched 3D plans (z-marching kernels)
// sharing one stream and one copy of the staggered parameters; the adjoint plan
// runs forward in reversed time.  Checkpoints hold every shot's wavefields
// (interior of the pitched arrays) and C-PML memory, lossless or as FP16/BF16 with
// a power-of-two scale per block.
//
// FwiElastic3D::run_optimal (lib/fwi.cpp:6770-6990) is the same loop with the
// elastic plans: the forward plan records the Ux, Uy and Uz data sets, the adjoint
// plan (backwardstepVelocity / backwardstepStress kernels) injects the three
// residuals at their receivers and records the wavelet gradient at the sources,
// and the correlation is FwiElastic3D::crossCorr; scaleGrad follows the last
// adjoint step.
#include <algorithm>
#include <cstring>
#include <memory>
#include <type_traits>
#include <vector>

#include <cuda_runtime.h>

#include "rsgpu.h"
#include "rsgpu_3d.h"
#include "rsgpu_adjoint.h"
#include "rsgpu_adjoint3d.h"
#include "rsgpu_host.h"
#include "rsgpu_plan3d.h"

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

static inline size_t rupa(size_t a, size_t b) { return (a + b - 1) / b * b; }

Adjoint3D::~Adjoint3D()
{
    fw.reset();
    bw.reset();
    dev_free(dbuf, stream);
    dev_free(ckpt, stream);
    if (stream) cudaStreamDestroy(stream);
}

rsgpu_status Adjoint3D::create(const rsgpu_config *c, const rsgpu_adjoint_opts *o, int k_, int ns,
                               const rsgpu_adjoint_shot *s)
{
    if (!c || !o || !s || ns < 1) { set_error("null config/options/shots or nshots < 1"); return RSGPU_ERR_ARG; }
    const bool el = c->physics == RSGPU_ELASTIC3D;
    if ((c->physics != RSGPU_ACOUSTIC3D && !el) || (k_ != RSGPU_KIND_RTM && k_ != RSGPU_KIND_FWI) ||
        (el && k_ != RSGPU_KIND_FWI)) {
        set_error("the 3D adjoint driver is built for acoustic RTM images and FWI gradients and elastic FWI gradients");
        return RSGPU_ERR_UNSUPPORTED;
    }
    if (el && o->misfit != RSGPU_MISFIT_DIFFERENCE) {
        set_error("elastic 3D: misfit %d: DIFFERENCE is built", o->misfit);
        return RSGPU_ERR_UNSUPPORTED;
    }
    if (k_ == RSGPU_KIND_FWI && (o->misfit < RSGPU_MISFIT_DIFFERENCE || o->misfit > RSGPU_MISFIT_ADAPTIVE_SINGLE)) {
        set_error("misfit %d: DIFFERENCE, CORRELATION, ADAPTIVE_GAUSS, ADAPTIVE_LINEAR and ADAPTIVE_SINGLE are built",
                  o->misfit);
        return RSGPU_ERR_UNSUPPORTED;
    }
    if (k_ == RSGPU_KIND_FWI && o->misfit == RSGPU_MISFIT_CORRELATION) {
        const int lim = 49152 / (c->precision == RSGPU_F64 ? 8 : 4);
        for (int i = 0; i < ns; i++)
            if (s[i].shot.nrec > lim) {
                set_error("shot %d: the CORRELATION misfit takes at most %d receivers per shot", i, lim);
                return RSGPU_ERR_UNSUPPORTED;
            }
    }
    // FwiAcoustic3D has no ADAPTIVE_SINGLE case: its switches fall through to the
    // DIFFERENCE code (lib/fwi.cpp:1631-1644, 1841-1852)
    misfit_type = o->misfit == RSGPU_MISFIT_ADAPTIVE_SINGLE ? RSGPU_MISFIT_DIFFERENCE : o->misfit;
    for (int i = 0; i < ns; i++) nrec_max = std::max(nrec_max, s[i].shot.nrec);
    if (o->ckpt_precision < RSGPU_CKPT_NATIVE || o->ckpt_precision > RSGPU_CKPT_BF16) {
        set_error("bad checkpoint precision %d", o->ckpt_precision);
        return RSGPU_ERR_ARG;
    }
    if (o->accum != RSGPU_ACCUM_REFERENCE && o->accum != RSGPU_ACCUM_F64) { set_error("bad accumulation %d", o->accum); return RSGPU_ERR_ARG; }
    if (o->snapmethod != RSGPU_SNAP_OPTIMAL && o->snapmethod != RSGPU_SNAP_FULL && o->snapmethod != RSGPU_SNAP_EDGES) {
        set_error("bad snapmethod %d", o->snapmethod);
        return RSGPU_ERR_ARG;
    }
    // FULL snapshots: RtmAcoustic3D::run.  FwiAcoustic3D::run correlates against its
    // unpadded snapshot with crossCorr's index range 1..n-1, which at the last interior
    // corner reads one element past the snapshot array (lib/fwi.cpp:1441-1459 with
    // Snapshot3D, lib/snap.cpp:1138-1195): not reproducible, so not offered.
    if (o->snapmethod != RSGPU_SNAP_OPTIMAL && (el || k_ != RSGPU_KIND_RTM || o->snapmethod == RSGPU_SNAP_EDGES)) {
        set_error("snapmethod %d: the 3D drivers offer FULL snapshots for the acoustic RTM image (RtmAcoustic3D::run) "
                  "and Revolve checkpointing otherwise", o->snapmethod);
        return RSGPU_ERR_UNSUPPORTED;
    }
    const int hy = o->nhy > 0 ? o->nhy : 1;
    if (k_ == RSGPU_KIND_RTM && (o->nhx < 1 || o->nhz < 1 || o->nhx % 2 == 0 || hy % 2 == 0 || o->nhz % 2 == 0)) {
        set_error("nhx, nhy and nhz must be odd and positive");
        return RSGPU_ERR_ARG;
    }
    for (int i = 0; i < ns; i++) {
        const rsgpu_shot &sh = s[i].shot;
        if (!el && (sh.src_field != RSGPU_PRESSURE || sh.rec_field != RSGPU_PRESSURE)) {
            set_error("shot %d: the acoustic 3D drivers take pressure sources and receivers", i);
            return RSGPU_ERR_UNSUPPORTED;
        }
        if (el && sh.rec_field != RSGPU_VX) {
            set_error("shot %d: elastic 3D FWI: the shot's receiver set is the Ux (RSGPU_VX) data set", i);
            return RSGPU_ERR_ARG;
        }
        if (el && (!s[i].gmap_vy || !s[i].gshift_vy || !s[i].data_vy || !s[i].gmap_vz || !s[i].gshift_vz ||
                   !s[i].data_vz || !s[i].vs)) {
            set_error("shot %d: elastic 3D FWI needs the Uy and Uz data sets (maps, shifts, data) and vs", i);
            return RSGPU_ERR_ARG;
        }
        if (sh.nsrc < 1 || sh.nrec < 1) { set_error("shot %d: needs sources and receivers", i); return RSGPU_ERR_ARG; }
        if (!s[i].data) { set_error("shot %d: data is null", i); return RSGPU_ERR_ARG; }
        if (s[i].srcilum) {
            set_error("shot %d: the 3D gradients have no source illumination (FwiAcoustic3D/FwiElastic3D::crossCorr)", i);
            return RSGPU_ERR_ARG;
        }
        if (k_ == RSGPU_KIND_FWI && (!s[i].vp || !s[i].rho)) { set_error("shot %d: vp/rho are null", i); return RSGPU_ERR_ARG; }
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) {
        cudaGetLastError();
        set_error("no CUDA device");
        return RSGPU_ERR_NODEVICE;
    }
    kind = k_;
    phys = el ? PHYS_E3D : PHYS_A3D;
    cfg = *c;
    nshots = ns;
    prec = c->precision;
    es = prec == PREC_F64 ? 8 : 4;
    acc = o->accum == RSGPU_ACCUM_F64 ? ACC_F64 : ACC_REF;
    ck = o->ckpt_precision;
    ck_es = ck == CK_NATIVE ? (size_t)es : 2;
    nhx = fwi() ? 1 : o->nhx;
    nhy = fwi() ? 1 : hy;
    nhz = fwi() ? 1 : o->nhz;
    snapmethod = o->snapmethod;
    if (snapmethod == RSGPU_SNAP_FULL) {
        snapinc = std::max(o->snapinc, 1);
        snapnt = (c->nt - 1) / snapinc + 1;
        enddiff = snap_enddiff(c->nt, c->dt, snapinc, prec);
        nslots = snapnt;
    } else {
        RevolveSchedule probe(c->nt, o->ncheck);
        ncheck = probe.snaps();
        nslots = ncheck;
    }
    CU(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));

    std::vector<rsgpu_shot> fs(ns), bs(ns);
    for (int i = 0; i < ns; i++) {
        fs[i] = s[i].shot;
        if (!fwi()) fs[i].nrec = 0;          // RTM: the forward run records nothing
        fs[i].rec_out = nullptr;
        bs[i] = s[i].shot;
        bs[i].nsrc = s[i].shot.nrec;         // the data, injected at the receivers
        bs[i].smap = s[i].shot.gmap;
        bs[i].sshift = s[i].shot.gshift;
        bs[i].wavelet = s[i].data;           // FWI: replaced by the residuals
        bs[i].nrec = fwi() ? s[i].shot.nsrc : 0;   // FWI: the wavelet gradient at the sources
        bs[i].gmap = s[i].shot.smap;
        bs[i].gshift = s[i].shot.sshift;
        bs[i].rec_out = nullptr;
    }
    // elastic: the forward plan records Ux, Uy and Uz; the adjoint plan injects the
    // three residuals and records the wavelet gradient at sources inside the
    // interior 1..n-2 of every axis (crossCorr records it inside its interior loop)
    std::vector<ShotSets> fsets, bsets;
    std::vector<std::vector<int>> wmaps(ns);
    if (el) {
        fsets.resize(ns);
        bsets.resize(ns);
        for (int i = 0; i < ns; i++) {
            const rsgpu_adjoint_shot &a = s[i];
            const int nr = a.shot.nrec;
            ShotSets &F = fsets[i], &B = bsets[i];
            F.nsrc = 1;
            F.src[0] = {a.shot.nsrc, a.shot.smap, a.shot.sshift, a.shot.src_field, a.shot.wavelet, nullptr, false};
            F.nrec = 3;
            F.rec[0] = {nr, a.shot.gmap, a.shot.gshift, RSGPU_VX, nullptr, nullptr, false};
            F.rec[1] = {nr, a.gmap_vy, a.gshift_vy, RSGPU_VY, nullptr, nullptr, false};
            F.rec[2] = {nr, a.gmap_vz, a.gshift_vz, RSGPU_VZ, nullptr, nullptr, false};
            B.nsrc = 3;
            B.src[0] = {nr, a.shot.gmap, a.shot.gshift, RSGPU_VX, a.data, nullptr, false};
            B.src[1] = {nr, a.gmap_vy, a.gshift_vy, RSGPU_VY, a.data_vy, nullptr, false};
            B.src[2] = {nr, a.gmap_vz, a.gshift_vz, RSGPU_VZ, a.data_vz, nullptr, false};
            std::vector<int> &wm = wmaps[i];
            wm.assign(a.shot.smap, a.shot.smap + 3 * a.shot.nsrc);
            for (int t = 0; t < a.shot.nsrc; t++) {
                const int *m = &wm[3 * t];
                if (m[0] < 1 || m[0] > a.shot.nx - 2 || m[1] < 1 || m[1] > a.shot.ny - 2 || m[2] < 1 ||
                    m[2] > a.shot.nz - 2)
                    wm[3 * t] = wm[3 * t + 1] = wm[3 * t + 2] = -1;
            }
            B.nrec = 1;
            B.rec[0] = {a.shot.nsrc, wm.data(), a.shot.sshift, a.shot.src_field, nullptr, nullptr, false};
            B.rec[0].at_point = true;
        }
    }
    fw.reset(new Plan3D());
    fw->shared_stream = stream;
    fw->gated_recording = fwi();
    ST(fw->create(c, ns, fs.data(), el ? fsets.data() : nullptr));
    bw.reset(new Plan3D());
    bw->shared_stream = stream;
    bw->reverse_time = true;
    bw->adjoint_steps = el;
    bw->share_params = fw.get();
    ST(bw->create(c, ns, bs.data(), el ? bsets.data() : nullptr));

    const size_t gs = acc == ACC_F64 ? 8 : (size_t)es;
    size_t off = 0;
    auto take = [&](size_t bytes) { size_t r = off; off = rupa(off + std::max<size_t>(bytes, 1), 256); return r; };
    for (auto *v : {&o_img, &o_vp, &o_rho, &o_obs, &o_g1, &o_valid, &o_vs, &o_obsy, &o_obsz, &o_g2}) v->assign(ns, 0);
    nx.resize(ns); ny.resize(ns); nz.resize(ns); nrec.resize(ns);
    for (int i = 0; i < ns; i++) {
        nx[i] = s[i].shot.nx; ny[i] = s[i].shot.ny; nz[i] = s[i].shot.nz; nrec[i] = s[i].shot.nrec;
        nxmax = std::max(nxmax, nx[i]);
        nymax = std::max(nymax, ny[i]);
        const size_t n3 = (size_t)nx[i] * ny[i] * nz[i];
        o_img[i] = take(n3 * nhx * nhy * nhz * gs);     // RTM image, or FWI vp gradient
        if (fwi()) {
            o_vp[i] = take(n3 * es);
            o_rho[i] = take(n3 * es);
            o_obs[i] = take((size_t)nrec[i] * cfg.nt * es);
            o_g1[i] = take(n3 * gs);
            o_valid[i] = take(sizeof(int) * nrec[i]);
            if (el) {
                o_vs[i] = take(n3 * es);
                o_obsy[i] = take((size_t)nrec[i] * cfg.nt * es);
                o_obsz[i] = take((size_t)nrec[i] * cfg.nt * es);
                o_g2[i] = take(n3 * gs);
            }
        }
    }
    const size_t corr_bytes = el ? (prec == PREC_F64 ? sizeof(Corr3DE<double>) : sizeof(Corr3DE<float>))
                            : fwi() ? (prec == PREC_F64 ? sizeof(Corr3DF<double>) : sizeof(Corr3DF<float>))
                                    : (prec == PREC_F64 ? sizeof(Corr3D<double>) : sizeof(Corr3D<float>));
    const size_t res_bytes = el ? (prec == PREC_F64 ? sizeof(Resid3E<double>) : sizeof(Resid3E<float>))
                                : (prec == PREC_F64 ? sizeof(Resid2D<double>) : sizeof(Resid2D<float>));
    o_corr = take(corr_bytes * ns);
    o_res = take(res_bytes * ns);
    o_misfit = take(sizeof(double) * ns);
    o_rpart = take(sizeof(double) * residual_partials(ns));
    const bool adaptive = fwi() && (misfit_type == RSGPU_MISFIT_ADAPTIVE_GAUSS ||
                                    misfit_type == RSGPU_MISFIT_ADAPTIVE_LINEAR);
    o_work.assign(ns, 0);
    o_tnorm.assign(ns, 0);
    if (adaptive) {
        for (int i = 0; i < ns; i++) {
            o_work[i] = take(adaptive_work_values(misfit_type, cfg.nt) * nrec[i] * es);
            o_tnorm[i] = take((size_t)nrec[i] * es);
        }
        o_atab = take(adaptive_table_bytes(prec, misfit_type, cfg.nt));
    }
    segs.clear();
    slot_elems = 0;
    for (int i = 0; i < ns; i++) {
        const Layout3D &L = fw->shots[i];
        auto add = [&](size_t byte_off, int rows, int cols, int pitch, int prow, long long pstride) {
            CkptSeg g{};
            g.src = (char *)fw->arena + byte_off;
            g.rows = rows; g.cols = cols; g.pitch = pitch; g.prow = prow; g.pstride = pstride;
            g.dst = (long long)slot_elems;
            slot_elems = rupa(slot_elems + (size_t)rows * cols, 64);
            segs.push_back(g);
        };
        const int l2 = 2 * cfg.lpml;
        if (snapmethod == RSGPU_SNAP_FULL) {
            // Snapshot3D::writeSnap: the nx*ny*nz interior of P (lib/snap.cpp:1138-1172)
            const size_t l = (size_t)cfg.lpml;
            add(L.f[A3_P] + fw->origin_bytes(L) + (l * L.plane + l * L.pitch + l) * es, ny[i] * nz[i], nx[i], L.pitch,
                ny[i], L.plane);
            continue;
        }
        for (int f = 0; f < fw->nf3(); f++)
            add(L.f[f] + fw->origin_bytes(L), L.nyp * L.nzp, L.nxp, L.pitch, L.nyp, L.plane);
        for (int k = 0; k < fw->npsi3(); k++) {
            add(L.psix[k], L.nzp * L.nyp, l2, l2, 0, 0);
            add(L.psiy[k], L.nzp * l2, L.nxp, L.nxp, 0, 0);
            add(L.psiz[k], l2 * L.nyp, L.nxp, L.nxp, 0, 0);
        }
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
    CU(cudaMemcpyAsync(D(o_segs), segs.data(), sizeof(CkptSeg) * segs.size(), cudaMemcpyHostToDevice, stream));
    std::vector<unsigned char> atab;
    if (adaptive) {
        atab.resize(adaptive_table_bytes(prec, misfit_type, cfg.nt));
        adaptive_fill_tables(prec, misfit_type, cfg.nt, atab.data());
        CU(cudaMemcpyAsync(D(o_atab), atab.data(), atab.size(), cudaMemcpyHostToDevice, stream));
    }
    std::vector<unsigned char> corr(corr_bytes * ns), res(res_bytes * ns);
    std::vector<std::vector<int>> valids(ns);   // host copies stay alive until the stream sync below
    for (int i = 0; i < ns && fwi(); i++) {
        const size_t n3 = (size_t)nx[i] * ny[i] * nz[i];
        CU(cudaMemcpyAsync(D(o_vp[i]), s[i].vp, n3 * es, cudaMemcpyHostToDevice, stream));
        CU(cudaMemcpyAsync(D(o_rho[i]), s[i].rho, n3 * es, cudaMemcpyHostToDevice, stream));
        CU(cudaMemcpyAsync(D(o_obs[i]), s[i].data, (size_t)nrec[i] * cfg.nt * es, cudaMemcpyHostToDevice, stream));
        if (el) {
            CU(cudaMemcpyAsync(D(o_vs[i]), s[i].vs, n3 * es, cudaMemcpyHostToDevice, stream));
            CU(cudaMemcpyAsync(D(o_obsy[i]), s[i].data_vy, (size_t)nrec[i] * cfg.nt * es, cudaMemcpyHostToDevice, stream));
            CU(cudaMemcpyAsync(D(o_obsz[i]), s[i].data_vz, (size_t)nrec[i] * cfg.nt * es, cudaMemcpyHostToDevice, stream));
        }
        // misfit mask: a receiver counts when its map lies on the grid (lib/fwi.cpp:1500)
        std::vector<int> &valid = valids[i];
        valid.resize(nrec[i]);
        for (int t = 0; t < nrec[i]; t++) {
            const int *m = s[i].shot.gmap + 3 * t;
            valid[t] = (m[0] >= 0 && m[1] >= 0 && m[2] >= 0) ? 0 : -1;
        }
        CU(cudaMemcpyAsync(D(o_valid[i]), valid.data(), sizeof(int) * valid.size(), cudaMemcpyHostToDevice, stream));
    }
    for (int i = 0; i < ns && el; i++) {
        const Layout3D &F = fw->shots[i], &B = bw->shots[i];
        char *fa = (char *)fw->arena, *ba = (char *)bw->arena;
        const size_t fo = fw->origin_bytes(F), bo = bw->origin_bytes(B);
        auto fill = [&](auto *d, auto *r) {
            using T = typename std::remove_const<typename std::remove_pointer<decltype(d->rx)>::type>::type;
            for (int k = 0; k < 9; k++) {
                d->ws[k] = (const T *)(fa + F.f[k] + fo);
                d->wr[k] = (const T *)(ba + B.f[k] + bo);
            }
            d->rx = (const T *)fw->param_base(i, ME_RX);
            d->ry = (const T *)fw->param_base(i, ME_RY);
            d->rz = (const T *)fw->param_base(i, ME_RZ);
            d->vp = (const T *)D(o_vp[i]);
            d->vs = (const T *)D(o_vs[i]);
            d->rho = (const T *)D(o_rho[i]);
            d->g[0] = D(o_img[i]);
            d->g[1] = D(o_g1[i]);
            d->g[2] = D(o_g2[i]);
            d->nx = nx[i]; d->ny = ny[i]; d->nz = nz[i]; d->pitch = F.pitch; d->lpml = cfg.lpml; d->plane = F.plane;
            const size_t obs[3] = {o_obs[i], o_obsy[i], o_obsz[i]};
            for (int k = 0; k < 3; k++) {
                r->mod[k] = (const T *)(fa + F.tracesk[k]);
                r->obs[k] = (const T *)D(obs[k]);
                r->res[k] = (T *)(ba + B.wavk[k]);
            }
            r->nrec = nrec[i];
            r->nt = cfg.nt;
        };
        if (prec == PREC_F64) {
            Corr3DE<double> d{};
            Resid3E<double> r{};
            fill(&d, &r);
            std::memcpy(corr.data() + i * sizeof d, &d, sizeof d);
            std::memcpy(res.data() + i * sizeof r, &r, sizeof r);
        } else {
            Corr3DE<float> d{};
            Resid3E<float> r{};
            fill(&d, &r);
            std::memcpy(corr.data() + i * sizeof d, &d, sizeof d);
            std::memcpy(res.data() + i * sizeof r, &r, sizeof r);
        }
    }
    for (int i = 0; i < ns && fwi() && !el; i++) {
        const Layout3D &F = fw->shots[i], &B = bw->shots[i];
        char *fa = (char *)fw->arena, *ba = (char *)bw->arena;
        const size_t fo = fw->origin_bytes(F), bo = bw->origin_bytes(B);
        auto fill = [&](auto *d, auto *r) {
            using T = typename std::remove_const<typename std::remove_pointer<decltype(d->wsp)>::type>::type;
            d->wsp = (const T *)(fa + F.f[A3_P] + fo);
            d->wrx = (const T *)(ba + B.f[A3_VX] + bo);
            d->wry = (const T *)(ba + B.f[A3_VY] + bo);
            d->wrz = (const T *)(ba + B.f[A3_VZ] + bo);
            d->rx = (const T *)fw->param_base(i, M3_RX);
            d->ry = (const T *)fw->param_base(i, M3_RY);
            d->rz = (const T *)fw->param_base(i, M3_RZ);
            d->vp = (const T *)D(o_vp[i]);
            d->rho = (const T *)D(o_rho[i]);
            d->g0 = D(o_img[i]);
            d->g1 = D(o_g1[i]);
            d->nx = nx[i]; d->ny = ny[i]; d->nz = nz[i]; d->pitch = F.pitch; d->lpml = cfg.lpml; d->plane = F.plane;
            r->mod = (const T *)(fa + F.traces);
            r->obs = (const T *)D(o_obs[i]);
            r->res = (T *)(ba + B.wav);
            r->rec_pt = (const int *)D(o_valid[i]);
            if (o_work[i]) {
                r->work = (decltype(r->work))D(o_work[i]);
                r->tnorm = (decltype(r->tnorm))D(o_tnorm[i]);
            }
            r->nrec = nrec[i];
            r->nt = cfg.nt;
        };
        if (prec == PREC_F64) {
            Corr3DF<double> d{};
            Resid2D<double> r{};
            fill(&d, &r);
            std::memcpy(corr.data() + i * sizeof d, &d, sizeof d);
            std::memcpy(res.data() + i * sizeof r, &r, sizeof r);
        } else {
            Corr3DF<float> d{};
            Resid2D<float> r{};
            fill(&d, &r);
            std::memcpy(corr.data() + i * sizeof d, &d, sizeof d);
            std::memcpy(res.data() + i * sizeof r, &r, sizeof r);
        }
    }
    for (int i = 0; i < ns && !fwi(); i++) {
        const Layout3D &F = fw->shots[i], &B = bw->shots[i];
        if (prec == PREC_F64) {
            Corr3D<double> d{};
            d.wsp = (const double *)((char *)fw->arena + F.f[A3_P] + fw->origin_bytes(F));
            d.wrp = (const double *)((char *)bw->arena + B.f[A3_P] + bw->origin_bytes(B));
            d.img = D(o_img[i]);
            d.nx = nx[i]; d.ny = ny[i]; d.nz = nz[i]; d.pitch = F.pitch; d.lpml = cfg.lpml; d.plane = F.plane;
            std::memcpy(corr.data() + i * sizeof d, &d, sizeof d);
        } else {
            Corr3D<float> d{};
            d.wsp = (const float *)((char *)fw->arena + F.f[A3_P] + fw->origin_bytes(F));
            d.wrp = (const float *)((char *)bw->arena + B.f[A3_P] + bw->origin_bytes(B));
            d.img = D(o_img[i]);
            d.nx = nx[i]; d.ny = ny[i]; d.nz = nz[i]; d.pitch = F.pitch; d.lpml = cfg.lpml; d.plane = F.plane;
            std::memcpy(corr.data() + i * sizeof d, &d, sizeof d);
        }
    }
    CU(cudaMemcpyAsync(D(o_corr), corr.data(), corr.size(), cudaMemcpyHostToDevice, stream));
    CU(cudaMemcpyAsync(D(o_res), res.data(), res.size(), cudaMemcpyHostToDevice, stream));
    CU(cudaStreamSynchronize(stream));
    return RSGPU_OK;
}

rsgpu_status Adjoint3D::slot_io(bool save, int slot)
{
    if (slot < 0 || slot >= nslots) { set_error("checkpoint slot %d outside [0,%d)", slot, nslots); return RSGPU_ERR_REVOLVE; }
    char *sl = (char *)ckpt + (size_t)slot * slot_elems * ck_es;
    float *sc = (float *)D(o_scales) + (size_t)slot * segs.size();
    cudaError_t e = save ? launch_ckpt_save(prec, ck, (const CkptSeg *)D(o_segs), (int)segs.size(), seg_rows, sl, sc,
                                            (unsigned *)D(o_maxbits), stream)
                         : launch_ckpt_load(prec, ck, (const CkptSeg *)D(o_segs), (int)segs.size(), seg_rows, sl, sc, stream);
    if (e != cudaSuccess) { set_error("checkpoint %s: %s", save ? "save" : "restore", cudaGetErrorString(e)); return RSGPU_ERR_CUDA; }
    launches += (save && ck != CK_NATIVE) ? 2 : 1;
    ckpt_bytes += (long long)(slot_elems * ck_es);
    return RSGPU_OK;
}

rsgpu_status Adjoint3D::correlate()
{
    cudaError_t e = elastic() ? launch_corr_fwi_e3d(prec, acc, D(o_corr), nshots, nxmax, nymax, cfg.dx, cfg.dy, cfg.dz, stream)
                    : fwi()   ? launch_corr_fwi_a3d(prec, acc, D(o_corr), nshots, nxmax, nymax, cfg.dx, cfg.dy, cfg.dz, stream)
                              : launch_corr_rtm_a3d(prec, acc, D(o_corr), nshots, nxmax, nymax, nhx, nhy, nhz, stream);
    if (e != cudaSuccess) { set_error("correlation launch: %s", cudaGetErrorString(e)); return RSGPU_ERR_CUDA; }
    launches += 1;
    return RSGPU_OK;
}

// RtmAcoustic3D::run (lib/rtm.cpp:640-733): as the 2D FULL driver, the P interior
// saved after steps 0, snapinc, ... and correlated at the adjoint times t with
// (t - enddiff) % snapinc == 0 against snapshot (t - enddiff)/snapinc.
rsgpu_status Adjoint3D::run_full()
{
    const int nt = cfg.nt;
    const long long l0 = fw->launches + bw->launches;
    launches = 0;
    fw_steps = bw_steps = ckpt_bytes = 0;
    ran = false;
    ST(fw->reset());
    ST(bw->reset());
    const size_t gs = acc == ACC_F64 ? 8 : (size_t)es;
    for (int i = 0; i < nshots; i++)
        CU(cudaMemsetAsync(D(o_img[i]), 0, (size_t)nx[i] * ny[i] * nz[i] * nhx * nhy * nhz * gs, stream));
    ST(fw->run(0, 1));
    ST(slot_io(true, 0));
    for (int k = 1; k < snapnt; k++) {
        ST(fw->run((k - 1) * snapinc + 1, snapinc));
        ST(slot_io(true, k));
    }
    const int done = (snapnt - 1) * snapinc + 1;
    if (done < nt) ST(fw->run(done, nt - done));
    fw_steps = nt;
    auto aligned = [&](int k) { return ((nt - 1 - k) - enddiff) % snapinc == 0; };
    for (int k = 0; k < nt;) {
        int e = k;
        while (e < nt && !aligned(e)) e++;
        const int n = (e < nt ? e + 1 : nt) - k;
        ST(bw->run(k, n));
        bw_steps += n;
        k += n;
        if (e < nt) {
            ST(slot_io(false, ((nt - 1 - e) - enddiff) / snapinc));
            ST(correlate());
        }
    }
    launches += fw->launches + bw->launches - l0;
    CU(cudaStreamSynchronize(stream));
    ST(fw->check_device_error());
    ST(bw->check_device_error());
    ran = true;
    return RSGPU_OK;
}

rsgpu_status Adjoint3D::run()
{
    if (snapmethod == RSGPU_SNAP_FULL) return run_full();
    const int nt = cfg.nt;
    const long long l0 = fw->launches + bw->launches;
    launches = 0;
    fw_steps = bw_steps = ckpt_bytes = 0;
    ST(fw->reset());
    ST(bw->reset());
    const size_t gs = acc == ACC_F64 ? 8 : (size_t)es;
    for (int i = 0; i < nshots; i++) {
        CU(cudaMemsetAsync(D(o_img[i]), 0, (size_t)nx[i] * ny[i] * nz[i] * nhx * nhy * nhz * gs, stream));
        if (fwi()) CU(cudaMemsetAsync(D(o_g1[i]), 0, (size_t)nx[i] * ny[i] * nz[i] * gs, stream));
        if (elastic()) CU(cudaMemsetAsync(D(o_g2[i]), 0, (size_t)nx[i] * ny[i] * nz[i] * gs, stream));
    }
    if (fwi()) ST(fw->set_recording(true));
    RevolveSchedule rev(nt, ncheck);
    for (;;) {
        const int oldcapo = rev.capo();
        const int a = rev.next();
        const int capo = rev.capo();
        if (a == RSGPU_ADVANCE) {
            ST(fw->run(oldcapo, capo - oldcapo));
            fw_steps += capo - oldcapo;
        } else if (a == RSGPU_TAKESHOT) {
            ST(slot_io(true, rev.check()));
        } else if (a == RSGPU_RESTORE) {
            ST(slot_io(false, rev.check()));
        } else if (a == RSGPU_FIRSTURN) {
            ST(fw->run(capo, 1));
            fw_steps += 1;
            if (fwi()) {
                ST(fw->set_recording(false));
                cudaError_t e = elastic() ? launch_residual_e3d(prec, acc, D(o_res), nshots, (double *)D(o_misfit), stream)
                                : o_atab ? launch_residual_adaptive(prec, acc, misfit_type, D(o_res), nshots, nrec_max,
                                                                    cfg.nt, D(o_atab), (double *)D(o_misfit), stream,
                                                                    false)
                                : misfit_type == RSGPU_MISFIT_CORRELATION
                                    ? launch_residual_corr(prec, acc, D(o_res), nshots, nrec_max, (double *)D(o_misfit),
                                                           stream, false)
                                    : launch_residual(prec, acc, D(o_res), nshots, (double *)D(o_misfit),
                                                      (double *)D(o_rpart), stream);
                if (e != cudaSuccess) { set_error("residual launch: %s", cudaGetErrorString(e)); return RSGPU_ERR_CUDA; }
                launches += elastic() || misfit_type == RSGPU_MISFIT_CORRELATION ? 1 : 2;
            }
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
        cudaError_t e = launch_scale_grad_e3d(prec, acc, D(o_corr), nshots, nxmax, nymax, stream);
        if (e != cudaSuccess) { set_error("scaleGrad launch: %s", cudaGetErrorString(e)); return RSGPU_ERR_CUDA; }
        launches += 1;
    }
    launches += fw->launches + bw->launches - l0;
    CU(cudaStreamSynchronize(stream));
    ST(fw->check_device_error());
    ST(bw->check_device_error());
    ran = true;
    return RSGPU_OK;
}

rsgpu_status Adjoint3D::read(int ns, const rsgpu_adjoint_shot *s)
{
    if (!ran) { set_error("no run to read"); return RSGPU_ERR_STATE; }
    if (ns != nshots || !s) { set_error("read expects the %d shots of the batch", nshots); return RSGPU_ERR_ARG; }
    const size_t gs = acc == ACC_F64 ? 8 : (size_t)es;
    std::vector<unsigned char> tmp;
    // add a device array of the accumulator type into a host array of the element type
    auto add_from = [&](void *host, size_t o, size_t n) -> rsgpu_status {
        tmp.resize(n * gs);
        CU(cudaMemcpyAsync(tmp.data(), D(o), n * gs, cudaMemcpyDeviceToHost, stream));
        CU(cudaStreamSynchronize(stream));
        if (es == 8) {
            double *h = (double *)host;
            const double *t = (const double *)tmp.data();
            for (size_t k = 0; k < n; k++) h[k] += t[k];
        } else if (gs == 8) {
            float *h = (float *)host;
            const double *t = (const double *)tmp.data();
            for (size_t k = 0; k < n; k++) h[k] = (float)((double)h[k] + t[k]);
        } else {
            float *h = (float *)host;
            const float *t = (const float *)tmp.data();
            for (size_t k = 0; k < n; k++) h[k] += t[k];
        }
        return RSGPU_OK;
    };
    if (fwi()) {
        std::vector<double> mis(nshots, 0.0);
        CU(cudaMemcpyAsync(mis.data(), D(o_misfit), sizeof(double) * nshots, cudaMemcpyDeviceToHost, stream));
        CU(cudaStreamSynchronize(stream));
        for (int i = 0; i < nshots; i++) {
            const size_t n3 = (size_t)nx[i] * ny[i] * nz[i];
            if (s[i].vpgrad) ST(add_from(s[i].vpgrad, o_img[i], n3));
            if (elastic()) {
                if (s[i].vsgrad) ST(add_from(s[i].vsgrad, o_g1[i], n3));
                if (s[i].rhograd) ST(add_from(s[i].rhograd, o_g2[i], n3));
            } else if (s[i].rhograd) {
                ST(add_from(s[i].rhograd, o_g1[i], n3));
            }
            if (s[i].shot.rec_out) ST(fw->read_traces(i, s[i].shot.rec_out, 0));
            if (elastic() && s[i].datamod_vy) ST(fw->read_traces(i, s[i].datamod_vy, 1));
            if (elastic() && s[i].datamod_vz) ST(fw->read_traces(i, s[i].datamod_vz, 2));
            if (s[i].wavgrad) ST(bw->read_traces(i, s[i].wavgrad));
            void *res_out[3] = {s[i].datares, elastic() ? s[i].datares_vy : nullptr,
                                elastic() ? s[i].datares_vz : nullptr};
            for (int k = 0; k < 3; k++) {
                if (!res_out[k]) continue;
                const size_t n = (size_t)nrec[i] * cfg.nt;
                tmp.resize(n * es);
                CU(cudaMemcpyAsync(tmp.data(), (char *)bw->arena + bw->shots[i].wavk[k], n * es,
                                   cudaMemcpyDeviceToHost, stream));
                CU(cudaStreamSynchronize(stream));
                if (es == 8) { double *h = (double *)res_out[k]; const double *t = (const double *)tmp.data(); for (size_t j = 0; j < n; j++) h[j] += t[j]; }
                else { float *h = (float *)res_out[k]; const float *t = (const float *)tmp.data(); for (size_t j = 0; j < n; j++) h[j] += t[j]; }
            }
            if (s[i].misfit) {
                if (acc == ACC_REF && es == 4) *s[i].misfit = (double)(float)((float)*s[i].misfit + (float)mis[i]);
                else *s[i].misfit += mis[i];
            }
        }
        return RSGPU_OK;
    }
    for (int i = 0; i < nshots; i++) {
        if (!s[i].image) continue;
        const size_t n = (size_t)nx[i] * ny[i] * nz[i] * nhx * nhy * nhz;
        tmp.resize(n * gs);
        CU(cudaMemcpyAsync(tmp.data(), D(o_img[i]), n * gs, cudaMemcpyDeviceToHost, stream));
        CU(cudaStreamSynchronize(stream));
        if (es == 8) {
            double *o = (double *)s[i].image;
            const double *t = (const double *)tmp.data();
            for (size_t k = 0; k < n; k++) o[k] += t[k];
        } else if (gs == 8) {
            float *o = (float *)s[i].image;
            const double *t = (const double *)tmp.data();
            for (size_t k = 0; k < n; k++) o[k] = (float)((double)o[k] + t[k]);
        } else {
            float *o = (float *)s[i].image;
            const float *t = (const float *)tmp.data();
            for (size_t k = 0; k < n; k++) o[k] += t[k];
        }
    }
    return RSGPU_OK;
}

}  // namespace rsgpu
