// Host runtime of the 3D propagator: the batch plan behind rsgpu_modelling and
// rsgpu_plan_* for RSGPU_ACOUSTIC3D.
//
// One device arena holds, per shot, the pitched fields (P, Vx, Vy, Vz), the
// C-PML memory of the three face pairs, the trace buffer, the staggered
// parameters (Rx, Ry, Rz, L) and the wavelets; a second buffer holds the shot
// descriptors, the tile table (TX3 x TY3 column blocks x z-chunks of every shot),
// coefficient rows, C-PML tables and injection/recording plans.  Each time step
// is three launches (velocity, stress, inject/record), every launch covering all
// shots.
#include <algorithm>
#include <cstring>
#include <map>
#include <vector>

#include <cuda.h>
#include <cuda_runtime.h>

#include "rsgpu.h"
#include "rsgpu_3d.h"
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

static inline size_t rup3(size_t a, size_t b) { return (a + b - 1) / b * b; }

// Index of the work array that stands in for field slot k in the adjoint velocity
// step (WorkE3 order: Sxx, Syy, Szz, Syz, Sxz, Sxy), -1 for the other slots.
static int work_slot(int k)
{
    switch (k) {
    case E3_SXX: return 0;
    case E3_SYY: return 1;
    case E3_SZZ: return 2;
    case E3_SYZ: return 3;
    case E3_SXZ: return 4;
    case E3_SXY: return 5;
    default: return -1;
    }
}


Plan3D::~Plan3D()
{
    dev_free(arena, stream);
    dev_free(d_meta, stream);
    dev_free(d_work, stream);
    if (stream && stream != shared_stream) cudaStreamDestroy(stream);
}

rsgpu_status Plan3D::create(const rsgpu_config *c, int ns, const rsgpu_shot *s, const ShotSets *sets)
{
    if (!c || !s || ns < 1) { set_error("null config/shots or nshots < 1"); return RSGPU_ERR_ARG; }
    if (c->physics != RSGPU_ACOUSTIC3D && c->physics != RSGPU_ELASTIC3D) { set_error("Plan3D: physics %d is not 3D", c->physics); return RSGPU_ERR_UNSUPPORTED; }
    phys = c->physics == RSGPU_ELASTIC3D ? PHYS_E3D : PHYS_A3D;
    if (c->precision < 0 || c->precision > 2) { set_error("bad precision %d", c->precision); return RSGPU_ERR_ARG; }
    if (c->lpml < 1 || c->nt < 1 || !(c->dt > 0) || !(c->dx > 0) || !(c->dy > 0) || !(c->dz > 0)) {
        set_error("lpml, nt, dt, dx, dy, dz must be positive");
        return RSGPU_ERR_ARG;
    }
    const int order = std::min(std::max(c->order, 1), 8);
    for (int i = 0; i < ns; i++) {
        const rsgpu_shot &sh = s[i];
        if (sh.nx < 1 || sh.ny < 1 || sh.nz < 1) { set_error("shot %d: empty model window", i); return RSGPU_ERR_ARG; }
        if (sh.nx + 2 * c->lpml <= order || sh.ny + 2 * c->lpml <= order || sh.nz + 2 * c->lpml <= order) {
            set_error("shot %d: padded grid smaller than stencil", i);
            return RSGPU_ERR_ARG;
        }
        for (int k = 0; k < np3(); k++)
            if (!sh.model[k]) { set_error("shot %d: model parameter %d is null", i, k); return RSGPU_ERR_ARG; }
        if (sh.nsrc < 0 || sh.nrec < 0) { set_error("shot %d: negative trace count", i); return RSGPU_ERR_ARG; }
        if (sh.nsrc > 0 && (!sh.smap || !sh.sshift || !sh.wavelet)) { set_error("shot %d: source arrays missing", i); return RSGPU_ERR_ARG; }
        if (sh.nrec > 0 && (!sh.gmap || !sh.gshift)) { set_error("shot %d: receiver arrays missing", i); return RSGPU_ERR_ARG; }
        if (sh.src_field < RSGPU_PRESSURE || sh.src_field > RSGPU_VZ) { set_error("shot %d: bad source field", i); return RSGPU_ERR_ARG; }
        if (sh.nrec > 0 && (sh.rec_field < RSGPU_PRESSURE || sh.rec_field > RSGPU_VZ)) { set_error("shot %d: bad receiver field", i); return RSGPU_ERR_ARG; }
    }
    nsets = phys == PHYS_E3D ? MAXSETS : 1;
    // the effective trace sets of every shot
    std::vector<ShotSets> eff(ns);
    for (int i = 0; i < ns; i++) {
        ShotSets &e = eff[i];
        if (sets) {
            e = sets[i];
        } else {
            e.nsrc = 1;
            e.src[0] = {s[i].nsrc, s[i].smap, s[i].sshift, s[i].src_field, s[i].wavelet, nullptr, false};
            e.nrec = 1;
            e.rec[0] = {s[i].nrec, s[i].gmap, s[i].gshift, s[i].rec_field, nullptr, s[i].rec_factor, false};
        }
        if (e.nsrc < 0 || e.nrec < 0 || e.nsrc > nsets || e.nrec > nsets) {
            set_error("shot %d: %d source and %d receiver sets (at most %d)", i, e.nsrc, e.nrec, nsets);
            return RSGPU_ERR_ARG;
        }
        for (int k = 0; k < e.nsrc; k++) {
            const TraceSet &t = e.src[k];
            if (t.n < 0 || (t.n > 0 && (!t.map || !t.shift || !t.data)) || t.field < RSGPU_PRESSURE || t.field > RSGPU_VZ) {
                set_error("shot %d: source set %d is malformed", i, k);
                return RSGPU_ERR_ARG;
            }
        }
        for (int k = 0; k < e.nrec; k++) {
            const TraceSet &t = e.rec[k];
            if (t.n < 0 || (t.n > 0 && (!t.map || !t.shift)) || t.field < RSGPU_PRESSURE || t.field > RSGPU_VZ ||
                (t.at_point && phys != PHYS_E3D)) {
                set_error("shot %d: receiver set %d is malformed", i, k);
                return RSGPU_ERR_ARG;
            }
            if (phys == PHYS_E3D && t.n > 0 && t.field == RSGPU_PRESSURE && !t.at_point && !t.factor) {
                set_error("shot %d: elastic 3D pressure receivers need rec_factor, (3*rho*vp^2 - 4*rho*vs^2)/3 at "
                          "each receiver's map point (WavesElastic3D::recordData, lib/waves.cpp:4285)", i);
                return RSGPU_ERR_ARG;
            }
        }
    }
    if (share_params && (share_params->nshots != ns || share_params->phys != phys || share_params->prec != c->precision)) {
        set_error("plans sharing parameters must hold the same shots");
        return RSGPU_ERR_ARG;
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) {
        cudaGetLastError();
        set_error("no CUDA device");
        return RSGPU_ERR_NODEVICE;
    }
    cfg = *c;
    cfg.order = order;
    prec = c->precision;
    nshots = ns;
    es = prec == PREC_F64 ? 8 : 4;
    zc = c->zchunk > 0 ? c->zchunk : 64;      // planes per z-chunk
    if (shared_stream) stream = shared_stream;
    else CU(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    const int lp = cfg.lpml;

    shots.resize(ns);
    size_t off = 0;
    auto take = [&](size_t bytes) { size_t o = off; off = rup3(off + std::max<size_t>(bytes, 1), 256); return o; };
    for (int i = 0; i < ns; i++) {
        Layout3D &L = shots[i];
        L.nxp = s[i].nx + 2 * lp; L.nyp = s[i].ny + 2 * lp; L.nzp = s[i].nz + 2 * lp;
        L.pitch = (int)rup3(GUARD + rup3(L.nxp, TX3) + GUARD, 32);
        L.rows = GUARD + (int)rup3(L.nyp, TY3) + GUARD;
        L.planes = GUARD + L.nzp + GUARD + 2;
        L.plane = (long long)L.pitch * L.rows;
        if ((long long)L.plane * L.planes > 0x7fffffffLL) {
            set_error("shot %d: padded 3D arrays of %lld cells exceed the kernels' 32-bit offsets", i,
                      (long long)L.plane * L.planes);
            return RSGPU_ERR_ARG;
        }
        const size_t fbytes = (size_t)L.plane * L.planes * es;
        for (int k = 0; k < nf3(); k++) L.f[k] = take(fbytes);
        for (int k = 0; k < npsi3(); k++) {
            L.psix[k] = take((size_t)L.nzp * L.nyp * 2 * lp * es);
            L.psiy[k] = take((size_t)L.nzp * 2 * lp * L.nxp * es);
            L.psiz[k] = take((size_t)2 * lp * L.nyp * L.nxp * es);
        }
        L.psi_end = off;
        const ShotSets &e = eff[i];
        L.nsrcsets = e.nsrc;
        L.nrecsets = e.nrec;
        for (int k = 0; k < e.nrec; k++) {
            L.nrecs[k] = e.rec[k].n;
            L.tracesk[k] = take((size_t)std::max(1, e.rec[k].n) * cfg.nt * es);
        }
        L.state_end = off;
        if (!share_params)
            for (int k = 0; k < np3(); k++) L.m[k] = take(fbytes);
        for (int k = 0; k < e.nsrc; k++) {
            L.nsrcs[k] = e.src[k].n;
            L.wavk[k] = take((size_t)std::max(1, e.src[k].n) * cfg.nt * es);
        }
        for (int k = 0; k < e.nrec; k++) L.rfack[k] = take((size_t)std::max(1, e.rec[k].n) * es);
        L.nrec = L.nrecs[0];
        L.nsrc = L.nsrcs[0];
        L.traces = L.tracesk[0];
        L.wav = L.wavk[0];
        L.rfac = L.rfack[0];
    }
    // injection / recording plans per (shot, set) (reference loop order: trace, z, y, x corner)
    const int nps = ns * nsets;
    std::vector<std::vector<long long>> inj_pt(nps), rec_pt(nps);
    std::vector<std::vector<int>> inj_start(nps), inj_tr(nps);
    std::vector<std::vector<double>> inj_w(nps), rec_w(nps);
    auto shift_of = [&](const void *p, int k) -> double {
        return prec == PREC_F64 ? ((const double *)p)[k] : (double)((const float *)p)[k];
    };
    auto tri = [&](double sft, double *w) {
        if (prec == PREC_F64) { w[0] = 1 - sft; w[1] = sft; }
        else { w[0] = (float)(1 - (float)sft); w[1] = (float)sft; }
    };
    for (int i = 0; i < ns; i++) {
        const Layout3D &L = shots[i];
        const ShotSets &e = eff[i];
        for (int k = 0; k < e.nsrc; k++) {
            const TraceSet &t = e.src[k];
            const int j = i * nsets + k;
            struct W3 { double v[3]; };
            std::map<long long, std::vector<std::pair<int, W3>>> per_pt;
            std::vector<long long> order_pts;
            for (int tr = 0; tr < t.n; tr++) {
                const int mx = t.map[3 * tr], my = t.map[3 * tr + 1], mz = t.map[3 * tr + 2];
                if (mx < 0 || my < 0 || mz < 0) continue;
                double xt[2], yt[2], zt[2];
                tri(shift_of(t.shift, 3 * tr), xt);
                tri(shift_of(t.shift, 3 * tr + 1), yt);
                tri(shift_of(t.shift, 3 * tr + 2), zt);
                for (int i1 = 0; i1 < 2; i1++)
                    for (int i2 = 0; i2 < 2; i2++)
                        for (int i3 = 0; i3 < 2; i3++) {
                            const int ix = lp + mx + i3, iy = lp + my + i2, iz = lp + mz + i1;
                            if (ix >= L.nxp || iy >= L.nyp || iz >= L.nzp) {
                                set_error("shot %d: source %d of set %d maps outside the grid", i, tr, k);
                                return RSGPU_ERR_ARG;
                            }
                            const long long p = iz * L.plane + (long long)iy * L.pitch + ix;
                            if (!per_pt.count(p)) order_pts.push_back(p);
                            per_pt[p].push_back({tr, W3{{xt[i3], yt[i2], zt[i1]}}});
                        }
            }
            inj_start[j].push_back(0);
            for (long long p : order_pts) {
                inj_pt[j].push_back(p);
                for (auto &cw : per_pt[p]) {
                    inj_tr[j].push_back(cw.first);
                    for (int q = 0; q < 3; q++) inj_w[j].push_back(cw.second.v[q]);
                }
                inj_start[j].push_back((int)inj_tr[j].size());
            }
        }
        for (int k = 0; k < e.nrec; k++) {
            const TraceSet &t = e.rec[k];
            const int j = i * nsets + k;
            for (int tr = 0; tr < t.n; tr++) {
                const int mx = t.map[3 * tr], my = t.map[3 * tr + 1], mz = t.map[3 * tr + 2];
                if (mx < 0 || my < 0 || mz < 0) {
                    rec_pt[j].push_back(-1);
                    for (int q = 0; q < 6; q++) rec_w[j].push_back(0);
                    continue;
                }
                if (lp + mx + 1 >= L.nxp || lp + my + 1 >= L.nyp || lp + mz + 1 >= L.nzp) {
                    set_error("shot %d: receiver %d of set %d maps outside the grid", i, tr, k);
                    return RSGPU_ERR_ARG;
                }
                rec_pt[j].push_back((long long)(lp + mz) * L.plane + (long long)(lp + my) * L.pitch + lp + mx);
                double w[2];
                for (int q = 0; q < 3; q++) {
                    tri(shift_of(t.shift, 3 * tr + q), w);
                    rec_w[j].push_back(w[0]);
                    rec_w[j].push_back(w[1]);
                }
            }
        }
    }
    std::vector<SetTables> tabs(nps);
    for (int j = 0; j < nps; j++) {
        SetTables &t = tabs[j];
        t.ip = take(inj_pt[j].size() * 8);
        t.is = take(std::max<size_t>(1, inj_start[j].size()) * 4);
        t.it = take(inj_tr[j].size() * 4);
        t.iw = take(inj_w[j].size() * es);
        t.rp = take(rec_pt[j].size() * 8);
        t.rw = take(rec_w[j].size() * es);
        t.ninj = (int)inj_pt[j].size();
        t.nrec = (int)rec_pt[j].size();
    }
    const size_t o_pml = take((size_t)12 * lp * es);
    rec_pt_offsets.assign(nps, 0);
    for (int j = 0; j < nps; j++) rec_pt_offsets[j] = tabs[j].rp;
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
    std::vector<unsigned char> hb;
    auto put_real = [&](size_t o, const std::vector<double> &v) -> rsgpu_status {
        if (v.empty()) return RSGPU_OK;
        hb.resize(v.size() * es);
        for (size_t k = 0; k < v.size(); k++) {
            if (es == 8) ((double *)hb.data())[k] = v[k];
            else ((float *)hb.data())[k] = (float)v[k];
        }
        CU(cudaMemcpy(A + o, hb.data(), hb.size(), cudaMemcpyHostToDevice));
        return RSGPU_OK;
    };
    auto put_raw = [&](size_t o, const void *p, size_t bytes) -> rsgpu_status {
        if (bytes) CU(cudaMemcpy(A + o, p, bytes, cudaMemcpyHostToDevice));
        return RSGPU_OK;
    };
    rsgpu_status st;
    for (int i = 0; i < ns; i++) {
        const Layout3D &L = shots[i];
        const ShotSets &e = eff[i];
        for (int k = 0; k < np3() && !share_params; k++) {
            cudaMemcpy3DParms p = {};
            p.srcPtr = make_cudaPitchedPtr(const_cast<void *>(s[i].model[k]), (size_t)L.nxp * es, L.nxp, L.nyp);
            p.dstPtr = make_cudaPitchedPtr(A + L.m[k] + origin_bytes(L), (size_t)L.pitch * es, L.pitch, L.rows);
            p.extent = make_cudaExtent((size_t)L.nxp * es, L.nyp, L.nzp);
            p.kind = cudaMemcpyHostToDevice;
            CU(cudaMemcpy3DAsync(&p, stream));
        }
        for (int k = 0; k < e.nsrc; k++)
            if (e.src[k].n > 0)
                CU(cudaMemcpyAsync(A + L.wavk[k], e.src[k].data, (size_t)e.src[k].n * cfg.nt * es,
                                   cudaMemcpyHostToDevice, stream));
        for (int k = 0; k < nsets; k++) {
            const int j = i * nsets + k;
            const SetTables &t = tabs[j];
            if ((st = put_raw(t.ip, inj_pt[j].data(), inj_pt[j].size() * 8)) != RSGPU_OK) return st;
            if ((st = put_raw(t.is, inj_start[j].data(), inj_start[j].size() * 4)) != RSGPU_OK) return st;
            if ((st = put_raw(t.it, inj_tr[j].data(), inj_tr[j].size() * 4)) != RSGPU_OK) return st;
            if ((st = put_real(t.iw, inj_w[j])) != RSGPU_OK) return st;
            if ((st = put_raw(t.rp, rec_pt[j].data(), rec_pt[j].size() * 8)) != RSGPU_OK) return st;
            if ((st = put_real(t.rw, rec_w[j])) != RSGPU_OK) return st;
        }
        for (int k = 0; k < e.nrec; k++)
            if (e.rec[k].factor && e.rec[k].n > 0) {
                std::vector<double> fac(e.rec[k].n);
                for (int t = 0; t < e.rec[k].n; t++) fac[t] = shift_of(e.rec[k].factor, t);
                if ((st = put_real(L.rfack[k], fac)) != RSGPU_OK) return st;
            }
    }
    {
        std::vector<unsigned char> tab((size_t)12 * lp * es);
        if (c->pml) std::memcpy(tab.data(), c->pml, tab.size());
        else pml_tables_host(lp, cfg.dt, prec, tab.data());
        if ((st = put_raw(o_pml, tab.data(), tab.size())) != RSGPU_OK) return st;
    }
    d_pml = A + o_pml;

    // tiles: column blocks x z-chunks of every shot
    std::vector<Tile3D> tiles;
    for (int i = 0; i < ns; i++) {
        const Layout3D &L = shots[i];
        for (int z0 = 0; z0 < L.nzp; z0 += zc)
            for (int y0 = 0; y0 < L.nyp; y0 += TY3)
                for (int x0 = 0; x0 < L.nxp; x0 += TX3) tiles.push_back({i, x0, y0, z0});
    }
    ntiles = (int)tiles.size();
    std::vector<unsigned char> cx, cy;
    coef_table_host(prec, cfg.dx, cfg.dy, cx);    // rows for dx then dy
    coef_table_host(prec, cfg.dz, cfg.dz, cy);    // rows for dz (first half)
    const size_t half = cx.size() / 2;
    std::vector<unsigned char> coefs(3 * half);
    std::memcpy(coefs.data(), cx.data(), 2 * half);
    std::memcpy(coefs.data() + 2 * half, cy.data(), half);
    const size_t shot_bytes = prec == PREC_F64 ? sizeof(Shot3D<double>) : sizeof(Shot3D<float>);
    const size_t ir_bytes = prec == PREC_F64 ? sizeof(InjRec3<double>) : sizeof(InjRec3<float>);
    const size_t m_shots = 0, m_ir = rup3(ns * shot_bytes, 256), m_tiles = rup3(m_ir + (size_t)nps * ir_bytes, 256);
    const size_t m_coef = rup3(m_tiles + tiles.size() * sizeof(Tile3D), 256);
    // fast mode: the tensor maps of the TMA-staged kernels
    const bool tma = prec == PREC_F32_FAST;
    const int nmap = phys == PHYS_E3D ? NMAP_E3 : NMAP_A3;
    const size_t m_maps = rup3(m_coef + coefs.size(), 256);
    // adjoint velocity through work arrays: a second set of shot descriptors and maps
    const bool wpass = tma && adjoint_steps && phys == PHYS_E3D;
    const size_t m_maps_w = rup3(m_maps + (tma ? (size_t)ns * nmap * sizeof(CUtensorMap) : 0), 256);
    const size_t m_shots_w = rup3(m_maps_w + (wpass ? (size_t)ns * NMAP_E3 * sizeof(CUtensorMap) : 0), 256);
    const size_t m_wdesc = rup3(m_shots_w + (wpass ? ns * shot_bytes : 0), 256);
    const size_t m_gate = rup3(m_wdesc + (wpass ? ns * sizeof(WorkE3) : 0), 256);
    const size_t m_end = m_gate + 256;
    std::vector<size_t> woff(ns, 0);
    if (wpass) {
        size_t wb = 0;
        for (int i = 0; i < ns; i++) {
            woff[i] = wb;
            wb = rup3(wb + 6 * (size_t)shots[i].plane * shots[i].planes * es, 256);
        }
        CU(dev_alloc(&d_work, wb, stream));
        CU(cudaMemsetAsync(d_work, 0, wb, stream));
    }
    CU(dev_alloc(&d_meta, m_end, stream));
    d_gate = reinterpret_cast<int *>((char *)d_meta + m_gate);
    d_err = d_gate + 1;
    std::vector<unsigned char> meta(m_end, 0);
    reinterpret_cast<int *>(meta.data() + m_gate)[0] = 1;   // recording on
    if (tma) {
        struct Spec { int slot; bool param; int boxw, boxh; };
        // VM_* then SM_* (rsgpu_3d.h)
        // acoustic: AM_* (rsgpu_3d.h)
        const Spec spec_a[NMAP_A3] = {
            {A3_P, false, WX3, HY3}, {A3_VX, false, TX3, TY3}, {A3_VY, false, TX3, TY3}, {A3_VZ, false, TX3, TY3},
            {M3_RX, true, TX3, TY3}, {M3_RY, true, TX3, TY3}, {M3_RZ, true, TX3, TY3},
            {A3_VX, false, WX3, TY3}, {A3_VY, false, TX3, HY3}, {A3_P, false, TX3, TY3}, {M3_L, true, TX3, TY3}};
        const Spec spec_e[NMAP_E3] = {
            {E3_SXX, false, WX3, TY3}, {E3_SXZ, false, WX3, TY3}, {E3_SXY, false, WX3, HY3},
            {E3_SYY, false, TX3, HY3}, {E3_SYZ, false, TX3, HY3},
            {E3_VX, false, TX3, TY3}, {E3_VY, false, TX3, TY3}, {E3_VZ, false, TX3, TY3},
            {ME_RX, true, TX3, TY3}, {ME_RY, true, TX3, TY3}, {ME_RZ, true, TX3, TY3},
            {E3_VX, false, WX3, HY3}, {E3_VY, false, WX3, HY3}, {E3_VZ, false, WX3, HY3},
            {E3_SXX, false, TX3, TY3}, {E3_SYY, false, TX3, TY3}, {E3_SZZ, false, TX3, TY3},
            {E3_SYZ, false, TX3, TY3}, {E3_SXZ, false, TX3, TY3}, {E3_SXY, false, TX3, TY3},
            {ME_L, true, TX3, TY3}, {ME_L2M, true, TX3, TY3}, {ME_MYZ, true, TX3, TY3},
            {ME_MXZ, true, TX3, TY3}, {ME_MXY, true, TX3, TY3}};
        const Spec *spec = phys == PHYS_E3D ? spec_e : spec_a;
        for (int i = 0; i < ns; i++) {
            const Layout3D &L = shots[i];
            for (int k = 0; k < nmap; k++) {
                const Spec &q = spec[k];
                // 2D map over the whole allocation: pitch x (rows * planes)
                void *base = q.param ? (void *)(param_base(i, q.slot) - origin_bytes(L)) : (void *)(A + L.f[q.slot]);
                void *m = meta.data() + m_maps + ((size_t)i * nmap + k) * sizeof(CUtensorMap);
                if (!encode_field_map_host(m, base, prec, L.pitch, L.rows * L.planes, q.boxw, q.boxh)) {
                    set_error("cuTensorMapEncodeTiled failed for map %d of shot %d", k, i);
                    return RSGPU_ERR_CUDA;
                }
                if (!wpass) continue;
                // the same map on the work array that stands in for a stress slot
                void *mw = meta.data() + m_maps_w + ((size_t)i * NMAP_E3 + k) * sizeof(CUtensorMap);
                const int ws = work_slot(q.param ? -1 : q.slot);
                void *wbase = ws < 0 ? base : (void *)((char *)d_work + woff[i] + (size_t)ws * L.plane * L.planes * es);
                if (!encode_field_map_host(mw, wbase, prec, L.pitch, L.rows * L.planes, q.boxw, q.boxh)) {
                    set_error("cuTensorMapEncodeTiled failed for work map %d of shot %d", k, i);
                    return RSGPU_ERR_CUDA;
                }
            }
        }
    }
    for (int i = 0; i < ns && wpass; i++) {
        const Layout3D &L = shots[i];
        const size_t fb = (size_t)L.plane * L.planes * es, org = origin_bytes(L);
        char *W = (char *)d_work + woff[i];
        // descriptors: the stress slots point at the work arrays
        Shot3D<float> d{};
        fill_shot<float>(reinterpret_cast<unsigned char *>(&d), i);
        for (int k = E3_SXX; k <= E3_SXY; k++) d.f[k] = (float *)(W + (size_t)work_slot(k) * fb + org);
        std::memcpy(meta.data() + m_shots_w + i * shot_bytes, &d, sizeof d);
        WorkE3 w{};
        const int sl[6] = {E3_SXX, E3_SYY, E3_SZZ, E3_SYZ, E3_SXZ, E3_SXY};
        for (int k = 0; k < 6; k++) {
            w.s[k] = (const float *)((char *)arena + L.f[sl[k]]);
            w.w[k] = (float *)(W + (size_t)k * fb);
        }
        auto pb = [&](int k) { return (const float *)(param_base(i, k) - org); };
        w.l = pb(ME_L); w.l2m = pb(ME_L2M); w.myz = pb(ME_MYZ); w.mxz = pb(ME_MXZ); w.mxy = pb(ME_MXY);
        w.n = (long long)L.plane * L.planes;
        std::memcpy(meta.data() + m_wdesc + i * sizeof(WorkE3), &w, sizeof w);
    }
    for (int i = 0; i < ns; i++) {
        const ShotSets &e = eff[i];
        if (prec == PREC_F64) fill_shot<double>(meta.data() + m_shots + i * shot_bytes, i);
        else fill_shot<float>(meta.data() + m_shots + i * shot_bytes, i);
        for (int k = 0; k < nsets; k++) {
            const TraceSet none{};
            const TraceSet &src = k < e.nsrc ? e.src[k] : none, &rec = k < e.nrec ? e.rec[k] : none;
            unsigned char *irp = meta.data() + m_ir + (size_t)(i * nsets + k) * ir_bytes;
            if (prec == PREC_F64) fill_set<double>(irp, i, k, src, rec, tabs[i * nsets + k]);
            else fill_set<float>(irp, i, k, src, rec, tabs[i * nsets + k]);
        }
    }
    std::memcpy(meta.data() + m_tiles, tiles.data(), tiles.size() * sizeof(Tile3D));
    std::memcpy(meta.data() + m_coef, coefs.data(), coefs.size());
    h_coefs = coefs;
    CU(cudaMemcpy(d_meta, meta.data(), m_end, cudaMemcpyHostToDevice));
    d_shots = (char *)d_meta + m_shots;
    d_injrec = (char *)d_meta + m_ir;
    d_tiles = (char *)d_meta + m_tiles;
    d_coefs = (char *)d_meta + m_coef;
    d_maps = tma ? (char *)d_meta + m_maps : nullptr;
    d_maps_w = wpass ? (char *)d_meta + m_maps_w : nullptr;
    d_shots_w = wpass ? (char *)d_meta + m_shots_w : nullptr;
    d_wdesc = wpass ? (char *)d_meta + m_wdesc : nullptr;
    CU(cudaStreamSynchronize(stream));
    return RSGPU_OK;
}

size_t Plan3D::origin_bytes(const Layout3D &L) const
{
    return ((size_t)GUARD * L.plane + (size_t)GUARD * L.pitch + GUARD) * es;
}

const char *Plan3D::param_base(int i, int k) const
{
    const Plan3D &o = share_params ? *share_params : *this;
    return (const char *)o.arena + o.shots[i].m[k] + o.origin_bytes(o.shots[i]);
}

template <typename T>
void Plan3D::fill_shot(unsigned char *sd, int i)
{
    char *A = (char *)arena;
    const Layout3D &L = shots[i];
    const size_t org = origin_bytes(L);
    Shot3D<T> d{};
    d.nxp = L.nxp; d.nyp = L.nyp; d.nzp = L.nzp; d.pitch = L.pitch; d.rows = L.rows;
    d.lpml = cfg.lpml; d.fs = cfg.fs; d.plane = L.plane;
    for (int k = 0; k < nf3(); k++) d.f[k] = (T *)(A + L.f[k] + org);
    for (int k = 0; k < np3(); k++) d.m[k] = (const T *)param_base(i, k);
    for (int k = 0; k < npsi3(); k++) {
        d.psix[k] = (T *)(A + L.psix[k]);
        d.psiy[k] = (T *)(A + L.psiy[k]);
        d.psiz[k] = (T *)(A + L.psiz[k]);
    }
    std::memcpy(sd, &d, sizeof d);
}

template <typename T>
void Plan3D::fill_set(unsigned char *irp, int i, int k, const TraceSet &src, const TraceSet &rec, const SetTables &t)
{
    char *A = (char *)arena;
    const Layout3D &L = shots[i];
    InjRec3<T> r{};
    r.ninj = t.ninj;
    r.kind_inj = t.ninj > 0 ? INJ3_P + src.field : INJ3_NONE;    // PRESSURE, VX, VY, VZ -> 1..4
    r.inj_pt = (const long long *)(A + t.ip);
    r.inj_start = (const int *)(A + t.is);
    r.inj_trace = (const int *)(A + t.it);
    r.inj_w = (const T *)(A + t.iw);
    r.wav = (const T *)(A + (k < L.nsrcsets ? L.wavk[k] : L.wavk[0]));
    r.nrec = t.nrec;
    r.kind_rec = t.nrec > 0 ? (rec.at_point ? REC3_WG_P : REC3_P) + rec.field : REC3_NONE;
    r.rec_pt = (const long long *)(A + t.rp);
    r.rec_w = (const T *)(A + t.rw);
    r.rec_out = (T *)(A + (k < L.nrecsets ? L.tracesk[k] : L.tracesk[0]));
    r.nt = cfg.nt;
    r.rev = reverse_time ? 1 : 0;
    r.rec_gate = gated_recording ? d_gate : nullptr;
    r.rec_factor = (const T *)(A + (k < L.nrecsets ? L.rfack[k] : L.rfack[0]));
    std::memcpy(irp, &r, sizeof r);
}

template <typename T>
static void make_args3(void *out, const Plan3D &p)
{
    Step3DArgs<T> a{};
    a.shots = (const Shot3D<T> *)p.d_shots;
    a.tiles = (const Tile3D *)p.d_tiles;
    a.ntiles = p.ntiles;
    a.order = p.cfg.order;
    a.zc = p.zc;
    a.lpml = p.cfg.lpml;
    a.dt = (T)p.cfg.dt; a.dx = (T)p.cfg.dx; a.dy = (T)p.cfg.dy; a.dz = (T)p.cfg.dz;
    a.rdx = (T)1 / a.dx; a.rdy = (T)1 / a.dy; a.rdz = (T)1 / a.dz;
    a.pml = (const T *)p.d_pml;
    a.maps = p.d_maps;
    a.err = p.d_err;
    const CoefSet3<T> &cs = *reinterpret_cast<const CoefSet3<T> *>(p.h_coefs.data());
    for (int k = 0; k < NCOEF; k++) {
        const T c[3] = {cs.cx[a.order * CROW3 + k], cs.cy[a.order * CROW3 + k], cs.cz[a.order * CROW3 + k]};
        for (int ax = 0; ax < 3; ax++) a.cf[ax][k] = a.cf2[ax][k][0] = a.cf2[ax][k][1] = c[ax];
    }
    std::memcpy(out, &a, sizeof a);
}

rsgpu_status Plan3D::reset()
{
    for (const auto &L : shots) CU(cudaMemsetAsync((char *)arena + L.f[0], 0, L.state_end - L.f[0], stream));
    return RSGPU_OK;
}

rsgpu_status Plan3D::step(int it)
{
    alignas(16) unsigned char args[sizeof(Step3DArgs<double>)];
    if (prec == PREC_F64) make_args3<double>(args, *this);
    else make_args3<float>(args, *this);
    cudaError_t e;
    if (phys == PHYS_E3D && d_wdesc) {
        // adjoint velocity: work arrays, then the forward TMA velocity kernel on them
        alignas(16) unsigned char wargs[sizeof(Step3DArgs<double>)];
        std::memcpy(wargs, args, sizeof wargs);
        Step3DArgs<float> &wa = *reinterpret_cast<Step3DArgs<float> *>(wargs);
        wa.shots = (const Shot3D<float> *)d_shots_w;
        wa.maps = d_maps_w;
        if ((e = launch_work_e3d(d_wdesc, nshots, stream)) != cudaSuccess) goto fail;
        if ((e = launch_step_e3d(prec, 0, 0, wargs, d_coefs, ntiles, stream)) != cudaSuccess) goto fail;
        if ((e = launch_step_e3d(prec, 1, 1, args, d_coefs, ntiles, stream)) != cudaSuccess) goto fail;
        if ((e = launch_injrec_e3d(prec, d_shots, d_injrec, nshots, nsets, cfg.dt, it, stream)) != cudaSuccess) goto fail;
        launches += 4;
        return RSGPU_OK;
    }
    if (phys == PHYS_E3D) {
        if ((e = launch_step_e3d(prec, 0, adjoint_steps, args, d_coefs, ntiles, stream)) != cudaSuccess) goto fail;
        if ((e = launch_step_e3d(prec, 1, adjoint_steps, args, d_coefs, ntiles, stream)) != cudaSuccess) goto fail;
        if ((e = launch_injrec_e3d(prec, d_shots, d_injrec, nshots, nsets, cfg.dt, it, stream)) != cudaSuccess) goto fail;
        launches += 3;
        return RSGPU_OK;
    }
    if ((e = launch_step_3d(prec, PHYS_A3D, 0, args, d_coefs, ntiles, stream)) != cudaSuccess) goto fail;
    if ((e = launch_step_3d(prec, PHYS_A3D, 1, args, d_coefs, ntiles, stream)) != cudaSuccess) goto fail;
    if ((e = launch_injrec_3d(prec, d_shots, d_injrec, nshots, cfg.dt, it, stream)) != cudaSuccess) goto fail;
    launches += 3;
    return RSGPU_OK;
fail:
    set_error("3D kernel launch failed: %s", cudaGetErrorString(e));
    return RSGPU_ERR_CUDA;
}

// Device-side error word (a bounded wait that gave up); read after a sync.
rsgpu_status Plan3D::check_device_error()
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

rsgpu_status Plan3D::set_recording(bool on)
{
    if (!gated_recording) { set_error("plan was created without gated recording"); return RSGPU_ERR_STATE; }
    CU(cudaMemsetAsync(d_gate, on ? 1 : 0, sizeof(int), stream));
    return RSGPU_OK;
}

rsgpu_status Plan3D::inject_record_only(int it)
{
    if (it < 0 || it >= cfg.nt) { set_error("step %d outside [0,%d)", it, cfg.nt); return RSGPU_ERR_ARG; }
    cudaError_t e = phys == PHYS_E3D ? launch_injrec_e3d(prec, d_shots, d_injrec, nshots, nsets, cfg.dt, it, stream)
                                     : launch_injrec_3d(prec, d_shots, d_injrec, nshots, cfg.dt, it, stream);
    if (e != cudaSuccess) { set_error("3D kernel launch failed: %s", cudaGetErrorString(e)); return RSGPU_ERR_CUDA; }
    launches += 1;
    return RSGPU_OK;
}

rsgpu_status Plan3D::run(int it0, int nsteps)
{
    if (it0 < 0 || nsteps < 0 || it0 + nsteps > cfg.nt) { set_error("step range [%d,%d) outside [0,%d)", it0, it0 + nsteps, cfg.nt); return RSGPU_ERR_ARG; }
    for (int k = 0; k < nsteps; k++) {
        rsgpu_status st = step(it0 + k);
        if (st != RSGPU_OK) return st;
    }
    return RSGPU_OK;
}

rsgpu_status Plan3D::read_traces(int shot, void *host_out, int set)
{
    if (shot < 0 || shot >= nshots) { set_error("bad shot %d", shot); return RSGPU_ERR_ARG; }
    const Layout3D &L = shots[shot];
    if (set < 0 || set >= std::max(1, L.nrecsets)) { set_error("bad receiver set %d", set); return RSGPU_ERR_ARG; }
    if (set >= L.nrecsets || L.nrecs[set] == 0) return RSGPU_OK;
    const size_t n = (size_t)L.nrecs[set] * cfg.nt;
    std::vector<unsigned char> tmp(n * es);
    CU(cudaMemcpyAsync(tmp.data(), (char *)arena + L.tracesk[set], n * es, cudaMemcpyDeviceToHost, stream));
    CU(cudaStreamSynchronize(stream));
    if (rsgpu_status st = check_device_error()) return st;
    if (es == 8) { double *o = (double *)host_out; const double *t = (const double *)tmp.data(); for (size_t k = 0; k < n; k++) o[k] += t[k]; }
    else { float *o = (float *)host_out; const float *t = (const float *)tmp.data(); for (size_t k = 0; k < n; k++) o[k] += t[k]; }
    return RSGPU_OK;
}

rsgpu_status Plan3D::read_field(int shot, int field, void *host_out)
{
    if (shot < 0 || shot >= nshots) { set_error("bad shot %d", shot); return RSGPU_ERR_ARG; }
    // acoustic: PRESSURE, VX, VY, VZ = slots 0..3; elastic: VX..SXY (codes 1..9) = slots 0..8
    const int slot = phys == PHYS_E3D ? field - 1 : field;
    if (slot < 0 || slot >= nf3()) { set_error("field %d not held by this 3D physics", field); return RSGPU_ERR_ARG; }
    const Layout3D &L = shots[shot];
    cudaMemcpy3DParms p = {};
    p.srcPtr = make_cudaPitchedPtr((char *)arena + L.f[slot] + origin_bytes(L), (size_t)L.pitch * es, L.pitch, L.rows);
    p.dstPtr = make_cudaPitchedPtr(host_out, (size_t)L.nxp * es, L.nxp, L.nyp);
    p.extent = make_cudaExtent((size_t)L.nxp * es, L.nyp, L.nzp);
    p.kind = cudaMemcpyDeviceToHost;
    CU(cudaMemcpy3DAsync(&p, stream));
    CU(cudaStreamSynchronize(stream));
    return RSGPU_OK;
}

}  // namespace rsgpu
