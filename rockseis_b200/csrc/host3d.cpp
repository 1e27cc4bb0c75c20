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

Plan3D::~Plan3D()
{
    if (arena) cudaFree(arena);
    if (d_meta) cudaFree(d_meta);
    if (stream && stream != shared_stream) cudaStreamDestroy(stream);
}

rsgpu_status Plan3D::create(const rsgpu_config *c, int ns, const rsgpu_shot *s)
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
        if (phys == PHYS_E3D && sh.nrec > 0 && sh.rec_field == RSGPU_PRESSURE && !sh.rec_factor) {
            set_error("shot %d: elastic 3D pressure receivers need rec_factor, (3*rho*vp^2 - 4*rho*vs^2)/3 at each "
                      "receiver's map point (WavesElastic3D::recordData, lib/waves.cpp:4285)", i);
            return RSGPU_ERR_ARG;
        }
        if (sh.nsrc < 0 || sh.nrec < 0) { set_error("shot %d: negative trace count", i); return RSGPU_ERR_ARG; }
        if (sh.nsrc > 0 && (!sh.smap || !sh.sshift || !sh.wavelet)) { set_error("shot %d: source arrays missing", i); return RSGPU_ERR_ARG; }
        if (sh.nrec > 0 && (!sh.gmap || !sh.gshift)) { set_error("shot %d: receiver arrays missing", i); return RSGPU_ERR_ARG; }
        if (sh.src_field < RSGPU_PRESSURE || sh.src_field > RSGPU_VZ) { set_error("shot %d: bad source field", i); return RSGPU_ERR_ARG; }
        if (sh.nrec > 0 && (sh.rec_field < RSGPU_PRESSURE || sh.rec_field > RSGPU_VZ)) { set_error("shot %d: bad receiver field", i); return RSGPU_ERR_ARG; }
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
        if ((long long)L.plane * 10 > 0x7fffffffLL) { set_error("shot %d: plane of %lld cells too large", i, L.plane); return RSGPU_ERR_ARG; }
        const size_t fbytes = (size_t)L.plane * L.planes * es;
        for (int k = 0; k < nf3(); k++) L.f[k] = take(fbytes);
        for (int k = 0; k < npsi3(); k++) {
            L.psix[k] = take((size_t)L.nzp * L.nyp * 2 * lp * es);
            L.psiy[k] = take((size_t)L.nzp * 2 * lp * L.nxp * es);
            L.psiz[k] = take((size_t)2 * lp * L.nyp * L.nxp * es);
        }
        L.psi_end = off;
        L.nrec = s[i].nrec;
        L.nsrc = s[i].nsrc;
        L.traces = take((size_t)std::max(1, s[i].nrec) * cfg.nt * es);
        L.state_end = off;
        for (int k = 0; k < np3(); k++) L.m[k] = take(fbytes);
        L.wav = take((size_t)std::max(1, s[i].nsrc) * cfg.nt * es);
        L.rfac = take((size_t)std::max(1, s[i].nrec) * es);
    }
    // injection / recording plans (reference loop order: trace, z, y, x corner)
    std::vector<std::vector<long long>> inj_pt(ns), rec_pt(ns);
    std::vector<std::vector<int>> inj_start(ns), inj_tr(ns);
    std::vector<std::vector<double>> inj_w(ns), rec_w(ns);
    auto shift_of = [&](const void *p, int k) -> double {
        return prec == PREC_F64 ? ((const double *)p)[k] : (double)((const float *)p)[k];
    };
    auto tri = [&](double sft, double *w) {
        if (prec == PREC_F64) { w[0] = 1 - sft; w[1] = sft; }
        else { w[0] = (float)(1 - (float)sft); w[1] = (float)sft; }
    };
    for (int i = 0; i < ns; i++) {
        const Layout3D &L = shots[i];
        struct W3 { double v[3]; };
        std::map<long long, std::vector<std::pair<int, W3>>> per_pt;
        std::vector<long long> order_pts;
        for (int t = 0; t < s[i].nsrc; t++) {
            const int mx = s[i].smap[3 * t], my = s[i].smap[3 * t + 1], mz = s[i].smap[3 * t + 2];
            if (mx < 0 || my < 0 || mz < 0) continue;
            double xt[2], yt[2], zt[2];
            tri(shift_of(s[i].sshift, 3 * t), xt);
            tri(shift_of(s[i].sshift, 3 * t + 1), yt);
            tri(shift_of(s[i].sshift, 3 * t + 2), zt);
            for (int i1 = 0; i1 < 2; i1++)
                for (int i2 = 0; i2 < 2; i2++)
                    for (int i3 = 0; i3 < 2; i3++) {
                        const int ix = lp + mx + i3, iy = lp + my + i2, iz = lp + mz + i1;
                        if (ix >= L.nxp || iy >= L.nyp || iz >= L.nzp) {
                            set_error("shot %d: source %d maps outside the grid", i, t);
                            return RSGPU_ERR_ARG;
                        }
                        const long long p = iz * L.plane + (long long)iy * L.pitch + ix;
                        if (!per_pt.count(p)) order_pts.push_back(p);
                        per_pt[p].push_back({t, W3{{xt[i3], yt[i2], zt[i1]}}});
                    }
        }
        inj_start[i].push_back(0);
        for (long long p : order_pts) {
            inj_pt[i].push_back(p);
            for (auto &cw : per_pt[p]) {
                inj_tr[i].push_back(cw.first);
                for (int k = 0; k < 3; k++) inj_w[i].push_back(cw.second.v[k]);
            }
            inj_start[i].push_back((int)inj_tr[i].size());
        }
        for (int t = 0; t < s[i].nrec; t++) {
            const int mx = s[i].gmap[3 * t], my = s[i].gmap[3 * t + 1], mz = s[i].gmap[3 * t + 2];
            if (mx < 0 || my < 0 || mz < 0) {
                rec_pt[i].push_back(-1);
                for (int k = 0; k < 6; k++) rec_w[i].push_back(0);
                continue;
            }
            if (lp + mx + 1 >= L.nxp || lp + my + 1 >= L.nyp || lp + mz + 1 >= L.nzp) {
                set_error("shot %d: receiver %d maps outside the grid", i, t);
                return RSGPU_ERR_ARG;
            }
            rec_pt[i].push_back((long long)(lp + mz) * L.plane + (long long)(lp + my) * L.pitch + lp + mx);
            double w[2];
            for (int k = 0; k < 3; k++) {
                tri(shift_of(s[i].gshift, 3 * t + k), w);
                rec_w[i].push_back(w[0]);
                rec_w[i].push_back(w[1]);
            }
        }
    }
    std::vector<size_t> o_ip(ns), o_is(ns), o_it(ns), o_iw(ns), o_rp(ns), o_rw(ns);
    for (int i = 0; i < ns; i++) {
        o_ip[i] = take(inj_pt[i].size() * 8);
        o_is[i] = take(inj_start[i].size() * 4);
        o_it[i] = take(inj_tr[i].size() * 4);
        o_iw[i] = take(inj_w[i].size() * es);
        o_rp[i] = take(rec_pt[i].size() * 8);
        o_rw[i] = take(rec_w[i].size() * es);
    }
    const size_t o_pml = take((size_t)12 * lp * es);
    rec_pt_offsets = o_rp;
    arena_bytes = off;
    if (cudaMalloc(&arena, arena_bytes) != cudaSuccess) {
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
        for (int k = 0; k < np3(); k++) {
            cudaMemcpy3DParms p = {};
            p.srcPtr = make_cudaPitchedPtr(const_cast<void *>(s[i].model[k]), (size_t)L.nxp * es, L.nxp, L.nyp);
            p.dstPtr = make_cudaPitchedPtr(A + L.m[k] + origin_bytes(L), (size_t)L.pitch * es, L.pitch, L.rows);
            p.extent = make_cudaExtent((size_t)L.nxp * es, L.nyp, L.nzp);
            p.kind = cudaMemcpyHostToDevice;
            CU(cudaMemcpy3DAsync(&p, stream));
        }
        if (s[i].nsrc > 0)
            CU(cudaMemcpyAsync(A + L.wav, s[i].wavelet, (size_t)s[i].nsrc * cfg.nt * es, cudaMemcpyHostToDevice, stream));
        if ((st = put_raw(o_ip[i], inj_pt[i].data(), inj_pt[i].size() * 8)) != RSGPU_OK) return st;
        if ((st = put_raw(o_is[i], inj_start[i].data(), inj_start[i].size() * 4)) != RSGPU_OK) return st;
        if ((st = put_raw(o_it[i], inj_tr[i].data(), inj_tr[i].size() * 4)) != RSGPU_OK) return st;
        if ((st = put_real(o_iw[i], inj_w[i])) != RSGPU_OK) return st;
        if ((st = put_raw(o_rp[i], rec_pt[i].data(), rec_pt[i].size() * 8)) != RSGPU_OK) return st;
        if ((st = put_real(o_rw[i], rec_w[i])) != RSGPU_OK) return st;
        if (s[i].rec_factor && s[i].nrec > 0) {
            std::vector<double> fac(s[i].nrec);
            for (int t = 0; t < s[i].nrec; t++) fac[t] = shift_of(s[i].rec_factor, t);
            if ((st = put_real(L.rfac, fac)) != RSGPU_OK) return st;
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
    const size_t m_shots = 0, m_ir = rup3(ns * shot_bytes, 256), m_tiles = rup3(m_ir + ns * ir_bytes, 256);
    const size_t m_coef = rup3(m_tiles + tiles.size() * sizeof(Tile3D), 256);
    const size_t m_gate = rup3(m_coef + coefs.size(), 256), m_end = m_gate + 256;
    CU(cudaMalloc(&d_meta, m_end));
    d_gate = reinterpret_cast<int *>((char *)d_meta + m_gate);
    std::vector<unsigned char> meta(m_end, 0);
    reinterpret_cast<int *>(meta.data() + m_gate)[0] = 1;   // recording on
    for (int i = 0; i < ns; i++) {
        if (prec == PREC_F64) fill_desc<double>(meta.data() + m_shots + i * shot_bytes, meta.data() + m_ir + i * ir_bytes,
                                                i, s[i], o_ip[i], o_is[i], o_it[i], o_iw[i], o_rp[i], o_rw[i],
                                                (int)inj_pt[i].size(), (int)rec_pt[i].size());
        else fill_desc<float>(meta.data() + m_shots + i * shot_bytes, meta.data() + m_ir + i * ir_bytes, i, s[i],
                              o_ip[i], o_is[i], o_it[i], o_iw[i], o_rp[i], o_rw[i], (int)inj_pt[i].size(),
                              (int)rec_pt[i].size());
    }
    std::memcpy(meta.data() + m_tiles, tiles.data(), tiles.size() * sizeof(Tile3D));
    std::memcpy(meta.data() + m_coef, coefs.data(), coefs.size());
    CU(cudaMemcpy(d_meta, meta.data(), m_end, cudaMemcpyHostToDevice));
    d_shots = (char *)d_meta + m_shots;
    d_injrec = (char *)d_meta + m_ir;
    d_tiles = (char *)d_meta + m_tiles;
    d_coefs = (char *)d_meta + m_coef;
    CU(cudaStreamSynchronize(stream));
    return RSGPU_OK;
}

size_t Plan3D::origin_bytes(const Layout3D &L) const
{
    return ((size_t)GUARD * L.plane + (size_t)GUARD * L.pitch + GUARD) * es;
}

template <typename T>
void Plan3D::fill_desc(unsigned char *sd, unsigned char *irp, int i, const rsgpu_shot &s, size_t o_ip, size_t o_is,
                       size_t o_it, size_t o_iw, size_t o_rp, size_t o_rw, int ninj, int nrec)
{
    char *A = (char *)arena;
    const Layout3D &L = shots[i];
    const size_t org = origin_bytes(L);
    Shot3D<T> d{};
    d.nxp = L.nxp; d.nyp = L.nyp; d.nzp = L.nzp; d.pitch = L.pitch; d.rows = L.rows;
    d.lpml = cfg.lpml; d.fs = cfg.fs; d.plane = L.plane;
    for (int k = 0; k < nf3(); k++) d.f[k] = (T *)(A + L.f[k] + org);
    for (int k = 0; k < np3(); k++) d.m[k] = (const T *)(A + L.m[k] + org);
    for (int k = 0; k < npsi3(); k++) {
        d.psix[k] = (T *)(A + L.psix[k]);
        d.psiy[k] = (T *)(A + L.psiy[k]);
        d.psiz[k] = (T *)(A + L.psiz[k]);
    }
    std::memcpy(sd, &d, sizeof d);
    InjRec3<T> r{};
    r.ninj = ninj;
    r.kind_inj = ninj > 0 ? INJ3_P + s.src_field : INJ3_NONE;    // PRESSURE, VX, VY, VZ -> 1..4
    r.inj_pt = (const long long *)(A + o_ip);
    r.inj_start = (const int *)(A + o_is);
    r.inj_trace = (const int *)(A + o_it);
    r.inj_w = (const T *)(A + o_iw);
    r.wav = (const T *)(A + L.wav);
    r.nrec = nrec;
    r.kind_rec = nrec > 0 ? REC3_P + s.rec_field : REC3_NONE;
    r.rec_pt = (const long long *)(A + o_rp);
    r.rec_w = (const T *)(A + o_rw);
    r.rec_out = (T *)(A + L.traces);
    r.nt = cfg.nt;
    r.rev = reverse_time ? 1 : 0;
    r.rec_gate = gated_recording ? d_gate : nullptr;
    r.rec_factor = (const T *)(A + L.rfac);
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
    if (phys == PHYS_E3D) {
        if ((e = launch_step_e3d(prec, 0, adjoint_steps, args, d_coefs, ntiles, stream)) != cudaSuccess) goto fail;
        if ((e = launch_step_e3d(prec, 1, adjoint_steps, args, d_coefs, ntiles, stream)) != cudaSuccess) goto fail;
        if ((e = launch_injrec_e3d(prec, d_shots, d_injrec, nshots, cfg.dt, it, stream)) != cudaSuccess) goto fail;
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

rsgpu_status Plan3D::set_recording(bool on)
{
    if (!gated_recording) { set_error("plan was created without gated recording"); return RSGPU_ERR_STATE; }
    CU(cudaMemsetAsync(d_gate, on ? 1 : 0, sizeof(int), stream));
    return RSGPU_OK;
}

rsgpu_status Plan3D::inject_record_only(int it)
{
    if (it < 0 || it >= cfg.nt) { set_error("step %d outside [0,%d)", it, cfg.nt); return RSGPU_ERR_ARG; }
    cudaError_t e = phys == PHYS_E3D ? launch_injrec_e3d(prec, d_shots, d_injrec, nshots, cfg.dt, it, stream)
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

rsgpu_status Plan3D::read_traces(int shot, void *host_out)
{
    if (shot < 0 || shot >= nshots) { set_error("bad shot %d", shot); return RSGPU_ERR_ARG; }
    const Layout3D &L = shots[shot];
    if (L.nrec == 0) return RSGPU_OK;
    const size_t n = (size_t)L.nrec * cfg.nt;
    std::vector<unsigned char> tmp(n * es);
    CU(cudaMemcpyAsync(tmp.data(), (char *)arena + L.traces, n * es, cudaMemcpyDeviceToHost, stream));
    CU(cudaStreamSynchronize(stream));
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
