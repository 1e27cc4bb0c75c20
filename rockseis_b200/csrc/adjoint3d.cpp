// RTM image driver for 3D acoustic shots (host runtime behind rsgpu_rtm_image and
// rsgpu_adjoint_* for RSGPU_ACOUSTIC3D).
//
// The reference's RtmAcoustic3D::run_optimal (lib/rtm.cpp:735-859) runs the same
// Revolve-driven loop as the 2D drivers: a forward propagator checkpointed in
// `ncheck` slots, an adjoint propagator fed with the recorded data, and a
// correlation of both pressures at every adjoint time level.  Here the forward and
// adjoint wavefields of all shots are two batched 3D plans (z-marching kernels)
// sharing one stream; the adjoint plan runs forward in reversed time.  Checkpoints
// hold every shot's four wavefields (interior of the pitched arrays) and C-PML
// memory, lossless or as FP16/BF16 with a power-of-two scale per block.
#include <algorithm>
#include <cstring>
#include <memory>
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
    if (dbuf) cudaFree(dbuf);
    if (ckpt) cudaFree(ckpt);
    if (stream) cudaStreamDestroy(stream);
}

rsgpu_status Adjoint3D::create(const rsgpu_config *c, const rsgpu_adjoint_opts *o, int kind, int ns,
                               const rsgpu_adjoint_shot *s)
{
    if (!c || !o || !s || ns < 1) { set_error("null config/options/shots or nshots < 1"); return RSGPU_ERR_ARG; }
    if (c->physics != RSGPU_ACOUSTIC3D || kind != RSGPU_KIND_RTM) {
        set_error("the 3D adjoint driver is built for acoustic RTM images");
        return RSGPU_ERR_UNSUPPORTED;
    }
    if (o->ckpt_precision < RSGPU_CKPT_NATIVE || o->ckpt_precision > RSGPU_CKPT_BF16) {
        set_error("bad checkpoint precision %d", o->ckpt_precision);
        return RSGPU_ERR_ARG;
    }
    if (o->accum != RSGPU_ACCUM_REFERENCE && o->accum != RSGPU_ACCUM_F64) { set_error("bad accumulation %d", o->accum); return RSGPU_ERR_ARG; }
    const int hy = o->nhy > 0 ? o->nhy : 1;
    if (o->nhx < 1 || o->nhz < 1 || o->nhx % 2 == 0 || hy % 2 == 0 || o->nhz % 2 == 0) {
        set_error("nhx, nhy and nhz must be odd and positive");
        return RSGPU_ERR_ARG;
    }
    for (int i = 0; i < ns; i++) {
        const rsgpu_shot &sh = s[i].shot;
        if (sh.src_field != RSGPU_PRESSURE || sh.rec_field != RSGPU_PRESSURE) {
            set_error("shot %d: the acoustic RTM driver takes pressure sources and receivers", i);
            return RSGPU_ERR_UNSUPPORTED;
        }
        if (sh.nsrc < 1 || sh.nrec < 1) { set_error("shot %d: needs sources and receivers", i); return RSGPU_ERR_ARG; }
        if (!s[i].data) { set_error("shot %d: data is null", i); return RSGPU_ERR_ARG; }
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) {
        cudaGetLastError();
        set_error("no CUDA device");
        return RSGPU_ERR_NODEVICE;
    }
    cfg = *c;
    nshots = ns;
    prec = c->precision;
    es = prec == PREC_F64 ? 8 : 4;
    acc = o->accum == RSGPU_ACCUM_F64 ? ACC_F64 : ACC_REF;
    ck = o->ckpt_precision;
    ck_es = ck == CK_NATIVE ? (size_t)es : 2;
    nhx = o->nhx; nhy = hy; nhz = o->nhz;
    {
        RevolveSchedule probe(c->nt, o->ncheck);
        ncheck = probe.snaps();
    }
    CU(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));

    std::vector<rsgpu_shot> fs(ns), bs(ns);
    for (int i = 0; i < ns; i++) {
        fs[i] = s[i].shot;
        fs[i].nrec = 0;                      // the forward run records nothing
        fs[i].rec_out = nullptr;
        bs[i] = s[i].shot;
        bs[i].nsrc = s[i].shot.nrec;         // the data, injected at the receivers
        bs[i].smap = s[i].shot.gmap;
        bs[i].sshift = s[i].shot.gshift;
        bs[i].wavelet = s[i].data;
        bs[i].nrec = 0;
        bs[i].rec_out = nullptr;
    }
    fw.reset(new Plan3D());
    fw->shared_stream = stream;
    ST(fw->create(c, ns, fs.data()));
    bw.reset(new Plan3D());
    bw->shared_stream = stream;
    bw->reverse_time = true;
    ST(bw->create(c, ns, bs.data()));

    const size_t gs = acc == ACC_F64 ? 8 : (size_t)es;
    size_t off = 0;
    auto take = [&](size_t bytes) { size_t r = off; off = rupa(off + std::max<size_t>(bytes, 1), 256); return r; };
    o_img.assign(ns, 0);
    nx.resize(ns); ny.resize(ns); nz.resize(ns);
    for (int i = 0; i < ns; i++) {
        nx[i] = s[i].shot.nx; ny[i] = s[i].shot.ny; nz[i] = s[i].shot.nz;
        nxmax = std::max(nxmax, nx[i]);
        nymax = std::max(nymax, ny[i]);
        o_img[i] = take((size_t)nx[i] * ny[i] * nz[i] * nhx * nhy * nhz * gs);
    }
    const size_t corr_bytes = prec == PREC_F64 ? sizeof(Corr3D<double>) : sizeof(Corr3D<float>);
    o_corr = take(corr_bytes * ns);
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
        for (int f = 0; f < 4; f++)
            add(L.f[f] + fw->origin_bytes(L), L.nyp * L.nzp, L.nxp, L.pitch, L.nyp, L.plane);
        for (int k = 0; k < 2; k++) {
            add(L.psix[k], L.nzp * L.nyp, l2, l2, 0, 0);
            add(L.psiy[k], L.nzp * l2, L.nxp, L.nxp, 0, 0);
            add(L.psiz[k], l2 * L.nyp, L.nxp, L.nxp, 0, 0);
        }
    }
    o_segs = take(sizeof(CkptSeg) * segs.size());
    o_scales = take(sizeof(float) * segs.size() * ncheck);
    o_maxbits = take(sizeof(unsigned) * segs.size());
    if (cudaMalloc(&dbuf, off) != cudaSuccess) {
        cudaGetLastError();
        set_error("device allocation of %zu bytes failed", off);
        return RSGPU_ERR_NOMEM;
    }
    const size_t ck_bytes = slot_elems * ck_es * (size_t)ncheck;
    if (cudaMalloc(&ckpt, ck_bytes) != cudaSuccess) {
        cudaGetLastError();
        set_error("checkpoint allocation of %zu bytes (%d slots) failed", ck_bytes, ncheck);
        return RSGPU_ERR_NOMEM;
    }
    CU(cudaMemsetAsync(dbuf, 0, off, stream));
    CU(cudaMemcpyAsync(D(o_segs), segs.data(), sizeof(CkptSeg) * segs.size(), cudaMemcpyHostToDevice, stream));
    std::vector<unsigned char> corr(corr_bytes * ns);
    for (int i = 0; i < ns; i++) {
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
    CU(cudaStreamSynchronize(stream));
    return RSGPU_OK;
}

rsgpu_status Adjoint3D::slot_io(bool save, int slot)
{
    if (slot < 0 || slot >= ncheck) { set_error("checkpoint slot %d outside [0,%d)", slot, ncheck); return RSGPU_ERR_REVOLVE; }
    char *sl = (char *)ckpt + (size_t)slot * slot_elems * ck_es;
    float *sc = (float *)D(o_scales) + (size_t)slot * segs.size();
    cudaError_t e = save ? launch_ckpt_save(prec, ck, (const CkptSeg *)D(o_segs), (int)segs.size(), sl, sc,
                                            (unsigned *)D(o_maxbits), stream)
                         : launch_ckpt_load(prec, ck, (const CkptSeg *)D(o_segs), (int)segs.size(), sl, sc, stream);
    if (e != cudaSuccess) { set_error("checkpoint %s: %s", save ? "save" : "restore", cudaGetErrorString(e)); return RSGPU_ERR_CUDA; }
    launches += (save && ck != CK_NATIVE) ? 2 : 1;
    ckpt_bytes += (long long)(slot_elems * ck_es);
    return RSGPU_OK;
}

rsgpu_status Adjoint3D::correlate()
{
    cudaError_t e = launch_corr_rtm_a3d(prec, acc, D(o_corr), nshots, nxmax, nymax, nhx, nhy, nhz, stream);
    if (e != cudaSuccess) { set_error("correlation launch: %s", cudaGetErrorString(e)); return RSGPU_ERR_CUDA; }
    launches += 1;
    return RSGPU_OK;
}

rsgpu_status Adjoint3D::run()
{
    const int nt = cfg.nt;
    const long long l0 = fw->launches + bw->launches;
    launches = 0;
    fw_steps = bw_steps = ckpt_bytes = 0;
    ST(fw->reset());
    ST(bw->reset());
    const size_t gs = acc == ACC_F64 ? 8 : (size_t)es;
    for (int i = 0; i < nshots; i++)
        CU(cudaMemsetAsync(D(o_img[i]), 0, (size_t)nx[i] * ny[i] * nz[i] * nhx * nhy * nhz * gs, stream));
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
    launches += fw->launches + bw->launches - l0;
    CU(cudaStreamSynchronize(stream));
    ran = true;
    return RSGPU_OK;
}

rsgpu_status Adjoint3D::read(int ns, const rsgpu_adjoint_shot *s)
{
    if (!ran) { set_error("no run to read"); return RSGPU_ERR_STATE; }
    if (ns != nshots || !s) { set_error("read expects the %d shots of the batch", nshots); return RSGPU_ERR_ARG; }
    const size_t gs = acc == ACC_F64 ? 8 : (size_t)es;
    std::vector<unsigned char> tmp;
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
