// Forward modelling of one acoustic 2D shot that allocates no device memory.
//
// Who needs it: callers that may not call cudaMalloc/cudaFree themselves or
// through this library -- for example a host application whose device memory
// is owned by another allocator (a framework's caching pool or a fixed
// budget), or one that cannot afford the device-wide synchronisation that
// cudaMalloc and cudaFree imply while other streams are running.  They hand in
// device buffers they already own for the inputs (staggered model, wavelet) and
// the output (traces); the wavefields, C-PML memory variables, staged
// parameters, tile tables, tensor maps and source/receiver plans live in one
// file-scope device array of NOALLOC_SCRATCH_BYTES.
//
// The kernels are the same ones rsgpu_modelling launches (fd2d_kernels.cuh);
// only the place of their working memory differs.
#include <cuda.h>
#include <algorithm>
#include <cstring>
#include <map>
#include <mutex>
#include <vector>

#include "rsgpu.h"
#include "rsgpu_host.h"
#include "rsgpu_internal.h"
#include "rsgpu_kernels.h"

namespace rsgpu {

// 32 MiB per device, held by every GPU that loads this library until the
// process exits (the array lives in the library's device image).
constexpr size_t NOALLOC_SCRATCH_BYTES = (size_t)32 << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

namespace {

std::mutex g_lock;                        // one call at a time in this process

// Device address of the scratch array on the current device.  In host code
// g_noalloc_scratch names a host-side stand-in, so the address comes from
// cudaGetSymbolAddress with the device current.  It is looked up on every call
// (the lookup allocates nothing): a cached address would go stale when the
// device's context is torn down and the module reloaded (cudaDeviceReset).
rsgpu_status scratch_address(unsigned char **out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        cudaGetLastError();
        set_error("no usable CUDA device for the no-allocation entry point");
        return RSGPU_ERR_NODEVICE;
    }
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
        set_error("cudaGetSymbolAddress of the scratch array failed: %s", cudaGetErrorString(e));
        return RSGPU_ERR_CUDA;
    }
    *out = static_cast<unsigned char *>(p);
    return RSGPU_OK;
}

inline size_t rup(size_t a, size_t b) { return (a + b - 1) / b * b; }

}  // namespace
}  // namespace rsgpu

using namespace rsgpu;

#define NA_CU(call)                                                                                \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess) {                                                                   \
            set_error("%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
            return RSGPU_ERR_CUDA;                                                                 \
        }                                                                                          \
    } while (0)

extern "C" rsgpu_status rsgpu_modelling_a2d_noalloc(const rsgpu_config *cfg, const rsgpu_shot *shot, void *stream)
{
    if (!cfg || !shot) { set_error("null config or shot"); return RSGPU_ERR_ARG; }
    if (cfg->physics != RSGPU_ACOUSTIC2D) { set_error("no-allocation modelling: acoustic 2D only"); return RSGPU_ERR_UNSUPPORTED; }
    if (cfg->precision != RSGPU_F32_EXACT && cfg->precision != RSGPU_F32_FAST) {
        set_error("no-allocation modelling: float precisions only");
        return RSGPU_ERR_UNSUPPORTED;
    }
    if (cfg->lpml < 1 || cfg->nt < 1 || !(cfg->dt > 0) || !(cfg->dx > 0) || !(cfg->dz > 0)) {
        set_error("lpml, nt, dt, dx, dz must be positive");
        return RSGPU_ERR_ARG;
    }
    const int order = std::min(std::max(cfg->order, 1), 8), lp = cfg->lpml, nt = cfg->nt, prec = cfg->precision;
    const int nxp = shot->nx + 2 * lp, nzp = shot->nz + 2 * lp;
    if (shot->nx < 1 || shot->nz < 1 || nxp <= order || nzp <= order) { set_error("model window too small"); return RSGPU_ERR_ARG; }
    for (int k = 0; k < 3; k++)
        if (!shot->model[k]) { set_error("model parameter %d is null", k); return RSGPU_ERR_ARG; }
    if (shot->nsrc < 0 || shot->nrec < 0) { set_error("negative trace count"); return RSGPU_ERR_ARG; }
    if (shot->nsrc > 0 && (!shot->smap || !shot->sshift || !shot->wavelet)) { set_error("source arrays missing"); return RSGPU_ERR_ARG; }
    if (shot->nrec > 0 && (!shot->gmap || !shot->gshift || !shot->rec_out)) { set_error("receiver arrays missing"); return RSGPU_ERR_ARG; }
    const int sf = shot->src_field, rf = shot->rec_field;
    if (sf != RSGPU_PRESSURE && sf != RSGPU_VX && sf != RSGPU_VZ) { set_error("bad source field"); return RSGPU_ERR_ARG; }
    if (shot->nrec > 0 && rf != RSGPU_PRESSURE && rf != RSGPU_VX && rf != RSGPU_VZ) { set_error("bad receiver field"); return RSGPU_ERR_ARG; }
    const int cfgi = (cfg->tile >= 0 && cfg->tile < tile_count_2d()) ? cfg->tile : TILECFG_DEFAULT;
    const TileShape ts = tile_shape_2d(cfgi);

    // ---- injection plan (contributions in the reference's loop order) and receivers
    const int pitch = (int)rup(GUARD + rup(nxp, 128) + GUARD, 32);
    const int rows = GUARD + (int)rup(nzp, 64) + GUARD;
    std::map<int, std::vector<int>> per_pt;          // target point -> contribution indices
    std::vector<int> order_pts, ctr;
    std::vector<float> cwx, cwz;
    const float *ssh = static_cast<const float *>(shot->sshift);
    for (int t = 0; t < shot->nsrc; t++) {
        const int mx = shot->smap[2 * t], mz = shot->smap[2 * t + 1];
        if (mx < 0 || mz < 0) continue;
        const float sx = ssh[2 * t], sz = ssh[2 * t + 1];
        const float xt[2] = {1 - sx, sx}, zt[2] = {1 - sz, sz};
        for (int i1 = 0; i1 < 2; i1++)
            for (int i2 = 0; i2 < 2; i2++) {
                const int ix = lp + mx + i2, iz = lp + mz + i1;
                if (ix >= nxp || iz >= nzp) { set_error("source %d maps outside the grid", t); return RSGPU_ERR_ARG; }
                const int p = iz * pitch + ix;
                if (!per_pt.count(p)) order_pts.push_back(p);
                per_pt[p].push_back((int)ctr.size());
                ctr.push_back(t); cwx.push_back(xt[i2]); cwz.push_back(zt[i1]);
            }
    }
    std::vector<int> inj_pt, inj_start(1, 0), inj_tr;
    std::vector<float> inj_wx, inj_wz;
    for (int p : order_pts) {
        inj_pt.push_back(p);
        for (int c : per_pt[p]) { inj_tr.push_back(ctr[c]); inj_wx.push_back(cwx[c]); inj_wz.push_back(cwz[c]); }
        inj_start.push_back((int)inj_tr.size());
    }
    std::vector<int> rec_pt;
    std::vector<float> rec_w;
    const float *gsh = static_cast<const float *>(shot->gshift);
    for (int t = 0; t < shot->nrec; t++) {
        const int mx = shot->gmap[2 * t], mz = shot->gmap[2 * t + 1];
        if (mx < 0 || mz < 0) { rec_pt.push_back(-1); rec_w.insert(rec_w.end(), 4, 0.f); continue; }
        if (lp + mx + 1 >= nxp || lp + mz + 1 >= nzp) { set_error("receiver %d maps outside the grid", t); return RSGPU_ERR_ARG; }
        rec_pt.push_back((lp + mz) * pitch + lp + mx);
        const float sx = gsh[2 * t], sz = gsh[2 * t + 1];
        rec_w.push_back(1 - sx); rec_w.push_back(sx); rec_w.push_back(1 - sz); rec_w.push_back(sz);
    }
    std::vector<Tile2D> tiles;
    for (int z0 = 0; z0 < nzp; z0 += ts.tz)
        for (int x0 = 0; x0 < nxp; x0 += ts.tx) {
            int fl = 0;
            if (x0 < order || x0 + ts.tx > nxp - order - 1) fl |= TILE_XEDGE;
            if (z0 < order || z0 + ts.tz > nzp - order - 1) fl |= TILE_ZEDGE;
            if (x0 < lp || x0 + ts.tx > nxp - lp) fl |= TILE_XPML;
            if (z0 < lp || z0 + ts.tz > nzp - lp) fl |= TILE_ZPML;
            tiles.push_back({0, x0, z0, fl});
        }
    std::vector<unsigned char> coefs;
    coef_table_host(prec, cfg->dx, cfg->dz, coefs);

    // ---- scratch layout: state and staged parameters first (cleared), then metadata
    size_t off = 0;
    auto take = [&](size_t bytes) { size_t o = off; off = rup(off + bytes, 256); return o; };
    const size_t fbytes = (size_t)pitch * rows * 4;
    size_t o_f[3], o_m[3], o_px[2], o_pz[2];
    for (auto &o : o_f) o = take(fbytes);
    for (auto &o : o_m) o = take(fbytes);
    for (auto &o : o_px) o = take((size_t)nzp * 2 * lp * 4);
    for (auto &o : o_pz) o = take((size_t)2 * lp * nxp * 4);
    const size_t cleared = off;
    const size_t o_meta = off;
    const size_t o_shot = take(sizeof(Shot2D<float>)), o_ir = take(sizeof(InjRec<float>));
    const size_t o_tiles = take(tiles.size() * sizeof(Tile2D)), o_coef = take(coefs.size());
    const size_t o_maps = take(NMAP2D * sizeof(CUtensorMap));
    const size_t o_ip = take(std::max<size_t>(1, inj_pt.size()) * 4), o_is = take(inj_start.size() * 4);
    const size_t o_it = take(std::max<size_t>(1, inj_tr.size()) * 4), o_wx = take(std::max<size_t>(1, inj_wx.size()) * 4);
    const size_t o_wz = take(std::max<size_t>(1, inj_wz.size()) * 4), o_rp = take(std::max<size_t>(1, rec_pt.size()) * 4);
    const size_t o_rw = take(std::max<size_t>(1, rec_w.size()) * 4), o_pml = take((size_t)12 * lp * 4);
    const size_t o_err = take(2 * sizeof(int));
    if (off > NOALLOC_SCRATCH_BYTES) {
        set_error("no-allocation modelling needs %zu bytes of scratch for this %dx%d padded grid; the library holds "
                  "%zu bytes -- use rsgpu_modelling instead", off, nxp, nzp, NOALLOC_SCRATCH_BYTES);
        return RSGPU_ERR_ARG;
    }

    std::lock_guard<std::mutex> guard(g_lock);
    unsigned char *S = nullptr;
    if (rsgpu_status s = scratch_address(&S)) return s;
    cudaStream_t st = static_cast<cudaStream_t>(stream);

    // ---- metadata, built on the host with device addresses inside the scratch
    std::vector<unsigned char> meta(off - o_meta, 0);
    auto at = [&](size_t o) { return meta.data() + (o - o_meta); };
    const size_t org = ((size_t)GUARD * pitch + GUARD) * 4;
    Shot2D<float> sd{};
    sd.nxp = nxp; sd.nzp = nzp; sd.pitch = pitch; sd.lpml = lp; sd.fs = cfg->fs;
    for (int k = 0; k < 3; k++) { sd.f[k] = (float *)(S + o_f[k] + org); sd.m[k] = (const float *)(S + o_m[k] + org); }
    for (int k = 0; k < 2; k++) { sd.psix[k] = (float *)(S + o_px[k]); sd.psiz[k] = (float *)(S + o_pz[k]); }
    std::memcpy(at(o_shot), &sd, sizeof sd);
    InjRec<float> ir{};
    ir.nt = nt;
    ir.ninjsets = 1;
    InjSet<float> &q = ir.inj[0];
    q.ninj = (int)inj_pt.size();
    q.kind = q.ninj == 0 ? INJ_NONE : sf == RSGPU_PRESSURE ? INJ_A2_P : sf == RSGPU_VX ? INJ_A2_VX : INJ_A2_VZ;
    q.pt = (const int *)(S + o_ip); q.start = (const int *)(S + o_is); q.trace = (const int *)(S + o_it);
    q.wx = (const float *)(S + o_wx); q.wz = (const float *)(S + o_wz);
    q.wav = static_cast<const float *>(shot->wavelet);
    ir.nrecsets = shot->nrec > 0 ? 1 : 0;
    RecSet<float> &r = ir.rec[0];
    r.nrec = shot->nrec;
    r.kind = shot->nrec == 0 ? REC_NONE : rf == RSGPU_PRESSURE ? REC_A2_P : rf == RSGPU_VX ? REC_A2_VX : REC_A2_VZ;
    r.pt = (const int *)(S + o_rp); r.w = (const float *)(S + o_rw); r.factor = nullptr;
    r.out = static_cast<float *>(shot->rec_out);
    std::memcpy(at(o_ir), &ir, sizeof ir);
    std::memcpy(at(o_tiles), tiles.data(), tiles.size() * sizeof(Tile2D));
    std::memcpy(at(o_coef), coefs.data(), coefs.size());
    for (int k = 0; k < 3; k++)
        if (!encode_field_map_host(at(o_maps) + k * sizeof(CUtensorMap), S + o_f[k], prec, pitch, rows, ts.tx + 2 * GUARD,
                                   ts.tz + 2 * GUARD)) {
            set_error("cuTensorMapEncodeTiled failed");
            return RSGPU_ERR_CUDA;
        }
    auto put = [&](size_t o, const void *src, size_t n) { if (n) std::memcpy(at(o), src, n); };
    put(o_ip, inj_pt.data(), inj_pt.size() * 4); put(o_is, inj_start.data(), inj_start.size() * 4);
    put(o_it, inj_tr.data(), inj_tr.size() * 4); put(o_wx, inj_wx.data(), inj_wx.size() * 4);
    put(o_wz, inj_wz.data(), inj_wz.size() * 4); put(o_rp, rec_pt.data(), rec_pt.size() * 4);
    put(o_rw, rec_w.data(), rec_w.size() * 4);
    if (cfg->pml) std::memcpy(at(o_pml), cfg->pml, (size_t)12 * lp * 4);
    else pml_tables_host(lp, cfg->dt, prec, at(o_pml));

    // ---- stage: clear wavefields, C-PML memory and parameter guards (the array
    // keeps the previous call's contents), copy the caller's parameters into the
    // pitched layout, upload the metadata
    NA_CU(cudaMemsetAsync(S, 0, cleared, st));
    for (int k = 0; k < 3; k++)
        NA_CU(cudaMemcpy2DAsync(S + o_m[k] + org, (size_t)pitch * 4, shot->model[k], (size_t)nxp * 4, (size_t)nxp * 4,
                                nzp, cudaMemcpyDeviceToDevice, st));
    NA_CU(cudaMemcpyAsync(S + o_meta, meta.data(), meta.size(), cudaMemcpyHostToDevice, st));

    // ---- the time loop: velocity, stress, insertSource + recordData per step
    Step2DArgs<float> a{};
    a.shots = (const Shot2D<float> *)(S + o_shot);
    a.tiles = (const Tile2D *)(S + o_tiles);
    a.ntiles = (int)tiles.size();
    a.order = order;
    a.dt = (float)cfg->dt; a.dx = (float)cfg->dx; a.dz = (float)cfg->dz;
    a.rdx = 1.0f / a.dx; a.rdz = 1.0f / a.dz;
    a.pml = (const float *)(S + o_pml);
    a.lpml = lp;
    int *derr = (int *)(S + o_err);
    // The error word is read back every CHECK_EVERY steps, so a call whose bounded
    // waits give up stops after at most that many more steps instead of queueing
    // all nt of them (each could wait out its own limit again).
    constexpr int CHECK_EVERY = 256;
    int err = 0;
    for (int it = 0; it < nt; it++) {
        for (int half = 0; half < 2; half++)
            NA_CU(launch_step_2d(prec, cfgi, PHYS_A2D, half, 0, &a, S + o_coef, S + o_maps, derr, a.ntiles, st));
        NA_CU(launch_injrec_2d(prec, S + o_shot, S + o_ir, 1, cfg->dt, it, nullptr, st));
        if ((it + 1) % CHECK_EVERY == 0 || it + 1 == nt) {
            NA_CU(cudaMemcpyAsync(&err, derr, sizeof(int), cudaMemcpyDeviceToHost, st));
            NA_CU(cudaStreamSynchronize(st));
            if (err) break;
        }
    }
    if (err) { set_error("a device-side wait exceeded its time limit (code %d)", err); return (rsgpu_status)err; }
    return RSGPU_OK;
}
