// Host side of the fused z-marching 2D step (kernels: fd2d_fused.cuh).
//
// setup_fused() builds, once per plan, the step's work items (strips of
// zm_strip_width() columns by bands of rows, ordered band-major so that CTAs
// running at the same time march neighbouring strips at the same depth), the
// per-item injection entries in the reference's set order, the flat list of
// receiver traces, and the TMA descriptors of the stress ring for both wavefield
// copies.  run_fused() advances an even number of steps with one launch each
// (replayed from a captured graph of 32 steps) so that the state ends in copy 0,
// where every other part of the library (checkpoints, correlations, read-back)
// expects it; a final odd step goes through the per-tile kernels.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include <cuda.h>
#include <cuda_runtime.h>

#include "rsgpu.h"
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

static inline size_t rup(size_t a, size_t b) { return (a + b - 1) / b * b; }

template <typename T>
static void fill_zm_args(std::vector<unsigned char> &out, const Plan &p, const void *items, int nitems,
                         const void *inj, const void *recs, int nrecs, const void *maps)
{
    Zm2DArgs<T> a{};
    a.shots = (const Shot2D<T> *)p.d_shots;
    a.plans = (const InjRec<T> *)p.d_injrec;
    a.items = (const ZmItem *)items;
    a.nitems = nitems;
    a.inj = (const int *)inj;
    a.recs = (const int4 *)recs;
    a.nrecs = nrecs;
    a.maps = maps;
    a.order = p.cfg.order;
    a.dt = (T)p.cfg.dt; a.dx = (T)p.cfg.dx; a.dz = (T)p.cfg.dz;
    a.rdx = (T)1 / a.dx; a.rdz = (T)1 / a.dz;
    a.pml = (const T *)p.d_pml;
    a.lpml = p.cfg.lpml;
    out.resize(sizeof a);
    std::memcpy(out.data(), &a, sizeof a);
}

rsgpu_status Plan::setup_fused(const std::vector<std::vector<int>> &inj_pts)
{
    const int ztx = zm_strip_width(), lp = cfg.lpml, o = cfg.order;
    const int nrf = phys == PHYS_E2D ? 3 : 1;
    const int ring[3] = {phys == PHYS_E2D ? (int)E2_SXX : (int)A2_P, E2_SZZ, E2_SXZ};
    int total_strips = 0, max_nzp = 0;
    for (const auto &L : shots) {
        total_strips += (L.nxp + ztx - 1) / ztx;
        max_nzp = std::max(max_nzp, L.nzp);
    }
    // band height: about three items per resident CTA, bands of at least 32 rows
    if (cfg.zchunk > 0) {
        zm_band = (int)rup((size_t)cfg.zchunk, 8);
    } else {
        const int res = zm_resident_ctas(prec, phys);
        int nz = (int)std::lround(3.0 * res / std::max(1, total_strips));
        nz = std::max(1, std::min(nz, std::max(1, max_nzp / 32)));
        zm_band = (int)rup((size_t)((max_nzp + nz - 1) / nz), 8);
    }
    const int band = zm_band;
    const int nbands = (max_nzp + band - 1) / band;
    std::vector<ZmItem> items;
    std::vector<std::vector<int>> index(nshots);   // per shot: item of (band, strip)
    for (int i = 0; i < nshots; i++) {
        const ShotLayout &L = shots[i];
        index[i].assign((size_t)((L.nzp + band - 1) / band) * ((L.nxp + ztx - 1) / ztx), -1);
    }
    for (int b = 0; b < nbands; b++)
        for (int i = 0; i < nshots; i++) {
            const ShotLayout &L = shots[i];
            const int z0 = b * band;
            if (z0 >= L.nzp) continue;
            const int z1 = std::min(z0 + band, (int)rup(L.nzp, 8));
            const int ns = (L.nxp + ztx - 1) / ztx;
            for (int st = 0; st < ns; st++) {
                ZmItem it{};
                it.shot = i;
                it.x0 = st * ztx;
                it.z0 = z0;
                it.z1 = z1;
                int fl = 0;
                if (it.x0 - 8 < o || it.x0 + ztx + 8 > L.nxp - o - 1) fl |= ZM_XEDGE;
                if (z0 - 8 < o || z1 + 8 > L.nzp - o - 1) fl |= ZM_ZEDGE;
                if (it.x0 - 8 < lp || it.x0 + ztx + 8 > L.nxp - lp) fl |= ZM_XPML;
                if (z0 - 8 < lp || z1 + 8 > L.nzp - lp) fl |= ZM_ZPML;
                it.flags = fl;
                index[i][(size_t)b * ns + st] = (int)items.size();
                items.push_back(it);
            }
        }
    zm_nitems = (int)items.size();
    // injection entries of each item, grouped by set in set order
    std::vector<std::vector<int>> per((size_t)zm_nitems * MAXSETS);
    for (int i = 0; i < nshots; i++) {
        const ShotLayout &L = shots[i];
        const int ns = (L.nxp + ztx - 1) / ztx;
        for (int k = 0; k < MAXSETS; k++) {
            const std::vector<int> &pts = inj_pts[(size_t)i * MAXSETS + k];
            for (size_t j = 0; j < pts.size(); j++) {
                const int iz = pts[j] / L.pitch, ix = pts[j] % L.pitch;
                const int item = index[i][(size_t)(iz / band) * ns + ix / ztx];
                if (item < 0) { set_error("shot %d: injection point outside the work items", i); return RSGPU_ERR_ARG; }
                per[(size_t)item * MAXSETS + k].push_back((k << 24) | (int)j);
            }
        }
    }
    std::vector<int> inj;
    for (int t = 0; t < zm_nitems; t++)
        for (int k = 0; k < MAXSETS; k++) {
            items[t].ie[k] = (int)inj.size();
            const auto &v = per[(size_t)t * MAXSETS + k];
            inj.insert(inj.end(), v.begin(), v.end());
            items[t].ie[k + 1] = (int)inj.size();
        }
    if (inj.empty()) inj.push_back(0);
    // every receiver trace of the batch
    std::vector<int> recs;
    for (int i = 0; i < nshots; i++)
        for (int k = 0; k < shots[i].nrecsets; k++)
            for (int tr = 0; tr < shots[i].nrecs[k]; tr++) {
                recs.push_back(i); recs.push_back(k); recs.push_back(tr); recs.push_back(0);
            }
    const int nrecs = (int)recs.size() / 4;
    if (recs.empty()) recs.assign(4, 0);
    // device tables: items | injection entries | receivers | tensor maps
    const size_t o_items = 0;
    const size_t o_inj = rup(o_items + items.size() * sizeof(ZmItem), 256);
    const size_t o_recs = rup(o_inj + inj.size() * sizeof(int), 256);
    const size_t o_maps = rup(o_recs + recs.size() * sizeof(int), 256);
    const size_t bytes = o_maps + (size_t)nshots * 2 * nrf * sizeof(CUtensorMap);
    std::vector<unsigned char> h(bytes, 0);
    std::memcpy(h.data() + o_items, items.data(), items.size() * sizeof(ZmItem));
    std::memcpy(h.data() + o_inj, inj.data(), inj.size() * sizeof(int));
    std::memcpy(h.data() + o_recs, recs.data(), recs.size() * sizeof(int));
    char *A = (char *)arena;
    for (int i = 0; i < nshots; i++) {
        const ShotLayout &L = shots[i];
        for (int c = 0; c < 2; c++)
            for (int r = 0; r < nrf; r++) {
                void *base = A + (c ? L.fb[ring[r]] : L.f[ring[r]]);
                void *m = h.data() + o_maps + (((size_t)i * 2 + c) * nrf + r) * sizeof(CUtensorMap);
                if (!encode_field_map_host(m, base, prec, L.pitch, L.rows, ztx + 32, 8)) {
                    set_error("cuTensorMapEncodeTiled failed for the stress ring of shot %d", i);
                    return RSGPU_ERR_CUDA;
                }
            }
    }
    CU(dev_alloc(&d_zm, bytes, stream));
    CU(cudaMemcpy(d_zm, h.data(), bytes, cudaMemcpyHostToDevice));
    char *Z = (char *)d_zm;
    if (prec == PREC_F64)
        fill_zm_args<double>(zm_args, *this, Z + o_items, zm_nitems, Z + o_inj, Z + o_recs, nrecs, Z + o_maps);
    else
        fill_zm_args<float>(zm_args, *this, Z + o_items, zm_nitems, Z + o_inj, Z + o_recs, nrecs, Z + o_maps);
    return RSGPU_OK;
}

rsgpu_status Plan::launch_fused(int it_base, bool dev_it, int cur, cudaEvent_t *ev)
{
    cudaError_t e;
    if (ev && (e = cudaEventRecordWithFlags(ev[0], stream, cudaEventRecordExternal)) != cudaSuccess) goto fail;
    if ((e = launch_zm_step_2d(prec, phys, zm_args.data(), d_coefs, d_it, cur, it_base, dev_it ? 1 : 0, zm_nitems,
                               stream)) != cudaSuccess)
        goto fail;
    if (ev && (e = cudaEventRecordWithFlags(ev[1], stream, cudaEventRecordExternal)) != cudaSuccess) goto fail;
    launches += 1;
    return RSGPU_OK;
fail:
    set_error("fused step launch failed: %s", cudaGetErrorString(e));
    return RSGPU_ERR_CUDA;
}

rsgpu_status Plan::run_fused(int it0, int nsteps)
{
    const int nf = nsteps & ~1;   // an even count leaves the state in copy 0
    cudaError_t e = launch_zm_set_run(d_it, it0, stream);
    if (e != cudaSuccess) { set_error("launch_zm_set_run: %s", cudaGetErrorString(e)); return RSGPU_ERR_CUDA; }
    launches += 1;
    int done = 0;
    const int G = graph_steps & ~1;
    if (use_graph && G >= 2 && nf >= G) {
        if (!zm_graph) {
            cudaGraph_t g;
            CU(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
            rsgpu_status st = RSGPU_OK;
            for (int s = 0; s < G && st == RSGPU_OK; s++)
                st = launch_fused(s, true, s & 1, (time_kernels && s < NTIMED) ? tev[s] : nullptr);
            if (st == RSGPU_OK && (e = launch_advance(d_it, G, stream)) != cudaSuccess) {
                set_error("launch_advance: %s", cudaGetErrorString(e));
                st = RSGPU_ERR_CUDA;
            }
            cudaError_t ce = cudaStreamEndCapture(stream, &g);
            if (st != RSGPU_OK) return st;
            if (ce != cudaSuccess) { set_error("graph capture failed: %s", cudaGetErrorString(ce)); return RSGPU_ERR_CUDA; }
            CU(cudaGraphInstantiate(&zm_graph, g, 0));
            cudaGraphDestroy(g);
            launches -= G;   // captured launches are counted at replay
        }
        while (nf - done >= G) {
            CU(cudaGraphLaunch(zm_graph, stream));
            launches += G + 1;
            done += G;
        }
    }
    for (; done < nf; done++)
        if (rsgpu_status st = launch_fused(it0 + done, false, done & 1)) return st;
    // the last fused step is recorded here (each launch records its predecessor)
    if ((e = launch_zm_record_2d(prec, zm_args.data(), d_it, 0, it0 + nf - 1, stream)) != cudaSuccess) {
        set_error("launch_zm_record_2d: %s", cudaGetErrorString(e));
        return RSGPU_ERR_CUDA;
    }
    launches += 1;
    if (nsteps & 1) return launch_step(it0 + nf, nullptr, adjoint_steps);
    return RSGPU_OK;
}

}  // namespace rsgpu
