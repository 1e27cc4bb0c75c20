// Host side of the column-marching elastic 2D half-steps (launch mode 4): work
// items (strip x band of every shot) and the tensor maps of the TMA row ring.
#include <algorithm>
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

static inline size_t rupm(size_t a, size_t b) { return (a + b - 1) / b * b; }

rsgpu_status Plan::setup_march(const std::vector<unsigned char> &coefs)
{
    // Band height: rows per work item.  One wave of CTAs covers the batch when the
    // strips x bands fill the SMs' resident slots; a band must be tall enough to
    // amortise its 16 rows of window warm-up.
    int dev = 0, nsm = 148;
    CU(cudaGetDevice(&dev));
    CU(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    int res = march_resident_ctas();
    if (res < 1) { set_error("the marching kernels cannot be resident on this device"); return RSGPU_ERR_CUDA; }
    long strips = 0;
    int nzmax = 0;
    for (const ShotLayout &L : shots) {
        strips += (L.nxp + MSTRIP2D - 1) / MSTRIP2D;
        nzmax = std::max(nzmax, L.nzp);
    }
    int band;
    if (cfg.zchunk > 0) {
        band = (int)rupm((size_t)cfg.zchunk, 8);
    } else {
        const long slots = (long)nsm * res;
        const long per = std::max(1L, slots / std::max(1L, strips));
        band = (int)rupm((size_t)((nzmax + per - 1) / per), 8);
        band = std::max(band, 32);
    }
    std::vector<MarchItem> items;
    for (int i = 0; i < nshots; i++) {
        const ShotLayout &L = shots[i];
        // strips that hold C-PML columns or columns with reduced-order stencils
        const int xlo = std::max(cfg.lpml, cfg.order), xhi = L.nxp - std::max(cfg.lpml, cfg.order + 1);
        for (int x0 = 0; x0 < L.nxp; x0 += MSTRIP2D) {
            const int flags = (x0 < xlo || x0 + MSTRIP2D > xhi) ? MARCH_XGEN : 0;
            for (int z0 = 0; z0 < L.nzp; z0 += band) items.push_back({i, x0, z0, std::min(z0 + band, L.nzp), flags});
        }
    }
    march_nitems = (int)items.size();
    march_band = band;
    // device tables: items | tensor maps (64-byte aligned)
    const size_t o_maps = rupm(items.size() * sizeof(MarchItem), 256);
    const size_t bytes = o_maps + (size_t)nshots * NMAP2D * sizeof(CUtensorMap);
    std::vector<unsigned char> h(bytes, 0);
    std::memcpy(h.data(), items.data(), items.size() * sizeof(MarchItem));
    char *A = (char *)arena;
    for (int i = 0; i < nshots; i++) {
        const ShotLayout &L = shots[i];
        for (int k = 0; k < NMAP2D; k++) {
            void *m = h.data() + o_maps + ((size_t)i * NMAP2D + k) * sizeof(CUtensorMap);
            if (!encode_field_map_host(m, A + L.f[k], prec, L.pitch, L.rows, MSTRIP2D + 2 * GUARD, 8)) {
                set_error("cuTensorMapEncodeTiled failed for the marching ring of shot %d", i);
                return RSGPU_ERR_CUDA;
            }
        }
    }
    CU(dev_alloc(&d_march, bytes, stream));
    CU(cudaMemcpy(d_march, h.data(), bytes, cudaMemcpyHostToDevice));
    March2DArgs &a = march_args;
    a.shots = (const Shot2D<float> *)d_shots;
    a.items = (const MarchItem *)d_march;
    a.maps = (const char *)d_march + o_maps;
    a.pml = (const float *)d_pml;
    a.coefs = (const float *)d_coefs;
    a.err = d_err;
    a.order = cfg.order;
    a.lpml = cfg.lpml;
    a.dt = (float)cfg.dt;
    // the full-order rows of the host CoefSet<float>: cx[9 * CROW] then cz[9 * CROW]
    const int crow = coef_row_stride();
    const float *cs = reinterpret_cast<const float *>(coefs.data());
    for (int k = 0; k < NCOEF; k++) {
        a.cx[k] = cs[cfg.order * crow + k];
        a.cz[k] = cs[9 * crow + cfg.order * crow + k];
    }
    return RSGPU_OK;
}

}  // namespace rsgpu
