// 3D RTM image and FWI gradient drivers behind the rsgpu_adjoint handle (host
// runtime, not ABI): acoustic RTM and FWI, elastic FWI.
#pragma once
#include <memory>
#include <vector>
#include <cuda_runtime.h>
#include "rsgpu.h"
#include "rsgpu_adjoint.h"
#include "rsgpu_plan3d.h"

namespace rsgpu {

class Adjoint3D {
public:
    ~Adjoint3D();
    rsgpu_status create(const rsgpu_config *c, const rsgpu_adjoint_opts *o, int kind, int ns,
                        const rsgpu_adjoint_shot *s);
    rsgpu_status run();
    rsgpu_status read(int ns, const rsgpu_adjoint_shot *s);

    int kind = RSGPU_KIND_RTM, nshots = 0, prec = 0, es = 4, acc = ACC_REF, ck = CK_NATIVE, nhx = 1, nhy = 1, nhz = 1;
    int phys = PHYS_A3D;
    int ncheck = 0, nslots = 0, nxmax = 0, nymax = 0;
    // FULL snapshots (RtmAcoustic3D::run): the P interior every snapinc steps
    int snapmethod = RSGPU_SNAP_OPTIMAL, snapinc = 1, snapnt = 0, enddiff = 0;
    int misfit_type = 0, nrec_max = 0;
    rsgpu_config cfg{};
    std::unique_ptr<Plan3D> fw, bw;
    cudaStream_t stream = nullptr;
    void *dbuf = nullptr, *ckpt = nullptr;
    size_t slot_elems = 0, ck_es = 4;
    int seg_rows = 1;                       // rows of the tallest checkpoint block
    std::vector<CkptSeg> segs;
    std::vector<size_t> o_img, o_vp, o_rho, o_obs, o_g1, o_valid;
    std::vector<size_t> o_vs, o_obsy, o_obsz, o_g2;    // elastic: vs, Uy/Uz data, density gradient
    size_t o_corr = 0, o_res = 0, o_misfit = 0, o_segs = 0, o_scales = 0, o_maxbits = 0;
    size_t o_rpart = 0;                     // residual pass: per-CTA partial misfits
    std::vector<size_t> o_work, o_tnorm;   // ADAPTIVE misfits: per-trace scratch and filter norms
    size_t o_atab = 0;                      // ADAPTIVE misfits: weights and summation-order tables
    std::vector<int> nx, ny, nz, nrec;
    bool fwi() const { return kind == RSGPU_KIND_FWI; }
    bool elastic() const { return phys == PHYS_E3D; }
    long long fw_steps = 0, bw_steps = 0, ckpt_bytes = 0, launches = 0;
    bool ran = false;

private:
    rsgpu_status run_full();
    rsgpu_status slot_io(bool save, int slot);
    rsgpu_status correlate();
    char *D(size_t o) const { return (char *)dbuf + o; }
};

}  // namespace rsgpu
