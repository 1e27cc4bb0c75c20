// 3D batch plan behind the opaque rsgpu_plan handle (host runtime, not ABI).
#pragma once
#include <cstddef>
#include <vector>
#include <cuda_runtime.h>
#include "rsgpu.h"
#include "rsgpu_kernels.h"
#include "rsgpu_plan.h"

namespace rsgpu {

// Byte offsets of one 3D shot's arrays inside the plan arena.
struct Layout3D {
    int nxp = 0, nyp = 0, nzp = 0, pitch = 0, rows = 0, planes = 0;
    long long plane = 0;
    int nrec = 0, nsrc = 0;                       // traces of set 0
    int nrecsets = 0, nsrcsets = 0;
    int nrecs[MAXSETS] = {}, nsrcs[MAXSETS] = {};
    size_t f[9] = {}, m[8] = {}, psix[6] = {}, psiy[6] = {}, psiz[6] = {};
    size_t psi_end = 0, state_end = 0;
    size_t traces = 0, wav = 0, rfac = 0;         // set 0
    size_t tracesk[MAXSETS] = {}, wavk[MAXSETS] = {}, rfack[MAXSETS] = {};
};

class Plan3D {
public:
    ~Plan3D();
    // sets: per shot the source/receiver trace sets (elastic: up to MAXSETS each);
    // null = the rsgpu_shot's own
    rsgpu_status create(const rsgpu_config *c, int ns, const rsgpu_shot *s, const ShotSets *sets = nullptr);
    rsgpu_status reset();
    rsgpu_status run(int it0, int nsteps);
    rsgpu_status step(int it);
    rsgpu_status read_traces(int shot, void *host_out, int set = 0);
    rsgpu_status read_field(int shot, int field, void *host_out);
    size_t origin_bytes(const Layout3D &L) const;
    rsgpu_status inject_record_only(int it);   // injection/recording of step it without propagation

    // fields, parameters and C-PML memory arrays per face pair of the physics
    int nf3() const { return phys == PHYS_E3D ? 9 : 4; }
    int np3() const { return phys == PHYS_E3D ? 8 : 4; }
    int npsi3() const { return phys == PHYS_E3D ? 6 : 2; }

    // options read by create()
    bool reverse_time = false;                 // wavelet/trace index nt-1-it at step it
    bool adjoint_steps = false;                // elastic: propagate with backwardstep* (adjoint kernels)
    bool gated_recording = false;              // recording obeys set_recording()
    const Plan3D *share_params = nullptr;      // use this plan's parameter arrays (same shots and
                                               // grids) instead of uploading a copy
    rsgpu_status set_recording(bool on);
    int *d_gate = nullptr;                     // recording switch (gated_recording)
    cudaStream_t shared_stream = nullptr;      // run on this caller-owned stream

    rsgpu_config cfg{};
    int prec = 0, phys = PHYS_A3D, nshots = 0, es = 4, zc = 64, ntiles = 0;
    int nsets = 1;                             // InjRec3 entries per shot (elastic: MAXSETS)
    std::vector<Layout3D> shots;
    std::vector<size_t> rec_pt_offsets;        // [shot*nsets + set]: arena offset of the receiver points (long long, -1 off grid)
    void *arena = nullptr, *d_meta = nullptr;
    size_t arena_bytes = 0;
    void *d_shots = nullptr, *d_injrec = nullptr, *d_tiles = nullptr, *d_coefs = nullptr, *d_pml = nullptr;
    std::vector<unsigned char> h_coefs;        // host copy of the CoefSet3 at d_coefs
    void *d_maps = nullptr;                    // elastic fast mode: NMAP_E3 tensor maps per shot
    // elastic fast adjoint plans: the velocity step runs the forward TMA kernel on work
    // arrays (launch_work_e3d); shot descriptors and maps whose stress slots are those
    void *d_work = nullptr, *d_shots_w = nullptr, *d_maps_w = nullptr, *d_wdesc = nullptr;
    int *d_err = nullptr;                      // device error word (bounded waits)
    rsgpu_status check_device_error();
    cudaStream_t stream = nullptr;
    long long launches = 0;

    // device address of parameter k of shot i (this plan's arena, or the shared plan's)
    const char *param_base(int i, int k) const;

private:
    struct SetTables {
        size_t ip, is, it, iw, rp, rw;
        int ninj, nrec;
    };
    template <typename T>
    void fill_shot(unsigned char *sd, int i);
    template <typename T>
    void fill_set(unsigned char *irp, int i, int k, const TraceSet &src, const TraceSet &rec, const SetTables &t);
};

}  // namespace rsgpu
