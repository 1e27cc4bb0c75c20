// Plan object behind the opaque rsgpu_plan handle (host runtime, not ABI).
#pragma once
#include <cstddef>
#include <vector>
#include <cuda_runtime.h>
#include "rsgpu.h"
#include "rsgpu_kernels.h"
#include "rsgpu_internal.h"

namespace rsgpu {

int esize(int prec);
inline int nfields(int phys) { return phys == PHYS_A2D ? 3 : phys == PHYS_E2D ? 5 : phys == PHYS_A3D ? 4 : 9; }
inline int nparams(int phys) { return phys == PHYS_A2D ? 3 : phys == PHYS_E2D ? 5 : phys == PHYS_A3D ? 4 : 8; }
inline int npsi(int phys) { return phys == PHYS_A2D ? 2 : 4; }

// One source or receiver trace set of a shot (host arrays; maps and shifts hold
// dim = 2 or 3 values per trace).
struct TraceSet {
    int n = 0;
    const int *map = nullptr;       // n*dim ints, -1 = off the grid
    const void *shift = nullptr;    // n*dim reals
    int field = RSGPU_PRESSURE;
    const void *data = nullptr;     // sources: n*nt wavelet / residual reals
    const void *factor = nullptr;   // receivers: elastic pressure divisor per trace, or null
    bool psum = false;              // receivers, elastic PRESSURE: record (Sxx + Szz) unhalved
    bool at_point = false;          // receivers, elastic 3D: the adjoint wavelet gradient, read at
                                    // the map point itself (no interpolation)
};
struct ShotSets {
    int nsrc = 0, nrec = 0;
    TraceSet src[MAXSETS], rec[MAXSETS];
};
// Arena offsets of one set's injection and recording plans.
struct SetOffsets {
    size_t ipt, istart, itr, iwx, iwz;
    int ninj;
    size_t rpt, rw, rfac;
};

// Byte offsets of one shot's arrays inside the plan arena.
struct ShotLayout {
    int nx = 0, nz = 0, nxp = 0, nzp = 0, pitch = 0, rows = 0;
    int nrec = 0, nsrc = 0;         // traces of set 0
    int nrecsets = 0, nsrcsets = 0;
    int nrecs[MAXSETS] = {}, nsrcs[MAXSETS] = {};
    size_t tracesk[MAXSETS] = {}, wavk[MAXSETS] = {};
    size_t f[9] = {}, m[8] = {}, psix[4] = {}, psiz[4] = {};
    size_t fb[5] = {}, psixb[2] = {}, psizb[2] = {};   // second copy (fused z-marching step)
    size_t traces = 0, wav = 0;
    size_t psi_end = 0;       // end of the wavefields + C-PML memory (a checkpoint's extent)
    size_t field_begin = 0;   // first byte of the zero-initialised state block
    size_t state_end = 0;     // one past its last byte (wavefields, C-PML memory, traces)
};

class Plan {
public:
    ~Plan();
    // sets: per shot the source/receiver trace sets; null = the rsgpu_shot's own
    rsgpu_status create(const rsgpu_config *c, int ns, const rsgpu_shot *s, const ShotSets *sets = nullptr);
    rsgpu_status reset();
    rsgpu_status run(int it0, int nsteps);
    rsgpu_status read_traces(int shot, void *host_out, int set = 0);
    rsgpu_status read_field(int shot, int field, void *host_out);
    rsgpu_status launch_step(int it_base, const int *it_dev, bool adj, cudaEvent_t *ev = nullptr);
    // fused z-marching step (one launch per time step, recording of the previous
    // step included); cur = the wavefield copy it reads
    rsgpu_status launch_fused(int it_base, bool dev_it, int cur, cudaEvent_t *ev = nullptr);
    rsgpu_status enable_timing();
    rsgpu_status kernel_times(float *ms_vel, float *ms_str);
    rsgpu_status check_device_error();
    // adjoint drivers: injection/recording of step `it` without propagation, and
    // switching the trace recording on/off in stream order
    rsgpu_status inject_record_only(int it);
    rsgpu_status set_recording(bool on);

    // options read by create()
    bool reverse_time = false;           // wavelet/trace index nt-1-it at step it
    bool adjoint_steps = false;          // propagate with the adjoint (backwardstep*) kernels
    bool gated_recording = false;        // recording obeys set_recording()
    cudaStream_t shared_stream = nullptr;  // run on this caller-owned stream

    rsgpu_config cfg{};
    int prec = 0, phys = 0, nshots = 0, tilecfg = 0, ntiles = 0;
    std::vector<ShotLayout> shots;
    std::vector<size_t> rec_pt_offsets;   // [shot*MAXSETS + set]: arena offset of the receiver points (-1 = off grid)
    void *arena = nullptr;
    size_t arena_bytes = 0, state_end = 0;
    void *d_meta = nullptr;
    void *d_shots = nullptr, *d_injrec = nullptr, *d_tiles = nullptr, *d_coefs = nullptr, *d_pml = nullptr;
    void *d_maps = nullptr;    // [nshots][NMAP2D] CUtensorMap
    int *d_it = nullptr;       // step counter read by graph-replayed kernels
    int *d_err = nullptr;      // device error word (bounded waits)
    int *d_gate = nullptr;     // recording switch (gated_recording)
    cudaStream_t stream = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    bool use_graph = true;
    int graph_steps = 32;
    long long launches = 0;
    // CUDA events recorded inside the graph around the half-step kernels of the
    // first NTIMED steps of every replayed chunk (kernel durations for rooflines)
    static const int NTIMED = 4;
    bool time_kernels = false;
    cudaEvent_t tev[NTIMED][3] = {};

    // fused z-marching step (fd2d_fused.cuh): chosen at create() for 2D forward
    // propagation unless launch_mode asks for the per-tile kernels
    bool fused = false;
    int zm_nitems = 0, zm_band = 0;
    std::vector<unsigned char> zm_args;   // Zm2DArgs<T> with device pointers into d_zm
    void *d_zm = nullptr;                 // items, injection entries, receiver list, tensor maps
    cudaGraphExec_t zm_graph = nullptr;

    // column-marching elastic half-steps (fd2d_march.cu, launch mode 4): chosen at
    // create() for FAST elastic forward propagation when launch_mode asks for it
    bool march = false;
    int march_nitems = 0, march_band = 0;
    March2DArgs march_args{};
    void *d_march = nullptr;              // work items and tensor maps

private:
    rsgpu_status run_fused(int it0, int nsteps);
    // builds the marching kernels' work items and tensor maps; coefs = the host CoefSet bytes
    rsgpu_status setup_march(const std::vector<unsigned char> &coefs);
    // builds the fused step's tables; inj_pts[shot*MAXSETS + set] = the set's CSR target offsets
    rsgpu_status setup_fused(const std::vector<std::vector<int>> &inj_pts);
    rsgpu_status check_config(const rsgpu_config *c, int ns, const rsgpu_shot *s, bool sets_given);
    int default_tile(long tiles32) const;   // tiles32: the batch's count of 32x32 tiles
    template <typename T>
    void fill_desc(unsigned char *sd, unsigned char *irp, const ShotLayout &L, size_t org, const SetOffsets *so,
                   const ShotSets &t);
};

}  // namespace rsgpu
