// Kernels of the FWI-gradient and RTM-image drivers (host runtime internals, not ABI).
#pragma once
#include <cmath>
#include <cstddef>
#include <cuda_runtime.h>
#include "rsgpu_kernels.h"

namespace rsgpu {

// Correlation inputs of one shot.  Field and parameter pointers are the origins
// (element (0,0) of the padded grid) of the pitched plan arrays; vp, rho and the
// outputs are dense [nz][nx] arrays of the unpadded window.
template <typename T>
struct Corr2D {
    const T *wsp;               // forward pressure
    const T *wrp, *wrx, *wrz;   // adjoint pressure, vx, vz
    const T *rx, *rz;           // staggered inverse densities of the forward plan
    const T *vp, *rho;          // unpadded models (FWI gradient scaling)
    void *g0, *g1;              // FWI: vpgrad, rhograd; RTM: g0 = image [nhz][nhx][nz][nx]
    void *ilum;                 // FWI: source illumination [nz][nx], or null
    int nx, nz, pitch, lpml;
};

// Elastic 2D correlation inputs of one shot (FwiElastic2D::crossCorr and scaleGrad).
template <typename T>
struct Corr2DE {
    const T *ws[5];             // forward Vx, Vz, Sxx, Szz, Sxz (origins)
    const T *wr[5];             // adjoint Vx, Vz, Sxx, Szz, Sxz
    const T *rx, *rz;
    const T *vp, *vs, *rho;     // unpadded models
    void *g[3];                 // lambda -> vp, mu -> vs, rho gradients [nz][nx]
    int nx, nz, pitch, lpml;
};

// Residuals of the three elastic data types (P, Ux, Uz) of one shot.
template <typename T>
struct Resid2DE {
    const T *mod[3];
    const T *obs[3];
    T *res[3];
    const int *rec_pt_vx;       // validity of a trace for the misfit: the Ux set's map
    int nrec, nt;
    T *work[2];                 // ADAPTIVE misfits: per-trace scratch of the Ux and Uz filters
    T *tnorm[2];                // ADAPTIVE misfits: the filters' squared norms per trace
};

// 3D image correlation inputs of one shot (RtmAcoustic3D::crossCorr).
template <typename T>
struct Corr3D {
    const T *wsp, *wrp;         // forward and adjoint pressure (origins of the pitched 3D arrays)
    void *img;                  // [nhz][nhy][nhx][nz][ny][nx]
    int nx, ny, nz, pitch, lpml, pad_;
    long long plane;            // elements per plane of the pitched arrays
};

// 3D FWI gradient correlation inputs of one shot (FwiAcoustic3D::crossCorr).
template <typename T>
struct Corr3DF {
    const T *wsp;               // forward pressure
    const T *wrx, *wry, *wrz;   // adjoint velocities
    const T *rx, *ry, *rz;      // staggered inverse densities
    const T *vp, *rho;          // unpadded models [nz][ny][nx]
    void *g0, *g1;              // vpgrad, rhograd [nz][ny][nx]
    int nx, ny, nz, pitch, lpml, pad_;
    long long plane;
};

// Elastic 3D correlation inputs of one shot (FwiElastic3D::crossCorr and scaleGrad).
template <typename T>
struct Corr3DE {
    const T *ws[9];             // forward Vx, Vy, Vz, Sxx, Syy, Szz, Syz, Sxz, Sxy (origins)
    const T *wr[9];             // adjoint fields, same order
    const T *rx, *ry, *rz;      // staggered inverse densities
    const T *vp, *vs, *rho;     // unpadded models [nz][ny][nx]
    void *g[3];                 // lambda -> vp, mu -> vs, rho gradients [nz][ny][nx]
    int nx, ny, nz, pitch, lpml, pad_;
    long long plane;
};

// Residuals of the three elastic 3D data types (Ux, Uy, Uz) of one shot.
template <typename T>
struct Resid3E {
    const T *mod[3];
    const T *obs[3];
    T *res[3];
    int nrec, nt;
};

// Residual and misfit of one shot (DIFFERENCE misfit).
template <typename T>
struct Resid2D {
    const T *mod;               // modelled data [nrec][nt] (forward plan traces)
    const T *obs;               // observed data [nrec][nt]
    T *res;                     // residual [nrec][nt] (adjoint plan source traces)
    const int *rec_pt;          // -1 for receivers off the grid (excluded from the misfit)
    int nrec, nt;
    T *work;                    // ADAPTIVE misfits: 5*nt scratch values per trace
    T *tnorm;                   // ADAPTIVE misfits: the shaping filter's squared norm per trace
};

// One shot's window of gradients / image for the global stack: component arrays of
// the accumulator type, [nh][nz][nx], placed at (x0, z0) of the global grid.
struct StackWin {
    const void *g[3];
    int nx, nz, x0, z0;
};
// Adds every shot's window into the global arrays out0..out2 (nxg*nzg*nh values of
// gbytes-byte type, components beyond ncomp unused), shots in order.
cudaError_t launch_stack_windows(int gbytes, const StackWin *w, int nshots, int ncomp, int nxg, int nzg, int nh,
                                 void *out0, void *out1, void *out2, cudaStream_t st);

// One contiguous 2D block of state copied into / out of a checkpoint slot.
struct CkptSeg {
    void *src;                  // first element
    int rows, cols, pitch;      // pitch in elements
    long long dst;              // element offset of the block inside a slot
    int prow;                   // 3D: rows per plane (0 = one 2D block)
    long long pstride;          // 3D: elements between planes
};

enum { ACC_REF = 0, ACC_F64 = 1 };

// Snapshot2D/3D's enddiff (lib/snap.cpp:334-337), evaluated in the element type:
// the adjoint time of the last snapshot minus that of the last forward step.
inline int snap_enddiff(int nt, double dt_cfg, int snapinc, int prec)
{
    const int snapnt = (nt - 1) / snapinc + 1;
    if (prec == PREC_F64) {
        const double dt = dt_cfg, snapdt = dt * snapinc;
        return (int)rintf((float)(((nt - 1) * dt - (snapnt - 1) * snapdt) / dt));
    }
    const float dt = (float)dt_cfg, snapdt = dt * snapinc;
    return (int)rintf(((nt - 1) * dt - (snapnt - 1) * snapdt) / dt);
}
enum { CK_NATIVE = 0, CK_F16 = 1, CK_BF16 = 2 };

// Gradient/image correlation of one adjoint time step over all shots.
cudaError_t launch_corr_fwi_a2d(int prec, int acc, const void *desc, int nshots, int nxmax, int nzmax, double dx,
                                double dz, cudaStream_t st);
cudaError_t launch_corr_rtm_a2d(int prec, int acc, const void *desc, int nshots, int nxmax, int nzmax, int nhx,
                                int nhz, cudaStream_t st);
// Residuals (mod - obs) and per-shot misfit (sum of r^2/2 over on-grid traces):
// ACC_REF in the element type, sequentially in the reference's order; ACC_F64 in
// double by fixed-order tree reductions (64 CTAs per shot, then their partials).
// partials: residual_partials(nshots) doubles of scratch.
cudaError_t launch_residual(int prec, int acc, const void *desc, int nshots, double *misfit, double *partials,
                            cudaStream_t st);
size_t residual_partials(int nshots);
// CORRELATION misfit (normalised zero-lag correlation per trace) and its residuals,
// with the 97th-percentile magnitude clip of the 2D driver when `clip`; nrec_max
// bounds the shared memory.
cudaError_t launch_residual_corr(int prec, int acc, const void *desc, int nshots, int nrec_max, double *misfit,
                                 cudaStream_t st, bool clip);
// ADAPTIVE_GAUSS / ADAPTIVE_LINEAR misfits (Wiener shaping filter per trace) and
// their residuals, with the 97th-percentile clip of the 2D drivers when `clip`.
// `tables` holds adaptive_table_bytes(prec, nt) bytes filled by
// adaptive_fill_tables; every Resid2D carries its work and tnorm arrays.
enum { ADAPT_GAUSS = 2, ADAPT_LINEAR = 3, ADAPT_SINGLE = 4 };
size_t adaptive_table_bytes(int prec, int mode, int nt);
void adaptive_fill_tables(int prec, int mode, int nt, void *host_tables);
// Per-trace scratch values of one filter (work) for a mode.
size_t adaptive_work_values(int mode, int nt);
cudaError_t launch_residual_adaptive(int prec, int acc, int mode, const void *desc, int nshots, int nrec_max, int nt,
                                     const void *tables, double *misfit, cudaStream_t st, bool clip);
// FwiElastic2D (lib/fwi.cpp:3002-3196, 3428-3753): ADAPTIVE_GAUSS / ADAPTIVE_LINEAR
// shape the Ux and Uz traces separately (`comp`: two Resid2D per shot, Ux then Uz,
// pointing into the Resid2DE arrays) and clip them together; ADAPTIVE_SINGLE shapes
// the Ux and Uz traces joined end to end with one filter, without a clip.  The P
// residual is zero.
cudaError_t launch_residual_adaptive_e2d(int prec, int acc, int mode, const void *desc, const void *comp, int nshots,
                                         int nrec_max, int nt, const void *tables, double *misfit, cudaStream_t st);
// The elastic CORRELATION misfit and residuals (P, Ux, Uz) with the reference's clips.
cudaError_t launch_residual_corr_e2d(int prec, int acc, const void *desc, int nshots, int nrec_max, double *misfit,
                                     cudaStream_t st);
cudaError_t launch_corr_fwi_e2d(int prec, int acc, const void *desc, int nshots, int nxmax, int nzmax, double dx,
                                double dz, cudaStream_t st);
cudaError_t launch_scale_grad_e2d(int prec, int acc, const void *desc, int nshots, int nxmax, int nzmax,
                                  cudaStream_t st);
cudaError_t launch_residual_e2d(int prec, int acc, const void *desc, int nshots, double *misfit, cudaStream_t st);
cudaError_t launch_corr_rtm_a3d(int prec, int acc, const void *desc, int nshots, int nxmax, int nymax, int nhx,
                                int nhy, int nhz, cudaStream_t st);
cudaError_t launch_corr_fwi_a3d(int prec, int acc, const void *desc, int nshots, int nxmax, int nymax, double dx,
                                double dy, double dz, cudaStream_t st);
// Elastic 3D (adjoint3d_elastic.cu): FwiElastic3D::crossCorr of one adjoint step,
// scaleGrad after the last one, and the DIFFERENCE residuals and misfit.
cudaError_t launch_corr_fwi_e3d(int prec, int acc, const void *desc, int nshots, int nxmax, int nymax, double dx,
                                double dy, double dz, cudaStream_t st);
cudaError_t launch_scale_grad_e3d(int prec, int acc, const void *desc, int nshots, int nxmax, int nymax,
                                  cudaStream_t st);
cudaError_t launch_residual_e3d(int prec, int acc, const void *desc, int nshots, double *misfit, cudaStream_t st);
// Checkpoint slot I/O.  scales[nseg] holds the power-of-two scale of each block
// for the 16-bit formats (written by save, read by load); max_rows is the largest
// `rows` of the blocks (it sizes the grid).
cudaError_t launch_ckpt_save(int prec, int ck, const CkptSeg *segs, int nseg, int max_rows, void *slot, float *scales,
                             unsigned *maxbits, cudaStream_t st);
cudaError_t launch_ckpt_load(int prec, int ck, const CkptSeg *segs, int nseg, int max_rows, const void *slot,
                             const float *scales, cudaStream_t st);
// The largest row count of a list of blocks.
inline int ckpt_max_rows(const CkptSeg *segs, size_t n)
{
    int m = 1;
    for (size_t i = 0; i < n; i++) m = segs[i].rows > m ? segs[i].rows : m;
    return m;
}

}  // namespace rsgpu
