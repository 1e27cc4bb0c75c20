/*
 * rsgpu.h -- C ABI of the B200 finite-difference wave-propagation library.
 *
 * This is the drop-in boundary beneath RockSeis's C++ drivers.  Each entry
 * point replaces the body of one reference method; the comment beside it cites
 * the reference interface (paths relative to the RockSeis source tree).
 *
 * Conventions
 *  - Plain pointers and sizes only.  Array layouts are the reference's:
 *      2D grids   a[iz*nx + ix]                (I2D, lib/waves.cpp:4)
 *      3D grids   a[iz*nx*ny + iy*nx + ix]     (I3D, lib/waves.cpp:8)
 *      traces     d[it + itr*nt]               (Idat, lib/waves.cpp:13)
 *      maps       Point2D<int> {x,z} / Point3D<int> {x,y,z} pairs, -1 = off grid
 *  - Element type of every real array is float for RSGPU_F32_* precisions
 *    and double for RSGPU_F64.
 *  - Output trace and image arrays are ACCUMULATED into (+=), exactly like the
 *    reference's recordData / crossCorr; callers pass zero-initialised arrays
 *    for a fresh result (the reference's Data2D/Image2D calloc).
 *  - Every call returns an rsgpu_status; nothing exits or throws.  The text of
 *    the last error on the calling thread is rsgpu_last_error().
 *  - No CPU fallback: without a usable CUDA device every compute entry point
 *    returns RSGPU_ERR_NODEVICE.
 */
#ifndef RSGPU_H
#define RSGPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RSGPU_ABI_VERSION 2

typedef enum {
    RSGPU_OK = 0,
    RSGPU_ERR_ARG = 1,          /* invalid argument (sizes, order, null pointers, ...) */
    RSGPU_ERR_CUDA = 2,         /* a CUDA runtime call failed */
    RSGPU_ERR_NOMEM = 3,        /* device or pinned-host allocation failed */
    RSGPU_ERR_STATE = 4,        /* call not valid in the plan's current state */
    RSGPU_ERR_TIMEOUT = 5,      /* a bounded device wait gave up */
    RSGPU_ERR_UNSUPPORTED = 6,  /* option not implemented for this physics */
    RSGPU_ERR_NODEVICE = 7,     /* no CUDA device / kernels not loadable */
    RSGPU_ERR_REVOLVE = 8       /* checkpoint schedule reported an error */
} rsgpu_status;

/* physics */
enum { RSGPU_ACOUSTIC2D = 0, RSGPU_ELASTIC2D = 1, RSGPU_ACOUSTIC3D = 2, RSGPU_ELASTIC3D = 3 };
/* arithmetic of the propagator:
 *   F32_EXACT: float, every operation rounded in the reference's order (no FMA);
 *              reproduces a stock float build of the reference bit for bit.
 *   F32_FAST : float, FMA and pre-scaled coefficients.
 *   F64      : double precision, exact reference order (the FP64 GPU oracle). */
enum { RSGPU_F32_EXACT = 0, RSGPU_F32_FAST = 1, RSGPU_F64 = 2 };
/* field codes: identical to the reference's rs_field (include/utils.h:22) */
enum { RSGPU_PRESSURE = 0, RSGPU_VX = 1, RSGPU_VY = 2, RSGPU_VZ = 3 };
/* misfit codes: identical to rs_fwimisfit (include/utils.h:26) */
enum {
    RSGPU_MISFIT_DIFFERENCE = 0,
    RSGPU_MISFIT_CORRELATION = 1,
    RSGPU_MISFIT_ADAPTIVE_GAUSS = 2,   /* Wiener shaping filter per trace, Gaussian weight */
    RSGPU_MISFIT_ADAPTIVE_LINEAR = 3,  /* Wiener shaping filter per trace, ramp weight */
    RSGPU_MISFIT_ADAPTIVE_SINGLE = 4   /* elastic 2D: one filter for the joined Ux/Uz traces;
                                          the acoustic drivers treat it as DIFFERENCE, as the
                                          reference's switch defaults do */
};
enum { RSGPU_INTERP_LINEAR = 0, RSGPU_INTERP_BSPLINE = 1, RSGPU_INTERP_SINC = 2 };   /* rs_interpmode */
/* checkpoint storage precision of the FWI/RTM gradient drivers */
enum { RSGPU_CKPT_NATIVE = 0, RSGPU_CKPT_F16 = 1, RSGPU_CKPT_BF16 = 2 };
/* revolve actions: identical to revolve_action (include/revolve.h:25) */
enum { RSGPU_ADVANCE = 0, RSGPU_TAKESHOT = 1, RSGPU_RESTORE = 2, RSGPU_FIRSTURN = 3,
       RSGPU_YOUTURN = 4, RSGPU_TERMINATE = 5, RSGPU_ERROR = 6 };

/* Run-wide settings shared by every shot of a batch (the reference's Modelling /
 * Fwi / Rtm object settings plus Der and Pml construction arguments). */
typedef struct {
    int physics;        /* RSGPU_ACOUSTIC2D ... */
    int precision;      /* RSGPU_F32_EXACT ... */
    int lpml;           /* Model::getLpml */
    int order;          /* Der order, clamped to 1..8 like Der::Der (lib/der.cpp:98-99) */
    int fs;             /* free surface (Model::getFs) */
    int nt;             /* time samples (Data::getNt) */
    double dx, dy, dz;  /* grid spacing (dy ignored in 2D) */
    double dt;          /* time step (Data::getDt) */
    const void *pml;    /* 12*lpml C-PML tables in the order A,B,C ltf; A,B,C ltf_stag;
                           A,B,C rbb; A,B,C rbb_stag (include/pml.h:31-81).  NULL: computed
                           by rsgpu_pml_tables with Smax = 1200. */
    int tile;           /* 2D kernel tile shape index (rsgpu_tile_shape), -1 = built-in default */
    int zchunk;         /* 3D: planes marched by one CTA (0 = 64); 2D fused step: rows per
                           work item (rounded up to 8; 0 = chosen from the batch size) */
    int launch_mode;    /* 2D propagation: 0 = library choice (the per-tile kernels, the
                           faster on B200), 1 = the same as 2 (a persistent variant of the
                           per-tile kernels measured slower and was removed),
                           2 = per-tile velocity and stress kernels, 3 = fused z-marching step:
                           velocity, stress and injection of a time step plus recording of
                           the previous one in one launch (forward propagation), 4 = column-
                           marching velocity and stress kernels (elastic, FAST arithmetic,
                           forward propagation; other plans use mode 2) */
    int reserved[5];
} rsgpu_config;

/* One shot (work item) of a batch.  nx/ny/nz are the UNPADDED window the
 * reference's local model holds; device arrays are (n + 2*lpml) per axis. */
typedef struct {
    int nx, ny, nz;
    /* Padded, staggered parameters in the order of the reference's Model getters:
     *  acoustic 2D: Rx, Rz, L              (ModelAcoustic2D::staggerModels, lib/model.cpp:1350)
     *  elastic 2D : Rx, Rz, L, L2M, M      (ModelElastic2D::staggerModels, lib/model.cpp:2720)
     *  acoustic 3D: Rx, Ry, Rz, L          (lib/model.cpp:1965)
     *  elastic 3D : Rx, Ry, Rz, L, L2M, M_yz, M_xz, M_xy   (lib/model.cpp:3371) */
    const void *model[8];
    /* source traces (Data2D/3D with SMAP maps, Geometry2D::makeMap lib/geometry.cpp:137) */
    int nsrc;
    const int *smap;            /* nsrc * dim ints */
    const void *sshift;         /* nsrc * dim reals */
    const void *wavelet;        /* nsrc * nt reals, trace-major */
    int src_field;              /* RSGPU_PRESSURE / RSGPU_VX / RSGPU_VY / RSGPU_VZ */
    /* receiver traces (GMAP) */
    int nrec;
    const int *gmap;
    const void *gshift;
    int rec_field;
    const void *rec_factor;     /* elastic pressure reciprocity divisor per trace, NULL = 1 */
    void *rec_out;              /* nrec * nt reals, accumulated (+=) */
} rsgpu_shot;

typedef struct rsgpu_plan rsgpu_plan;

/* ---------------------------------------------------------------------------
 * Library
 * ------------------------------------------------------------------------- */
int rsgpu_abi_version(void);
const char *rsgpu_last_error(void);
/* Number of CUDA devices visible, or 0. */
int rsgpu_device_count(void);

/* ---------------------------------------------------------------------------
 * Forward modelling
 * ------------------------------------------------------------------------- */

/* Replaces ModellingAcoustic2D::run (lib/modelling.cpp:197-291),
 * ModellingElastic2D::run (lib/modelling.cpp:545-645), ModellingAcoustic3D::run
 * (lib/modelling.cpp:363-474) and ModellingElastic3D::run (lib/modelling.cpp:727-850):
 * nt time steps of forwardstepVelocity, forwardstepStress, insertSource and
 * recordData for every shot of the batch, all shots advancing together.
 * Host arrays in, host traces accumulated into shots[i].rec_out. */
rsgpu_status rsgpu_modelling(const rsgpu_config *cfg, int nshots, const rsgpu_shot *shots);

/* The same work split into steps, for callers that keep the batch resident:
 * create uploads models/maps/wavelets once; run advances steps on the device;
 * read copies one shot's traces to the host (accumulating). */
rsgpu_status rsgpu_plan_create(const rsgpu_config *cfg, int nshots, const rsgpu_shot *shots, rsgpu_plan **plan);
rsgpu_status rsgpu_plan_reset(rsgpu_plan *plan);                 /* zero wavefields, C-PML memory, traces */
rsgpu_status rsgpu_plan_run(rsgpu_plan *plan, int it0, int nsteps);
rsgpu_status rsgpu_plan_read_traces(rsgpu_plan *plan, int shot, void *host_out);
rsgpu_status rsgpu_plan_sync(rsgpu_plan *plan);
/* cudaStream_t of the plan (as void*), for callers that time it with events */
void *rsgpu_plan_stream(rsgpu_plan *plan);
/* Device launches of the propagator kernels issued since the plan was created. */
long long rsgpu_plan_launch_count(rsgpu_plan *plan);
/* Kernel timing: enable_timing makes the captured time loop record CUDA events
 * around the velocity and stress launches of the first steps of each replayed
 * chunk; kernel_times returns their mean durations (ms) from the last replay. */
rsgpu_status rsgpu_plan_enable_timing(rsgpu_plan *plan);
rsgpu_status rsgpu_plan_kernel_times(rsgpu_plan *plan, float *ms_velocity, float *ms_stress);
/* How a 2D plan propagates (no counterpart in the reference): the launch mode in
 * use (3 = fused z-marching step, whose one launch per step rsgpu_plan_kernel_times
 * reports as ms_velocity with ms_stress 0; 4 = column-marching half-steps; 2 =
 * per-tile velocity and stress kernels), and the
 * work items of modes 3 and 4 with their height in rows (0 otherwise). */
rsgpu_status rsgpu_plan_info(rsgpu_plan *plan, int *launch_mode, int *work_items, int *band_rows);
/* Copy one wavefield (reference field code, SXX=4.. for elastic) of one shot to the host
 * in the reference's padded layout (for step-level parity tests). */
rsgpu_status rsgpu_plan_read_field(rsgpu_plan *plan, int shot, int field, void *host_out);
void rsgpu_plan_destroy(rsgpu_plan *plan);

/* Forward modelling of ONE acoustic 2D shot that allocates no device memory.
 * No counterpart in the reference: it exists for callers that cannot call
 * cudaMalloc/cudaFree -- an application whose device memory belongs to another
 * allocator or to a fixed budget, or one that cannot accept the device-wide
 * synchronisation those calls imply while its other streams run.  Such a caller
 * passes DEVICE buffers it owns for shot->model[0..2] (Rx, Rz, L, padded
 * reference layout), shot->wavelet (nsrc*nt) and shot->rec_out (nrec*nt,
 * accumulated); maps and shifts stay in host memory.  All working memory
 * (wavefields, C-PML memory, staged parameters, plans) lives in one static
 * 32 MiB device array per GPU, held by every GPU that loads the library until
 * the process exits; a grid that needs more is rejected with RSGPU_ERR_ARG.
 * Float precisions only; results equal rsgpu_modelling's.  Every call, the
 * first on a device included, looks up the array's device address on the
 * current device (cudaGetSymbolAddress, which allocates nothing), so make each
 * call outside stream capture.  The call blocks: it waits for its work on
 * `stream` (a cudaStream_t, 0 = default) to finish before it returns.  Every
 * call shares the array and clears what must start at zero; calls are
 * serialised by a process-wide lock, and work from two calls must not be made
 * to overlap on the GPU: overlapping calls would race on the array. */
rsgpu_status rsgpu_modelling_a2d_noalloc(const rsgpu_config *cfg, const rsgpu_shot *shot, void *stream);

/* ---------------------------------------------------------------------------
 * FWI gradient and RTM image (adjoint path with Revolve checkpointing)
 * ------------------------------------------------------------------------- */
/* How the gradient / image and the misfit are summed over the nt adjoint steps:
 *   ACCUM_REFERENCE: in the propagator's element type, in the reference's order
 *                    (with RSGPU_F32_EXACT: bit-identical to the reference);
 *   ACCUM_F64      : per-step contributions added in double on the GPU, misfit
 *                    summed in double (fixed-order tree). */
enum { RSGPU_ACCUM_REFERENCE = 0, RSGPU_ACCUM_F64 = 1 };

typedef struct {
    int ncheck;          /* Revolve snapshots (Fwi::setNcheck / Rtm::setNcheck); values outside
                            [2, nt] fall back to Revolve::adjust(nt) like the reference */
    int ckpt_precision;  /* RSGPU_CKPT_NATIVE (lossless) / RSGPU_CKPT_F16 / RSGPU_CKPT_BF16: the
                            checkpoint slots hold the state as 16-bit values with a power-of-two
                            scale per array */
    int accum;           /* RSGPU_ACCUM_* */
    int misfit;          /* RSGPU_MISFIT_*: DIFFERENCE; CORRELATION (acoustic 2D lib/fwi.cpp:617-645,
                            808-849 with the 97th-percentile residual clip; acoustic 3D
                            :1511-1540, 1696-1722 without it; elastic 2D :2939-3001, 3309-3426
                            with the x/z and P clips); ADAPTIVE_GAUSS / ADAPTIVE_LINEAR (acoustic
                            2D :646-735, 851-1014, acoustic 3D :1541-1630, 1725-1840, elastic 2D
                            :3002-3148, 3428-3674); ADAPTIVE_SINGLE (elastic 2D :3149-3196,
                            3675-3753).  The elastic 3D gradient takes DIFFERENCE only */
    int nhx, nhz;        /* RTM extended-image lags (Rtm::setNhx/setNhz; odd, 1 = zero lag) */
    int nhy;             /* 3D RTM y lags (Rtm::setNhy; odd, 0 or 1 = zero lag) */
    int snapmethod;      /* RSGPU_SNAP_OPTIMAL: Revolve checkpointing (run_optimal);
                            RSGPU_SNAP_FULL: the forward pressure saved every snapinc steps and
                            correlated at those steps only (FwiAcoustic2D::run, lib/fwi.cpp:1030-1156;
                            RtmAcoustic2D::run, lib/rtm.cpp:222-326); acoustic 2D;
                            RSGPU_SNAP_EDGES: RtmAcoustic2D::run_edge (lib/rtm.cpp:328-421), the
                            RTM image from the wavefield's four edge lines saved every snapinc
                            steps, the source wavefield re-propagated from them */
    int snapinc;         /* FULL: snapshot increment (Fwi/Rtm snapinc; < 1 means 1) */
    int noreverse;       /* FULL FWI: forward run and misfit only (Fwi::setNoreverse) */
    int reserved[6];
} rsgpu_adjoint_opts;
enum { RSGPU_SNAP_OPTIMAL = 0, RSGPU_SNAP_FULL = 1, RSGPU_SNAP_EDGES = 2 };

/* One shot of FwiAcoustic2D::run_optimal (lib/fwi.cpp:1159-1332),
 * RtmAcoustic2D::run_optimal (lib/rtm.cpp:423-545), FwiElastic2D::run_optimal
 * (lib/fwi.cpp:3937-4143) or FwiElastic3D::run_optimal (lib/fwi.cpp:6770-6990).
 * `shot` carries the padded model, the source (wavelet, SMAP maps) and the
 * receiver maps (GMAP) exactly as for rsgpu_modelling.  Acoustic: src_field and
 * rec_field are RSGPU_PRESSURE.  Elastic 2D: shot.rec_field is RSGPU_PRESSURE (the
 * P data set) and the Ux/Uz sets (VX/VZ maps of the same receivers) are given by
 * the *_vx / *_vz members.  Elastic 3D: the shot's own receiver set is the Ux set
 * (shot.rec_field RSGPU_VX: data, shot.rec_out, datares), the Uy and Uz sets are
 * the *_vy and *_vz members (same trace count); vpgrad, vsgrad, rhograd and the
 * models are [nz][ny][nx].  The reference requires every data set.  Every output
 * is ACCUMULATED (+=) and may be NULL when not wanted. */
typedef struct {
    rsgpu_shot shot;      /* shot.rec_out: FWI modelled data (datamodP), nrec*nt */
    const void *vp;       /* FWI: unpadded vp, nz*nx (ModelAcoustic2D::getVp) */
    const void *rho;      /* FWI: unpadded density, nz*nx (getR) */
    const void *data;     /* FWI: recorded data (datarecP); RTM: the data to migrate; nrec*nt */
    void *vpgrad;         /* FWI: nz*nx (vpgrad image) */
    void *rhograd;        /* FWI: nz*nx */
    void *wavgrad;        /* FWI: nsrc*nt wavelet gradient (SMAP recording of the adjoint P) */
    void *datares;        /* FWI: nrec*nt residuals (dataresP) */
    double *misfit;       /* FWI: one value, accumulated */
    void *image;          /* RTM: nhz*nhx*nz*nx (pimage, Image2D layout); 3D: nhz*nhy*nhx*nz*ny*nx */
    /* elastic 2D only */
    const int *gmap_vx, *gmap_vz;          /* GMAP of the Ux (VX) and Uz (VZ) data sets */
    const void *gshift_vx, *gshift_vz;
    const void *data_vx, *data_vz;         /* recorded Ux / Uz data, nrec*nt */
    const void *vs;                        /* unpadded vs, nz*nx (scaleGrad) */
    void *vsgrad;                          /* nz*nx */
    void *datamod_vx, *datamod_vz;         /* modelled Ux / Uz data */
    void *datares_vx, *datares_vz;         /* Ux / Uz residuals */
    /* elastic 3D only: the Uy data set */
    const int *gmap_vy;
    const void *gshift_vy;
    const void *data_vy;
    void *datamod_vy, *datares_vy;
    /* acoustic 2D FWI: source illumination, nz*nx (FwiAcoustic2D::setSrcilum;
       srcilum -= vpscale*Pfw*Pfw in crossCorr, lib/fwi.cpp:565-567), NULL = off */
    void *srcilum;
} rsgpu_adjoint_shot;

/* FwiAcoustic2D<float>::run_optimal (cfg->physics RSGPU_ACOUSTIC2D),
 * FwiElastic2D<float>::run_optimal (RSGPU_ELASTIC2D), FwiAcoustic3D (RSGPU_ACOUSTIC3D)
 * or FwiElastic3D<float>::run_optimal (RSGPU_ELASTIC3D, DIFFERENCE misfit) for a
 * batch of shots. */
rsgpu_status rsgpu_fwi_gradient(const rsgpu_config *cfg, const rsgpu_adjoint_opts *opts, int nshots,
                                const rsgpu_adjoint_shot *shots);
/* RtmAcoustic2D<float>::run_optimal (RSGPU_ACOUSTIC2D) or RtmAcoustic3D<float>::run_optimal
 * (RSGPU_ACOUSTIC3D, lib/rtm.cpp:735-859) for a batch of shots. */
rsgpu_status rsgpu_rtm_image(const rsgpu_config *cfg, const rsgpu_adjoint_opts *opts, int nshots,
                             const rsgpu_adjoint_shot *shots);

/* The same drivers with the batch resident on the device between runs (no
 * counterpart in the reference; for repeated gradients of one batch):
 * create uploads models, maps and data; run computes one gradient / image of
 * every shot on the device; read adds the results of the last run into the
 * host outputs of `shots` (the same array that create received, or one with the
 * same shapes); stats reports the work of the last run. */
typedef struct rsgpu_adjoint rsgpu_adjoint;
enum { RSGPU_KIND_FWI = 0, RSGPU_KIND_RTM = 1 };
rsgpu_status rsgpu_adjoint_create(const rsgpu_config *cfg, const rsgpu_adjoint_opts *opts, int kind, int nshots,
                                  const rsgpu_adjoint_shot *shots, rsgpu_adjoint **adj);
rsgpu_status rsgpu_adjoint_run(rsgpu_adjoint *adj);
rsgpu_status rsgpu_adjoint_read(rsgpu_adjoint *adj, int nshots, const rsgpu_adjoint_shot *shots);
/* Image2D::stackImage (lib/image.cpp:348-438) of the last run's per-shot results
 * into global images, done on the device (the reference stacks per-shot files on
 * the master, Inversion*::runGrad lib/inversion.cpp:309-321): shot i's window is
 * added at global column ix_start[i] and row iz_start[i] (the reference's
 * (int)(ox_local/dx - ox_global/dx) in the element type; parts outside the global
 * grid are dropped), shots in batch order, onto the running global images held in
 * the host arrays out* (uploaded, stacked, written back: batch after batch this is
 * the reference's shot-by-shot stack): FWI acoustic (vpgrad, rhograd), elastic
 * (vpgrad, vsgrad, rhograd), RTM (image with its lags, out0).  2D drivers. */
rsgpu_status rsgpu_adjoint_stack(rsgpu_adjoint *adj, int nxg, int nzg, const int *ix_start, const int *iz_start,
                                 void *out0, void *out1, void *out2);
/* forward steps, adjoint steps, checkpoint bytes written + read, kernel launches */
rsgpu_status rsgpu_adjoint_stats(rsgpu_adjoint *adj, long long *fw_steps, long long *bw_steps,
                                 long long *ckpt_bytes, long long *launches);
void *rsgpu_adjoint_stream(rsgpu_adjoint *adj);
void rsgpu_adjoint_destroy(rsgpu_adjoint *adj);

/* ---------------------------------------------------------------------------
 * Host preprocessing (restatements of the reference's host-side code; callers
 * that hold reference objects pass the reference's own arrays instead)
 * ------------------------------------------------------------------------- */

/* Interp<T>::interp (lib/interp.cpp:123-186, Data2D and Data3D alike): resample
 * ntr traces of n1 samples (origin o1, interval d1, trace-major [ntr][n1]) onto n2
 * samples (o2, d2) with the reference's LINEAR, BSPLINE (4-tap) or SINC (6-tap)
 * kernel; samples whose stencil leaves the input trace are zero.  Host arrays of
 * the precision's element type.  LINEAR and BSPLINE are bit-identical to the
 * reference; SINC evaluates sin on the GPU (equal after rounding in practice). */
rsgpu_status rsgpu_interp_traces(int precision, int mode, int ntr, int n1, double o1, double d1, const void *in,
                                 int n2, double o2, double d2, void *out);

/* Failure-detection self test (no counterpart in the reference): launches one CTA
 * that waits on a barrier nothing completes.  The kernel's bounded wait (the same
 * one every TMA stage uses) gives up after 2 s, records the time-out in a device
 * error word and returns, so the call returns RSGPU_ERR_TIMEOUT and the device stays
 * usable for further calls.  Any other status means the failure path is broken. */
rsgpu_status rsgpu_selftest_bounded_wait(void);

/* Plans and gradient drivers take their device memory from a library-owned
 * stream-ordered pool per device that keeps up to 8 GiB of freed blocks mapped
 * between calls (so a call that creates and destroys a plan does not map and
 * unmap its arena every time).  This returns every cached block of the current
 * device to the driver; it synchronises the device.  No reference counterpart. */
rsgpu_status rsgpu_release_cached_memory(void);

/* ------------------------------------------------------------------ shot-gather files
 * The reference's .rss container (File::writeHeader / readHeader, lib/file.cpp:184-250):
 * magic "R0CKS", data_format, header_format, type, Nheader, Ndims, N[9], D[9], O[9],
 * then per trace Nheader header values and N1 samples.  Trace files
 * (Data2D::write / read, lib/data.cpp:463-635; Data3D::write :1265-1320) carry the
 * source and receiver coordinates as trace headers: (sx, sz, gx, gz) in 2D,
 * (sx, sy, sz, gx, gy, gz) in 3D, in the sample type.  precision: RSGPU_F32_EXACT or
 * RSGPU_F32_FAST (float files) or RSGPU_F64 (double files). */
enum { RSGPU_RSS_GENERIC = 0, RSGPU_RSS_REGULAR = 1, RSGPU_RSS_DATA2D = 2, RSGPU_RSS_DATA3D = 3 };
typedef struct {
    int data_format, header_format, type;
    long long nheader, ndims;
    long long n[9];
    double d[9], o[9];
} rsgpu_rss_header;
rsgpu_status rsgpu_rss_read_header(const char *path, rsgpu_rss_header *h);
/* Data2D::write (dim 2) / Data3D::write (dim 3): ntrace traces of nt samples;
 * scoords/gcoords hold dim values per trace ([x, z] or [x, y, z]). */
rsgpu_status rsgpu_rss_write_traces(const char *path, int precision, int dim, long long nt, double dt, double ot,
                                    long long ntrace, const void *scoords, const void *gcoords, const void *data);
/* Traces [first, first+count) of a Data2D/Data3D file; any output may be NULL. */
rsgpu_status rsgpu_rss_read_traces(const char *path, int precision, long long first, long long count, void *scoords,
                                   void *gcoords, void *data);
/* ModelAcoustic2D::writeVp and the other model writers (lib/model.cpp:1283-1313):
 * a REGULAR file, N1 = nx, N2 = ny (pass 0 in 2D: the file records 1), N3 = nz;
 * values [nz][ny][nx]. */
rsgpu_status rsgpu_rss_write_model(const char *path, int precision, int nx, int ny, int nz, double dx, double dy,
                                   double dz, double ox, double oy, double oz, const void *values);
rsgpu_status rsgpu_rss_read_model(const char *path, int precision, long long count, void *values);

/* Sort (lib/sort.cpp:132-1055): gathers of a trace file by source, receiver or CMP
 * position (CMP snapped to dx, dy bins), ordered by x, y, z (order 0), y, x, z (1)
 * or z, x, y (2), each gather's traces in file order; and the gather queue of the
 * MPI drivers: rsgpu_sort_next gives the first gather that is NOT_STARTED or
 * FAILED (Sort::get2DGather()), reading a gather marks it RUNNING, the caller
 * marks it FINISHED or FAILED (a failed gather is handed out again). */
enum { RSGPU_SORT_SOURCE = 0, RSGPU_SORT_RECEIVER = 1, RSGPU_SORT_CMP = 2 };
enum { RSGPU_GATHER_FINISHED = 0, RSGPU_GATHER_RUNNING = 1, RSGPU_GATHER_NOT_STARTED = 2, RSGPU_GATHER_FAILED = 3 };
typedef struct rsgpu_sort rsgpu_sort;
rsgpu_status rsgpu_sort_create(const char *path, int key, double dx, double dy, int order, rsgpu_sort **out);
void rsgpu_sort_destroy(rsgpu_sort *s);
rsgpu_status rsgpu_sort_info(const rsgpu_sort *s, long long *ngathers, long long *ntraces, long long *nt);
long long rsgpu_sort_gather_size(const rsgpu_sort *s, long long number);
long long rsgpu_sort_next(const rsgpu_sort *s);
int rsgpu_sort_status(const rsgpu_sort *s, long long number);
rsgpu_status rsgpu_sort_set_status(rsgpu_sort *s, long long number, int status);
/* Sort::get2DGather(number) / get3DGather(number): coordinates and samples of the
 * gather's traces (reciprocity swaps sources and receivers). */
rsgpu_status rsgpu_sort_read_gather(rsgpu_sort *s, long long number, int reciprocity, void *scoords, void *gcoords,
                                    void *data);
/* Sort::createEmptydataset: an output trace file with the survey's headers and n1
 * zero samples per trace; Sort::put2DGather / put3DGather: a gather written to its
 * traces' places in such a file. */
rsgpu_status rsgpu_sort_create_output(const rsgpu_sort *s, const char *path, long long n1, double d1, double o1);
rsgpu_status rsgpu_sort_write_gather(const rsgpu_sort *s, const char *path, long long number, int reciprocity,
                                     long long n1, const void *scoords, const void *gcoords, const void *data);

/* 2D kernel tile shapes, the search space of the tile autotuner (no counterpart in
 * the reference, whose loops have no tiles).  rsgpu_tile_count returns how many
 * shapes the library holds for `precision`; rsgpu_tile_shape gives shape `idx`:
 * the tile's x and z extent, the rows each thread updates and the CTAs per SM the
 * kernel is compiled for.  Index i is the value of rsgpu_config.tile that selects
 * it.  FP64 holds shapes 0 and 3 only; other indices return RSGPU_ERR_ARG there. */
int rsgpu_tile_count(int precision);
rsgpu_status rsgpu_tile_shape(int precision, int idx, int *tx, int *tz, int *rows_per_thread, int *ctas_per_sm);

/* Pml::computeABC with Amax=0, Kmax=2, Smax=1200 (lib/pml.cpp:79-126). */
rsgpu_status rsgpu_pml_tables(int lpml, double dt, int precision, void *out12);

/* Model*::staggerModels (lib/model.cpp:93-240, 1350-1411, 1965, 2720-2802, 3371-3475):
 * pad by lpml with edge replication, form moduli, stagger, invert density,
 * free-surface adjustments.  vs is ignored for acoustic physics.  out[] receives
 * the parameters in the rsgpu_shot.model order, each (nx+2l)(ny+2l)(nz+2l). */
rsgpu_status rsgpu_stagger_model(int physics, int nx, int ny, int nz, int lpml, int fs, int precision,
                                 const void *vp, const void *vs, const void *rho, void *const *out);

/* Data2D/3D::makeMap -> Geometry2D/3D::makeMap (lib/data.cpp:440-460, 1116-1141;
 * lib/geometry.cpp:137-230, 303-420) with zero padding arguments.  coords: ntr*dim
 * doubles (x,z) or (x,y,z) holding the T-typed coordinates; n/o/d: model size,
 * origin and spacing per axis as in Model::getGeom; gshift: per-axis staggering
 * shift in cells (the reference uses -0.5 along the component of a VX/VY/VZ
 * trace set, 0 otherwise; NULL = all 0).  map gets -1 where off the grid. */
rsgpu_status rsgpu_make_map(int dim, int precision, int ntr, const double *coords, const int *n, const double *o,
                            const double *d, const double *gshift, int *map, void *shift);

/* ---------------------------------------------------------------------------
 * Checkpoint schedule
 * ------------------------------------------------------------------------- */
/* Revolve<T>::revolve action trace for (nt, ncheck) (lib/revolve.cpp:150-305).
 * Writes up to max (action, capo, check) triples; returns the count through *n. */
rsgpu_status rsgpu_revolve_trace(int nt, int ncheck, int max, int *actions, int *capos, int *checks, int *n);
/* Revolve<T>::numforw (lib/revolve.cpp:31-62) */
int rsgpu_revolve_numforw(int nt, int ncheck);

#ifdef __cplusplus
}
#endif
#endif /* RSGPU_H */
