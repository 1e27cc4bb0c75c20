// Internal declarations shared by the CUDA translation units and the host runtime
// of librsgpu.  Nothing here crosses the C ABI (include/rsgpu.h is the boundary).
//
// Device layout of one shot ("window") of a batch
// -----------------------------------------------
// Every field and parameter of a shot is a pitched 2D (or 3D) array with a zero
// guard margin of GUARD cells on every side, so that a tile with its halo never
// reads outside the allocation and the stencil needs no bounds checks.  The
// guard cells are never written; the reference's reduced-order stencil near the
// array ends is reproduced with per-point coefficient rows whose unused taps are
// zero, so the guard values never reach a result.
//
//   element (ix, iz) of field f  =  f.origin[iz * pitch + ix]      (2D)
//   element (ix, iy, iz)         =  f.origin[(iz * nyp_alloc + iy) * pitch + ix]  (3D)
//
// pitch is a multiple of 4 elements and origin is 16-byte aligned, so quads of
// four x-neighbours are loaded as one vector.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace rsgpu {

constexpr int GUARD = 8;      // halo of the 16-tap staggered stencil (order 8)
constexpr int NCOEF = 8;      // taps per side of the widest stencil

// Field slots.  Acoustic 2D: P, Vx, Vz.  Elastic 2D: Vx, Vz, Sxx, Szz, Sxz.
enum { A2_P = 0, A2_VX = 1, A2_VZ = 2 };
enum { E2_VX = 0, E2_VZ = 1, E2_SXX = 2, E2_SZZ = 3, E2_SXZ = 4 };
// Parameter slots.  Acoustic: Rx, Rz, L.  Elastic: Rx, Rz, L, L2M, M.
enum { M_RX = 0, M_RZ = 1, M_L = 2, M_L2M = 3, M_M = 4 };

// Per-shot descriptor read by the 2D kernels.  psix arrays are [nzp][2*lpml]
// (left strip columns 0..lpml-1, right strip columns lpml..2*lpml-1);
// psiz arrays are [2*lpml][nxp] (top rows, then bottom rows).
template <typename T>
struct Shot2D {
    int nxp, nzp, pitch, lpml;
    int fs;            // free surface flag (elastic: Szz = 0 on row lpml)
    int pad_[3];
    T *f[5];
    const T *m[5];
    T *psix[4];
    T *psiz[4];
    // Second copy of the wavefields and of the velocity C-PML memory (psix/psiz 0
    // and 1) for the fused z-marching step kernel, which reads one copy and writes
    // the other (null when the plan does not use it).
    T *fb[5];
    T *psixb[2];
    T *psizb[2];
};

// One CTA work item: shot index, tile origin and flags.
struct Tile2D {
    int shot, x0, z0, flags;
};
enum {
    TILE_XEDGE = 1,   // some x-point of the tile is within `order` of an array end
    TILE_ZEDGE = 2,
    TILE_XPML = 4,    // tile intersects the left/right C-PML strips
    TILE_ZPML = 8,
    TILE_FSROW = 16,  // tile contains the free-surface row
};

// PML tables on the device: 12 arrays of lpml entries, in the order
// A,B,C ltf; A,B,C ltf_stag; A,B,C rbb; A,B,C rbb_stag.
enum { PT_A = 0, PT_B = 1, PT_C = 2 };
enum { PT_LTF = 0, PT_LTF_STAG = 3, PT_RBB = 6, PT_RBB_STAG = 9 };

// Source injection / receiver recording plan for one shot (all device pointers).
// A shot has up to MAXSETS source sets and MAXSETS receiver sets (e.g. the P, Vx
// and Vz residuals an elastic adjoint injects, or the three data types its forward
// records).  Injection: per set a CSR list over unique target points,
// contributions in the reference's loop order (trace, then z-corner, then
// x-corner), so that several traces hitting one cell add in the same order as on
// the CPU.  Sets are injected one after another, then recorded.
constexpr int MAXSETS = 3;
template <typename T>
struct InjSet {
    int ninj;               // unique injection target points
    int kind;               // see InjKind
    const int *pt;          // [ninj] linear offset (iz*pitch + ix) from field origin
    const int *start;       // [ninj+1] CSR into contributions
    const int *trace;       // [ncontrib] trace index
    const T *wx;            // [ncontrib] xtri weight (1 - shift.x or shift.x)
    const T *wz;            // [ncontrib] ytri weight
    const T *wav;           // [ntr * nt] trace-major wavelet / residual
};
template <typename T>
struct RecSet {
    int nrec;               // receiver traces
    int kind;               // see RecKind
    const int *pt;          // [nrec] offset of the (ix,iz) corner, or -1 if off-grid
    const T *w;             // [nrec*4] weights x0, x1, z0, z1
    const T *factor;        // [nrec] reciprocity divisor for elastic pressure
    T *out;                 // [nrec * nt] trace-major output (accumulated with +=)
};
template <typename T>
struct InjRec {
    int ninjsets, nrecsets;
    int nt;
    int rev;                // 1: step `it` reads wav[nt-1-it] and writes out[nt-1-it]
                            //    (adjoint propagation run forward in reversed time)
    const int *rec_gate;    // if non-null, recording happens only while *rec_gate != 0
    InjSet<T> inj[MAXSETS];
    RecSet<T> rec[MAXSETS];
};
enum InjKind {
    INJ_NONE = 0,
    INJ_A2_P = 1,     // P   += dt*L *w   (acoustic pressure source)
    INJ_A2_VX = 2,    // Vx  += dt*Rx*w
    INJ_A2_VZ = 3,    // Vz  += dt*Rz*w
    INJ_E2_P = 4,     // Sxx -= dt*w ; Szz -= dt*w  (elastic explosive source)
    INJ_E2_VX = 5,
    INJ_E2_VZ = 6,
};
enum RecKind {
    REC_NONE = 0,
    REC_A2_P = 1, REC_A2_VX = 2, REC_A2_VZ = 3,
    REC_E2_P = 4, REC_E2_VX = 5, REC_E2_VZ = 6,
    REC_E2_PSUM = 7,  // xtri*ytri*(Sxx + Szz) in T: the elastic wavelet gradient (lib/fwi.cpp:2681-2697)
};

// Arguments of one 2D half-step launch (passed by value).
template <typename T>
struct Step2DArgs {
    const Shot2D<T> *shots;
    const Tile2D *tiles;
    int ntiles;
    int order;
    T dt, dx, dz;
    T rdx, rdz;        // RN(1/dx), RN(1/dz): reciprocal-division mode only
    const T *pml;      // 12*lpml C-PML tables
    int lpml;
};

// ---- fused z-marching 2D step (fd2d_fused.cuh)
// One work item: rows [z0, z1) (multiples of 8) of the strip [x0, x0+TX) of a shot,
// and its injection entries per trace set, ie[s]..ie[s+1] in the item entry list.
struct ZmItem {
    int shot, x0, z0, z1, flags;
    int ie[MAXSETS + 1];
};
enum { ZM_XEDGE = 1, ZM_ZEDGE = 2, ZM_XPML = 4, ZM_ZPML = 8 };

template <typename T>
struct Zm2DArgs {
    const Shot2D<T> *shots;
    const InjRec<T> *plans;       // per shot (injection and recording sets)
    const ZmItem *items;
    int nitems;
    const int *inj;               // item injection entries: (set << 24) | CSR index
    const int4 *recs;             // every receiver trace of the batch: (shot, set, trace, 0)
    int nrecs;
    const void *maps;             // CUtensorMap [shot][copy][ring field]
    int order;
    T dt, dx, dz;
    T rdx, rdz;
    const T *pml;                 // 12*lpml C-PML tables
    int lpml;
};

// ---- column-marching elastic 2D half-steps (fd2d_march.cu, launch mode 4)
// One work item: rows [z0, z1) of the strip [x0, x0 + MSTRIP2D) of a shot.
constexpr int MSTRIP2D = 128;
struct MarchItem {
    int shot, x0, z0, z1, flags;
};
enum { MARCH_XGEN = 1 };   // the strip holds C-PML or reduced-order columns
struct March2DArgs {
    const Shot2D<float> *shots;
    const MarchItem *items;
    const void *maps;             // CUtensorMap [shot][NMAP2D] with box (MSTRIP2D + 16) x 8 rows
    const float *pml;             // 12*lpml C-PML tables
    const float *coefs;           // CoefSet<float> (per-K rows, divided by the spacing)
    int *err;                     // device error word (bounded waits)
    int order, lpml;
    float dt;
    float cx[NCOEF], cz[NCOEF];   // the full-order rows of coefs
};

}  // namespace rsgpu
