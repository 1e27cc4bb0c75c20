// 3D propagation: device descriptors and launchers (host runtime internals, not ABI).
//
// Device layout of one 3D shot: every field and parameter is a pitched array of
// planes with a zero guard of GUARD cells on every side in x and y and GUARD
// planes below and GUARD+2 above in z, so that a z-marching column with its
// 16-plane register window and its x/y halos never leaves the allocation.
//   element (ix, iy, iz) = origin[iz * plane + iy * pitch + ix],  plane = pitch * rows
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "rsgpu_internal.h"

namespace rsgpu {

constexpr int TX3 = 32;   // x columns per CTA (one warp row)
constexpr int TY3 = 8;    // y rows per CTA
constexpr int WX3 = TX3 + 16, HY3 = TY3 + 16;   // a tile with its 8-cell x or y halos

enum { A3_P = 0, A3_VX = 1, A3_VY = 2, A3_VZ = 3 };
enum { M3_RX = 0, M3_RY = 1, M3_RZ = 2, M3_L = 3 };
// Elastic 3D field slots (the reference's rs_field codes minus one) and parameters
// (the rsgpu_shot.model order: ModelElastic3D::staggerModels, lib/model.cpp:3371).
enum { E3_VX = 0, E3_VY = 1, E3_VZ = 2, E3_SXX = 3, E3_SYY = 4, E3_SZZ = 5, E3_SYZ = 6, E3_SXZ = 7, E3_SXY = 8 };
enum { ME_RX = 0, ME_RY = 1, ME_RZ = 2, ME_L = 3, ME_L2M = 4, ME_MYZ = 5, ME_MXZ = 6, ME_MXY = 7 };

template <typename T>
struct Shot3D {
    int nxp, nyp, nzp, pitch;
    int rows, lpml, fs, pad_;
    long long plane;          // elements per plane
    T *f[9];                  // acoustic: P, Vx, Vy, Vz; elastic: E3_* slots
    const T *m[8];            // acoustic: Rx, Ry, Rz, L; elastic: ME_* slots
    // C-PML memory per face pair, x [nzp][nyp][2L], y [nzp][2L][nxp], z [2L][nyp][nxp].
    // Acoustic: [0] velocity step (P derivatives), [1] stress step.  Elastic: [0..2]
    // the velocity step's Vx, Vy, Vz updates, [3] the normal stresses, [4] Sxz (x, z),
    // Syz (y) ... see fd3d_elastic.cu for the assignment of each update.
    T *psix[6], *psiy[6], *psiz[6];
};

// Tensor maps of the acoustic 3D TMA kernels (FAST), per shot, over whole pitched
// arrays like the elastic ones:
//   velocity: P {48 x 24} (x and y halos); Vx, Vy, Vz, Rx, Ry, Rz {32 x 8}
//   stress:   Vx {48 x 8} (x halo); Vy {32 x 24} (y halo); P, L {32 x 8}
enum {
    AM_PH = 0, AM_VX, AM_VY, AM_VZ, AM_RX, AM_RY, AM_RZ, AM_VXH, AM_VYH, AM_P, AM_L,
    NMAP_A3
};

// Work arrays of the elastic adjoint velocity step (FAST): per shot the allocation
// bases of the six stresses (Sxx, Syy, Szz, Syz, Sxz, Sxy), of L, L2M, M_yz, M_xz,
// M_xy, of the six work arrays in the same order, and the elements of one field
// allocation (a multiple of 4; every base 16-byte aligned).
struct WorkE3 {
    const float *s[6];
    const float *l, *l2m, *myz, *mxz, *mxy;
    float *w[6];
    long long n;
};
cudaError_t launch_work_e3d(const void *desc, int nshots, cudaStream_t st);

// One CTA: a TX3 x TY3 column block of one shot, marching planes [z0, z0 + zc).
struct Tile3D {
    int shot, x0, y0, z0;
};

template <typename T>
struct Step3DArgs {
    // the full-order coefficient rows of x, y and z (row `order` of CoefSet3; fast
    // mode: pre-divided by the spacing), kept in the launch's parameter space so
    // that the taps take them as constant operands; cf2 holds each value twice
    // (the operand of a paired f32x2 multiply-add)
    alignas(16) T cf2[3][NCOEF][2];
    T cf[3][NCOEF];
    const Shot3D<T> *shots;
    const Tile3D *tiles;
    int ntiles, order, zc, lpml;
    T dt, dx, dy, dz;
    T rdx, rdy, rdz;
    const T *pml;
    const void *maps;          // elastic fast mode: NMAP_E3 CUtensorMaps per shot (null: no TMA kernels)
    int *err;                  // device error word (a bounded wait that gave up)
};

// Tensor maps of the elastic 3D TMA kernels, per shot: 2D maps over a whole
// pitched array (pitch x rows*planes) with the box each staged tile needs.
//   velocity: Sxx, Sxz {48 x 8} (x halo); Sxy {48 x 24} (x and y halos);
//             Syy, Syz {32 x 24} (y halo); Vx, Vy, Vz, Rx, Ry, Rz {32 x 8}
//   stress:   Vx, Vy, Vz {48 x 24}; the six stresses and L, L2M, M_yz, M_xz, M_xy {32 x 8}
enum {
    VM_SXX = 0, VM_SXZ, VM_SXY, VM_SYY, VM_SYZ, VM_VX, VM_VY, VM_VZ, VM_RX, VM_RY, VM_RZ,
    SM_VX, SM_VY, SM_VZ, SM_SXX, SM_SYY, SM_SZZ, SM_SYZ, SM_SXZ, SM_SXY, SM_L, SM_L2M, SM_MYZ, SM_MXZ, SM_MXY,
    NMAP_E3
};

constexpr int CROW3 = 9;
template <typename T>
struct CoefSet3 {
    T cx[9 * CROW3];
    T cy[9 * CROW3];
    T cz[9 * CROW3];
};

// Source injection / receiver recording (trilinear, 8 corners), one CTA per shot.
// Contributions are kept in the reference's loop order: trace, z, y, x corner.
template <typename T>
struct InjRec3 {
    int ninj, kind_inj;
    const long long *inj_pt;   // [ninj] element offset from the field origin
    const int *inj_start;      // [ninj+1]
    const int *inj_trace;      // [ncontrib]
    const T *inj_w;            // [ncontrib][3] x, y, z weights
    const T *wav;              // [ntr * nt]
    int nrec, kind_rec;
    const long long *rec_pt;   // [nrec] offset of the (x0, y0, z0) corner, -1 off the grid
    const T *rec_w;            // [nrec][6] x0 x1 y0 y1 z0 z1
    T *rec_out;                // [nrec * nt], accumulated
    int nt;
    int rev;                   // 1: step it reads wav[nt-1-it] and writes rec_out[nt-1-it]
    const int *rec_gate;       // if non-null, recording happens only while *rec_gate != 0
    const T *rec_factor;       // elastic pressure: per-receiver divisor (3*rho*vp^2 - 4*rho*vs^2)/3
};
enum { INJ3_NONE = 0, INJ3_P = 1, INJ3_VX = 2, INJ3_VY = 3, INJ3_VZ = 4 };
enum { REC3_NONE = 0, REC3_P = 1, REC3_VX = 2, REC3_VY = 3, REC3_VZ = 4,
       // elastic 3D wavelet gradient (FwiElastic3D::crossCorr, lib/fwi.cpp:5217-5258):
       // out[it] = value at the map point (rec_pt) of Sxx + Syy + Szz, or the average
       // of the velocity and its lower neighbour along its own axis
       REC3_WG_P = 5, REC3_WG_VX = 6, REC3_WG_VY = 7, REC3_WG_VZ = 8 };

cudaError_t launch_step_3d(int prec, int physics, int half, const void *args, const void *coefs, int grid,
                           cudaStream_t st);
// Elastic 3D half-steps (fd3d_elastic.cu); adj selects backwardstepVelocity/Stress.
cudaError_t launch_step_e3d(int prec, int half, int adj, const void *args, const void *coefs, int grid,
                            cudaStream_t st);
// Elastic 3D injection then recording, one CTA per shot: plans[shot*nsets + k]
// holds source set k and receiver set k; every set is injected, then every set
// recorded.
cudaError_t launch_injrec_e3d(int prec, const void *shots, const void *plans, int nshots, int nsets, double dt,
                              int it, cudaStream_t st);
cudaError_t launch_injrec_3d(int prec, const void *shots, const void *plans, int nshots, double dt, int it,
                             cudaStream_t st);

}  // namespace rsgpu
