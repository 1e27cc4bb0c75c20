// Elastic 3D staggered-grid propagator (WavesElastic3D, lib/waves.cpp:2465-4400).
//
// Nine fields (Vx, Vy, Vz, Sxx, Syy, Szz, Syz, Sxz, Sxy), eight staggered
// parameters (Rx, Ry, Rz, L, L2M, M_yz, M_xz, M_xy).  As in the acoustic 3D
// kernels (fd3d.cu) each CTA owns a TX3 x TY3 block of (x, y) columns of one shot
// and marches a chunk of z planes; per plane:
//   - z-derivatives come from 16-plane register windows per column;
//   - x- and y-derivatives from the current plane's operands staged in shared
//     memory with an 8-cell halo on the axes they are differentiated along;
//   - the C-PML memory update and correction of every derivative is fused.
// The adjoint steps (backwardstepVelocity / backwardstepStress, lib/waves.cpp:
// 3260-4104) are the same kernels with other operands: the velocity step
// differentiates the work arrays L2M*Sxx + L*Syy + L*Szz, ..., M_xy*Sxy, ...
// (formed on the fly from the stresses and moduli), and the stress step adds
// dt*derivative without the moduli, each normal stress taking one derivative.
//
// Per point the operations follow the reference's order (x part, C-PML x, y part,
// C-PML y, z part, C-PML z per field; normal stresses share one memory per axis;
// free surface Szz = 0 on row lpml before the z memory), so MODE_IEEE reproduces
// the reference's float arithmetic bit for bit.  Assignment of the C-PML memory
// arrays (each used by exactly one update):
//   psix[0] Vx  (Sxx, staggered)   psiy[0] Vx  (Sxy)          psiz[0] Vx  (Sxz)
//   psix[1] Vy  (Sxy)              psiy[1] Vy  (Syy, stag.)   psiz[1] Vy  (Syz)
//   psix[2] Vz  (Sxz)              psiy[2] Vz  (Syz)          psiz[2] Vz  (Szz, stag.)
//   psix[3] normal stresses (Vx)   psiy[3] normal (Vy)        psiz[3] normal (Vz)
//   psix[4] Sxz (Vz, stag.)        psiy[4] Syz (Vz, stag.)    psiz[4] Sxz (Vx, stag.)
//   psix[5] Sxy (Vy, stag.)        psiy[5] Sxy (Vx, stag.)    psiz[5] Syz (Vy, stag.)
#include "fd2d_kernels.cuh"
#include "rsgpu_3d.h"

namespace rsgpu {
namespace {

template <typename T>
__device__ __forceinline__ void load_coefs3e(CoefSet3<T> &s, const CoefSet3<T> *g)
{
    const T *src = reinterpret_cast<const T *>(g);
    T *dst = reinterpret_cast<T *>(&s);
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    for (int i = tid; i < (int)(sizeof(CoefSet3<T>) / sizeof(T)); i += blockDim.x * blockDim.y) dst[i] = src[i];
}

// Copy the shot descriptor into shared memory: the field pointers are then read
// from a space that the kernel's global stores cannot alias, so the compiler may
// keep or re-read them freely instead of reloading them from global memory after
// every store.  Visible after the block's next barrier.
template <typename T>
__device__ __forceinline__ void stage_shot(Shot3D<T> &dst, const Shot3D<T> *src)
{
    constexpr int n = sizeof(Shot3D<T>) / sizeof(int);
    static_assert(sizeof(Shot3D<T>) % sizeof(int) == 0, "descriptor size");
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    if (tid < n) reinterpret_cast<int *>(&dst)[tid] = reinterpret_cast<const int *>(src)[tid];
}

// Staggered derivative with all NCOEF taps: b[0] = f[i-7] (forward) or f[i-8]
// (backward); sum_k (b[8+k] - b[7-k]) c_k in the reference's order.
template <typename T, int MODE>
__device__ __forceinline__ T taps3(const T *b, int s, const T *cu, T d, T r)
{
    using A = Ar<T, MODE>;
    T acc = A::mul(A::sub(b[8 * s], b[7 * s]), cu[0]);
#pragma unroll
    for (int k = 1; k < NCOEF; k++) acc = A::mad(acc, A::sub(b[(8 + k) * s], b[(7 - k) * s]), cu[k]);
    return (MODE == MODE_FAST) ? acc : A::div(acc, d, r);
}
template <typename T, int MODE>
__device__ __forceinline__ T taps3_reg(const T (&q)[16], const T *cu, T d, T r)
{
    using A = Ar<T, MODE>;
    T acc = A::mul(A::sub(q[8], q[7]), cu[0]);
#pragma unroll
    for (int k = 1; k < NCOEF; k++) acc = A::mad(acc, A::sub(q[8 + k], q[7 - k]), cu[k]);
    return (MODE == MODE_FAST) ? acc : A::div(acc, d, r);
}

// Operands of the velocity step: the stresses (forward) or the work arrays of
// backwardstepVelocity (lib/waves.cpp:3307, 3353, 3399, 3446, 3491, 3535, 3582,
// 3628, 3672), evaluated in the reference's expression order.
enum { OP_XX = 0, OP_YY = 1, OP_ZZ = 2, OP_XY = 3, OP_XZ = 4, OP_YZ = 5 };
template <typename T, int MODE, bool ADJ, typename I>
__device__ __forceinline__ T opnd(const Shot3D<T> &sh, I o, int kind)
{
    using A = Ar<T, MODE>;
    if (!ADJ) {
        const int f = kind == OP_XX ? E3_SXX : kind == OP_YY ? E3_SYY : kind == OP_ZZ ? E3_SZZ
                    : kind == OP_XY ? E3_SXY : kind == OP_XZ ? E3_SXZ : E3_SYZ;
        return sh.f[f][o];
    }
    if (kind == OP_XY) return A::mul(sh.m[ME_MXY][o], sh.f[E3_SXY][o]);
    if (kind == OP_XZ) return A::mul(sh.m[ME_MXZ][o], sh.f[E3_SXZ][o]);
    if (kind == OP_YZ) return A::mul(sh.m[ME_MYZ][o], sh.f[E3_SYZ][o]);
    const T l = sh.m[ME_L][o], l2m = sh.m[ME_L2M][o];
    const T sxx = sh.f[E3_SXX][o], syy = sh.f[E3_SYY][o], szz = sh.f[E3_SZZ][o];
    const T cx = kind == OP_XX ? l2m : l, cy = kind == OP_YY ? l2m : l, cz = kind == OP_ZZ ? l2m : l;
    return A::add(A::add(A::mul(cx, sxx), A::mul(cy, syy)), A::mul(cz, szz));
}

// Reduced-order z stencil reading the operands from global memory (the reference's
// rule near the array ends; rarely taken).
template <typename T, int MODE, bool ADJ>
__device__ __noinline__ T stencil_z_op(const Shot3D<T> &sh, long long o, long long plane, int K, const T *c, bool fw,
                                       int kind, T d, T r)
{
    using A = Ar<T, MODE>;
    if (K <= 0) return T(0);
    auto at = [&](int k) -> T { return opnd<T, MODE, ADJ>(sh, o + (long long)k * plane, kind); };
    T acc = A::mul(fw ? A::sub(at(1), at(0)) : A::sub(at(0), at(-1)), c[0]);
    for (int k = 1; k < K; k++) {
        const T dl = fw ? A::sub(at(k + 1), at(-k)) : A::sub(at(k), at(-k - 1));
        acc = A::mad(acc, dl, c[k]);
    }
    return (MODE == MODE_FAST) ? acc : A::div(acc, d, r);
}

// Shared-memory tiles of one plane: W = TX3 + 16 columns with an x halo, H = TY3 + 16
// rows with a y halo.
constexpr int WX = TX3 + 16, HY = TY3 + 16;

// ---------------------------------------------------------------- velocity step
// Vx += dt*Rx*(Dx+ XX) [x psi0 stag] + (Dy- XY) [y psi0] + (Dz- XZ) [z psi0]
// Vy += dt*Ry*(Dx- XY) [x psi1] + (Dy+ YY) [y psi1 stag] + (Dz- YZ) [z psi1]
// Vz += dt*Rz*(Dx- XZ) [x psi2] + (Dy- YZ) [y psi2] + (Dz+ ZZ) [z psi2 stag]
// (lib/waves.cpp:2465-2846; adjoint operands lib/waves.cpp:3260-3712)
template <typename T>
struct VelSmem {
    T xx[2][TY3][WX];     // XX operand, x halo
    T xy[2][HY][WX];      // XY operand, x and y halos
    T xz[2][TY3][WX];     // XZ operand, x halo
    T yy[2][HY][TX3];     // YY operand, y halo
    T yz[2][HY][TX3];     // YZ operand, y halo
    CoefSet3<T> cs;
};

template <typename T, int MODE, bool ADJ>
__global__ void __launch_bounds__(TX3 *TY3, 2) e3d_velocity(Step3DArgs<T> a, const CoefSet3<T> *coefs)
{
    using A = Ar<T, MODE>;
    extern __shared__ __align__(16) unsigned char smraw[];
    VelSmem<T> &S = *reinterpret_cast<VelSmem<T> *>(smraw);
    __shared__ Shot3D<T> shs;
    const Tile3D tl = a.tiles[blockIdx.x];
    stage_shot(shs, a.shots + tl.shot);
    load_coefs3e(S.cs, coefs);
    __syncthreads();
    const int tx = threadIdx.x, ty = threadIdx.y;
    const Shot3D<T> &sh = shs;
    const int ix = tl.x0 + tx, iy = tl.y0 + ty;
    const int nxp = sh.nxp, nyp = sh.nyp, nzp = sh.nzp, pitch = sh.pitch, L = a.lpml, order = a.order;
    const long long plane = sh.plane;
    const int col = iy * pitch + ix;
    T *Vx = sh.f[E3_VX], *Vy = sh.f[E3_VY], *Vz = sh.f[E3_VZ];
    const T *Rx = sh.m[ME_RX], *Ry = sh.m[ME_RY], *Rz = sh.m[ME_RZ];
    const bool in_grid = ix < nxp && iy < nyp;
    const int Kxf = kfw(ix, nxp, order), Kxb = kbw(ix, nxp, order);
    const int Kyf = kfw(iy, nyp, order), Kyb = kbw(iy, nyp, order);
    int xb = 0, xc = 0, yb = 0, yc = 0;
    const int xi = in_grid ? xstrip(ix, nxp, L, xb, xc) : -1;
    const int yi = in_grid ? xstrip(iy, nyp, L, yb, yc) : -1;
    const int z0 = tl.z0, ze = min(z0 + a.zc, nzp);
    const int hx = tx < 8 ? -8 : TX3 - 8;   // x halo column of threads tx < 16
    // z windows: XZ and YZ backward (planes z-8..z+7), ZZ forward (z-7..z+8)
    T qxz[16], qyz[16], qzz[16];
#pragma unroll
    for (int j = 0; j < 16; j++) {
        qxz[j] = opnd<T, MODE, ADJ>(sh, (long long)(z0 - 8 + j) * plane + col, OP_XZ);
        qyz[j] = opnd<T, MODE, ADJ>(sh, (long long)(z0 - 8 + j) * plane + col, OP_YZ);
        qzz[j] = opnd<T, MODE, ADJ>(sh, (long long)(z0 - 7 + j) * plane + col, OP_ZZ);
    }
    long long o = (long long)z0 * plane + col;
    T vx = Vx[o], vy = Vy[o], vz = Vz[o], rx = __ldg(Rx + o), ry = __ldg(Ry + o), rz = __ldg(Rz + o);
    T cxx = opnd<T, MODE, ADJ>(sh, o, OP_XX), cxy = opnd<T, MODE, ADJ>(sh, o, OP_XY), cyy = opnd<T, MODE, ADJ>(sh, o, OP_YY);
    T hxx = 0, hxy = 0, hxz = 0, vxy0 = 0, vxy1 = 0, vyy0 = 0, vyy1 = 0, vyz0 = 0, vyz1 = 0;
    if (tx < 16) {
        hxx = opnd<T, MODE, ADJ>(sh, o + hx, OP_XX);
        hxy = opnd<T, MODE, ADJ>(sh, o + hx, OP_XY);
        hxz = opnd<T, MODE, ADJ>(sh, o + hx, OP_XZ);
    }
    if (ty < 8) {
        vxy0 = opnd<T, MODE, ADJ>(sh, o - 8 * pitch, OP_XY); vxy1 = opnd<T, MODE, ADJ>(sh, o + TY3 * pitch, OP_XY);
        vyy0 = opnd<T, MODE, ADJ>(sh, o - 8 * pitch, OP_YY); vyy1 = opnd<T, MODE, ADJ>(sh, o + TY3 * pitch, OP_YY);
        vyz0 = opnd<T, MODE, ADJ>(sh, o - 8 * pitch, OP_YZ); vyz1 = opnd<T, MODE, ADJ>(sh, o + TY3 * pitch, OP_YZ);
    }
    const T *cux = a.cf[0], *cuy = a.cf[1], *cuz = a.cf[2];
    __syncthreads();
    for (int iz = z0; iz < ze; iz++, o += plane) {
        const int b = (iz - z0) & 1;
        S.xx[b][ty][tx + 8] = cxx;
        S.xy[b][ty + 8][tx + 8] = cxy;
        S.xz[b][ty][tx + 8] = qxz[8];
        S.yy[b][ty + 8][tx] = cyy;
        S.yz[b][ty + 8][tx] = qyz[8];
        if (tx < 16) {
            const int c = tx < 8 ? tx : tx + TX3;
            S.xx[b][ty][c] = hxx;
            S.xy[b][ty + 8][c] = hxy;
            S.xz[b][ty][c] = hxz;
        }
        if (ty < 8) {
            S.xy[b][ty][tx + 8] = vxy0; S.xy[b][ty + TY3 + 8][tx + 8] = vxy1;
            S.yy[b][ty][tx] = vyy0; S.yy[b][ty + TY3 + 8][tx] = vyy1;
            S.yz[b][ty][tx] = vyz0; S.yz[b][ty + TY3 + 8][tx] = vyz1;
        }
        // next plane's inputs (the plane after the chunk lies inside the allocation; unused)
        const long long on = o + plane;
        const T nvx = Vx[on], nvy = Vy[on], nvz = Vz[on];
        const T nrx = __ldg(Rx + on), nry = __ldg(Ry + on), nrz = __ldg(Rz + on);
        const T ncxx = opnd<T, MODE, ADJ>(sh, on, OP_XX), ncxy = opnd<T, MODE, ADJ>(sh, on, OP_XY),
                ncyy = opnd<T, MODE, ADJ>(sh, on, OP_YY);
        if (tx < 16) {
            hxx = opnd<T, MODE, ADJ>(sh, on + hx, OP_XX);
            hxy = opnd<T, MODE, ADJ>(sh, on + hx, OP_XY);
            hxz = opnd<T, MODE, ADJ>(sh, on + hx, OP_XZ);
        }
        if (ty < 8) {
            vxy0 = opnd<T, MODE, ADJ>(sh, on - 8 * pitch, OP_XY); vxy1 = opnd<T, MODE, ADJ>(sh, on + TY3 * pitch, OP_XY);
            vyy0 = opnd<T, MODE, ADJ>(sh, on - 8 * pitch, OP_YY); vyy1 = opnd<T, MODE, ADJ>(sh, on + TY3 * pitch, OP_YY);
            vyz0 = opnd<T, MODE, ADJ>(sh, on - 8 * pitch, OP_YZ); vyz1 = opnd<T, MODE, ADJ>(sh, on + TY3 * pitch, OP_YZ);
        }
        __syncthreads();
        const int Kzf = kfw(iz, nzp, order), Kzb = kbw(iz, nzp, order);
        int zb = 0, zc = 0;
        const int zi = in_grid ? xstrip(iz, nzp, L, zb, zc) : -1;
        const long long px = ((long long)iz * nyp + iy) * 2 * L + xc;
        const long long py = ((long long)iz * 2 * L + yc) * nxp + ix;
        const long long pz = ((long long)zc * nyp + iy) * nxp + ix;
        // ---- Vx
        {
            const T *c = &S.xx[b][ty][tx + 8];
            const T d1 = (Kxf == order) ? taps3<T, MODE>(c - 7, 1, cux, a.dx, a.rdx)
                                        : stencil_k<T, MODE>(c, 1, Kxf, S.cs.cx + Kxf * CROW3, true, a.dx, a.rdx);
            const T *cy = &S.xy[b][ty + 8][tx + 8];
            const T d2 = (Kyb == order) ? taps3<T, MODE>(cy - 8 * WX, WX, cuy, a.dy, a.rdy)
                                        : stencil_k<T, MODE>(cy, WX, Kyb, S.cs.cy + Kyb * CROW3, false, a.dy, a.rdy);
            const T d3 = (Kzb == order) ? taps3_reg<T, MODE>(qxz, cuz, a.dz, a.rdz)
                                        : stencil_z_op<T, MODE, ADJ>(sh, o, plane, Kzb, S.cs.cz + Kzb * CROW3, false, OP_XZ, a.dz, a.rdz);
            const T am = A::mul(a.dt, rx);
            vx = A::mad(vx, am, d1);
            if (xi >= 0) vx = pml_correct<T, MODE>(vx, am, d1, sh.psix[0] + px, a.pml, L, xb + 3, xi);
            vx = A::mad(vx, am, d2);
            if (yi >= 0) vx = pml_correct<T, MODE>(vx, am, d2, sh.psiy[0] + py, a.pml, L, yb, yi);
            vx = A::mad(vx, am, d3);
            if (zi >= 0) vx = pml_correct<T, MODE>(vx, am, d3, sh.psiz[0] + pz, a.pml, L, zb, zi);
            Vx[o] = vx;
        }
        // ---- Vy
        {
            const T *c = &S.xy[b][ty + 8][tx + 8];
            const T d1 = (Kxb == order) ? taps3<T, MODE>(c - 8, 1, cux, a.dx, a.rdx)
                                        : stencil_k<T, MODE>(c, 1, Kxb, S.cs.cx + Kxb * CROW3, false, a.dx, a.rdx);
            const T *cy = &S.yy[b][ty + 8][tx];
            const T d2 = (Kyf == order) ? taps3<T, MODE>(cy - 7 * TX3, TX3, cuy, a.dy, a.rdy)
                                        : stencil_k<T, MODE>(cy, TX3, Kyf, S.cs.cy + Kyf * CROW3, true, a.dy, a.rdy);
            const T d3 = (Kzb == order) ? taps3_reg<T, MODE>(qyz, cuz, a.dz, a.rdz)
                                        : stencil_z_op<T, MODE, ADJ>(sh, o, plane, Kzb, S.cs.cz + Kzb * CROW3, false, OP_YZ, a.dz, a.rdz);
            const T am = A::mul(a.dt, ry);
            vy = A::mad(vy, am, d1);
            if (xi >= 0) vy = pml_correct<T, MODE>(vy, am, d1, sh.psix[1] + px, a.pml, L, xb, xi);
            vy = A::mad(vy, am, d2);
            if (yi >= 0) vy = pml_correct<T, MODE>(vy, am, d2, sh.psiy[1] + py, a.pml, L, yb + 3, yi);
            vy = A::mad(vy, am, d3);
            if (zi >= 0) vy = pml_correct<T, MODE>(vy, am, d3, sh.psiz[1] + pz, a.pml, L, zb, zi);
            Vy[o] = vy;
        }
        // ---- Vz
        {
            const T *c = &S.xz[b][ty][tx + 8];
            const T d1 = (Kxb == order) ? taps3<T, MODE>(c - 8, 1, cux, a.dx, a.rdx)
                                        : stencil_k<T, MODE>(c, 1, Kxb, S.cs.cx + Kxb * CROW3, false, a.dx, a.rdx);
            const T *cy = &S.yz[b][ty + 8][tx];
            const T d2 = (Kyb == order) ? taps3<T, MODE>(cy - 8 * TX3, TX3, cuy, a.dy, a.rdy)
                                        : stencil_k<T, MODE>(cy, TX3, Kyb, S.cs.cy + Kyb * CROW3, false, a.dy, a.rdy);
            const T d3 = (Kzf == order) ? taps3_reg<T, MODE>(qzz, cuz, a.dz, a.rdz)
                                        : stencil_z_op<T, MODE, ADJ>(sh, o, plane, Kzf, S.cs.cz + Kzf * CROW3, true, OP_ZZ, a.dz, a.rdz);
            const T am = A::mul(a.dt, rz);
            vz = A::mad(vz, am, d1);
            if (xi >= 0) vz = pml_correct<T, MODE>(vz, am, d1, sh.psix[2] + px, a.pml, L, xb, xi);
            vz = A::mad(vz, am, d2);
            if (yi >= 0) vz = pml_correct<T, MODE>(vz, am, d2, sh.psiy[2] + py, a.pml, L, yb, yi);
            vz = A::mad(vz, am, d3);
            if (zi >= 0) vz = pml_correct<T, MODE>(vz, am, d3, sh.psiz[2] + pz, a.pml, L, zb + 3, zi);
            Vz[o] = vz;
        }
        // windows advance one plane
#pragma unroll
        for (int j = 0; j < 15; j++) { qxz[j] = qxz[j + 1]; qyz[j] = qyz[j + 1]; qzz[j] = qzz[j + 1]; }
        qxz[15] = opnd<T, MODE, ADJ>(sh, o + 8 * plane, OP_XZ);
        qyz[15] = opnd<T, MODE, ADJ>(sh, o + 8 * plane, OP_YZ);
        qzz[15] = opnd<T, MODE, ADJ>(sh, o + 9 * plane, OP_ZZ);
        vx = nvx; vy = nvy; vz = nvz; rx = nrx; ry = nry; rz = nrz;
        cxx = ncxx; cxy = ncxy; cyy = ncyy;
    }
}

// ---------------------------------------------------------------- stress step
// Forward (lib/waves.cpp:2849-3257):
//   Dx- Vx: Sxx += dt*L2M*d, Syy += dt*L*d, Szz += dt*L*d  [x psi3 shared]
//   Dy- Vy: Sxx += L, Syy += L2M, Szz += L                  [y psi3]
//   Dz- Vz: Sxx += L, Syy += L, Szz += L2M; free surface Szz = 0 on row lpml; [z psi3]
//   Sxz += dt*M_xz*(Dx+ Vz) [x psi4 stag] ; (Dz+ Vx) [z psi4 stag]
//   Syz += dt*M_yz*(Dz+ Vy) [z psi5 stag] ; (Dy+ Vz) [y psi4 stag]
//   Sxy += dt*M_xy*(Dy+ Vx) [y psi5 stag] ; (Dx+ Vy) [x psi5 stag]
// Adjoint (lib/waves.cpp:3715-4101): Sxx += dt*(Dx- Vx) [x psi3], Syy += dt*(Dy- Vy)
// [y psi3], Szz += dt*(Dz- Vz), free surface, [z psi3]; shear stresses as above
// with dt in place of dt*M.
template <typename T>
struct StrSmem {
    T vx[2][HY][WX];
    T vy[2][HY][WX];
    T vz[2][HY][WX];
    CoefSet3<T> cs;
};

template <typename T, int MODE, bool ADJ>
__global__ void __launch_bounds__(TX3 *TY3, 2) e3d_stress(Step3DArgs<T> a, const CoefSet3<T> *coefs)
{
    using A = Ar<T, MODE>;
    extern __shared__ __align__(16) unsigned char smraw[];
    StrSmem<T> &S = *reinterpret_cast<StrSmem<T> *>(smraw);
    __shared__ Shot3D<T> shs;
    const Tile3D tl = a.tiles[blockIdx.x];
    stage_shot(shs, a.shots + tl.shot);
    load_coefs3e(S.cs, coefs);
    __syncthreads();
    const int tx = threadIdx.x, ty = threadIdx.y;
    const Shot3D<T> &sh = shs;
    const int ix = tl.x0 + tx, iy = tl.y0 + ty;
    const int nxp = sh.nxp, nyp = sh.nyp, nzp = sh.nzp, pitch = sh.pitch, L = a.lpml, order = a.order;
    const long long plane = sh.plane;
    const int col = iy * pitch + ix;
    const T *Vx = sh.f[E3_VX], *Vy = sh.f[E3_VY], *Vz = sh.f[E3_VZ];
    T *Sxx = sh.f[E3_SXX], *Syy = sh.f[E3_SYY], *Szz = sh.f[E3_SZZ];
    T *Syz = sh.f[E3_SYZ], *Sxz = sh.f[E3_SXZ], *Sxy = sh.f[E3_SXY];
    const bool in_grid = ix < nxp && iy < nyp;
    const int Kxf = kfw(ix, nxp, order), Kxb = kbw(ix, nxp, order);
    const int Kyf = kfw(iy, nyp, order), Kyb = kbw(iy, nyp, order);
    int xb = 0, xc = 0, yb = 0, yc = 0;
    const int xi = in_grid ? xstrip(ix, nxp, L, xb, xc) : -1;
    const int yi = in_grid ? xstrip(iy, nyp, L, yb, yc) : -1;
    const int z0 = tl.z0, ze = min(z0 + a.zc, nzp);
    const int hx = tx < 8 ? -8 : TX3 - 8;
    // z windows: Vz backward (planes z-8..z+7), Vx and Vy forward (z-7..z+8)
    T qz[16], qx[16], qy[16];
#pragma unroll
    for (int j = 0; j < 16; j++) {
        qz[j] = Vz[(long long)(z0 - 8 + j) * plane + col];
        qx[j] = Vx[(long long)(z0 - 7 + j) * plane + col];
        qy[j] = Vy[(long long)(z0 - 7 + j) * plane + col];
    }
    long long o = (long long)z0 * plane + col;
    T sxx = Sxx[o], syy = Syy[o], szz = Szz[o], syz = Syz[o], sxz = Sxz[o], sxy = Sxy[o];
    T l = 0, l2m = 0, myz = 0, mxz = 0, mxy = 0;
    if (!ADJ) {
        l = __ldg(sh.m[ME_L] + o); l2m = __ldg(sh.m[ME_L2M] + o);
        myz = __ldg(sh.m[ME_MYZ] + o); mxz = __ldg(sh.m[ME_MXZ] + o); mxy = __ldg(sh.m[ME_MXY] + o);
    }
    T hvx = 0, hvy = 0, hvz = 0, yx0 = 0, yx1 = 0, yy0 = 0, yy1 = 0, yz0 = 0, yz1 = 0;
    if (tx < 16) { hvx = Vx[o + hx]; hvy = Vy[o + hx]; hvz = Vz[o + hx]; }
    if (ty < 8) {
        yx0 = Vx[o - 8 * pitch]; yx1 = Vx[o + TY3 * pitch];
        yy0 = Vy[o - 8 * pitch]; yy1 = Vy[o + TY3 * pitch];
        yz0 = Vz[o - 8 * pitch]; yz1 = Vz[o + TY3 * pitch];
    }
    const T *cux = a.cf[0], *cuy = a.cf[1], *cuz = a.cf[2];
    __syncthreads();
    for (int iz = z0; iz < ze; iz++, o += plane) {
        const int b = (iz - z0) & 1;
        S.vx[b][ty + 8][tx + 8] = qx[7];
        S.vy[b][ty + 8][tx + 8] = qy[7];
        S.vz[b][ty + 8][tx + 8] = qz[8];
        if (tx < 16) {
            const int c = tx < 8 ? tx : tx + TX3;
            S.vx[b][ty + 8][c] = hvx; S.vy[b][ty + 8][c] = hvy; S.vz[b][ty + 8][c] = hvz;
        }
        if (ty < 8) {
            S.vx[b][ty][tx + 8] = yx0; S.vx[b][ty + TY3 + 8][tx + 8] = yx1;
            S.vy[b][ty][tx + 8] = yy0; S.vy[b][ty + TY3 + 8][tx + 8] = yy1;
            S.vz[b][ty][tx + 8] = yz0; S.vz[b][ty + TY3 + 8][tx + 8] = yz1;
        }
        const long long on = o + plane;
        const T nsxx = Sxx[on], nsyy = Syy[on], nszz = Szz[on], nsyz = Syz[on], nsxz = Sxz[on], nsxy = Sxy[on];
        T nl = 0, nl2m = 0, nmyz = 0, nmxz = 0, nmxy = 0;
        if (!ADJ) {
            nl = __ldg(sh.m[ME_L] + on); nl2m = __ldg(sh.m[ME_L2M] + on);
            nmyz = __ldg(sh.m[ME_MYZ] + on); nmxz = __ldg(sh.m[ME_MXZ] + on); nmxy = __ldg(sh.m[ME_MXY] + on);
        }
        if (tx < 16) { hvx = Vx[on + hx]; hvy = Vy[on + hx]; hvz = Vz[on + hx]; }
        if (ty < 8) {
            yx0 = Vx[on - 8 * pitch]; yx1 = Vx[on + TY3 * pitch];
            yy0 = Vy[on - 8 * pitch]; yy1 = Vy[on + TY3 * pitch];
            yz0 = Vz[on - 8 * pitch]; yz1 = Vz[on + TY3 * pitch];
        }
        __syncthreads();
        const int Kzf = kfw(iz, nzp, order), Kzb = kbw(iz, nzp, order);
        int zb = 0, zc = 0;
        const int zi = in_grid ? xstrip(iz, nzp, L, zb, zc) : -1;
        const long long px = ((long long)iz * nyp + iy) * 2 * L + xc;
        const long long py = ((long long)iz * 2 * L + yc) * nxp + ix;
        const long long pz = ((long long)zc * nyp + iy) * nxp + ix;
        const T *cvx = &S.vx[b][ty + 8][tx + 8], *cvy = &S.vy[b][ty + 8][tx + 8], *cvz = &S.vz[b][ty + 8][tx + 8];
        // ---- normal stresses
        {
            const T dxx = (Kxb == order) ? taps3<T, MODE>(cvx - 8, 1, cux, a.dx, a.rdx)
                                         : stencil_k<T, MODE>(cvx, 1, Kxb, S.cs.cx + Kxb * CROW3, false, a.dx, a.rdx);
            const T dyy = (Kyb == order) ? taps3<T, MODE>(cvy - 8 * WX, WX, cuy, a.dy, a.rdy)
                                         : stencil_k<T, MODE>(cvy, WX, Kyb, S.cs.cy + Kyb * CROW3, false, a.dy, a.rdy);
            const T dzz = (Kzb == order) ? taps3_reg<T, MODE>(qz, cuz, a.dz, a.rdz)
                                         : stencil_k<T, MODE>(Vz + o, (int)plane, Kzb, S.cs.cz + Kzb * CROW3, false, a.dz, a.rdz);
            const bool fsrow = sh.fs && iz == L;
            if (!ADJ) {
                const T a2 = A::mul(a.dt, l2m), a1 = A::mul(a.dt, l);
                auto upd3 = [&](T d, T cxx_, T cyy_, T czz_) {
                    sxx = A::mad(sxx, cxx_, d); syy = A::mad(syy, cyy_, d); szz = A::mad(szz, czz_, d);
                };
                auto pml3 = [&](T d, T *psi, int base, int idx, T cxx_, T cyy_, T czz_) {
                    const T tA = __ldg(a.pml + (base + PT_A) * L + idx), tB = __ldg(a.pml + (base + PT_B) * L + idx),
                            tC = __ldg(a.pml + (base + PT_C) * L + idx);
                    const T p = A::mad(A::mul(tB, *psi), tA, d);
                    *psi = p;
                    const T cq = A::mad(p, tC, d);
                    sxx = A::msub(sxx, cxx_, cq); syy = A::msub(syy, cyy_, cq); szz = A::msub(szz, czz_, cq);
                };
                upd3(dxx, a2, a1, a1);
                if (xi >= 0) pml3(dxx, sh.psix[3] + px, xb, xi, a2, a1, a1);
                upd3(dyy, a1, a2, a1);
                if (yi >= 0) pml3(dyy, sh.psiy[3] + py, yb, yi, a1, a2, a1);
                upd3(dzz, a1, a1, a2);
                if (fsrow) szz = T(0);
                if (zi >= 0) pml3(dzz, sh.psiz[3] + pz, zb, zi, a1, a1, a2);
            } else {
                sxx = A::mad(sxx, a.dt, dxx);
                if (xi >= 0) sxx = pml_correct<T, MODE>(sxx, a.dt, dxx, sh.psix[3] + px, a.pml, L, xb, xi);
                syy = A::mad(syy, a.dt, dyy);
                if (yi >= 0) syy = pml_correct<T, MODE>(syy, a.dt, dyy, sh.psiy[3] + py, a.pml, L, yb, yi);
                szz = A::mad(szz, a.dt, dzz);
                if (fsrow) szz = T(0);
                if (zi >= 0) szz = pml_correct<T, MODE>(szz, a.dt, dzz, sh.psiz[3] + pz, a.pml, L, zb, zi);
            }
            Sxx[o] = sxx; Syy[o] = syy; Szz[o] = szz;
        }
        // ---- Sxz: Dx+ Vz, Dz+ Vx
        {
            const T d1 = (Kxf == order) ? taps3<T, MODE>(cvz - 7, 1, cux, a.dx, a.rdx)
                                        : stencil_k<T, MODE>(cvz, 1, Kxf, S.cs.cx + Kxf * CROW3, true, a.dx, a.rdx);
            const T d2 = (Kzf == order) ? taps3_reg<T, MODE>(qx, cuz, a.dz, a.rdz)
                                        : stencil_k<T, MODE>(Vx + o, (int)plane, Kzf, S.cs.cz + Kzf * CROW3, true, a.dz, a.rdz);
            const T am = ADJ ? a.dt : A::mul(a.dt, mxz);
            sxz = A::mad(sxz, am, d1);
            if (xi >= 0) sxz = pml_correct<T, MODE>(sxz, am, d1, sh.psix[4] + px, a.pml, L, xb + 3, xi);
            sxz = A::mad(sxz, am, d2);
            if (zi >= 0) sxz = pml_correct<T, MODE>(sxz, am, d2, sh.psiz[4] + pz, a.pml, L, zb + 3, zi);
            Sxz[o] = sxz;
        }
        // ---- Syz: Dz+ Vy, Dy+ Vz
        {
            const T d1 = (Kzf == order) ? taps3_reg<T, MODE>(qy, cuz, a.dz, a.rdz)
                                        : stencil_k<T, MODE>(Vy + o, (int)plane, Kzf, S.cs.cz + Kzf * CROW3, true, a.dz, a.rdz);
            const T d2 = (Kyf == order) ? taps3<T, MODE>(cvz - 7 * WX, WX, cuy, a.dy, a.rdy)
                                        : stencil_k<T, MODE>(cvz, WX, Kyf, S.cs.cy + Kyf * CROW3, true, a.dy, a.rdy);
            const T am = ADJ ? a.dt : A::mul(a.dt, myz);
            syz = A::mad(syz, am, d1);
            if (zi >= 0) syz = pml_correct<T, MODE>(syz, am, d1, sh.psiz[5] + pz, a.pml, L, zb + 3, zi);
            syz = A::mad(syz, am, d2);
            if (yi >= 0) syz = pml_correct<T, MODE>(syz, am, d2, sh.psiy[4] + py, a.pml, L, yb + 3, yi);
            Syz[o] = syz;
        }
        // ---- Sxy: Dy+ Vx, Dx+ Vy
        {
            const T d1 = (Kyf == order) ? taps3<T, MODE>(cvx - 7 * WX, WX, cuy, a.dy, a.rdy)
                                        : stencil_k<T, MODE>(cvx, WX, Kyf, S.cs.cy + Kyf * CROW3, true, a.dy, a.rdy);
            const T d2 = (Kxf == order) ? taps3<T, MODE>(cvy - 7, 1, cux, a.dx, a.rdx)
                                        : stencil_k<T, MODE>(cvy, 1, Kxf, S.cs.cx + Kxf * CROW3, true, a.dx, a.rdx);
            const T am = ADJ ? a.dt : A::mul(a.dt, mxy);
            sxy = A::mad(sxy, am, d1);
            if (yi >= 0) sxy = pml_correct<T, MODE>(sxy, am, d1, sh.psiy[5] + py, a.pml, L, yb + 3, yi);
            sxy = A::mad(sxy, am, d2);
            if (xi >= 0) sxy = pml_correct<T, MODE>(sxy, am, d2, sh.psix[5] + px, a.pml, L, xb + 3, xi);
            Sxy[o] = sxy;
        }
#pragma unroll
        for (int j = 0; j < 15; j++) { qz[j] = qz[j + 1]; qx[j] = qx[j + 1]; qy[j] = qy[j + 1]; }
        qz[15] = Vz[o + 8 * plane];
        qx[15] = Vx[o + 9 * plane];
        qy[15] = Vy[o + 9 * plane];
        sxx = nsxx; syy = nsyy; szz = nszz; syz = nsyz; sxz = nsxz; sxy = nsxy;
        l = nl; l2m = nl2m; myz = nmyz; mxz = nmxz; mxy = nmxy;
    }
}

// ---------------------------------------------------------------- fast-mode kernels
// RSGPU_F32_FAST versions of the two half-steps: the same stencils, C-PML and
// update order, with derivatives that share an axis and a direction computed in
// pairs -- one 64-bit shared load and one FADD2/FFMA2 per tap for two fields -- and
// the full-order coefficients taken from the launch's parameter space.
//   velocity: x backward (XY, XZ), y backward (XY, YZ), z backward (XZ, YZ);
//             single: x forward XX, y forward YY, z forward ZZ
//   stress:   x forward (Vz, Vy), y forward (Vz, Vx), z forward (Vx, Vy);
//             single: x backward Vx, y backward Vy, z backward Vz
__device__ __forceinline__ float2 taps_pair(const float2 *b, int s, const float (&c2)[NCOEF][2])
{
    using A2 = Ar2<float, MODE_FAST>;
    const float2 *cc = reinterpret_cast<const float2 *>(c2);
    float2 acc = A2::mul(A2::sub(b[8 * s], b[7 * s]), cc[0]);
#pragma unroll
    for (int k = 1; k < NCOEF; k++) acc = A2::acc(acc, A2::sub(b[(8 + k) * s], b[(7 - k) * s]), cc[k]);
    return acc;
}
__device__ __forceinline__ float2 taps_pair_reg(const float2 (&q)[16], const float (&c2)[NCOEF][2])
{
    using A2 = Ar2<float, MODE_FAST>;
    const float2 *cc = reinterpret_cast<const float2 *>(c2);
    float2 acc = A2::mul(A2::sub(q[8], q[7]), cc[0]);
#pragma unroll
    for (int k = 1; k < NCOEF; k++) acc = A2::acc(acc, A2::sub(q[8 + k], q[7 - k]), cc[k]);
    return acc;
}

struct VelSmemF {
    float xx[2][TY3][WX];      // XX, x halo
    float2 xq[2][TY3][WX];     // (XY, XZ), x halo
    float2 yq[2][HY][TX3];     // (XY, YZ), y halo
    float yy[2][HY][TX3];      // YY, y halo
    CoefSet3<float> cs;
};

template <bool ADJ>
__global__ void __launch_bounds__(TX3 *TY3, 2) e3d_velocity_fast(Step3DArgs<float> a, const CoefSet3<float> *coefs)
{
    using T = float;
    constexpr int MODE = MODE_FAST;
    using A = Ar<T, MODE>;
    extern __shared__ __align__(16) unsigned char smraw[];
    VelSmemF &S = *reinterpret_cast<VelSmemF *>(smraw);
    __shared__ Shot3D<T> shs;
    const Tile3D tl = a.tiles[blockIdx.x];
    stage_shot(shs, a.shots + tl.shot);
    load_coefs3e(S.cs, coefs);
    __syncthreads();
    const int tx = threadIdx.x, ty = threadIdx.y;
    const Shot3D<T> &sh = shs;
    const int ix = tl.x0 + tx, iy = tl.y0 + ty;
    const int nxp = sh.nxp, nyp = sh.nyp, nzp = sh.nzp, pitch = sh.pitch, L = a.lpml, order = a.order;
    const int plane = (int)sh.plane;   // a field holds fewer than 2^31 elements
    const int col = iy * pitch + ix;
    T *Vx = sh.f[E3_VX], *Vy = sh.f[E3_VY], *Vz = sh.f[E3_VZ];
    const T *Rx = sh.m[ME_RX], *Ry = sh.m[ME_RY], *Rz = sh.m[ME_RZ];
    const bool in_grid = ix < nxp && iy < nyp;
    const int Kxf = kfw(ix, nxp, order), Kxb = kbw(ix, nxp, order);
    const int Kyf = kfw(iy, nyp, order), Kyb = kbw(iy, nyp, order);
    int xb = 0, xc = 0, yb = 0, yc = 0;
    const int xi = in_grid ? xstrip(ix, nxp, L, xb, xc) : -1;
    const int yi = in_grid ? xstrip(iy, nyp, L, yb, yc) : -1;
    const int z0 = tl.z0, ze = min(z0 + a.zc, nzp);
    const int hx = tx < 8 ? -8 : TX3 - 8;
    // z windows: (XZ, YZ) backward (planes z-8..z+7), ZZ forward (z-7..z+8)
    float2 qp[16];
    T qzz[16];
#pragma unroll
    for (int j = 0; j < 16; j++) {
        const int oj = (z0 - 8 + j) * plane + col;
        qp[j] = make_float2(opnd<T, MODE, ADJ>(sh, oj, OP_XZ), opnd<T, MODE, ADJ>(sh, oj, OP_YZ));
        qzz[j] = opnd<T, MODE, ADJ>(sh, (z0 - 7 + j) * plane + col, OP_ZZ);
    }
    int o = z0 * plane + col;
    T vx = Vx[o], vy = Vy[o], vz = Vz[o], rx = __ldg(Rx + o), ry = __ldg(Ry + o), rz = __ldg(Rz + o);
    T cxx = opnd<T, MODE, ADJ>(sh, o, OP_XX), cxy = opnd<T, MODE, ADJ>(sh, o, OP_XY), cyy = opnd<T, MODE, ADJ>(sh, o, OP_YY);
    T hxx = 0, hxy = 0, hxz = 0;
    if (tx < 16) {
        hxx = opnd<T, MODE, ADJ>(sh, o + hx, OP_XX);
        hxy = opnd<T, MODE, ADJ>(sh, o + hx, OP_XY);
        hxz = opnd<T, MODE, ADJ>(sh, o + hx, OP_XZ);
    }
    T vxy0 = opnd<T, MODE, ADJ>(sh, o - 8 * pitch, OP_XY), vxy1 = opnd<T, MODE, ADJ>(sh, o + TY3 * pitch, OP_XY);
    T vyy0 = opnd<T, MODE, ADJ>(sh, o - 8 * pitch, OP_YY), vyy1 = opnd<T, MODE, ADJ>(sh, o + TY3 * pitch, OP_YY);
    T vyz0 = opnd<T, MODE, ADJ>(sh, o - 8 * pitch, OP_YZ), vyz1 = opnd<T, MODE, ADJ>(sh, o + TY3 * pitch, OP_YZ);
    __syncthreads();
    for (int iz = z0; iz < ze; iz++, o += plane) {
        const int b = (iz - z0) & 1;
        S.xx[b][ty][tx + 8] = cxx;
        S.xq[b][ty][tx + 8] = make_float2(cxy, qp[8].x);
        S.yq[b][ty + 8][tx] = make_float2(cxy, qp[8].y);
        S.yy[b][ty + 8][tx] = cyy;
        if (tx < 16) {
            const int c = tx < 8 ? tx : tx + TX3;
            S.xx[b][ty][c] = hxx;
            S.xq[b][ty][c] = make_float2(hxy, hxz);
        }
        S.yq[b][ty][tx] = make_float2(vxy0, vyz0);
        S.yq[b][ty + TY3 + 8][tx] = make_float2(vxy1, vyz1);
        S.yy[b][ty][tx] = vyy0;
        S.yy[b][ty + TY3 + 8][tx] = vyy1;
        // next plane's inputs (the plane after the chunk lies inside the allocation; unused)
        const int on = o + plane;
        const T nvx = Vx[on], nvy = Vy[on], nvz = Vz[on];
        const T nrx = __ldg(Rx + on), nry = __ldg(Ry + on), nrz = __ldg(Rz + on);
        const T ncxx = opnd<T, MODE, ADJ>(sh, on, OP_XX), ncxy = opnd<T, MODE, ADJ>(sh, on, OP_XY),
                ncyy = opnd<T, MODE, ADJ>(sh, on, OP_YY);
        if (tx < 16) {
            hxx = opnd<T, MODE, ADJ>(sh, on + hx, OP_XX);
            hxy = opnd<T, MODE, ADJ>(sh, on + hx, OP_XY);
            hxz = opnd<T, MODE, ADJ>(sh, on + hx, OP_XZ);
        }
        vxy0 = opnd<T, MODE, ADJ>(sh, on - 8 * pitch, OP_XY); vxy1 = opnd<T, MODE, ADJ>(sh, on + TY3 * pitch, OP_XY);
        vyy0 = opnd<T, MODE, ADJ>(sh, on - 8 * pitch, OP_YY); vyy1 = opnd<T, MODE, ADJ>(sh, on + TY3 * pitch, OP_YY);
        vyz0 = opnd<T, MODE, ADJ>(sh, on - 8 * pitch, OP_YZ); vyz1 = opnd<T, MODE, ADJ>(sh, on + TY3 * pitch, OP_YZ);
        __syncthreads();
        const int Kzf = kfw(iz, nzp, order), Kzb = kbw(iz, nzp, order);
        int zb = 0, zc = 0;
        const int zi = in_grid ? xstrip(iz, nzp, L, zb, zc) : -1;
        const int px = (iz * nyp + iy) * 2 * L + xc;
        const int py = (iz * 2 * L + yc) * nxp + ix;
        const int pz = (zc * nyp + iy) * nxp + ix;
        // full-order derivatives, then the reduced-order ones near the array ends
        const T *cx1 = &S.xx[b][ty][tx + 8];
        T dxx = taps3<T, MODE>(cx1 - 7, 1, a.cf[0], a.dx, a.rdx);
        const float2 *cxq = &S.xq[b][ty][tx + 8];
        float2 dxq = taps_pair(cxq - 8, 1, a.cf2[0]);
        const float2 *cyq = &S.yq[b][ty + 8][tx];
        float2 dyq = taps_pair(cyq - 8 * TX3, TX3, a.cf2[1]);
        const T *cy1 = &S.yy[b][ty + 8][tx];
        T dyy = taps3<T, MODE>(cy1 - 7 * TX3, TX3, a.cf[1], a.dy, a.rdy);
        float2 dzq = taps_pair_reg(qp, a.cf2[2]);
        T dzz = taps3_reg<T, MODE>(qzz, a.cf[2], a.dz, a.rdz);
        if (Kxf != order) dxx = stencil_k<T, MODE>(cx1, 1, Kxf, S.cs.cx + Kxf * CROW3, true, a.dx, a.rdx);
        if (Kxb != order) {
            const T *c = reinterpret_cast<const T *>(cxq);
            dxq.x = stencil_k<T, MODE>(c, 2, Kxb, S.cs.cx + Kxb * CROW3, false, a.dx, a.rdx);
            dxq.y = stencil_k<T, MODE>(c + 1, 2, Kxb, S.cs.cx + Kxb * CROW3, false, a.dx, a.rdx);
        }
        if (Kyb != order) {
            const T *c = reinterpret_cast<const T *>(cyq);
            dyq.x = stencil_k<T, MODE>(c, 2 * TX3, Kyb, S.cs.cy + Kyb * CROW3, false, a.dy, a.rdy);
            dyq.y = stencil_k<T, MODE>(c + 1, 2 * TX3, Kyb, S.cs.cy + Kyb * CROW3, false, a.dy, a.rdy);
        }
        if (Kyf != order) dyy = stencil_k<T, MODE>(cy1, TX3, Kyf, S.cs.cy + Kyf * CROW3, true, a.dy, a.rdy);
        if (Kzb != order) {
            dzq.x = stencil_z_op<T, MODE, ADJ>(sh, o, plane, Kzb, S.cs.cz + Kzb * CROW3, false, OP_XZ, a.dz, a.rdz);
            dzq.y = stencil_z_op<T, MODE, ADJ>(sh, o, plane, Kzb, S.cs.cz + Kzb * CROW3, false, OP_YZ, a.dz, a.rdz);
        }
        if (Kzf != order)
            dzz = stencil_z_op<T, MODE, ADJ>(sh, o, plane, Kzf, S.cs.cz + Kzf * CROW3, true, OP_ZZ, a.dz, a.rdz);
        // ---- Vx: Dx+ XX, Dy- XY, Dz- XZ
        {
            const T am = A::mul(a.dt, rx);
            vx = A::mad(vx, am, dxx);
            if (xi >= 0) vx = pml_correct<T, MODE>(vx, am, dxx, sh.psix[0] + px, a.pml, L, xb + 3, xi);
            vx = A::mad(vx, am, dyq.x);
            if (yi >= 0) vx = pml_correct<T, MODE>(vx, am, dyq.x, sh.psiy[0] + py, a.pml, L, yb, yi);
            vx = A::mad(vx, am, dzq.x);
            if (zi >= 0) vx = pml_correct<T, MODE>(vx, am, dzq.x, sh.psiz[0] + pz, a.pml, L, zb, zi);
            Vx[o] = vx;
        }
        // ---- Vy: Dx- XY, Dy+ YY, Dz- YZ
        {
            const T am = A::mul(a.dt, ry);
            vy = A::mad(vy, am, dxq.x);
            if (xi >= 0) vy = pml_correct<T, MODE>(vy, am, dxq.x, sh.psix[1] + px, a.pml, L, xb, xi);
            vy = A::mad(vy, am, dyy);
            if (yi >= 0) vy = pml_correct<T, MODE>(vy, am, dyy, sh.psiy[1] + py, a.pml, L, yb + 3, yi);
            vy = A::mad(vy, am, dzq.y);
            if (zi >= 0) vy = pml_correct<T, MODE>(vy, am, dzq.y, sh.psiz[1] + pz, a.pml, L, zb, zi);
            Vy[o] = vy;
        }
        // ---- Vz: Dx- XZ, Dy- YZ, Dz+ ZZ
        {
            const T am = A::mul(a.dt, rz);
            vz = A::mad(vz, am, dxq.y);
            if (xi >= 0) vz = pml_correct<T, MODE>(vz, am, dxq.y, sh.psix[2] + px, a.pml, L, xb, xi);
            vz = A::mad(vz, am, dyq.y);
            if (yi >= 0) vz = pml_correct<T, MODE>(vz, am, dyq.y, sh.psiy[2] + py, a.pml, L, yb, yi);
            vz = A::mad(vz, am, dzz);
            if (zi >= 0) vz = pml_correct<T, MODE>(vz, am, dzz, sh.psiz[2] + pz, a.pml, L, zb + 3, zi);
            Vz[o] = vz;
        }
#pragma unroll
        for (int j = 0; j < 15; j++) { qp[j] = qp[j + 1]; qzz[j] = qzz[j + 1]; }
        qp[15] = make_float2(opnd<T, MODE, ADJ>(sh, o + 8 * plane, OP_XZ), opnd<T, MODE, ADJ>(sh, o + 8 * plane, OP_YZ));
        qzz[15] = opnd<T, MODE, ADJ>(sh, o + 9 * plane, OP_ZZ);
        vx = nvx; vy = nvy; vz = nvz; rx = nrx; ry = nry; rz = nrz;
        cxx = ncxx; cxy = ncxy; cyy = ncyy;
    }
}

struct StrSmemF {
    float sx[2][TY3][WX];      // Vx, x halo
    float2 px[2][TY3][WX];     // (Vz, Vy), x halo
    float sy[2][HY][TX3];      // Vy, y halo
    float2 py[2][HY][TX3];     // (Vz, Vx), y halo
    CoefSet3<float> cs;
};

template <bool ADJ>
__global__ void __launch_bounds__(TX3 *TY3, 2) e3d_stress_fast(Step3DArgs<float> a, const CoefSet3<float> *coefs)
{
    using T = float;
    constexpr int MODE = MODE_FAST;
    using A = Ar<T, MODE>;
    extern __shared__ __align__(16) unsigned char smraw[];
    StrSmemF &S = *reinterpret_cast<StrSmemF *>(smraw);
    __shared__ Shot3D<T> shs;
    const Tile3D tl = a.tiles[blockIdx.x];
    stage_shot(shs, a.shots + tl.shot);
    load_coefs3e(S.cs, coefs);
    __syncthreads();
    const int tx = threadIdx.x, ty = threadIdx.y;
    const Shot3D<T> &sh = shs;
    const int ix = tl.x0 + tx, iy = tl.y0 + ty;
    const int nxp = sh.nxp, nyp = sh.nyp, nzp = sh.nzp, pitch = sh.pitch, L = a.lpml, order = a.order;
    const int plane = (int)sh.plane;   // a field holds fewer than 2^31 elements
    const int col = iy * pitch + ix;
    const T *Vx = sh.f[E3_VX], *Vy = sh.f[E3_VY], *Vz = sh.f[E3_VZ];
    T *Sxx = sh.f[E3_SXX], *Syy = sh.f[E3_SYY], *Szz = sh.f[E3_SZZ];
    T *Syz = sh.f[E3_SYZ], *Sxz = sh.f[E3_SXZ], *Sxy = sh.f[E3_SXY];
    const bool in_grid = ix < nxp && iy < nyp;
    const int Kxf = kfw(ix, nxp, order), Kxb = kbw(ix, nxp, order);
    const int Kyf = kfw(iy, nyp, order), Kyb = kbw(iy, nyp, order);
    int xb = 0, xc = 0, yb = 0, yc = 0;
    const int xi = in_grid ? xstrip(ix, nxp, L, xb, xc) : -1;
    const int yi = in_grid ? xstrip(iy, nyp, L, yb, yc) : -1;
    const int z0 = tl.z0, ze = min(z0 + a.zc, nzp);
    const int hx = tx < 8 ? -8 : TX3 - 8;
    // z windows: Vz backward (planes z-8..z+7), (Vx, Vy) forward (z-7..z+8)
    T qz[16];
    float2 qv[16];
#pragma unroll
    for (int j = 0; j < 16; j++) {
        qz[j] = Vz[(z0 - 8 + j) * plane + col];
        const int oj = (z0 - 7 + j) * plane + col;
        qv[j] = make_float2(Vx[oj], Vy[oj]);
    }
    int o = z0 * plane + col;
    T sxx = Sxx[o], syy = Syy[o], szz = Szz[o], syz = Syz[o], sxz = Sxz[o], sxy = Sxy[o];
    T l = 0, l2m = 0, myz = 0, mxz = 0, mxy = 0;
    if (!ADJ) {
        l = __ldg(sh.m[ME_L] + o); l2m = __ldg(sh.m[ME_L2M] + o);
        myz = __ldg(sh.m[ME_MYZ] + o); mxz = __ldg(sh.m[ME_MXZ] + o); mxy = __ldg(sh.m[ME_MXY] + o);
    }
    T hvx = 0, hvy = 0, hvz = 0;
    if (tx < 16) { hvx = Vx[o + hx]; hvy = Vy[o + hx]; hvz = Vz[o + hx]; }
    T yx0 = Vx[o - 8 * pitch], yx1 = Vx[o + TY3 * pitch];
    T yy0 = Vy[o - 8 * pitch], yy1 = Vy[o + TY3 * pitch];
    T yz0 = Vz[o - 8 * pitch], yz1 = Vz[o + TY3 * pitch];
    __syncthreads();
    for (int iz = z0; iz < ze; iz++, o += plane) {
        const int b = (iz - z0) & 1;
        const T cvx = qv[7].x, cvy = qv[7].y, cvz = qz[8];
        S.sx[b][ty][tx + 8] = cvx;
        S.px[b][ty][tx + 8] = make_float2(cvz, cvy);
        S.sy[b][ty + 8][tx] = cvy;
        S.py[b][ty + 8][tx] = make_float2(cvz, cvx);
        if (tx < 16) {
            const int c = tx < 8 ? tx : tx + TX3;
            S.sx[b][ty][c] = hvx;
            S.px[b][ty][c] = make_float2(hvz, hvy);
        }
        S.sy[b][ty][tx] = yy0; S.sy[b][ty + TY3 + 8][tx] = yy1;
        S.py[b][ty][tx] = make_float2(yz0, yx0); S.py[b][ty + TY3 + 8][tx] = make_float2(yz1, yx1);
        const int on = o + plane;
        const T nsxx = Sxx[on], nsyy = Syy[on], nszz = Szz[on], nsyz = Syz[on], nsxz = Sxz[on], nsxy = Sxy[on];
        T nl = 0, nl2m = 0, nmyz = 0, nmxz = 0, nmxy = 0;
        if (!ADJ) {
            nl = __ldg(sh.m[ME_L] + on); nl2m = __ldg(sh.m[ME_L2M] + on);
            nmyz = __ldg(sh.m[ME_MYZ] + on); nmxz = __ldg(sh.m[ME_MXZ] + on); nmxy = __ldg(sh.m[ME_MXY] + on);
        }
        if (tx < 16) { hvx = Vx[on + hx]; hvy = Vy[on + hx]; hvz = Vz[on + hx]; }
        yx0 = Vx[on - 8 * pitch]; yx1 = Vx[on + TY3 * pitch];
        yy0 = Vy[on - 8 * pitch]; yy1 = Vy[on + TY3 * pitch];
        yz0 = Vz[on - 8 * pitch]; yz1 = Vz[on + TY3 * pitch];
        __syncthreads();
        const int Kzf = kfw(iz, nzp, order), Kzb = kbw(iz, nzp, order);
        int zb = 0, zc = 0;
        const int zi = in_grid ? xstrip(iz, nzp, L, zb, zc) : -1;
        const int px = (iz * nyp + iy) * 2 * L + xc;
        const int py = (iz * 2 * L + yc) * nxp + ix;
        const int pz = (zc * nyp + iy) * nxp + ix;
        const T *csx = &S.sx[b][ty][tx + 8];
        T dxx = taps3<T, MODE>(csx - 8, 1, a.cf[0], a.dx, a.rdx);
        const float2 *cpx = &S.px[b][ty][tx + 8];
        float2 dxp = taps_pair(cpx - 7, 1, a.cf2[0]);                 // (Dx+ Vz, Dx+ Vy)
        const T *csy = &S.sy[b][ty + 8][tx];
        T dyy = taps3<T, MODE>(csy - 8 * TX3, TX3, a.cf[1], a.dy, a.rdy);
        const float2 *cpy = &S.py[b][ty + 8][tx];
        float2 dyp = taps_pair(cpy - 7 * TX3, TX3, a.cf2[1]);         // (Dy+ Vz, Dy+ Vx)
        T dzz = taps3_reg<T, MODE>(qz, a.cf[2], a.dz, a.rdz);
        float2 dzp = taps_pair_reg(qv, a.cf2[2]);                     // (Dz+ Vx, Dz+ Vy)
        if (Kxb != order) dxx = stencil_k<T, MODE>(csx, 1, Kxb, S.cs.cx + Kxb * CROW3, false, a.dx, a.rdx);
        if (Kxf != order) {
            const T *c = reinterpret_cast<const T *>(cpx);
            dxp.x = stencil_k<T, MODE>(c, 2, Kxf, S.cs.cx + Kxf * CROW3, true, a.dx, a.rdx);
            dxp.y = stencil_k<T, MODE>(c + 1, 2, Kxf, S.cs.cx + Kxf * CROW3, true, a.dx, a.rdx);
        }
        if (Kyb != order) dyy = stencil_k<T, MODE>(csy, TX3, Kyb, S.cs.cy + Kyb * CROW3, false, a.dy, a.rdy);
        if (Kyf != order) {
            const T *c = reinterpret_cast<const T *>(cpy);
            dyp.x = stencil_k<T, MODE>(c, 2 * TX3, Kyf, S.cs.cy + Kyf * CROW3, true, a.dy, a.rdy);
            dyp.y = stencil_k<T, MODE>(c + 1, 2 * TX3, Kyf, S.cs.cy + Kyf * CROW3, true, a.dy, a.rdy);
        }
        if (Kzb != order) dzz = stencil_k<T, MODE>(Vz + o, (int)plane, Kzb, S.cs.cz + Kzb * CROW3, false, a.dz, a.rdz);
        if (Kzf != order) {
            dzp.x = stencil_k<T, MODE>(Vx + o, (int)plane, Kzf, S.cs.cz + Kzf * CROW3, true, a.dz, a.rdz);
            dzp.y = stencil_k<T, MODE>(Vy + o, (int)plane, Kzf, S.cs.cz + Kzf * CROW3, true, a.dz, a.rdz);
        }
        // ---- normal stresses
        {
            const bool fsrow = sh.fs && iz == L;
            if (!ADJ) {
                const T a2 = A::mul(a.dt, l2m), a1 = A::mul(a.dt, l);
                auto upd3 = [&](T d, T cxx_, T cyy_, T czz_) {
                    sxx = A::mad(sxx, cxx_, d); syy = A::mad(syy, cyy_, d); szz = A::mad(szz, czz_, d);
                };
                auto pml3 = [&](T d, T *psi, int base, int idx, T cxx_, T cyy_, T czz_) {
                    const T tA = __ldg(a.pml + (base + PT_A) * L + idx), tB = __ldg(a.pml + (base + PT_B) * L + idx),
                            tC = __ldg(a.pml + (base + PT_C) * L + idx);
                    const T p = A::mad(A::mul(tB, *psi), tA, d);
                    *psi = p;
                    const T cq = A::mad(p, tC, d);
                    sxx = A::msub(sxx, cxx_, cq); syy = A::msub(syy, cyy_, cq); szz = A::msub(szz, czz_, cq);
                };
                upd3(dxx, a2, a1, a1);
                if (xi >= 0) pml3(dxx, sh.psix[3] + px, xb, xi, a2, a1, a1);
                upd3(dyy, a1, a2, a1);
                if (yi >= 0) pml3(dyy, sh.psiy[3] + py, yb, yi, a1, a2, a1);
                upd3(dzz, a1, a1, a2);
                if (fsrow) szz = T(0);
                if (zi >= 0) pml3(dzz, sh.psiz[3] + pz, zb, zi, a1, a1, a2);
            } else {
                sxx = A::mad(sxx, a.dt, dxx);
                if (xi >= 0) sxx = pml_correct<T, MODE>(sxx, a.dt, dxx, sh.psix[3] + px, a.pml, L, xb, xi);
                syy = A::mad(syy, a.dt, dyy);
                if (yi >= 0) syy = pml_correct<T, MODE>(syy, a.dt, dyy, sh.psiy[3] + py, a.pml, L, yb, yi);
                szz = A::mad(szz, a.dt, dzz);
                if (fsrow) szz = T(0);
                if (zi >= 0) szz = pml_correct<T, MODE>(szz, a.dt, dzz, sh.psiz[3] + pz, a.pml, L, zb, zi);
            }
            Sxx[o] = sxx; Syy[o] = syy; Szz[o] = szz;
        }
        // ---- Sxz: Dx+ Vz, Dz+ Vx
        {
            const T am = ADJ ? a.dt : A::mul(a.dt, mxz);
            sxz = A::mad(sxz, am, dxp.x);
            if (xi >= 0) sxz = pml_correct<T, MODE>(sxz, am, dxp.x, sh.psix[4] + px, a.pml, L, xb + 3, xi);
            sxz = A::mad(sxz, am, dzp.x);
            if (zi >= 0) sxz = pml_correct<T, MODE>(sxz, am, dzp.x, sh.psiz[4] + pz, a.pml, L, zb + 3, zi);
            Sxz[o] = sxz;
        }
        // ---- Syz: Dz+ Vy, Dy+ Vz
        {
            const T am = ADJ ? a.dt : A::mul(a.dt, myz);
            syz = A::mad(syz, am, dzp.y);
            if (zi >= 0) syz = pml_correct<T, MODE>(syz, am, dzp.y, sh.psiz[5] + pz, a.pml, L, zb + 3, zi);
            syz = A::mad(syz, am, dyp.x);
            if (yi >= 0) syz = pml_correct<T, MODE>(syz, am, dyp.x, sh.psiy[4] + py, a.pml, L, yb + 3, yi);
            Syz[o] = syz;
        }
        // ---- Sxy: Dy+ Vx, Dx+ Vy
        {
            const T am = ADJ ? a.dt : A::mul(a.dt, mxy);
            sxy = A::mad(sxy, am, dyp.y);
            if (yi >= 0) sxy = pml_correct<T, MODE>(sxy, am, dyp.y, sh.psiy[5] + py, a.pml, L, yb + 3, yi);
            sxy = A::mad(sxy, am, dxp.y);
            if (xi >= 0) sxy = pml_correct<T, MODE>(sxy, am, dxp.y, sh.psix[5] + px, a.pml, L, xb + 3, xi);
            Sxy[o] = sxy;
        }
#pragma unroll
        for (int j = 0; j < 15; j++) { qz[j] = qz[j + 1]; qv[j] = qv[j + 1]; }
        qz[15] = Vz[o + 8 * plane];
        qv[15] = make_float2(Vx[o + 9 * plane], Vy[o + 9 * plane]);
        sxx = nsxx; syy = nsyy; szz = nszz; syz = nsyz; sxz = nsxz; sxy = nsxy;
        l = nl; l2m = nl2m; myz = nmyz; mxz = nmxz; mxy = nmxy;
    }
}

// ---------------------------------------------------------------- fast mode with TMA-staged planes
// The forward velocity step and both stress steps of RSGPU_F32_FAST with every
// plane tile brought in by TMA (cp.async.bulk.tensor.2d, one thread issuing,
// completion on an mbarrier per stage) NSTG3 - 1 planes ahead of the plane being
// computed: the loads in flight no longer depend on registers or resident warps.
// The z-derivatives still come from 16-plane register windows, refilled by plain
// loads eight planes ahead.  Same stencils, C-PML and update order as
// e3d_velocity_fast / e3d_stress_fast.  Every wait is bounded (2 s): on timeout the
// CTA records RSGPU_ERR_TIMEOUT in the error word and stops.
constexpr int NSTG3 = 3;

struct VelStageT {
    float xx[TY3][WX];         // Sxx, x halo
    float xz[TY3][WX];         // Sxz, x halo
    float xy[HY][WX];          // Sxy, x and y halos
    float yy[HY][TX3];         // Syy, y halo
    float yz[HY][TX3];         // Syz, y halo
    float pv[6][TY3][TX3];     // Vx, Vy, Vz, Rx, Ry, Rz
};
struct StrStageT {
    float v[3][HY][WX];        // Vx, Vy, Vz, x and y halos
    float sv[6][TY3][TX3];     // Sxx, Syy, Szz, Syz, Sxz, Sxy
    float mv[5][TY3][TX3];     // L, L2M, M_yz, M_xz, M_xy (forward only)
};
static_assert(sizeof(VelStageT) % 128 == 0 && sizeof(StrStageT) % 128 == 0, "TMA destinations stay 128-byte aligned");
static_assert(sizeof(float) * TY3 * WX % 128 == 0 && sizeof(float) * HY * WX % 128 == 0 &&
              sizeof(float) * HY * TX3 % 128 == 0 && sizeof(float) * TY3 * TX3 % 128 == 0, "tile sizes");
constexpr uint32_t VEL_STAGE_BYTES = sizeof(VelStageT);
constexpr uint32_t STR_STAGE_BYTES_FW = sizeof(StrStageT);
constexpr uint32_t STR_STAGE_BYTES_ADJ = sizeof(StrStageT) - sizeof(float) * 5 * TY3 * TX3;

template <typename Stage>
struct TmaSmem {
    Stage st[NSTG3];
    uint64_t bar[NSTG3];
    CoefSet3<float> cs;
};
template <typename Stage>
constexpr size_t tma_smem_bytes() { return sizeof(TmaSmem<Stage>) + 128; }   // + alignment slack

// (a - b) pairs of two arrays with the same tap spacing: sum_k c_k (p[(8+k)s] - p[(7-k)s])
__device__ __forceinline__ float2 taps_pair2(const float *p, const float *q, int sp, int sq,
                                             const float (&c2)[NCOEF][2])
{
    using A2 = Ar2<float, MODE_FAST>;
    const float2 *cc = reinterpret_cast<const float2 *>(c2);
    float2 acc = A2::mul(A2::sub(make_float2(p[8 * sp], q[8 * sq]), make_float2(p[7 * sp], q[7 * sq])), cc[0]);
#pragma unroll
    for (int k = 1; k < NCOEF; k++)
        acc = A2::acc(acc, A2::sub(make_float2(p[(8 + k) * sp], q[(8 + k) * sq]),
                                   make_float2(p[(7 - k) * sp], q[(7 - k) * sq])), cc[k]);
    return acc;
}

// Allocation row of plane iz, padded row iy_alloc (guards included).
__device__ __forceinline__ int alloc_row(const Shot3D<float> &sh, int iz, int iy_alloc)
{
    return (GUARD + iz) * sh.rows + iy_alloc;
}

__global__ void __launch_bounds__(TX3 *TY3, 2) e3d_velocity_tma(Step3DArgs<float> a, const CoefSet3<float> *coefs)
{
    using T = float;
    constexpr int MODE = MODE_FAST;
    using A = Ar<T, MODE>;
    extern __shared__ unsigned char smraw[];
    TmaSmem<VelStageT> &S =
        *reinterpret_cast<TmaSmem<VelStageT> *>((reinterpret_cast<uintptr_t>(smraw) + 127) & ~uintptr_t(127));
    __shared__ Shot3D<T> shs;
    const Tile3D tl = a.tiles[blockIdx.x];
    stage_shot(shs, a.shots + tl.shot);
    load_coefs3e(S.cs, coefs);
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    if (tid == 0)
        for (int k = 0; k < NSTG3; k++) mbar_init(&S.bar[k], 1);
    __syncthreads();
    const Shot3D<T> &sh = shs;
    const CUtensorMap *M = reinterpret_cast<const CUtensorMap *>(a.maps) + (size_t)tl.shot * NMAP_E3;
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int x0 = tl.x0, y0 = tl.y0;
    const int ix = x0 + tx, iy = y0 + ty;
    const int nxp = sh.nxp, nyp = sh.nyp, nzp = sh.nzp, pitch = sh.pitch, L = a.lpml, order = a.order;
    const int plane = (int)sh.plane;
    const int col = iy * pitch + ix;
    T *Vx = sh.f[E3_VX], *Vy = sh.f[E3_VY], *Vz = sh.f[E3_VZ];
    const bool in_grid = ix < nxp && iy < nyp;
    const int Kxf = kfw(ix, nxp, order), Kxb = kbw(ix, nxp, order);
    const int Kyf = kfw(iy, nyp, order), Kyb = kbw(iy, nyp, order);
    int xb = 0, xc = 0, yb = 0, yc = 0;
    const int xi = in_grid ? xstrip(ix, nxp, L, xb, xc) : -1;
    const int yi = in_grid ? xstrip(iy, nyp, L, yb, yc) : -1;
    const int z0 = tl.z0, ze = min(z0 + a.zc, nzp);
    // stage k <- plane iz: every box starts on a 16-byte boundary (x0 and x0 + 8 are
    // multiples of 4 floats)
    auto issue = [&](int iz, int k) {
        VelStageT &g = S.st[k];
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        mbar_expect_tx(&S.bar[k], VEL_STAGE_BYTES);
        const int rh = alloc_row(sh, iz, GUARD + y0), ry = alloc_row(sh, iz, y0);
        tma_load_2d(g.xx, M + VM_SXX, &S.bar[k], x0, rh);
        tma_load_2d(g.xz, M + VM_SXZ, &S.bar[k], x0, rh);
        tma_load_2d(g.xy, M + VM_SXY, &S.bar[k], x0, ry);
        tma_load_2d(g.yy, M + VM_SYY, &S.bar[k], x0 + GUARD, ry);
        tma_load_2d(g.yz, M + VM_SYZ, &S.bar[k], x0 + GUARD, ry);
#pragma unroll
        for (int q = 0; q < 6; q++) tma_load_2d(g.pv[q], M + VM_VX + q, &S.bar[k], x0 + GUARD, rh);
    };
    if (tid == 0)
        for (int j = 0; j < NSTG3 - 1 && z0 + j < ze; j++) issue(z0 + j, j);
    // z windows: (XZ, YZ) backward (planes z-8..z+7), ZZ forward (z-7..z+8)
    const T *Sxz = sh.f[E3_SXZ], *Syz = sh.f[E3_SYZ], *Szz = sh.f[E3_SZZ];
    float2 qp[16];
    T qzz[16];
#pragma unroll
    for (int j = 0; j < 16; j++) {
        const int oj = (z0 - 8 + j) * plane + col;
        qp[j] = make_float2(Sxz[oj], Syz[oj]);
        qzz[j] = Szz[(z0 - 7 + j) * plane + col];
    }
    int o = z0 * plane + col;
    for (int iz = z0; iz < ze; iz++, o += plane) {
        const int j = iz - z0, k = j % NSTG3;
        if (tid == 0 && iz + NSTG3 - 1 < ze) issue(iz + NSTG3 - 1, (j + NSTG3 - 1) % NSTG3);
        // window refills of this iteration, in flight while the stage arrives
        const float2 nq = make_float2(Sxz[o + 8 * plane], Syz[o + 8 * plane]);
        const T nzz = Szz[o + 9 * plane];
        if (!__syncthreads_and(mbar_wait_bounded(&S.bar[k], (uint32_t)(j / NSTG3) & 1u, a.err))) return;
        const VelStageT &g = S.st[k];
        const int Kzf = kfw(iz, nzp, order), Kzb = kbw(iz, nzp, order);
        int zb = 0, zc = 0;
        const int zi = in_grid ? xstrip(iz, nzp, L, zb, zc) : -1;
        const int px = (iz * nyp + iy) * 2 * L + xc;
        const int py = (iz * 2 * L + yc) * nxp + ix;
        const int pz = (zc * nyp + iy) * nxp + ix;
        const T *cxx = &g.xx[ty][tx + 8], *cxy = &g.xy[ty + 8][tx + 8], *cxz = &g.xz[ty][tx + 8];
        const T *cyy = &g.yy[ty + 8][tx], *cyz = &g.yz[ty + 8][tx];
        T dxx = taps3<T, MODE>(cxx - 7, 1, a.cf[0], a.dx, a.rdx);
        float2 dxq = taps_pair2(cxy - 8, cxz - 8, 1, 1, a.cf2[0]);                  // (Dx- XY, Dx- XZ)
        float2 dyq = taps_pair2(cxy - 8 * WX, cyz - 8 * TX3, WX, TX3, a.cf2[1]);  // (Dy- XY, Dy- YZ)
        T dyy = taps3<T, MODE>(cyy - 7 * TX3, TX3, a.cf[1], a.dy, a.rdy);
        float2 dzq = taps_pair_reg(qp, a.cf2[2]);
        T dzz = taps3_reg<T, MODE>(qzz, a.cf[2], a.dz, a.rdz);
        if (Kxf != order) dxx = stencil_k<T, MODE>(cxx, 1, Kxf, S.cs.cx + Kxf * CROW3, true, a.dx, a.rdx);
        if (Kxb != order) {
            dxq.x = stencil_k<T, MODE>(cxy, 1, Kxb, S.cs.cx + Kxb * CROW3, false, a.dx, a.rdx);
            dxq.y = stencil_k<T, MODE>(cxz, 1, Kxb, S.cs.cx + Kxb * CROW3, false, a.dx, a.rdx);
        }
        if (Kyb != order) {
            dyq.x = stencil_k<T, MODE>(cxy, WX, Kyb, S.cs.cy + Kyb * CROW3, false, a.dy, a.rdy);
            dyq.y = stencil_k<T, MODE>(cyz, TX3, Kyb, S.cs.cy + Kyb * CROW3, false, a.dy, a.rdy);
        }
        if (Kyf != order) dyy = stencil_k<T, MODE>(cyy, TX3, Kyf, S.cs.cy + Kyf * CROW3, true, a.dy, a.rdy);
        if (Kzb != order) {
            dzq.x = stencil_z_op<T, MODE, false>(sh, o, plane, Kzb, S.cs.cz + Kzb * CROW3, false, OP_XZ, a.dz, a.rdz);
            dzq.y = stencil_z_op<T, MODE, false>(sh, o, plane, Kzb, S.cs.cz + Kzb * CROW3, false, OP_YZ, a.dz, a.rdz);
        }
        if (Kzf != order)
            dzz = stencil_z_op<T, MODE, false>(sh, o, plane, Kzf, S.cs.cz + Kzf * CROW3, true, OP_ZZ, a.dz, a.rdz);
        T vx = g.pv[0][ty][tx], vy = g.pv[1][ty][tx], vz = g.pv[2][ty][tx];
        // ---- Vx: Dx+ XX, Dy- XY, Dz- XZ
        {
            const T am = A::mul(a.dt, g.pv[3][ty][tx]);
            vx = A::mad(vx, am, dxx);
            if (xi >= 0) vx = pml_correct<T, MODE>(vx, am, dxx, sh.psix[0] + px, a.pml, L, xb + 3, xi);
            vx = A::mad(vx, am, dyq.x);
            if (yi >= 0) vx = pml_correct<T, MODE>(vx, am, dyq.x, sh.psiy[0] + py, a.pml, L, yb, yi);
            vx = A::mad(vx, am, dzq.x);
            if (zi >= 0) vx = pml_correct<T, MODE>(vx, am, dzq.x, sh.psiz[0] + pz, a.pml, L, zb, zi);
            Vx[o] = vx;
        }
        // ---- Vy: Dx- XY, Dy+ YY, Dz- YZ
        {
            const T am = A::mul(a.dt, g.pv[4][ty][tx]);
            vy = A::mad(vy, am, dxq.x);
            if (xi >= 0) vy = pml_correct<T, MODE>(vy, am, dxq.x, sh.psix[1] + px, a.pml, L, xb, xi);
            vy = A::mad(vy, am, dyy);
            if (yi >= 0) vy = pml_correct<T, MODE>(vy, am, dyy, sh.psiy[1] + py, a.pml, L, yb + 3, yi);
            vy = A::mad(vy, am, dzq.y);
            if (zi >= 0) vy = pml_correct<T, MODE>(vy, am, dzq.y, sh.psiz[1] + pz, a.pml, L, zb, zi);
            Vy[o] = vy;
        }
        // ---- Vz: Dx- XZ, Dy- YZ, Dz+ ZZ
        {
            const T am = A::mul(a.dt, g.pv[5][ty][tx]);
            vz = A::mad(vz, am, dxq.y);
            if (xi >= 0) vz = pml_correct<T, MODE>(vz, am, dxq.y, sh.psix[2] + px, a.pml, L, xb, xi);
            vz = A::mad(vz, am, dyq.y);
            if (yi >= 0) vz = pml_correct<T, MODE>(vz, am, dyq.y, sh.psiy[2] + py, a.pml, L, yb, yi);
            vz = A::mad(vz, am, dzz);
            if (zi >= 0) vz = pml_correct<T, MODE>(vz, am, dzz, sh.psiz[2] + pz, a.pml, L, zb + 3, zi);
            Vz[o] = vz;
        }
#pragma unroll
        for (int q = 0; q < 15; q++) { qp[q] = qp[q + 1]; qzz[q] = qzz[q + 1]; }
        qp[15] = nq;
        qzz[15] = nzz;
        __syncthreads();   // stage k is refilled next iteration
    }
}

template <bool ADJ>
__global__ void __launch_bounds__(TX3 *TY3, 2) e3d_stress_tma(Step3DArgs<float> a, const CoefSet3<float> *coefs)
{
    using T = float;
    constexpr int MODE = MODE_FAST;
    using A = Ar<T, MODE>;
    extern __shared__ unsigned char smraw[];
    TmaSmem<StrStageT> &S =
        *reinterpret_cast<TmaSmem<StrStageT> *>((reinterpret_cast<uintptr_t>(smraw) + 127) & ~uintptr_t(127));
    __shared__ Shot3D<T> shs;
    const Tile3D tl = a.tiles[blockIdx.x];
    stage_shot(shs, a.shots + tl.shot);
    load_coefs3e(S.cs, coefs);
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    if (tid == 0)
        for (int k = 0; k < NSTG3; k++) mbar_init(&S.bar[k], 1);
    __syncthreads();
    const Shot3D<T> &sh = shs;
    const CUtensorMap *M = reinterpret_cast<const CUtensorMap *>(a.maps) + (size_t)tl.shot * NMAP_E3;
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int x0 = tl.x0, y0 = tl.y0;
    const int ix = x0 + tx, iy = y0 + ty;
    const int nxp = sh.nxp, nyp = sh.nyp, nzp = sh.nzp, pitch = sh.pitch, L = a.lpml, order = a.order;
    const int plane = (int)sh.plane;
    const int col = iy * pitch + ix;
    const T *Vx = sh.f[E3_VX], *Vy = sh.f[E3_VY], *Vz = sh.f[E3_VZ];
    T *Sxx = sh.f[E3_SXX], *Syy = sh.f[E3_SYY], *Szz = sh.f[E3_SZZ];
    T *Syz = sh.f[E3_SYZ], *Sxz = sh.f[E3_SXZ], *Sxy = sh.f[E3_SXY];
    const bool in_grid = ix < nxp && iy < nyp;
    const int Kxf = kfw(ix, nxp, order), Kxb = kbw(ix, nxp, order);
    const int Kyf = kfw(iy, nyp, order), Kyb = kbw(iy, nyp, order);
    int xb = 0, xc = 0, yb = 0, yc = 0;
    const int xi = in_grid ? xstrip(ix, nxp, L, xb, xc) : -1;
    const int yi = in_grid ? xstrip(iy, nyp, L, yb, yc) : -1;
    const int z0 = tl.z0, ze = min(z0 + a.zc, nzp);
    auto issue = [&](int iz, int k) {
        StrStageT &g = S.st[k];
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        mbar_expect_tx(&S.bar[k], ADJ ? STR_STAGE_BYTES_ADJ : STR_STAGE_BYTES_FW);
        const int rh = alloc_row(sh, iz, GUARD + y0), ry = alloc_row(sh, iz, y0);
#pragma unroll
        for (int q = 0; q < 3; q++) tma_load_2d(g.v[q], M + SM_VX + q, &S.bar[k], x0, ry);
#pragma unroll
        for (int q = 0; q < 6; q++) tma_load_2d(g.sv[q], M + SM_SXX + q, &S.bar[k], x0 + GUARD, rh);
        if (!ADJ) {
#pragma unroll
            for (int q = 0; q < 5; q++) tma_load_2d(g.mv[q], M + SM_L + q, &S.bar[k], x0 + GUARD, rh);
        }
    };
    if (tid == 0)
        for (int j = 0; j < NSTG3 - 1 && z0 + j < ze; j++) issue(z0 + j, j);
    // z windows: Vz backward (planes z-8..z+7), (Vx, Vy) forward (z-7..z+8)
    T qz[16];
    float2 qv[16];
#pragma unroll
    for (int j = 0; j < 16; j++) {
        qz[j] = Vz[(z0 - 8 + j) * plane + col];
        const int oj = (z0 - 7 + j) * plane + col;
        qv[j] = make_float2(Vx[oj], Vy[oj]);
    }
    int o = z0 * plane + col;
    for (int iz = z0; iz < ze; iz++, o += plane) {
        const int j = iz - z0, k = j % NSTG3;
        if (tid == 0 && iz + NSTG3 - 1 < ze) issue(iz + NSTG3 - 1, (j + NSTG3 - 1) % NSTG3);
        const T nz = Vz[o + 8 * plane];
        const float2 nv = make_float2(Vx[o + 9 * plane], Vy[o + 9 * plane]);
        if (!__syncthreads_and(mbar_wait_bounded(&S.bar[k], (uint32_t)(j / NSTG3) & 1u, a.err))) return;
        const StrStageT &g = S.st[k];
        const int Kzf = kfw(iz, nzp, order), Kzb = kbw(iz, nzp, order);
        int zb = 0, zc = 0;
        const int zi = in_grid ? xstrip(iz, nzp, L, zb, zc) : -1;
        const int px = (iz * nyp + iy) * 2 * L + xc;
        const int py = (iz * 2 * L + yc) * nxp + ix;
        const int pz = (zc * nyp + iy) * nxp + ix;
        const T *cvx = &g.v[0][ty + 8][tx + 8], *cvy = &g.v[1][ty + 8][tx + 8], *cvz = &g.v[2][ty + 8][tx + 8];
        T dxx = taps3<T, MODE>(cvx - 8, 1, a.cf[0], a.dx, a.rdx);
        float2 dxp = taps_pair2(cvz - 7, cvy - 7, 1, 1, a.cf2[0]);                  // (Dx+ Vz, Dx+ Vy)
        T dyy = taps3<T, MODE>(cvy - 8 * WX, WX, a.cf[1], a.dy, a.rdy);
        float2 dyp = taps_pair2(cvz - 7 * WX, cvx - 7 * WX, WX, WX, a.cf2[1]);     // (Dy+ Vz, Dy+ Vx)
        T dzz = taps3_reg<T, MODE>(qz, a.cf[2], a.dz, a.rdz);
        float2 dzp = taps_pair_reg(qv, a.cf2[2]);                                   // (Dz+ Vx, Dz+ Vy)
        if (Kxb != order) dxx = stencil_k<T, MODE>(cvx, 1, Kxb, S.cs.cx + Kxb * CROW3, false, a.dx, a.rdx);
        if (Kxf != order) {
            dxp.x = stencil_k<T, MODE>(cvz, 1, Kxf, S.cs.cx + Kxf * CROW3, true, a.dx, a.rdx);
            dxp.y = stencil_k<T, MODE>(cvy, 1, Kxf, S.cs.cx + Kxf * CROW3, true, a.dx, a.rdx);
        }
        if (Kyb != order) dyy = stencil_k<T, MODE>(cvy, WX, Kyb, S.cs.cy + Kyb * CROW3, false, a.dy, a.rdy);
        if (Kyf != order) {
            dyp.x = stencil_k<T, MODE>(cvz, WX, Kyf, S.cs.cy + Kyf * CROW3, true, a.dy, a.rdy);
            dyp.y = stencil_k<T, MODE>(cvx, WX, Kyf, S.cs.cy + Kyf * CROW3, true, a.dy, a.rdy);
        }
        if (Kzb != order) dzz = stencil_k<T, MODE>(Vz + o, plane, Kzb, S.cs.cz + Kzb * CROW3, false, a.dz, a.rdz);
        if (Kzf != order) {
            dzp.x = stencil_k<T, MODE>(Vx + o, plane, Kzf, S.cs.cz + Kzf * CROW3, true, a.dz, a.rdz);
            dzp.y = stencil_k<T, MODE>(Vy + o, plane, Kzf, S.cs.cz + Kzf * CROW3, true, a.dz, a.rdz);
        }
        T sxx = g.sv[0][ty][tx], syy = g.sv[1][ty][tx], szz = g.sv[2][ty][tx];
        T syz = g.sv[3][ty][tx], sxz = g.sv[4][ty][tx], sxy = g.sv[5][ty][tx];
        // ---- normal stresses
        {
            const bool fsrow = sh.fs && iz == L;
            if (!ADJ) {
                const T l = g.mv[0][ty][tx], l2m = g.mv[1][ty][tx];
                const T a2 = A::mul(a.dt, l2m), a1 = A::mul(a.dt, l);
                auto upd3 = [&](T d, T cxx_, T cyy_, T czz_) {
                    sxx = A::mad(sxx, cxx_, d); syy = A::mad(syy, cyy_, d); szz = A::mad(szz, czz_, d);
                };
                auto pml3 = [&](T d, T *psi, int base, int idx, T cxx_, T cyy_, T czz_) {
                    const T tA = __ldg(a.pml + (base + PT_A) * L + idx), tB = __ldg(a.pml + (base + PT_B) * L + idx),
                            tC = __ldg(a.pml + (base + PT_C) * L + idx);
                    const T p = A::mad(A::mul(tB, *psi), tA, d);
                    *psi = p;
                    const T cq = A::mad(p, tC, d);
                    sxx = A::msub(sxx, cxx_, cq); syy = A::msub(syy, cyy_, cq); szz = A::msub(szz, czz_, cq);
                };
                upd3(dxx, a2, a1, a1);
                if (xi >= 0) pml3(dxx, sh.psix[3] + px, xb, xi, a2, a1, a1);
                upd3(dyy, a1, a2, a1);
                if (yi >= 0) pml3(dyy, sh.psiy[3] + py, yb, yi, a1, a2, a1);
                upd3(dzz, a1, a1, a2);
                if (fsrow) szz = T(0);
                if (zi >= 0) pml3(dzz, sh.psiz[3] + pz, zb, zi, a1, a1, a2);
            } else {
                sxx = A::mad(sxx, a.dt, dxx);
                if (xi >= 0) sxx = pml_correct<T, MODE>(sxx, a.dt, dxx, sh.psix[3] + px, a.pml, L, xb, xi);
                syy = A::mad(syy, a.dt, dyy);
                if (yi >= 0) syy = pml_correct<T, MODE>(syy, a.dt, dyy, sh.psiy[3] + py, a.pml, L, yb, yi);
                szz = A::mad(szz, a.dt, dzz);
                if (fsrow) szz = T(0);
                if (zi >= 0) szz = pml_correct<T, MODE>(szz, a.dt, dzz, sh.psiz[3] + pz, a.pml, L, zb, zi);
            }
            Sxx[o] = sxx; Syy[o] = syy; Szz[o] = szz;
        }
        // ---- Sxz: Dx+ Vz, Dz+ Vx
        {
            const T am = ADJ ? a.dt : A::mul(a.dt, g.mv[3][ty][tx]);
            sxz = A::mad(sxz, am, dxp.x);
            if (xi >= 0) sxz = pml_correct<T, MODE>(sxz, am, dxp.x, sh.psix[4] + px, a.pml, L, xb + 3, xi);
            sxz = A::mad(sxz, am, dzp.x);
            if (zi >= 0) sxz = pml_correct<T, MODE>(sxz, am, dzp.x, sh.psiz[4] + pz, a.pml, L, zb + 3, zi);
            Sxz[o] = sxz;
        }
        // ---- Syz: Dz+ Vy, Dy+ Vz
        {
            const T am = ADJ ? a.dt : A::mul(a.dt, g.mv[2][ty][tx]);
            syz = A::mad(syz, am, dzp.y);
            if (zi >= 0) syz = pml_correct<T, MODE>(syz, am, dzp.y, sh.psiz[5] + pz, a.pml, L, zb + 3, zi);
            syz = A::mad(syz, am, dyp.x);
            if (yi >= 0) syz = pml_correct<T, MODE>(syz, am, dyp.x, sh.psiy[4] + py, a.pml, L, yb + 3, yi);
            Syz[o] = syz;
        }
        // ---- Sxy: Dy+ Vx, Dx+ Vy
        {
            const T am = ADJ ? a.dt : A::mul(a.dt, g.mv[4][ty][tx]);
            sxy = A::mad(sxy, am, dyp.y);
            if (yi >= 0) sxy = pml_correct<T, MODE>(sxy, am, dyp.y, sh.psiy[5] + py, a.pml, L, yb + 3, yi);
            sxy = A::mad(sxy, am, dxp.y);
            if (xi >= 0) sxy = pml_correct<T, MODE>(sxy, am, dxp.y, sh.psix[5] + px, a.pml, L, xb + 3, xi);
            Sxy[o] = sxy;
        }
#pragma unroll
        for (int q = 0; q < 15; q++) { qz[q] = qz[q + 1]; qv[q] = qv[q + 1]; }
        qz[15] = nz;
        qv[15] = nv;
        __syncthreads();   // stage k is refilled next iteration
    }
}

// ---------------------------------------------------------------- sources and receivers
// One CTA per shot: injection of every source set (lib/waves.cpp:4104-4244), then,
// after a barrier, recording of every receiver set (lib/waves.cpp:4247-4400) of
// the same step.
template <typename T, int MODE>
__device__ void inject_set(const Shot3D<T> &sh, const InjRec3<T> &pl, T dt, int it)
{
    using A = Ar<T, MODE == MODE_FAST ? MODE_FAST : MODE_IEEE>;
    if (pl.kind_inj == INJ3_P) {
        // Sxx, Syy, Szz -= dt*wav*xtri*ytri*ztri
        for (int q = threadIdx.x; q < pl.ninj; q += blockDim.x) {
            const long long p = pl.inj_pt[q];
            T sxx = sh.f[E3_SXX][p], syy = sh.f[E3_SYY][p], szz = sh.f[E3_SZZ][p];
            for (int c = pl.inj_start[q]; c < pl.inj_start[q + 1]; c++) {
                const T w = pl.wav[(long long)pl.inj_trace[c] * pl.nt + it];
                const T s = A::mul(A::mul(A::mul(A::mul(dt, w), pl.inj_w[3 * c]), pl.inj_w[3 * c + 1]), pl.inj_w[3 * c + 2]);
                sxx = A::sub(sxx, s); syy = A::sub(syy, s); szz = A::sub(szz, s);
            }
            sh.f[E3_SXX][p] = sxx; sh.f[E3_SYY][p] = syy; sh.f[E3_SZZ][p] = szz;
        }
    } else if (pl.kind_inj != INJ3_NONE) {
        // Vx += dt*Rx*wav*xtri*ytri*ztri (likewise Vy, Vz)
        const int k = pl.kind_inj - INJ3_VX;
        T *F = sh.f[E3_VX + k];
        const T *Mod = sh.m[ME_RX + k];
        for (int q = threadIdx.x; q < pl.ninj; q += blockDim.x) {
            const long long p = pl.inj_pt[q];
            T v = F[p];
            const T dm = A::mul(dt, Mod[p]);
            for (int c = pl.inj_start[q]; c < pl.inj_start[q + 1]; c++) {
                const T w = pl.wav[(long long)pl.inj_trace[c] * pl.nt + it];
                v = A::add(v, A::mul(A::mul(A::mul(A::mul(dm, w), pl.inj_w[3 * c]), pl.inj_w[3 * c + 1]),
                                     pl.inj_w[3 * c + 2]));
            }
            F[p] = v;
        }
    }
}

template <typename T, int MODE>
__device__ void record_set(const Shot3D<T> &sh, const InjRec3<T> &pl, int it)
{
    using A = Ar<T, MODE == MODE_FAST ? MODE_FAST : MODE_IEEE>;
    if (pl.kind_rec == REC3_NONE || (pl.rec_gate && *pl.rec_gate == 0)) return;
    for (int tr = threadIdx.x; tr < pl.nrec; tr += blockDim.x) {
        const long long p = pl.rec_pt[tr];
        if (p < 0) continue;
        T *out = pl.rec_out + (long long)tr * pl.nt + it;
        if (pl.kind_rec >= REC3_WG_P) {
            // wavelet gradient, assigned: 1.0*(Sxx + Syy + Szz) or 0.5*(v + v[-1]) in double
            if (pl.kind_rec == REC3_WG_P) {
                *out = A::add(A::add(sh.f[E3_SXX][p], sh.f[E3_SYY][p]), sh.f[E3_SZZ][p]);
            } else {
                const int k = pl.kind_rec - REC3_WG_VX;
                const long long step = k == 0 ? 1 : k == 1 ? (long long)sh.pitch : sh.plane;
                const T *F = sh.f[E3_VX + k];
                *out = (T)__dmul_rn(0.5, (double)A::add(F[p], F[p - step]));
            }
            continue;
        }
        const T *w = pl.rec_w + 6 * tr;
        T acc = *out;
        if (pl.kind_rec == REC3_P) {
            // (1./3.)*xtri*ytri*ztri*F/factor in double, added to the T-typed sample, for
            // Sxx, Syy, Szz at each corner (lib/waves.cpp:4290-4300)
            const double fac = (double)pl.rec_factor[tr];
            for (int i1 = 0; i1 < 2; i1++)
                for (int i2 = 0; i2 < 2; i2++)
                    for (int i3 = 0; i3 < 2; i3++) {
                        const long long q = p + i1 * sh.plane + (long long)i2 * sh.pitch + i3;
                        const double c = __dmul_rn(__dmul_rn(__dmul_rn(1.0 / 3.0, (double)w[i3]), (double)w[2 + i2]),
                                                   (double)w[4 + i1]);
                        acc = (T)__dadd_rn((double)acc, __ddiv_rn(__dmul_rn(c, (double)sh.f[E3_SXX][q]), fac));
                        acc = (T)__dadd_rn((double)acc, __ddiv_rn(__dmul_rn(c, (double)sh.f[E3_SYY][q]), fac));
                        acc = (T)__dadd_rn((double)acc, __ddiv_rn(__dmul_rn(c, (double)sh.f[E3_SZZ][q]), fac));
                    }
        } else {
            const T *F = sh.f[E3_VX + (pl.kind_rec - REC3_VX)];
            for (int i1 = 0; i1 < 2; i1++)
                for (int i2 = 0; i2 < 2; i2++)
                    for (int i3 = 0; i3 < 2; i3++)
                        acc = A::add(acc, A::mul(A::mul(A::mul(w[i3], w[2 + i2]), w[4 + i1]),
                                                 F[p + i1 * sh.plane + (long long)i2 * sh.pitch + i3]));
        }
        *out = acc;
    }
}

template <typename T, int MODE>
__global__ void inject_record_e3d(const Shot3D<T> *shots, const InjRec3<T> *plans, int nsets, T dt, int it0)
{
    const Shot3D<T> &sh = shots[blockIdx.x];
    const InjRec3<T> *pl = plans + (long long)blockIdx.x * nsets;
    const int it = pl[0].rev ? pl[0].nt - 1 - it0 : it0;
    for (int k = 0; k < nsets; k++) {
        if (k) __syncthreads();
        inject_set<T, MODE>(sh, pl[k], dt, it);
    }
    __syncthreads();
    for (int k = 0; k < nsets; k++) record_set<T, MODE>(sh, pl[k], it);
}

template <bool ADJ>
cudaError_t step_e3_fast(int half, const void *args, const void *coefs, int grid, cudaStream_t st)
{
    const Step3DArgs<float> &a = *reinterpret_cast<const Step3DArgs<float> *>(args);
    const dim3 block(TX3, TY3);
    if (a.maps && !(half == 0 && ADJ)) {
        // TMA-staged planes (the adjoint velocity step differentiates work arrays formed
        // from five fields and keeps the register-staged kernel)
        if (half == 0) {
            auto k = e3d_velocity_tma;
            static const cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                              (int)tma_smem_bytes<VelStageT>());
            if (e != cudaSuccess) return e;
            k<<<grid, block, tma_smem_bytes<VelStageT>(), st>>>(a, (const CoefSet3<float> *)coefs);
        } else {
            auto k = e3d_stress_tma<ADJ>;
            static const cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                              (int)tma_smem_bytes<StrStageT>());
            if (e != cudaSuccess) return e;
            k<<<grid, block, tma_smem_bytes<StrStageT>(), st>>>(a, (const CoefSet3<float> *)coefs);
        }
        return cudaGetLastError();
    }
    if (half == 0) {
        auto k = e3d_velocity_fast<ADJ>;
        static const cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                          (int)sizeof(VelSmemF));
        if (e != cudaSuccess) return e;
        k<<<grid, block, sizeof(VelSmemF), st>>>(a, (const CoefSet3<float> *)coefs);
    } else {
        auto k = e3d_stress_fast<ADJ>;
        static const cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                          (int)sizeof(StrSmemF));
        if (e != cudaSuccess) return e;
        k<<<grid, block, sizeof(StrSmemF), st>>>(a, (const CoefSet3<float> *)coefs);
    }
    return cudaGetLastError();
}

template <typename T, int MODE, bool ADJ>
cudaError_t step_e3(int half, const void *args, const void *coefs, int grid, cudaStream_t st)
{
    const Step3DArgs<T> &a = *reinterpret_cast<const Step3DArgs<T> *>(args);
    const dim3 block(TX3, TY3);
    if (half == 0) {
        auto k = e3d_velocity<T, MODE, ADJ>;
        static const cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                          (int)sizeof(VelSmem<T>));
        if (e != cudaSuccess) return e;
        k<<<grid, block, sizeof(VelSmem<T>), st>>>(a, (const CoefSet3<T> *)coefs);
    } else {
        auto k = e3d_stress<T, MODE, ADJ>;
        static const cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                          (int)sizeof(StrSmem<T>));
        if (e != cudaSuccess) return e;
        k<<<grid, block, sizeof(StrSmem<T>), st>>>(a, (const CoefSet3<T> *)coefs);
    }
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_step_e3d(int prec, int half, int adj, const void *args, const void *coefs, int grid,
                            cudaStream_t st)
{
    if (prec == PREC_F64)
        return adj ? step_e3<double, MODE_IEEE, true>(half, args, coefs, grid, st)
                   : step_e3<double, MODE_IEEE, false>(half, args, coefs, grid, st);
    if (prec == PREC_F32_EXACT)
        return adj ? step_e3<float, MODE_IEEE, true>(half, args, coefs, grid, st)
                   : step_e3<float, MODE_IEEE, false>(half, args, coefs, grid, st);
    return adj ? step_e3_fast<true>(half, args, coefs, grid, st) : step_e3_fast<false>(half, args, coefs, grid, st);
}

// Work arrays of the adjoint velocity step (FAST arithmetic), the operands that
// opnd<.., ADJ=true> forms per tap, computed once per point over a shot's whole field
// allocation: W_xx = L2M Sxx + L Syy + L Szz, W_yy, W_zz likewise, W_yz = M_yz Syz,
// W_xz = M_xz Sxz, W_xy = M_xy Sxy.  The forward TMA velocity kernel then
// differentiates them as it differentiates stresses.  Four values per thread.
__global__ void __launch_bounds__(256) e3d_work_arrays(const WorkE3 *desc)
{
    using A = Ar<float, MODE_FAST>;
    const WorkE3 &e = desc[blockIdx.y];
    const long long n4 = e.n / 4;
    auto ld = [](const float *p, long long k) { return __ldg(reinterpret_cast<const float4 *>(p) + k); };
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n4; k += (long long)gridDim.x * blockDim.x) {
        const float4 sxx = ld(e.s[0], k), syy = ld(e.s[1], k), szz = ld(e.s[2], k);
        const float4 l = ld(e.l, k), l2m = ld(e.l2m, k);
        float4 wxx, wyy, wzz;
        const float *pxx = &sxx.x, *pyy = &syy.x, *pzz = &szz.x, *pl = &l.x, *pl2m = &l2m.x;
        float *oxx = &wxx.x, *oyy = &wyy.x, *ozz = &wzz.x;
#pragma unroll
        for (int c = 0; c < 4; c++) {
            oxx[c] = A::add(A::add(A::mul(pl2m[c], pxx[c]), A::mul(pl[c], pyy[c])), A::mul(pl[c], pzz[c]));
            oyy[c] = A::add(A::add(A::mul(pl[c], pxx[c]), A::mul(pl2m[c], pyy[c])), A::mul(pl[c], pzz[c]));
            ozz[c] = A::add(A::add(A::mul(pl[c], pxx[c]), A::mul(pl[c], pyy[c])), A::mul(pl2m[c], pzz[c]));
        }
        reinterpret_cast<float4 *>(e.w[0])[k] = wxx;
        reinterpret_cast<float4 *>(e.w[1])[k] = wyy;
        reinterpret_cast<float4 *>(e.w[2])[k] = wzz;
        const float4 syz = ld(e.s[3], k), sxz = ld(e.s[4], k), sxy = ld(e.s[5], k);
        const float4 myz = ld(e.myz, k), mxz = ld(e.mxz, k), mxy = ld(e.mxy, k);
        reinterpret_cast<float4 *>(e.w[3])[k] = make_float4(A::mul(myz.x, syz.x), A::mul(myz.y, syz.y),
                                                            A::mul(myz.z, syz.z), A::mul(myz.w, syz.w));
        reinterpret_cast<float4 *>(e.w[4])[k] = make_float4(A::mul(mxz.x, sxz.x), A::mul(mxz.y, sxz.y),
                                                            A::mul(mxz.z, sxz.z), A::mul(mxz.w, sxz.w));
        reinterpret_cast<float4 *>(e.w[5])[k] = make_float4(A::mul(mxy.x, sxy.x), A::mul(mxy.y, sxy.y),
                                                            A::mul(mxy.z, sxy.z), A::mul(mxy.w, sxy.w));
    }
}

cudaError_t launch_work_e3d(const void *desc, int nshots, cudaStream_t st)
{
    e3d_work_arrays<<<dim3(4 * 148, (unsigned)nshots), 256, 0, st>>>((const WorkE3 *)desc);
    return cudaGetLastError();
}

cudaError_t launch_injrec_e3d(int prec, const void *shots, const void *plans, int nshots, int nsets, double dt,
                              int it, cudaStream_t st)
{
    if (prec == PREC_F64)
        inject_record_e3d<double, MODE_IEEE><<<nshots, 256, 0, st>>>((const Shot3D<double> *)shots,
                                                                     (const InjRec3<double> *)plans, nsets, dt, it);
    else if (prec == PREC_F32_EXACT)
        inject_record_e3d<float, MODE_IEEE><<<nshots, 256, 0, st>>>((const Shot3D<float> *)shots,
                                                                    (const InjRec3<float> *)plans, nsets, (float)dt,
                                                                    it);
    else
        inject_record_e3d<float, MODE_FAST><<<nshots, 256, 0, st>>>((const Shot3D<float> *)shots,
                                                                    (const InjRec3<float> *)plans, nsets, (float)dt,
                                                                    it);
    return cudaGetLastError();
}

}  // namespace rsgpu
