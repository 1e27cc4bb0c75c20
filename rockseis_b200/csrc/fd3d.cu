// 3D acoustic staggered-grid propagator (WavesAcoustic3D, lib/waves.cpp:710-1190).
//
// Each CTA owns a TX3 x TY3 block of (x, y) columns of one shot and marches up
// the z axis through a chunk of planes.  Per plane:
//   - the z-derivative comes from a 16-plane register window per column
//     (fw: planes z-7..z+8, bw: z-8..z+7), shifted by one plane per step, so a
//     column's stencil values are loaded from HBM once;
//   - the x- and y-derivatives come from the plane tile staged in shared memory
//     with an 8-cell x/y halo (the centre from the register window, the halo
//     from L2-resident neighbours);
//   - the C-PML memory-variable update and correction of each face pair are fused
//     into the same pass.
// Arithmetic follows the reference operation by operation (MODE_IEEE: separately
// rounded ops and IEEE division; MODE_FAST: FMA, coefficients pre-divided).  Near
// the array ends the reference's reduced-order stencils are evaluated by
// stencil_k (the same rules as in 2D).  One launch covers all tiles of all shots.
#include <type_traits>

#include "fd2d_kernels.cuh"
#include "rsgpu_3d.h"

namespace rsgpu {
namespace {

static_assert(TX3 >= 16 && TY3 >= 8, "the halo fetch assigns one x-halo column per thread tx < 16 and two y-halo rows "
                                     "per thread ty < 8");

template <typename T>
__device__ __forceinline__ void load_coefs3(CoefSet3<T> &s, const CoefSet3<T> *g)
{
    const T *src = reinterpret_cast<const T *>(g);
    T *dst = reinterpret_cast<T *>(&s);
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    for (int i = tid; i < (int)(sizeof(CoefSet3<T>) / sizeof(T)); i += blockDim.x * blockDim.y) dst[i] = src[i];
}

// Staggered derivative with all NCOEF taps around b[7] (fw: b[0] = f[i-7]) or
// b[8] (bw: b[0] = f[i-8]); in both cases sum_k (b[8+k*s] - b[7-k*s]) c_k.  The
// coefficients are read from shared memory (one broadcast per tap), which keeps
// them out of the register file.
template <typename T, int MODE>
__device__ __forceinline__ T taps(const T *b, int s, const T *cu, T d, T r)
{
    using A = Ar<T, MODE>;
    T acc = A::mul(A::sub(b[8 * s], b[7 * s]), cu[0]);
#pragma unroll
    for (int k = 1; k < NCOEF; k++) acc = A::mad(acc, A::sub(b[(8 + k) * s], b[(7 - k) * s]), cu[k]);
    return (MODE == MODE_FAST) ? acc : A::div(acc, d, r);
}
template <typename T, int MODE>
__device__ __forceinline__ T taps_reg(const T (&q)[16], const T *cu, T d, T r)
{
    using A = Ar<T, MODE>;
    T acc = A::mul(A::sub(q[8], q[7]), cu[0]);
#pragma unroll
    for (int k = 1; k < NCOEF; k++) acc = A::mad(acc, A::sub(q[8 + k], q[7 - k]), cu[k]);
    return (MODE == MODE_FAST) ? acc : A::div(acc, d, r);
}

// Velocity half-step (lib/waves.cpp:710-851):
//   Vx += dt*Rx*Dx+P [x C-PML, staggered tables], Vy likewise in y, Vz in z.
// Software pipelined: the point-wise inputs and the x/y halo of plane iz+1 are
// requested while plane iz is computed, so their latency overlaps the arithmetic.
// (Plane ze, read by the last prefetch, lies inside the allocation; a value read
// there belongs to the next z-chunk and is not used.)
template <typename T, int MODE>
__global__ void __launch_bounds__(TX3 *TY3, 3) a3d_velocity(Step3DArgs<T> a, const CoefSet3<T> *coefs)
{
    using A = Ar<T, MODE>;
    __shared__ CoefSet3<T> cs;
    __shared__ T sPb[2][TY3 + 16][TX3 + 16];   // ping-pong: one barrier per plane
    load_coefs3(cs, coefs);
    const int tx = threadIdx.x, ty = threadIdx.y;
    const Tile3D tl = a.tiles[blockIdx.x];
    const Shot3D<T> &sh = a.shots[tl.shot];
    const int ix = tl.x0 + tx, iy = tl.y0 + ty;
    const int nxp = sh.nxp, nyp = sh.nyp, nzp = sh.nzp, pitch = sh.pitch, L = a.lpml, order = a.order;
    const long long plane = sh.plane;
    const int col = iy * pitch + ix;
    const T *P = sh.f[A3_P];
    T *Vx = sh.f[A3_VX], *Vy = sh.f[A3_VY], *Vz = sh.f[A3_VZ];
    const T *Rx = sh.m[M3_RX], *Ry = sh.m[M3_RY], *Rz = sh.m[M3_RZ];
    const bool in_grid = ix < nxp && iy < nyp;
    const int Kx = kfw(ix, nxp, order), Ky = kfw(iy, nyp, order);
    int xb = 0, xc = 0, yb = 0, yc = 0;
    const int xi = in_grid ? xstrip(ix, nxp, L, xb, xc) : -1;
    const int yi = in_grid ? xstrip(iy, nyp, L, yb, yc) : -1;
    const int z0 = tl.z0, ze = min(z0 + a.zc, nzp);
    // x halo: threads tx < 16 fetch one column each (tx < 8 left, 8..15 right);
    // y halo: threads ty < 8 fetch one row below and one above the block
    const int hx = tx < 8 ? -8 : TX3 - 8;
    T q[16];
#pragma unroll
    for (int j = 0; j < 16; j++) q[j] = P[(z0 - 7 + j) * plane + col];
    long long o = (long long)z0 * plane + col;
    T vx = Vx[o], vy = Vy[o], vz = Vz[o], rx = __ldg(Rx + o), ry = __ldg(Ry + o), rz = __ldg(Rz + o);
    T hxv = tx < 16 ? P[o + hx] : T(0);
    T hy0 = ty < 8 ? P[o - 8 * pitch] : T(0), hy1 = ty < 8 ? P[o + TY3 * pitch] : T(0);
    const T *cux = cs.cx + order * CROW3, *cuy = cs.cy + order * CROW3, *cuz = cs.cz + order * CROW3;
    for (int iz = z0; iz < ze; iz++, o += plane) {
        // the buffer written here was last read two planes ago, before the
        // previous plane's barrier
        T (*sP)[TX3 + 16] = sPb[(iz - z0) & 1];
        sP[ty + 8][tx + 8] = q[7];
        if (tx < 16) sP[ty + 8][tx < 8 ? tx : tx + TX3] = hxv;
        if (ty < 8) {
            sP[ty][tx + 8] = hy0;
            sP[ty + TY3 + 8][tx + 8] = hy1;
        }
        // next plane's inputs
        const long long on = o + plane;
        const T nvx = Vx[on], nvy = Vy[on], nvz = Vz[on];
        const T nrx = __ldg(Rx + on), nry = __ldg(Ry + on), nrz = __ldg(Rz + on);
        if (tx < 16) hxv = P[on + hx];
        if (ty < 8) {
            hy0 = P[on - 8 * pitch];
            hy1 = P[on + TY3 * pitch];
        }
        __syncthreads();
        const T *cx = &sP[ty + 8][tx + 8];
        const T dfx = (Kx == order) ? taps<T, MODE>(cx - 7, 1, cux, a.dx, a.rdx)
                                    : stencil_ki<T, MODE>(cx, 1, Kx, cs.cx + Kx * CROW3, true, a.dx, a.rdx);
        const T dfy = (Ky == order) ? taps<T, MODE>(cx - 7 * (TX3 + 16), TX3 + 16, cuy, a.dy, a.rdy)
                                    : stencil_ki<T, MODE>(cx, TX3 + 16, Ky, cs.cy + Ky * CROW3, true, a.dy, a.rdy);
        const int Kz = kfw(iz, nzp, order);
        const T dfz = (Kz == order) ? taps_reg<T, MODE>(q, cuz, a.dz, a.rdz)
                                    : stencil_ki<T, MODE>(P + o, (int)plane, Kz, cs.cz + Kz * CROW3, true, a.dz, a.rdz);
        T am = A::mul(a.dt, rx);
        vx = A::mad(vx, am, dfx);
        if (xi >= 0)
            vx = pml_correct<T, MODE>(vx, am, dfx, sh.psix[0] + ((long long)iz * nyp + iy) * 2 * L + xc, a.pml, L,
                                      xb + 3, xi);
        Vx[o] = vx;
        am = A::mul(a.dt, ry);
        vy = A::mad(vy, am, dfy);
        if (yi >= 0)
            vy = pml_correct<T, MODE>(vy, am, dfy, sh.psiy[0] + ((long long)iz * 2 * L + yc) * nxp + ix, a.pml, L,
                                      yb + 3, yi);
        Vy[o] = vy;
        am = A::mul(a.dt, rz);
        vz = A::mad(vz, am, dfz);
        int zb = 0, zc = 0;
        const int zi = in_grid ? xstrip(iz, nzp, L, zb, zc) : -1;
        if (zi >= 0)
            vz = pml_correct<T, MODE>(vz, am, dfz, sh.psiz[0] + ((long long)zc * nyp + iy) * nxp + ix, a.pml, L,
                                      zb + 3, zi);
        Vz[o] = vz;
#pragma unroll
        for (int j = 0; j < 15; j++) q[j] = q[j + 1];
        q[15] = P[o + 9 * plane];
        vx = nvx; vy = nvy; vz = nvz; rx = nrx; ry = nry; rz = nrz;
    }
}

// Stress half-step (lib/waves.cpp:854-998):
//   P += dt*L*Dx-Vx [x C-PML]; P += dt*L*Dy-Vy [y]; P += dt*L*Dz-Vz [z].
// Pipelined like the velocity half-step.
template <typename T, int MODE>
__global__ void __launch_bounds__(TX3 *TY3, 3) a3d_stress(Step3DArgs<T> a, const CoefSet3<T> *coefs)
{
    using A = Ar<T, MODE>;
    __shared__ CoefSet3<T> cs;
    __shared__ T sVxb[2][TY3][TX3 + 16];       // ping-pong: one barrier per plane
    __shared__ T sVyb[2][TY3 + 16][TX3];
    load_coefs3(cs, coefs);
    const int tx = threadIdx.x, ty = threadIdx.y;
    const Tile3D tl = a.tiles[blockIdx.x];
    const Shot3D<T> &sh = a.shots[tl.shot];
    const int ix = tl.x0 + tx, iy = tl.y0 + ty;
    const int nxp = sh.nxp, nyp = sh.nyp, nzp = sh.nzp, pitch = sh.pitch, L = a.lpml, order = a.order;
    const long long plane = sh.plane;
    const int col = iy * pitch + ix;
    T *P = sh.f[A3_P];
    const T *Vx = sh.f[A3_VX], *Vy = sh.f[A3_VY], *Vz = sh.f[A3_VZ];
    const T *Lm = sh.m[M3_L];
    const bool in_grid = ix < nxp && iy < nyp;
    const int Kx = kbw(ix, nxp, order), Ky = kbw(iy, nyp, order);
    int xb = 0, xc = 0, yb = 0, yc = 0;
    const int xi = in_grid ? xstrip(ix, nxp, L, xb, xc) : -1;
    const int yi = in_grid ? xstrip(iy, nyp, L, yb, yc) : -1;
    const int z0 = tl.z0, ze = min(z0 + a.zc, nzp);
    const int hx = tx < 8 ? -8 : TX3 - 8;
    T q[16];
#pragma unroll
    for (int j = 0; j < 16; j++) q[j] = Vz[(z0 - 8 + j) * plane + col];
    long long o = (long long)z0 * plane + col;
    T p = P[o], lm = __ldg(Lm + o), vxc = Vx[o], vyc = Vy[o];
    T hxv = tx < 16 ? Vx[o + hx] : T(0);
    T hy0 = ty < 8 ? Vy[o - 8 * pitch] : T(0), hy1 = ty < 8 ? Vy[o + TY3 * pitch] : T(0);
    const T *cux = cs.cx + order * CROW3, *cuy = cs.cy + order * CROW3, *cuz = cs.cz + order * CROW3;
    for (int iz = z0; iz < ze; iz++, o += plane) {
        T (*sVx)[TX3 + 16] = sVxb[(iz - z0) & 1];
        T (*sVy)[TX3] = sVyb[(iz - z0) & 1];
        sVx[ty][tx + 8] = vxc;
        sVy[ty + 8][tx] = vyc;
        if (tx < 16) sVx[ty][tx < 8 ? tx : tx + TX3] = hxv;
        if (ty < 8) {
            sVy[ty][tx] = hy0;
            sVy[ty + TY3 + 8][tx] = hy1;
        }
        const long long on = o + plane;
        const T np_ = P[on], nlm = __ldg(Lm + on), nvx = Vx[on], nvy = Vy[on];
        if (tx < 16) hxv = Vx[on + hx];
        if (ty < 8) {
            hy0 = Vy[on - 8 * pitch];
            hy1 = Vy[on + TY3 * pitch];
        }
        __syncthreads();
        const T *cx = &sVx[ty][tx + 8];
        const T *cy = &sVy[ty + 8][tx];
        const T d1 = (Kx == order) ? taps<T, MODE>(cx - 8, 1, cux, a.dx, a.rdx)
                                   : stencil_ki<T, MODE>(cx, 1, Kx, cs.cx + Kx * CROW3, false, a.dx, a.rdx);
        const T d2 = (Ky == order) ? taps<T, MODE>(cy - 8 * TX3, TX3, cuy, a.dy, a.rdy)
                                   : stencil_ki<T, MODE>(cy, TX3, Ky, cs.cy + Ky * CROW3, false, a.dy, a.rdy);
        const int Kz = kbw(iz, nzp, order);
        const T d3 = (Kz == order) ? taps_reg<T, MODE>(q, cuz, a.dz, a.rdz)
                                   : stencil_ki<T, MODE>(Vz + o, (int)plane, Kz, cs.cz + Kz * CROW3, false, a.dz, a.rdz);
        const T am = A::mul(a.dt, lm);
        p = A::mad(p, am, d1);
        if (xi >= 0)
            p = pml_correct<T, MODE>(p, am, d1, sh.psix[1] + ((long long)iz * nyp + iy) * 2 * L + xc, a.pml, L, xb,
                                     xi);
        p = A::mad(p, am, d2);
        if (yi >= 0)
            p = pml_correct<T, MODE>(p, am, d2, sh.psiy[1] + ((long long)iz * 2 * L + yc) * nxp + ix, a.pml, L, yb,
                                     yi);
        p = A::mad(p, am, d3);
        int zb = 0, zc = 0;
        const int zi = in_grid ? xstrip(iz, nzp, L, zb, zc) : -1;
        if (zi >= 0)
            p = pml_correct<T, MODE>(p, am, d3, sh.psiz[1] + ((long long)zc * nyp + iy) * nxp + ix, a.pml, L, zb,
                                     zi);
        P[o] = p;
#pragma unroll
        for (int j = 0; j < 15; j++) q[j] = q[j + 1];
        q[15] = Vz[o + 8 * plane];
        p = np_; lm = nlm; vxc = nvx; vyc = nvy;
    }
}

// Source injection then receiver recording of one step, one CTA per shot
// (lib/waves.cpp:999-1190).
template <typename T, int MODE>
__global__ void inject_record_3d(const Shot3D<T> *shots, const InjRec3<T> *plans, T dt, int it)
{
    using A = Ar<T, MODE == MODE_FAST ? MODE_FAST : MODE_IEEE>;
    const Shot3D<T> &sh = shots[blockIdx.x];
    const InjRec3<T> &pl = plans[blockIdx.x];
    it = pl.rev ? pl.nt - 1 - it : it;
    if (pl.kind_inj != INJ3_NONE) {
        T *F = sh.f[pl.kind_inj == INJ3_P ? A3_P : pl.kind_inj == INJ3_VX ? A3_VX : pl.kind_inj == INJ3_VY ? A3_VY : A3_VZ];
        const T *Mod = sh.m[pl.kind_inj == INJ3_P ? M3_L : pl.kind_inj == INJ3_VX ? M3_RX : pl.kind_inj == INJ3_VY ? M3_RY : M3_RZ];
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
    if (pl.kind_rec == REC3_NONE || (pl.rec_gate && *pl.rec_gate == 0)) return;
    __syncthreads();
    const T *F = sh.f[pl.kind_rec == REC3_P ? A3_P : pl.kind_rec == REC3_VX ? A3_VX : pl.kind_rec == REC3_VY ? A3_VY : A3_VZ];
    for (int tr = threadIdx.x; tr < pl.nrec; tr += blockDim.x) {
        const long long p = pl.rec_pt[tr];
        if (p < 0) continue;
        const T *w = pl.rec_w + 6 * tr;
        T *out = pl.rec_out + (long long)tr * pl.nt + it;
        T acc = *out;
        for (int i1 = 0; i1 < 2; i1++)
            for (int i2 = 0; i2 < 2; i2++)
                for (int i3 = 0; i3 < 2; i3++)
                    acc = A::add(acc, A::mul(A::mul(A::mul(w[i3], w[2 + i2]), w[4 + i1]),
                                             F[p + i1 * sh.plane + (long long)i2 * sh.pitch + i3]));
        *out = acc;
    }
}

// ---------------------------------------------------------------- fast mode with TMA-staged planes
// The two half-steps of RSGPU_F32_FAST with every plane tile brought in by TMA
// (cp.async.bulk.tensor.2d issued by one thread, completion on an mbarrier per
// stage) two planes ahead of the plane being computed, so the loads in flight do
// not depend on registers or resident warps.  The z-derivative still comes from the
// 16-plane register window, refilled by a plain load eight planes ahead.  Same
// stencils, C-PML and update order as a3d_velocity / a3d_stress.  Every wait is
// bounded (2 s): on timeout the CTA records RSGPU_ERR_TIMEOUT and stops.
constexpr int NSTG_A3 = 3;

struct A3VelStage {
    float p[HY3][WX3];         // P with its x and y halos
    float pv[6][TY3][TX3];     // Vx, Vy, Vz, Rx, Ry, Rz
};
struct A3StrStage {
    float vx[TY3][WX3];        // Vx, x halo
    float vy[HY3][TX3];        // Vy, y halo
    float pl[2][TY3][TX3];     // P, L
};
static_assert(sizeof(A3VelStage) % 128 == 0 && sizeof(A3StrStage) % 128 == 0, "TMA destinations stay 128-byte aligned");
static_assert(sizeof(float) * HY3 * WX3 % 128 == 0 && sizeof(float) * TY3 * WX3 % 128 == 0 &&
              sizeof(float) * HY3 * TX3 % 128 == 0 && sizeof(float) * TY3 * TX3 % 128 == 0, "tile sizes");

template <typename Stage>
struct A3Smem {
    Stage st[NSTG_A3];
    uint64_t bar[NSTG_A3];
    CoefSet3<float> cs;
};
template <typename Stage>
constexpr size_t a3_smem_bytes() { return sizeof(A3Smem<Stage>) + 128; }   // + alignment slack

// Allocation row of plane iz, padded row iy_alloc (guards included).
__device__ __forceinline__ int a3_row(const Shot3D<float> &sh, int iz, int iy_alloc)
{
    return (GUARD + iz) * sh.rows + iy_alloc;
}

__global__ void __launch_bounds__(TX3 *TY3, 3) a3d_velocity_tma(Step3DArgs<float> a, const CoefSet3<float> *coefs)
{
    using T = float;
    constexpr int MODE = MODE_FAST;
    using A = Ar<T, MODE>;
    extern __shared__ unsigned char smraw[];
    A3Smem<A3VelStage> &S =
        *reinterpret_cast<A3Smem<A3VelStage> *>((reinterpret_cast<uintptr_t>(smraw) + 127) & ~uintptr_t(127));
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX3 + tx;
    const Tile3D tl = a.tiles[blockIdx.x];
    const Shot3D<T> &sh = a.shots[tl.shot];
    load_coefs3(S.cs, coefs);
    if (tid == 0)
        for (int k = 0; k < NSTG_A3; k++) mbar_init(&S.bar[k], 1);
    __syncthreads();
    const CUtensorMap *M = reinterpret_cast<const CUtensorMap *>(a.maps) + (size_t)tl.shot * NMAP_A3;
    const int x0 = tl.x0, y0 = tl.y0, ix = x0 + tx, iy = y0 + ty;
    const int nxp = sh.nxp, nyp = sh.nyp, nzp = sh.nzp, pitch = sh.pitch, L = a.lpml, order = a.order;
    const long long plane = sh.plane;
    const int col = iy * pitch + ix;
    const T *P = sh.f[A3_P];
    T *Vx = sh.f[A3_VX], *Vy = sh.f[A3_VY], *Vz = sh.f[A3_VZ];
    const bool in_grid = ix < nxp && iy < nyp;
    const int Kx = kfw(ix, nxp, order), Ky = kfw(iy, nyp, order);
    int xb = 0, xc = 0, yb = 0, yc = 0;
    const int xi = in_grid ? xstrip(ix, nxp, L, xb, xc) : -1;
    const int yi = in_grid ? xstrip(iy, nyp, L, yb, yc) : -1;
    const int z0 = tl.z0, ze = min(z0 + a.zc, nzp);
    // stage k <- plane iz; the boxes start on 16-byte boundaries (x0, x0 + 8 multiples of 4)
    auto issue = [&](int iz, int k) {
        A3VelStage &g = S.st[k];
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        mbar_expect_tx(&S.bar[k], (uint32_t)sizeof(A3VelStage));
        tma_load_2d(g.p, M + AM_PH, &S.bar[k], x0, a3_row(sh, iz, y0));
        for (int q = 0; q < 6; q++) tma_load_2d(g.pv[q], M + AM_VX + q, &S.bar[k], x0 + GUARD, a3_row(sh, iz, GUARD + y0));
    };
    if (tid == 0)
        for (int j = 0; j < NSTG_A3 - 1 && z0 + j < ze; j++) issue(z0 + j, j);
    T q[16];                                     // P, planes z-7..z+8 (forward z-derivative)
#pragma unroll
    for (int j = 0; j < 16; j++) q[j] = P[(z0 - 7 + j) * plane + col];
    const T *cux = S.cs.cx + order * CROW3, *cuy = S.cs.cy + order * CROW3, *cuz = S.cs.cz + order * CROW3;
    long long o = (long long)z0 * plane + col;
    for (int iz = z0; iz < ze; iz++, o += plane) {
        const int j = iz - z0, k = j % NSTG_A3;
        if (tid == 0 && iz + NSTG_A3 - 1 < ze) issue(iz + NSTG_A3 - 1, (j + NSTG_A3 - 1) % NSTG_A3);
        const T nq = P[o + 9 * plane];          // window refill, in flight while the stage arrives
        if (!__syncthreads_and(mbar_wait_bounded(&S.bar[k], (uint32_t)(j / NSTG_A3) & 1u, a.err))) return;
        const A3VelStage &g = S.st[k];
        const T *cx = &g.p[ty + 8][tx + 8];
        const T dfx = (Kx == order) ? taps<T, MODE>(cx - 7, 1, cux, a.dx, a.rdx)
                                    : stencil_ki<T, MODE>(cx, 1, Kx, S.cs.cx + Kx * CROW3, true, a.dx, a.rdx);
        const T dfy = (Ky == order) ? taps<T, MODE>(cx - 7 * WX3, WX3, cuy, a.dy, a.rdy)
                                    : stencil_ki<T, MODE>(cx, WX3, Ky, S.cs.cy + Ky * CROW3, true, a.dy, a.rdy);
        const int Kz = kfw(iz, nzp, order);
        const T dfz = (Kz == order) ? taps_reg<T, MODE>(q, cuz, a.dz, a.rdz)
                                    : stencil_ki<T, MODE>(P + o, (int)plane, Kz, S.cs.cz + Kz * CROW3, true, a.dz, a.rdz);
        T vx = g.pv[0][ty][tx], vy = g.pv[1][ty][tx], vz = g.pv[2][ty][tx];
        T am = A::mul(a.dt, g.pv[3][ty][tx]);
        vx = A::mad(vx, am, dfx);
        if (xi >= 0)
            vx = pml_correct<T, MODE>(vx, am, dfx, sh.psix[0] + ((long long)iz * nyp + iy) * 2 * L + xc, a.pml, L,
                                      xb + 3, xi);
        Vx[o] = vx;
        am = A::mul(a.dt, g.pv[4][ty][tx]);
        vy = A::mad(vy, am, dfy);
        if (yi >= 0)
            vy = pml_correct<T, MODE>(vy, am, dfy, sh.psiy[0] + ((long long)iz * 2 * L + yc) * nxp + ix, a.pml, L,
                                      yb + 3, yi);
        Vy[o] = vy;
        am = A::mul(a.dt, g.pv[5][ty][tx]);
        vz = A::mad(vz, am, dfz);
        int zb = 0, zc = 0;
        const int zi = in_grid ? xstrip(iz, nzp, L, zb, zc) : -1;
        if (zi >= 0)
            vz = pml_correct<T, MODE>(vz, am, dfz, sh.psiz[0] + ((long long)zc * nyp + iy) * nxp + ix, a.pml, L,
                                      zb + 3, zi);
        Vz[o] = vz;
#pragma unroll
        for (int jj = 0; jj < 15; jj++) q[jj] = q[jj + 1];
        q[15] = nq;
        __syncthreads();   // stage k is refilled next iteration
    }
}

__global__ void __launch_bounds__(TX3 *TY3, 3) a3d_stress_tma(Step3DArgs<float> a, const CoefSet3<float> *coefs)
{
    using T = float;
    constexpr int MODE = MODE_FAST;
    using A = Ar<T, MODE>;
    extern __shared__ unsigned char smraw[];
    A3Smem<A3StrStage> &S =
        *reinterpret_cast<A3Smem<A3StrStage> *>((reinterpret_cast<uintptr_t>(smraw) + 127) & ~uintptr_t(127));
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX3 + tx;
    const Tile3D tl = a.tiles[blockIdx.x];
    const Shot3D<T> &sh = a.shots[tl.shot];
    load_coefs3(S.cs, coefs);
    if (tid == 0)
        for (int k = 0; k < NSTG_A3; k++) mbar_init(&S.bar[k], 1);
    __syncthreads();
    const CUtensorMap *M = reinterpret_cast<const CUtensorMap *>(a.maps) + (size_t)tl.shot * NMAP_A3;
    const int x0 = tl.x0, y0 = tl.y0, ix = x0 + tx, iy = y0 + ty;
    const int nxp = sh.nxp, nyp = sh.nyp, nzp = sh.nzp, pitch = sh.pitch, L = a.lpml, order = a.order;
    const long long plane = sh.plane;
    const int col = iy * pitch + ix;
    T *P = sh.f[A3_P];
    const T *Vz = sh.f[A3_VZ];
    const bool in_grid = ix < nxp && iy < nyp;
    const int Kx = kbw(ix, nxp, order), Ky = kbw(iy, nyp, order);
    int xb = 0, xc = 0, yb = 0, yc = 0;
    const int xi = in_grid ? xstrip(ix, nxp, L, xb, xc) : -1;
    const int yi = in_grid ? xstrip(iy, nyp, L, yb, yc) : -1;
    const int z0 = tl.z0, ze = min(z0 + a.zc, nzp);
    auto issue = [&](int iz, int k) {
        A3StrStage &g = S.st[k];
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        mbar_expect_tx(&S.bar[k], (uint32_t)sizeof(A3StrStage));
        const int rh = a3_row(sh, iz, GUARD + y0);
        tma_load_2d(g.vx, M + AM_VXH, &S.bar[k], x0, rh);
        tma_load_2d(g.vy, M + AM_VYH, &S.bar[k], x0 + GUARD, a3_row(sh, iz, y0));
        tma_load_2d(g.pl[0], M + AM_P, &S.bar[k], x0 + GUARD, rh);
        tma_load_2d(g.pl[1], M + AM_L, &S.bar[k], x0 + GUARD, rh);
    };
    if (tid == 0)
        for (int j = 0; j < NSTG_A3 - 1 && z0 + j < ze; j++) issue(z0 + j, j);
    T q[16];                                     // Vz, planes z-8..z+7 (backward z-derivative)
#pragma unroll
    for (int j = 0; j < 16; j++) q[j] = Vz[(z0 - 8 + j) * plane + col];
    const T *cux = S.cs.cx + order * CROW3, *cuy = S.cs.cy + order * CROW3, *cuz = S.cs.cz + order * CROW3;
    long long o = (long long)z0 * plane + col;
    for (int iz = z0; iz < ze; iz++, o += plane) {
        const int j = iz - z0, k = j % NSTG_A3;
        if (tid == 0 && iz + NSTG_A3 - 1 < ze) issue(iz + NSTG_A3 - 1, (j + NSTG_A3 - 1) % NSTG_A3);
        const T nq = Vz[o + 8 * plane];
        if (!__syncthreads_and(mbar_wait_bounded(&S.bar[k], (uint32_t)(j / NSTG_A3) & 1u, a.err))) return;
        const A3StrStage &g = S.st[k];
        const T *cx = &g.vx[ty][tx + 8];
        const T *cy = &g.vy[ty + 8][tx];
        const T d1 = (Kx == order) ? taps<T, MODE>(cx - 8, 1, cux, a.dx, a.rdx)
                                   : stencil_ki<T, MODE>(cx, 1, Kx, S.cs.cx + Kx * CROW3, false, a.dx, a.rdx);
        const T d2 = (Ky == order) ? taps<T, MODE>(cy - 8 * TX3, TX3, cuy, a.dy, a.rdy)
                                   : stencil_ki<T, MODE>(cy, TX3, Ky, S.cs.cy + Ky * CROW3, false, a.dy, a.rdy);
        const int Kz = kbw(iz, nzp, order);
        const T d3 = (Kz == order) ? taps_reg<T, MODE>(q, cuz, a.dz, a.rdz)
                                   : stencil_ki<T, MODE>(Vz + o, (int)plane, Kz, S.cs.cz + Kz * CROW3, false, a.dz, a.rdz);
        T p = g.pl[0][ty][tx];
        const T am = A::mul(a.dt, g.pl[1][ty][tx]);
        p = A::mad(p, am, d1);
        if (xi >= 0)
            p = pml_correct<T, MODE>(p, am, d1, sh.psix[1] + ((long long)iz * nyp + iy) * 2 * L + xc, a.pml, L, xb,
                                     xi);
        p = A::mad(p, am, d2);
        if (yi >= 0)
            p = pml_correct<T, MODE>(p, am, d2, sh.psiy[1] + ((long long)iz * 2 * L + yc) * nxp + ix, a.pml, L, yb,
                                     yi);
        p = A::mad(p, am, d3);
        int zb = 0, zc = 0;
        const int zi = in_grid ? xstrip(iz, nzp, L, zb, zc) : -1;
        if (zi >= 0)
            p = pml_correct<T, MODE>(p, am, d3, sh.psiz[1] + ((long long)zc * nyp + iy) * nxp + ix, a.pml, L, zb,
                                     zi);
        P[o] = p;
#pragma unroll
        for (int jj = 0; jj < 15; jj++) q[jj] = q[jj + 1];
        q[15] = nq;
        __syncthreads();
    }
}

template <typename T, int MODE>
cudaError_t step3(int half, const void *args, const void *coefs, int grid, cudaStream_t st)
{
    const Step3DArgs<T> &a = *reinterpret_cast<const Step3DArgs<T> *>(args);
    const dim3 block(TX3, TY3);
    if constexpr (MODE == MODE_FAST && std::is_same<T, float>::value) {
        if (a.maps) {
            // TMA-staged planes (the plan builds the maps in fast mode)
            if (half == 0) {
                auto k = a3d_velocity_tma;
                const size_t sm = a3_smem_bytes<A3VelStage>();
                cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
                if (e != cudaSuccess) return e;
                k<<<grid, block, sm, st>>>(a, (const CoefSet3<float> *)coefs);
            } else {
                auto k = a3d_stress_tma;
                const size_t sm = a3_smem_bytes<A3StrStage>();
                cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
                if (e != cudaSuccess) return e;
                k<<<grid, block, sm, st>>>(a, (const CoefSet3<float> *)coefs);
            }
            return cudaGetLastError();
        }
    }
    if (half == 0) a3d_velocity<T, MODE><<<grid, block, 0, st>>>(a, (const CoefSet3<T> *)coefs);
    else a3d_stress<T, MODE><<<grid, block, 0, st>>>(a, (const CoefSet3<T> *)coefs);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_step_3d(int prec, int physics, int half, const void *args, const void *coefs, int grid,
                           cudaStream_t st)
{
    if (physics != PHYS_A3D) return cudaErrorInvalidValue;
    if (prec == PREC_F64) return step3<double, MODE_IEEE>(half, args, coefs, grid, st);
    if (prec == PREC_F32_EXACT) return step3<float, MODE_IEEE>(half, args, coefs, grid, st);
    return step3<float, MODE_FAST>(half, args, coefs, grid, st);
}

cudaError_t launch_injrec_3d(int prec, const void *shots, const void *plans, int nshots, double dt, int it,
                             cudaStream_t st)
{
    if (prec == PREC_F64)
        inject_record_3d<double, MODE_IEEE><<<nshots, 256, 0, st>>>((const Shot3D<double> *)shots,
                                                                    (const InjRec3<double> *)plans, dt, it);
    else if (prec == PREC_F32_EXACT)
        inject_record_3d<float, MODE_IEEE><<<nshots, 256, 0, st>>>((const Shot3D<float> *)shots,
                                                                   (const InjRec3<float> *)plans, (float)dt, it);
    else
        inject_record_3d<float, MODE_FAST><<<nshots, 256, 0, st>>>((const Shot3D<float> *)shots,
                                                                   (const InjRec3<float> *)plans, (float)dt, it);
    return cudaGetLastError();
}

}  // namespace rsgpu
