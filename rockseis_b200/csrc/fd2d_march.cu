// Column-marching elastic 2D half-steps (FAST arithmetic, forward propagation;
// rsgpu_config.launch_mode 4).
//
// A CTA of MW warps owns a strip of MSTRIP2D columns of one shot and a band of rows
// [z0, z1) and walks down the band one row at a time; every thread holds one
// column.
//   - The two fields that are z-differentiated live in 16-row register windows
//     (one new row enters each window per step).  The z-derivatives are FMA sums
//     over the window in row order with -c / +c terms: the summation order of the
//     per-tile FAST kernels (dz_stream_f32), so both give bit-identical wavefields.
//   - The fields that are x-differentiated arrive by TMA in a circular ring of
//     RING_ROWS rows (MNS chunks of MCH rows), MSTRIP2D + 16 columns wide (the x
//     halo), filled up to three chunks ahead; x-derivatives are scalar FMAs in the
//     per-tile kernels' tap order (dx_quad).
//   - Point-wise inputs (the updated fields, densities and moduli) are loaded one
//     row ahead into registers; their rows two chunks ahead are prefetched into L2
//     by bulk prefetches issued beside the ring's TMA loads.
// Rows and strips away from the C-PML strips and the array ends run a lean path;
// the others run the general path, which applies the reduced-order stencils near
// the array ends (lib/der.cpp's rule, from the ring row or the register window)
// and the C-PML memory updates operation by operation like the per-tile kernels
// (lib/waves.cpp:1416-1735).
#include "fd2d_kernels.cuh"

namespace rsgpu {

namespace {

constexpr int MW = 4;                        // warps per CTA
constexpr int MNT = 32 * MW;                 // threads per CTA (one column each)
constexpr int MRW = MSTRIP2D + 2 * GUARD;    // ring row: the strip plus the x halo
constexpr int MCH = 8;                       // rows per TMA chunk
constexpr int MNS = 4;                       // chunks in the ring
constexpr int RING_ROWS = MCH * MNS;         // a power of two: ring row = r & (RING_ROWS - 1)
constexpr int MINB_MARCH = 4;                // resident CTAs per SM requested from the allocator
static_assert(MSTRIP2D == 32 * MW, "one column per thread");
static_assert((RING_ROWS & (RING_ROWS - 1)) == 0, "ring rows");

constexpr int WIN = 15 + MCH;               // window registers: 16 rows for each row of a group
template <int NF>                             // NF ring fields (velocity 3, stress 2)
struct MarchSmem {
    float ring[NF][RING_ROWS][MRW];
    float coef[2 * 9 * CROW];   // CoefSet<float>: per-K x rows, then per-K z rows
    uint64_t bar[MNS];
};
constexpr size_t march_smem(int nf) { return nf == 3 ? sizeof(MarchSmem<3>) : sizeof(MarchSmem<2>); }

// L2 prefetch of `bytes` contiguous bytes (16-byte aligned start and size).
__device__ __forceinline__ void prefetch_l2(const void *p, uint32_t bytes)
{
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

// x-derivative of one column on a ring row; `row` points at the column.
// FW: f[i+k+1] - f[i-k]; BW: f[i+k] - f[i-k-1]; taps in dx_quad's order.
template <bool FW>
__device__ __forceinline__ float dx_col(const float *row, const float *c)
{
    float acc = FW ? (row[1] - row[0]) * c[0] : (row[0] - row[-1]) * c[0];
#pragma unroll
    for (int k = 1; k < NCOEF; k++) {
        const float dl = FW ? row[k + 1] - row[-k] : row[k] - row[-k - 1];
        acc = fmaf(dl, c[k], acc);
    }
    return acc;
}

// Reduced-order stencils of K pairs (stencil_k's arithmetic) near the array ends,
// unrolled with the taps beyond K predicated off: on a ring row (x, sk_row) or on
// a register window (z, sk_at: forward and backward windows both hold the taps
// at 8+k / 7-k).  c = the K row of the coefficient table in shared memory.
template <bool FW>
__device__ __forceinline__ float sk_row(const float *row, int K, const float *c)
{
    float acc = (FW ? row[1] - row[0] : row[0] - row[-1]) * c[0];
#pragma unroll
    for (int k = 1; k < NCOEF; k++)
        if (k < K) acc = fmaf(FW ? row[k + 1] - row[-k] : row[k] - row[-k - 1], c[k], acc);
    return K == 0 ? 0.f : acc;
}
// One C-PML memory update with the memory value already loaded (pml_correct's
// arithmetic): psi = B*psi + A*df; F -= a*(psi + C*df).
__device__ __forceinline__ float pml_step(float F, float a, float df, float &psi, const float *tab, int L, int base,
                                          int idx)
{
    const float tA = __ldg(tab + (base + PT_A) * L + idx), tB = __ldg(tab + (base + PT_B) * L + idx),
                tC = __ldg(tab + (base + PT_C) * L + idx);
    psi = fmaf(tA, df, tB * psi);
    return fmaf(-a, fmaf(tC, df, psi), F);
}

// F += am*d1 [x memory] ; F += am*d2 [z memory]  (update_field, FAST)
template <bool GEN>
__device__ __forceinline__ float upd(float F, float am, float d1, float d2, int xi, float &px, int xtab, int zi,
                                     float &pz, int ztab, const float *pml, int L)
{
    F = fmaf(am, d1, F);
    if (GEN && xi >= 0) F = pml_step(F, am, d1, px, pml, L, xtab, xi);
    F = fmaf(am, d2, F);
    if (GEN && zi >= 0) F = pml_step(F, am, d2, pz, pml, L, ztab, zi);
    return F;
}

// Per-thread geometry.
struct Lane {
    int cx;         // field column
    int rc;         // its ring column
    int xi, xb, xc; // C-PML x strip index / table base / psix column (xi = -1: none)
    int kf, kb;     // forward / backward stencil pairs at the column
    bool in;        // column inside the padded grid
};

__device__ __forceinline__ Lane make_lane(const MarchItem &it, const Shot2D<float> &sh, int L, int order)
{
    Lane n{};
    n.cx = it.x0 + (int)threadIdx.x;
    n.rc = GUARD + (int)threadIdx.x;
    n.xi = xstrip(n.cx, sh.nxp, L, n.xb, n.xc);
    n.kf = kfw(n.cx, sh.nxp, order);
    n.kb = kbw(n.cx, sh.nxp, order);
    n.in = n.cx < sh.nxp;
    return n;
}

// Ring control: chunk c holds field rows z0 - 8 + MCH*c .. +MCH-1 of the NF ring
// fields in ring rows MCH*(c % MNS)..; the n-th use of a chunk slot waits on
// parity n & 1.
template <int NF>
struct Ring {
    MarchSmem<NF> *S;
    const CUtensorMap *m[NF];
    int x0, z0, nch;
    __device__ __forceinline__ void issue(int c) const
    {
        const int s = c % MNS;
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        mbar_expect_tx(&S->bar[s], (uint32_t)(NF * MCH * MRW * sizeof(float)));
        // allocation row of field row z0 - 8 + MCH*c is z0 + MCH*c; allocation column x0
        // is field column x0 - 8 (x0 is a multiple of the strip: 16-byte aligned)
#pragma unroll
        for (int f = 0; f < NF; f++) tma_load_2d(&S->ring[f][MCH * s][0], m[f], &S->bar[s], x0, z0 + MCH * c);
    }
    __device__ __forceinline__ bool wait(int c, int *err) const
    {
        return c >= nch || mbar_wait_bounded(&S->bar[c % MNS], (uint32_t)((c / MNS) & 1), err);
    }
};

// Rows zrow..zrow+7 of the point-wise fields, prefetched into L2 (one row of the
// strip per thread, NP fields).
template <int NP>
__device__ __forceinline__ void prefetch_rows(const float *const *pf, int pitch, int x0, int zrow, int z1)
{
    const int t = threadIdx.x;
    if (t < NP * MCH) {
        const int f = t / MCH, z = zrow + t % MCH;
        if (z < z1) prefetch_l2(pf[f] + (long)z * pitch + x0, MSTRIP2D * sizeof(float));
    }
}

// Rows [zlo, zhi) need neither reduced-order z stencils nor z C-PML memory.
__device__ __forceinline__ void plain_rows(int nzp, int L, int order, int &zlo, int &zhi)
{
    zlo = max(L, order);
    zhi = nzp - max(L, order + 1);
}

// Windows over a group of MCH rows starting at zg (ring row r0 = zg - z0 + 8):
// the backward window wA[q] = ring row r0 - 8 + q, the forward window wB[q] =
// ring row r0 - 7 + q; row zg + i reads wA[i..i+15] / wB[i..i+15].  Entries 0..14
// carry over from the previous group; 15..22 are loaded at the group's start.
template <int NF>
__device__ __forceinline__ void win_fill(const MarchSmem<NF> &S, int fa, int fb, int r0, int rc, float (&wA)[WIN],
                                         float (&wB)[WIN])
{
    const int ra = (r0 + 7) & (RING_ROWS - 1), rb = (r0 + 8) & (RING_ROWS - 1);
    wA[15] = S.ring[fa][ra][rc];
#pragma unroll
    for (int q = 0; q < MCH - 1; q++) wA[16 + q] = S.ring[fa][rb + q][rc];
#pragma unroll
    for (int q = 0; q < MCH; q++) wB[15 + q] = S.ring[fb][rb + q][rc];
}
__device__ __forceinline__ void win_shift(float (&wA)[WIN], float (&wB)[WIN], int by)
{
#pragma unroll
    for (int q = 0; q < 15; q++) { wA[q] = wA[q + by]; wB[q] = wB[q + by]; }
}
__device__ __forceinline__ void win_shift1(float (&wA)[WIN], float (&wB)[WIN])
{
#pragma unroll
    for (int q = 0; q < WIN - 1; q++) { wA[q] = wA[q + 1]; wB[q] = wB[q + 1]; }
}
// 16 consecutive window rows from offset i
template <int I>
__device__ __forceinline__ float dz_at(const float (&w)[WIN], const float *c)
{
    float acc = 0.f;
#pragma unroll
    for (int q = 0; q < 16; q++) acc = fmaf(w[I + q], q < 8 ? -c[7 - q] : c[q - 8], acc);
    return acc;
}
template <int I>
__device__ __forceinline__ float sk_at(const float (&w)[WIN], int K, const float *c)
{
    float acc = (w[I + 8] - w[I + 7]) * c[0];
#pragma unroll
    for (int k = 1; k < NCOEF; k++)
        if (k < K) acc = fmaf(w[I + 8 + k] - w[I + 7 - k], c[k], acc);
    return K == 0 ? 0.f : acc;
}

// ------------------------------------------------------------------ velocity rows
// Vx += dt*Rx*(Dx+Sxx [x psi0, staggered tables] + Dz-Sxz [z psi0]);
// Vz += dt*Rz*(Dx-Sxz [x psi1] + Dz+Szz [z psi1, staggered])   (lib/waves.cpp:1416-1566)
// Ring fields: [0] Sxx, [1] Sxz (backward window), [2] Szz (forward window).
struct VelPts {
    float vx, vz, rx, rz;
};
struct VelCtx {
    const Shot2D<float> *sh;
    float *Vx, *Vz;
    const float *Rx, *Rz;
    int pitch, nzp, nxp, L, order;
};

// Row zg + I of a group; rr = its ring row (masked).  GEN: C-PML strips and
// reduced-order stencils.
template <bool GEN, int I>
__device__ __forceinline__ void vel_row(const March2DArgs &a, const VelCtx &c, const MarchSmem<3> &S, const Lane &n,
                                        int z, int rr, bool more, const float (&wA)[WIN], const float (&wB)[WIN],
                                        VelPts &cur)
{
    const int o = z * c.pitch + n.cx;
    VelPts nxt = cur;
    if (more) {   // next row's point-wise inputs, in flight during this row
        const int o1 = o + c.pitch;
        nxt = {c.Vx[o1], c.Vz[o1], __ldg(c.Rx + o1), __ldg(c.Rz + o1)};
    }
    int zi = -1, zbt = 0, zr = 0, px = 0, pz = 0;
    float mx0 = 0.f, mx1 = 0.f, mz0 = 0.f, mz1 = 0.f;
    if (GEN) {
        zi = n.in ? zstrip(z, c.nzp, c.L, zbt, zr) : -1;
        px = z * 2 * c.L + n.xc;
        pz = zr * c.nxp + n.cx;
        if (n.xi >= 0) { mx0 = c.sh->psix[0][px]; mx1 = c.sh->psix[1][px]; }
        if (zi >= 0) { mz0 = c.sh->psiz[0][pz]; mz1 = c.sh->psiz[1][pz]; }
    }
    const float *rxx = &S.ring[0][rr][n.rc], *rxz = &S.ring[1][rr][n.rc];
    float d1 = dx_col<true>(rxx, a.cx);    // Dx+ Sxx
    float e1 = dx_col<false>(rxz, a.cx);   // Dx- Sxz
    float d2 = dz_at<I>(wA, a.cz);         // Dz- Sxz
    float e2 = dz_at<I>(wB, a.cz);         // Dz+ Szz
    if (GEN) {
        if (n.kf != c.order) d1 = sk_row<true>(rxx, n.kf, S.coef + n.kf * CROW);
        if (n.kb != c.order) e1 = sk_row<false>(rxz, n.kb, S.coef + n.kb * CROW);
        const int kzb = kbw(z, c.nzp, c.order), kzf = kfw(z, c.nzp, c.order);
        if (kzb != c.order) d2 = sk_at<I>(wA, kzb, S.coef + (9 + kzb) * CROW);
        if (kzf != c.order) e2 = sk_at<I>(wB, kzf, S.coef + (9 + kzf) * CROW);
    }
    c.Vx[o] = upd<GEN>(cur.vx, a.dt * cur.rx, d1, d2, n.xi, mx0, n.xb + 3, zi, mz0, zbt, a.pml, c.L);
    c.Vz[o] = upd<GEN>(cur.vz, a.dt * cur.rz, e1, e2, n.xi, mx1, n.xb, zi, mz1, zbt + 3, a.pml, c.L);
    if (GEN) {
        if (n.xi >= 0) { c.sh->psix[0][px] = mx0; c.sh->psix[1][px] = mx1; }
        if (zi >= 0) { c.sh->psiz[0][pz] = mz0; c.sh->psiz[1][pz] = mz1; }
    }
    cur = nxt;
}

// ------------------------------------------------------------------ stress rows
// Sxx += dt*L2M*Dx-Vx + dt*L*Dz-Vz, Szz += dt*L*Dx-Vx + dt*L2M*Dz-Vz (one x and one
// z memory variable for both, psi2); free surface: Szz = 0 on row lpml;
// Sxz += dt*M*(Dx+Vz [x psi3, staggered] + Dz+Vx [z psi3, staggered])
// (lib/waves.cpp:1571-1735).  Ring fields: [0] Vx (forward window), [1] Vz
// (backward window); both also x-differentiated.
struct StrPts {
    float sxx, szz, sxz, lm, l2m, mu;
};
struct StrCtx {
    const Shot2D<float> *sh;
    float *Sxx, *Szz, *Sxz;
    const float *Lm, *L2M, *Mu;
    int pitch, nzp, nxp, L, order, fsrow;
};

template <bool GEN, int I>
__device__ __forceinline__ void str_row(const March2DArgs &a, const StrCtx &c, const MarchSmem<2> &S, const Lane &n,
                                        int z, int rr, bool more, const float (&wA)[WIN], const float (&wB)[WIN],
                                        StrPts &cur)
{
    const int o = z * c.pitch + n.cx;
    StrPts nxt = cur;
    if (more) {
        const int o1 = o + c.pitch;
        nxt = {c.Sxx[o1], c.Szz[o1], c.Sxz[o1], __ldg(c.Lm + o1), __ldg(c.L2M + o1), __ldg(c.Mu + o1)};
    }
    int zi = -1, zbt = 0, zr = 0, px = 0, pz = 0;
    float mx2 = 0.f, mx3 = 0.f, mz2 = 0.f, mz3 = 0.f;
    if (GEN) {
        zi = n.in ? zstrip(z, c.nzp, c.L, zbt, zr) : -1;
        px = z * 2 * c.L + n.xc;
        pz = zr * c.nxp + n.cx;
        if (n.xi >= 0) { mx2 = c.sh->psix[2][px]; mx3 = c.sh->psix[3][px]; }
        if (zi >= 0) { mz2 = c.sh->psiz[2][pz]; mz3 = c.sh->psiz[3][pz]; }
    }
    const float *rvx = &S.ring[0][rr][n.rc], *rvz = &S.ring[1][rr][n.rc];
    float d1 = dx_col<false>(rvx, a.cx);   // Dx- Vx
    float e1 = dx_col<true>(rvz, a.cx);    // Dx+ Vz
    float d2 = dz_at<I>(wA, a.cz);         // Dz- Vz
    float e2 = dz_at<I>(wB, a.cz);         // Dz+ Vx
    if (GEN) {
        if (n.kb != c.order) d1 = sk_row<false>(rvx, n.kb, S.coef + n.kb * CROW);
        if (n.kf != c.order) e1 = sk_row<true>(rvz, n.kf, S.coef + n.kf * CROW);
        const int kzb = kbw(z, c.nzp, c.order), kzf = kfw(z, c.nzp, c.order);
        if (kzb != c.order) d2 = sk_at<I>(wA, kzb, S.coef + (9 + kzb) * CROW);
        if (kzf != c.order) e2 = sk_at<I>(wB, kzf, S.coef + (9 + kzf) * CROW);
    }
    // normal stresses (update_normal, forward): one x and one z memory for both
    const float a2 = a.dt * cur.l2m, a1 = a.dt * cur.lm;
    float xx = fmaf(a2, d1, cur.sxx);
    float zz = fmaf(a1, d1, cur.szz);
    if (GEN && n.xi >= 0) {
        const float *tb = a.pml + n.xb * c.L + n.xi;
        const float tA = __ldg(tb + PT_A * c.L), tB = __ldg(tb + PT_B * c.L), tC = __ldg(tb + PT_C * c.L);
        mx2 = fmaf(tA, d1, tB * mx2);
        const float cq = fmaf(tC, d1, mx2);
        xx = fmaf(-a2, cq, xx);
        zz = fmaf(-a1, cq, zz);
    }
    xx = fmaf(a1, d2, xx);
    zz = fmaf(a2, d2, zz);
    if (GEN && zi >= 0) {
        const float *tb = a.pml + zbt * c.L + zi;
        const float tA = __ldg(tb + PT_A * c.L), tB = __ldg(tb + PT_B * c.L), tC = __ldg(tb + PT_C * c.L);
        mz2 = fmaf(tA, d2, tB * mz2);
        const float cq = fmaf(tC, d2, mz2);
        xx = fmaf(-a1, cq, xx);
        zz = fmaf(-a2, cq, zz);
    }
    if (GEN && z == c.fsrow) zz = 0.f;
    c.Sxx[o] = xx;
    c.Szz[o] = zz;
    c.Sxz[o] = upd<GEN>(cur.sxz, a.dt * cur.mu, e1, e2, n.xi, mx3, n.xb + 3, zi, mz3, zbt + 3, a.pml, c.L);
    if (GEN) {
        if (n.xi >= 0) { c.sh->psix[2][px] = mx2; c.sh->psix[3][px] = mx3; }
        if (zi >= 0) { c.sh->psiz[2][pz] = mz2; c.sh->psiz[3][pz] = mz3; }
    }
    cur = nxt;
}

// Kernel prologue shared by both half-steps: barriers, the first ring chunks and
// the coefficient table.
template <int NF>
__device__ __forceinline__ Ring<NF> march_begin(const March2DArgs &a, MarchSmem<NF> &S, const MarchItem &it,
                                                const int (&fields)[NF])
{
    const CUtensorMap *M = reinterpret_cast<const CUtensorMap *>(a.maps) + (size_t)it.shot * NMAP2D;
    Ring<NF> R;
    R.S = &S;
#pragma unroll
    for (int f = 0; f < NF; f++) R.m[f] = M + fields[f];
    R.x0 = it.x0;
    R.z0 = it.z0;
    R.nch = (it.z1 - it.z0 + 15) / MCH + 1;
    if (threadIdx.x == 0) {
        for (int s = 0; s < MNS; s++) mbar_init(&S.bar[s], 1);
        for (int c = 0; c < MNS && c < R.nch; c++) R.issue(c);
    }
    for (int k = threadIdx.x; k < 2 * 9 * CROW; k += MNT) S.coef[k] = a.coefs[k];
    __syncthreads();   // barriers initialised, coefficients in place
    return R;
}

// Start of row group g (rows z0 + 8g ..): chunk g+2 has arrived and every thread
// is done with chunk g (group g reads chunks g+1 and g+2), whose slot then
// receives chunk g+4.
template <int NF, int NP>
__device__ __forceinline__ bool group_begin(const March2DArgs &a, const Ring<NF> &R, int g, const float *const *pf,
                                            int pitch, int z1)
{
    if (!__syncthreads_and(R.wait(g + 2, a.err))) return false;
    if (threadIdx.x == 0 && g + MNS < R.nch) R.issue(g + MNS);
    prefetch_rows<NP>(pf, pitch, R.x0, R.z0 + MCH * (g + 2), z1);
    return true;
}

}  // namespace

__global__ void __launch_bounds__(MNT, MINB_MARCH) e2d_march_velocity(const March2DArgs a)
{
    extern __shared__ __align__(128) unsigned char smraw[];
    MarchSmem<3> &S = *reinterpret_cast<MarchSmem<3> *>(smraw);
    const MarchItem it = a.items[blockIdx.x];
    const Shot2D<float> &sh = a.shots[it.shot];
    const Ring<3> R = march_begin<3>(a, S, it, {E2_SXX, E2_SXZ, E2_SZZ});
    const VelCtx c{&sh, sh.f[E2_VX], sh.f[E2_VZ], sh.m[M_RX], sh.m[M_RZ], sh.pitch, sh.nzp, sh.nxp, a.lpml, a.order};
    const Lane n = make_lane(it, sh, c.L, c.order);
    const int z0 = it.z0, z1 = it.z1;
    const float *pf[4] = {c.Vx, c.Vz, c.Rx, c.Rz};
    prefetch_rows<4>(pf, c.pitch, it.x0, z0, z1);
    prefetch_rows<4>(pf, c.pitch, it.x0, z0 + MCH, z1);
    const int o0 = z0 * c.pitch + n.cx;
    VelPts cur{c.Vx[o0], c.Vz[o0], __ldg(c.Rx + o0), __ldg(c.Rz + o0)};
    if (!__syncthreads_and(R.wait(0, a.err) && R.wait(1, a.err))) return;
    // windows before the first group: Sxz ring rows 0..14, Szz ring rows 1..15
    float wA[WIN], wB[WIN];
#pragma unroll
    for (int q = 0; q < 15; q++) { wA[q] = S.ring[1][q][n.rc]; wB[q] = S.ring[2][q + 1][n.rc]; }
    int zlo, zhi;
    plain_rows(c.nzp, c.L, c.order, zlo, zhi);
    const bool xplain = !(it.flags & MARCH_XGEN);
    for (int g = 0;; g++) {
        const int zg = z0 + MCH * g;
        if (zg >= z1) break;
        if (!group_begin<3, 4>(a, R, g, pf, c.pitch, z1)) return;
        const int r0 = (zg - z0 + 8) & (RING_ROWS - 1);
        win_fill<3>(S, 1, 2, zg - z0 + 8, n.rc, wA, wB);
        if (xplain && zg >= zlo && zg + MCH <= min(zhi, z1)) {
            const bool more = zg + MCH < z1;
            vel_row<false, 0>(a, c, S, n, zg + 0, r0 + 0, true, wA, wB, cur);
            vel_row<false, 1>(a, c, S, n, zg + 1, r0 + 1, true, wA, wB, cur);
            vel_row<false, 2>(a, c, S, n, zg + 2, r0 + 2, true, wA, wB, cur);
            vel_row<false, 3>(a, c, S, n, zg + 3, r0 + 3, true, wA, wB, cur);
            vel_row<false, 4>(a, c, S, n, zg + 4, r0 + 4, true, wA, wB, cur);
            vel_row<false, 5>(a, c, S, n, zg + 5, r0 + 5, true, wA, wB, cur);
            vel_row<false, 6>(a, c, S, n, zg + 6, r0 + 6, true, wA, wB, cur);
            vel_row<false, 7>(a, c, S, n, zg + 7, r0 + 7, more, wA, wB, cur);
            win_shift(wA, wB, MCH);
        } else {
            const int ze = min(zg + MCH, z1);
#pragma unroll 1
            for (int z = zg; z < zg + MCH; z++) {
                if (z < ze) vel_row<true, 0>(a, c, S, n, z, r0 + z - zg, z + 1 < z1, wA, wB, cur);
                win_shift1(wA, wB);
            }
        }
    }
    // every chunk issued has been waited for: the last group waits for chunk nch-1
}

__global__ void __launch_bounds__(MNT, MINB_MARCH) e2d_march_stress(const March2DArgs a)
{
    extern __shared__ __align__(128) unsigned char smraw[];
    MarchSmem<2> &S = *reinterpret_cast<MarchSmem<2> *>(smraw);
    const MarchItem it = a.items[blockIdx.x];
    const Shot2D<float> &sh = a.shots[it.shot];
    const Ring<2> R = march_begin<2>(a, S, it, {E2_VX, E2_VZ});
    const StrCtx c{&sh, sh.f[E2_SXX], sh.f[E2_SZZ], sh.f[E2_SXZ], sh.m[M_L], sh.m[M_L2M], sh.m[M_M],
                   sh.pitch, sh.nzp, sh.nxp, a.lpml, a.order, sh.fs ? a.lpml : -1};
    const Lane n = make_lane(it, sh, c.L, c.order);
    const int z0 = it.z0, z1 = it.z1;
    const float *pf[6] = {c.Sxx, c.Szz, c.Sxz, c.Lm, c.L2M, c.Mu};
    prefetch_rows<6>(pf, c.pitch, it.x0, z0, z1);
    prefetch_rows<6>(pf, c.pitch, it.x0, z0 + MCH, z1);
    const int o0 = z0 * c.pitch + n.cx;
    StrPts cur{c.Sxx[o0], c.Szz[o0], c.Sxz[o0], __ldg(c.Lm + o0), __ldg(c.L2M + o0), __ldg(c.Mu + o0)};
    if (!__syncthreads_and(R.wait(0, a.err) && R.wait(1, a.err))) return;
    // windows before the first group: Vz ring rows 0..14, Vx ring rows 1..15
    float wA[WIN], wB[WIN];
#pragma unroll
    for (int q = 0; q < 15; q++) { wA[q] = S.ring[1][q][n.rc]; wB[q] = S.ring[0][q + 1][n.rc]; }
    int zlo, zhi;
    plain_rows(c.nzp, c.L, c.order, zlo, zhi);
    const bool xplain = !(it.flags & MARCH_XGEN);
    for (int g = 0;; g++) {
        const int zg = z0 + MCH * g;
        if (zg >= z1) break;
        if (!group_begin<2, 6>(a, R, g, pf, c.pitch, z1)) return;
        const int r0 = (zg - z0 + 8) & (RING_ROWS - 1);
        win_fill<2>(S, 1, 0, zg - z0 + 8, n.rc, wA, wB);
        if (xplain && zg >= zlo && zg + MCH <= min(zhi, z1) && (c.fsrow < zg || c.fsrow >= zg + MCH)) {
            const bool more = zg + MCH < z1;
            str_row<false, 0>(a, c, S, n, zg + 0, r0 + 0, true, wA, wB, cur);
            str_row<false, 1>(a, c, S, n, zg + 1, r0 + 1, true, wA, wB, cur);
            str_row<false, 2>(a, c, S, n, zg + 2, r0 + 2, true, wA, wB, cur);
            str_row<false, 3>(a, c, S, n, zg + 3, r0 + 3, true, wA, wB, cur);
            str_row<false, 4>(a, c, S, n, zg + 4, r0 + 4, true, wA, wB, cur);
            str_row<false, 5>(a, c, S, n, zg + 5, r0 + 5, true, wA, wB, cur);
            str_row<false, 6>(a, c, S, n, zg + 6, r0 + 6, true, wA, wB, cur);
            str_row<false, 7>(a, c, S, n, zg + 7, r0 + 7, more, wA, wB, cur);
            win_shift(wA, wB, MCH);
        } else {
            const int ze = min(zg + MCH, z1);
#pragma unroll 1
            for (int z = zg; z < zg + MCH; z++) {
                if (z < ze) str_row<true, 0>(a, c, S, n, z, r0 + z - zg, z + 1 < z1, wA, wB, cur);
                win_shift1(wA, wB);
            }
        }
    }
}

// ------------------------------------------------------------------ host side
int march_smem_bytes() { return (int)march_smem(3); }

int march_resident_ctas()
{
    int nv = 0, ns = 0;
    if (cudaFuncSetAttribute(e2d_march_velocity, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)march_smem(3)) != cudaSuccess ||
        cudaFuncSetAttribute(e2d_march_stress, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)march_smem(2)) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nv, e2d_march_velocity, MNT, march_smem(3)) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&ns, e2d_march_stress, MNT, march_smem(2)) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return nv < ns ? nv : ns;
}

cudaError_t launch_march_2d(int half, const March2DArgs &a, int nitems, cudaStream_t st)
{
    // set once per process (thread-safe static initialisation)
    static const cudaError_t attr = [] {
        cudaError_t e = cudaFuncSetAttribute(e2d_march_velocity, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)march_smem(3));
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(e2d_march_stress, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)march_smem(2));
        return e;
    }();
    if (attr != cudaSuccess) return attr;
    if (half == 0) e2d_march_velocity<<<nitems, MNT, march_smem(3), st>>>(a);
    else e2d_march_stress<<<nitems, MNT, march_smem(2), st>>>(a);
    return cudaGetLastError();
}

}  // namespace rsgpu
