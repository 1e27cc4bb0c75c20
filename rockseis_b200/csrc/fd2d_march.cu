// Column-marching elastic 2D half-steps (FAST arithmetic, forward propagation;
// rsgpu_config.launch_mode 4).
//
// The per-tile kernels (fd2d_kernels.cuh) re-read a 16-row halo for every 32-row
// tile and spend a third of their instructions on addressing and register moves;
// these kernels march instead.  A CTA of MW warps owns a strip of MSTRIP columns
// of one shot and a band of rows [z0, z1) and walks down the band one row at a
// time.  Every thread holds one column:
//   - the two fields that are z-differentiated live in 16-row register windows
//     (one new row enters each window per step), and the z-derivatives are FMA
//     sums over the window in row order with -c / +c terms: the summation order
//     of the per-tile FAST kernels (dz_stream_f32), so both give bit-identical
//     wavefields;
//   - the fields that are x-differentiated arrive by TMA in a ring of MNS slots
//     of MCH rows, MSTRIP + 16 columns wide (the x halo), filled two chunks
//     ahead; x-derivatives are scalar FMAs in the per-tile kernels' tap order;
//   - point-wise inputs (the updated fields, densities and moduli) are read
//     from global memory; their rows two chunks ahead are prefetched into L2 by
//     bulk prefetches issued beside the ring's TMA loads.
// Reduced-order stencils near the array ends (lib/der.cpp's rule) replace the
// full-order result per point, read straight from the wavefields in global
// memory, and the C-PML memory updates follow the per-tile kernels operation by
// operation (lib/waves.cpp:1416-1735).
#include "fd2d_kernels.cuh"

namespace rsgpu {

namespace {

constexpr int MW = 4;                    // warps per CTA
constexpr int MNT = 32 * MW;             // threads per CTA
constexpr int MRW = MSTRIP2D + 2 * GUARD;  // ring row: the strip plus the x halo
constexpr int MCH = 8;                   // rows per TMA chunk
constexpr int MNS = 3;                   // ring slots
constexpr int MNF = 2;                   // ring fields of a half-step
constexpr int MINB_MARCH = 4;            // resident CTAs per SM requested from the allocator
static_assert(MSTRIP2D == 32 * MW, "one column per thread");

struct MarchSmem {
    float ring[MNS][MNF][MCH][MRW];
    uint64_t bar[MNS];
};
constexpr size_t MARCH_SMEM = sizeof(MarchSmem) + 128;   // + alignment slack
constexpr uint32_t CHUNK_BYTES = (uint32_t)(MNF * MCH * MRW * sizeof(float));


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

// z-derivative from a 16-row window w (forward: rows z-7..z+8; backward: rows
// z-8..z+7): sum in row order of cz[q] * w[q], cz[q] = -c[7-q] (q < 8), +c[q-8]
// (q >= 8), starting from zero.
__device__ __forceinline__ float dz_win(const float (&w)[16], const float *c)
{
    float acc = 0.f;
#pragma unroll
    for (int q = 0; q < 16; q++) acc = fmaf(w[q], q < 8 ? -c[7 - q] : c[q - 8], acc);
    return acc;
}

// Reduced-order stencil of K pairs at one point (stencil_k's arithmetic, FAST),
// inlined so that the rare edge points cost no call around the live windows.
__device__ __forceinline__ float sk(const float *center, int stride, int K, const float *c, bool fw)
{
    if (K == 0) return 0.f;
    float acc = (fw ? center[stride] - center[0] : center[0] - center[-stride]) * c[0];
#pragma unroll 1
    for (int k = 1; k < K; k++) {
        const float dl = fw ? center[(k + 1) * stride] - center[-k * stride] : center[k * stride] - center[-(k + 1) * stride];
        acc = fmaf(dl, c[k], acc);
    }
    return acc;
}

// F += am*d1 [x memory] ; F += am*d2 [z memory]  (update_field, FAST)
__device__ __forceinline__ float upd(float F, float am, float d1, float d2, int xi, float *px, int xtab, int zi,
                                     float *pz, int ztab, const float *pml, int L)
{
    F = fmaf(am, d1, F);
    if (xi >= 0) F = pml_correct<float, MODE_FAST>(F, am, d1, px, pml, L, xtab, xi);
    F = fmaf(am, d2, F);
    if (zi >= 0) F = pml_correct<float, MODE_FAST>(F, am, d2, pz, pml, L, ztab, zi);
    return F;
}

// Per-thread geometry shared by both half-steps.
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
    const int cl = threadIdx.x;
    n.cx = it.x0 + cl;
    n.rc = GUARD + cl;
    n.xi = xstrip(n.cx, sh.nxp, L, n.xb, n.xc);
    n.kf = kfw(n.cx, sh.nxp, order);
    n.kb = kbw(n.cx, sh.nxp, order);
    n.in = n.cx < sh.nxp;
    return n;
}

// Ring control: chunk c holds field rows z0 - 8 + MCH*c .. +MCH-1 of both ring
// fields in slot c % MNS; the n-th use of a slot waits on parity n & 1.
struct Ring {
    MarchSmem *S;
    const CUtensorMap *m0, *m1;
    int x0, z0, nch;
    __device__ __forceinline__ void issue(int c) const
    {
        const int s = c % MNS;
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        mbar_expect_tx(&S->bar[s], CHUNK_BYTES);
        // allocation row of field row z0 - 8 + MCH*c is z0 + MCH*c; allocation column x0
        // is field column x0 - 8 (x0 is a multiple of the strip: 16-byte aligned)
        tma_load_2d(&S->ring[s][0][0][0], m0, &S->bar[s], x0, z0 + MCH * c);
        tma_load_2d(&S->ring[s][1][0][0], m1, &S->bar[s], x0, z0 + MCH * c);
    }
    __device__ __forceinline__ bool wait(int c, int *err) const
    {
        return mbar_wait_bounded(&S->bar[c % MNS], (uint32_t)((c / MNS) & 1), err);
    }
};

// Ring row r (r = z - z0 + 8) of field f, given the slots of chunks g+1 (s1) and
// g+2 (s2) for the group g whose rows are r = 8(g+1) + i.
__device__ __forceinline__ const float *ring_row(const MarchSmem *S, int s1, int s2, int f, int rr)
{
    return rr < MCH ? &S->ring[s1][f][rr][0] : &S->ring[s2][f][rr - MCH][0];
}

// Rows of the point-wise fields prefetched into L2 for group g (8 rows from z0 + 8g).
template <int NP>
__device__ __forceinline__ void prefetch_rows(const float *const (&pf)[NP], int pitch, int x0, int zrow, int nzp)
{
    const int t = threadIdx.x;
    if (t < NP * MCH) {
        const int f = t / MCH, z = zrow + t % MCH;
        if (z >= 0 && z < nzp) prefetch_l2(pf[f] + (long)z * pitch + x0, MSTRIP2D * sizeof(float));
    }
}

}  // namespace

// ------------------------------------------------------------------ velocity half-step
// Vx += dt*Rx*(Dx+Sxx [x psi0, staggered tables] + Dz-Sxz [z psi0]);
// Vz += dt*Rz*(Dx-Sxz [x psi1] + Dz+Szz [z psi1, staggered])   (lib/waves.cpp:1416-1566)
// Ring fields: [0] Sxx, [1] Sxz (also the backward window's leading row);
// the forward window (Szz) is refilled from global memory one row ahead.
__global__ void __launch_bounds__(MNT, MINB_MARCH) e2d_march_velocity(const March2DArgs a)
{
    extern __shared__ unsigned char smraw[];
    MarchSmem *S = reinterpret_cast<MarchSmem *>((reinterpret_cast<uintptr_t>(smraw) + 127) & ~uintptr_t(127));
    const MarchItem it = a.items[blockIdx.x];
    const Shot2D<float> &sh = a.shots[it.shot];
    const int L = a.lpml, order = a.order, pitch = sh.pitch, nzp = sh.nzp, nxp = sh.nxp;
    const int z0 = it.z0, z1 = it.z1;
    const CUtensorMap *M = reinterpret_cast<const CUtensorMap *>(a.maps) + (size_t)it.shot * NMAP2D;
    const Ring R{S, M + E2_SXX, M + E2_SXZ, it.x0, z0, (z1 - z0 + 15) / MCH + 1};
    if (threadIdx.x == 0) {
        for (int s = 0; s < MNS; s++) mbar_init(&S->bar[s], 1);
        for (int c = 0; c < MNS && c < R.nch; c++) R.issue(c);
    }
    const Lane n = make_lane(it, sh, L, order);
    const float *Sxx = sh.f[E2_SXX], *Sxz = sh.f[E2_SXZ], *Szz = sh.f[E2_SZZ];
    float *Vx = sh.f[E2_VX], *Vz = sh.f[E2_VZ];
    const float *Rx = sh.m[M_RX], *Rz = sh.m[M_RZ];
    const float *pf[5] = {Vx, Vz, Rx, Rz, Szz};
    prefetch_rows<5>(pf, pitch, it.x0, z0, nzp);
    prefetch_rows<5>(pf, pitch, it.x0, z0 + MCH, nzp);
    // forward window (Szz rows z-8..z+7 before the step at z) and its next row
    float wB[16];
#pragma unroll
    for (int q = 0; q < 16; q++) wB[q] = Szz[(z0 - 8 + q) * pitch + n.cx];
    float nB = Szz[(z0 + 8) * pitch + n.cx];
    __syncthreads();   // barriers initialised
    if (!__syncthreads_and(R.wait(0, a.err) && R.wait(1, a.err))) return;
    // backward window (Sxz rows z-9..z+6 before the step at z): ring rows 0..14
    float wA[16];
    wA[0] = 0.f;
#pragma unroll
    for (int q = 1; q < 16; q++) wA[q] = ring_row(S, 0, 1, 1, q - 1)[n.rc];
    int s1 = 1, s2 = 2;
    for (int zb = z0; zb < z1; zb += 16) {
#pragma unroll
        for (int u = 0; u < 16; u++) {
            const int z = zb + u;
            if (z >= z1) break;
            const int i = u & 7;
            if (i == 0) {
                const int g = (z - z0) >> 3;
                if (!__syncthreads_and(g + 2 >= R.nch || R.wait(g + 2, a.err))) return;
                if (threadIdx.x == 0 && g + 3 < R.nch) R.issue(g + 3);
                prefetch_rows<5>(pf, pitch, it.x0, z0 + MCH * (g + 2), nzp);
                s1 = (g + 1) % MNS;
                s2 = (g + 2) % MNS;
            }
            const int o = z * pitch + n.cx;
            const float vx = Vx[o], vz = Vz[o], rx = __ldg(Rx + o), rz = __ldg(Rz + o);
            // windows: Sxz gains row z+7 (ring row r+7), Szz row z+8
#pragma unroll
            for (int q = 0; q < 15; q++) { wA[q] = wA[q + 1]; wB[q] = wB[q + 1]; }
            wA[15] = ring_row(S, s1, s2, 1, i + 7)[n.rc];
            wB[15] = nB;
            if (z + 1 < z1) nB = Szz[o + 9 * pitch];
            float d1 = dx_col<true>(ring_row(S, s1, s2, 0, i) + n.rc, a.cx);    // Dx+ Sxx
            float e1 = dx_col<false>(ring_row(S, s1, s2, 1, i) + n.rc, a.cx);   // Dx- Sxz
            float d2 = dz_win(wA, a.cz);                                         // Dz- Sxz
            float e2 = dz_win(wB, a.cz);                                         // Dz+ Szz
            if (n.kf != order) d1 = sk(Sxx + o, 1, n.kf, a.coefs + n.kf * CROW, true);
            if (n.kb != order) e1 = sk(Sxz + o, 1, n.kb, a.coefs + n.kb * CROW, false);
            const int kzb = kbw(z, nzp, order), kzf = kfw(z, nzp, order);
            if (kzb != order) d2 = sk(Sxz + o, pitch, kzb, a.coefs + 9 * CROW + kzb * CROW, false);
            if (kzf != order) e2 = sk(Szz + o, pitch, kzf, a.coefs + 9 * CROW + kzf * CROW, true);
            int zbt = 0, zr = 0;
            const int zi = n.in ? zstrip(z, nzp, L, zbt, zr) : -1;
            const int px = z * 2 * L + n.xc, pz = zr * nxp + n.cx;
            Vx[o] = upd(vx, a.dt * rx, d1, d2, n.xi, sh.psix[0] + px, n.xb + 3, zi, sh.psiz[0] + pz, zbt, a.pml, L);
            Vz[o] = upd(vz, a.dt * rz, e1, e2, n.xi, sh.psix[1] + px, n.xb, zi, sh.psiz[1] + pz, zbt + 3, a.pml, L);
        }
    }
    // every chunk issued has been waited for: the last group waits for chunk nch-1
}

// ------------------------------------------------------------------ stress half-step
// Sxx += dt*L2M*Dx-Vx + dt*L*Dz-Vz, Szz += dt*L*Dx-Vx + dt*L2M*Dz-Vz (one x and one
// z memory variable for both, psi2); free surface: Szz = 0 on row lpml;
// Sxz += dt*M*(Dx+Vz [x psi3, staggered] + Dz+Vx [z psi3, staggered])
// (lib/waves.cpp:1571-1735).  Ring fields: [0] Vx (forward window), [1] Vz
// (backward window); both also x-differentiated.
__global__ void __launch_bounds__(MNT, MINB_MARCH) e2d_march_stress(const March2DArgs a)
{
    extern __shared__ unsigned char smraw[];
    MarchSmem *S = reinterpret_cast<MarchSmem *>((reinterpret_cast<uintptr_t>(smraw) + 127) & ~uintptr_t(127));
    const MarchItem it = a.items[blockIdx.x];
    const Shot2D<float> &sh = a.shots[it.shot];
    const int L = a.lpml, order = a.order, pitch = sh.pitch, nzp = sh.nzp, nxp = sh.nxp;
    const int z0 = it.z0, z1 = it.z1;
    const CUtensorMap *M = reinterpret_cast<const CUtensorMap *>(a.maps) + (size_t)it.shot * NMAP2D;
    const Ring R{S, M + E2_VX, M + E2_VZ, it.x0, z0, (z1 - z0 + 15) / MCH + 1};
    if (threadIdx.x == 0) {
        for (int s = 0; s < MNS; s++) mbar_init(&S->bar[s], 1);
        for (int c = 0; c < MNS && c < R.nch; c++) R.issue(c);
    }
    const Lane n = make_lane(it, sh, L, order);
    const float *Vx = sh.f[E2_VX], *Vz = sh.f[E2_VZ];
    float *Sxx = sh.f[E2_SXX], *Szz = sh.f[E2_SZZ], *Sxz = sh.f[E2_SXZ];
    const float *Lm = sh.m[M_L], *L2M = sh.m[M_L2M], *Mu = sh.m[M_M];
    const float *pf[6] = {Sxx, Szz, Sxz, Lm, L2M, Mu};
    prefetch_rows<6>(pf, pitch, it.x0, z0, nzp);
    prefetch_rows<6>(pf, pitch, it.x0, z0 + MCH, nzp);
    const int fsrow = sh.fs ? L : -1;
    __syncthreads();
    if (!__syncthreads_and(R.wait(0, a.err) && R.wait(1, a.err))) return;
    // backward window (Vz rows z-9..z+6 before the step at z): ring rows 0..14 of field 1;
    // forward window (Vx rows z-8..z+7): ring rows 0..15 of field 0
    float wA[16], wB[16];
    wA[0] = 0.f;
#pragma unroll
    for (int q = 1; q < 16; q++) wA[q] = ring_row(S, 0, 1, 1, q - 1)[n.rc];
#pragma unroll
    for (int q = 0; q < 16; q++) wB[q] = ring_row(S, 0, 1, 0, q)[n.rc];
    int s1 = 1, s2 = 2;
    for (int zb = z0; zb < z1; zb += 16) {
#pragma unroll
        for (int u = 0; u < 16; u++) {
            const int z = zb + u;
            if (z >= z1) break;
            const int i = u & 7;
            if (i == 0) {
                const int g = (z - z0) >> 3;
                if (!__syncthreads_and(g + 2 >= R.nch || R.wait(g + 2, a.err))) return;
                if (threadIdx.x == 0 && g + 3 < R.nch) R.issue(g + 3);
                prefetch_rows<6>(pf, pitch, it.x0, z0 + MCH * (g + 2), nzp);
                s1 = (g + 1) % MNS;
                s2 = (g + 2) % MNS;
            }
            const int o = z * pitch + n.cx;
            const float sxx = Sxx[o], szz = Szz[o], sxz = Sxz[o];
            const float lm = __ldg(Lm + o), l2m = __ldg(L2M + o), mu = __ldg(Mu + o);
#pragma unroll
            for (int q = 0; q < 15; q++) { wA[q] = wA[q + 1]; wB[q] = wB[q + 1]; }
            wA[15] = ring_row(S, s1, s2, 1, i + 7)[n.rc];   // Vz row z+7
            wB[15] = ring_row(S, s1, s2, 0, i + 8)[n.rc];   // Vx row z+8
            float d1 = dx_col<false>(ring_row(S, s1, s2, 0, i) + n.rc, a.cx);   // Dx- Vx
            float e1 = dx_col<true>(ring_row(S, s1, s2, 1, i) + n.rc, a.cx);    // Dx+ Vz
            float d2 = dz_win(wA, a.cz);                                         // Dz- Vz
            float e2 = dz_win(wB, a.cz);                                         // Dz+ Vx
            if (n.kb != order) d1 = sk(Vx + o, 1, n.kb, a.coefs + n.kb * CROW, false);
            if (n.kf != order) e1 = sk(Vz + o, 1, n.kf, a.coefs + n.kf * CROW, true);
            const int kzb = kbw(z, nzp, order), kzf = kfw(z, nzp, order);
            if (kzb != order) d2 = sk(Vz + o, pitch, kzb, a.coefs + 9 * CROW + kzb * CROW, false);
            if (kzf != order) e2 = sk(Vx + o, pitch, kzf, a.coefs + 9 * CROW + kzf * CROW, true);
            int zbt = 0, zr = 0;
            const int zi = n.in ? zstrip(z, nzp, L, zbt, zr) : -1;
            // normal stresses (update_normal, forward)
            const float a2 = a.dt * l2m, a1 = a.dt * lm;
            float xx = fmaf(a2, d1, sxx);
            float zz = fmaf(a1, d1, szz);
            if (n.xi >= 0) {
                float *ps = sh.psix[2] + z * 2 * L + n.xc;
                const float *tb = a.pml + n.xb * L + n.xi;
                const float tA = __ldg(tb + PT_A * L), tB = __ldg(tb + PT_B * L), tC = __ldg(tb + PT_C * L);
                const float p = fmaf(tA, d1, tB * *ps);
                *ps = p;
                const float cq = fmaf(tC, d1, p);
                xx = fmaf(-a2, cq, xx);
                zz = fmaf(-a1, cq, zz);
            }
            xx = fmaf(a1, d2, xx);
            zz = fmaf(a2, d2, zz);
            if (zi >= 0) {
                float *ps = sh.psiz[2] + zr * nxp + n.cx;
                const float *tb = a.pml + zbt * L + zi;
                const float tA = __ldg(tb + PT_A * L), tB = __ldg(tb + PT_B * L), tC = __ldg(tb + PT_C * L);
                const float p = fmaf(tA, d2, tB * *ps);
                *ps = p;
                const float cq = fmaf(tC, d2, p);
                xx = fmaf(-a1, cq, xx);
                zz = fmaf(-a2, cq, zz);
            }
            if (z == fsrow) zz = 0.f;
            Sxx[o] = xx;
            Szz[o] = zz;
            // shear stress
            Sxz[o] = upd(sxz, a.dt * mu, e1, e2, n.xi, sh.psix[3] + z * 2 * L + n.xc, n.xb + 3, zi,
                         sh.psiz[3] + zr * nxp + n.cx, zbt + 3, a.pml, L);
        }
    }
}

// ------------------------------------------------------------------ host side
int march_smem_bytes() { return (int)MARCH_SMEM; }

int march_resident_ctas()
{
    int nv = 0, ns = 0;
    if (cudaFuncSetAttribute(e2d_march_velocity, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)MARCH_SMEM) != cudaSuccess ||
        cudaFuncSetAttribute(e2d_march_stress, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)MARCH_SMEM) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nv, e2d_march_velocity, MNT, MARCH_SMEM) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&ns, e2d_march_stress, MNT, MARCH_SMEM) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return nv < ns ? nv : ns;
}

cudaError_t launch_march_2d(int half, const March2DArgs &a, int nitems, cudaStream_t st)
{
    static bool attr = false;
    if (!attr) {
        cudaError_t e = cudaFuncSetAttribute(e2d_march_velocity, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)MARCH_SMEM);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(e2d_march_stress, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)MARCH_SMEM);
        if (e != cudaSuccess) return e;
        attr = true;
    }
    if (half == 0) e2d_march_velocity<<<nitems, MNT, MARCH_SMEM, st>>>(a);
    else e2d_march_stress<<<nitems, MNT, MARCH_SMEM, st>>>(a);
    return cudaGetLastError();
}

}  // namespace rsgpu
