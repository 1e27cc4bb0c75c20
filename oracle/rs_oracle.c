/*
 * rs_oracle.c -- CPU restatement of the RockSeis finite-difference hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  The test-suite uses this file as the checker for
 * the CUDA library (rockseis_b200/librsgpu.so); the product never links or
 * calls it.  It is pinned against the unmodified reference (oracle/_ref,
 * built from the reference's own sources) by tests/test_oracle_pin.py and
 * against the committed fixtures in tests/golden/.
 *
 * Scope: one shot, float arithmetic in the reference's operation order (build
 * with -ffp-contract=off), inputs already preprocessed the way the reference's
 * Model/Pml/Geometry classes hold them:
 *   - padded staggered parameters (Rx, Rz, L [, L2M, M]) in a[iz*nxp + ix];
 *   - C-PML tables, 12 arrays of lpml: A,B,C ltf; A,B,C ltf_stag; A,B,C rbb; A,B,C rbb_stag;
 *   - trace maps (x,z) and shifts as produced by Geometry2D::makeMap;
 *   - traces d[it + itr*nt].
 * Reference functions restated (paths relative to the RockSeis tree):
 *   Der::ddx_fw/ddz_fw/ddx_bw/ddz_bw       lib/der.cpp:155-540
 *   WavesAcoustic2D::forwardstep*           lib/waves.cpp:217-404
 *   WavesAcoustic2D::insertSource/record    lib/waves.cpp:407-595
 *   WavesElastic2D::forwardstep*            lib/waves.cpp:1416-1735
 *   WavesElastic2D::backwardstep*           lib/waves.cpp:1738-2080
 *   WavesElastic2D::insertSource/record     lib/waves.cpp:2085-2288
 *   FwiAcoustic2D::crossCorr                lib/fwi.cpp:511-571
 *   FwiAcoustic2D::computeMisfit/Residuals  lib/fwi.cpp:574-1027 (DIFFERENCE)
 *   FwiAcoustic2D::run_optimal              lib/fwi.cpp:1159-1332 (all states kept in memory)
 *   RtmAcoustic2D::crossCorr/run_optimal    lib/rtm.cpp:191-219, 423-545
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* optimised staggered coefficients per half-length K (lib/der.cpp:3-53) */
static const double COEF[9][8] = {
    {0, 0, 0, 0, 0, 0, 0, 0},
    {(double)1.0029f, 0, 0, 0, 0, 0, 0, 0},
    {1.188401e+0, -7.046382e-2, 0, 0, 0, 0, 0, 0},
    {1.216624e+0, -9.197724e-2, 1.300041e-2, 0, 0, 0, 0, 0},
    {1.230862e+0, -1.034123e-1, 2.011671e-2, -3.245760e-3, 0, 0, 0, 0},
    {1.239407e+0, -1.105315e-1, 2.496329e-2, -5.804879e-3, 9.358680e-4, 0, 0, 0},
    {1.245095e+0, -1.153979e-1, 2.848442e-2, -7.899473e-3, 1.898222e-3, -2.935304e-4, 0, 0},
    {1.249150e+0, -1.189375e-1, 3.116091e-2, -9.623004e-3, 2.812069e-3, -6.655106e-4, 9.728191e-5, 0},
    {1.252186e+0, -1.216289e-1, 3.326513e-2, -1.105777e-2, 3.647865e-3, -1.066144e-3, 2.437491e-4, -3.351959e-5},
};

typedef struct {
    int nxp, nzp;      /* padded grid */
    int lpml, order, fs;
    float dx, dz, dt;
    int nt;
} orc_grid;

/* Coefficient pairs used at index i of an axis of length n: the reference's three
 * loops overwrite each other near the ends, the last writer defines the rule. */
static int k_fw(int i, int n, int order)
{
    if (i >= n - 1) return 0;
    if (i >= n - order - 1) return n - 1 - i;
    if (i >= order - 1) return order;
    return i + 1;
}
static int k_bw(int i, int n, int order)
{
    if (i >= n - order) return n - i;
    if (i >= order) return order;
    return i;
}

/* forward staggered derivative at linear index p along stride s; pos/n for the order rule */
static float d_fw(const float *f, long p, long s, int pos, int n, int order, float d)
{
    int K = k_fw(pos, n, order);
    if (K == 0) return 0.0f;
    float c[8];
    for (int k = 0; k < K; k++) c[k] = (float)COEF[K][k];
    float acc = (f[p + s] - f[p]) * c[0];
    for (int k = 1; k < K; k++) acc += (f[p + (k + 1) * s] - f[p - k * s]) * c[k];
    return acc / d;
}
static float d_bw(const float *f, long p, long s, int pos, int n, int order, float d)
{
    int K = k_bw(pos, n, order);
    if (K == 0) return 0.0f;
    float c[8];
    for (int k = 0; k < K; k++) c[k] = (float)COEF[K][k];
    float acc = (f[p] - f[p - s]) * c[0];
    for (int k = 1; k < K; k++) acc += (f[p + k * s] - f[p - (k + 1) * s]) * c[k];
    return acc / d;
}

/* whole-array derivatives (which: 0 x_fw, 2 z_fw, 3 x_bw, 5 z_bw), for Der parity tests */
void orc_der2d(int nxp, int nzp, int order, float dx, float dz, int which, const float *f, float *df)
{
    for (int iz = 0; iz < nzp; iz++)
        for (int ix = 0; ix < nxp; ix++) {
            long p = (long)iz * nxp + ix;
            switch (which) {
            case 0: df[p] = d_fw(f, p, 1, ix, nxp, order, dx); break;
            case 2: df[p] = d_fw(f, p, nxp, iz, nzp, order, dz); break;
            case 3: df[p] = d_bw(f, p, 1, ix, nxp, order, dx); break;
            default: df[p] = d_bw(f, p, nxp, iz, nzp, order, dz); break;
            }
        }
}

/* C-PML strip of a coordinate: returns table index (or -1) and sets table base (0 ltf, 6 rbb) */
static int strip(int i, int n, int L, int *base, int *slot)
{
    if (i < L) { *base = 0; *slot = i; return i; }
    if (i >= n - L) { *base = 6; *slot = L + (i - (n - L)); return i - (n - L); }
    return -1;
}

/* psi = B*psi + A*df ;  F -= a*(psi + C*df)   (lib/waves.cpp:252-253) */
static float cpml(float F, float a, float df, float *psi, const float *tab, int L, int base, int idx)
{
    *psi = tab[(base + 1) * L + idx] * (*psi) + tab[(base + 0) * L + idx] * df;
    return F - a * (*psi + tab[(base + 2) * L + idx] * df);
}

/* ------------------------------------------------------------------ wave state */
typedef struct {
    orc_grid g;
    int elastic;
    float *f[5];          /* A: P,Vx,Vz   E: Vx,Vz,Sxx,Szz,Sxz */
    float *psix[4];       /* [nzp][2L] */
    float *psiz[4];       /* [2L][nxp] */
} orc_state;

static void st_alloc(orc_state *s, const orc_grid *g, int elastic)
{
    s->g = *g;
    s->elastic = elastic;
    long n = (long)g->nxp * g->nzp;
    int nf = elastic ? 5 : 3, np = elastic ? 4 : 2;
    for (int k = 0; k < 5; k++) s->f[k] = k < nf ? calloc(n, sizeof(float)) : NULL;
    for (int k = 0; k < 4; k++) {
        s->psix[k] = k < np ? calloc((long)g->nzp * 2 * g->lpml, sizeof(float)) : NULL;
        s->psiz[k] = k < np ? calloc((long)g->nxp * 2 * g->lpml, sizeof(float)) : NULL;
    }
}
static void st_free(orc_state *s)
{
    for (int k = 0; k < 5; k++) free(s->f[k]);
    for (int k = 0; k < 4; k++) { free(s->psix[k]); free(s->psiz[k]); }
}
static long st_bytes_fields(const orc_state *s) { return (long)s->g.nxp * s->g.nzp * (s->elastic ? 5 : 3); }
static void st_copy_fields(float *dst, const orc_state *s)
{
    long n = (long)s->g.nxp * s->g.nzp;
    for (int k = 0; k < (s->elastic ? 5 : 3); k++) memcpy(dst + k * n, s->f[k], n * sizeof(float));
}

/* ------------------------------------------------------------------ acoustic 2D step */
static void a2d_step(orc_state *s, const float *Rx, const float *Rz, const float *Lm, const float *tab)
{
    const orc_grid *g = &s->g;
    const int nx = g->nxp, nz = g->nzp, L = g->lpml;
    float *P = s->f[0], *Vx = s->f[1], *Vz = s->f[2];
    int b, sl, t;
    for (int iz = 0; iz < nz; iz++)
        for (int ix = 0; ix < nx; ix++) {
            long p = (long)iz * nx + ix;
            float dfx = d_fw(P, p, 1, ix, nx, g->order, g->dx);
            float ax = g->dt * Rx[p];
            Vx[p] += ax * dfx;
            if ((t = strip(ix, nx, L, &b, &sl)) >= 0) Vx[p] = cpml(Vx[p], ax, dfx, &s->psix[0][(long)iz * 2 * L + sl], tab, L, b + 3, t);
            float dfz = d_fw(P, p, nx, iz, nz, g->order, g->dz);
            float az = g->dt * Rz[p];
            Vz[p] += az * dfz;
            if ((t = strip(iz, nz, L, &b, &sl)) >= 0) Vz[p] = cpml(Vz[p], az, dfz, &s->psiz[0][(long)sl * nx + ix], tab, L, b + 3, t);
        }
    for (int iz = 0; iz < nz; iz++)
        for (int ix = 0; ix < nx; ix++) {
            long p = (long)iz * nx + ix;
            float al = g->dt * Lm[p];
            float dfx = d_bw(Vx, p, 1, ix, nx, g->order, g->dx);
            P[p] += al * dfx;
            if ((t = strip(ix, nx, L, &b, &sl)) >= 0) P[p] = cpml(P[p], al, dfx, &s->psix[1][(long)iz * 2 * L + sl], tab, L, b, t);
            float dfz = d_bw(Vz, p, nx, iz, nz, g->order, g->dz);
            P[p] += al * dfz;
            if ((t = strip(iz, nz, L, &b, &sl)) >= 0) P[p] = cpml(P[p], al, dfz, &s->psiz[1][(long)sl * nx + ix], tab, L, b, t);
        }
}

/* ------------------------------------------------------------------ elastic 2D steps */
static void e2d_vel(orc_state *s, const float *Rx, const float *Rz, const float *Lm, const float *L2M,
                    const float *M, const float *tab, int adj)
{
    const orc_grid *g = &s->g;
    const int nx = g->nxp, nz = g->nzp, L = g->lpml;
    float *Vx = s->f[0], *Vz = s->f[1], *Sxx = s->f[2], *Szz = s->f[3], *Sxz = s->f[4];
    long n = (long)nx * nz;
    const float *w1 = Sxx, *w2 = Sxz, *w3 = Szz;
    float *b1 = NULL, *b2 = NULL, *b3 = NULL;
    if (adj) {
        /* adjoint work arrays (lib/waves.cpp:1774, 1812, 1885) */
        b1 = malloc(n * sizeof(float)); b2 = malloc(n * sizeof(float)); b3 = malloc(n * sizeof(float));
        for (long p = 0; p < n; p++) {
            b1[p] = L2M[p] * Sxx[p] + Lm[p] * Szz[p];
            b2[p] = M[p] * Sxz[p];
            b3[p] = Lm[p] * Sxx[p] + L2M[p] * Szz[p];
        }
        w1 = b1; w2 = b2; w3 = b3;
    }
    int b, sl, t;
    for (int iz = 0; iz < nz; iz++)
        for (int ix = 0; ix < nx; ix++) {
            long p = (long)iz * nx + ix;
            float a = g->dt * Rx[p];
            float d1 = d_fw(w1, p, 1, ix, nx, g->order, g->dx);
            Vx[p] += a * d1;
            if ((t = strip(ix, nx, L, &b, &sl)) >= 0) Vx[p] = cpml(Vx[p], a, d1, &s->psix[0][(long)iz * 2 * L + sl], tab, L, b + 3, t);
            float d2 = d_bw(w2, p, nx, iz, nz, g->order, g->dz);
            Vx[p] += a * d2;
            if ((t = strip(iz, nz, L, &b, &sl)) >= 0) Vx[p] = cpml(Vx[p], a, d2, &s->psiz[0][(long)sl * nx + ix], tab, L, b, t);
            a = g->dt * Rz[p];
            d1 = d_bw(w2, p, 1, ix, nx, g->order, g->dx);
            Vz[p] += a * d1;
            if ((t = strip(ix, nx, L, &b, &sl)) >= 0) Vz[p] = cpml(Vz[p], a, d1, &s->psix[1][(long)iz * 2 * L + sl], tab, L, b, t);
            d2 = d_fw(w3, p, nx, iz, nz, g->order, g->dz);
            Vz[p] += a * d2;
            if ((t = strip(iz, nz, L, &b, &sl)) >= 0) Vz[p] = cpml(Vz[p], a, d2, &s->psiz[1][(long)sl * nx + ix], tab, L, b + 3, t);
        }
    free(b1); free(b2); free(b3);
}

static void e2d_str(orc_state *s, const float *Lm, const float *L2M, const float *M, const float *tab, int adj)
{
    const orc_grid *g = &s->g;
    const int nx = g->nxp, nz = g->nzp, L = g->lpml;
    float *Vx = s->f[0], *Vz = s->f[1], *Sxx = s->f[2], *Szz = s->f[3], *Sxz = s->f[4];
    int b, sl, t;
    for (int iz = 0; iz < nz; iz++)
        for (int ix = 0; ix < nx; ix++) {
            long p = (long)iz * nx + ix;
            float d1 = d_bw(Vx, p, 1, ix, nx, g->order, g->dx);
            float d2 = d_bw(Vz, p, nx, iz, nz, g->order, g->dz);
            if (!adj) {
                float a2 = g->dt * L2M[p], a1 = g->dt * Lm[p];
                Sxx[p] += a2 * d1;
                Szz[p] += a1 * d1;
                if ((t = strip(ix, nx, L, &b, &sl)) >= 0) {
                    float *ps = &s->psix[2][(long)iz * 2 * L + sl];
                    *ps = tab[(b + 1) * L + t] * (*ps) + tab[b * L + t] * d1;
                    Sxx[p] -= a2 * (*ps + tab[(b + 2) * L + t] * d1);
                    Szz[p] -= a1 * (*ps + tab[(b + 2) * L + t] * d1);
                }
                Sxx[p] += a1 * d2;
                Szz[p] += a2 * d2;
                if ((t = strip(iz, nz, L, &b, &sl)) >= 0) {
                    float *ps = &s->psiz[2][(long)sl * nx + ix];
                    *ps = tab[(b + 1) * L + t] * (*ps) + tab[b * L + t] * d2;
                    Sxx[p] -= a1 * (*ps + tab[(b + 2) * L + t] * d2);
                    Szz[p] -= a2 * (*ps + tab[(b + 2) * L + t] * d2);
                }
            } else {
                Sxx[p] += g->dt * d1;
                if ((t = strip(ix, nx, L, &b, &sl)) >= 0) Sxx[p] = cpml(Sxx[p], g->dt, d1, &s->psix[2][(long)iz * 2 * L + sl], tab, L, b, t);
                Szz[p] += g->dt * d2;
                if ((t = strip(iz, nz, L, &b, &sl)) >= 0) Szz[p] = cpml(Szz[p], g->dt, d2, &s->psiz[2][(long)sl * nx + ix], tab, L, b, t);
            }
            if (g->fs && iz == L) Szz[p] = 0.0f;
            float a = adj ? g->dt : g->dt * M[p];
            d1 = d_fw(Vz, p, 1, ix, nx, g->order, g->dx);
            Sxz[p] += a * d1;
            if ((t = strip(ix, nx, L, &b, &sl)) >= 0) Sxz[p] = cpml(Sxz[p], a, d1, &s->psix[3][(long)iz * 2 * L + sl], tab, L, b + 3, t);
            d2 = d_fw(Vx, p, nx, iz, nz, g->order, g->dz);
            Sxz[p] += a * d2;
            if ((t = strip(iz, nz, L, &b, &sl)) >= 0) Sxz[p] = cpml(Sxz[p], a, d2, &s->psiz[3][(long)sl * nx + ix], tab, L, b + 3, t);
        }
}

/* ------------------------------------------------------------------ sources / receivers */
/* field codes (include/utils.h:22): 0 PRESSURE, 1 VX, 3 VZ */
static void inject(orc_state *s, const float *Mod, int field, int ntr, const int *map, const float *shift,
                   const float *wav, int it)
{
    const orc_grid *g = &s->g;
    const int nx = g->nxp, L = g->lpml;
    for (int i = 0; i < ntr; i++) {
        if (map[2 * i] < 0 || map[2 * i + 1] < 0) continue;
        float xt[2] = {1 - shift[2 * i], shift[2 * i]}, zt[2] = {1 - shift[2 * i + 1], shift[2 * i + 1]};
        for (int i1 = 0; i1 < 2; i1++)
            for (int i2 = 0; i2 < 2; i2++) {
                long p = (long)(L + map[2 * i + 1] + i1) * nx + (L + map[2 * i] + i2);
                float w = wav[it + (long)i * g->nt];
                if (!s->elastic) {
                    float *F = field == 0 ? s->f[0] : field == 1 ? s->f[1] : s->f[2];
                    F[p] += g->dt * Mod[p] * w * xt[i2] * zt[i1];
                } else if (field == 0) {
                    s->f[2][p] -= g->dt * w * xt[i2] * zt[i1];
                    s->f[3][p] -= g->dt * w * xt[i2] * zt[i1];
                } else {
                    float *F = field == 1 ? s->f[0] : s->f[1];
                    F[p] += g->dt * Mod[p] * w * xt[i2] * zt[i1];
                }
            }
    }
}

static void record(const orc_state *s, int field, int ntr, const int *map, const float *shift, const float *factor,
                   float *out, int it)
{
    const orc_grid *g = &s->g;
    const int nx = g->nxp, L = g->lpml;
    for (int i = 0; i < ntr; i++) {
        if (map[2 * i] < 0 || map[2 * i + 1] < 0) continue;
        float xt[2] = {1 - shift[2 * i], shift[2 * i]}, zt[2] = {1 - shift[2 * i + 1], shift[2 * i + 1]};
        float *o = &out[it + (long)i * g->nt];
        for (int i1 = 0; i1 < 2; i1++)
            for (int i2 = 0; i2 < 2; i2++) {
                long p = (long)(L + map[2 * i + 1] + i1) * nx + (L + map[2 * i] + i2);
                if (!s->elastic) {
                    const float *F = field == 0 ? s->f[0] : field == 1 ? s->f[1] : s->f[2];
                    *o += xt[i2] * zt[i1] * F[p];
                } else if (field == 0) {
                    float fac = factor ? factor[i] : 1.0f;
                    *o += (1. / 2.) * xt[i2] * zt[i1] * s->f[2][p] / fac;
                    *o += (1. / 2.) * xt[i2] * zt[i1] * s->f[3][p] / fac;
                } else {
                    const float *F = field == 1 ? s->f[0] : s->f[1];
                    *o += xt[i2] * zt[i1] * F[p];
                }
            }
    }
}

static const float *src_mod_a2d(int field, const float *Rx, const float *Rz, const float *Lm)
{
    return field == 0 ? Lm : field == 1 ? Rx : Rz;
}

/* ------------------------------------------------------------------ drivers */
/* ModellingAcoustic2D::run for one shot.  models: Rx, Rz, L.  nsteps <= nt steps
 * are run (nsteps < nt gives a bounded sample for CPU timing).  state_out, if
 * given, receives P,Vx,Vz after the last step. */
int orc_mod_a2d(const orc_grid *g, const float *Rx, const float *Rz, const float *Lm, const float *tab,
                int ns, const int *smap, const float *sshift, const float *wav, int sfield,
                int nr, const int *gmap, const float *gshift, int rfield, float *out, int nsteps, float *state_out)
{
    orc_state s;
    st_alloc(&s, g, 0);
    for (int it = 0; it < nsteps; it++) {
        a2d_step(&s, Rx, Rz, Lm, tab);
        inject(&s, src_mod_a2d(sfield, Rx, Rz, Lm), sfield, ns, smap, sshift, wav, it);
        record(&s, rfield, nr, gmap, gshift, NULL, out, it);
    }
    if (state_out) st_copy_fields(state_out, &s);
    st_free(&s);
    return 0;
}

/* ModellingElastic2D::run for one shot.  models: Rx, Rz, L, L2M, M. */
int orc_mod_e2d(const orc_grid *g, const float *Rx, const float *Rz, const float *Lm, const float *L2M,
                const float *M, const float *tab, int ns, const int *smap, const float *sshift, const float *wav,
                int sfield, int nr, const int *gmap, const float *gshift, int rfield, const float *factor, float *out,
                int nsteps, float *state_out)
{
    orc_state s;
    st_alloc(&s, g, 1);
    const float *smod = sfield == 1 ? Rx : Rz;
    for (int it = 0; it < nsteps; it++) {
        e2d_vel(&s, Rx, Rz, Lm, L2M, M, tab, 0);
        e2d_str(&s, Lm, L2M, M, tab, 0);
        inject(&s, smod, sfield, ns, smap, sshift, wav, it);
        record(&s, rfield, nr, gmap, gshift, factor, out, it);
    }
    if (state_out) st_copy_fields(state_out, &s);
    st_free(&s);
    return 0;
}

/* One adjoint (backward) elastic step from a given state, for step-level tests.
 * state: Vx,Vz,Sxx,Szz,Sxz in/out; C-PML memory starts at zero. */
int orc_e2d_adjoint_steps(const orc_grid *g, const float *Rx, const float *Rz, const float *Lm, const float *L2M,
                          const float *M, const float *tab, int nsteps, float *state)
{
    orc_state s;
    st_alloc(&s, g, 1);
    long n = (long)g->nxp * g->nzp;
    for (int k = 0; k < 5; k++) memcpy(s.f[k], state + k * n, n * sizeof(float));
    for (int it = 0; it < nsteps; it++) {
        e2d_vel(&s, Rx, Rz, Lm, L2M, M, tab, 1);
        e2d_str(&s, Lm, L2M, M, tab, 1);
    }
    st_copy_fields(state, &s);
    st_free(&s);
    return 0;
}

/* Forward pressure paired with the adjoint field at time index `it` by the
 * reference's Revolve-driven loops: at FIRSTURN (it = nt-1) the forward field has
 * just been stepped to it; at every YOUTURN the forward field was advanced only to
 * the state before step it (lib/fwi.cpp:1213-1217, 1281-1289; lib/rtm.cpp:459-524),
 * i.e. the state after step it-1, and the zero initial state for it = 0. */
static const float *fw_state_at(const float *Ps, const float *zero, long n, int nt, int it)
{
    if (it == nt - 1) return Ps + (size_t)it * n;
    if (it == 0) return zero;
    return Ps + (size_t)(it - 1) * n;
}

/* FwiAcoustic2D::crossCorr (lib/fwi.cpp:511-571), unpadded interior 1..n-2 */
static void a2d_corr(const orc_grid *g, int nx, int nz, const float *Vp, const float *Rho, const float *Rx,
                     const float *Rz, const float *wsp, const float *wrx, const float *wrz, float *vpgrad,
                     float *rhograd)
{
    const int L = g->lpml, nxp = g->nxp;
    const float dx = g->dx, dz = g->dz;
    for (int ix = 1; ix < nx - 1; ix++)
        for (int iz = 1; iz < nz - 1; iz++) {
            long q = (long)(iz + L) * nxp + (ix + L);
            float vpscale = -2.0 / (Vp[(long)iz * nx + ix]);
            float rhoscale1 = -1.0 / (Rho[(long)iz * nx + ix]);
            float mrxx = (wrx[q] - wrx[q - 1]) / dx;
            float mrzz = (wrz[q] - wrz[q - nxp]) / dz;
            vpgrad[(long)iz * nx + ix] -= vpscale * wsp[q] * (mrxx + mrzz);
            rhograd[(long)iz * nx + ix] -= rhoscale1 * wsp[q] * (mrxx + mrzz);
            float uderx = 0.5 * wrx[q] * Rx[q] * (wsp[q + 1] - wsp[q]) / dx;
            uderx += 0.5 * wrx[q - 1] * Rx[q - 1] * (wsp[q] - wsp[q - 1]) / dx;
            float uderz = 0.5 * wrz[q] * Rz[q] * (wsp[q + nxp] - wsp[q]) / dz;
            uderz += 0.5 * wrz[q - nxp] * Rz[q - nxp] * (wsp[q] - wsp[q - nxp]) / dz;
            rhograd[(long)iz * nx + ix] += (uderx + uderz);
        }
}

static int cmp_float(const void *a, const void *b)
{
    const float x = *(const float *)a, y = *(const float *)b;
    return (x > y) - (x < y);
}

/* CORRELATION misfit and residuals of one shot's pressure traces, shared by the 2D
 * and 3D drivers (FwiAcoustic2D: lib/fwi.cpp:617-645, 808-849; FwiAcoustic3D:
 * lib/fwi.cpp:1511-1540, 1696-1722).  Per trace in float: n1 = sqrt(sum m*m),
 * n2 = sqrt(sum o*o) (zero -> 1), n3 = sum m*o / (n1*n2); the misfit adds
 * -(m*o/(n1*n2)) over the traces on the grid; every trace's residual is
 * -(o/(n1*n2) - (m/(n1*n1))*n3).  With `clip` (2D only) the residuals at or above
 * the magnitude at index 97*nt*nr/100 of the ascending sort are set to zero. */
static int corr_misfit(int nr, int nt, const int *valid, const float *datamod, const float *obs, int clip,
                       float *datares, float *mis)
{
    for (int tr = 0; tr < nr; tr++) {
        const float *m = datamod + (long)tr * nt, *o = obs + (long)tr * nt;
        float n1 = 0.0f, n2 = 0.0f, n3 = 0.0f;
        for (int it = 0; it < nt; it++) {
            n1 += m[it] * m[it];
            n2 += o[it] * o[it];
            n3 += m[it] * o[it];
        }
        n1 = sqrtf(n1);
        n2 = sqrtf(n2);
        if (n1 == 0) n1 = 1.0f;
        if (n2 == 0) n2 = 1.0f;
        if (valid[tr])
            for (int it = 0; it < nt; it++) {
                float v = (float)((-1.0) * (m[it] * o[it] / (n1 * n2)));
                *mis += v;
            }
        n3 /= (n1 * n2);
        float *r = datares + (long)tr * nt;
        for (int it = 0; it < nt; it++) r[it] = (float)((-1.0) * 1 * ((o[it] / (n1 * n2)) - (m[it] / (n1 * n1)) * n3));
    }
    if (!clip) return 0;
    const long tot = (long)nt * nr;
    float *fres = malloc(tot * sizeof(float));
    if (!fres) return -1;
    for (long k = 0; k < tot; k++) fres[k] = fabsf(datares[k]);
    qsort(fres, tot, sizeof(float), cmp_float);
    const float pclip = fres[(long)((97ul * (unsigned long)nt * (unsigned long)nr) / 100ul)];
    for (long k = 0; k < tot; k++)
        if (fabsf(datares[k]) >= pclip) datares[k] = 0.0f;
    free(fres);
    return 0;
}

/* FwiAcoustic2D::run_optimal with the DIFFERENCE (misfit_type 0) or CORRELATION (1) misfit and pressure data, one shot.
 * The forward states are kept for every step instead of being recomputed from
 * checkpoints; recomputation is deterministic, so the gradient is the same.
 * The pairing of forward and adjoint time levels follows fw_state_at().
 * vp, rho: unpadded models [nz][nx]; outputs accumulate (+=) like the reference. */
int orc_fwi_a2d(const orc_grid *g, int nx, int nz, const float *vp, const float *rho, const float *Rx,
                const float *Rz, const float *Lm, const float *tab, int ns, const int *smap, const float *sshift,
                const float *wav, int nr, const int *gmap, const float *gshift, const float *obs, int misfit_type,
                float *vpgrad, float *rhograd, float *wavgrad, float *datamod, float *datares, double *misfit)
{
    const int nt = g->nt;
    const long n = (long)g->nxp * g->nzp;
    float *Ps = malloc((size_t)nt * n * sizeof(float));
    if (!Ps) return -1;
    orc_state fw, bw;
    st_alloc(&fw, g, 0);
    st_alloc(&bw, g, 0);
    for (int it = 0; it < nt; it++) {
        a2d_step(&fw, Rx, Rz, Lm, tab);
        inject(&fw, Lm, 0, ns, smap, sshift, wav, it);
        record(&fw, 0, nr, gmap, gshift, NULL, datamod, it);
        memcpy(Ps + (size_t)it * n, fw.f[0], n * sizeof(float));
    }
    float mis = 0.0f;
    if (misfit_type == 0) {
        /* computeMisfit / computeResiduals, DIFFERENCE (lib/fwi.cpp:597-611, 798-806) */
        for (int tr = 0; tr < nr; tr++) {
            if (gmap[2 * tr] >= 0 && gmap[2 * tr + 1] >= 0)
                for (int it = 0; it < nt; it++) {
                    float r = datamod[it + (long)tr * nt] - obs[it + (long)tr * nt];
                    mis += 0.5 * r * r;
                }
            for (int it = 0; it < nt; it++) datares[it + (long)tr * nt] = 1 * (datamod[it + (long)tr * nt] - obs[it + (long)tr * nt]);
        }
    } else {
        /* CORRELATION (lib/fwi.cpp:617-645, 808-849), with the percentile clip */
        int *valid = malloc(nr * sizeof(int));
        if (!valid) return -1;
        for (int tr = 0; tr < nr; tr++) valid[tr] = gmap[2 * tr] >= 0 && gmap[2 * tr + 1] >= 0;
        const int rc = corr_misfit(nr, nt, valid, datamod, obs, 1, datares, &mis);
        free(valid);
        if (rc) return rc;
    }
    *misfit = mis;
    float *zero = calloc(n, sizeof(float));
    for (int it = nt - 1; it >= 0; it--) {
        if (it < nt - 1) a2d_step(&bw, Rx, Rz, Lm, tab);
        inject(&bw, Lm, 0, nr, gmap, gshift, datares, it);
        a2d_corr(g, nx, nz, vp, rho, Rx, Rz, fw_state_at(Ps, zero, n, nt, it), bw.f[1], bw.f[2], vpgrad, rhograd);
        record(&bw, 0, ns, smap, sshift, NULL, wavgrad, it);
    }
    free(zero);
    st_free(&fw);
    st_free(&bw);
    free(Ps);
    return 0;
}

/* RtmAcoustic2D::run_optimal, zero or extended lags (lib/rtm.cpp:191-219, 423-545). */
int orc_rtm_a2d(const orc_grid *g, int nx, int nz, const float *Rx, const float *Rz, const float *Lm,
                const float *tab, int ns, const int *smap, const float *sshift, const float *wav, int nr,
                const int *gmap, const float *gshift, const float *data, int nhx, int nhz, float *image)
{
    const int nt = g->nt, L = g->lpml, nxp = g->nxp;
    const long n = (long)g->nxp * g->nzp;
    float *Ps = malloc((size_t)nt * n * sizeof(float));
    if (!Ps) return -1;
    orc_state fw, bw;
    st_alloc(&fw, g, 0);
    st_alloc(&bw, g, 0);
    for (int it = 0; it < nt; it++) {
        a2d_step(&fw, Rx, Rz, Lm, tab);
        inject(&fw, Lm, 0, ns, smap, sshift, wav, it);
        memcpy(Ps + (size_t)it * n, fw.f[0], n * sizeof(float));
    }
    float *zero = calloc(n, sizeof(float));
    for (int it = nt - 1; it >= 0; it--) {
        if (it < nt - 1) a2d_step(&bw, Rx, Rz, Lm, tab);
        inject(&bw, Lm, 0, nr, gmap, gshift, data, it);
        const float *ws = fw_state_at(Ps, zero, n, nt, it), *wr = bw.f[0];
        for (int ihx = 0; ihx < nhx; ihx++) {
            int hx = -(nhx - 1) / 2 + ihx;
            for (int ihz = 0; ihz < nhz; ihz++) {
                int hz = -(nhz - 1) / 2 + ihz;
                for (int ix = 0; ix < nx; ix++) {
                    if (ix - hx < 0 || ix - hx >= nx || ix + hx < 0 || ix + hx >= nx) continue;
                    for (int iz = 0; iz < nz; iz++) {
                        if (iz - hz < 0 || iz - hz >= nz || iz + hz < 0 || iz + hz >= nz) continue;
                        image[(((long)ihz * nhx + ihx) * nz + iz) * nx + ix] +=
                            ws[(long)(iz - hz + L) * nxp + (ix - hx + L)] * wr[(long)(iz + hz + L) * nxp + (ix + hx + L)];
                    }
                }
            }
        }
    }
    free(zero);
    st_free(&fw);
    st_free(&bw);
    free(Ps);
    return 0;
}

long orc_state_size(int nxp, int nzp, int elastic) { return (long)nxp * nzp * (elastic ? 5 : 3); }

/* ================================================================== acoustic 3D
 * WavesAcoustic3D::forwardstepVelocity/Stress (lib/waves.cpp:710-998),
 * insertSource/recordData (lib/waves.cpp:999-1190), ModellingAcoustic3D::run
 * (lib/modelling.cpp:363-474).  Arrays a[(iz*nyp + iy)*nxp + ix]; C-PML memory
 * per face pair: x [nzp][nyp][2L], y [nzp][2L][nxp], z [2L][nyp][nxp]. */
typedef struct {
    int nxp, nyp, nzp;
    int lpml, order, fs;
    float dx, dy, dz, dt;
    int nt;
} orc_grid3;

typedef struct {
    orc_grid3 g;
    float *f[4];            /* P, Vx, Vy, Vz */
    float *px[2], *py[2], *pz[2];   /* [0] velocity step (P), [1] stress step (Vxx, Vyy, Vzz) */
} orc_state3;

static void st3_alloc(orc_state3 *s, const orc_grid3 *g)
{
    s->g = *g;
    long n = (long)g->nxp * g->nyp * g->nzp;
    for (int k = 0; k < 4; k++) s->f[k] = calloc(n, sizeof(float));
    for (int k = 0; k < 2; k++) {
        s->px[k] = calloc((long)g->nzp * g->nyp * 2 * g->lpml, sizeof(float));
        s->py[k] = calloc((long)g->nzp * 2 * g->lpml * g->nxp, sizeof(float));
        s->pz[k] = calloc((long)2 * g->lpml * g->nyp * g->nxp, sizeof(float));
    }
}
static void st3_free(orc_state3 *s)
{
    for (int k = 0; k < 4; k++) free(s->f[k]);
    for (int k = 0; k < 2; k++) { free(s->px[k]); free(s->py[k]); free(s->pz[k]); }
}

static void a3d_step(orc_state3 *s, const float *Rx, const float *Ry, const float *Rz, const float *Lm,
                     const float *tab)
{
    const orc_grid3 *g = &s->g;
    const int nx = g->nxp, ny = g->nyp, nz = g->nzp, L = g->lpml, o = g->order;
    const long sy = nx, sz = (long)nx * ny;
    float *P = s->f[0], *Vx = s->f[1], *Vy = s->f[2], *Vz = s->f[3];
    int b, sl, t;
    for (int iz = 0; iz < nz; iz++)
        for (int iy = 0; iy < ny; iy++)
            for (int ix = 0; ix < nx; ix++) {
                long p = iz * sz + iy * sy + ix;
                float d = d_fw(P, p, 1, ix, nx, o, g->dx), a = g->dt * Rx[p];
                Vx[p] += a * d;
                if ((t = strip(ix, nx, L, &b, &sl)) >= 0)
                    Vx[p] = cpml(Vx[p], a, d, &s->px[0][((long)iz * ny + iy) * 2 * L + sl], tab, L, b + 3, t);
                d = d_fw(P, p, sy, iy, ny, o, g->dy);
                a = g->dt * Ry[p];
                Vy[p] += a * d;
                if ((t = strip(iy, ny, L, &b, &sl)) >= 0)
                    Vy[p] = cpml(Vy[p], a, d, &s->py[0][((long)iz * 2 * L + sl) * nx + ix], tab, L, b + 3, t);
                d = d_fw(P, p, sz, iz, nz, o, g->dz);
                a = g->dt * Rz[p];
                Vz[p] += a * d;
                if ((t = strip(iz, nz, L, &b, &sl)) >= 0)
                    Vz[p] = cpml(Vz[p], a, d, &s->pz[0][((long)sl * ny + iy) * nx + ix], tab, L, b + 3, t);
            }
    for (int iz = 0; iz < nz; iz++)
        for (int iy = 0; iy < ny; iy++)
            for (int ix = 0; ix < nx; ix++) {
                long p = iz * sz + iy * sy + ix;
                float al = g->dt * Lm[p];
                float d = d_bw(Vx, p, 1, ix, nx, o, g->dx);
                P[p] += al * d;
                if ((t = strip(ix, nx, L, &b, &sl)) >= 0)
                    P[p] = cpml(P[p], al, d, &s->px[1][((long)iz * ny + iy) * 2 * L + sl], tab, L, b, t);
                d = d_bw(Vy, p, sy, iy, ny, o, g->dy);
                P[p] += al * d;
                if ((t = strip(iy, ny, L, &b, &sl)) >= 0)
                    P[p] = cpml(P[p], al, d, &s->py[1][((long)iz * 2 * L + sl) * nx + ix], tab, L, b, t);
                d = d_bw(Vz, p, sz, iz, nz, o, g->dz);
                P[p] += al * d;
                if ((t = strip(iz, nz, L, &b, &sl)) >= 0)
                    P[p] = cpml(P[p], al, d, &s->pz[1][((long)sl * ny + iy) * nx + ix], tab, L, b, t);
            }
}

/* field codes: 0 PRESSURE, 1 VX, 2 VY, 3 VZ; maps (x,y,z) */
static void inject3(orc_state3 *s, const float *Mod, int field, int ntr, const int *map, const float *shift,
                    const float *wav, int it)
{
    const orc_grid3 *g = &s->g;
    const int nx = g->nxp, ny = g->nyp, L = g->lpml;
    float *F = s->f[field == 0 ? 0 : field];
    for (int i = 0; i < ntr; i++) {
        const int *m = map + 3 * i;
        const float *sh = shift + 3 * i;
        if (m[0] < 0 || m[1] < 0 || m[2] < 0) continue;
        float xt[2] = {1 - sh[0], sh[0]}, yt[2] = {1 - sh[1], sh[1]}, zt[2] = {1 - sh[2], sh[2]};
        float w = wav[it + (long)i * g->nt];
        for (int i1 = 0; i1 < 2; i1++)
            for (int i2 = 0; i2 < 2; i2++)
                for (int i3 = 0; i3 < 2; i3++) {
                    long p = ((long)(L + m[2] + i1) * ny + (L + m[1] + i2)) * nx + (L + m[0] + i3);
                    F[p] += g->dt * Mod[p] * w * xt[i3] * yt[i2] * zt[i1];
                }
    }
}

static void record3(const orc_state3 *s, int field, int ntr, const int *map, const float *shift, float *out, int it)
{
    const orc_grid3 *g = &s->g;
    const int nx = g->nxp, ny = g->nyp, L = g->lpml;
    const float *F = s->f[field == 0 ? 0 : field];
    for (int i = 0; i < ntr; i++) {
        const int *m = map + 3 * i;
        const float *sh = shift + 3 * i;
        if (m[0] < 0 || m[1] < 0 || m[2] < 0) continue;
        float xt[2] = {1 - sh[0], sh[0]}, yt[2] = {1 - sh[1], sh[1]}, zt[2] = {1 - sh[2], sh[2]};
        float *o = &out[it + (long)i * g->nt];
        for (int i1 = 0; i1 < 2; i1++)
            for (int i2 = 0; i2 < 2; i2++)
                for (int i3 = 0; i3 < 2; i3++) {
                    long p = ((long)(L + m[2] + i1) * ny + (L + m[1] + i2)) * nx + (L + m[0] + i3);
                    *o += xt[i3] * yt[i2] * zt[i1] * F[p];
                }
    }
}

/* ModellingAcoustic3D::run for one shot.  models: Rx, Ry, Rz, L (padded). */
int orc_mod_a3d(const orc_grid3 *g, const float *Rx, const float *Ry, const float *Rz, const float *Lm,
                const float *tab, int ns, const int *smap, const float *sshift, const float *wav, int sfield, int nr,
                const int *gmap, const float *gshift, int rfield, float *out, int nsteps, float *state_out)
{
    orc_state3 s;
    st3_alloc(&s, g);
    const float *smod = sfield == 0 ? Lm : sfield == 1 ? Rx : sfield == 2 ? Ry : Rz;
    for (int it = 0; it < nsteps; it++) {
        a3d_step(&s, Rx, Ry, Rz, Lm, tab);
        inject3(&s, smod, sfield, ns, smap, sshift, wav, it);
        record3(&s, rfield, nr, gmap, gshift, out, it);
    }
    if (state_out) {
        long n = (long)g->nxp * g->nyp * g->nzp;
        for (int k = 0; k < 4; k++) memcpy(state_out + k * n, s.f[k], n * sizeof(float));
    }
    st3_free(&s);
    return 0;
}

/* ================================================================== elastic 2D FWI gradient
 * FwiElastic2D::crossCorr (lib/fwi.cpp:2591-2775) on the interior 1..n-2 of the
 * unpadded window: fw = forward Vx,Vz,Sxx,Szz,Sxz, bw = adjoint fields.  vpg holds
 * the lambda correlation, vsg the mu correlation until scaleGrad. */
static void e2d_corr(const orc_grid *g, int nx, int nz, const float *Rx, const float *Rz, float *const *fw,
                     float *const *bw, float *vpg, float *vsg, float *rhog, int sfield, int ns, const int *smap,
                     const float *sshift, float *wavgrad, int it)
{
    const int L = g->lpml, P = g->nxp;
    const float dx = g->dx, dz = g->dz;
    const float *wsx = fw[0], *wsz = fw[1], *wsxx = fw[2], *wszz = fw[3], *wsxz = fw[4];
    const float *wrx = bw[0], *wrz = bw[1], *rsxx = bw[2], *rszz = bw[3], *rsxz = bw[4];
    for (int ix = 1; ix < nx - 1; ix++)
        for (int iz = 1; iz < nz - 1; iz++) {
            long q = (long)(iz + L) * P + (ix + L), u = (long)iz * nx + ix;
            float msxx = (wsx[q] - wsx[q - 1]) / dx;
            float mszz = (wsz[q] - wsz[q - P]) / dz;
            vpg[u] -= (msxx + mszz) * (rsxx[q] + rszz[q]);
            float msxz1 = (wsx[q - 1] - wsx[q - 1 - P]) / dz + (wsz[q - P] - wsz[q - 1 - P]) / dx;
            float msxz2 = (wsx[q] - wsx[q - P]) / dz + (wsz[q + 1 - P] - wsz[q - P]) / dx;
            float msxz3 = (wsx[q - 1 + P] - wsx[q - 1]) / dz + (wsz[q] - wsz[q - 1]) / dx;
            float msxz4 = (wsx[q + P] - wsx[q]) / dz + (wsz[q + 1] - wsz[q]) / dx;
            float mrxz1 = rsxz[q - 1 - P], mrxz2 = rsxz[q - P], mrxz3 = rsxz[q - 1], mrxz4 = rsxz[q];
            vsg[u] += (2.0) * (msxx * rszz[q] + mszz * rsxx[q]) -
                      0.25 * (msxz1 * mrxz1 + msxz2 * mrxz2 + msxz3 * mrxz3 + msxz4 * mrxz4);
            for (int i = 0; i < ns && wavgrad; i++) {
                if (smap[2 * i] != ix || smap[2 * i + 1] != iz) continue;
                float xt[2] = {1 - sshift[2 * i], sshift[2 * i]}, zt[2] = {1 - sshift[2 * i + 1], sshift[2 * i + 1]};
                for (int i1 = 0; i1 < 2; i1++)
                    for (int i2 = 0; i2 < 2; i2++) {
                        long r = q + (long)i1 * P + i2;
                        float v = sfield == 0 ? rsxx[r] + rszz[r] : sfield == 1 ? wrx[r] : wrz[r];
                        wavgrad[it + (long)i * g->nt] += xt[i2] * zt[i1] * v;
                    }
            }
            float uderx = 0.5 * wrx[q] * Rx[q] * (wsxx[q + 1] - wsxx[q]) / dx;
            uderx += 0.5 * wrx[q - 1] * Rx[q - 1] * (wsxx[q] - wsxx[q - 1]) / dx;
            uderx += 0.5 * wrx[q] * Rx[q] * (wsxz[q] - wsxz[q - P]) / dz;
            uderx += 0.5 * wrx[q - 1] * Rx[q - 1] * (wsxz[q - 1] - wsxz[q - 1 - P]) / dz;
            float uderz = 0.5 * wrz[q] * Rz[q] * (wsxz[q] - wsxz[q - 1]) / dx;
            uderz += 0.5 * wrz[q - P] * Rz[q - P] * (wsxz[q - P] - wsxz[q - 1 - P]) / dx;
            uderz += 0.5 * wrz[q] * Rz[q] * (wszz[q + P] - wszz[q]) / dz;
            uderz += 0.5 * wrz[q - P] * Rz[q - P] * (wszz[q] - wszz[q - P]) / dz;
            rhog[u] -= (uderx + uderz);
        }
}

/* FwiElastic2D::scaleGrad (lib/fwi.cpp:2778-2849) */
static void e2d_scale(int nx, int nz, const float *Vp, const float *Vs, const float *Rho, float *vpg, float *vsg,
                      float *rhog)
{
    for (int ix = 0; ix < nx; ix++)
        for (int iz = 0; iz < nz; iz++) {
            long u = (long)iz * nx + ix;
            float vpscale = 2.0 * Rho[u] * Vp[u];
            float vsscale = 2.0 * Rho[u] * Vs[u];
            float rhoscale1 = Vp[u] * Vp[u] - 2.0 * Vs[u] * Vs[u];
            float rhoscale2 = Vs[u] * Vs[u];
            float lambda = vpg[u], mu = vsg[u];
            vpg[u] = vpscale * lambda;
            vsg[u] = vsscale * mu - 2.0 * vsscale * lambda;
            float rho = rhog[u];
            rhog[u] = rhoscale1 * lambda + rhoscale2 * mu + rho;
        }
}

/* FwiElastic2D CORRELATION misfit and residuals (lib/fwi.cpp:2939-3001, 3309-3426)
 * for the P, Ux, Uz components (c = 0, 1, 2 at offsets c*nr*nt): per trace and
 * component, norms in float as in the acoustic case; the misfit adds
 * (rp + rx + rz) with non-finite terms set to zero, over the traces whose Ux map
 * is on the grid; residuals for every trace.  Clips: x and z share the larger of
 * their two 97th-percentile magnitudes, and a sample whose x residual reaches it
 * loses both its x and z residual; P has its own clip; non-finite residuals are
 * set to zero. */
static int fin(float v) { return !isnan(v) && !isinf(v); }

static float kth_mag(const float *r, long tot, long pos, float *buf)
{
    for (long k = 0; k < tot; k++) buf[k] = fabsf(r[k]);
    qsort(buf, tot, sizeof(float), cmp_float);
    return buf[pos];
}

static int e2d_corr_misfit(int nr, int nt, const int *gmap_vx, const float *mods, const float *obs, float *ress, float *mis)
{
    const long nd = (long)nr * nt;
    for (int tr = 0; tr < nr; tr++) {
        float n1[3], n2[3], n3[3];
        for (int c = 0; c < 3; c++) {
            const float *m = mods + c * nd + (long)tr * nt, *o = obs + c * nd + (long)tr * nt;
            n1[c] = n2[c] = n3[c] = 0.0f;
            for (int it = 0; it < nt; it++) {
                n1[c] += m[it] * m[it];
                n2[c] += o[it] * o[it];
                n3[c] += m[it] * o[it];
            }
            n1[c] = sqrtf(n1[c]);
            n2[c] = sqrtf(n2[c]);
            if (n1[c] == 0) n1[c] = 1.0f;
            if (n2[c] == 0) n2[c] = 1.0f;
        }
        if (gmap_vx[2 * tr] >= 0 && gmap_vx[2 * tr + 1] >= 0)
            for (int it = 0; it < nt; it++) {
                float r[3];
                for (int c = 0; c < 3; c++) {
                    const long k = c * nd + (long)tr * nt + it;
                    r[c] = (float)((-1.0) * (mods[k] * obs[k] / (n1[c] * n2[c])));
                    if (!fin(r[c])) r[c] = 0.0f;
                }
                *mis += (r[0] + r[1] + r[2]);
            }
        for (int c = 0; c < 3; c++) {
            n3[c] /= (n1[c] * n2[c]);
            for (int it = 0; it < nt; it++) {
                const long k = c * nd + (long)tr * nt + it;
                ress[k] = (float)((-1.0) * ((obs[k] / (n1[c] * n2[c])) - (mods[k] / (n1[c] * n1[c])) * n3[c]));
            }
        }
    }
    float *buf = malloc(nd * sizeof(float));
    if (!buf) return -1;
    const long pos = (long)((97ul * (unsigned long)nt * (unsigned long)nr) / 100ul);
    float *rp = ress, *rx = ress + nd, *rz = ress + 2 * nd;
    float pclip = kth_mag(rx, nd, pos, buf);
    const float zclip = kth_mag(rz, nd, pos, buf);
    if (zclip > pclip) pclip = zclip;
    for (long k = 0; k < nd; k++) {
        if (fabsf(rx[k]) >= pclip) { rx[k] = 0.0f; rz[k] = 0.0f; }
        if (!fin(rx[k])) rx[k] = 0.0f;
        if (!fin(rz[k])) rz[k] = 0.0f;
    }
    pclip = kth_mag(rp, nd, pos, buf);
    for (long k = 0; k < nd; k++) {
        if (fabsf(rp[k]) >= pclip) rp[k] = 0.0f;
        if (!fin(rp[k])) rp[k] = 0.0f;
    }
    free(buf);
    return 0;
}

/* FwiElastic2D::run_optimal with the DIFFERENCE (misfit_type 0) or CORRELATION (1) misfit: P, Ux (VX) and Uz (VZ)
 * data at the receivers; all forward states kept in memory.  maps: gmap[3] /
 * gshift[3] for the P, VX and VZ trace sets; obs/mods/ress: [3][nr][nt]. */
int orc_fwi_e2d(const orc_grid *g, int nx, int nz, const float *vp, const float *vs, const float *rho,
                const float *Rx, const float *Rz, const float *Lm, const float *L2M, const float *M, const float *tab,
                int ns, const int *smap, const float *sshift, const float *wav, int sfield, int nr,
                const int *const *gmap, const float *const *gshift, const float *obs, int misfit_type, float *vpg,
                float *vsg, float *rhog, float *wavgrad, float *mods, float *ress, double *misfit)
{
    const int nt = g->nt;
    const long n = (long)g->nxp * g->nzp, nd = (long)nr * nt;
    float *Ps = malloc((size_t)nt * 5 * n * sizeof(float));
    if (!Ps) return -1;
    orc_state fw, bw;
    st_alloc(&fw, g, 1);
    st_alloc(&bw, g, 1);
    const float *smod = sfield == 1 ? Rx : Rz;
    for (int it = 0; it < nt; it++) {
        e2d_vel(&fw, Rx, Rz, Lm, L2M, M, tab, 0);
        e2d_str(&fw, Lm, L2M, M, tab, 0);
        inject(&fw, smod, sfield, ns, smap, sshift, wav, it);
        record(&fw, 0, nr, gmap[0], gshift[0], NULL, mods, it);
        record(&fw, 1, nr, gmap[1], gshift[1], NULL, mods + nd, it);
        record(&fw, 3, nr, gmap[2], gshift[2], NULL, mods + 2 * nd, it);
        for (int k = 0; k < 5; k++) memcpy(Ps + ((size_t)it * 5 + k) * n, fw.f[k], n * sizeof(float));
    }
    float mis = 0.0f;
    if (misfit_type == 0) {
        /* computeMisfit / computeResiduals (lib/fwi.cpp:2852-2905, 3227-3290), DIFFERENCE */
        for (int tr = 0; tr < nr; tr++) {
            const int valid = gmap[1][2 * tr] >= 0 && gmap[1][2 * tr + 1] >= 0;
            for (int it = 0; it < nt; it++) {
                long k = it + (long)tr * nt;
                float rp = mods[k] - obs[k], rx = mods[nd + k] - obs[nd + k], rz = mods[2 * nd + k] - obs[2 * nd + k];
                if (valid) mis += 0.5 * (rp * rp + rx * rx + rz * rz);
                ress[k] = rp;
                ress[nd + k] = rx;
                ress[2 * nd + k] = rz;
            }
        }
    } else if (e2d_corr_misfit(nr, nt, gmap[1], mods, obs, ress, &mis)) {
        return -1;
    }
    *misfit = mis;
    float *zero = calloc(5 * n, sizeof(float));
    for (int it = nt - 1; it >= 0; it--) {
        if (it < nt - 1) {
            e2d_vel(&bw, Rx, Rz, Lm, L2M, M, tab, 1);
            e2d_str(&bw, Lm, L2M, M, tab, 1);
        }
        inject(&bw, NULL, 0, nr, gmap[0], gshift[0], ress, it);
        inject(&bw, Rx, 1, nr, gmap[1], gshift[1], ress + nd, it);
        inject(&bw, Rz, 3, nr, gmap[2], gshift[2], ress + 2 * nd, it);
        const float *st = it == nt - 1 ? Ps + (size_t)it * 5 * n : it == 0 ? zero : Ps + (size_t)(it - 1) * 5 * n;
        float *fwf[5];
        for (int k = 0; k < 5; k++) fwf[k] = (float *)st + k * n;
        e2d_corr(g, nx, nz, Rx, Rz, fwf, bw.f, vpg, vsg, rhog, sfield, ns, smap, sshift, wavgrad, it);
    }
    e2d_scale(nx, nz, vp, vs, rho, vpg, vsg, rhog);
    free(zero);
    st_free(&fw);
    st_free(&bw);
    free(Ps);
    return 0;
}

/* RtmAcoustic3D::run_optimal with (nhx, nhy, nhz) lags (lib/rtm.cpp:601-637, 735-859),
 * forward pressure kept for every step; pairing as fw_state_at().
 * image [nhz][nhy][nhx][nz][ny][nx]. */
int orc_rtm_a3d(const orc_grid3 *g, int nx, int ny, int nz, const float *Rx, const float *Ry, const float *Rz,
                const float *Lm, const float *tab, int ns, const int *smap, const float *sshift, const float *wav,
                int nr, const int *gmap, const float *gshift, const float *data, int nhx, int nhy, int nhz,
                float *image)
{
    const int nt = g->nt, L = g->lpml, nxp = g->nxp, nyp = g->nyp;
    const long n = (long)g->nxp * g->nyp * g->nzp;
    float *Ps = malloc((size_t)nt * n * sizeof(float));
    if (!Ps) return -1;
    orc_state3 fw, bw;
    st3_alloc(&fw, g);
    st3_alloc(&bw, g);
    for (int it = 0; it < nt; it++) {
        a3d_step(&fw, Rx, Ry, Rz, Lm, tab);
        inject3(&fw, Lm, 0, ns, smap, sshift, wav, it);
        memcpy(Ps + (size_t)it * n, fw.f[0], n * sizeof(float));
    }
    float *zero = calloc(n, sizeof(float));
    for (int it = nt - 1; it >= 0; it--) {
        if (it < nt - 1) a3d_step(&bw, Rx, Ry, Rz, Lm, tab);
        inject3(&bw, Lm, 0, nr, gmap, gshift, data, it);
        const float *ws = fw_state_at(Ps, zero, n, nt, it), *wr = bw.f[0];
        for (int ihx = 0; ihx < nhx; ihx++) {
            int hx = -(nhx - 1) / 2 + ihx;
            for (int ihy = 0; ihy < nhy; ihy++) {
                int hy = -(nhy - 1) / 2 + ihy;
                for (int ihz = 0; ihz < nhz; ihz++) {
                    int hz = -(nhz - 1) / 2 + ihz;
                    for (int ix = 0; ix < nx; ix++) {
                        if (ix - hx < 0 || ix - hx >= nx || ix + hx < 0 || ix + hx >= nx) continue;
                        for (int iy = 0; iy < ny; iy++) {
                            if (iy - hy < 0 || iy - hy >= ny || iy + hy < 0 || iy + hy >= ny) continue;
                            for (int iz = 0; iz < nz; iz++) {
                                if (iz - hz < 0 || iz - hz >= nz || iz + hz < 0 || iz + hz >= nz) continue;
                                long ii = ((((long)ihz * nhy + ihy) * nhx + ihx) * nz + iz) * (long)nx * ny +
                                          (long)iy * nx + ix;
                                long ps = ((long)(iz - hz + L) * nyp + (iy - hy + L)) * nxp + (ix - hx + L);
                                long pr = ((long)(iz + hz + L) * nyp + (iy + hy + L)) * nxp + (ix + hx + L);
                                image[ii] += ws[ps] * wr[pr];
                            }
                        }
                    }
                }
            }
        }
    }
    free(zero);
    st3_free(&fw);
    st3_free(&bw);
    free(Ps);
    return 0;
}

/* FwiAcoustic3D::crossCorr (lib/fwi.cpp:1403-1466) on 1..n-1 of the unpadded window.
 * The reference's last z-term uses the adjoint Vz of the cell below in y (iy-1),
 * with Rz of the cell above in z (iz-1); that is restated as it is. */
static void a3d_corr(const orc_grid3 *g, int nx, int ny, int nz, const float *Vp, const float *Rho, const float *Rx,
                     const float *Ry, const float *Rz, const float *wsp, const float *wrx, const float *wry,
                     const float *wrz, float *vpgrad, float *rhograd)
{
    const int L = g->lpml;
    const long sy = g->nxp, sz = (long)g->nxp * g->nyp;
    const float dx = g->dx, dy = g->dy, dz = g->dz;
    for (int ix = 1; ix < nx; ix++)
        for (int iy = 1; iy < ny; iy++)
            for (int iz = 1; iz < nz; iz++) {
                long q = (iz + L) * sz + (iy + L) * sy + (ix + L);
                long u = ((long)iz * ny + iy) * nx + ix;
                float vpscale = -2.0 / (Vp[u]);
                float rhoscale1 = -1.0 / (Rho[u]);
                float mrxx = (wrx[q] - wrx[q - 1]) / dx;
                float mryy = (wry[q] - wry[q - sy]) / dy;
                float mrzz = (wrz[q] - wrz[q - sz]) / dz;
                vpgrad[u] -= vpscale * wsp[q] * (mrxx + mryy + mrzz);
                rhograd[u] -= rhoscale1 * wsp[q] * (mrxx + mryy + mrzz);
                float uderx = (0.5) * wrx[q] * Rx[q] * (wsp[q + 1] - wsp[q]) / dx;
                uderx += (0.5) * wrx[q - 1] * Rx[q - 1] * (wsp[q] - wsp[q - 1]) / dx;
                float udery = (0.5) * wry[q] * Ry[q] * (wsp[q + sy] - wsp[q]) / dy;
                udery += (0.5) * wry[q - sy] * Ry[q - sy] * (wsp[q] - wsp[q - sy]) / dy;
                float uderz = (0.5) * wrz[q] * Rz[q] * (wsp[q + sz] - wsp[q]) / dz;
                uderz += (0.5) * wrz[q - sy] * Rz[q - sz] * (wsp[q] - wsp[q - sz]) / dz;
                rhograd[u] += (uderx + udery + uderz);
            }
}

/* FwiAcoustic3D::run_optimal with the DIFFERENCE (misfit_type 0) or CORRELATION (1, no clip in 3D) misfit and pressure data, one shot,
 * all forward pressures kept (pairing as fw_state_at()). */
int orc_fwi_a3d(const orc_grid3 *g, int nx, int ny, int nz, const float *vp, const float *rho, const float *Rx,
                const float *Ry, const float *Rz, const float *Lm, const float *tab, int ns, const int *smap,
                const float *sshift, const float *wav, int nr, const int *gmap, const float *gshift, const float *obs,
                int misfit_type, float *vpgrad, float *rhograd, float *wavgrad, float *datamod, float *datares,
                double *misfit)
{
    const int nt = g->nt;
    const long n = (long)g->nxp * g->nyp * g->nzp;
    float *Ps = malloc((size_t)nt * n * sizeof(float));
    if (!Ps) return -1;
    orc_state3 fw, bw;
    st3_alloc(&fw, g);
    st3_alloc(&bw, g);
    for (int it = 0; it < nt; it++) {
        a3d_step(&fw, Rx, Ry, Rz, Lm, tab);
        inject3(&fw, Lm, 0, ns, smap, sshift, wav, it);
        record3(&fw, 0, nr, gmap, gshift, datamod, it);
        memcpy(Ps + (size_t)it * n, fw.f[0], n * sizeof(float));
    }
    float mis = 0.0f;
    if (misfit_type == 0) {
        for (int tr = 0; tr < nr; tr++) {
            const int valid = gmap[3 * tr] >= 0 && gmap[3 * tr + 1] >= 0 && gmap[3 * tr + 2] >= 0;
            for (int it = 0; it < nt; it++) {
                long k = it + (long)tr * nt;
                float r = datamod[k] - obs[k];
                if (valid) mis += 0.5 * r * r;
                datares[k] = 1 * (datamod[k] - obs[k]);
            }
        }
    } else {
        int *valid = malloc(nr * sizeof(int));
        if (!valid) return -1;
        for (int tr = 0; tr < nr; tr++) valid[tr] = gmap[3 * tr] >= 0 && gmap[3 * tr + 1] >= 0 && gmap[3 * tr + 2] >= 0;
        const int rc = corr_misfit(nr, nt, valid, datamod, obs, 0, datares, &mis);
        free(valid);
        if (rc) return rc;
    }
    *misfit = mis;
    float *zero = calloc(n, sizeof(float));
    for (int it = nt - 1; it >= 0; it--) {
        if (it < nt - 1) a3d_step(&bw, Rx, Ry, Rz, Lm, tab);
        inject3(&bw, Lm, 0, nr, gmap, gshift, datares, it);
        a3d_corr(g, nx, ny, nz, vp, rho, Rx, Ry, Rz, fw_state_at(Ps, zero, n, nt, it), bw.f[1], bw.f[2], bw.f[3],
                 vpgrad, rhograd);
        record3(&bw, 0, ns, smap, sshift, wavgrad, it);
    }
    free(zero);
    st3_free(&fw);
    st3_free(&bw);
    free(Ps);
    return 0;
}

/* Interp<float>::interp (lib/interp.cpp:38-186) for trace-major float traces:
 * mode 0 LINEAR (pad 1), 1 BSPLINE (pad 2), 2 SINC (pad 3); the C expressions
 * keep the reference's float/double mix (double literals promote). */
static float orc_sinc(float x)
{
    if (x == 0.0) return 1.0f;
    return (float)(sin(3.14159265358979323846 * x) / (3.14159265358979323846 * x));
}

int orc_interp(int mode, int ntr, int n1, float o1, float d1, const float *in, int n2, float o2, float d2, float *out)
{
    const int pad = mode == 0 ? 1 : mode == 1 ? 2 : 3;
    for (int i = 0; i < ntr; i++)
        for (long j = 0; j < n2; j++) {
            const float val = o2 + (float)j * d2;
            const long i0 = (long)((val - o1) / d1) - (pad - 1);
            float *o = out + (long)i * n2 + j;
            if (i0 < 0 || i0 + (2 * pad) - 1 > (long)n1 - 1) { *o = 0.0f; continue; }
            const float x0 = o1 + (float)(i0 + (pad - 1)) * d1;
            const float d = (val - x0) / d1;
            const float *m = in + (long)i * n1 + i0;
            if (mode == 0) {
                *o = (float)((1.0 - d) * m[0] + d * m[1]);
            } else if (mode == 1) {
                const float xp = (float)(d + 1.0), om = (float)(1.0 - d);
                const float a0 = (float)(((-(1.0 / 6.0) * xp + 1.0) * xp - 2.0) * xp + (4.0 / 3.0));
                const float a1 = (float)((0.5 * d - 1.0) * d * d + (2.0 / 3.0));
                const float a2 = (float)((0.5 * om - 1.0) * om * om + (2.0 / 3.0));
                const float a3 = (float)(1.0 - a0 - a1 - a2);
                *o = a0 * m[0] + a1 * m[1] + a2 * m[2] + a3 * m[3];
            } else {
                float acc = 0.0f;
                for (int k = 0; k < 6; k++)
                    acc = acc + m[k] * orc_sinc((float)((2.0 - k) + d)) * orc_sinc((float)(((2.0 - k) + d) / 3.0));
                *o = acc;
            }
        }
    return 0;
}
