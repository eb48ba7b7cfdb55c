/*
 * ifos_restate.c -- TEST INFRASTRUCTURE ONLY: the CPU oracle for the
 * IFOS2D forward/adjoint propagation path, written from scratch in plain C.
 *
 * It restates, in its own data layout (one padded plane per field, halo H on
 * every side), the arithmetic of the reference's propagation kernels so that
 * it can be pinned bit-for-bit against the reference compiled in place
 * (oracle/_ref) and then serve, without the reference tree, as the checker of
 * the CUDA path.  Every function cites the reference code it follows.  Float
 * and double promotions follow the reference's C expressions (a literal such
 * as 2.0 or 0.5 makes the expression double before the final store), because
 * the pin is bit-exact.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "ifos_oracle.h"

#define H 8
#define PI_D 3.141592653589793

typedef struct {
    orc_cfg c;
    int nx, ny, P, fdoh, psv, sh;
    size_t plane;
    float hc[7];
    /* CPML profiles, index 1..2FW (0 unused) */
    float *Kx, *ax, *bx, *Kxh, *axh, *bxh, *Ky, *ay, *by, *Kyh, *ayh, *byh;
} grid_t;

static inline size_t ix(const grid_t *g, int j, int i) {
    return (size_t)(j - 1 + H) * (size_t)g->P + (size_t)(i - 1 + H);
}
#define A(arr, j, i) (arr)[ix(g, (j), (i))]

static float *plane(const grid_t *g) { return calloc(g->plane, sizeof(float)); }

/* ------------------------------------------------------------------------ */
/* FD coefficients, src/holbergcoeff.c:37-108.  Row 0 is Taylor, rows 1-4 are
 * Holberg's coefficients for a maximum relative group-velocity error of 0.1,
 * 0.5, 1 and 3 percent (Holberg 1987).  Column 0 is the reference's
 * grid-points-per-wavelength figure, 1..6 the stencil weights. */
static const double fd_table[5][6][7] = {
    {{23.0, 1.0, 0, 0, 0, 0, 0},
     {8.0, 9.0 / 8.0, -1.0 / 24.0, 0, 0, 0, 0},
     {6.0, 75.0 / 64.0, -25.0 / 384.0, 3.0 / 640.0, 0, 0, 0},
     {5.0, 1225.0 / 1024.0, -245.0 / 3072.0, 49.0 / 5120.0, -5.0 / 7168.0, 0, 0},
     {5.0, 19845.0 / 16384.0, -735.0 / 8192.0, 567.0 / 40960.0, -405.0 / 229376.0, 35.0 / 294912.0, 0},
     {4.0, 160083.0 / 131072.0, -12705.0 / 131072.0, 22869.0 / 1310720.0, -5445.0 / 1835008.0,
      847.0 / 2359296.0, -63.0 / 2883584.0}},
    {{49.7, 1.0010, 0, 0, 0, 0, 0},
     {8.32, 1.1382, -0.046414, 0, 0, 0, 0},
     {4.77, 1.1965, -0.078804, 0.0081781, 0, 0, 0},
     {3.69, 1.2257, -0.099537, 0.018063, -0.0026274, 0, 0},
     {3.19, 1.2415, -0.11231, 0.026191, -0.0064682, 0.001191, 0},
     {2.91, 1.2508, -0.12034, 0.032131, -0.010142, 0.0029857, -0.00066667}},
    {{22.2, 1.0050, 0, 0, 0, 0, 0},
     {5.65, 1.1534, -0.052806, 0, 0, 0, 0},
     {3.74, 1.2111, -0.088313, 0.011768, 0, 0, 0},
     {3.11, 1.2367, -0.10815, 0.023113, -0.0046905, 0, 0},
     {2.80, 1.2496, -0.11921, 0.031130, -0.0093272, 0.0025161, 0},
     {2.62, 1.2568, -0.12573, 0.036423, -0.013132, 0.0047484, -0.0015979}},
    {{15.8, 1.0100, 0, 0, 0, 0, 0},
     {4.80, 1.1640, -0.057991, 0, 0, 0, 0},
     {3.39, 1.2192, -0.094070, 0.014608, 0, 0, 0},
     {2.90, 1.2422, -0.11269, 0.026140, -0.0064054, 0, 0},
     {2.65, 1.2534, -0.12257, 0.033755, -0.011081, 0.0036784, 0},
     {2.51, 1.2596, -0.12825, 0.038550, -0.014763, 0.0058619, -0.0024538}},
    {{9.16, 1.0300, 0, 0, 0, 0, 0},
     {3.47, 1.1876, -0.072518, 0, 0, 0, 0},
     {2.91, 1.2341, -0.10569, 0.022589, 0, 0, 0},
     {2.61, 1.2516, -0.12085, 0.032236, -0.011459, 0, 0},
     {2.45, 1.2596, -0.12829, 0.038533, -0.014681, 0.0072580, 0},
     {2.36, 1.2640, -0.13239, 0.042217, -0.017803, 0.0081959, -0.0051848}},
};

int orc_fd_coeffs(const orc_cfg *c, float *hc7) {
    if (c->fdorder < 2 || c->fdorder > 12 || (c->fdorder & 1) || c->maxrelerror < 0 || c->maxrelerror > 4)
        return 1;
    for (int k = 0; k < 7; k++) hc7[k] = (float)fd_table[c->maxrelerror][c->fdorder / 2 - 1][k];
    return 0;
}

/* ------------------------------------------------------------------------ */
/* CPML profiles, src/PML_pro.c:83-316 (d0 from the INRIA report, alpha from
 * Festa & Vilotte).  `abs()` on the float d in the reference truncates to
 * int, so `a` stays 0 wherever |d| < 1 (src/PML_pro.c:171-172). */
static void pml_side(float d0, float thick, float origin, int lo, int hi, int left, int clamp, float DH, float DT,
                     float npower, float kmax, float amax, int base, float *d, float *K, float *al, float *a, float *b,
                     float *dh_, float *Kh, float *alh, float *ah, float *bh, float d0_half) {
    for (int i = lo; i <= hi; i++) {
        int h = i - base;
        K[h] = 1.0f;
        Kh[h] = 1.0f;
        float xval = DH * (i - 1);
        float absc, norm;
        absc = left ? origin - xval : xval - origin;
        if (absc >= 0.0) {
            norm = absc / thick;
            d[h] = d0 * pow(norm, npower);
            K[h] = 1.0 + (kmax - 1.0) * pow(norm, npower);
            al[h] = amax * (1.0 - norm);
        }
        absc = left ? origin - (xval + DH / 2.0) : xval + DH / 2.0 - origin;
        if (absc >= 0.0) {
            norm = absc / thick;
            dh_[h] = d0_half * pow(norm, npower);
            Kh[h] = 1.0 + (kmax - 1.0) * pow(norm, npower);
            alh[h] = amax * (1.0 - norm);
        }
        if (clamp) {
            if (al[h] < 0.0) al[h] = 0.0;
            if (alh[h] < 0.0) alh[h] = 0.0;
        }
        b[h] = exp(-(d[h] / K[h] + al[h]) * DT);
        bh[h] = exp(-(dh_[h] / Kh[h] + alh[h]) * DT);
        if ((int)d[h] != 0) a[h] = d[h] * (b[h] - 1.0) / (K[h] * (d[h] + K[h] * al[h]));
        if ((int)dh_[h] != 0) ah[h] = dh_[h] * (bh[h] - 1.0) / (Kh[h] * (dh_[h] + Kh[h] * alh[h]));
    }
}

/* out: 20 arrays of n = 2FW, each 0-based [h-1]:
 * d_x K_x alpha_x a_x b_x | half x | d_y K_y alpha_y a_y b_y | half y */
static void pml_all(const orc_cfg *c, float **arr /* 20 arrays, 1-based, length 2FW+1 */) {
    const float DH = c->dh, DT = c->dt, npower = c->npower, kmax = c->k_max_pml;
    const int FW = c->fw, NX = c->nx, NY = c->ny;
    const float amax = 2.0 * PI_D * (c->fpml / 2.0);
    float thick_x = FW * DH, thick_y = FW * DH;
    float Rcoef = 0.001f;
    float d0_x = -(npower + 1) * c->vppml * log(Rcoef) / (2.0 * thick_x);
    float d0_y = -(npower + 1) * c->vppml * log(Rcoef) / (2.0 * thick_y);
    float xl = thick_x, xr = (NX - 1) * DH - thick_x;
    pml_side(d0_x, thick_x, xl, 1, FW, 1, 1, DH, DT, npower, kmax, amax, 0, arr[0], arr[1], arr[2], arr[3], arr[4],
             arr[5], arr[6], arr[7], arr[8], arr[9], d0_x);
    pml_side(d0_x, thick_x, xr, NX - FW + 1, NX, 0, 1, DH, DT, npower, kmax, amax, NX - 2 * FW, arr[0], arr[1],
             arr[2], arr[3], arr[4], arr[5], arr[6], arr[7], arr[8], arr[9], d0_x);
    float yt = thick_y, yb = (NY - 1) * DH - thick_y;
    pml_side(d0_y, thick_y, yt, 1, FW, 1, 0, DH, DT, npower, kmax, amax, 0, arr[10], arr[11], arr[12], arr[13],
             arr[14], arr[15], arr[16], arr[17], arr[18], arr[19], d0_y);
    /* src/PML_pro.c:299 uses d0_x for the half-node profile of this side */
    pml_side(d0_y, thick_y, yb, NY - FW + 1, NY, 0, 0, DH, DT, npower, kmax, amax, NY - 2 * FW, arr[10], arr[11],
             arr[12], arr[13], arr[14], arr[15], arr[16], arr[17], arr[18], arr[19], d0_x);
}

int orc_pml_profiles(const orc_cfg *c, float *out) {
    int n = 2 * c->fw;
    float *arr[20];
    for (int k = 0; k < 20; k++) arr[k] = calloc((size_t)n + 1, sizeof(float));
    pml_all(c, arr);
    for (int k = 0; k < 20; k++) {
        memcpy(out + (size_t)k * n, arr[k] + 1, (size_t)n * sizeof(float));
        free(arr[k]);
    }
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Source signals, src/wavelet.c:29-133 (analytic shapes only). */
int orc_wavelet(const orc_cfg *c, int shape, int nsrc, const float *srcpos, float *signals) {
    const float DT = c->dt;
    for (int nt = 1; nt <= c->nt; nt++) {
        float t = (float)nt * DT;
        for (int k = 0; k < nsrc; k++) {
            float tshift = srcpos[3 * nsrc + k], fc = srcpos[4 * nsrc + k], a = srcpos[5 * nsrc + k];
            float ts = 1.0 / fc, amp = 0.0f, tau, ag;
            switch (shape) {
                case 1:
                    tau = PI_D * (t - 1.5 * ts - tshift) / (ts);
                    amp = (((1.0 - 2.0 * tau * tau) * exp(-tau * tau)));
                    break;
                case 2:
                    if ((t < tshift) || (t > (tshift + ts))) amp = 0.0;
                    else amp = ((sin(2.0 * PI_D * (t - tshift) * fc) - 0.5 * sin(4.0 * PI_D * (t - tshift) * fc)));
                    break;
                case 4:
                    if ((t < tshift) || (t > (tshift + ts))) amp = 0.0;
                    else amp = pow(sin(PI_D * (t - tshift) / ts), 3.0);
                    break;
                case 5:
                    ts = 1.2 / fc;
                    ag = PI_D * PI_D * fc * fc;
                    amp = -2.0 * ag * (t - ts) * exp(-ag * (t - ts) * (t - ts));
                    break;
                case 6:
                    amp = 0.0;
                    if (nt == 1 + (int)floor(tshift / DT + 0.5)) amp = 1.0;
                    break;
                case 8:
                    if (t < tshift) amp = 0.0;
                    if ((t >= tshift) && (t <= (tshift + ts)))
                        amp = (ts / (0.75 * PI_D)) *
                              (0.5 - 0.75 * cos(PI_D * (t - tshift) / ts) + 0.25 * pow(cos(PI_D * (t - tshift) / ts), 3.0));
                    if (t > (tshift + ts)) amp = ts / (0.75 * PI_D);
                    break;
                default:
                    return 1;
            }
            signals[(size_t)k * c->nt + (nt - 1)] = amp * a;
        }
    }
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Residual, L2, energy for LNORM=2, VELOCITY=0, no windows/kills:
 * src/calc_res.c:137-281, src/calc_energy.c, src/calc_misfit.c.  Seismograms
 * are integrated by running sums times DT; the residual is time-reversed; the
 * norms are accumulated in float. */
int orc_calc_res(const orc_cfg *c, int ntr, int ns, const float *obs, const float *syn, float *diff, double *l2,
                 double *energy, double *misfit) {
    const float DT = c->dt;
    float L2 = 0.0f, E = 0.0f, M = 0.0f;
    float *is = malloc(sizeof(float) * (size_t)ns), *id = malloc(sizeof(float) * (size_t)ns);
    for (int i = 0; i < ntr; i++) {
        const float *s = syn + (size_t)i * ns, *d = obs + (size_t)i * ns;
        float rs = 0.0f, rd = 0.0f;
        for (int j = 0; j < ns; j++) {
            rs += s[j];
            is[j] = rs * DT;
            rd += d[j];
            id[j] = rd * DT;
        }
        for (int j = 0; j < ns; j++) {
            float r = is[j] - id[j];
            diff[(size_t)i * ns + (ns - 1 - j)] = r;
            L2 += r * r;
        }
        for (int j = 0; j < ns; j++) E += id[j] * id[j];
        for (int j = 0; j < ns; j++) {
            float r = id[j] - is[j];
            M += r * r;
        }
    }
    free(is);
    free(id);
    *l2 = L2;
    *energy = E;
    *misfit = M;
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Shot state */
typedef struct {
    /* model (halo planes so the ghost ring fits) */
    float *rho, *vp, *vs, *taus, *taup, *rip, *rjp, *uipjp, *tausipjp;
    /* visco coefficients */
    float *fipjp, *f, *g, **dip, **d, **e;
    float bip[ORC_MAX_L + 1], bjm[ORC_MAX_L + 1], cip[ORC_MAX_L + 1], cjm[ORC_MAX_L + 1], eta[ORC_MAX_L + 1];
    float sumu, sumpi;
    /* wavefields */
    float *vx, *vy, *sxx, *syy, *sxy, *vxp1, *vyp1, *vz, *sxz, *syz, *vzp1, *sp;
    float **r, **p, **q, **t, **o;
    /* CPML memory: x strips NY x 2FW, y strips 2FW x NX (1-based h) */
    float *psi_sxx_x, *psi_sxy_x, *psi_vxx, *psi_vyx, *psi_vxxs, *psi_sxz_x, *psi_vzx;
    float *psi_syy_y, *psi_sxy_y, *psi_vyy, *psi_vxy, *psi_syz_y, *psi_vzy;
} shot_t;

#define PX(arr, j, h) (arr)[(size_t)((j)-1) * (size_t)(2 * g->c.fw) + (size_t)((h)-1)]
#define PY(arr, h, i) (arr)[(size_t)((h)-1) * (size_t)g->nx + (size_t)((i)-1)]

/* periodic one-cell material ring of a single rank, src/matcopy_elastic.c:59-141 */
static void ghost_ring(const grid_t *g, float *m) {
    const int NX = g->nx, NY = g->ny;
    for (int i = 0; i <= NX + 1; i++) A(m, NY + 1, i) = A(m, 1, i);
    for (int i = 0; i <= NX + 1; i++) A(m, 0, i) = A(m, NY, i);
    for (int j = 0; j <= NY + 1; j++) A(m, j, NX + 1) = A(m, j, 1);
    for (int j = 0; j <= NY + 1; j++) A(m, j, 0) = A(m, j, NX);
}

static void setup_model(const grid_t *g, shot_t *s, const orc_shot_io *io) {
    const orc_cfg *c = &g->c;
    const int NX = g->nx, NY = g->ny, L = c->L;
    s->rho = plane(g); s->vp = plane(g); s->vs = plane(g); s->taus = plane(g); s->taup = plane(g);
    s->rip = plane(g); s->rjp = plane(g); s->uipjp = plane(g); s->tausipjp = plane(g);
    for (int j = 1; j <= NY; j++)
        for (int i = 1; i <= NX; i++) {
            size_t k = (size_t)(j - 1) * NX + (i - 1);
            A(s->rho, j, i) = io->rho[k];
            A(s->vp, j, i) = io->vp[k];
            A(s->vs, j, i) = c->acoustic ? 0.0f : io->vs[k];
            A(s->taus, j, i) = io->taus ? io->taus[k] : c->tau;
            A(s->taup, j, i) = io->taup ? io->taup[k] : c->tau;
        }
    ghost_ring(g, s->rho);
    ghost_ring(g, s->vp);
    ghost_ring(g, s->vs);
    if (L && !c->acoustic) { ghost_ring(g, s->taus); ghost_ring(g, s->taup); }
    if (L && c->acoustic) ghost_ring(g, s->taup); /* src/matcopy_viscac.c: rho, pi, taup */
    /* harmonic shear modulus at (i+1/2, j+1/2), src/av_mue.c:45-61 */
    if (!c->acoustic)
        for (int j = 1; j <= NY; j++)
            for (int i = 1; i <= NX; i++) {
                float u1 = A(s->rho, j, i) * A(s->vs, j, i) * A(s->vs, j, i);
                float u2 = A(s->rho, j, i + 1) * A(s->vs, j, i + 1) * A(s->vs, j, i + 1);
                float u3 = A(s->rho, j + 1, i) * A(s->vs, j + 1, i) * A(s->vs, j + 1, i);
                float u4 = A(s->rho, j + 1, i + 1) * A(s->vs, j + 1, i + 1) * A(s->vs, j + 1, i + 1);
                float v = 4.0 / ((1.0 / u1) + (1.0 / u2) + (1.0 / u3) + (1.0 / u4));
                if ((u1 == 0.0) || (u2 == 0.0) || (u3 == 0.0) || (u4 == 0.0)) v = 0.0;
                A(s->uipjp, j, i) = v;
            }
    /* reciprocal averaged densities, src/av_rho.c:26-33 */
    for (int j = 1; j <= NY; j++)
        for (int i = 1; i <= NX; i++) {
            A(s->rjp, j, i) = 1.0 / (0.5 * (A(s->rho, j, i) + A(s->rho, j + 1, i)));
            A(s->rip, j, i) = 1.0 / (0.5 * (A(s->rho, j, i) + A(s->rho, j, i + 1)));
        }
    if (!L) return;
    /* src/av_tau.c:25-29 (unused by the acoustic update) */
    for (int j = 1; j <= NY; j++)
        for (int i = 1; i <= NX; i++)
            A(s->tausipjp, j, i) =
                0.25 * (A(s->taus, j, i) + A(s->taus, j, i + 1) + A(s->taus, j + 1, i) + A(s->taus, j + 1, i + 1));
    /* relaxation: eta_l = DT*2*pi*FL_l (src/readmod.c:44-49,
     * src/readmod_viscac.c:47-50), then the coefficient set of
     * src/prepare_update_s.c:33-77; the acoustic set of
     * src/prepare_update_p.c:44-64 (g, bjm, cjm, e) is the same formulas */
    float pts[ORC_MAX_L + 1];
    for (int l = 1; l <= L; l++) {
        pts[l] = 1.0 / (2.0 * PI_D * c->fl[l - 1]);
        s->eta[l] = c->dt / pts[l];
    }
    float ws = 2.0 * PI_D * c->f_ref;
    float sumu = 0.0f, sumpi = 0.0f;
    for (int l = 1; l <= L; l++) {
        sumu = sumu + ((ws * ws * pts[l] * pts[l]) / (1.0 + ws * ws * pts[l] * pts[l]));
        sumpi = sumpi + ((ws * ws * pts[l] * pts[l]) / (1.0 + ws * ws * pts[l] * pts[l]));
    }
    s->sumu = sumu;
    s->sumpi = sumpi;
    s->fipjp = plane(g); s->f = plane(g); s->g = plane(g);
    s->dip = calloc((size_t)L + 1, sizeof(float *));
    s->d = calloc((size_t)L + 1, sizeof(float *));
    s->e = calloc((size_t)L + 1, sizeof(float *));
    for (int l = 1; l <= L; l++) { s->dip[l] = plane(g); s->d[l] = plane(g); s->e[l] = plane(g); }
    const float DT = c->dt;
    for (int j = 1; j <= NY; j++)
        for (int i = 1; i <= NX; i++) {
            float mu = (A(s->vs, j, i) * A(s->vs, j, i) * A(s->rho, j, i)) / (1.0 + sumu * A(s->taus, j, i));
            float pi = (A(s->vp, j, i) * A(s->vp, j, i) * A(s->rho, j, i)) / (1.0 + sumpi * A(s->taup, j, i));
            float muipjp = A(s->uipjp, j, i) / (1.0 + sumu * A(s->tausipjp, j, i));
            A(s->fipjp, j, i) = muipjp * DT * (1.0 + L * A(s->tausipjp, j, i));
            A(s->f, j, i) = mu * DT * (1.0 + L * A(s->taus, j, i));
            A(s->g, j, i) = pi * DT * (1.0 + L * A(s->taup, j, i));
            for (int l = 1; l <= L; l++) {
                s->bip[l] = 1.0 / (1.0 + (s->eta[l] * 0.5));
                s->bjm[l] = 1.0 / (1.0 + (s->eta[l] * 0.5));
                s->cip[l] = 1.0 - (s->eta[l] * 0.5);
                s->cjm[l] = 1.0 - (s->eta[l] * 0.5);
                A(s->dip[l], j, i) = muipjp * s->eta[l] * A(s->tausipjp, j, i);
                A(s->d[l], j, i) = mu * s->eta[l] * A(s->taus, j, i);
                A(s->e[l], j, i) = pi * s->eta[l] * A(s->taup, j, i);
            }
        }
}

static float **planes(const grid_t *g, int n) {
    float **v = calloc((size_t)n + 1, sizeof(float *));
    for (int l = 1; l <= n; l++) v[l] = plane(g);
    return v;
}

static void alloc_state(const grid_t *g, shot_t *s) {
    const int L = g->c.L;
    float **fl[] = {&s->vx, &s->vy, &s->sxx, &s->syy, &s->sxy, &s->vxp1, &s->vyp1,
                    &s->vz, &s->sxz, &s->syz, &s->vzp1, &s->sp};
    for (size_t k = 0; k < sizeof(fl) / sizeof(fl[0]); k++) *fl[k] = plane(g);
    if (L) { s->r = planes(g, L); s->p = planes(g, L); s->q = planes(g, L); s->t = planes(g, L); s->o = planes(g, L); }
    size_t nxs = (size_t)g->ny * 2 * g->c.fw + 1, nys = (size_t)2 * g->c.fw * g->nx + 1;
    float **px[] = {&s->psi_sxx_x, &s->psi_sxy_x, &s->psi_vxx, &s->psi_vyx, &s->psi_vxxs, &s->psi_sxz_x, &s->psi_vzx};
    float **py[] = {&s->psi_syy_y, &s->psi_sxy_y, &s->psi_vyy, &s->psi_vxy, &s->psi_syz_y, &s->psi_vzy};
    for (size_t k = 0; k < 7; k++) *px[k] = calloc(nxs, sizeof(float));
    for (size_t k = 0; k < 6; k++) *py[k] = calloc(nys, sizeof(float));
}

static void zero_state(const grid_t *g, shot_t *s) {
    const int L = g->c.L;
    float *fl[] = {s->vx, s->vy, s->sxx, s->syy, s->sxy, s->vxp1, s->vyp1, s->vz, s->sxz, s->syz, s->vzp1, s->sp};
    for (size_t k = 0; k < 12; k++) memset(fl[k], 0, g->plane * sizeof(float));
    for (int l = 1; l <= L; l++) {
        memset(s->r[l], 0, g->plane * sizeof(float)); memset(s->p[l], 0, g->plane * sizeof(float));
        memset(s->q[l], 0, g->plane * sizeof(float)); memset(s->t[l], 0, g->plane * sizeof(float));
        memset(s->o[l], 0, g->plane * sizeof(float));
    }
    size_t nxs = (size_t)g->ny * 2 * g->c.fw + 1, nys = (size_t)2 * g->c.fw * g->nx + 1;
    float *px[] = {s->psi_sxx_x, s->psi_sxy_x, s->psi_vxx, s->psi_vyx, s->psi_vxxs, s->psi_sxz_x, s->psi_vzx};
    float *py[] = {s->psi_syy_y, s->psi_sxy_y, s->psi_vyy, s->psi_vxy, s->psi_syz_y, s->psi_vzy};
    for (size_t k = 0; k < 7; k++) memset(px[k], 0, nxs * sizeof(float));
    for (size_t k = 0; k < 6; k++) memset(py[k], 0, nys * sizeof(float));
}

/* CPML strip membership, src/update_v_PML.c:177-228 */
static inline int in_left(const grid_t *g, int i) { return !g->c.boundary && i <= g->c.fw; }
static inline int in_right(const grid_t *g, int i) { return !g->c.boundary && i >= g->nx - g->c.fw + 1; }
static inline int in_top(const grid_t *g, int j) { return !g->c.free_surf && j <= g->c.fw; }
static inline int in_bot(const grid_t *g, int j) { return j >= g->ny - g->c.fw + 1; }

/* psi = b*psi + a*d; d = d/K + psi (the CPML recursion of every kernel) */
static inline float cpml(float *psi, float b, float a, float K, float d) {
    *psi = b * *psi + a * d;
    return d / K + *psi;
}
#define CPML_X(arr, j, i, pb, pa, pK, d)                                                                     \
    do {                                                                                                      \
        if (in_left(g, i)) d = cpml(&PX(arr, j, i), pb[i], pa[i], pK[i], d);                                  \
        if (in_right(g, i)) {                                                                                 \
            int h1_ = (i) - g->nx + 2 * g->c.fw;                                                              \
            d = cpml(&PX(arr, j, h1_), pb[h1_], pa[h1_], pK[h1_], d);                                         \
        }                                                                                                     \
    } while (0)
#define CPML_Y(arr, j, i, pb, pa, pK, d)                                                                     \
    do {                                                                                                      \
        if (in_top(g, j)) d = cpml(&PY(arr, j, i), pb[j], pa[j], pK[j], d);                                   \
        if (in_bot(g, j)) {                                                                                   \
            int h1_ = (j) - g->ny + 2 * g->c.fw;                                                              \
            d = cpml(&PY(arr, h1_, i), pb[h1_], pa[h1_], pK[h1_], d);                                         \
        }                                                                                                     \
    } while (0)

/* staggered first differences: forward (+) reads f[k+m] - f[k-m+1],
 * backward (-) reads f[k+m-1] - f[k-m]; summed in the reference's order,
 * the m=1 term starting the sum as in its written-out expressions
 * (src/update_v_PML.c:164-175) */
static inline float dfx_fwd(const grid_t *g, const float *f, int j, int i) {
    float s = g->hc[1] * (A(f, j, i + 1) - A(f, j, i));
    for (int m = 2; m <= g->fdoh; m++) s += g->hc[m] * (A(f, j, i + m) - A(f, j, i - m + 1));
    return s;
}
static inline float dfx_bwd(const grid_t *g, const float *f, int j, int i) {
    float s = g->hc[1] * (A(f, j, i) - A(f, j, i - 1));
    for (int m = 2; m <= g->fdoh; m++) s += g->hc[m] * (A(f, j, i + m - 1) - A(f, j, i - m));
    return s;
}
static inline float dfy_fwd(const grid_t *g, const float *f, int j, int i) {
    float s = g->hc[1] * (A(f, j + 1, i) - A(f, j, i));
    for (int m = 2; m <= g->fdoh; m++) s += g->hc[m] * (A(f, j + m, i) - A(f, j - m + 1, i));
    return s;
}
static inline float dfy_bwd(const grid_t *g, const float *f, int j, int i) {
    float s = g->hc[1] * (A(f, j, i) - A(f, j - 1, i));
    for (int m = 2; m <= g->fdoh; m++) s += g->hc[m] * (A(f, j + m - 1, i) - A(f, j - m, i));
    return s;
}

/* the same sums accumulated from zero, as the reference's generic loops do
 * (its FDORDER 10/12 default branches: src/update_v_acoustic_PML.c:396-409,
 * src/update_p_PML.c:275-287, src/update_s_visc_PML.c:615-660) */
static inline float dfx_fwd_z(const grid_t *g, const float *f, int j, int i) {
    float s = 0.0f;
    for (int m = 1; m <= g->fdoh; m++) s += g->hc[m] * (A(f, j, i + m) - A(f, j, i - m + 1));
    return s;
}
static inline float dfx_bwd_z(const grid_t *g, const float *f, int j, int i) {
    float s = 0.0f;
    for (int m = 1; m <= g->fdoh; m++) s += g->hc[m] * (A(f, j, i + m - 1) - A(f, j, i - m));
    return s;
}
static inline float dfy_fwd_z(const grid_t *g, const float *f, int j, int i) {
    float s = 0.0f;
    for (int m = 1; m <= g->fdoh; m++) s += g->hc[m] * (A(f, j + m, i) - A(f, j - m + 1, i));
    return s;
}
static inline float dfy_bwd_z(const grid_t *g, const float *f, int j, int i) {
    float s = 0.0f;
    for (int m = 1; m <= g->fdoh; m++) s += g->hc[m] * (A(f, j + m - 1, i) - A(f, j - m, i));
    return s;
}

static int quirk_hi(const grid_t *g) { return g->c.fdorder >= 10 && !g->c.hi_order_corrected; }

/* ---- velocity half step ------------------------------------------------ */
/* P-SV: src/update_v_PML.c:161-252 (orders 2-8 form, used for every order
 * when hi_order_corrected) and :466-528 (reference 10/12 branches). */
static void update_v_psv(const grid_t *g, shot_t *s, int sw) {
    const float DT = g->c.dt, DH = g->c.dh;
    const float dtdh = DT * DT / DH;
    for (int j = 1; j <= g->ny; j++)
        for (int i = 1; i <= g->nx; i++) {
            if (quirk_hi(g)) {
                /* one written-out sum per component (src/update_v_PML.c:469-490) */
                float ax_ = dfx_fwd(g, s->sxx, j, i), ay_ = dfy_fwd(g, s->syy, j, i);
                for (int m = 1; m <= g->fdoh; m++) ax_ += g->hc[m] * (A(s->sxy, j + m - 1, i) - A(s->sxy, j - m, i));
                for (int m = 1; m <= g->fdoh; m++) ay_ += g->hc[m] * (A(s->sxy, j, i + m - 1) - A(s->sxy, j, i - m));
                A(s->vx, j, i) += ax_ * dtdh * A(s->rip, j, i);
                A(s->vy, j, i) += ay_ * dtdh * A(s->rjp, j, i);
                continue;
            }
            float sxx_x = dfx_fwd(g, s->sxx, j, i);
            float sxy_x = dfx_bwd(g, s->sxy, j, i);
            float sxy_y = dfy_bwd(g, s->sxy, j, i);
            float syy_y = dfy_fwd(g, s->syy, j, i);
            CPML_X(s->psi_sxx_x, j, i, g->bxh, g->axh, g->Kxh, sxx_x);
            CPML_X(s->psi_sxy_x, j, i, g->bx, g->ax, g->Kx, sxy_x);
            CPML_Y(s->psi_syy_y, j, i, g->byh, g->ayh, g->Kyh, syy_y);
            CPML_Y(s->psi_sxy_y, j, i, g->by, g->ay, g->Ky, sxy_y);
            if (sw == 0) {
                A(s->vxp1, j, i) = A(s->rip, j, i) * (sxx_x + sxy_y) / DH;
                A(s->vyp1, j, i) = A(s->rjp, j, i) * (sxy_x + syy_y) / DH;
            } else {
                A(s->vxp1, j, i) += A(s->vx, j, i) * DT;
                A(s->vyp1, j, i) += A(s->vy, j, i) * DT;
            }
            A(s->vx, j, i) += DT * A(s->rip, j, i) * (sxx_x + sxy_y) / DH;
            A(s->vy, j, i) += DT * A(s->rjp, j, i) * (sxy_x + syy_y) / DH;
        }
}

/* SH: src/update_v_PML_SH.c:61-297 (CPML on every order); vzp1 keeps the old
 * velocity (:98). */
static void update_v_sh(const grid_t *g, shot_t *s) {
    const float DT = g->c.dt, DH = g->c.dh;
    for (int j = 1; j <= g->ny; j++)
        for (int i = 1; i <= g->nx; i++) {
            float sxz_x = dfx_bwd(g, s->sxz, j, i);
            float syz_y = dfy_fwd(g, s->syz, j, i);
            CPML_X(s->psi_sxz_x, j, i, g->bx, g->ax, g->Kx, sxz_x);
            CPML_Y(s->psi_syz_y, j, i, g->byh, g->ayh, g->Kyh, syz_y);
            A(s->vzp1, j, i) = A(s->vz, j, i);
            A(s->vz, j, i) += A(s->rjp, j, i) * DT * (sxz_x + syz_y) / (DH);
        }
}

/* acoustic: src/update_v_acoustic_PML.c:72-148 and the 10/12 default :396-409 */
static void update_v_ac(const grid_t *g, shot_t *s, int sw) {
    const float DT = g->c.dt, DH = g->c.dh;
    const float dtdh = DT * DT / DH;
    for (int j = 1; j <= g->ny; j++)
        for (int i = 1; i <= g->nx; i++) {
            const int q = quirk_hi(g);
            float sp_x = q ? dfx_fwd_z(g, s->sp, j, i) : dfx_fwd(g, s->sp, j, i);
            float sp_y = q ? dfy_fwd_z(g, s->sp, j, i) : dfy_fwd(g, s->sp, j, i);
            if (q) {
                A(s->vx, j, i) += sp_x * dtdh * A(s->rip, j, i);
                A(s->vy, j, i) += sp_y * dtdh * A(s->rjp, j, i);
                continue;
            }
            CPML_X(s->psi_sxx_x, j, i, g->bxh, g->axh, g->Kxh, sp_x);
            CPML_Y(s->psi_syy_y, j, i, g->byh, g->ayh, g->Kyh, sp_y);
            if (sw == 0) {
                A(s->vxp1, j, i) = A(s->rip, j, i) * (sp_x) / DH;
                A(s->vyp1, j, i) = A(s->rjp, j, i) * (sp_y) / DH;
            } else {
                A(s->vxp1, j, i) += A(s->vx, j, i) * DT;
                A(s->vyp1, j, i) += A(s->vy, j, i) * DT;
            }
            A(s->vx, j, i) += DT * A(s->rip, j, i) * (sp_x) / DH;
            A(s->vy, j, i) += DT * A(s->rjp, j, i) * (sp_y) / DH;
        }
}

/* point forces after the velocity update: forward src/update_v_PML.c:553-564,
 * src/update_v_PML_SH.c:327-333; adjoint (residuals at the receivers,
 * unscaled) :567-578 and src/update_v_PML_SH.c:338-345. */
static void inject_v(const grid_t *g, shot_t *s, int sw, int nt, int n, const float *pos, const float *sig0,
                     const float *sig1, const float *sigz) {
    const float DT = g->c.dt, DH = g->c.dh;
    const int NT = g->c.nt;
    for (int l = 0; l < n; l++) {
        int i = (int)pos[l], j = (int)pos[n + l];
        if (sw == 0) {
            if (g->psv) {
                float azi_rad = pos[6 * n + l] * PI_D / 180;
                int type = (int)pos[7 * n + l];
                float s0 = sig0[(size_t)l * NT + nt - 1], s1 = sig1[(size_t)l * NT + nt - 1];
                if (type == 2) A(s->vx, j, i) += (DT * A(s->rip, j, i) * s1) / (DH * DH);
                if (type == 3) A(s->vy, j, i) += (DT * A(s->rjp, j, i) * s1) / (DH * DH);
                if (type == 4) {
                    A(s->vx, j, i) += (DT * A(s->rip, j, i) * sin(azi_rad) * s0) / (DH * DH);
                    A(s->vy, j, i) += (DT * A(s->rjp, j, i) * cos(azi_rad) * s0) / (DH * DH);
                }
            }
            if (g->sh && !g->c.acoustic)
                A(s->vz, j, i) += (A(s->rjp, j, i) * DT * 1.0 * sigz[(size_t)l * NT + nt - 1]) / (DH * DH);
        } else {
            if (g->psv) {
                int at = g->c.adjoint_type;
                float s0 = sig0[(size_t)l * NT + nt - 1], s1 = sig1[(size_t)l * NT + nt - 1];
                if (at == 1) {
                    A(s->vx, j, i) += s0;
                    A(s->vy, j, i) += s1;
                }
                if (at == 2) A(s->vy, j, i) += s1;
                if (at == 3) A(s->vx, j, i) += s0;
            }
            if (g->sh && !g->c.acoustic) A(s->vz, j, i) += sigz[(size_t)l * NT + nt - 1];
        }
    }
}

/* ---- stress half step --------------------------------------------------- */
/* P-SV elastic: src/update_s_elastic_PML.c:151-241 (orders 2-8 form) and
 * :442-535 (reference 10/12 branches). */
static void update_s_psv_el(const grid_t *g, shot_t *s) {
    const float DT = g->c.dt, DH = g->c.dh;
    const float dhi = DT / DH;
    for (int j = 1; j <= g->ny; j++)
        for (int i = 1; i <= g->nx; i++) {
            float vxx = dfx_bwd(g, s->vx, j, i) * dhi;
            float vyx = dfx_fwd(g, s->vy, j, i) * dhi;
            float vxy = dfy_fwd(g, s->vx, j, i) * dhi;
            float vyy = dfy_bwd(g, s->vy, j, i) * dhi;
            if (quirk_hi(g)) {
                float fipjp = A(s->uipjp, j, i) * DT, f = A(s->vs, j, i) * DT, gg = A(s->vp, j, i) * DT;
                A(s->sxy, j, i) += (fipjp * (vxy + vyx));
                A(s->sxx, j, i) += (gg * (vxx + vyy)) - (2.0 * f * vyy);
                A(s->syy, j, i) += (gg * (vxx + vyy)) - (2.0 * f * vxx);
                continue;
            }
            CPML_X(s->psi_vxx, j, i, g->bx, g->ax, g->Kx, vxx);
            CPML_X(s->psi_vyx, j, i, g->bxh, g->axh, g->Kxh, vyx);
            CPML_Y(s->psi_vyy, j, i, g->by, g->ay, g->Ky, vyy);
            CPML_Y(s->psi_vxy, j, i, g->byh, g->ayh, g->Kyh, vxy);
            float fipjp = A(s->uipjp, j, i);
            float rho = A(s->rho, j, i), u = A(s->vs, j, i), pi = A(s->vp, j, i);
            float f = rho * u * u;
            float gg = rho * ((pi * pi) - 2 * u * u);
            A(s->sxy, j, i) += fipjp * (vyx + vxy);
            A(s->sxx, j, i) += gg * (vxx + vyy) + (2.0 * f * vxx);
            A(s->syy, j, i) += gg * (vxx + vyy) + (2.0 * f * vyy);
        }
}

/* P-SV viscoelastic, L standard linear solids: src/update_s_visc_PML.c:
 * orders 2-8 with CPML :62-516, reference 10/12 = default branch without
 * CPML :518-660. */
static void update_s_psv_visc(const grid_t *g, shot_t *s) {
    const float DT = g->c.dt, DH = g->c.dh;
    const int L = g->c.L;
    const float dhi = 1.0 / DH, dthalbe = DT / 2.0;
    for (int j = 1; j <= g->ny; j++)
        for (int i = 1; i <= g->nx; i++) {
            const int q = quirk_hi(g);
            float vxx = (q ? dfx_bwd_z(g, s->vx, j, i) : dfx_bwd(g, s->vx, j, i)) * dhi;
            float vyx = (q ? dfx_fwd_z(g, s->vy, j, i) : dfx_fwd(g, s->vy, j, i)) * dhi;
            float vxy = (q ? dfy_fwd_z(g, s->vx, j, i) : dfy_fwd(g, s->vx, j, i)) * dhi;
            float vyy = (q ? dfy_bwd_z(g, s->vy, j, i) : dfy_bwd(g, s->vy, j, i)) * dhi;
            if (!q) {
                CPML_X(s->psi_vxx, j, i, g->bx, g->ax, g->Kx, vxx);
                CPML_X(s->psi_vyx, j, i, g->bxh, g->axh, g->Kxh, vyx);
                CPML_Y(s->psi_vyy, j, i, g->by, g->ay, g->Ky, vyy);
                CPML_Y(s->psi_vxy, j, i, g->byh, g->ayh, g->Kyh, vxy);
            }
            float sumr = 0.0f, sump = 0.0f, sumq = 0.0f;
            for (int l = 1; l <= L; l++) {
                sumr += A(s->r[l], j, i);
                sump += A(s->p[l], j, i);
                sumq += A(s->q[l], j, i);
            }
            float fipjp = A(s->fipjp, j, i), f = A(s->f, j, i), gg = A(s->g, j, i);
            A(s->sxy, j, i) += (fipjp * (vxy + vyx)) + (dthalbe * sumr);
            A(s->sxx, j, i) += (gg * (vxx + vyy)) - (2.0 * f * vyy) + (dthalbe * sump);
            A(s->syy, j, i) += (gg * (vxx + vyy)) - (2.0 * f * vxx) + (dthalbe * sumq);
            sumr = sump = sumq = 0.0f;
            for (int l = 1; l <= L; l++) {
                float *rr = &A(s->r[l], j, i), *pp = &A(s->p[l], j, i), *qq = &A(s->q[l], j, i);
                *rr = s->bip[l] * (*rr * s->cip[l] - (A(s->dip[l], j, i) * (vxy + vyx)));
                *pp = s->bjm[l] * (*pp * s->cjm[l] - (A(s->e[l], j, i) * (vxx + vyy)) + (2.0 * A(s->d[l], j, i) * vyy));
                *qq = s->bjm[l] * (*qq * s->cjm[l] - (A(s->e[l], j, i) * (vxx + vyy)) + (2.0 * A(s->d[l], j, i) * vxx));
                sumr += *rr;
                sump += *pp;
                sumq += *qq;
            }
            A(s->sxy, j, i) += (dthalbe * sumr);
            A(s->sxx, j, i) += (dthalbe * sump);
            A(s->syy, j, i) += (dthalbe * sumq);
        }
}

/* SH elastic: src/update_s_elastic_PML_SH.c:60-400; SH visco:
 * src/update_s_visc_PML_SH.c:59-476 (CPML on every order for both). */
static void update_s_sh(const grid_t *g, shot_t *s) {
    const float DT = g->c.dt, DH = g->c.dh;
    const int L = g->c.L;
    const float dhi = L ? (float)(1.0 / DH) : DT / DH, dthalbe = DT / 2.0;
    for (int j = 1; j <= g->ny; j++)
        for (int i = 1; i <= g->nx; i++) {
            float vzx = dfx_fwd(g, s->vz, j, i) * dhi;
            float vzy = dfy_bwd(g, s->vz, j, i) * dhi;
            CPML_X(s->psi_vzx, j, i, g->bxh, g->axh, g->Kxh, vzx);
            CPML_Y(s->psi_vzy, j, i, g->by, g->ay, g->Ky, vzy);
            if (!L) {
                float fipjp = A(s->uipjp, j, i);
                float f = A(s->rho, j, i) * A(s->vs, j, i) * A(s->vs, j, i);
                A(s->sxz, j, i) += (fipjp * vzx);
                A(s->syz, j, i) += (f * vzy);
            } else {
                float sumo = 0.0f, sumt = 0.0f;
                for (int l = 1; l <= L; l++) {
                    sumo += A(s->o[l], j, i);
                    sumt += A(s->t[l], j, i);
                }
                A(s->sxz, j, i) += (A(s->fipjp, j, i) * vzx) + (dthalbe * sumo);
                A(s->syz, j, i) += (A(s->f, j, i) * vzy) + (dthalbe * sumt);
                sumo = sumt = 0.0f;
                for (int l = 1; l <= L; l++) {
                    float *oo = &A(s->o[l], j, i), *tt = &A(s->t[l], j, i);
                    *oo = s->bip[l] * (*oo * s->cip[l] - (A(s->dip[l], j, i) * vzx));
                    *tt = s->bjm[l] * (*tt * s->cjm[l] - (A(s->d[l], j, i) * vzy));
                    sumt += *tt;
                    sumo += *oo;
                }
                A(s->sxz, j, i) += (dthalbe * sumo);
                A(s->syz, j, i) += (dthalbe * sumt);
            }
        }
}

/* acoustic pressure: src/update_p_PML.c:55-273 and the 10/12 default :275-287 */
static void update_p_ac(const grid_t *g, shot_t *s) {
    const float DT = g->c.dt, DH = g->c.dh;
    const float dhi = DT / DH;
    for (int j = 1; j <= g->ny; j++)
        for (int i = 1; i <= g->nx; i++) {
            if (quirk_hi(g)) {
                float vxx = dfx_bwd_z(g, s->vx, j, i), vyy = dfy_bwd_z(g, s->vy, j, i);
                float gg = A(s->vp, j, i) * DT;
                A(s->sp, j, i) += (gg * (vxx + vyy)) * dhi;
                continue;
            }
            float vxx = dfx_bwd(g, s->vx, j, i) * dhi;
            float vyy = dfy_bwd(g, s->vy, j, i) * dhi;
            CPML_X(s->psi_vxx, j, i, g->bx, g->ax, g->Kx, vxx);
            CPML_Y(s->psi_vyy, j, i, g->by, g->ay, g->Ky, vyy);
            float gg = A(s->rho, j, i) * (A(s->vp, j, i) * A(s->vp, j, i));
            A(s->sp, j, i) += gg * (vxx + vyy);
        }
}

/* viscoacoustic pressure with L relaxation mechanisms:
 * src/update_p_visc_PML.c:61-146 (FDORDER 2: written-out differences and
 * CPML, whose vyx/vxy memories it also advances) and :148-182 (every other
 * order: the generic loop from zero, without CPML) */
static void update_p_visc(const grid_t *g, shot_t *s) {
    const float DT = g->c.dt, DH = g->c.dh;
    const float dhi = 1.0 / DH, dthalbe = DT / 2.0;
    const int L = g->c.L;
    for (int j = 1; j <= g->ny; j++)
        for (int i = 1; i <= g->nx; i++) {
            float vxx, vyy;
            if (g->c.fdorder == 2) {
                vxx = dfx_bwd(g, s->vx, j, i) * dhi;
                float vyx = dfx_fwd(g, s->vy, j, i) * dhi;
                float vxy = dfy_fwd(g, s->vx, j, i) * dhi;
                vyy = dfy_bwd(g, s->vy, j, i) * dhi;
                CPML_X(s->psi_vxx, j, i, g->bx, g->ax, g->Kx, vxx);
                CPML_X(s->psi_vyx, j, i, g->bxh, g->axh, g->Kxh, vyx);
                CPML_Y(s->psi_vyy, j, i, g->by, g->ay, g->Ky, vyy);
                CPML_Y(s->psi_vxy, j, i, g->byh, g->ayh, g->Kyh, vxy);
            } else {
                vxx = dfx_bwd_z(g, s->vx, j, i) * dhi;
                vyy = dfy_bwd_z(g, s->vy, j, i) * dhi;
            }
            float sump = 0.0f;
            for (int l = 1; l <= L; l++) sump += A(s->p[l], j, i);
            A(s->sp, j, i) += (A(s->g, j, i) * (vxx + vyy)) + (dthalbe * sump);
            sump = 0.0f;
            for (int l = 1; l <= L; l++) {
                float *pp = &A(s->p[l], j, i);
                *pp = s->bjm[l] * (*pp * s->cjm[l] - (A(s->e[l], j, i) * (vxx + vyy)));
                sump += *pp;
            }
            A(s->sp, j, i) += (dthalbe * sump);
        }
}

/* explosive source (forward) / pressure residual (adjoint, ADJOINT_TYPE 4),
 * src/psource.c:37-74 */
static void psource(const grid_t *g, shot_t *s, int nt, int n, const float *pos, const float *sig, int sw) {
    const float DH = g->c.dh;
    const int NT = g->c.nt;
    for (int l = 0; l < n; l++) {
        int i = (int)pos[l], j = (int)pos[n + l];
        const float *sl = sig + (size_t)l * NT - 1; /* 1-based */
        float amp = 0.0f;
        if (sw == 0) {
            if (nt == 1) amp = sl[nt + 1] / (2.0 * DH * DH);
            if ((nt > 1) && (nt < NT)) amp = (sl[nt + 1] - sl[nt - 1]) / (2.0 * DH * DH);
            if (nt == NT) amp = -sl[nt - 1] / (2.0 * DH * DH);
        } else {
            amp = sl[nt];
        }
        if (!g->c.acoustic) {
            A(s->sxx, j, i) += 0.5 * amp;
            A(s->syy, j, i) += 0.5 * amp;
        } else {
            A(s->sp, j, i) += amp;
        }
    }
}

/* free surface by imaging at j=1: src/surface_elastic_PML.c:47-106,
 * src/surface_PML.c:61-173, src/surface_acoustic_PML.c:28-38 */
static void surface(const grid_t *g, shot_t *s) {
    const float DT = g->c.dt, DH = g->c.dh;
    const int L = g->c.L, fdoh = g->fdoh, j = 1;
    const float dh24 = 1.0 / DH, dthalbe = DT / 2.0;
    if (g->c.acoustic) {
        for (int i = 1; i <= g->nx; i++) {
            A(s->sp, j, i) = 0;
            for (int m = 1; m <= fdoh; m++) A(s->sp, j - m, i) = -A(s->sp, j + m, i);
        }
        return;
    }
    if (g->psv)
        for (int i = 1; i <= g->nx; i++) {
            A(s->syy, j, i) = 0.0;
            if (L)
                for (int l = 1; l <= L; l++) A(s->q[l], j, i) = 0.0;
            float vxx = 0.0f, vyy = 0.0f;
            for (int m = 1; m <= fdoh; m++) {
                A(s->syy, j - m, i) = -A(s->syy, j + m, i);
                A(s->sxy, j - m, i) = -A(s->sxy, j + m - 1, i);
                vxx += g->hc[m] * (A(s->vx, j, i + m - 1) - A(s->vx, j, i - m));
                vyy += g->hc[m] * (A(s->vy, j + m - 1, i) - A(s->vy, j - m, i));
            }
            vxx *= dh24;
            vyy *= dh24;
            CPML_X(s->psi_vxxs, j, i, g->bx, g->ax, g->Kx, vxx);
            float rho = A(s->rho, j, i), u = A(s->vs, j, i), pi = A(s->vp, j, i);
            if (!L) {
                float fjm = rho * u * u * 2.0;
                float gg = rho * ((pi * pi) - 2 * u * u);
                A(s->sxx, j, i) += -DT * ((gg * gg) / (gg + fjm) * vxx + gg * vyy);
            } else {
                float taus = A(s->taus, j, i), taup = A(s->taup, j, i);
                float mu = (u * u * rho) / (1.0 + s->sumu * taus);
                float pm = (pi * pi * rho) / (1.0 + s->sumpi * taup);
                float sump = 0.0f;
                for (int l = 1; l <= L; l++) sump += A(s->p[l], j, i);
                float fjm = mu * 2.0 * (1.0 + L * taus);
                float gg = pm * (1.0 + L * taup);
                A(s->sxx, j, i) += -(DT * (gg - fjm) * (gg - fjm) * vxx / gg) - (DT * (gg - fjm) * vyy) - (dthalbe * sump);
                sump = 0.0f;
                for (int l = 1; l <= L; l++) {
                    float bjm = s->eta[l] / (1.0 + (s->eta[l] * 0.5));
                    float djm = 2.0 * mu * taus;
                    float e = pm * taup;
                    A(s->p[l], j, i) += bjm * (((djm - e) * ((fjm / gg) - 1.0) * vxx) - ((djm - e) * vyy));
                    sump += A(s->p[l], j, i);
                }
                A(s->sxx, j, i) += (dthalbe * sump);
            }
        }
    if (g->sh)
        for (int i = 1; i <= g->nx; i++) {
            A(s->syz, j, i) = 0.0;
            for (int m = 1; m <= fdoh; m++) {
                A(s->syz, j - m, i) = -A(s->syz, j + m, i);
                A(s->sxz, j - m, i) = -A(s->sxz, j + m - 1, i);
            }
        }
}

/* receivers, src/seismo_ssg.c:26-140 */
static void seismo(const grid_t *g, shot_t *s, int nt, int ntr, const int *rec, float *sec) {
    const int NT = g->c.nt, SEISMO = g->c.seismo;
    const float dhi = g->c.dt / g->c.dh;
    float *svx = sec, *svy = sec + (size_t)ntr * NT, *svz = sec + (size_t)2 * ntr * NT;
    float *sp_ = sec + (size_t)3 * ntr * NT, *scurl = sec + (size_t)4 * ntr * NT, *sdiv = sec + (size_t)5 * ntr * NT;
    for (int itr = 0; itr < ntr; itr++) {
        int i = rec[itr], j = rec[ntr + itr];
        size_t o = (size_t)itr * NT + (nt - 1);
        int want_v = SEISMO == 1 || SEISMO == 4 || SEISMO == 5;
        int want_p = SEISMO == 2 || SEISMO == 4 || SEISMO == 5;
        int want_cd = SEISMO == 3 || SEISMO == 4;
        if (want_cd) {
            float vxx = 0, vyy = 0, vyx = 0, vxy = 0;
            for (int m = 1; m <= g->fdoh; m++) {
                vxx += g->hc[m] * (A(s->vx, j, i + m - 1) - A(s->vx, j, i - m));
                vyy += g->hc[m] * (A(s->vy, j + m - 1, i) - A(s->vy, j - m, i));
                vyx += g->hc[m] * (A(s->vy, j, i + m) - A(s->vy, j, i - m + 1));
                vxy += g->hc[m] * (A(s->vx, j + m, i) - A(s->vx, j - m + 1, i));
            }
            vxx *= dhi; vyy *= dhi; vyx *= dhi; vxy *= dhi;
            sdiv[o] = (vxx + vyy) * sqrt(A(s->vp, j, i));
            scurl[o] = !g->c.acoustic ? (vxy - vyx) * sqrt(A(s->vs, j, i)) : 0;
        }
        if (want_v) {
            if (SEISMO == 4 || g->psv) {
                svx[o] = A(s->vx, j, i);
                svy[o] = A(s->vy, j, i);
            }
            if (g->sh) svz[o] = A(s->vz, j, i);
        }
        if (want_p && (SEISMO != 5 || g->psv)) {
            if (!g->c.acoustic) sp_[o] = -A(s->sxx, j, i) - A(s->syy, j, i);
            else sp_[o] = -A(s->sp, j, i);
        }
    }
}

static void get_plane(const grid_t *g, float *dst, const float *src) {
    for (int j = 1; j <= g->ny; j++)
        for (int i = 1; i <= g->nx; i++) dst[(size_t)(j - 1) * g->nx + (i - 1)] = A(src, j, i);
}

static void fields_out(const grid_t *g, shot_t *s, float *out) {
    const float *fl[ORC_NF] = {s->vx, s->vy, s->sxx, s->syy, s->sxy, s->vxp1, s->vyp1, s->vz, s->sxz, s->syz, s->vzp1, s->sp};
    size_t n = (size_t)g->nx * g->ny;
    for (int k = 0; k < ORC_NF; k++) get_plane(g, out + k * n, fl[k]);
}

/* one full time step in the reference driver's order, src/IFOS2D.c:1680-1803 */
static void step(const grid_t *g, shot_t *s, int nt, int sw, const orc_shot_io *io, const float *adjx,
                 const float *adjy, const float *adjz, const float *backpos) {
    const orc_cfg *c = &g->c;
    int n = sw ? io->ntr : io->nsrc;
    const float *pos = sw ? backpos : io->srcpos;
    if (!c->acoustic) {
        if (g->psv) update_v_psv(g, s, sw);
        if (g->sh) update_v_sh(g, s);
    } else {
        update_v_ac(g, s, sw);
    }
    if (sw == 0) inject_v(g, s, 0, nt, n, pos, io->signals, io->signals, io->signals);
    else inject_v(g, s, 1, nt, n, pos, adjx, adjy, adjz);
    if (!c->acoustic) {
        if (g->psv) { if (c->L) update_s_psv_visc(g, s); else update_s_psv_el(g, s); }
        if (g->sh) update_s_sh(g, s);
    } else if (c->L) {
        update_p_visc(g, s);
    } else {
        update_p_ac(g, s);
    }
    /* update_v_PML and update_v_acoustic_PML assign the global SOURCE_TYPE
     * from each source's type column as they inject forces
     * (src/update_v_PML.c:558), so the explosive source below fires when the
     * LAST source of the shot is of type 1. */
    int stype = c->source_type;
    if (sw == 0 && g->psv && n > 0) stype = (int)pos[7 * n + (n - 1)];
    if (sw == 0 && stype == 1 && g->psv) psource(g, s, nt, n, pos, io->signals, 0);
    if (sw == 1 && c->adjoint_type == 4) psource(g, s, nt, n, pos, adjz, 1);
    if (c->free_surf) surface(g, s);
}

int orc_run_shot(const orc_cfg *cfg, orc_shot_io *io) {
    grid_t G, *g = &G;
    memset(g, 0, sizeof G);
    g->c = *cfg;
    g->nx = cfg->nx;
    g->ny = cfg->ny;
    g->P = cfg->nx + 2 * H;
    g->plane = (size_t)(cfg->ny + 2 * H) * (size_t)g->P;
    g->fdoh = cfg->fdorder / 2;
    g->psv = cfg->wavetype == 1 || cfg->wavetype == 3;
    g->sh = cfg->wavetype == 2 || cfg->wavetype == 3;
    if (cfg->parameterization != 1) return 3; /* the restatement covers vp, vs, rho only */
    if (orc_fd_coeffs(cfg, g->hc)) return 1;
    if (g->fdoh + 1 > H) return 2;
    float *prof[20];
    int n2 = 2 * cfg->fw;
    for (int k = 0; k < 20; k++) prof[k] = calloc((size_t)n2 + 1, sizeof(float));
    pml_all(cfg, prof);
    g->Kx = prof[1]; g->ax = prof[3]; g->bx = prof[4];
    g->Kxh = prof[6]; g->axh = prof[8]; g->bxh = prof[9];
    g->Ky = prof[11]; g->ay = prof[13]; g->by = prof[14];
    g->Kyh = prof[16]; g->ayh = prof[18]; g->byh = prof[19];

    shot_t S, *s = &S;
    memset(s, 0, sizeof S);
    setup_model(g, s, io);
    alloc_state(g, s);

    const int NT = cfg->nt, NX = g->nx, NY = g->ny;
    const int ntdtinv = (int)ceil((float)NT / (float)cfg->dtinv);
    const size_t N = (size_t)NX * NY;
    /* forward snapshots, slot-major (slot k holds forward step 1+k*DTINV) */
    int ncomp = 0;
    float *snap = NULL;
    if (io->run_adjoint) {
        ncomp = g->psv ? (cfg->acoustic ? 3 : 5) : 0;
        if (g->sh) ncomp += 3;
        snap = calloc((size_t)ntdtinv * ncomp * N, sizeof(float));
        if (!snap) return 3;
    }
    float *sec = io->sections;
    if (sec) memset(sec, 0, sizeof(float) * (size_t)ORC_NS * io->ntr * NT);
    int nsteps = io->nsteps > 0 && io->nsteps <= NT ? io->nsteps : NT;
    int *is_snap = calloc((size_t)NT + 2, sizeof(int));
    int hin = 0;
    for (int nt = 1; nt <= nsteps; nt++) {
        step(g, s, nt, 0, io, NULL, NULL, NULL, NULL);
        if (cfg->seismo && sec) seismo(g, s, nt, io->ntr, io->recpos, sec);
        if ((nt - 1) % cfg->dtinv == 0) {
            is_snap[nt] = 1;
            if (io->run_adjoint) {
                float *base = snap + (size_t)hin * ncomp * N;
                int k = 0;
                if (g->psv) {
                    get_plane(g, base + (size_t)k++ * N, s->vxp1);
                    get_plane(g, base + (size_t)k++ * N, s->vyp1);
                    if (!cfg->acoustic) {
                        get_plane(g, base + (size_t)k++ * N, s->sxx);
                        get_plane(g, base + (size_t)k++ * N, s->syy);
                        get_plane(g, base + (size_t)k++ * N, s->sxy);
                    } else {
                        get_plane(g, base + (size_t)k++ * N, s->sp);
                    }
                }
                if (g->sh) {
                    get_plane(g, base + (size_t)k++ * N, s->vzp1);
                    get_plane(g, base + (size_t)k++ * N, s->sxz);
                    get_plane(g, base + (size_t)k++ * N, s->syz);
                }
                hin++;
            }
        }
    }
    if (io->fields) fields_out(g, s, io->fields);

    if (io->run_adjoint) {
        const int ntr = io->ntr;
        const float *adjx = io->adj, *adjy = io->adj + (size_t)ntr * NT, *adjz = io->adj + (size_t)2 * ntr * NT;
        float *backpos = calloc((size_t)2 * (ntr > 0 ? ntr : 1), sizeof(float));
        for (int i = 0; i < ntr; i++) {
            backpos[i] = (float)io->recpos[i];
            backpos[ntr + i] = (float)io->recpos[ntr + i];
        }
        zero_state(g, s);
        float *wl = calloc(N, sizeof(float)), *wm = calloc(N, sizeof(float)), *wr = calloc(N, sizeof(float));
        float *wmz = calloc(N, sizeof(float)), *wrz = calloc(N, sizeof(float));
        int hin_a = 1;
        for (int nt = 1; nt <= NT; nt++) {
            step(g, s, nt, 1, io, adjx, adjy, adjz, backpos);
            if (is_snap[NT - nt + 1]) {
                /* zero-lag correlation, src/IFOS2D.c:2379-2419 */
                const float *base = snap + (size_t)(ntdtinv - hin_a) * ncomp * N;
                for (int j = 1; j <= NY; j++)
                    for (int i = 1; i <= NX; i++) {
                        size_t q = (size_t)(j - 1) * NX + (i - 1);
                        int k = 0;
                        if (g->psv) {
                            float frx = base[k++ * N + q], fry = base[k++ * N + q];
                            wr[q] += (A(s->vxp1, j, i) * frx) + (A(s->vyp1, j, i) * fry);
                            if (!cfg->acoustic) {
                                float fx = base[k++ * N + q], fy = base[k++ * N + q], fu = base[k++ * N + q];
                                float sxx = A(s->sxx, j, i), syy = A(s->syy, j, i), sxy = A(s->sxy, j, i);
                                wl[q] += (fx + fy) * (sxx + syy);
                                float rho = A(s->rho, j, i), u = A(s->vs, j, i), pi = A(s->vp, j, i);
                                float muss = rho * u * u;
                                float lamss = rho * pi * pi - 2.0 * muss;
                                if (u > 0.0)
                                    wm[q] += ((1.0 / (muss * muss)) * (fu * sxy)) +
                                             (.25 * (fx + fy * (sxx + syy)) / ((lamss + muss) * (lamss + muss))) +
                                             (.25 * (fx - fy * (sxx - syy)) / (muss * muss));
                            } else {
                                float fp = base[k++ * N + q];
                                wl[q] += (fp) * (A(s->sp, j, i));
                            }
                        }
                        if (g->sh) {
                            float frz = base[k++ * N + q], fxz = base[k++ * N + q], fyz = base[k++ * N + q];
                            wrz[q] += A(s->vzp1, j, i) * frz;
                            float muss = A(s->rho, j, i) * A(s->vs, j, i) * A(s->vs, j, i);
                            wmz[q] += (1.0 / (muss * muss)) * (fxz * A(s->sxz, j, i) + fyz * A(s->syz, j, i));
                        }
                    }
                hin_a++;
            }
        }
        if (io->adj_fields) fields_out(g, s, io->adj_fields);
        if (io->grads) {
            /* per-shot assembly, PARAMETERIZATION=1, src/IFOS2D.c:2477-2601 */
            float *G_ = io->grads;
            memset(G_, 0, sizeof(float) * ORC_NG * N);
            memcpy(G_ + ORC_G_LAM_RAW * N, wl, N * sizeof(float));
            memcpy(G_ + ORC_G_MU_RAW * N, wm, N * sizeof(float));
            memcpy(G_ + ORC_G_RHO_RAW * N, wr, N * sizeof(float));
            memcpy(G_ + ORC_G_MU_Z_RAW * N, wmz, N * sizeof(float));
            memcpy(G_ + ORC_G_RHO_Z_RAW * N, wrz, N * sizeof(float));
            const float DT = cfg->dt;
            for (int j = 1; j <= NY; j++)
                for (int i = 1; i <= NX; i++) {
                    size_t q = (size_t)(j - 1) * NX + (i - 1);
                    float rho = A(s->rho, j, i), u = A(s->vs, j, i), pi = A(s->vp, j, i);
                    float lam = 0, mu = 0;
                    if (g->psv) {
                        lam = -DT * wl[q];
                        float muss = !cfg->acoustic ? rho * u * u : 0;
                        float lamss = rho * pi * pi - 2.0 * muss;
                        if (!cfg->acoustic) lam = (1.0 / (4.0 * (lamss + muss) * (lamss + muss))) * lam;
                        else lam = (1.0 / ((lamss + muss) * (lamss + muss))) * lam;
                        G_[ORC_G_VP * N + q] = 2.0 * pi * rho * lam;
                        if (!cfg->acoustic) {
                            mu = -DT * wm[q];
                            G_[ORC_G_VS * N + q] = -4.0 * rho * u * lam + 2.0 * rho * u * mu;
                        } else {
                            G_[ORC_G_VS * N + q] = wm[q];
                        }
                        float rho_s = -DT * wr[q];
                        if (!cfg->acoustic)
                            G_[ORC_G_RHO * N + q] = ((pi * pi) - (2.0 * u * u)) * lam + u * u * mu + rho_s;
                        else
                            G_[ORC_G_RHO * N + q] = ((pi * pi) * lam) + rho_s;
                    }
                    if (g->sh && !cfg->acoustic) {
                        float mu_z = -DT * wmz[q];
                        G_[ORC_G_VS_Z * N + q] = (2.0 * rho * u * mu_z);
                        float rho_s_z = -DT * wrz[q];
                        G_[ORC_G_RHO_Z * N + q] = ((u * u * mu_z) + rho_s_z);
                    } else {
                        G_[ORC_G_VS_Z * N + q] = wmz[q];
                        G_[ORC_G_RHO_Z * N + q] = wrz[q];
                    }
                }
        }
        free(wl); free(wm); free(wr); free(wmz); free(wrz); free(backpos);
    }
    free(snap);
    free(is_snap);
    for (int k = 0; k < 20; k++) free(prof[k]);
    /* the oracle runs in short-lived test processes; the planes below are the
     * large allocations */
    float *big[] = {s->rho, s->vp, s->vs, s->taus, s->taup, s->rip, s->rjp, s->uipjp, s->tausipjp, s->vx, s->vy,
                    s->sxx, s->syy, s->sxy, s->vxp1, s->vyp1, s->vz, s->sxz, s->syz, s->vzp1, s->sp,
                    s->psi_sxx_x, s->psi_sxy_x, s->psi_vxx, s->psi_vyx, s->psi_vxxs, s->psi_sxz_x, s->psi_vzx,
                    s->psi_syy_y, s->psi_sxy_y, s->psi_vyy, s->psi_vxy, s->psi_syz_y, s->psi_vzy};
    for (size_t k = 0; k < sizeof(big) / sizeof(big[0]); k++) free(big[k]);
    if (cfg->L && !cfg->acoustic) {
        for (int l = 1; l <= cfg->L; l++) {
            free(s->dip[l]); free(s->d[l]); free(s->e[l]);
        }
        free(s->dip); free(s->d); free(s->e); free(s->fipjp); free(s->f); free(s->g);
    }
    if (cfg->L)
        for (int l = 1; l <= cfg->L; l++) {
            free(s->r[l]); free(s->p[l]); free(s->q[l]); free(s->t[l]); free(s->o[l]);
        }
    return 0;
}
