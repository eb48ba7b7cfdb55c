/*
 * ref_harness.c -- TEST INFRASTRUCTURE ONLY (built into oracle/_ref/).
 *
 * Implements ifos_oracle.h by calling the reference's own kernel functions,
 * compiled in place from the IFOS2D source tree, in the order of the
 * reference driver.  This file contains no propagation arithmetic of its own:
 * it allocates the reference's NR-style arrays (util.c), sets the reference's
 * global scalars (globvar.h, compiled from the reference tree), and calls
 *   setup   matcopy_elastic/matcopy/matcopy_viscac, av_mue, av_rho, av_tau,
 *           prepare_update_s/_p, PML_pro, holbergcoeff (src/IFOS2D.c:773-943)
 *   forward update_v_PML(_SH), update_s_*_PML(_SH), update_p(_visc)_PML,
 *           psource, surface_*,
 *           seismo_ssg, snapshot store               (src/IFOS2D.c:1651-1894)
 *   adjoint the same kernels with sw=1 + zero-lag correlation
 *                                                    (src/IFOS2D.c:2224-2438)
 *   gradient assembly, PARAMETERIZATION 1 and 3      (src/IFOS2D.c:2471-2611)
 * The propagation kernels read PARAMETERIZATION from the globals themselves;
 * the assembly below follows the driver's branches for 1 and 3.
 */
#include "fd.h"
#include "globvar.h"
#include "ifos_oracle.h"

/* ---- globals the driver (IFOS2D.c) owns and kernels read through extern ---- */
static void set_globals(const orc_cfg *c) {
    static FILE *devnull = NULL;
    if (!devnull) devnull = fopen("/dev/null", "w");
    FP = devnull;
    NX = NXG = c->nx;
    NY = NYG = c->ny;
    NT = c->nt;
    DH = c->dh;
    DT = c->dt;
    FDORDER = c->fdorder;
    MAXRELERROR = c->maxrelerror;
    FW = c->fw;
    FREE_SURF = c->free_surf;
    BOUNDARY = c->boundary;
    VPPML = c->vppml;
    FPML = c->fpml;
    npower = c->npower;
    k_max_PML = c->k_max_pml;
    L = c->L;
    F_REF = c->f_ref;
    TAU = c->tau;
    WAVETYPE = c->wavetype;
    ACOUSTIC = c->acoustic;
    PARAMETERIZATION = c->parameterization;
    VELOCITY = c->velocity;
    SEISMO = c->seismo;
    SOURCE_TYPE = c->source_type;
    ADJOINT_TYPE = c->adjoint_type;
    NPROCX = NPROCY = 1;
    NPROC = 1;
    MYID = 0;
    POS[1] = POS[2] = 0;
    IENDX = NX;
    IENDY = NY;
    VERBOSE = 0;
    TRKILL = 0;
    TIMEWIN = 0;
    NORMALIZE = 0;
    NDT = 1;
    if (FL) { free_vector(FL, 1, ORC_MAX_L); FL = NULL; }
    FL = vector(1, ORC_MAX_L);
    for (int l = 1; l <= ORC_MAX_L; l++) FL[l] = c->fl[l - 1];
}

#define PLANE(p, k, nx, ny) ((p) + (size_t)(k) * (size_t)(nx) * (size_t)(ny))

static void put_plane(float *dst, float **m, int nx, int ny) {
    for (int j = 1; j <= ny; j++)
        for (int i = 1; i <= nx; i++) dst[(size_t)(j - 1) * nx + (i - 1)] = m[j][i];
}

int orc_fd_coeffs(const orc_cfg *c, float *hc7) {
    set_globals(c);
    float *hc = holbergcoeff();
    for (int i = 0; i <= 6; i++) hc7[i] = hc[i];
    free_vector(hc, 0, 6);
    return 0;
}

int orc_pml_profiles(const orc_cfg *c, float *out) {
    set_globals(c);
    int n = 2 * FW;
    float *a[20];
    for (int k = 0; k < 20; k++) a[k] = vector(1, n);
    PML_pro(a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7], a[8], a[9],
            a[10], a[11], a[12], a[13], a[14], a[15], a[16], a[17], a[18], a[19]);
    for (int k = 0; k < 20; k++) {
        for (int i = 1; i <= n; i++) out[(size_t)k * n + (i - 1)] = a[k][i];
        free_vector(a[k], 1, n);
    }
    return 0;
}

int orc_wavelet(const orc_cfg *c, int shape, int nsrc, const float *srcpos, float *signals) {
    set_globals(c);
    SOURCE_SHAPE = shape;
    float **sp = matrix(1, 8, 1, nsrc);
    for (int r = 1; r <= 8; r++)
        for (int l = 1; l <= nsrc; l++) sp[r][l] = srcpos[(size_t)(r - 1) * nsrc + (l - 1)];
    float **s = wavelet(sp, nsrc, 1, 0, 0);
    for (int l = 1; l <= nsrc; l++)
        for (int t = 1; t <= NT; t++) signals[(size_t)(l - 1) * NT + (t - 1)] = s[l][t];
    free_matrix(sp, 1, 8, 1, nsrc);
    return 0;
}

int orc_calc_res(const orc_cfg *c, int ntr, int ns, const float *obs, const float *syn,
                 float *diff, double *l2, double *energy, double *misfit) {
    set_globals(c);
    float **d = matrix(1, ntr, 1, ns), **s = matrix(1, ntr, 1, ns);
    float **df = matrix(1, ntr, 1, ns), **dfo = matrix(1, ntr, 1, ns);
    int **rl = imatrix(1, 3, 1, ntr);
    for (int i = 1; i <= ntr; i++) {
        rl[1][i] = rl[2][i] = 1;
        rl[3][i] = i;
        for (int j = 1; j <= ns; j++) {
            d[i][j] = obs[(size_t)(i - 1) * ns + (j - 1)];
            s[i][j] = syn[(size_t)(i - 1) * ns + (j - 1)];
        }
    }
    float **srcpos = matrix(1, 8, 1, 1);
    double L2 = calc_res(d, s, df, dfo, ntr, ns, 2, 0.0f, 0, 1, 1, ntr, rl, 1, 1, 1, srcpos, rl);
    double E = calc_energy(d, ntr, ns, 0.0f, ntr, rl, 1, 1, 1, srcpos, rl);
    double M = calc_misfit(d, s, ntr, ns, 2, 0.0f, 0, 1, 1, ntr, rl, 1, 1, 1, srcpos, rl);
    for (int i = 1; i <= ntr; i++)
        for (int j = 1; j <= ns; j++) diff[(size_t)(i - 1) * ns + (j - 1)] = df[i][j];
    *l2 = L2;
    *energy = E;
    *misfit = M;
    free_matrix(d, 1, ntr, 1, ns);
    free_matrix(s, 1, ntr, 1, ns);
    free_matrix(df, 1, ntr, 1, ns);
    free_matrix(dfo, 1, ntr, 1, ns);
    free_matrix(srcpos, 1, 8, 1, 1);
    free_imatrix(rl, 1, 3, 1, ntr);
    return 0;
}

int orc_run_shot(const orc_cfg *c, orc_shot_io *io) {
    set_globals(c);
    const int nd = FDORDER / 2 + 1;
    const int lo_y = -nd + 1, hi_y = NY + nd, lo_x = -nd + 1, hi_x = NX + nd;
#define MAT() matrix(lo_y, hi_y, lo_x, hi_x)
#define FREEMAT(m) free_matrix(m, lo_y, hi_y, lo_x, hi_x)
    const int psv = (WAVETYPE == 1 || WAVETYPE == 3);
    const int sh = (WAVETYPE == 2 || WAVETYPE == 3);
    const int ntdtinv = (int)ceil((float)NT / (float)c->dtinv);
    const int nsnap = NT / c->dtinv;  /* allocation depth, src/IFOS2D.c:541 */

    float *hc = holbergcoeff();

    /* model */
    float **prho = MAT(), **ppi = MAT(), **pu = MAT(), **prip = MAT(), **prjp = MAT();
    float **puipjp = MAT(), **ptaus = MAT(), **ptaup = MAT(), **ptausipjp = MAT();
    for (int j = 1; j <= NY; j++)
        for (int i = 1; i <= NX; i++) {
            size_t k = (size_t)(j - 1) * NX + (i - 1);
            prho[j][i] = io->rho[k];
            ppi[j][i] = io->vp[k];
            pu[j][i] = ACOUSTIC ? 0.0f : io->vs[k];
            ptaus[j][i] = io->taus ? io->taus[k] : TAU;
            ptaup[j][i] = io->taup ? io->taup[k] : TAU;
        }
    /* viscoelastic coefficient arrays */
    float ***pr = NULL, ***pp = NULL, ***pq = NULL, ***dip = NULL, ***d = NULL, ***e = NULL;
    float ***pt = NULL, ***po = NULL;
    float **fipjp = NULL, **f = NULL, **g = NULL;
    float *bip = NULL, *bjm = NULL, *cip = NULL, *cjm = NULL, *etajm = NULL, *etaip = NULL, *peta = NULL;
    if (L) {
        pr = f3tensor(lo_y, hi_y, lo_x, hi_x, 1, L);
        pp = f3tensor(lo_y, hi_y, lo_x, hi_x, 1, L);
        pq = f3tensor(lo_y, hi_y, lo_x, hi_x, 1, L);
        pt = f3tensor(lo_y, hi_y, lo_x, hi_x, 1, L);
        po = f3tensor(lo_y, hi_y, lo_x, hi_x, 1, L);
        dip = f3tensor(lo_y, hi_y, lo_x, hi_x, 1, L);
        d = f3tensor(lo_y, hi_y, lo_x, hi_x, 1, L);
        e = f3tensor(lo_y, hi_y, lo_x, hi_x, 1, L);
        fipjp = MAT();
        f = MAT();
        g = MAT();
        bip = vector(1, L);
        bjm = vector(1, L);
        cip = vector(1, L);
        cjm = vector(1, L);
        etajm = vector(1, L);
        etaip = vector(1, L);
        peta = vector(1, L);
        /* eta as readmod computes it (src/readmod.c:44-49) */
        for (int l = 1; l <= L; l++) {
            float pts = 1.0 / (2.0 * PI * FL[l]);
            peta[l] = DT / pts;
        }
    }

    /* material ghost ring + averages (src/IFOS2D.c:906-943) */
    if (L && !ACOUSTIC) matcopy(prho, ppi, pu, ptaus, ptaup);
    else if (L) matcopy_viscac(prho, ppi, ptaup);
    else matcopy_elastic(prho, ppi, pu);
    if (!ACOUSTIC) av_mue(pu, puipjp, prho);
    av_rho(prho, prip, prjp);
    if (!ACOUSTIC && L) av_tau(ptaus, ptausipjp);
    if (L && !ACOUSTIC)
        prepare_update_s(etajm, etaip, peta, fipjp, pu, puipjp, ppi, prho, ptaus, ptaup, ptausipjp, f, g,
                         bip, bjm, cip, cjm, dip, d, e);
    else if (L)
        prepare_update_p(etajm, peta, ppi, prho, ptaup, g, bjm, cjm, e);

    /* CPML profiles (src/IFOS2D.c:816) */
    int n2 = 2 * FW > 0 ? 2 * FW : 1;
    float *d_x = vector(1, n2), *K_x = vector(1, n2), *alpha_prime_x = vector(1, n2), *a_x = vector(1, n2),
          *b_x = vector(1, n2);
    float *d_x_half = vector(1, n2), *K_x_half = vector(1, n2), *alpha_prime_x_half = vector(1, n2),
          *a_x_half = vector(1, n2), *b_x_half = vector(1, n2);
    float *d_y = vector(1, n2), *K_y = vector(1, n2), *alpha_prime_y = vector(1, n2), *a_y = vector(1, n2),
          *b_y = vector(1, n2);
    float *d_y_half = vector(1, n2), *K_y_half = vector(1, n2), *alpha_prime_y_half = vector(1, n2),
          *a_y_half = vector(1, n2), *b_y_half = vector(1, n2);
    PML_pro(d_x, K_x, alpha_prime_x, a_x, b_x, d_x_half, K_x_half, alpha_prime_x_half, a_x_half, b_x_half,
            d_y, K_y, alpha_prime_y, a_y, b_y, d_y_half, K_y_half, alpha_prime_y_half, a_y_half, b_y_half);

    float **psi_sxx_x = matrix(1, NY, 1, n2), **psi_syy_y = matrix(1, n2, 1, NX);
    float **psi_sxy_y = matrix(1, n2, 1, NX), **psi_sxy_x = matrix(1, NY, 1, n2);
    float **psi_vxx = matrix(1, NY, 1, n2), **psi_vxxs = matrix(1, NY, 1, n2);
    float **psi_vyy = matrix(1, n2, 1, NX), **psi_vxy = matrix(1, n2, 1, NX);
    float **psi_vyx = matrix(1, NY, 1, n2);
    float **psi_sxz_x = matrix(1, NY, 1, n2), **psi_syz_y = matrix(1, n2, 1, NX);
    float **psi_vzx = matrix(1, NY, 1, n2), **psi_vzy = matrix(1, n2, 1, NX);

    /* wavefields */
    float **pvx = MAT(), **pvy = MAT(), **pvxp1 = MAT(), **pvyp1 = MAT(), **pvxm1 = MAT(), **pvym1 = MAT();
    float **psxx = MAT(), **psyy = MAT(), **psxy = MAT(), **psp = MAT();
    float **pvz = MAT(), **pvzp1 = MAT(), **pvzm1 = MAT(), **psxz = MAT(), **psyz = MAT();
    float **ux = MAT(), **uy = MAT(), **uxy = MAT(), **uyx = MAT(), **uttx = MAT(), **utty = MAT();
    float **uxz = MAT(), **uyz = MAT(), **absorb_coeff = MAT(), **u_ac = MAT();

    /* sources: srcpos_loc rows 1..8 */
    int nsrc = io->nsrc;
    float **srcpos_loc = matrix(1, 8, 1, nsrc > 0 ? nsrc : 1);
    float **signals = matrix(1, nsrc > 0 ? nsrc : 1, 1, NT);
    for (int l = 1; l <= nsrc; l++) {
        for (int r = 1; r <= 8; r++) srcpos_loc[r][l] = io->srcpos[(size_t)(r - 1) * nsrc + (l - 1)];
        for (int t = 1; t <= NT; t++) signals[l][t] = io->signals[(size_t)(l - 1) * NT + (t - 1)];
    }
    /* receivers */
    int ntr = io->ntr;
    int ntr1 = ntr > 0 ? ntr : 1;
    int **recpos_loc = imatrix(1, 3, 1, ntr1);
    for (int i = 1; i <= ntr; i++) {
        recpos_loc[1][i] = io->recpos[i - 1];
        recpos_loc[2][i] = io->recpos[ntr + i - 1];
        recpos_loc[3][i] = i;
    }
    float **sectionvx = matrix(1, ntr1, 1, NT), **sectionvy = matrix(1, ntr1, 1, NT);
    float **sectionvz = matrix(1, ntr1, 1, NT), **sectionp = matrix(1, ntr1, 1, NT);
    float **sectioncurl = matrix(1, ntr1, 1, NT), **sectiondiv = matrix(1, ntr1, 1, NT);

    /* snapshots (src/IFOS2D.c:534-591) */
    float ***fw_x = NULL, ***fw_y = NULL, ***fw_u = NULL, ***fw_p = NULL, ***fw_rx = NULL, ***fw_ry = NULL;
    float ***fw_rz = NULL, ***fw_xz = NULL, ***fw_yz = NULL;
    int nsl = nsnap > 0 ? nsnap : 1;
    if (io->run_adjoint) {
        if (psv) {
            fw_rx = f3tensor(lo_y, hi_y, lo_x, hi_x, 1, nsl);
            fw_ry = f3tensor(lo_y, hi_y, lo_x, hi_x, 1, nsl);
            if (!ACOUSTIC) {
                fw_x = f3tensor(lo_y, hi_y, lo_x, hi_x, 1, nsl);
                fw_y = f3tensor(lo_y, hi_y, lo_x, hi_x, 1, nsl);
                fw_u = f3tensor(lo_y, hi_y, lo_x, hi_x, 1, nsl);
            } else {
                fw_p = f3tensor(lo_y, hi_y, lo_x, hi_x, 1, nsl);
            }
        }
        if (sh) {
            fw_rz = f3tensor(lo_y, hi_y, lo_x, hi_x, 1, nsl);
            fw_xz = f3tensor(lo_y, hi_y, lo_x, hi_x, 1, nsl);
            fw_yz = f3tensor(lo_y, hi_y, lo_x, hi_x, 1, nsl);
        }
    }
    int *DTINV_help = ivector(1, NT);

    /* ------------------------- forward (src/IFOS2D.c:1651-1894) ------------------------- */
    int hin = 1, hin1 = 1;
    int nsteps = io->nsteps > 0 && io->nsteps <= NT ? io->nsteps : NT;
    for (int nt = 1; nt <= nsteps; nt++) {
        if (!ACOUSTIC) {
            if (psv)
                update_v_PML(1, NX, 1, NY, nt, pvx, pvxp1, pvxm1, pvy, pvyp1, pvym1, uttx, utty, psxx, psyy, psxy,
                             prip, prjp, srcpos_loc, signals, signals, nsrc, absorb_coeff, hc, 0, 0, K_x, a_x, b_x,
                             K_x_half, a_x_half, b_x_half, K_y, a_y, b_y, K_y_half, a_y_half, b_y_half, psi_sxx_x,
                             psi_syy_y, psi_sxy_y, psi_sxy_x);
            if (sh)
                update_v_PML_SH(1, NX, 1, NY, nt, pvz, pvzp1, pvzm1, psxz, psyz, prjp, srcpos_loc, signals, signals,
                                nsrc, absorb_coeff, hc, 0, 0, K_x, a_x, b_x, K_x_half, a_x_half, b_x_half, K_y, a_y,
                                b_y, K_y_half, a_y_half, b_y_half, psi_sxz_x, psi_syz_y);
        } else {
            update_v_acoustic_PML(1, NX, 1, NY, nt, pvx, pvxp1, pvxm1, pvy, pvyp1, pvym1, psp, prip, prjp,
                                  srcpos_loc, signals, signals, nsrc, absorb_coeff, hc, 0, 0, K_x_half, a_x_half,
                                  b_x_half, K_y_half, a_y_half, b_y_half, psi_sxx_x, psi_syy_y);
        }
        if (L) {
            if (psv && !ACOUSTIC)
                update_s_visc_PML(1, NX, 1, NY, pvx, pvy, ux, uy, uxy, uyx, psxx, psyy, psxy, ppi, pu, puipjp, prho,
                                  hc, 0, pr, pp, pq, fipjp, f, g, bip, bjm, cip, cjm, d, e, dip, K_x, a_x, b_x,
                                  K_x_half, a_x_half, b_x_half, K_y, a_y, b_y, K_y_half, a_y_half, b_y_half, psi_vxx,
                                  psi_vyy, psi_vxy, psi_vyx);
            if (psv && ACOUSTIC)
                update_p_visc_PML(1, NX, 1, NY, pvx, pvy, psp, ppi, prho, hc, 0, pp, g, bjm, cjm, e, K_x, a_x, b_x,
                                  K_x_half, a_x_half, b_x_half, K_y, a_y, b_y, K_y_half, a_y_half, b_y_half, psi_vxx,
                                  psi_vyy, psi_vxy, psi_vyx);
            if (sh)
                update_s_visc_PML_SH(1, NX, 1, NY, pvz, psxz, psyz, pt, po, bip, bjm, cip, cjm, d, dip, fipjp, f, hc,
                                     0, K_x, a_x, b_x, K_x_half, a_x_half, b_x_half, K_y, a_y, b_y, K_y_half,
                                     a_y_half, b_y_half, psi_vzx, psi_vzy);
        } else {
            if (psv) {
                if (!ACOUSTIC)
                    update_s_elastic_PML(1, NX, 1, NY, pvx, pvy, ux, uy, uxy, uyx, psxx, psyy, psxy, ppi, pu, puipjp,
                                         absorb_coeff, prho, hc, 0, K_x, a_x, b_x, K_x_half, a_x_half, b_x_half, K_y,
                                         a_y, b_y, K_y_half, a_y_half, b_y_half, psi_vxx, psi_vyy, psi_vxy, psi_vyx);
                else
                    update_p_PML(1, NX, 1, NY, pvx, pvy, psp, u_ac, ppi, absorb_coeff, prho, hc, 0, K_x, a_x, b_x,
                                 K_x_half, a_x_half, b_x_half, K_y, a_y, b_y, K_y_half, a_y_half, b_y_half, psi_vxx,
                                 psi_vyy, psi_vxy, psi_vyx);
            }
            if (sh)
                update_s_elastic_PML_SH(1, NX, 1, NY, pvz, psxz, psyz, uxz, uyz, hc, 0, K_x, a_x, b_x, K_x_half,
                                        a_x_half, b_x_half, K_y, a_y, b_y, K_y_half, a_y_half, b_y_half, psi_vzx,
                                        psi_vzy, puipjp, pu, prho);
        }
        if ((SOURCE_TYPE == 1) && psv) psource(nt, psxx, psyy, psp, srcpos_loc, signals, nsrc, 0);
        if (FREE_SURF) {
            if (!ACOUSTIC) {
                if (L)
                    surface_PML(1, pvx, pvy, psxx, psyy, psxy, psyz, pp, pq, ppi, pu, prho, ptaup, ptaus, etajm, peta,
                                hc, K_x, a_x, b_x, psi_vxxs, ux, uy, uxy, uyz, psxz, uxz);
                else
                    surface_elastic_PML(1, pvx, pvy, psxx, psyy, psxy, psyz, ppi, pu, prho, hc, K_x, a_x, b_x,
                                        psi_vxxs, ux, uy, uxy, uyz, psxz, uxz);
            } else {
                surface_acoustic_PML(1, psp);
            }
        }
        if (SEISMO)
            seismo_ssg(nt, ntr, recpos_loc, sectionvx, sectionvy, sectionvz, sectionp, sectioncurl, sectiondiv, pvx,
                       pvy, pvz, psxx, psyy, psp, ppi, pu, hc);
        if (nt == hin1) {
            if (io->run_adjoint) {
                for (int j = 1; j <= NY; j++)
                    for (int i = 1; i <= NX; i++) {
                        if (psv) {
                            fw_rx[j][i][hin] = pvxp1[j][i];
                            fw_ry[j][i][hin] = pvyp1[j][i];
                            if (!ACOUSTIC) {
                                fw_x[j][i][hin] = psxx[j][i];
                                fw_y[j][i][hin] = psyy[j][i];
                                fw_u[j][i][hin] = psxy[j][i];
                            } else {
                                fw_p[j][i][hin] = psp[j][i];
                            }
                        }
                        if (sh) {
                            fw_rz[j][i][hin] = pvzp1[j][i];
                            fw_xz[j][i][hin] = psxz[j][i];
                            fw_yz[j][i][hin] = psyz[j][i];
                        }
                    }
                hin++;
                hin1 = hin1 + c->dtinv;
            }
            DTINV_help[nt] = 1;
        }
    }
    if (io->sections) {
        float **secs[ORC_NS] = {sectionvx, sectionvy, sectionvz, sectionp, sectioncurl, sectiondiv};
        for (int k = 0; k < ORC_NS; k++)
            for (int i = 1; i <= ntr; i++)
                for (int t = 1; t <= NT; t++)
                    io->sections[((size_t)k * ntr + (i - 1)) * NT + (t - 1)] = secs[k][i][t];
    }
    float **fl[ORC_NF] = {pvx, pvy, psxx, psyy, psxy, pvxp1, pvyp1, pvz, psxz, psyz, pvzp1, psp};
    if (io->fields)
        for (int k = 0; k < ORC_NF; k++) put_plane(PLANE(io->fields, k, NX, NY), fl[k], NX, NY);

    /* ------------------------- adjoint (src/IFOS2D.c:2156-2438) ------------------------- */
    if (io->run_adjoint) {
        float **wc_shot = MAT(), **wc_rho_shot = MAT(), **wc_u_shot = MAT();
        float **wc_rho_z = MAT(), **wc_u_z = MAT();
        float **diffx = matrix(1, ntr1, 1, NT), **diffy = matrix(1, ntr1, 1, NT), **diffz = matrix(1, ntr1, 1, NT);
        for (int i = 1; i <= ntr; i++)
            for (int t = 1; t <= NT; t++) {
                diffx[i][t] = io->adj[((size_t)0 * ntr + (i - 1)) * NT + (t - 1)];
                diffy[i][t] = io->adj[((size_t)1 * ntr + (i - 1)) * NT + (t - 1)];
                diffz[i][t] = io->adj[((size_t)2 * ntr + (i - 1)) * NT + (t - 1)];
            }
        float **srcpos_loc_back = matrix(1, 6, 1, ntr1);
        for (int i = 1; i <= ntr; i++) {
            srcpos_loc_back[1][i] = recpos_loc[1][i];
            srcpos_loc_back[2][i] = recpos_loc[2][i];
        }
        /* zero wavefields (src/IFOS2D.c:2193-2213) */
        if (L && ACOUSTIC)
            zero_fdveps_viscac(-nd + 1, NY + nd, -nd + 1, NX + nd, pvx, pvy, psp, pvxp1, pvyp1, psi_sxx_x, psi_sxy_x,
                               psi_vxx, psi_vyx, psi_syy_y, psi_sxy_y, psi_vyy, psi_vxy, psi_vxxs, pp);
        else if (L)
            zero_fdveps_visc(-nd + 1, NY + nd, -nd + 1, NX + nd, pvx, pvy, pvz, psxx, psyy, psxy, psxz, psyz, ux, uy,
                             uxy, pvxp1, pvyp1, psi_sxx_x, psi_sxy_x, psi_sxz_x, psi_vxx, psi_vyx, psi_vzx, psi_syy_y,
                             psi_sxy_y, psi_syz_y, psi_vyy, psi_vxy, psi_vzy, psi_vxxs, pr, pp, pq, pt, po);
        else if (!ACOUSTIC)
            zero_fdveps(-nd + 1, NY + nd, -nd + 1, NX + nd, pvx, pvy, pvz, psxx, psyy, psxy, psxz, psyz, ux, uy, uxy,
                        pvxp1, pvyp1, psi_sxx_x, psi_sxy_x, psi_sxz_x, psi_vxx, psi_vyx, psi_vzx, psi_syy_y,
                        psi_sxy_y, psi_syz_y, psi_vyy, psi_vxy, psi_vzy, psi_vxxs);
        else
            zero_fdveps_ac(-nd + 1, NY + nd, -nd + 1, NX + nd, pvx, pvy, psp, pvxp1, pvyp1, psi_sxx_x, psi_sxy_x,
                           psi_vxx, psi_vyx, psi_syy_y, psi_sxy_y, psi_vyy, psi_vxy, psi_vxxs);
        int hin_a = 1;
        for (int nt = 1; nt <= NT; nt++) {
            if (!ACOUSTIC) {
                if (psv)
                    update_v_PML(1, NX, 1, NY, nt, pvx, pvxp1, pvxm1, pvy, pvyp1, pvym1, uttx, utty, psxx, psyy, psxy,
                                 prip, prjp, srcpos_loc_back, diffx, diffy, ntr, absorb_coeff, hc, 0, 1, K_x, a_x,
                                 b_x, K_x_half, a_x_half, b_x_half, K_y, a_y, b_y, K_y_half, a_y_half, b_y_half,
                                 psi_sxx_x, psi_syy_y, psi_sxy_y, psi_sxy_x);
                if (sh)
                    update_v_PML_SH(1, NX, 1, NY, nt, pvz, pvzp1, pvzm1, psxz, psyz, prjp, srcpos_loc_back, diffz,
                                    diffz, ntr, absorb_coeff, hc, 0, 1, K_x, a_x, b_x, K_x_half, a_x_half, b_x_half,
                                    K_y, a_y, b_y, K_y_half, a_y_half, b_y_half, psi_sxz_x, psi_syz_y);
            } else {
                update_v_acoustic_PML(1, NX, 1, NY, nt, pvx, pvxp1, pvxm1, pvy, pvyp1, pvym1, psp, prip, prjp,
                                      srcpos_loc_back, diffx, diffy, ntr, absorb_coeff, hc, 0, 1, K_x_half, a_x_half,
                                      b_x_half, K_y_half, a_y_half, b_y_half, psi_sxx_x, psi_syy_y);
            }
            if (L) {
                if (psv && !ACOUSTIC)
                    update_s_visc_PML(1, NX, 1, NY, pvx, pvy, ux, uy, uxy, uyx, psxx, psyy, psxy, ppi, pu, puipjp,
                                      prho, hc, 0, pr, pp, pq, fipjp, f, g, bip, bjm, cip, cjm, d, e, dip, K_x, a_x,
                                      b_x, K_x_half, a_x_half, b_x_half, K_y, a_y, b_y, K_y_half, a_y_half, b_y_half,
                                      psi_vxx, psi_vyy, psi_vxy, psi_vyx);
                if (psv && ACOUSTIC)
                    update_p_visc_PML(1, NX, 1, NY, pvx, pvy, psp, ppi, prho, hc, 0, pp, g, bjm, cjm, e, K_x, a_x,
                                      b_x, K_x_half, a_x_half, b_x_half, K_y, a_y, b_y, K_y_half, a_y_half, b_y_half,
                                      psi_vxx, psi_vyy, psi_vxy, psi_vyx);
                if (sh)
                    update_s_visc_PML_SH(1, NX, 1, NY, pvz, psxz, psyz, pt, po, bip, bjm, cip, cjm, d, dip, fipjp, f,
                                         hc, 0, K_x, a_x, b_x, K_x_half, a_x_half, b_x_half, K_y, a_y, b_y, K_y_half,
                                         a_y_half, b_y_half, psi_vzx, psi_vzy);
            } else {
                if (!ACOUSTIC) {
                    if (psv)
                        update_s_elastic_PML(1, NX, 1, NY, pvx, pvy, ux, uy, uxy, uyx, psxx, psyy, psxy, ppi, pu,
                                             puipjp, absorb_coeff, prho, hc, 0, K_x, a_x, b_x, K_x_half, a_x_half,
                                             b_x_half, K_y, a_y, b_y, K_y_half, a_y_half, b_y_half, psi_vxx, psi_vyy,
                                             psi_vxy, psi_vyx);
                    if (sh)
                        update_s_elastic_PML_SH(1, NX, 1, NY, pvz, psxz, psyz, uxz, uyz, hc, 0, K_x, a_x, b_x,
                                                K_x_half, a_x_half, b_x_half, K_y, a_y, b_y, K_y_half, a_y_half,
                                                b_y_half, psi_vzx, psi_vzy, puipjp, pu, prho);
                } else {
                    update_p_PML(1, NX, 1, NY, pvx, pvy, psp, u_ac, ppi, absorb_coeff, prho, hc, 0, K_x, a_x, b_x,
                                 K_x_half, a_x_half, b_x_half, K_y, a_y, b_y, K_y_half, a_y_half, b_y_half, psi_vxx,
                                 psi_vyy, psi_vxy, psi_vyx);
                }
            }
            if (ADJOINT_TYPE == 4) psource(nt, psxx, psyy, psp, srcpos_loc_back, diffz, ntr, 1);
            if (FREE_SURF) {
                if (!ACOUSTIC) {
                    if (L)
                        surface_PML(1, pvx, pvy, psxx, psyy, psxy, psyz, pp, pq, ppi, pu, prho, ptaup, ptaus, etajm,
                                    peta, hc, K_x, a_x, b_x, psi_vxxs, ux, uy, uxy, uyz, psxz, uxz);
                    else
                        surface_elastic_PML(1, pvx, pvy, psxx, psyy, psxy, psyz, ppi, pu, prho, hc, K_x, a_x, b_x,
                                            psi_vxxs, ux, uy, uxy, uyz, psxz, uxz);
                } else {
                    surface_acoustic_PML(1, psp);
                }
            }
            /* zero-lag correlation (src/IFOS2D.c:2379-2419) */
            if (DTINV_help[NT - nt + 1] == 1) {
                int s = ntdtinv - hin_a + 1;
                for (int j = 1; j <= NY; j++)
                    for (int i = 1; i <= NX; i++) {
                        if (psv) {
                            wc_rho_shot[j][i] += (pvxp1[j][i] * fw_rx[j][i][s]) + (pvyp1[j][i] * fw_ry[j][i][s]);
                            if (!ACOUSTIC)
                                wc_shot[j][i] += (fw_x[j][i][s] + fw_y[j][i][s]) * (psxx[j][i] + psyy[j][i]);
                            else
                                wc_shot[j][i] += (fw_p[j][i][s]) * (psp[j][i]);
                            if (!ACOUSTIC) {
                                float muss = prho[j][i] * pu[j][i] * pu[j][i];
                                float lamss = prho[j][i] * ppi[j][i] * ppi[j][i] - 2.0 * muss;
                                if (pu[j][i] > 0.0) {
                                    wc_u_shot[j][i] +=
                                        ((1.0 / (muss * muss)) * (fw_u[j][i][s] * psxy[j][i])) +
                                        (.25 * (fw_x[j][i][s] + fw_y[j][i][s] * (psxx[j][i] + psyy[j][i])) /
                                         ((lamss + muss) * (lamss + muss))) +
                                        (.25 * (fw_x[j][i][s] - fw_y[j][i][s] * (psxx[j][i] - psyy[j][i])) /
                                         (muss * muss));
                                }
                            }
                        }
                        if (sh) {
                            wc_rho_z[j][i] += pvzp1[j][i] * fw_rz[j][i][s];
                            float muss = prho[j][i] * pu[j][i] * pu[j][i];
                            wc_u_z[j][i] += (1.0 / (muss * muss)) *
                                            (fw_xz[j][i][s] * psxz[j][i] + fw_yz[j][i][s] * psyz[j][i]);
                        }
                    }
                hin_a++;
            }
        }
        if (io->adj_fields)
            for (int k = 0; k < ORC_NF; k++) put_plane(PLANE(io->adj_fields, k, NX, NY), fl[k], NX, NY);

        /* gradient assembly (src/IFOS2D.c:2471-2611); PARAMETERIZATION 3 keeps
           each -DT-scaled sum (:2498-2500, :2527-2530, :2551-2554, :2581-2584, :2605-2608) */
        if (io->grads) {
            float **lam = MAT(), **mu = MAT(), **rho_s = MAT(), **mu_z = MAT(), **rho_s_z = MAT();
            put_plane(PLANE(io->grads, ORC_G_LAM_RAW, NX, NY), wc_shot, NX, NY);
            put_plane(PLANE(io->grads, ORC_G_MU_RAW, NX, NY), wc_u_shot, NX, NY);
            put_plane(PLANE(io->grads, ORC_G_RHO_RAW, NX, NY), wc_rho_shot, NX, NY);
            put_plane(PLANE(io->grads, ORC_G_MU_Z_RAW, NX, NY), wc_u_z, NX, NY);
            put_plane(PLANE(io->grads, ORC_G_RHO_Z_RAW, NX, NY), wc_rho_z, NX, NY);
            if (psv) {
                for (int j = 1; j <= NY; j++)
                    for (int i = 1; i <= NX; i++) {
                        lam[j][i] = -DT * wc_shot[j][i];
                        if (PARAMETERIZATION == 3) {
                            wc_shot[j][i] = lam[j][i];
                            continue;
                        }
                        float muss = !ACOUSTIC ? prho[j][i] * pu[j][i] * pu[j][i] : 0;
                        float lamss = prho[j][i] * ppi[j][i] * ppi[j][i] - 2.0 * muss;
                        if (!ACOUSTIC)
                            lam[j][i] = (1.0 / (4.0 * (lamss + muss) * (lamss + muss))) * lam[j][i];
                        else
                            lam[j][i] = (1.0 / ((lamss + muss) * (lamss + muss))) * lam[j][i];
                        wc_shot[j][i] = 2.0 * ppi[j][i] * prho[j][i] * lam[j][i];
                    }
                if (!ACOUSTIC)
                    for (int j = 1; j <= NY; j++)
                        for (int i = 1; i <= NX; i++) {
                            mu[j][i] = -DT * wc_u_shot[j][i];
                            if (PARAMETERIZATION == 3)
                                wc_u_shot[j][i] = mu[j][i];
                            else
                                wc_u_shot[j][i] = -4.0 * prho[j][i] * pu[j][i] * lam[j][i] +
                                                  2.0 * prho[j][i] * pu[j][i] * mu[j][i];
                        }
                for (int j = 1; j <= NY; j++)
                    for (int i = 1; i <= NX; i++) {
                        rho_s[j][i] = -DT * wc_rho_shot[j][i];
                        if (PARAMETERIZATION == 3)
                            wc_rho_shot[j][i] = rho_s[j][i];
                        else if (!ACOUSTIC)
                            wc_rho_shot[j][i] = ((ppi[j][i] * ppi[j][i]) - (2.0 * pu[j][i] * pu[j][i])) * lam[j][i] +
                                                pu[j][i] * pu[j][i] * mu[j][i] + rho_s[j][i];
                        else
                            wc_rho_shot[j][i] = ((ppi[j][i] * ppi[j][i]) * lam[j][i]) + rho_s[j][i];
                    }
            }
            if (sh && !ACOUSTIC) {
                for (int j = 1; j <= NY; j++)
                    for (int i = 1; i <= NX; i++) {
                        mu_z[j][i] = -DT * wc_u_z[j][i];
                        wc_u_z[j][i] = PARAMETERIZATION == 3 ? mu_z[j][i] : (2.0 * prho[j][i] * pu[j][i] * mu_z[j][i]);
                    }
                for (int j = 1; j <= NY; j++)
                    for (int i = 1; i <= NX; i++) {
                        rho_s_z[j][i] = -DT * wc_rho_z[j][i];
                        wc_rho_z[j][i] = PARAMETERIZATION == 3 ? rho_s_z[j][i]
                                                               : ((pu[j][i] * pu[j][i] * mu_z[j][i]) + rho_s_z[j][i]);
                    }
            }
            put_plane(PLANE(io->grads, ORC_G_VP, NX, NY), wc_shot, NX, NY);
            put_plane(PLANE(io->grads, ORC_G_VS, NX, NY), wc_u_shot, NX, NY);
            put_plane(PLANE(io->grads, ORC_G_RHO, NX, NY), wc_rho_shot, NX, NY);
            put_plane(PLANE(io->grads, ORC_G_VS_Z, NX, NY), wc_u_z, NX, NY);
            put_plane(PLANE(io->grads, ORC_G_RHO_Z, NX, NY), wc_rho_z, NX, NY);
            FREEMAT(lam); FREEMAT(mu); FREEMAT(rho_s); FREEMAT(mu_z); FREEMAT(rho_s_z);
        }
        FREEMAT(wc_shot); FREEMAT(wc_rho_shot); FREEMAT(wc_u_shot); FREEMAT(wc_rho_z); FREEMAT(wc_u_z);
        free_matrix(diffx, 1, ntr1, 1, NT);
        free_matrix(diffy, 1, ntr1, 1, NT);
        free_matrix(diffz, 1, ntr1, 1, NT);
        free_matrix(srcpos_loc_back, 1, 6, 1, ntr1);
    }

    /* release (leaks of the few vectors are harmless in a test process, but free the big ones) */
    if (io->run_adjoint) {
        float ***snaps[9] = {fw_x, fw_y, fw_u, fw_p, fw_rx, fw_ry, fw_rz, fw_xz, fw_yz};
        for (int k = 0; k < 9; k++)
            if (snaps[k]) free_f3tensor(snaps[k], lo_y, hi_y, lo_x, hi_x, 1, nsl);
    }
    float **all[] = {prho, ppi, pu, prip, prjp, puipjp, ptaus, ptaup, ptausipjp, pvx, pvy, pvxp1, pvyp1, pvxm1, pvym1,
                     psxx, psyy, psxy, psp, pvz, pvzp1, pvzm1, psxz, psyz, ux, uy, uxy, uyx, uttx, utty, uxz, uyz,
                     absorb_coeff, u_ac};
    for (size_t k = 0; k < sizeof(all) / sizeof(all[0]); k++) FREEMAT(all[k]);
    if (L) {
        float ***t3[] = {pr, pp, pq, pt, po, dip, d, e};
        for (size_t k = 0; k < sizeof(t3) / sizeof(t3[0]); k++) free_f3tensor(t3[k], lo_y, hi_y, lo_x, hi_x, 1, L);
        FREEMAT(fipjp); FREEMAT(f); FREEMAT(g);
    }
    free_matrix(sectionvx, 1, ntr1, 1, NT);
    free_matrix(sectionvy, 1, ntr1, 1, NT);
    free_matrix(sectionvz, 1, ntr1, 1, NT);
    free_matrix(sectionp, 1, ntr1, 1, NT);
    free_matrix(sectioncurl, 1, ntr1, 1, NT);
    free_matrix(sectiondiv, 1, ntr1, 1, NT);
    free_matrix(srcpos_loc, 1, 8, 1, nsrc > 0 ? nsrc : 1);
    free_matrix(signals, 1, nsrc > 0 ? nsrc : 1, 1, NT);
    free_imatrix(recpos_loc, 1, 3, 1, ntr1);
    free_ivector(DTINV_help, 1, NT);
    free_vector(hc, 0, 6);
    return 0;
#undef MAT
#undef FREEMAT
}
