/*
 * ifos_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * One C interface implemented twice:
 *   - oracle/_ref/libifosref.so : the reference's own kernel sources
 *     (the IFOS2D src directory) compiled in place and driven in the order of the
 *     reference driver's shot loop (src/IFOS2D.c:1651-1894 forward,
 *     :2224-2438 adjoint, :2471-2611 gradient assembly);
 *   - oracle/liboracle.so        : a from-scratch plain-C restatement of the
 *     same algorithm (oracle/restate/ifos_restate.c).
 * Tests use them as checkers for the CUDA path.  Nothing in the product links,
 * loads or calls either library.
 *
 * Layout conventions (both implementations):
 *   model / gradient / field planes are NY x NX, row-major, x (i) fastest,
 *   element (j,i) of the reference's 1-based grid at [(j-1)*NX + (i-1)];
 *   seismogram planes are ntr x NT, sample nt (1-based) at [itr*NT + nt-1].
 */
#ifndef IFOS_ORACLE_H
#define IFOS_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_MAX_L 8

typedef struct orc_cfg {
    int nx, ny, nt;
    float dh, dt;
    int fdorder, maxrelerror;
    int fw, free_surf, boundary;
    float vppml, fpml, npower, k_max_pml;
    int L;                 /* relaxation mechanisms, 0 = elastic */
    float f_ref, tau;
    float fl[ORC_MAX_L];
    int wavetype;          /* 1 P-SV, 2 SH, 3 both */
    int acoustic;
    int parameterization;  /* 1: vp, vs, rho; 3: lambda, mu, rho (compiled reference only) */
    int velocity;          /* 0: displacement-type snapshots (stress) */
    int seismo;            /* 1..5 */
    int source_type;       /* forward source mechanism: 1 explosive, 2/3 force x/y, 4 rotated */
    int adjoint_type;      /* 1 vx+vy, 2 vy, 3 vx, 4 p */
    int dtinv;
    int hi_order_corrected;/* restatement only: 1 = FDORDER 10/12 P-SV and
                              acoustic branches use the CPML form of orders
                              2-8; 0 = the reference's own 10/12 branches
                              (src/update_v_PML.c:466-528,
                              src/update_s_elastic_PML.c:442-535).  The
                              reference library always behaves as 0. */
} orc_cfg;

/* Field planes written to orc_shot_io.fields / adj_fields, in this order. */
enum {
    ORC_F_VX = 0, ORC_F_VY, ORC_F_SXX, ORC_F_SYY, ORC_F_SXY, ORC_F_VXP1, ORC_F_VYP1,
    ORC_F_VZ, ORC_F_SXZ, ORC_F_SYZ, ORC_F_VZP1, ORC_F_SP, ORC_NF
};
/* Seismogram planes written to orc_shot_io.sections, in this order. */
enum { ORC_S_VX = 0, ORC_S_VY, ORC_S_VZ, ORC_S_P, ORC_S_CURL, ORC_S_DIV, ORC_NS };
/* Gradient planes written to orc_shot_io.grads, in this order:
 * raw zero-lag correlations (before the -DT scaling), then the per-shot
 * assembled gradients of the reference (PARAMETERIZATION=1). */
enum {
    ORC_G_LAM_RAW = 0,  /* waveconv_shot    (src/IFOS2D.c:2390) */
    ORC_G_MU_RAW,       /* waveconv_u_shot  (src/IFOS2D.c:2398) */
    ORC_G_RHO_RAW,      /* waveconv_rho_shot(src/IFOS2D.c:2385) */
    ORC_G_VP,           /* waveconv_shot after assembly (src/IFOS2D.c:2491) */
    ORC_G_VS,           /* waveconv_u_shot after assembly (src/IFOS2D.c:2520) */
    ORC_G_RHO,          /* waveconv_rho_shot after assembly (src/IFOS2D.c:2580) */
    ORC_G_MU_Z_RAW,     /* waveconv_u_shot_z   (src/IFOS2D.c:2412) */
    ORC_G_RHO_Z_RAW,    /* waveconv_rho_shot_z (src/IFOS2D.c:2410) */
    ORC_G_VS_Z,         /* SH vs gradient (src/IFOS2D.c:2549) */
    ORC_G_RHO_Z,        /* SH rho gradient (src/IFOS2D.c:2600) */
    ORC_NG
};

typedef struct orc_shot_io {
    /* model planes NY*NX; taup/taus may be NULL (then TAU everywhere) */
    const float *vp, *vs, *rho, *taup, *taus;
    /* sources: 8*nsrc floats laid out like the reference's srcpos_loc rows
     * 1..8 (x, y in grid points, 0, tshift, fc, amp, azimuth, type) */
    int nsrc;
    const float *srcpos;
    const float *signals;     /* nsrc*NT source signals (forward) */
    int ntr;
    const int *recpos;        /* 2*ntr: grid x (1-based) row, then grid y row */
    int nsteps;               /* forward steps to run, 1..NT */
    float *sections;          /* ORC_NS planes ntr*NT, or NULL */
    float *fields;            /* ORC_NF planes after the forward loop, or NULL */
    int run_adjoint;          /* 1: adjoint loop over NT steps + gradients */
    const float *adj;         /* 3 planes ntr*NT: adjoint sources for vx, vy,
                                 and vz (SH) or p (ADJOINT_TYPE 4); these are
                                 the time-reversed residual sections the
                                 reference passes to update_v_PML(sw=1) */
    float *grads;             /* ORC_NG planes, or NULL */
    float *adj_fields;        /* ORC_NF planes after the adjoint loop, or NULL */
} orc_shot_io;

/* Run one shot.  Returns 0 on success. */
int orc_run_shot(const orc_cfg *cfg, orc_shot_io *io);

/* CPML profiles, 6 arrays of 2*FW floats each per direction, in the order
 * d, K, alpha', a, b for integer nodes then half nodes; x then y
 * (20 arrays * 2FW).  Matches PML_pro (src/PML_pro.c:83-316). */
int orc_pml_profiles(const orc_cfg *cfg, float *out);

/* FD coefficients hc[0..6] (src/holbergcoeff.c:37-108). */
int orc_fd_coeffs(const orc_cfg *cfg, float *hc7);

/* Source signals nsrc*NT for SOURCE_SHAPE `shape` (src/wavelet.c:29-133). */
int orc_wavelet(const orc_cfg *cfg, int shape, int nsrc, const float *srcpos, float *signals);

/* Residual / misfit / energy of one component for LNORM=2 with the given
 * trace-kill vector (may be NULL).  Mirrors calc_res (src/calc_res.c:24-309),
 * calc_misfit (src/calc_misfit.c:24-232) and calc_energy
 * (src/calc_energy.c:24-175).  obs/syn/diff are ntr*ns. */
int orc_calc_res(const orc_cfg *cfg, int ntr, int ns, const float *obs, const float *syn,
                 float *diff, double *l2, double *energy, double *misfit);

#ifdef __cplusplus
}
#endif
#endif
