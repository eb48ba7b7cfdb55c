/* Role-compatible entry points of libifos_compat.so.
 *
 * The reference's per-kernel functions under their own names and signatures,
 * so that the unmodified IFOS2D driver (src/IFOS2D.c) links against the GPU
 * library instead of its own kernels.  They read the driver's globals
 * (src/globvar.h: NX, NY, NT, DT, DH, FDORDER, FW, FREE_SURF, BOUNDARY,
 * POS, NPROCX, NPROCY, L, FL, F_REF, VELOCITY, PARAMETERIZATION, WAVETYPE,
 * SEISMO, ACOUSTIC, SOURCE_TYPE, ADJOINT_TYPE), which the program linking this
 * library defines, and act on the caller's arrays as allocated by
 * src/util.c matrix()/f3tensor()/vector(): each call mirrors the arrays it
 * reads to the device, computes there, and copies the arrays it writes back
 * before returning.  Results are bit-identical to the reference functions on
 * the same inputs, including their side outputs (rate fields ux/uy/uxy/uxz/uyz,
 * the free-surface ghost rows, the SOURCE_TYPE global set by update_v_PML).
 *
 * infoout, absorb_coeff and the unused m1/utt arrays are accepted and ignored
 * as in the reference.  A CUDA failure prints its cause and exits with
 * status 1, where the reference's declare_error() aborts.
 */
#ifndef IFOS_COMPAT_H
#define IFOS_COMPAT_H

#ifdef __cplusplus
extern "C" {
#endif

/* src/fd.h:384-389 (src/update_v_PML.c:29) */
void update_v_PML(int nx1, int nx2, int ny1, int ny2, int nt, float **vx, float **vxp1, float **vxm1, float **vy,
                  float **vyp1, float **vym1, float **uttx, float **utty, float **sxx, float **syy, float **sxy,
                  float **rip, float **rjp, float **srcpos_loc, float **signals, float **signals1, int nsrc,
                  float **absorb_coeff, float *hc, int infoout, int sw, float *K_x, float *a_x, float *b_x,
                  float *K_x_half, float *a_x_half, float *b_x_half, float *K_y, float *a_y, float *b_y,
                  float *K_y_half, float *a_y_half, float *b_y_half, float **psi_sxx_x, float **psi_syy_y,
                  float **psi_sxy_y, float **psi_sxy_x);

/* src/fd.h:352-357 (src/update_s_elastic_PML.c:28) */
void update_s_elastic_PML(int nx1, int nx2, int ny1, int ny2, float **vx, float **vy, float **ux, float **uy,
                          float **uxy, float **uyx, float **sxx, float **syy, float **sxy, float **pi, float **u,
                          float **uipjp, float **absorb_coeff, float **rho, float *hc, int infoout, float *K_x,
                          float *a_x, float *b_x, float *K_x_half, float *a_x_half, float *b_x_half, float *K_y,
                          float *a_y, float *b_y, float *K_y_half, float *a_y_half, float *b_y_half, float **psi_vxx,
                          float **psi_vyy, float **psi_vxy, float **psi_vyx);

/* src/fd.h:363-369 (src/update_s_visc_PML.c:28) */
void update_s_visc_PML(int nx1, int nx2, int ny1, int ny2, float **vx, float **vy, float **ux, float **uy,
                       float **uxy, float **uyx, float **sxx, float **syy, float **sxy, float **pi, float **u,
                       float **uipjp, float **rho, float *hc, int infoout, float ***r, float ***p, float ***q,
                       float **fipjp, float **f, float **g, float *bip, float *bjm, float *cip, float *cjm,
                       float ***d, float ***e, float ***dip, float *K_x, float *a_x, float *b_x, float *K_x_half,
                       float *a_x_half, float *b_x_half, float *K_y, float *a_y, float *b_y, float *K_y_half,
                       float *a_y_half, float *b_y_half, float **psi_vxx, float **psi_vyy, float **psi_vxy,
                       float **psi_vyx);

/* src/fd.h:286 (src/surface_elastic_PML.c:26) */
void surface_elastic_PML(int ndepth, float **vx, float **vy, float **sxx, float **syy, float **sxy, float **syz,
                         float **pi, float **u, float **rho, float *hc, float *K_x, float *a_x, float *b_x,
                         float **psi_vxx, float **ux, float **uy, float **uxy, float **uyz, float **sxz,
                         float **uxz);

/* src/fd.h:288 (src/surface_PML.c:25) */
void surface_PML(int ndepth, float **vx, float **vy, float **sxx, float **syy, float **sxy, float **syz, float ***p,
                 float ***q, float **ppi, float **pu, float **prho, float **ptaup, float **ptaus, float *etajm,
                 float *peta, float *hc, float *K_x, float *a_x, float *b_x, float **psi_vxx, float **ux,
                 float **uy, float **uxy, float **uyz, float **sxz, float **uxz);

/* src/fd.h:206-207 (src/psource.c:26) */
void psource(int nt, float **sxx, float **syy, float **sp, float **srcpos_loc, float **signals, int nsrc, int sw);

/* src/fd.h:262-265 (src/seismo_ssg.c:26) */
void seismo_ssg(int lsamp, int ntr, int **recpos, float **sectionvx, float **sectionvy, float **sectionvz,
                float **sectionp, float **sectioncurl, float **sectiondiv, float **vx, float **vy, float **vz,
                float **sxx, float **syy, float **sp, float **pi, float **u, float *hc);

/* src/fd.h:391-394 (src/update_v_PML_SH.c:29) */
void update_v_PML_SH(int nx1, int nx2, int ny1, int ny2, int nt, float **vz, float **vzp1, float **vzm1, float **sxz,
                     float **syz, float **rjp, float **srcpos_loc, float **signals, float **signals1, int nsrc,
                     float **absorb_coeff, float *hc, int infoout, int sw, float *K_x, float *a_x, float *b_x,
                     float *K_x_half, float *a_x_half, float *b_x_half, float *K_y, float *a_y, float *b_y,
                     float *K_y_half, float *a_y_half, float *b_y_half, float **psi_sxz_x, float **psi_syz_y);

/* src/fd.h:313-314 (src/update_s_elastic_PML_SH.c:28) */
void update_s_elastic_PML_SH(int nx1, int nx2, int ny1, int ny2, float **vz, float **sxz, float **syz, float **uxz,
                             float **uyz, float *hc, int infoout, float *K_x, float *a_x, float *b_x,
                             float *K_x_half, float *a_x_half, float *b_x_half, float *K_y, float *a_y, float *b_y,
                             float *K_y_half, float *a_y_half, float *b_y_half, float **psi_vzx, float **psi_vzy,
                             float **uipjp, float **u, float **rho);

/* src/fd.h:316 (src/update_s_visc_PML_SH.c:29) */
void update_s_visc_PML_SH(int nx1, int nx2, int ny1, int ny2, float **vz, float **sxz, float **syz, float ***t,
                          float ***o, float *bip, float *bjm, float *cip, float *cjm, float ***d, float ***dip,
                          float **fipjp, float **f, float *hc, int infoout, float *K_x, float *a_x, float *b_x,
                          float *K_x_half, float *a_x_half, float *b_x_half, float *K_y, float *a_y, float *b_y,
                          float *K_y_half, float *a_y_half, float *b_y_half, float **psi_vzx, float **psi_vzy);

/* src/fd.h:502-507 (src/update_v_acoustic_PML.c) */
void update_v_acoustic_PML(int nx1, int nx2, int ny1, int ny2, int nt, float **vx, float **vxp1, float **vxm1,
                           float **vy, float **vyp1, float **vym1, float **sp, float **rip, float **rjp,
                           float **srcpos_loc, float **signals, float **signals1, int nsrc, float **absorb_coeff,
                           float *hc, int infoout, int sw, float *K_x_half, float *a_x_half, float *b_x_half,
                           float *K_y_half, float *a_y_half, float *b_y_half, float **psi_sxx_x, float **psi_syy_y);

/* src/fd.h:509-513 (src/update_p_PML.c:28) */
void update_p_PML(int nx1, int nx2, int ny1, int ny2, float **vx, float **vy, float **sp, float **u, float **pi,
                  float **absorb_coeff, float **rho, float *hc, int infoout, float *K_x, float *a_x, float *b_x,
                  float *K_x_half, float *a_x_half, float *b_x_half, float *K_y, float *a_y, float *b_y,
                  float *K_y_half, float *a_y_half, float *b_y_half, float **psi_vxx, float **psi_vyy,
                  float **psi_vxy, float **psi_vyx);

/* src/fd.h:556-560 (src/update_p_visc_PML.c:30) */
void update_p_visc_PML(int nx1, int nx2, int ny1, int ny2, float **vx, float **vy, float **sp, float **pi,
                       float **rho, float *hc, int infoout, float ***p, float **g, float *bjm, float *cjm, float ***e,
                       float *K_x, float *a_x, float *b_x, float *K_x_half, float *a_x_half, float *b_x_half,
                       float *K_y, float *a_y, float *b_y, float *K_y_half, float *a_y_half, float *b_y_half,
                       float **psi_vxx, float **psi_vyy, float **psi_vxy, float **psi_vyx);

/* src/fd.h:515 (src/surface_acoustic_PML.c:23) */
void surface_acoustic_PML(int ndepth, float **sp);

/* Release the device mirrors held for the caller's arrays (optional; the
 * mirrors are otherwise kept for reuse until the process exits). */
void ifos_compat_release(void);

#ifdef __cplusplus
}
#endif

#endif /* IFOS_COMPAT_H */
