/*
 * driver_stubs.c -- TEST INFRASTRUCTURE ONLY (linked into oracle/_ref/IFOS2D
 * and IFOS2D_compat).
 *
 * The four reference routines that need FFTW3 or libstfinv (absent here):
 * source-time-function inversion (src/stf.c), its convolution
 * (src/conv_FD.c) and the Hilbert envelope (src/calc_envelope.c,
 * src/calc_hilbert.c).  They run only with INV_STF=1 or LNORM 5-8, which the
 * driver test does not use; reaching one aborts loudly.
 */
#include <stdio.h>
#include <stdlib.h>

static void off_path(const char *what) {
    fprintf(stderr, "oracle/_ref driver: %s needs FFTW3/libstfinv, which this build leaves out\n", what);
    abort();
}
void stf(FILE *fp, float **sectionvy, float **sectionvy_obs, float **sectionvy_conv, float *source_time_function,
         int **recpos, int **recpos_loc, int ntr_glob, int ntr, float **srcpos, int ishot, int ns, int iter,
         int nsrc_glob, float F_LOW_PASS, int SH, int nsrc_loc) {
    (void)fp; (void)sectionvy; (void)sectionvy_obs; (void)sectionvy_conv; (void)source_time_function;
    (void)recpos; (void)recpos_loc; (void)ntr_glob; (void)ntr; (void)srcpos; (void)ishot; (void)ns; (void)iter;
    (void)nsrc_glob; (void)F_LOW_PASS; (void)SH; (void)nsrc_loc;
    off_path("stf");
}
void conv_FD(float *a, float *b, float *c, int ns) { (void)a; (void)b; (void)c; (void)ns; off_path("conv_FD"); }
void calc_hilbert(float **a, float **b, int ns, int ntr) { (void)a; (void)b; (void)ns; (void)ntr; off_path("calc_hilbert"); }
void calc_envelope(float **a, float **b, int ns, int ntr) { (void)a; (void)b; (void)ns; (void)ntr; off_path("calc_envelope"); }
