/*
 * ref_stubs.c -- TEST INFRASTRUCTURE ONLY (built into oracle/_ref/).
 *
 * Link stand-ins for reference entry points that need FFTW3 or SU file input
 * (absent here) and are off the path the oracle exercises (LNORM=2, analytic
 * source wavelets).  Each aborts loudly if ever reached.
 */
#include <stdio.h>
#include <stdlib.h>

static void off_path(const char *what) {
    fprintf(stderr, "oracle/_ref: %s is off the oracle's path (needs FFTW3/SU input)\n", what);
    abort();
}
void calc_envelope(float **a, float **b, int ns, int ntr) { (void)a; (void)b; (void)ns; (void)ntr; off_path("calc_envelope"); }
void calc_hilbert(float **a, float **b, int ns, int ntr) { (void)a; (void)b; (void)ns; (void)ntr; off_path("calc_hilbert"); }
void inseis_source_wavelet(float *a, int nt, int ishot, int sh, int stf) {
    (void)a; (void)nt; (void)ishot; (void)sh; (void)stf; off_path("inseis_source_wavelet");
}
/* model file merging of src/mergemod.c (called by the file writers of
 * src/matrix_operations.c, which the smoothing oracle links but never calls) */
void mergemod(char modfile[74], int format) { (void)modfile; (void)format; off_path("mergemod"); }
