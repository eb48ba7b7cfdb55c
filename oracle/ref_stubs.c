/*
 * ref_stubs.c -- TEST INFRASTRUCTURE ONLY (built into oracle/_ref/).
 *
 * Link stand-ins for reference entry points that need FFTW3 or SU file input
 * (absent here) and are off the path the oracle exercises (LNORM=2, analytic
 * source wavelets); those abort loudly if ever reached.  The file writers
 * and the parameter broadcast below are single-rank no-ops.
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
/* model file merging of src/mergemod.c and the per-rank model writer of
 * src/writemod.c: src/calc_mat_change_test.c writes the updated model and
 * the L-BFGS difference vectors through them after its arithmetic; the files
 * are off the oracle's path, so both are no-ops here */
void mergemod(char modfile[74], int format) { (void)modfile; (void)format; }
void writemod(char modfile[74], float **array, int format) { (void)modfile; (void)array; (void)format; }
/* src/exchange_par.c broadcasts the parameters from rank 0; with one rank
 * that is the identity */
void exchange_par(void) {}
