/*
 * writers_harness.c -- TEST INFRASTRUCTURE ONLY (linked into
 * oracle/_ref/libifoswriters.so with the reference's own writemod.c,
 * mergemod.c, writedsk.c, readdsk.c, matrix_operations.c and util.c as
 * compiled for the driver).  It defines the driver's globals (src/globvar.h)
 * and sets the ones the file writers read, for a single-rank run.
 */
#include "fd.h"
#include "globvar.h"

void orc_writer_globals(int nx, int ny) {
    static FILE *devnull = NULL;
    if (!devnull) devnull = fopen("/dev/null", "w");
    FP = devnull;
    NX = NXG = nx;
    NY = NYG = ny;
    IDX = IDY = 1;
    POS[1] = POS[2] = 0;
    MYID = 0;
    NPROCX = NPROCY = NPROC = 1;
    VERBOSE = 0;
}
