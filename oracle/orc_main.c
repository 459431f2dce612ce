/* Command-line driver for the CPU oracle: runs the STEP_7 program in a
 * directory holding input.dat (TEST INFRASTRUCTURE ONLY).
 * usage: orc_main <dir> [threads] [tanh_mode] [heat bits] */
#include "step7.h"
#include <stdio.h>
#include <stdlib.h>

int main(int argc, char **argv)
{
    if (argc < 2) { fprintf(stderr, "usage: %s <dir> [threads] [tanh_mode] [heat]\n", argv[0]); return 2; }
    int nt = argc > 2 ? atoi(argv[2]) : 0;
    int tm = argc > 3 ? atoi(argv[3]) : 0;
    int ht = argc > 4 ? atoi(argv[4]) : 0;
    int rc = orc_main(argv[1], nt, tm, ht);
    if (rc) fprintf(stderr, "orc_main failed: %d\n", rc);
    return rc ? 1 : 0;
}
