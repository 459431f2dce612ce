/*
 * step7.h -- CPU oracle: a C restatement of the reference's serial STEP_7
 * program (giacomofalcucci/BGK_PCM, directory STEP_7/).
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product (bgk_pcm_b200/, include/)
 * links, loads or calls this code; only tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py use it, and only as the checker.
 *
 * Parity status: the reference is Fortran and no Fortran compiler exists in
 * this image, so the reference cannot be built here.  The restatement is
 * pinned instead against golden vectors produced by executing the reference's
 * own STEP_7 source text with a Fortran-subset interpreter
 * (tests/golden/make_golden.py, run where the reference sources are mounted),
 * see tests/test_oracle_golden.py.
 *
 * Layout: every field is (0:Nx+1, 0:Ny+1) column-major, exactly like the
 * reference's allocatable arrays (STEP_7/setup.f90:34-77): element (i,j) is at
 * offset i + (Nx+2)*j.
 */
#ifndef BGK_ORACLE_STEP7_H
#define BGK_ORACLE_STEP7_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* The 21 input.dat values in file order (STEP_7/setup.f90:7-31). */
typedef struct orc_params {
    int iter, noutput, dump, Nx, Ny;
    double Re, rho0, rho1, tau_f, tau_g, T0, T_in_sol, grav, eps,
           stefan_number, T_width, length;
    int westBC, eastBC, northBC, southBC;
} orc_params;

/* Field identifiers (same numbering as the product's BGK_FIELD_*). */
enum {
    ORC_F0 = 0,            /* f0..f8   : 0..8   */
    ORC_G0 = 9,            /* g0..g8   : 9..17  */
    ORC_RHO = 18, ORC_T = 19, ORC_U = 20, ORC_V = 21,
    ORC_PHI = 22, ORC_PHI_PREC = 23,
    ORC_RHO2 = 24, ORC_T2 = 25, ORC_U2 = 26, ORC_V2 = 27,
    ORC_FP0 = 28,          /* fp0..fp8 : 28..36 */
    ORC_GP0 = 37,          /* gp0..gp8 : 37..45 */
    ORC_NFIELDS = 46
};

typedef struct orc_state orc_state;

/* input.dat parser (STEP_7/setup.f90:5-32); returns 0 or a negative code. */
int orc_read_input(const char *path, orc_params *p);

/* setup: allocation + derived constants (STEP_7/setup.f90:34-115). */
orc_state *orc_create(const orc_params *p);
void orc_destroy(orc_state *s);

/* 0 = libm tanh (as the reference), 1 = bgk_portable_tanh (bit-exact mode). */
void orc_set_tanh_mode(orc_state *s, int mode);
/* 1 = keep collision.f90's ft/gt temporaries in double (the smooth,
 * differentiable form); 0 = their implicit REAL(4) (the reference). */
void orc_set_smooth(orc_state *s, int smooth);
/* Heated wall of STEP_DOCONCURRENT's preprocessor options, as bits:
 * ORC_HEAT_RIGHT = FROMRIGHT (east wall at Tin, west wall zero-gradient,
 * liquid strip on the east side), ORC_HEAT_BOTTOM = FROMBOTTOM (initial
 * liquid layer along the south wall); 0 = STEP_7 (heated west wall).
 * Both bits = both macros defined.  Set before orc_initialization. */
enum { ORC_HEAT_RIGHT = 1, ORC_HEAT_BOTTOM = 2 };
void orc_set_heat(orc_state *s, int heat);
/* OpenMP threads for the hot loops (0 = leave the runtime default). */
void orc_set_threads(int n);

/* The reference's subroutines, one call each. */
void orc_initialization(orc_state *s);
void orc_bc_f(orc_state *s);
void orc_bc_g(orc_state *s);
void orc_streaming(orc_state *s);
void orc_moments_pre(orc_state *s);
void orc_phase_field(orc_state *s);
void orc_forces(orc_state *s);
void orc_collision(orc_state *s);
void orc_moments(orc_state *s);

/* n full time steps in the STEP_7/main.f90:60-69 order; advances it. */
void orc_step(orc_state *s, int n);

/* Direct access to a field (ORC_* id); NX2 = Nx+2 is the leading dimension. */
double *orc_field(orc_state *s, int id);
int orc_get_it(const orc_state *s);
void orc_set_it(orc_state *s, int it);

/* Output routines; files are written into the directory given to
 * orc_open_outputs (fort.64, fort.69, non-dim_bulk_numbers.dat, fort.666,
 * fort.667, fort.668, log.dat, Nusselt.dat, Output_XXXXXXXX.vtk). */
int orc_open_outputs(orc_state *s, const char *dir);
void orc_close_outputs(orc_state *s);
void orc_diag(orc_state *s);
void orc_probe(orc_state *s);
void orc_prof_x(orc_state *s);
void orc_prof_y(orc_state *s);
void orc_field_check(orc_state *s);
void orc_out2d(orc_state *s);
/* Reductions used by field_check (STEP_7/field_check.f90:9-17): sums of
 * rho, T, phi over the interior in reference loop order, and #(phi>0). */
void orc_sums(orc_state *s, double out[4]);

/* The whole program of STEP_7/main.f90 run inside dir (reads dir/input.dat,
 * writes the reference's output files there).  Returns 0 on success. */
int orc_main(const char *dir, int nthreads, int tanh_mode, int heat);

/* bgk_portable_tanh, exported for the tests. */
double orc_portable_tanh(double x);

#ifdef __cplusplus
}
#endif
#endif
