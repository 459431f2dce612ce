/*
 * step7.c -- CPU oracle: C restatement of the reference's serial STEP_7
 * program (giacomofalcucci/BGK_PCM).  TEST INFRASTRUCTURE ONLY: the product
 * never links or calls this file; tests, smoke() and bench.py's CPU-baseline
 * leg use it as the checker.
 *
 * Every routine below cites the reference file:line it restates.  Arithmetic
 * is written with the reference's evaluation order (Fortran evaluates a chain
 * of + or * left to right; parenthesised groups first) and must be compiled
 * with -ffp-contract=off so that no a*b+c is fused: gfortran -O3 for generic
 * x86-64 (STEP_7/Makefile:5-7) emits no FMA.  `x**2.0d0` is x*x, which is how
 * gfortran expands a real power of 2.0.
 *
 * Quirks reproduced on purpose (each one changes results):
 *  - forces: `beta` is never declared and forces.f90 has no `implicit none`,
 *    so it is an implicit default REAL (4 bytes): its value is rounded to
 *    float and promoted back (STEP_7/forces.f90:13).
 *  - collision: the temporaries are declared as ft00..ft08 / gt00..gt08
 *    (STEP_7/collision.f90:11-12) but the code assigns ft0..ft8 / gt0..gt8
 *    (collision.f90:84-120), which are therefore implicit REAL(4) as well:
 *    each regularized population is rounded to float before the relaxation
 *    f = ft - omega*(ft - feq) is evaluated in double.
 *  - BC_f with code 4 never writes f6(Nx+1,0) nor f7(Nx+1,Ny+1); streaming
 *    reads them, so they keep their initial equilibrium values.
 *  - BC_g's north/south copies run after its west/east fills, so the corner
 *    halos take the west/east values.
 *  - moments leaves T, u, v as the average of the post-collision moments and
 *    the pre-collision ones (STEP_7/moments.f90:20-24).
 *  - diag's Ny**3 is a default (32-bit) INTEGER product and wraps.
 * The OpenMP loops split only the j range of loops without reductions, so a
 * multi-threaded run is bit-identical to a serial one (STEP_OPENMP/ adds the
 * same directives to the same loops).
 */
#include "step7.h"
#include "../include/bgk_portable_tanh.h"

#include <errno.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

struct orc_state {
    orc_params p;
    int Nx, Ny, NX2, NY2;
    size_t A;
    double *fld[ORC_NFIELDS];
    double *x, *y;
    /* shared.f90 scalars */
    double kvisc, alpha, T0, Tin, rho0, rho1, eps, T_in_sol;
    double w[9], cx[9], cy[9];
    double omega_g, omega_f, tau_g, tau_f, grav;
    double mass, length;
    double T_crit, T_act, T_width, f_plus, f_minus;
    double u0, v0, cs, cs2, cs4, delta_T, stefan_number, Re, Mach;
    double Nu[40], Nu2[40], Nu3[40];
    int it, iter, it0, a, b, samplex, sampley, interf, dump, noutput;
    int westBC, eastBC, northBC, southBC;
    int deltaOut, itOut;
    int tanh_mode;
    int smooth;            /* 1: keep ft/gt in double (the differentiable form) */
    int heat;              /* ORC_HEAT_* bits (STEP_DOCONCURRENT's FROMRIGHT / FROMBOTTOM) */
    /* diag.f90's melt_front/melt_front_expected are locals that are not
     * assigned on every path; they are carried from call to call here. */
    double diag_melt_front, diag_melt_front_expected;
    char dir[1024];
    FILE *u64, *u69, *u164, *u666, *u667, *u668;
};

#define IX(i, j) ((size_t)(i) + (size_t)s->NX2 * (size_t)(j))
#define F(k) (s->fld[ORC_F0 + (k)])
#define G(k) (s->fld[ORC_G0 + (k)])
#define FP(k) (s->fld[ORC_FP0 + (k)])
#define GP(k) (s->fld[ORC_GP0 + (k)])
#define RHO (s->fld[ORC_RHO])
#define TT (s->fld[ORC_T])
#define UU (s->fld[ORC_U])
#define VV (s->fld[ORC_V])
#define PHI (s->fld[ORC_PHI])
#define PHIP (s->fld[ORC_PHI_PREC])
#define RHO2 (s->fld[ORC_RHO2])
#define T2 (s->fld[ORC_T2])
#define U2 (s->fld[ORC_U2])
#define V2 (s->fld[ORC_V2])

void orc_set_threads(int n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

/* ---------------------------------------------------------------- input */

/* List-directed read of "label value [anything]" (STEP_7/setup.f90:7-31):
 * the label goes into a CHARACTER(1) and is discarded, the value is the
 * second blank/comma separated token; reals may use a d/D exponent. */
static int next_value(FILE *fp, char *tok, size_t n)
{
    char line[4096];
    while (fgets(line, sizeof line, fp)) {
        char *save = NULL;
        char *t1 = strtok_r(line, " \t,\r\n", &save);
        if (!t1) return -1; /* a blank record: list-directed read fails */
        char *t2 = strtok_r(NULL, " \t,\r\n", &save);
        if (!t2) return -1;
        strncpy(tok, t2, n - 1);
        tok[n - 1] = 0;
        return 0;
    }
    return -1;
}

static int parse_real(const char *t, double *out)
{
    char buf[256];
    size_t n = strlen(t);
    if (n >= sizeof buf) return -1;
    for (size_t i = 0; i <= n; i++) {
        char c = t[i];
        buf[i] = (c == 'd' || c == 'D') ? 'e' : c;
    }
    char *end = NULL;
    errno = 0;
    double v = strtod(buf, &end);
    if (end == buf || *end != 0 || errno) return -1;
    *out = v;
    return 0;
}

static int parse_int(const char *t, int *out)
{
    char *end = NULL;
    errno = 0;
    long v = strtol(t, &end, 10);
    if (end == t || *end != 0 || errno) return -1;
    *out = (int)v;
    return 0;
}

int orc_read_input(const char *path, orc_params *p)
{
    FILE *fp = fopen(path, "r");
    if (!fp) return -1;
    char tok[256];
    int rc = 0;
#define RI(field) do { if (rc == 0 && (next_value(fp, tok, sizeof tok) || parse_int(tok, &p->field))) rc = -2; } while (0)
#define RR(field) do { if (rc == 0 && (next_value(fp, tok, sizeof tok) || parse_real(tok, &p->field))) rc = -2; } while (0)
    RI(iter); RI(noutput); RI(dump); RI(Nx); RI(Ny);
    RR(Re); RR(rho0); RR(rho1); RR(tau_f); RR(tau_g); RR(T0); RR(T_in_sol);
    RR(grav); RR(eps); RR(stefan_number); RR(T_width); RR(length);
    RI(westBC); RI(eastBC); RI(northBC); RI(southBC);
#undef RI
#undef RR
    fclose(fp);
    return rc;
}

/* ---------------------------------------------------------------- setup */

/* STEP_7/setup.f90:34-115 */
orc_state *orc_create(const orc_params *p)
{
    if (p->Nx < 1 || p->Ny < 1) return NULL;
    orc_state *s = (orc_state *)calloc(1, sizeof *s);
    if (!s) return NULL;
    s->p = *p;
    s->Nx = p->Nx;
    s->Ny = p->Ny;
    s->NX2 = p->Nx + 2;
    s->NY2 = p->Ny + 2;
    s->A = (size_t)s->NX2 * (size_t)s->NY2;
    for (int k = 0; k < ORC_NFIELDS; k++) {
        s->fld[k] = (double *)calloc(s->A, sizeof(double));
        if (!s->fld[k]) { orc_destroy(s); return NULL; }
    }
    s->x = (double *)calloc((size_t)s->NX2, sizeof(double));
    s->y = (double *)calloc((size_t)s->NY2, sizeof(double));
    s->iter = p->iter; s->noutput = p->noutput; s->dump = p->dump;
    s->Re = p->Re; s->rho0 = p->rho0; s->rho1 = p->rho1;
    s->tau_f = p->tau_f; s->tau_g = p->tau_g; s->T0 = p->T0;
    s->T_in_sol = p->T_in_sol; s->grav = p->grav; s->eps = p->eps;
    s->stefan_number = p->stefan_number; s->T_width = p->T_width;
    s->length = p->length;
    s->westBC = p->westBC; s->eastBC = p->eastBC;
    s->northBC = p->northBC; s->southBC = p->southBC;

    s->w[0] = 4.0 / 9.0;
    s->w[1] = 1.0 / 9.0; s->w[2] = 1.0 / 9.0; s->w[3] = 1.0 / 9.0; s->w[4] = 1.0 / 9.0;
    s->w[5] = 1.0 / 36.0; s->w[6] = 1.0 / 36.0; s->w[7] = 1.0 / 36.0; s->w[8] = 1.0 / 36.0;

    s->x[0] = 0.0; s->y[0] = 0.0;
    for (int i = 1; i <= s->Nx + 1; i++) s->x[i] = s->x[i - 1] + 1.0;
    for (int j = 1; j <= s->Ny + 1; j++) s->y[j] = s->y[j - 1] + 1.0;

    s->cs = sqrt(1.0 / 3.0);
    s->cs2 = 1.0 / 3.0;
    s->cs4 = 1.0 / 9.0;
    s->omega_f = 1.0 / s->tau_f;
    s->omega_g = 1.0 / s->tau_g;
    s->kvisc = s->cs2 * (s->tau_f - 0.5);
    s->alpha = s->cs2 * (s->tau_g - 0.5);
    s->samplex = 40;
    s->sampley = 20;
    s->a = s->Nx / s->samplex;
    s->b = s->Ny / s->sampley;
    return s;
}

void orc_destroy(orc_state *s)
{
    if (!s) return;
    orc_close_outputs(s);
    for (int k = 0; k < ORC_NFIELDS; k++) free(s->fld[k]);
    free(s->x);
    free(s->y);
    free(s);
}

void orc_set_tanh_mode(orc_state *s, int mode) { s->tanh_mode = mode; }
void orc_set_smooth(orc_state *s, int smooth) { s->smooth = smooth; }
void orc_set_heat(orc_state *s, int heat) { s->heat = heat; }
double *orc_field(orc_state *s, int id) { return (id >= 0 && id < ORC_NFIELDS) ? s->fld[id] : NULL; }
int orc_get_it(const orc_state *s) { return s->it; }
void orc_set_it(orc_state *s, int it) { s->it = it; }

/* Equilibrium of the 9 populations for prefactor r (rho or T) and velocity
 * (u,v), in the exact expression order of STEP_7/initialization.f90:104-128,
 * STEP_7/collision.f90:19-37 and STEP_7/BC_f.f90 (w*r computed first; the
 * diagonal terms are 4.5d0*upv*upv = (4.5*upv)*upv). */
static inline void feq9(const double *w, double r, double u, double v, double *e)
{
    double uu = u * u, vv = v * v;
    double uv = 1.5 * (uu + vv);
    double upv = u + v, umv = u - v;
    e[0] = w[0] * r * (1.0 - uv);
    e[1] = w[1] * r * (1.0 + 3.0 * u + 4.5 * uu - uv);
    e[2] = w[2] * r * (1.0 + 3.0 * v + 4.5 * vv - uv);
    e[3] = w[3] * r * (1.0 - 3.0 * u + 4.5 * uu - uv);
    e[4] = w[4] * r * (1.0 - 3.0 * v + 4.5 * vv - uv);
    e[5] = w[5] * r * (1.0 + 3.0 * upv + 4.5 * upv * upv - uv);
    e[6] = w[6] * r * (1.0 - 3.0 * umv + 4.5 * umv * umv - uv);
    e[7] = w[7] * r * (1.0 - 3.0 * upv + 4.5 * upv * upv - uv);
    e[8] = w[8] * r * (1.0 + 3.0 * umv + 4.5 * umv * umv - uv);
}

/* ------------------------------------------------------- initialization */

/* STEP_7/initialization.f90:5-152; with heat bits, the branches of
 * STEP_DOCONCURRENT/initialization.f90:16-62 (T/rho), :122-137 (T buffer)
 * and :208-222 (phi). */
void orc_initialization(orc_state *s)
{
    const int Nx = s->Nx, Ny = s->Ny;
    const int right = s->heat & ORC_HEAT_RIGHT, bottom = s->heat & ORC_HEAT_BOTTOM;
    s->interf = Nx / 40;
    s->Tin = s->T0;
    s->u0 = s->Re * s->kvisc / s->length;
    s->v0 = 0.0;
    s->Mach = s->u0 / s->cs;

    for (int j = 0; j <= Ny + 1; j++)
        for (int i = 0; i <= Nx + 1; i++) {
            /* liquid layer: rows 0..interf (FROMBOTTOM; interf = Nx/40 also
             * here), columns Nx-interf+1..Nx+1 (FROMRIGHT) or 0..interf */
            const int liquid = bottom ? (j <= s->interf) : right ? (i >= Nx - s->interf + 1) : (i <= s->interf);
            TT[IX(i, j)] = liquid ? s->T0 : s->T_in_sol;
            RHO[IX(i, j)] = liquid ? s->rho1 : s->rho0;
        }
    for (size_t q = 0; q < s->A; q++) { UU[q] = s->u0; VV[q] = s->v0; }

    static const double cx[9] = {0, 1, 0, -1, 0, 1, -1, -1, 1};
    static const double cy[9] = {0, 0, 1, 0, -1, 1, 1, -1, -1};
    memcpy(s->cx, cx, sizeof cx);
    memcpy(s->cy, cy, sizeof cy);

    if (bottom) {
        /* `do i = 0,Ny+1; T(i,0) = Tin`: the index runs to Ny+1 along x, so
         * with Ny > Nx it continues past the end of row 0 into row 1 (column-
         * major storage, no bounds check): the first Ny+2 cells in memory */
        for (int i = 0; i <= Ny + 1; i++) TT[i] = s->Tin;
    } else if (right) {
        for (int j = 0; j <= Ny + 1; j++) TT[IX(Nx + 1, j)] = s->Tin;
    } else {
        for (int j = 0; j <= Ny + 1; j++) TT[IX(0, j)] = s->Tin;
    }
    for (int i = 0; i <= Nx + 1; i++) {
        UU[IX(i, Ny + 1)] = 0.0; VV[IX(i, Ny + 1)] = 0.0;
        UU[IX(i, 0)] = 0.0; VV[IX(i, 0)] = 0.0;
    }
    if (s->westBC == 3) {
        for (size_t q = 0; q < s->A; q++) { UU[q] = 0.0; VV[q] = 0.0; }
        for (int j = 0; j <= Ny + 1; j++) RHO[IX(0, j)] = s->rho1;
    }
    for (int j = 1; j <= Ny; j++) {
        if (s->westBC == 1) {
            UU[IX(0, j)] = s->u0;
            VV[IX(0, j)] = s->v0;
        } else if (s->westBC == 2) {
            double ny1 = (double)(Ny + 1);
            UU[IX(0, j)] = -(6.0 * s->u0 / (ny1 * ny1)) * (s->y[j] * s->y[j] - ny1 * s->y[j]);
            VV[IX(0, j)] = s->v0;
        }
    }
    for (int j = 0; j <= Ny + 1; j++)
        for (int i = 0; i <= Nx + 1; i++) {
            size_t q = IX(i, j);
            double e[9];
            feq9(s->w, RHO[q], UU[q], VV[q], e);
            for (int k = 0; k < 9; k++) F(k)[q] = e[k];
            feq9(s->w, TT[q], UU[q], VV[q], e);
            for (int k = 0; k < 9; k++) G(k)[q] = e[k];
        }
    for (size_t q = 0; q < s->A; q++) { PHI[q] = -1.0; PHIP[q] = -1.0; }
    /* FROMRIGHT's phi strip starts at Nx-interf, one column left of its T
     * strip; FROMBOTTOM keeps the west phi strip */
    const int p0 = right ? Nx - s->interf : 0, p1 = right ? Nx + 1 : s->interf;
    for (int j = 0; j <= Ny + 1; j++)
        for (int i = p0; i <= p1; i++) {
            PHI[IX(i, j)] = 1.0;
            PHIP[IX(i, j)] = 1.0;
        }
    s->it = 0;
}

/* ----------------------------------------------------------------- BC_f */

/* STEP_7/BC_f.f90:5-200, all branches, in source order W, E, N, S. */
void orc_bc_f(orc_state *s)
{
    const int Nx = s->Nx, Ny = s->Ny;
    const double *w = s->w;
    double uu, vv, uv, upv, umv;
    /* WEST */
    if (s->westBC == 0) {
        for (int j = 0; j <= Ny + 1; j++)
            for (int k = 0; k < 9; k++) F(k)[IX(0, j)] = F(k)[IX(Nx, j)];
    } else if (s->westBC == 1) {
        uu = s->u0 * s->u0; vv = s->v0 * s->v0; uv = 1.5 * (uu + vv);
        upv = s->u0 + s->v0; umv = s->u0 - s->v0;
        for (int j = 1; j <= Ny; j++) {
            double r = RHO[IX(1, j)];
            F(1)[IX(0, j)] = w[1] * r * (1.0 + 3.0 * s->u0 + 4.5 * uu - uv);
            F(5)[IX(0, j)] = w[5] * r * (1.0 + 3.0 * upv + 4.5 * upv * upv - uv);
            F(8)[IX(0, j)] = w[8] * r * (1.0 + 3.0 * umv + 4.5 * umv * umv - uv);
            UU[IX(0, j)] = s->u0;
            VV[IX(0, j)] = s->v0;
            RHO[IX(0, j)] = RHO[IX(1, j)];
        }
    } else if (s->westBC == 2) {
        for (int j = 0; j <= Ny + 1; j++) {
            double u = UU[IX(0, j)];
            uu = u * u; vv = s->v0 * s->v0; uv = 1.5 * (uu + vv);
            upv = u + s->v0; umv = u - s->v0;
            double r = RHO[IX(1, j)];
            F(1)[IX(0, j)] = w[1] * r * (1.0 + 3.0 * u + 4.5 * uu - uv);
            F(5)[IX(0, j)] = w[5] * r * (1.0 + 3.0 * upv + 4.5 * upv * upv - uv);
            F(8)[IX(0, j)] = w[8] * r * (1.0 + 3.0 * umv + 4.5 * umv * umv - uv);
        }
    } else if (s->westBC == 3) {
        for (int j = 0; j <= Ny + 1; j++) {
            double u = UU[IX(1, j)], v = VV[IX(1, j)];
            uu = u * u; vv = v * v; uv = 1.5 * (uu + vv);
            upv = u + v; umv = u - v;
            F(1)[IX(0, j)] = w[1] * s->rho1 * (1.0 + 3.0 * u + 4.5 * uu - uv);
            F(5)[IX(0, j)] = w[5] * s->rho1 * (1.0 + 3.0 * upv + 4.5 * upv * upv - uv);
            F(8)[IX(0, j)] = w[8] * s->rho1 * (1.0 + 3.0 * umv + 4.5 * umv * umv - uv);
            UU[IX(0, j)] = u;
            VV[IX(0, j)] = v;
            RHO[IX(0, j)] = s->rho1;
        }
    } else if (s->westBC == 4) {
        for (int j = 1; j <= Ny; j++) {
            F(1)[IX(0, j)] = F(3)[IX(1, j)];
            F(8)[IX(0, j)] = F(6)[IX(1, j - 1)];
            F(5)[IX(0, j)] = F(7)[IX(1, j + 1)];
        }
    }
    /* EAST */
    if (s->eastBC == 0) {
        for (int j = 0; j <= Ny + 1; j++)
            for (int k = 0; k < 9; k++) F(k)[IX(Nx + 1, j)] = F(k)[IX(1, j)];
    } else if (s->eastBC == 3) {
        for (int j = 1; j <= Ny; j++) {
            double u = UU[IX(Nx, j)], v = VV[IX(Nx, j)];
            uu = u * u; vv = v * v; uv = 1.5 * (uu + vv);
            upv = u + v; umv = u - v;
            F(3)[IX(Nx + 1, j)] = w[3] * s->rho0 * (1.0 - 3.0 * u + 4.5 * uu - uv);
            F(6)[IX(Nx + 1, j)] = w[6] * s->rho0 * (1.0 - 3.0 * umv + 4.5 * umv * umv - uv);
            F(7)[IX(Nx + 1, j)] = w[7] * s->rho0 * (1.0 - 3.0 * upv + 4.5 * upv * upv - uv);
            UU[IX(Nx + 1, j)] = u;
            VV[IX(Nx + 1, j)] = v;
            RHO[IX(Nx + 1, j)] = s->rho0;
        }
    } else if (s->eastBC == 4) {
        for (int j = 1; j <= Ny; j++) {
            F(3)[IX(Nx + 1, j)] = F(1)[IX(Nx, j)];
            F(6)[IX(Nx + 1, j)] = F(8)[IX(Nx, j + 1)];
            F(7)[IX(Nx + 1, j)] = F(5)[IX(Nx, j - 1)];
        }
    }
    /* NORTH */
    if (s->northBC == 0) {
        for (int i = 0; i <= Nx + 1; i++)
            for (int k = 0; k < 9; k++) F(k)[IX(i, Ny + 1)] = F(k)[IX(i, 1)];
    } else if (s->northBC == 4) {
        for (int i = 1; i <= Nx; i++) {
            F(4)[IX(i, Ny + 1)] = F(2)[IX(i, Ny)];
            F(7)[IX(i, Ny + 1)] = F(5)[IX(i - 1, Ny)];
            F(8)[IX(i, Ny + 1)] = F(6)[IX(i + 1, Ny)];
            RHO[IX(i, Ny + 1)] = RHO[IX(i, Ny)];
            UU[IX(i, Ny + 1)] = 0.0;
            VV[IX(i, Ny + 1)] = 0.0;
        }
        F(8)[IX(0, Ny + 1)] = F(6)[IX(1, Ny)];
    } else if (s->northBC == 5) {
        for (int i = 0; i <= Nx + 1; i++) {
            F(4)[IX(i, Ny + 1)] = F(2)[IX(i, Ny - 1)];
            F(7)[IX(i, Ny + 1)] = F(6)[IX(i, Ny - 1)];
            F(8)[IX(i, Ny + 1)] = F(5)[IX(i, Ny - 1)];
        }
    } else if (s->northBC == 6) {
        for (int i = 0; i <= Nx + 1; i++) {
            F(4)[IX(i, Ny + 1)] = F(4)[IX(i, Ny)];
            F(7)[IX(i, Ny + 1)] = F(7)[IX(i, Ny)];
            F(8)[IX(i, Ny + 1)] = F(8)[IX(i, Ny)];
        }
    } else if (s->northBC == 1) {
        uu = s->u0 * s->u0; vv = s->v0 * s->v0; uv = 1.5 * (uu + vv);
        upv = s->u0 + s->v0; umv = s->u0 - s->v0;
        for (int i = 0; i <= Nx + 1; i++) {
            double r = RHO[IX(i, Ny)];
            F(4)[IX(i, Ny + 1)] = w[4] * r * (1.0 - 3.0 * s->v0 + 4.5 * vv - uv);
            F(7)[IX(i, Ny + 1)] = w[7] * r * (1.0 - 3.0 * upv + 4.5 * upv * upv - uv);
            F(8)[IX(i, Ny + 1)] = w[8] * r * (1.0 + 3.0 * umv + 4.5 * umv * umv - uv);
        }
    }
    /* SOUTH */
    if (s->southBC == 0) {
        for (int i = 0; i <= Nx + 1; i++)
            for (int k = 0; k < 9; k++) F(k)[IX(i, 0)] = F(k)[IX(i, Ny)];
    } else if (s->southBC == 4) {
        for (int i = 1; i <= Nx; i++) {
            F(2)[IX(i, 0)] = F(4)[IX(i, 1)];
            F(5)[IX(i, 0)] = F(7)[IX(i + 1, 1)];
            F(6)[IX(i, 0)] = F(8)[IX(i - 1, 1)];
            RHO[IX(i, 0)] = RHO[IX(i, 1)];
            UU[IX(i, 0)] = 0.0;
            VV[IX(i, 0)] = 0.0;
        }
        F(5)[IX(0, 0)] = F(7)[IX(1, 1)];
    } else if (s->southBC == 6) {
        for (int i = 0; i <= Nx + 1; i++) {
            F(2)[IX(i, 0)] = F(2)[IX(i, 1)];
            F(5)[IX(i, 0)] = F(5)[IX(i, 1)];
            F(6)[IX(i, 0)] = F(6)[IX(i, 1)];
        }
    }
}

/* ----------------------------------------------------------------- BC_g */

/* STEP_7/BC_g.f90:5-64 (no branches: W Dirichlet Tin, E zero-gradient T,
 * N/S copies of all nine g, T and phi).  With ORC_HEAT_RIGHT, the FROMRIGHT
 * branches of STEP_DOCONCURRENT/BC_g.f90:13-45: W zero-gradient T, whose g1,
 * g5, g8 take the -x equilibrium polynomials of directions 3, 7, 6 (the
 * sign flip is the reference's), E Dirichlet Tin.  DOCONCURRENT's loops run
 * over j = 0..Ny / 0..Ny+1; rows 0 and Ny+1 are overwritten by the N/S copies
 * below, so j = 1..Ny gives the same arrays. */
void orc_bc_g(orc_state *s)
{
    const int Nx = s->Nx, Ny = s->Ny;
    const double *w = s->w;
    if (s->heat & ORC_HEAT_RIGHT) {
        for (int j = 1; j <= Ny; j++) {
            double u = UU[IX(0, j)], v = VV[IX(0, j)];
            double uu = u * u, vv = v * v, uv = 1.5 * (uu + vv);
            double upv = u + v, umv = u - v;
            double t = TT[IX(1, j)];
            G(1)[IX(0, j)] = w[1] * t * (1.0 - 3.0 * u + 4.5 * uu - uv);
            G(5)[IX(0, j)] = w[5] * t * (1.0 - 3.0 * upv + 4.5 * upv * upv - uv);
            G(8)[IX(0, j)] = w[8] * t * (1.0 - 3.0 * umv + 4.5 * umv * umv - uv);
            TT[IX(0, j)] = TT[IX(1, j)];
        }
        for (int j = 1; j <= Ny; j++) {
            double u = UU[IX(Nx + 1, j)], v = VV[IX(Nx + 1, j)];
            double uu = u * u, vv = v * v, uv = 1.5 * (uu + vv);
            double upv = u + v, umv = u - v;
            G(3)[IX(Nx + 1, j)] = w[3] * s->Tin * (1.0 - 3.0 * u + 4.5 * uu - uv);
            G(6)[IX(Nx + 1, j)] = w[6] * s->Tin * (1.0 - 3.0 * umv + 4.5 * umv * umv - uv);
            G(7)[IX(Nx + 1, j)] = w[7] * s->Tin * (1.0 - 3.0 * upv + 4.5 * upv * upv - uv);
            TT[IX(Nx + 1, j)] = s->Tin;
        }
    }
    for (int j = 1; j <= Ny && !(s->heat & ORC_HEAT_RIGHT); j++) {
        double u = UU[IX(0, j)], v = VV[IX(0, j)];
        double uu = u * u, vv = v * v, uv = 1.5 * (uu + vv);
        double upv = u + v, umv = u - v;
        G(1)[IX(0, j)] = w[1] * s->Tin * (1.0 + 3.0 * u + 4.5 * uu - uv);
        G(5)[IX(0, j)] = w[5] * s->Tin * (1.0 + 3.0 * upv + 4.5 * upv * upv - uv);
        G(8)[IX(0, j)] = w[8] * s->Tin * (1.0 + 3.0 * umv + 4.5 * umv * umv - uv);
        TT[IX(0, j)] = s->Tin;
    }
    for (int j = 1; j <= Ny && !(s->heat & ORC_HEAT_RIGHT); j++) {
        double u = UU[IX(Nx + 1, j)], v = VV[IX(Nx + 1, j)];
        double uu = u * u, vv = v * v, uv = 1.5 * (uu + vv);
        double upv = u + v, umv = u - v;
        double t = TT[IX(Nx, j)];
        G(3)[IX(Nx + 1, j)] = w[3] * t * (1.0 - 3.0 * u + 4.5 * uu - uv);
        G(6)[IX(Nx + 1, j)] = w[6] * t * (1.0 - 3.0 * umv + 4.5 * umv * umv - uv);
        G(7)[IX(Nx + 1, j)] = w[7] * t * (1.0 - 3.0 * upv + 4.5 * upv * upv - uv);
        TT[IX(Nx + 1, j)] = TT[IX(Nx, j)];
    }
    for (int i = 0; i <= Nx + 1; i++) {
        for (int k = 0; k < 9; k++) G(k)[IX(i, Ny + 1)] = G(k)[IX(i, Ny)];
        TT[IX(i, Ny + 1)] = TT[IX(i, Ny)];
        PHI[IX(i, Ny + 1)] = PHI[IX(i, Ny)];
    }
    for (int i = 0; i <= Nx + 1; i++) {
        for (int k = 0; k < 9; k++) G(k)[IX(i, 0)] = G(k)[IX(i, 1)];
        TT[IX(i, 0)] = TT[IX(i, 1)];
        PHI[IX(i, 0)] = PHI[IX(i, 1)];
    }
}

/* ------------------------------------------------------------ streaming */

/* STEP_7/streaming.f90:5-27: pull fp_k(i,j) = f_k(i-cx_k, j-cy_k). */
void orc_streaming(orc_state *s)
{
    const int Nx = s->Nx, Ny = s->Ny;
#pragma omp parallel for schedule(static)
    for (int j = 1; j <= Ny; j++)
        for (int i = 1; i <= Nx; i++) {
            size_t q = IX(i, j);
            FP(0)[q] = F(0)[IX(i, j)];
            FP(1)[q] = F(1)[IX(i - 1, j)];
            FP(2)[q] = F(2)[IX(i, j - 1)];
            FP(3)[q] = F(3)[IX(i + 1, j)];
            FP(4)[q] = F(4)[IX(i, j + 1)];
            FP(5)[q] = F(5)[IX(i - 1, j - 1)];
            FP(6)[q] = F(6)[IX(i + 1, j - 1)];
            FP(7)[q] = F(7)[IX(i + 1, j + 1)];
            FP(8)[q] = F(8)[IX(i - 1, j + 1)];
            GP(0)[q] = G(0)[IX(i, j)];
            GP(1)[q] = G(1)[IX(i - 1, j)];
            GP(2)[q] = G(2)[IX(i, j - 1)];
            GP(3)[q] = G(3)[IX(i + 1, j)];
            GP(4)[q] = G(4)[IX(i, j + 1)];
            GP(5)[q] = G(5)[IX(i - 1, j - 1)];
            GP(6)[q] = G(6)[IX(i + 1, j - 1)];
            GP(7)[q] = G(7)[IX(i + 1, j + 1)];
            GP(8)[q] = G(8)[IX(i - 1, j + 1)];
        }
}

/* ----------------------------------------------------------- momentsPre */

/* STEP_7/momentsPre.f90:5-23 */
void orc_moments_pre(orc_state *s)
{
    const int Nx = s->Nx, Ny = s->Ny;
#pragma omp parallel for schedule(static)
    for (int j = 1; j <= Ny; j++)
        for (int i = 1; i <= Nx; i++) {
            size_t q = IX(i, j);
            double f0 = FP(0)[q], f1 = FP(1)[q], f2 = FP(2)[q], f3 = FP(3)[q], f4 = FP(4)[q];
            double f5 = FP(5)[q], f6 = FP(6)[q], f7 = FP(7)[q], f8 = FP(8)[q];
            double rho = f0 + f1 + f2 + f3 + f4 + f5 + f6 + f7 + f8;
            double t = GP(0)[q] + GP(1)[q] + GP(2)[q] + GP(3)[q] + GP(4)[q]
                     + GP(5)[q] + GP(6)[q] + GP(7)[q] + GP(8)[q];
            double irho = 1.0 / rho;
            double u = irho * (f1 - f3 + f5 - f6 - f7 + f8);
            double v = irho * (f2 - f4 + f5 + f6 - f7 - f8);
            RHO[q] = rho; TT[q] = t; UU[q] = u; VV[q] = v;
            RHO2[q] = rho; T2[q] = t; U2[q] = u; V2[q] = v;
        }
}

/* ---------------------------------------------------------- phase_field */

static inline double sq(double x) { return x * x; }

/* STEP_7/phase_field.f90:11-52 (Succi's kinetic phase selector). */
void orc_phase_field(orc_state *s)
{
    const int Nx = s->Nx, Ny = s->Ny;
    s->T_act = 0.0;
    s->T_crit = 273.0;
    s->f_plus = 0.5;
    s->f_minus = 0.5;
    memcpy(PHIP, PHI, s->A * sizeof(double));
    const double T_crit = s->T_crit, T_act = s->T_act, T_width = s->T_width;
    const double f_plus = s->f_plus, f_minus = s->f_minus;
    const int portable = s->tanh_mode == 1;
#pragma omp parallel for schedule(static)
    for (int j = 1; j <= Ny; j++)
        for (int i = 1; i <= Nx; i++) {
            double t = TT[IX(i, j)];
            double ap = ((t - T_crit) - T_act) / T_width;
            double am = ((t - T_crit) + T_act) / T_width;
            double thp = portable ? bgk_portable_tanh(ap) : tanh(ap);
            double thm = portable ? bgk_portable_tanh(am) : tanh(am);
            double react_plus = 0.5 * (1.0 + thp);
            double react_minus = 0.5 * (1.0 - thm);
            const double *pp = PHIP;
            double k_plus = sq(0.5 * (1.0 + pp[IX(i, j)]))
                          + sq(0.5 * (1.0 + pp[IX(i + 1, j)]))
                          + sq(0.5 * (1.0 + pp[IX(i, j + 1)]))
                          + sq(0.5 * (1.0 + pp[IX(i - 1, j)]))
                          + sq(0.5 * (1.0 + pp[IX(i, j - 1)]))
                          + sq(0.5 * (1.0 + pp[IX(i + 1, j + 1)]))
                          + sq(0.5 * (1.0 + pp[IX(i - 1, j + 1)]))
                          + sq(0.5 * (1.0 + pp[IX(i - 1, j - 1)]))
                          + sq(0.5 * (1.0 + pp[IX(i + 1, j - 1)]));
            double k_minus = sq(0.5 * (1.0 - pp[IX(i, j)]))
                           + sq(0.5 * (1.0 - pp[IX(i + 1, j)]))
                           + sq(0.5 * (1.0 - pp[IX(i, j + 1)]))
                           + sq(0.5 * (1.0 - pp[IX(i - 1, j)]))
                           + sq(0.5 * (1.0 - pp[IX(i, j - 1)]))
                           + sq(0.5 * (1.0 - pp[IX(i + 1, j + 1)]))
                           + sq(0.5 * (1.0 - pp[IX(i - 1, j + 1)]))
                           + sq(0.5 * (1.0 - pp[IX(i - 1, j - 1)]))
                           + sq(0.5 * (1.0 - pp[IX(i + 1, j - 1)]));
            k_plus = (k_plus / 8.0) * react_plus;
            k_minus = (k_minus / 8.0) * react_minus;
            double p0 = pp[IX(i, j)];
            PHI[IX(i, j)] = p0 + (f_plus * k_plus * (1.0 - p0) - f_minus * k_minus * (1.0 + p0));
        }
}

/* --------------------------------------------------------------- forces */

/* STEP_7/forces.f90:12-28.  `beta` is an implicit REAL(4). */
void orc_forces(orc_state *s)
{
    const int Nx = s->Nx, Ny = s->Ny;
    s->delta_T = s->T0 - s->T_in_sol;
    const float beta = (float)((1.0 - s->rho1 / s->rho0) / s->delta_T);
    const double delta_T = s->delta_T, stefan = s->stefan_number;
    const double grav = s->grav, omega_f = s->omega_f;
#pragma omp parallel for schedule(static)
    for (int j = 1; j <= Ny; j++)
        for (int i = 1; i <= Nx; i++) {
            size_t q = IX(i, j);
            double phi = PHI[q], phip = PHIP[q], rho = RHO[q];
            double t = TT[q] - (delta_T / stefan * (phi - phip) / 2.0);
            TT[q] = t;
            double forceY = rho * grav * (double)beta * t * (1.0 + phi / 2.0);
            double forceX = -(1.0 * UU[q] * (1.0 - phi) * 0.5);
            forceY = forceY - 1.0 * VV[q] * (1.0 - phi) * 0.5;
            UU[q] = UU[q] + forceX / (omega_f * rho);
            VV[q] = VV[q] + forceY / (omega_f * rho);
        }
}

/* ------------------------------------------------------------ collision */

/* STEP_7/collision.f90:14-152: regularized BGK for f and g. */
void orc_collision(orc_state *s)
{
    const int Nx = s->Nx, Ny = s->Ny;
    const double cs2 = s->cs2, omf = s->omega_f, omg = s->omega_g;
    const double m = -cs2, q1 = 1.0 - cs2;
    double C[9];
    for (int k = 0; k < 9; k++) C[k] = (0.5 * s->w[k]) / (cs2 * cs2);
#pragma omp parallel for schedule(static)
    for (int j = 1; j <= Ny; j++)
        for (int i = 1; i <= Nx; i++) {
            size_t q = IX(i, j);
            double fe[9], ge[9], d[9], e[9];
            float ft[9], gt[9]; /* implicit REAL(4): ft0..ft8, gt0..gt8 are undeclared */
            feq9(s->w, RHO[q], UU[q], VV[q], fe);
            feq9(s->w, TT[q], UU[q], VV[q], ge);
            for (int k = 0; k < 9; k++) { d[k] = FP(k)[q] - fe[k]; e[k] = GP(k)[q] - ge[k]; }
            double pxx = m * d[0] + q1 * d[1] + m * d[2] + q1 * d[3] + m * d[4]
                       + q1 * d[5] + q1 * d[6] + q1 * d[7] + q1 * d[8];
            double pyy = m * d[0] + m * d[1] + q1 * d[2] + m * d[3] + q1 * d[4]
                       + q1 * d[5] + q1 * d[6] + q1 * d[7] + q1 * d[8];
            double pxy = 1.0 * d[5] - 1.0 * d[6] + 1.0 * d[7] - 1.0 * d[8];
            double txx = m * e[0] + q1 * e[1] + m * e[2] + q1 * e[3] + m * e[4]
                       + q1 * e[5] + q1 * e[6] + q1 * e[7] + q1 * e[8];
            double tyy = m * e[0] + m * e[1] + q1 * e[2] + m * e[3] + q1 * e[4]
                       + q1 * e[5] + q1 * e[6] + q1 * e[7] + q1 * e[8];
            double txy = 1.0 * e[5] - 1.0 * e[6] + 1.0 * e[7] - 1.0 * e[8];
            ft[0] = fe[0] + C[0] * (m * pxx + m * pyy);
            ft[1] = fe[1] + C[1] * (q1 * pxx + m * pyy);
            ft[2] = fe[2] + C[2] * (m * pxx + q1 * pyy);
            ft[3] = fe[3] + C[3] * (q1 * pxx + m * pyy);
            ft[4] = fe[4] + C[4] * (m * pxx + q1 * pyy);
            ft[5] = fe[5] + C[5] * (q1 * pxx + q1 * pyy + 2.0 * pxy);
            ft[6] = fe[6] + C[6] * (q1 * pxx + q1 * pyy - 2.0 * pxy);
            ft[7] = fe[7] + C[7] * (q1 * pxx + q1 * pyy + 2.0 * pxy);
            ft[8] = fe[8] + C[8] * (q1 * pxx + q1 * pyy - 2.0 * pxy);
            gt[0] = ge[0] + C[0] * (m * txx + m * tyy);
            gt[1] = ge[1] + C[1] * (q1 * txx + m * tyy);
            gt[2] = ge[2] + C[2] * (m * txx + q1 * tyy);
            gt[3] = ge[3] + C[3] * (q1 * txx + m * tyy);
            gt[4] = ge[4] + C[4] * (m * txx + q1 * tyy);
            gt[5] = ge[5] + C[5] * (q1 * txx + q1 * tyy + 2.0 * txy);
            gt[6] = ge[6] + C[6] * (q1 * txx + q1 * tyy - 2.0 * txy);
            gt[7] = ge[7] + C[7] * (q1 * txx + q1 * tyy + 2.0 * txy);
            gt[8] = ge[8] + C[8] * (q1 * txx + q1 * tyy - 2.0 * txy);
            if (s->smooth) {
                /* the differentiable form: ft/gt kept in double */
                double fd[9], gd[9];
                fd[0] = fe[0] + C[0] * (m * pxx + m * pyy);
                fd[1] = fe[1] + C[1] * (q1 * pxx + m * pyy);
                fd[2] = fe[2] + C[2] * (m * pxx + q1 * pyy);
                fd[3] = fe[3] + C[3] * (q1 * pxx + m * pyy);
                fd[4] = fe[4] + C[4] * (m * pxx + q1 * pyy);
                fd[5] = fe[5] + C[5] * (q1 * pxx + q1 * pyy + 2.0 * pxy);
                fd[6] = fe[6] + C[6] * (q1 * pxx + q1 * pyy - 2.0 * pxy);
                fd[7] = fe[7] + C[7] * (q1 * pxx + q1 * pyy + 2.0 * pxy);
                fd[8] = fe[8] + C[8] * (q1 * pxx + q1 * pyy - 2.0 * pxy);
                gd[0] = ge[0] + C[0] * (m * txx + m * tyy);
                gd[1] = ge[1] + C[1] * (q1 * txx + m * tyy);
                gd[2] = ge[2] + C[2] * (m * txx + q1 * tyy);
                gd[3] = ge[3] + C[3] * (q1 * txx + m * tyy);
                gd[4] = ge[4] + C[4] * (m * txx + q1 * tyy);
                gd[5] = ge[5] + C[5] * (q1 * txx + q1 * tyy + 2.0 * txy);
                gd[6] = ge[6] + C[6] * (q1 * txx + q1 * tyy - 2.0 * txy);
                gd[7] = ge[7] + C[7] * (q1 * txx + q1 * tyy + 2.0 * txy);
                gd[8] = ge[8] + C[8] * (q1 * txx + q1 * tyy - 2.0 * txy);
                for (int k = 0; k < 9; k++) {
                    F(k)[q] = fd[k] - omf * (fd[k] - fe[k]);
                    G(k)[q] = gd[k] - omg * (gd[k] - ge[k]);
                }
                continue;
            }
            for (int k = 0; k < 9; k++) {
                F(k)[q] = (double)ft[k] - omf * ((double)ft[k] - fe[k]);
                G(k)[q] = (double)gt[k] - omg * ((double)gt[k] - ge[k]);
            }
        }
}

/* -------------------------------------------------------------- moments */

/* STEP_7/moments.f90:8-27 */
void orc_moments(orc_state *s)
{
    const int Nx = s->Nx, Ny = s->Ny;
#pragma omp parallel for schedule(static)
    for (int j = 1; j <= Ny; j++)
        for (int i = 1; i <= Nx; i++) {
            size_t q = IX(i, j);
            double f0 = F(0)[q], f1 = F(1)[q], f2 = F(2)[q], f3 = F(3)[q], f4 = F(4)[q];
            double f5 = F(5)[q], f6 = F(6)[q], f7 = F(7)[q], f8 = F(8)[q];
            double rho = f0 + f1 + f2 + f3 + f4 + f5 + f6 + f7 + f8;
            double irho = 1.0 / rho;
            double temp_T = G(0)[q] + G(1)[q] + G(2)[q] + G(3)[q] + G(4)[q]
                          + G(5)[q] + G(6)[q] + G(7)[q] + G(8)[q];
            double temp_u = irho * (f1 - f3 + f5 - f6 - f7 + f8);
            double temp_v = irho * (f2 - f4 + f5 + f6 - f7 - f8);
            RHO[q] = rho;
            TT[q] = (temp_T + T2[q]) * 0.5;
            UU[q] = (temp_u + U2[q]) * 0.5;
            VV[q] = (temp_v + V2[q]) * 0.5;
        }
}

/* STEP_7/main.f90:60-69 */
void orc_step(orc_state *s, int n)
{
    for (int t = 0; t < n; t++) {
        s->it += 1;
        orc_bc_f(s);
        orc_bc_g(s);
        orc_streaming(s);
        orc_moments_pre(s);
        orc_phase_field(s);
        orc_forces(s);
        orc_collision(s);
        orc_moments(s);
    }
}

/* -------------------------------------------------------------- outputs */

/* Fortran Ew.d edit descriptor: 0.ddddddE+xx, right-justified in w. */
static void fmt_E(char *out, int w, int d, double x)
{
    char body[160];
    if (x == 0.0) {
        snprintf(body, sizeof body, "0.%0*dE+00", d, 0);
    } else {
        double ax = fabs(x);
        char tmp[80];
        snprintf(tmp, sizeof tmp, "%.*e", d - 1, ax); /* d.ddd e+xx */
        int ex = atoi(strchr(tmp, 'e') + 1);
        char digits[80]; int nd = 0;
        for (const char *c = tmp; *c && *c != 'e'; c++) if (*c >= '0' && *c <= '9') digits[nd++] = *c;
        digits[nd] = 0;
        int e10 = ex + 1;
        if (e10 >= -99 && e10 <= 99)
            snprintf(body, sizeof body, "%s0.%sE%c%02d", x < 0 ? "-" : "", digits, e10 < 0 ? '-' : '+', abs(e10));
        else
            snprintf(body, sizeof body, "%s0.%s%c%03d", x < 0 ? "-" : "", digits, e10 < 0 ? '-' : '+', abs(e10));
    }
    snprintf(out, 64, "%*.*s", w, 60, body);
}

/* gfortran list-directed REAL(8): 17 significant digits. */
static void fmt_list(char *out, double x)
{
    double ax = fabs(x);
    if (x != 0.0 && (ax < 0.1 || ax >= 1e16)) {
        char tmp[64];
        snprintf(tmp, sizeof tmp, "%.16E", x);
        char *e = strchr(tmp, 'E');
        int ex = atoi(e + 1);
        *e = 0;
        snprintf(out, 64, "%s E%c%03d", tmp, ex < 0 ? '-' : '+', abs(ex));
        /* gfortran prints no blank before E */
        char *b = strchr(out, ' ');
        if (b) memmove(b, b + 1, strlen(b));
    } else {
        int intdig = ax >= 1.0 ? (int)floor(log10(ax)) + 1 : 0;
        int frac = 17 - (intdig > 0 ? intdig : 0);
        if (intdig == 0) frac = 17;
        snprintf(out, 64, "%.*f", frac, x);
    }
}

int orc_open_outputs(orc_state *s, const char *dir)
{
    snprintf(s->dir, sizeof s->dir, "%s", dir);
    char path[1200];
#define OPEN_UNIT(fp, name, mode) do { snprintf(path, sizeof path, "%s/%s", dir, name); fp = fopen(path, mode); if (!fp) return -1; } while (0)
    OPEN_UNIT(s->u64, "fort.64", "w");
    OPEN_UNIT(s->u69, "fort.69", "w");
    OPEN_UNIT(s->u164, "non-dim_bulk_numbers.dat", "w");
    OPEN_UNIT(s->u666, "fort.666", "w");
    OPEN_UNIT(s->u667, "fort.667", "w");
    OPEN_UNIT(s->u668, "fort.668", "w");
#undef OPEN_UNIT
    return 0;
}

void orc_close_outputs(orc_state *s)
{
    FILE **u[] = {&s->u64, &s->u69, &s->u164, &s->u666, &s->u667, &s->u668};
    for (size_t k = 0; k < sizeof u / sizeof u[0]; k++)
        if (*u[k]) { fclose(*u[k]); *u[k] = NULL; }
}

/* STEP_7/diag.f90:15-116 */
void orc_diag(orc_state *s)
{
    const int Nx = s->Nx, Ny = s->Ny;
    long long Ny_2 = Ny / 2, i_liq = Nx / 20, i_sol = Nx - Nx / 20;
    double Delta_Temp = s->T0 - s->T_in_sol;
    if (PHI[IX(i_liq, Ny_2)] < 1.0) i_liq = 2;
    if (PHI[IX(i_sol, Ny_2)] > 0.0) i_sol = Nx - 1;
    (void)i_liq; (void)i_sol;
    double beta_gras = (s->rho0 / s->rho1 - 1.0) / Delta_Temp;
    int32_t ny3 = (int32_t)((uint32_t)Ny * (uint32_t)Ny * (uint32_t)Ny);
    double Gras = s->grav * beta_gras * Delta_Temp * (double)ny3 / (s->kvisc * s->kvisc);
    double Pr = (2.0 * s->tau_f - 1.0) / (2.0 * s->tau_g - 1.0);
    double Ray = Pr * Gras;
    double Fou = s->alpha * (double)s->it / (double)(Ny * Ny);
    double theta = s->stefan_number * Fou;
    double theta1 = pow(Ray, -0.5);
    double theta2 = (double)(Nx / Ny) * pow(Ray, -0.25);
    if (s->u69) {
        char b[8][64];
        fmt_list(b[0], beta_gras); fmt_list(b[1], s->grav); fmt_list(b[2], Gras);
        fmt_list(b[3], Delta_Temp); fmt_list(b[4], Pr); fmt_list(b[5], Ray);
        fmt_list(b[6], Fou); fmt_list(b[7], theta);
        fprintf(s->u69, " beta_gras, grav, Gras, Delta_Temp, Pr, Ray, Fou, theta\n");
        fprintf(s->u69, " ");
        for (int k = 0; k < 8; k++) fprintf(s->u69, " %s", b[k]);
        fprintf(s->u69, "\n ---------------------------------------------\n");
        fflush(s->u69);
    }
    double Nus = pow(2.0 * theta, -0.5)
               + (0.35 * pow(Ray, 0.25) - pow(2.0 * theta, -0.5))
               * pow(1.0 + pow(0.0175 * pow(Ray, 0.75) * pow(theta, 1.5), -2.0), -0.5);
    double Nus_comp = 0.0;
    for (int j = 1; j <= Ny; j++)
        Nus_comp = Nus_comp + (double)Ny * ((s->Tin - TT[IX(2, j)]) / 2.0) / Delta_Temp;
    Nus_comp = Nus_comp / (double)Ny;
    double Nus_comp_2 = 0.0;
    for (int j = 1; j <= Ny; j++) {
        double grad_T = fabs((-(3.0 * TT[IX(1, j)]) + 4.0 * TT[IX(2, j)] - TT[IX(3, j)]) / 2.0);
        Nus_comp_2 = Nus_comp_2 + (double)Ny * grad_T / Delta_Temp;
    }
    Nus_comp_2 = Nus_comp_2 / (double)Ny;
    if (s->it % 100 == 0) {
        double melt = 0.0;
        for (int j = 1; j <= Ny; j++)
            for (int i = 1; i <= Nx; i++)
                if (PHI[IX(i, j)] > 0.0) melt = melt + 1.0;
        melt = melt / (double)(Nx * Ny);
        if (theta <= theta1) {
            s->diag_melt_front = (double)Ny / pow(2.0 * theta, -0.5);
            s->diag_melt_front_expected = (double)Ny / Nus;
        } else if (theta > theta1 && theta < theta2) {
            double mf = 0.0;
            for (int j = 1; j <= Ny; j++)
                for (int i = 1; i <= Nx; i++)
                    if (PHI[IX(i, j)] == 0.0) mf = mf + (double)i;
            s->diag_melt_front = mf / (double)Ny;
            s->diag_melt_front_expected = (double)Ny * theta * pow(Ray, 0.25);
        }
        if (s->u164) {
            double vals[11] = {theta, Nus, Nus_comp, Nus_comp_2, melt, s->diag_melt_front,
                               s->diag_melt_front_expected, Gras, Pr, Ray, Fou};
            fprintf(s->u164, "%8d", s->it);
            for (int k = 0; k < 11; k++) { char b[64]; fmt_E(b, 13, 6, vals[k]); fprintf(s->u164, " %s", b); }
            fprintf(s->u164, "\n");
            fflush(s->u164);
        }
    }
}

static void write_row5(FILE *f, int idx, double a, double b, double c, double d, double e)
{
    double v[5] = {a, b, c, d, e};
    fprintf(f, "%8d", idx);
    for (int k = 0; k < 5; k++) { char s[64]; fmt_E(s, 14, 6, v[k]); fprintf(f, "%s ", s); }
    fprintf(f, "\n");
}

/* STEP_7/probe.f90:5-12 */
void orc_probe(orc_state *s)
{
    if (!s->u666) return;
    size_t q = IX(s->Nx / 2, s->Ny / 2);
    write_row5(s->u666, s->it, UU[q], VV[q], RHO[q], TT[q], PHI[q]);
    fflush(s->u666);
}

/* STEP_7/prof_x.f90:5-16 */
void orc_prof_x(orc_state *s)
{
    if (!s->u667) return;
    fprintf(s->u667, "# t=%7d\n", s->it);
    for (int i = 1; i <= s->Nx; i++) {
        size_t q = IX(i, s->Ny / 2);
        write_row5(s->u667, i, UU[q], VV[q], RHO[q], TT[q], PHI[q]);
    }
    fprintf(s->u667, "\n\n");
    fflush(s->u667);
}

/* STEP_7/prof_y.f90:5-16 */
void orc_prof_y(orc_state *s)
{
    if (!s->u668) return;
    fprintf(s->u668, "# t=%7d\n", s->it);
    for (int j = 1; j <= s->Ny; j++) {
        size_t q = IX(s->Nx / 2, j);
        write_row5(s->u668, j, UU[q], VV[q], RHO[q], TT[q], PHI[q]);
    }
    fprintf(s->u668, "\n\n");
    fflush(s->u668);
}

void orc_sums(orc_state *s, double out[4])
{
    double m = 0.0, t = 0.0, p = 0.0, c = 0.0;
    for (int j = 1; j <= s->Ny; j++)
        for (int i = 1; i <= s->Nx; i++) {
            size_t q = IX(i, j);
            m = m + RHO[q];
            t = t + TT[q];
            p = p + PHI[q];
            if (PHI[q] > 0.0) c = c + 1.0;
        }
    out[0] = m; out[1] = t; out[2] = p; out[3] = c;
}

/* STEP_7/field_check.f90:9-24 */
void orc_field_check(orc_state *s)
{
    double sums[4];
    orc_sums(s, sums);
    double n = (double)(s->Nx * s->Ny);
    double mass_aver = sums[0] / n, temp_aver = sums[1] / n, phi_aver = sums[2] / n;
    if (s->u64) {
        char a[64], b[64], c[64];
        fmt_E(a, 16, 8, mass_aver); fmt_E(b, 16, 8, temp_aver); fmt_E(c, 16, 8, phi_aver);
        fprintf(s->u64, "%8d %s %s %s \n", s->it, a, b, c);
        fflush(s->u64);
    }
}

/* STEP_7/out2d.f90:8-62: ASCII VTK structured grid including the halos. */
void orc_out2d(orc_state *s)
{
    char path[1200];
    snprintf(path, sizeof path, "%s/Output_%08d.vtk", s->dir[0] ? s->dir : ".", s->it);
    FILE *f = fopen(path, "w");
    if (!f) return;
    const int Nx = s->Nx, Ny = s->Ny;
    fprintf(f, "# vtk DataFile Version 2.0\nGriglia strutturata\nASCII\nDATASET STRUCTURED_GRID\n");
    fprintf(f, "DIMENSIONS%8d%8d%8d\n", Nx + 2, Ny + 2, 1);
    fprintf(f, "POINTS%15d float\n", (Nx + 2) * (Ny + 2));
    for (int l = 0; l <= Ny + 1; l++)
        for (int i = 0; i <= Nx + 1; i++) fprintf(f, "%12d%12d%12d\n", i, l, 1);
    fprintf(f, "POINT_DATA%15d\n", (Nx + 2) * (Ny + 2));
    char b[64], c[64];
    fprintf(f, "SCALARS DENSITY float 1\nLOOKUP_TABLE default\n");
    for (int l = 0; l <= Ny + 1; l++)
        for (int i = 0; i <= Nx + 1; i++) { fmt_list(b, RHO[IX(i, l)]); fprintf(f, "   %s     \n", b); }
    fprintf(f, "SCALARS Temperature float 1\nLOOKUP_TABLE default\n");
    for (int l = 0; l <= Ny + 1; l++)
        for (int i = 0; i <= Nx + 1; i++) { fmt_list(b, TT[IX(i, l)]); fprintf(f, "   %s     \n", b); }
    fprintf(f, "SCALARS Phase_Field float 1\nLOOKUP_TABLE default\n");
    for (int l = 0; l <= Ny + 1; l++)
        for (int i = 0; i <= Nx + 1; i++) { fmt_list(b, PHI[IX(i, l)]); fprintf(f, "   %s     \n", b); }
    fprintf(f, "VECTORS VELOCITY float\n");
    for (int l = 0; l <= Ny + 1; l++)
        for (int i = 0; i <= Nx + 1; i++) {
            fmt_list(b, UU[IX(i, l)]); fmt_list(c, VV[IX(i, l)]);
            fprintf(f, "   %s        %s        0.0000000000000000     \n", b, c);
        }
    fclose(f);
}

/* STEP_7/main.f90:18-122 (restart path excluded: dump_out is commented out
 * in the reference and dump_in does not restore phi). */
int orc_main(const char *dir, int nthreads, int tanh_mode, int heat)
{
    char path[1200];
    snprintf(path, sizeof path, "%s/input.dat", dir);
    orc_params p;
    if (orc_read_input(path, &p)) return -1;
    orc_set_threads(nthreads);
    orc_state *s = orc_create(&p);
    if (!s) return -2;
    s->tanh_mode = tanh_mode;
    s->heat = heat;
    if (orc_open_outputs(s, dir)) { orc_destroy(s); return -3; }
    snprintf(path, sizeof path, "%s/log.dat", dir);
    FILE *lg = fopen(path, "w");
    if (lg) { fprintf(lg, " iteration    mass\n ====================\n"); fclose(lg); }
    s->it = 0;
    s->it0 = 1;
    orc_initialization(s);
    s->deltaOut = s->iter / s->noutput;
    s->itOut = s->deltaOut;
    orc_out2d(s);
    for (int it = s->it0; it <= s->iter; it++) {
        orc_step(s, 1);
        if (it % 1000 == 0) {
            orc_diag(s);
            orc_probe(s);
            orc_prof_x(s);
            orc_prof_y(s);
            orc_field_check(s);
            lg = fopen(path, "a");
            if (lg) { fprintf(lg, "%8d %10.4f\n", it, s->mass); fclose(lg); }
        }
        if (it == s->itOut || it == s->iter) {
            orc_out2d(s);
            char np[1200];
            snprintf(np, sizeof np, "%s/Nusselt.dat", dir);
            FILE *nf = fopen(np, "w");
            if (nf) {
                for (int i = 0; i < s->samplex; i++)
                    fprintf(nf, "%8d %10.4f %10.4f %10.4f\n", i + 1, s->Nu[i], s->Nu2[i], s->Nu3[i]);
                fclose(nf);
            }
            s->itOut = s->itOut + s->deltaOut;
        }
    }
    orc_destroy(s);
    return 0;
}

/* The check-mode tanh, exported so tests can compare it with libm. */
double orc_portable_tanh(double x) { return bgk_portable_tanh(x); }
