/*
 * bgk_internal.h -- device state and kernel launchers shared by the CUDA
 * translation units of libbgkpcm.  Not part of the public ABI.
 *
 * Device data layout (FP64 form)
 *  - Populations: compact interior planes, no halo.  A buffer holds the nine
 *    planes of one distribution; plane k, row y (0..Ny-1), column x
 *    (0..Nx-1) is at k*plane + y*P + x, P = Nx rounded up to 32 elements so
 *    that every row starts on a 256-byte boundary.  f and g are kept twice
 *    (A/B ping-pong): a step pulls from buffer `cur` and writes buffer
 *    `cur^1`.  The reference's f/g halos are not stored: with the no-slip
 *    code 4 every halo value streaming reads is a function of the interior
 *    (bounce-back, STEP_7/BC_f.f90:62-68,101-107,125-136,181-192) or of a
 *    per-row boundary array (STEP_7/BC_g.f90:7-31), except the two corner
 *    populations f6(Nx+1,0) and f7(Nx+1,Ny+1) that BC_f never writes; those
 *    two numbers are kept in `corner`.  With any other wall code the f halo
 *    cells carry state of their own (periodic copies, inflow equilibria,
 *    values that persist from step to step), so they are kept in a ring
 *    (`fring`, see ring_idx) that a boundary kernel updates before each step
 *    exactly as BC_f does, and the step pulls from it.
 *  - phi: compact interior plane, A/B ping-pong (its 3x3 stencil reads the
 *    previous step's values).  Columns 0 and Nx+1 are frozen boundary values
 *    (phiW/phiE per row); rows 0 and Ny+1 are copies of rows 1 and Ny.
 *  - tcol: T(Nx, j) from the previous step's `moments`, read by the east
 *    boundary of g (STEP_7/BC_g.f90:21-31); A/B ping-pong.
 *  - Mirrors: rho, T, u, v, phi in the reference layout (Nx+2)x(Ny+2) with
 *    halos.  The fused kernel writes their interiors only on the last two
 *    steps of a bgk_step call; a small kernel applies the reference's halo
 *    rules before the last one, so downloads see exactly what the
 *    reference's arrays hold after `moments`.
 *  - Staged state (allocated on first use): the reference's remaining arrays
 *    f, g, fp, gp (with halos), rho2, T2, u2, v2, phi_prec; the mirrors double
 *    as the staged rho, T, u, v, phi.
 */
#ifndef BGK_INTERNAL_H
#define BGK_INTERNAL_H

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "../../include/bgk_pcm.h"

namespace bgk {

/* Physics constants in the form the kernels use them.  Every value is
 * computed on the host with the reference's expression (file:line beside
 * each), so kernels reproduce its roundings. */
struct Consts {
    int Nx, Ny;
    double w[9];           /* setup.f90:79-87                                */
    double cs2;            /* setup.f90:99                                   */
    double m_cs2;          /* (  - cs2)        collision.f90:34              */
    double q_cs2;          /* (1 - cs2)        collision.f90:35              */
    double C[9];           /* (0.5*w_k)/(cs2*cs2) collision.f90:84-100       */
    double omega_f, omega_g;         /* setup.f90:102-103                   */
    double T_crit, T_act, T_width;   /* phase_field.f90:11-12, input        */
    double f_plus, f_minus;          /* phase_field.f90:14-15               */
    double dts;            /* delta_T/stefan_number   forces.f90:15          */
    double grav;
    double beta;           /* REAL(4) beta promoted   forces.f90:13          */
    double Tin;            /* initialization.f90:9 (scalar hot wall)        */
    double u0, v0;         /* initialization.f90:11-12                      */
    double rho0, rho1, T0, T_in_sol;
    int interf;            /* initialization.f90:5                           */
    int heat;              /* BGK_HEAT_* bits (STEP_DOCONCURRENT's options)  */
};

/* Device pointers of one fused step. Ref-layout mirrors use pitch NX2. */
template <typename T>
struct StepPtrs {
    const T *fin, *gin;
    T *fout, *gout;
    const T *phin;
    T *phout;
    const double *tcin;
    double *tcout;
    const double *gW;      /* [3][Ny]  g1,g5,g8 west values, row j at j-1   */
    const double *pE;      /* [3][Ny]  east equilibrium polynomials k=3,6,7 */
    const double *phiW, *phiE;   /* [Ny]                                    */
    const double *tin;     /* per-row hot wall [Ny], or null (scalar Tin)   */
    double *mrho, *mT, *mu, *mv, *mphi;  /* mirrors, or null               */
    const double *ring;    /* f halo ring [9][ring_len] (walls other than 4) */
    long long ring_len;
    long long plane;       /* elements per population plane                */
    int P;                 /* row pitch (elements)                          */
    int NX2;               /* mirror pitch                                   */
};

/* Offset of halo cell (i, j) of the reference's (0:Nx+1, 0:Ny+1) layout in
 * one population's ring: column 0 (rows 0..Ny+1, corners included), column
 * Nx+1 (rows 0..Ny+1), row 0 (columns 1..Nx), row Ny+1 (columns 1..Nx). */
__host__ __device__ inline long long ring_idx(int Nx, int Ny, int i, int j)
{
    if (i == 0) return j;
    if (i == Nx + 1) return (long long)(Ny + 2) + j;
    if (j == 0) return 2LL * (Ny + 2) + (i - 1);
    return 2LL * (Ny + 2) + Nx + (i - 1);
}
__host__ __device__ inline long long ring_length(int Nx, int Ny) { return 2LL * (Ny + 2) + 2LL * Nx; }

struct LowpScale {
    float sf, sg;          /* FP16 form: stored = deviation * s            */
    float inv_sf, inv_sg;
};

} // namespace bgk

struct bgk_ctx {
    bgk_params p;
    bgk_options opt;
    bgk::Consts c;
    int dev;
    cudaStream_t stream;
    int Nx, Ny, NX2, NY2;
    size_t A;              /* (Nx+2)*(Ny+2)                                 */
    int P;                 /* compact pitch                                 */
    long long plane;       /* Ny*P                                          */
    size_t esz;            /* bytes per stored population element           */
    size_t phisz;          /* bytes per stored phi element (4 or 8)          */
    int it;

    /* fused state (each buffer has a 256-byte guard on both sides: the
     * shared-memory pipeline copies row segments that start 16 bytes before a
     * band and may end 16 bytes after a row) */
    void *fbuf[2], *gbuf[2], *phibuf[2];
    void *raw[6];          /* allocation bases of fbuf, gbuf, phibuf        */
    int *errflag;          /* device: nonzero after a bounded wait gave up   */
    int cur;
    double *tcol[2];
    double *gW, *pE, *phiW, *phiE;
    double *tin_rows;      /* device [Ny] or null                           */
    double *tright;        /* BGK_HEAT_RIGHT: [Ny] of Tin, the east wall's T  */
                           /* column in place of the lagged T(Nx,j)          */
    double *tin_host;      /* host copy [Ny] or null                        */
    bool bc_dirty;
    bgk::LowpScale scale;

    /* reference-layout mirrors / staged arrays */
    double *mrho, *mT, *mu, *mv, *mphi;
    double *sf[9], *sg[9], *sfp[9], *sgp[9];
    double *sphip, *srho2, *sT2, *su2, *sv2;
    bool staged_alloc;
    int mode;              /* 0 = fused state is current, 1 = staged        */
    int stage_pos;         /* 0 at a step boundary                          */
    bool pristine;         /* nothing changed since bgk_initialize           */

    double *scratch;       /* A doubles                                     */
    double *red;           /* reduction partials; red[0..3] = results        */
    double *corner;        /* f6(Nx+1,0), f7(Nx+1,Ny+1) (never written by BC_f) */
    /* launch-bound grids (up to 2^21 nodes): the plain steps of a call
     * replay a captured CUDA graph of GRAPH_STEPS steps, one per starting
     * buffer (BGK_GRAPH=0 disables) */
    cudaGraphExec_t step_graph[2];
    bool graph_on, graph_failed;
    bool ring;             /* a wall other than code 4: f halos in fring     */
    double *fring;         /* [9][ring_len] f halo cells (ring_idx), or null */
    long long ring_len;
    int red_n;
    double *pinned;        /* small pinned host buffer                      */

    /* launch shape of the fused kernels: strip height (0 = automatic) and
     * L2 prefetch distance in rows (0 = off); BGK_STRIP_H / BGK_PREFETCH_ROWS
     * override the defaults at bgk_create */
    int tune_H, tune_pf;
    /* kernel choice: 1 = shared-memory pipeline (default), 0 = register
     * pulls; pipeline depth and CTAs per SM (BGK_PIPE, BGK_PIPE_D,
     * BGK_PIPE_CTAS) */
    int tune_pipe, tune_D, tune_ctas, nsm;
    int tune_flow;         /* 1: reduced-precision steps between outputs in one
                            * dataflow launch (BGK_FLOW)                    */
    void *flow_buf;        /* its ticket counter and per-tile step counts   */
    int flow_stall;        /* test of the error path: dependency waits of a
                            * dataflow launch never succeed (BGK_FLOW_STALL) */
    size_t flow_bytes;
    void *adj_ws;          /* adjoint workspace kept between bgk_adjoint_run calls */
    size_t adj_ws_bytes;
};

namespace bgk {

/* kernels_f64.cu (compiled with --fmad=false: the reference's roundings) */
/* T column the step's east g halos use: T(Nx,j) of the previous step
 * (tcol[buf]), or the constant Tin column with BGK_HEAT_RIGHT */
inline const double *east_tcol(const bgk_ctx *c, int buf) { return c->tright ? c->tright : c->tcol[buf]; }

cudaError_t launch_init_f64(bgk_ctx *c);
cudaError_t launch_bc_prep(bgk_ctx *c);
cudaError_t launch_ring_bc(bgk_ctx *c);            /* BC_f + BC_g halos + bc_prep, walls other than 4 */
cudaError_t launch_macro_halos(bgk_ctx *c);
/* moments: write rho, T, u, v, phi of every node (the last step of a call);
 * edge_halos: write instead the halo cells those fields get from this step's
 * edge nodes (the step before the last of a call, FP64 pipeline only) */
cudaError_t launch_fused_f64(bgk_ctx *c, bool moments, bool edge_halos = false);
cudaError_t launch_flow_f64(bgk_ctx *c, int nsteps);     /* dataflow steps, no moments */
cudaError_t launch_staged(bgk_ctx *c, int stage);   /* 1..8 in main.f90 order */
cudaError_t launch_compact_to_staged(bgk_ctx *c);
cudaError_t launch_staged_to_compact(bgk_ctx *c);
cudaError_t launch_ref_to_compact(bgk_ctx *c, int field, const double *ref);
cudaError_t launch_compact_to_ref(bgk_ctx *c, int field, double *ref, int which);
cudaError_t launch_field_sums(bgk_ctx *c, int j0, int nrows);   /* -> c->red[0..3] */
size_t rows_bytes(const bgk_ctx *c, int nrows);                 /* packed slab halo rows */
cudaError_t launch_rows_copy(bgk_ctx *c, int j0, int nrows, void *buf, bool unpack);
cudaError_t launch_fused_f64_ptrs(bgk_ctx *c, const double *fin, const double *gin, const double *phin,
                                  const double *tcin, double *fout, double *gout, double *phout, double *tcout);

/* kernels_fast.cu (FMA allowed): FP64-FMA, FP32 and FP16 forms */
cudaError_t launch_fused_fast(bgk_ctx *c, bool moments, bool edge_halos = false);
cudaError_t launch_init_lowp(bgk_ctx *c);
cudaError_t launch_flow_lowp(bgk_ctx *c, int nsteps);   /* dataflow steps, no moments */
cudaError_t launch_flow_fast(bgk_ctx *c, int nsteps);   /* FMA FP64 or reduced precision */

} // namespace bgk

/* capi.cu helpers shared with adjoint.cu */
int bgk_internal_fail(int code, const char *msg);
int bgk_internal_prepare_fused(bgk_ctx *c);   /* device, fused state, BC arrays */
int bgk_internal_advance(bgk_ctx *c, int nsteps); /* fused steps, no mirror writes */

#endif
