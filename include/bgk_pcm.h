/*
 * bgk_pcm.h -- C ABI of the B200 (sm_100a) implementation of the BGK_PCM
 * time step: D2Q9 double-distribution thermal lattice Boltzmann (f = flow,
 * g = temperature), regularized BGK collision, buoyancy + solid drag forcing
 * and the kinetic phase-field update with latent-heat feedback.
 *
 * The reference (giacomofalcucci/BGK_PCM, STEP_7/) has no library interface:
 * its boundary is a set of argument-less Fortran subroutines that mutate the
 * module `shared` (STEP_7/shared.f90:1-104), called in a fixed order from
 * STEP_7/main.f90:60-69.  Each entry point below replaces one of them (cited
 * per function); bgk_step replaces the whole sequence with one fused kernel
 * per time step.  The only C interop precedent in the reference is
 * STEP_7/get_mem.c:23 bound by STEP_7/get_mem_mod.f90:7, and these functions
 * follow the same style: plain C types, bind(c)-friendly.
 *
 * Conventions
 *  - Every function returns BGK_OK (0) or a negative BGK_ERR_* code and never
 *    exits, aborts or traps; bgk_last_error() describes the last failure of
 *    the calling thread.
 *  - Host arrays use the reference layout: a field is (0:Nx+1, 0:Ny+1)
 *    column-major (x fastest), halos included, with a leading dimension
 *    ld >= Nx+2 (ld = Nx+2 for a Fortran array declared like the reference's).
 *  - A context owns its device buffers and one CUDA stream; it is used by one
 *    host thread at a time.  Calls that return data synchronise the stream;
 *    bgk_step and the stage entry points only enqueue work.
 *  - There is no CPU fallback: a context can only be created on a CUDA device
 *    of compute capability 10.0 (B200), and every step runs on it.
 */
#ifndef BGK_PCM_H
#define BGK_PCM_H

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------ status codes */
#define BGK_OK               0
#define BGK_ERR_ARG         -1  /* invalid argument                              */
#define BGK_ERR_UNSUPPORTED -2  /* valid input the chosen path does not implement */
#define BGK_ERR_CUDA        -3  /* CUDA runtime or launch failure                 */
#define BGK_ERR_OOM         -4  /* device or host allocation failed               */
#define BGK_ERR_STATE       -5  /* call not allowed in the current state          */
#define BGK_ERR_IO          -6  /* file could not be read or written              */
#define BGK_ERR_NONFINITE   -7  /* a reduction found NaN or Inf                    */

/* ------------------------------------------------------------- parameters */
/* The 21 input.dat values in file order (STEP_7/setup.f90:7-31). */
typedef struct bgk_params {
    int iter, noutput, dump, Nx, Ny;
    double Re, rho0, rho1, tau_f, tau_g, T0, T_in_sol, grav, eps,
           stefan_number, T_width, length;
    int westBC, eastBC, northBC, southBC;
} bgk_params;

/* Storage/arithmetic form of the populations. */
#define BGK_PREC_F64   0  /* plain FP64 (the reference's mykind = dp)                  */
#define BGK_PREC_F32   1  /* FP32 deviations f_i - w_i*rho0, g_i - w_i*T0, FP32 math    */
#define BGK_PREC_F16   2  /* FP16 deviations with a per-field scale, FP32 math          */
#define BGK_PREC_F32X  3  /* FP32 deviations, FP64 math, phi in FP64                   */

/* tanh used by the phase-field selector (STEP_7/phase_field.f90:20-21) in
 * the FP64 forms (BGK_PREC_F64, BGK_PREC_F32X).  The default, portable tanh
 * (bgk_portable_tanh.h, a few ulp from libm) is evaluated the same way by the
 * CPU oracle, so the FP64 step equals it bit for bit; it costs 1.4-2.5 % of
 * the step's throughput on B200 against CUDA's tanh.  The FP32 and FP16 forms
 * always use CUDA's tanhf. */
#define BGK_TANH_PORTABLE 0  /* bit-identical to the CPU oracle (default)          */
#define BGK_TANH_DEVICE   1  /* CUDA's tanh                                         */

typedef struct bgk_options {
    int precision;   /* BGK_PREC_*                                              */
    int tanh_mode;   /* BGK_TANH_* (FP64 forms)                                 */
    int fma;         /* FP64 only: 0 = the reference's exact operation order    */
                     /* (no fused multiply-add); 1 = FMA-contracted variant      */
    int device;      /* CUDA device ordinal, or -1 for the current device        */
    int smooth;      /* FP64 only: 0 = the reference's roundings, including the  */
                     /* REAL(4) temporaries ft0..ft8 / gt0..gt8 of               */
                     /* STEP_7/collision.f90:84-120 (implicitly typed); 1 = keep */
                     /* them in double, which makes the step a smooth function   */
                     /* of its inputs (the form the adjoint differentiates)      */
    int heat;        /* BGK_HEAT_* bits: the heated wall (0 = west, STEP_7)      */
} bgk_options;

/* Heating options of the reference's STEP_DOCONCURRENT variant, which it
 * selects with preprocessor macros at build time; here they are bits of
 * bgk_options.heat, chosen at bgk_create:
 *  BGK_HEAT_RIGHT  (FROMRIGHT, STEP_DOCONCURRENT/BC_g.f90:13-45 and
 *                  initialization.f90:30-60,128-133,208-214): the east wall
 *                  is held at Tin and the west wall is zero-gradient in T
 *                  (its g1, g5, g8 use the polynomials of directions 3, 7, 6,
 *                  with T(1,j) of the previous step); the initial liquid
 *                  strip is T/rho at columns >= Nx-interf+1 and phi at
 *                  columns >= Nx-interf.  FP64 forms only.
 *  BGK_HEAT_BOTTOM (FROMBOTTOM, initialization.f90:16-28,123-127): the
 *                  initial liquid layer is rows 0..interf (interf = Nx/40);
 *                  the walls are STEP_7's.  Its T buffer loop `T(i,0) = Tin,
 *                  i = 0..Ny+1` runs along x and, with Ny > Nx, on into row
 *                  1; that is reproduced.  Every precision form.
 * Both bits = both macros defined (T/rho layer from FROMBOTTOM, phi strip and
 * walls from FROMRIGHT).  The packed-row exchange (the y-slab
 * decomposition) refuses both bits; bgk_advance and the adjoint refuse
 * BGK_HEAT_RIGHT. */
#define BGK_HEAT_WEST    0
#define BGK_HEAT_RIGHT   1
#define BGK_HEAT_BOTTOM  2

/* ----------------------------------------------------------------- fields */
/* Field ids for bgk_upload / bgk_download; the names are the reference's
 * arrays (STEP_7/shared.f90:36-79). */
#define BGK_FIELD_F0        0   /* f0..f8   =  0..8  */
#define BGK_FIELD_G0        9   /* g0..g8   =  9..17 */
#define BGK_FIELD_RHO      18
#define BGK_FIELD_T        19
#define BGK_FIELD_U        20
#define BGK_FIELD_V        21
#define BGK_FIELD_PHI      22
#define BGK_FIELD_PHI_PREC 23
#define BGK_FIELD_RHO2     24
#define BGK_FIELD_T2       25
#define BGK_FIELD_U2       26
#define BGK_FIELD_V2       27
#define BGK_FIELD_FP0      28   /* fp0..fp8 = 28..36 */
#define BGK_FIELD_GP0      37   /* gp0..gp8 = 37..45 */
#define BGK_NFIELDS        46

typedef struct bgk_ctx bgk_ctx;

/* Thread-local description of the last failure ("" if none). */
const char *bgk_last_error(void);

/* Parse input.dat (list-directed "label value" records, d/D exponents and
 * trailing comments accepted).  Replaces STEP_7/setup.f90:5-32. */
int bgk_read_input(const char *path, bgk_params *out);

/* Allocate device state and derive the constants (weights, omega_f, omega_g,
 * kvisc, alpha).  Replaces STEP_7/setup.f90:34-115.  opt may be NULL
 * (FP64, portable tanh, exact order, current device, heated west wall: the
 * same as a zero-initialized bgk_options).  Walls: the FP64 step (fused and staged)
 * runs every BC_f code of STEP_7/BC_f.f90 (0 periodic, 1 fixed velocity, 2
 * parabolic inflow, 3 fixed pressure, 4 no-slip, 5 symmetric, 6 open); with
 * a wall other than code 4 the fused step keeps the f halo cells in a ring
 * that a one-block kernel updates before each step as BC_f does.  The
 * reduced-precision forms, bgk_advance, the packed-row exchange and the
 * adjoint implement the no-slip code 4, the only code any shipped input
 * uses (UTIL/input.dat.0-3). */
int bgk_create(const bgk_params *p, const bgk_options *opt, bgk_ctx **out);
int bgk_destroy(bgk_ctx *ctx);

/* Fill every field with the reference's initial condition: liquid strip
 * i <= Nx/40 at (T0, rho1, phi=+1), solid elsewhere at (T_in_sol, rho0,
 * phi=-1), equilibrium populations; sets it = 0.  Replaces
 * STEP_7/initialization.f90:5-152. */
int bgk_initialize(bgk_ctx *ctx);

/* nsteps fused time steps, each equivalent to STEP_7/main.f90:60-69
 * (BC_f, BC_g, streaming, momentsPre, phase_field, forces, collision,
 * moments); advances it by nsteps.  Afterwards rho, T, u, v, phi (with
 * halos) are as the reference leaves them after `moments`. */
int bgk_step(bgk_ctx *ctx, int nsteps);

/* One reference subroutine each, unfused, on the complete reference state
 * (FP64 contexts only).  Calling them in the order of STEP_7/main.f90:60-69
 * gives results bit-identical to bgk_step(ctx, 1).  bgk_moments increments it.
 * A context may switch between staged and fused stepping at step
 * boundaries (after bgk_moments). */
int bgk_bc_f(bgk_ctx *ctx);          /* STEP_7/BC_f.f90:1-207         */
int bgk_bc_g(bgk_ctx *ctx);          /* STEP_7/BC_g.f90:1-71          */
int bgk_streaming(bgk_ctx *ctx);     /* STEP_7/streaming.f90:1-33     */
int bgk_moments_pre(bgk_ctx *ctx);   /* STEP_7/momentsPre.f90:1-71    */
int bgk_phase_field(bgk_ctx *ctx);   /* STEP_7/phase_field.f90:1-63   */
int bgk_forces(bgk_ctx *ctx);        /* STEP_7/forces.f90:1-43        */
int bgk_collision(bgk_ctx *ctx);     /* STEP_7/collision.f90:1-158    */
int bgk_moments(bgk_ctx *ctx);       /* STEP_7/moments.f90:1-74       */

/* Copy one field between the host (reference layout, leading dimension ld)
 * and the device.  After bgk_step the fields f, g, rho, T, u, v, phi and
 * phi_prec can be downloaded; the momentsPre copies (rho2, T2, u2, v2) and
 * the streamed populations (fp, gp) exist only in the staged state.
 * Uploading f, g, rho, T, u, v or phi replaces that part of the state, the
 * way STEP_7/dump_in.f90:9-18 overwrites the module arrays. */
int bgk_upload(bgk_ctx *ctx, int field, const double *host, int ld);
int bgk_download(bgk_ctx *ctx, int field, double *host, int ld);

/* Copy the rectangle i0..i0+ni-1, j0..j0+nj-1 (reference indices, halos
 * allowed) of a field into host[a + ld*b].  Used for the probe, the x/y
 * profiles and the wall-gradient columns of the diagnostics
 * (STEP_7/probe.f90, prof_x.f90, prof_y.f90, diag.f90:63-76) without copying
 * the whole field. */
int bgk_download_region(bgk_ctx *ctx, int field, int i0, int j0, int ni, int nj,
                        double *host, int ld);

/* Interior reductions in FP64 for field_check/diag
 * (STEP_7/field_check.f90:9-17, STEP_7/diag.f90:82-91):
 * out[0] = sum rho, out[1] = sum T, out[2] = sum phi, out[3] = #(phi > 0).
 * Returns BGK_ERR_NONFINITE (with out filled) if a sum is NaN or Inf. */
int bgk_field_sums(bgk_ctx *ctx, double out[4]);

/* Time-step counter `it` (STEP_7/main.f90:54). */
int bgk_get_it(const bgk_ctx *ctx, int *it);
int bgk_set_it(bgk_ctx *ctx, int it);

/* Hot-wall temperature per row: tin[j-1] is Tin for row j = 1..Ny
 * (generalises the scalar Tin of STEP_7/BC_g.f90:13-16; tin = NULL restores
 * the scalar Tin = T0 of STEP_7/initialization.f90:9).  The heated wall is
 * the west one: a context created with BGK_HEAT_RIGHT refuses a per-row tin. */
int bgk_set_tin(bgk_ctx *ctx, const double *tin, int ny);

/* Wait for all work queued on the context's stream. */
int bgk_sync(bgk_ctx *ctx);

/* The context's CUDA stream (a cudaStream_t), so a caller can order its own
 * work or timing events with the library's kernels.  No reference
 * counterpart (the reference has no device streams). */
int bgk_get_stream(bgk_ctx *ctx, void **stream);

/* ----------------------------------------------------- differentiation form */
/* Loss L = sum_p (phi(i_p, j_p) - phi_target_p)^2 on the state reached after
 * nsteps fused steps from the current state. */
typedef struct bgk_adjoint_spec {
    int nsteps;                /* forward steps from the current state           */
    int checkpoint_every;      /* K > 0: snapshot every K steps; 0: K =
                                * ceil(sqrt(nsteps)), or the binomial schedule
                                * when those snapshots do not fit in free
                                * device memory; < 0: binomial schedule with
                                * -checkpoint_every state slots               */
    int nprobes;
    const int *probe_i;        /* reference indices, 1..Nx                       */
    const int *probe_j;        /* 1..Ny                                          */
    const double *phi_target;  /* nprobes values                                 */
} bgk_adjoint_spec;

/* L and its gradient with respect to the per-row hot-wall temperatures
 * (grad_tin[j-1] = dL/dTin_j, the Tin of STEP_7/BC_g.f90:13-16 generalised
 * per row by bgk_set_tin) and to the thermal relaxation time tau_g
 * (STEP_7/setup.f90:103), by a hand-written reverse of the fused step run
 * backward in time with checkpoint-and-recompute: snapshots every K steps,
 * each K-step segment recomputed forward before it is reversed, or, when
 * memory is short, a binomial (revolve) schedule over a fixed number of
 * state slots that recomputes each step a few times instead.  No
 * reference counterpart (the reference has no derivatives).  Requires an FP64
 * context created with opt.smooth = 1 (the differentiable form).  The
 * context is left at the final state, exactly as bgk_step(ctx, nsteps)
 * leaves it.  grad_tin may be NULL.  The workspace (snapshots, recompute
 * buffer, partials) stays allocated in the context for the next call unless
 * it exceeds a quarter of the device memory; bgk_destroy frees it. */
int bgk_adjoint_run(bgk_ctx *ctx, const bgk_adjoint_spec *spec, double *loss,
                    double *grad_tin, double *grad_tau_g);

/* ---------------------------------------------------- allocation-free sums */
/* Rows the static scratch of bgk_field_sums_static holds: 4 doubles per row,
 * 1 MiB per device. */
#define BGK_STATIC_SUMS_MAX_NY 32768

/* The four sums of bgk_field_sums -- total density, total temperature,
 * total liquid fraction and the number of liquid nodes (phi > 0) over the
 * interior -- over fields the caller keeps in its own device memory,
 * computed without allocating anything.  This entry point has no
 * counterpart in the reference.
 *
 * For a caller that cannot allocate device memory mid-run: a host that owns
 * its rho/T/phi arrays on the GPU and must not create a context (bgk_create
 * allocates the whole step state) nor call cudaMalloc/cudaFree (cudaFree
 * synchronizes the device, and a fixed device-memory budget may leave no
 * room).  The scratch is a static __device__ array inside the library.
 *
 * rho, T, phi: device arrays of the current device in the reference layout
 * (0:Nx+1, 0:Ny+1), i fastest, row j at offset j*ld; the interior
 * i = 1..Nx, j = 1..Ny is summed.  out: 4 doubles of device memory, written
 * asynchronously on `stream` (a cudaStream_t; NULL = the legacy default
 * stream): out[0] = sum rho, out[1] = sum T, out[2] = sum phi,
 * out[3] = #(phi > 0).  The call does not wait and does not check the sums
 * for NaN or Inf.  Agrees with bgk_field_sums to rounding (another order of
 * addition); deterministic for given Nx, Ny.
 *
 * Limits and rules:
 *  - Ny > BGK_STATIC_SUMS_MAX_NY is rejected with BGK_ERR_ARG before any
 *    device work.
 *  - Nothing in the scratch has to start at zero: every slot a call reads is
 *    written earlier by the same call.
 *  - The first call on each device looks up the scratch address
 *    (cudaGetSymbolAddress) and caches it for the device's current CUDA
 *    context; make that first call before any stream capture begins.  After
 *    the context is replaced (cudaDeviceReset, or another context made
 *    current), the next call repeats the lookup, and that call too belongs
 *    outside a stream capture.
 *  - All calls on one device share the scratch.  Calls that can overlap in
 *    time (on different streams, or from host threads without ordering
 *    between them) race and return wrong sums; calls on one stream are
 *    ordered and safe. */
int bgk_field_sums_static(const double *rho, const double *T, const double *phi, int Nx, int Ny,
                          int ld, void *stream, double *out);

/* ------------------------------------------------ y-slab decomposition */
/* A domain split into slabs of rows, one context per slab, each holding
 * copies ("ghost rows") of its neighbours' rows on every side that is a cut
 * rather than a wall.  The step treats a context's first and last rows as
 * the N/S walls, so a ghost row's own update is wrong and the error moves
 * one row inward per step; with H ghost rows a slab takes H steps and then
 * replaces its ghost rows by the neighbours' current rows, and every real
 * row is bit-identical to the undivided run.  No reference counterpart:
 * the reference runs on one node (STEP_OPENMP splits loops, not the
 * domain). */

/* nsteps fused steps without writing the reference-layout fields (rho, T,
 * u, v, phi and halos keep their values): the steps between two halo
 * exchanges.  The populations, phi and it advance exactly as in bgk_step;
 * the last two steps before fields are read must go through bgk_step. */
int bgk_advance(bgk_ctx *ctx, int nsteps);

/* Bytes of nrows packed rows of the step state: the 18 population planes at
 * the context's storage size, phi, and the east T column, each section
 * padded to 16 bytes. */
int bgk_rows_bytes(const bgk_ctx *ctx, int nrows, size_t *bytes);

/* Pack interior rows j0 .. j0+nrows-1 (0-based; reference rows j0+1 ..) of
 * the current step state into dev_buf, or unpack dev_buf into them: device
 * memory of the context's device, 16-byte aligned, bgk_rows_bytes long.
 * Asynchronous on the context's stream; the rows' reference-layout fields
 * are not updated by unpack. */
int bgk_rows_pack(bgk_ctx *ctx, int j0, int nrows, void *dev_buf);
int bgk_rows_unpack(bgk_ctx *ctx, int j0, int nrows, const void *dev_buf);

/* bgk_field_sums over interior rows j0 .. j0+nrows-1 only (a slab's own
 * rows, without its ghost rows); the full range gives bgk_field_sums bit
 * for bit. */
int bgk_field_sums_rows(bgk_ctx *ctx, int j0, int nrows, double out[4]);

/* Complete binary snapshot (populations, phi, frozen boundary values, it)
 * -- unlike the reference's text dump (STEP_7/dump_out.f90:5-18), which omits
 * phi and phi_prec.  A snapshot restores into a context of the same size,
 * precision and heat bits (BGK_ERR_ARG otherwise). */
int bgk_save(bgk_ctx *ctx, const char *path);
int bgk_load(bgk_ctx *ctx, const char *path);

#ifdef __cplusplus
}
#endif
#endif /* BGK_PCM_H */
