/*
 * capi.cu -- the extern "C" boundary of libbgkpcm (include/bgk_pcm.h):
 * context life cycle, parameter handling, host<->device transfers in the
 * reference layout, and the step drivers.  Kernels live in kernels_f64.cu
 * (reference operation order) and kernels_fast.cu (FMA / reduced precision).
 */
#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdint>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "bgk_internal.h"

using bgk::Consts;

/* Reduced-precision field conversions are implemented in kernels_fast.cu. */
int lowp_compact_to_ref(bgk_ctx *c, int field, double *ref, int prev);
int lowp_ref_to_compact(bgk_ctx *c, int field, const double *ref);

namespace {

thread_local char g_err[512] = "";

int fail(int code, const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof g_err, fmt, ap);
    va_end(ap);
    return code;
}

int cuda_fail(cudaError_t e, const char *what)
{
    return fail(BGK_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

#define CK(call, what)                                   \
    do {                                                 \
        cudaError_t e_ = (call);                         \
        if (e_ != cudaSuccess) return cuda_fail(e_, what); \
    } while (0)

bool all_bc4(const bgk_params &p)
{
    return p.westBC == 4 && p.eastBC == 4 && p.northBC == 4 && p.southBC == 4;
}

/* ------------------------------------------------------------- input.dat */

/* One list-directed record "label value ...": the value is the second token
 * separated by blanks, tabs or commas (STEP_7/setup.f90:7-31 reads every
 * record as `read(112,*) id(k), value`). */
int next_value(FILE *fp, std::string &tok)
{
    char line[4096];
    if (!fgets(line, sizeof line, fp)) return -1;
    const char *sep = " \t,\r\n";
    char *save = nullptr;
    char *t1 = strtok_r(line, sep, &save);
    if (!t1) return -1;
    char *t2 = strtok_r(nullptr, sep, &save);
    if (!t2) return -1;
    tok = t2;
    return 0;
}

int to_real(const std::string &t, double &out)
{
    std::string b = t;
    for (char &ch : b)
        if (ch == 'd' || ch == 'D') ch = 'e';
    char *end = nullptr;
    errno = 0;
    double v = strtod(b.c_str(), &end);
    if (end == b.c_str() || *end != 0 || errno) return -1;
    out = v;
    return 0;
}

int to_int(const std::string &t, int &out)
{
    char *end = nullptr;
    errno = 0;
    long v = strtol(t.c_str(), &end, 10);
    if (end == t.c_str() || *end != 0 || errno) return -1;
    out = (int)v;
    return 0;
}

/* setup.f90:79-115, forces.f90:12-13, phase_field.f90:11-15,
 * initialization.f90:5-13, collision.f90:84-100. Host arithmetic is built
 * without contraction, so these match the reference bit for bit. */
Consts make_consts(const bgk_params &p)
{
    Consts c{};
    c.Nx = p.Nx;
    c.Ny = p.Ny;
    c.w[0] = 4.0 / 9.0;
    for (int k = 1; k <= 4; k++) c.w[k] = 1.0 / 9.0;
    for (int k = 5; k <= 8; k++) c.w[k] = 1.0 / 36.0;
    c.cs2 = 1.0 / 3.0;
    c.m_cs2 = -c.cs2;
    c.q_cs2 = 1.0 - c.cs2;
    for (int k = 0; k < 9; k++) c.C[k] = (0.5 * c.w[k]) / (c.cs2 * c.cs2);
    c.omega_f = 1.0 / p.tau_f;
    c.omega_g = 1.0 / p.tau_g;
    const double kvisc = c.cs2 * (p.tau_f - 0.5);
    c.T_crit = 273.0;
    c.T_act = 0.0;
    c.T_width = p.T_width;
    c.f_plus = 0.5;
    c.f_minus = 0.5;
    const double delta_T = p.T0 - p.T_in_sol;
    c.dts = delta_T / p.stefan_number;
    c.grav = p.grav;
    const float beta32 = (float)((1.0 - p.rho1 / p.rho0) / delta_T);
    c.beta = (double)beta32;
    c.Tin = p.T0;
    c.u0 = p.Re * kvisc / p.length;
    c.v0 = 0.0;
    c.rho0 = p.rho0;
    c.rho1 = p.rho1;
    c.T0 = p.T0;
    c.T_in_sol = p.T_in_sol;
    c.interf = p.Nx / 40;
    return c;
}

int check_params(const bgk_params &p)
{
    if (p.Nx < 1 || p.Ny < 1) return fail(BGK_ERR_ARG, "Nx and Ny must be >= 1 (got %d, %d)", p.Nx, p.Ny);
    if ((long long)(p.Nx + 2) * (p.Ny + 2) > (1LL << 40)) return fail(BGK_ERR_ARG, "grid too large");
    const double r[] = {p.Re, p.rho0, p.rho1, p.tau_f, p.tau_g, p.T0, p.T_in_sol, p.grav, p.eps,
                        p.stefan_number, p.T_width, p.length};
    for (double v : r)
        if (!std::isfinite(v)) return fail(BGK_ERR_ARG, "non-finite real parameter");
    if (p.tau_f == 0.0 || p.tau_g == 0.0) return fail(BGK_ERR_ARG, "tau_f and tau_g must be non-zero");
    if (p.rho0 == 0.0) return fail(BGK_ERR_ARG, "rho0 must be non-zero (forces.f90:13 divides by it)");
    if (p.T0 == p.T_in_sol) return fail(BGK_ERR_ARG, "T0 == T_in_sol: beta = (1-rho1/rho0)/(T0-T_in_sol) is undefined");
    if (p.stefan_number == 0.0) return fail(BGK_ERR_ARG, "stefan_number must be non-zero");
    if (p.T_width == 0.0) return fail(BGK_ERR_ARG, "T_width must be non-zero");
    if (p.length == 0.0) return fail(BGK_ERR_ARG, "length must be non-zero (u0 = Re*kvisc/length)");
    const int bcs[] = {p.westBC, p.eastBC, p.northBC, p.southBC};
    const char *nm[] = {"westBC", "eastBC", "northBC", "southBC"};
    static const int ok_w[] = {0, 1, 2, 3, 4}, ok_e[] = {0, 3, 4}, ok_n[] = {0, 1, 4, 5, 6}, ok_s[] = {0, 4, 6};
    const int *oks[] = {ok_w, ok_e, ok_n, ok_s};
    const int nok[] = {5, 3, 5, 3};
    for (int b = 0; b < 4; b++) {
        bool ok = false;
        for (int k = 0; k < nok[b]; k++) ok |= (bcs[b] == oks[b][k]);
        if (!ok) return fail(BGK_ERR_UNSUPPORTED, "%s = %d has no branch in STEP_7/BC_f.f90", nm[b], bcs[b]);
    }
    return BGK_OK;
}

template <typename T>
int dalloc(T **p, size_t bytes, const char *what)
{
    void *q = nullptr;
    cudaError_t e = cudaMalloc(&q, bytes ? bytes : 16);
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        return fail(BGK_ERR_OOM, "cudaMalloc(%zu bytes) for %s: %s", bytes, what, cudaGetErrorString(e));
    }
    *p = (T *)q;
    return BGK_OK;
}

#define DA(ptr, bytes, what)                          \
    do {                                              \
        int rc_ = dalloc(&(ptr), (bytes), (what));    \
        if (rc_) { bgk_destroy(c); return rc_; }      \
    } while (0)

int set_device(const bgk_ctx *c)
{
    cudaError_t e = cudaSetDevice(c->dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
    return BGK_OK;
}

int alloc_staged(bgk_ctx *c)
{
    if (c->staged_alloc) return BGK_OK;
    const size_t bytes = c->A * sizeof(double);
    double **all[] = {&c->sphip, &c->srho2, &c->sT2, &c->su2, &c->sv2};
    for (int k = 0; k < 9; k++) {
        int rc;
        if ((rc = dalloc(&c->sf[k], bytes, "staged f"))) return rc;
        if ((rc = dalloc(&c->sg[k], bytes, "staged g"))) return rc;
        if ((rc = dalloc(&c->sfp[k], bytes, "staged fp"))) return rc;
        if ((rc = dalloc(&c->sgp[k], bytes, "staged gp"))) return rc;
        CK(cudaMemsetAsync(c->sf[k], 0, bytes, c->stream), "memset");
        CK(cudaMemsetAsync(c->sg[k], 0, bytes, c->stream), "memset");
        CK(cudaMemsetAsync(c->sfp[k], 0, bytes, c->stream), "memset");
        CK(cudaMemsetAsync(c->sgp[k], 0, bytes, c->stream), "memset");
    }
    for (double **p : all) {
        int rc;
        if ((rc = dalloc(p, bytes, "staged field"))) return rc;
        CK(cudaMemsetAsync(*p, 0, bytes, c->stream), "memset");
    }
    c->staged_alloc = true;
    return BGK_OK;
}

/* Make the reference-layout (staged) state current. */
int ensure_staged(bgk_ctx *c)
{
    if (c->opt.precision != BGK_PREC_F64)
        return fail(BGK_ERR_UNSUPPORTED, "the staged (per-subroutine) path exists for FP64 contexts only");
    if (c->mode == 1) return BGK_OK;
    int rc = alloc_staged(c);
    if (rc) return rc;
    if (c->pristine) {
        /* straight after bgk_initialize: the complete initial arrays,
         * halos included (initialization.f90 fills every cell) */
        c->mode = 1;
        CK(bgk::launch_init_f64(c), "init (staged)");
    } else {
        CK(bgk::launch_compact_to_staged(c), "compact_to_staged");
        /* phi_prec = phi of the previous step with the same halos */
        CK(bgk::launch_compact_to_ref(c, BGK_FIELD_PHI_PREC, c->sphip, 1), "phi_prec");
    }
    c->mode = 1;
    c->stage_pos = 0;
    return BGK_OK;
}

/* Make the compact (fused) state current; allowed at step boundaries. */
int ensure_fused(bgk_ctx *c)
{
    if (c->mode == 0) return BGK_OK;
    if (c->stage_pos != 0)
        return fail(BGK_ERR_STATE, "the staged step is incomplete (last stage %d); finish it with bgk_moments",
                    c->stage_pos);
    CK(bgk::launch_staged_to_compact(c), "staged_to_compact");
    c->mode = 0;
    c->bc_dirty = true;
    return BGK_OK;
}

double *staged_field_ptr(bgk_ctx *c, int f)
{
    if (f >= BGK_FIELD_F0 && f < BGK_FIELD_F0 + 9) return c->sf[f - BGK_FIELD_F0];
    if (f >= BGK_FIELD_G0 && f < BGK_FIELD_G0 + 9) return c->sg[f - BGK_FIELD_G0];
    if (f >= BGK_FIELD_FP0 && f < BGK_FIELD_FP0 + 9) return c->sfp[f - BGK_FIELD_FP0];
    if (f >= BGK_FIELD_GP0 && f < BGK_FIELD_GP0 + 9) return c->sgp[f - BGK_FIELD_GP0];
    switch (f) {
    case BGK_FIELD_RHO: return c->mrho;
    case BGK_FIELD_T: return c->mT;
    case BGK_FIELD_U: return c->mu;
    case BGK_FIELD_V: return c->mv;
    case BGK_FIELD_PHI: return c->mphi;
    case BGK_FIELD_PHI_PREC: return c->sphip;
    case BGK_FIELD_RHO2: return c->srho2;
    case BGK_FIELD_T2: return c->sT2;
    case BGK_FIELD_U2: return c->su2;
    case BGK_FIELD_V2: return c->sv2;
    }
    return nullptr;
}

double *mirror_ptr(bgk_ctx *c, int f)
{
    switch (f) {
    case BGK_FIELD_RHO: return c->mrho;
    case BGK_FIELD_T: return c->mT;
    case BGK_FIELD_U: return c->mu;
    case BGK_FIELD_V: return c->mv;
    case BGK_FIELD_PHI: return c->mphi;
    }
    return nullptr;
}

bool is_intermediate(int f)
{
    return f == BGK_FIELD_RHO2 || f == BGK_FIELD_T2 || f == BGK_FIELD_U2 || f == BGK_FIELD_V2 ||
           (f >= BGK_FIELD_FP0 && f < BGK_FIELD_GP0 + 9);
}

/* Device pointer to a full reference-layout copy of `field`, materialising
 * it into the scratch buffer when the current state does not hold it in
 * that layout. */
int field_source(bgk_ctx *c, int field, const double **src)
{
    if (c->mode == 1) {
        *src = staged_field_ptr(c, field);
        return BGK_OK;
    }
    if (double *m = mirror_ptr(c, field)) {
        *src = m;
        return BGK_OK;
    }
    if (is_intermediate(field))
        return fail(BGK_ERR_STATE, "field %d (momentsPre copy or streamed population) exists only in the staged "
                                   "state; call the stage entry points to materialise it", field);
    if (c->opt.precision != BGK_PREC_F64) {
        int rc = lowp_compact_to_ref(c, field, c->scratch, field == BGK_FIELD_PHI_PREC);
        if (rc) return rc;
    } else {
        CK(bgk::launch_compact_to_ref(c, field, c->scratch, field == BGK_FIELD_PHI_PREC), "compact_to_ref");
    }
    *src = c->scratch;
    return BGK_OK;
}

} // namespace

int bgk_internal_fail(int code, const char *msg) { return fail(code, "%s", msg); }

int bgk_internal_prepare_fused(bgk_ctx *c)
{
    if (!all_bc4(c->p))
        return fail(BGK_ERR_UNSUPPORTED, "the fused step implements the no-slip code 4 on every wall");
    if (c->opt.heat & BGK_HEAT_RIGHT)
        return fail(BGK_ERR_UNSUPPORTED, "BGK_HEAT_RIGHT runs on bgk_step and the stage entry points only");
    int rc = set_device(c);
    if (rc) return rc;
    if ((rc = ensure_fused(c))) return rc;
    if (c->bc_dirty) {
        CK(bgk::launch_bc_prep(c), "bc_prep");
        c->bc_dirty = false;
    }
    return BGK_OK;
}

/* n fused steps without the reference-layout moments and halos (the
 * mirrors keep their values from before): the adjoint's forward pass
 * between snapshots, whose last chunk goes through bgk_step. */
int bgk_internal_advance(bgk_ctx *c, int nsteps)
{
    int rc = bgk_internal_prepare_fused(c);
    if (rc) return rc;
    c->pristine = false;
    const bool exact = c->opt.precision == BGK_PREC_F64 && !c->opt.fma;
    for (int t = 0; t < nsteps; t++) {
        if (exact) CK(bgk::launch_fused_f64(c, false), "fused step");
        else CK(bgk::launch_fused_fast(c, false), "fused step");
        c->cur ^= 1;
        c->it += 1;
    }
    return BGK_OK;
}

extern "C" {

const char *bgk_last_error(void) { return g_err; }

int bgk_read_input(const char *path, bgk_params *out)
{
    if (!path || !out) return fail(BGK_ERR_ARG, "null argument");
    FILE *fp = fopen(path, "r");
    if (!fp) return fail(BGK_ERR_IO, "cannot open %s (the reference opens input.dat with status='old')", path);
    bgk_params p{};
    std::string t;
    int rc = 0;
    int *ints1[] = {&p.iter, &p.noutput, &p.dump, &p.Nx, &p.Ny};
    double *reals[] = {&p.Re, &p.rho0, &p.rho1, &p.tau_f, &p.tau_g, &p.T0, &p.T_in_sol, &p.grav, &p.eps,
                       &p.stefan_number, &p.T_width, &p.length};
    int *ints2[] = {&p.westBC, &p.eastBC, &p.northBC, &p.southBC};
    int rec = 0;
    for (int *v : ints1) { rec++; if (!rc && (next_value(fp, t) || to_int(t, *v))) rc = rec; }
    for (double *v : reals) { rec++; if (!rc && (next_value(fp, t) || to_real(t, *v))) rc = rec; }
    for (int *v : ints2) { rec++; if (!rc && (next_value(fp, t) || to_int(t, *v))) rc = rec; }
    fclose(fp);
    if (rc) return fail(BGK_ERR_IO, "%s: record %d is missing or malformed", path, rc);
    *out = p;
    return BGK_OK;
}

/* CK for bgk_create once the context exists: free it before failing */
#define CKC(call, what)                                                    \
    do {                                                                   \
        cudaError_t e_ = (call);                                           \
        if (e_ != cudaSuccess) { bgk_destroy(c); return cuda_fail(e_, what); } \
    } while (0)

/* ------------------------------------------------------ step graphs */

/* Steps per captured graph: even, so a replay ends on the buffer it starts
 * from. */
constexpr int GRAPH_STEPS = 32;

static void drop_step_graphs(bgk_ctx *c)
{
    for (int b = 0; b < 2; b++)
        if (c->step_graph[b]) {
            cudaGraphExecDestroy(c->step_graph[b]);
            c->step_graph[b] = nullptr;
        }
}

/* One plain step (no moments): the halo-ring update first where it applies. */
static cudaError_t launch_plain_step(bgk_ctx *c, bool exact)
{
    if (c->ring) {
        cudaError_t e = bgk::launch_ring_bc(c);
        if (e != cudaSuccess) return e;
    }
    return exact ? bgk::launch_fused_f64(c, false) : bgk::launch_fused_fast(c, false);
}

/* Capture GRAPH_STEPS plain steps starting from buffer c->cur into
 * c->step_graph[c->cur].  Every kernel involved has been launched once
 * before (its attributes are set), so the capture holds kernel launches
 * only.  Returns false (and leaves graphs off for the context) on failure. */
static bool capture_step_graph(bgk_ctx *c, bool exact)
{
    const int start = c->cur;
    cudaGraph_t g = nullptr;
    if (cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        (void)cudaGetLastError();
        return false;
    }
    cudaError_t e = cudaSuccess;
    for (int k = 0; k < GRAPH_STEPS && e == cudaSuccess; k++) {
        e = launch_plain_step(c, exact);
        c->cur ^= 1;
    }
    const cudaError_t e2 = cudaStreamEndCapture(c->stream, &g);
    c->cur = start;
    cudaGraphExec_t x = nullptr;
    if (e == cudaSuccess && e2 == cudaSuccess && g && cudaGraphInstantiate(&x, g, 0) == cudaSuccess) {
        c->step_graph[start] = x;
    } else {
        x = nullptr;
    }
    if (g) cudaGraphDestroy(g);
    (void)cudaGetLastError();
    return x != nullptr;
}

int bgk_create(const bgk_params *pp, const bgk_options *opt, bgk_ctx **out)
{
    if (!pp || !out) return fail(BGK_ERR_ARG, "null argument");
    *out = nullptr;
    int rc = check_params(*pp);
    if (rc) return rc;
    bgk_options o{BGK_PREC_F64, BGK_TANH_PORTABLE, 0, -1, 0, BGK_HEAT_WEST};
    if (opt) o = *opt;
    if (o.heat < 0 || o.heat > (BGK_HEAT_RIGHT | BGK_HEAT_BOTTOM)) return fail(BGK_ERR_ARG, "bad heat bits %d", o.heat);
    if ((o.heat & BGK_HEAT_RIGHT) && o.precision != BGK_PREC_F64)
        return fail(BGK_ERR_UNSUPPORTED, "BGK_HEAT_RIGHT is implemented in the FP64 forms only");
    if (o.precision < BGK_PREC_F64 || o.precision > BGK_PREC_F32X) return fail(BGK_ERR_ARG, "bad precision %d", o.precision);
    if (o.tanh_mode != BGK_TANH_DEVICE && o.tanh_mode != BGK_TANH_PORTABLE) return fail(BGK_ERR_ARG, "bad tanh_mode");
    /* the FP32 and FP16 forms are bit-exact with nothing: CUDA's tanhf */
    if (o.precision == BGK_PREC_F32 || o.precision == BGK_PREC_F16) o.tanh_mode = BGK_TANH_DEVICE;
    if (o.precision != BGK_PREC_F64 && !all_bc4(*pp))
        return fail(BGK_ERR_UNSUPPORTED, "reduced-precision forms implement the no-slip code 4 on every wall only");

    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) {
        (void)cudaGetLastError();
        return fail(BGK_ERR_CUDA, "no CUDA device available (%s); this library has no CPU path",
                    e != cudaSuccess ? cudaGetErrorString(e) : "0 devices");
    }
    int dev = o.device;
    if (dev < 0) CK(cudaGetDevice(&dev), "cudaGetDevice");
    if (dev >= ndev) return fail(BGK_ERR_ARG, "device %d out of range (%d devices)", dev, ndev);
    cudaDeviceProp prop;
    CK(cudaGetDeviceProperties(&prop, dev), "cudaGetDeviceProperties");
    if (prop.major != 10) return fail(BGK_ERR_UNSUPPORTED, "device %d is sm_%d%d; this build targets sm_100a (B200)",
                                      dev, prop.major, prop.minor);
    CK(cudaSetDevice(dev), "cudaSetDevice");

    bgk_ctx *c = new (std::nothrow) bgk_ctx();
    if (!c) return fail(BGK_ERR_OOM, "host allocation");
    c->p = *pp;
    c->opt = o;
    c->c = make_consts(*pp);
    c->c.heat = o.heat;
    c->dev = dev;
    c->Nx = pp->Nx;
    c->Ny = pp->Ny;
    c->NX2 = pp->Nx + 2;
    c->NY2 = pp->Ny + 2;
    c->A = (size_t)c->NX2 * (size_t)c->NY2;
    c->P = (pp->Nx + 31) / 32 * 32;
    c->plane = (long long)c->P * pp->Ny;
    c->esz = o.precision == BGK_PREC_F64 ? 8 : (o.precision == BGK_PREC_F16 ? 2 : 4);
    /* phi: FP64 in the FP64 and FP32X forms; FP32 (storage and phase-field
     * arithmetic) in the FP32 and FP16 forms unless BGK_LP_PHI64=1 */
    c->phisz = (o.precision == BGK_PREC_F64 || o.precision == BGK_PREC_F32X) ? 8 : 4;
    if (o.precision == BGK_PREC_F32 || o.precision == BGK_PREC_F16) {
        const char *v = getenv("BGK_LP_PHI64");
        if (v && atoi(v) == 1) c->phisz = 8;
    }
    c->it = 0;
    c->cur = 0;
    c->bc_dirty = true;
    c->tune_H = 0;
    c->tune_pf = 2;
    c->tune_pipe = 1;
    c->tune_D = 0;
    c->tune_ctas = 0;
    if (const char *v = getenv("BGK_STRIP_H")) c->tune_H = atoi(v);
    if (const char *v = getenv("BGK_PREFETCH_ROWS")) c->tune_pf = atoi(v);
    if (const char *v = getenv("BGK_PIPE")) c->tune_pipe = atoi(v);
    if (const char *v = getenv("BGK_PIPE_D")) c->tune_D = atoi(v);
    if (const char *v = getenv("BGK_PIPE_CTAS")) c->tune_ctas = atoi(v);
    c->tune_flow = 0;
    if (const char *v = getenv("BGK_FLOW")) c->tune_flow = atoi(v);
    c->step_graph[0] = c->step_graph[1] = nullptr;
    c->graph_failed = false;
    c->graph_on = (long long)pp->Nx * pp->Ny <= (1LL << 21);
    if (const char *v = getenv("BGK_GRAPH")) c->graph_on = c->graph_on && atoi(v) != 0;
    c->flow_stall = 0;
    if (const char *v = getenv("BGK_FLOW_STALL")) c->flow_stall = atoi(v) == 1;
    {
        cudaDeviceProp pr;
        c->nsm = (cudaGetDeviceProperties(&pr, dev) == cudaSuccess) ? pr.multiProcessorCount : 148;
    }
    e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) { delete c; return cuda_fail(e, "cudaStreamCreate"); }

    /* 9 planes per distribution, then slack for the pipeline's last row
     * segment (a band of 128 columns + 16 bytes may run past the last row) */
    const size_t popbytes = (size_t)(9 * c->plane + 2 * c->P + 256) * c->esz;
    const size_t phibytes = (size_t)(c->plane + 2 * c->P + 256) * c->phisz;
    const size_t guard = 256;
    for (int b = 0; b < 2; b++) {
        DA(c->raw[b], popbytes + 2 * guard, "f populations");
        DA(c->raw[2 + b], popbytes + 2 * guard, "g populations");
        DA(c->raw[4 + b], phibytes + 2 * guard, "phi");
        CKC(cudaMemsetAsync(c->raw[b], 0, popbytes + 2 * guard, c->stream), "memset");
        CKC(cudaMemsetAsync(c->raw[2 + b], 0, popbytes + 2 * guard, c->stream), "memset");
        CKC(cudaMemsetAsync(c->raw[4 + b], 0, phibytes + 2 * guard, c->stream), "memset");
        c->fbuf[b] = (char *)c->raw[b] + guard;
        c->gbuf[b] = (char *)c->raw[2 + b] + guard;
        c->phibuf[b] = (char *)c->raw[4 + b] + guard;
        DA(c->tcol[b], (size_t)c->Ny * sizeof(double), "T column");
    }
    DA(c->errflag, sizeof(int), "error flag");
    CKC(cudaMemsetAsync(c->errflag, 0, sizeof(int), c->stream), "memset");
    DA(c->gW, 3 * (size_t)c->Ny * sizeof(double), "west g");
    DA(c->pE, 3 * (size_t)c->Ny * sizeof(double), "east poly");
    DA(c->phiW, (size_t)c->Ny * sizeof(double), "phi west");
    DA(c->phiE, (size_t)c->Ny * sizeof(double), "phi east");
    const size_t abytes = c->A * sizeof(double);
    DA(c->mrho, abytes, "rho");
    DA(c->mT, abytes, "T");
    DA(c->mu, abytes, "u");
    DA(c->mv, abytes, "v");
    DA(c->mphi, abytes, "phi mirror");
    DA(c->scratch, abytes, "scratch");
    c->red_n = 4 + 4 * 592;
    DA(c->red, (size_t)c->red_n * sizeof(double), "reduction");
    DA(c->corner, 2 * sizeof(double), "corners");
    /* walls other than the no-slip code 4 (FP64 only): the f halo ring.
     * BGK_HEAT_RIGHT runs there too: its west g halos take T(1,j) of the
     * previous step, which the ring step keeps in the T mirror (edge nodes
     * write their moments every step) and bc_prep reads before each step */
    c->ring = o.precision == BGK_PREC_F64 && (!all_bc4(*pp) || (o.heat & BGK_HEAT_RIGHT));
    c->ring_len = bgk::ring_length(c->Nx, c->Ny);
    c->fring = nullptr;
    if (c->ring) {
        DA(c->fring, (size_t)9 * (size_t)c->ring_len * sizeof(double), "f halo ring");
        CKC(cudaMemsetAsync(c->fring, 0, (size_t)9 * (size_t)c->ring_len * sizeof(double), c->stream), "memset");
    }
    c->tright = nullptr;
    if (o.heat & BGK_HEAT_RIGHT) {
        DA(c->tright, (size_t)c->Ny * sizeof(double), "east T column");
        std::vector<double> col((size_t)c->Ny, c->c.Tin);
        e = cudaMemcpy(c->tright, col.data(), col.size() * sizeof(double), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) { bgk_destroy(c); return cuda_fail(e, "east T column"); }
    }
    e = cudaMallocHost(&c->pinned, 64 * sizeof(double));
    if (e != cudaSuccess) { bgk_destroy(c); return cuda_fail(e, "cudaMallocHost"); }
    CKC(cudaStreamSynchronize(c->stream), "create");
    *out = c;
    return BGK_OK;
}

int bgk_destroy(bgk_ctx *c)
{
    if (!c) return BGK_OK;
    cudaSetDevice(c->dev);
    if (c->stream) cudaStreamSynchronize(c->stream);
    void *ptrs[] = {c->raw[0], c->raw[1], c->raw[2], c->raw[3], c->raw[4], c->raw[5], c->errflag,
                    c->tcol[0], c->tcol[1], c->gW, c->pE, c->phiW, c->phiE, c->tin_rows,
                    c->mrho, c->mT, c->mu, c->mv, c->mphi, c->sphip, c->srho2, c->sT2, c->su2, c->sv2,
                    c->scratch, c->red, c->corner, c->fring, c->flow_buf, c->tright};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    for (int k = 0; k < 9; k++) {
        if (c->sf[k]) cudaFree(c->sf[k]);
        if (c->sg[k]) cudaFree(c->sg[k]);
        if (c->sfp[k]) cudaFree(c->sfp[k]);
        if (c->sgp[k]) cudaFree(c->sgp[k]);
    }
    drop_step_graphs(c);
    if (c->pinned) cudaFreeHost(c->pinned);
    if (c->adj_ws) cudaFree(c->adj_ws);
    free(c->tin_host);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return BGK_OK;
}

int bgk_initialize(bgk_ctx *c)
{
    if (!c) return fail(BGK_ERR_ARG, "null context");
    int rc = set_device(c);
    if (rc) return rc;
    drop_step_graphs(c);   /* the reduced-precision scales are set anew */
    c->cur = 0;
    c->mode = 0;
    if (c->opt.precision == BGK_PREC_F64) {
        CK(bgk::launch_init_f64(c), "init");
    } else {
        CK(bgk::launch_init_lowp(c), "init");
    }
    c->it = 0;
    c->stage_pos = 0;
    c->bc_dirty = true;
    c->pristine = true;
    CK(cudaStreamSynchronize(c->stream), "initialize");
    return BGK_OK;
}

int bgk_step(bgk_ctx *c, int nsteps)
{
    if (!c) return fail(BGK_ERR_ARG, "null context");
    if (nsteps < 0) return fail(BGK_ERR_ARG, "nsteps < 0");
    if (nsteps == 0) return BGK_OK;
    if (!all_bc4(c->p) && !c->ring)
        return fail(BGK_ERR_UNSUPPORTED, "the reduced-precision forms implement the no-slip code 4 on every wall");
    int rc = set_device(c);
    if (rc) return rc;
    if ((rc = ensure_fused(c))) return rc;
    if (c->bc_dirty && !c->ring) {
        CK(bgk::launch_bc_prep(c), "bc_prep");
        c->bc_dirty = false;
    }
    c->pristine = false;
    const bool f64 = c->opt.precision == BGK_PREC_F64;
    const bool exact = f64 && !c->opt.fma;
    int t = 0;
    if (c->tune_flow && !c->ring && nsteps > 2) {
        /* the steps before the two that write the moments in one launch
         * (BGK_FLOW=1), or in one launch each with tiles handed out on
         * demand (BGK_FLOW=2) */
        const int nflow = nsteps - 2;
        for (int done = 0; done < nflow;) {
            const int n = c->tune_flow == 2 ? 1 : nflow;
            if (exact) CK(bgk::launch_flow_f64(c, n), "dataflow steps");
            else CK(bgk::launch_flow_fast(c, n), "dataflow steps");
            c->cur ^= n & 1;
            c->it += n;
            done += n;
        }
        t = nflow;
    }
    /* Launch-bound grids: the plain steps before the last two as replays of
     * a captured graph (the kernels and their order are those of the loop
     * below, so the results are the same bit for bit) */
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(c->stream, &cap) != cudaSuccess) {
        (void)cudaGetLastError();
        cap = cudaStreamCaptureStatusActive;
    }
    /* (a caller capturing the context's stream into a graph of its own gets
     * the direct launches) */
    if (c->graph_on && !c->graph_failed && !c->tune_flow && cap == cudaStreamCaptureStatusNone &&
        nsteps - 2 - t >= GRAPH_STEPS + 1) {
        if (!c->step_graph[c->cur ^ 1] || !c->step_graph[c->cur]) {
            /* one step launched directly first sets every kernel's attributes */
            CK(launch_plain_step(c, exact), "fused step");
            c->cur ^= 1;
            c->it += 1;
            t += 1;
            if (!c->step_graph[c->cur] && !capture_step_graph(c, exact)) c->graph_failed = true;
        }
        while (!c->graph_failed && c->step_graph[c->cur] && nsteps - 2 - t >= GRAPH_STEPS) {
            CK(cudaGraphLaunch(c->step_graph[c->cur], c->stream), "step graph");
            c->it += GRAPH_STEPS;
            t += GRAPH_STEPS;
        }
    }
    /* The reference's arrays after the call: the last step's moments, with
     * halos copied from the step before (STEP_7/BC_f.f90, BC_g.f90).  On the
     * FP64 pipeline the step before the last writes those halo cells itself
     * from its edge nodes; otherwise it writes all its moments and a
     * macro-halo pass copies them before the last step. */
    const bool eh = f64 && c->tune_pipe && !c->ring && nsteps >= 2;
    for (; t < nsteps; t++) {
        const bool last = (t == nsteps - 1);
        const bool prev = (t == nsteps - 2);
        const bool mom = last || (prev && !eh);
        if (c->ring) {
            /* BC_f and the halo part of BC_g every step, then the west/east
             * g values from this step's velocity halos (STEP_7/BC_g.f90:7-31) */
            CK(bgk::launch_ring_bc(c), "ring boundary");
        } else if (last && !eh) {
            CK(bgk::launch_macro_halos(c), "macro_halos");
        }
        if (exact) CK(bgk::launch_fused_f64(c, mom, prev && eh), "fused step");
        else CK(bgk::launch_fused_fast(c, mom, prev && eh), "fused step");
        c->cur ^= 1;
        c->it += 1;
    }
    return BGK_OK;
}

static int stage_call(bgk_ctx *c, int stage)
{
    if (!c) return fail(BGK_ERR_ARG, "null context");
    int rc = set_device(c);
    if (rc) return rc;
    if ((rc = ensure_staged(c))) return rc;
    c->pristine = false;
    CK(bgk::launch_staged(c, stage), "stage kernel");
    if (stage == 8) {
        c->stage_pos = 0;
        c->it += 1;
    } else {
        c->stage_pos = stage;
    }
    return BGK_OK;
}

int bgk_bc_f(bgk_ctx *c) { return stage_call(c, 1); }
int bgk_bc_g(bgk_ctx *c) { return stage_call(c, 2); }
int bgk_streaming(bgk_ctx *c) { return stage_call(c, 3); }
int bgk_moments_pre(bgk_ctx *c) { return stage_call(c, 4); }
int bgk_phase_field(bgk_ctx *c) { return stage_call(c, 5); }
int bgk_forces(bgk_ctx *c) { return stage_call(c, 6); }
int bgk_collision(bgk_ctx *c) { return stage_call(c, 7); }
int bgk_moments(bgk_ctx *c) { return stage_call(c, 8); }

int bgk_upload(bgk_ctx *c, int field, const double *host, int ld)
{
    if (!c || !host) return fail(BGK_ERR_ARG, "null argument");
    if (field < 0 || field >= BGK_NFIELDS) return fail(BGK_ERR_ARG, "bad field id %d", field);
    if (ld < c->NX2) return fail(BGK_ERR_ARG, "ld (%d) < Nx+2 (%d)", ld, c->NX2);
    int rc = set_device(c);
    if (rc) return rc;
    if (c->mode == 0 && is_intermediate(field)) {
        if ((rc = ensure_staged(c))) return rc;
    }
    if (field == BGK_FIELD_PHI_PREC && c->mode == 0 && c->opt.precision == BGK_PREC_F64) {
        if ((rc = ensure_staged(c))) return rc;
    }
    const size_t w = (size_t)c->NX2 * sizeof(double);
    double *dst;
    if (c->mode == 1) dst = staged_field_ptr(c, field);
    else if (double *m = mirror_ptr(c, field)) dst = m;
    else dst = c->scratch;
    CK(cudaMemcpy2DAsync(dst, w, host, (size_t)ld * sizeof(double), w, c->NY2, cudaMemcpyHostToDevice, c->stream),
       "upload copy");
    if (c->mode == 0) {
        if (c->opt.precision == BGK_PREC_F64) {
            CK(bgk::launch_ref_to_compact(c, field, dst), "upload convert");
        } else {
            if ((rc = lowp_ref_to_compact(c, field, dst))) return rc;
        }
    }
    if (field == BGK_FIELD_U || field == BGK_FIELD_V || field == BGK_FIELD_PHI) c->bc_dirty = true;
    c->pristine = false;
    CK(cudaStreamSynchronize(c->stream), "upload");
    return BGK_OK;
}

int bgk_download(bgk_ctx *c, int field, double *host, int ld)
{
    if (!c || !host) return fail(BGK_ERR_ARG, "null argument");
    if (field < 0 || field >= BGK_NFIELDS) return fail(BGK_ERR_ARG, "bad field id %d", field);
    if (ld < c->NX2) return fail(BGK_ERR_ARG, "ld (%d) < Nx+2 (%d)", ld, c->NX2);
    return bgk_download_region(c, field, 0, 0, c->NX2, c->NY2, host, ld);
}

int bgk_download_region(bgk_ctx *c, int field, int i0, int j0, int ni, int nj, double *host, int ld)
{
    if (!c || !host) return fail(BGK_ERR_ARG, "null argument");
    if (field < 0 || field >= BGK_NFIELDS) return fail(BGK_ERR_ARG, "bad field id %d", field);
    if (ni < 0 || nj < 0 || i0 < 0 || j0 < 0 || i0 + ni > c->NX2 || j0 + nj > c->NY2)
        return fail(BGK_ERR_ARG, "region (%d,%d)+(%d,%d) outside 0..Nx+1 x 0..Ny+1", i0, j0, ni, nj);
    if (ld < ni) return fail(BGK_ERR_ARG, "ld (%d) < ni (%d)", ld, ni);
    if (ni == 0 || nj == 0) return BGK_OK;
    int rc = set_device(c);
    if (rc) return rc;
    const double *src = nullptr;
    if ((rc = field_source(c, field, &src))) return rc;
    const size_t spitch = (size_t)c->NX2 * sizeof(double);
    CK(cudaMemcpy2DAsync(host, (size_t)ld * sizeof(double), src + (size_t)i0 + (size_t)c->NX2 * j0, spitch,
                         (size_t)ni * sizeof(double), nj, cudaMemcpyDeviceToHost, c->stream),
       "download copy");
    CK(cudaStreamSynchronize(c->stream), "download");
    return BGK_OK;
}

static int field_sums_range(bgk_ctx *c, int j0, int nrows, double out[4])
{
    if (!c || !out) return fail(BGK_ERR_ARG, "null argument");
    if (j0 < 0 || nrows < 1 || (long long)j0 + nrows > c->Ny)
        return fail(BGK_ERR_ARG, "rows %d..%d outside 0..%d", j0, j0 + nrows - 1, c->Ny - 1);
    int rc = set_device(c);
    if (rc) return rc;
    CK(bgk::launch_field_sums(c, j0, nrows), "field sums");
    CK(cudaMemcpyAsync(c->pinned, c->red, 4 * sizeof(double), cudaMemcpyDeviceToHost, c->stream), "sums copy");
    CK(cudaStreamSynchronize(c->stream), "field sums");
    for (int k = 0; k < 4; k++) out[k] = c->pinned[k];
    for (int k = 0; k < 4; k++)
        if (!std::isfinite(out[k])) return fail(BGK_ERR_NONFINITE, "field sum %d is not finite", k);
    return BGK_OK;
}

int bgk_field_sums(bgk_ctx *c, double out[4])
{
    if (!c) return fail(BGK_ERR_ARG, "null context");
    return field_sums_range(c, 0, c->Ny, out);
}

int bgk_field_sums_rows(bgk_ctx *c, int j0, int nrows, double out[4]) { return field_sums_range(c, j0, nrows, out); }

int bgk_advance(bgk_ctx *c, int nsteps)
{
    if (!c) return fail(BGK_ERR_ARG, "null context");
    if (nsteps < 0) return fail(BGK_ERR_ARG, "nsteps < 0");
    if (nsteps == 0) return BGK_OK;
    return bgk_internal_advance(c, nsteps);
}

int bgk_rows_bytes(const bgk_ctx *c, int nrows, size_t *bytes)
{
    if (!c || !bytes) return fail(BGK_ERR_ARG, "null argument");
    if (nrows < 1 || nrows > c->Ny) return fail(BGK_ERR_ARG, "nrows %d outside 1..%d", nrows, c->Ny);
    *bytes = bgk::rows_bytes(c, nrows);
    return BGK_OK;
}

static int rows_copy(bgk_ctx *c, int j0, int nrows, const void *buf, bool unpack)
{
    if (!c || !buf) return fail(BGK_ERR_ARG, "null argument");
    if (j0 < 0 || nrows < 1 || (long long)j0 + nrows > c->Ny)
        return fail(BGK_ERR_ARG, "rows %d..%d outside 0..%d", j0, j0 + nrows - 1, c->Ny - 1);
    if ((uintptr_t)buf & 15u) return fail(BGK_ERR_ARG, "row buffer is not 16-byte aligned");
    if (!all_bc4(c->p))
        return fail(BGK_ERR_UNSUPPORTED, "packed rows belong to the fused step, which implements the no-slip "
                                         "code 4 on every wall");
    if (c->opt.heat)
        return fail(BGK_ERR_UNSUPPORTED, "the packed-row exchange implements the heated west wall only");
    int rc = set_device(c);
    if (rc) return rc;
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, buf) != cudaSuccess) {
        cudaGetLastError();
        return fail(BGK_ERR_ARG, "row buffer is not a CUDA pointer");
    }
    if (!(at.type == cudaMemoryTypeManaged || (at.type == cudaMemoryTypeDevice && at.device == c->dev)))
        return fail(BGK_ERR_ARG, "row buffer is not device memory of the context's device");
    if ((rc = ensure_fused(c))) return rc;
    CK(bgk::launch_rows_copy(c, j0, nrows, const_cast<void *>(buf), unpack), unpack ? "rows unpack" : "rows pack");
    if (unpack) c->pristine = false;
    return BGK_OK;
}

int bgk_rows_pack(bgk_ctx *c, int j0, int nrows, void *buf) { return rows_copy(c, j0, nrows, buf, false); }

int bgk_rows_unpack(bgk_ctx *c, int j0, int nrows, const void *buf) { return rows_copy(c, j0, nrows, buf, true); }

int bgk_get_it(const bgk_ctx *c, int *it)
{
    if (!c || !it) return fail(BGK_ERR_ARG, "null argument");
    *it = c->it;
    return BGK_OK;
}

int bgk_set_it(bgk_ctx *c, int it)
{
    if (!c) return fail(BGK_ERR_ARG, "null context");
    c->it = it;
    return BGK_OK;
}

int bgk_set_tin(bgk_ctx *c, const double *tin, int ny)
{
    if (!c) return fail(BGK_ERR_ARG, "null context");
    int rc = set_device(c);
    if (rc) return rc;
    drop_step_graphs(c);   /* the halo-ring update reads the tin pointer */
    if (!tin) {
        if (c->tin_rows) { cudaFree(c->tin_rows); c->tin_rows = nullptr; }
        free(c->tin_host);
        c->tin_host = nullptr;
        c->bc_dirty = true;
        return BGK_OK;
    }
    if (ny != c->Ny) return fail(BGK_ERR_ARG, "tin has %d rows, expected Ny = %d", ny, c->Ny);
    if (c->opt.heat & BGK_HEAT_RIGHT)
        return fail(BGK_ERR_UNSUPPORTED, "a per-row tin sets the west wall, which BGK_HEAT_RIGHT leaves adiabatic");
    for (int j = 0; j < ny; j++)
        if (!std::isfinite(tin[j])) return fail(BGK_ERR_ARG, "tin[%d] is not finite", j);
    if (!c->tin_rows) {
        if ((rc = dalloc(&c->tin_rows, (size_t)ny * sizeof(double), "tin"))) return rc;
        c->tin_host = (double *)malloc((size_t)ny * sizeof(double));
        if (!c->tin_host) return fail(BGK_ERR_OOM, "host allocation");
    }
    memcpy(c->tin_host, tin, (size_t)ny * sizeof(double));
    CK(cudaMemcpyAsync(c->tin_rows, c->tin_host, (size_t)ny * sizeof(double), cudaMemcpyHostToDevice, c->stream),
       "tin copy");
    CK(cudaStreamSynchronize(c->stream), "set_tin");
    c->bc_dirty = true;
    return BGK_OK;
}

int bgk_sync(bgk_ctx *c)
{
    if (!c) return fail(BGK_ERR_ARG, "null context");
    int rc = set_device(c);
    if (rc) return rc;
    CK(cudaStreamSynchronize(c->stream), "sync");
    int flag = 0;
    CK(cudaMemcpy(&flag, c->errflag, sizeof(int), cudaMemcpyDeviceToHost), "error flag");
    if (flag) {
        cudaMemset(c->errflag, 0, sizeof(int));
        return fail(BGK_ERR_CUDA, "a bounded wait inside a step kernel gave up (code %d); results are invalid", flag);
    }
    return BGK_OK;
}

int bgk_get_stream(bgk_ctx *c, void **stream)
{
    if (!c || !stream) return fail(BGK_ERR_ARG, "null argument");
    *stream = (void *)c->stream;
    return BGK_OK;
}

/* Snapshot layout: magic, header ints, then raw device buffers. */
static const char kMagic[8] = {'B', 'G', 'K', 'S', 'N', 'A', 'P', '1'};

int bgk_save(bgk_ctx *c, const char *path)
{
    if (!c || !path) return fail(BGK_ERR_ARG, "null argument");
    int rc = set_device(c);
    if (rc) return rc;
    if ((rc = ensure_fused(c))) return rc;
    FILE *fp = fopen(path, "wb");
    if (!fp) return fail(BGK_ERR_IO, "cannot write %s", path);
    const int hdr[8] = {c->Nx, c->Ny, c->opt.precision, c->it, c->P, c->tin_host ? 1 : 0, c->ring ? 1 : 0,
                        c->opt.heat};
    bool ok = fwrite(kMagic, 1, 8, fp) == 8 && fwrite(hdr, sizeof hdr, 1, fp) == 1;
    const size_t popbytes = (size_t)9 * c->plane * c->esz;
    const size_t phibytes = (size_t)c->plane * c->phisz;
    std::vector<char> buf(std::max(popbytes, c->A * sizeof(double)));
    auto put = [&](const void *dev, size_t bytes) {
        if (!ok) return;
        if (cudaMemcpy(buf.data(), dev, bytes, cudaMemcpyDeviceToHost) != cudaSuccess) { ok = false; return; }
        ok = fwrite(buf.data(), 1, bytes, fp) == bytes;
    };
    cudaStreamSynchronize(c->stream);
    put(c->fbuf[c->cur], popbytes);
    put(c->gbuf[c->cur], popbytes);
    put(c->phibuf[c->cur], phibytes);
    put(c->phibuf[c->cur ^ 1], phibytes);
    put(c->tcol[c->cur], (size_t)c->Ny * sizeof(double));
    put(c->corner, 2 * sizeof(double));
    put(c->mrho, c->A * sizeof(double));
    put(c->mT, c->A * sizeof(double));
    put(c->mu, c->A * sizeof(double));
    put(c->mv, c->A * sizeof(double));
    put(c->mphi, c->A * sizeof(double));
    if (c->ring) put(c->fring, (size_t)9 * (size_t)c->ring_len * sizeof(double));
    if (ok && c->opt.precision == BGK_PREC_F16) ok = fwrite(&c->scale, sizeof c->scale, 1, fp) == 1;
    if (ok && c->tin_host) ok = fwrite(c->tin_host, sizeof(double), c->Ny, fp) == (size_t)c->Ny;
    if (fclose(fp) != 0) ok = false;
    if (!ok) return fail(BGK_ERR_IO, "writing snapshot %s failed", path);
    return BGK_OK;
}

int bgk_load(bgk_ctx *c, const char *path)
{
    if (!c || !path) return fail(BGK_ERR_ARG, "null argument");
    int rc = set_device(c);
    if (rc) return rc;
    drop_step_graphs(c);   /* the snapshot may carry other scales or a tin */
    FILE *fp = fopen(path, "rb");
    if (!fp) return fail(BGK_ERR_IO, "cannot read %s", path);
    char mg[8];
    int hdr[8];
    bool ok = fread(mg, 1, 8, fp) == 8 && memcmp(mg, kMagic, 8) == 0 && fread(hdr, sizeof hdr, 1, fp) == 1;
    if (!ok) { fclose(fp); return fail(BGK_ERR_IO, "%s is not a snapshot", path); }
    if (hdr[7] != c->opt.heat) {
        fclose(fp);
        return fail(BGK_ERR_ARG, "snapshot was written with heat bits %d; the context has %d", hdr[7], c->opt.heat);
    }
    if (hdr[0] != c->Nx || hdr[1] != c->Ny || hdr[2] != c->opt.precision || hdr[4] != c->P ||
        hdr[6] != (c->ring ? 1 : 0)) {
        fclose(fp);
        return fail(BGK_ERR_ARG, "snapshot is %dx%d precision %d; context is %dx%d precision %d", hdr[0], hdr[1],
                    hdr[2], c->Nx, c->Ny, c->opt.precision);
    }
    const size_t popbytes = (size_t)9 * c->plane * c->esz;
    const size_t phibytes = (size_t)c->plane * c->phisz;
    std::vector<char> buf(std::max(popbytes, c->A * sizeof(double)));
    auto get = [&](void *dev, size_t bytes) {
        if (!ok) return;
        if (fread(buf.data(), 1, bytes, fp) != bytes) { ok = false; return; }
        ok = cudaMemcpy(dev, buf.data(), bytes, cudaMemcpyHostToDevice) == cudaSuccess;
    };
    cudaStreamSynchronize(c->stream);
    c->cur = 0;
    c->mode = 0;
    c->stage_pos = 0;
    c->pristine = false;
    get(c->fbuf[0], popbytes);
    get(c->gbuf[0], popbytes);
    get(c->phibuf[0], phibytes);
    get(c->phibuf[1], phibytes);
    get(c->tcol[0], (size_t)c->Ny * sizeof(double));
    get(c->corner, 2 * sizeof(double));
    get(c->mrho, c->A * sizeof(double));
    get(c->mT, c->A * sizeof(double));
    get(c->mu, c->A * sizeof(double));
    get(c->mv, c->A * sizeof(double));
    get(c->mphi, c->A * sizeof(double));
    if (c->ring) get(c->fring, (size_t)9 * (size_t)c->ring_len * sizeof(double));
    if (ok && c->opt.precision == BGK_PREC_F16) ok = fread(&c->scale, sizeof c->scale, 1, fp) == 1;
    std::vector<double> tin;
    if (ok && hdr[5]) {
        tin.resize(c->Ny);
        ok = fread(tin.data(), sizeof(double), c->Ny, fp) == (size_t)c->Ny;
    }
    fclose(fp);
    if (!ok) return fail(BGK_ERR_IO, "reading snapshot %s failed", path);
    c->it = hdr[3];
    c->bc_dirty = true;
    return bgk_set_tin(c, hdr[5] ? tin.data() : nullptr, c->Ny);
}

} // extern "C"
