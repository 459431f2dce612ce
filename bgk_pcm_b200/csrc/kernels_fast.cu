/*
 * kernels_fast.cu -- kernels built with multiply-add contraction:
 *  - the FMA variant of the fused FP64 step (same source as the exact one,
 *    fused_f64.cuh; parity with the reference is then within rounding, not
 *    bit-for-bit);
 *  - the reduced-precision forms (FP32 / FP16 deviation storage).
 */
#include <cuda_fp16.h>

#include <atomic>

#include "bgk_internal.h"
#include "bgk_math.cuh"
#include "../../include/bgk_portable_tanh.h"

namespace bgk {
namespace {

__device__ __forceinline__ double select_tanh(double x, int mode)
{
    return mode == BGK_TANH_PORTABLE ? bgk_portable_tanh(x) : tanh(x);
}

#include "fused_f64.cuh"
#include "fused_pipe.cuh"

int strip_height(const bgk_ctx *c)
{
    if (c->tune_H > 0) return c->tune_H;
    const int bx = (c->Nx + FUSED_BX - 1) / FUSED_BX;
    int H = 16;
    while (H > 2 && (long long)bx * ((c->Ny + H - 1) / H) < 148LL * 8) H /= 2;
    return H;
}

} // namespace

cudaError_t launch_fused_lowp(bgk_ctx *c, bool moments);


/* Step pointers of a dataflow launch: s0 steps the current buffers into
 * the other ones, s1 back (no moments written). */
static void flow_ptrs(const bgk_ctx *c, StepPtrs<double> &s0, StepPtrs<double> &s1)
{
    StepPtrs<double> s{};
    s.gW = c->gW; s.pE = c->pE; s.phiW = c->phiW; s.phiE = c->phiE;
    s.plane = c->plane; s.P = c->P; s.NX2 = c->NX2;
    s0 = s;
    s1 = s;
    const int a = c->cur, b = c->cur ^ 1;
    s0.fin = (const double *)c->fbuf[a]; s0.gin = (const double *)c->gbuf[a];
    s0.fout = (double *)c->fbuf[b]; s0.gout = (double *)c->gbuf[b];
    s0.phin = (const double *)c->phibuf[a]; s0.phout = (double *)c->phibuf[b];
    s0.tcin = east_tcol(c, a); s0.tcout = c->tcol[b];
    s1.fin = (const double *)c->fbuf[b]; s1.gin = (const double *)c->gbuf[b];
    s1.fout = (double *)c->fbuf[a]; s1.gout = (double *)c->gbuf[a];
    s1.phin = (const double *)c->phibuf[b]; s1.phout = (double *)c->phibuf[a];
    s1.tcin = east_tcol(c, b); s1.tcout = c->tcol[a];
}

cudaError_t launch_flow_lowp(bgk_ctx *c, int nsteps);

/* nsteps steps of the FMA-contracted FP64 variant or of a reduced-precision
 * form in one dataflow launch (walls of code 4, no moments). */
cudaError_t launch_flow_fast(bgk_ctx *c, int nsteps)
{
    if (c->opt.precision != BGK_PREC_F64) return launch_flow_lowp(c, nsteps);
    StepPtrs<double> s0, s1;
    flow_ptrs(c, s0, s1);
    return launch_flow_pipe_f64(c, s0, s1, nsteps);
}

cudaError_t launch_fused_fast(bgk_ctx *c, bool moments, bool edge_halos)
{
    if (c->opt.precision != BGK_PREC_F64) return launch_fused_lowp(c, moments);
    StepPtrs<double> s{};
    const int src = c->cur, dst = c->cur ^ 1;
    s.fin = (const double *)c->fbuf[src]; s.gin = (const double *)c->gbuf[src];
    s.fout = (double *)c->fbuf[dst]; s.gout = (double *)c->gbuf[dst];
    s.phin = (const double *)c->phibuf[src]; s.phout = (double *)c->phibuf[dst];
    s.tcin = east_tcol(c, src); s.tcout = c->tcol[dst];
    s.gW = c->gW; s.pE = c->pE; s.phiW = c->phiW; s.phiE = c->phiE; s.tin = c->tin_rows;
    s.mrho = c->mrho; s.mT = c->mT; s.mu = c->mu; s.mv = c->mv; s.mphi = c->mphi;
    s.plane = c->plane; s.P = c->P; s.NX2 = c->NX2;
    s.ring = c->fring; s.ring_len = c->ring_len;
    const int H = strip_height(c);
    dim3 grd((c->Nx + FUSED_BX - 1) / FUSED_BX, (c->Ny + H - 1) / H);
    if (c->tune_pipe || c->ring) return launch_fused_pipe_f64(c, s, moments, edge_halos);
    return launch_fused_f64_variant(c, grd, s, H, moments);
}

namespace {

/* ------------------------------------------------------------------------
 * Reduced-precision forms.
 *
 * Stored: deviations fd_k = f_k - w_k*rho0 and gd_k = g_k - w_k*T0 as float
 * (FP32 form) or as half(dev * scale) (FP16 form, one power-of-two scale per
 * distribution); phi as float in both.  Arithmetic is FP32 except the
 * latent-heat update of T (FP64), the east-wall g values and the moments
 * written to the FP64 mirrors.  With the deviations the equilibria become
 *   feqd_k = w_k (rho0 Q_k + drho (1 + Q_k)),  Q_k = poly_k(u,v) - 1,
 * and the regularized BGK update is feqd_k + (1 - omega) C_k S_k(Pi_neq),
 * which is the reference's ft - omega (ft - feq) without forming ft.
 * ---------------------------------------------------------------------- */

template <typename AT>
struct ConstsLP {
    int Nx, Ny;
    AT w[9];
    AT cf[9], cg[9];         /* (1 - omega) * (0.5 w_k / cs2^2)             */
    AT m, q;                 /* -cs2, 1 - cs2                                */
    AT rho0, T0;
    AT T0mTcrit;             /* T0 - T_crit                                  */
    AT inv_T_width;
    AT f_plus, f_minus;
    AT gb;                   /* grav * beta                                  */
    AT omega_f;
    AT inv_omega_f;          /* 1 / omega_f = tau_f                          */
    /* 1 - sum_k w[k] in exact arithmetic over the rounded weights (-7.45e-9
     * for float).  Added to the k = 0 equilibrium times the density and
     * temperature deviations, so that sum_k feq_k = drho and sum_k geq_k =
     * dT hold to rounding.  Without it every collision multiplies the
     * deviations by (1 + 7.45e-9): over 20,000 steps a systematic drift of
     * 1.5e-4 of (T - T0), which moves the melting front. */
    AT wcorr;
    /* The same rounding scales the first moment of the equilibria:
     * 3 sum_k w_k c_kx^2 = 1 + 2^-27 for the float weights, so every
     * collision multiplied the momentum (and the heat flux) by that factor,
     * a uniform anti-damping force that made the FP32 form's velocity drift
     * from the FP64 path's in proportion to the step count (6.5e-5 of max
     * |u| after 10k steps at 4096^2).  mcorr = (3 sum w c^2 - 1)/2 times
     * rho*u (T*u) is taken from the +x and added to the -x population (and
     * likewise in y), which leaves the mass and the second moments that the
     * regularization reads unchanged. */
    AT mcorr;
    double dts, T0d, rho0d;
    double T0mTcrit_d, inv_T_width_d;
    double w_d[9];
};

template <typename S> struct Codec;
/* ld: read-only global load (ld.global.nc) -- global memory only.
 * lds: plain load, for the shared-memory stages of the pipeline kernel. */
template <> struct Codec<float> {
    static __device__ __forceinline__ float ld(const float *p, float) { return __ldg(p); }
    static __device__ __forceinline__ float lds(const float *p, float) { return *p; }
    static __device__ __forceinline__ void st(float *p, float v, float) { *p = v; }
};
template <> struct Codec<__half> {
    static __device__ __forceinline__ float ld(const __half *p, float inv) { return __half2float(__ldg(p)) * inv; }
    static __device__ __forceinline__ float lds(const __half *p, float inv) { return __half2float(*p) * inv; }
    static __device__ __forceinline__ void st(__half *p, float v, float s) { *p = __float2half_rn(v * s); }
};

__device__ __forceinline__ float tanh_lp(float x, int mode)
{
    return mode == BGK_TANH_PORTABLE ? (float)bgk_portable_tanh((double)x) : tanhf(x);
}

template <typename AT>
__device__ __forceinline__ void qpoly(AT u, AT v, AT *Q)
{
    const AT uu = u * u, vv = v * v, uv = (AT)1.5 * (uu + vv);
    const AT upv = u + v, umv = u - v;
    const AT three = (AT)3, f45 = (AT)4.5;
    Q[0] = -uv;
    Q[1] = three * u + f45 * uu - uv;
    Q[2] = three * v + f45 * vv - uv;
    Q[3] = -three * u + f45 * uu - uv;
    Q[4] = -three * v + f45 * vv - uv;
    Q[5] = three * upv + f45 * upv * upv - uv;
    Q[6] = -three * umv + f45 * umv * umv - uv;
    Q[7] = -three * upv + f45 * upv * upv - uv;
    Q[8] = three * umv + f45 * umv * umv - uv;
}

template <typename AT>
__device__ __forceinline__ void reg_relax_lp(const ConstsLP<AT> &c, const AT *in, const AT *eq, const AT *cc,
                                             AT *out)
{
    AT d[9];
#pragma unroll
    for (int k = 0; k < 9; k++) d[k] = in[k] - eq[k];
    const AT m = c.m, q = c.q;
    const AT pxx = m * (d[0] + d[2] + d[4]) + q * (d[1] + d[3] + d[5] + d[6] + d[7] + d[8]);
    const AT pyy = m * (d[0] + d[1] + d[3]) + q * (d[2] + d[4] + d[5] + d[6] + d[7] + d[8]);
    const AT pxy = d[5] - d[6] + d[7] - d[8];
    const AT s0 = m * (pxx + pyy);
    const AT s1 = q * pxx + m * pyy;
    const AT s2 = m * pxx + q * pyy;
    const AT sqq = q * (pxx + pyy);
    const AT s5 = sqq + (AT)2 * pxy, s6 = sqq - (AT)2 * pxy;
    out[0] = eq[0] + cc[0] * s0;
    out[1] = eq[1] + cc[1] * s1;
    out[2] = eq[2] + cc[2] * s2;
    out[3] = eq[3] + cc[3] * s1;
    out[4] = eq[4] + cc[4] * s2;
    out[5] = eq[5] + cc[5] * s5;
    out[6] = eq[6] + cc[6] * s6;
    out[7] = eq[7] + cc[7] * s5;
    out[8] = eq[8] + cc[8] * s6;
}

template <typename S, typename PT>
struct LpPtrs {
    const S *fin, *gin;
    S *fout, *gout;
    const PT *phin;
    PT *phout;
    const double *tcin;
    double *tcout;
    const double *gW, *pE, *phiW, *phiE, *corner;
    double *mrho, *mT, *mu, *mv, *mphi;
    long long plane;
    int P, NX2;
    float sf, sg, inv_sf, inv_sg;
};

/* PT: storage and arithmetic type of the phase field (float, or double
 * with the phase-field update -- selector terms, tanh, liquid fraction --
 * evaluated in FP64). */
template <typename PT>
__device__ __forceinline__ PT tanh_pt(PT x, int mode);
template <>
__device__ __forceinline__ float tanh_pt<float>(float x, int mode) { return tanh_lp(x, mode); }
template <>
__device__ __forceinline__ double tanh_pt<double>(double x, int mode)
{
    return mode == BGK_TANH_PORTABLE ? bgk_portable_tanh(x) : tanh(x);
}

/* Phase-field storage.  The update of STEP_7/phase_field.f90:22-48 needs,
 * per cell, the two bases 1 + phi and 1 - phi (of the selector terms
 * (1/2 (1 +- phi))^2 and of the update itself).  A codec gives both for a
 * stored word, phi in double, and the encoding of an updated value; phi is
 * stored as itself, in float or in double. */
template <typename PS> struct PhiCodec;
template <> struct PhiCodec<float> {
    using A = float;
    static __device__ __forceinline__ float onep(float s) { return 1.f + s; }
    static __device__ __forceinline__ float onem(float s) { return 1.f - s; }
    static __device__ __forceinline__ double dec(float s) { return (double)s; }
    static __device__ __forceinline__ float from_d(double phi) { return (float)phi; }
    static __device__ __forceinline__ float update(float s, float kpp, float kmm)
    {
        return s + (0.5f * kpp * (1.f - s) - 0.5f * kmm * (1.f + s));
    }
};
template <> struct PhiCodec<double> {
    using A = double;
    static __device__ __forceinline__ double onep(double s) { return 1.0 + s; }
    static __device__ __forceinline__ double onem(double s) { return 1.0 - s; }
    static __device__ __forceinline__ double dec(double s) { return s; }
    static __device__ __forceinline__ double from_d(double phi) { return phi; }
    static __device__ __forceinline__ double update(double s, double kpp, double kmm)
    {
        return s + (0.5 * kpp * (1.0 - s) - 0.5 * kmm * (1.0 + s));
    }
};

/* One node of a reduced-precision step after its pulls (deviations in AT):
 * momentsPre, phase field (PT), latent heat (FP64), forces, collision,
 * stores, moments.  Shared by the register-pull and pipeline kernels.
 *
 * Conservation closure.  In exact arithmetic the collision leaves sum_k f_k
 * and sum_k g_k unchanged (the latter after the latent heat).  Evaluated in
 * FP32 it does not: the g equilibrium carries terms w_k T0 Q_k of ~30 K
 * against an energy deviation of a few K, and in a steady flow the same
 * rounding recurs at a node every step, so it acts as a spurious heat (and
 * mass) source.  At 256^2 that source moved T by 1.7e-4 dT and the melt
 * front by 0.002 cells after 20k steps.  So the rest populations are the
 * residuals: f_0 = drho - sum_{k>0} f_k in AT, and g_0 = dT - sum_{k>0} g_k
 * in FP64, with dT, the node's energy deviation, also summed and carried
 * through the latent heat in FP64 (the energy bookkeeping of the
 * liquid-fraction update).  The stored populations then carry the node's
 * mass and energy up to the rounding of f_0 and g_0 themselves. */
template <typename S, typename PT, typename AT, int TANH, bool MOM>
__device__ __forceinline__ void node_lp(const LpPtrs<S, PT> &s, const ConstsLP<AT> &c, int x, int y, long long cc,
                                        bool E, AT *f, AT *g, typename PhiCodec<PT>::A kp,
                                        typename PhiCodec<PT>::A km, PT q0)
{
    using PC = PhiCodec<PT>;
    using PA = typename PC::A;
    using C = Codec<S>;
    const long long pl = s.plane;
    /* momentsPre (deviations; the energy in FP64) */
    AT drho = 0;
    double dTd = 0.0;
#pragma unroll
    for (int k = 0; k < 9; k++) { drho += f[k]; dTd += (double)g[k]; }
    AT dT = (AT)dTd;
    const AT rho = c.rho0 + drho;
    const AT irho = (AT)1 / rho;
    AT u = irho * (f[1] - f[3] + f[5] - f[6] - f[7] + f[8]);
    AT v = irho * (f[2] - f[4] + f[5] + f[6] - f[7] - f[8]);
    const AT dT2 = dT, u2 = u, v2 = v;

    /* phase_field (in PA) */
    const PA one = (PA)1, half = (PA)0.5;
    const PA th = tanh_pt<PA>(((PA)c.T0mTcrit_d + (PA)dT) * (PA)c.inv_T_width_d, TANH);
    const PA kpp = kp * (PA)0.125 * (half * (one + th));
    const PA kmm = km * (PA)0.125 * (half * (one - th));
    const PT qn = PC::update(q0, kpp, kmm);
    const double p0d = PC::dec(q0), pnd = PC::dec(qn);
    const AT phn = (AT)pnd;

    /* forces: latent heat in FP64, on the change of the stored phi */
    dTd -= c.dts * (pnd - p0d) * 0.5;
    dT = (AT)dTd;
    const AT T = c.T0 + dT;
    const AT omp = (AT)1 - phn;
    const AT forceY = rho * c.gb * T * ((AT)1 + (AT)0.5 * phn) - (AT)0.5 * v * omp;
    const AT forceX = (AT)-0.5 * u * omp;
    const AT iw = irho * c.inv_omega_f;     /* 1 / (omega_f rho), one division less */
    u = u + forceX * iw;
    v = v + forceY * iw;

    /* collision */
    AT Q[9], eq[9], out[9];
    qpoly(u, v, Q);
#pragma unroll
    for (int k = 0; k < 9; k++) eq[k] = c.w[k] * (c.rho0 * Q[k] + drho * ((AT)1 + Q[k]));
    eq[0] += c.wcorr * drho;
    {
        const AT mx = c.mcorr * rho * u, my = c.mcorr * rho * v;
        eq[1] -= mx; eq[3] += mx;
        eq[2] -= my; eq[4] += my;
    }
    reg_relax_lp(c, f, eq, c.cf, out);
    {
        AT r = drho;                        /* mass closure */
#pragma unroll
        for (int k = 1; k < 9; k++) r -= out[k];
        out[0] = r;
    }
#pragma unroll
    for (int k = 0; k < 9; k++) { C::st(s.fout + k * pl + cc, (float)out[k], s.sf); f[k] = out[k]; }
#pragma unroll
    for (int k = 0; k < 9; k++) eq[k] = c.w[k] * (c.T0 * Q[k] + dT * ((AT)1 + Q[k]));
    eq[0] += c.wcorr * dT;
    {
        const AT mx = c.mcorr * T * u, my = c.mcorr * T * v;
        eq[1] -= mx; eq[3] += mx;
        eq[2] -= my; eq[4] += my;
    }
    reg_relax_lp(c, g, eq, c.cg, out);
    {
        double r = dTd;                     /* energy closure */
#pragma unroll
        for (int k = 1; k < 9; k++) r -= (double)out[k];
        out[0] = (AT)r;
    }
#pragma unroll
    for (int k = 0; k < 9; k++) C::st(s.gout + k * pl + cc, (float)out[k], s.sg);
    s.phout[cc] = qn;

    if (MOM || E) {
        AT sg = 0;
#pragma unroll
        for (int k = 0; k < 9; k++) sg += out[k];
        const double Tm = c.T0d + 0.5 * ((double)sg + (double)dT2);
        if (E) s.tcout[y] = Tm;
        if (MOM) {
            AT sf = 0;
#pragma unroll
            for (int k = 0; k < 9; k++) sf += f[k];
            const AT rm = c.rho0 + sf;
            const AT irm = (AT)1 / rm;
            const AT tu = irm * (f[1] - f[3] + f[5] - f[6] - f[7] + f[8]);
            const AT tv = irm * (f[2] - f[4] + f[5] + f[6] - f[7] - f[8]);
            const size_t q = (size_t)(x + 1) + (size_t)s.NX2 * (size_t)(y + 1);
            s.mrho[q] = (double)c.rho0 + (double)sf;
            s.mT[q] = Tm;
            s.mu[q] = 0.5 * ((double)tu + (double)u2);
            s.mv[q] = 0.5 * ((double)tv + (double)v2);
            s.mphi[q] = pnd;
        }
    }
}

template <typename S, typename PT, typename AT, int TANH, bool MOM>
__global__ void __launch_bounds__(FUSED_BX)
fused_lowp_kernel(LpPtrs<S, PT> s, ConstsLP<AT> c, int H, int pf)
{
    const int Nx = c.Nx, Ny = c.Ny;
    const int x = blockIdx.x * FUSED_BX + threadIdx.x;
    if (x >= Nx) return;
    const int y0 = blockIdx.y * H;
    const int y1 = min(y0 + H, Ny);
    const long long pl = s.plane;
    const int P = s.P;
    const bool W = (x == 0), E = (x == Nx - 1);
    const S *__restrict__ F = s.fin;
    const S *__restrict__ G = s.gin;
    const PT *__restrict__ PH = s.phin;
    const float isf = s.inv_sf, isg = s.inv_sg;

    using PC = PhiCodec<PT>;
    using PA = typename PC::A;
    PA ap[3], am[3];   /* per row y-1, y, y+1: sums over x-1..x+1 of (1/2 (1 +- phi))^2 */
    PT pc[3];          /* and the stored phi of column x */
    auto load_row = [&](int r, int slot) {
        const int rc = r < 0 ? 0 : (r >= Ny ? Ny - 1 : r);
        const PT *row = PH + (long long)rc * P;
        const PT pL = W ? PC::from_d(s.phiW[rc]) : row[x - 1];
        const PT pM = row[x];
        const PT pR = E ? PC::from_d(s.phiE[rc]) : row[x + 1];
        const PA h = (PA)0.5;
        const PA a0 = h * PC::onep(pL), a1 = h * PC::onep(pM), a2 = h * PC::onep(pR);
        const PA b0 = h * PC::onem(pL), b1 = h * PC::onem(pM), b2 = h * PC::onem(pR);
        ap[slot] = a0 * a0 + a1 * a1 + a2 * a2;
        am[slot] = b0 * b0 + b1 * b1 + b2 * b2;
        pc[slot] = pM;
    };
    load_row(y0 - 1, 0);
    load_row(y0, 1);

    const int x0 = blockIdx.x * FUSED_BX, ncols = min(FUSED_BX, Nx - x0);
    for (int y = y0; y < y1; y++) {
        if (pf > 0) prefetch_row(F, G, PH, pl, P, x0, ncols, y + pf, Ny);
        load_row(y + 1, 2);
        const bool Sb = (y == 0), N = (y == Ny - 1);
        const long long cc = (long long)y * P + x;
        AT f[9], g[9];
        using C = Codec<S>;
        f[0] = (AT)C::ld(F + cc, isf);
        f[1] = (AT)C::ld(W ? F + 3 * pl + cc : F + 1 * pl + cc - 1, isf);
        f[2] = (AT)C::ld(Sb ? F + 4 * pl + cc : F + 2 * pl + cc - P, isf);
        f[3] = (AT)C::ld(E ? F + 1 * pl + cc : F + 3 * pl + cc + 1, isf);
        f[4] = (AT)C::ld(N ? F + 2 * pl + cc : F + 4 * pl + cc + P, isf);
        f[5] = (AT)C::ld((W || Sb) ? F + 7 * pl + cc : F + 5 * pl + cc - P - 1, isf);
        f[6] = (AT)C::ld((E || Sb) ? F + 8 * pl + cc : F + 6 * pl + cc - P + 1, isf);
        f[7] = (AT)C::ld((E || N) ? F + 5 * pl + cc : F + 7 * pl + cc + P + 1, isf);
        f[8] = (AT)C::ld((W || N) ? F + 6 * pl + cc : F + 8 * pl + cc + P - 1, isf);
        if (E && Sb) f[6] = (AT)(s.corner[0] - c.w_d[6] * c.rho0d);
        if (E && N) f[7] = (AT)(s.corner[1] - c.w_d[7] * c.rho0d);

        const int ym = Sb ? y : y - 1, yp = N ? y : y + 1;
        const long long cm = (long long)ym * P + x, cp = (long long)yp * P + x;
        g[0] = (AT)C::ld(G + cc, isg);
        g[2] = (AT)C::ld(G + 2 * pl + cm, isg);
        g[4] = (AT)C::ld(G + 4 * pl + cp, isg);
        if (W) {
            g[1] = (AT)(s.gW[y] - c.w_d[1] * c.T0d);
            g[5] = (AT)(s.gW[Ny + ym] - c.w_d[5] * c.T0d);
            g[8] = (AT)(s.gW[2 * Ny + yp] - c.w_d[8] * c.T0d);
        } else {
            g[1] = (AT)C::ld(G + 1 * pl + cc - 1, isg);
            g[5] = (AT)C::ld(G + 5 * pl + cm - 1, isg);
            g[8] = (AT)C::ld(G + 8 * pl + cp - 1, isg);
        }
        if (E) {
            g[3] = (AT)(c.w_d[3] * s.tcin[y] * s.pE[y] - c.w_d[3] * c.T0d);
            g[6] = (AT)(c.w_d[6] * s.tcin[ym] * s.pE[Ny + ym] - c.w_d[6] * c.T0d);
            g[7] = (AT)(c.w_d[7] * s.tcin[yp] * s.pE[2 * Ny + yp] - c.w_d[7] * c.T0d);
        } else {
            g[3] = (AT)C::ld(G + 3 * pl + cc + 1, isg);
            g[6] = (AT)C::ld(G + 6 * pl + cm + 1, isg);
            g[7] = (AT)C::ld(G + 7 * pl + cp + 1, isg);
        }

        node_lp<S, PT, AT, TANH, MOM>(s, c, x, y, cc, E, f, g, (ap[0] + ap[1]) + ap[2], (am[0] + am[1]) + am[2], pc[1]);

        ap[0] = ap[1]; ap[1] = ap[2];
        am[0] = am[1]; am[1] = am[2];
        pc[0] = pc[1]; pc[1] = pc[2];
    }
}

/* Pipeline consumers of the reduced-precision step, shared by the
 * per-step kernel and the multi-step (dataflow) kernel below.
 *
 * lp_window_start: the 3x3 phase-field window's first two rows (y0-1, y0)
 * for column x, from global memory. */
template <typename S, typename PT, typename AT>
__device__ __forceinline__ void lp_window_start(const LpPtrs<S, PT> &s, const ConstsLP<AT> &c, int x, int y0,
                                                bool W, bool E, typename PhiCodec<PT>::A *ap,
                                                typename PhiCodec<PT>::A *am, PT *pc)
{
    using PC = PhiCodec<PT>;
    using PA = typename PC::A;
    const PA h = (PA)0.5;
    const int Ny = c.Ny;
    for (int slot = 0; slot < 2; slot++) {
        const int rr = y0 - 1 + slot;
        const int rc = rr < 0 ? 0 : (rr >= Ny ? Ny - 1 : rr);
        const PT *row = s.phin + (long long)rc * s.P;
        const PT pL = W ? PC::from_d(s.phiW[rc]) : row[x - 1];
        const PT pM = row[x];
        const PT pR = E ? PC::from_d(s.phiE[rc]) : row[x + 1];
        const PA a0 = h * PC::onep(pL), a1 = h * PC::onep(pM), a2 = h * PC::onep(pR);
        const PA b0 = h * PC::onem(pL), b1 = h * PC::onem(pM), b2 = h * PC::onem(pR);
        ap[slot] = a0 * a0 + a1 * a1 + a2 * a2;
        am[slot] = b0 * b0 + b1 * b1 + b2 * b2;
        pc[slot] = pM;
    }
}

/* lp_window_stage: the same two rows from a dataflow stage (slots 1, 2). */
template <typename S, typename PT, typename AT>
__device__ __forceinline__ void lp_window_stage(const LpPtrs<S, PT> &s, const ConstsLP<AT> &c, int y0, int tid, bool W,
                                                bool E, const unsigned char *stage, typename PhiCodec<PT>::A *ap,
                                                typename PhiCodec<PT>::A *am, PT *pc)
{
    using Gm = PipeGeom<S, PT>;
    using PC = PhiCodec<PT>;
    using PA = typename PC::A;
    const PA h = (PA)0.5;
    const int Ny = c.Ny;
    for (int slot = 0; slot < 2; slot++) {
        const int rr = y0 - 1 + slot;
        const int rc = rr < 0 ? 0 : (rr >= Ny ? Ny - 1 : rr);
        const PT *row = reinterpret_cast<const PT *>(stage + 18 * Gm::POP_BYTES + (1 + slot) * Gm::PHI_BYTES);
        const PT pL = W ? PC::from_d(s.phiW[rc]) : row[Gm::ALP + tid - 1];
        const PT pM = row[Gm::ALP + tid];
        const PT pR = E ? PC::from_d(s.phiE[rc]) : row[Gm::ALP + tid + 1];
        const PA a0 = h * PC::onep(pL), a1 = h * PC::onep(pM), a2 = h * PC::onep(pR);
        const PA b0 = h * PC::onem(pL), b1 = h * PC::onem(pM), b2 = h * PC::onem(pR);
        ap[slot] = a0 * a0 + a1 * a1 + a2 * a2;
        am[slot] = b0 * b0 + b1 * b1 + b2 * b2;
        pc[slot] = pM;
    }
}

/* lp_row: node (x, y) from a filled stage: the window's new row y+1, the
 * pulls (bounce-back and boundary values from global memory), node_lp, and
 * the window shift. */
template <typename S, typename PT, typename AT, int TANH, bool MOM>
__device__ __forceinline__ void lp_row(const LpPtrs<S, PT> &s, const ConstsLP<AT> &c, const unsigned char *stage,
                                       int x, int y, int tid, bool W, bool E, typename PhiCodec<PT>::A *ap,
                                       typename PhiCodec<PT>::A *am, PT *pc)
{
    using Gm = PipeGeom<S, PT>;
    using C = Codec<S>;
    using PC = PhiCodec<PT>;
    using PA = typename PC::A;
    const PA h = (PA)0.5;
    const int Ny = c.Ny;
    const long long pl = s.plane;
    const S *__restrict__ F = s.fin;
    const float isf = s.inv_sf, isg = s.inv_sg;
    const S *sp = reinterpret_cast<const S *>(stage);
    const S *sg = sp + 9 * Gm::RW;
    const PT *sphi = reinterpret_cast<const PT *>(stage + 18 * Gm::POP_BYTES);
    const bool Sb = (y == 0), N = (y == Ny - 1);
    const long long cc = (long long)y * s.P + x;
    const int col = tid + Gm::AL;
    {
        const int rc = (y + 1 >= Ny) ? Ny - 1 : y + 1;
        const PT pL = W ? PC::from_d(s.phiW[rc]) : sphi[Gm::ALP + tid - 1];
        const PT pM = sphi[Gm::ALP + tid];
        const PT pR = E ? PC::from_d(s.phiE[rc]) : sphi[Gm::ALP + tid + 1];
        const PA a0 = h * PC::onep(pL), a1 = h * PC::onep(pM), a2 = h * PC::onep(pR);
        const PA b0 = h * PC::onem(pL), b1 = h * PC::onem(pM), b2 = h * PC::onem(pR);
        ap[2] = a0 * a0 + a1 * a1 + a2 * a2;
        am[2] = b0 * b0 + b1 * b1 + b2 * b2;
        pc[2] = pM;
    }
    AT f[9], g[9];
    f[0] = (AT)C::lds(sp + 0 * Gm::RW + col, isf);
    f[1] = (AT)C::lds(W ? sp + 3 * Gm::RW + col : sp + 1 * Gm::RW + col - 1, isf);
    f[2] = (AT)C::lds(sp + 2 * Gm::RW + col, isf);
    f[3] = (AT)C::lds(E ? sp + 1 * Gm::RW + col : sp + 3 * Gm::RW + col + 1, isf);
    f[4] = (AT)C::lds(sp + 4 * Gm::RW + col, isf);
    f[5] = (AT)C::lds(sp + 5 * Gm::RW + col - 1, isf);
    f[6] = (AT)C::lds(sp + 6 * Gm::RW + col + 1, isf);
    f[7] = (AT)C::lds(sp + 7 * Gm::RW + col + 1, isf);
    f[8] = (AT)C::lds(sp + 8 * Gm::RW + col - 1, isf);
    if (W || E || Sb || N) {
        if (Sb) f[2] = (AT)C::ld(F + 4 * pl + cc, isf);
        if (N) f[4] = (AT)C::ld(F + 2 * pl + cc, isf);
        if (W || Sb) f[5] = (AT)C::ld(F + 7 * pl + cc, isf);
        if (E || Sb) f[6] = (E && Sb) ? (AT)(s.corner[0] - c.w_d[6] * c.rho0d) : (AT)C::ld(F + 8 * pl + cc, isf);
        if (E || N) f[7] = (E && N) ? (AT)(s.corner[1] - c.w_d[7] * c.rho0d) : (AT)C::ld(F + 5 * pl + cc, isf);
        if (W || N) f[8] = (AT)C::ld(F + 6 * pl + cc, isf);
    }
    const int ym = Sb ? y : y - 1, yp = N ? y : y + 1;
    g[0] = (AT)C::lds(sg + 0 * Gm::RW + col, isg);
    g[2] = (AT)C::lds(sg + 2 * Gm::RW + col, isg);
    g[4] = (AT)C::lds(sg + 4 * Gm::RW + col, isg);
    if (W) {
        g[1] = (AT)(s.gW[y] - c.w_d[1] * c.T0d);
        g[5] = (AT)(s.gW[Ny + ym] - c.w_d[5] * c.T0d);
        g[8] = (AT)(s.gW[2 * Ny + yp] - c.w_d[8] * c.T0d);
    } else {
        g[1] = (AT)C::lds(sg + 1 * Gm::RW + col - 1, isg);
        g[5] = (AT)C::lds(sg + 5 * Gm::RW + col - 1, isg);
        g[8] = (AT)C::lds(sg + 8 * Gm::RW + col - 1, isg);
    }
    if (E) {
        g[3] = (AT)(c.w_d[3] * s.tcin[y] * s.pE[y] - c.w_d[3] * c.T0d);
        g[6] = (AT)(c.w_d[6] * s.tcin[ym] * s.pE[Ny + ym] - c.w_d[6] * c.T0d);
        g[7] = (AT)(c.w_d[7] * s.tcin[yp] * s.pE[2 * Ny + yp] - c.w_d[7] * c.T0d);
    } else {
        g[3] = (AT)C::lds(sg + 3 * Gm::RW + col + 1, isg);
        g[6] = (AT)C::lds(sg + 6 * Gm::RW + col + 1, isg);
        g[7] = (AT)C::lds(sg + 7 * Gm::RW + col + 1, isg);
    }
    node_lp<S, PT, AT, TANH, MOM>(s, c, x, y, cc, E, f, g, (ap[0] + ap[1]) + ap[2], (am[0] + am[1]) + am[2], pc[1]);
    ap[0] = ap[1]; ap[1] = ap[2];
    am[0] = am[1]; am[1] = am[2];
    pc[0] = pc[1]; pc[1] = pc[2];
}

/* The reduced-precision step on the shared-memory pipeline of
 * fused_pipe.cuh: identical producer, consumers decode deviations from the
 * stage and call node_lp. */
template <typename S, typename PT, typename AT, int D, int TANH, bool MOM>
__global__ void __launch_bounds__(PIPE_THREADS, 4)
fused_pipe_lp_kernel(LpPtrs<S, PT> s, ConstsLP<AT> c, PipeSched sch, int *errflag)
{
    using Gm = PipeGeom<S, PT>;
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t *full = reinterpret_cast<uint64_t *>(smem);
    uint64_t *empty = full + D;
    unsigned char *stages = smem + Gm::HEADER;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int Nx = c.Nx, Ny = c.Ny;
    if (tid == 0) {
        for (int d = 0; d < D; d++) {
            mbar_init(&full[d], 1);
            mbar_init(&empty[d], PIPE_CWARPS);
        }
        mbar_fence_init();
    }
    __syncthreads();
    pdl_wait();
    if (warp == PIPE_CWARPS) {
        if (lane != 0) return;
        PipeIter it;
        long long r = 0;
        bool ok = it.start(sch, Ny);
        while (ok) {
            const int st = (int)(r % D);
            if (r >= D && !mbar_wait(&empty[st], (uint32_t)(((r / D) - 1) & 1))) {
                atomicExch(errflag, 1);
                break;
            }
            pipe_issue<S, PT>(s.fin, s.gin, s.phin, s.plane, s.P, Ny, it.x0, it.y,
                              stages + (size_t)st * Gm::STAGE_BYTES, &full[st]);
            r++;
            ok = it.next();
        }
        for (long long q = (r > D ? r - D : 0); q < r; q++)
            if (!mbar_wait(&full[q % D], (uint32_t)((q / D) & 1))) atomicExch(errflag, 2);
        pdl_allow_next();
        return;
    }
    using PA = typename PhiCodec<PT>::A;
    PipeIter it;
    long long r = 0;
    bool ok = it.start(sch, Ny);
    while (ok) {
        const int x = it.x0 + tid;
        const bool active = x < Nx;
        const bool W = (x == 0), E = (x == Nx - 1);
        PA ap[3], am[3];   /* per row y-1, y, y+1: sums over x-1..x+1 of (1/2 (1 +- phi))^2 */
        PT pc[3];          /* and the stored phi of column x */
        if (active) lp_window_start(s, c, x, it.y, W, E, ap, am, pc);
        const int tile = it.t;
        bool failed = false;
        do {
            const int y = it.y;
            const int st = (int)(r % D);
            if (!__all_sync(0xffffffffu, mbar_wait(&full[st], (uint32_t)((r / D) & 1)))) {
                atomicExch(errflag, 3);
                failed = true;
                break;
            }
            if (active)
                lp_row<S, PT, AT, TANH, MOM>(s, c, stages + (size_t)st * Gm::STAGE_BYTES, x, y, tid, W, E, ap, am,
                                             pc);
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty[st]);
            r++;
            ok = it.next();
        } while (ok && it.t == tile);
        if (failed) break;
    }
    pdl_allow_next();
}

/* Multi-step (dataflow) form of the reduced-precision pipeline: the
 * schedule, its ordering and its waits are described with FlowCtl in
 * pipe_common.cuh. */
template <typename S, typename PT, typename AT, int D, int TANH>
__global__ void __launch_bounds__(PIPE_THREADS, 4)
flow_pipe_lp_kernel(LpPtrs<S, PT> s0, LpPtrs<S, PT> s1, ConstsLP<AT> c, PipeSched sch, FlowCtl fl, int *errflag)
{
    static_assert(D <= 8, "stage tags hold 8 stages");
    using Gm = PipeGeom<S, PT>;
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ int warps_done[8];
    uint64_t *full = reinterpret_cast<uint64_t *>(smem);
    uint64_t *empty = full + D;
    StageTag *tag = reinterpret_cast<StageTag *>(smem + 128);
    unsigned char *stages = smem + Gm::HEADER;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int Nx = c.Nx, Ny = c.Ny;
    if (tid == 0) {
        for (int d = 0; d < D; d++) {
            mbar_init(&full[d], 1);
            mbar_init(&empty[d], PIPE_CWARPS);
            warps_done[d] = 0;
        }
        mbar_fence_init();
    }
    __syncthreads();
    const long long total = (long long)fl.nsteps * sch.ntiles;
    if (warp == PIPE_CWARPS) {
        /* ---------------- producer ---------------- */
        if (lane != 0) return;
        long long r = 0;
        bool bad = false;
        /* the next ticket is claimed one tile ahead, so its round trip
         * overlaps the current tile's copies; a claimed ticket is always
         * larger than the one in progress, so the schedule stays free of
         * deadlock */
        unsigned long long next = atomicAdd(fl.ticket, 1ull);
        while (!bad) {
            const unsigned long long item = next;
            if (item >= (unsigned long long)total) break;
            next = atomicAdd(fl.ticket, 1ull);
            const int k = (int)(item / sch.ntiles), t = (int)(item % sch.ntiles);
            if (k > 0) {
                /* items of the first step read what earlier launches wrote
                 * (ordered by the launch boundary); later ones read other
                 * CTAs' stores of this launch through the bulk copies */
                if (!flow_deps(fl.done, t, sch, (unsigned)k + fl.stall, errflag)) {
                    atomicExch(errflag, 4);
                    break;
                }
                fence_proxy_async_global();
            }
            const LpPtrs<S, PT> &sk = (k & 1) ? s1 : s0;
            const int x0 = (t % sch.nbands) * sch.bx, y0 = (t / sch.nbands) * sch.H;
            const int y1 = min(y0 + sch.H, Ny);
            for (int y = y0; y < y1; y++) {
                const int st = (int)(r % D);
                if (r >= D && !mbar_wait(&empty[st], (uint32_t)(((r / D) - 1) & 1))) {
                    atomicExch(errflag, 1);
                    bad = true;
                    break;
                }
                tag[st] = StageTag{k, t, y, (y == y0 ? TAG_FIRST : 0) | (y == y1 - 1 ? TAG_LAST : 0)};
                pipe_issue_w<S, PT>(sk.fin, sk.gin, sk.phin, sk.plane, sk.P, Ny, x0, y, y == y0,
                                    stages + (size_t)st * Gm::STAGE_BYTES_W, &full[st]);
                r++;
            }
        }
        /* a stage with no data tells the consumers to leave */
        if (!bad) {
            const int st = (int)(r % D);
            if (r < D || mbar_wait(&empty[st], (uint32_t)(((r / D) - 1) & 1))) {
                tag[st] = StageTag{-1, -1, -1, TAG_END};
                mbar_arrive(&full[st]);
                r++;
            } else {
                atomicExch(errflag, 1);
            }
        }
        /* do not retire while copies into this CTA's shared memory are in flight */
        for (long long q = (r > D ? r - D : 0); q < r; q++)
            if (!mbar_wait(&full[q % D], (uint32_t)((q / D) & 1))) atomicExch(errflag, 2);
        return;
    }
    /* ---------------- consumers ---------------- */
    using PA = typename PhiCodec<PT>::A;
    PA ap[3], am[3];
    PT pc[3];
    for (long long r = 0;; r++) {
        const int st = (int)(r % D);
        if (!__all_sync(0xffffffffu, mbar_wait(&full[st], (uint32_t)((r / D) & 1)))) {
            atomicExch(errflag, 3);
            break;
        }
        const StageTag tg = tag[st];
        if (tg.flags & TAG_END) break;
        const LpPtrs<S, PT> &sk = (tg.k & 1) ? s1 : s0;
        const int x = (tg.t % sch.nbands) * sch.bx + tid;
        const bool W = (x == 0), E = (x == Nx - 1);
        if (x < Nx) {
            const unsigned char *stg = stages + (size_t)st * Gm::STAGE_BYTES_W;
            if (tg.flags & TAG_FIRST) lp_window_stage(sk, c, tg.y, tid, W, E, stg, ap, am, pc);
            lp_row<S, PT, AT, TANH, false>(sk, c, stg, x, tg.y, tid, W, E, ap, am, pc);
        }
        if ((tg.flags & TAG_LAST) && fl.nsteps > 1) {
            /* this warp's part of the tile is stored: the warp barrier orders
             * the lanes' stores before lane 0's fence, whose cumulativity
             * makes them visible device-wide (the pattern of a grid-wide
             * barrier); the last of the four warps publishes the tile's step */
            __syncwarp();
            if (lane == 0) {
                __threadfence();
                if (atomicAdd(&warps_done[st], 1) == PIPE_CWARPS - 1) {
                    warps_done[st] = 0;
                    __threadfence();
                    st_release_u32(fl.done + tg.t, (unsigned)tg.k + 1);
                }
            }
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[st]);
    }
}

template <typename S, typename PT, typename AT, int D, int T, bool M>
cudaError_t pipe_lp_launch(bgk_ctx *c, const LpPtrs<S, PT> &s, const ConstsLP<AT> &lp, int ctas)
{
    using Gm = PipeGeom<S, PT>;
    const size_t smem = Gm::smem_bytes(D);
    static std::atomic<unsigned long long> done{0};
    const cudaError_t e = pipe_configure(fused_pipe_lp_kernel<S, PT, AT, D, T, M>, smem, c->dev, done);
    if (e != cudaSuccess) return e;
    /* no more CTAs per SM in the grid than can be resident */
    static std::atomic<int> occ{0};
    const int fit = pipe_occupancy(fused_pipe_lp_kernel<S, PT, AT, D, T, M>, smem, occ);
    if (fit > 0 && ctas > fit) ctas = fit;
    int grid;
    const PipeSched sch = pipe_sched(c, ctas, 8, &grid);
    /* plain launch: programmatic dependent launch measured 3-10 % slower for
     * these forms (the kernel's griddepcontrol instructions are no-ops then) */
    fused_pipe_lp_kernel<S, PT, AT, D, T, M><<<grid, PIPE_THREADS, smem, c->stream>>>(s, lp, sch, c->errflag);
    return cudaGetLastError();
}

template <typename S, typename PT, typename AT, int D>
cudaError_t pipe_lp_dispatch(bgk_ctx *c, const LpPtrs<S, PT> &s, const ConstsLP<AT> &lp, bool mom, int ctas)
{
    if (c->opt.tanh_mode == BGK_TANH_PORTABLE)
        return mom ? pipe_lp_launch<S, PT, AT, D, BGK_TANH_PORTABLE, true>(c, s, lp, ctas)
                   : pipe_lp_launch<S, PT, AT, D, BGK_TANH_PORTABLE, false>(c, s, lp, ctas);
    return mom ? pipe_lp_launch<S, PT, AT, D, BGK_TANH_DEVICE, true>(c, s, lp, ctas)
               : pipe_lp_launch<S, PT, AT, D, BGK_TANH_DEVICE, false>(c, s, lp, ctas);
}

/* Initial condition in deviation storage (STEP_7/initialization.f90 with
 * the no-slip walls: u = v = u0 inside, 0 on rows 0 and Ny+1). */
template <typename S, typename PT>
__global__ void init_lowp_kernel(Consts c, S *fd, S *gd, PT *ph0, PT *ph1, long long plane, int P,
                                 float sf, float sg)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= c.Nx || y >= c.Ny) return;
    const int i = x + 1, j = y + 1;
    const double T = init_T(c, i, j);
    const double rho = init_rho(c, i, j);
    double Pq[9];
    eq_poly(c.u0, c.v0, Pq);
    const long long cc = (long long)y * P + x;
    for (int k = 0; k < 9; k++) {
        Codec<S>::st(fd + k * plane + cc, (float)(c.w[k] * rho * Pq[k] - c.w[k] * c.rho0), sf);
        Codec<S>::st(gd + k * plane + cc, (float)(c.w[k] * T * Pq[k] - c.w[k] * c.T0), sg);
    }
    const PT phi = PhiCodec<PT>::from_d(init_phi(c, i));
    ph0[cc] = phi;
    ph1[cc] = phi;
}

/* reference-layout field <-> one compact deviation plane */
template <typename S>
__global__ void lp_ref_to_plane(Consts c, const double *ref, S *dst, int P, double base, float scale)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= c.Nx || y >= c.Ny) return;
    const double v = ref[(size_t)(x + 1) + (size_t)(c.Nx + 2) * (size_t)(y + 1)];
    Codec<S>::st(dst + (long long)y * P + x, (float)(v - base), scale);
}

template <typename S>
__global__ void lp_plane_to_ref(Consts c, const S *src, int P, double *ref, double base, float inv_scale,
                                const double *halo_src, int ci, int cj, const double *corner)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i > c.Nx + 1 || j > c.Ny + 1) return;
    const size_t q = (size_t)i + (size_t)(c.Nx + 2) * (size_t)j;
    if (i >= 1 && i <= c.Nx && j >= 1 && j <= c.Ny)
        ref[q] = base + (double)Codec<S>::ld(src + (long long)(j - 1) * P + (i - 1), inv_scale);
    else if (halo_src)
        ref[q] = halo_src[q];
    else
        ref[q] = (corner && i == ci && j == cj) ? corner[0] : 0.0;
}

/* reference-layout phi <-> a stored phi plane (any phi codec) */
template <typename PT>
__global__ void phi_ref_to_plane(Consts c, const double *ref, PT *dst, int P)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= c.Nx || y >= c.Ny) return;
    dst[(long long)y * P + x] = PhiCodec<PT>::from_d(ref[(size_t)(x + 1) + (size_t)(c.Nx + 2) * (size_t)(y + 1)]);
}

template <typename PT>
__global__ void phi_plane_to_ref(Consts c, const PT *src, int P, double *ref, const double *halo_src)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i > c.Nx + 1 || j > c.Ny + 1) return;
    const size_t q = (size_t)i + (size_t)(c.Nx + 2) * (size_t)j;
    if (i >= 1 && i <= c.Nx && j >= 1 && j <= c.Ny)
        ref[q] = PhiCodec<PT>::dec(src[(long long)(j - 1) * P + (i - 1)]);
    else
        ref[q] = halo_src[q];
}

__global__ void lp_tcol_kernel(Consts c, const double *ref, double *tcol)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x + 1;
    if (j <= c.Ny) tcol[j - 1] = ref[(size_t)c.Nx + (size_t)(c.Nx + 2) * (size_t)j];
}

template <typename AT>
ConstsLP<AT> make_lp(const bgk_ctx *b)
{
    const Consts &c = b->c;
    ConstsLP<AT> l{};
    l.Nx = c.Nx;
    l.Ny = c.Ny;
    for (int k = 0; k < 9; k++) {
        l.w[k] = (AT)c.w[k];
        l.w_d[k] = c.w[k];
        l.cf[k] = (AT)((1.0 - c.omega_f) * c.C[k]);
        l.cg[k] = (AT)((1.0 - c.omega_g) * c.C[k]);
    }
    l.m = (AT)c.m_cs2;
    l.q = (AT)c.q_cs2;
    l.rho0 = (AT)c.rho0;
    l.T0 = (AT)c.T0;
    l.T0mTcrit = (AT)(c.T0 - c.T_crit - c.T_act);
    l.inv_T_width = (AT)(1.0 / c.T_width);
    l.f_plus = (AT)c.f_plus;
    l.f_minus = (AT)c.f_minus;
    l.gb = (AT)(c.grav * c.beta);
    l.omega_f = (AT)c.omega_f;
    l.inv_omega_f = (AT)(1.0 / c.omega_f);
    {
        double ws = 0.0;   /* exact: nine floats of similar size sum without rounding in double */
        for (int k = 0; k < 9; k++) ws += (double)l.w[k];
        l.wcorr = (AT)(1.0 - ws);
        /* 2 w1 + 4 w5 and three times it are exact in double */
        const double m = 3.0 * (2.0 * (double)l.w[1] + 4.0 * (double)l.w[5]) - 1.0;
        l.mcorr = (AT)(0.5 * m);
    }
    l.dts = c.dts;
    l.T0mTcrit_d = c.T0 - c.T_crit - c.T_act;
    l.inv_T_width_d = 1.0 / c.T_width;
    l.T0d = c.T0;
    l.rho0d = c.rho0;
    return l;
}

template <typename S, typename PT, typename AT>
cudaError_t launch_lowp_t(bgk_ctx *c, bool moments)
{
    LpPtrs<S, PT> s{};
    const int src = c->cur, dst = c->cur ^ 1;
    s.fin = (const S *)c->fbuf[src]; s.gin = (const S *)c->gbuf[src];
    s.fout = (S *)c->fbuf[dst]; s.gout = (S *)c->gbuf[dst];
    s.phin = (const PT *)c->phibuf[src]; s.phout = (PT *)c->phibuf[dst];
    s.tcin = c->tcol[src]; s.tcout = c->tcol[dst];
    s.gW = c->gW; s.pE = c->pE; s.phiW = c->phiW; s.phiE = c->phiE; s.corner = c->corner;
    s.mrho = c->mrho; s.mT = c->mT; s.mu = c->mu; s.mv = c->mv; s.mphi = c->mphi;
    s.plane = c->plane; s.P = c->P; s.NX2 = c->NX2;
    s.sf = c->scale.sf; s.sg = c->scale.sg; s.inv_sf = c->scale.inv_sf; s.inv_sg = c->scale.inv_sg;
    const ConstsLP<AT> lp = make_lp<AT>(c);
    const int H = strip_height(c);
    dim3 grd((c->Nx + FUSED_BX - 1) / FUSED_BX, (c->Ny + H - 1) / H);
    if (c->tune_pipe) {
        /* stages of ~10 KB (FP32) / ~5 KB (FP16).  Measured on B200 (FP32,
         * 3/4 stages x 4/5 CTAs per SM x H = 4/8/16 at 1024^2, 2048^2,
         * 3072^2, 4096^2 and 16384x4096): 4 stages; 5 CTAs per SM up to
         * 2^22 nodes (+7 % at 1024^2, +13 % at 2048^2: 35.4 against 31.3
         * GLUPS), 4 above (5 loses 3-16 % there). */
        const int D = c->tune_D > 0 ? c->tune_D : 4;
        const int ctas = c->tune_ctas > 0 ? c->tune_ctas : ((long long)c->Nx * c->Ny <= (1LL << 22) ? 5 : 4);
        if (D <= 3) return pipe_lp_dispatch<S, PT, AT, 3>(c, s, lp, moments, ctas);
        if (D >= 6) return pipe_lp_dispatch<S, PT, AT, 6>(c, s, lp, moments, ctas);
        return pipe_lp_dispatch<S, PT, AT, 4>(c, s, lp, moments, ctas);
    }
#define BGK_LP(T, M) fused_lowp_kernel<S, PT, AT, T, M><<<grd, FUSED_BX, 0, c->stream>>>(s, lp, H, c->tune_pf)
    if (c->opt.tanh_mode == BGK_TANH_PORTABLE) {
        if (moments) BGK_LP(BGK_TANH_PORTABLE, true); else BGK_LP(BGK_TANH_PORTABLE, false);
    } else {
        if (moments) BGK_LP(BGK_TANH_DEVICE, true); else BGK_LP(BGK_TANH_DEVICE, false);
    }
#undef BGK_LP
    return cudaGetLastError();
}

/* nsteps steps of a reduced-precision form in one dataflow launch (no
 * moments written); the state advances from buffer cur to cur ^ (nsteps & 1). */
template <typename S, typename PT, typename AT>
cudaError_t launch_flow_t(bgk_ctx *c, int nsteps)
{
    constexpr int D = 4;
    LpPtrs<S, PT> s0{};
    const int a = c->cur, b = c->cur ^ 1;
    s0.gW = c->gW; s0.pE = c->pE; s0.phiW = c->phiW; s0.phiE = c->phiE; s0.corner = c->corner;
    s0.plane = c->plane; s0.P = c->P; s0.NX2 = c->NX2;
    s0.sf = c->scale.sf; s0.sg = c->scale.sg; s0.inv_sf = c->scale.inv_sf; s0.inv_sg = c->scale.inv_sg;
    LpPtrs<S, PT> s1 = s0;
    s0.fin = (const S *)c->fbuf[a]; s0.gin = (const S *)c->gbuf[a]; s0.fout = (S *)c->fbuf[b]; s0.gout = (S *)c->gbuf[b];
    s0.phin = (const PT *)c->phibuf[a]; s0.phout = (PT *)c->phibuf[b]; s0.tcin = c->tcol[a]; s0.tcout = c->tcol[b];
    s1.fin = (const S *)c->fbuf[b]; s1.gin = (const S *)c->gbuf[b]; s1.fout = (S *)c->fbuf[a]; s1.gout = (S *)c->gbuf[a];
    s1.phin = (const PT *)c->phibuf[b]; s1.phout = (PT *)c->phibuf[a]; s1.tcin = c->tcol[b]; s1.tcout = c->tcol[a];
    const ConstsLP<AT> lp = make_lp<AT>(c);
    int grid;
    const PipeSched sch = pipe_sched(c, c->tune_ctas > 0 ? c->tune_ctas : 4, 8, &grid);
    const size_t need = sizeof(unsigned long long) + (size_t)sch.ntiles * sizeof(unsigned);
    if (c->flow_bytes < need) {
        if (c->flow_buf) cudaFree(c->flow_buf);
        c->flow_buf = nullptr;
        c->flow_bytes = 0;
        cudaError_t e = cudaMalloc(&c->flow_buf, need);
        if (e != cudaSuccess) return e;
        c->flow_bytes = need;
    }
    cudaError_t e = cudaMemsetAsync(c->flow_buf, 0, need, c->stream);
    if (e != cudaSuccess) return e;
    FlowCtl fl;
    fl.ticket = (unsigned long long *)c->flow_buf;
    fl.done = (unsigned *)((char *)c->flow_buf + sizeof(unsigned long long));
    fl.nsteps = nsteps;
    fl.stall = c->flow_stall ? (1u << 30) : 0u;
    using Gm = PipeGeom<S, PT>;
    const size_t smem = Gm::smem_bytes_w(D);
    if (c->opt.tanh_mode == BGK_TANH_PORTABLE) {
        static std::atomic<unsigned long long> done{0};
        if ((e = pipe_configure(flow_pipe_lp_kernel<S, PT, AT, D, BGK_TANH_PORTABLE>, smem, c->dev, done))) return e;
        flow_pipe_lp_kernel<S, PT, AT, D, BGK_TANH_PORTABLE><<<grid, PIPE_THREADS, smem, c->stream>>>(s0, s1, lp, sch,
                                                                                                     fl, c->errflag);
    } else {
        static std::atomic<unsigned long long> done{0};
        if ((e = pipe_configure(flow_pipe_lp_kernel<S, PT, AT, D, BGK_TANH_DEVICE>, smem, c->dev, done))) return e;
        flow_pipe_lp_kernel<S, PT, AT, D, BGK_TANH_DEVICE><<<grid, PIPE_THREADS, smem, c->stream>>>(s0, s1, lp, sch,
                                                                                                   fl, c->errflag);
    }
    return cudaGetLastError();
}

} // namespace

cudaError_t launch_flow_lowp(bgk_ctx *c, int nsteps)
{
    const bool p64 = c->phisz == 8;
    if (c->opt.precision == BGK_PREC_F32X) return launch_flow_t<float, double, double>(c, nsteps);
    if (c->opt.precision == BGK_PREC_F32)
        return p64 ? launch_flow_t<float, double, float>(c, nsteps) : launch_flow_t<float, float, float>(c, nsteps);
    return p64 ? launch_flow_t<__half, double, float>(c, nsteps) : launch_flow_t<__half, float, float>(c, nsteps);
}

cudaError_t launch_fused_lowp(bgk_ctx *c, bool moments)

{
    const bool p64 = c->phisz == 8;
    if (c->opt.precision == BGK_PREC_F32X) return launch_lowp_t<float, double, double>(c, moments);
    if (c->opt.precision == BGK_PREC_F32)
        return p64 ? launch_lowp_t<float, double, float>(c, moments) : launch_lowp_t<float, float, float>(c, moments);
    return p64 ? launch_lowp_t<__half, double, float>(c, moments) : launch_lowp_t<__half, float, float>(c, moments);
}

/* FP16 scales: powers of two that put the largest deviations expected in
 * the benchmark cavities (|fd| < ~0.1, |gd| < ~50) near 2^6 .. 2^10, far from
 * both the FP16 overflow (65504) and its subnormal range (< 6.1e-5). */
static void set_scales(bgk_ctx *c)
{
    if (c->opt.precision == BGK_PREC_F16) {
        c->scale.sf = 1024.0f;
        c->scale.sg = 16.0f;
    } else {
        c->scale.sf = 1.0f;
        c->scale.sg = 1.0f;
    }
    c->scale.inv_sf = 1.0f / c->scale.sf;
    c->scale.inv_sg = 1.0f / c->scale.sg;
}

cudaError_t launch_init_lowp(bgk_ctx *c)
{
    set_scales(c);
    /* mirrors, corners and the T column come from the FP64 initial condition */
    void *fb = c->fbuf[c->cur], *gb = c->gbuf[c->cur];
    c->fbuf[c->cur] = nullptr;
    c->gbuf[c->cur] = nullptr;
    const int mode = c->mode;
    c->mode = 2;   /* neither compact FP64 nor staged: mirrors only */
    cudaError_t e = launch_init_f64(c);
    c->mode = mode;
    c->fbuf[c->cur] = fb;
    c->gbuf[c->cur] = gb;
    if (e != cudaSuccess) return e;
    dim3 blk(32, 8), grd((c->Nx + 31) / 32, (c->Ny + 7) / 8);
    const bool p64 = c->phisz == 8;
#define BGK_INIT(S, PT, sf_, sg_)                                                                        \
    init_lowp_kernel<S, PT><<<grd, blk, 0, c->stream>>>(c->c, (S *)fb, (S *)gb, (PT *)c->phibuf[0],     \
                                                        (PT *)c->phibuf[1], c->plane, c->P, sf_, sg_)
    if (c->opt.precision != BGK_PREC_F16) {
        if (p64) BGK_INIT(float, double, 1.f, 1.f); else BGK_INIT(float, float, 1.f, 1.f);
    } else {
        if (p64) BGK_INIT(__half, double, c->scale.sf, c->scale.sg);
        else BGK_INIT(__half, float, c->scale.sf, c->scale.sg);
    }
#undef BGK_INIT
    return cudaGetLastError();
}

template <typename S>
static int lp_to_compact(bgk_ctx *c, int field, const double *ref)
{
    dim3 blk(32, 8), grd((c->Nx + 31) / 32, (c->Ny + 7) / 8);
    if (field >= BGK_FIELD_F0 && field < BGK_FIELD_F0 + 9) {
        const int k = field - BGK_FIELD_F0;
        lp_ref_to_plane<S><<<grd, blk, 0, c->stream>>>(c->c, ref, (S *)c->fbuf[c->cur] + k * c->plane, c->P,
                                                       c->c.w[k] * c->c.rho0, c->scale.sf);
        if (k == 6 || k == 7) {
            const size_t q = (k == 6) ? (size_t)(c->Nx + 1) : (size_t)(c->Nx + 1) + (size_t)c->NX2 * (size_t)(c->Ny + 1);
            if (cudaMemcpyAsync(c->corner + (k - 6), ref + q, sizeof(double), cudaMemcpyDeviceToDevice, c->stream))
                return BGK_ERR_CUDA;
        }
    } else if (field >= BGK_FIELD_G0 && field < BGK_FIELD_G0 + 9) {
        const int k = field - BGK_FIELD_G0;
        lp_ref_to_plane<S><<<grd, blk, 0, c->stream>>>(c->c, ref, (S *)c->gbuf[c->cur] + k * c->plane, c->P,
                                                       c->c.w[k] * c->c.T0, c->scale.sg);
    } else if (field == BGK_FIELD_PHI) {
        for (int b = 0; b < 2; b++) {
            if (c->phisz == 8)
                phi_ref_to_plane<double><<<grd, blk, 0, c->stream>>>(c->c, ref, (double *)c->phibuf[b], c->P);
            else
                phi_ref_to_plane<float><<<grd, blk, 0, c->stream>>>(c->c, ref, (float *)c->phibuf[b], c->P);
        }
    } else if (field == BGK_FIELD_T) {
        lp_tcol_kernel<<<(c->Ny + 127) / 128, 128, 0, c->stream>>>(c->c, ref, c->tcol[c->cur]);
    } else if (field != BGK_FIELD_RHO && field != BGK_FIELD_U && field != BGK_FIELD_V) {
        return BGK_ERR_UNSUPPORTED;
    }
    return cudaGetLastError() == cudaSuccess ? BGK_OK : BGK_ERR_CUDA;
}

template <typename S>
static int lp_to_ref(bgk_ctx *c, int field, double *ref, int prev)
{
    dim3 blk(32, 8), grd((c->NX2 + 31) / 32, (c->NY2 + 7) / 8);
    const int b = prev ? (c->cur ^ 1) : c->cur;
    if (field >= BGK_FIELD_F0 && field < BGK_FIELD_F0 + 9) {
        const int k = field - BGK_FIELD_F0;
        const double *cn = (k == 6) ? c->corner : (k == 7 ? c->corner + 1 : nullptr);
        lp_plane_to_ref<S><<<grd, blk, 0, c->stream>>>(c->c, (const S *)c->fbuf[b] + k * c->plane, c->P, ref,
                                                       c->c.w[k] * c->c.rho0, c->scale.inv_sf, nullptr, c->Nx + 1,
                                                       k == 6 ? 0 : c->Ny + 1, cn);
    } else if (field >= BGK_FIELD_G0 && field < BGK_FIELD_G0 + 9) {
        const int k = field - BGK_FIELD_G0;
        lp_plane_to_ref<S><<<grd, blk, 0, c->stream>>>(c->c, (const S *)c->gbuf[b] + k * c->plane, c->P, ref,
                                                       c->c.w[k] * c->c.T0, c->scale.inv_sg, nullptr, -1, -1, nullptr);
    } else if (field == BGK_FIELD_PHI_PREC) {
        if (c->phisz == 8)
            phi_plane_to_ref<double><<<grd, blk, 0, c->stream>>>(c->c, (const double *)c->phibuf[b], c->P, ref, c->mphi);
        else
            phi_plane_to_ref<float><<<grd, blk, 0, c->stream>>>(c->c, (const float *)c->phibuf[b], c->P, ref, c->mphi);
    } else {
        return BGK_ERR_UNSUPPORTED;
    }
    return cudaGetLastError() == cudaSuccess ? BGK_OK : BGK_ERR_CUDA;
}

} // namespace bgk

int lowp_ref_to_compact(bgk_ctx *c, int field, const double *ref)
{
    return c->opt.precision != BGK_PREC_F16 ? bgk::lp_to_compact<float>(c, field, ref)
                                            : bgk::lp_to_compact<__half>(c, field, ref);
}

int lowp_compact_to_ref(bgk_ctx *c, int field, double *ref, int prev)
{
    return c->opt.precision != BGK_PREC_F16 ? bgk::lp_to_ref<float>(c, field, ref, prev)
                                            : bgk::lp_to_ref<__half>(c, field, ref, prev);
}
