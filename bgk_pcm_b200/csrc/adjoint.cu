/*
 * adjoint.cu -- the differentiation form: a hand-written reverse of the fused
 * FP64 step (smooth form, see bgk_options.smooth) run backward in time with
 * checkpoint-and-recompute.
 *
 * One reverse step (forward step n: S(n-1) -> S(n)) is one kernel, fused in
 * gather form.  At node i it
 *  1. gathers the adjoint of the state S(n) at i -- lambda_f[k], lambda_g[k],
 *     lambda_phi and (east column) lambda of T(Nx, y) -- from the local
 *     partials Pi(n+1) that the reverse of step n+1 left at the nodes that
 *     read those values: the node that pulled the population (i + c_k), the
 *     node itself when the pull was a bounce-back, the rows that read a
 *     clamped (copied) halo row of g or phi, and the 3x3 stencils that read
 *     phi(i);
 *  2. recomputes the forward node update of step n from S(n-1);
 *  3. applies the vector-Jacobian product of that update and stores the
 *     partials Pi(n)(i): the adjoints of the 18 pulled populations, of the
 *     two 3x3 selector sums (k+, k-) and of phi_prec(i).
 * Each step therefore reads S(n-1) and Pi(n+1) once and writes Pi(n) once.
 * Parameter gradients: d/d omega_g per block (deterministic partial sums),
 * d/dTin per row from the west nodes' pulled-g partials.
 *
 * Forward states come from snapshots every K steps; each K-step segment is
 * recomputed with the fused kernel before it is reversed, except the last
 * one, whose states the forward pass writes into the segment buffer.
 */
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <vector>

#include "bgk_internal.h"
#include "bgk_math.cuh"
#include "../../include/bgk_portable_tanh.h"

namespace {

using bgk::Consts;

#include "pipe_common.cuh"

constexpr int NPI = 21;          /* partial planes: f[9], g[9], k+, k-, phi_prec */
constexpr int AB_X = 64, AB_Y = 4;

__constant__ int d_cx[9] = {0, 1, 0, -1, 0, 1, -1, -1, 1};
__constant__ int d_cy[9] = {0, 0, 1, 0, -1, 1, 1, -1, -1};
__constant__ int d_opp[9] = {0, 3, 4, 1, 2, 7, 8, 5, 6};
/* A_k, B_k, E_k of S_k = A_k Pxx + B_k Pyy + 2 E_k Pxy (collision.f90:84-100);
 * the same coefficients weight d_k in Pxx, Pyy, Pxy. */
__constant__ int d_AisQ[9] = {0, 1, 0, 1, 0, 1, 1, 1, 1};
__constant__ int d_BisQ[9] = {0, 0, 1, 0, 1, 1, 1, 1, 1};
__constant__ double d_E[9] = {0, 0, 0, 0, 0, 1, -1, 1, -1};

struct AdjPtrs {
    const double *f, *g, *phi, *tcol;      /* state S(n-1), compact          */
    const double *pin;                     /* Pi(n+1): NPI planes            */
    double *pout;                          /* Pi(n)                          */
    const double *gW, *pE, *phiW, *phiE, *corner;
    double *omg_acc;                       /* per-block running sums         */
    const double *dgW;                     /* d gW_k / d Tin per row         */
    double inv_T_width;                    /* 1 / T_width                    */
    double inv_omega_f;                    /* 1 / omega_f = tau_f            */
    double *gtin;                          /* dL/dTin per row                */
    long long plane;
    int P;
    int tanh_mode;
};

__device__ __forceinline__ double tanh_sel(double x, int mode)
{
    return mode == BGK_TANH_PORTABLE ? bgk_portable_tanh(x) : tanh(x);
}

__host__ __device__ constexpr int cx_of(int k) { return (k == 1 || k == 5 || k == 8) ? 1 : ((k == 3 || k == 6 || k == 7) ? -1 : 0); }
__host__ __device__ constexpr int cy_of(int k) { return (k == 2 || k == 5 || k == 6) ? 1 : ((k == 4 || k == 7 || k == 8) ? -1 : 0); }

/* The equilibrium polynomial P_k(u, v) = 1 + 3 c_k.u + 4.5 (c_k.u)^2 -
 * 1.5 |u|^2 (same value as eq_poly up to rounding) and its gradient. */
__device__ __forceinline__ double poly_k(int k, double u, double v, double &du, double &dv)
{
    const double cx = cx_of(k), cy = cy_of(k);
    const double cu = cx * u + cy * v;
    du = 3.0 * cx + 9.0 * cu * cx - 3.0 * u;
    dv = 3.0 * cy + 9.0 * cu * cy - 3.0 * v;
    return 1.0 + 3.0 * cu + 4.5 * cu * cu - 1.5 * (u * u + v * v);
}


/* Vector-Jacobian product of one node update (smooth form).
 * in : pulled f, g; selector sums kp, km; phi_prec p0; output adjoints
 *      Fo_b (f post-collision), Go_b (g post-collision), Tm_b (moments T
 *      written for the east boundary) and the adjoint of the new phi in
 *      gathered form: phi_b = d0 + aplus'(phn) * skp + aminus'(phn) * skm,
 *      where the selector-term derivatives are taken at the new value phn
 *      (the value the next step's stencils read).
 * out: f_b, g_b (pulled), kp_b, km_b, p0_b, omg_b (d/d omega_g). */
template <class FOB, class GOB, class OUTF, class OUTG>
__device__ __forceinline__ void node_vjp(const Consts &c, int tanh_mode, const double *f, const double *g, double kp, double km,
                         double p0, FOB Fo_b, GOB Go_b, double d0, double skp, double skm,
                         double Tm_b, OUTF out_fb, OUTG out_gb, double &kp_b, double &km_b, double &p0_b,
                         double &omg_b, double inv_Tw, double inv_of)
{
    const double m = c.m_cs2, q = c.q_cs2;
    /* ---- forward recompute ---- */
    double rho = 0.0, T = 0.0;
#pragma unroll
    for (int k = 0; k < 9; k++) { rho += f[k]; T += g[k]; }
    const double irho = 1.0 / rho;
    const double mx = f[1] - f[3] + f[5] - f[6] - f[7] + f[8];
    const double my = f[2] - f[4] + f[5] + f[6] - f[7] - f[8];
    const double u = irho * mx, v = irho * my;
    const double arg = ((T - c.T_crit) - c.T_act) * inv_Tw;
    const double th = tanh_sel(arg, tanh_mode);
    const double rp = 0.5 * (1.0 + th), rm = 0.5 * (1.0 - th);
    const double KP = (kp / 8.0) * rp, KM = (km / 8.0) * rm;
    const double phn = p0 + (c.f_plus * KP * (1.0 - p0) - c.f_minus * KM * (1.0 + p0));
    const double phn_b = d0 + 0.5 * (1.0 + phn) * skp - 0.5 * (1.0 - phn) * skm;
    const double Tf = T - c.dts * (phn - p0) / 2.0;
    const double gb = c.grav * c.beta;
    const double onep = 1.0 + phn / 2.0;
    const double FY0 = rho * gb * Tf * onep;
    const double omp = 1.0 - phn;
    const double FX = -(u * omp * 0.5);
    const double FY = FY0 - v * omp * 0.5;
    const double iorho = irho * inv_of;   /* 1 / (omega_f rho) */
    const double uf = u + FX * iorho, vf = v + FY * iorho;
    /* non-equilibrium moments of g; the polynomials P_k(uf, vf) and their
     * gradients are formed per k where they are used (fewer live registers) */
    double txx = 0.0, tyy = 0.0, txy = 0.0;
#pragma unroll
    for (int k = 0; k < 9; k++) {
        double du, dv;
        const double e = g[k] - c.w[k] * Tf * poly_k(k, uf, vf, du, dv);
        txx += (d_AisQ[k] ? q : m) * e;
        tyy += (d_BisQ[k] ? q : m) * e;
        txy += d_E[k] * e;
    }

    /* ---- reverse ---- */
    const double hT = 0.5 * Tm_b;      /* moments T = (sum g + T2) / 2 */
    /* g collision: go_k = geq_k + (1-omega_g) C_k Sg_k; f likewise */
    const double cg = 1.0 - c.omega_g, cf = 1.0 - c.omega_f;
    double txxb = 0.0, tyyb = 0.0, txyb = 0.0, pxxb = 0.0, pyyb = 0.0, pxyb = 0.0;
    omg_b = 0.0;
#pragma unroll
    for (int k = 0; k < 9; k++) {
        const double A = d_AisQ[k] ? q : m, B = d_BisQ[k] ? q : m;
        const double Gob = Go_b(k) + hT;
        const double Sg = A * txx + B * tyy + 2.0 * d_E[k] * txy;
        omg_b += Gob * (-c.C[k] * Sg);
        const double sb = Gob * cg * c.C[k];
        txxb += sb * A; tyyb += sb * B; txyb += 2.0 * sb * d_E[k];
        const double sf = Fo_b(k) * cf * c.C[k];
        pxxb += sf * A; pyyb += sf * B; pxyb += 2.0 * sf * d_E[k];
    }
    double rhob = 0.0, Tfb = 0.0, ufb = 0.0, vfb = 0.0;
#pragma unroll
    for (int j = 0; j < 9; j++) {
        const double A = d_AisQ[j] ? q : m, B = d_BisQ[j] ? q : m;
        const double eb = A * txxb + B * tyyb + d_E[j] * txyb;
        const double db = A * pxxb + B * pyyb + d_E[j] * pxyb;
        const double geqb = (Go_b(j) + hT) - eb;
        const double feqb = Fo_b(j) - db;
        double du, dv;
        const double Pj = poly_k(j, uf, vf, du, dv);
        rhob += feqb * c.w[j] * Pj;
        Tfb += geqb * c.w[j] * Pj;
        const double Pb = c.w[j] * (feqb * rho + geqb * Tf);
        ufb += Pb * du;
        vfb += Pb * dv;
    }
    /* velocity shift */
    double ub = ufb, vb = vfb;
    const double FXb = ufb * iorho, FYb = vfb * iorho;
    const double orhob = -(ufb * FX + vfb * FY) * (iorho * iorho);
    rhob += c.omega_f * orhob;
    /* drag and buoyancy */
    const double FY0b = FYb;
    vb += -0.5 * omp * FYb;
    double phnb = 0.5 * v * FYb;
    ub += -0.5 * omp * FXb;
    phnb += 0.5 * u * FXb;
    rhob += FY0b * gb * Tf * onep;
    Tfb += FY0b * rho * gb * onep;
    phnb += FY0b * rho * gb * Tf * 0.5;
    /* latent heat */
    double Tb = Tfb;
    phnb += -0.5 * c.dts * Tfb;
    p0_b = 0.5 * c.dts * Tfb;
    /* phase field */
    const double PHb = phn_b + phnb;
    p0_b += PHb * (1.0 - c.f_plus * KP - c.f_minus * KM);
    const double KPb = PHb * c.f_plus * (1.0 - p0);
    const double KMb = -PHb * c.f_minus * (1.0 + p0);
    kp_b = KPb * rp / 8.0;
    km_b = KMb * rm / 8.0;
    const double rpb = KPb * kp / 8.0, rmb = KMb * km / 8.0;
    const double thb = 0.5 * rpb - 0.5 * rmb;
    Tb += thb * (1.0 - th * th) * inv_Tw;
    Tb += hT;
    /* momentsPre */
    const double mxb = ub * irho, myb = vb * irho;
    const double irhob = ub * mx + vb * my;
    rhob += -irhob * irho * irho;
    /* pulled-population adjoints: the collision term (recomputed from the
     * six moment adjoints) plus the moment terms */
#pragma unroll
    for (int j = 0; j < 9; j++) {
        const double A = d_AisQ[j] ? q : m, B = d_BisQ[j] ? q : m;
        const double eb = A * txxb + B * tyyb + d_E[j] * txyb;
        const double db = A * pxxb + B * pyyb + d_E[j] * pxyb;
        out_fb(j, db + (rhob + cx_of(j) * mxb + cy_of(j) * myb));
        out_gb(j, eb + Tb);
    }
}

__device__ __forceinline__ double PI(const AdjPtrs &s, int k, int x, int y)
{
    return s.pin[k * s.plane + (long long)y * s.P + x];
}

/* dL/dTin contributions of one step's pulled-g partials at row y (west
 * column): pop 1 reads the west value of its own row, pop 5 that of row y-1
 * (clamped), pop 8 that of row y+1 (clamped). */
__device__ __forceinline__ double tin_partial(const double *pi, long long plane, int P, int Ny, const double *dgW,
                                              int y)
{
    auto at = [&](int k, int yy) { return pi[(9 + k) * plane + (long long)yy * P]; };
    double a = at(1, y) * dgW[y];
    double b5 = 0.0, b8 = 0.0;
    if (y + 1 < Ny) b5 += at(5, y + 1);
    if (y == 0) b5 += at(5, 0);
    if (y - 1 >= 0) b8 += at(8, y - 1);
    if (y == Ny - 1) b8 += at(8, Ny - 1);
    return a + b5 * dgW[Ny + y] + b8 * dgW[2 * Ny + y];
}

/* 2 blocks (16 warps) per SM: 128 registers, a few spilled words. */
__global__ void __launch_bounds__(AB_X *AB_Y, 2)
adj_step_kernel(AdjPtrs s, Consts c)
{
    const int Nx = c.Nx, Ny = c.Ny;
    const int x = blockIdx.x * AB_X + threadIdx.x;
    const int y = blockIdx.y * AB_Y + threadIdx.y;
    const bool active = x < Nx && y < Ny;
    double omg_b = 0.0;
    if (active) {
        const long long pl = s.plane;
        const int P = s.P;
        const long long cc = (long long)y * P + x;
        const bool W = x == 0, E = x == Nx - 1, S = y == 0, N = y == Ny - 1;

        /* 1. gather the adjoint of S(n) at this node */
        double lf[9], lg[9];
#pragma unroll
        for (int k = 0; k < 9; k++) {
            const int xd = x + d_cx[k], yd = y + d_cy[k];
            if (xd >= 0 && xd < Nx && yd >= 0 && yd < Ny) {
                lf[k] = PI(s, k, xd, yd);
            } else {
                /* read by this node's own bounce-back of opp(k), except the
                 * two frozen corners (pop 6 at (Nx,1), pop 7 at (Nx,Ny)) */
                const bool corner6 = (k == 8) && E && S;
                const bool corner7 = (k == 5) && E && N;
                lf[k] = (corner6 || corner7) ? 0.0 : PI(s, d_opp[k], x, y);
            }
            double a = 0.0;
            if (xd >= 0 && xd < Nx) {
                if (yd >= 0 && yd < Ny) a += PI(s, 9 + k, xd, yd);
                if (d_cy[k] == 1 && y == 0) a += PI(s, 9 + k, xd, 0);
                if (d_cy[k] == -1 && y == Ny - 1) a += PI(s, 9 + k, xd, Ny - 1);
            }
            lg[k] = a;
        }
        /* phi: own direct partial + the 3x3 stencils that read this cell */
        double skp = 0.0, skm = 0.0;
        for (int dy = -1; dy <= 1; dy++) {
            for (int dx = -1; dx <= 1; dx++) {
                const int xd = x - dx;
                if (xd < 0 || xd >= Nx) continue;
                const int yd = y - dy;
                if (yd >= 0 && yd < Ny) { skp += PI(s, 18, xd, yd); skm += PI(s, 19, xd, yd); }
                if (dy == -1 && y == 0) { skp += PI(s, 18, xd, 0); skm += PI(s, 19, xd, 0); }
                if (dy == 1 && y == Ny - 1) { skp += PI(s, 18, xd, Ny - 1); skm += PI(s, 19, xd, Ny - 1); }
            }
        }
        /* dL/dTin from Pi(n+1) (the partials of the later step), one
         * thread per row, so the per-row sums keep a fixed order */
        if (W) s.gtin[y] += tin_partial(s.pin, pl, P, Ny, s.dgW, y);
        const double ph = s.phi[cc];        /* phi_prec of step n */
        const double d0 = PI(s, 20, x, y);
        /* T(Nx, y) written by this (east) node: read by the east pulls of
         * pops 3 (same row), 6 (row y+1, or row 0 itself) and 7 (row y-1, or
         * row Ny-1 itself) of the next step */
        double lT = 0.0;
        if (E) {
            lT += PI(s, 9 + 3, x, y) * c.w[3] * s.pE[y];
            double a6 = 0.0, a7 = 0.0;
            if (y + 1 < Ny) a6 += PI(s, 9 + 6, x, y + 1);
            if (y == 0) a6 += PI(s, 9 + 6, x, 0);
            if (y - 1 >= 0) a7 += PI(s, 9 + 7, x, y - 1);
            if (y == Ny - 1) a7 += PI(s, 9 + 7, x, Ny - 1);
            lT += a6 * c.w[6] * s.pE[Ny + y] + a7 * c.w[7] * s.pE[2 * Ny + y];
        }

        /* 2. pulled inputs of step n from S(n-1) (as fused_f64_kernel) */
        const double *F = s.f, *G = s.g;
        double f[9], g[9];
        f[0] = F[cc];
        f[1] = *(W ? F + 3 * pl + cc : F + 1 * pl + cc - 1);
        f[2] = *(S ? F + 4 * pl + cc : F + 2 * pl + cc - P);
        f[3] = *(E ? F + 1 * pl + cc : F + 3 * pl + cc + 1);
        f[4] = *(N ? F + 2 * pl + cc : F + 4 * pl + cc + P);
        f[5] = *((W || S) ? F + 7 * pl + cc : F + 5 * pl + cc - P - 1);
        f[6] = *((E || S) ? F + 8 * pl + cc : F + 6 * pl + cc - P + 1);
        f[7] = *((E || N) ? F + 5 * pl + cc : F + 7 * pl + cc + P + 1);
        f[8] = *((W || N) ? F + 6 * pl + cc : F + 8 * pl + cc + P - 1);
        if (E && S) f[6] = s.corner[0];
        if (E && N) f[7] = s.corner[1];
        const int ym = S ? y : y - 1, yp = N ? y : y + 1;
        const long long cm = (long long)ym * P + x, cp = (long long)yp * P + x;
        g[0] = G[cc];
        g[1] = *(W ? s.gW + y : G + 1 * pl + cc - 1);
        g[2] = G[2 * pl + cm];
        g[4] = G[4 * pl + cp];
        g[5] = *(W ? s.gW + Ny + ym : G + 5 * pl + cm - 1);
        g[8] = *(W ? s.gW + 2 * Ny + yp : G + 8 * pl + cp - 1);
        if (E) {
            g[3] = c.w[3] * s.tcol[y] * s.pE[y];
            g[6] = c.w[6] * s.tcol[ym] * s.pE[Ny + ym];
            g[7] = c.w[7] * s.tcol[yp] * s.pE[2 * Ny + yp];
        } else {
            g[3] = G[3 * pl + cc + 1];
            g[6] = G[6 * pl + cm + 1];
            g[7] = G[7 * pl + cp + 1];
        }
        double kp = 0.0, km = 0.0;
        for (int dy = -1; dy <= 1; dy++) {
            const int r = min(max(y + dy, 0), Ny - 1);
            for (int dx = -1; dx <= 1; dx++) {
                const int xs = x + dx;
                const double p = xs < 0 ? s.phiW[r] : (xs >= Nx ? s.phiE[r] : s.phi[(long long)r * P + xs]);
                kp += bgk::aplus(p);
                km += bgk::aminus(p);
            }
        }

        /* 3. vector-Jacobian product -> Pi(n) */
        double fb[9], gbv[9], kpb, kmb, p0b;
        node_vjp(c, s.tanh_mode, f, g, kp, km, ph, [&](int k) { return lf[k]; }, [&](int k) { return lg[k]; }, d0,
                 skp, skm, lT, [&](int k, double v) { fb[k] = v; }, [&](int k, double v) { gbv[k] = v; }, kpb, kmb,
                 p0b, omg_b, s.inv_T_width, s.inv_omega_f);
#pragma unroll
        for (int k = 0; k < 9; k++) {
            s.pout[k * pl + cc] = fb[k];
            s.pout[(9 + k) * pl + cc] = gbv[k];
        }
        s.pout[18 * pl + cc] = kpb;
        s.pout[19 * pl + cc] = kmb;
        s.pout[20 * pl + cc] = p0b;
    }
    /* deterministic per-block accumulation of d/d omega_g */
    __shared__ double red[AB_X * AB_Y];
    const int t = threadIdx.y * AB_X + threadIdx.x;
    red[t] = omg_b;
    __syncthreads();
    for (int o = AB_X * AB_Y / 2; o > 0; o >>= 1) {
        if (t < o) red[t] += red[t + o];
        __syncthreads();
    }
    if (t == 0) s.omg_acc[blockIdx.y * gridDim.x + blockIdx.x] += red[0];
}

/* ------------------------------------------------------------------------
 * The reverse step on the shared-memory pipeline (default).  Same
 * arithmetic as adj_step_kernel; the loads are decoupled from the
 * ~200-register node VJP: one producer lane per CTA streams, for each row y
 * of a 128-column tile, 40 row segments into a stage with bulk asynchronous
 * copies (16 bytes of neighbours on each side of the band):
 *    0..8   Pi_k(n+1)        row y + c_ky (clamped)   gather of lambda_f
 *    9..17  Pi_(9+k)(n+1)    row y + c_ky (clamped)   gather of lambda_g
 *   18, 19  Pi_k+, Pi_k-     row y + 1 (clamped)      3x3 gather window
 *   20      Pi_phi_prec      row y
 *   21..29  f_k(n-1)         row y - c_ky (clamped)   pulls
 *   30..38  g_k(n-1)         row y - c_ky (clamped)
 *   39      phi(n-1)         row y + 1 (clamped)      3x3 stencil window
 * Consumers keep the rows y-1 and y of the two 3x3 windows in registers.
 * Values that a boundary node needs outside the staged rows (bounce-back
 * partials, the clamped halo rows, the east T column, the west Tin terms)
 * are read from global memory, as in adj_step_kernel.
 * ---------------------------------------------------------------------- */
constexpr int ADJ_AL = 2;                                 /* 16 bytes of doubles */
constexpr int ADJ_RW = PIPE_BX + 2 * ADJ_AL;
constexpr int ADJ_SEG_BYTES = ADJ_RW * (int)sizeof(double);
constexpr int ADJ_NSEG = 40;
constexpr int ADJ_STAGE_BYTES = ADJ_NSEG * ADJ_SEG_BYTES;
constexpr int ADJ_HEADER = 256;
/* Wall tables: the values a west (x = 0) or east (x = Nx-1) node reads from
 * global memory outside the staged rows, for every row of a tile (at most
 * ADJ_BND_ROWS rows, the largest tile height adj_sched picks).  The warp
 * that holds the wall node fills its table once per tile, one lane per row,
 * so the loads of all rows are in flight together; the node then reads them
 * from shared memory.  Without the tables the wall lane issued ~20 dependent
 * global loads per row and the CTAs of the two wall bands set the kernel's
 * duration.  Value v of row r is at table[v * ADJ_BND_ROWS + r]. */
constexpr int ADJ_BND_ROWS = 64;
constexpr int ADJ_BND_VALS = 10;
enum : int { BW_PHI, BW_BB1, BW_BB8, BW_BB5, BW_GW0, BW_GW1, BW_GW2, BW_F5, BW_F8 };       /* west */
enum : int { BE_PHI, BE_BB3, BE_BB7, BE_BB6, BE_LT, BE_G3, BE_G6, BE_G7, BE_F6, BE_F7 };  /* east */
static_assert(BW_F8 < ADJ_BND_VALS && BE_F7 < ADJ_BND_VALS, "wall table width");
constexpr int ADJ_BND_BYTES = 2 * ADJ_BND_VALS * ADJ_BND_ROWS * (int)sizeof(double);
/* stages D and CTAs per SM: (2, 2) keeps a stage in flight while the
 * consumers work (168 registers); (1, 3) trades that for 50 % more warps
 * (128 registers) */
__host__ __device__ constexpr size_t adj_smem(int D)
{
    return (size_t)ADJ_HEADER + (size_t)D * ADJ_STAGE_BYTES + (size_t)ADJ_BND_BYTES;
}
static_assert(2 * (adj_smem(2) + 1024) <= 228 * 1024, "two CTAs per SM");
static_assert(3 * (adj_smem(1) + 1024) <= 228 * 1024, "three CTAs per SM");

__host__ __device__ constexpr int opp_of(int k) { return k == 0 ? 0 : (k <= 4 ? (k + 1) % 4 + 1 : (k + 1) % 4 + 5); }
static_assert(opp_of(1) == 3 && opp_of(2) == 4 && opp_of(3) == 1 && opp_of(4) == 2, "opposites");
static_assert(opp_of(5) == 7 && opp_of(6) == 8 && opp_of(7) == 5 && opp_of(8) == 6, "opposites");

__device__ __forceinline__ int clamp_row(int r, int Ny) { return r < 0 ? 0 : (r >= Ny ? Ny - 1 : r); }

__device__ __forceinline__ double warp_total(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

/* Producer: the 40 row-segment copies of work item (x0, y), segments of RW
 * doubles (band width + 2 * ADJ_AL). */
template <int RW>
__device__ __forceinline__ void adj_issue_t(const AdjPtrs &s, int Ny, int x0, int y, unsigned char *stage,
                                            uint64_t *full)
{
    constexpr int ADJ_SEG_BYTES = RW * (int)sizeof(double);
    mbar_arrive_expect_tx(full, ADJ_NSEG * ADJ_SEG_BYTES);
    const long long pl = s.plane;
    const int P = s.P;
#pragma unroll 1
    for (int k = 0; k < 9; k++) {
        const long long o1 = (long long)clamp_row(y + cy_of(k), Ny) * P + x0 - ADJ_AL;
        const long long o2 = (long long)clamp_row(y - cy_of(k), Ny) * P + x0 - ADJ_AL;
        bulk_g2s(stage + k * ADJ_SEG_BYTES, s.pin + k * pl + o1, ADJ_SEG_BYTES, full);
        bulk_g2s(stage + (9 + k) * ADJ_SEG_BYTES, s.pin + (9 + k) * pl + o1, ADJ_SEG_BYTES, full);
        bulk_g2s(stage + (21 + k) * ADJ_SEG_BYTES, s.f + k * pl + o2, ADJ_SEG_BYTES, full);
        bulk_g2s(stage + (30 + k) * ADJ_SEG_BYTES, s.g + k * pl + o2, ADJ_SEG_BYTES, full);
    }
    const long long op = (long long)clamp_row(y + 1, Ny) * P + x0 - ADJ_AL;
    const long long oy = (long long)y * P + x0 - ADJ_AL;
    bulk_g2s(stage + 18 * ADJ_SEG_BYTES, s.pin + 18 * pl + op, ADJ_SEG_BYTES, full);
    bulk_g2s(stage + 19 * ADJ_SEG_BYTES, s.pin + 19 * pl + op, ADJ_SEG_BYTES, full);
    bulk_g2s(stage + 20 * ADJ_SEG_BYTES, s.pin + 20 * pl + oy, ADJ_SEG_BYTES, full);
    bulk_g2s(stage + 39 * ADJ_SEG_BYTES, s.phi + op, ADJ_SEG_BYTES, full);
}

__device__ __forceinline__ void adj_issue(const AdjPtrs &s, int Ny, int x0, int y, unsigned char *stage,
                                          uint64_t *full)
{
    adj_issue_t<ADJ_RW>(s, Ny, x0, y, stage, full);
}

/* Fill the wall tables for rows ty0 .. ty0 + nrows - 1 of a tile, lane r
 * taking rows r, r + 32, ...: west node x = 0 into bw, east node x = Nx - 1
 * into be, each value read or formed exactly as the row loop of
 * adj_step_kernel does.  The west node's dL/dTin update, which needs only
 * Pi(n+1), is made here as well (row y's entry is updated by this lane
 * alone in the step). */
__device__ __forceinline__ void adj_fill_walls(const AdjPtrs &s, const Consts &c, const double *__restrict__ PIN,
                                               int ty0, int nrows, bool west, bool east, int lane, double *bw,
                                               double *be)
{
    const long long pl = s.plane;
    const int P = s.P, Nx = c.Nx, Ny = c.Ny;
    for (int r = lane; r < nrows; r += 32) {
        const int y = ty0 + r;
        const bool S = (y == 0), N = (y == Ny - 1);
        const int ym = S ? y : y - 1, yp = N ? y : y + 1;
        const int rc = clamp_row(y + 1, Ny);
        if (east) {
            const int x = Nx - 1;
            const long long cc = (long long)y * P + x;
            double *t = be + r;
            t[BE_PHI * ADJ_BND_ROWS] = s.phiE[rc];
            t[BE_BB3 * ADJ_BND_ROWS] = PIN[3 * pl + cc];
            t[BE_BB7 * ADJ_BND_ROWS] = PIN[7 * pl + cc];
            t[BE_BB6 * ADJ_BND_ROWS] = PIN[6 * pl + cc];
            /* T(Nx, y) is read by the east pulls of pops 3, 6 and 7 of the
             * next step */
            double lT = 0.0;
            lT += PIN[(9 + 3) * pl + cc] * c.w[3] * s.pE[y];
            double a6 = 0.0, a7 = 0.0;
            if (y + 1 < Ny) a6 += PIN[(9 + 6) * pl + cc + P];
            if (y == 0) a6 += PIN[(9 + 6) * pl + x];
            if (y - 1 >= 0) a7 += PIN[(9 + 7) * pl + cc - P];
            if (y == Ny - 1) a7 += PIN[(9 + 7) * pl + (long long)(Ny - 1) * P + x];
            lT += a6 * c.w[6] * s.pE[Ny + y] + a7 * c.w[7] * s.pE[2 * Ny + y];
            t[BE_LT * ADJ_BND_ROWS] = lT;
            t[BE_G3 * ADJ_BND_ROWS] = c.w[3] * s.tcol[y] * s.pE[y];
            t[BE_G6 * ADJ_BND_ROWS] = c.w[6] * s.tcol[ym] * s.pE[Ny + ym];
            t[BE_G7 * ADJ_BND_ROWS] = c.w[7] * s.tcol[yp] * s.pE[2 * Ny + yp];
            t[BE_F6 * ADJ_BND_ROWS] = S ? s.corner[0] : s.f[8 * pl + cc];
            t[BE_F7 * ADJ_BND_ROWS] = N ? s.corner[1] : s.f[5 * pl + cc];
        }
        if (west) {
            const long long cc = (long long)y * P;
            double *t = bw + r;
            t[BW_PHI * ADJ_BND_ROWS] = s.phiW[rc];
            t[BW_BB1 * ADJ_BND_ROWS] = PIN[1 * pl + cc];
            t[BW_BB8 * ADJ_BND_ROWS] = PIN[8 * pl + cc];
            t[BW_BB5 * ADJ_BND_ROWS] = PIN[5 * pl + cc];
            t[BW_GW0 * ADJ_BND_ROWS] = s.gW[y];
            t[BW_GW1 * ADJ_BND_ROWS] = s.gW[Ny + ym];
            t[BW_GW2 * ADJ_BND_ROWS] = s.gW[2 * Ny + yp];
            t[BW_F5 * ADJ_BND_ROWS] = s.f[7 * pl + cc];
            t[BW_F8 * ADJ_BND_ROWS] = s.f[6 * pl + cc];
            s.gtin[y] += tin_partial(PIN, pl, P, Ny, s.dgW, y);
        }
    }
}

/* Sum of a Pi row over columns x-1..x+1 inside the domain. */
__device__ __forceinline__ double row3(const double *v, int i, bool hasL, bool hasR)
{
    return (hasL ? v[i - 1] : 0.0) + v[i] + (hasR ? v[i + 1] : 0.0);
}

/* Register split (WSPLIT): the CTA is two warpgroups, the four consumer
 * warps and a producer warpgroup whose warp 4 lane 0 issues the copies.  It
 * is launched with ADJ_LAUNCH_REGS registers per thread; the producer
 * warpgroup gives all but ADJ_PROD_REGS back (setmaxnreg.dec) and the
 * consumers take them (setmaxnreg.inc to ADJ_CONS_REGS), so the node VJP
 * runs without spills at two CTAs per SM.  The two shares add up to the
 * launch allocation exactly: ADJ_CONS_REGS + ADJ_PROD_REGS =
 * 2 * ADJ_LAUNCH_REGS; the host checks the kernel's register count before
 * it selects this variant. */
constexpr int ADJ_LAUNCH_REGS = 128, ADJ_PROD_REGS = 40, ADJ_CONS_REGS = 216;
static_assert(ADJ_CONS_REGS + ADJ_PROD_REGS == 2 * ADJ_LAUNCH_REGS, "register split must match the launch");
static_assert(ADJ_CONS_REGS % 8 == 0 && ADJ_PROD_REGS % 8 == 0 && ADJ_PROD_REGS >= 24, "setmaxnreg granularity");

template <int ADJ_D, int ADJ_CTAS, bool WSPLIT = false>
__global__ void __launch_bounds__(WSPLIT ? 256 : PIPE_THREADS, ADJ_CTAS)
adj_pipe_kernel(AdjPtrs s, Consts c, PipeSched sch, int *errflag)
{
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t *full = reinterpret_cast<uint64_t *>(smem);
    uint64_t *empty = full + ADJ_D;
    unsigned char *stages = smem + ADJ_HEADER;
    double *bwall = reinterpret_cast<double *>(stages + (size_t)ADJ_D * ADJ_STAGE_BYTES);   /* wall tables */
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int Nx = c.Nx, Ny = c.Ny;
    if (tid == 0) {
        for (int d = 0; d < ADJ_D; d++) {
            mbar_init(&full[d], 1);
            mbar_init(&empty[d], PIPE_CWARPS);
        }
        mbar_fence_init();
    }
    __syncthreads();
    pdl_allow_next();
    pdl_wait();
    if (warp >= PIPE_CWARPS) {
        if constexpr (WSPLIT) asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;" ::"n"(ADJ_PROD_REGS));
        if (warp != PIPE_CWARPS || lane != 0) return;
        PipeIter it;
        long long r = 0;
        bool ok = it.start(sch, Ny);
        while (ok) {
            const int st = (int)(r % ADJ_D);
            if (r >= ADJ_D && !mbar_wait(&empty[st], (uint32_t)(((r / ADJ_D) - 1) & 1))) {
                atomicExch(errflag, 11);
                break;
            }
            adj_issue(s, Ny, it.x0, it.y, stages + (size_t)st * ADJ_STAGE_BYTES, &full[st]);
            r++;
            ok = it.next();
        }
        /* do not retire while copies into this CTA's shared memory are in flight */
        for (long long q = (r > ADJ_D ? r - ADJ_D : 0); q < r; q++)
            if (!mbar_wait(&full[q % ADJ_D], (uint32_t)((q / ADJ_D) & 1))) atomicExch(errflag, 12);
        return;
    }

    if constexpr (WSPLIT) asm volatile("setmaxnreg.inc.sync.aligned.u32 %0;" ::"n"(ADJ_CONS_REGS));
    const long long pl = s.plane;
    const int P = s.P;
    const double *__restrict__ PIN = s.pin;
    double omg_sum = 0.0;
    PipeIter it;
    long long r = 0;
    bool ok = it.start(sch, Ny);
    while (ok) {
        const int x = it.x0 + tid;
        const bool active = x < Nx;
        const bool W = (x == 0), E = (x == Nx - 1);
        const bool hasL = x > 0, hasR = x + 1 < Nx;
        /* windows: phi of columns x-1..x+1 and the Pi_k+/Pi_k- row sums, rows
         * y-1, y (slots 0, 1); slot 2 is filled from the stage */
        double ph[3][3], rk[3], rm[3];
        if (active) {
#pragma unroll
            for (int slot = 0; slot < 2; slot++) {
                const int rr = it.y - 1 + slot;
                const int rc = clamp_row(rr, Ny);
                const double *row = s.phi + (long long)rc * P;
                ph[slot][0] = W ? s.phiW[rc] : row[x - 1];
                ph[slot][1] = row[x];
                ph[slot][2] = E ? s.phiE[rc] : row[x + 1];
                if (rr >= 0) {
                    rk[slot] = row3(PIN + 18 * pl + (long long)rr * P, x, hasL, hasR);
                    rm[slot] = row3(PIN + 19 * pl + (long long)rr * P, x, hasL, hasR);
                } else {
                    rk[slot] = 0.0;
                    rm[slot] = 0.0;
                }
            }
        }
        /* wall tables of this tile, filled by the warp that holds the west
         * or east node (warp-private: only that warp's lanes touch them) */
        const int ty0 = it.y;
        const int eoff = Nx - 1 - it.x0;
        const bool wwest = it.x0 == 0 && warp == 0;
        const bool weast = eoff < PIPE_BX && warp == (eoff >> 5);
        if (wwest || weast) {
            int nrows = it.y1 - it.y;
            if (nrows > ADJ_BND_ROWS) {         /* adj_sched never picks such H */
                if (lane == 0) atomicExch(errflag, 14);
                nrows = ADJ_BND_ROWS;
            }
            __syncwarp();
            adj_fill_walls(s, c, PIN, ty0, nrows, wwest, weast, lane, bwall, bwall + ADJ_BND_VALS * ADJ_BND_ROWS);
            __syncwarp();
        }
        const int tile = it.t;
        bool failed = false;
        do {
            const int y = it.y;
            const int st = (int)(r % ADJ_D);
            if (!__all_sync(0xffffffffu, mbar_wait(&full[st], (uint32_t)((r / ADJ_D) & 1)))) {
                atomicExch(errflag, 13);
                failed = true;
                break;
            }
            double *stg = reinterpret_cast<double *>(stages + (size_t)st * ADJ_STAGE_BYTES);
            bool wrote = false;
            if (active) {
                const bool S = (y == 0), N = (y == Ny - 1);
                const long long cc = (long long)y * P + x;
                const int col = tid + ADJ_AL;
                /* this row's entries of the wall tables */
                const int rl = (y - ty0) & (ADJ_BND_ROWS - 1);
                auto wv = [&](int v) { return bwall[v * ADJ_BND_ROWS + rl]; };
                auto ev = [&](int v) { return bwall[(ADJ_BND_VALS + v) * ADJ_BND_ROWS + rl]; };
                /* new row y+1 of both windows */
                {
                    const double *sph = stg + 39 * ADJ_RW;
                    ph[2][0] = W ? wv(BW_PHI) : sph[col - 1];
                    ph[2][1] = sph[col];
                    ph[2][2] = E ? ev(BE_PHI) : sph[col + 1];
                    if (y + 1 < Ny) {
                        rk[2] = row3(stg + 18 * ADJ_RW, col, hasL, hasR);
                        rm[2] = row3(stg + 19 * ADJ_RW, col, hasL, hasR);
                    } else {
                        rk[2] = 0.0;
                        rm[2] = 0.0;
                    }
                }

                /* 1. the adjoint of S(n) at this node.  lambda_f[k] and
                 * lambda_g[k] are the stage words at (segment k or 9+k,
                 * column x + c_kx); each such word is read by this thread
                 * only, so a boundary node writes its own gathered value over
                 * it and the VJP reads every lambda from the stage. */
                if (W || E || S || N) {
                    wrote = true;
#pragma unroll
                    for (int k = 0; k < 9; k++) {
                        const int xd = x + cx_of(k), yd = y + cy_of(k);
                        const bool xin = xd >= 0 && xd < Nx, yin = yd >= 0 && yd < Ny;
                        double *wf = stg + k * ADJ_RW + col + cx_of(k);
                        double *wg = stg + (9 + k) * ADJ_RW + col + cx_of(k);
                        if (!(xin && yin)) {
                            /* read by this node's own bounce-back of opp(k),
                             * except the two frozen corners (pop 6 at (Nx,1),
                             * pop 7 at (Nx,Ny)) */
                            const bool corner6 = (k == 8) && E && S;
                            const bool corner7 = (k == 5) && E && N;
                            double v;
                            if (cx_of(k) == -1 && W)
                                v = wv(k == 3 ? BW_BB1 : (k == 6 ? BW_BB8 : BW_BB5));
                            else if (cx_of(k) == 1 && E)
                                v = ev(k == 1 ? BE_BB3 : (k == 5 ? BE_BB7 : BE_BB6));
                            else
                                v = PIN[opp_of(k) * pl + cc];
                            *wf = (corner6 || corner7) ? 0.0 : v;
                        }
                        double a = 0.0;
                        if (xin) {
                            if (yin) a += *wg;
                            if (cy_of(k) == 1 && S) a += PIN[(9 + k) * pl + xd];
                            if (cy_of(k) == -1 && N) a += PIN[(9 + k) * pl + (long long)(Ny - 1) * P + xd];
                        }
                        *wg = a;
                    }
                }
                const double skp = rk[0] + rk[1] + rk[2] + (S ? rk[1] : 0.0) + (N ? rk[1] : 0.0);
                const double skm = rm[0] + rm[1] + rm[2] + (S ? rm[1] : 0.0) + (N ? rm[1] : 0.0);
                const double d0 = stg[20 * ADJ_RW + col];
                /* T(Nx, y) partial (east); the west node's dL/dTin update was
                 * made when the wall table was filled */
                const double lT = E ? ev(BE_LT) : 0.0;

                /* 2. pulled inputs of step n from S(n-1), as the forward pipeline */
                const double *sp = stg + 21 * ADJ_RW, *sg = stg + 30 * ADJ_RW;
                const double *F = s.f;
                double f[9], g[9];
                f[0] = sp[0 * ADJ_RW + col];
                f[1] = W ? sp[3 * ADJ_RW + col] : sp[1 * ADJ_RW + col - 1];
                f[2] = sp[2 * ADJ_RW + col];
                f[3] = E ? sp[1 * ADJ_RW + col] : sp[3 * ADJ_RW + col + 1];
                f[4] = sp[4 * ADJ_RW + col];
                f[5] = sp[5 * ADJ_RW + col - 1];
                f[6] = sp[6 * ADJ_RW + col + 1];
                f[7] = sp[7 * ADJ_RW + col + 1];
                f[8] = sp[8 * ADJ_RW + col - 1];
                if (W || E || S || N) {
                    if (S) f[2] = F[4 * pl + cc];
                    if (N) f[4] = F[2 * pl + cc];
                    if (W) f[5] = wv(BW_F5);
                    else if (S) f[5] = F[7 * pl + cc];
                    if (E) f[6] = ev(BE_F6);
                    else if (S) f[6] = F[8 * pl + cc];
                    if (E) f[7] = ev(BE_F7);
                    else if (N) f[7] = F[5 * pl + cc];
                    if (W) f[8] = wv(BW_F8);
                    else if (N) f[8] = F[6 * pl + cc];
                }
                g[0] = sg[0 * ADJ_RW + col];
                g[2] = sg[2 * ADJ_RW + col];
                g[4] = sg[4 * ADJ_RW + col];
                if (W) {
                    g[1] = wv(BW_GW0);
                    g[5] = wv(BW_GW1);
                    g[8] = wv(BW_GW2);
                } else {
                    g[1] = sg[1 * ADJ_RW + col - 1];
                    g[5] = sg[5 * ADJ_RW + col - 1];
                    g[8] = sg[8 * ADJ_RW + col - 1];
                }
                if (E) {
                    g[3] = ev(BE_G3);
                    g[6] = ev(BE_G6);
                    g[7] = ev(BE_G7);
                } else {
                    g[3] = sg[3 * ADJ_RW + col + 1];
                    g[6] = sg[6 * ADJ_RW + col + 1];
                    g[7] = sg[7 * ADJ_RW + col + 1];
                }
                /* selector sums in the forward kernel's order */
                const double kp = bgk::aplus(ph[1][1]) + bgk::aplus(ph[1][2]) + bgk::aplus(ph[2][1]) +
                                  bgk::aplus(ph[1][0]) + bgk::aplus(ph[0][1]) + bgk::aplus(ph[2][2]) +
                                  bgk::aplus(ph[2][0]) + bgk::aplus(ph[0][0]) + bgk::aplus(ph[0][2]);
                const double km = bgk::aminus(ph[1][1]) + bgk::aminus(ph[1][2]) + bgk::aminus(ph[2][1]) +
                                  bgk::aminus(ph[1][0]) + bgk::aminus(ph[0][1]) + bgk::aminus(ph[2][2]) +
                                  bgk::aminus(ph[2][0]) + bgk::aminus(ph[0][0]) + bgk::aminus(ph[0][2]);

                /* 3. vector-Jacobian product -> Pi(n) */
                const double *lam = stg + col;
                double *po = s.pout + cc;
                double kpb, kmb, p0b, omg_b;
                node_vjp(c, s.tanh_mode, f, g, kp, km, ph[1][1],
                         [&](int k) { return lam[k * ADJ_RW + cx_of(k)]; },
                         [&](int k) { return lam[(9 + k) * ADJ_RW + cx_of(k)]; }, d0, skp, skm, lT,
                         [&](int k, double v) { po[k * pl] = v; }, [&](int k, double v) { po[(9 + k) * pl] = v; },
                         kpb, kmb, p0b, omg_b, s.inv_T_width, s.inv_omega_f);
                omg_sum += omg_b;
                s.pout[18 * pl + cc] = kpb;
                s.pout[19 * pl + cc] = kmb;
                s.pout[20 * pl + cc] = p0b;
#pragma unroll
                for (int k = 0; k < 3; k++) {
                    ph[0][k] = ph[1][k];
                    ph[1][k] = ph[2][k];
                }
                rk[0] = rk[1]; rk[1] = rk[2];
                rm[0] = rm[1]; rm[1] = rm[2];
            }
            /* generic-proxy writes into the stage are ordered before the
             * producer's next bulk copy into it */
            if (__any_sync(0xffffffffu, wrote)) asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty[st]);
            r++;
            ok = it.next();
        } while (ok && it.t == tile);
        if (failed) break;
    }
    /* d/d omega_g: one running partial per consumer warp, in a fixed order */
    omg_sum = warp_total(omg_sum);
    if (lane == 0) s.omg_acc[blockIdx.x * PIPE_CWARPS + warp] += omg_sum;
}

/* Tile height for the reverse step: the H that minimises the waves of tiles
 * times (H + 1), the 1 standing for the per-tile window prologue. */
PipeSched adj_sched(const bgk_ctx *c, int ctas_per_sm, int bx, int *grid)
{
    PipeSched sch{};   /* tiles of H rows (ranges = 0): the wall tables hold one tile */
    sch.bx = bx;
    sch.nbands = (c->Nx + bx - 1) / bx;
    const long long slots = (long long)c->nsm * ctas_per_sm;
    long long best = -1;
    int bestH = 1;
    for (int H = 1; H <= ADJ_BND_ROWS; H++) {
        const long long tiles = (long long)sch.nbands * ((c->Ny + H - 1) / H);
        const long long waves = (tiles + slots - 1) / slots;
        const long long cost = waves * (H + 1);
        if (best < 0 || cost < best) { best = cost; bestH = H; }
        if (H >= c->Ny) break;
    }
    if (c->tune_H > 0) bestH = c->tune_H < ADJ_BND_ROWS ? c->tune_H : ADJ_BND_ROWS;   /* wall tables */
    sch.H = bestH;
    sch.nstrips = (c->Ny + bestH - 1) / bestH;
    sch.ntiles = sch.nbands * sch.nstrips;
    *grid = (int)(sch.ntiles < slots ? sch.ntiles : slots);
    return sch;
}

/* dL/dTin per row from the west nodes' pulled-g partials of one step (the
 * step kernel folds in those of the step after it; this kernel takes the
 * partials of step 1 at the end of the sweep). */
__global__ void adj_tin_kernel(const double *pi, long long plane, int P, int Ny, const double *dgW, double *grad)
{
    for (int y = threadIdx.x; y < Ny; y += blockDim.x) grad[y] += tin_partial(pi, plane, P, Ny, dgW, y);
}

/* d gW_k / d Tin = w_k * poly_k(u(0,j), v(0,j)) for k = 1, 5, 8 */
__global__ void adj_dgw_kernel(Consts c, const double *mu, const double *mv, double *dgW)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x + 1;
    if (j > c.Ny) return;
    const size_t q = (size_t)(c.Nx + 2) * j;
    double P[9];
    bgk::eq_poly(mu[q], mv[q], P);
    dgW[j - 1] = c.w[1] * P[1];
    dgW[c.Ny + j - 1] = c.w[5] * P[5];
    dgW[2 * c.Ny + j - 1] = c.w[8] * P[8];
}

/* Loss and its seed: Pi(N+1)[phi_prec] = 2 (phi - target) at the probes
 * (serial, so repeated probes add deterministically). */
__global__ void adj_seed_kernel(const double *phi, long long plane, int P, int np, const int *pi_, const int *pj,
                                const double *target, double *seed_plane, double *loss)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double L = 0.0;
    for (int p = 0; p < np; p++) {
        const long long q = (long long)(pj[p] - 1) * P + (pi_[p] - 1);
        const double r = phi[q] - target[p];
        L += r * r;
        seed_plane[q] += 2.0 * r;
    }
    *loss = L;
}

__global__ void adj_sum_kernel(const double *acc, int n, double *out)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double s = 0.0;
    for (int i = 0; i < n; i++) s += acc[i];
    *out = s;
}

} // namespace

extern "C" int bgk_adjoint_run(bgk_ctx *c, const bgk_adjoint_spec *spec, double *loss, double *grad_tin,
                               double *grad_tau_g)
{
    if (!c || !spec || !loss || !grad_tau_g) return bgk_internal_fail(BGK_ERR_ARG, "null argument");
    if (c->opt.precision != BGK_PREC_F64 || !c->opt.smooth)
        return bgk_internal_fail(BGK_ERR_UNSUPPORTED, "the adjoint differentiates the smooth FP64 form: create the "
                                                      "context with precision BGK_PREC_F64 and smooth = 1");
    const int N = spec->nsteps;
    if (N < 1) return bgk_internal_fail(BGK_ERR_ARG, "nsteps must be >= 1");
    if (spec->nprobes < 1 || !spec->probe_i || !spec->probe_j || !spec->phi_target)
        return bgk_internal_fail(BGK_ERR_ARG, "at least one probe is needed");
    for (int p = 0; p < spec->nprobes; p++)
        if (spec->probe_i[p] < 1 || spec->probe_i[p] > c->Nx || spec->probe_j[p] < 1 || spec->probe_j[p] > c->Ny)
            return bgk_internal_fail(BGK_ERR_ARG, "probe outside 1..Nx x 1..Ny");
    int rc = bgk_internal_prepare_fused(c);
    if (rc) return rc;

    cudaStream_t st = c->stream;
    const long long pl = c->plane;
    const int Ny = c->Ny;
    /* one stored state: f (9 planes), g (9), phi (1), T column (Ny, padded),
     * with a guard before and after it: the fused step's shared-memory
     * pipeline copies row segments that start 16 bytes before a band and may
     * run up to a band (128 elements) past the last row of a plane */
    const long long tc_pad = ((long long)Ny + 31) / 32 * 32;
    const size_t state_guard = 256;     /* elements on each side */
    const size_t state_elems = (size_t)(19 * pl + tc_pad) + 2 * state_guard;
    const size_t state_bytes = state_elems * sizeof(double);

    /* Checkpoint schedule.  K > 0: snapshots every K steps, each K-step
     * segment recomputed into a buffer of K + 1 states and reversed (the
     * sqrt(N) scheme; K = ceil(sqrt(N)) when checkpoint_every is 0).  When
     * that does not fit in free device memory, or when checkpoint_every < 0,
     * a binomial schedule (Griewank's revolve, written as a recursion) with
     * a fixed number of state slots: -checkpoint_every of them, or as many
     * as fit.  Both give the same gradient bit for bit. */
    int K = spec->checkpoint_every > 0 ? spec->checkpoint_every : (int)std::ceil(std::sqrt((double)N));
    if (K > N) K = N;
    const int nsnap = (N + K - 1) / K;    /* snapshots of S(0), S(K), ...    */
    const size_t fixed_bytes = 2 * ((size_t)NPI * pl + 2 * state_guard) * sizeof(double) + 8 * (size_t)Ny * 8 +
                               (64u << 20);
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
        (void)cudaGetLastError();
        return bgk_internal_fail(BGK_ERR_CUDA, "cudaMemGetInfo failed");
    }
    free_b += c->adj_ws_bytes;            /* a cached workspace can be given back */
    const size_t margin = (size_t)1 << 30;
    const size_t avail = free_b > fixed_bytes + margin ? free_b - fixed_bytes - margin : 0;
    bool binomial = spec->checkpoint_every < 0 || (size_t)(nsnap + K + 1) * state_bytes > avail;
    int nslots = 0;                        /* binomial: state slots incl. S(0) */
    if (binomial) {
        nslots = spec->checkpoint_every < 0 ? -spec->checkpoint_every : (int)(avail / state_bytes) - 2;
        if (nslots > N) nslots = N;
        if (nslots < 1 || (size_t)(nslots + 2) * state_bytes > avail)
            return bgk_internal_fail(BGK_ERR_OOM, "not enough device memory for the adjoint's checkpoints");
    }

    /* reverse-step kernel: the shared-memory pipeline (adj_pipe_kernel), or
     * the register gather (adj_step_kernel) when the context selects the
     * register-pull kernels */
    const int akind = c->tune_pipe ? 1 : 0;
    dim3 blk(AB_X, AB_Y), grd((c->Nx + AB_X - 1) / AB_X, (Ny + AB_Y - 1) / AB_Y);
    int pgrid = 0, partials = 0;
    PipeSched psch{};
    /* variant of the reverse step: 2 = two stages, two CTAs per SM and the
     * producer/consumer register split (default, when the kernel's launch
     * register count makes the split exact); 0 = the same without the
     * split; 1 = one stage, three CTAs per SM (BGK_ADJ_PIPE selects) */
    int adj_var = 2;
    if (const char *v = getenv("BGK_ADJ_PIPE")) adj_var = atoi(v);
    if (adj_var == 2) {
        cudaFuncAttributes fa{};
        if (cudaFuncGetAttributes(&fa, adj_pipe_kernel<2, 2, true>) != cudaSuccess ||
            fa.numRegs != ADJ_LAUNCH_REGS) {
            (void)cudaGetLastError();
            adj_var = 0;
        }
    }
    if (adj_var < 0 || adj_var > 2) adj_var = 2;
    const int adj_ctas = adj_var == 1 ? 3 : 2;
    if (akind == 1) {
        psch = adj_sched(c, adj_ctas, PIPE_BX, &pgrid);
        partials = PIPE_CWARPS;
    }
    const int nblk = akind ? pgrid * partials : (int)(grd.x * grd.y);

    /* Workspace: one device allocation, carved in 256-byte aligned pieces.
     * It stays in the context for the next call (freed by bgk_destroy)
     * unless it is larger than a quarter of the device memory.
     * sqrt(N): nsnap snapshots + K+1 segment states; binomial: nslots slots
     * + 2 work states.  State i of a block at base + i * state_elems. */
    const size_t nstates_a = binomial ? (size_t)nslots : (size_t)nsnap;
    const size_t nstates_b = binomial ? 2 : (size_t)(K + 1);
    const size_t pi_bytes = ((size_t)NPI * pl + 2 * state_guard) * sizeof(double);
    const size_t piece[] = {nstates_a * state_bytes, nstates_b * state_bytes, pi_bytes, pi_bytes,
                            (size_t)nblk * sizeof(double), 3 * (size_t)Ny * sizeof(double),
                            (size_t)Ny * sizeof(double), 4 * sizeof(double),
                            (size_t)spec->nprobes * sizeof(int) + 16, (size_t)spec->nprobes * sizeof(int) + 16,
                            (size_t)spec->nprobes * sizeof(double)};
    constexpr int NPIECE = (int)(sizeof(piece) / sizeof(piece[0]));
    size_t off[NPIECE], ws_bytes = 0;
    for (int i = 0; i < NPIECE; i++) {
        off[i] = ws_bytes;
        ws_bytes += (piece[i] + 255) / 256 * 256;
    }
    if (c->adj_ws_bytes < ws_bytes) {
        if (c->adj_ws) cudaFree(c->adj_ws);
        c->adj_ws = nullptr;
        c->adj_ws_bytes = 0;
        if (cudaMalloc(&c->adj_ws, ws_bytes) != cudaSuccess) {
            (void)cudaGetLastError();
            c->adj_ws = nullptr;
            return bgk_internal_fail(BGK_ERR_OOM, "adjoint workspace allocation failed");
        }
        c->adj_ws_bytes = ws_bytes;
    }
    auto cleanup = [&]() {
        if (c->adj_ws_bytes > total_b / 4) {
            cudaFree(c->adj_ws);
            c->adj_ws = nullptr;
            c->adj_ws_bytes = 0;
        }
    };
    char *wsb = static_cast<char *>(c->adj_ws);
    auto at = [&](int i) { return static_cast<void *>(wsb + off[i]); };
    double *snaps = static_cast<double *>(at(0)) + state_guard;
    double *seg = static_cast<double *>(at(1)) + state_guard;
    /* partial planes Pi, guarded like the states (the pipelined reverse step
     * copies row segments of them) */
    double *pi[2] = {static_cast<double *>(at(2)) + state_guard, static_cast<double *>(at(3)) + state_guard};
    double *omg_acc = static_cast<double *>(at(4));
    double *dgW = static_cast<double *>(at(5));
    double *gtin = static_cast<double *>(at(6));
    double *scal = static_cast<double *>(at(7));
    int *dpi = static_cast<int *>(at(8));
    int *dpj = static_cast<int *>(at(9));
    double *dtg = static_cast<double *>(at(10));
#define ACK(call)                                                                   \
    do {                                                                            \
        cudaError_t e_ = (call);                                                    \
        if (e_ != cudaSuccess) {                                                    \
            cleanup();                                                              \
            return bgk_internal_fail(BGK_ERR_CUDA, cudaGetErrorString(e_));         \
        }                                                                           \
    } while (0)
    auto copy_state_in = [&](double *dst, int buf) -> cudaError_t {
        cudaError_t e;
        if ((e = cudaMemcpyAsync(dst, c->fbuf[buf], 9 * pl * sizeof(double), cudaMemcpyDeviceToDevice, st))) return e;
        if ((e = cudaMemcpyAsync(dst + 9 * pl, c->gbuf[buf], 9 * pl * sizeof(double), cudaMemcpyDeviceToDevice, st)))
            return e;
        if ((e = cudaMemcpyAsync(dst + 18 * pl, c->phibuf[buf], pl * sizeof(double), cudaMemcpyDeviceToDevice, st)))
            return e;
        return cudaMemcpyAsync(dst + 19 * pl, c->tcol[buf], Ny * sizeof(double), cudaMemcpyDeviceToDevice, st);
    };
    auto copy_state_out = [&](int buf, const double *src) -> cudaError_t {
        cudaError_t e;
        if ((e = cudaMemcpyAsync(c->fbuf[buf], src, 9 * pl * sizeof(double), cudaMemcpyDeviceToDevice, st))) return e;
        if ((e = cudaMemcpyAsync(c->gbuf[buf], src + 9 * pl, 9 * pl * sizeof(double), cudaMemcpyDeviceToDevice, st)))
            return e;
        if ((e = cudaMemcpyAsync(c->phibuf[buf], src + 18 * pl, pl * sizeof(double), cudaMemcpyDeviceToDevice, st)))
            return e;
        return cudaMemcpyAsync(c->tcol[buf], src + 19 * pl, Ny * sizeof(double), cudaMemcpyDeviceToDevice, st);
    };
    /* one fused forward step between two stored states */
    auto fwd = [&](const double *a, double *b) -> cudaError_t {
        return bgk::launch_fused_f64_ptrs(c, a, a + 9 * pl, a + 18 * pl, a + 19 * pl, b, b + 9 * pl, b + 18 * pl,
                                          b + 19 * pl);
    };
    /* one reverse step: forward step n, from S(n-1) */
    int pin = 0;
    auto rstep = [&](const double *S0) -> cudaError_t {
        AdjPtrs a{};
        a.f = S0; a.g = S0 + 9 * pl; a.phi = S0 + 18 * pl; a.tcol = S0 + 19 * pl;
        a.pin = pi[pin]; a.pout = pi[pin ^ 1];
        a.gW = c->gW; a.pE = c->pE; a.phiW = c->phiW; a.phiE = c->phiE; a.corner = c->corner;
        a.omg_acc = omg_acc;
        a.dgW = dgW; a.gtin = gtin;
        a.inv_T_width = 1.0 / c->c.T_width;
        a.inv_omega_f = 1.0 / c->c.omega_f;
        a.plane = pl; a.P = c->P;
        a.tanh_mode = c->opt.tanh_mode;
        if (akind == 1)
        {
            cudaError_t e;
            if (adj_var == 1)
                e = pdl_launch(adj_pipe_kernel<1, 3>, pgrid, PIPE_THREADS, adj_smem(1), st, a, c->c, psch, c->errflag);
            else if (adj_var == 2)
                e = pdl_launch(adj_pipe_kernel<2, 2, true>, pgrid, 256, adj_smem(2), st, a, c->c, psch, c->errflag);
            else
                e = pdl_launch(adj_pipe_kernel<2, 2>, pgrid, PIPE_THREADS, adj_smem(2), st, a, c->c, psch, c->errflag);
            if (e != cudaSuccess) return e;
        }
        else
            adj_step_kernel<<<grd, blk, 0, st>>>(a, c->c);
        pin ^= 1;
        return cudaGetLastError();
    };

    if (akind == 1) {
        static std::atomic<unsigned long long> done{0};
        static std::atomic<unsigned long long> done1{0}, done2{0};
        if (adj_var == 1) ACK(pipe_configure(adj_pipe_kernel<1, 3>, adj_smem(1), c->dev, done1));
        else if (adj_var == 2) ACK(pipe_configure(adj_pipe_kernel<2, 2, true>, adj_smem(2), c->dev, done2));
        else ACK(pipe_configure(adj_pipe_kernel<2, 2>, adj_smem(2), c->dev, done));
    }
    ACK(cudaMemcpyAsync(dpi, spec->probe_i, spec->nprobes * sizeof(int), cudaMemcpyHostToDevice, st));
    ACK(cudaMemcpyAsync(dpj, spec->probe_j, spec->nprobes * sizeof(int), cudaMemcpyHostToDevice, st));
    ACK(cudaMemcpyAsync(dtg, spec->phi_target, spec->nprobes * sizeof(double), cudaMemcpyHostToDevice, st));
    adj_dgw_kernel<<<(Ny + 127) / 128, 128, 0, st>>>(c->c, c->mu, c->mv, dgW);
    ACK(cudaGetLastError());

    /* forward pass on the context (snapshots every K steps in the sqrt(N)
     * scheme; S(0) only in the binomial one) */
    ACK(copy_state_in(snaps, c->cur));
    bool last_in_seg = false;             /* the last segment's states are in seg */
    if (binomial) {
        rc = bgk_step(c, N);
        if (rc) { cleanup(); return rc; }
    } else {
        for (int n0 = 0; n0 < N; n0 += K) {
            const int len = (n0 + K < N) ? K : N - n0;
            if (n0 + len < N) {
                rc = bgk_internal_advance(c, len);
                if (rc) { cleanup(); return rc; }
                ACK(copy_state_in(snaps + (size_t)((n0 + len) / K) * state_elems, c->cur));
            } else if (len >= 3) {
                /* last segment: S(n0+1) .. S(N-2) go straight into the
                 * segment buffer, so the reverse sweep need not recompute
                 * them; S(N-2) is copied into the context, whose last two
                 * steps run through bgk_step (moments and halos), and S(N-1)
                 * is copied back from the context's other buffer */
                rc = bgk_internal_prepare_fused(c);
                if (rc) { cleanup(); return rc; }
                const double *s0 = snaps + (size_t)(n0 / K) * state_elems;
                for (int n = n0 + 1; n <= N - 2; n++)
                    ACK(fwd(n - 1 == n0 ? s0 : seg + (size_t)(n - 1 - n0) * state_elems,
                            seg + (size_t)(n - n0) * state_elems));
                ACK(copy_state_out(c->cur, seg + (size_t)(N - 2 - n0) * state_elems));
                c->it += len - 2;
                c->pristine = false;
                rc = bgk_step(c, 2);
                if (rc) { cleanup(); return rc; }
                ACK(copy_state_in(seg + (size_t)(N - 1 - n0) * state_elems, c->cur ^ 1));
                last_in_seg = true;
            } else {
                rc = bgk_step(c, len);
                if (rc) { cleanup(); return rc; }
            }
        }
    }
    /* loss and seed */
    ACK(cudaMemsetAsync(pi[0], 0, (size_t)NPI * pl * sizeof(double), st));
    ACK(cudaMemsetAsync(omg_acc, 0, (size_t)nblk * sizeof(double), st));
    ACK(cudaMemsetAsync(gtin, 0, (size_t)Ny * sizeof(double), st));
    adj_seed_kernel<<<1, 32, 0, st>>>((const double *)c->phibuf[c->cur], pl, c->P, spec->nprobes, dpi, dpj, dtg,
                                      pi[0] + 20 * pl, scal);
    ACK(cudaGetLastError());

    if (!binomial) {
        /* reverse sweep, one segment at a time */
        for (int sgi = nsnap - 1; sgi >= 0; sgi--) {
            const int n0 = sgi * K;
            const int n1 = (n0 + K < N) ? n0 + K : N;
            /* S(n0) is the snapshot itself; S(n0+1) .. S(n1-1) are recomputed
             * into seg[1 .. n1-n0-1] */
            auto state = [&](int n) {
                return n == n0 ? snaps + (size_t)sgi * state_elems : seg + (size_t)(n - n0) * state_elems;
            };
            if (!(last_in_seg && sgi == nsnap - 1))
                for (int n = n0 + 1; n < n1; n++) ACK(fwd(state(n - 1), state(n)));
            for (int n = n1; n > n0; n--) ACK(rstep(state(n - 1)));
        }
    } else {
        double *work[2] = {seg, seg + state_elems};
        auto slot = [&](int i) { return snaps + (size_t)i * state_elems; };
        /* S(a + steps) from S(a) in src into dst (dst is a slot or work[1]):
         * the intermediate states alternate between work[0] and dst itself,
         * in the parity that ends on dst */
        auto advance = [&](const double *src, int steps, double *dst) -> cudaError_t {
            const double *cur = src;
            for (int i = 1; i <= steps; i++) {
                double *next = ((steps - i) % 2 == 0) ? dst : work[0];
                cudaError_t e = fwd(cur, next);
                if (e != cudaSuccess) return e;
                cur = next;
            }
            return cudaSuccess;
        };
        /* C(cp + r, cp): steps reversible with cp checkpoints and r repetitions */
        auto beta = [](int cp, int r) {
            double v = 1.0;
            for (int i = 1; i <= cp; i++) v = v * (double)(r + i) / (double)i;
            return v;
        };
        /* reverse forward steps b, b-1, ..., a+1; S(a) is in slot ia; slots
         * ia+1 .. nslots-1 are free */
        std::function<cudaError_t(int, int, int)> rev = [&](int a, int b, int ia) -> cudaError_t {
            const int n = b - a;
            const int nfree = nslots - 1 - ia;
            cudaError_t e;
            if (n == 1) return rstep(slot(ia));
            if (nfree == 0) {
                for (int k = b; k > a; k--) {
                    if (k - 1 == a) {
                        e = rstep(slot(ia));
                    } else {
                        if ((e = advance(slot(ia), k - 1 - a, work[1])) != cudaSuccess) return e;
                        e = rstep(work[1]);
                    }
                    if (e != cudaSuccess) return e;
                }
                return cudaSuccess;
            }
            /* fewest repetitions r with C(cp + r, cp) >= n; the first
             * checkpoint goes l steps ahead, l in [n - C(cp - 1 + r, cp - 1),
             * C(cp + r - 1, cp)] (right part reversible with one checkpoint
             * less, left part with one repetition less); the middle of that
             * range is within ~1 % of the fewest forward steps */
            const int cp = nfree + 1;
            int r = 0;
            while (beta(cp, r) < (double)n) r++;
            const double rmax = beta(cp - 1, r), lmax = beta(cp, r - 1);
            const int lo = rmax >= (double)(n - 1) ? 1 : n - (int)rmax;
            const int hi = lmax >= (double)(n - 1) ? n - 1 : (int)lmax;
            int l = (lo + hi) / 2;
            if (l < 1) l = 1;
            if (l > n - 1) l = n - 1;
            const int m = a + l;
            if ((e = advance(slot(ia), l, slot(ia + 1))) != cudaSuccess) return e;
            if ((e = rev(m, b, ia + 1)) != cudaSuccess) return e;
            return rev(a, m, ia);
        };
        ACK(rev(0, N, 0));
    }
    adj_tin_kernel<<<1, 1024, 0, st>>>(pi[pin], pl, c->P, Ny, dgW, gtin);
    ACK(cudaGetLastError());
    adj_sum_kernel<<<1, 32, 0, st>>>(omg_acc, nblk, scal + 1);
    ACK(cudaGetLastError());
    double host[2];
    ACK(cudaMemcpyAsync(host, scal, 2 * sizeof(double), cudaMemcpyDeviceToHost, st));
    if (grad_tin) ACK(cudaMemcpyAsync(grad_tin, gtin, (size_t)Ny * sizeof(double), cudaMemcpyDeviceToHost, st));
    int flag = 0;
    ACK(cudaMemcpyAsync(&flag, c->errflag, sizeof(int), cudaMemcpyDeviceToHost, st));
    ACK(cudaStreamSynchronize(st));
    if (flag) {
        cudaMemsetAsync(c->errflag, 0, sizeof(int), st);
        cudaStreamSynchronize(st);
        cleanup();
        return bgk_internal_fail(BGK_ERR_CUDA, "a bounded wait inside an adjoint or step kernel gave up; "
                                               "the gradient is invalid");
    }
    *loss = host[0];
    /* omega_g = 1/tau_g */
    const double tau_g = c->p.tau_g;
    *grad_tau_g = host[1] * (-1.0 / (tau_g * tau_g));
    cleanup();
#undef ACK
    return BGK_OK;
}
