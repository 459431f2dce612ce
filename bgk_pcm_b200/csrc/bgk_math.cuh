/*
 * bgk_math.cuh -- per-node formulas of the reference, written once in the
 * reference's evaluation order and shared by the fused and staged FP64
 * kernels (and by the host-side constant setup).
 *
 * Compiled into a translation unit built with --fmad=false, each expression
 * below is rounded operation by operation exactly as gfortran -O3 evaluates
 * the Fortran source on x86-64 (no fused multiply-add, left-to-right chains).
 */
#ifndef BGK_MATH_CUH
#define BGK_MATH_CUH

#include "bgk_internal.h"

#if defined(__CUDACC__)
#define BGK_HD __host__ __device__ __forceinline__
#else
#define BGK_HD inline
#endif

namespace bgk {

/* The initial condition of cell (i,j), 0 <= i <= Nx+1, 0 <= j <= Ny+1:
 * STEP_7/initialization.f90:15-26,45-47,137-151, with the heat bits selecting
 * the FROMRIGHT / FROMBOTTOM branches of STEP_DOCONCURRENT/initialization.f90
 * (:16-62 the liquid layer of T and rho, :122-137 the T buffer, :208-222 the
 * phi strip).  FROMBOTTOM's T buffer loop `do i = 0,Ny+1; T(i,0) = Tin` runs
 * along x and, with Ny > Nx, continues into row 1 of the column-major
 * array: it covers the first Ny+2 cells in memory. */
BGK_HD bool init_liquid(const Consts &c, int i, int j)
{
    if (c.heat & BGK_HEAT_BOTTOM) return j <= c.interf;
    if (c.heat & BGK_HEAT_RIGHT) return i >= c.Nx - c.interf + 1;
    return i <= c.interf;
}

BGK_HD double init_T(const Consts &c, int i, int j)
{
    const long long q = (long long)i + (long long)(c.Nx + 2) * j;
    const bool buffer = (c.heat & BGK_HEAT_BOTTOM) ? q <= (long long)c.Ny + 1
                      : (c.heat & BGK_HEAT_RIGHT) ? i == c.Nx + 1 : i == 0;
    return buffer ? c.Tin : (init_liquid(c, i, j) ? c.T0 : c.T_in_sol);
}

BGK_HD double init_rho(const Consts &c, int i, int j) { return init_liquid(c, i, j) ? c.rho1 : c.rho0; }

/* FROMRIGHT's phi strip starts one column left of its T strip */
BGK_HD double init_phi(const Consts &c, int i)
{
    return ((c.heat & BGK_HEAT_RIGHT) ? i >= c.Nx - c.interf : i <= c.interf) ? 1.0 : -1.0;
}

/* The nine equilibrium polynomials of STEP_7/collision.f90:19-27
 * (and initialization.f90:110-118, BC_g.f90:13-15,25-27): the factor that
 * multiplies w_k*rho (or w_k*T).  Note 4.5d0*upv*upv == (4.5*upv)*upv. */
BGK_HD void eq_poly(double u, double v, double *P)
{
    double uu = u * u;
    double vv = v * v;
    double uv = 1.5 * (uu + vv);
    double upv = u + v;
    double umv = u - v;
    P[0] = 1.0 - uv;
    P[1] = ((1.0 + 3.0 * u) + 4.5 * uu) - uv;
    P[2] = ((1.0 + 3.0 * v) + 4.5 * vv) - uv;
    P[3] = ((1.0 - 3.0 * u) + 4.5 * uu) - uv;
    P[4] = ((1.0 - 3.0 * v) + 4.5 * vv) - uv;
    P[5] = ((1.0 + 3.0 * upv) + (4.5 * upv) * upv) - uv;
    P[6] = ((1.0 - 3.0 * umv) + (4.5 * umv) * umv) - uv;
    P[7] = ((1.0 - 3.0 * upv) + (4.5 * upv) * upv) - uv;
    P[8] = ((1.0 + 3.0 * umv) + (4.5 * umv) * umv) - uv;
}

/* Regularized BGK for one distribution (STEP_7/collision.f90:42-150):
 * in = streamed populations, eq = equilibria, out = post-collision. */
template <bool REF32 = true>
BGK_HD void regularize_relax(const Consts &c, const double *in, const double *eq,
                             double omega, double *out)
{
    const double m = c.m_cs2, q = c.q_cs2;
    double d0 = in[0] - eq[0], d1 = in[1] - eq[1], d2 = in[2] - eq[2];
    double d3 = in[3] - eq[3], d4 = in[4] - eq[4], d5 = in[5] - eq[5];
    double d6 = in[6] - eq[6], d7 = in[7] - eq[7], d8 = in[8] - eq[8];
    double pxx = m * d0 + q * d1 + m * d2 + q * d3 + m * d4
               + q * d5 + q * d6 + q * d7 + q * d8;
    double pyy = m * d0 + m * d1 + q * d2 + m * d3 + q * d4
               + q * d5 + q * d6 + q * d7 + q * d8;
    double pxy = ((d5 - d6) + d7) - d8;
    double mxx = m * pxx, qxx = q * pxx, myy = m * pyy, qyy = q * pyy;
    double tp = 2.0 * pxy;
    double s0 = mxx + myy;
    double s1 = qxx + myy;
    double s2 = mxx + qyy;
    double sqq = qxx + qyy;
    double s5 = sqq + tp;
    double s6 = sqq - tp;
    /* ft0..ft8 / gt0..gt8 are undeclared in collision.f90, hence implicit
     * REAL(4): the regularized population is rounded to float, then the
     * relaxation is evaluated in double with it (REF32; the smooth form
     * keeps it in double). */
    double ft0 = eq[0] + c.C[0] * s0;
    if (REF32) ft0 = (double)(float)ft0;
    double ft1 = eq[1] + c.C[1] * s1;
    if (REF32) ft1 = (double)(float)ft1;
    double ft2 = eq[2] + c.C[2] * s2;
    if (REF32) ft2 = (double)(float)ft2;
    double ft3 = eq[3] + c.C[3] * s1;
    if (REF32) ft3 = (double)(float)ft3;
    double ft4 = eq[4] + c.C[4] * s2;
    if (REF32) ft4 = (double)(float)ft4;
    double ft5 = eq[5] + c.C[5] * s5;
    if (REF32) ft5 = (double)(float)ft5;
    double ft6 = eq[6] + c.C[6] * s6;
    if (REF32) ft6 = (double)(float)ft6;
    double ft7 = eq[7] + c.C[7] * s5;
    if (REF32) ft7 = (double)(float)ft7;
    double ft8 = eq[8] + c.C[8] * s6;
    if (REF32) ft8 = (double)(float)ft8;
    out[0] = ft0 - omega * (ft0 - eq[0]);
    out[1] = ft1 - omega * (ft1 - eq[1]);
    out[2] = ft2 - omega * (ft2 - eq[2]);
    out[3] = ft3 - omega * (ft3 - eq[3]);
    out[4] = ft4 - omega * (ft4 - eq[4]);
    out[5] = ft5 - omega * (ft5 - eq[5]);
    out[6] = ft6 - omega * (ft6 - eq[6]);
    out[7] = ft7 - omega * (ft7 - eq[7]);
    out[8] = ft8 - omega * (ft8 - eq[8]);
}

/* Sum of nine populations, left to right (momentsPre.f90:8-11). */
BGK_HD double sum9(const double *a)
{
    return a[0] + a[1] + a[2] + a[3] + a[4] + a[5] + a[6] + a[7] + a[8];
}
BGK_HD double xmom(const double *a) { return a[1] - a[3] + a[5] - a[6] - a[7] + a[8]; }
BGK_HD double ymom(const double *a) { return a[2] - a[4] + a[5] + a[6] - a[7] - a[8]; }

/* Phase-field selector terms (phase_field.f90:22-42): (0.5*(1 +/- phi))**2. */
BGK_HD double aplus(double p) { double t = 0.5 * (1.0 + p); return t * t; }
BGK_HD double aminus(double p) { double t = 0.5 * (1.0 - p); return t * t; }

/* phase_field.f90:44-48 given the two 3x3 sums and the tanh value. */
BGK_HD double phi_update(const Consts &c, double kp, double km, double th, double p0)
{
    double react_plus = 0.5 * (1.0 + th);
    double react_minus = 0.5 * (1.0 - th);
    kp = (kp / 8.0) * react_plus;
    km = (km / 8.0) * react_minus;
    return p0 + (c.f_plus * kp * (1.0 - p0) - c.f_minus * km * (1.0 + p0));
}

/* x / y for y > 0, skipping the division when x is a zero: 0 / y is that
 * zero with its sign, bit for bit.  Where the liquid fraction is 1 (and
 * wherever u is exactly 0, as in the symmetric bulk of the cavity) the drag
 * numerator is +-0; on B200 a warp whose lanes divide zeros runs the
 * division measurably slower, so those lanes sit the division out. */
BGK_HD double div_pos(double x, double y) { return x == 0.0 ? x : x / y; }

/* forces.f90:15-27: latent heat on T, buoyancy + drag, velocity shift. */
BGK_HD void apply_forces(const Consts &c, double phi, double phip, double rho,
                         double &T, double &u, double &v)
{
    T = T - (c.dts * (phi - phip) / 2.0);
    double forceY = rho * c.grav * c.beta * T * (1.0 + phi / 2.0);
    double forceX = -(u * (1.0 - phi) * 0.5);
    forceY = forceY - v * (1.0 - phi) * 0.5;
    /* omega_f * rho > 0 (rho is a sum of positive populations) */
    u = u + div_pos(forceX, c.omega_f * rho);
    v = v + div_pos(forceY, c.omega_f * rho);
}

} // namespace bgk
#endif
