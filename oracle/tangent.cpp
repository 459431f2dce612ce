/*
 * tangent.cpp -- forward-mode (tangent) derivative of the reference's time
 * step, for checking the adjoint.  TEST INFRASTRUCTURE ONLY.
 *
 * The STEP_7 routines on the no-slip cavity (BC_f code 4, BC_g,
 * streaming, momentsPre, phase_field, forces, collision, moments; files and
 * lines as cited in step7.c) are restated once more, templated on the
 * scalar type, in the smooth form (collision's ft/gt temporaries kept in
 * double, as bgk_options.smooth selects).  Instantiated with double it must
 * reproduce step7.c's smooth form bit for bit (checked by the tests);
 * instantiated with a dual number (value, derivative) it propagates the
 * derivative along one direction of the parameters: the per-row hot-wall
 * temperatures Tin[j] and tau_g.  tanh' = 1 - tanh^2.
 */
#include <cmath>
#include <cstddef>
#include <cstring>
#include <vector>

#include "step7.h"

namespace {

struct Dual {
    double v, d;
    Dual(double a = 0.0, double b = 0.0) : v(a), d(b) {}
};
inline Dual operator+(Dual a, Dual b) { return {a.v + b.v, a.d + b.d}; }
inline Dual operator-(Dual a, Dual b) { return {a.v - b.v, a.d - b.d}; }
inline Dual operator-(Dual a) { return {-a.v, -a.d}; }
inline Dual operator*(Dual a, Dual b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }
inline Dual operator/(Dual a, Dual b) { return {a.v / b.v, (a.d * b.v - a.v * b.d) / (b.v * b.v)}; }
inline Dual tanh_(Dual a)
{
    double t = std::tanh(a.v);
    return {t, (1.0 - t * t) * a.d};
}
inline double tanh_(double a) { return std::tanh(a); }
inline double val(double a) { return a; }
inline double val(Dual a) { return a.v; }

template <typename T>
struct State {
    int Nx, Ny, NX2;
    std::vector<T> f[9], g[9], fp[9], gp[9];
    std::vector<T> rho, TT, u, v, phi, phip, T2, u2, v2;
    T omega_f, omega_g, tau_g;
    std::vector<T> tin;                 /* rows 1..Ny at index j */
    double w[9], cs2, grav, rho0, rho1, T0, T_in_sol, stefan, T_width;
    size_t ix(int i, int j) const { return (size_t)i + (size_t)NX2 * (size_t)j; }
};

template <typename T>
void eq9(const double *w, T r, T u, T v, T *e)
{
    T uu = u * u, vv = v * v;
    T uv = T(1.5) * (uu + vv);
    T upv = u + v, umv = u - v;
    e[0] = T(w[0]) * r * (T(1.0) - uv);
    e[1] = T(w[1]) * r * (T(1.0) + T(3.0) * u + T(4.5) * uu - uv);
    e[2] = T(w[2]) * r * (T(1.0) + T(3.0) * v + T(4.5) * vv - uv);
    e[3] = T(w[3]) * r * (T(1.0) - T(3.0) * u + T(4.5) * uu - uv);
    e[4] = T(w[4]) * r * (T(1.0) - T(3.0) * v + T(4.5) * vv - uv);
    e[5] = T(w[5]) * r * (T(1.0) + T(3.0) * upv + T(4.5) * upv * upv - uv);
    e[6] = T(w[6]) * r * (T(1.0) - T(3.0) * umv + T(4.5) * umv * umv - uv);
    e[7] = T(w[7]) * r * (T(1.0) - T(3.0) * upv + T(4.5) * upv * upv - uv);
    e[8] = T(w[8]) * r * (T(1.0) + T(3.0) * umv + T(4.5) * umv * umv - uv);
}

/* STEP_7/initialization.f90 (Re = 0: u = v = 0) */
template <typename T>
void init(State<T> &s, const orc_params &p)
{
    s.Nx = p.Nx; s.Ny = p.Ny; s.NX2 = p.Nx + 2;
    const size_t A = (size_t)(p.Nx + 2) * (p.Ny + 2);
    for (int k = 0; k < 9; k++) { s.f[k].assign(A, T(0)); s.g[k].assign(A, T(0)); s.fp[k].assign(A, T(0)); s.gp[k].assign(A, T(0)); }
    for (auto *a : {&s.rho, &s.TT, &s.u, &s.v, &s.phi, &s.phip, &s.T2, &s.u2, &s.v2}) a->assign(A, T(0));
    s.w[0] = 4.0 / 9.0;
    for (int k = 1; k <= 4; k++) s.w[k] = 1.0 / 9.0;
    for (int k = 5; k <= 8; k++) s.w[k] = 1.0 / 36.0;
    s.cs2 = 1.0 / 3.0;
    s.grav = p.grav; s.rho0 = p.rho0; s.rho1 = p.rho1; s.T0 = p.T0; s.T_in_sol = p.T_in_sol;
    s.stefan = p.stefan_number; s.T_width = p.T_width;
    s.omega_f = T(1.0 / p.tau_f);
    const int interf = p.Nx / 40;
    for (int j = 0; j <= p.Ny + 1; j++)
        for (int i = 0; i <= p.Nx + 1; i++) {
            size_t q = s.ix(i, j);
            s.TT[q] = T(i <= interf ? p.T0 : p.T_in_sol);
            s.rho[q] = T(i <= interf ? p.rho1 : p.rho0);
            if (i == 0) s.TT[q] = T(p.T0);
            T e[9];
            eq9(s.w, s.rho[q], T(0), T(0), e);
            for (int k = 0; k < 9; k++) s.f[k][q] = e[k];
            eq9(s.w, s.TT[q], T(0), T(0), e);
            for (int k = 0; k < 9; k++) s.g[k][q] = e[k];
            s.phi[q] = T(i <= interf ? 1.0 : -1.0);
            s.phip[q] = s.phi[q];
        }
}

template <typename T>
void step(State<T> &s)
{
    const int Nx = s.Nx, Ny = s.Ny;
    auto &f = s.f; auto &g = s.g; auto &fp = s.fp; auto &gp = s.gp;
    /* BC_f code 4 (STEP_7/BC_f.f90:62-68,101-107,125-136,181-192) */
    for (int j = 1; j <= Ny; j++) {
        f[1][s.ix(0, j)] = f[3][s.ix(1, j)];
        f[8][s.ix(0, j)] = f[6][s.ix(1, j - 1)];
        f[5][s.ix(0, j)] = f[7][s.ix(1, j + 1)];
    }
    for (int j = 1; j <= Ny; j++) {
        f[3][s.ix(Nx + 1, j)] = f[1][s.ix(Nx, j)];
        f[6][s.ix(Nx + 1, j)] = f[8][s.ix(Nx, j + 1)];
        f[7][s.ix(Nx + 1, j)] = f[5][s.ix(Nx, j - 1)];
    }
    for (int i = 1; i <= Nx; i++) {
        f[4][s.ix(i, Ny + 1)] = f[2][s.ix(i, Ny)];
        f[7][s.ix(i, Ny + 1)] = f[5][s.ix(i - 1, Ny)];
        f[8][s.ix(i, Ny + 1)] = f[6][s.ix(i + 1, Ny)];
    }
    f[8][s.ix(0, Ny + 1)] = f[6][s.ix(1, Ny)];
    for (int i = 1; i <= Nx; i++) {
        f[2][s.ix(i, 0)] = f[4][s.ix(i, 1)];
        f[5][s.ix(i, 0)] = f[7][s.ix(i + 1, 1)];
        f[6][s.ix(i, 0)] = f[8][s.ix(i - 1, 1)];
    }
    f[5][s.ix(0, 0)] = f[7][s.ix(1, 1)];
    /* BC_g (STEP_7/BC_g.f90:7-64), u = v = 0 on the walls */
    for (int j = 1; j <= Ny; j++) {
        T e[9];
        eq9(s.w, s.tin[j], T(0), T(0), e);
        g[1][s.ix(0, j)] = e[1]; g[5][s.ix(0, j)] = e[5]; g[8][s.ix(0, j)] = e[8];
    }
    for (int j = 1; j <= Ny; j++) {
        T e[9];
        eq9(s.w, s.TT[s.ix(Nx, j)], T(0), T(0), e);
        g[3][s.ix(Nx + 1, j)] = e[3]; g[6][s.ix(Nx + 1, j)] = e[6]; g[7][s.ix(Nx + 1, j)] = e[7];
    }
    for (int i = 0; i <= Nx + 1; i++) {
        for (int k = 0; k < 9; k++) g[k][s.ix(i, Ny + 1)] = g[k][s.ix(i, Ny)];
        s.phi[s.ix(i, Ny + 1)] = s.phi[s.ix(i, Ny)];
    }
    for (int i = 0; i <= Nx + 1; i++) {
        for (int k = 0; k < 9; k++) g[k][s.ix(i, 0)] = g[k][s.ix(i, 1)];
        s.phi[s.ix(i, 0)] = s.phi[s.ix(i, 1)];
    }
    /* streaming (STEP_7/streaming.f90:5-27) */
    static const int cx[9] = {0, 1, 0, -1, 0, 1, -1, -1, 1}, cy[9] = {0, 0, 1, 0, -1, 1, 1, -1, -1};
    for (int j = 1; j <= Ny; j++)
        for (int i = 1; i <= Nx; i++)
            for (int k = 0; k < 9; k++) {
                fp[k][s.ix(i, j)] = f[k][s.ix(i - cx[k], j - cy[k])];
                gp[k][s.ix(i, j)] = g[k][s.ix(i - cx[k], j - cy[k])];
            }
    /* momentsPre (STEP_7/momentsPre.f90:5-23) */
    for (int j = 1; j <= Ny; j++)
        for (int i = 1; i <= Nx; i++) {
            size_t q = s.ix(i, j);
            T r = fp[0][q] + fp[1][q] + fp[2][q] + fp[3][q] + fp[4][q] + fp[5][q] + fp[6][q] + fp[7][q] + fp[8][q];
            T t = gp[0][q] + gp[1][q] + gp[2][q] + gp[3][q] + gp[4][q] + gp[5][q] + gp[6][q] + gp[7][q] + gp[8][q];
            T ir = T(1.0) / r;
            s.rho[q] = r; s.TT[q] = t;
            s.u[q] = ir * (fp[1][q] - fp[3][q] + fp[5][q] - fp[6][q] - fp[7][q] + fp[8][q]);
            s.v[q] = ir * (fp[2][q] - fp[4][q] + fp[5][q] + fp[6][q] - fp[7][q] - fp[8][q]);
            s.T2[q] = t; s.u2[q] = s.u[q]; s.v2[q] = s.v[q];
        }
    /* phase_field (STEP_7/phase_field.f90:11-52) */
    s.phip = s.phi;
    for (int j = 1; j <= Ny; j++)
        for (int i = 1; i <= Nx; i++) {
            size_t q = s.ix(i, j);
            T th = tanh_(((s.TT[q] - T(273.0)) - T(0.0)) / T(s.T_width));
            T rp = T(0.5) * (T(1.0) + th), rm = T(0.5) * (T(1.0) - th);
            const int di[9] = {0, 1, 0, -1, 0, 1, -1, -1, 1}, dj[9] = {0, 0, 1, 0, -1, 1, 1, -1, -1};
            T kp(0.0), km(0.0);
            for (int a = 0; a < 9; a++) {
                T pp = s.phip[s.ix(i + di[a], j + dj[a])];
                T x = T(0.5) * (T(1.0) + pp), y = T(0.5) * (T(1.0) - pp);
                kp = (a == 0) ? x * x : kp + x * x;
                km = (a == 0) ? y * y : km + y * y;
            }
            kp = (kp / T(8.0)) * rp;
            km = (km / T(8.0)) * rm;
            T p0 = s.phip[q];
            s.phi[q] = p0 + (T(0.5) * kp * (T(1.0) - p0) - T(0.5) * km * (T(1.0) + p0));
        }
    /* forces (STEP_7/forces.f90:12-28); beta is REAL(4) */
    const double dT = s.T0 - s.T_in_sol;
    const double beta = (double)(float)((1.0 - s.rho1 / s.rho0) / dT);
    for (int j = 1; j <= Ny; j++)
        for (int i = 1; i <= Nx; i++) {
            size_t q = s.ix(i, j);
            T ph = s.phi[q], pp = s.phip[q], r = s.rho[q];
            T t = s.TT[q] - (T(dT / s.stefan) * (ph - pp) / T(2.0));
            s.TT[q] = t;
            T fy = r * T(s.grav) * T(beta) * t * (T(1.0) + ph / T(2.0));
            T fx = -(s.u[q] * (T(1.0) - ph) * T(0.5));
            fy = fy - s.v[q] * (T(1.0) - ph) * T(0.5);
            s.u[q] = s.u[q] + fx / (s.omega_f * r);
            s.v[q] = s.v[q] + fy / (s.omega_f * r);
        }
    /* collision (STEP_7/collision.f90:14-152), smooth form */
    const T m(-s.cs2), q1(1.0 - s.cs2);
    T C[9];
    for (int k = 0; k < 9; k++) C[k] = T((0.5 * s.w[k]) / (s.cs2 * s.cs2));
    for (int j = 1; j <= Ny; j++)
        for (int i = 1; i <= Nx; i++) {
            size_t q = s.ix(i, j);
            T fe[9], ge[9], d[9], e[9];
            eq9(s.w, s.rho[q], s.u[q], s.v[q], fe);
            eq9(s.w, s.TT[q], s.u[q], s.v[q], ge);
            for (int k = 0; k < 9; k++) { d[k] = fp[k][q] - fe[k]; e[k] = gp[k][q] - ge[k]; }
            T pxx = m * d[0] + q1 * d[1] + m * d[2] + q1 * d[3] + m * d[4] + q1 * d[5] + q1 * d[6] + q1 * d[7] + q1 * d[8];
            T pyy = m * d[0] + m * d[1] + q1 * d[2] + m * d[3] + q1 * d[4] + q1 * d[5] + q1 * d[6] + q1 * d[7] + q1 * d[8];
            T pxy = d[5] - d[6] + d[7] - d[8];
            T txx = m * e[0] + q1 * e[1] + m * e[2] + q1 * e[3] + m * e[4] + q1 * e[5] + q1 * e[6] + q1 * e[7] + q1 * e[8];
            T tyy = m * e[0] + m * e[1] + q1 * e[2] + m * e[3] + q1 * e[4] + q1 * e[5] + q1 * e[6] + q1 * e[7] + q1 * e[8];
            T txy = e[5] - e[6] + e[7] - e[8];
            T S[9], Sg[9];
            S[0] = m * pxx + m * pyy; S[1] = q1 * pxx + m * pyy; S[2] = m * pxx + q1 * pyy;
            S[3] = q1 * pxx + m * pyy; S[4] = m * pxx + q1 * pyy;
            S[5] = q1 * pxx + q1 * pyy + T(2.0) * pxy; S[6] = q1 * pxx + q1 * pyy - T(2.0) * pxy;
            S[7] = q1 * pxx + q1 * pyy + T(2.0) * pxy; S[8] = q1 * pxx + q1 * pyy - T(2.0) * pxy;
            Sg[0] = m * txx + m * tyy; Sg[1] = q1 * txx + m * tyy; Sg[2] = m * txx + q1 * tyy;
            Sg[3] = q1 * txx + m * tyy; Sg[4] = m * txx + q1 * tyy;
            Sg[5] = q1 * txx + q1 * tyy + T(2.0) * txy; Sg[6] = q1 * txx + q1 * tyy - T(2.0) * txy;
            Sg[7] = q1 * txx + q1 * tyy + T(2.0) * txy; Sg[8] = q1 * txx + q1 * tyy - T(2.0) * txy;
            for (int k = 0; k < 9; k++) {
                T ft = fe[k] + C[k] * S[k];
                T gt = ge[k] + C[k] * Sg[k];
                f[k][q] = ft - s.omega_f * (ft - fe[k]);
                g[k][q] = gt - s.omega_g * (gt - ge[k]);
            }
        }
    /* moments (STEP_7/moments.f90:8-27) */
    for (int j = 1; j <= Ny; j++)
        for (int i = 1; i <= Nx; i++) {
            size_t q = s.ix(i, j);
            T r = f[0][q] + f[1][q] + f[2][q] + f[3][q] + f[4][q] + f[5][q] + f[6][q] + f[7][q] + f[8][q];
            T ir = T(1.0) / r;
            T t = g[0][q] + g[1][q] + g[2][q] + g[3][q] + g[4][q] + g[5][q] + g[6][q] + g[7][q] + g[8][q];
            T tu = ir * (f[1][q] - f[3][q] + f[5][q] - f[6][q] - f[7][q] + f[8][q]);
            T tv = ir * (f[2][q] - f[4][q] + f[5][q] + f[6][q] - f[7][q] - f[8][q]);
            s.rho[q] = r;
            s.TT[q] = (t + s.T2[q]) * T(0.5);
            s.u[q] = (tu + s.u2[q]) * T(0.5);
            s.v[q] = (tv + s.v2[q]) * T(0.5);
        }
}

} // namespace

extern "C" {

/* Loss sum_p (phi(i_p,j_p) - target_p)^2 after nsteps steps of the
 * no-slip cavity from the initial condition, with hot-wall temperatures
 * tin[j-1] (j = 1..Ny) and tau_g; dloss = its derivative along (dtin,
 * dtau_g).  phi_out (optional, (Nx+2)(Ny+2)) receives the final phi. */
int orc_tangent_loss(const orc_params *p, const double *tin, const double *dtin, double dtau_g, int nsteps,
                     int np, const int *pi, const int *pj, const double *target, double *loss, double *dloss,
                     double *phi_out)
{
    if (p->westBC != 4 || p->eastBC != 4 || p->northBC != 4 || p->southBC != 4 || p->Re != 0.0) return -1;
    State<Dual> s;
    init(s, *p);
    s.tin.assign((size_t)p->Ny + 2, Dual(0.0));
    for (int j = 1; j <= p->Ny; j++) s.tin[j] = Dual(tin[j - 1], dtin ? dtin[j - 1] : 0.0);
    Dual tau(p->tau_g, dtau_g);
    s.omega_g = Dual(1.0) / tau;
    for (int n = 0; n < nsteps; n++) step(s);
    Dual L(0.0);
    for (int a = 0; a < np; a++) {
        Dual r = s.phi[s.ix(pi[a], pj[a])] - Dual(target[a]);
        L = L + r * r;
    }
    *loss = L.v;
    *dloss = L.d;
    if (phi_out)
        for (size_t q = 0; q < s.phi.size(); q++) phi_out[q] = s.phi[q].v;
    return 0;
}

/* The same restatement in plain double (its values must equal step7.c's
 * smooth form with the same per-row Tin). */
int orc_tangent_plain(const orc_params *p, const double *tin, int nsteps, double *phi_out, double *T_out)
{
    State<double> s;
    init(s, *p);
    s.tin.assign((size_t)p->Ny + 2, 0.0);
    for (int j = 1; j <= p->Ny; j++) s.tin[j] = tin[j - 1];
    s.omega_g = 1.0 / p->tau_g;
    for (int n = 0; n < nsteps; n++) step(s);
    memcpy(phi_out, s.phi.data(), s.phi.size() * sizeof(double));
    memcpy(T_out, s.TT.data(), s.TT.size() * sizeof(double));
    return 0;
}

} // extern "C"
