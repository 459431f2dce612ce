/*
 * kernels_f64.cu -- FP64 kernels in the reference's exact operation order.
 * Built with --fmad=false so no multiply-add is contracted (the reference is
 * compiled by gfortran -O3 for generic x86-64, which has no FMA).
 *
 *  - init_kernel            STEP_7/initialization.f90:5-152
 *  - bc_prep_kernel         per-row boundary values for the fused step
 *                           (STEP_7/BC_g.f90:7-31 west/east terms, frozen phi
 *                           columns)
 *  - macro_halo_kernel      the halo assignments of STEP_7/BC_f.f90 (code 4)
 *                           and STEP_7/BC_g.f90 that touch rho, u, v, T, phi
 *  - fused_f64_kernel       one whole time step (STEP_7/main.f90:60-69)
 *  - staged_*               one kernel per reference subroutine
 *  - conversions between the compact state and the reference layout
 *  - field_sums_kernel      FP64 interior reductions (field_check / diag)
 */
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

struct Staged {
    double *f[9], *g[9], *fp[9], *gp[9];
    double *rho, *T, *u, *v, *phi, *phip, *rho2, *T2, *u2, *v2;
    const double *tin;
};

/* ------------------------------------------------------------------ init */

/* STEP_7/initialization.f90:15-152, one thread per reference cell
 * (i,j) in 0..Nx+1 x 0..Ny+1.  Writes the mirrors (rho,T,u,v,phi with halos),
 * the compact populations (interior) or the staged arrays, and phi twice
 * (phi and phi_prec are equal after initialization).  The heat bits select
 * STEP_DOCONCURRENT/initialization.f90's FROMRIGHT / FROMBOTTOM branches
 * (:16-62 T/rho, :122-137 T buffer, :208-222 phi). */
__global__ void init_kernel(Consts c, int westBC, StepPtrs<double> s, double *fcomp, double *gcomp,
                            double *phc0, double *phc1, Staged st, bool staged, double *corner, double *tcol,
                            double *ring, long long RL)
{
    const int NX2 = c.Nx + 2, NY2 = c.Ny + 2;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= NX2 || j >= NY2) return;
    const int Nx = c.Nx, Ny = c.Ny;
    const double T = init_T(c, i, j);
    double rho = init_rho(c, i, j);
    double u = c.u0, v = c.v0;
    const size_t q = (size_t)i + (size_t)NX2 * (size_t)j;
    if (j == 0 || j == Ny + 1) { u = 0.0; v = 0.0; }
    if (westBC == 3) {
        u = 0.0; v = 0.0;
        if (i == 0) rho = c.rho1;
    }
    if (i == 0 && j >= 1 && j <= Ny) {
        if (westBC == 1) { u = c.u0; v = c.v0; }
        else if (westBC == 2) {
            double ny1 = (double)(Ny + 1);
            double yj = (double)j;
            u = -(6.0 * c.u0 / (ny1 * ny1)) * (yj * yj - ny1 * yj);
            v = c.v0;
        }
    }
    double P[9];
    eq_poly(u, v, P);
    const double phi = init_phi(c, i);
    s.mrho[q] = rho; s.mT[q] = T; s.mu[q] = u; s.mv[q] = v; s.mphi[q] = phi;
    double fe[9], ge[9];
    for (int k = 0; k < 9; k++) { fe[k] = c.w[k] * rho * P[k]; ge[k] = c.w[k] * T * P[k]; }
    if (staged) {
        for (int k = 0; k < 9; k++) { st.f[k][q] = fe[k]; st.g[k][q] = ge[k]; }
        st.phip[q] = phi;
    }
    if (fcomp && i >= 1 && i <= Nx && j >= 1 && j <= Ny) {
        const long long cc = (long long)(j - 1) * s.P + (i - 1);
        for (int k = 0; k < 9; k++) {
            fcomp[k * s.plane + cc] = fe[k];
            gcomp[k * s.plane + cc] = ge[k];
        }
        phc0[cc] = phi;
        phc1[cc] = phi;
    }
    if (i == Nx + 1 && j == 0) corner[0] = fe[6];
    if (i == Nx + 1 && j == Ny + 1) corner[1] = fe[7];
    if (i == Nx && j >= 1 && j <= Ny) tcol[j - 1] = T;
    if (ring && (i == 0 || i == Nx + 1 || j == 0 || j == Ny + 1))
        for (int k = 0; k < 9; k++) ring[k * RL + ring_idx(Nx, Ny, i, j)] = fe[k];
}

/* ------------------------------------------------------- boundary prep */

/* West g values (BC_g.f90:7-17) per row, the east equilibrium polynomials
 * (BC_g.f90:21-31: g_k(Nx+1,j) = w_k*T(Nx,j)*poly_k(u(Nx+1,j),v(Nx+1,j))),
 * and the frozen phi columns.  tin = per-row hot wall or null (scalar).
 * With BGK_HEAT_RIGHT (STEP_DOCONCURRENT/BC_g.f90:13-17) the west values are
 * w_k*T(1,j)*poly of directions 3, 7, 6, T(1,j) being the previous step's
 * (the T mirror, which the ring step writes at edge nodes every step); this
 * then runs before every step. */
__device__ __forceinline__ void bc_prep_row(const Consts &c, const double *mu, const double *mv,
                                            const double *mphi, const double *mT, const double *tin, double *gW,
                                            double *pE, double *phiW, double *phiE, int j)
{
    const int Ny = c.Ny, NX2 = c.Nx + 2;
    double P[9];
    const size_t qw = (size_t)NX2 * j, qe = (size_t)(c.Nx + 1) + (size_t)NX2 * j;
    eq_poly(mu[qw], mv[qw], P);
    if (c.heat & BGK_HEAT_RIGHT) {
        const double T1 = mT[qw + 1];
        gW[0 * Ny + j - 1] = c.w[1] * T1 * P[3];
        gW[1 * Ny + j - 1] = c.w[5] * T1 * P[7];
        gW[2 * Ny + j - 1] = c.w[8] * T1 * P[6];
    } else {
        const double Tin = tin ? tin[j - 1] : c.Tin;
        gW[0 * Ny + j - 1] = c.w[1] * Tin * P[1];
        gW[1 * Ny + j - 1] = c.w[5] * Tin * P[5];
        gW[2 * Ny + j - 1] = c.w[8] * Tin * P[8];
    }
    eq_poly(mu[qe], mv[qe], P);
    pE[0 * Ny + j - 1] = P[3];
    pE[1 * Ny + j - 1] = P[6];
    pE[2 * Ny + j - 1] = P[7];
    phiW[j - 1] = mphi[qw];
    phiE[j - 1] = mphi[qe];
}

__global__ void bc_prep_kernel(Consts c, const double *mu, const double *mv, const double *mphi,
                               const double *mT, const double *tin, double *gW, double *pE, double *phiW,
                               double *phiE)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x + 1;
    if (j > c.Ny) return;
    bc_prep_row(c, mu, mv, mphi, mT, tin, gW, pE, phiW, phiE, j);
}

/* Halo cells between population rings and reference-layout arrays (pitch
 * Nx+2): block row y copies population k0 + y to or from refs.p[y]
 * (to_ring: ref -> ring, else ring -> ref). */
struct Ptr9 {
    double *p[9];
};

__global__ void ring_ref_copy(int Nx, int Ny, double *ring, long long RL, Ptr9 refs, int k0, bool to_ring)
{
    const long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (r >= RL) return;
    const int k = k0 + blockIdx.y;
    int i, j;
    if (r < Ny + 2) { i = 0; j = (int)r; }
    else if (r < 2LL * (Ny + 2)) { i = Nx + 1; j = (int)(r - (Ny + 2)); }
    else if (r < 2LL * (Ny + 2) + Nx) { i = (int)(r - 2LL * (Ny + 2)) + 1; j = 0; }
    else { i = (int)(r - 2LL * (Ny + 2) - Nx) + 1; j = Ny + 1; }
    double *ref = refs.p[blockIdx.y];
    const size_t q = (size_t)i + (size_t)(Nx + 2) * (size_t)j;
    if (to_ring) ring[k * RL + r] = ref[q];
    else ref[q] = ring[k * RL + r];
}

/* ------------------------------------------------------ macroscopic halos */

/* The assignments of BC_f (code 4 north/south: rho copy, u=v=0;
 * STEP_7/BC_f.f90:125-134,181-190) and of BC_g (T west/east, then T and phi
 * north/south copies; STEP_7/BC_g.f90:7-64) on the mirrors, which hold the
 * previous step's moments.  One block: west/east first, then north/south. */
__global__ void macro_halo_kernel(Consts c, double *rho, double *T, double *u, double *v,
                                  double *phi, const double *tin)
{
    const int Nx = c.Nx, Ny = c.Ny, NX2 = Nx + 2;
#define Q(i, j) ((size_t)(i) + (size_t)NX2 * (size_t)(j))
    for (int i = 1 + threadIdx.x; i <= Nx; i += blockDim.x) {
        rho[Q(i, Ny + 1)] = rho[Q(i, Ny)];
        u[Q(i, Ny + 1)] = 0.0; v[Q(i, Ny + 1)] = 0.0;
        rho[Q(i, 0)] = rho[Q(i, 1)];
        u[Q(i, 0)] = 0.0; v[Q(i, 0)] = 0.0;
    }
    for (int j = 1 + threadIdx.x; j <= Ny; j += blockDim.x) {
        T[Q(0, j)] = tin ? tin[j - 1] : c.Tin;
        T[Q(Nx + 1, j)] = T[Q(Nx, j)];
    }
    __syncthreads();
    for (int i = threadIdx.x; i <= Nx + 1; i += blockDim.x) {
        T[Q(i, Ny + 1)] = T[Q(i, Ny)];
        phi[Q(i, Ny + 1)] = phi[Q(i, Ny)];
        T[Q(i, 0)] = T[Q(i, 1)];
        phi[Q(i, 0)] = phi[Q(i, 1)];
    }
#undef Q
}

#include "fused_f64.cuh"
#include "fused_pipe.cuh"

/* --------------------------------------------------------- staged kernels */

#define SQ(i, j) ((size_t)(i) + (size_t)NX2 * (size_t)(j))

/* STEP_7/BC_f.f90:5-200, every branch, west, east, north, south in order. */
__global__ void staged_bc_f(Staged s, Consts c, int wbc, int ebc, int nbc, int sbc)
{
    const int Nx = c.Nx, Ny = c.Ny, NX2 = Nx + 2;
    const double *w = c.w;
    const int t0 = threadIdx.x, nt = blockDim.x;
    double P[9];
    /* WEST */
    if (wbc == 0) {
        for (int j = t0; j <= Ny + 1; j += nt)
            for (int k = 0; k < 9; k++) s.f[k][SQ(0, j)] = s.f[k][SQ(Nx, j)];
    } else if (wbc == 1) {
        eq_poly(c.u0, c.v0, P);
        for (int j = 1 + t0; j <= Ny; j += nt) {
            double r = s.rho[SQ(1, j)];
            s.f[1][SQ(0, j)] = w[1] * r * P[1];
            s.f[5][SQ(0, j)] = w[5] * r * P[5];
            s.f[8][SQ(0, j)] = w[8] * r * P[8];
            s.u[SQ(0, j)] = c.u0;
            s.v[SQ(0, j)] = c.v0;
            s.rho[SQ(0, j)] = s.rho[SQ(1, j)];
        }
    } else if (wbc == 2) {
        for (int j = t0; j <= Ny + 1; j += nt) {
            eq_poly(s.u[SQ(0, j)], c.v0, P);
            double r = s.rho[SQ(1, j)];
            s.f[1][SQ(0, j)] = w[1] * r * P[1];
            s.f[5][SQ(0, j)] = w[5] * r * P[5];
            s.f[8][SQ(0, j)] = w[8] * r * P[8];
        }
    } else if (wbc == 3) {
        for (int j = t0; j <= Ny + 1; j += nt) {
            double u1 = s.u[SQ(1, j)], v1 = s.v[SQ(1, j)];
            eq_poly(u1, v1, P);
            s.f[1][SQ(0, j)] = w[1] * c.rho1 * P[1];
            s.f[5][SQ(0, j)] = w[5] * c.rho1 * P[5];
            s.f[8][SQ(0, j)] = w[8] * c.rho1 * P[8];
            s.u[SQ(0, j)] = u1;
            s.v[SQ(0, j)] = v1;
            s.rho[SQ(0, j)] = c.rho1;
        }
    } else if (wbc == 4) {
        for (int j = 1 + t0; j <= Ny; j += nt) {
            s.f[1][SQ(0, j)] = s.f[3][SQ(1, j)];
            s.f[8][SQ(0, j)] = s.f[6][SQ(1, j - 1)];
            s.f[5][SQ(0, j)] = s.f[7][SQ(1, j + 1)];
        }
    }
    __syncthreads();
    /* EAST */
    if (ebc == 0) {
        for (int j = t0; j <= Ny + 1; j += nt)
            for (int k = 0; k < 9; k++) s.f[k][SQ(Nx + 1, j)] = s.f[k][SQ(1, j)];
    } else if (ebc == 3) {
        for (int j = 1 + t0; j <= Ny; j += nt) {
            double un = s.u[SQ(Nx, j)], vn = s.v[SQ(Nx, j)];
            eq_poly(un, vn, P);
            s.f[3][SQ(Nx + 1, j)] = w[3] * c.rho0 * P[3];
            s.f[6][SQ(Nx + 1, j)] = w[6] * c.rho0 * P[6];
            s.f[7][SQ(Nx + 1, j)] = w[7] * c.rho0 * P[7];
            s.u[SQ(Nx + 1, j)] = un;
            s.v[SQ(Nx + 1, j)] = vn;
            s.rho[SQ(Nx + 1, j)] = c.rho0;
        }
    } else if (ebc == 4) {
        for (int j = 1 + t0; j <= Ny; j += nt) {
            s.f[3][SQ(Nx + 1, j)] = s.f[1][SQ(Nx, j)];
            s.f[6][SQ(Nx + 1, j)] = s.f[8][SQ(Nx, j + 1)];
            s.f[7][SQ(Nx + 1, j)] = s.f[5][SQ(Nx, j - 1)];
        }
    }
    __syncthreads();
    /* NORTH */
    if (nbc == 0) {
        for (int i = t0; i <= Nx + 1; i += nt)
            for (int k = 0; k < 9; k++) s.f[k][SQ(i, Ny + 1)] = s.f[k][SQ(i, 1)];
    } else if (nbc == 4) {
        for (int i = 1 + t0; i <= Nx; i += nt) {
            s.f[4][SQ(i, Ny + 1)] = s.f[2][SQ(i, Ny)];
            s.f[7][SQ(i, Ny + 1)] = s.f[5][SQ(i - 1, Ny)];
            s.f[8][SQ(i, Ny + 1)] = s.f[6][SQ(i + 1, Ny)];
            s.rho[SQ(i, Ny + 1)] = s.rho[SQ(i, Ny)];
            s.u[SQ(i, Ny + 1)] = 0.0;
            s.v[SQ(i, Ny + 1)] = 0.0;
        }
        if (t0 == 0) s.f[8][SQ(0, Ny + 1)] = s.f[6][SQ(1, Ny)];
    } else if (nbc == 5) {
        for (int i = t0; i <= Nx + 1; i += nt) {
            s.f[4][SQ(i, Ny + 1)] = s.f[2][SQ(i, Ny - 1)];
            s.f[7][SQ(i, Ny + 1)] = s.f[6][SQ(i, Ny - 1)];
            s.f[8][SQ(i, Ny + 1)] = s.f[5][SQ(i, Ny - 1)];
        }
    } else if (nbc == 6) {
        for (int i = t0; i <= Nx + 1; i += nt) {
            s.f[4][SQ(i, Ny + 1)] = s.f[4][SQ(i, Ny)];
            s.f[7][SQ(i, Ny + 1)] = s.f[7][SQ(i, Ny)];
            s.f[8][SQ(i, Ny + 1)] = s.f[8][SQ(i, Ny)];
        }
    } else if (nbc == 1) {
        eq_poly(c.u0, c.v0, P);
        for (int i = t0; i <= Nx + 1; i += nt) {
            double r = s.rho[SQ(i, Ny)];
            s.f[4][SQ(i, Ny + 1)] = w[4] * r * P[4];
            s.f[7][SQ(i, Ny + 1)] = w[7] * r * P[7];
            s.f[8][SQ(i, Ny + 1)] = w[8] * r * P[8];
        }
    }
    __syncthreads();
    /* SOUTH */
    if (sbc == 0) {
        for (int i = t0; i <= Nx + 1; i += nt)
            for (int k = 0; k < 9; k++) s.f[k][SQ(i, 0)] = s.f[k][SQ(i, Ny)];
    } else if (sbc == 4) {
        for (int i = 1 + t0; i <= Nx; i += nt) {
            s.f[2][SQ(i, 0)] = s.f[4][SQ(i, 1)];
            s.f[5][SQ(i, 0)] = s.f[7][SQ(i + 1, 1)];
            s.f[6][SQ(i, 0)] = s.f[8][SQ(i - 1, 1)];
            s.rho[SQ(i, 0)] = s.rho[SQ(i, 1)];
            s.u[SQ(i, 0)] = 0.0;
            s.v[SQ(i, 0)] = 0.0;
        }
        if (t0 == 0) s.f[5][SQ(0, 0)] = s.f[7][SQ(1, 1)];
    } else if (sbc == 6) {
        for (int i = t0; i <= Nx + 1; i += nt) {
            s.f[2][SQ(i, 0)] = s.f[2][SQ(i, 1)];
            s.f[5][SQ(i, 0)] = s.f[5][SQ(i, 1)];
            s.f[6][SQ(i, 0)] = s.f[6][SQ(i, 1)];
        }
    }
}

/* STEP_7/BC_g.f90:5-64 */
__global__ void staged_bc_g(Staged s, Consts c)
{
    const int Nx = c.Nx, Ny = c.Ny, NX2 = Nx + 2;
    const double *w = c.w;
    double P[9];
    if (c.heat & BGK_HEAT_RIGHT) {
        /* STEP_DOCONCURRENT/BC_g.f90:13-17, 35-39 (FROMRIGHT) */
        for (int j = 1 + threadIdx.x; j <= Ny; j += blockDim.x) {
            eq_poly(s.u[SQ(0, j)], s.v[SQ(0, j)], P);
            const double t = s.T[SQ(1, j)];
            s.g[1][SQ(0, j)] = w[1] * t * P[3];
            s.g[5][SQ(0, j)] = w[5] * t * P[7];
            s.g[8][SQ(0, j)] = w[8] * t * P[6];
            s.T[SQ(0, j)] = s.T[SQ(1, j)];
        }
        for (int j = 1 + threadIdx.x; j <= Ny; j += blockDim.x) {
            eq_poly(s.u[SQ(Nx + 1, j)], s.v[SQ(Nx + 1, j)], P);
            s.g[3][SQ(Nx + 1, j)] = w[3] * c.Tin * P[3];
            s.g[6][SQ(Nx + 1, j)] = w[6] * c.Tin * P[6];
            s.g[7][SQ(Nx + 1, j)] = w[7] * c.Tin * P[7];
            s.T[SQ(Nx + 1, j)] = c.Tin;
        }
    }
    for (int j = 1 + threadIdx.x; j <= Ny && !(c.heat & BGK_HEAT_RIGHT); j += blockDim.x) {
        const double Tin = s.tin ? s.tin[j - 1] : c.Tin;
        eq_poly(s.u[SQ(0, j)], s.v[SQ(0, j)], P);
        s.g[1][SQ(0, j)] = w[1] * Tin * P[1];
        s.g[5][SQ(0, j)] = w[5] * Tin * P[5];
        s.g[8][SQ(0, j)] = w[8] * Tin * P[8];
        s.T[SQ(0, j)] = Tin;
    }
    for (int j = 1 + threadIdx.x; j <= Ny && !(c.heat & BGK_HEAT_RIGHT); j += blockDim.x) {
        eq_poly(s.u[SQ(Nx + 1, j)], s.v[SQ(Nx + 1, j)], P);
        const double t = s.T[SQ(Nx, j)];
        s.g[3][SQ(Nx + 1, j)] = w[3] * t * P[3];
        s.g[6][SQ(Nx + 1, j)] = w[6] * t * P[6];
        s.g[7][SQ(Nx + 1, j)] = w[7] * t * P[7];
        s.T[SQ(Nx + 1, j)] = s.T[SQ(Nx, j)];
    }
    __syncthreads();
    for (int i = threadIdx.x; i <= Nx + 1; i += blockDim.x) {
        for (int k = 0; k < 9; k++) s.g[k][SQ(i, Ny + 1)] = s.g[k][SQ(i, Ny)];
        s.T[SQ(i, Ny + 1)] = s.T[SQ(i, Ny)];
        s.phi[SQ(i, Ny + 1)] = s.phi[SQ(i, Ny)];
    }
    __syncthreads();
    for (int i = threadIdx.x; i <= Nx + 1; i += blockDim.x) {
        for (int k = 0; k < 9; k++) s.g[k][SQ(i, 0)] = s.g[k][SQ(i, 1)];
        s.T[SQ(i, 0)] = s.T[SQ(i, 1)];
        s.phi[SQ(i, 0)] = s.phi[SQ(i, 1)];
    }
}

/* --------------------------------------------- ring boundary (codes != 4) */

/* BC_f (STEP_7/BC_f.f90:5-200, every branch, west, east, north, south in that
 * order) on the fused state: interior f from the compact planes of the
 * current buffer, halo f in the ring, rho/u/v in the mirrors (which hold the
 * previous step's moments on the edge rows and columns and the reference's
 * halo values).  Then the macroscopic halo assignments of BC_g
 * (STEP_7/BC_g.f90:7-64): T west/east, then T and phi north/south, and
 * bc_prep's per-row west/east values.  Three launches (ring_k1..k3 below)
 * keep every phase after the phases whose cells it reads, as in the
 * reference.  The g halos themselves are not stored: the step computes them
 * (west and east from bc_prep's per-row values, north and south as
 * copies). */
struct RingF {
    const double *fc;      /* compact planes (current buffer) */
    double *ring;
    long long plane, RL;
    int P, Nx, Ny;
    __device__ double get(int k, int i, int j) const
    {
        if (i >= 1 && i <= Nx && j >= 1 && j <= Ny) return fc[k * plane + (long long)(j - 1) * P + (i - 1)];
        return ring[k * RL + ring_idx(Nx, Ny, i, j)];
    }
    __device__ void set(int k, int i, int j, double v) const { ring[k * RL + ring_idx(Nx, Ny, i, j)] = v; }
};

/* The phases of the boundary update, one cell (row j or column i) per
 * call, with the reference's formulas and ranges. */
__device__ __forceinline__ void ring_west(const Consts &c, const RingF &F, double *rho, double *u, double *v,
                                          int wbc, int j)
{
    const int Nx = c.Nx, Ny = c.Ny, NX2 = Nx + 2;
    const double *w = c.w;
    double P[9];
    if (wbc == 0) {
        double q[9];
#pragma unroll
        for (int k = 0; k < 9; k++) q[k] = F.get(k, Nx, j);
#pragma unroll
        for (int k = 0; k < 9; k++) F.set(k, 0, j, q[k]);
    } else if (wbc == 1) {
        if (j < 1 || j > Ny) return;
        eq_poly(c.u0, c.v0, P);
        double r = rho[SQ(1, j)];
        F.set(1, 0, j, w[1] * r * P[1]);
        F.set(5, 0, j, w[5] * r * P[5]);
        F.set(8, 0, j, w[8] * r * P[8]);
        u[SQ(0, j)] = c.u0;
        v[SQ(0, j)] = c.v0;
        rho[SQ(0, j)] = rho[SQ(1, j)];
    } else if (wbc == 2) {
        eq_poly(u[SQ(0, j)], c.v0, P);
        double r = rho[SQ(1, j)];
        F.set(1, 0, j, w[1] * r * P[1]);
        F.set(5, 0, j, w[5] * r * P[5]);
        F.set(8, 0, j, w[8] * r * P[8]);
    } else if (wbc == 3) {
        double u1 = u[SQ(1, j)], v1 = v[SQ(1, j)];
        eq_poly(u1, v1, P);
        F.set(1, 0, j, w[1] * c.rho1 * P[1]);
        F.set(5, 0, j, w[5] * c.rho1 * P[5]);
        F.set(8, 0, j, w[8] * c.rho1 * P[8]);
        u[SQ(0, j)] = u1;
        v[SQ(0, j)] = v1;
        rho[SQ(0, j)] = c.rho1;
    } else if (wbc == 4) {
        if (j < 1 || j > Ny) return;
        const double a = F.get(3, 1, j), b = F.get(6, 1, j - 1), d = F.get(7, 1, j + 1);
        F.set(1, 0, j, a);
        F.set(8, 0, j, b);
        F.set(5, 0, j, d);
    }
}

__device__ __forceinline__ void ring_east(const Consts &c, const RingF &F, double *rho, double *u, double *v,
                                          int ebc, int j)
{
    const int Nx = c.Nx, Ny = c.Ny, NX2 = Nx + 2;
    const double *w = c.w;
    double P[9];
    if (ebc == 0) {
        double q[9];
#pragma unroll
        for (int k = 0; k < 9; k++) q[k] = F.get(k, 1, j);
#pragma unroll
        for (int k = 0; k < 9; k++) F.set(k, Nx + 1, j, q[k]);
    } else if (ebc == 3) {
        if (j < 1 || j > Ny) return;
        double un = u[SQ(Nx, j)], vn = v[SQ(Nx, j)];
        eq_poly(un, vn, P);
        F.set(3, Nx + 1, j, w[3] * c.rho0 * P[3]);
        F.set(6, Nx + 1, j, w[6] * c.rho0 * P[6]);
        F.set(7, Nx + 1, j, w[7] * c.rho0 * P[7]);
        u[SQ(Nx + 1, j)] = un;
        v[SQ(Nx + 1, j)] = vn;
        rho[SQ(Nx + 1, j)] = c.rho0;
    } else if (ebc == 4) {
        if (j < 1 || j > Ny) return;
        const double a = F.get(1, Nx, j), b = F.get(8, Nx, j + 1), d = F.get(5, Nx, j - 1);
        F.set(3, Nx + 1, j, a);
        F.set(6, Nx + 1, j, b);
        F.set(7, Nx + 1, j, d);
    }
}

__device__ __forceinline__ void ring_north(const Consts &c, const RingF &F, double *rho, double *u, double *v,
                                           int nbc, int i)
{
    const int Nx = c.Nx, Ny = c.Ny, NX2 = Nx + 2;
    const double *w = c.w;
    double P[9];
    if (nbc == 0) {
        double q[9];
#pragma unroll
        for (int k = 0; k < 9; k++) q[k] = F.get(k, i, 1);
#pragma unroll
        for (int k = 0; k < 9; k++) F.set(k, i, Ny + 1, q[k]);
    } else if (nbc == 4) {
        if (i == 0) {
            F.set(8, 0, Ny + 1, F.get(6, 1, Ny));
            return;
        }
        if (i > Nx) return;
        const double a = F.get(2, i, Ny), b = F.get(5, i - 1, Ny), d = F.get(6, i + 1, Ny);
        F.set(4, i, Ny + 1, a);
        F.set(7, i, Ny + 1, b);
        F.set(8, i, Ny + 1, d);
        rho[SQ(i, Ny + 1)] = rho[SQ(i, Ny)];
        u[SQ(i, Ny + 1)] = 0.0;
        v[SQ(i, Ny + 1)] = 0.0;
    } else if (nbc == 5) {
        const double a = F.get(2, i, Ny - 1), b = F.get(6, i, Ny - 1), d = F.get(5, i, Ny - 1);
        F.set(4, i, Ny + 1, a);
        F.set(7, i, Ny + 1, b);
        F.set(8, i, Ny + 1, d);
    } else if (nbc == 6) {
        const double a = F.get(4, i, Ny), b = F.get(7, i, Ny), d = F.get(8, i, Ny);
        F.set(4, i, Ny + 1, a);
        F.set(7, i, Ny + 1, b);
        F.set(8, i, Ny + 1, d);
    } else if (nbc == 1) {
        eq_poly(c.u0, c.v0, P);
        double r = rho[SQ(i, Ny)];
        F.set(4, i, Ny + 1, w[4] * r * P[4]);
        F.set(7, i, Ny + 1, w[7] * r * P[7]);
        F.set(8, i, Ny + 1, w[8] * r * P[8]);
    }
}

__device__ __forceinline__ void ring_south(const Consts &c, const RingF &F, double *rho, double *u, double *v,
                                           int sbc, int i)
{
    const int Nx = c.Nx, Ny = c.Ny, NX2 = Nx + 2;
    if (sbc == 0) {
        double q[9];
#pragma unroll
        for (int k = 0; k < 9; k++) q[k] = F.get(k, i, Ny);
#pragma unroll
        for (int k = 0; k < 9; k++) F.set(k, i, 0, q[k]);
    } else if (sbc == 4) {
        if (i == 0) {
            F.set(5, 0, 0, F.get(7, 1, 1));
            return;
        }
        if (i > Nx) return;
        const double a = F.get(4, i, 1), b = F.get(7, i + 1, 1), d = F.get(8, i - 1, 1);
        F.set(2, i, 0, a);
        F.set(5, i, 0, b);
        F.set(6, i, 0, d);
        rho[SQ(i, 0)] = rho[SQ(i, 1)];
        u[SQ(i, 0)] = 0.0;
        v[SQ(i, 0)] = 0.0;
    } else if (sbc == 6) {
        const double a = F.get(2, i, 1), b = F.get(5, i, 1), d = F.get(6, i, 1);
        F.set(2, i, 0, a);
        F.set(5, i, 0, b);
        F.set(6, i, 0, d);
    }
}

/* BC_g's T west/east (T(Nx,j) of the previous moments is tcol; with
 * BGK_HEAT_RIGHT, T(1,j) of the previous step is in the mirror and the east
 * wall is Tin), rows j = 1..Ny */
__device__ __forceinline__ void ring_g_west_east(const Consts &c, double *T, const double *tin, const double *tcol,
                                                 int j)
{
    const int Nx = c.Nx, NX2 = Nx + 2;
    if (c.heat & BGK_HEAT_RIGHT) {
        T[SQ(0, j)] = T[SQ(1, j)];
        T[SQ(Nx + 1, j)] = c.Tin;
    } else {
        T[SQ(0, j)] = tin ? tin[j - 1] : c.Tin;
        T[SQ(Nx + 1, j)] = tcol[j - 1];
    }
}

/* The update runs as three launches; within one, phases that neither read
 * nor write each other's cells run side by side, one thread per cell.
 *  1. BC_f west and east.  West writes column 0 and reads columns 1 and Nx;
 *     east writes column Nx+1 and reads columns 1 and Nx.
 *  2. BC_f north and south, and BC_g's T west/east.  North writes row Ny+1
 *     and reads rows Ny-1, Ny and 1; south writes row 0 and reads rows 1
 *     and Ny; BC_g touches only T, which BC_f neither reads nor writes.  The
 *     one exception, north code 5 reading row Ny-1 = 0 when Ny = 1, runs
 *     south as a launch of its own after north.
 *  3. BC_g's T and phi north (row Ny+1 from row Ny, whose ends step 2
 *     wrote) and south (row 0 from row 1), and bc_prep's per-row values
 *     (from the u, v halos of step 1 and the T mirror).
 * Each launch sees what the previous ones wrote (stream order), as each
 * phase of the reference sees the phases before it. */
__global__ void ring_k1(Consts c, RingF F, double *rho, double *u, double *v, int wbc, int ebc)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x, n = c.Ny + 2;
    if (t < n) ring_west(c, F, rho, u, v, wbc, t);
    else if (t < 2 * n) ring_east(c, F, rho, u, v, ebc, t - n);
}

__global__ void ring_k2(Consts c, RingF F, double *rho, double *u, double *v, double *T, const double *tin,
                        const double *tcol, int nbc, int sbc, bool with_south)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x, m = c.Nx + 2;
    const int ns = with_south ? m : 0;
    if (t < m) ring_north(c, F, rho, u, v, nbc, t);
    else if (t < m + ns) ring_south(c, F, rho, u, v, sbc, t - m);
    else if (t < m + ns + c.Ny) ring_g_west_east(c, T, tin, tcol, t - m - ns + 1);
}

__global__ void ring_k2_south(Consts c, RingF F, double *rho, double *u, double *v, int sbc)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < c.Nx + 2) ring_south(c, F, rho, u, v, sbc, t);
}

__global__ void ring_k3(Consts c, double *T, double *phi, const double *mu, const double *mv, const double *tin,
                        double *gW, double *pE, double *phiW, double *phiE)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x, m = c.Nx + 2, Ny = c.Ny, NX2 = c.Nx + 2;
    if (t < m) {
        T[SQ(t, Ny + 1)] = T[SQ(t, Ny)];
        phi[SQ(t, Ny + 1)] = phi[SQ(t, Ny)];
    } else if (t < 2 * m) {
        const int i = t - m;
        T[SQ(i, 0)] = T[SQ(i, 1)];
        phi[SQ(i, 0)] = phi[SQ(i, 1)];
    } else if (t < 2 * m + Ny) {
        bc_prep_row(c, mu, mv, phi, T, tin, gW, pE, phiW, phiE, t - 2 * m + 1);
    }
}

#define INTERIOR_IJ()                                             \
    const int Nx = c.Nx, Ny = c.Ny, NX2 = Nx + 2;                 \
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;      \
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;      \
    if (i > Nx || j > Ny) return;                                 \
    const size_t q = SQ(i, j);                                    \
    (void)Nx; (void)Ny;

/* STEP_7/streaming.f90:5-27 */
__global__ void staged_streaming(Staged s, Consts c)
{
    INTERIOR_IJ();
    s.fp[0][q] = s.f[0][SQ(i, j)];
    s.fp[1][q] = s.f[1][SQ(i - 1, j)];
    s.fp[2][q] = s.f[2][SQ(i, j - 1)];
    s.fp[3][q] = s.f[3][SQ(i + 1, j)];
    s.fp[4][q] = s.f[4][SQ(i, j + 1)];
    s.fp[5][q] = s.f[5][SQ(i - 1, j - 1)];
    s.fp[6][q] = s.f[6][SQ(i + 1, j - 1)];
    s.fp[7][q] = s.f[7][SQ(i + 1, j + 1)];
    s.fp[8][q] = s.f[8][SQ(i - 1, j + 1)];
    s.gp[0][q] = s.g[0][SQ(i, j)];
    s.gp[1][q] = s.g[1][SQ(i - 1, j)];
    s.gp[2][q] = s.g[2][SQ(i, j - 1)];
    s.gp[3][q] = s.g[3][SQ(i + 1, j)];
    s.gp[4][q] = s.g[4][SQ(i, j + 1)];
    s.gp[5][q] = s.g[5][SQ(i - 1, j - 1)];
    s.gp[6][q] = s.g[6][SQ(i + 1, j - 1)];
    s.gp[7][q] = s.g[7][SQ(i + 1, j + 1)];
    s.gp[8][q] = s.g[8][SQ(i - 1, j + 1)];
}

/* STEP_7/momentsPre.f90:5-23 */
__global__ void staged_moments_pre(Staged s, Consts c)
{
    INTERIOR_IJ();
    double f[9], g[9];
    for (int k = 0; k < 9; k++) { f[k] = s.fp[k][q]; g[k] = s.gp[k][q]; }
    const double rho = sum9(f), T = sum9(g);
    const double irho = 1.0 / rho;
    const double u = irho * xmom(f), v = irho * ymom(f);
    s.rho[q] = rho; s.T[q] = T; s.u[q] = u; s.v[q] = v;
    s.rho2[q] = rho; s.T2[q] = T; s.u2[q] = u; s.v2[q] = v;
}

/* STEP_7/phase_field.f90:19 (phi_prec = phi over the whole array) */
__global__ void staged_copy(double *dst, const double *src, size_t n)
{
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x)
        dst[q] = src[q];
}

/* STEP_7/phase_field.f90:21-52 */
template <int TANH>
__global__ void staged_phase_field(Staged s, Consts c)
{
    INTERIOR_IJ();
    const double *pp = s.phip;
    const double th = select_tanh(((s.T[q] - c.T_crit) - c.T_act) / c.T_width, TANH);
    const double kp = aplus(pp[SQ(i, j)]) + aplus(pp[SQ(i + 1, j)]) + aplus(pp[SQ(i, j + 1)])
                    + aplus(pp[SQ(i - 1, j)]) + aplus(pp[SQ(i, j - 1)]) + aplus(pp[SQ(i + 1, j + 1)])
                    + aplus(pp[SQ(i - 1, j + 1)]) + aplus(pp[SQ(i - 1, j - 1)]) + aplus(pp[SQ(i + 1, j - 1)]);
    const double km = aminus(pp[SQ(i, j)]) + aminus(pp[SQ(i + 1, j)]) + aminus(pp[SQ(i, j + 1)])
                    + aminus(pp[SQ(i - 1, j)]) + aminus(pp[SQ(i, j - 1)]) + aminus(pp[SQ(i + 1, j + 1)])
                    + aminus(pp[SQ(i - 1, j + 1)]) + aminus(pp[SQ(i - 1, j - 1)]) + aminus(pp[SQ(i + 1, j - 1)]);
    s.phi[q] = phi_update(c, kp, km, th, pp[q]);
}

/* STEP_7/forces.f90:12-28 */
__global__ void staged_forces(Staged s, Consts c)
{
    INTERIOR_IJ();
    double T = s.T[q], u = s.u[q], v = s.v[q];
    apply_forces(c, s.phi[q], s.phip[q], s.rho[q], T, u, v);
    s.T[q] = T; s.u[q] = u; s.v[q] = v;
}

/* STEP_7/collision.f90:14-152 */
template <bool REF32>
__global__ void staged_collision(Staged s, Consts c)
{
    INTERIOR_IJ();
    double Pq[9], in[9], eq[9], out[9];
    const double rho = s.rho[q], T = s.T[q];
    eq_poly(s.u[q], s.v[q], Pq);
    for (int k = 0; k < 9; k++) { in[k] = s.fp[k][q]; eq[k] = c.w[k] * rho * Pq[k]; }
    regularize_relax<REF32>(c, in, eq, c.omega_f, out);
    for (int k = 0; k < 9; k++) s.f[k][q] = out[k];
    for (int k = 0; k < 9; k++) { in[k] = s.gp[k][q]; eq[k] = c.w[k] * T * Pq[k]; }
    regularize_relax<REF32>(c, in, eq, c.omega_g, out);
    for (int k = 0; k < 9; k++) s.g[k][q] = out[k];
}

/* STEP_7/moments.f90:8-27 */
__global__ void staged_moments(Staged s, Consts c)
{
    INTERIOR_IJ();
    double f[9], g[9];
    for (int k = 0; k < 9; k++) { f[k] = s.f[k][q]; g[k] = s.g[k][q]; }
    const double rho = sum9(f);
    const double irho = 1.0 / rho;
    const double tT = sum9(g);
    const double tu = irho * xmom(f), tv = irho * ymom(f);
    s.rho[q] = rho;
    s.T[q] = (tT + s.T2[q]) * 0.5;
    s.u[q] = (tu + s.u2[q]) * 0.5;
    s.v[q] = (tv + s.v2[q]) * 0.5;
}

/* ------------------------------------------------------------ conversions */

/* compact (cur) populations -> staged reference arrays (interior), plus the
 * two frozen corners; other f/g halo cells carry no state with code 4. */
__global__ void compact_to_staged_kernel(Staged s, Consts c, const double *fc, const double *gc,
                                         long long plane, int P, const double *corner)
{
    INTERIOR_IJ();
    const long long cc = (long long)(j - 1) * P + (i - 1);
    for (int k = 0; k < 9; k++) { s.f[k][q] = fc[k * plane + cc]; s.g[k][q] = gc[k * plane + cc]; }
    if (i == Nx && j == 1) s.f[6][SQ(Nx + 1, 0)] = corner[0];
    if (i == Nx && j == Ny) s.f[7][SQ(Nx + 1, Ny + 1)] = corner[1];
}

__global__ void staged_to_compact_kernel(Staged s, Consts c, double *fc, double *gc, double *phc,
                                         double *phc_prev, long long plane, int P, double *corner,
                                         double *tcol)
{
    INTERIOR_IJ();
    const long long cc = (long long)(j - 1) * P + (i - 1);
    for (int k = 0; k < 9; k++) { fc[k * plane + cc] = s.f[k][q]; gc[k * plane + cc] = s.g[k][q]; }
    phc[cc] = s.phi[q];
    phc_prev[cc] = s.phip[q];
    if (i == Nx) tcol[j - 1] = s.T[q];
    if (i == Nx && j == 1) corner[0] = s.f[6][SQ(Nx + 1, 0)];
    if (i == Nx && j == Ny) corner[1] = s.f[7][SQ(Nx + 1, Ny + 1)];
}

/* one reference-layout field -> compact plane (interior only) */
__global__ void ref_to_plane_kernel(Consts c, const double *ref, double *plane_dst, int P)
{
    INTERIOR_IJ();
    plane_dst[(long long)(j - 1) * P + (i - 1)] = ref[q];
}

/* compact plane -> reference layout; halos zero except the optional corner */
__global__ void plane_to_ref_kernel(Consts c, const double *plane_src, int P, double *ref,
                                    const double *halo_src, int corner_i, int corner_j, const double *corner)
{
    const int Nx = c.Nx, Ny = c.Ny, NX2 = Nx + 2;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i > Nx + 1 || j > Ny + 1) return;
    const size_t q = SQ(i, j);
    if (i >= 1 && i <= Nx && j >= 1 && j <= Ny)
        ref[q] = plane_src[(long long)(j - 1) * P + (i - 1)];
    else if (halo_src)
        ref[q] = halo_src[q];
    else
        ref[q] = (corner && i == corner_i && j == corner_j) ? corner[0] : 0.0;
}

/* T(Nx, j) of a reference-layout field -> tcol */
__global__ void ref_to_tcol_kernel(Consts c, const double *ref, double *tcol)
{
    const int Ny = c.Ny, NX2 = c.Nx + 2;
    const int j = blockIdx.x * blockDim.x + threadIdx.x + 1;
    if (j <= Ny) tcol[j - 1] = ref[SQ(c.Nx, j)];
}

/* ---------------------------------------------------------------- sums */

constexpr int SUM_BLOCKS = 592;   /* 4 x 148 SMs */
constexpr int SUM_THREADS = 256;

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

/* Deterministic two-pass FP64 reduction: a fixed grid strides over the
 * interior in a fixed order, each block reduces with warp shuffles and
 * writes 4 partials; one block then adds the partials in index order. */
__global__ void field_sums_kernel(Consts c, const double *rho, const double *T, const double *phi,
                                  double *partial, int j0, int nrows)
{
    const int Nx = c.Nx, NX2 = Nx + 2;
    const long long n = (long long)Nx * nrows;
    double a = 0.0, b = 0.0, p = 0.0, k = 0.0;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t % Nx) + 1, j = (int)(t / Nx) + 1 + j0;
        const size_t q = SQ(i, j);
        a += rho[q];
        b += T[q];
        const double ph = phi[q];
        p += ph;
        k += (ph > 0.0) ? 1.0 : 0.0;
    }
    __shared__ double sh[4][SUM_THREADS / 32];
    a = warp_sum(a); b = warp_sum(b); p = warp_sum(p); k = warp_sum(k);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) { sh[0][wid] = a; sh[1][wid] = b; sh[2][wid] = p; sh[3][wid] = k; }
    __syncthreads();
    if (threadIdx.x < 4) {
        double acc = 0.0;
        for (int w = 0; w < SUM_THREADS / 32; w++) acc += sh[threadIdx.x][w];
        partial[4 + threadIdx.x * SUM_BLOCKS + blockIdx.x] = acc;
    }
}

__global__ void field_sums_final(double *partial)
{
    const int r = threadIdx.x;   /* 4 threads */
    if (r >= 4) return;
    double acc = 0.0;
    for (int b = 0; b < SUM_BLOCKS; b++) acc += partial[4 + r * SUM_BLOCKS + b];
    partial[r] = acc;
}

Staged staged_of(bgk_ctx *c)
{
    Staged s;
    for (int k = 0; k < 9; k++) { s.f[k] = c->sf[k]; s.g[k] = c->sg[k]; s.fp[k] = c->sfp[k]; s.gp[k] = c->sgp[k]; }
    s.rho = c->mrho; s.T = c->mT; s.u = c->mu; s.v = c->mv; s.phi = c->mphi;
    s.phip = c->sphip; s.rho2 = c->srho2; s.T2 = c->sT2; s.u2 = c->su2; s.v2 = c->sv2;
    s.tin = c->tin_rows;
    return s;
}

dim3 interior_grid(const bgk_ctx *c, dim3 blk)
{
    return dim3((c->Nx + blk.x - 1) / blk.x, (c->Ny + blk.y - 1) / blk.y);
}

double *corner_ptr(bgk_ctx *c) { return c->corner; }

} // namespace


cudaError_t launch_init_f64(bgk_ctx *c)
{
    StepPtrs<double> s{};
    s.mrho = c->mrho; s.mT = c->mT; s.mu = c->mu; s.mv = c->mv; s.mphi = c->mphi;
    s.plane = c->plane; s.P = c->P; s.NX2 = c->NX2;
    dim3 blk(32, 8), grd((c->NX2 + 31) / 32, (c->NY2 + 7) / 8);
    const bool staged = c->mode == 1;
    init_kernel<<<grd, blk, 0, c->stream>>>(
        c->c, c->p.westBC, s,
        staged ? nullptr : (double *)c->fbuf[c->cur],
        staged ? nullptr : (double *)c->gbuf[c->cur],
        (double *)c->phibuf[0], (double *)c->phibuf[1], staged_of(c), staged,
        c->corner, c->tcol[c->cur], (!staged && c->ring) ? c->fring : nullptr, c->ring_len);
    return cudaGetLastError();
}

cudaError_t launch_ring_bc(bgk_ctx *c)
{
    RingF F;
    F.fc = (const double *)c->fbuf[c->cur];
    F.ring = c->fring;
    F.plane = c->plane;
    F.RL = c->ring_len;
    F.P = c->P;
    F.Nx = c->Nx;
    F.Ny = c->Ny;
    const int Nx = c->Nx, Ny = c->Ny, nb = 256;
    const bool with_south = !(c->p.northBC == 5 && Ny < 2);
    const int n1 = 2 * (Ny + 2), n2 = (Nx + 2) * (with_south ? 2 : 1) + Ny, n3 = 2 * (Nx + 2) + Ny;
    ring_k1<<<(n1 + nb - 1) / nb, nb, 0, c->stream>>>(c->c, F, c->mrho, c->mu, c->mv, c->p.westBC, c->p.eastBC);
    ring_k2<<<(n2 + nb - 1) / nb, nb, 0, c->stream>>>(c->c, F, c->mrho, c->mu, c->mv, c->mT, c->tin_rows,
                                                      c->tcol[c->cur], c->p.northBC, c->p.southBC, with_south);
    if (!with_south)
        ring_k2_south<<<(Nx + 2 + nb - 1) / nb, nb, 0, c->stream>>>(c->c, F, c->mrho, c->mu, c->mv, c->p.southBC);
    ring_k3<<<(n3 + nb - 1) / nb, nb, 0, c->stream>>>(c->c, c->mT, c->mphi, c->mu, c->mv, c->tin_rows, c->gW, c->pE,
                                                      c->phiW, c->phiE);
    return cudaGetLastError();
}

cudaError_t launch_bc_prep(bgk_ctx *c)
{
    int n = c->Ny;
    bc_prep_kernel<<<(n + 127) / 128, 128, 0, c->stream>>>(c->c, c->mu, c->mv, c->mphi, c->mT, c->tin_rows,
                                                            c->gW, c->pE, c->phiW, c->phiE);
    return cudaGetLastError();
}

cudaError_t launch_macro_halos(bgk_ctx *c)
{
    macro_halo_kernel<<<1, 1024, 0, c->stream>>>(c->c, c->mrho, c->mT, c->mu, c->mv, c->mphi, c->tin_rows);
    return cudaGetLastError();
}

static int strip_height(const bgk_ctx *c)
{
    /* enough blocks to fill 148 SMs several times over, but tall strips */
    if (c->tune_H > 0) return c->tune_H;
    const int bx = (c->Nx + FUSED_BX - 1) / FUSED_BX;
    int H = 16;
    while (H > 2 && (long long)bx * ((c->Ny + H - 1) / H) < 148LL * 8) H /= 2;
    return H;
}


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

/* nsteps exact-order FP64 steps in one dataflow launch (walls of code 4). */
cudaError_t launch_flow_f64(bgk_ctx *c, int nsteps)
{
    StepPtrs<double> s0, s1;
    flow_ptrs(c, s0, s1);
    return launch_flow_pipe_f64(c, s0, s1, nsteps);
}

cudaError_t launch_fused_f64(bgk_ctx *c, bool moments, bool edge_halos)
{
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
    /* walls other than code 4 run on the pipeline kernel only */
    if (c->tune_pipe || c->ring) return launch_fused_pipe_f64(c, s, moments, edge_halos);
    return launch_fused_f64_variant(c, grd, s, H, moments);
}

/* One fused step between explicit state buffers (no moments written):
 * used by the adjoint to recompute checkpointed segments. */
cudaError_t launch_fused_f64_ptrs(bgk_ctx *c, const double *fin, const double *gin, const double *phin,
                                  const double *tcin, double *fout, double *gout, double *phout, double *tcout)
{
    StepPtrs<double> s{};
    s.fin = fin; s.gin = gin; s.fout = fout; s.gout = gout;
    s.phin = phin; s.phout = phout; s.tcin = tcin; s.tcout = tcout;
    s.gW = c->gW; s.pE = c->pE; s.phiW = c->phiW; s.phiE = c->phiE;
    s.mrho = c->mrho; s.mT = c->mT; s.mu = c->mu; s.mv = c->mv; s.mphi = c->mphi;
    s.plane = c->plane; s.P = c->P; s.NX2 = c->NX2;
    const int H = strip_height(c);
    dim3 grd((c->Nx + FUSED_BX - 1) / FUSED_BX, (c->Ny + H - 1) / H);
    if (c->tune_pipe) return launch_fused_pipe_f64(c, s, false);
    return launch_fused_f64_variant(c, grd, s, H, false);
}

cudaError_t launch_staged(bgk_ctx *c, int stage)
{
    Staged s = staged_of(c);
    dim3 blk(64, 4);
    dim3 grd = interior_grid(c, blk);
    switch (stage) {
    case 1: staged_bc_f<<<1, 1024, 0, c->stream>>>(s, c->c, c->p.westBC, c->p.eastBC, c->p.northBC, c->p.southBC); break;
    case 2: staged_bc_g<<<1, 1024, 0, c->stream>>>(s, c->c); break;
    case 3: staged_streaming<<<grd, blk, 0, c->stream>>>(s, c->c); break;
    case 4: staged_moments_pre<<<grd, blk, 0, c->stream>>>(s, c->c); break;
    case 5:
        staged_copy<<<592, 256, 0, c->stream>>>(s.phip, s.phi, c->A);
        if (c->opt.tanh_mode == BGK_TANH_PORTABLE)
            staged_phase_field<BGK_TANH_PORTABLE><<<grd, blk, 0, c->stream>>>(s, c->c);
        else
            staged_phase_field<BGK_TANH_DEVICE><<<grd, blk, 0, c->stream>>>(s, c->c);
        break;
    case 6: staged_forces<<<grd, blk, 0, c->stream>>>(s, c->c); break;
    case 7:
        if (c->opt.smooth) staged_collision<false><<<grd, blk, 0, c->stream>>>(s, c->c);
        else staged_collision<true><<<grd, blk, 0, c->stream>>>(s, c->c);
        break;
    case 8: staged_moments<<<grd, blk, 0, c->stream>>>(s, c->c); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

/* the f halo cells between the ring and the staged arrays */
static cudaError_t ring_staged(bgk_ctx *c, bool to_ring)
{
    Ptr9 refs;
    for (int k = 0; k < 9; k++) refs.p[k] = c->sf[k];
    dim3 grd((unsigned)((c->ring_len + 255) / 256), 9);
    ring_ref_copy<<<grd, 256, 0, c->stream>>>(c->Nx, c->Ny, c->fring, c->ring_len, refs, 0, to_ring);
    return cudaGetLastError();
}

/* the f halo cells of population k between the ring and a reference-layout field */
static cudaError_t ring_field(bgk_ctx *c, int k, double *ref, bool to_ring)
{
    Ptr9 refs{};
    refs.p[0] = ref;
    dim3 grd((unsigned)((c->ring_len + 255) / 256), 1);
    ring_ref_copy<<<grd, 256, 0, c->stream>>>(c->Nx, c->Ny, c->fring, c->ring_len, refs, k, to_ring);
    return cudaGetLastError();
}

cudaError_t launch_compact_to_staged(bgk_ctx *c)
{
    Staged s = staged_of(c);
    dim3 blk(64, 4);
    compact_to_staged_kernel<<<interior_grid(c, blk), blk, 0, c->stream>>>(
        s, c->c, (const double *)c->fbuf[c->cur], (const double *)c->gbuf[c->cur], c->plane, c->P, corner_ptr(c));
    if (c->ring) return ring_staged(c, false);
    return cudaGetLastError();
}

cudaError_t launch_staged_to_compact(bgk_ctx *c)
{
    Staged s = staged_of(c);
    dim3 blk(64, 4);
    staged_to_compact_kernel<<<interior_grid(c, blk), blk, 0, c->stream>>>(
        s, c->c, (double *)c->fbuf[c->cur], (double *)c->gbuf[c->cur], (double *)c->phibuf[c->cur],
        (double *)c->phibuf[c->cur ^ 1], c->plane, c->P, corner_ptr(c), c->tcol[c->cur]);
    if (c->ring) return ring_staged(c, true);
    return cudaGetLastError();
}

/* Upload helper for the fused state: `ref` is a device copy of one field in
 * the reference layout. */
cudaError_t launch_ref_to_compact(bgk_ctx *c, int field, const double *ref)
{
    dim3 blk(64, 4), grd = interior_grid(c, blk);
    if (field >= BGK_FIELD_F0 && field < BGK_FIELD_F0 + 9) {
        const int k = field - BGK_FIELD_F0;
        ref_to_plane_kernel<<<grd, blk, 0, c->stream>>>(c->c, ref, (double *)c->fbuf[c->cur] + k * c->plane, c->P);
        if (c->ring) {
            cudaError_t e = ring_field(c, k, const_cast<double *>(ref), true);
            if (e != cudaSuccess) return e;
        }
        if (k == 6 || k == 7) {
            const size_t q = (k == 6) ? (size_t)(c->Nx + 1) : (size_t)(c->Nx + 1) + (size_t)c->NX2 * (size_t)(c->Ny + 1);
            cudaError_t e = cudaMemcpyAsync(corner_ptr(c) + (k - 6), ref + q, sizeof(double),
                                            cudaMemcpyDeviceToDevice, c->stream);
            if (e != cudaSuccess) return e;
        }
    } else if (field >= BGK_FIELD_G0 && field < BGK_FIELD_G0 + 9) {
        const int k = field - BGK_FIELD_G0;
        ref_to_plane_kernel<<<grd, blk, 0, c->stream>>>(c->c, ref, (double *)c->gbuf[c->cur] + k * c->plane, c->P);
    } else if (field == BGK_FIELD_PHI) {
        ref_to_plane_kernel<<<grd, blk, 0, c->stream>>>(c->c, ref, (double *)c->phibuf[0], c->P);
        ref_to_plane_kernel<<<grd, blk, 0, c->stream>>>(c->c, ref, (double *)c->phibuf[1], c->P);
    } else if (field == BGK_FIELD_T) {
        ref_to_tcol_kernel<<<(c->Ny + 127) / 128, 128, 0, c->stream>>>(c->c, ref, c->tcol[c->cur]);
    }
    return cudaGetLastError();
}

/* Download helper for the fused state: writes a reference-layout field into
 * device memory `ref`.  which = 0: current buffer, 1: previous (phi_prec). */
cudaError_t launch_compact_to_ref(bgk_ctx *c, int field, double *ref, int which)
{
    dim3 blk(32, 8), grd((c->NX2 + 31) / 32, (c->NY2 + 7) / 8);
    const int b = which ? (c->cur ^ 1) : c->cur;
    if (field >= BGK_FIELD_F0 && field < BGK_FIELD_F0 + 9) {
        const int k = field - BGK_FIELD_F0;
        const double *cn = (k == 6) ? corner_ptr(c) : (k == 7 ? corner_ptr(c) + 1 : nullptr);
        plane_to_ref_kernel<<<grd, blk, 0, c->stream>>>(c->c, (const double *)c->fbuf[b] + k * c->plane, c->P, ref,
                                                         nullptr, c->Nx + 1, k == 6 ? 0 : c->Ny + 1, cn);
        /* the ring holds the halo of the current step only */
        if (c->ring && !which) return ring_field(c, k, ref, false);
    } else if (field >= BGK_FIELD_G0 && field < BGK_FIELD_G0 + 9) {
        const int k = field - BGK_FIELD_G0;
        plane_to_ref_kernel<<<grd, blk, 0, c->stream>>>(c->c, (const double *)c->gbuf[b] + k * c->plane, c->P, ref,
                                                         nullptr, -1, -1, nullptr);
    } else if (field == BGK_FIELD_PHI_PREC) {
        plane_to_ref_kernel<<<grd, blk, 0, c->stream>>>(c->c, (const double *)c->phibuf[b], c->P, ref,
                                                         c->mphi, -1, -1, nullptr);
    } else {
        return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

/* Interior rows j0 .. j0+nrows-1 (0-based); results land in c->red[0..3]. */
cudaError_t launch_field_sums(bgk_ctx *c, int j0, int nrows)
{
    field_sums_kernel<<<SUM_BLOCKS, SUM_THREADS, 0, c->stream>>>(c->c, c->mrho, c->mT, c->mphi, c->red, j0,
                                                                  nrows);
    field_sums_final<<<1, 32, 0, c->stream>>>(c->red);
    return cudaGetLastError();
}

/* ------------------------------------------------------- slab halo rows */

/* Packed rows: 20 sections (f_0..f_8, g_0..g_8 of TE, phi of TP, the east
 * T column of double), each nrows x Nx elements (the T column nrows) and
 * padded to 16 bytes.  blockIdx.y is the section; a grid-stride loop over
 * its elements.  UNPACK copies the other way. */
__host__ __device__ inline size_t rows_section_bytes(long long elems, int esz)
{
    return ((size_t)elems * (size_t)esz + 15) / 16 * 16;
}

template <typename TE, typename TP, bool UNPACK>
__global__ void rows_copy_kernel(TE *f, TE *g, TP *phi, double *tcol, long long pl, int P, int Nx, int j0,
                                 int nrows, unsigned char *buf)
{
    const int sec = blockIdx.y;
    const long long n = (long long)Nx * nrows;
    const size_t sec_pop = rows_section_bytes(n, (int)sizeof(TE));
    if (sec < 19) {
        size_t off;
        if (sec < 18) off = (size_t)sec * sec_pop;
        else off = 18 * sec_pop;
        for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
             t += (long long)gridDim.x * blockDim.x) {
            const long long r = t / Nx, x = t % Nx;
            const long long q = (long long)(j0 + r) * P + x;
            if (sec < 18) {
                TE *plane = (sec < 9 ? f + (long long)sec * pl : g + (long long)(sec - 9) * pl);
                TE *b = reinterpret_cast<TE *>(buf + off);
                if (UNPACK) plane[q] = b[t];
                else b[t] = plane[q];
            } else {
                TP *b = reinterpret_cast<TP *>(buf + off);
                if (UNPACK) phi[q] = b[t];
                else b[t] = phi[q];
            }
        }
    } else {
        double *b = reinterpret_cast<double *>(buf + 18 * sec_pop + rows_section_bytes(n, (int)sizeof(TP)));
        for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nrows;
             t += (long long)gridDim.x * blockDim.x) {
            if (UNPACK) tcol[j0 + t] = b[t];
            else b[t] = tcol[j0 + t];
        }
    }
}

size_t rows_bytes(const bgk_ctx *c, int nrows)
{
    const long long n = (long long)c->Nx * nrows;
    return 18 * rows_section_bytes(n, c->esz) + rows_section_bytes(n, c->phisz) + rows_section_bytes(nrows, 8);
}

template <typename TE, typename TP>
static cudaError_t rows_copy_t(bgk_ctx *c, int j0, int nrows, unsigned char *buf, bool unpack)
{
    const int cur = c->cur;
    TE *f = static_cast<TE *>(c->fbuf[cur]);
    TE *g = static_cast<TE *>(c->gbuf[cur]);
    TP *phi = static_cast<TP *>(c->phibuf[cur]);
    const long long n = (long long)c->Nx * nrows;
    long long bx = (n + 255) / 256;
    if (bx > 1184) bx = 1184;
    const dim3 grd((unsigned)bx, 20);
    if (unpack)
        rows_copy_kernel<TE, TP, true><<<grd, 256, 0, c->stream>>>(f, g, phi, c->tcol[cur], c->plane, c->P, c->Nx,
                                                                   j0, nrows, buf);
    else
        rows_copy_kernel<TE, TP, false><<<grd, 256, 0, c->stream>>>(f, g, phi, c->tcol[cur], c->plane, c->P,
                                                                    c->Nx, j0, nrows, buf);
    return cudaGetLastError();
}

cudaError_t launch_rows_copy(bgk_ctx *c, int j0, int nrows, void *buf, bool unpack)
{
    unsigned char *b = static_cast<unsigned char *>(buf);
    if (c->esz == 8) return rows_copy_t<unsigned long long, unsigned long long>(c, j0, nrows, b, unpack);
    if (c->esz == 4)
        return c->phisz == 8 ? rows_copy_t<unsigned int, unsigned long long>(c, j0, nrows, b, unpack)
                             : rows_copy_t<unsigned int, unsigned int>(c, j0, nrows, b, unpack);
    return c->phisz == 8 ? rows_copy_t<unsigned short, unsigned long long>(c, j0, nrows, b, unpack)
                         : rows_copy_t<unsigned short, unsigned int>(c, j0, nrows, b, unpack);
}

} // namespace bgk
