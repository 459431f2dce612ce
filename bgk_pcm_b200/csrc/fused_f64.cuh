/*
 * fused_f64.cuh -- the fused FP64 time-step kernel.  Included by
 * kernels_f64.cu (built with --fmad=false: bit-for-bit the reference's
 * operation order) and by kernels_fast.cu (built with multiply-add
 * contraction: the FMA variant, same source).  Must be included inside an
 * anonymous namespace within namespace bgk, after select_tanh.
 */
#ifndef BGK_FUSED_F64_CUH
#define BGK_FUSED_F64_CUH

/* ------------------------------------------------------------ fused step */

constexpr int FUSED_BX = 128;

/* Bulk prefetch of one row segment into L2 (sm_90+ bulk-copy unit): a hint
 * that keeps DRAM requests in flight without registers or shared memory.
 * ptr must be 16-byte aligned, bytes a multiple of 16. */
__device__ __forceinline__ void prefetch_l2(const void *ptr, unsigned bytes)
{
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(ptr), "r"(bytes) : "memory");
}

/* Threads 0..18 of a strip block prefetch source row r of the nine f
 * planes, the nine g planes and the phi plane for columns x0..x0+127. */
template <typename T, typename TP>
__device__ __forceinline__ void prefetch_row(const T *F, const T *G, const TP *PH, long long pl, int P, int x0,
                                             int ncols, int r, int Ny)
{
    const int t = threadIdx.x;
    if (t >= 19 || r >= Ny) return;
    const long long off = (long long)r * P + x0;
    const void *ptr;
    unsigned bytes;
    if (t < 18) {
        ptr = (t < 9 ? F + t * pl : G + (t - 9) * pl) + off;
        bytes = (unsigned)(ncols * sizeof(T));
    } else {
        ptr = PH + off;
        bytes = (unsigned)(ncols * sizeof(TP));
    }
    bytes = (bytes + 15u) & ~15u;
    prefetch_l2(ptr, bytes);
}

/* The halo cells of rho, T, u, v and phi that STEP_7's BC_f (code 4) and
 * BC_g copy from the edge nodes at the start of a step
 * (STEP_7/BC_f.f90:127-134,183-190, BC_g.f90:7-64), written by the edge
 * node (x, y) of the step before: rm, Tm, phn are its moments.  After the
 * last step of a call the reference's arrays hold these lagged halos. */
__device__ __forceinline__ void edge_halos_f64(const StepPtrs<double> &s, const Consts &c, int x, int y, bool W,
                                               bool E, bool S, bool N, double rm, double Tm, double phn)
{
    const int Nx = c.Nx, Ny = c.Ny, i = x + 1, j = y + 1;
    const size_t X = (size_t)s.NX2;
    if (N) {
        const size_t q = (size_t)i + X * (size_t)(Ny + 1);
        s.mrho[q] = rm; s.mu[q] = 0.0; s.mv[q] = 0.0; s.mT[q] = Tm; s.mphi[q] = phn;
    }
    if (S) {
        const size_t q = (size_t)i;
        s.mrho[q] = rm; s.mu[q] = 0.0; s.mv[q] = 0.0; s.mT[q] = Tm; s.mphi[q] = phn;
    }
    if (E) {
        s.mT[(size_t)(Nx + 1) + X * (size_t)j] = Tm;
        if (N) { s.mT[(size_t)(Nx + 1) + X * (size_t)(Ny + 1)] = Tm; s.mphi[(size_t)(Nx + 1) + X * (size_t)(Ny + 1)] = s.phiE[Ny - 1]; }
        if (S) { s.mT[(size_t)(Nx + 1)] = Tm; s.mphi[(size_t)(Nx + 1)] = s.phiE[0]; }
    }
    if (W) {
        const double tw = s.tin ? s.tin[y] : c.Tin;
        s.mT[X * (size_t)j] = tw;
        if (N) { s.mT[X * (size_t)(Ny + 1)] = tw; s.mphi[X * (size_t)(Ny + 1)] = s.phiW[Ny - 1]; }
        if (S) { s.mT[0] = tw; s.mphi[0] = s.phiW[0]; }
    }
}

/* One node of the fused step after its pulls: momentsPre, phase_field,
 * forces, collision, stores and (when required) moments.  Shared by the
 * register-pull kernel below and the shared-memory pipeline kernel
 * (fused_pipe.cuh), so both round identically. */
template <int TANH, bool MOM, bool REF32, bool RING = false, bool EH = false>
__device__ __forceinline__ void node_f64(const StepPtrs<double> &s, const Consts &c, int x, int y, long long cc,
                                         bool E, double *f, double *g, const double (&ap)[3][3],
                                         const double (&am)[3][3], const double *pc, bool edge = false,
                                         bool W = false, bool S = false, bool N = false)
{
    const long long pl = s.plane;
    /* momentsPre */
    const double rho = sum9(f);
    double T = sum9(g);
    const double irho = 1.0 / rho;
    double u = irho * xmom(f);
    double v = irho * ymom(f);
    const double T2 = T, u2 = u, v2 = v;

    /* phase_field */
    const double th = select_tanh(((T - c.T_crit) - c.T_act) / c.T_width, TANH);
    const double kp = ap[1][1] + ap[1][2] + ap[2][1] + ap[1][0] + ap[0][1]
                    + ap[2][2] + ap[2][0] + ap[0][0] + ap[0][2];
    const double km = am[1][1] + am[1][2] + am[2][1] + am[1][0] + am[0][1]
                    + am[2][2] + am[2][0] + am[0][0] + am[0][2];
    const double p0 = pc[1];
    const double phn = phi_update(c, kp, km, th, p0);

    /* forces */
    apply_forces(c, phn, p0, rho, T, u, v);

    /* collision */
    double Pq[9], eq[9], out[9];
    eq_poly(u, v, Pq);
#pragma unroll
    for (int k = 0; k < 9; k++) eq[k] = c.w[k] * rho * Pq[k];
    regularize_relax<REF32>(c, f, eq, c.omega_f, out);
#pragma unroll
    for (int k = 0; k < 9; k++) { s.fout[k * pl + cc] = out[k]; f[k] = out[k]; }
#pragma unroll
    for (int k = 0; k < 9; k++) eq[k] = c.w[k] * T * Pq[k];
    regularize_relax<REF32>(c, g, eq, c.omega_g, out);
#pragma unroll
    for (int k = 0; k < 9; k++) s.gout[k * pl + cc] = out[k];
    s.phout[cc] = phn;

    /* moments (all nodes on output steps; column Nx every step; with a wall
     * other than code 4, every edge node every step: the next step's BC_f
     * reads rho, u and v there) */
    const bool wm = MOM || (RING && edge);
    const bool eh = EH && edge;
    if (wm || E || eh) {
        const double Tm = (sum9(out) + T2) * 0.5;
        if (E) s.tcout[y] = Tm;
        if (eh) edge_halos_f64(s, c, x, y, W, E, S, N, sum9(f), Tm, phn);
        if (wm) {
            const double rm = sum9(f);
            const double irm = 1.0 / rm;
            const double tu = irm * xmom(f);
            const double tv = irm * ymom(f);
            const size_t q = (size_t)(x + 1) + (size_t)s.NX2 * (size_t)(y + 1);
            s.mrho[q] = rm;
            s.mT[q] = Tm;
            s.mu[q] = (tu + u2) * 0.5;
            s.mv[q] = (tv + v2) * 0.5;
            s.mphi[q] = phn;
        }
    }

}

/* One thread owns one column x of a strip of H rows and marches up it.  The
 * 3x3 phi stencil is kept as per-cell selector terms (aplus/aminus) of a
 * sliding 3-row window, so each phi value is loaded and squared once per row
 * instead of nine times.  Populations are pulled from the neighbours
 * (STEP_7/streaming.f90:5-27) with the no-slip boundary folded in:
 *  f: a pull from outside the domain takes the opposite population of the
 *     same node (bounce-back), except f6 at (Nx,1) and f7 at (Nx,Ny), which
 *     read the never-written corner halos (kept in corner[0..1]);
 *  g: rows 0/Ny+1 are copies of rows 1/Ny (clamp y), column 0 is the west
 *     value, column Nx+1 is w_k*T(Nx,y)*poly_k (east, previous moments). */
template <int TANH, bool MOM, bool REF32>
__global__ void __launch_bounds__(FUSED_BX, 4)
fused_f64_kernel(StepPtrs<double> s, Consts c, const double *__restrict__ corner, int H, int pf)
{
    const int Nx = c.Nx, Ny = c.Ny;
    const int x = blockIdx.x * FUSED_BX + threadIdx.x;
    if (x >= Nx) return;
    const int y0 = blockIdx.y * H;
    const int y1 = min(y0 + H, Ny);
    const long long pl = s.plane;
    const int P = s.P;
    const bool W = (x == 0), E = (x == Nx - 1);
    const double *__restrict__ F = s.fin;
    const double *__restrict__ G = s.gin;
    const double *__restrict__ PH = s.phin;

    double ap[3][3], am[3][3], pc[3];
    auto load_row = [&](int r, int slot) {
        const int rc = r < 0 ? 0 : (r >= Ny ? Ny - 1 : r);
        const double *row = PH + (long long)rc * P;
        const double pL = *(W ? (s.phiW + rc) : (row + x - 1));
        const double pM = row[x];
        const double pR = *(E ? (s.phiE + rc) : (row + x + 1));
        ap[slot][0] = aplus(pL); ap[slot][1] = aplus(pM); ap[slot][2] = aplus(pR);
        am[slot][0] = aminus(pL); am[slot][1] = aminus(pM); am[slot][2] = aminus(pR);
        pc[slot] = pM;
    };
    load_row(y0 - 1, 0);
    load_row(y0, 1);

    const int x0 = blockIdx.x * FUSED_BX, ncols = min(FUSED_BX, Nx - x0);
    for (int y = y0; y < y1; y++) {
        if (pf > 0) prefetch_row(F, G, PH, pl, P, x0, ncols, y + pf, Ny);
        load_row(y + 1, 2);
        const bool S = (y == 0), N = (y == Ny - 1);
        const long long cc = (long long)y * P + x;

        /* streaming (pull) with bounce-back */
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
        if (E && S) f[6] = corner[0];
        if (E && N) f[7] = corner[1];

        /* streaming of g with the BC_g halo values */
        const int ym = S ? y : y - 1, yp = N ? y : y + 1;
        const long long cm = (long long)ym * P + x, cp = (long long)yp * P + x;
        g[0] = G[cc];
        g[1] = *(W ? s.gW + y : G + 1 * pl + cc - 1);
        g[2] = G[2 * pl + cm];
        g[4] = G[4 * pl + cp];
        g[5] = *(W ? s.gW + Ny + ym : G + 5 * pl + cm - 1);
        g[8] = *(W ? s.gW + 2 * Ny + yp : G + 8 * pl + cp - 1);
        if (E) {
            g[3] = c.w[3] * s.tcin[y] * s.pE[y];
            g[6] = c.w[6] * s.tcin[ym] * s.pE[Ny + ym];
            g[7] = c.w[7] * s.tcin[yp] * s.pE[2 * Ny + yp];
        } else {
            g[3] = G[3 * pl + cc + 1];
            g[6] = G[6 * pl + cm + 1];
            g[7] = G[7 * pl + cp + 1];
        }

        node_f64<TANH, MOM, REF32>(s, c, x, y, cc, E, f, g, ap, am, pc);

#pragma unroll
        for (int k = 0; k < 3; k++) {
            ap[0][k] = ap[1][k]; ap[1][k] = ap[2][k];
            am[0][k] = am[1][k]; am[1][k] = am[2][k];
        }
        pc[0] = pc[1]; pc[1] = pc[2];
    }
}

/* Launch the fused kernel with the template arguments the context selects. */
inline cudaError_t launch_fused_f64_variant(const bgk_ctx *c, dim3 grd, const StepPtrs<double> &s, int H, bool mom)
{
    const bool portable = c->opt.tanh_mode == BGK_TANH_PORTABLE;
    const bool ref32 = !c->opt.smooth;
#define BGK_LAUNCH(T, M, R) fused_f64_kernel<T, M, R><<<grd, FUSED_BX, 0, c->stream>>>(s, c->c, c->corner, H, c->tune_pf)
    if (portable) {
        if (mom) { if (ref32) BGK_LAUNCH(BGK_TANH_PORTABLE, true, true); else BGK_LAUNCH(BGK_TANH_PORTABLE, true, false); }
        else { if (ref32) BGK_LAUNCH(BGK_TANH_PORTABLE, false, true); else BGK_LAUNCH(BGK_TANH_PORTABLE, false, false); }
    } else {
        if (mom) { if (ref32) BGK_LAUNCH(BGK_TANH_DEVICE, true, true); else BGK_LAUNCH(BGK_TANH_DEVICE, true, false); }
        else { if (ref32) BGK_LAUNCH(BGK_TANH_DEVICE, false, true); else BGK_LAUNCH(BGK_TANH_DEVICE, false, false); }
    }
#undef BGK_LAUNCH
    return cudaGetLastError();
}

#endif
