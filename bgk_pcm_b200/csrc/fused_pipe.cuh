/*
 * fused_pipe.cuh -- the fused step with a shared-memory pipeline.
 *
 * The register-pull kernel (fused_f64.cuh) issues its 18 population loads and
 * then computes: with ~128 registers per thread only ~16 warps fit on an SM,
 * and the loads of a warp are not in flight while it computes, so the kernel
 * is latency-bound below the HBM roofline.  Here the loads are decoupled:
 *
 *  - one producer warp per CTA streams, for each row the CTA will compute,
 *    the 18 population row-segments (f and g planes, each at its pull source
 *    row y - c_y, clamped into the domain) and the next phi row into a ring of
 *    D shared-memory stages with bulk asynchronous copies (cp.async.bulk,
 *    completion counted in bytes on a per-stage mbarrier);
 *  - four consumer warps (one node per thread) wait for a stage, pull their
 *    populations from shared memory (x +/- 1 is a neighbouring word, no
 *    misaligned global access), compute the node with the same device
 *    function as the register-pull kernel (node_f64), write the results and
 *    release the stage on a second mbarrier.
 * A CTA owns tiles of 128 columns x H rows (persistent, round-robin); the
 * producer runs D rows ahead across tile boundaries.  Row segments start 16
 * bytes before the band (the population buffers carry 256-byte guards), so
 * every copy is 16-byte aligned.  Boundary nodes read their bounce-back and
 * boundary values from global memory, as in the register-pull kernel.
 *
 * Every wait is bounded (about a second); on expiry the thread records a code
 * in errflag and leaves its loop, and the producer waits (bounded) for all of
 * its copies before it exits.  No multicast, no clusters.
 *
 * Include inside an anonymous namespace in namespace bgk after fused_f64.cuh.
 */
#ifndef BGK_FUSED_PIPE_CUH
#define BGK_FUSED_PIPE_CUH

#include "pipe_common.cuh"

/* Stage geometry for storage type S (populations) and PT (phi). */
template <typename S, typename PT>
struct PipeGeom {
    static constexpr int AL = 16 / (int)sizeof(S);       /* left pad (elements) */
    static constexpr int RW = PIPE_BX + 2 * AL;
    static constexpr int ALP = 16 / (int)sizeof(PT);
    static constexpr int RWP = PIPE_BX + 2 * ALP;
    static constexpr int POP_BYTES = RW * (int)sizeof(S);
    static constexpr int PHI_BYTES = RWP * (int)sizeof(PT);
    static constexpr int STAGE_BYTES = (18 * POP_BYTES + PHI_BYTES + 127) / 128 * 128;
    static constexpr int TX_BYTES = 18 * POP_BYTES + PHI_BYTES;
    static constexpr int HEADER = 256;                    /* mbarriers (2 x 16 max) */
    static size_t smem_bytes(int D) { return (size_t)HEADER + (size_t)D * STAGE_BYTES; }
    /* dataflow stages also carry a tile's first two window rows of phi */
    static constexpr int STAGE_BYTES_W = (18 * POP_BYTES + 3 * PHI_BYTES + 127) / 128 * 128;
    static size_t smem_bytes_w(int D) { return (size_t)HEADER + (size_t)D * STAGE_BYTES_W; }
};

__constant__ int pipe_cy[9] = {0, 0, 1, 0, -1, 1, 1, -1, -1};

/* Producer: issue the 19 row-segment copies of work item (x0, y) into a stage. */
template <typename S, typename PT>
__device__ __forceinline__ void pipe_issue(const S *F, const S *G, const PT *PH, long long pl, int P, int Ny, int x0,
                                           int y, unsigned char *stage, uint64_t *full)
{
    using Gm = PipeGeom<S, PT>;
    mbar_arrive_expect_tx(full, Gm::TX_BYTES);
#pragma unroll 1
    for (int k = 0; k < 9; k++) {
        int r = y - pipe_cy[k];
        r = r < 0 ? 0 : (r >= Ny ? Ny - 1 : r);
        const long long off = (long long)r * P + x0 - Gm::AL;
        bulk_g2s(stage + k * Gm::POP_BYTES, F + k * pl + off, Gm::POP_BYTES, full);
        bulk_g2s(stage + (9 + k) * Gm::POP_BYTES, G + k * pl + off, Gm::POP_BYTES, full);
    }
    const int rp = (y + 1 >= Ny) ? Ny - 1 : y + 1;
    bulk_g2s(stage + 18 * Gm::POP_BYTES, PH + (long long)rp * P + x0 - Gm::ALP, Gm::PHI_BYTES, full);
}

/* Pipeline consumers of the FP64 step, shared by the per-step kernel and
 * the multi-step (dataflow) kernel.
 *
 * f64_window_start: the selector terms of the phase-field window's first
 * two rows (y0-1, y0) for column x, from global memory. */
__device__ __forceinline__ void f64_window_start(const StepPtrs<double> &s, int Ny, int x, int y0, bool W, bool E,
                                                 double (&ap)[3][3], double (&am)[3][3], double *pc)
{
    for (int slot = 0; slot < 2; slot++) {
        const int rr = y0 - 1 + slot;
        const int rc = rr < 0 ? 0 : (rr >= Ny ? Ny - 1 : rr);
        const double *row = s.phin + (long long)rc * s.P;
        const double pL = W ? s.phiW[rc] : row[x - 1];
        const double pM = row[x];
        const double pR = E ? s.phiE[rc] : row[x + 1];
        ap[slot][0] = aplus(pL); ap[slot][1] = aplus(pM); ap[slot][2] = aplus(pR);
        am[slot][0] = aminus(pL); am[slot][1] = aminus(pM); am[slot][2] = aminus(pR);
        pc[slot] = pM;
    }
}

/* f64_row: node (x, y) from a filled stage -- the window's new row y+1,
 * the pulls (bounce-back, or the halo ring with other wall codes, and the
 * g boundary values), node_f64, and the window shift. */
template <int TANH, bool MOM, bool REF32, bool RING, bool EH = false>
__device__ __forceinline__ void f64_row(const StepPtrs<double> &s, const Consts &c, const double *__restrict__ corner,
                                        const unsigned char *stage, int x, int y, int tid, bool W, bool E,
                                        double (&ap)[3][3], double (&am)[3][3], double *pc)
{
    using Gm = PipeGeom<double, double>;
    const int Nx = c.Nx, Ny = c.Ny;
    const long long pl = s.plane;
    const double *__restrict__ F = s.fin;
    const double *stg = reinterpret_cast<const double *>(stage);
    const double *sp = stg;                                    /* f planes */
    const double *sg = stg + 9 * Gm::RW;                       /* g planes */
    const double *sphi = stg + 18 * Gm::RW;
    const bool S = (y == 0), N = (y == Ny - 1);
    const long long cc = (long long)y * s.P + x;
    const int col = tid + Gm::AL;
    /* new phi row y+1 of the window */
    {
        const int rc = (y + 1 >= Ny) ? Ny - 1 : y + 1;
        const double pL = W ? s.phiW[rc] : sphi[Gm::ALP + tid - 1];
        const double pM = sphi[Gm::ALP + tid];
        const double pR = E ? s.phiE[rc] : sphi[Gm::ALP + tid + 1];
        ap[2][0] = aplus(pL); ap[2][1] = aplus(pM); ap[2][2] = aplus(pR);
        am[2][0] = aminus(pL); am[2][1] = aminus(pM); am[2][2] = aminus(pR);
        pc[2] = pM;
    }
    double f[9], g[9];
    f[0] = sp[0 * Gm::RW + col];
    f[1] = W ? sp[3 * Gm::RW + col] : sp[1 * Gm::RW + col - 1];
    f[2] = sp[2 * Gm::RW + col];
    f[3] = E ? sp[1 * Gm::RW + col] : sp[3 * Gm::RW + col + 1];
    f[4] = sp[4 * Gm::RW + col];
    f[5] = sp[5 * Gm::RW + col - 1];
    f[6] = sp[6 * Gm::RW + col + 1];
    f[7] = sp[7 * Gm::RW + col + 1];
    f[8] = sp[8 * Gm::RW + col - 1];
    if (RING) {
        /* pulls from outside the domain read the halo ring, which the
         * boundary kernel filled as BC_f does */
        if (W || E || S || N) {
            const double *R = s.ring;
            const long long RL = s.ring_len;
            const int i = x + 1, j = y + 1;
            if (W) f[1] = R[1 * RL + ring_idx(Nx, Ny, 0, j)];
            if (S) f[2] = R[2 * RL + ring_idx(Nx, Ny, i, 0)];
            if (E) f[3] = R[3 * RL + ring_idx(Nx, Ny, Nx + 1, j)];
            if (N) f[4] = R[4 * RL + ring_idx(Nx, Ny, i, Ny + 1)];
            if (W || S) f[5] = R[5 * RL + ring_idx(Nx, Ny, i - 1, j - 1)];
            if (E || S) f[6] = R[6 * RL + ring_idx(Nx, Ny, i + 1, j - 1)];
            if (E || N) f[7] = R[7 * RL + ring_idx(Nx, Ny, i + 1, j + 1)];
            if (W || N) f[8] = R[8 * RL + ring_idx(Nx, Ny, i - 1, j + 1)];
        }
    } else if (W || E || S || N) {
        /* bounce-back values that are not in the stage */
        if (S) f[2] = F[4 * pl + cc];
        if (N) f[4] = F[2 * pl + cc];
        if (W || S) f[5] = F[7 * pl + cc];
        if (E || S) f[6] = (E && S) ? corner[0] : F[8 * pl + cc];
        if (E || N) f[7] = (E && N) ? corner[1] : F[5 * pl + cc];
        if (W || N) f[8] = F[6 * pl + cc];
    }
    const int ym = S ? y : y - 1, yp = N ? y : y + 1;
    g[0] = sg[0 * Gm::RW + col];
    g[2] = sg[2 * Gm::RW + col];
    g[4] = sg[4 * Gm::RW + col];
    if (W) {
        g[1] = s.gW[y];
        g[5] = s.gW[Ny + ym];
        g[8] = s.gW[2 * Ny + yp];
    } else {
        g[1] = sg[1 * Gm::RW + col - 1];
        g[5] = sg[5 * Gm::RW + col - 1];
        g[8] = sg[8 * Gm::RW + col - 1];
    }
    if (E) {
        g[3] = c.w[3] * s.tcin[y] * s.pE[y];
        g[6] = c.w[6] * s.tcin[ym] * s.pE[Ny + ym];
        g[7] = c.w[7] * s.tcin[yp] * s.pE[2 * Ny + yp];
    } else {
        g[3] = sg[3 * Gm::RW + col + 1];
        g[6] = sg[6 * Gm::RW + col + 1];
        g[7] = sg[7 * Gm::RW + col + 1];
    }
    node_f64<TANH, MOM, REF32, RING, EH>(s, c, x, y, cc, E, f, g, ap, am, pc, W || E || S || N, W, S, N);
#pragma unroll
    for (int k = 0; k < 3; k++) {
        ap[0][k] = ap[1][k]; ap[1][k] = ap[2][k];
        am[0][k] = am[1][k]; am[1][k] = am[2][k];
    }
    pc[0] = pc[1]; pc[1] = pc[2];
}

/* Dataflow producer: as pipe_issue, and on a tile's first row y also the
 * phi rows y-1 (clamped) and y, the window the consumers start the tile
 * with, into the stage's two extra row slots. */
template <typename S, typename PT>
__device__ __forceinline__ void pipe_issue_w(const S *F, const S *G, const PT *PH, long long pl, int P, int Ny,
                                             int x0, int y, bool first, unsigned char *stage, uint64_t *full)
{
    using Gm = PipeGeom<S, PT>;
    mbar_arrive_expect_tx(full, Gm::TX_BYTES + (first ? 2 * Gm::PHI_BYTES : 0));
#pragma unroll 1
    for (int k = 0; k < 9; k++) {
        int r = y - pipe_cy[k];
        r = r < 0 ? 0 : (r >= Ny ? Ny - 1 : r);
        const long long off = (long long)r * P + x0 - Gm::AL;
        bulk_g2s(stage + k * Gm::POP_BYTES, F + k * pl + off, Gm::POP_BYTES, full);
        bulk_g2s(stage + (9 + k) * Gm::POP_BYTES, G + k * pl + off, Gm::POP_BYTES, full);
    }
    const int rp = (y + 1 >= Ny) ? Ny - 1 : y + 1;
    unsigned char *sphi = stage + 18 * Gm::POP_BYTES;
    bulk_g2s(sphi, PH + (long long)rp * P + x0 - Gm::ALP, Gm::PHI_BYTES, full);
    if (first) {
        const int rm = y > 0 ? y - 1 : 0;
        bulk_g2s(sphi + Gm::PHI_BYTES, PH + (long long)rm * P + x0 - Gm::ALP, Gm::PHI_BYTES, full);
        bulk_g2s(sphi + 2 * Gm::PHI_BYTES, PH + (long long)y * P + x0 - Gm::ALP, Gm::PHI_BYTES, full);
    }
}

/* The FP64 window's first two rows from a dataflow stage (slots 1 and 2). */
__device__ __forceinline__ void f64_window_stage(const StepPtrs<double> &s, int Ny, int y0, int tid, bool W, bool E,
                                                 const unsigned char *stage, double (&ap)[3][3], double (&am)[3][3],
                                                 double *pc)
{
    using Gm = PipeGeom<double, double>;
    for (int slot = 0; slot < 2; slot++) {
        const int rr = y0 - 1 + slot;
        const int rc = rr < 0 ? 0 : (rr >= Ny ? Ny - 1 : rr);
        const double *row = reinterpret_cast<const double *>(stage + 18 * Gm::POP_BYTES + (1 + slot) * Gm::PHI_BYTES);
        const double pL = W ? s.phiW[rc] : row[Gm::ALP + tid - 1];
        const double pM = row[Gm::ALP + tid];
        const double pR = E ? s.phiE[rc] : row[Gm::ALP + tid + 1];
        ap[slot][0] = aplus(pL); ap[slot][1] = aplus(pM); ap[slot][2] = aplus(pR);
        am[slot][0] = aminus(pL); am[slot][1] = aminus(pM); am[slot][2] = aminus(pR);
        pc[slot] = pM;
    }
}

template <int D, int TANH, bool MOM, bool REF32, bool RING = false, bool EH = false>
__global__ void __launch_bounds__(PIPE_THREADS, 3)
fused_pipe_f64_kernel(StepPtrs<double> s, Consts c, const double *__restrict__ corner, PipeSched sch, int *errflag)
{
    using Gm = PipeGeom<double, double>;
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
    pdl_allow_next();
    pdl_wait();

    if (warp == PIPE_CWARPS) {
        /* ---------------- producer ---------------- */
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
            pipe_issue<double, double>(s.fin, s.gin, s.phin, s.plane, s.P, Ny, it.x0, it.y,
                                       stages + (size_t)st * Gm::STAGE_BYTES, &full[st]);
            r++;
            ok = it.next();
        }
        /* do not retire while copies into this CTA's shared memory are in flight */
        for (long long q = (r > D ? r - D : 0); q < r; q++)
            if (!mbar_wait(&full[q % D], (uint32_t)((q / D) & 1))) atomicExch(errflag, 2);
        return;
    }

    /* ---------------- consumers ---------------- */
    PipeIter it;
    long long r = 0;
    bool ok = it.start(sch, Ny);
    while (ok) {
        const int x = it.x0 + tid;
        const bool active = x < Nx;
        const bool W = (x == 0), E = (x == Nx - 1);
        double ap[3][3], am[3][3], pc[3];
        if (active) f64_window_start(s, Ny, x, it.y, W, E, ap, am, pc);
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
                f64_row<TANH, MOM, REF32, RING, EH>(s, c, corner, stages + (size_t)st * Gm::STAGE_BYTES, x, y, tid, W,
                                                    E, ap, am, pc);
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty[st]);
            r++;
            ok = it.next();
        } while (ok && it.t == tile);
        if (failed) break;
    }
}

/* The FP64 step as a multi-step (dataflow) launch: the schedule of FlowCtl
 * (pipe_common.cuh) over the consumers above, walls of code 4, no moments;
 * s0 steps buffer A to B, s1 steps B to A. */
template <int D, int TANH, bool REF32>
__global__ void __launch_bounds__(PIPE_THREADS, 3)
flow_pipe_f64_kernel(StepPtrs<double> s0, StepPtrs<double> s1, Consts c, const double *__restrict__ corner,
                     PipeSched sch, FlowCtl fl, int *errflag)
{
    static_assert(D <= 8, "stage tags hold 8 stages");
    using Gm = PipeGeom<double, double>;
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
            const StepPtrs<double> &sk = (k & 1) ? s1 : s0;
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
                pipe_issue_w<double, double>(sk.fin, sk.gin, sk.phin, sk.plane, sk.P, Ny, x0, y, y == y0,
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
    double ap[3][3], am[3][3], pc[3];
    for (long long r = 0;; r++) {
        const int st = (int)(r % D);
        if (!__all_sync(0xffffffffu, mbar_wait(&full[st], (uint32_t)((r / D) & 1)))) {
            atomicExch(errflag, 3);
            break;
        }
        const StageTag tg = tag[st];
        if (tg.flags & TAG_END) break;
        const StepPtrs<double> &sk = (tg.k & 1) ? s1 : s0;
        const int x = (tg.t % sch.nbands) * sch.bx + tid;
        const bool W = (x == 0), E = (x == Nx - 1);
        if (x < Nx) {
            const unsigned char *stg = stages + (size_t)st * Gm::STAGE_BYTES_W;
            if (tg.flags & TAG_FIRST) f64_window_stage(sk, Ny, tg.y, tid, W, E, stg, ap, am, pc);
            f64_row<TANH, false, REF32, false>(sk, c, corner, stg, x, tg.y, tid, W, E, ap, am, pc);
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

/* nsteps FP64 steps in one dataflow launch (walls of code 4, no moments).
 * flow_buf: the context's ticket counter and per-tile step counts. */
template <int T, bool R>
inline cudaError_t flow_f64_launch_t(bgk_ctx *c, const StepPtrs<double> &s0, const StepPtrs<double> &s1, int nsteps)
{
    constexpr int D = 2;
    using Gm = PipeGeom<double, double>;
    const size_t smem = Gm::smem_bytes_w(D);
    static std::atomic<unsigned long long> done{0};
    cudaError_t e = pipe_configure(flow_pipe_f64_kernel<D, T, R>, smem, c->dev, done);
    if (e != cudaSuccess) return e;
    int grid;
    const PipeSched sch = pipe_sched(c, c->tune_ctas > 0 ? c->tune_ctas : 3, 4, &grid);
    const size_t need = sizeof(unsigned long long) + (size_t)sch.ntiles * sizeof(unsigned);
    if (c->flow_bytes < need) {
        if (c->flow_buf) cudaFree(c->flow_buf);
        c->flow_buf = nullptr;
        c->flow_bytes = 0;
        if ((e = cudaMalloc(&c->flow_buf, need)) != cudaSuccess) return e;
        c->flow_bytes = need;
    }
    if ((e = cudaMemsetAsync(c->flow_buf, 0, need, c->stream)) != cudaSuccess) return e;
    FlowCtl fl;
    fl.ticket = (unsigned long long *)c->flow_buf;
    fl.done = (unsigned *)((char *)c->flow_buf + sizeof(unsigned long long));
    fl.nsteps = nsteps;
    fl.stall = c->flow_stall ? (1u << 30) : 0u;
    flow_pipe_f64_kernel<D, T, R><<<grid, PIPE_THREADS, smem, c->stream>>>(s0, s1, c->c, c->corner, sch, fl,
                                                                          c->errflag);
    return cudaGetLastError();
}

inline cudaError_t launch_flow_pipe_f64(bgk_ctx *c, const StepPtrs<double> &s0, const StepPtrs<double> &s1,
                                        int nsteps)
{
    const bool portable = c->opt.tanh_mode == BGK_TANH_PORTABLE;
    const bool ref32 = !c->opt.smooth;
    if (portable)
        return ref32 ? flow_f64_launch_t<BGK_TANH_PORTABLE, true>(c, s0, s1, nsteps)
                     : flow_f64_launch_t<BGK_TANH_PORTABLE, false>(c, s0, s1, nsteps);
    return ref32 ? flow_f64_launch_t<BGK_TANH_DEVICE, true>(c, s0, s1, nsteps)
                 : flow_f64_launch_t<BGK_TANH_DEVICE, false>(c, s0, s1, nsteps);
}

template <int D, int T, bool M, bool R, bool RING = false, bool EH = false>
inline cudaError_t pipe_f64_launch(const bgk_ctx *c, const StepPtrs<double> &s, int ctas)
{
    using Gm = PipeGeom<double, double>;
    const size_t smem = Gm::smem_bytes(D);
    static std::atomic<unsigned long long> done{0};
    const cudaError_t e = pipe_configure(fused_pipe_f64_kernel<D, T, M, R, RING, EH>, smem, c->dev, done);
    if (e != cudaSuccess) return e;
    int grid;
    const PipeSched sch = pipe_sched(c, ctas, 4, &grid, 32, 2);
    /* programmatic dependent launch on grids of up to 2^21 nodes, whose
     * steps are short enough (tens of microseconds) for the launch gap to
     * matter: +9 % at 512^2; on larger grids it measured ~1 % slower */
    if ((long long)c->Nx * c->Ny <= (1LL << 21))
        return pdl_launch(fused_pipe_f64_kernel<D, T, M, R, RING, EH>, grid, PIPE_THREADS, smem, c->stream, s, c->c,
                          (const double *)c->corner, sch, c->errflag);
    fused_pipe_f64_kernel<D, T, M, R, RING, EH><<<grid, PIPE_THREADS, smem, c->stream>>>(s, c->c, c->corner, sch,
                                                                                       c->errflag);
    return cudaGetLastError();
}

/* Walls other than code 4: two stages (the default depth), the halo ring. */
inline cudaError_t pipe_f64_ring_dispatch(const bgk_ctx *c, const StepPtrs<double> &s, bool mom, int ctas)
{
    const bool portable = c->opt.tanh_mode == BGK_TANH_PORTABLE;
    const bool ref32 = !c->opt.smooth;
    if (portable) {
        if (mom) return ref32 ? pipe_f64_launch<2, BGK_TANH_PORTABLE, true, true, true>(c, s, ctas)
                              : pipe_f64_launch<2, BGK_TANH_PORTABLE, true, false, true>(c, s, ctas);
        return ref32 ? pipe_f64_launch<2, BGK_TANH_PORTABLE, false, true, true>(c, s, ctas)
                     : pipe_f64_launch<2, BGK_TANH_PORTABLE, false, false, true>(c, s, ctas);
    }
    if (mom) return ref32 ? pipe_f64_launch<2, BGK_TANH_DEVICE, true, true, true>(c, s, ctas)
                          : pipe_f64_launch<2, BGK_TANH_DEVICE, true, false, true>(c, s, ctas);
    return ref32 ? pipe_f64_launch<2, BGK_TANH_DEVICE, false, true, true>(c, s, ctas)
                 : pipe_f64_launch<2, BGK_TANH_DEVICE, false, false, true>(c, s, ctas);
}

template <int D>
inline cudaError_t pipe_f64_dispatch(const bgk_ctx *c, const StepPtrs<double> &s, bool mom, int ctas, bool eh)
{
    const bool portable = c->opt.tanh_mode == BGK_TANH_PORTABLE;
    const bool ref32 = !c->opt.smooth;
    if (eh && !mom) {
        if (portable)
            return ref32 ? pipe_f64_launch<D, BGK_TANH_PORTABLE, false, true, false, true>(c, s, ctas)
                         : pipe_f64_launch<D, BGK_TANH_PORTABLE, false, false, false, true>(c, s, ctas);
        return ref32 ? pipe_f64_launch<D, BGK_TANH_DEVICE, false, true, false, true>(c, s, ctas)
                     : pipe_f64_launch<D, BGK_TANH_DEVICE, false, false, false, true>(c, s, ctas);
    }
    if (portable) {
        if (mom) return ref32 ? pipe_f64_launch<D, BGK_TANH_PORTABLE, true, true>(c, s, ctas)
                              : pipe_f64_launch<D, BGK_TANH_PORTABLE, true, false>(c, s, ctas);
        return ref32 ? pipe_f64_launch<D, BGK_TANH_PORTABLE, false, true>(c, s, ctas)
                     : pipe_f64_launch<D, BGK_TANH_PORTABLE, false, false>(c, s, ctas);
    }
    if (mom) return ref32 ? pipe_f64_launch<D, BGK_TANH_DEVICE, true, true>(c, s, ctas)
                          : pipe_f64_launch<D, BGK_TANH_DEVICE, true, false>(c, s, ctas);
    return ref32 ? pipe_f64_launch<D, BGK_TANH_DEVICE, false, true>(c, s, ctas)
                 : pipe_f64_launch<D, BGK_TANH_DEVICE, false, false>(c, s, ctas);
}

/* Pipeline depth 2..4 stages of ~20 KB.  Measured on B200 at 2048^2 and
 * 4096^2: 2 stages with 3 CTAs per SM (12 consumer warps) is best (92 % /
 * 88 % of the copy bandwidth); more stages or CTAs lose occupancy or issue
 * slots. */
inline cudaError_t launch_fused_pipe_f64(const bgk_ctx *c, const StepPtrs<double> &s, bool mom, bool eh = false)
{
    if (c->ring) return pipe_f64_ring_dispatch(c, s, mom, c->tune_ctas > 0 ? c->tune_ctas : 3);
    const int D = c->tune_D > 0 ? c->tune_D : 2;
    const int ctas = c->tune_ctas > 0 ? c->tune_ctas : (D <= 2 ? 3 : 2);
    switch (D) {
    case 2: return pipe_f64_dispatch<2>(c, s, mom, ctas, eh);
    case 4: return pipe_f64_dispatch<4>(c, s, mom, ctas, eh);
    default: return pipe_f64_dispatch<3>(c, s, mom, ctas, eh);
    }
}

#endif
