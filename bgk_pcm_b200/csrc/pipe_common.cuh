/*
 * pipe_common.cuh -- building blocks of the shared-memory pipeline kernels
 * (the fused step in fused_pipe.cuh, the adjoint step in adjoint.cu):
 * mbarrier helpers with bounded waits, the bulk global->shared copy, the
 * persistent tile iterator and the tile scheduler.
 *
 * One producer warp (one active lane) per CTA issues cp.async.bulk copies of
 * row segments into a ring of D stages, completion counted in bytes on a
 * per-stage "full" mbarrier; PIPE_CWARPS consumer warps compute from a stage
 * and release it on its "empty" mbarrier.  No clusters, no multicast.
 *
 * Include inside an anonymous namespace, after bgk_internal.h and <atomic>.
 */
#ifndef BGK_PIPE_COMMON_CUH
#define BGK_PIPE_COMMON_CUH

constexpr int PIPE_BX = 128;
constexpr int PIPE_CWARPS = PIPE_BX / 32;
constexpr int PIPE_THREADS = PIPE_BX + 32;
constexpr long long PIPE_WAIT_LIMIT = 1LL << 24;   /* x ~64 ns sleeps: ~1 s */

struct PipeSched {
    int nbands, H, nstrips, ntiles;
    int bx;                 /* band (tile) width in columns */
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok)
                 : "r"(smem_u32(bar)), "r"(parity)
                 : "memory");
    return ok != 0;
}

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

/* Bounded wait: false after ~PIPE_WAIT_LIMIT polls or about a second of
 * wall clock, whichever comes first (a try_wait may itself suspend the
 * thread for a while before it reports an incomplete phase). */
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity)
{
    unsigned long long t0 = 0;
    for (long long i = 0; i < PIPE_WAIT_LIMIT; i++) {
        if (mbar_try_wait(bar, parity)) return true;
        if (i > 32) __nanosleep(64);
        if (i == 1024) t0 = global_ns();
        if (i > 1024 && (i & 1023) == 0 && global_ns() - t0 > 1000000000ull) return false;
    }
    return false;
}

__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

/* Iterate this CTA's work items in order: tiles t = blockIdx.x, +gridDim.x,
 * ..., rows y0..y1-1 of each.  next() returns false at the end.  (Equal
 * contiguous row ranges per CTA instead, which leave no partial last wave,
 * measured 18-28 % slower on B200: concurrently running CTAs then stream
 * rows spread over the whole plane instead of one band of rows.) */
struct PipeIter {
    int t, y, y1, x0;
    PipeSched sch;
    int Ny;
    __device__ bool start(const PipeSched &s, int Ny_)
    {
        sch = s;
        Ny = Ny_;
        t = blockIdx.x;
        return open();
    }
    __device__ bool open()
    {
        if (t >= sch.ntiles) return false;
        const int band = t % sch.nbands, strip = t / sch.nbands;
        x0 = band * sch.bx;
        y = strip * sch.H;
        y1 = min(y + sch.H, Ny);
        return true;
    }
    __device__ bool next()
    {
        if (++y < y1) return true;
        t += gridDim.x;
        return open();
    }
};

/* Tile height: max_H rows, halved down to min_H while there are fewer
 * than 10 tiles per resident CTA, then down to 1 while there are fewer than
 * 4 (small grids, e.g. 512^2 runs best at H = 1).  Taller tiles start fewer
 * phase-field windows and pipeline fills; shorter ones leave a smaller
 * partial last wave.  Measured on B200 (FP64, 200-1000 steps): max_H = 32,
 * min_H = 2 give H = 2 at 1024^2 (17.0 GLUPS against 16.2 with H = 4), 4 at
 * 2048^2 (18.9; 8/16/32: 18.6/17.8/16.5), 16 at 3072^2 and 4096^2 (+1.5 %,
 * +2.7 % over H = 4) and 32 at 16384x4096 (+2.6 %); the reduced-precision
 * forms run best at H = 8 throughout (no max_H: H starts at base_H). */
inline PipeSched pipe_sched(const bgk_ctx *c, int ctas_per_sm, int base_H, int *grid, int max_H = 0,
                            int min_H = 0)
{
    PipeSched sch{};
    sch.bx = PIPE_BX;
    sch.nbands = (c->Nx + PIPE_BX - 1) / PIPE_BX;
    const long long slots = (long long)c->nsm * ctas_per_sm;
    auto tiles = [&](int h) { return (long long)sch.nbands * ((c->Ny + h - 1) / h); };
    int H = max_H > base_H ? max_H : base_H;
    const int lo = min_H > 0 ? min_H : base_H;
    while (H > lo && tiles(H) < 10 * slots) H /= 2;
    while (H > 1 && tiles(H) < 4 * slots) H /= 2;
    if (c->tune_H > 0) H = c->tune_H;
    sch.H = H;
    sch.nstrips = (c->Ny + H - 1) / H;
    sch.ntiles = sch.nbands * sch.nstrips;
    *grid = (int)(sch.ntiles < slots ? sch.ntiles : slots);
    return sch;
}

/* Raise the kernel's dynamic shared-memory limit once per device (the
 * attribute belongs to the device's context).  Devices past 63 set it on
 * every launch. */
template <typename K>
inline cudaError_t pipe_configure(K kernel, size_t smem, int dev, std::atomic<unsigned long long> &done)
{
    const unsigned long long bit = (dev >= 0 && dev < 64) ? (1ull << dev) : 0ull;
    if (bit && (done.load(std::memory_order_acquire) & bit)) return cudaSuccess;
    const cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess && bit) done.fetch_or(bit, std::memory_order_release);
    return e;
}

/* Resident CTAs per SM of a pipeline kernel with `smem` bytes of dynamic
 * shared memory (registers and shared memory decide), queried once per
 * kernel; 0 if the query fails. */
template <typename K>
inline int pipe_occupancy(K kernel, size_t smem, std::atomic<int> &cached)
{
    int n = cached.load(std::memory_order_acquire);
    if (n > 0) return n;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, PIPE_THREADS, smem) != cudaSuccess) {
        (void)cudaGetLastError();
        return 0;
    }
    cached.store(n, std::memory_order_release);
    return n;
}

/* Programmatic dependent launch.  Where it pays (the FP64 step on small
 * grids, the adjoint's reverse step) a pipeline kernel is launched with
 * programmatic stream serialization: its CTAs may be scheduled while the
 * previous kernel on the stream drains, set up their shared memory and
 * mbarriers, and then wait (griddepcontrol.wait) until that kernel has
 * completed and its writes are visible.  Nothing reads or writes global
 * memory before the wait.  A CTA allows the next kernel to be scheduled
 * (griddepcontrol.launch_dependents), which takes effect once every CTA of
 * this grid has done so or exited.  Under a plain launch both instructions
 * are no-ops. */
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_allow_next() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

template <typename... KArgs, typename... Args>
inline cudaError_t pdl_launch(void (*kernel)(KArgs...), int grid, int block, size_t smem, cudaStream_t st,
                              Args &&...args)
{
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3((unsigned)block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

/* ------------------------------------------------------------------------
 * Multi-step (dataflow) pipeline kernels (the FP64 step in fused_pipe.cuh,
 * the reduced-precision forms in kernels_fast.cu).
 *
 * One launch advances nsteps steps, so the grid does not drain and refill
 * at every step boundary.  Work items are (step k, tile t) in step-major
 * order, taken from a ticket counter by the producer of whichever CTA is
 * free.  An item may start once the 3x3 tile neighbourhood of t has
 * completed step k-1 (done[t'] >= k).  That covers every value the item
 * reads -- pull rows y +- 1, the phase-field stencil, the 16-byte pads into
 * the neighbouring bands, the east T column at rows y +- 1 -- and, because
 * the two buffers alternate, every value it overwrites: its own rows of the
 * buffer that step k-1 pulled from, which only items of that neighbourhood
 * read.  Every dependency holds a smaller ticket, claimed by a running CTA,
 * so the smallest unfinished ticket can always proceed and the schedule
 * needs no co-residency.
 *
 * Ordering: each consumer warp's stores of a tile are fenced (a warp
 * barrier, then membar.gl by one lane) before the last of its four warps
 * releases done[t] (a one-step launch has no readers and skips this); a producer acquires the
 * flags, then orders the bulk copies (async proxy) after that with
 * fence.proxy.async, and hands the stage to its consumers through the
 * stage's mbarrier.  Every wait is bounded; on expiry the error flag is set
 * and every CTA leaves.
 * ---------------------------------------------------------------------- */
struct FlowCtl {
    unsigned long long *ticket; /* next work item (zero at launch)         */
    unsigned *done;     /* [ntiles]: steps completed by each tile (zero)   */
    int nsteps;
    unsigned stall;     /* added to every dependency target: 0, or (to test
                         * the error path) a count no tile reaches        */
};
struct StageTag {
    int k, t, y, flags;
};
constexpr int TAG_FIRST = 1, TAG_LAST = 2, TAG_END = 4;

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned *p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_u32(unsigned *p, unsigned v)
{
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void fence_proxy_async_global() { asm volatile("fence.proxy.async.global;" ::: "memory"); }

/* Wait (bounded) until every tile of the 3x3 neighbourhood of t has done
 * `need` steps; false on expiry or once another CTA raised the error flag.
 * The nine counts are read together (relaxed, one round trip to L2 per
 * poll); once all suffice, an acquire fence orders what follows after the
 * stores that the counts publish. */
__device__ __forceinline__ unsigned ld_relaxed_u32(const unsigned *p)
{
    unsigned v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void fence_acquire_gpu() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }

__device__ bool flow_deps(const unsigned *done, int t, const PipeSched &sch, unsigned need, const int *errflag)
{
    const int b = t % sch.nbands, st = t / sch.nbands;
    const unsigned *p[9];
    int n = 0;
    for (int ds = -1; ds <= 1; ds++) {
        const int ss = st + ds;
        if (ss < 0 || ss >= sch.nstrips) continue;
        for (int db = -1; db <= 1; db++) {
            const int bb = b + db;
            if (bb < 0 || bb >= sch.nbands) continue;
            p[n++] = done + (long long)ss * sch.nbands + bb;
        }
    }
    const unsigned long long t0 = global_ns();
    for (long long i = 0;; i++) {
        unsigned v[9];
#pragma unroll
        for (int q = 0; q < 9; q++)
            if (q < n) v[q] = ld_relaxed_u32(p[q]);
        bool ok = true;
#pragma unroll
        for (int q = 0; q < 9; q++)
            if (q < n && v[q] < need) ok = false;
        if (ok) break;
        if (i > PIPE_WAIT_LIMIT) return false;
        if ((i & 255) == 255 && (*(volatile const int *)errflag || global_ns() - t0 > 1000000000ull)) return false;
        if (i > 32) __nanosleep(64);
    }
    fence_acquire_gpu();
    return true;
}

#endif
