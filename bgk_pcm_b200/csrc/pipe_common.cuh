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

/* Bounded wait: false after ~PIPE_WAIT_LIMIT polls. */
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity)
{
    for (long long i = 0; i < PIPE_WAIT_LIMIT; i++) {
        if (mbar_try_wait(bar, parity)) return true;
        if (i > 32) __nanosleep(64);
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
 * ..., rows y0..y1-1 of each.  next() returns false at the end. */
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

/* Tile height: base_H rows (measured best on B200: 4 for FP64, 8 for the
 * reduced-precision forms; taller tiles leave a partial last wave, shorter
 * ones lose a little per tile), halved down to 1 while there are fewer than
 * 4 tiles per resident CTA (small grids, e.g. 512^2 runs best at H = 1). */
inline PipeSched pipe_sched(const bgk_ctx *c, int ctas_per_sm, int base_H, int *grid)
{
    PipeSched sch;
    sch.bx = PIPE_BX;
    sch.nbands = (c->Nx + PIPE_BX - 1) / PIPE_BX;
    const long long slots = (long long)c->nsm * ctas_per_sm;
    int H = base_H;
    while (H > 1 && (long long)sch.nbands * ((c->Ny + H - 1) / H) < 4 * slots) H /= 2;
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

#endif
