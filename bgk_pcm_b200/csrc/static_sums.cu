/*
 * static_sums.cu -- bgk_field_sums_static: the interior FP64 sums of
 * bgk_field_sums (STEP_7/field_check.f90:9-17, STEP_7/diag.f90:82-91) over
 * device fields the caller owns, with no allocation of any kind.
 *
 * Two launches on the caller's stream:
 *   1. row_sums_kernel   one 128-thread block per interior row j writes the
 *                        row's four sums into the static row-partials array;
 *   2. rows_final_kernel one block adds the row partials in a fixed order and
 *                        writes out[0..3].
 * The order of every addition is fixed by Nx and Ny alone, so a call is
 * deterministic.  It is not the order of bgk_field_sums (a fixed 592-block
 * grid), so the two agree to rounding, not bit for bit.
 *
 * Scratch: g_row_partials, a file-scope __device__ array of
 * 4 * BGK_STATIC_SUMS_MAX_NY doubles (1 MiB per device).  Its device address
 * is looked up with cudaGetSymbolAddress on the first call in each CUDA
 * context of a device and cached under that context's unique id, so a
 * context that replaces the old one (cudaDeviceReset, or a caller's own
 * driver-API context) gets its own lookup instead of a stale address.  Every
 * slot a call reads was written earlier by the same call, so no part of the
 * scratch has to start at zero and nothing is cleared between calls.  All
 * calls on one device share the array: calls that can overlap in time race.
 */
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <mutex>

#include <cuda.h>            /* driver types only; entry points come from the runtime */
#include <cuda_runtime.h>

#include "bgk_pcm.h"
#include "bgk_internal.h"

namespace {

constexpr int ROW_THREADS = 128;
constexpr int FINAL_THREADS = 256;          /* 64 threads per sum */
constexpr int MAX_DEVICES = 64;

static __device__ __align__(256) double g_row_partials[4 * BGK_STATIC_SUMS_MAX_NY];

/* The scratch address per device, valid for the context it was looked up in. */
struct ScratchAddr {
    unsigned long long ctx_id = 0;
    double *ptr = nullptr;
};
ScratchAddr g_partials_addr[MAX_DEVICES];
std::mutex g_partials_mu;

/* Unique id of the calling thread's current CUDA context (0 if none), via
 * the driver entry points the runtime hands out, so the library needs no
 * link dependency on the driver library. */
unsigned long long current_ctx_id()
{
    using GetCurrent = CUresult (*)(CUcontext *);
    using GetId = CUresult (*)(CUcontext, unsigned long long *);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<GetCurrent>(f);
        f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<GetId>(f);
        cudaGetLastError();
    });
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (!get_current || !get_id || get_current(&ctx) != CUDA_SUCCESS || !ctx) return 0;
    if (get_id(ctx, &id) != CUDA_SUCCESS) return 0;
    return id;
}

/* The scratch address in the current context of device dev: looked up on
 * the first call in that context, cached afterwards. */
int scratch_address(int dev, double **out)
{
    std::lock_guard<std::mutex> lock(g_partials_mu);
    ScratchAddr &a = g_partials_addr[dev];
    const unsigned long long id = current_ctx_id();
    if (a.ptr && id != 0 && a.ctx_id == id) {
        *out = a.ptr;
        return BGK_OK;
    }
    void *addr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&addr, g_row_partials);
    if (e != cudaSuccess || !addr) {
        cudaGetLastError();
        char msg[200];
        std::snprintf(msg, sizeof msg, "bgk_field_sums_static: cudaGetSymbolAddress failed: %s",
                      cudaGetErrorString(e));
        return bgk_internal_fail(BGK_ERR_CUDA, msg);
    }
    /* the lookup makes the context current if nothing was; cache under its id
     * (an id of 0, no context known, is never a cache hit) */
    a.ctx_id = id != 0 ? id : current_ctx_id();
    a.ptr = static_cast<double *>(addr);
    *out = a.ptr;
    return BGK_OK;
}

__device__ __forceinline__ double warp_total(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

/* Block j-1 sums interior row j; part is laid out [4][Ny]. */
__global__ void __launch_bounds__(ROW_THREADS)
row_sums_kernel(const double *rho, const double *T, const double *phi, int Nx, int Ny, long long ld,
                double *part)
{
    const int j = blockIdx.x + 1;
    const size_t row = (size_t)j * (size_t)ld;
    double a = 0.0, b = 0.0, p = 0.0, k = 0.0;
    for (int i = threadIdx.x + 1; i <= Nx; i += ROW_THREADS) {
        a += rho[row + i];
        b += T[row + i];
        const double ph = phi[row + i];
        p += ph;
        k += (ph > 0.0) ? 1.0 : 0.0;
    }
    __shared__ double sh[4][ROW_THREADS / 32];
    a = warp_total(a); b = warp_total(b); p = warp_total(p); k = warp_total(k);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) { sh[0][wid] = a; sh[1][wid] = b; sh[2][wid] = p; sh[3][wid] = k; }
    __syncthreads();
    if (threadIdx.x < 4) {
        double acc = 0.0;
        for (int w = 0; w < ROW_THREADS / 32; w++) acc += sh[threadIdx.x][w];
        part[(size_t)threadIdx.x * Ny + (j - 1)] = acc;
    }
}

/* Threads 64r..64r+63 add the Ny partials of sum r. */
__global__ void __launch_bounds__(FINAL_THREADS)
rows_final_kernel(const double *part, int Ny, double *out)
{
    const int r = threadIdx.x >> 6, l = threadIdx.x & 63;
    double acc = 0.0;
    for (int j = l; j < Ny; j += 64) acc += part[(size_t)r * Ny + j];
    acc = warp_total(acc);
    __shared__ double sh[FINAL_THREADS / 32];
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 4) out[threadIdx.x] = sh[2 * threadIdx.x] + sh[2 * threadIdx.x + 1];
}

int fail(int code, const char *fmt, long long a = 0, long long b = 0)
{
    char msg[256];
    std::snprintf(msg, sizeof msg, fmt, a, b);
    return bgk_internal_fail(code, msg);
}

/* Device memory of the current device (or managed memory) only: a pageable
 * host pointer would fault inside the kernel. */
int check_device_pointer(const void *ptr, int dev, const char *name)
{
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, ptr) != cudaSuccess) {
        cudaGetLastError();
        char msg[160];
        std::snprintf(msg, sizeof msg, "bgk_field_sums_static: %s is not a CUDA pointer", name);
        return bgk_internal_fail(BGK_ERR_ARG, msg);
    }
    const bool ok = at.type == cudaMemoryTypeManaged || (at.type == cudaMemoryTypeDevice && at.device == dev);
    if (!ok) {
        char msg[160];
        std::snprintf(msg, sizeof msg, "bgk_field_sums_static: %s is not device memory of the current device",
                      name);
        return bgk_internal_fail(BGK_ERR_ARG, msg);
    }
    return BGK_OK;
}

} // namespace

extern "C" int bgk_field_sums_static(const double *rho, const double *T, const double *phi, int Nx, int Ny,
                                     int ld, void *stream, double *out)
{
    if (!rho || !T || !phi || !out) return fail(BGK_ERR_ARG, "bgk_field_sums_static: null pointer");
    if (Nx < 1 || Ny < 1) return fail(BGK_ERR_ARG, "bgk_field_sums_static: Nx (%lld) and Ny (%lld) must be >= 1", Nx, Ny);
    if (Ny > BGK_STATIC_SUMS_MAX_NY)
        return fail(BGK_ERR_ARG,
                    "bgk_field_sums_static: Ny = %lld exceeds the static scratch, which holds %lld rows; "
                    "use bgk_field_sums on a context instead",
                    Ny, BGK_STATIC_SUMS_MAX_NY);
    if ((long long)ld < (long long)Nx + 2)
        return fail(BGK_ERR_ARG, "bgk_field_sums_static: ld (%lld) < Nx + 2 (%lld)", ld, (long long)Nx + 2);
    const uintptr_t mis = ((uintptr_t)rho | (uintptr_t)T | (uintptr_t)phi | (uintptr_t)out) & 7u;
    if (mis) return fail(BGK_ERR_ARG, "bgk_field_sums_static: a pointer is not 8-byte aligned");

    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return fail(BGK_ERR_CUDA, "bgk_field_sums_static: no CUDA device (there is no CPU path)");
    }
    if (dev < 0 || dev >= MAX_DEVICES) return fail(BGK_ERR_ARG, "bgk_field_sums_static: device %lld out of range", dev);
    int rc;
    if ((rc = check_device_pointer(rho, dev, "rho")) || (rc = check_device_pointer(T, dev, "T")) ||
        (rc = check_device_pointer(phi, dev, "phi")) || (rc = check_device_pointer(out, dev, "out")))
        return rc;

    double *part = nullptr;
    if ((rc = scratch_address(dev, &part))) return rc;

    cudaStream_t s = static_cast<cudaStream_t>(stream);
    row_sums_kernel<<<Ny, ROW_THREADS, 0, s>>>(rho, T, phi, Nx, Ny, (long long)ld, part);
    rows_final_kernel<<<1, FINAL_THREADS, 0, s>>>(part, Ny, out);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        char msg[200];
        std::snprintf(msg, sizeof msg, "bgk_field_sums_static: launch failed: %s", cudaGetErrorString(e));
        return bgk_internal_fail(BGK_ERR_CUDA, msg);
    }
    return BGK_OK;
}
