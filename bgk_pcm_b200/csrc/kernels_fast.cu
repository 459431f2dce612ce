/*
 * kernels_fast.cu -- kernels built with multiply-add contraction:
 *  - the FMA variant of the fused FP64 step (same source as the exact one,
 *    fused_f64.cuh; parity with the reference is then within rounding, not
 *    bit-for-bit);
 *  - the reduced-precision forms (FP32 / FP16 deviation storage).
 */
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

int strip_height(const bgk_ctx *c)
{
    const int bx = (c->Nx + FUSED_BX - 1) / FUSED_BX;
    int H = 16;
    while (H > 2 && (long long)bx * ((c->Ny + H - 1) / H) < 148LL * 8) H /= 2;
    return H;
}

} // namespace

cudaError_t launch_fused_fast(bgk_ctx *c, bool moments)
{
    if (c->opt.precision != BGK_PREC_F64) return cudaErrorNotSupported;
    StepPtrs<double> s{};
    const int src = c->cur, dst = c->cur ^ 1;
    s.fin = (const double *)c->fbuf[src]; s.gin = (const double *)c->gbuf[src];
    s.fout = (double *)c->fbuf[dst]; s.gout = (double *)c->gbuf[dst];
    s.phin = (const double *)c->phibuf[src]; s.phout = (double *)c->phibuf[dst];
    s.tcin = c->tcol[src]; s.tcout = c->tcol[dst];
    s.gW = c->gW; s.pE = c->pE; s.phiW = c->phiW; s.phiE = c->phiE;
    s.mrho = c->mrho; s.mT = c->mT; s.mu = c->mu; s.mv = c->mv; s.mphi = c->mphi;
    s.plane = c->plane; s.P = c->P; s.NX2 = c->NX2;
    const int H = strip_height(c);
    dim3 grd((c->Nx + FUSED_BX - 1) / FUSED_BX, (c->Ny + H - 1) / H);
    if (c->opt.tanh_mode == BGK_TANH_PORTABLE) {
        if (moments) fused_f64_kernel<BGK_TANH_PORTABLE, true><<<grd, FUSED_BX, 0, c->stream>>>(s, c->c, c->corner, H);
        else fused_f64_kernel<BGK_TANH_PORTABLE, false><<<grd, FUSED_BX, 0, c->stream>>>(s, c->c, c->corner, H);
    } else {
        if (moments) fused_f64_kernel<BGK_TANH_DEVICE, true><<<grd, FUSED_BX, 0, c->stream>>>(s, c->c, c->corner, H);
        else fused_f64_kernel<BGK_TANH_DEVICE, false><<<grd, FUSED_BX, 0, c->stream>>>(s, c->c, c->corner, H);
    }
    return cudaGetLastError();
}

cudaError_t launch_init_lowp(bgk_ctx *c)
{
    (void)c;
    return cudaErrorNotSupported;
}

} // namespace bgk

int lowp_compact_to_ref(bgk_ctx *c, int field, double *ref, int prev)
{
    (void)c; (void)field; (void)ref; (void)prev;
    return BGK_ERR_UNSUPPORTED;
}

int lowp_ref_to_compact(bgk_ctx *c, int field, const double *ref)
{
    (void)c; (void)field; (void)ref;
    return BGK_ERR_UNSUPPORTED;
}
