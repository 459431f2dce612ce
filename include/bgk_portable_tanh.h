/*
 * bgk_portable_tanh.h -- a hyperbolic tangent built only from IEEE-754
 * double-precision +, -, *, / and exact power-of-two scaling.
 *
 * Purpose: the reference's phase-field selector calls tanh once per node
 * (STEP_7/phase_field.f90:20-21).  The host libm tanh and CUDA's tanh may
 * differ by an ulp or two, which makes the GPU step and its CPU oracle differ
 * in the last bits even when every other operation is identical.  With this
 * function selected on both sides (BGK_TANH_PORTABLE), each correctly-rounded
 * operation happens in the same order on the CPU (compiled with
 * -ffp-contract=off) and on the GPU (compiled with --fmad=false), so the two
 * results are bit-identical and a parity test can demand exact equality.
 * The production path uses CUDA's own tanh.
 *
 * Method (from the mathematics; no library constants):
 *   tanh(|x|) = -m / (2 + m),  m = expm1(-2|x|)
 *   expm1(y)  = 2^k (e^r - 1) + (2^k - 1),  y = k ln2 + r, |r| <= ln2/2
 *   (Cody & Waite two-constant reduction: ln2 split into a 32-bit head and a
 *   correction so that k*head is exact), e^r - 1 by its Taylor series to
 *   degree 13, evaluated in Horner form.  Coefficients are 1/n! rounded to
 *   nearest double (computed with exact rational arithmetic).
 *   The reduction and the Horner steps are explicit fused multiply-adds
 *   (C99 fma, IEEE-754 fusedMultiplyAdd: one rounding), which both the host
 *   libm and the GPU evaluate exactly as specified, so they stay
 *   bit-identical even where the surrounding code forbids contraction; on
 *   the GPU this halves the function's floating-point operations.
 * Accuracy: a few ulp over the whole real line (checked against libm by the
 * CPU test-suite).  This is a checking aid, not a replacement for tanh.
 */
#ifndef BGK_PORTABLE_TANH_H
#define BGK_PORTABLE_TANH_H

#include <math.h>
#include <stdint.h>
#include <string.h>

#if defined(__CUDACC__)
#define BGK_PT_HD __host__ __device__ __forceinline__
#else
#define BGK_PT_HD static inline
#endif

/* 2^k for -1022 <= k <= 1023, built from its bit pattern (exact). */
BGK_PT_HD double bgk_pt_pow2i(int k)
{
    uint64_t bits = (uint64_t)(k + 1023) << 52;
    double d;
#if defined(__CUDA_ARCH__)
    d = __longlong_as_double((long long)bits);
#else
    memcpy(&d, &bits, sizeof d);
#endif
    return d;
}

/* e^y - 1 for y <= 0 (the only range tanh needs). */
BGK_PT_HD double bgk_pt_expm1_neg(double y)
{
    const double inv_ln2 = 0x1.71547652b82fep+0;   /* 1/ln 2            */
    const double ln2_hi  = 0x1.62e42ff000000p-1;   /* ln 2, 32-bit head */
    const double ln2_lo  = -0x1.718432a1b0e26p-35; /* ln 2 - ln2_hi     */
    /* e^-40 < 2^-57: below this, e^y - 1 rounds to -1 exactly */
    if (y < -40.0) return -1.0;
    double kd = fma(y, inv_ln2, 0.5);
    /* floor without libm: truncate toward zero, fix negative non-integers */
    double t = (double)(long long)kd;
    if (t > kd) t = t - 1.0;
    int k = (int)t;
    double r = fma(-t, ln2_lo, fma(-t, ln2_hi, y));
    /* e^r - 1 = r(1 + r/2 + r^2/6 + ... + r^12/13!) */
    double p = 0x1.6124613a86d09p-33;              /* 1/13! */
    p = fma(p, r, 0x1.1eed8eff8d898p-29);          /* 1/12! */
    p = fma(p, r, 0x1.ae64567f544e4p-26);          /* 1/11! */
    p = fma(p, r, 0x1.27e4fb7789f5cp-22);          /* 1/10! */
    p = fma(p, r, 0x1.71de3a556c734p-19);          /* 1/9!  */
    p = fma(p, r, 0x1.a01a01a01a01ap-16);          /* 1/8!  */
    p = fma(p, r, 0x1.a01a01a01a01ap-13);          /* 1/7!  */
    p = fma(p, r, 0x1.6c16c16c16c17p-10);          /* 1/6!  */
    p = fma(p, r, 0x1.1111111111111p-7);           /* 1/5!  */
    p = fma(p, r, 0x1.5555555555555p-5);           /* 1/4!  */
    p = fma(p, r, 0x1.5555555555555p-3);           /* 1/3!  */
    p = fma(p, r, 0.5);                            /* 1/2!  */
    p = fma(p, r, 1.0);                            /* 1/1!  */
    double em = p * r;                             /* e^r - 1 */
    if (k == 0) return em;
    double s = bgk_pt_pow2i(k);
    return (s * (em + 1.0)) - 1.0;
}

BGK_PT_HD double bgk_portable_tanh(double x)
{
    double ax = x < 0.0 ? -x : x;
    double th;
    if (ax == 0.0) return x;
    if (ax > 22.0) {
        th = 1.0;
    } else {
        double m = bgk_pt_expm1_neg(-2.0 * ax);
        th = -m / (2.0 + m);
    }
    return x < 0.0 ? -th : th;
}

#endif /* BGK_PORTABLE_TANH_H */
