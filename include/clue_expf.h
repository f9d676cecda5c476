/*
 * clue_expf.h — the single-precision exponential used by the Gaussian and
 * exponential convolutional kernels, with identical results on the host (C/C++)
 * and on the device (CUDA).
 *
 * Why a library-owned exp: the reference evaluates `math::exp`, which is
 * `std::exp` on its serial CPU backend and CUDA's `::exp` on the GPU
 * (CLUEstering internal/math/exp/exp.hpp:19-29). Neither is correctly rounded,
 * and the two disagree by up to an ulp, so a density that must be reproduced
 * bit for bit by a CPU checker cannot use either. This function is written
 * from the mathematics with a named published method:
 *
 *   - Cody & Waite argument reduction (W. J. Cody, W. Waite, "Software Manual
 *     for the Elementary Functions", 1980): x = n*ln2 + r with
 *     n = rint(x*log2(e)) and ln2 split into a 16-significant-bit head
 *     (so n*head is exact for |n| < 256) and a tail;
 *   - e^r on |r| <= ln2/2 by its Taylor series to degree 7 in Horner form with
 *     fused multiply-adds (truncation error < 2^-27 relative);
 *   - reconstruction e^x = p * 2^n as two exact power-of-two scalings so that
 *     results in the subnormal range are rounded exactly once.
 *
 * Every step is an IEEE-754 single operation with round-to-nearest (fmaf is
 * correctly rounded in C99 and CUDA alike), so host and device return the same
 * bits. The error against the exact exponential is checked by the test suite
 * (at most 1 ulp over the normal range).
 */
#ifndef CLUE_EXPF_H
#define CLUE_EXPF_H

#include <stdint.h>
#include <string.h>

#if defined(__CUDACC__)
#define CLUE_EXPF_QUAL static __host__ __device__ __forceinline__
#else
#define CLUE_EXPF_QUAL static inline
#endif

#if defined(__CUDA_ARCH__)
#define CLUE_FMAF(a, b, c) __fmaf_rn((a), (b), (c))
#define CLUE_FMUL(a, b) __fmul_rn((a), (b))
#define CLUE_FSUB(a, b) __fsub_rn((a), (b))
#define CLUE_RINTF(a) rintf(a)
#else
#include <math.h>
#define CLUE_FMAF(a, b, c) fmaf((a), (b), (c))
#define CLUE_FMUL(a, b) ((a) * (b))
#define CLUE_FSUB(a, b) ((a) - (b))
#define CLUE_RINTF(a) rintf(a)
#endif

CLUE_EXPF_QUAL float clue_bits_to_float(uint32_t b) {
  float f;
#if defined(__CUDA_ARCH__)
  f = __uint_as_float(b);
#else
  memcpy(&f, &b, sizeof f);
#endif
  return f;
}

/* 2^e for e in [-126, 127], built from its exponent bits (exact). */
CLUE_EXPF_QUAL float clue_pow2i(int e) { return clue_bits_to_float((uint32_t)(e + 127) << 23); }

/* clue_expf for x in [underflow_at, overflow_at] (no NaN): the same operations
 * without the special-case tests, so it returns the same bits there. */
CLUE_EXPF_QUAL float clue_expf_core(float x) {
  const float log2e = 1.44269502162933349609375f;  /* 0x3fb8aa3b */
  const float ln2_hi = 0.693145751953125f;          /* 0x3f317200, 16 significant bits */
  const float ln2_lo = 1.428606765330187e-06f;      /* 0x35bfbe8e = ln2 - ln2_hi */
  const float fn = CLUE_RINTF(CLUE_FMUL(x, log2e));
  /* r = (x - n*hi) - n*lo; n*hi is exact, so the first subtraction is exact too
   * (Sterbenz) for the range handled here. */
  const float r = CLUE_FSUB(CLUE_FSUB(x, CLUE_FMUL(fn, ln2_hi)), CLUE_FMUL(fn, ln2_lo));
  /* Taylor coefficients 1/k!, k = 7..0, each rounded to float. */
  float p = 1.98412701138295233249664306640625e-04f; /* 1/7! */
  p = CLUE_FMAF(p, r, 1.38888892251998186111450195312e-03f); /* 1/6! */
  p = CLUE_FMAF(p, r, 8.33333376795053482055664062500e-03f); /* 1/5! */
  p = CLUE_FMAF(p, r, 4.16666679084300994873046875000e-02f); /* 1/4! */
  p = CLUE_FMAF(p, r, 1.66666671633720397949218750000e-01f); /* 1/3! */
  p = CLUE_FMAF(p, r, 0.5f);
  p = CLUE_FMAF(p, r, 1.0f);
  p = CLUE_FMAF(p, r, 1.0f);
  const int n = (int)fn;
  const int n1 = n / 2;
  const int n2 = n - n1;
  /* p * 2^n1 stays in the normal range (exact); the second scaling rounds once. */
  return CLUE_FMUL(CLUE_FMUL(p, clue_pow2i(n1)), clue_pow2i(n2));
}

CLUE_EXPF_QUAL float clue_expf(float x) {
  /* ln(2^128) rounded down to float: above it the result overflows. */
  const float overflow_at = 88.72283935546875f;
  /* Below ln(2^-150) the exact result is under half the smallest subnormal. */
  const float underflow_at = -103.97207641601562f;
  if (x != x)
    return x;
  if (x > overflow_at)
    return clue_bits_to_float(0x7f800000u); /* +inf */
  if (x < underflow_at)
    return 0.0f;
  return clue_expf_core(x);
}

#endif /* CLUE_EXPF_H */
