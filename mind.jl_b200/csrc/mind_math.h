/*
 * mind_math.h — project-owned elementary functions and the Philox stream,
 * compiled identically for the host and for sm_100a.
 *
 * Why these exist: FP64 parity between the CUDA path and the CPU oracle is
 * defined bit for bit.  glibc's and CUDA's exp/log differ in the last bit on
 * some arguments, and spiking networks amplify a last-bit difference into a
 * different raster.  Both sides therefore call these functions, built only
 * from IEEE-754 correctly rounded +, -, *, /, fma and exact bit operations, in
 * a fixed order; host code is compiled with -ffp-contract=off and device code
 * with -fmad=false so no other fusion happens.
 *
 * Methods (constants derived by gen_mathconst.py from exact arithmetic):
 *   exp  Cody-Waite additive reduction x = k ln2 + r, |r| <= ln2/2, then the
 *        degree-13 Taylor polynomial of e^r by Horner with fma, scaled by 2^k.
 *   log  x = 2^e m with m in [sqrt2/2, sqrt2); ln m = 2 atanh(s), s = (m-1)/(m+1),
 *        summed as f - s (f - R) with R the atanh series in s^2 to s^22.
 *   pow  exp(y log x) (used for Q10 factors; exact for y == 0).
 * Accuracy against glibc is checked by tests/test_math_rng.py (a few ulp at most).
 *
 * Philox4x32-10 follows Salmon, Moraes, Dror and Shaw, "Parallel random
 * numbers: as easy as 1, 2, 3" (SC'11), with its published multipliers and
 * Weyl key increments; the per-instance stream layout is the one the reference
 * keeps for NEURON's nrnran123 (src/runtime/cuda/micro.jl:3-77).
 */
#ifndef MIND_MATH_H
#define MIND_MATH_H

#include <stdint.h>
#include <math.h>
#ifndef __CUDACC__
#include <string.h>
#endif

#ifdef __CUDACC__
#define MIND_HD __host__ __device__ __forceinline__
#else
#define MIND_HD static inline
#endif

/* ---- constants: output of gen_mathconst.py ---- */
#define MIND_LN2_HI 0x1.62e42fee00000p-1
#define MIND_LN2_LO 0x1.a39ef35793c76p-33
#define MIND_INV_LN2 0x1.71547652b82fep+0
#define MIND_SQRT2 0x1.6a09e667f3bcdp+0
#define MIND_INV_2P32P1 0x1.fffffffe00000p-33
#define MIND_EXP_C2 0x1.0000000000000p-1
#define MIND_EXP_C3 0x1.5555555555555p-3
#define MIND_EXP_C4 0x1.5555555555555p-5
#define MIND_EXP_C5 0x1.1111111111111p-7
#define MIND_EXP_C6 0x1.6c16c16c16c17p-10
#define MIND_EXP_C7 0x1.a01a01a01a01ap-13
#define MIND_EXP_C8 0x1.a01a01a01a01ap-16
#define MIND_EXP_C9 0x1.71de3a556c734p-19
#define MIND_EXP_C10 0x1.27e4fb7789f5cp-22
#define MIND_EXP_C11 0x1.ae64567f544e4p-26
#define MIND_EXP_C12 0x1.1eed8eff8d898p-29
#define MIND_EXP_C13 0x1.6124613a86d09p-33
#define MIND_LOG_C1 0x1.5555555555555p-1
#define MIND_LOG_C2 0x1.999999999999ap-2
#define MIND_LOG_C3 0x1.2492492492492p-2
#define MIND_LOG_C4 0x1.c71c71c71c71cp-3
#define MIND_LOG_C5 0x1.745d1745d1746p-3
#define MIND_LOG_C6 0x1.3b13b13b13b14p-3
#define MIND_LOG_C7 0x1.1111111111111p-3
#define MIND_LOG_C8 0x1.e1e1e1e1e1e1ep-4
#define MIND_LOG_C9 0x1.af286bca1af28p-4
#define MIND_LOG_C10 0x1.8618618618618p-4
#define MIND_LOG_C11 0x1.642c8590b2164p-4

MIND_HD uint64_t mind_bits(double x) {
#ifdef __CUDA_ARCH__
    return (uint64_t)__double_as_longlong(x);
#else
    uint64_t b;
    memcpy(&b, &x, sizeof b);
    return b;
#endif
}

MIND_HD double mind_from_bits(uint64_t b) {
#ifdef __CUDA_ARCH__
    return __longlong_as_double((long long)b);
#else
    double x;
    memcpy(&x, &b, sizeof x);
    return x;
#endif
}

/* 2^k for k in [-1022, 1023], exact. */
MIND_HD double mind_pow2i(int k) { return mind_from_bits((uint64_t)(k + 1023) << 52); }

/* p * 2^k for any int k, exact unless the result is subnormal or overflows. */
MIND_HD double mind_scale2(double p, int k) {
    if (k > 1023) return (p * mind_pow2i(1023)) * mind_pow2i(k - 1023 > 1023 ? 1023 : k - 1023);
    if (k < -1022) {
        int rest = k + 1022;
        if (rest < -1022) rest = -1022;
        return (p * mind_pow2i(-1022)) * mind_pow2i(rest);
    }
    return p * mind_pow2i(k);
}

MIND_HD double mind_exp(double x) {
    if (x != x) return x;
    if (x > 709.782712893384) return INFINITY;
    if (x < -745.1332191019412) return 0.0;
    double kf = floor(x * MIND_INV_LN2 + 0.5);
    int k = (int)kf;
    double r = (x - kf * MIND_LN2_HI) - kf * MIND_LN2_LO;
    double p = MIND_EXP_C13;
    p = fma(p, r, MIND_EXP_C12);
    p = fma(p, r, MIND_EXP_C11);
    p = fma(p, r, MIND_EXP_C10);
    p = fma(p, r, MIND_EXP_C9);
    p = fma(p, r, MIND_EXP_C8);
    p = fma(p, r, MIND_EXP_C7);
    p = fma(p, r, MIND_EXP_C6);
    p = fma(p, r, MIND_EXP_C5);
    p = fma(p, r, MIND_EXP_C4);
    p = fma(p, r, MIND_EXP_C3);
    p = fma(p, r, MIND_EXP_C2);
    p = fma(p, r, 1.0);
    p = fma(p, r, 1.0);
    return mind_scale2(p, k);
}

MIND_HD double mind_log(double x) {
    if (x != x) return x;
    if (x < 0.0) return NAN;
    if (x == 0.0) return -INFINITY;
    if (x == INFINITY) return x;
    int adjust = 0;
    if (x < 0x1p-1022) {
        x = x * 0x1p54;
        adjust = -54;
    }
    uint64_t b = mind_bits(x);
    int e = (int)((b >> 52) & 0x7ff) - 1023 + adjust;
    double m = mind_from_bits((b & 0x000fffffffffffffULL) | 0x3ff0000000000000ULL);
    if (m > MIND_SQRT2) {
        m = m * 0.5;
        e += 1;
    }
    double f = m - 1.0;
    double s = f / (2.0 + f);
    double z = s * s;
    double R = MIND_LOG_C11;
    R = fma(R, z, MIND_LOG_C10);
    R = fma(R, z, MIND_LOG_C9);
    R = fma(R, z, MIND_LOG_C8);
    R = fma(R, z, MIND_LOG_C7);
    R = fma(R, z, MIND_LOG_C6);
    R = fma(R, z, MIND_LOG_C5);
    R = fma(R, z, MIND_LOG_C4);
    R = fma(R, z, MIND_LOG_C3);
    R = fma(R, z, MIND_LOG_C2);
    R = fma(R, z, MIND_LOG_C1);
    R = R * z;
    double lm = f - s * (f - R);
    double ef = (double)e;
    return ef * MIND_LN2_HI + (lm + ef * MIND_LN2_LO);
}

MIND_HD double mind_pow(double x, double y) {
    if (y == 0.0 || x == 1.0) return 1.0;
    if (x > 0.0) return mind_exp(y * mind_log(x));
    if (x == 0.0) return y > 0.0 ? 0.0 : INFINITY;
    if (y == floor(y)) {
        double magnitude = mind_exp(y * mind_log(-x));
        double half = y * 0.5;
        return half == floor(half) ? magnitude : -magnitude;
    }
    return NAN;
}

/* x / 0.001, bit for bit equal to the IEEE quotient, without a division.
 * 1000 is the correctly rounded reciprocal of the double 0.001 and differs from
 * 1/0.001 by 0.19 units in its last place, so q0 = x*1000 lies within one ulp of
 * x/0.001; the residual x - q0*0.001 is then exact in one FMA, and one correction
 * step rounds to the IEEE quotient (Markstein's theorem: P. W. Markstein,
 * "Computation of elementary functions on the IBM RISC System/6000 processor",
 * IBM J. Res. Dev. 34(1), 1990; J.-M. Muller et al., Handbook of Floating-Point
 * Arithmetic, chapter on FMA-based division).  The theorem assumes no underflow
 * or overflow, so magnitudes outside [2^-900, 2^900], and non-finite values,
 * take the division; zeros come back unchanged, as 0/0.001 keeps the sign. */
/* AlphaSynapse's alpha(x) (mod/AlphaSynapse.mod FUNCTION alpha): x exp(1 - x) on
 * [0, 10], else 0. */
MIND_HD double mind_alpha(double x) { return (x < 0.0 || x > 10.0) ? 0.0 : x * mind_exp(1.0 - x); }

MIND_HD double mind_div_milli(double x) {
    const double ax = fabs(x);
    if (ax >= 0x1p-900 && ax <= 0x1p+900) {
        const double q0 = x * 1000.0;
        const double r = fma(-q0, 0.001, x);
        return fma(r, 1000.0, q0);
    }
    return x == 0.0 ? x : x / 0.001;
}

/* ---- Philox4x32-10 ---- */
#define MIND_PHILOX_M0 0xD2511F53u
#define MIND_PHILOX_M1 0xCD9E8D57u
#define MIND_PHILOX_W0 0x9E3779B9u
#define MIND_PHILOX_W1 0xBB67AE85u

/* In place: ctr <- Philox4x32-10(ctr, key). */
MIND_HD void mind_philox4x32_10(uint32_t ctr[4], uint32_t key0, uint32_t key1) {
    uint32_t a = ctr[0], b = ctr[1], c = ctr[2], d = ctr[3];
    for (int round = 0; round < 10; ++round) {
        uint64_t p0 = (uint64_t)MIND_PHILOX_M0 * (uint64_t)a;
        uint64_t p1 = (uint64_t)MIND_PHILOX_M1 * (uint64_t)c;
        uint32_t na = (uint32_t)(p1 >> 32) ^ b ^ key0;
        uint32_t nb = (uint32_t)p1;
        uint32_t nc = (uint32_t)(p0 >> 32) ^ d ^ key1;
        uint32_t nd = (uint32_t)p0;
        a = na;
        b = nb;
        c = nc;
        d = nd;
        key0 += MIND_PHILOX_W0;
        key1 += MIND_PHILOX_W1;
    }
    ctr[0] = a;
    ctr[1] = b;
    ctr[2] = c;
    ctr[3] = d;
}

/*
 * One random stream of one mechanism instance, in the nrnran123 layout the
 * reference keeps per row: a 34-bit draw counter, three 32-bit ids
 * (id1 = logical id low word, id2 = high word, id3 = digest low word ^ stream)
 * and the four words of the current Philox block.  The Philox counter block
 * is (counter >> 2, id3, id1, id2) under key (seed low, seed high).
 */
typedef struct MindRan {
    uint64_t counter;
    uint32_t id1, id2, id3;
    uint32_t words[4];
} MindRan;

MIND_HD void mind_ran_refresh(MindRan *s, uint64_t seed) {
    uint32_t ctr[4] = {(uint32_t)(s->counter >> 2), s->id3, s->id1, s->id2};
    mind_philox4x32_10(ctr, (uint32_t)seed, (uint32_t)(seed >> 32));
    s->words[0] = ctr[0];
    s->words[1] = ctr[1];
    s->words[2] = ctr[2];
    s->words[3] = ctr[3];
}

/* initialize_random_kernel!: ids from the logical id and digest, then setseq(0). */
MIND_HD void mind_ran_init(MindRan *s, uint64_t logical_id, uint64_t digest, uint32_t stream,
                           uint64_t seed) {
    s->id1 = (uint32_t)logical_id;
    s->id2 = (uint32_t)(logical_id >> 32);
    s->id3 = (uint32_t)digest ^ stream;
    s->counter = 0;
    mind_ran_refresh(s, seed);
}

/* random_setseq: counter <- trunc(sequence) (0 outside [0, 2^40-1]); regenerate words. */
MIND_HD void mind_ran_setseq(MindRan *s, double sequence, uint64_t seed) {
    double bounded = (sequence >= 0.0 && sequence <= 1099511627775.0) ? sequence : 0.0;
    s->counter = ((uint64_t)trunc(bounded)) & 0x3ffffffffULL;
    mind_ran_refresh(s, seed);
}

/* Uniform in (0,1): consume word counter&3; after the fourth word advance the block. */
MIND_HD double mind_ran_uniform(MindRan *s, uint64_t seed) {
    uint32_t which = (uint32_t)(s->counter & 3u);
    uint32_t word = s->words[which];
    uint64_t next = (s->counter + 1u) & 0x3ffffffffULL;
    s->counter = next;
    if (which == 3u) {
        if (next == 0u) {
            /* Carry into the ids in the order id3, id1, id2. */
            s->id3 += 1u;
            if (s->id3 == 0u) {
                s->id1 += 1u;
                if (s->id1 == 0u) s->id2 += 1u;
            }
        }
        mind_ran_refresh(s, seed);
    }
    return ((double)word + 1.0) * MIND_INV_2P32P1;
}

/* random_negexp(stream) with unit mean: -log(u). */
MIND_HD double mind_ran_negexp(MindRan *s, uint64_t seed) {
    return -mind_log(mind_ran_uniform(s, seed)) * 1.0;
}

#endif /* MIND_MATH_H */
