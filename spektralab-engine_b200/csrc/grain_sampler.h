/* The grain random-number path, compiled identically for the device (CUDA) and for the host checker
 * (C99), so that the Philox words and the Poisson counts for the same lambda agree bit for bit.
 *
 *   Philox4x32-10     Salmon, Moraes, Dror and Shaw, "Parallel random numbers: as easy as 1, 2, 3", SC 2011;
 *                     counter (pixel, stream, j, 0), key (seed, 0), words consumed x, y, z, w
 *                     (reference kernels/spk_common.h:23-67)
 *   uniform           u = ((word >> 8) + 0.5) * 2^-24
 *   Poisson, lam>=10  Hormann's transformed rejection with squeeze (PTRS), "The transformed rejection
 *                     method for generating Poisson random variables", Insurance: Mathematics and
 *                     Economics 12 (1993); at most 64 tries, then floor(lam)
 *   Poisson, lam<10   multiply uniforms until the product falls to exp(-lam), at most 512 steps
 *   lgamma(k + 1)     Stirling series with five correction terms, shifted up to 7 by recurrence
 *   sub-layer draw    q = clamp(d/D, 1e-6, 0.999999); sat = 1 - q u 0.999999; lam = (n / sat) q;
 *                     Poisson(lam) (D / n) sat  (reference kernels/fx_random.h:19-99)
 *
 * Elementary functions. The sampler needs log, exp, sqrt and cos in binary32. Vendor libraries round
 * these differently in the last place, so both builds use the functions below:
 *   spk_logf  x = m 2^e with m in [sqrt(1/2), sqrt(2)); f = m - 1, s = f / (2 + f);
 *             log m = 2 atanh s = 2 (s + s^3/3 + s^5/5 + s^7/7 + s^9/9 + s^11/11) (|s| <= 0.1716);
 *             log x = e ln2_hi + (log m + e ln2_lo)   (Cody and Waite's split of ln 2)
 *   spk_expf  n = rint(x log2 e); r = (x - n ln2_hi) - n ln2_lo; exp r by its Taylor series to r^8
 *             in Horner form (|r| <= 0.347); times 2^n built in the exponent field
 *   spk_cosf  k = rint(x 2/pi); r = x - k pi/2 in three parts; the sine or cosine Taylor series on
 *             |r| <= pi/4 to degree 9 or 10, sign and choice from k mod 4
 *   sqrt      the correctly rounded square root (IEEE 754), identical everywhere
 * Every product, sum and quotient is written as an explicitly rounded operation (SPK_MUL, SPK_ADD,
 * SPK_DIV, SPK_FMA), so no compiler contraction can change a result.
 */
#ifndef SPKB_GRAIN_SAMPLER_H
#define SPKB_GRAIN_SAMPLER_H

#include <stdint.h>

#if defined(__CUDACC__)
#define SPK_HD __host__ __device__ __forceinline__
#if defined(__CUDA_ARCH__)
#define SPK_MUL(a, b) __fmul_rn((a), (b))
#define SPK_ADD(a, b) __fadd_rn((a), (b))
#define SPK_SUB(a, b) __fsub_rn((a), (b))
#define SPK_DIV(a, b) __fdiv_rn((a), (b))
#define SPK_FMA(a, b, c) __fmaf_rn((a), (b), (c))
#define SPK_SQRT(a) __fsqrt_rn(a)
#define SPK_FLOOR(a) floorf(a)
#define SPK_RINT(a) rintf(a)
#else
#include <math.h>
#define SPK_MUL(a, b) ((a) * (b))
#define SPK_ADD(a, b) ((a) + (b))
#define SPK_SUB(a, b) ((a) - (b))
#define SPK_DIV(a, b) ((a) / (b))
#define SPK_FMA(a, b, c) fmaf((a), (b), (c))
#define SPK_SQRT(a) sqrtf(a)
#define SPK_FLOOR(a) floorf(a)
#define SPK_RINT(a) rintf(a)
#endif
#else
#include <math.h>
#define SPK_HD static inline
/* host builds of this header compile with -ffp-contract=off */
#define SPK_MUL(a, b) ((a) * (b))
#define SPK_ADD(a, b) ((a) + (b))
#define SPK_SUB(a, b) ((a) - (b))
#define SPK_DIV(a, b) ((a) / (b))
#define SPK_FMA(a, b, c) fmaf((a), (b), (c))
#define SPK_SQRT(a) sqrtf(a)
#define SPK_FLOOR(a) floorf(a)
#define SPK_RINT(a) rintf(a)
#endif

#define SPK_PHILOX_M0 0xD2511F53u
#define SPK_PHILOX_M1 0xCD9E8D57u
#define SPK_PHILOX_W0 0x9E3779B9u
#define SPK_PHILOX_W1 0xBB67AE85u
#define SPK_STREAM_GRAIN(c, l) ((c) + 10u * (l))
#define SPK_STREAM_MICRO(c) (100u + (c))

typedef struct {
    uint32_t x, y, z, w;
} spk_u4;

SPK_HD uint32_t spk_bits(float f) {
    union {
        float f;
        uint32_t u;
    } v;
    v.f = f;
    return v.u;
}
SPK_HD float spk_float(uint32_t u) {
    union {
        float f;
        uint32_t u;
    } v;
    v.u = u;
    return v.f;
}

SPK_HD spk_u4 spk_philox(spk_u4 c, uint32_t k0, uint32_t k1) {
    for (int r = 0; r < 10; ++r) {
        const uint64_t p0 = (uint64_t)SPK_PHILOX_M0 * c.x;
        const uint64_t p1 = (uint64_t)SPK_PHILOX_M1 * c.z;
        spk_u4 n;
        n.x = (uint32_t)(p1 >> 32) ^ c.y ^ k0;
        n.y = (uint32_t)p1;
        n.z = (uint32_t)(p0 >> 32) ^ c.w ^ k1;
        n.w = (uint32_t)p0;
        c = n;
        k0 += SPK_PHILOX_W0;
        k1 += SPK_PHILOX_W1;
    }
    return c;
}

SPK_HD float spk_uniform(uint32_t word) { return SPK_MUL((float)(word >> 8) + 0.5f, 5.9604644775390625e-08f); }

/* One generator per (pixel, stream). */
typedef struct {
    uint32_t pixel, stream, seed, j, used;
    spk_u4 block;
} spk_stream;

SPK_HD void spk_stream_init(spk_stream* g, uint32_t pixel, uint32_t stream, uint32_t seed) {
    g->pixel = pixel;
    g->stream = stream;
    g->seed = seed;
    g->j = 0;
    g->used = 4;
}

SPK_HD float spk_stream_uniform(spk_stream* g) {
    if (g->used == 4) {
        spk_u4 c;
        c.x = g->pixel;
        c.y = g->stream;
        c.z = g->j;
        c.w = 0u;
        g->block = spk_philox(c, g->seed, 0u);
        ++g->j;
        g->used = 0;
    }
    const uint32_t w = g->used == 0 ? g->block.x : g->used == 1 ? g->block.y : g->used == 2 ? g->block.z : g->block.w;
    ++g->used;
    return spk_uniform(w);
}

/* ---- elementary functions (method above) ---- */

#define SPK_LN2_HI 0.693145751953125f        /* ln 2 rounded to 16 significant bits: exact products */
#define SPK_LN2_LO 1.42860682030941723212e-6f /* ln 2 - SPK_LN2_HI */

SPK_HD float spk_logf(float x) {
    uint32_t u = spk_bits(x);
    if (!(x > 0.0f)) return x == 0.0f ? spk_float(0xFF800000u) : spk_float(0x7FC00000u);
    if (u >= 0x7F800000u) return x; /* +inf or NaN */
    int e = 0;
    if (u < 0x00800000u) { /* subnormal: scale into the normal range */
        x = SPK_MUL(x, 8388608.0f);
        u = spk_bits(x);
        e = -23;
    }
    /* m in [sqrt(1/2), sqrt(2)): take the exponent of x * sqrt(2) */
    const uint32_t ub = u + (0x3F800000u - 0x3F3504F3u);
    e += (int)(ub >> 23) - 127;
    const float m = spk_float((ub & 0x007FFFFFu) + 0x3F3504F3u);
    const float f = SPK_SUB(m, 1.0f);
    const float s = SPK_DIV(f, SPK_ADD(2.0f, f));
    const float z = SPK_MUL(s, s);
    float p = 0.090909090909090909f;            /* 1/11 */
    p = SPK_FMA(p, z, 0.111111111111111111f);   /* 1/9 */
    p = SPK_FMA(p, z, 0.142857142857142857f);   /* 1/7 */
    p = SPK_FMA(p, z, 0.2f);                    /* 1/5 */
    p = SPK_FMA(p, z, 0.333333333333333333f);   /* 1/3 */
    /* log m = 2 s + 2 s z p, written as f - (f - 2 s) ... keep it simple: 2s (1 + z p) */
    const float two_s = SPK_ADD(s, s);
    const float lm = SPK_FMA(SPK_MUL(two_s, z), p, two_s);
    const float fe = (float)e;
    return SPK_FMA(fe, SPK_LN2_HI, SPK_FMA(fe, SPK_LN2_LO, lm));
}

SPK_HD float spk_expf(float x) {
    if (x != x) return x;
    if (x > 88.72283905206835f) return spk_float(0x7F800000u);
    if (x < -103.97208f) return 0.0f;
    const float n = SPK_RINT(SPK_MUL(x, 1.44269504088896341f));
    const float r = SPK_FMA(-n, SPK_LN2_LO, SPK_FMA(-n, SPK_LN2_HI, x));
    /* Taylor series of e^r to r^8, Horner form */
    float p = 2.48015873015873016e-05f;           /* 1/8! */
    p = SPK_FMA(p, r, 1.98412698412698413e-04f);  /* 1/7! */
    p = SPK_FMA(p, r, 1.38888888888888889e-03f);  /* 1/6! */
    p = SPK_FMA(p, r, 8.33333333333333333e-03f);  /* 1/5! */
    p = SPK_FMA(p, r, 4.16666666666666667e-02f);  /* 1/4! */
    p = SPK_FMA(p, r, 1.66666666666666667e-01f);  /* 1/3! */
    p = SPK_FMA(p, r, 0.5f);
    p = SPK_FMA(p, r, 1.0f);
    p = SPK_FMA(p, r, 1.0f);
    int k = (int)n;
    /* 2^k in two steps so that k down to -149 and up to 128 stay representable */
    const int k1 = k / 2, k2 = k - k1;
    const float s1 = spk_float((uint32_t)(k1 + 127) << 23);
    const float s2 = k2 >= -126 ? spk_float((uint32_t)(k2 + 127) << 23) : 0.0f;
    return SPK_MUL(SPK_MUL(p, s1), s2);
}

#define SPK_PIO2_1 1.5707963705062866e+00f  /* pi/2 in three parts, the first two with 12 trailing zero bits */
#define SPK_PIO2_2 -4.3711388286737929e-08f
#define SPK_PIO2_3 -1.7151245100059209e-15f

SPK_HD float spk_sin_poly(float r) {
    const float z = SPK_MUL(r, r);
    float p = 2.75573192239858907e-06f;            /* 1/9! */
    p = SPK_FMA(p, z, -1.98412698412698413e-04f);  /* -1/7! */
    p = SPK_FMA(p, z, 8.33333333333333333e-03f);   /* 1/5! */
    p = SPK_FMA(p, z, -1.66666666666666667e-01f);  /* -1/3! */
    return SPK_FMA(SPK_MUL(r, z), p, r);
}
SPK_HD float spk_cos_poly(float r) {
    const float z = SPK_MUL(r, r);
    float p = -2.75573192239858907e-07f;           /* -1/10! */
    p = SPK_FMA(p, z, 2.48015873015873016e-05f);   /* 1/8! */
    p = SPK_FMA(p, z, -1.38888888888888889e-03f);  /* -1/6! */
    p = SPK_FMA(p, z, 4.16666666666666667e-02f);   /* 1/4! */
    p = SPK_FMA(p, z, -0.5f);
    return SPK_FMA(z, p, 1.0f);
}

/* cos for |x| up to a few thousand (the sampler calls it on (0, 2 pi]) */
SPK_HD float spk_cosf(float x) {
    const float k = SPK_RINT(SPK_MUL(x, 0.636619772367581343f));
    float r = SPK_FMA(-k, SPK_PIO2_1, x);
    r = SPK_FMA(-k, SPK_PIO2_2, r);
    r = SPK_FMA(-k, SPK_PIO2_3, r);
    const int q = ((int)k) & 3;
    if (q == 0) return spk_cos_poly(r);
    if (q == 1) return -spk_sin_poly(r);
    if (q == 2) return -spk_cos_poly(r);
    return spk_sin_poly(r);
}

/* ---- the sampler ---- */

#define SPK_TWO_PI 6.283185307179586f
#define SPK_LOG_TWO_PI 0x1.d67f1ep+0f /* spk_logf(SPK_TWO_PI), bit for bit (0x3FEB3F8F) */

SPK_HD float spk_lgamma_k(float x) {
    if (x == 1.0f || x == 2.0f) return 0.0f;
    float x0 = x;
    int n = 0;
    if (x <= 7.0f) {
        n = (int)(7.0f - x);
        x0 = SPK_ADD(x, (float)n);
    }
    const float x2 = SPK_DIV(1.0f, SPK_MUL(x0, x0));
    float g = 8.417508417508418e-04f;
    g = SPK_ADD(SPK_MUL(g, x2), -5.952380952380952e-04f);
    g = SPK_ADD(SPK_MUL(g, x2), 7.936507936507937e-04f);
    g = SPK_ADD(SPK_MUL(g, x2), -2.777777777777778e-03f);
    g = SPK_ADD(SPK_MUL(g, x2), 8.333333333333333e-02f);
    const float t1 = SPK_ADD(SPK_DIV(g, x0), SPK_MUL(0.5f, SPK_LOG_TWO_PI));
    float gl = SPK_SUB(SPK_ADD(t1, SPK_MUL(SPK_SUB(x0, 0.5f), spk_logf(x0))), x0);
    if (x <= 7.0f) {
        for (int i = 0; i < n; ++i) {
            gl = SPK_SUB(gl, spk_logf(SPK_SUB(x0, 1.0f)));
            x0 = SPK_SUB(x0, 1.0f);
        }
    }
    return gl;
}

/* PTRS in pieces, so that a caller can run every draw's first attempt in lockstep and finish the
 * rest apart. Attempt `it` of a draw takes uniforms 2 it (U) and 2 it + 1 (V) of its stream. */
typedef struct {
    float lam, loglam, b, a, invalpha, loginvalpha, vr;
} spk_ptrs;

#define SPK_PTRS_REJECT 0
#define SPK_PTRS_ACCEPT 1
#define SPK_PTRS_TEST 2 /* neither squeeze decides: the full test follows */

/* the constants of the squeeze: lam, b, a, vr */
SPK_HD void spk_ptrs_init(spk_ptrs* p, float lam) {
    const float slam = SPK_SQRT(lam);
    p->lam = lam;
    p->b = SPK_ADD(0.931f, SPK_MUL(2.53f, slam));
    p->a = SPK_ADD(-0.059f, SPK_MUL(0.02483f, p->b));
    p->vr = SPK_SUB(0.9277f, SPK_DIV(3.6224f, SPK_SUB(p->b, 2.0f)));
}

/* the constants only the full test reads: log lam, 1 / alpha and its log (after spk_ptrs_init) */
SPK_HD void spk_ptrs_init_test(spk_ptrs* p) {
    p->loglam = spk_logf(p->lam);
    p->invalpha = SPK_ADD(1.1239f, SPK_DIV(1.1328f, SPK_SUB(p->b, 3.4f)));
    p->loginvalpha = spk_logf(p->invalpha);
}

/* the candidate k of an attempt and its two squeezes */
SPK_HD int spk_ptrs_squeeze(const spk_ptrs* p, float u, float V, float* k_out, float* us_out) {
    const float U = SPK_SUB(u, 0.5f);
    const float us = SPK_SUB(0.5f, fabsf(U));
    const float k =
        SPK_FLOOR(SPK_ADD(SPK_ADD(SPK_MUL(SPK_ADD(SPK_DIV(SPK_MUL(2.0f, p->a), us), p->b), U), p->lam), 0.43f));
    *k_out = k;
    *us_out = us;
    if (us >= 0.07f && V <= p->vr) return SPK_PTRS_ACCEPT;
    if (k < 0.0f || (us < 0.013f && V > us)) return SPK_PTRS_REJECT;
    return SPK_PTRS_TEST;
}

/* the full acceptance test: log V + log(1/alpha) - log(a / us^2 + b) <= -lam + k log lam - log k! */
SPK_HD int spk_ptrs_test(const spk_ptrs* p, float V, float k, float us) {
    const float L = SPK_SUB(SPK_ADD(spk_logf(V), p->loginvalpha),
                            spk_logf(SPK_ADD(SPK_DIV(p->a, SPK_MUL(us, us)), p->b)));
    const float Rt = SPK_SUB(SPK_ADD(-p->lam, SPK_MUL(k, p->loglam)), spk_lgamma_k(SPK_ADD(k, 1.0f)));
    return L <= Rt;
}

/* attempts it0..63 on a generator positioned at attempt it0's first uniform; floor(lam) after 64 */
SPK_HD float spk_ptrs_from(const spk_ptrs* p, spk_stream* g, int it0) {
    for (int it = it0; it < 64; ++it) {
        const float u = spk_stream_uniform(g);
        const float V = spk_stream_uniform(g);
        float k, us;
        const int r = spk_ptrs_squeeze(p, u, V, &k, &us);
        if (r == SPK_PTRS_ACCEPT) return k;
        if (r == SPK_PTRS_REJECT) continue;
        if (spk_ptrs_test(p, V, k, us)) return k;
    }
    return SPK_FLOOR(p->lam);
}

/* lam < 10 (and NaN): multiply uniforms until the product falls to exp(-lam) */
SPK_HD float spk_poisson_product(float lam, spk_stream* g) {
    const float E = spk_expf(-lam);
    float X = 0.0f;
    float prod = 1.0f;
    for (int it = 0; it < 512; ++it) {
        prod = SPK_MUL(prod, spk_stream_uniform(g));
        if (prod > E) {
            X = SPK_ADD(X, 1.0f);
        } else {
            return X;
        }
    }
    return X;
}

SPK_HD float spk_poisson(float lam, uint32_t pixel, uint32_t stream, uint32_t seed) {
    spk_stream g;
    spk_stream_init(&g, pixel, stream, seed);
    if (lam >= 10.0f) {
        spk_ptrs p;
        spk_ptrs_init(&p, lam);
        spk_ptrs_init_test(&p);
        return spk_ptrs_from(&p, &g, 0);
    }
    return spk_poisson_product(lam, &g);
}

/* lam for a sub-layer draw; a NaN density gives NaN (and then no draws) */
SPK_HD float spk_sublayer_lambda(float d, float D, float n, float u, float* sat_out) {
    float q = SPK_DIV(d, D);
    q = q < 1e-6f ? 1e-6f : (q > 0.999999f ? 0.999999f : q);
    const float sat = SPK_SUB(1.0f, SPK_MUL(SPK_MUL(q, u), 0.999999f));
    *sat_out = sat;
    return SPK_MUL(SPK_DIV(n, sat), q);
}

SPK_HD float spk_sublayer_draw(float d, float D, float n, float u, uint32_t pixel, uint32_t stream, uint32_t seed) {
    float sat;
    const float lam = spk_sublayer_lambda(d, D, n, u, &sat);
    return SPK_MUL(spk_poisson(lam, pixel, stream, seed), SPK_MUL(SPK_DIV(D, n), sat));
}

/* Box-Muller lognormal of mean m and standard deviation s from words x, y of block 0 */
SPK_HD float spk_lognormal(float m, float s, uint32_t pixel, uint32_t stream, uint32_t seed) {
    spk_stream g;
    spk_stream_init(&g, pixel, stream, seed);
    const float u1 = spk_stream_uniform(&g);
    const float u2 = spk_stream_uniform(&g);
    const float z = SPK_MUL(SPK_SQRT(SPK_MUL(-2.0f, spk_logf(u1))), spk_cosf(SPK_MUL(SPK_TWO_PI, u2)));
    const float sig = SPK_SQRT(spk_logf(SPK_ADD(1.0f, SPK_DIV(SPK_MUL(s, s), SPK_MUL(m, m)))));
    const float mu = SPK_SUB(spk_logf(m), SPK_MUL(SPK_MUL(0.5f, sig), sig));
    return spk_expf(SPK_ADD(mu, SPK_MUL(sig, z)));
}

#endif /* SPKB_GRAIN_SAMPLER_H */
