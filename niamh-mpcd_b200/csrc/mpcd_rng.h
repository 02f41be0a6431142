/*
 * mpcd_rng.h -- counter-based random variates for the MPCD solvent timestep.
 *
 * The reference draws every random number from one global sequential
 * generator (Mersenne Twister or xoshiro, mpcd/subroutines/rand.c:40-275), so
 * the value a cell or particle receives depends on the order in which the
 * serial loops visit them.  A GPU step visits cells and particles in no fixed
 * order, so here every variate is a pure function of
 *
 *     (seed, replica, step, stream, entity id, draw index)
 *
 * computed with Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random
 * numbers: as easy as 1, 2, 3", SC'11).  The same header compiles as C99 for
 * the host and as CUDA for sm_100a, and the floating-point steps use only
 * correctly rounded operations written out explicitly (no contraction into
 * FMA unless an fma is written), so host and device produce bit-identical
 * draws.  That lets a CPU checker consume exactly the numbers the GPU used.
 *
 * Distributions follow the reference's own methods:
 *   - uniform on [0,1) from a 32-bit word scaled by 2^-32, as genrand_real
 *     (rand.c:365-368);
 *   - random unit axis in 3D by Marsaglia's rejection method, as ranvec3D
 *     (rand.c:708-722);
 *   - Gaussian by the polar Box-Muller method in single precision, as
 *     genrand_gauss (rand.c:473-498), scaled in double by sqrt(kT/m) as
 *     genrand_gaussMB (rand.c:510-513).  The natural logarithm is a
 *     deterministic atanh-series evaluation (ln m = 2 atanh((m-1)/(m+1))).
 */
#ifndef MPCD_RNG_H
#define MPCD_RNG_H

#include <stdint.h>

#if defined(__CUDACC__)
#define MPCD_HD __host__ __device__ __forceinline__
#else
#define MPCD_HD static inline
#include <math.h>
#include <string.h>
#endif

/* Streams: which random quantity of a step a counter belongs to. */
enum {
    MPCD_STREAM_SHIFT = 1,   /* grid shift, 3 uniforms per step            */
    MPCD_STREAM_AXIS = 2,    /* SRD rotation axis, per cell                */
    MPCD_STREAM_THERMAL = 3, /* Andersen thermal velocities, per particle  */
    MPCD_STREAM_GHOST = 4,   /* phantom-particle momentum, per cell        */
    MPCD_STREAM_LC = 5,      /* Maier-Saupe Metropolis uniforms, per particle */
    MPCD_STREAM_ORTH = 6,    /* orthogonal-axis choice, per cell           */
    /* initial state (step 0), per particle: */
    MPCD_STREAM_INIT_POS = 7, /* positions, 4 uniforms per placement attempt */
    MPCD_STREAM_INIT_VEL = 8, /* velocities                                  */
    MPCD_STREAM_INIT_ORI = 9, /* orientations                                */
    MPCD_STREAM_RETHERM = 10, /* bounce-limit re-thermalisation, per particle,
                                 4 draws per re-thermalisation of a step    */
    /* re-placement of a particle that left the grid, per particle and step: */
    MPCD_STREAM_ESCAPE_POS = 11, /* position, DIM uniforms per attempt       */
    MPCD_STREAM_ESCAPE_VEL = 12, /* velocity, DIM normals                    */
    MPCD_STREAM_ESCAPE_ORI = 13, /* nematic orientation, one uniform         */
    MPCD_STREAM_VICSEK = 14      /* Vicsek cone, 2 (3D) or 1 (2D) uniforms per
                                    particle                                   */
};

/* Maximum Philox blocks a rejection loop may consume (2 attempts per block).
 * Failure probability for the polar method is (1-pi/4)^64 < 1e-42. */
#define MPCD_RNG_MAX_BLOCKS 32

/* ---- exactly rounded primitives (no implicit contraction) -------------- */
#if defined(__CUDA_ARCH__)
#define MPCD_FMUL(a, b) __fmul_rn((a), (b))
#define MPCD_FADD(a, b) __fadd_rn((a), (b))
#define MPCD_FSUB(a, b) __fsub_rn((a), (b))
#define MPCD_FDIV(a, b) __fdiv_rn((a), (b))
#define MPCD_FSQRT(a) __fsqrt_rn((a))
#define MPCD_FFMA(a, b, c) __fmaf_rn((a), (b), (c))
#define MPCD_DMUL(a, b) __dmul_rn((a), (b))
#define MPCD_DADD(a, b) __dadd_rn((a), (b))
#define MPCD_DSUB(a, b) __dsub_rn((a), (b))
#define MPCD_DSQRT(a) __dsqrt_rn((a))
#define MPCD_DDIV(a, b) __ddiv_rn((a), (b))
#else
/* Host builds must use -ffp-contract=off so these stay single operations. */
#define MPCD_FMUL(a, b) ((float)(a) * (float)(b))
#define MPCD_FADD(a, b) ((float)(a) + (float)(b))
#define MPCD_FSUB(a, b) ((float)(a) - (float)(b))
#define MPCD_FDIV(a, b) ((float)(a) / (float)(b))
#define MPCD_FSQRT(a) sqrtf((a))
#define MPCD_FFMA(a, b, c) fmaf((a), (b), (c))
#define MPCD_DMUL(a, b) ((double)(a) * (double)(b))
#define MPCD_DADD(a, b) ((double)(a) + (double)(b))
#define MPCD_DSUB(a, b) ((double)(a) - (double)(b))
#define MPCD_DSQRT(a) sqrt((a))
#define MPCD_DDIV(a, b) ((double)(a) / (double)(b))
#endif

typedef struct {
    uint32_t x, y, z, w;
} mpcd_u4;

MPCD_HD uint32_t mpcd_mulhi32(uint32_t a, uint32_t b) {
#if defined(__CUDA_ARCH__)
    return __umulhi(a, b);
#else
    return (uint32_t)(((uint64_t)a * (uint64_t)b) >> 32);
#endif
}

/* Philox4x32-10: ten rounds of the published S-box with Weyl key bumps. */
MPCD_HD mpcd_u4 mpcd_philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                            uint64_t key) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
    const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
    uint32_t k0 = (uint32_t)key, k1 = (uint32_t)(key >> 32);
    int r;
    for (r = 0; r < 10; ++r) {
        uint32_t hi0 = mpcd_mulhi32(M0, c0), lo0 = M0 * c0;
        uint32_t hi1 = mpcd_mulhi32(M1, c2), lo1 = M1 * c2;
        uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
        c0 = n0;
        c1 = lo1;
        c2 = n2;
        c3 = lo0;
        k0 += W0;
        k1 += W1;
    }
    mpcd_u4 o;
    o.x = c0;
    o.y = c1;
    o.z = c2;
    o.w = c3;
    return o;
}

/* Counter block for (stream, entity, block index) of one replica and step. */
MPCD_HD mpcd_u4 mpcd_block(uint64_t seed, uint32_t replica, uint32_t step,
                           uint32_t stream, uint32_t id, uint32_t blk) {
    return mpcd_philox(id, step, (stream << 24) | (blk & 0x00FFFFFFu), replica,
                       seed);
}

MPCD_HD uint32_t mpcd_lane(mpcd_u4 r, int k) {
    return k == 0 ? r.x : (k == 1 ? r.y : (k == 2 ? r.z : r.w));
}

/* uniform double on [0,1): exact multiple of 2^-32, as genrand_real. */
MPCD_HD double mpcd_u01(uint32_t v) { return (double)v * 0x1p-32; }

/* uniform float on [0,1): exact multiple of 2^-24. */
MPCD_HD float mpcd_u01f(uint32_t v) {
    return (float)(v >> 8) * 0x1p-24f;
}

MPCD_HD uint32_t mpcd_f2u(float f) {
#if defined(__CUDA_ARCH__)
    return __float_as_uint(f);
#else
    uint32_t u;
    memcpy(&u, &f, 4);
    return u;
#endif
}
MPCD_HD float mpcd_u2f(uint32_t u) {
#if defined(__CUDA_ARCH__)
    return __uint_as_float(u);
#else
    float f;
    memcpy(&f, &u, 4);
    return f;
#endif
}

/* Natural log of a positive normal float, evaluated identically on host and
 * device: x = m 2^e with m in [sqrt(1/2), sqrt(2)), ln m = 2 atanh(s),
 * s = (m-1)/(m+1), series through s^11.  Max error about 1 ulp. */
MPCD_HD float mpcd_logf(float x) {
    uint32_t b = mpcd_f2u(x);
    int ex = (int)((b >> 23) & 0xFFu) - 127;
    float m = mpcd_u2f((b & 0x007FFFFFu) | 0x3F800000u);
    if (m > 1.41421354f) {
        m = MPCD_FMUL(m, 0.5f);
        ex += 1;
    }
    float f = MPCD_FSUB(m, 1.0f);
    float s = MPCD_FDIV(f, MPCD_FADD(2.0f, f));
    float s2 = MPCD_FMUL(s, s);
    /* 1/11, 1/9, 1/7, 1/5, 1/3 */
    float p = MPCD_FFMA(s2, 0x1.745d18p-4f, 0x1.c71c72p-4f);
    p = MPCD_FFMA(s2, p, 0x1.24924ap-3f);
    p = MPCD_FFMA(s2, p, 0x1.99999ap-3f);
    p = MPCD_FFMA(s2, p, 0x1.555556p-2f);
    float t = MPCD_FMUL(2.0f, s);
    float lnm = MPCD_FFMA(MPCD_FMUL(t, s2), p, t);
    float fe = (float)ex;
    /* ln 2 split so that fe*LN2_HI is exact for |e| < 2^8 */
    return MPCD_FFMA(fe, 0x1.62e400p-1f, MPCD_FFMA(fe, 0x1.7f7d1cp-20f, lnm));
}

/* Grid shift for a step: three uniforms in [0,1) (x, y, z), as ranshift
 * (rand.c:678-696) produces them.  Axes beyond dim are zero. */
MPCD_HD void mpcd_rng_shift(uint64_t seed, uint32_t replica, uint32_t step,
                            int dim, double s[3]) {
    mpcd_u4 r = mpcd_block(seed, replica, step, MPCD_STREAM_SHIFT, 0u, 0u);
    s[0] = mpcd_u01(r.x);
    s[1] = dim >= 2 ? mpcd_u01(r.y) : 0.0;
    s[2] = dim >= 3 ? mpcd_u01(r.z) : 0.0;
}

/* Random unit vector on S^2 by Marsaglia's method (ranvec3D, rand.c:708-722):
 * x,y uniform in [-1,1), reject x^2+y^2 > 1, v = (2x sqrt(1-s), 2y sqrt(1-s),
 * 1-2s). */
MPCD_HD void mpcd_rng_axis3(uint64_t seed, uint32_t replica, uint32_t step,
                            uint32_t cell, double v[3]) {
    uint32_t blk;
    for (blk = 0; blk < MPCD_RNG_MAX_BLOCKS; ++blk) {
        mpcd_u4 r = mpcd_block(seed, replica, step, MPCD_STREAM_AXIS, cell, blk);
        int a;
        for (a = 0; a < 2; ++a) {
            double x = MPCD_DSUB(MPCD_DMUL(2.0, mpcd_u01(a ? r.z : r.x)), 1.0);
            double y = MPCD_DSUB(MPCD_DMUL(2.0, mpcd_u01(a ? r.w : r.y)), 1.0);
            double s = MPCD_DADD(MPCD_DMUL(x, x), MPCD_DMUL(y, y));
            if (s <= 1.0) {
                double f = MPCD_DMUL(2.0, MPCD_DSQRT(MPCD_DSUB(1.0, s)));
                v[0] = MPCD_DMUL(f, x);
                v[1] = MPCD_DMUL(f, y);
                v[2] = MPCD_DSUB(1.0, MPCD_DMUL(2.0, s));
                return;
            }
        }
    }
    v[0] = 0.0;
    v[1] = 0.0;
    v[2] = 1.0;
}

/* Pair of standard normals by the polar method in single precision
 * (genrand_gauss, rand.c:473-498).  'pair' selects independent pairs for the
 * same entity (e.g. components 0,1 and 2 of a 3D thermal velocity). */
MPCD_HD void mpcd_rng_normal2(uint64_t seed, uint32_t replica, uint32_t step,
                              uint32_t stream, uint32_t id, uint32_t pair,
                              float g[2]) {
    uint32_t blk;
    for (blk = 0; blk < MPCD_RNG_MAX_BLOCKS; ++blk) {
        mpcd_u4 r = mpcd_block(seed, replica, step, stream, id,
                               (pair << 8) | blk);
        int a;
        for (a = 0; a < 2; ++a) {
            float x1 = MPCD_FSUB(MPCD_FMUL(2.0f, mpcd_u01f(a ? r.z : r.x)), 1.0f);
            float x2 = MPCD_FSUB(MPCD_FMUL(2.0f, mpcd_u01f(a ? r.w : r.y)), 1.0f);
            float w = MPCD_FADD(MPCD_FMUL(x1, x1), MPCD_FMUL(x2, x2));
            if (w < 1.0f && w > 0.0f) {
                float f = MPCD_FSQRT(
                    MPCD_FDIV(MPCD_FMUL(-2.0f, mpcd_logf(w)), w));
                g[0] = MPCD_FMUL(x1, f);
                g[1] = MPCD_FMUL(x2, f);
                return;
            }
        }
    }
    g[0] = 0.0f;
    g[1] = 0.0f;
}

/* The k-th standard normal of an entity's sequence (k = 0,1 from pair 0,
 * k = 2,3 from pair 1, ...). */
MPCD_HD float mpcd_rng_normal(uint64_t seed, uint32_t replica, uint32_t step,
                              uint32_t stream, uint32_t id, uint32_t k) {
    float g[2];
    mpcd_rng_normal2(seed, replica, step, stream, id, k >> 1, g);
    return (k & 1u) ? g[1] : g[0];
}

/* The k-th uniform double of an entity's sequence (four per Philox block). */
MPCD_HD double mpcd_rng_uniform(uint64_t seed, uint32_t replica, uint32_t step,
                                uint32_t stream, uint32_t id, uint32_t k) {
    mpcd_u4 r = mpcd_block(seed, replica, step, stream, id, k >> 2);
    return mpcd_u01(mpcd_lane(r, (int)(k & 3u)));
}

/* The Cartesian axis of a cell's orthogonal-axis SRD rotation: the
 * reference's CA = (int)DIM * genrand_real() (stochrotMPC, mpc.c:1289) with
 * the cell's first uniform of its own stream, in 0..dim-1. */
MPCD_HD int mpcd_rng_orth_axis(uint64_t seed, uint32_t replica, uint32_t step,
                               uint32_t cell, int dim) {
    int ca = (int)(MPCD_DMUL((double)dim, mpcd_rng_uniform(seed, replica, step,
                                                          MPCD_STREAM_ORTH, cell, 0u)));
    return ca < dim ? ca : dim - 1;
}

#endif /* MPCD_RNG_H */
