// plis_stream.h — the random stream and the scalar numerics of the tau-leaping step.
//
// This header is compiled unchanged by nvcc (device code of the CUDA step) and by g++ (the FP64/FP32
// host oracle under oracle/, which is test infrastructure).  Everything here is plain IEEE-754
// arithmetic (+ - * / sqrt floor fma), integer operations and bit manipulation, so both compilers
// produce the same bits provided no floating-point contraction is added behind our back:
// nvcc gets -fmad=false, g++ gets -ffp-contract=off.  Explicit fma() calls are used where wanted
// (they are correctly rounded on both sides).
//
// What lives here and why:
//  * Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy as 1, 2, 3", SC'11):
//    a counter-based generator.  The reference keeps one stateful cuRAND MRG32k3a state per
//    subvolume (PLISCuda/src/init.cu:3-13, 192 bytes each, read-modify-written on every draw);
//    here a draw is a pure function of (seed, replica, subvolume, step, attempt, channel, sub),
//    so no generator state lives in memory and a step can be replayed bit-exactly.
//  * exp / log written from the mathematics: Cody-Waite range reduction by ln 2 followed by the
//    Taylor series of e^r (|r| <= ln2/2), and the atanh series ln m = 2 atanh((m-1)/(m+1)) for
//    m in [sqrt(1/2), sqrt(2)).  The split of ln 2 into a 32-bit head and a tail was derived with
//    mpmath; the series coefficients are 1/n! and 1/(2k+1) rounded to nearest.
//  * ln k! : exact table for k <= 16 (mpmath, rounded to nearest), Stirling's series above.
//  * Poisson variates: inversion by sequential search for lambda < 10, and PTRS
//    (W. Hormann, "The transformed rejection method for generating Poisson random variables",
//    Insurance: Mathematics and Economics 12 (1993) 39-45) for lambda >= 10.
//    The reference calls curand_poisson (PLISCuda/src/leap.cu:27, :51).
//  * Exponential variates -ln(U)/a (the reference: -logf(curand_uniform)/a, PLISCuda/src/tau.cu:193-194).
#ifndef PLIS_STREAM_H_
#define PLIS_STREAM_H_

#include <stdint.h>

#if defined(__CUDACC__)
#define PLIS_HD __host__ __device__ __forceinline__
#define PLIS_FMA(a, b, c) fma((a), (b), (c))
#define PLIS_FMAF(a, b, c) fmaf((a), (b), (c))
#define PLIS_FLOOR(x) floor(x)
#define PLIS_FLOORF(x) floorf(x)
#define PLIS_SQRT(x) sqrt(x)
#define PLIS_SQRTF(x) sqrtf(x)
#define PLIS_FABS(x) fabs(x)
#define PLIS_FABSF(x) fabsf(x)
#else
#include <math.h>
#include <string.h>
#define PLIS_HD static inline
#define PLIS_FMA(a, b, c) fma((a), (b), (c))
#define PLIS_FMAF(a, b, c) fmaf((a), (b), (c))
#define PLIS_FLOOR(x) floor(x)
#define PLIS_FLOORF(x) floorf(x)
#define PLIS_SQRT(x) sqrt(x)
#define PLIS_SQRTF(x) sqrtf(x)
#define PLIS_FABS(x) fabs(x)
#define PLIS_FABSF(x) fabsf(x)
#endif

// ------------------------------------------------------------------------------------------------
// bit casts
// ------------------------------------------------------------------------------------------------
PLIS_HD uint64_t plis_d2u(double x) {
#if defined(__CUDA_ARCH__)
  return (uint64_t)__double_as_longlong(x);
#else
  uint64_t u; memcpy(&u, &x, 8); return u;
#endif
}
PLIS_HD double plis_u2d(uint64_t u) {
#if defined(__CUDA_ARCH__)
  return __longlong_as_double((long long)u);
#else
  double x; memcpy(&x, &u, 8); return x;
#endif
}
PLIS_HD uint32_t plis_f2u(float x) {
#if defined(__CUDA_ARCH__)
  return (uint32_t)__float_as_uint(x);
#else
  uint32_t u; memcpy(&u, &x, 4); return u;
#endif
}
PLIS_HD float plis_u2f(uint32_t u) {
#if defined(__CUDA_ARCH__)
  return __uint_as_float(u);
#else
  float x; memcpy(&x, &u, 4); return x;
#endif
}

#define PLIS_INF_D (plis_u2d(0x7FF0000000000000ull))
#define PLIS_NAN_D (plis_u2d(0x7FF8000000000000ull))
#define PLIS_INF_F (plis_u2f(0x7F800000u))
#define PLIS_NAN_F (plis_u2f(0x7FC00000u))

PLIS_HD int plis_isinf_d(double x) { return (plis_d2u(x) & 0x7FFFFFFFFFFFFFFFull) == 0x7FF0000000000000ull; }
PLIS_HD int plis_isinf_f(float x) { return (plis_f2u(x) & 0x7FFFFFFFu) == 0x7F800000u; }

// ------------------------------------------------------------------------------------------------
// Philox4x32-10
// ------------------------------------------------------------------------------------------------
#define PLIS_PHILOX_M0 0xD2511F53u
#define PLIS_PHILOX_M1 0xCD9E8D57u
#define PLIS_PHILOX_W0 0x9E3779B9u
#define PLIS_PHILOX_W1 0xBB67AE85u

typedef struct plis_u32x4 { uint32_t x, y, z, w; } plis_u32x4;

PLIS_HD plis_u32x4 plis_philox4x32_10(plis_u32x4 c, uint32_t k0, uint32_t k1) {
#if defined(__CUDA_ARCH__)
#pragma unroll
#endif
  for (int i = 0; i < 10; ++i) {
    uint64_t p0 = (uint64_t)PLIS_PHILOX_M0 * (uint64_t)c.x;
    uint64_t p1 = (uint64_t)PLIS_PHILOX_M1 * (uint64_t)c.z;
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    plis_u32x4 n;
    n.x = hi1 ^ c.y ^ k0;
    n.y = lo1;
    n.z = hi0 ^ c.w ^ k1;
    n.w = lo0;
    c = n;
    k0 += PLIS_PHILOX_W0;
    k1 += PLIS_PHILOX_W1;
  }
  return c;
}

// ------------------------------------------------------------------------------------------------
// Counter layout.  One "channel" of one subvolume in one phase of one attempt of one step owns the
// sub-stream (c.y low 12 bits = sub, incremented per Philox block).  A sub-stream holds 4096 blocks
// (8192 binary64 or 16384 binary32 uniforms); the step never needs more than 64 blocks from one
// (PTRS gives up after 64 rejections, the inversion search draws one uniform):
//   c.x = subvolume index (within its replica)
//   c.y = channel << 12 | sub          (channel < 2^20)
//   c.z = step (low 32 bits)
//   c.w = phase << 28 | (attempt & 0xFFF) << 16 | (step >> 32) & 0xFFFF
//   key = (seed low 32, seed high 32 xor replica * 0x632BE5AB)
// ------------------------------------------------------------------------------------------------
enum {
  PLIS_PHASE_TAU = 1,    // exponential next-event times drawn while classifying
  PLIS_PHASE_LEAP = 2,   // Poisson firings of non-critical reactions and diffusions
  PLIS_PHASE_CRIT = 3,   // the single critical event of a LEAP_CR subvolume
  PLIS_PHASE_SSA = 4,    // the exact event of the arg-min subvolume
  PLIS_PHASE_INIT = 5    // synthetic initial states (generators)
};

#define PLIS_CH_DIFF_BASE 0x40000u  // diffusion channels: base + species * 8 + slot
PLIS_HD uint32_t plis_ch_react(uint32_t r) { return r; }
PLIS_HD uint32_t plis_ch_diff(uint32_t s, uint32_t slot) { return PLIS_CH_DIFF_BASE + s * 8u + slot; }
// Grouped channels: the single uniforms of the inversion-searched draws (means below
// PLIS_LEAP_INV_MAX) of a group come from shared Philox blocks, four uniforms per block (uniform i of
// a group: word i % 4 of block i / 4).  Reactions 4g .. 4g+3 form group g; the six
// neighbour slots of one species form its diffusion group.  Draws searched by PTRS keep their own
// channels (plis_ch_react, plis_ch_diff).
// The leap's draws search by inversion up to a mean of 20 (the stand-alone samplers below switch to
// PTRS at 10): a search from 0 costs about lambda + 3 sqrt(lambda) iterations of a few operations for
// the slowest lane of a warp, where PTRS costs a few hundred divergent instructions per draw, and
// the two cross near 20.  Both searches are exact samplers, so the mean only picks the algorithm.
#define PLIS_LEAP_INV_MAX 20.0
#define PLIS_CH_RGROUP_BASE 0x20000u  // + reaction group
#define PLIS_CH_DGROUP_BASE 0x60000u  // + species
PLIS_HD uint32_t plis_ch_rgroup(uint32_t g) { return PLIS_CH_RGROUP_BASE + g; }
PLIS_HD uint32_t plis_ch_dgroup(uint32_t s) { return PLIS_CH_DGROUP_BASE + s; }

// Pooled draws.  A leap of a network with many channels, most of them with tiny means, draws the
// channels of small mean together: walking the reactions (in order) and then the diffusing species
// (in order), a channel whose mean is below PLIS_POOL_CUT joins the pool while the pool's total mean
// stays at most PLIS_POOL_MAX (a species joins with its n neighbour slots, weight n * mean).  The
// pool's total K ~ Poisson(total) comes by inversion from word x of block 0 of the pool channel;
// event e (0-based) takes block e + 1: word x picks the channel with probability weight / total
// (cumulative weights in walking order), word y the neighbour slot of a diffusion event,
// slot = (y * n) >> 32.  Given K the channel counts are multinomial, so every pooled channel's count
// is Poisson(mean) and independent of the others, as a draw per channel would be (Poisson splitting;
// up to the 2^-32 resolution of the choices).  The other channels draw as before.
#define PLIS_CH_POOL 0x7FFFFu
#define PLIS_POOL_CUT 0.125
#define PLIS_POOL_MAX 1.0
PLIS_HD uint32_t plis_pool_slot(uint32_t y, uint32_t n) { return (uint32_t)(((uint64_t)y * (uint64_t)n) >> 32); }

typedef struct plis_stream {
  plis_u32x4 ctr;
  uint32_t k0, k1;
  plis_u32x4 buf;
  int avail;  // 32-bit words left in buf
} plis_stream;

PLIS_HD plis_stream plis_stream_make(uint64_t seed, uint32_t replica, uint32_t cell, uint32_t phase,
                                     uint64_t step, uint32_t attempt, uint32_t channel) {
  plis_stream s;
  s.ctr.x = cell;
  s.ctr.y = (channel & 0xFFFFFu) << 12;
  s.ctr.z = (uint32_t)step;
  s.ctr.w = ((phase & 0xFu) << 28) | ((attempt & 0xFFFu) << 16) | (uint32_t)((step >> 32) & 0xFFFFu);
  s.k0 = (uint32_t)seed;
  s.k1 = (uint32_t)(seed >> 32) ^ (replica * 0x632BE5ABu);
  s.buf.x = s.buf.y = s.buf.z = s.buf.w = 0u;
  s.avail = 0;
  return s;
}

PLIS_HD void plis_stream_refill(plis_stream* s) {
  s->buf = plis_philox4x32_10(s->ctr, s->k0, s->k1);
  s->ctr.y = (s->ctr.y & 0xFFFFF000u) | ((s->ctr.y + 1u) & 0xFFFu);
  s->avail = 4;
}

PLIS_HD uint32_t plis_stream_u32(plis_stream* s) {
  if (s->avail == 0) plis_stream_refill(s);
  uint32_t r;
  switch (s->avail) {
    case 4: r = s->buf.x; break;
    case 3: r = s->buf.y; break;
    case 2: r = s->buf.z; break;
    default: r = s->buf.w; break;
  }
  s->avail -= 1;
  return r;
}

// Uniform double strictly inside (0,1): 52 random bits, (x + 1/2) * 2^-52.  Exact in binary64.
PLIS_HD double plis_uniform_d(plis_stream* s) {
  uint32_t hi = plis_stream_u32(s);
  uint32_t lo = plis_stream_u32(s);
  uint64_t x = (((uint64_t)hi << 32) | (uint64_t)lo) >> 12;
  return ((double)x + 0.5) * 2.220446049250313e-16;  // 2^-52
}

// Uniform float strictly inside (0,1): 23 random bits, (x + 1/2) * 2^-23.  Exact in binary32.
PLIS_HD float plis_uniform_f(plis_stream* s) {
  uint32_t x = plis_stream_u32(s) >> 9;
  return ((float)x + 0.5f) * 1.1920928955078125e-07f;  // 2^-23
}

// Uniforms 0 .. n-1 of a group (n <= 8): u[i] for every i whose bit is set in `need` (the others may
// be left unset).  `g` is the group's stream (plis_stream_make with the group channel); its blocks
// are computed here, only those holding a needed uniform.  Uniform i is word i%4 of block i/4 in both
// precisions: binary64 takes all 32 bits of the word, (w + 1/2) 2^-32 (exact in binary64; an
// inversion search from 0 only ever compares it with a CDF, and 2^-32 resolution leaves unreached
// only upper tails of probability below 2^-33), binary32 the top 23 bits as plis_uniform_f does.
PLIS_HD plis_u32x4 plis_group_block(const plis_stream* g, uint32_t b) {
  plis_u32x4 ctr = g->ctr;
  ctr.y = (ctr.y & 0xFFFFF000u) | (b & 0xFFFu);
  return plis_philox4x32_10(ctr, g->k0, g->k1);
}

PLIS_HD double plis_u32_to_uniform_d(uint32_t w) {
  return ((double)w + 0.5) * 2.3283064365386963e-10;  // 2^-32
}

PLIS_HD float plis_u32_to_uniform_f(uint32_t w) {
  uint32_t x = w >> 9;
  return ((float)x + 0.5f) * 1.1920928955078125e-07f;  // 2^-23
}

// Precomputed round keys.  The ten round keys of plis_philox4x32_10 under the key plis_stream_make
// derives from (seed, replica) are rk0[i] = k0 + i W0, rk1[i] = k1 + i W1; a caller that holds them
// (the step kernels keep them in their arguments) computes a block without the key schedule, with
// the same result as plis_philox4x32_10 / plis_group_block.
PLIS_HD void plis_round_keys(uint64_t seed, uint32_t replica, uint32_t rk0[10], uint32_t rk1[10]) {
  const plis_stream s = plis_stream_make(seed, replica, 0u, 0u, 0u, 0u, 0u);
  for (int i = 0; i < 10; ++i) {
    rk0[i] = s.k0 + (uint32_t)i * PLIS_PHILOX_W0;
    rk1[i] = s.k1 + (uint32_t)i * PLIS_PHILOX_W1;
  }
}

PLIS_HD plis_u32x4 plis_philox4x32_10_rk(plis_u32x4 c, const uint32_t rk0[10], const uint32_t rk1[10]) {
#if defined(__CUDA_ARCH__)
#pragma unroll
#endif
  for (int i = 0; i < 10; ++i) {
    uint64_t p0 = (uint64_t)PLIS_PHILOX_M0 * (uint64_t)c.x;
    uint64_t p1 = (uint64_t)PLIS_PHILOX_M1 * (uint64_t)c.z;
    plis_u32x4 n;
    n.x = (uint32_t)(p1 >> 32) ^ c.y ^ rk0[i];
    n.y = (uint32_t)p1;
    n.z = (uint32_t)(p0 >> 32) ^ c.w ^ rk1[i];
    n.w = (uint32_t)p0;
    c = n;
  }
  return c;
}

PLIS_HD plis_u32x4 plis_group_block_rk(const plis_stream* g, uint32_t b, const uint32_t rk0[10], const uint32_t rk1[10]) {
  plis_u32x4 ctr = g->ctr;
  ctr.y = (ctr.y & 0xFFFFF000u) | (b & 0xFFFu);
  return plis_philox4x32_10_rk(ctr, rk0, rk1);
}

// plis_group_uniforms_d / _f with precomputed round keys (same uniforms)
PLIS_HD void plis_group_uniforms_rk_d(const plis_stream* g, uint32_t need, double* u, int n, const uint32_t rk0[10],
                                      const uint32_t rk1[10]) {
#if defined(__CUDA_ARCH__)
#pragma unroll
#endif
  for (int b = 0; b < 2; ++b) {
    if (4 * b < n && (need >> (4 * b)) & 15u) {
      const plis_u32x4 w = plis_group_block_rk(g, (uint32_t)b, rk0, rk1);
      u[4 * b] = plis_u32_to_uniform_d(w.x);
      if (4 * b + 1 < n) u[4 * b + 1] = plis_u32_to_uniform_d(w.y);
      if (4 * b + 2 < n) u[4 * b + 2] = plis_u32_to_uniform_d(w.z);
      if (4 * b + 3 < n) u[4 * b + 3] = plis_u32_to_uniform_d(w.w);
    }
  }
}

PLIS_HD void plis_group_uniforms_rk_f(const plis_stream* g, uint32_t need, float* u, int n, const uint32_t rk0[10],
                                      const uint32_t rk1[10]) {
#if defined(__CUDA_ARCH__)
#pragma unroll
#endif
  for (int b = 0; b < 2; ++b) {
    if (4 * b < n && (need >> (4 * b)) & 15u) {
      const plis_u32x4 w = plis_group_block_rk(g, (uint32_t)b, rk0, rk1);
      u[4 * b] = plis_u32_to_uniform_f(w.x);
      if (4 * b + 1 < n) u[4 * b + 1] = plis_u32_to_uniform_f(w.y);
      if (4 * b + 2 < n) u[4 * b + 2] = plis_u32_to_uniform_f(w.z);
      if (4 * b + 3 < n) u[4 * b + 3] = plis_u32_to_uniform_f(w.w);
    }
  }
}

PLIS_HD void plis_group_uniforms_d(const plis_stream* g, uint32_t need, double* u, int n) {
#if defined(__CUDA_ARCH__)
#pragma unroll
#endif
  for (int b = 0; b < 2; ++b) {
    if (4 * b < n && (need >> (4 * b)) & 15u) {
      const plis_u32x4 w = plis_group_block(g, (uint32_t)b);
      u[4 * b] = plis_u32_to_uniform_d(w.x);
      if (4 * b + 1 < n) u[4 * b + 1] = plis_u32_to_uniform_d(w.y);
      if (4 * b + 2 < n) u[4 * b + 2] = plis_u32_to_uniform_d(w.z);
      if (4 * b + 3 < n) u[4 * b + 3] = plis_u32_to_uniform_d(w.w);
    }
  }
}

PLIS_HD void plis_group_uniforms_f(const plis_stream* g, uint32_t need, float* u, int n) {
#if defined(__CUDA_ARCH__)
#pragma unroll
#endif
  for (int b = 0; b < 2; ++b) {
    if (4 * b < n && (need >> (4 * b)) & 15u) {
      const plis_u32x4 w = plis_group_block(g, (uint32_t)b);
      u[4 * b] = plis_u32_to_uniform_f(w.x);
      if (4 * b + 1 < n) u[4 * b + 1] = plis_u32_to_uniform_f(w.y);
      if (4 * b + 2 < n) u[4 * b + 2] = plis_u32_to_uniform_f(w.z);
      if (4 * b + 3 < n) u[4 * b + 3] = plis_u32_to_uniform_f(w.w);
    }
  }
}

// ------------------------------------------------------------------------------------------------
// exp / log, binary64
// ------------------------------------------------------------------------------------------------
#define PLIS_LN2_HI 0.6931471803691238      // ln 2 rounded to 32 significant bits
#define PLIS_LN2_LO 1.9082149292705877e-10  // ln 2 - PLIS_LN2_HI
#define PLIS_INV_LN2 1.4426950408889634
#define PLIS_SQRT2 1.4142135623730951
#define PLIS_HALF_LN_2PI 0.9189385332046728

// 2^k for -1022 <= k <= 1023, by construction of the exponent field (exact).
PLIS_HD double plis_pow2i(int k) { return plis_u2d((uint64_t)(k + 1023) << 52); }

PLIS_HD double plis_exp(double x) {
  if (x != x) return x;
  if (x < -745.2) return 0.0;
  if (x > 709.78) return PLIS_INF_D;
  double kd = PLIS_FLOOR(x * PLIS_INV_LN2 + 0.5);
  int k = (int)kd;
  double r = (x - kd * PLIS_LN2_HI) - kd * PLIS_LN2_LO;
  // Taylor series of e^r through r^13 (|r| <= 0.3466: truncation < 5e-18)
  double p = 1.6059043836821613e-10;
  p = PLIS_FMA(p, r, 2.08767569878681e-09);
  p = PLIS_FMA(p, r, 2.505210838544172e-08);
  p = PLIS_FMA(p, r, 2.755731922398589e-07);
  p = PLIS_FMA(p, r, 2.7557319223985893e-06);
  p = PLIS_FMA(p, r, 2.48015873015873e-05);
  p = PLIS_FMA(p, r, 0.0001984126984126984);
  p = PLIS_FMA(p, r, 0.001388888888888889);
  p = PLIS_FMA(p, r, 0.008333333333333333);
  p = PLIS_FMA(p, r, 0.041666666666666664);
  p = PLIS_FMA(p, r, 0.16666666666666666);
  p = PLIS_FMA(p, r, 0.5);
  p = PLIS_FMA(p, r, 1.0);
  p = PLIS_FMA(p, r, 1.0);
  if (k >= -1022) {
    if (k > 1023) return (p * plis_pow2i(1023)) * 2.0;
    return p * plis_pow2i(k);
  }
  return (p * plis_pow2i(k + 60)) * 8.673617379884035e-19;  // 2^-60; rounds once into the subnormals
}

// e^x for -708 < x < 709 (normal results): plis_exp without its NaN and range tests, the same operations
// and therefore the same bits on that domain.  The leap's e^-lambda (0 <= lambda < PLIS_LEAP_INV_MAX).
PLIS_HD double plis_exp_normal(double x) {
  double kd = PLIS_FLOOR(x * PLIS_INV_LN2 + 0.5);
  int k = (int)kd;
  double r = (x - kd * PLIS_LN2_HI) - kd * PLIS_LN2_LO;
  double p = 1.6059043836821613e-10;
  p = PLIS_FMA(p, r, 2.08767569878681e-09);
  p = PLIS_FMA(p, r, 2.505210838544172e-08);
  p = PLIS_FMA(p, r, 2.755731922398589e-07);
  p = PLIS_FMA(p, r, 2.7557319223985893e-06);
  p = PLIS_FMA(p, r, 2.48015873015873e-05);
  p = PLIS_FMA(p, r, 0.0001984126984126984);
  p = PLIS_FMA(p, r, 0.001388888888888889);
  p = PLIS_FMA(p, r, 0.008333333333333333);
  p = PLIS_FMA(p, r, 0.041666666666666664);
  p = PLIS_FMA(p, r, 0.16666666666666666);
  p = PLIS_FMA(p, r, 0.5);
  p = PLIS_FMA(p, r, 1.0);
  p = PLIS_FMA(p, r, 1.0);
  return p * plis_pow2i(k);
}

PLIS_HD double plis_log(double x) {
  if (!(x > 0.0)) return (x == 0.0) ? -PLIS_INF_D : PLIS_NAN_D;
  if (plis_isinf_d(x)) return x;
  uint64_t b = plis_d2u(x);
  int e = (int)((b >> 52) & 0x7FF);
  if (e == 0) {  // subnormal: scale by 2^54 exactly
    x = x * 18014398509481984.0;
    b = plis_d2u(x);
    e = (int)((b >> 52) & 0x7FF) - 54;
  }
  e -= 1023;
  double m = plis_u2d((b & 0x000FFFFFFFFFFFFFull) | 0x3FF0000000000000ull);  // [1, 2)
  if (m > PLIS_SQRT2) { m = m * 0.5; e += 1; }
  double s = (m - 1.0) / (m + 1.0);
  double s2 = s * s;
  // atanh series: ln m = 2 (s + s^3/3 + ... + s^21/21); |s| <= 0.1716
  double q = 0.047619047619047616;
  q = PLIS_FMA(q, s2, 0.05263157894736842);
  q = PLIS_FMA(q, s2, 0.058823529411764705);
  q = PLIS_FMA(q, s2, 0.06666666666666667);
  q = PLIS_FMA(q, s2, 0.07692307692307693);
  q = PLIS_FMA(q, s2, 0.09090909090909091);
  q = PLIS_FMA(q, s2, 0.1111111111111111);
  q = PLIS_FMA(q, s2, 0.14285714285714285);
  q = PLIS_FMA(q, s2, 0.2);
  q = PLIS_FMA(q, s2, 0.3333333333333333);
  double lm = 2.0 * PLIS_FMA(s * s2, q, s);
  double ed = (double)e;
  return ed * PLIS_LN2_HI + (ed * PLIS_LN2_LO + lm);
}

// ln k!  (k >= 0)
PLIS_HD double plis_lnfact(double k) {
  if (k <= 16.0) {
    int i = (int)k;
    switch (i) {
      case 0: case 1: return 0.0;
      case 2: return 0.6931471805599453;
      case 3: return 1.791759469228055;
      case 4: return 3.1780538303479458;
      case 5: return 4.787491742782046;
      case 6: return 6.579251212010101;
      case 7: return 8.525161361065415;
      case 8: return 10.60460290274525;
      case 9: return 12.801827480081469;
      case 10: return 15.104412573075516;
      case 11: return 17.502307845873887;
      case 12: return 19.987214495661885;
      case 13: return 22.552163853123425;
      case 14: return 25.19122118273868;
      case 15: return 27.89927138384089;
      default: return 30.671860106080672;
    }
  }
  // Stirling: ln Gamma(z) = (z - 1/2) ln z - z + ln(2 pi)/2 + 1/(12z) - 1/(360z^3) + 1/(1260z^5)
  //                         - 1/(1680z^7) + 1/(1188z^9),  z = k + 1 >= 18
  double z = k + 1.0;
  double w = 1.0 / z;
  double w2 = w * w;
  double c = 0.0008417508417508417;
  c = 0.0005952380952380953 - w2 * c;
  c = 0.0007936507936507937 - w2 * c;
  c = 0.002777777777777778 - w2 * c;
  c = 0.08333333333333333 - w2 * c;
  return ((z - 0.5) * plis_log(z) - z) + (PLIS_HALF_LN_2PI + w * c);
}

// ------------------------------------------------------------------------------------------------
// Poisson, binary64
// ------------------------------------------------------------------------------------------------
// 1/k rounded to nearest, k = 0..200 (entry 0 unused): the inversion search multiplies by it
// instead of dividing.  On the device it sits in constant memory; every active lane of a warp is at
// the same k, so the read is a broadcast.
#define PLIS_INV_K_VALUES \
    0.0, 1.0, 0.5, 0.3333333333333333, 0.25, 0.2,\
    0.16666666666666666, 0.14285714285714285, 0.125, 0.1111111111111111, 0.1, 0.09090909090909091,\
    0.08333333333333333, 0.07692307692307693, 0.07142857142857142, 0.06666666666666667, 0.0625, 0.058823529411764705,\
    0.05555555555555555, 0.05263157894736842, 0.05, 0.047619047619047616, 0.045454545454545456, 0.043478260869565216,\
    0.041666666666666664, 0.04, 0.038461538461538464, 0.037037037037037035, 0.03571428571428571, 0.034482758620689655,\
    0.03333333333333333, 0.03225806451612903, 0.03125, 0.030303030303030304, 0.029411764705882353, 0.02857142857142857,\
    0.027777777777777776, 0.02702702702702703, 0.02631578947368421, 0.02564102564102564, 0.025, 0.024390243902439025,\
    0.023809523809523808, 0.023255813953488372, 0.022727272727272728, 0.022222222222222223, 0.021739130434782608, 0.02127659574468085,\
    0.020833333333333332, 0.02040816326530612, 0.02, 0.0196078431372549, 0.019230769230769232, 0.018867924528301886,\
    0.018518518518518517, 0.01818181818181818, 0.017857142857142856, 0.017543859649122806, 0.017241379310344827, 0.01694915254237288,\
    0.016666666666666666, 0.01639344262295082, 0.016129032258064516, 0.015873015873015872, 0.015625, 0.015384615384615385,\
    0.015151515151515152, 0.014925373134328358, 0.014705882352941176, 0.014492753623188406, 0.014285714285714285, 0.014084507042253521,\
    0.013888888888888888, 0.0136986301369863, 0.013513513513513514, 0.013333333333333334, 0.013157894736842105, 0.012987012987012988,\
    0.01282051282051282, 0.012658227848101266, 0.0125, 0.012345679012345678, 0.012195121951219513, 0.012048192771084338,\
    0.011904761904761904, 0.011764705882352941, 0.011627906976744186, 0.011494252873563218, 0.011363636363636364, 0.011235955056179775,\
    0.011111111111111112, 0.01098901098901099, 0.010869565217391304, 0.010752688172043012, 0.010638297872340425, 0.010526315789473684,\
    0.010416666666666666, 0.010309278350515464, 0.01020408163265306, 0.010101010101010102, 0.01, 0.009900990099009901,\
    0.00980392156862745, 0.009708737864077669, 0.009615384615384616, 0.009523809523809525, 0.009433962264150943, 0.009345794392523364,\
    0.009259259259259259, 0.009174311926605505, 0.00909090909090909, 0.009009009009009009, 0.008928571428571428, 0.008849557522123894,\
    0.008771929824561403, 0.008695652173913044, 0.008620689655172414, 0.008547008547008548, 0.00847457627118644, 0.008403361344537815,\
    0.008333333333333333, 0.008264462809917356, 0.00819672131147541, 0.008130081300813009, 0.008064516129032258, 0.008,\
    0.007936507936507936, 0.007874015748031496, 0.0078125, 0.007751937984496124, 0.007692307692307693, 0.007633587786259542,\
    0.007575757575757576, 0.007518796992481203, 0.007462686567164179, 0.007407407407407408, 0.007352941176470588, 0.0072992700729927005,\
    0.007246376811594203, 0.007194244604316547, 0.007142857142857143, 0.0070921985815602835, 0.007042253521126761, 0.006993006993006993,\
    0.006944444444444444, 0.006896551724137931, 0.00684931506849315, 0.006802721088435374, 0.006756756756756757, 0.006711409395973154,\
    0.006666666666666667, 0.006622516556291391, 0.006578947368421052, 0.006535947712418301, 0.006493506493506494, 0.0064516129032258064,\
    0.00641025641025641, 0.006369426751592357, 0.006329113924050633, 0.006289308176100629, 0.00625, 0.006211180124223602,\
    0.006172839506172839, 0.006134969325153374, 0.006097560975609756, 0.006060606060606061, 0.006024096385542169, 0.005988023952095809,\
    0.005952380952380952, 0.005917159763313609, 0.0058823529411764705, 0.005847953216374269, 0.005813953488372093, 0.005780346820809248,\
    0.005747126436781609, 0.005714285714285714, 0.005681818181818182, 0.005649717514124294, 0.0056179775280898875, 0.00558659217877095,\
    0.005555555555555556, 0.0055248618784530384, 0.005494505494505495, 0.00546448087431694, 0.005434782608695652, 0.005405405405405406,\
    0.005376344086021506, 0.0053475935828877, 0.005319148936170213, 0.005291005291005291, 0.005263157894736842, 0.005235602094240838,\
    0.005208333333333333, 0.0051813471502590676, 0.005154639175257732, 0.005128205128205128, 0.00510204081632653, 0.005076142131979695,\
    0.005050505050505051, 0.005025125628140704, 0.005,
#if defined(__CUDA_ARCH__)
static __constant__ double plis_inv_k_tab[201] = {PLIS_INV_K_VALUES};
#else
static const double plis_inv_k_tab[201] = {PLIS_INV_K_VALUES};
#endif

#define PLIS_POISSON_BIG 1099511627776.0  // 2^40: returned for lambda >= 2^40 (counts overflow anyway)

// Poisson(lam) for lam < 10 by inversion (sequential search from 0), given emlam = exp(-lam):
// draws that share a mean (the per-neighbour diffusion draws of one species) share the exp.
// inversion by sequential search from the uniform u (plis_poisson_small_d without its draw)
PLIS_HD double plis_poisson_inv_d(double u, double lam, double emlam) {
  double p = emlam;
  double F = p;
  double k = 0.0;
  int ki = 0;
  while (u > F) {
    k += 1.0;
    ki += 1;
    p = (p * lam) * plis_inv_k_tab[ki];
    F += p;
    if (p <= F * 8.673617379884035e-19 || ki >= 200) break;  // tail below 2^-60: stop
  }
  return k;
}

PLIS_HD double plis_poisson_small_d(plis_stream* st, double lam, double emlam) {
  double u = plis_uniform_d(st);
  double p = emlam;
  double F = p;
  double k = 0.0;
  int ki = 0;
  while (u > F) {
    k += 1.0;
    ki += 1;
    p = (p * lam) * plis_inv_k_tab[ki];
    F += p;
    if (p <= F * 8.673617379884035e-19 || ki >= 200) break;  // tail below 2^-60: stop
  }
  return k;
}

PLIS_HD double plis_poisson_d(plis_stream* st, double lam) {
  if (!(lam > 0.0)) return 0.0;
  if (lam >= PLIS_POISSON_BIG) return PLIS_POISSON_BIG;
  if (lam < 10.0) {
    // inversion by sequential search
    return plis_poisson_small_d(st, lam, plis_exp(-lam));
  }
  // PTRS, Hormann (1993).  ln(lambda) is needed only by the full acceptance test, which the squeeze
  // (us >= 0.07 && V <= vr) spares about 86 % of the draws, so it is computed on first use.
  double slam = PLIS_SQRT(lam);
  double loglam = -1.0;
  double b = 0.931 + 2.53 * slam;
  double a = -0.059 + 0.02483 * b;
  double invalpha = 1.1239 + 1.1328 / (b - 3.4);
  double vr = 0.9277 - 3.6224 / (b - 2.0);
  for (int it = 0; it < 64; ++it) {
    double U = plis_uniform_d(st) - 0.5;
    double V = plis_uniform_d(st);
    double us = 0.5 - PLIS_FABS(U);
    double k = PLIS_FLOOR((2.0 * a / us + b) * U + lam + 0.43);
    if (us >= 0.07 && V <= vr) return k;
    if (k < 0.0 || (us < 0.013 && V > us)) continue;
    double lhs = plis_log(V) + plis_log(invalpha) - plis_log(a / (us * us) + b);
    if (loglam < 0.0) loglam = plis_log(lam);  // lambda >= 10: ln(lambda) > 2
    double rhs = -lam + k * loglam - plis_lnfact(k);
    if (lhs <= rhs) return k;
  }
  return PLIS_FLOOR(lam);
}

// Integer value of a drawn count (clamped at 2^40 so the conversion is always defined).
PLIS_HD long long plis_count_d(double k) { return k >= PLIS_POISSON_BIG ? (1LL << 40) : (long long)k; }

PLIS_HD double plis_exponential_d(plis_stream* st, double rate) {
  double u = plis_uniform_d(st);
  return -plis_log(u) / rate;
}

// ------------------------------------------------------------------------------------------------
// binary32 variants (the FP32 precision form).  Same methods, shorter series; Poisson means of 10
// and above are sampled by the binary64 PTRS.
// ------------------------------------------------------------------------------------------------
#define PLIS_LN2_HI_F 0.69311523f      // ln 2 rounded to 12 significant bits
#define PLIS_LN2_LO_F 3.1946183e-05f   // ln 2 - PLIS_LN2_HI_F
#define PLIS_INV_LN2_F 1.442695f
#define PLIS_SQRT2_F 1.4142135f

PLIS_HD float plis_pow2i_f(int k) { return plis_u2f((uint32_t)(k + 127) << 23); }

PLIS_HD float plis_expf(float x) {
  if (x != x) return x;
  if (x < -103.9f) return 0.0f;
  if (x > 88.72f) return PLIS_INF_F;
  float kf = PLIS_FLOORF(x * PLIS_INV_LN2_F + 0.5f);
  int k = (int)kf;
  float r = (x - kf * PLIS_LN2_HI_F) - kf * PLIS_LN2_LO_F;
  float p = 2.4801588e-05f;  // Taylor through r^8
  p = PLIS_FMAF(p, r, 0.0001984127f);
  p = PLIS_FMAF(p, r, 0.0013888889f);
  p = PLIS_FMAF(p, r, 0.008333334f);
  p = PLIS_FMAF(p, r, 0.041666668f);
  p = PLIS_FMAF(p, r, 0.16666667f);
  p = PLIS_FMAF(p, r, 0.5f);
  p = PLIS_FMAF(p, r, 1.0f);
  p = PLIS_FMAF(p, r, 1.0f);
  if (k >= -126) {
    if (k > 127) return (p * plis_pow2i_f(127)) * 2.0f;
    return p * plis_pow2i_f(k);
  }
  return (p * plis_pow2i_f(k + 30)) * 9.3132257e-10f;  // 2^-30
}

// e^x for -87 < x < 88 (normal results): plis_expf without its NaN and range tests, the same bits there.
PLIS_HD float plis_expf_normal(float x) {
  float kf = PLIS_FLOORF(x * PLIS_INV_LN2_F + 0.5f);
  int k = (int)kf;
  float r = (x - kf * PLIS_LN2_HI_F) - kf * PLIS_LN2_LO_F;
  float p = 2.4801588e-05f;
  p = PLIS_FMAF(p, r, 0.0001984127f);
  p = PLIS_FMAF(p, r, 0.0013888889f);
  p = PLIS_FMAF(p, r, 0.008333334f);
  p = PLIS_FMAF(p, r, 0.041666668f);
  p = PLIS_FMAF(p, r, 0.16666667f);
  p = PLIS_FMAF(p, r, 0.5f);
  p = PLIS_FMAF(p, r, 1.0f);
  p = PLIS_FMAF(p, r, 1.0f);
  return p * plis_pow2i_f(k);
}

PLIS_HD float plis_logf(float x) {
  if (!(x > 0.0f)) return (x == 0.0f) ? -PLIS_INF_F : PLIS_NAN_F;
  if (plis_isinf_f(x)) return x;
  uint32_t b = plis_f2u(x);
  int e = (int)((b >> 23) & 0xFF);
  if (e == 0) {
    x = x * 16777216.0f;  // 2^24
    b = plis_f2u(x);
    e = (int)((b >> 23) & 0xFF) - 24;
  }
  e -= 127;
  float m = plis_u2f((b & 0x007FFFFFu) | 0x3F800000u);
  if (m > PLIS_SQRT2_F) { m = m * 0.5f; e += 1; }
  float s = (m - 1.0f) / (m + 1.0f);
  float s2 = s * s;
  float q = 0.09090909f;  // through s^11/11
  q = PLIS_FMAF(q, s2, 0.11111111f);
  q = PLIS_FMAF(q, s2, 0.14285715f);
  q = PLIS_FMAF(q, s2, 0.2f);
  q = PLIS_FMAF(q, s2, 0.33333334f);
  float lm = 2.0f * PLIS_FMAF(s * s2, q, s);
  float ef = (float)e;
  return ef * PLIS_LN2_HI_F + (ef * PLIS_LN2_LO_F + lm);
}

PLIS_HD double plis_poisson_inv_f(float u, float lam, float emlam) {
  float p = emlam;
  float F = p;
  float k = 0.0f;
  int ki = 0;
  while (u > F) {
    k += 1.0f;
    ki += 1;
    p = (p * lam) * (float)plis_inv_k_tab[ki];
    F += p;
    if (p <= F * 2.9802322e-08f || ki >= 100) break;  // tail below 2^-25
  }
  return (double)k;
}

PLIS_HD double plis_poisson_small_f(plis_stream* st, float lam, float emlam) {
  float u = plis_uniform_f(st);
  float p = emlam;
  float F = p;
  float k = 0.0f;
  int ki = 0;
  while (u > F) {
    k += 1.0f;
    ki += 1;
    p = (p * lam) * (float)plis_inv_k_tab[ki];
    F += p;
    if (p <= F * 2.9802322e-08f || ki >= 100) break;  // tail below 2^-25
  }
  return (double)k;
}

// Returns the count as a double (exact integer), like plis_poisson_d.
PLIS_HD double plis_poisson_f(plis_stream* st, float lam) {
  if (!(lam > 0.0f)) return 0.0;
  if (lam < 10.0f) return plis_poisson_small_f(st, lam, plis_expf(-lam));
  // lambda >= 10: the PTRS acceptance test compares ln-probabilities of size ~lambda*ln(lambda),
  // which binary32 cannot resolve (its spacing near 1e6 is 0.125), so it runs in binary64.
  return plis_poisson_d(st, (double)lam);
}

#endif  // PLIS_STREAM_H_
