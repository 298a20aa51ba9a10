// Counter-based random numbers shared bit-for-bit by the CUDA kernels and the
// host code (connection rules, the FP64 oracle).
//
// The reference draws its Poisson input from one cuRAND XORWOW state per
// direct connection (src/poiss_gen.cu:33-41 curand_init, :62 curand_poisson)
// and its random connectivity from the cuRAND host API (src/random.cu).
// Keeping a 48-byte generator state per connection costs HBM traffic on every
// step, so this build keys every draw by (seed, stream, step) instead:
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy
// as 1, 2, 3", SC'11) has no state, so nothing is read or written per draw.
//
// Poisson counts for lambda < NGPU_POISSON_INV_MAX use inversion by sequential
// search with a single uniform and only correctly rounded IEEE double
// operations (explicit *_rn intrinsics on the device, no contraction), so the
// GPU and the CPU oracle produce identical integer counts. Larger lambda uses
// Hoermann's PTRS transformed rejection ("The transformed rejection method for
// generating Poisson random variables", 1993), whose log/lgamma calls make it
// statistically but not bit-wise reproducible across host and device.
#pragma once
#include <stdint.h>
#include <math.h>

#if defined(__CUDACC__)
#define NG_HD __host__ __device__ __forceinline__
#else
#define NG_HD inline
#endif

namespace ngpu {

// random-number stream purposes (folded into the Philox key)
enum RngTag : uint32_t {
  RNG_TAG_POISSON_DIRECT = 1,   // poisson_generator direct connections
  RNG_TAG_POISSON_NODE = 2,     // CreatePoissonGenerator nodes
  RNG_TAG_CONNECT = 3,          // host connection rules
  RNG_TAG_ARRAY = 4,            // RandomUniform / RandomNormal arrays
  RNG_TAG_SOURCE_SET = 5,       // per-target source sampling
  RNG_TAG_MLP = 6               // step-proposer training samples
};

struct Philox4 {
  uint32_t v[4];
};

NG_HD void ng_mulhilo(uint32_t a, uint32_t b, uint32_t &hi, uint32_t &lo) {
#if defined(__CUDA_ARCH__)
  lo = a * b;
  hi = __umulhi(a, b);
#else
  uint64_t p = (uint64_t)a * (uint64_t)b;
  lo = (uint32_t)p;
  hi = (uint32_t)(p >> 32);
#endif
}

// Philox4x32 with 10 rounds.
NG_HD Philox4 philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2,
                            uint32_t c3, uint32_t k0, uint32_t k1) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
  const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
  for (int r = 0; r < 10; r++) {
    uint32_t hi0, lo0, hi1, lo1;
    ng_mulhilo(M0, c0, hi0, lo0);
    ng_mulhilo(M1, c2, hi1, lo1);
    uint32_t n0 = hi1 ^ c1 ^ k0;
    uint32_t n2 = hi0 ^ c3 ^ k1;
    c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
    k0 += W0; k1 += W1;
  }
  Philox4 out;
  out.v[0] = c0; out.v[1] = c1; out.v[2] = c2; out.v[3] = c3;
  return out;
}

// One block of 4x32 random bits for (seed, tag, stream, step, draw index).
NG_HD Philox4 ng_random_block(uint64_t seed, uint32_t tag, uint64_t stream,
                              int64_t step, uint32_t draw) {
  uint32_t k0 = (uint32_t)seed;
  uint32_t k1 = (uint32_t)(seed >> 32) ^ (tag * 0x85EBCA6Bu);
  uint64_t st = (uint64_t)step;
  return philox4x32_10((uint32_t)stream, (uint32_t)(stream >> 32),
                       (uint32_t)st,
                       (uint32_t)(st >> 32) ^ (draw << 16) ^ (draw >> 16),
                       k0, k1);
}

// uniform double in the open interval (0,1) from 64 random bits (53 used)
NG_HD double ng_u01(uint32_t a, uint32_t b) {
  uint64_t k = ((uint64_t)a << 21) ^ (uint64_t)(b >> 11);
  k &= ((uint64_t)1 << 53) - 1;
  return ((double)k + 0.5) * (1.0 / 9007199254740992.0);
}

// exact double arithmetic helpers (no FMA contraction on either side)
#if defined(__CUDA_ARCH__)
#define NG_DMUL(a, b) __dmul_rn((a), (b))
#define NG_DADD(a, b) __dadd_rn((a), (b))
#define NG_DDIV(a, b) __ddiv_rn((a), (b))
#else
#define NG_DMUL(a, b) ((a) * (b))
#define NG_DADD(a, b) ((a) + (b))
#define NG_DDIV(a, b) ((a) / (b))
#endif

#define NGPU_POISSON_INV_MAX 10.0

// Inversion by sequential search. exp_neg_lambda = exp(-lambda) is computed
// once on the host so no transcendental is evaluated here.
NG_HD uint32_t ng_poisson_inversion(double lambda, double exp_neg_lambda,
                                    double u) {
  uint32_t n = 0;
  double p = exp_neg_lambda;
  double F = p;
  while (u > F && n < 200) {
    n++;
    p = NG_DDIV(NG_DMUL(p, lambda), (double)n);
    F = NG_DADD(F, p);
  }
  return n;
}

// PTRS for lambda >= NGPU_POISSON_INV_MAX (Hoermann 1993, algorithm PTRS).
NG_HD uint32_t ng_poisson_ptrs(double lambda, uint64_t seed, uint32_t tag,
                               uint64_t stream, int64_t step) {
  double slam = sqrt(lambda);
  double loglam = log(lambda);
  double b = 0.931 + 2.53 * slam;
  double a = -0.059 + 0.02483 * b;
  double invalpha = 1.1239 + 1.1328 / (b - 3.4);
  double vr = 0.9277 - 3.6224 / (b - 2.0);
  for (uint32_t draw = 0; draw < 256; draw++) {
    Philox4 r = ng_random_block(seed, tag, stream, step, draw);
    double U = ng_u01(r.v[0], r.v[1]) - 0.5;
    double V = ng_u01(r.v[2], r.v[3]);
    double us = 0.5 - fabs(U);
    double k = floor((2.0 * a / us + b) * U + lambda + 0.43);
    if (us >= 0.07 && V <= vr) return (uint32_t)k;
    if (k < 0.0 || (us < 0.013 && V > us)) continue;
    if (log(V) + log(invalpha) - log(a / (us * us) + b)
        <= -lambda + k * loglam - lgamma(k + 1.0)) {
      return (uint32_t)k;
    }
  }
  return (uint32_t)floor(lambda + 0.5);
}

// Poisson count for one (stream, step).
NG_HD uint32_t ng_poisson(double lambda, double exp_neg_lambda, uint64_t seed,
                          uint32_t tag, uint64_t stream, int64_t step) {
  if (!(lambda > 0.0)) return 0;
  if (lambda < NGPU_POISSON_INV_MAX) {
    Philox4 r = ng_random_block(seed, tag, stream, step, 0);
    return ng_poisson_inversion(lambda, exp_neg_lambda, ng_u01(r.v[0], r.v[1]));
  }
  return ng_poisson_ptrs(lambda, seed, tag, stream, step);
}

// Poisson CDF table entries per generator (inversion thresholds)
#define NGPU_CDF_LEN 201

// Inversion thresholds of the direct-connection sampler: thr[k] = F(k) 2^32
// rounded to the nearest integer and saturated at 2^32 - 1, where F(k) is
// the Poisson CDF formed by the recurrence of ng_poisson_inversion (same
// double operations on every host). A count for a 32-bit uniform u is the
// number of leading thresholds with u >= thr[k], so P(count > k) =
// 1 - thr[k] / 2^32, the CDF to 2^-32. Integer compares make the device
// search cheap and identical on the host.
NG_HD void ng_poisson_thresholds(double lambda, double exp_neg_lambda, uint32_t *thr) {
  double p = exp_neg_lambda;
  double F = p;
  for (int n = 0; n < NGPU_CDF_LEN; n++) {
    if (n > 0) {
      p = NG_DDIV(NG_DMUL(p, lambda), (double)n);
      F = NG_DADD(F, p);
    }
    const double v = floor(NG_DADD(NG_DMUL(F, 4294967296.0), 0.5));
    thr[n] = v >= 4294967295.0 ? 0xFFFFFFFFu : (uint32_t)v;
  }
}

// Count of the direct-connection sampler for lambda < NGPU_POISSON_INV_MAX:
// u is word 0 of the Philox block of (seed, POISSON_DIRECT, stream, step).
NG_HD uint32_t ng_poisson_count_thr(uint32_t u, const uint32_t *thr) {
  uint32_t n = 0;
  while (n < NGPU_CDF_LEN - 1 && u >= thr[n]) n++;
  return n;
}

// Direct-connection Poisson count for one (stream, step): inversion against
// the thresholds below NGPU_POISSON_INV_MAX, PTRS above.
NG_HD uint32_t ng_poisson_direct(double lambda, const uint32_t *thr, uint64_t seed,
                                 uint64_t stream, int64_t step) {
  if (!(lambda > 0.0)) return 0;
  if (lambda < NGPU_POISSON_INV_MAX) {
    Philox4 r = ng_random_block(seed, RNG_TAG_POISSON_DIRECT, stream, step, 0);
    return ng_poisson_count_thr(r.v[0], thr);
  }
  return ng_poisson_ptrs(lambda, seed, RNG_TAG_POISSON_DIRECT, stream, step);
}

// fixed-point accumulation of synaptic input: 32 fractional bits
#define NGPU_ACC_SCALE 4294967296.0
#define NGPU_ACC_INV_SCALE (1.0 / 4294967296.0)

NG_HD long long ng_to_fixed(float v) {
#if defined(__CUDA_ARCH__)
  return __double2ll_rn((double)v * NGPU_ACC_SCALE);
#else
  return llrint((double)v * NGPU_ACC_SCALE);
#endif
}

}  // namespace ngpu
