// Device-side building blocks shared by the kernel translation units:
// spike push, input folding, the RK5 (Cash-Karp) step and the per-neuron RK5
// update with its single-group and batched (segment-table) kernels.
// Included by ngpu_kernels.cu and ngpu_rk5_batch.cu only.
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include "ngpu_device.h"
#include "ngpu_kernels.h"
#include "ngpu_models.h"
#include "ngpu_rk5_models.cuh"
#include "ngpu_rng.h"
#include "ngpu_f32x2.cuh"
#include "ngpu_step_proposer.cuh"
#include <cooperative_groups.h>

namespace ngpu {

namespace cg = cooperative_groups;

#define NGPU_BLOCK 128

// Programmatic dependent launch (sm_90+): the RK5 update and its finishing
// launch are issued with programmatic stream serialization, so the next
// kernel's blocks may be scheduled before this one has finished. pdl_wait()
// blocks until the preceding kernel has completed and its memory is
// visible (a no-op for a kernel launched without the attribute); each block
// calls pdl_trigger() once it has started, so the dependent kernel's blocks
// can take the slots that this grid's last wave frees and wait there.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

inline bool PdlEnabled() {
  static int on = -1;
  if (on < 0) {
    const char *e = getenv("NGB200_PDL");
    on = (e != nullptr && atoi(e) == 0) ? 0 : 1;
  }
  return on == 1;
}

// k<<<grid, block, 0, s>>>(args...) with programmatic stream serialization
template <typename... KArgs, typename... Args>
inline void launch_pdl(void (*k)(KArgs...), dim3 grid, dim3 block, cudaStream_t s,
                       Args... args) {
  if (!PdlEnabled()) {
    k<<<grid, block, 0, s>>>(args...);
    return;
  }
  cudaLaunchConfig_t cfg;
  memset(&cfg, 0, sizeof(cfg));
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  memset(at, 0, sizeof(at));
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, k, args...);
}

__device__ __forceinline__ bool pbit(const unsigned *mask, int j) {
  return (mask[j >> 5] >> (j & 31)) & 1u;
}

// ---------------------------------------------------------------------------
// spikes
// ---------------------------------------------------------------------------
__device__ __forceinline__ void push_spike(const PushArgs &pa, StepCtx *ctx,
                                           int node, int local, float height,
                                           long long T, double t_now,
                                           int den_delay_steps) {
  // the ring slot of step T, the step of ctx (every caller pushes the
  // spikes of its context's step)
  const int slot = ctx->ring_slot;
  int pos = atomicAdd(&pa.ring_cnt[slot], 1);
  if (pos < pa.ring_C) {
    long long k = (long long)slot * pa.ring_C + pos;
    pa.ring_src[k] = (unsigned)node;
    pa.ring_h[k] = height;
  } else {
    atomicOr(&ctx->err, (unsigned)DERR_RING_OVERFLOW);
  }
  pa.last_spike_T[node] = (int)T;
  pa.last_spike_h[node] = height;
  // the spike reaches the node's own dendrites (STDP post rule) at once or
  // den_delay_steps later (src/spike_buffer.cu:164-167, 265-300)
  if (den_delay_steps == 0) {
    pa.last_rev_T[node] = (int)T;
  } else if (pa.rev_cnt != nullptr) {
    if (den_delay_steps < pa.rev_R) {
      const int rs = (int)((T + den_delay_steps) % pa.rev_R);
      const int rp = atomicAdd(&pa.rev_cnt[rs], 1);
      if (rp < pa.rev_C) pa.rev_src[(long long)rs * pa.rev_C + rp] = (unsigned)node;
      else atomicOr(&ctx->err, (unsigned)DERR_REV_OVERFLOW);
    } else {
      atomicOr(&ctx->err, (unsigned)DERR_REV_OVERFLOW);
    }
  }
  if (pa.spike_count != nullptr) pa.spike_count[local]++;
  if (pa.rec_times != nullptr) {
    int n = pa.n_rec[local];
    // one slot is kept unused, as in src/spike_buffer.cu:183-186
    if (n < pa.max_rec - 1) {
      pa.rec_times[(long long)local * pa.max_rec + n] = (float)t_now;
      pa.n_rec[local] = n + 1;
    }
  }
}

// This group's accumulators that the update of step T0 + it + 1 folds: the
// slot written by the delivery of step T0 + it (StepCtx::acc_in_slot).
__device__ __forceinline__ long long *acc_in(const InputArgs &in, int slot) {
  return in.acc + acc_slot_offset(slot, in.acc_slots, in.acc_par) + in.acc_base;
}

// whether that slot may hold input: no stamps, or stamped by a delivery of
// step T0 + it (one load that every thread of the block shares)
__device__ __forceinline__ bool acc_live(const InputArgs &in, int slot, long long T0,
                                         long long it) {
  if (in.acc_stamp == nullptr) return true;
  return __ldcg(in.acc_stamp + (in.acc_slots > 1 ? slot : 0)) == T0 + it;
}

// Poisson count of one direct connection for the step T_prev (the
// reference's draw for that step); t_rel is the step's time relative to the
// generator's origin and the connection's delay, and the count is 0 outside
// the generator's active window. SMALL / LARGE: whether rates below / at or above
// NGPU_POISSON_INV_MAX per step are drawn; a count that is not drawn is 0.
// Small rates: the 32-bit uniform against the generator's inversion
// thresholds (ng_poisson_count_thr): the thresholds do not decrease, so
// the count below 8 is the number of the first 8 thresholds at or under u
// (8 independent integer compares; t8 holds them, in the kernel parameters
// for a uniform drive), and the search goes on in the table only in the
// rare case that all 8 are.
template <bool SMALL, bool LARGE>
__device__ __forceinline__ unsigned direct_count(double t_rel, float start, float stop,
                                                 double lam, const unsigned *thr,
                                                 const unsigned *t8,
                                                 unsigned long long seed,
                                                 unsigned long long stream, long long T_prev) {
  if (!(t_rel >= (double)start && t_rel <= (double)stop)) return 0;
  unsigned n = 0;
  if (lam < NGPU_POISSON_INV_MAX) {
    if constexpr (SMALL) {
      if (lam > 0.0) {
        const unsigned u = ng_random_block(seed, RNG_TAG_POISSON_DIRECT, stream, T_prev, 0).v[0];
#pragma unroll
        for (int k = 0; k < 8; k++) n += (u >= t8[k]) ? 1u : 0u;
        if (n == 8) {
          while (n < NGPU_CDF_LEN - 1 && u >= thr[n]) n++;
        }
      }
    }
  } else {
    if constexpr (LARGE) n = ng_poisson_ptrs(lam, seed, RNG_TAG_POISSON_DIRECT, stream, T_prev);
  }
  return n;
}

// Sum of the pending synaptic input of one node per port (fixed point):
// accumulator contents (cleared here) plus the Poisson direct connections
// drawn for the previous step. pre_acc: the accumulator values already
// fetched (port q at pre_acc[q]), or null. LARGE = false leaves out the
// connections of NGPU_POISSON_INV_MAX or more expected spikes per step:
// the update kernels of RK5 neurons, simple-model neurons and parrots use it,
// and k_poisson_large adds those draws into the accumulators before them
// (the large-rate sampler needs many registers, and inlined it raised the
// update kernels' register count and spills).
template <int NP, bool LARGE = true>
__device__ __forceinline__ void input_sum(const InputArgs &in, int i,
                                          int n_pad, int np, long long it,
                                          double t0, float dt, int pending,
                                          long long T0, int acc_slot, long long *s,
                                          bool dry = false,
                                          const long long *pre_acc = nullptr) {
  const bool live = pre_acc != nullptr || acc_live(in, acc_slot, T0, it);
#pragma unroll
  for (int q = 0; q < NP; q++) {
    s[q] = 0;
    if (q < np && live) {
      long long *a = acc_in(in, acc_slot) + (long long)q * n_pad + i;
      long long v = pre_acc ? pre_acc[q] : *a;
      if (v != 0 && !(in.dry || dry)) *a = 0;
      s[q] = v;
    }
  }
  if (pending && in.ud) {
    const double t = t0 + (double)dt * (double)it;
    const double t_rel = t - (double)in.ud_origin - (double)in.ud_delay;
    const unsigned n = direct_count<true, LARGE>(
        t_rel, in.ud_start, in.ud_stop, in.ud_lambda, in.ud_thr, in.ud_thr8, in.seed,
        in.ud_stream0 + (unsigned long long)i, T0 + it);
    if (n > 0) {
      const long long v = ng_to_fixed(in.ud_w * (float)n);
#pragma unroll
      for (int q = 0; q < NP; q++) {
        if (q == in.ud_port) s[q] += v;
      }
    }
  } else if (pending && in.dc_off != nullptr) {
    unsigned b = in.dc_off[i], e = in.dc_off[i + 1];
    if (b < e) {
      // time of the step whose draws are pending (neural_time_ of that step)
      double t = t0 + (double)dt * (double)it;
      long long T_prev = T0 + it;
      for (unsigned c = b; c < e; c++) {
        unsigned gen = in.dc_gen[c];
        double t_rel = t - (double)in.gen_origin[gen] - (double)in.dc_delay[c];
        const unsigned *thr = in.gen_thr + (size_t)gen * NGPU_CDF_LEN;
        const unsigned n = direct_count<true, LARGE>(
            t_rel, in.gen_start[gen], in.gen_stop[gen], in.gen_lambda[gen], thr, thr, in.seed,
            in.dc_stream[c], T_prev);
        if (n > 0) {
          long long v = ng_to_fixed(in.dc_weight[c] * (float)n);
          int port = in.dc_port[c];
#pragma unroll
          for (int q = 0; q < NP; q++) {
            if (q == port) s[q] += v;
          }
        }
      }
    }
  }
}

__device__ __forceinline__ float fold_value(float var, long long s, float w) {
  return (float)((double)var + (double)s * NGPU_ACC_INV_SCALE * (double)w);
}

// ---------------------------------------------------------------------------
// RK5 (Cash-Karp) step and update, following src/rk5.h:57-162
// ---------------------------------------------------------------------------
// err^e for err > 0 with e = -0.2 or -0.25 (step-size controller): the
// special-function unit's base-2 logarithm and power
__device__ __forceinline__ float ctrl_pow(float err, float e) {
  return ex2_approx(e * lg2_approx(err));
}

// Cash-Karp coefficients as pairs (c, c): one operand of the packed stage
// arithmetic, read from the constant bank.
struct Rk5PairConsts {
  float2 a21, a31, a32, a41, a42, a43, a51, a52, a53, a54, a61, a62, a63, a64, a65;
  float2 a71, a73, a74, a76, e1, e3, e4, e5, e6;
};
#define NGPU_PAIR(c) {rk5c::c, rk5c::c}
static __constant__ Rk5PairConsts c_rk5[1] = {{
    NGPU_PAIR(a21), NGPU_PAIR(a31), NGPU_PAIR(a32), NGPU_PAIR(a41), NGPU_PAIR(a42),
    NGPU_PAIR(a43), NGPU_PAIR(a51), NGPU_PAIR(a52), NGPU_PAIR(a53), NGPU_PAIR(a54),
    NGPU_PAIR(a61), NGPU_PAIR(a62), NGPU_PAIR(a63), NGPU_PAIR(a64), NGPU_PAIR(a65),
    NGPU_PAIR(a71), NGPU_PAIR(a73), NGPU_PAIR(a74), NGPU_PAIR(a76), NGPU_PAIR(e1),
    NGPU_PAIR(e3), NGPU_PAIR(e4), NGPU_PAIR(e5), NGPU_PAIR(e6)}};
#undef NGPU_PAIR
#define NGPU_C2(name) (c_rk5[cz].name)

// error scale |y| + |h k1| + scal_min of one pair of variables
__device__ __forceinline__ void rk5_err_scale(f2 y, f2 k1, float h, float &s0, float &s1) {
  float y0, y1, k0, k1s;
  f2_unpack(y, y0, y1);
  f2_unpack(k1, k0, k1s);
  s0 = fabsf(y0) + fabsf(k0 * h) + rk5c::scal_min;
  s1 = fabsf(y1) + fabsf(k1s * h) + rk5c::scal_min;
}

// One RK5 step (src/rk5.h:57-147): Cash-Karp stages, error estimate and
// step-size control, retried with a smaller step until accepted. The state
// variables are processed as pairs (y[2j], y[2j+1]) with packed FP32x2
// arithmetic, which rounds every half as the scalar operation would; an odd
// variable count is padded with a zero variable. Kept from the reference:
// the error scale |y| + |h k1| + 0.1 with the step size before clamping, the
// clamp to [h_min, h_max], the escape at h <= h_min (1 + 1e-5) (h_min_thr:
// the largest float at or below that double), the reduction to at least
// 0.1 h (in double) and the growth rules. The scaled errors |e_i| / ys_i
// are products with the reciprocal of ys_i; when their maximum, times
// 1 / eps, lies within 1e-5 of 1 the norm is recomputed in FP64 (IEEE
// quotients) so that the accept / reject decision is the exact one.
template <class M, int NP>
__device__ __forceinline__ void rk5_step(double &x, float *y, float &h,
                                         float h_min, float h_min_thr, float h_max,
                                         const float *p, const float *q,
                                         float refr, int np, float inv_eps,
                                         unsigned &evals, float &h_acc, float &err_acc) {
  using namespace rk5c;
  constexpr int NV = M::NVAR;
  constexpr int NH = (NV + 1) / 2;
  constexpr int NVP = 2 * NH;
  // K1: the derivative at the start (kept across retries); K2..K4 while
  // stages need them; S6 / P5 / PE: running sums of the sixth stage's
  // input, the fifth-order solution and the error estimate, formed in the
  // reference's order of terms as soon as their terms exist, so that K2..K5
  // are not live at the same time
  f2 Y[NH], K1[NH], K2[NH], K3[NH], K4[NH], YN[NH];
  float d[NVP], yn[NVP];
#pragma unroll
  for (int j = 0; j < NVP; j++) d[j] = 0.0f;
#pragma unroll
  for (int j = 0; j < NH; j++) Y[j] = f2_pack(y[2 * j], (2 * j + 1 < NV) ? y[2 * j + 1] : 0.0f);
  M::deriv(y, d, p, q, refr, np);
  evals++;
#pragma unroll
  for (int j = 0; j < NH; j++) K1[j] = f2_pack(d[2 * j], d[2 * j + 1]);
  // the error scale |y| + |h k1| + scal_min uses the step size the call
  // starts with; it is formed where the error is (fewer live registers)
  const float h_in = h;
  float err = 0.0f;
  for (int guard = 0;; guard++) {
    // an index the compiler cannot see is 0: the coefficient pairs are read
    // from the constant bank in every attempt instead of being hoisted out
    // of the retry loop into registers (24 pairs = 48 registers)
    int cz;
    asm volatile("mov.u32 %0, 0;" : "=r"(cz));
    h = fmaxf(fminf(h, h_max), h_min);
    const f2 HH = f2_pack(h, h);
    // stage 2
    const f2 HA21 = f2_mul(HH, NGPU_C2(a21));
#pragma unroll
    for (int j = 0; j < NH; j++) {
      YN[j] = f2_fma(HA21, K1[j], Y[j]);
      f2_unpack(YN[j], yn[2 * j], yn[2 * j + 1]);
    }
    M::deriv(yn, d, p, q, refr, np);
#pragma unroll
    for (int j = 0; j < NH; j++) K2[j] = f2_pack(d[2 * j], d[2 * j + 1]);
    // stage 3
#pragma unroll
    for (int j = 0; j < NH; j++) {
      f2 t = f2_mul(NGPU_C2(a31), K1[j]);
      t = f2_fma(NGPU_C2(a32), K2[j], t);
      YN[j] = f2_fma(HH, t, Y[j]);
      f2_unpack(YN[j], yn[2 * j], yn[2 * j + 1]);
    }
    M::deriv(yn, d, p, q, refr, np);
#pragma unroll
    for (int j = 0; j < NH; j++) K3[j] = f2_pack(d[2 * j], d[2 * j + 1]);
    // stage 4
#pragma unroll
    for (int j = 0; j < NH; j++) {
      f2 t = f2_mul(NGPU_C2(a41), K1[j]);
      t = f2_fma(NGPU_C2(a42), K2[j], t);
      t = f2_fma(NGPU_C2(a43), K3[j], t);
      YN[j] = f2_fma(HH, t, Y[j]);
      f2_unpack(YN[j], yn[2 * j], yn[2 * j + 1]);
    }
    M::deriv(yn, d, p, q, refr, np);
#pragma unroll
    for (int j = 0; j < NH; j++) K4[j] = f2_pack(d[2 * j], d[2 * j + 1]);
    // stage 5 input; the terms of K2..K4 in the later sums
    f2 S6[NH], P5[NH], PE[NH];
#pragma unroll
    for (int j = 0; j < NH; j++) {
      f2 t = f2_mul(NGPU_C2(a51), K1[j]);
      t = f2_fma(NGPU_C2(a52), K2[j], t);
      t = f2_fma(NGPU_C2(a53), K3[j], t);
      t = f2_fma(NGPU_C2(a54), K4[j], t);
      YN[j] = f2_fma(HH, t, Y[j]);
      f2_unpack(YN[j], yn[2 * j], yn[2 * j + 1]);
      f2 u = f2_mul(NGPU_C2(a61), K1[j]);
      u = f2_fma(NGPU_C2(a62), K2[j], u);
      u = f2_fma(NGPU_C2(a63), K3[j], u);
      S6[j] = f2_fma(NGPU_C2(a64), K4[j], u);
      f2 v = f2_mul(NGPU_C2(a71), K1[j]);
      v = f2_fma(NGPU_C2(a73), K3[j], v);
      P5[j] = f2_fma(NGPU_C2(a74), K4[j], v);
      f2 e = f2_mul(NGPU_C2(e1), K1[j]);
      e = f2_fma(NGPU_C2(e3), K3[j], e);
      PE[j] = f2_fma(NGPU_C2(e4), K4[j], e);
    }
    M::deriv(yn, d, p, q, refr, np);
    // stage 6 input (K5 = d)
#pragma unroll
    for (int j = 0; j < NH; j++) {
      const f2 k5 = f2_pack(d[2 * j], d[2 * j + 1]);
      YN[j] = f2_fma(HH, f2_fma(NGPU_C2(a65), k5, S6[j]), Y[j]);
      f2_unpack(YN[j], yn[2 * j], yn[2 * j + 1]);
      PE[j] = f2_fma(NGPU_C2(e5), k5, PE[j]);
    }
    M::deriv(yn, d, p, q, refr, np);
    evals += 5;
    // fifth-order solution and the scaled error of the embedded estimate (K6 = d)
    err = 0.0f;
#pragma unroll
    for (int j = 0; j < NH; j++) {
      const f2 k6 = f2_pack(d[2 * j], d[2 * j + 1]);
      YN[j] = f2_fma(HH, f2_fma(NGPU_C2(a76), k6, P5[j]), Y[j]);
      PE[j] = f2_mul(HH, f2_fma(NGPU_C2(e6), k6, PE[j]));
      float v0, v1, s0, s1;
      f2_unpack(PE[j], v0, v1);
      rk5_err_scale(Y[j], K1[j], h_in, s0, s1);
      err = fmaxf(err, fmaxf(fabsf(v0) * rcp_approx(s0), fabsf(v1) * rcp_approx(s1)));
    }
    err *= inv_eps;
    bool accept = err <= 1.0f;
    if (fabsf(err - 1.0f) < 1.0e-5f) {
      // borderline: the norm in FP64 with IEEE quotients decides
      double e64 = 0.0;
#pragma unroll
      for (int j = 0; j < NH; j++) {
        float v0, v1, s0, s1;
        f2_unpack(PE[j], v0, v1);
        rk5_err_scale(Y[j], K1[j], h_in, s0, s1);
        e64 = fmax(e64, fabs((double)v0 / (double)s0));
        e64 = fmax(e64, fabs((double)v1 / (double)s1));
      }
      accept = e64 * (double)inv_eps <= 1.0;
    }
    if (accept || h <= h_min_thr) break;
    if (guard >= 256) break;
    const float h_new = h * coeff * ctrl_pow(err, exp_dec);
    const double h01 = 0.1 * (double)h;
    h = (float)(((double)h_new > h01) ? (double)h_new : h01);
  }
  x += h;
  h_acc = h;
  err_acc = err;
  if (err > err_min) {
    h = h * coeff * ctrl_pow(err, exp_inc);
  } else {
    h = (float)(5.0 * (double)h);
  }
#pragma unroll
  for (int j = 0; j < NH; j++) {
    float a, b;
    f2_unpack(YN[j], a, b);
    y[2 * j] = a;
    if (2 * j + 1 < NV) y[2 * j + 1] = b;
  }
}
#undef NGPU_C2

template <class M>
struct ModelTraits;

// input var / weight mapping and the param column of den_delay and
// refractory_step for every RK5 model
#define NGPU_TRAITS(MODEL, IN_BASE, IN_STEP, W_BASE, W_STEP, REFR, DEN)   \
  template <int NP>                                                       \
  struct ModelTraits<MODEL<NP>> {                                         \
    enum { in_base = IN_BASE, in_step = IN_STEP, w_base = W_BASE,         \
           w_step = W_STEP, refr = REFR, den = DEN };                     \
  };
NGPU_TRAITS(AeifCondBeta, 3, 2, A_NSP + 3, 4, A_refr, A_den_delay)
NGPU_TRAITS(AeifCondAlpha, 3, 2, A_NSP + 2, 3, A_refr, A_den_delay)
NGPU_TRAITS(AeifPscAlpha, 3, 2, A_NSP + 1, 2, A_refr, A_den_delay)
NGPU_TRAITS(AeifPscExp, 2, 1, -1, 0, A_refr, A_den_delay)
NGPU_TRAITS(AeifPscDelta, 0, 0, -1, 0, A_refr, A_den_delay)
NGPU_TRAITS(IzhCondBeta, 3, 2, I_NSP + 3, 4, I_refr, I_den_delay)

__device__ __forceinline__ void block_add_u64(unsigned long long v,
                                              unsigned long long *dst, int blk = -1) {
  // per warp: a shuffle sum, then one reduction into the block's counter
  // whose result is not waited for (red.global.add), so a finished block
  // frees its SM slot at once (a barrier and a load-add-store of the
  // counter by one thread held every block for an L2 round trip)
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0 && v != 0) atomicAdd(dst + (blk >= 0 ? blk : (int)blockIdx.x), v);
}

// Appends one accepted sub-step (features at its start, training target) to
// the group's step log; one atomic per warp.
__device__ __forceinline__ void log_step_sample(const GroupArgs &g, const float *f,
                                                float target) {
  const unsigned mask = __activemask();
  const int lane = threadIdx.x & 31;
  const int leader = __ffs(mask) - 1;
  const unsigned rank = __popc(mask & ((1u << lane) - 1u));
  unsigned base = 0;
  if (lane == leader) base = atomicAdd(g.log_count, (unsigned)__popc(mask));
  base = __shfl_sync(mask, base, leader);
  const unsigned idx = base + rank;
  if (idx < (unsigned)g.log_cap) {
    float4 *dst = reinterpret_cast<float4 *>(g.log_buf + (size_t)idx * 8);
    dst[0] = make_float4(f[0], f[1], f[2], f[3]);
    dst[1] = make_float4(f[4], f[5], target, 0.0f);
  }
}

// Parameters of neuron i when they are not all group-uniform: the per-neuron
// columns named in pmask, the uniform value otherwise, and the reciprocals
// formed in registers.
template <class M, bool UNI>
__device__ __forceinline__ void rk5_load_params(const GroupArgs &g, int i, bool active,
                                                float *p_loc, float *q_loc) {
  if (!UNI) {
#pragma unroll
    for (int j = 0; j < (UNI ? 1 : M::NPARAM); j++) {
      if (j < g.nparam) {
        p_loc[j] = (active && pbit(g.pmask, j)) ? g.param[(long long)j * g.n_pad + i] : g.puni[j];
      } else {
        p_loc[j] = 1.0f;
      }
      q_loc[j] = 1.0f / p_loc[j];
    }
  }
}

// One sub-step of the plain controller (src/rk5.h:57-162) followed by the
// model's spike test; true once the time step is complete.
template <class M, int NP>
__device__ __forceinline__ bool rk5_plain_substep(const GroupArgs &g, const PushArgs &pa,
                                                  StepCtx *ctx, int i, float *y, double &x,
                                                  float &h, float &refr, int &guard,
                                                  const float *p, const float *q, int np,
                                                  float inv_eps, double x1, long long T,
                                                  int den, bool dry, unsigned &evals) {
  float h_acc, err_acc;
  const float hmax = (float)(x1 - x);
  rk5_step<M, NP>(x, y, h, g.h_min, g.h_min_thr, hmax, p, q, refr, np, inv_eps, evals, h_acc,
                  err_acc);
  bool end_step = (x >= x1 - (double)g.h_min);
  if (M::external(y, p, refr, end_step, g.dt)) {
    if (!dry) push_spike(pa, ctx, g.i_node_0 + i, i, 1.0f, T, x1, den);
  }
  if (++guard > g.max_substeps) {
    atomicOr(&ctx->err, (unsigned)DERR_RK5_STUCK);
    end_step = true;
  }
  return end_step;
}

// end-of-step state of neuron i
template <class M, int NP>
__device__ __forceinline__ void rk5_store(const GroupArgs &g, int i, const float *y, float h,
                                          double x, double x1, float refr, bool write_refr) {
  using Tr = ModelTraits<M>;
#pragma unroll
  for (int j = 0; j < M::NVAR; j++) {
    // (every variable column exists for 2-4 ports, see rk5_neuron)
    if ((NP >= 2 && NP <= 4) || j < g.nvar) g.var[(long long)j * g.n_pad + i] = y[j];
  }
  g.h[i] = h;
  g.dx[i] = (float)(x - x1);
  if (write_refr) g.param[(long long)Tr::refr * g.n_pad + i] = refr;
}

// Hands neuron i (segment seg of a batched launch, 128-neuron tile tile)
// over to the straggler queue; false if the queue has no room (the caller
// then carries on). One reservation per group of converged threads (a warp
// lies within one tile, so the group shares the sub-queue).
template <int NV>
__device__ __forceinline__ bool rk5_enqueue(const Rk5Queue &qu, int seg, int tile, int i,
                                            const float *y, double x, float h, float refr,
                                            int guard) {
  if (8 + NV > qu.stride) return false;
  const int lane_q = tile & (NGPU_QLANES - 1);
  cg::coalesced_group grp = cg::coalesced_threads();
  unsigned base = 0;
  if (grp.thread_rank() == 0) base = atomicAdd(&qu.hdr->lane[lane_q].tail, grp.size());
  base = grp.shfl(base, 0);
  const unsigned k = base + grp.thread_rank();
  if (k >= (unsigned)qu.sub_cap) return false;
  float *r = qu.rec + ((size_t)lane_q * qu.sub_cap + k) * qu.stride;
  r[0] = __int_as_float(i);
  r[1] = __int_as_float(seg);
  r[2] = __int_as_float(guard);
  r[3] = h;
  r[4] = refr;
  *reinterpret_cast<double *>(r + 6) = x;
#pragma unroll
  for (int j = 0; j < NV; j++) r[8 + j] = y[j];
  return true;
}

// Finishes a straggler record: the rest of the time step of its neuron with
// the same sub-step sequence as the uninterrupted loop.
template <class M, int NP, bool UNI>
__device__ __forceinline__ void rk5_resume(const GroupArgs &g, const PushArgs &pa, StepCtx *ctx,
                                           const float *p_uni, const float *q_uni, int np,
                                           const float *r, unsigned &evals, bool dry) {
  using Tr = ModelTraits<M>;
  if constexpr (NP >= 2 && NP <= 4) np = NP;   // as in rk5_neuron
  const int i = __float_as_int(r[0]);
  int guard = __float_as_int(r[2]);
  float h = r[3];
  float refr = r[4];
  double x = *reinterpret_cast<const double *>(r + 6);
  float y[M::NVAR];
#pragma unroll
  for (int j = 0; j < M::NVAR; j++) y[j] = r[8 + j];
  float p_loc[UNI ? 1 : M::NPARAM];
  float q_loc[UNI ? 1 : M::NPARAM];
  rk5_load_params<M, UNI>(g, i, true, p_loc, q_loc);
  const float *p = UNI ? p_uni : p_loc;
  const float *q = UNI ? q_uni : q_loc;
  const long long it = ctx->it;
  const double x1 = ctx->t0 + (double)g.dt * (double)(it + 1);
  const long long T = ctx->T0 + it + 1;
  const float inv_eps = g.inv_eps;
  // group-wide dendritic delay: the steps formed on the host
  const int den = (UNI && g.den_delay_col == Tr::den) ? g.den_steps
                                                       : (int)roundf(p[Tr::den] / g.dt);
  bool end_step = false;
  while (!end_step) {
    end_step = rk5_plain_substep<M, NP>(g, pa, ctx, i, y, x, h, refr, guard, p, q, np, inv_eps,
                                        x1, T, den, dry, evals);
  }
  if (!dry) {
    rk5_store<M, NP>(g, i, y, h, x, x1, refr, true);
  } else if (y[0] == 1.2345e30f) {
    g.h[i] = h + (float)x;        // keeps the timing run from being optimised away
  }
}

// Records of the queue's last update launch: per-sub-queue counts and their
// prefix in s_pref[0..NGPU_QLANES]; returns the total. Whole blocks call it.
__device__ __forceinline__ unsigned rk5_queue_prefix(const Rk5Queue &qu, unsigned *s_pref) {
  if (threadIdx.x < NGPU_QLANES) {
    unsigned c = qu.hdr->lane[threadIdx.x].tail;
    c = c < (unsigned)qu.sub_cap ? c : (unsigned)qu.sub_cap;
    unsigned incl = c;
#pragma unroll
    for (int o = 1; o < NGPU_QLANES; o <<= 1) {
      const unsigned v = __shfl_up_sync(0xffffffffu, incl, o);
      if ((int)threadIdx.x >= o) incl += v;
    }
    s_pref[threadIdx.x + 1] = incl;
    if (threadIdx.x == 0) s_pref[0] = 0;
  }
  __syncthreads();
  return s_pref[NGPU_QLANES];
}

// record number t (< the total) in sub-queue order
__device__ __forceinline__ const float *rk5_queue_record(const Rk5Queue &qu,
                                                         const unsigned *s_pref, unsigned t) {
  int lo = 0, hi = NGPU_QLANES;       // the sub-queue with s_pref[lo] <= t < s_pref[lo + 1]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (s_pref[mid] <= t) lo = mid; else hi = mid;
  }
  return qu.rec + ((size_t)lo * qu.sub_cap + (t - s_pref[lo])) * qu.stride;
}

// The last block of a finishing launch empties the queue for the next
// update; every block has read the record count by then.
__device__ __forceinline__ void rk5_queue_reset(const Rk5Queue &qu) {
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned prev = atomicAdd(&qu.hdr->done, 1u);
    if (prev == gridDim.x - 1) {
      for (int j = 0; j < NGPU_QLANES; j++) qu.hdr->lane[j].tail = 0u;
      qu.hdr->done = 0u;
    }
  }
}

// Integrates neuron i of group g over one time step (one thread per
// neuron). UNI: every parameter except the refractory counter is
// group-uniform and is read from p_uni / q_uni (reciprocals); otherwise the
// parameters are loaded per neuron and q is formed in registers.
// MODE STEP_PLAIN: the reference's controller; STEP_LOG: the same, and every
// sub-step that starts with a controller guess shorter than the rest of the
// time step is logged for training the proposer. (The learned proposer runs
// in the straggler queue's finishing launch, k_rk5_finish_learned, after a
// STEP_PLAIN update with the queue on.)
// With a straggler queue (STEP_PLAIN), a neuron still inside the step after
// its first sub-step is handed over to the queue (segment seg). pre_col /
// pre_acc: the neuron's state columns (M::NVAR state variables, refractory
// counter, step size, time offset) and accumulators already fetched, or null.
template <class M, int NP, bool UNI, int MODE>
__device__ __forceinline__ void rk5_neuron(const GroupArgs &g, const InputArgs &in,
                                           const PushArgs &pa, StepCtx *ctx, int i,
                                           const float *p_uni, const float *q_uni,
                                           unsigned &evals, bool dry_run,
                                           const Rk5Queue *qu = nullptr,
                                           int seg = 0, const float *pre_col = nullptr,
                                           const long long *pre_acc = nullptr, int tile = -1) {
  using Tr = ModelTraits<M>;
  const bool dry = g.dry || dry_run;
  // the launchers pick the template port count NP = np for 2..4 ports (1
  // serves 0 and 1), so there the count is a compile-time constant
  const int np = (NP >= 2 && NP <= 4) ? NP : in.np;
  const long long it = ctx->it;
  const long long T0 = ctx->T0;
  const double t0 = ctx->t0;
  const int pending = ctx->poisson_pending;
  const int n_pad = g.n_pad;
  // the pending input is summed before the state is loaded, so that the state
  // is not live across the Poisson draws (fewer registers and spills)
  constexpr int NPI = (M::NPV == 0) ? 1 : NP;
  long long s[NPI];
  input_sum<NPI, false>(in, i, n_pad, np, it, t0, g.dt, pending, T0, ctx->acc_in_slot, s, dry,
                          pre_acc);
  float y[M::NVAR];
#pragma unroll
  for (int j = 0; j < M::NVAR; j++) {
    y[j] = ((NP >= 2 && NP <= 4) || j < g.nvar)
               ? (pre_col ? pre_col[j] : g.var[(long long)j * n_pad + i])
                                  : 0.0f;
  }
  float p_loc[UNI ? 1 : M::NPARAM];
  float q_loc[UNI ? 1 : M::NPARAM];
  rk5_load_params<M, UNI>(g, i, true, p_loc, q_loc);
  const float *p = UNI ? p_uni : p_loc;
  const float *q = UNI ? q_uni : q_loc;
  float refr = pre_col ? pre_col[M::NVAR] : g.param[(long long)Tr::refr * n_pad + i];
  // fold the previous step's input
#pragma unroll
  for (int qq = 0; qq < NPI; qq++) {
    if (qq < np && s[qq] != 0) {
      const int vi = Tr::in_base + qq * Tr::in_step;
      const float w = (Tr::w_base >= 0) ? p[Tr::w_base + qq * Tr::w_step] : 1.0f;
      y[vi] = fold_value(y[vi], s[qq], w);
    }
  }
  const float refr0 = refr;
  const double x1 = t0 + (double)g.dt * (double)(it + 1);
  double x = t0 + (double)g.dt * (double)it +
             (double)(pre_col ? pre_col[M::NVAR + 2] : g.dx[i]);
  float h = pre_col ? pre_col[M::NVAR + 1] : g.h[i];
  const float h_min = g.h_min;
  const float inv_eps = g.inv_eps;
  const long long T = T0 + it + 1;
  // group-wide dendritic delay: the steps formed on the host
  const int den = (UNI && g.den_delay_col == Tr::den) ? g.den_steps
                                                       : (int)roundf(p[Tr::den] / g.dt);
  bool end_step = false;
  int guard = 0;
  float h_acc, err_acc;
  if constexpr (MODE == STEP_LOG) {
    while (!end_step) {
      const float hmax = (float)(x1 - x);
      float f[6];
      bool lg = false;
      if (h < hmax && !dry) {
        ProposerFeatures<M>::get(y, p, h, g.dt, f);
        lg = true;
      }
      rk5_step<M, NP>(x, y, h, h_min, g.h_min_thr, hmax, p, q, refr, np, inv_eps, evals, h_acc,
                      err_acc);
      if (lg) log_step_sample(g, f, proposer_target(h_acc, err_acc, g.dt));
      end_step = (x >= x1 - (double)h_min);
      if (M::external(y, p, refr, end_step, g.dt)) {
        if (!dry) push_spike(pa, ctx, g.i_node_0 + i, i, 1.0f, T, x1, den);
      }
      if (++guard > g.max_substeps) {
        atomicOr(&ctx->err, (unsigned)DERR_RK5_STUCK);
        break;
      }
    }
  } else {
    while (!end_step) {
      end_step = rk5_plain_substep<M, NP>(g, pa, ctx, i, y, x, h, refr, guard, p, q, np,
                                          inv_eps, x1, T, den, dry, evals);
      if (!end_step && guard == 1 && qu != nullptr) {
        if (rk5_enqueue<M::NVAR>(*qu, seg, tile >= 0 ? tile : (i >> 7), i, y, x, h, refr,
                                 guard))
          return;
      }
    }
  }
  if (!dry) {
    rk5_store<M, NP>(g, i, y, h, x, x1, refr, refr != refr0);
  } else if (y[0] == 1.2345e30f) {
    // keeps the dry run from being optimised away; never true in practice
    g.h[i] = h + (float)x;
  }
}

// One RK5 group per launch; its arguments live in the constant
// kernel-parameter block, so uniform parameters cost no loads.
template <class M, int NP, bool UNI, int MINB, int MODE>
__global__ void __launch_bounds__(NGPU_BLOCK, MINB)
k_rk5_update(const __grid_constant__ GroupArgs g, const __grid_constant__ InputArgs in,
             const __grid_constant__ PushArgs pa, StepCtx *ctx) {
  pdl_wait();
  pdl_trigger();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned evals = 0;
  const bool queued = (MODE == STEP_PLAIN) && g.q.cap > 0;
  if (i < g.n) rk5_neuron<M, NP, UNI, MODE>(g, in, pa, ctx, i, g.puni, g.pinv, evals, false,
                                            queued ? &g.q : nullptr, 0);
  if (g.blk_evals != nullptr) block_add_u64(evals, g.blk_evals);
}

// Integrates neuron i through the W consecutive steps of a window (plain
// controller), its state in registers from the first step to the last: each
// step reads its own step context (ctxs[k]), folds that step's pending input
// (its accumulator slot, filled before the window by earlier deliveries, and
// its Poisson draws) and integrates the step with rk5_neuron's sub-step
// sequence; the time offset is rounded to float between steps, as
// rk5_neuron stores it, so the result is the one-step path's, bit for bit.
// Spikes go to each step's ring slot. FREE: a lane whose step ended begins
// its next step while the others go on, so a warp takes as many sub-steps
// as its slowest lane over the window, not the sum over the steps of each
// step's slowest lane (busy networks: 6 % less time for the window update
// of the 1e6-neuron network at 26 Hz); without it the warp's lanes go
// through the steps together, the tighter loop where every neuron takes
// one sub-step per step. Both give the same results.
template <class M, int NP, bool UNI, bool FREE>
__device__ __forceinline__ void rk5_window_neuron(const GroupArgs &g, const InputArgs &in,
                                                  const PushArgs &pa, StepCtx *ctxs, int W,
                                                  int i, const float *p_uni,
                                                  const float *q_uni, unsigned &evals) {
  using Tr = ModelTraits<M>;
  const int np = (NP >= 2 && NP <= 4) ? NP : in.np;
  const int n_pad = g.n_pad;
  constexpr int NPI = (M::NPV == 0) ? 1 : NP;
  float y[M::NVAR];
#pragma unroll
  for (int j = 0; j < M::NVAR; j++)
    y[j] = ((NP >= 2 && NP <= 4) || j < g.nvar) ? g.var[(long long)j * n_pad + i] : 0.0f;
  float p_loc[UNI ? 1 : M::NPARAM];
  float q_loc[UNI ? 1 : M::NPARAM];
  rk5_load_params<M, UNI>(g, i, true, p_loc, q_loc);
  const float *p = UNI ? p_uni : p_loc;
  const float *q = UNI ? q_uni : q_loc;
  float refr = g.param[(long long)Tr::refr * n_pad + i];
  const float refr0 = refr;
  float h = g.h[i];
  float dxf = g.dx[i];
  const int den = (UNI && g.den_delay_col == Tr::den) ? g.den_steps
                                                       : (int)roundf(p[Tr::den] / g.dt);
  StepCtx *ctx = ctxs;
  double x1 = 0.0, x = 0.0;
  long long T = 0;
  int guard = 0, k = 0;
  auto begin_step = [&]() {
    ctx = ctxs + k;
    const long long it = ctx->it;
    const long long T0 = ctx->T0;
    const double t0 = ctx->t0;
    long long s[NPI];
    input_sum<NPI, false>(in, i, n_pad, np, it, t0, g.dt, ctx->poisson_pending, T0,
                          ctx->acc_in_slot, s);
#pragma unroll
    for (int qq = 0; qq < NPI; qq++) {
      if (qq < np && s[qq] != 0) {
        const int vi = Tr::in_base + qq * Tr::in_step;
        const float w = (Tr::w_base >= 0) ? p[Tr::w_base + qq * Tr::w_step] : 1.0f;
        y[vi] = fold_value(y[vi], s[qq], w);
      }
    }
    x1 = t0 + (double)g.dt * (double)(it + 1);
    x = t0 + (double)g.dt * (double)it + (double)dxf;
    T = T0 + it + 1;
    guard = 0;
  };
  if constexpr (FREE) {
    begin_step();
    while (true) {
      if (rk5_plain_substep<M, NP>(g, pa, ctx, i, y, x, h, refr, guard, p, q, np, g.inv_eps,
                                   x1, T, den, false, evals)) {
        dxf = (float)(x - x1);
        if (++k == W) break;
        begin_step();
      }
    }
  } else {
    for (k = 0; k < W; k++) {
      begin_step();
      bool end_step = false;
      while (!end_step) {
        end_step = rk5_plain_substep<M, NP>(g, pa, ctx, i, y, x, h, refr, guard, p, q, np,
                                            g.inv_eps, x1, T, den, false, evals);
      }
      dxf = (float)(x - x1);
    }
  }
#pragma unroll
  for (int j = 0; j < M::NVAR; j++) {
    if ((NP >= 2 && NP <= 4) || j < g.nvar) g.var[(long long)j * n_pad + i] = y[j];
  }
  g.h[i] = h;
  g.dx[i] = dxf;
  if (refr != refr0) g.param[(long long)Tr::refr * n_pad + i] = refr;
}

// One RK5 group through a window of W steps (several steps per launch);
// MINB: the register cap of the single-step variant the autotuner chose.
template <class M, int NP, bool UNI, int MINB, bool FREE = false>
__global__ void __launch_bounds__(NGPU_BLOCK, MINB)
k_rk5_window(const __grid_constant__ GroupArgs g, const __grid_constant__ InputArgs in,
             const __grid_constant__ PushArgs pa, StepCtx *ctxs, int W) {
  pdl_wait();
  pdl_trigger();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned evals = 0;
  if (i < g.n)
    rk5_window_neuron<M, NP, UNI, FREE>(g, in, pa, ctxs, W, i, g.puni, g.pinv, evals);
  if (g.blk_evals != nullptr) block_add_u64(evals, g.blk_evals);
}

// Many RK5 groups of one model through a window of W steps in one launch
// (the batched form of k_rk5_window): block b integrates its 128 neurons of
// segment blk_seg[b]; the segment's uniform parameters are staged in shared
// memory.
template <class M, int NP, bool UNI, int MINB>
__global__ void __launch_bounds__(NGPU_BLOCK, MINB)
k_rk5_window_seg(const SegArgs *__restrict__ segs, const int *__restrict__ blk_seg,
                 unsigned long long *blk_evals, StepCtx *ctxs, int W) {
  pdl_wait();
  pdl_trigger();
  __shared__ float s_p[M::NPARAM], s_q[M::NPARAM];
  const int seg = blk_seg[blockIdx.x];
  const SegArgs &S = segs[seg];
  if (UNI) {
    for (int j = threadIdx.x; j < M::NPARAM; j += blockDim.x) {
      s_p[j] = S.g.puni[j];
      s_q[j] = S.g.pinv[j];
    }
    __syncthreads();
  }
  const int i = (blockIdx.x - S.blk0) * blockDim.x + threadIdx.x;
  unsigned evals = 0;
  if (i < S.g.n)
    rk5_window_neuron<M, NP, UNI, false>(S.g, S.in, S.pa, ctxs, W, i, s_p, s_q, evals);
  if (blk_evals != nullptr) block_add_u64(evals, blk_evals);
}

// ---------------------------------------------------------------------------
// Persistent RK5 update with TMA prefetch of the neuron state. Each block
// walks the 128-neuron tiles blockIdx.x, blockIdx.x + gridDim.x, ...; the
// state columns (variables, refractory counter, step size, time offset) and
// accumulators of the next two tiles are brought into shared memory by 1-D
// bulk copies (cp.async.bulk, completion counted on an mbarrier) while the
// block integrates the current tile, so no warp waits for HBM at the start
// of its neurons. Group-uniform parameters only (they are in the constant
// bank); the arithmetic is rk5_neuron's.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void mbar_expect_tx(uint64_t *mbar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
               : : "r"(smem_u32(mbar)), "r"(bytes) : "memory");
}

// global -> shared bulk copy (16-byte aligned addresses, size a multiple of 16)
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes,
                                         uint64_t *mbar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
      : : "r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(mbar)) : "memory");
}

template <class M, int NP>
struct Rk5TileStage {
  enum { NC = M::NVAR + 3, NPI = (M::NPV == 0) ? 1 : NP };
  float col[NC][NGPU_BLOCK];          // variables, refractory, h, dx
  long long acc[NPI][NGPU_BLOCK];     // accumulators per port
};

template <class M, int NP>
__device__ __forceinline__ void rk5_issue_tile(Rk5TileStage<M, NP> &st, uint64_t *bar,
                                               const GroupArgs &g, const long long *acc,
                                               int n_acc, int t) {
  using Tr = ModelTraits<M>;
  const long long o = (long long)t * NGPU_BLOCK;
  const uint32_t cb = NGPU_BLOCK * sizeof(float), ab = NGPU_BLOCK * sizeof(long long);
  const int nv = g.nvar < M::NVAR ? g.nvar : M::NVAR;
  mbar_expect_tx(bar, (uint32_t)(nv + 3) * cb + (uint32_t)n_acc * ab);
  for (int j = 0; j < nv; j++) bulk_g2s(st.col[j], g.var + (long long)j * g.n_pad + o, cb, bar);
  bulk_g2s(st.col[M::NVAR], g.param + (long long)Tr::refr * g.n_pad + o, cb, bar);
  bulk_g2s(st.col[M::NVAR + 1], g.h + o, cb, bar);
  bulk_g2s(st.col[M::NVAR + 2], g.dx + o, cb, bar);
  for (int q = 0; q < n_acc; q++) bulk_g2s(st.acc[q], acc + (long long)q * g.n_pad + o, ab, bar);
}

template <class M, int NP, int MINB>
__global__ void __launch_bounds__(NGPU_BLOCK, MINB)
k_rk5_update_tiles(const __grid_constant__ GroupArgs g, const __grid_constant__ InputArgs in,
                   const __grid_constant__ PushArgs pa, StepCtx *ctx) {
  pdl_wait();
  pdl_trigger();
  using St = Rk5TileStage<M, NP>;
  __shared__ alignas(128) St s_st[2];
  __shared__ alignas(8) uint64_t s_bar[2];
  const int n_tiles = (g.n + NGPU_BLOCK - 1) / NGPU_BLOCK;
  const int n_acc = in.np < (int)St::NPI ? in.np : (int)St::NPI;
  const int G = gridDim.x;
  if (threadIdx.x == 0) {
    mbar_init(&s_bar[0], 1);
    mbar_init(&s_bar[1], 1);
  }
  __syncthreads();
  // this step's input half (thread 0 issues every copy)
  const long long *acc = threadIdx.x == 0 ? acc_in(in, ctx->acc_in_slot) : nullptr;
  if (threadIdx.x == 0) {
    if ((int)blockIdx.x < n_tiles) rk5_issue_tile<M, NP>(s_st[0], &s_bar[0], g, acc, n_acc, blockIdx.x);
    if ((int)blockIdx.x + G < n_tiles)
      rk5_issue_tile<M, NP>(s_st[1], &s_bar[1], g, acc, n_acc, blockIdx.x + G);
  }
  const Rk5Queue *qu = g.q.cap > 0 ? &g.q : nullptr;
  unsigned evals = 0;
  int k = 0;
  for (int t = blockIdx.x; t < n_tiles; t += G, k++) {
    const int s = k & 1;
    const bool ok = __syncthreads_and(
        mbar_wait(&s_bar[s], (k >> 1) & 1, NGPU_WAIT_ITERS, (g.wait_test & WAIT_TEST_FIRST) != 0));
    if (!ok) {
      // a copy did not land: leave this block's remaining tiles untouched,
      // after waiting (bounded) for the copies in flight, which write into
      // this block's shared memory; if that wait runs out too, the host is
      // told that the device state is lost
      if (threadIdx.x == 0) {
        atomicOr(&ctx->err, (unsigned)DERR_TILE_TIMEOUT);
        bool drained = mbar_wait(&s_bar[s], (k >> 1) & 1, NGPU_WAIT_ITERS);
        if (t + G < n_tiles)
          drained = mbar_wait(&s_bar[s ^ 1], ((k + 1) >> 1) & 1, NGPU_WAIT_ITERS) && drained;
        if (!drained) atomicOr(&ctx->err, (unsigned)DERR_TILE_DRAIN);
      }
      __syncthreads();
      break;
    }
    float pc[St::NC];
    long long pq[St::NPI];
#pragma unroll
    for (int j = 0; j < St::NC; j++) pc[j] = s_st[s].col[j][threadIdx.x];
#pragma unroll
    for (int q = 0; q < St::NPI; q++) pq[q] = s_st[s].acc[q][threadIdx.x];
    __syncthreads();                    // stage s is free again
    if (threadIdx.x == 0 && t + 2 * G < n_tiles) {
      proxy_fence_async_smem();         // order the reads above before the copy
      rk5_issue_tile<M, NP>(s_st[s], &s_bar[s], g, acc, n_acc, t + 2 * G);
    }
    const int i = t * NGPU_BLOCK + threadIdx.x;
    if (i < g.n) rk5_neuron<M, NP, true, STEP_PLAIN>(g, in, pa, ctx, i, g.puni, g.pinv, evals,
                                                     false, qu, 0, pc, pq);
  }
  if (g.blk_evals != nullptr) block_add_u64(evals, g.blk_evals);
}

// Second launch of a queued update: one straggler record per thread.
template <class M, int NP, bool UNI>
__global__ void __launch_bounds__(NGPU_BLOCK, 1)
k_rk5_finish(const __grid_constant__ GroupArgs g, const __grid_constant__ InputArgs in,
             const __grid_constant__ PushArgs pa, StepCtx *ctx) {
  // the next launch may be scheduled at once (its own wait still holds it
  // until this grid has completed); then wait for the update's records
  pdl_trigger();
  pdl_wait();
  __shared__ unsigned s_pref[NGPU_QLANES + 1];
  const unsigned n = rk5_queue_prefix(g.q, s_pref);
  if (n == 0) return;             // the same for every block: nothing to reset
  unsigned evals = 0;
  for (unsigned k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    rk5_resume<M, NP, UNI>(g, pa, ctx, g.puni, g.pinv, in.np, rk5_queue_record(g.q, s_pref, k),
                           evals, g.dry != 0);
  }
  if (g.blk_evals != nullptr) block_add_u64(evals, g.blk_evals);
  rk5_queue_reset(g.q);
}

// Many RK5 groups of one model in one launch (independent networks of a
// parameter sweep, for instance): block b integrates segment blk_seg[b],
// whose arguments are read from the device segment table; the segment's
// uniform parameters are staged in shared memory.
template <class M, int NP, bool UNI, int MINB, int MODE>
__global__ void __launch_bounds__(NGPU_BLOCK, MINB)
k_rk5_update_seg(const SegArgs *__restrict__ segs, const int *__restrict__ blk_seg,
                 unsigned long long *blk_evals, int dry, StepCtx *ctx,
                 const __grid_constant__ Rk5Queue qu) {
  pdl_wait();
  pdl_trigger();
  __shared__ float s_p[M::NPARAM], s_q[M::NPARAM];
  const int seg = blk_seg[blockIdx.x];
  const SegArgs &S = segs[seg];
  if (UNI) {
    for (int j = threadIdx.x; j < M::NPARAM; j += blockDim.x) {
      s_p[j] = S.g.puni[j];
      s_q[j] = S.g.pinv[j];
    }
    __syncthreads();
  }
  const int i = (blockIdx.x - S.blk0) * blockDim.x + threadIdx.x;
  unsigned evals = 0;
  const bool queued = (MODE == STEP_PLAIN) && qu.cap > 0;
  if (i < S.g.n)
    rk5_neuron<M, NP, UNI, MODE>(S.g, S.in, S.pa, ctx, i, s_p, s_q, evals, dry != 0,
                                 queued ? &qu : nullptr, seg, nullptr, nullptr, blockIdx.x);
  if (blk_evals != nullptr) block_add_u64(evals, blk_evals);
}

// Second launch of a queued batched update: one straggler record per
// thread, with the arguments of the record's segment.
template <class M, int NP, bool UNI>
__global__ void __launch_bounds__(NGPU_BLOCK, 1)
k_rk5_finish_seg(const SegArgs *__restrict__ segs, unsigned long long *blk_evals, int dry,
                 StepCtx *ctx, const __grid_constant__ Rk5Queue qu) {
  // the next launch may be scheduled at once (its own wait still holds it
  // until this grid has completed); then wait for the update's records
  pdl_trigger();
  pdl_wait();
  __shared__ unsigned s_pref[NGPU_QLANES + 1];
  const unsigned n = rk5_queue_prefix(qu, s_pref);
  if (n == 0) return;             // the same for every block: nothing to reset
  unsigned evals = 0;
  for (unsigned k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const float *r = rk5_queue_record(qu, s_pref, k);
    const SegArgs &R = segs[__float_as_int(r[1])];
    rk5_resume<M, NP, UNI>(R.g, R.pa, ctx, R.g.puni, R.g.pinv, R.in.np, r, evals,
                           R.g.dry || dry != 0);
  }
  if (blk_evals != nullptr) block_add_u64(evals, blk_evals);
  rk5_queue_reset(qu);
}

// Finishing launch of an update with the learned step proposer: the update
// is the plain kernel with the straggler queue on, so a neuron whose first
// sub-step (the controller's guess) completes the time step, the common
// case, never waits for a tensor-core round; the records of the others are
// taken 128 per CTA, which integrates them in lock-step rounds of one
// sub-step: each round in which a record's next step is shorter than the
// rest of the time step is one CTA-wide MMA of the proposer network
// (src/rk5.h:57-162 for the sub-step; the proposal replaces the
// controller's guess, the error test still accepts or rejects). SEG: records
// of a batched launch (the record's segment gives its arguments; g0 is the
// first segment's, for the proposer's weights and margin).
template <class M, int NP, bool UNI, bool SEG>
__global__ void __launch_bounds__(NGPU_BLOCK, 1)
k_rk5_finish_learned(const __grid_constant__ GroupArgs g0, const __grid_constant__ PushArgs pa0,
                     int np0, const SegArgs *__restrict__ segs, unsigned long long *blk_evals,
                     int dry, StepCtx *ctx, const __grid_constant__ Rk5Queue qu) {
  using Tr = ModelTraits<M>;
  pdl_trigger();
  pdl_wait();
  __shared__ unsigned s_pref[NGPU_QLANES + 1];
  const unsigned n = rk5_queue_prefix(qu, s_pref);
  if (n == 0) return;             // the same for every block: nothing to reset
  __shared__ ProposerSmem ps;
  proposer_alloc(ps);
  bool staged = false, failed = false;
  unsigned evals = 0;
  const long long it = ctx->it;
  const long long T = ctx->T0 + it + 1;
  for (unsigned base = blockIdx.x * NGPU_BLOCK; base < n; base += gridDim.x * NGPU_BLOCK) {
    const unsigned k = base + threadIdx.x;
    const bool act = k < n;
    const float *r = act ? rk5_queue_record(qu, s_pref, k) : nullptr;
    const int seg = (SEG && act) ? __float_as_int(r[1]) : 0;
    const GroupArgs &g = SEG ? segs[seg].g : g0;
    const PushArgs &pa = SEG ? segs[seg].pa : pa0;
    const int np = (NP >= 2 && NP <= 4) ? NP : (SEG ? segs[seg].in.np : np0);
    const int i = act ? __float_as_int(r[0]) : 0;
    int guard = act ? __float_as_int(r[2]) : 0;
    float h = act ? r[3] : 0.0f;
    float refr = act ? r[4] : 0.0f;
    double x = act ? *reinterpret_cast<const double *>(r + 6) : 0.0;
    float y[M::NVAR];
#pragma unroll
    for (int j = 0; j < M::NVAR; j++) y[j] = act ? r[8 + j] : 0.0f;
    float p_loc[UNI ? 1 : M::NPARAM];
    float q_loc[UNI ? 1 : M::NPARAM];
    rk5_load_params<M, UNI>(g, i, act, p_loc, q_loc);
    const float *p = UNI ? g.puni : p_loc;
    const float *q = UNI ? g.pinv : q_loc;
    const double x1 = ctx->t0 + (double)g.dt * (double)(it + 1);
    const int den = (UNI && g.den_delay_col == Tr::den) ? g.den_steps
                                                         : (int)roundf(p[Tr::den] / g.dt);
    const bool dry_g = dry != 0 || g.dry != 0;
    bool end = !act;
    while (__syncthreads_or(!end)) {
      const float hmax = !end ? (float)(x1 - x) : 0.0f;
      const bool want = !end && !failed && h < hmax;
      if (__syncthreads_or(want)) {
        if (!staged) {
          proposer_stage_weights(ps, g0.mlp);
          staged = true;
        }
        float f[6] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
        if (want) ProposerFeatures<M>::get(y, p, h, g.dt, f);
        float o = 0.0f;
        if (proposer_round(ps, want, f, o, &ctx->err, g0.wait_test)) {
          if (want) {
            // the proposal may shrink the controller's guess by at most 4x
            // (after a low-error step it then still grows, >= 1.25x) and
            // enlarge it by at most 16x: a network queried outside its
            // training distribution cannot stall or blow up the integration
            const float hp = g.dt * exp2f(o - g0.mlp_margin);
            h = fminf(fmaxf(fminf(fmaxf(hp, 0.25f * h), 16.0f * h), g.h_min), hmax);
          }
        } else {
          failed = true;
        }
      }
      if (!end) {
        end = rk5_plain_substep<M, NP>(g, pa, ctx, i, y, x, h, refr, guard, p, q, np, g.inv_eps,
                                       x1, T, den, dry_g, evals);
      }
    }
    if (act && !dry_g) rk5_store<M, NP>(g, i, y, h, x, x1, refr, true);
  }
  proposer_teardown(ps, failed);
  if (blk_evals != nullptr) block_add_u64(evals, blk_evals);
  rk5_queue_reset(qu);
}

}  // namespace ngpu
