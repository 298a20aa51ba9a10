// Simulation kernels for sm_100a.
//
// Per time step the driver launches (captured in CUDA graphs of a chunk of
// steps):
//   1. the node updates: one launch per RK5 group or batch of RK5 groups
//      (ngpu_kernels_common.cuh, ngpu_rk5_batch.cu) plus its straggler
//      finishing launch, and one launch for the groups of simple models; each
//      folds the pending synaptic input of the previous step into the state
//      (the reference's GetSpikes and PoissGenSendSpikeKernel,
//      src/get_spike.cu:116-140, src/poiss_gen.cu:43-74), integrates the step
//      and appends emitted spikes to this step's ring slot
//      (src/spike_buffer.cu:143-228);
//   2. k_deliver: expands the (source, delay) groups that fall due in this
//      step into fixed-point accumulator additions, with the STDP pre-spike
//      rule (src/spike_buffer.cu:233-302, src/nested_loop.cu:39-167,
//      src/get_spike.cu:48-85); without plastic synapses it runs on a second
//      stream beside the node updates;
//   3. k_stdp_post: STDP post-spike rule over incoming plastic synapses of the
//      neurons that spiked (src/rev_spike.cu:41-75);
//   4. k_record (multimeter columns); k_advance only for networks without
//      delivery.
// No host synchronisation happens inside a step; each step of a chunk reads
// its own device-resident copy of the step context (k_step_prologue).
#include <cuda_runtime.h>
#include <math.h>
#include <stdlib.h>
#include "ngpu_device.h"
#include "ngpu_kernels.h"
#include "ngpu_models.h"
#include "ngpu_rk5_models.cuh"
#include "ngpu_rng.h"
#include "ngpu_kernels_common.cuh"
#include "ngpu_deliver.cuh"

namespace ngpu {

int Rk5VariantCount(int np, int all_uniform) { return (all_uniform && np <= 4) ? NGPU_RK5_VARIANTS : 1; }

bool LaunchRk5Update(int model, int np, const GroupArgs &g,
                     const InputArgs &in, const PushArgs &pa, StepCtx *ctx,
                     cudaStream_t s, const DeliverArgs *del, int n_del) {
  if (g.n <= 0) return false;
  if (del != nullptr && (del->nd <= 0 || del->e_syn != nullptr || n_del <= 0)) del = nullptr;
  switch (model) {
    case RK5_AEIF_COND_BETA: return LaunchRk5AeifCondBeta(np, g, in, pa, ctx, s, del, n_del);
    case RK5_AEIF_COND_ALPHA: return LaunchRk5AeifCondAlpha(np, g, in, pa, ctx, s, del, n_del);
    case RK5_AEIF_PSC_ALPHA:
    case RK5_AEIF_PSC_EXP:
    case RK5_AEIF_PSC_DELTA: return LaunchRk5AeifPsc(model, np, g, in, pa, ctx, s, del, n_del);
    case RK5_IZHIKEVICH_COND_BETA: return LaunchRk5IzhCondBeta(np, g, in, pa, ctx, s, del, n_del);
    default: return false;
  }
}

bool LaunchRk5Window(int model, int np, bool free_lanes, const GroupArgs &g, const InputArgs &in,
                     const PushArgs &pa, StepCtx *ctxs, int W, cudaStream_t s) {
  if (g.n <= 0) return true;
  switch (model) {
    case RK5_AEIF_COND_BETA: return LaunchRk5WindowAeifCondBeta(np, free_lanes, g, in, pa, ctxs, W, s);
    case RK5_AEIF_COND_ALPHA: return LaunchRk5WindowAeifCondAlpha(np, free_lanes, g, in, pa, ctxs, W, s);
    case RK5_AEIF_PSC_ALPHA:
    case RK5_AEIF_PSC_EXP:
    case RK5_AEIF_PSC_DELTA: return LaunchRk5WindowAeifPsc(model, np, free_lanes, g, in, pa, ctxs, W, s);
    case RK5_IZHIKEVICH_COND_BETA: return LaunchRk5WindowIzhCondBeta(np, free_lanes, g, in, pa, ctxs, W, s);
    default: return false;
  }
}

// floats of a straggler record for the kernel instance LaunchRk5Update picks
template <template <int> class MT>
static int rk5_nvar(int np) {
  switch (np) {
    case 0:
    case 1: return MT<1>::NVAR;
    case 2: return MT<2>::NVAR;
    case 3: return MT<3>::NVAR;
    case 4: return MT<4>::NVAR;
    default: return np <= 8 ? MT<8>::NVAR : MT<20>::NVAR;
  }
}

int Rk5RecordFloats(int model, int np) {
  int nv = 0;
  switch (model) {
    case RK5_AEIF_COND_BETA: nv = rk5_nvar<AeifCondBeta>(np); break;
    case RK5_AEIF_COND_ALPHA: nv = rk5_nvar<AeifCondAlpha>(np); break;
    case RK5_AEIF_PSC_ALPHA: nv = rk5_nvar<AeifPscAlpha>(np); break;
    case RK5_AEIF_PSC_EXP: nv = rk5_nvar<AeifPscExp>(np); break;
    case RK5_AEIF_PSC_DELTA: nv = AeifPscDelta<1>::NVAR; break;
    case RK5_IZHIKEVICH_COND_BETA: nv = rk5_nvar<IzhCondBeta>(np); break;
    default: return 0;
  }
  return (8 + nv + 3) / 4 * 4;
}

// ---------------------------------------------------------------------------
// iaf_psc_exp: exact propagator update (src/iaf_psc_exp.cu:94-119)
// ---------------------------------------------------------------------------
__device__ __forceinline__ float gparam(const GroupArgs &g, int j, int i) {
  return pbit(g.pmask, j) ? g.param[(long long)j * g.n_pad + i] : g.puni[j];
}

__device__ __forceinline__ void iaf_psc_exp_node(const GroupArgs &g, const InputArgs &in,
                                                 const PushArgs &pa, StepCtx *ctx, int i) {
  const long long it = ctx->it, T0 = ctx->T0;
  const double t0 = ctx->t0;
  const int n_pad = g.n_pad;
  float *var = g.var;
  float I_ex = var[i], I_in = var[n_pad + i];
  float V = var[2 * n_pad + i], refr = var[3 * n_pad + i];
  long long s[2];
  input_sum<2, false>(in, i, n_pad, 2, it, t0, g.dt, ctx->poisson_pending, T0,
               ctx->acc_in_slot, s);
  if (s[0] != 0) I_ex = fold_value(I_ex, s[0], 1.0f);
  if (s[1] != 0) I_in = fold_value(I_in, s[1], 1.0f);
  const float I_e = gparam(g, 3, i), Theta = gparam(g, 4, i);
  const float V_reset = gparam(g, 5, i), t_ref = gparam(g, 8, i);
  const float P20 = gparam(g, 10, i), P11ex = gparam(g, 11, i);
  const float P11in = gparam(g, 12, i), P21ex = gparam(g, 13, i);
  const float P21in = gparam(g, 14, i), P22 = gparam(g, 15, i);
  if (refr > 0.0f) {
    refr -= 1.0f;
  } else {
    V = V * P22 + I_ex * P21ex + I_in * P21in + I_e * P20;
  }
  I_ex *= P11ex;
  I_in *= P11in;
  if (V >= Theta) {
    const long long T = T0 + it + 1;
    const double t_now = t0 + (double)g.dt * (double)(it + 1);
    const int den = (int)roundf(gparam(g, 9, i) / g.dt);
    push_spike(pa, ctx, g.i_node_0 + i, i, 1.0f, T, t_now, den);
    V = V_reset;
    refr = (float)(int)roundf(t_ref / g.dt);
  }
  var[i] = I_ex;
  var[n_pad + i] = I_in;
  var[2 * n_pad + i] = V;
  var[3 * n_pad + i] = refr;
}

__global__ void __launch_bounds__(NGPU_BLOCK)
k_iaf_psc_exp(GroupArgs g, InputArgs in, PushArgs pa, StepCtx *ctx) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < g.n) iaf_psc_exp_node(g, in, pa, ctx, i);
}

void LaunchIafPscExpUpdate(const GroupArgs &g, const InputArgs &in,
                           const PushArgs &pa, StepCtx *ctx, cudaStream_t s) {
  if (g.n <= 0) return;
  k_iaf_psc_exp<<<(g.n + NGPU_BLOCK - 1) / NGPU_BLOCK, NGPU_BLOCK, 0, s>>>(
      g, in, pa, ctx);
}

// ---------------------------------------------------------------------------
// iaf_psc_exp_g and iaf_psc_exp_hc (src/iaf_psc_exp_g.cu:39-66,
// src/iaf_psc_exp_hc.cu:33-59): one exponential current, exact propagators
// of the group. gc = P11, P22, P21, P20, Theta_rel, V_reset_rel, refractory
// steps. Variables I_syn, V_m_rel, refractory_step; parameter I_e.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void iaf_psc_exp_g_node(const GroupArgs &g, const InputArgs &in,
                                                   const PushArgs &pa, StepCtx *ctx, int i) {
  const long long it = ctx->it, T0 = ctx->T0;
  const double t0 = ctx->t0;
  const int n_pad = g.n_pad;
  float *var = g.var;
  float I_syn = var[i], V = var[n_pad + i], refr = var[2 * n_pad + i];
  long long s[1];
  input_sum<1, false>(in, i, n_pad, 1, it, t0, g.dt, ctx->poisson_pending, T0,
               ctx->acc_in_slot, s);
  if (s[0] != 0) I_syn = fold_value(I_syn, s[0], 1.0f);
  const float I_e = gparam(g, 0, i);
  if (refr > 0.0f) {
    refr -= 1.0f;
  } else {
    V = V * g.gc[1] + I_syn * g.gc[2] + I_e * g.gc[3];
  }
  I_syn *= g.gc[0];
  if (V >= g.gc[4]) {
    const long long T = T0 + it + 1;
    const double t_now = t0 + (double)g.dt * (double)(it + 1);
    push_spike(pa, ctx, g.i_node_0 + i, i, 1.0f, T, t_now, 0);
    V = g.gc[5];
    refr = g.gc[6];
  }
  var[i] = I_syn;
  var[n_pad + i] = V;
  var[2 * n_pad + i] = refr;
}

// ---------------------------------------------------------------------------
// izhikevich (src/izhikevich.cu:38-72): forward Euler, the input of the
// previous step added to V_m. The quadratic is evaluated with double
// constants, i.e. in FP64, as in the reference. gc = V_th, a, b, c, d,
// refractory steps, h. Variables I_syn, V_m, u, refractory_step; parameters
// I_e, den_delay.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void izhikevich_node(const GroupArgs &g, const InputArgs &in,
                                                const PushArgs &pa, StepCtx *ctx, int i) {
  const long long it = ctx->it, T0 = ctx->T0;
  const double t0 = ctx->t0;
  const int n_pad = g.n_pad;
  float *var = g.var;
  float I_syn = var[i], V = var[n_pad + i], u = var[2 * n_pad + i];
  float refr = var[3 * n_pad + i];
  long long s[1];
  input_sum<1, false>(in, i, n_pad, 1, it, t0, g.dt, ctx->poisson_pending, T0,
               ctx->acc_in_slot, s);
  if (s[0] != 0) I_syn = fold_value(I_syn, s[0], 1.0f);
  const float I_e = gparam(g, 0, i);
  const float h = g.gc[6], a = g.gc[1], b = g.gc[2];
  if (refr > 0.0f) {
    refr -= 1.0f;
  } else {
    const float v_old = V, u_old = u;
    V += h * (0.04 * v_old * v_old + 5.0 * v_old + 140.0 - u_old + I_e) + I_syn;
    u += h * a * (b * v_old - u_old);
  }
  I_syn = 0.0f;
  if (V >= g.gc[0]) {
    const long long T = T0 + it + 1;
    const double t_now = t0 + (double)g.dt * (double)(it + 1);
    const int den = (int)roundf(gparam(g, 1, i) / g.dt);
    push_spike(pa, ctx, g.i_node_0 + i, i, 1.0f, T, t_now, den);
    V = g.gc[3];
    u += g.gc[4];
    refr = g.gc[5] < 0.0f ? 0.0f : g.gc[5];
  }
  var[i] = I_syn;
  var[n_pad + i] = V;
  var[2 * n_pad + i] = u;
  var[3 * n_pad + i] = refr;
}

// ---------------------------------------------------------------------------
// izhikevich_psc_exp, _2s, _5s (src/izhikevich_psc_exp.cu:40-76,
// src/izhikevich_psc_exp_2s.cu:41-83): NSUB forward-Euler sub-steps of
// dt / NSUB per time step, each followed by the decay of the exponential
// current; a refractory neuron only decays its current. gc = V_th, a, b, c,
// d, refractory steps, sub-step h, current decay per sub-step.
// ---------------------------------------------------------------------------
template <int NSUB>
__device__ __forceinline__ void izh_psc_exp_node(const GroupArgs &g, const InputArgs &in,
                                                 const PushArgs &pa, StepCtx *ctx, int i) {
  const long long it = ctx->it, T0 = ctx->T0;
  const double t0 = ctx->t0;
  const int n_pad = g.n_pad;
  float *var = g.var;
  float I_syn = var[i], V = var[n_pad + i], u = var[2 * n_pad + i];
  float refr = var[3 * n_pad + i];
  long long s[1];
  input_sum<1, false>(in, i, n_pad, 1, it, t0, g.dt, ctx->poisson_pending, T0,
               ctx->acc_in_slot, s);
  if (s[0] != 0) I_syn = fold_value(I_syn, s[0], 1.0f);
  const float I_e = gparam(g, 0, i);
  const float h = g.gc[6], a = g.gc[1], b = g.gc[2], C_syn = g.gc[7];
  if (refr > 0.0f) {
    refr -= 1.0f;
#pragma unroll
    for (int k = 0; k < NSUB; k++) I_syn *= C_syn;
  } else {
#pragma unroll
    for (int k = 0; k < NSUB; k++) {
      const float v_old = V, u_old = u;
      V += h * (0.04 * v_old * v_old + 5.0 * v_old + 140.0 - u_old + I_syn + I_e);
      u += h * a * (b * v_old - u_old);
      I_syn *= C_syn;
    }
  }
  if (V >= g.gc[0]) {
    const long long T = T0 + it + 1;
    const double t_now = t0 + (double)g.dt * (double)(it + 1);
    const int den = (int)roundf(gparam(g, 1, i) / g.dt);
    push_spike(pa, ctx, g.i_node_0 + i, i, 1.0f, T, t_now, den);
    V = g.gc[3];
    u += g.gc[4];
    refr = g.gc[5] < 0.0f ? 0.0f : g.gc[5];
  }
  var[i] = I_syn;
  var[n_pad + i] = V;
  var[2 * n_pad + i] = u;
  var[3 * n_pad + i] = refr;
}

// one node of a simple model (kind: ModelKind; n_sub: Euler sub-steps of
// the izhikevich_psc_exp family)
__device__ __forceinline__ void simple_node(int kind, int n_sub, const GroupArgs &g,
                                            const InputArgs &in, const PushArgs &pa,
                                            StepCtx *ctx, int i) {
  switch (kind) {
    case MK_IAF_PSC_EXP: iaf_psc_exp_node(g, in, pa, ctx, i); break;
    case MK_IAF_PSC_EXP_G: iaf_psc_exp_g_node(g, in, pa, ctx, i); break;
    case MK_IZHIKEVICH: izhikevich_node(g, in, pa, ctx, i); break;
    case MK_IZH_PSC_EXP:
      if (n_sub == 5) izh_psc_exp_node<5>(g, in, pa, ctx, i);
      else if (n_sub == 2) izh_psc_exp_node<2>(g, in, pa, ctx, i);
      else izh_psc_exp_node<1>(g, in, pa, ctx, i);
      break;
    default: break;
  }
}

__global__ void __launch_bounds__(NGPU_BLOCK)
k_simple(GroupArgs g, InputArgs in, PushArgs pa, StepCtx *ctx, int kind, int n_sub) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < g.n) simple_node(kind, n_sub, g, in, pa, ctx, i);
}

// Many groups of simple models in one launch: block b updates 128 nodes of
// segment blk_seg[b] (the cortical column's eight populations are one
// launch per step instead of eight).
__global__ void __launch_bounds__(NGPU_BLOCK)
k_simple_seg(const SegArgs *__restrict__ segs, const int *__restrict__ blk_seg, StepCtx *ctx) {
  const SegArgs &S = segs[blk_seg[blockIdx.x]];
  const int i = (blockIdx.x - S.blk0) * blockDim.x + threadIdx.x;
  if (i < S.g.n) simple_node(S.kind, S.n_sub, S.g, S.in, S.pa, ctx, i);
}

void LaunchSimpleBatch(const SegArgs *segs, const int *blk_seg, int n_blocks, StepCtx *ctx,
                       cudaStream_t s) {
  if (n_blocks <= 0) return;
  k_simple_seg<<<n_blocks, NGPU_BLOCK, 0, s>>>(segs, blk_seg, ctx);
}

void LaunchSimpleNeuronUpdate(int kind, int n_sub, const GroupArgs &g, const InputArgs &in,
                              const PushArgs &pa, StepCtx *ctx, cudaStream_t s) {
  if (g.n <= 0) return;
  const dim3 grid((g.n + NGPU_BLOCK - 1) / NGPU_BLOCK), block(NGPU_BLOCK);
  k_simple<<<grid, block, 0, s>>>(g, in, pa, ctx, kind, n_sub);
}

// ---------------------------------------------------------------------------
// spike_generator (src/spike_generator.cu:37-55)
// ---------------------------------------------------------------------------
__global__ void k_spike_generator(GroupArgs g, PushArgs pa, StepCtx *ctx) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.n) return;
  const long long it = ctx->it, T0 = ctx->T0;
  const long long step = T0 + it;
  int b = g.sg_next[i];
  if (b < g.sg_off[i + 1] && (long long)g.sg_step[b] == step) {
    const long long T = step + 1;
    const double t_now = ctx->t0 + (double)g.dt * (double)(it + 1);
    push_spike(pa, ctx, g.i_node_0 + i, i, g.sg_height[b], T, t_now, 0);
    g.sg_next[i] = b + 1;
  }
}

void LaunchSpikeGeneratorUpdate(const GroupArgs &g, const PushArgs &pa,
                                StepCtx *ctx, cudaStream_t s) {
  if (g.n <= 0) return;
  k_spike_generator<<<(g.n + NGPU_BLOCK - 1) / NGPU_BLOCK, NGPU_BLOCK, 0, s>>>(
      g, pa, ctx);
}

// ---------------------------------------------------------------------------
// parrot_neuron (src/parrot_neuron.cu:48-70)
// ---------------------------------------------------------------------------
__global__ void k_parrot(GroupArgs g, InputArgs in, PushArgs pa,
                         StepCtx *ctx) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.n) return;
  const long long it = ctx->it, T0 = ctx->T0;
  const double t0 = ctx->t0;
  const int n_pad = g.n_pad;
  float *var = g.var;
  long long s[2];
  input_sum<2, false>(in, i, n_pad, 2, it, t0, g.dt, ctx->poisson_pending, T0,
               ctx->acc_in_slot, s);
  float sh = var[i];
  if (s[0] != 0) sh = fold_value(sh, s[0], 1.0f);
  if (s[1] != 0) var[n_pad + i] = fold_value(var[n_pad + i], s[1], 0.0f);
  var[2 * n_pad + i] = sh;
  if (sh != 0.0f) {
    if (gparam(g, 0, i) == 0.0f) sh = 1.0f;
    const long long T = T0 + it + 1;
    const double t_now = t0 + (double)g.dt * (double)(it + 1);
    const int den = (int)roundf(gparam(g, 1, i) / g.dt);
    push_spike(pa, ctx, g.i_node_0 + i, i, sh, T, t_now, den);
    var[i] = 0.0f;
  } else {
    var[i] = sh;
  }
}

void LaunchParrotUpdate(const GroupArgs &g, const InputArgs &in,
                        const PushArgs &pa, StepCtx *ctx, cudaStream_t s) {
  if (g.n <= 0) return;
  k_parrot<<<(g.n + NGPU_BLOCK - 1) / NGPU_BLOCK, NGPU_BLOCK, 0, s>>>(g, in,
                                                                     pa, ctx);
}

// ---------------------------------------------------------------------------
// spike_detector (src/spike_detector.cu:43-66)
// ---------------------------------------------------------------------------
__global__ void k_spike_detector(GroupArgs g, InputArgs in, StepCtx *ctx) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.n) return;
  const int n_pad = g.n_pad;
  float *var = g.var;
  long long s[1];
  input_sum<1>(in, i, n_pad, 1, ctx->it, ctx->t0, g.dt, ctx->poisson_pending,
               ctx->T0, ctx->acc_in_slot, s);
  float sh = var[i];
  if (s[0] != 0) sh = fold_value(sh, s[0], 1.0f);
  if (sh != 0.0f) {
    if (gparam(g, 0, i) == 0.0f) sh = 1.0f;
    var[i] = 0.0f;
  } else {
    var[i] = sh;
  }
  var[n_pad + i] = sh;
}

void LaunchSpikeDetectorUpdate(const GroupArgs &g, const InputArgs &in,
                               StepCtx *ctx, cudaStream_t s) {
  if (g.n <= 0) return;
  k_spike_detector<<<(g.n + NGPU_BLOCK - 1) / NGPU_BLOCK, NGPU_BLOCK, 0, s>>>(
      g, in, ctx);
}

// ---------------------------------------------------------------------------
// CreatePoissonGenerator nodes: one count per node per step pushed as a
// spike of that height (src/poisson.cu:26-54)
// ---------------------------------------------------------------------------
// The reference draws the counts in blocks of ceil(1e5 / n) steps and zeroes
// counts above 5 lambda in the first step of every block only
// (src/poisson.cu:45-88: the fix-up kernel covers n_node entries).
__global__ void k_poisson_nodes(GroupArgs g, PushArgs pa, double lambda,
                                double explam, unsigned long long seed,
                                StepCtx *ctx) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.n) return;
  const long long it = ctx->it, T0 = ctx->T0;
  const long long T = T0 + it + 1;
  unsigned n = ng_poisson(lambda, explam, seed, RNG_TAG_POISSON_NODE,
                          (unsigned long long)(g.i_node_0 + i), T);
  const long long block_steps = (100000 - 1) / g.n + 1;
  if ((T - 1) % block_steps == 0 && (float)n > (float)lambda * 5.0f) n = 0;
  if (n > 0) {
    const double t_now = ctx->t0 + (double)g.dt * (double)(it + 1);
    push_spike(pa, ctx, g.i_node_0 + i, i, (float)n, T, t_now, 0);
  }
}

void LaunchPoissonNodesUpdate(const GroupArgs &g, const PushArgs &pa,
                              double lambda, double explam,
                              unsigned long long seed, StepCtx *ctx,
                              cudaStream_t s) {
  if (g.n <= 0) return;
  k_poisson_nodes<<<(g.n + NGPU_BLOCK - 1) / NGPU_BLOCK, NGPU_BLOCK, 0, s>>>(
      g, pa, lambda, explam, seed, ctx);
}

// ---------------------------------------------------------------------------
// input fold outside the step loop
// ---------------------------------------------------------------------------
__global__ void k_fold_input(GroupArgs g, InputArgs in, StepCtx *ctx) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.n || in.np <= 0 || in.in_var < 0) return;
  long long s[4];
  const int np = in.np < 4 ? in.np : 4;
  input_sum<4>(in, i, g.n_pad, np, ctx->it, ctx->t0, g.dt, ctx->poisson_pending,
               ctx->T0, ctx->acc_in_slot, s);
  for (int q = 0; q < np; q++) {
    if (s[q] == 0) continue;
    float w;
    if (in.w_param) {
      w = gparam(g, in.w_col + q * in.w_col_step, i);
    } else {
      w = in.w_const[q];
    }
    float *v = g.var + (long long)(in.in_var + q * in.in_step) * g.n_pad + i;
    *v = fold_value(*v, s[q], w);
  }
  // ports beyond 4 (RK5 groups with many receptors)
  for (int q = 4; q < in.np; q++) {
    long long *a = acc_in(in, ctx->acc_in_slot) + (long long)q * g.n_pad + i;
    long long sv = *a;
    if (sv == 0) continue;
    *a = 0;
    float w = in.w_param ? gparam(g, in.w_col + q * in.w_col_step, i)
                         : in.w_const[3];
    float *v = g.var + (long long)(in.in_var + q * in.in_step) * g.n_pad + i;
    *v = fold_value(*v, sv, w);
  }
}

// Poisson direct connections of NGPU_POISSON_INV_MAX or more expected spikes
// per step into a group of RK5 neurons, simple-model neurons or parrots:
// drawn here, before the group's update, and added into the accumulator slot
// that the update folds (those update kernels leave these connections out). The draws are the ones the update would make
// and the accumulators hold fixed-point integers, so the folded input is the
// same bit for bit. One thread per node, the only writer of its slots at
// this point of the step (the delivery that filled this half has finished).
__global__ void k_poisson_large(GroupArgs g, InputArgs in, StepCtx *ctx) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.n || !ctx->poisson_pending) return;
  const long long it = ctx->it, T0 = ctx->T0;
  const double t = ctx->t0 + (double)g.dt * (double)it;
  long long *acc = acc_in(in, ctx->acc_in_slot) + i;
  // the slot may now hold input: stamp it for the update (one store; a
  // stamp on a slot that stays zero only costs the update its loads)
  if (i == 0 && in.acc_stamp != nullptr)
    in.acc_stamp[in.acc_slots > 1 ? ctx->acc_in_slot : 0] = T0 + it;
  if (in.ud) {
    const unsigned n = direct_count<false, true>(
        t - (double)in.ud_origin - (double)in.ud_delay, in.ud_start, in.ud_stop, in.ud_lambda,
        nullptr, nullptr, in.seed, in.ud_stream0 + (unsigned long long)i, T0 + it);
    if (n > 0) acc[(long long)in.ud_port * g.n_pad] += ng_to_fixed(in.ud_w * (float)n);
  } else if (in.dc_off != nullptr) {
    const unsigned b = in.dc_off[i], e = in.dc_off[i + 1];
    for (unsigned c = b; c < e; c++) {
      const unsigned gen = in.dc_gen[c];
      const unsigned n = direct_count<false, true>(
          t - (double)in.gen_origin[gen] - (double)in.dc_delay[c], in.gen_start[gen],
          in.gen_stop[gen], in.gen_lambda[gen], nullptr, nullptr, in.seed,
          in.dc_stream[c], T0 + it);
      if (n > 0) acc[(long long)in.dc_port[c] * g.n_pad] += ng_to_fixed(in.dc_weight[c] * (float)n);
    }
  }
}

void LaunchPoissonLarge(const GroupArgs &g, const InputArgs &in, StepCtx *ctx,
                        cudaStream_t s) {
  if (g.n <= 0) return;
  k_poisson_large<<<(g.n + 127) / 128, 128, 0, s>>>(g, in, ctx);
}

__global__ void k_clear_pending(StepCtx *ctx) { ctx->poisson_pending = 0; }

void LaunchFoldInput(const GroupArgs &g, const InputArgs &in, StepCtx *ctx,
                     cudaStream_t s) {
  if (g.n <= 0) return;
  k_fold_input<<<(g.n + NGPU_BLOCK - 1) / NGPU_BLOCK, NGPU_BLOCK, 0, s>>>(
      g, in, ctx);
}

void LaunchClearPending(StepCtx *ctx, cudaStream_t s) {
  k_clear_pending<<<1, 1, 0, s>>>(ctx);
}

// register cap of the static delivery kernels: 4 blocks of 256 threads per
// SM (64 registers, no spill; 6 and 8 blocks spill 80-230 bytes)
#define NGPU_DELIVER_MINB 4
template <bool PLASTIC>
__global__ void __launch_bounds__(256, PLASTIC ? 1 : NGPU_DELIVER_MINB)
k_deliver(DeliverArgs d, SynGroupTable syn, StepCtx *ctx) {
  deliver_blocks<PLASTIC>(d, syn, ctx, blockIdx.x, gridDim.x);
}

// the register cap of the window delivery (blocks per SM): 3, or 2 where
// NGB200_WINDOW_DELIVER_BLOCKS says so
static int WindowDeliverCap() {
  static const int cap = [] {
    const char *e = getenv("NGB200_WINDOW_DELIVER_BLOCKS");
    return (e != nullptr && atoi(e) == 2) ? 2 : 3;
  }();
  return cap;
}

// Spike bookkeeping of a window, by the threads of one block: the spikes of
// the steps T_b + c_lo ... T_b + c_hi - 1 (T_b the step of ctx) are counted
// into ctx->n_spikes, then the ring slots of the steps T_b + first_off ...
// T_b + first_off + n - 1 are emptied for the steps that will write them
// (the two ranges may share ring slots: counted first).
struct WindowBook {
  long long first_off;
  int n;
  long long c_lo, c_hi;
};

__device__ __forceinline__ void window_book_block(int *ring_cnt, int ring_R, int ring_C,
                                                  StepCtx *ctx, const WindowBook &bk) {
  __shared__ unsigned long long s_cnt[256];
  const long long T_b = ctx->T0 + ctx->it + 1;
  unsigned long long cnt = 0;
  for (long long rel = bk.c_lo + threadIdx.x; rel < bk.c_hi; rel += blockDim.x) {
    if (T_b + rel < 0) continue;
    const int c = ring_cnt[ring_add(ctx->ring_slot, rel, ring_R)];
    cnt += (unsigned long long)(c < ring_C ? c : ring_C);
  }
  s_cnt[threadIdx.x] = cnt;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int j = 1; j < (int)blockDim.x; j++) cnt += s_cnt[j];
    ctx->n_spikes += cnt;
  }
  for (int k = threadIdx.x; k < bk.n; k += blockDim.x) {
    const long long rel = bk.first_off + k;
    if (T_b + rel >= 0) ring_cnt[ring_add(ctx->ring_slot, rel, ring_R)] = 0;
  }
}

// Delivery before a window of integrated steps: the accumulator slots of
// the steps T_b + v_lo ... T_b + v_lo + v_n - 1 (T_b: the step of ctx, the
// window's first step) filled from the spike ring at the delays
// d.delays[di0 ...]; the last block to finish (every block has then read
// the ring) does the window's bookkeeping (one launch less per window).
// MINB: resident blocks per SM the registers are capped for. The window
// delivery keeps two items in flight per warp (105 registers uncapped): 3
// blocks per SM spill a few words, 2 blocks do not;
// NGB200_WINDOW_DELIVER_BLOCKS picks one (default 3).
template <int MINB>
__global__ void __launch_bounds__(256, MINB)
k_deliver_window(DeliverArgs d, StepCtx *ctx, int v_lo, int v_n, int di0, int D_lo, int D_hi,
                 WindowBook bk) {
  deliver_window_blocks(d, ctx, v_lo, v_n, di0, D_lo, D_hi, blockIdx.x, gridDim.x);
  __shared__ bool s_last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    s_last = atomicAdd(d.done, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  window_book_block(d.ring_cnt_w, d.ring_R, d.ring_C, ctx, bk);
  if (threadIdx.x == 0) *d.done = 0u;
}

// the bookkeeping alone (a window with nothing to deliver)
__global__ void k_window_book(int *ring_cnt, int ring_R, int ring_C, StepCtx *ctx, WindowBook bk) {
  window_book_block(ring_cnt, ring_R, ring_C, ctx, bk);
}

void LaunchDeliverWindow(const DeliverArgs &d, StepCtx *ctx, int v_lo, int v_n, int di0,
                         int D_lo, int D_hi, long long book_first_off, int book_n,
                         long long c_lo, long long c_hi, int n_blocks, cudaStream_t s) {
  const WindowBook bk = {book_first_off, book_n, c_lo, c_hi};
  // no slot to fill, or no connection from a spiking source (di0 out of
  // range): the bookkeeping alone
  if (d.nd <= 0 || v_n <= 0 || di0 < 0 || di0 >= d.nd) {
    k_window_book<<<1, 256, 0, s>>>(d.ring_cnt_w, d.ring_R, d.ring_C, ctx, bk);
    return;
  }
  if (WindowDeliverCap() == 2)
    k_deliver_window<2><<<n_blocks, 256, 0, s>>>(d, ctx, v_lo, v_n, di0, D_lo, D_hi, bk);
  else
    k_deliver_window<3><<<n_blocks, 256, 0, s>>>(d, ctx, v_lo, v_n, di0, D_lo, D_hi, bk);
}

// Resident delivery blocks per SM, at most 3: the delivery runs beside the
// node updates, and a larger grid takes SM slots from them without
// delivering faster (measured on the silent and the 26 Hz scale networks).
int DeliverBlocksPerSM() {
  int nb = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_deliver<false>, 256, 0) != cudaSuccess)
    return 3;
  return nb > 3 ? 3 : (nb > 0 ? nb : 1);
}

// Resident blocks per SM of the static delivery kernel (no cap).
int DeliverOccupancy() {
  int nb = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_deliver<false>, 256, 0) != cudaSuccess)
    return 8;
  return nb > 0 ? nb : 1;
}

// Resident blocks per SM of the window delivery: its grid is resident at
// once, so that its warps go through the items in order together.
int DeliverWindowOccupancy() {
  int nb = 0;
  const cudaError_t e =
      WindowDeliverCap() == 2
          ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_deliver_window<2>, 256, 0)
          : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_deliver_window<3>, 256, 0);
  if (e != cudaSuccess) return WindowDeliverCap();
  return nb > 0 ? nb : 1;
}

void LaunchDeliver(const DeliverArgs &d, const SynGroupTable &syn,
                   StepCtx *ctx, int n_blocks, cudaStream_t s) {
  if (d.nd <= 0) return;
  if (d.e_syn != nullptr) k_deliver<true><<<n_blocks, 256, 0, s>>>(d, syn, ctx);
  else k_deliver<false><<<n_blocks, 256, 0, s>>>(d, syn, ctx);
}

// ---------------------------------------------------------------------------
// STDP post-spike rule: neurons that spiked in this step, over their
// incoming plastic synapses (src/rev_spike.cu:41-75)
// ---------------------------------------------------------------------------
// STDP post rule for one node whose spike reached its dendrites in step T:
// every incoming plastic synapse with a pre-synaptic arrival stamp
// 0 <= T - stamp < 16384 (src/rev_spike.cu:41-55); one warp per node,
// a node is handled once per step.
// One block per node, four incoming edges per thread in flight: the edge
// indices, then the gathers of group, stamp and weight, then the updates.
__device__ __forceinline__ void post_rule_node(const DeliverArgs &d, const SynGroupTable &syn,
                                               unsigned node, long long T) {
  __shared__ int s_first;
  __syncthreads();
  if (threadIdx.x == 0) s_first = (atomicExch(&d.last_post_T[node], (int)T) != (int)T);
  __syncthreads();
  if (!s_first) return;
  const unsigned long long beg = d.rev_off[node], end = d.rev_off[node + 1];
  const unsigned B = blockDim.x;
  for (unsigned long long r0 = beg + threadIdx.x; r0 < end; r0 += 4ull * B) {
    unsigned e[4];
    int sg[4], st[4];
    float w[4];
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const unsigned long long r = r0 + (unsigned long long)u * B;
      if (r < end) e[u] = d.rev_edge[r];
    }
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const unsigned long long r = r0 + (unsigned long long)u * B;
      if (r < end) {
        sg[u] = d.e_syn[e[u]];
        st[u] = d.e_stamp[e[u]];
        w[u] = d.e_w[e[u]];
      }
    }
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const unsigned long long r = r0 + (unsigned long long)u * B;
      if (r < end) {
        const long long Dt_int = T - (long long)st[u];
        if (sg[u] > 0 && Dt_int >= 0 && Dt_int < NGPU_MAX_SYN_DT)
          d.e_w[e[u]] = syn_update(syn, sg[u], w[u], d.dt * (float)Dt_int);
      }
    }
  }
}

// Nodes whose spike reaches their dendrites in this step after a dendritic
// delay: their last post-spike step is set before this step's deliveries
// (src/spike_buffer.cu:299-301 runs before the delivery of the step).
__global__ void k_rev_arrive(DeliverArgs d, StepCtx *ctx) {
  const long long T = ctx->T0 + ctx->it + 1;
  const int slot = (int)(T % d.rev_R);
  int cnt = d.rev_cnt[slot];
  cnt = cnt < d.rev_C ? cnt : d.rev_C;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < cnt; k += gridDim.x * blockDim.x)
    d.last_rev_T[d.rev_src[(long long)slot * d.rev_C + k]] = (int)T;
}

void LaunchRevArrive(const DeliverArgs &d, StepCtx *ctx, cudaStream_t s) {
  k_rev_arrive<<<148, 256, 0, s>>>(d, ctx);
}

__global__ void __launch_bounds__(256)
k_stdp_post(DeliverArgs d, SynGroupTable syn, StepCtx *ctx) {
  const long long T = ctx->T0 + ctx->it + 1;
  const int slot = ctx->ring_slot;
  int cnt = d.ring_cnt[slot];
  cnt = cnt < d.ring_C ? cnt : d.ring_C;
  // one block per node: spikes of this step without dendritic delay
  for (int item = blockIdx.x; item < cnt; item += gridDim.x) {
    const unsigned node = d.ring_src[(long long)slot * d.ring_C + item];
    if (d.last_rev_T[node] != (int)T) continue;   // dendritic delay > 0 (block-uniform)
    post_rule_node(d, syn, node, T);
  }
  // spikes of earlier steps reaching the dendrites now
  if (d.rev_cnt != nullptr) {
    const int rslot = (int)(T % d.rev_R);
    int rcnt = d.rev_cnt[rslot];
    rcnt = rcnt < d.rev_C ? rcnt : d.rev_C;
    for (int item = blockIdx.x; item < rcnt; item += gridDim.x)
      post_rule_node(d, syn, d.rev_src[(long long)rslot * d.rev_C + item], T);
  }
  finish_step(d, ctx, gridDim.x);
}

void LaunchStdpPost(const DeliverArgs &d, const SynGroupTable &syn,
                    StepCtx *ctx, int n_blocks, cudaStream_t s) {
  k_stdp_post<<<n_blocks, 256, 0, s>>>(d, syn, ctx);
}

// ---------------------------------------------------------------------------
// multimeter records and step bookkeeping
// ---------------------------------------------------------------------------
__global__ void k_record(const RecCol *cols, int n_cols, float *buf,
                         long long cap_rows, const int *last_spike_T,
                         const float *last_spike_h, int initial, float dt,
                         StepCtx *ctx) {
  const long long row = ctx->rec_row;
  if (row >= cap_rows) {
    if (blockIdx.x == 0 && threadIdx.x == 0)
      atomicOr(&ctx->err, (unsigned)DERR_REC_OVERFLOW);
    return;
  }
  const long long it = ctx->it;
  const long long T = ctx->T0 + it + 1;
  float *r = buf + row * (n_cols + 1);
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c == 0) {
    double t = initial ? ctx->t0 : ctx->t0 + (double)dt * (double)(it + 1);
    r[0] = (float)t;
  }
  if (c < n_cols) {
    RecCol col = cols[c];
    float v;
    if (col.spike) {
      v = (!initial && col.has_out && last_spike_T[col.node] == (int)T)
              ? last_spike_h[col.node] : 0.0f;
    } else {
      v = *col.ptr;
    }
    r[1 + c] = v;
  }
}

void LaunchRecord(const RecCol *cols, int n_cols, float *buf, long long cap_rows,
                  const int *last_spike_T, const float *last_spike_h,
                  int initial, float dt, StepCtx *ctx, cudaStream_t s) {
  int nb = (n_cols + 1 + 255) / 256;
  k_record<<<nb, 256, 0, s>>>(cols, n_cols, buf, cap_rows, last_spike_T,
                              last_spike_h, initial, dt, ctx);
}

// bit 0: the step bookkeeping of a network without delivery (see
// step_bookkeeping); bit 1: advance the recording row of the context
__global__ void k_advance(int *ring_cnt, int ring_R, int ring_C, int flags,
                          StepCtx *ctx) {
  if (flags & 1) step_bookkeeping(ring_cnt, ring_R, ring_C, ctx);
  if (flags & 2) ctx->rec_row += 1;
}

// Per-step copies of the step context for a chunk of n steps: step k of the
// chunk reads copy k (its step index, recording row, pending Poisson draws),
// so no kernel has to advance a shared context between the steps of a chunk
// and each step needs no bookkeeping launch of its own.
__global__ void k_step_prologue(const StepCtx *base, StepCtx *copies, int n, int rec) {
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    StepCtx c = *base;
    c.it = base->it + k;
    if (k > 0) c.poisson_pending = 1;
    c.rec_row = base->rec_row + (rec ? k : 0);
    c.err = 0u;
    c.n_spikes = 0ull;
    ctx_set_slots(c);
    copies[k] = c;
  }
}

// Folds the chunk's per-step contexts back into the base context: step
// index, pending draws, recording row, error bits and spike count.
__global__ void k_step_epilogue(StepCtx *base, const StepCtx *copies, int n, int rec) {
  __shared__ unsigned long long s_sp[256];
  __shared__ unsigned s_err[256];
  unsigned long long sp = 0;
  unsigned err = 0;
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    sp += copies[k].n_spikes;
    err |= copies[k].err;
  }
  s_sp[threadIdx.x] = sp;
  s_err[threadIdx.x] = err;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int j = 1; j < (int)blockDim.x; j++) {
      sp += s_sp[j];
      err |= s_err[j];
    }
    base->n_spikes += sp;
    base->err |= err;
    base->it += n;
    ctx_set_slots(*base);
    if (n > 0) base->poisson_pending = 1;
    if (rec) base->rec_row += n;
  }
}

void LaunchStepPrologue(const StepCtx *base, StepCtx *copies, int n, int rec, cudaStream_t s) {
  k_step_prologue<<<1, 256, 0, s>>>(base, copies, n, rec);
}

void LaunchStepEpilogue(StepCtx *base, const StepCtx *copies, int n, int rec, cudaStream_t s) {
  k_step_epilogue<<<1, 256, 0, s>>>(base, copies, n, rec);
}

void LaunchAdvance(int *ring_cnt, int ring_R, int ring_C, int flags,
                   StepCtx *ctx, cudaStream_t s) {
  k_advance<<<1, 1, 0, s>>>(ring_cnt, ring_R, ring_C, flags, ctx);
}

// ---------------------------------------------------------------------------
// calibration kernels
// ---------------------------------------------------------------------------
// beta-function conductance normalisation (src/aeif_cond_beta.cu:58-87)
__global__ void k_calib_beta(int n, int n_pad, float *param, int np,
                             int nsp, int npp, int col_rise, int col_decay,
                             int col_g0, int col_refr) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  param[(long long)col_refr * n_pad + i] = 0.0f;
  for (int q = 0; q < np; q++) {
    float tr = param[(long long)(nsp + npp * q + col_rise) * n_pad + i];
    float td = param[(long long)(nsp + npp * q + col_decay) * n_pad + i];
    float denom1 = td - tr;
    float denom2 = 0.0f;
    if (denom1 != 0.0f) {
      float t_p = td * tr * logf(td / tr) / denom1;
      denom2 = expf(-t_p / td) - expf(-t_p / tr);
    }
    float g0;
    if (denom2 == 0.0f) {
      g0 = (float)(M_E / (double)td);
    } else {
      g0 = (float)((1.0 / (double)tr - 1.0 / (double)td) / (double)denom2);
    }
    param[(long long)(nsp + npp * q + col_g0) * n_pad + i] = g0;
  }
}

// alpha-function normalisation e/tau (src/aeif_cond_alpha.cu:63-68)
__global__ void k_calib_alpha(int n, int n_pad, float *param, int np, int nsp,
                              int npp, int col_tau, int col_out, int col_refr) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  param[(long long)col_refr * n_pad + i] = 0.0f;
  for (int q = 0; q < np; q++) {
    float tau = param[(long long)(nsp + npp * q + col_tau) * n_pad + i];
    param[(long long)(nsp + npp * q + col_out) * n_pad + i] =
        (float)(M_E / (double)tau);
  }
}

__global__ void k_calib_refr(int n, int n_pad, float *param, int col_refr) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  param[(long long)col_refr * n_pad + i] = 0.0f;
}

void LaunchCalibrateRk5(int model, const GroupArgs &g, int np,
                        cudaStream_t s) {
  if (g.n <= 0) return;
  int nb = (g.n + NGPU_BLOCK - 1) / NGPU_BLOCK;
  switch (model) {
    case RK5_AEIF_COND_BETA:
      k_calib_beta<<<nb, NGPU_BLOCK, 0, s>>>(g.n, g.n_pad, g.param, np, A_NSP,
                                             4, 1, 2, 3, A_refr);
      break;
    case RK5_IZHIKEVICH_COND_BETA:
      k_calib_beta<<<nb, NGPU_BLOCK, 0, s>>>(g.n, g.n_pad, g.param, np, I_NSP,
                                             4, 1, 2, 3, I_refr);
      break;
    case RK5_AEIF_COND_ALPHA:
      k_calib_alpha<<<nb, NGPU_BLOCK, 0, s>>>(g.n, g.n_pad, g.param, np, A_NSP,
                                              3, 1, 2, A_refr);
      break;
    case RK5_AEIF_PSC_ALPHA:
      k_calib_alpha<<<nb, NGPU_BLOCK, 0, s>>>(g.n, g.n_pad, g.param, np, A_NSP,
                                              2, 0, 1, A_refr);
      break;
    default:
      k_calib_refr<<<nb, NGPU_BLOCK, 0, s>>>(g.n, g.n_pad, g.param, A_refr);
  }
}

// exact-integration propagators (src/iaf_psc_exp.cu:53-91)
__device__ double propagator_32(double tau_syn, double tau, double C,
                                double h) {
  const double P32_linear = 1.0 / (2.0 * C * tau * tau) * h * h
                            * (tau_syn - tau) * exp(-h / tau);
  const double P32_singular = h / C * exp(-h / tau);
  const double P32 = -tau / (C * (1.0 - tau / tau_syn)) * exp(-h / tau_syn)
                     * expm1(h * (1.0 / tau_syn - 1.0 / tau));
  const double dev_P32 = fabs(P32 - P32_singular);
  if (tau == tau_syn ||
      (fabs(tau - tau_syn) < 0.1 && dev_P32 > 2.0 * fabs(P32_linear))) {
    return P32_singular;
  }
  return P32;
}

__global__ void k_calib_iaf(int n, int n_pad, float *param, float h) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float *col = param + i;
  const long long P = n_pad;
  float tau_m = col[0 * P], C_m = col[1 * P];
  float tau_ex = col[6 * P], tau_in = col[7 * P];
  float P22 = expf(-h / tau_m);
  col[11 * P] = expf(-h / tau_ex);
  col[12 * P] = expf(-h / tau_in);
  col[15 * P] = P22;
  col[13 * P] = (float)propagator_32(tau_ex, tau_m, C_m, h);
  col[14 * P] = (float)propagator_32(tau_in, tau_m, C_m, h);
  col[10 * P] = (float)((double)(tau_m / C_m) * (1.0 - (double)P22));
}

void LaunchCalibrateIaf(const GroupArgs &g, float h, cudaStream_t s) {
  if (g.n <= 0) return;
  k_calib_iaf<<<(g.n + NGPU_BLOCK - 1) / NGPU_BLOCK, NGPU_BLOCK, 0, s>>>(
      g.n, g.n_pad, g.param, h);
}

// ---------------------------------------------------------------------------
// parameter / variable access helpers
// ---------------------------------------------------------------------------
__global__ void k_fill_float(float *p, long long n, float v) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  for (; i < n; i += (long long)gridDim.x * blockDim.x) p[i] = v;
}
__global__ void k_fill_int(int *p, long long n, int v) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  for (; i < n; i += (long long)gridDim.x * blockDim.x) p[i] = v;
}
__global__ void k_scatter_float(float *col, const int *idx, int n, float v,
                                const float *vals, int stride) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  col[idx[k]] = vals ? vals[(long long)k * stride] : v;
}
__global__ void k_gather_float(const float *col, const int *idx, int n,
                               float *out, int stride) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  out[(long long)k * stride] = col[idx[k]];
}

static int grid_for(long long n) {
  long long b = (n + 255) / 256;
  if (b > 148 * 32) b = 148 * 32;
  if (b < 1) b = 1;
  return (int)b;
}

void LaunchFillFloat(float *p, long long n, float v, cudaStream_t s) {
  if (n <= 0) return;
  k_fill_float<<<grid_for(n), 256, 0, s>>>(p, n, v);
}
void LaunchFillInt(int *p, long long n, int v, cudaStream_t s) {
  if (n <= 0) return;
  k_fill_int<<<grid_for(n), 256, 0, s>>>(p, n, v);
}
void LaunchScatterFloat(float *col, const int *idx, int n, float v,
                        const float *vals, int vals_stride, cudaStream_t s) {
  if (n <= 0) return;
  k_scatter_float<<<(n + 255) / 256, 256, 0, s>>>(col, idx, n, v, vals,
                                                  vals_stride);
}
void LaunchGatherFloat(const float *col, const int *idx, int n, float *out,
                       int out_stride, cudaStream_t s) {
  if (n <= 0) return;
  k_gather_float<<<(n + 255) / 256, 256, 0, s>>>(col, idx, n, out, out_stride);
}

}  // namespace ngpu
