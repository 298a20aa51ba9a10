// Synaptic delivery (the reference's SpikeBufferUpdate / NestedLoop /
// NestedLoopFunction0, src/spike_buffer.cu:233-302, src/nested_loop.cu:39-167,
// src/get_spike.cu:48-85) and the synapse-model updates of the STDP rules.
// Included by ngpu_kernels.cu (the delivery and STDP kernels) and by the RK5
// launch header (delivery blocks fused into the update grid).
#pragma once
#include "ngpu_kernels_common.cuh"

namespace ngpu {

// ---------------------------------------------------------------------------
// synapse models (src/stdp.cu:24-51, src/test_syn_model.cu:24-30)
// ---------------------------------------------------------------------------
// x^mu; the exponents of additive (0) and multiplicative (1) STDP, the
// common settings, need no pow (pow(x, 0) is 1 and pow(x, 1) is x exactly)
__device__ __forceinline__ double pow_mu(double x, double mu) {
  if (mu == 0.0) return 1.0;
  if (mu == 1.0) return x;
  return pow(x, mu);
}

__device__ __forceinline__ float syn_update(const SynGroupTable &syn, int sg,
                                            float w, float Dt) {
  int type = syn.type[sg - 1];
  const float *prm = syn.param[sg - 1];
  if (type == 2) {
    double tau_plus = prm[0], tau_minus = prm[1], lambda = prm[2];
    double alpha = prm[3], mu_plus = prm[4], mu_minus = prm[5];
    double Wmax = prm[6];
    double w0 = w, w1;
    if (Dt >= 0.0f) {
      double fact = lambda * exp(-(double)Dt / tau_plus);
      w1 = w0 + fact * Wmax * pow_mu(1.0 - w0 / Wmax, mu_plus);
    } else {
      double fact = -alpha * lambda * exp((double)Dt / tau_minus);
      w1 = w0 + fact * Wmax * pow_mu(w0 / Wmax, mu_minus);
    }
    w1 = w1 > 0.0 ? w1 : 0.0;
    w1 = w1 < Wmax ? w1 : Wmax;
    return (float)w1;
  } else if (type == 1) {
    return w + (prm[1] + prm[0] * Dt);
  }
  return w;
}

// End-of-step work of plastic networks, fused into the step's last kernel:
// the last block to finish empties this step's dendritic-delay slot, which
// every block of the post rule has read by then. (The step index itself
// never changes during a chunk of steps: each step reads its own copy of the
// step context, see k_step_prologue.)
__device__ __forceinline__ void finish_step(const DeliverArgs &d, StepCtx *ctx, int nblk) {
  if (d.advance_flags == 0) return;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    unsigned prev = atomicAdd(d.done, 1u);
    if (prev == (unsigned)nblk - 1) {
      __threadfence();
      if ((d.advance_flags & 1) && d.rev_cnt != nullptr) {
        const long long T = ctx->T0 + ctx->it + 1;
        d.rev_cnt[(int)(T % d.rev_R)] = 0;
      }
      *d.done = 0u;
      __threadfence();
    }
  }
}

// Spike count of step T - 1 (complete: every kernel of that step has ended)
// and the emptying of the ring slot that step T + 1 fills. Called once per
// step, by the step's delivery or by k_advance; the slot of T + 1 is never
// read in step T (deliveries read T - 1 ... T - max delay of a ring with
// max delay + 2 slots).
__device__ __forceinline__ void step_bookkeeping(int *ring_cnt, int ring_R, int ring_C,
                                                 StepCtx *ctx) {
  const int s = ctx->ring_slot;                 // slot of step T
  const int c = ring_cnt[s > 0 ? s - 1 : ring_R - 1];
  ctx->n_spikes += (unsigned long long)(c < ring_C ? c : ring_C);
  ring_cnt[s + 1 < ring_R ? s + 1 : 0] = 0;
}

// ---------------------------------------------------------------------------
// synaptic delivery: one warp per (spike, delay) group. PLASTIC: the
// network has plastic synapses (the STDP pre rule runs on every edge); the
// static instance does not carry that path's registers.
// ---------------------------------------------------------------------------
// Edges beg..end of one (spike, delay) group without plasticity, delivered
// by a whole warp into the accumulators acc: eight edges per lane in flight;
// edges are read once per spike, so they are loaded with the streaming
// (evict-first) hint.
__device__ __forceinline__ void deliver_static_edges(const DeliverArgs &d, long long *acc,
                                                     unsigned long long beg,
                                                     unsigned long long end, float height,
                                                     int lane) {
  for (unsigned long long e0 = beg + lane; e0 < end; e0 += 256) {
    unsigned sl[8];
    float wv[8];
#pragma unroll
    for (int u = 0; u < 8; u++) {
      const unsigned long long e = e0 + 32 * u;
      if (e < end) {
        sl[u] = __ldcs(d.e_slot + e);
        wv[u] = __ldcs(d.e_w + e);
      }
    }
#pragma unroll
    for (int u = 0; u < 8; u++) {
      const unsigned long long e = e0 + 32 * u;
      if (e < end) {
        atomicAdd((unsigned long long *)(acc + sl[u]),
                  (unsigned long long)ng_to_fixed(height * wv[u]));
      }
    }
  }
}

// Delivery work of block blk of nblk delivery blocks (any block size that
// is a multiple of 32, at most 256 threads): the whole grid of k_deliver, or
// the first blocks of a fused RK5 update (k_rk5_update_deliver).
template <bool PLASTIC>
__device__ __forceinline__ void deliver_blocks(const DeliverArgs &d, const SynGroupTable &syn,
                                               StepCtx *ctx, int blk, int nblk) {
  const long long T = ctx->T0 + ctx->it + 1;
  // the slot the update of T + 1 folds, and the ring slot of step T
  const int out_slot = ctx->acc_out_slot;
  const int ring_T = ctx->ring_slot;
  long long *const acc = d.acc + acc_slot_offset(out_slot, d.acc_slots, d.acc_par);
  long long *const stamp =
      d.acc_stamp != nullptr ? d.acc_stamp + (d.acc_slots > 1 ? out_slot : 0) : nullptr;
  if (d.step_book && blk == 0 && threadIdx.x == 0)
    step_bookkeeping(d.ring_cnt_w, d.ring_R, d.ring_C, ctx);
  const int lane = threadIdx.x & 31;
  const int warp = (blk * (int)blockDim.x + (int)threadIdx.x) >> 5;
  const int n_warps = (nblk * (int)blockDim.x) >> 5;
  const bool warp_scan = d.nd <= 32;
  unsigned long long events = 0;
  // the edges of one (spike, delay) item: spike j of ring slot `slot` at
  // distinct-delay index di; called by whole warps
  auto deliver_item = [&](int di, unsigned src, float height) {
    const unsigned long long gi = (unsigned long long)src * d.nd + di;
    const unsigned long long beg = d.grp_off[gi], end = d.grp_off[gi + 1];
    if (lane == 0) events += end - beg;
    if constexpr (!PLASTIC) {
      deliver_static_edges(d, acc, beg, end, height, lane);
    } else {
      // plastic network: four edges per lane in flight, then the
      // post-synaptic last-spike gathers of all four, then the updates
      for (unsigned long long e0 = beg + lane; e0 < end; e0 += 128) {
        unsigned sl[4], post[4];
        float wv[4];
        int sgv[4], lr[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
          const unsigned long long e = e0 + 32 * u;
          if (e < end) {
            sl[u] = d.e_slot[e];
            wv[u] = d.e_w[e];
            sgv[u] = d.e_syn[e];
            post[u] = sgv[u] > 0 ? d.e_post[e] : 0u;
          }
        }
#pragma unroll
        for (int u = 0; u < 4; u++) {
          const unsigned long long e = e0 + 32 * u;
          if (e < end && sgv[u] > 0) lr[u] = d.last_rev_T[post[u]];
        }
#pragma unroll
        for (int u = 0; u < 4; u++) {
          const unsigned long long e = e0 + 32 * u;
          if (e < end) {
            atomicAdd((unsigned long long *)(acc + sl[u]),
                      (unsigned long long)ng_to_fixed(height * wv[u]));
            if (sgv[u] > 0) {
              // pre-spike rule with the last post spike (src/get_spike.cu:73-83)
              d.e_stamp[e] = (int)T;
              const long long Dt_int = T - (long long)lr[u];
              if (Dt_int > 0 && Dt_int < NGPU_MAX_SYN_DT) {
                d.e_w[e] = syn_update(syn, sgv[u], wv[u], -d.dt * (float)Dt_int);
              }
            }
          }
        }
      }
    }
  };
  if (warp_scan) {
    // per-delay spike counts and their prefix in registers of every warp
    int my_slot = 0, my_incl = 0, total;
    int c = 0;
    if (lane < d.nd) {
      int slot = ring_T - d.delays[lane];       // delays are below ring_R
      if (slot < 0) slot += d.ring_R;
      my_slot = slot;
      c = d.ring_cnt[slot];
      c = c < d.ring_C ? c : d.ring_C;
    }
    my_incl = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int v = __shfl_up_sync(0xffffffffu, my_incl, o);
      if (lane >= o) my_incl += v;
    }
    total = __shfl_sync(0xffffffffu, my_incl, 31);
    // the slot may receive input this step: one store (see acc_stamp; a
    // store per item, all to one word, held the grid's end for the L2 to
    // serialise them)
    if (warp == 0 && lane == 0 && total > 0 && stamp != nullptr) *stamp = T;
    for (int item = warp; item < total; item += n_warps) {
      // first delay whose inclusive prefix exceeds the item
      // (item < total, so some lane's inclusive prefix exceeds it)
      const unsigned m = __ballot_sync(0xffffffffu, my_incl > item);
      const int di = __ffs(m) - 1;
      const int slot = __shfl_sync(0xffffffffu, my_slot, di);
      const int prev = __shfl_sync(0xffffffffu, my_incl, di > 0 ? di - 1 : 0);
      const long long k = (long long)slot * d.ring_C + (item - (di > 0 ? prev : 0));
      deliver_item(di, d.ring_src[k], d.ring_h[k]);
    }
  } else {
    // more than 32 distinct delays: every delay has a fixed set of G warps,
    // which read its spike count themselves and take its spikes in turn (no
    // prefix over the delays, no search); with fewer warps than delays each
    // warp takes every n_warps-th delay
    const bool per_delay = n_warps >= d.nd;
    const int G = per_delay ? n_warps / d.nd : 1;
    if (!per_delay || warp < G * d.nd) {
      for (int di = per_delay ? warp % d.nd : warp; di < d.nd; di += per_delay ? d.nd : n_warps) {
        int slot = ring_T - d.delays[di];
        if (slot < 0) slot += d.ring_R;
        // the warp's first ring entry is loaded together with the slot's
        // spike count, not after it (one dependent load less per item; an
        // entry past the count is within the slot and is not used)
        const int j0 = per_delay ? warp / d.nd : 0;
        const long long k0 = (long long)slot * d.ring_C + j0;
        unsigned src0 = 0u;
        float h0 = 0.0f;
        if (j0 < d.ring_C) {
          src0 = d.ring_src[k0];
          h0 = d.ring_h[k0];
        }
        int c = d.ring_cnt[slot];
        c = c < d.ring_C ? c : d.ring_C;
        // one stamp store per delay with spikes (the delay's first warp)
        if (j0 == 0 && c > 0 && lane == 0 && stamp != nullptr) *stamp = T;
        if (j0 < c) deliver_item(di, src0, h0);
        for (int j = j0 + G; j < c; j += G) {
          const long long k = (long long)slot * d.ring_C + j;
          deliver_item(di, d.ring_src[k], d.ring_h[k]);
        }
      }
    }
  }
  if (d.blk_events != nullptr) {
    // per warp, a reduction whose result is not waited for (see block_add_u64)
    for (int o = 16; o > 0; o >>= 1) events += __shfl_down_sync(0xffffffffu, events, o);
    if (lane == 0 && events != 0) atomicAdd(d.blk_events + blk, events);
  }
  finish_step(d, ctx, nblk);
}

// Delivery before a window of integrated steps (networks without plastic
// synapses, k_rk5_window): the accumulator slots of the steps
// T_b + v_lo ... T_b + v_lo + v_n - 1 (T_b: the step of ctx, the window's
// first step) receive every spike that arrives in them, at each delay D of
// a spiking source (d.delays[di0 ...]): the spikes of step v - D, all
// emitted before the window since a window is no longer than the shortest
// such delay + 1 steps. The slot of step v is the one the update of step
// v + 1 folds, filled as the one-step delivery of step v fills it, so each
// slot gets all its input in one launch, where a delivery of the window's
// own spikes at all their delays would add into every slot once per delay,
// each time from HBM.
//
// The items (slot, delay, spike) are ordered by slot, then delay, and warp
// w takes the items w, w + n_warps, w + 2 n_warps, ...: the warps go
// through the order together, so one or two slots are written at a time
// and stay in L2. The (slot, delay) pairs are taken 32 at a time, a lane
// each, and a scan of their spike counts gives every pair's first item, so
// a warp finds its own items without looking at the others'. A warp's
// items are software-pipelined: an item's spike entry and edge range load
// while the previous item's edges are in flight.
__device__ __forceinline__ void deliver_window_blocks(const DeliverArgs &d, const StepCtx *ctx,
                                                      int v_lo, int v_n, int di0, int D_lo,
                                                      int D_hi, int blk, int nblk) {
  const unsigned full = 0xffffffffu;
  const long long T_b = ctx->T0 + ctx->it + 1;
  const int ring_b = ctx->ring_slot, acc_b = ctx->acc_out_slot;
  const int lane = threadIdx.x & 31;
  const int warp = (blk * (int)blockDim.x + (int)threadIdx.x) >> 5;
  const int n_warps = (nblk * (int)blockDim.x) >> 5;
  const int nd_s = d.nd - di0;                 // delays of spiking sources
  const int P = v_n * nd_s;
  // the delays in registers (lane i: delay di0 + i), where they fit
  const int my_delay = (lane < nd_s) ? d.delays[di0 + lane] : 0;
  // a quiet window: no spike in the emission steps T_b + v_lo - D_hi ...
  // T_b + v_lo + v_n - 1 - D_lo, one round of independent loads
  {
    const int span = (v_n - 1) + (D_hi - D_lo) + 1;
    int any = 0;
    for (int i = lane; i < span; i += 32) {
      const long long rel_s = (long long)v_lo - D_hi + i;
      if (T_b + rel_s >= 0) any |= d.ring_cnt[ring_add(ring_b, rel_s, d.ring_R)];
    }
    if (!__any_sync(full, any != 0)) return;
  }
  // the round (32 pairs, a lane each): pair values, this warp's first item
  // of each pair (r_j), the lanes with items left (m)
  int p0 = -32, base = 0, total = 0;
  int r_v = 0, r_di = 0, r_c = 0, r_j = 0, r_slot = 0;
  unsigned m = 0u;
  // the current pair's items: jj, jj + n_warps, ... below cl
  bool in_pair = false;
  int jj = 0, cl = 0, dil = 0, slot_l = 0, v_slot = 0;
  // the previous item, its edge range loaded
  bool has_prev = false;
  unsigned long long pbeg = 0, pend = 0;
  float ph = 0.0f;
  long long *pacc = nullptr;
  unsigned long long events = 0;
  while (true) {
    // the next item of this warp in the order (warp-uniform control flow)
    bool got = false;
    if (in_pair) {
      jj += n_warps;
      got = jj < cl;
      in_pair = got;
    }
    while (!got) {
      if (m == 0u) {
        if (p0 >= 0) base = (base + total) % n_warps;
        p0 += 32;
        if (p0 >= P) break;
        const int p = p0 + lane;
        r_v = p / nd_s;
        r_di = di0 + (p - r_v * nd_s);
        r_c = 0;
        r_slot = 0;
        const int D = __shfl_sync(full, my_delay, (r_di - di0) & 31);
        if (p < P) {
          // emission step
          const long long rel_s = (long long)v_lo + r_v - (nd_s <= 32 ? D : d.delays[r_di]);
          if (T_b + rel_s >= 0) {
            r_slot = ring_add(ring_b, rel_s, d.ring_R);
            const int c = d.ring_cnt[r_slot];
            r_c = c < d.ring_C ? c : d.ring_C;
          }
        }
        int incl = r_c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int v = __shfl_up_sync(full, incl, o);
          if (lane >= o) incl += v;
        }
        total = __shfl_sync(full, incl, 31);
        // item j of the pair is item base + (incl - r_c) + j of the order
        r_j = warp - (base + incl - r_c) % n_warps;
        if (r_j < 0) r_j += n_warps;
        m = __ballot_sync(full, r_j < r_c);
        continue;
      }
      const int l = __ffs(m) - 1;
      m &= m - 1;
      jj = __shfl_sync(full, r_j, l);
      cl = __shfl_sync(full, r_c, l);
      dil = __shfl_sync(full, r_di, l);
      slot_l = __shfl_sync(full, r_slot, l);
      const long long rv = (long long)v_lo + __shfl_sync(full, r_v, l);
      v_slot = ring_add(acc_b, rv, d.acc_slots);
      // one stamp store per (slot, delay) pair with spikes: by the warp of its first item
      if (jj == 0 && lane == 0 && d.acc_stamp != nullptr) d.acc_stamp[v_slot] = T_b + rv;
      in_pair = true;
      got = true;
    }
    if (!got) break;
    // this item's spike entry
    const long long kk = (long long)slot_l * d.ring_C + jj;
    const unsigned src = d.ring_src[kk];
    const float height = d.ring_h[kk];
    // the previous item's first 256 edges, loaded before this item's edge range
    unsigned sl[8];
    float wv[8];
    const int n_mine = has_prev ? (int)(pend - pbeg < 256ull ? pend - pbeg : 256ull) - lane : 0;
    {
      const unsigned *ps = d.e_slot + pbeg + lane;
      const float *pw = d.e_w + pbeg + lane;
#pragma unroll
      for (int u = 0; u < 8; u++) {
        if (32 * u < n_mine) {
          sl[u] = __ldcs(ps + 32 * u);
          wv[u] = __ldcs(pw + 32 * u);
        }
      }
    }
    const unsigned long long e_i = (unsigned long long)src * d.nd + dil;
    const unsigned long long beg = d.grp_off[e_i], end = d.grp_off[e_i + 1];
#pragma unroll
    for (int u = 0; u < 8; u++) {
      if (32 * u < n_mine)
        atomicAdd((unsigned long long *)(pacc + sl[u]),
                  (unsigned long long)ng_to_fixed(ph * wv[u]));
    }
    if (has_prev && pend > pbeg + 256) deliver_static_edges(d, pacc, pbeg + 256, pend, ph, lane);
    if (lane == 0) events += end - beg;
    pbeg = beg;
    pend = end;
    ph = height;
    pacc = d.acc + acc_slot_offset(v_slot, d.acc_slots, d.acc_par);
    has_prev = true;
  }
  if (has_prev) deliver_static_edges(d, pacc, pbeg, pend, ph, lane);
  if (d.blk_events != nullptr) {
    // per warp, a reduction whose result is not waited for (see block_add_u64)
    for (int o = 16; o > 0; o >>= 1) events += __shfl_down_sync(full, events, o);
    if (lane == 0 && events != 0) atomicAdd(d.blk_events + blk, events);
  }
}

}  // namespace ngpu
