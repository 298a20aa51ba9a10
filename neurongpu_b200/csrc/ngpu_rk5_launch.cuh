// Launchers of the single-group RK5 update kernels (plain controller
// variants chosen by the autotuner, step logging, learned proposer) and the
// straggler finishing launch. Included by one translation unit per model
// family (ngpu_rk5_<model>.cu), so that their template instances compile in
// parallel.
#pragma once
#include <type_traits>

#include "ngpu_kernels_common.cuh"
#include "ngpu_deliver.cuh"

namespace ngpu {

// The RK5 update of one group with the step's synaptic delivery in the same
// grid (networks without plastic synapses): blocks 0 .. n_del - 1 deliver
// (the work of k_deliver's grid), the others integrate the neurons. The
// delivery of step T reads spikes of earlier steps and adds into the
// accumulator half that the update of T + 1 folds, while the update of T
// folds the other half and writes ring slot T: disjoint data, so the two
// run side by side without a second stream, and the next step's update,
// launched with programmatic stream serialization, may be scheduled while
// this grid's last wave runs (one launch per step instead of a fork, a
// delivery launch and a join). The delivery blocks come first so that they
// are scheduled in the first wave.
template <class M, int NP, int MINB>
__global__ void __launch_bounds__(NGPU_BLOCK, MINB)
k_rk5_update_deliver(const __grid_constant__ GroupArgs g, const __grid_constant__ InputArgs in,
                     const __grid_constant__ PushArgs pa, StepCtx *ctx,
                     const __grid_constant__ DeliverArgs d, int n_del) {
  pdl_wait();
  pdl_trigger();
  if ((int)blockIdx.x < n_del) {
    __shared__ SynGroupTable no_syn;          // static synapses only: never read
    deliver_blocks<false>(d, no_syn, ctx, blockIdx.x, n_del);
    return;
  }
  const int blk = (int)blockIdx.x - n_del;
  const int i = blk * NGPU_BLOCK + threadIdx.x;
  unsigned evals = 0;
  const bool queued = g.q.cap > 0;
  if (i < g.n) rk5_neuron<M, NP, true, STEP_PLAIN>(g, in, pa, ctx, i, g.puni, g.pinv, evals, false,
                                                   queued ? &g.q : nullptr, 0);
  if (g.blk_evals != nullptr) block_add_u64(evals, g.blk_evals, blk);
}

// grid of the persistent tile kernel: as many blocks as are resident at once
// (at most one per tile)
template <class M, int NP, int MINB>
static int tile_grid(int n_tiles) {
  static int resident = 0;
  if (resident == 0) {
    int dev = 0, n_sm = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_rk5_update_tiles<M, NP, MINB>,
                                                  NGPU_BLOCK, 0);
    resident = (n_sm > 0 ? n_sm : 148) * (per_sm > 0 ? per_sm : 1);
  }
  return n_tiles < resident ? n_tiles : resident;
}

// The tile kernel's bulk copies need 16-byte aligned column and accumulator
// starts (cudaMalloc bases, columns of n_pad = a multiple of 128 entries).
static bool tiles_aligned(const GroupArgs &g, const InputArgs &in) {
  auto al = [](const void *p) { return ((uintptr_t)p & 15u) == 0; };
  return al(g.var) && al(g.param) && al(g.h) && al(g.dx) && al(in.acc + in.acc_base) &&
         ((in.acc_par * sizeof(long long)) & 15u) == 0 && (g.n_pad % NGPU_BLOCK) == 0;
}

template <class M, int NP>
static bool launch_rk5(const GroupArgs &g, const InputArgs &in, const PushArgs &pa,
                       StepCtx *ctx, cudaStream_t s, const DeliverArgs *del = nullptr,
                       int n_del = 0) {
  dim3 grid((g.n + NGPU_BLOCK - 1) / NGPU_BLOCK), block(NGPU_BLOCK);
  constexpr bool kProposer = ProposerFeatures<M>::supported && NP <= 2;
  if (g.step_mode == STEP_LOG) {
    // step logging: conductance AdEx, <= 2 ports
    if constexpr (kProposer) {
      if (g.all_uniform) k_rk5_update<M, NP, true, 1, STEP_LOG><<<grid, block, 0, s>>>(g, in, pa, ctx);
      else k_rk5_update<M, NP, false, 1, STEP_LOG><<<grid, block, 0, s>>>(g, in, pa, ctx);
    }
    return false;
  }
  // the learned proposer: the plain update of the chosen variant with the
  // straggler queue, the proposer in the queue's finishing launch
  const bool learned = g.step_mode == STEP_LEARNED;
  if (learned && !kProposer) return false;
  auto finish = [&](auto uni) {
    constexpr bool U = decltype(uni)::value;
    if (g.q.cap <= 0) return;
    if (learned) {
      if constexpr (kProposer) {
        const SegArgs *no_segs = nullptr;
        launch_pdl(k_rk5_finish_learned<M, NP, U, false>, dim3(g.q.fin_blocks), block, s, g, pa,
                   in.np, no_segs, g.blk_evals, g.dry, ctx, g.q);
      }
    } else {
      launch_pdl(k_rk5_finish<M, NP, U>, dim3(g.q.fin_blocks), block, s, g, in, pa, ctx);
    }
  };
  if (g.all_uniform) {
    if constexpr (NP <= 4) {
      // occupancy variants chosen by the autotuner (register cap per thread)
      const bool tile_v = g.variant == 4 || g.variant == 5 || g.variant == 7 || g.variant == 8;
      const int variant = (tile_v && !tiles_aligned(g, in)) ? 1 : g.variant;
      const int n_tiles = (int)grid.x;
      if (del != nullptr && Rk5FusesDelivery(variant)) {
        const dim3 fgrid(grid.x + n_del);
        switch (variant) {
          case 1: launch_pdl(k_rk5_update_deliver<M, NP, 5>, fgrid, block, s, g, in, pa, ctx, *del, n_del); break;
          case 2: launch_pdl(k_rk5_update_deliver<M, NP, 6>, fgrid, block, s, g, in, pa, ctx, *del, n_del); break;
          case 3: launch_pdl(k_rk5_update_deliver<M, NP, 8>, fgrid, block, s, g, in, pa, ctx, *del, n_del); break;
          case 6: launch_pdl(k_rk5_update_deliver<M, NP, 4>, fgrid, block, s, g, in, pa, ctx, *del, n_del); break;
          default: launch_pdl(k_rk5_update_deliver<M, NP, 1>, fgrid, block, s, g, in, pa, ctx, *del, n_del); break;
        }
        finish(std::true_type());
        return true;
      }
      switch (variant) {
        case 1: launch_pdl(k_rk5_update<M, NP, true, 5, STEP_PLAIN>, grid, block, s, g, in, pa, ctx); break;
        case 2: launch_pdl(k_rk5_update<M, NP, true, 6, STEP_PLAIN>, grid, block, s, g, in, pa, ctx); break;
        case 3: launch_pdl(k_rk5_update<M, NP, true, 8, STEP_PLAIN>, grid, block, s, g, in, pa, ctx); break;
        case 4:
          launch_pdl(k_rk5_update_tiles<M, NP, 5>, dim3(tile_grid<M, NP, 5>(n_tiles)), block, s, g, in, pa, ctx);
          break;
        case 5:
          launch_pdl(k_rk5_update_tiles<M, NP, 6>, dim3(tile_grid<M, NP, 6>(n_tiles)), block, s, g, in, pa, ctx);
          break;
        case 6: launch_pdl(k_rk5_update<M, NP, true, 4, STEP_PLAIN>, grid, block, s, g, in, pa, ctx); break;
        case 7:
          launch_pdl(k_rk5_update_tiles<M, NP, 4>, dim3(tile_grid<M, NP, 4>(n_tiles)), block, s, g, in, pa, ctx);
          break;
        case 8:
          launch_pdl(k_rk5_update_tiles<M, NP, 3>, dim3(tile_grid<M, NP, 3>(n_tiles)), block, s, g, in, pa, ctx);
          break;
        default: launch_pdl(k_rk5_update<M, NP, true, 1, STEP_PLAIN>, grid, block, s, g, in, pa, ctx); break;
      }
    } else {
      launch_pdl(k_rk5_update<M, NP, true, 1, STEP_PLAIN>, grid, block, s, g, in, pa, ctx);
    }
    finish(std::true_type());
  } else {
    launch_pdl(k_rk5_update<M, NP, false, 1, STEP_PLAIN>, grid, block, s, g, in, pa, ctx);
    finish(std::false_type());
  }
  return false;
}

// The window kernel (several steps per launch) with the register cap of the
// group's chosen single-step variant.
template <class M, int NP>
static void launch_rk5_window(bool free_lanes, const GroupArgs &g, const InputArgs &in,
                              const PushArgs &pa, StepCtx *ctxs, int W, cudaStream_t s) {
  const dim3 grid((g.n + NGPU_BLOCK - 1) / NGPU_BLOCK), block(NGPU_BLOCK);
  if (!g.all_uniform) {
    launch_pdl(k_rk5_window<M, NP, false, 1>, grid, block, s, g, in, pa, ctxs, W);
    return;
  }
  // the register cap for 6 blocks per SM was the fastest window kernel on
  // the 1e6-neuron network whatever the single-step variant (4.19 bio-s per
  // wall-s against 4.00-4.01 for 5 and 8 blocks and 3.60 for 4); variant 0
  // (no cap) and the 4-block variants keep their own
  switch (g.variant) {
    case 0: launch_pdl(k_rk5_window<M, NP, true, 1>, grid, block, s, g, in, pa, ctxs, W); break;
    case 6:
    case 7:
    case 8: launch_pdl(k_rk5_window<M, NP, true, 4>, grid, block, s, g, in, pa, ctxs, W); break;
    default:
      // busy networks: lanes go through the window's steps at their own pace
      if (free_lanes)
        launch_pdl(k_rk5_window<M, NP, true, 6, true>, grid, block, s, g, in, pa, ctxs, W);
      else
        launch_pdl(k_rk5_window<M, NP, true, 6>, grid, block, s, g, in, pa, ctxs, W);
      break;
  }
}

// windows: 1-4 ports (the group kinds that WindowSteps admits)
template <template <int> class MT>
static bool launch_rk5_window_model(int np, bool free_lanes, const GroupArgs &g,
                                    const InputArgs &in, const PushArgs &pa, StepCtx *ctxs,
                                    int W, cudaStream_t s) {
  switch (np) {
    case 0:
    case 1: launch_rk5_window<MT<1>, 1>(free_lanes, g, in, pa, ctxs, W, s); return true;
    case 2: launch_rk5_window<MT<2>, 2>(free_lanes, g, in, pa, ctxs, W, s); return true;
    case 3: launch_rk5_window<MT<3>, 3>(free_lanes, g, in, pa, ctxs, W, s); return true;
    case 4: launch_rk5_window<MT<4>, 4>(free_lanes, g, in, pa, ctxs, W, s); return true;
    default: return false;
  }
}

template <template <int> class MT>
static bool launch_rk5_model(int np, const GroupArgs &g, const InputArgs &in,
                             const PushArgs &pa, StepCtx *ctx, cudaStream_t s,
                             const DeliverArgs *del, int n_del) {
  switch (np) {
    case 0:
    case 1: return launch_rk5<MT<1>, 1>(g, in, pa, ctx, s, del, n_del);
    case 2: return launch_rk5<MT<2>, 2>(g, in, pa, ctx, s, del, n_del);
    case 3: return launch_rk5<MT<3>, 3>(g, in, pa, ctx, s, del, n_del);
    case 4: return launch_rk5<MT<4>, 4>(g, in, pa, ctx, s, del, n_del);
    default:
      if (np <= 8) return launch_rk5<MT<8>, 8>(g, in, pa, ctx, s);
      return launch_rk5<MT<20>, 20>(g, in, pa, ctx, s);
  }
}

}  // namespace ngpu
