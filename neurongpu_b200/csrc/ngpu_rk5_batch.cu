// Batched RK5 update: many node groups of one model and port count in one
// launch through a device segment table (k_rk5_update_seg), e.g. the
// independent networks of a parameter sweep. Kept in its own translation unit
// so that its template instances compile in parallel with ngpu_kernels.cu.
#include <cstring>

#include "ngpu_kernels_common.cuh"

namespace ngpu {

template <class M, int NP>
static void launch_rk5_seg(const Rk5Batch &b, StepCtx *ctx, cudaStream_t s) {
  dim3 grid(b.n_blocks), block(NGPU_BLOCK);
  constexpr bool kProposer = ProposerFeatures<M>::supported && NP <= 2;
  if (b.mode == STEP_LOG) {
    if constexpr (kProposer) {
      if (b.uni) k_rk5_update_seg<M, NP, true, 1, STEP_LOG><<<grid, block, 0, s>>>(b.segs, b.blk_seg, b.blk_evals, b.dry, ctx, b.q);
      else k_rk5_update_seg<M, NP, false, 1, STEP_LOG><<<grid, block, 0, s>>>(b.segs, b.blk_seg, b.blk_evals, b.dry, ctx, b.q);
    }
    return;
  }
  // the learned proposer: the plain update of the chosen variant with the
  // straggler queue, the proposer in the queue's finishing launch
  const bool learned = b.mode == STEP_LEARNED;
  if (learned && !kProposer) return;
  if constexpr (NP <= 4) {
    if (b.uni) {
      switch (b.variant) {
        case 1: launch_pdl(k_rk5_update_seg<M, NP, true, 5, STEP_PLAIN>, grid, block, s, b.segs, b.blk_seg, b.blk_evals, b.dry, ctx, b.q); break;
        case 2: launch_pdl(k_rk5_update_seg<M, NP, true, 6, STEP_PLAIN>, grid, block, s, b.segs, b.blk_seg, b.blk_evals, b.dry, ctx, b.q); break;
        case 3: launch_pdl(k_rk5_update_seg<M, NP, true, 8, STEP_PLAIN>, grid, block, s, b.segs, b.blk_seg, b.blk_evals, b.dry, ctx, b.q); break;
        default: launch_pdl(k_rk5_update_seg<M, NP, true, 1, STEP_PLAIN>, grid, block, s, b.segs, b.blk_seg, b.blk_evals, b.dry, ctx, b.q); break;
      }
    } else {
      launch_pdl(k_rk5_update_seg<M, NP, false, 1, STEP_PLAIN>, grid, block, s, b.segs, b.blk_seg, b.blk_evals, b.dry, ctx, b.q);
    }
    if (b.q.cap > 0 && learned) {
      if constexpr (kProposer) {
        PushArgs no_pa;
        memset(&no_pa, 0, sizeof(no_pa));
        if (b.uni) launch_pdl(k_rk5_finish_learned<M, NP, true, true>, dim3(b.q.fin_blocks), block, s, b.first, no_pa, 0, b.segs, b.blk_evals, b.dry, ctx, b.q);
        else launch_pdl(k_rk5_finish_learned<M, NP, false, true>, dim3(b.q.fin_blocks), block, s, b.first, no_pa, 0, b.segs, b.blk_evals, b.dry, ctx, b.q);
      }
    } else if (b.q.cap > 0) {
      if (b.uni) launch_pdl(k_rk5_finish_seg<M, NP, true>, dim3(b.q.fin_blocks), block, s, b.segs, b.blk_evals, b.dry, ctx, b.q);
      else launch_pdl(k_rk5_finish_seg<M, NP, false>, dim3(b.q.fin_blocks), block, s, b.segs, b.blk_evals, b.dry, ctx, b.q);
    }
  }
}

// windows of W steps: the window kernel with the register cap for 5 blocks
// per SM (the batched kernel's segment arguments raise its register need:
// at 6 blocks it spills 112 bytes) unless the batch's variant is 0 (no
// cap); per-neuron parameters without a cap
template <class M, int NP>
static void launch_rk5_window_seg(const Rk5Batch &b, StepCtx *ctxs, int W, cudaStream_t s) {
  const dim3 grid(b.n_blocks), block(NGPU_BLOCK);
  if (!b.uni) {
    launch_pdl(k_rk5_window_seg<M, NP, false, 1>, grid, block, s, b.segs, b.blk_seg, b.blk_evals,
               ctxs, W);
  } else if (b.variant == 0) {
    launch_pdl(k_rk5_window_seg<M, NP, true, 1>, grid, block, s, b.segs, b.blk_seg, b.blk_evals,
               ctxs, W);
  } else {
    launch_pdl(k_rk5_window_seg<M, NP, true, 5>, grid, block, s, b.segs, b.blk_seg, b.blk_evals,
               ctxs, W);
  }
}

template <template <int> class MT>
static void launch_rk5_window_seg_model(const Rk5Batch &b, StepCtx *ctxs, int W, cudaStream_t s) {
  switch (b.np) {
    case 0:
    case 1: launch_rk5_window_seg<MT<1>, 1>(b, ctxs, W, s); break;
    case 2: launch_rk5_window_seg<MT<2>, 2>(b, ctxs, W, s); break;
    case 3: launch_rk5_window_seg<MT<3>, 3>(b, ctxs, W, s); break;
    case 4: launch_rk5_window_seg<MT<4>, 4>(b, ctxs, W, s); break;
    default: break;
  }
}

template <template <int> class MT>
static void launch_rk5_seg_model(const Rk5Batch &b, StepCtx *ctx, cudaStream_t s) {
  switch (b.np) {
    case 0:
    case 1: launch_rk5_seg<MT<1>, 1>(b, ctx, s); break;
    case 2: launch_rk5_seg<MT<2>, 2>(b, ctx, s); break;
    case 3: launch_rk5_seg<MT<3>, 3>(b, ctx, s); break;
    case 4: launch_rk5_seg<MT<4>, 4>(b, ctx, s); break;
    default: break;
  }
}

bool StepProposerSupported(int model, int np) {
  return np >= 1 && np <= 2 && (model == RK5_AEIF_COND_BETA || model == RK5_AEIF_COND_ALPHA);
}

bool Rk5BatchSupported(int model, int np) {
  return np <= 4 && model >= RK5_AEIF_COND_BETA && model <= RK5_IZHIKEVICH_COND_BETA;
}

void LaunchRk5Batch(const Rk5Batch &b, StepCtx *ctx, cudaStream_t s) {
  if (b.n_blocks <= 0) return;
  switch (b.model) {
    case RK5_AEIF_COND_BETA: launch_rk5_seg_model<AeifCondBeta>(b, ctx, s); break;
    case RK5_AEIF_COND_ALPHA: launch_rk5_seg_model<AeifCondAlpha>(b, ctx, s); break;
    case RK5_AEIF_PSC_ALPHA: launch_rk5_seg_model<AeifPscAlpha>(b, ctx, s); break;
    case RK5_AEIF_PSC_EXP: launch_rk5_seg_model<AeifPscExp>(b, ctx, s); break;
    case RK5_AEIF_PSC_DELTA: launch_rk5_seg<AeifPscDelta<1>, 1>(b, ctx, s); break;
    case RK5_IZHIKEVICH_COND_BETA: launch_rk5_seg_model<IzhCondBeta>(b, ctx, s); break;
    default: break;
  }
}

void LaunchRk5BatchWindow(const Rk5Batch &b, StepCtx *ctxs, int W, cudaStream_t s) {
  if (b.n_blocks <= 0) return;
  switch (b.model) {
    case RK5_AEIF_COND_BETA: launch_rk5_window_seg_model<AeifCondBeta>(b, ctxs, W, s); break;
    case RK5_AEIF_COND_ALPHA: launch_rk5_window_seg_model<AeifCondAlpha>(b, ctxs, W, s); break;
    case RK5_AEIF_PSC_ALPHA: launch_rk5_window_seg_model<AeifPscAlpha>(b, ctxs, W, s); break;
    case RK5_AEIF_PSC_EXP: launch_rk5_window_seg_model<AeifPscExp>(b, ctxs, W, s); break;
    case RK5_AEIF_PSC_DELTA: launch_rk5_window_seg<AeifPscDelta<1>, 1>(b, ctxs, W, s); break;
    case RK5_IZHIKEVICH_COND_BETA: launch_rk5_window_seg_model<IzhCondBeta>(b, ctxs, W, s); break;
    default: break;
  }
}

}  // namespace ngpu
