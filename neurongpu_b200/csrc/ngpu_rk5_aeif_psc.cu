// Single-group RK5 update launches of the current-based AdEx models (aeif_psc_alpha, aeif_psc_exp, aeif_psc_delta) (template instances of
// ngpu_rk5_launch.cuh, compiled in their own translation unit).
#include "ngpu_rk5_launch.cuh"

namespace ngpu {

bool LaunchRk5AeifPsc(int model, int np, const GroupArgs &g, const InputArgs &in,
                      const PushArgs &pa, StepCtx *ctx, cudaStream_t s, const DeliverArgs *del,
                      int n_del) {
  switch (model) {
    case RK5_AEIF_PSC_ALPHA: return launch_rk5_model<AeifPscAlpha>(np, g, in, pa, ctx, s, del, n_del);
    case RK5_AEIF_PSC_EXP: return launch_rk5_model<AeifPscExp>(np, g, in, pa, ctx, s, del, n_del);
    case RK5_AEIF_PSC_DELTA: return launch_rk5<AeifPscDelta<1>, 1>(g, in, pa, ctx, s, del, n_del);
    default: return false;
  }
}

bool LaunchRk5WindowAeifPsc(int model, int np, bool free_lanes, const GroupArgs &g,
                            const InputArgs &in, const PushArgs &pa, StepCtx *ctxs, int W,
                            cudaStream_t s) {
  switch (model) {
    case RK5_AEIF_PSC_ALPHA:
      return launch_rk5_window_model<AeifPscAlpha>(np, free_lanes, g, in, pa, ctxs, W, s);
    case RK5_AEIF_PSC_EXP:
      return launch_rk5_window_model<AeifPscExp>(np, free_lanes, g, in, pa, ctxs, W, s);
    case RK5_AEIF_PSC_DELTA:
      launch_rk5_window<AeifPscDelta<1>, 1>(free_lanes, g, in, pa, ctxs, W, s);
      return true;
    default: return false;
  }
}

}  // namespace ngpu
