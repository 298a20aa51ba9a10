// Single-group RK5 update launches of aeif_cond_beta (template instances of
// ngpu_rk5_launch.cuh, compiled in their own translation unit).
#include "ngpu_rk5_launch.cuh"

namespace ngpu {

bool LaunchRk5AeifCondBeta(int np, const GroupArgs &g, const InputArgs &in, const PushArgs &pa,
          StepCtx *ctx, cudaStream_t s, const DeliverArgs *del, int n_del) {
  return launch_rk5_model<AeifCondBeta>(np, g, in, pa, ctx, s, del, n_del);
}

bool LaunchRk5WindowAeifCondBeta(int np, bool free_lanes, const GroupArgs &g, const InputArgs &in,
                       const PushArgs &pa, StepCtx *ctxs, int W, cudaStream_t s) {
  return launch_rk5_window_model<AeifCondBeta>(np, free_lanes, g, in, pa, ctxs, W, s);
}

}  // namespace ngpu
