// Host-callable launchers for the simulation kernels (ngpu_kernels.cu).
#pragma once
#include <cuda_runtime.h>
#include "ngpu_device.h"

namespace ngpu {

struct RecCol {
  const float *ptr;   // address of the recorded value (null for "spike")
  int node;           // global node id (for "spike")
  int spike;          // 1: spike height recorded in this step, else 0
  int has_out;        // node stores spikes (reference quirk of "spike")
};

// per-step node updates
bool LaunchRk5Update(int model, int np, const GroupArgs &g,
                     const InputArgs &in, const PushArgs &pa, StepCtx *ctx,
                     cudaStream_t s, const DeliverArgs *del = nullptr, int n_del = 0);
// number of RK5 kernel variants (GroupArgs::variant) for a group
int Rk5VariantCount(int np, int all_uniform);
// RK5 kernel variants of a group with uniform parameters (2-4 ports):
// 0 no register cap; 1, 2, 3: caps for 5, 6, 8 resident blocks per SM;
// 4, 5: persistent kernel with shared-memory prefetch of the state, caps for
// 5 and 6 blocks per SM; 6: cap for 4 blocks per SM; 7, 8: persistent
// kernel with caps for 4 and 3 blocks per SM
#define NGPU_RK5_VARIANTS 9
// per-model launchers (one translation unit each); with del != nullptr the
// step's delivery (n_del blocks) runs in the update's grid when the chosen
// variant allows it (returns true then)
bool LaunchRk5AeifCondBeta(int np, const GroupArgs &g, const InputArgs &in, const PushArgs &pa,
                           StepCtx *ctx, cudaStream_t s, const DeliverArgs *del, int n_del);
bool LaunchRk5AeifCondAlpha(int np, const GroupArgs &g, const InputArgs &in, const PushArgs &pa,
                            StepCtx *ctx, cudaStream_t s, const DeliverArgs *del, int n_del);
bool LaunchRk5AeifPsc(int model, int np, const GroupArgs &g, const InputArgs &in,
                      const PushArgs &pa, StepCtx *ctx, cudaStream_t s, const DeliverArgs *del,
                      int n_del);
bool LaunchRk5IzhCondBeta(int np, const GroupArgs &g, const InputArgs &in, const PushArgs &pa,
                          StepCtx *ctx, cudaStream_t s, const DeliverArgs *del, int n_del);
// several steps per launch: one RK5 group through the W steps whose step
// contexts are ctxs[0 .. W-1] (plain controller, 1-4 ports; false if the
// model or port count has no window kernel); free_lanes: a lane whose step
// ended begins its next step while the others go on (busy networks)
bool LaunchRk5Window(int model, int np, bool free_lanes, const GroupArgs &g, const InputArgs &in,
                     const PushArgs &pa, StepCtx *ctxs, int W, cudaStream_t s);
bool LaunchRk5WindowAeifCondBeta(int np, bool free_lanes, const GroupArgs &g,
                                 const InputArgs &in, const PushArgs &pa, StepCtx *ctxs, int W,
                                 cudaStream_t s);
bool LaunchRk5WindowAeifCondAlpha(int np, bool free_lanes, const GroupArgs &g,
                                  const InputArgs &in, const PushArgs &pa, StepCtx *ctxs, int W,
                                  cudaStream_t s);
bool LaunchRk5WindowAeifPsc(int model, int np, bool free_lanes, const GroupArgs &g,
                            const InputArgs &in, const PushArgs &pa, StepCtx *ctxs, int W,
                            cudaStream_t s);
bool LaunchRk5WindowIzhCondBeta(int np, bool free_lanes, const GroupArgs &g, const InputArgs &in,
                                const PushArgs &pa, StepCtx *ctxs, int W, cudaStream_t s);
// whether the variant's update grid can carry the delivery blocks (the
// register-capped one-block-per-tile variants; not the persistent ones)
inline bool Rk5FusesDelivery(int variant) {
  return variant == 0 || variant == 1 || variant == 2 || variant == 3 || variant == 6;
}
// floats per straggler record (Rk5Queue::stride) of an RK5 model / port count
int Rk5RecordFloats(int model, int np);

// several RK5 groups of one model and port count in one launch: a device
// segment table (one SegArgs per group) and a block -> segment map
struct Rk5Batch {
  int model, np;
  int uni;                        // every segment has all_uniform set
  int variant;                    // occupancy variant (as GroupArgs::variant)
  int dry;                        // timing run: compute, store nothing
  int mode;                       // StepMode shared by every segment
  int n_blocks;
  const SegArgs *segs;
  const int *blk_seg;
  unsigned long long *blk_evals;  // [n_blocks] or null
  Rk5Queue q;                     // straggler queue of the launch (cap 0: off)
  GroupArgs first;                // the first segment's arguments (proposer weights, margin)
};
bool Rk5BatchSupported(int model, int np);
void LaunchRk5Batch(const Rk5Batch &b, StepCtx *ctx, cudaStream_t s);
// a batch through the W steps of a window (plain controller)
void LaunchRk5BatchWindow(const Rk5Batch &b, StepCtx *ctxs, int W, cudaStream_t s);
// step logging / learned proposer available for this model and port count
bool StepProposerSupported(int model, int np);
void LaunchIafPscExpUpdate(const GroupArgs &g, const InputArgs &in,
                           const PushArgs &pa, StepCtx *ctx, cudaStream_t s);
// iaf_psc_exp_g / _hc (MK_IAF_PSC_EXP_G), izhikevich (MK_IZHIKEVICH) and
// izhikevich_psc_exp with n_sub Euler sub-steps (MK_IZH_PSC_EXP); the group
// constants are in GroupArgs::gc
void LaunchSimpleNeuronUpdate(int kind, int n_sub, const GroupArgs &g, const InputArgs &in,
                              const PushArgs &pa, StepCtx *ctx, cudaStream_t s);
// groups of iaf_psc_exp / iaf_psc_exp_g / izhikevich / izhikevich_psc_exp in
// one launch through a segment table (SegArgs::kind, n_sub; block -> segment)
void LaunchSimpleBatch(const SegArgs *segs, const int *blk_seg, int n_blocks, StepCtx *ctx,
                       cudaStream_t s);
void LaunchSpikeGeneratorUpdate(const GroupArgs &g, const PushArgs &pa,
                                StepCtx *ctx, cudaStream_t s);
void LaunchParrotUpdate(const GroupArgs &g, const InputArgs &in,
                        const PushArgs &pa, StepCtx *ctx, cudaStream_t s);
void LaunchSpikeDetectorUpdate(const GroupArgs &g, const InputArgs &in,
                               StepCtx *ctx, cudaStream_t s);
void LaunchPoissonNodesUpdate(const GroupArgs &g, const PushArgs &pa,
                              double lambda, double explam,
                              unsigned long long seed, StepCtx *ctx,
                              cudaStream_t s);
// folds pending input outside the step loop (end of a session)
void LaunchFoldInput(const GroupArgs &g, const InputArgs &in, StepCtx *ctx,
                     cudaStream_t s);
void LaunchClearPending(StepCtx *ctx, cudaStream_t s);
// draws a group's Poisson direct connections of NGPU_POISSON_INV_MAX or more
// expected spikes per step into its accumulators (before the update of RK5
// neurons, simple-model neurons or parrots, which leaves them out)
void LaunchPoissonLarge(const GroupArgs &g, const InputArgs &in, StepCtx *ctx,
                        cudaStream_t s);

// synaptic delivery and plasticity
void LaunchDeliver(const DeliverArgs &d, const SynGroupTable &syn,
                   StepCtx *ctx, int n_blocks, cudaStream_t s);
// around a window: the accumulator slots of the steps T_b + v_lo ...
// T_b + v_lo + v_n - 1 (T_b: the step of ctx) filled from the spike ring at
// the delays d.delays[di0 ...] (those of spiking sources, D_lo ... D_hi
// steps); then, in the
// same launch, the spike count of the steps T_b + c_lo ... T_b + c_hi - 1
// into ctx and the ring slots of the steps T_b + book_first_off ...
// + book_n - 1 emptied
void LaunchDeliverWindow(const DeliverArgs &d, StepCtx *ctx, int v_lo, int v_n, int di0,
                         int D_lo, int D_hi, long long book_first_off, int book_n,
                         long long c_lo, long long c_hi, int n_blocks, cudaStream_t s);
// spike exchange of partitioned networks (ngpu_remote.cu)
void LaunchPackRemote(const int *ring_cnt, const unsigned *ring_src, const float *ring_h,
                      int ring_R, int ring_C, const StepCtx *ctx, int n_steps,
                      const unsigned char *exported, unsigned *out, long long cap,
                      cudaStream_t s);
void LaunchUnpackRemote(const unsigned *in, long long count, const int *lut, int lut_n,
                        int *ring_cnt, unsigned *ring_src, float *ring_h, int ring_R, int ring_C,
                        StepCtx *ctx, int n_steps, cudaStream_t s);
// resident 256-thread delivery blocks per SM (grid = SMs x this)
int DeliverBlocksPerSM();
int DeliverOccupancy();
int DeliverWindowOccupancy();
// dendritic-delay arrivals of this step (before the delivery kernel)
void LaunchRevArrive(const DeliverArgs &d, StepCtx *ctx, cudaStream_t s);
void LaunchStdpPost(const DeliverArgs &d, const SynGroupTable &syn,
                    StepCtx *ctx, int n_blocks, cudaStream_t s);

// recording and step bookkeeping
void LaunchRecord(const RecCol *cols, int n_cols, float *buf, long long cap_rows,
                  const int *last_spike_T, const float *last_spike_h,
                  int initial, float dt, StepCtx *ctx, cudaStream_t s);
void LaunchAdvance(int *ring_cnt, int ring_R, int ring_C, int flags,
                   StepCtx *ctx, cudaStream_t s);
// per-step context copies of a chunk of n steps (before / after the steps)
void LaunchStepPrologue(const StepCtx *base, StepCtx *copies, int n, int rec, cudaStream_t s);
void LaunchStepEpilogue(StepCtx *base, const StepCtx *copies, int n, int rec, cudaStream_t s);

// calibration
void LaunchCalibrateRk5(int model, const GroupArgs &g, int np,
                        cudaStream_t s);
void LaunchCalibrateIaf(const GroupArgs &g, float h, cudaStream_t s);

// learned RK5 step proposer (ngpu_step_proposer.cu)
void MlpBuildImage(const float *params, MlpImage *img);
void MlpInitParams(float *params, unsigned long long seed, float b3);
// mean gradient and loss over n samples [n][8] (features, target)
float MlpGradients(const float *d_data, int n, const float *params, float *grad,
                   cudaStream_t s);
// Adam on FP32 params (in/out), mini-batches of blocks x 64 samples
void MlpTrain(const float *d_data, int n, float *params, int steps, int blocks, float lr,
              unsigned long long seed, float *loss_first, float *loss_last, cudaStream_t s);
// tensor-core inference on n feature rows [n][6]
void MlpInfer(const float *d_x6, int n, const MlpImage *d_img, float *d_out, unsigned *d_err,
              cudaStream_t s);

// utilities
void LaunchFillFloat(float *p, long long n, float v, cudaStream_t s);
void LaunchFillInt(int *p, long long n, int v, cudaStream_t s);
void LaunchScatterFloat(float *col, const int *idx, int n, float v,
                        const float *vals, int vals_stride, cudaStream_t s);
void LaunchGatherFloat(const float *col, const int *idx, int n, float *out,
                       int out_stride, cudaStream_t s);

}  // namespace ngpu
