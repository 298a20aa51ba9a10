// Device-side data layout shared by the kernels and the host driver.
//
// Layout in HBM (one simulation instance):
//   * per node group, state and parameters as structure-of-arrays columns of
//     length n_pad (n rounded up to 128): var[j*n_pad + i], param[j*n_pad + i];
//     RK5 groups add h[i] (adaptive step) and dx[i] (offset of the neuron's
//     integration time from the step boundary, replacing the reference's FP64
//     per-neuron time x, src/rk5.h:27-55).
//   * acc[slot]: 64-bit fixed-point input accumulators (32 fractional bits),
//     one per (target node, receptor port); slot = acc_base + port*n_pad + i.
//     Integer addition is associative, so delivery order never changes results.
//   * out-edges in CSR order by (source, delay): e_slot (u32 accumulator slot)
//     and e_w (f32 weight) = 8 bytes per synapse; grp_off[src*nd + di] gives
//     the edge range of source src for the di-th distinct delay.
//   * a ring of per-step spike lists (R = max delay + 1 slots), replacing the
//     per-source shift queues of src/spike_buffer.cu:143-302.
#pragma once
#include <stdint.h>
#include "ngpu_rng.h"

namespace ngpu {

#define NGPU_MAX_PARAM 128      // per-neuron parameters of one model
#define NGPU_MAX_VAR 64         // per-neuron variables of one model
#define NGPU_MAX_DELAYS 1024    // distinct delay values (steps)
#define NGPU_MAX_SYN_GROUPS 32
#define NGPU_MAX_SYN_PARAM 8
#define NGPU_MAX_SYN_DT 16384   // STDP window in steps (src/syn_model.h:21)
#define NGPU_RK5_MAX_SUBSTEPS 200000

// error bits written by kernels into StepCtx::err
enum DeviceError : unsigned {
  DERR_RING_OVERFLOW = 1u,      // more spikes in one step than ring capacity
  DERR_RK5_STUCK = 2u,          // adaptive integration exceeded substep cap
  DERR_REC_OVERFLOW = 4u,       // recording buffer overflow
  DERR_NAN_STATE = 8u,
  DERR_PROPOSER_TIMEOUT = 16u,  // a tensor-core completion wait of the step proposer timed out
  DERR_REV_OVERFLOW = 32u,      // dendritic delay above its maximum or too many dendritic arrivals
  // a shared-memory prefetch of the RK5 update did not complete in time: the
  // block leaves its remaining tiles untouched (their neurons skip the step)
  DERR_TILE_TIMEOUT = 64u,
  // after DERR_TILE_TIMEOUT the block's wait for its copies still in flight
  // also ran out, so a copy may land in shared memory after the block has
  // exited: the host treats the device state as lost (Simulate fails and
  // every later call is refused until the simulator is reset)
  DERR_TILE_DRAIN = 128u
};

// Bits of GroupArgs::wait_test (test hook, 0 in normal runs): the marked
// bounded waits give up at once, as if their limit had run out, so that
// their time-out paths can be exercised without a fault or a hang.
enum WaitTest : int {
  WAIT_TEST_FIRST = 1,          // the tile prefetch wait; the first MMA wait of a proposal round
  WAIT_TEST_SECOND = 2          // the second MMA wait of a proposal round
};

#if defined(__CUDACC__)
#define NGPU_HD __host__ __device__ __forceinline__
#else
#define NGPU_HD inline
#endif

// Parity bookkeeping of a proposal round's completion barrier. A round
// commits two tensor-core completions (layer 1, then layer 2) and waits for
// them in order; phase_in is the parity of the first. Returns the parity
// to keep in ProposerSmem::phase: after a complete round the parity of the
// next round's first completion (two phases later: phase_in again); after a
// failed wait the parity of the completion still pending, which the
// teardown waits for before the tensor memory is released (ok1: the first
// wait succeeded, ok2: the second).
NGPU_HD uint32_t proposer_phase_after(uint32_t phase_in, bool ok1, bool ok2) {
  if (!ok1) return phase_in;            // layer 1 still pending
  if (!ok2) return phase_in ^ 1u;       // layer 2 still pending
  return phase_in;                      // both completed
}

// Iterations of a bounded mbarrier wait (each try_wait may also suspend the
// thread for a hardware-defined time)
#define NGPU_WAIT_ITERS (1 << 22)

struct StepCtx {
  long long it;                 // iteration index within the current session
  long long T0;                 // time index at session start
  double t0;                    // time (ms) at session start
  int poisson_pending;          // Poisson draws of step it-1 not yet folded
  unsigned err;                 // DeviceError bits
  long long rec_row;            // next row of the recording buffer
  unsigned long long n_spikes;  // spikes pushed (all time)
  // ring sizes and the slots of this step, formed when the step index is
  // set (ctx_set_slots): kernels index the rings without a 64-bit division
  int acc_slots;                // accumulator ring (0 or 1: one buffer)
  int ring_R;                   // spike ring
  int acc_in_slot;              // accumulator slot of step T - 1 (folded by this step)
  int acc_out_slot;             // accumulator slot of step T (this step's delivery)
  int ring_slot;                // spike-ring slot of step T
};

// the slots of the step T = T0 + it + 1 of c
NGPU_HD void ctx_set_slots(StepCtx &c) {
  const long long T = c.T0 + c.it + 1;
  c.acc_in_slot = c.acc_slots > 1 ? (int)((T - 1) % c.acc_slots) : 0;
  c.acc_out_slot = c.acc_slots > 1 ? (int)(T % c.acc_slots) : 0;
  c.ring_slot = c.ring_R > 0 ? (int)(T % c.ring_R) : 0;
}

// (slot + k) mod n for a ring of n slots and a small offset k (|k| < 2^30)
NGPU_HD int ring_add(int slot, long long k, int n) {
  if (n <= 1) return 0;
  int r = (int)((slot + k) % n);
  return r < 0 ? r + n : r;
}

// Where a node's spike goes and what bookkeeping it updates.
struct PushArgs {
  unsigned *ring_src;
  float *ring_h;
  int *ring_cnt;
  int ring_R;
  int ring_C;
  int *last_spike_T;
  float *last_spike_h;
  int *last_rev_T;
  int *spike_count;             // per group-local node, may be null
  float *rec_times;             // [n * max_rec], may be null
  int *n_rec;
  int max_rec;
  // dendritic-delay ring (plastic networks): nodes whose spike reaches their
  // own dendrites in step T are listed in slot T % rev_R
  unsigned *rev_src;
  int *rev_cnt;
  int rev_R, rev_C;
};

// Offset of accumulator slot `slot` in a ring of `slots` slots of `stride`
// accumulators each (the slot of step T: the delivery of step T adds into
// it and the update of step T + 1 folds and clears it; 0 for one buffer).
NGPU_HD long long acc_slot_offset(int slot, int slots, long long stride) {
  return slots > 1 ? (long long)slot * stride : 0;
}

// Per-group input folding: acc (+ Poisson direct connections) into state.
struct InputArgs {
  long long *acc;               // global accumulator array
  long long acc_base;           // this group's first slot
  // accumulators per slot (0: one buffer). Deliveries of step T add into
  // slot T mod acc_slots and the update of step T + 1 folds and clears it,
  // so the update of a step and the delivery of the same step touch
  // different slots and may run concurrently.
  long long acc_par;
  int acc_slots;                // 2, or max delay + 2 where steps run in windows
  // per slot, the last step whose delivery (or large-rate Poisson pre-pass)
  // added into it, or null: a slot stamped with another step holds zeros,
  // and its loads are skipped
  long long *acc_stamp;
  int np;                       // receptor ports
  int in_var;                   // var column of port-0 input
  int in_step;                  // column stride between ports
  int w_param;                  // weight from a port parameter?
  int w_col;                    // param column of port-0 weight
  int w_col_step;               // param column stride between ports
  float w_const[4];             // constant weights (w_param == 0)
  // Poisson direct connections into this group's nodes, CSR by local node
  const unsigned *dc_off;       // [n+1] or null
  const unsigned *dc_gen;       // generator index
  const unsigned char *dc_port;
  const float *dc_weight;
  const float *dc_delay;
  const unsigned long long *dc_stream;
  const float *gen_rate;        // per generator node
  const float *gen_origin;
  const float *gen_start;
  const float *gen_stop;
  const double *gen_lambda;     // rate*dt/1000 as the reference computes it
  const double *gen_explam;     // exp(-lambda)
  const unsigned *gen_thr;      // [gen * NGPU_CDF_LEN + k] inversion thresholds (ng_poisson_thresholds)
  unsigned long long seed;
  int dry;                      // timing run: leave the accumulators as they are
  // Uniform drive: every node of the group has exactly one direct connection,
  // all from generator ud_gen with the same port, weight and delay and with
  // consecutive random streams ud_stream0 + i. The per-node connection
  // arrays are then not read at all.
  int ud;
  int ud_port;
  float ud_w, ud_delay, ud_origin, ud_start, ud_stop;
  double ud_lambda, ud_explam;
  const unsigned *ud_thr;       // the generator's thresholds
  unsigned ud_thr8[8];          // its first 8 thresholds (kernel parameters)
  unsigned long long ud_stream0;
};


// Inference image of the learned RK5 step proposer (6 -> 32 -> 32 -> 1 MLP):
// BF16 weight tiles already in the UMMA K-major layout of the kernels' shared
// memory, FP32 output-layer parameters.
#define NGPU_MLP_NPARAM 1313      // FP32 parameters: W1 32x6, b1 32, W2 32x32, b2 32, w3 32, b3
enum MlpParamOffset {
  MLP_W1 = 0, MLP_B1 = 192, MLP_W2 = 224, MLP_B2 = 1248, MLP_W3 = 1280, MLP_B3 = 1312
};
struct MlpImage {
  unsigned w1[32 * 16 / 2];     // N 32 x K 16 bf16 (K 0..5 weights, K 6 bias)
  unsigned w2[32 * 32 / 2];     // N 32 x K 32 bf16
  float b2[32];
  float w3[32];
  float b3;
  float pad_[31];
};

// RK5 update modes
enum StepMode { STEP_PLAIN = 0, STEP_LOG = 1, STEP_LEARNED = 2 };

// Straggler queue of one RK5 update (plain controller). A neuron that is
// still inside the time step after its first sub-step saves its state to a
// record and leaves its warp; a second launch finishes the records densely,
// one neuron per thread, so a warp never carries 31 idle lanes while one
// neuron near a spike takes many short sub-steps. Resuming from a record
// repeats exactly the arithmetic of the uninterrupted loop.
// The records are split over NGPU_QLANES sub-queues by tile (128 neurons)
// index, each with its own counter on its own 128-byte line: reservations of
// different tiles then do not contend for one address.
#define NGPU_QLANES 32
struct Rk5QueueHdr {
  struct Lane {
    unsigned tail;              // records reserved in this sub-queue (may pass sub_cap)
    unsigned pad_[31];
  } lane[NGPU_QLANES];
  unsigned done;                // finishing blocks done (the last one resets the header)
  unsigned pad_[31];
};
struct Rk5Queue {
  Rk5QueueHdr *hdr;
  float *rec;                   // [NGPU_QLANES][sub_cap][stride]: node, segment, sub-steps,
                                // h, refractory, pad, time (double), state variables
  int cap;                      // NGPU_QLANES * sub_cap; 0: queue off
  int sub_cap;                  // records per sub-queue: 128 x its tiles
  int stride;                   // floats per record, a multiple of 4
  int fin_blocks;               // grid of the finishing launch
};

struct GroupArgs {
  int n;                        // nodes
  int n_pad;                    // column length
  int i_node_0;                 // first global node id
  int nvar, nparam;             // per-neuron columns in use
  float *var;                   // [nvar][n_pad]
  float *param;                 // [nparam][n_pad]
  float *h;                     // RK5 step size
  float *dx;                    // RK5 time offset
  unsigned pmask[NGPU_MAX_PARAM / 32];  // bit j: param j read per neuron
  float puni[NGPU_MAX_PARAM];   // uniform parameter values
  float pinv[NGPU_MAX_PARAM];   // 1 / puni[j] (IEEE division on the host)
  float gc[8];                  // constants derived from group parameters (propagators,
                                // thresholds, refractory steps) of the non-RK5 models
  int all_uniform;              // every parameter but refractory_step uniform
  int variant;                  // RK5 kernel variant (occupancy target)
  int dry;                      // timing run: compute everything, store nothing
  float h_min;
  float h_min_thr;              // largest float <= h_min * (1 + 1e-5) in double (RK5 escape)
  float dt;                     // time resolution (ms)
  float eps;                    // RK5 tolerance
  float inv_eps;                // 1 / eps (IEEE division on the host)
  int max_substeps;             // RK5 sub-steps per neuron and step before DERR_RK5_STUCK
  int wait_test;                // WaitTest bits (0 in normal runs)
  int den_steps;                // round(den_delay / dt) of the uniform value
  int den_delay_col;            // param column of den_delay or -1
  unsigned long long *blk_evals;  // per-block RK5 derivative evaluations
  Rk5Queue q;                   // straggler queue of the single-group launch
  // learned step proposer (STEP_LEARNED) and accepted-step logging (STEP_LOG)
  int step_mode;
  float mlp_margin;             // proposal = dt * 2^(output - margin)
  const MlpImage *mlp;
  float *log_buf;               // [log_cap][8]: 6 features, target, 0
  unsigned *log_count;
  int log_cap;
  // spike generator data
  const int *sg_off;            // [n+1]
  const int *sg_step;           // spike step index
  const float *sg_height;
  int *sg_next;
};

// One RK5 group of a batched launch: its arguments and its first block.
struct SegArgs {
  GroupArgs g;
  InputArgs in;
  PushArgs pa;
  int blk0;
  int kind;                     // ModelKind (batched launch of simple models)
  int n_sub;                    // Euler sub-steps (izhikevich_psc_exp family)
  int pad_;
};

struct SynGroupTable {
  int n;                        // number of synapse groups (index 1..n)
  int type[NGPU_MAX_SYN_GROUPS];          // 1: test_syn_model, 2: stdp
  float param[NGPU_MAX_SYN_GROUPS][NGPU_MAX_SYN_PARAM];
};

struct DeliverArgs {
  const unsigned long long *grp_off;   // [n_src*nd + 1]
  const unsigned *e_slot;
  float *e_w;
  const unsigned char *e_syn;          // null if no plastic synapse exists
  int *e_stamp;                        // arrival step of last pre spike
  const unsigned *e_post;              // target node id (plastic networks)
  long long *acc;
  long long acc_par;                   // accumulators per slot (0: one buffer)
  int acc_slots;                       // slots of the accumulator ring (see InputArgs)
  long long *acc_stamp;                // per slot, the last step added into it, or null
  const unsigned *ring_src;
  const float *ring_h;
  const int *ring_cnt;
  int ring_R, ring_C;
  int nd;
  const int *delays;                   // [nd] distinct delays in steps, ascending
  const int *delay_di;                 // [delays[nd-1] + 1] delay -> its index, or -1
  int *last_rev_T;
  int *last_post_T;
  const unsigned *rev_src;             // dendritic-delay ring (see PushArgs)
  int *rev_cnt;
  int rev_R, rev_C;
  const unsigned long long *rev_off;   // [n_nodes+1] incoming plastic edges
  const unsigned *rev_edge;
  float dt;
  unsigned long long *blk_events;      // per-block delivered events
  // step bookkeeping at the start of the delivery (block 0): count the
  // spikes of step T - 1 and empty the ring slot of step T + 1 (the
  // simulator sets it; the ring then has max delay + 2 slots)
  int step_book;
  // bit 0: the last block clears the dendritic-delay slot of this step
  // (plastic networks, the step's last kernel)
  int advance_flags;
  int *ring_cnt_w;
  unsigned *done;                      // blocks finished (reset by the last)
};

}  // namespace ngpu
