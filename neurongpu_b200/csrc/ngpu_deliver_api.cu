// Standalone spike delivery through the C ABI: one batch of spikes through a
// caller-owned CSR synapse graph into caller-owned fixed-point accumulators,
// using the simulator's delivery kernel (k_deliver in ngpu_kernels.cu).
//
// The kernel reads spikes from per-delay slots of a spike ring; this entry
// point builds that ring in scratch device memory (allocated per call),
// buckets the caller's spikes into it by delay index, runs the delivery and
// releases the scratch.
#include <cuda_runtime.h>
#include <string.h>

#include "ngpu_device.h"
#include "ngpu_kernels.h"
#include "ngpu_deliver.cuh"

namespace ngpu {

// spike k of the batch goes to ring slot (nd - di[k]) so that the kernel,
// run at time index T = nd + 1 with delays[di] = di + 1, finds it there
__global__ void k_bucket_spikes(const unsigned *src, const float *h, const int *di, int n,
                                int nd, unsigned *ring_src, float *ring_h, int *ring_cnt,
                                int C, unsigned *err) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  int d = di[k];
  if (d < 0 || d >= nd) {
    atomicOr(err, 1u);
    return;
  }
  int slot = nd - d;
  int pos = atomicAdd(&ring_cnt[slot], 1);
  if (pos < C) {
    ring_src[(long long)slot * C + pos] = src[k];
    ring_h[(long long)slot * C + pos] = h[k];
  } else {
    atomicOr(err, 2u);
  }
}

__global__ void k_prepare_batch(StepCtx *ctx, int *delays, int *ring_cnt, int nd) {
  int t = threadIdx.x;
  if (t == 0) {
    ctx->it = 0;
    ctx->T0 = nd;          // T = T0 + it + 1 = nd + 1
    ctx->t0 = 0.0;
    ctx->err = 0;
    ctx->acc_slots = 0;    // one accumulator buffer
    ctx->ring_R = nd + 1;
    ctx_set_slots(*ctx);
  }
  for (int k = t; k < nd; k += blockDim.x) delays[k] = k + 1;
  for (int k = t; k < nd + 1; k += blockDim.x) ring_cnt[k] = 0;
}

// Grid of a standalone delivery: every SM of the current device with as
// many delivery blocks as fit (nothing else runs beside it here, unlike the
// simulator's delivery), cached per device.
static int StandaloneDeliverBlocks() {
  static int cached[64] = {0};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) return 148 * 8;
  if (dev < 64 && cached[dev] > 0) return cached[dev];
  int n_sm = 0, per_sm = 0;
  if (cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n_sm <= 0)
    n_sm = 148;
  per_sm = DeliverOccupancy();
  const int blocks = n_sm * (per_sm > 0 ? per_sm : 1);
  if (dev < 64) cached[dev] = blocks;
  return blocks;
}

int DeliverBatch(const unsigned long long *grp_off, const unsigned *e_slot, const float *e_w,
                 int nd, const unsigned *spike_src, const float *spike_h, const int *spike_di,
                 int n_spikes, long long *acc, cudaStream_t stream, unsigned *ring_src,
                 float *ring_h, int *ring_cnt, int *delays, StepCtx *ctx, unsigned *err) {
  const int C = n_spikes > 0 ? n_spikes : 1;
  k_prepare_batch<<<1, 128, 0, stream>>>(ctx, delays, ring_cnt, nd);
  if (n_spikes > 0) {
    k_bucket_spikes<<<(n_spikes + 255) / 256, 256, 0, stream>>>(
        spike_src, spike_h, spike_di, n_spikes, nd, ring_src, ring_h, ring_cnt, C, err);
  }
  DeliverArgs d;
  memset(&d, 0, sizeof(d));
  d.grp_off = grp_off;
  d.e_slot = e_slot;
  d.e_w = (float *)e_w;
  d.acc = acc;
  d.ring_src = ring_src;
  d.ring_h = ring_h;
  d.ring_cnt = ring_cnt;
  d.ring_R = nd + 1;
  d.ring_C = C;
  d.nd = nd;
  d.delays = delays;
  SynGroupTable syn;
  memset(&syn, 0, sizeof(syn));
  LaunchDeliver(d, syn, ctx, StandaloneDeliverBlocks(), stream);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

}  // namespace ngpu

using namespace ngpu;

extern "C" int NGB200_DeliverSpikes(const unsigned long long *grp_off, const unsigned *e_slot,
                                    const float *e_w, int nd, const unsigned *spike_src,
                                    const float *spike_h, const int *spike_di, int n_spikes,
                                    long long *acc, void *stream) {
  if (nd <= 0 || nd > NGPU_MAX_DELAYS || n_spikes < 0) return 1;
  cudaStream_t s = (cudaStream_t)stream;
  const long long C = n_spikes > 0 ? n_spikes : 1;
  const long long R = nd + 1;
  unsigned *ring_src = nullptr, *err = nullptr;
  float *ring_h = nullptr;
  int *ring_cnt = nullptr, *delays = nullptr;
  StepCtx *ctx = nullptr;
  int rc = 0;
  if (cudaMalloc(&ring_src, sizeof(unsigned) * R * C) != cudaSuccess ||
      cudaMalloc(&ring_h, sizeof(float) * R * C) != cudaSuccess ||
      cudaMalloc(&ring_cnt, sizeof(int) * R) != cudaSuccess ||
      cudaMalloc(&delays, sizeof(int) * nd) != cudaSuccess ||
      cudaMalloc(&ctx, sizeof(StepCtx)) != cudaSuccess ||
      cudaMalloc(&err, sizeof(unsigned)) != cudaSuccess) {
    rc = 2;
  } else {
    cudaMemsetAsync(err, 0, sizeof(unsigned), s);
    if (DeliverBatch(grp_off, e_slot, e_w, nd, spike_src, spike_h, spike_di, n_spikes, acc, s,
                     ring_src, ring_h, ring_cnt, delays, ctx, err) != 0) {
      rc = 3;
    }
    unsigned h_err = 0;
    if (cudaMemcpyAsync(&h_err, err, sizeof(unsigned), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess) {
      rc = 3;
    } else if (h_err) {
      rc = 4;
    }
  }
  cudaFree(ring_src);
  cudaFree(ring_h);
  cudaFree(ring_cnt);
  cudaFree(delays);
  cudaFree(ctx);
  cudaFree(err);
  return rc;
}

namespace ngpu {

// event e's target slot and weight of the streaming-delivery probe: a
// multiplicative hash of e spreads the targets over the whole slot array
__global__ void k_probe_edges(unsigned *e_slot, float *e_w, long long n_events, long long n_slots) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n_events;
       e += (long long)gridDim.x * blockDim.x) {
    const unsigned long long h = (unsigned long long)e * 0x9E3779B97F4A7C15ull;
    e_slot[e] = (unsigned)((h >> 17) % (unsigned long long)n_slots);
    e_w[e] = 0.05f;
  }
}

// the delivery's inner loop (deliver_static_edges) over the whole edge
// array in chunks of 256 edges per warp, without the ring and CSR lookups
__global__ void __launch_bounds__(256) k_probe_deliver(DeliverArgs d, long long n_events) {
  const int lane = threadIdx.x & 31;
  const long long warp = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const long long n_warps = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long c = warp * 256; c < n_events; c += n_warps * 256) {
    const unsigned long long end = (unsigned long long)(c + 256 < n_events ? c + 256 : n_events);
    deliver_static_edges(d, d.acc, (unsigned long long)c, end, 1.0f, lane);
  }
}

}  // namespace ngpu

// The rate (events/s) at which this GPU delivers synaptic events when
// nothing else limits the delivery: n_events edges (4-byte target slot and
// 4-byte weight read once, evict-first) added as 64-bit fixed-point values
// into n_slots accumulators by the delivery's inner loop with the grid of a
// standalone delivery, timed over reps launches after one warm-up launch.
// The bound of the simulator's delivery kernel when its events per step are
// this many into this many accumulators (the ring and CSR lookups of the
// real kernel add a chain of dependent loads per (spike, delay) item).
// Allocates and frees its arrays; returns 0, 2 on an allocation failure.
extern "C" int NGB200_StreamingDeliveryRate(long long n_slots, long long n_events, int reps,
                                            double *events_per_s) {
  using namespace ngpu;
  if (n_slots <= 0 || n_events <= 0 || reps <= 0 || events_per_s == nullptr) return 1;
  long long *acc = nullptr;
  unsigned *e_slot = nullptr;
  float *e_w = nullptr;
  cudaStream_t s = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int rc = 0;
  if (cudaMalloc(&acc, sizeof(long long) * n_slots) != cudaSuccess ||
      cudaMalloc(&e_slot, sizeof(unsigned) * n_events) != cudaSuccess ||
      cudaMalloc(&e_w, sizeof(float) * n_events) != cudaSuccess ||
      cudaStreamCreate(&s) != cudaSuccess || cudaEventCreate(&e0) != cudaSuccess ||
      cudaEventCreate(&e1) != cudaSuccess) {
    rc = 2;
  } else {
    cudaMemsetAsync(acc, 0, sizeof(long long) * n_slots, s);
    k_probe_edges<<<1184, 256, 0, s>>>(e_slot, e_w, n_events, n_slots);
    DeliverArgs d;
    memset(&d, 0, sizeof(d));
    d.e_slot = e_slot;
    d.e_w = e_w;
    d.acc = acc;
    const int blocks = StandaloneDeliverBlocks();
    k_probe_deliver<<<blocks, 256, 0, s>>>(d, n_events);
    cudaEventRecord(e0, s);
    for (int r = 0; r < reps; r++) k_probe_deliver<<<blocks, 256, 0, s>>>(d, n_events);
    cudaEventRecord(e1, s);
    float ms = 0.0f;
    if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess ||
        ms <= 0.0f) {
      rc = 3;
    } else {
      *events_per_s = (double)n_events * reps / (ms * 1e-3);
    }
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (s) cudaStreamDestroy(s);
  cudaFree(acc);
  cudaFree(e_slot);
  cudaFree(e_w);
  return rc;
}
