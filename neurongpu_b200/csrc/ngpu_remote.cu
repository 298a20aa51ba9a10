// Spike exchange of a network partitioned over hosts (one GPU per host
// process): the reference sends the spikes of nodes with remote targets to
// their hosts every step over MPI (src/spike_mpi.cu:284-486,
// src/neurongpu.cu:490-521) and pushes the received ones into the spike
// buffers of its remote-node images. Here a host packs the spikes of its
// exported nodes of the last n steps (n: the shortest delay of a remote
// connection, so none of them is due before the exchange), the hosts
// all-gather the packed lists with their own collective, and every host
// pushes the spikes of the remote nodes it has images of into its spike
// ring at the steps they were emitted; the ring's delivery then reaches the
// image nodes' targets at the connection delays.
#include <cuda_runtime.h>

#include "ngpu_device.h"
#include "ngpu_kernels.h"

namespace ngpu {

// one block per step of the packed range (steps T_next - n ... T_next - 1,
// T_next the step after the last one run): the spikes of exported nodes,
// appended as (step offset, node, height bits) after a 4-word header
// [count, overflow, 0, 0]
__global__ void k_pack_remote(const int *ring_cnt, const unsigned *ring_src, const float *ring_h,
                              int ring_R, int ring_C, const StepCtx *ctx, int n_steps,
                              const unsigned char *exported, unsigned *out, long long cap) {
  const int k = blockIdx.x;
  const int slot = ring_add(ctx->ring_slot, (long long)k - n_steps, ring_R);
  int c = ring_cnt[slot];
  c = c < ring_C ? c : ring_C;
  for (int j = threadIdx.x; j < c; j += blockDim.x) {
    const long long e = (long long)slot * ring_C + j;
    const unsigned src = ring_src[e];
    if (!exported[src]) continue;
    const unsigned pos = atomicAdd(&out[0], 1u);
    if ((long long)pos < cap) {
      unsigned *r = out + 4 + 3ll * pos;
      r[0] = (unsigned)k;
      r[1] = src;
      r[2] = __float_as_uint(ring_h[e]);
    } else {
      out[1] = 1u;
    }
  }
}

// the list of one other host: each spike of a remote node with an image
// here goes into the ring slot of its step. The spike counter of the step
// context counts this host's own spikes: the bookkeeping of the next step
// counts the last packed step's slot, images included, so those are taken
// off here.
__global__ void k_unpack_remote(const unsigned *in, long long count, const int *lut, int lut_n,
                                int *ring_cnt, unsigned *ring_src, float *ring_h, int ring_R,
                                int ring_C, StepCtx *ctx, int n_steps) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < count;
       i += (long long)gridDim.x * blockDim.x) {
    const unsigned *r = in + 4 + 3 * i;
    const unsigned k = r[0], src = r[1];
    if (k >= (unsigned)n_steps || src >= (unsigned)lut_n) continue;
    const int img = lut[src];
    if (img < 0) continue;
    const int slot = ring_add(ctx->ring_slot, (long long)k - n_steps, ring_R);
    const int pos = atomicAdd(&ring_cnt[slot], 1);
    if (pos < ring_C) {
      ring_src[(long long)slot * ring_C + pos] = (unsigned)img;
      ring_h[(long long)slot * ring_C + pos] = __uint_as_float(r[2]);
    } else {
      atomicOr(&ctx->err, (unsigned)DERR_RING_OVERFLOW);
    }
    if (k == (unsigned)n_steps - 1) atomicAdd(&ctx->n_spikes, ~0ull);   // minus one
  }
}

void LaunchPackRemote(const int *ring_cnt, const unsigned *ring_src, const float *ring_h,
                      int ring_R, int ring_C, const StepCtx *ctx, int n_steps,
                      const unsigned char *exported, unsigned *out, long long cap,
                      cudaStream_t s) {
  cudaMemsetAsync(out, 0, 4 * sizeof(unsigned), s);
  if (n_steps > 0)
    k_pack_remote<<<n_steps, 256, 0, s>>>(ring_cnt, ring_src, ring_h, ring_R, ring_C, ctx,
                                           n_steps, exported, out, cap);
}

void LaunchUnpackRemote(const unsigned *in, long long count, const int *lut, int lut_n,
                        int *ring_cnt, unsigned *ring_src, float *ring_h, int ring_R, int ring_C,
                        StepCtx *ctx, int n_steps, cudaStream_t s) {
  if (count <= 0) return;
  const long long blocks = (count + 255) / 256;
  k_unpack_remote<<<(int)(blocks < 1184 ? blocks : 1184), 256, 0, s>>>(
      in, count, lut, lut_n, ring_cnt, ring_src, ring_h, ring_R, ring_C, ctx, n_steps);
}

}  // namespace ngpu
