// NGB200_DeliverSpikesNoAlloc: the standalone delivery of
// ngpu_deliver_api.cu without any device allocation. Its scratch (the
// per-delay spike lists, the step context and an error word) lives in one
// file-scope __device__ array, so the call never runs cudaMalloc / cudaFree.
//
// Who needs it: a host program that has handed all device memory to its own
// allocator, or that drives delivery from a loop which must not stall. A
// cudaMalloc / cudaFree in the step path can fail there, or synchronise the
// device and block the caller's other streams.
//
// The array costs every GPU that loads the library NGB200_NOALLOC_SCRATCH
// bytes until the process exits. All calls share it and a call leaves its
// contents behind: the spike-list counters and the error word are cleared at
// the start of each call, and two calls that overlap on the GPU (for example
// on two streams, or from two host threads) race on it.
#include <cuda_runtime.h>
#include <mutex>

#include "ngpu_device.h"

// one batch: (nd + 1) * n_spikes ring entries of 8 bytes at most
#define NGB200_NOALLOC_MAX_ENTRIES (1 << 20)
#define NGB200_NOALLOC_HEADER 16384
#define NGB200_NOALLOC_SCRATCH (NGB200_NOALLOC_HEADER + 8ull * NGB200_NOALLOC_MAX_ENTRIES)

static __device__ __align__(256) unsigned char g_noalloc_scratch[NGB200_NOALLOC_SCRATCH];

namespace ngpu {
int DeliverBatch(const unsigned long long *grp_off, const unsigned *e_slot, const float *e_w,
                 int nd, const unsigned *spike_src, const float *spike_h, const int *spike_di,
                 int n_spikes, long long *acc, cudaStream_t stream, unsigned *ring_src,
                 float *ring_h, int *ring_cnt, int *delays, StepCtx *ctx, unsigned *err);
}

namespace {

std::mutex g_setup_mutex;
unsigned char *g_scratch_addr[64] = {nullptr};

// Device address of the scratch array on the current device. The host-side
// name g_noalloc_scratch is only a stand-in: kernels must be given this
// address, which is looked up once per device with that device current and
// kept for the life of the process (a cudaDeviceReset ends the context it
// belongs to; the entry point is documented as not usable after one).
unsigned char *scratch_on_current_device() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (g_scratch_addr[dev] == nullptr) {
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess) return nullptr;
    g_scratch_addr[dev] = (unsigned char *)p;
  }
  return g_scratch_addr[dev];
}

__global__ void k_clear_word(unsigned *w) { *w = 0u; }

}  // namespace

extern "C" int NGB200_DeliverSpikesNoAlloc(const unsigned long long *grp_off,
                                           const unsigned *e_slot, const float *e_w, int nd,
                                           const unsigned *spike_src, const float *spike_h,
                                           const int *spike_di, int n_spikes, long long *acc,
                                           void *stream) {
  if (nd <= 0 || nd > NGPU_MAX_DELAYS || n_spikes < 0) return 1;
  const long long C = n_spikes > 0 ? n_spikes : 1;
  if ((long long)(nd + 1) * C > NGB200_NOALLOC_MAX_ENTRIES) return 5;
  unsigned char *base = scratch_on_current_device();
  if (base == nullptr) return 3;
  cudaStream_t s = (cudaStream_t)stream;
  // header: step context, error word, delay table, per-slot counts
  ngpu::StepCtx *ctx = (ngpu::StepCtx *)base;
  unsigned *err = (unsigned *)(base + 256);
  int *delays = (int *)(base + 512);                  // nd <= 1024 ints
  int *ring_cnt = (int *)(base + 512 + 4 * 1024);     // nd + 1 <= 1025 ints
  const long long R = nd + 1;
  unsigned *ring_src = (unsigned *)(base + NGB200_NOALLOC_HEADER);
  float *ring_h = (float *)(base + NGB200_NOALLOC_HEADER + 4 * R * C);
  k_clear_word<<<1, 1, 0, s>>>(err);
  int rc = 0;
  if (ngpu::DeliverBatch(grp_off, e_slot, e_w, nd, spike_src, spike_h, spike_di, n_spikes, acc,
                         s, ring_src, ring_h, ring_cnt, delays, ctx, err) != 0) {
    rc = 3;
  }
  unsigned h_err = 0;
  if (cudaMemcpyAsync(&h_err, err, sizeof(unsigned), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess) {
    return 3;
  }
  if (rc == 0 && h_err) rc = 4;
  return rc;
}
