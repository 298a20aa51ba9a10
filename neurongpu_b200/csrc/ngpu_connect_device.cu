// Device-side connection builder: the connection rules draw straight into a
// device edge store, and the delivery graph (CSR by source and delay) is
// built on the GPU with a stable radix sort, so a 1e9-synapse network never
// passes through host memory.
//
// Rules and their random streams follow the host restatement kept with the
// oracle (the same Philox counters, the same sampling algorithm), so the
// graph is identical to it edge for edge; rule semantics as in
// src/connect_rules.h:48-400 (golosio/NeuronGPU), with the independent
// per-target sampling of fixed_indegree / fixed_outdegree.
#include <cuda_runtime.h>
#include <stdint.h>
#include <cub/cub.cuh>
#include "ngpu_connect_device.h"
#include "ngpu_rng.h"

namespace ngpu {

enum { CERR_DELAY_SMALL = 1u, CERR_DELAY_LARGE = 2u, CERR_PORT = 4u, CERR_SYN = 8u };

__device__ __forceinline__ void put_edge(const RuleArgs &a, long long ia, int s, int t) {
  const float delay = a.d_arr ? a.d_arr[ia] : a.delay;
  if (!(delay >= a.dt)) {
    atomicOr(a.err, (unsigned)CERR_DELAY_SMALL);
    return;
  }
  const float r = roundf(delay / a.dt);
  if (r > 65535.0f) {
    atomicOr(a.err, (unsigned)CERR_DELAY_LARGE);
    return;
  }
  const long long k = a.base + ia;
  a.e.src[k] = (uint32_t)s;
  a.e.tgt[k] = (uint32_t)t;
  a.e.port[k] = a.port;
  a.e.syn[k] = a.syn;
  a.e.w[k] = a.w_arr ? a.w_arr[ia] : a.w;
  a.e.d[k] = (uint16_t)r;
}

__device__ __forceinline__ int rule_src(const RuleArgs &a, long long k) {
  return a.src_arr ? a.src_arr[k] : a.src0 + (int)k;
}
__device__ __forceinline__ int rule_tgt(const RuleArgs &a, long long k) {
  return a.tgt_arr ? a.tgt_arr[k] : a.tgt0 + (int)k;
}

__global__ void k_rule_one_to_one(RuleArgs a, long long n) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
       k += (long long)gridDim.x * blockDim.x)
    put_edge(a, k, rule_src(a, k), rule_tgt(a, k));
}

__global__ void k_rule_all_to_all(RuleArgs a, long long ns, long long nt) {
  const long long n = ns * nt;
  for (long long ia = blockIdx.x * (long long)blockDim.x + threadIdx.x; ia < n;
       ia += (long long)gridDim.x * blockDim.x) {
    const long long it = ia / ns, is = ia - it * ns;
    put_edge(a, ia, rule_src(a, is), rule_tgt(a, it));
  }
}

__global__ void k_rule_fixed_total(RuleArgs a, long long n, long long ns, long long nt) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
       k += (long long)gridDim.x * blockDim.x) {
    Philox4 r = ng_random_block(a.seed, RNG_TAG_CONNECT, a.call, (unsigned long long)k, 0);
    const int is = (int)(r.v[0] % (uint32_t)ns);
    const int it = (int)(r.v[1] % (uint32_t)nt);
    put_edge(a, k, rule_src(a, is), rule_tgt(a, it));
  }
}

// K distinct pool indices per outer node (target for fixed_indegree, source
// for fixed_outdegree): partial Fisher-Yates when the pool is small
// (n_pool < 5 K), otherwise rejection of repeats with an open-addressing set;
// each thread keeps its permutation / set in its own scratch slice.
__global__ void k_rule_fixed_degree(RuleArgs a, long long n_outer, long long n_pool, int K,
                                    int indeg, int *scratch, long long slice) {
  const long long nthr = (long long)gridDim.x * blockDim.x;
  const long long tid = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  int *buf = scratch + tid * slice;
  const bool small = n_pool < 5LL * K;
  int cap = 16;
  while (cap < 2 * K) cap <<= 1;
  for (long long o = tid; o < n_outer; o += nthr) {
    if (small) {
      for (long long j = 0; j < n_pool; j++) buf[j] = (int)j;
      for (int i = 0; i < K; i++) {
        Philox4 r = ng_random_block(a.seed, RNG_TAG_SOURCE_SET, a.call, (unsigned long long)o,
                                    (uint32_t)i);
        const long long j = i + (long long)(r.v[0] % (uint32_t)(n_pool - i));
        const int tmp = buf[i];
        buf[i] = buf[j];
        buf[j] = tmp;
        const int pick = buf[i];
        const long long ia = o * K + i;
        put_edge(a, ia, indeg ? rule_src(a, pick) : rule_src(a, o),
                 indeg ? rule_tgt(a, o) : rule_tgt(a, pick));
      }
    } else {
      for (int j = 0; j < cap; j++) buf[j] = -1;
      uint32_t draw = 0;
      for (int i = 0; i < K; i++) {
        int j;
        for (;;) {
          Philox4 r = ng_random_block(a.seed, RNG_TAG_SOURCE_SET, a.call, (unsigned long long)o,
                                      draw++);
          j = (int)(r.v[0] % (uint32_t)n_pool);
          uint32_t h = ((uint32_t)j * 0x9E3779B1u) & (uint32_t)(cap - 1);
          bool dup = false;
          while (buf[h] >= 0) {
            if (buf[h] == j) {
              dup = true;
              break;
            }
            h = (h + 1) & (uint32_t)(cap - 1);
          }
          if (!dup) {
            buf[h] = j;
            break;
          }
        }
        const long long ia = o * K + i;
        put_edge(a, ia, indeg ? rule_src(a, j) : rule_src(a, o),
                 indeg ? rule_tgt(a, o) : rule_tgt(a, j));
      }
    }
  }
}

static int grid_for(long long n, int block) {
  long long g = (n + block - 1) / block;
  if (g > 148LL * 32) g = 148LL * 32;
  return (int)(g > 0 ? g : 1);
}

void DevRuleOneToOne(const RuleArgs &a, long long n, cudaStream_t s) {
  if (n > 0) k_rule_one_to_one<<<grid_for(n, 256), 256, 0, s>>>(a, n);
}
void DevRuleAllToAll(const RuleArgs &a, long long ns, long long nt, cudaStream_t s) {
  if (ns * nt > 0) k_rule_all_to_all<<<grid_for(ns * nt, 256), 256, 0, s>>>(a, ns, nt);
}
void DevRuleFixedTotal(const RuleArgs &a, long long n, long long ns, long long nt,
                       cudaStream_t s) {
  if (n > 0) k_rule_fixed_total<<<grid_for(n, 256), 256, 0, s>>>(a, n, ns, nt);
}

long long DevRuleFixedDegreeScratchInts(long long n_pool, int K) {
  if (n_pool < 5LL * K) return n_pool;
  long long cap = 16;
  while (cap < 2LL * K) cap <<= 1;
  return cap;
}

void DevRuleFixedDegree(const RuleArgs &a, long long n_outer, long long n_pool, int K, int indeg,
                        int *scratch, long long slice, int n_threads, cudaStream_t s) {
  if (n_outer <= 0 || K <= 0) return;
  const int block = 128;
  const int grid = (n_threads + block - 1) / block;
  k_rule_fixed_degree<<<grid, block, 0, s>>>(a, n_outer, n_pool, K, indeg, scratch, slice);
}

// ---------------------------------------------------------------------------
// CSR by (source, delay index), stable in insertion order
// ---------------------------------------------------------------------------
__global__ void k_delay_hist(const uint16_t *d, long long n, unsigned *hist) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
       k += (long long)gridDim.x * blockDim.x)
    atomicAdd(&hist[d[k]], 1u);
}

__global__ void k_make_keys(const uint32_t *src, const uint16_t *d, const int *delay_index,
                            int nd, long long n, uint32_t *keys, uint32_t *vals,
                            unsigned *counts) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
       k += (long long)gridDim.x * blockDim.x) {
    const uint32_t key = src[k] * (uint32_t)nd + (uint32_t)delay_index[d[k]];
    keys[k] = key;
    vals[k] = (uint32_t)k;
    atomicAdd(&counts[key], 1u);
  }
}

__global__ void k_csr_gather(const uint32_t *order, long long n, EdgeStore e, uint32_t *c_tgt,
                             uint8_t *c_port, uint8_t *c_syn, float *c_w) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
       k += (long long)gridDim.x * blockDim.x) {
    const uint32_t o = order[k];
    c_tgt[k] = e.tgt[o];
    c_port[k] = e.port[o];
    c_syn[k] = e.syn[o];
    c_w[k] = e.w[o];
  }
}

void DevDelayHistogram(const uint16_t *d, long long n, unsigned *hist65536, cudaStream_t s) {
  cudaMemsetAsync(hist65536, 0, sizeof(unsigned) * 65536, s);
  if (n > 0) k_delay_hist<<<grid_for(n, 256), 256, 0, s>>>(d, n, hist65536);
}

static unsigned bits_for(unsigned long long v) {
  unsigned b = 1;
  while (b < 32 && (1ull << b) <= v) b++;
  return b;
}

cudaError_t DevBuildCSR(const EdgeStore &e, long long n, const int *d_delay_index, int nd,
                        long long n_keys, unsigned long long *grp_off, uint32_t *c_tgt,
                        uint8_t *c_port, uint8_t *c_syn, float *c_w, cudaStream_t s) {
  cudaError_t err = cudaSuccess;
  uint32_t *keys = nullptr, *keys2 = nullptr, *vals = nullptr, *vals2 = nullptr;
  unsigned *counts = nullptr;
  void *tmp = nullptr;
  size_t tmp_bytes = 0, tmp2 = 0;
  const int nn = (int)n;
#define CK(x) do { err = (x); if (err != cudaSuccess) goto done; } while (0)
  CK(cudaMallocAsync((void **)&counts, sizeof(unsigned) * (size_t)(n_keys + 1), s));
  CK(cudaMemsetAsync(counts, 0, sizeof(unsigned) * (size_t)(n_keys + 1), s));
  if (n > 0) {
    CK(cudaMallocAsync((void **)&keys, sizeof(uint32_t) * (size_t)n, s));
    CK(cudaMallocAsync((void **)&keys2, sizeof(uint32_t) * (size_t)n, s));
    CK(cudaMallocAsync((void **)&vals, sizeof(uint32_t) * (size_t)n, s));
    CK(cudaMallocAsync((void **)&vals2, sizeof(uint32_t) * (size_t)n, s));
    k_make_keys<<<grid_for(n, 256), 256, 0, s>>>(e.src, e.d, d_delay_index, nd, n, keys, vals,
                                                 counts);
    CK(cudaGetLastError());
    CK(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, keys, keys2, vals, vals2, nn, 0,
                                       bits_for((unsigned long long)n_keys), s));
  }
  CK(cub::DeviceScan::ExclusiveSum(nullptr, tmp2, counts, grp_off, (int)(n_keys + 1), s));
  if (tmp2 > tmp_bytes) tmp_bytes = tmp2;
  CK(cudaMallocAsync(&tmp, tmp_bytes > 0 ? tmp_bytes : 16, s));
  if (n > 0) {
    CK(cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, keys, keys2, vals, vals2, nn, 0,
                                       bits_for((unsigned long long)n_keys), s));
    k_csr_gather<<<grid_for(n, 256), 256, 0, s>>>(vals2, n, e, c_tgt, c_port, c_syn, c_w);
    CK(cudaGetLastError());
  }
  tmp2 = tmp_bytes;
  CK(cub::DeviceScan::ExclusiveSum(tmp, tmp2, counts, grp_off, (int)(n_keys + 1), s));
done:
#undef CK
  if (keys) cudaFreeAsync(keys, s);
  if (keys2) cudaFreeAsync(keys2, s);
  if (vals) cudaFreeAsync(vals, s);
  if (vals2) cudaFreeAsync(vals2, s);
  if (counts) cudaFreeAsync(counts, s);
  if (tmp) cudaFreeAsync(tmp, s);
  return err;
}

// ---------------------------------------------------------------------------
// delivery arrays and the incoming plastic lists
// ---------------------------------------------------------------------------
__global__ void k_csr_slots(const uint32_t *c_tgt, const uint8_t *c_port, const uint8_t *c_syn,
                            long long n, SlotTables t, uint32_t *slot, unsigned *err) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
       k += (long long)gridDim.x * blockDim.x) {
    const uint32_t tg = c_tgt[k];
    const int g = t.node_group[tg];
    const int port = c_port[k];
    if (port >= t.n_port[g]) {
      atomicOr(err, (unsigned)CERR_PORT);
      slot[k] = 0;
      continue;
    }
    if (c_syn[k] > t.n_syn_groups) atomicOr(err, (unsigned)CERR_SYN);
    slot[k] = (uint32_t)(t.acc_base[g] + (long long)port * t.n_pad[g] + (tg - t.i_node_0[g]));
  }
}

void DevCsrSlots(const uint32_t *c_tgt, const uint8_t *c_port, const uint8_t *c_syn,
                 long long n, const SlotTables &t, uint32_t *slot, unsigned *err,
                 cudaStream_t s) {
  if (n > 0) k_csr_slots<<<grid_for(n, 256), 256, 0, s>>>(c_tgt, c_port, c_syn, n, t, slot, err);
}

__global__ void k_plastic_keys(const uint32_t *c_tgt, const uint8_t *c_syn, long long n,
                               uint32_t sentinel, uint32_t *keys, uint32_t *vals,
                               unsigned *counts, unsigned *any) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
       k += (long long)gridDim.x * blockDim.x) {
    const bool pl = c_syn[k] > 0;
    const uint32_t key = pl ? c_tgt[k] : sentinel;
    keys[k] = key;
    vals[k] = (uint32_t)k;
    if (pl) {
      atomicAdd(&counts[key], 1u);
      *any = 1u;
    }
  }
}

cudaError_t DevPlasticLists(const uint32_t *c_tgt, const uint8_t *c_syn, long long n,
                            long long n_nodes, unsigned long long *rev_off,
                            uint32_t **rev_edge_out, long long *n_plastic, cudaStream_t s) {
  cudaError_t err = cudaSuccess;
  uint32_t *keys = nullptr, *keys2 = nullptr, *vals = nullptr, *vals2 = nullptr;
  unsigned *counts = nullptr, *any = nullptr;
  void *tmp = nullptr;
  size_t tmp_bytes = 0, tmp2 = 0;
  unsigned long long total = 0;
  *rev_edge_out = nullptr;
  *n_plastic = 0;
  const int nn = (int)n;
#define CK(x) do { err = (x); if (err != cudaSuccess) goto done; } while (0)
  CK(cudaMallocAsync((void **)&counts, sizeof(unsigned) * (size_t)(n_nodes + 1), s));
  CK(cudaMemsetAsync(counts, 0, sizeof(unsigned) * (size_t)(n_nodes + 1), s));
  CK(cudaMallocAsync((void **)&any, sizeof(unsigned), s));
  CK(cudaMemsetAsync(any, 0, sizeof(unsigned), s));
  CK(cudaMallocAsync((void **)&keys, sizeof(uint32_t) * (size_t)(n > 0 ? n : 1), s));
  CK(cudaMallocAsync((void **)&keys2, sizeof(uint32_t) * (size_t)(n > 0 ? n : 1), s));
  CK(cudaMallocAsync((void **)&vals, sizeof(uint32_t) * (size_t)(n > 0 ? n : 1), s));
  CK(cudaMallocAsync((void **)&vals2, sizeof(uint32_t) * (size_t)(n > 0 ? n : 1), s));
  if (n > 0) {
    k_plastic_keys<<<grid_for(n, 256), 256, 0, s>>>(c_tgt, c_syn, n, (uint32_t)n_nodes, keys,
                                                    vals, counts, any);
    CK(cudaGetLastError());
    CK(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, keys, keys2, vals, vals2, nn, 0,
                                       bits_for((unsigned long long)n_nodes + 1), s));
  }
  CK(cub::DeviceScan::ExclusiveSum(nullptr, tmp2, counts, rev_off, (int)(n_nodes + 1), s));
  if (tmp2 > tmp_bytes) tmp_bytes = tmp2;
  CK(cudaMallocAsync(&tmp, tmp_bytes > 0 ? tmp_bytes : 16, s));
  if (n > 0)
    CK(cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, keys, keys2, vals, vals2, nn, 0,
                                       bits_for((unsigned long long)n_nodes + 1), s));
  tmp2 = tmp_bytes;
  CK(cub::DeviceScan::ExclusiveSum(tmp, tmp2, counts, rev_off, (int)(n_nodes + 1), s));
  CK(cudaMemcpyAsync(&total, rev_off + n_nodes, sizeof(unsigned long long),
                     cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  *n_plastic = (long long)total;
  // the plastic edges are the first `total` sorted entries (non-plastic keys
  // sort last); keep them, in CSR order within each target
  CK(cudaMalloc((void **)rev_edge_out, sizeof(uint32_t) * (size_t)(total > 0 ? total : 1)));
  if (total > 0)
    CK(cudaMemcpyAsync(*rev_edge_out, vals2, sizeof(uint32_t) * (size_t)total,
                       cudaMemcpyDeviceToDevice, s));
done:
#undef CK
  if (keys) cudaFreeAsync(keys, s);
  if (keys2) cudaFreeAsync(keys2, s);
  if (vals) cudaFreeAsync(vals, s);
  if (vals2) cudaFreeAsync(vals2, s);
  if (counts) cudaFreeAsync(counts, s);
  if (any) cudaFreeAsync(any, s);
  if (tmp) cudaFreeAsync(tmp, s);
  return err;
}

}  // namespace ngpu
