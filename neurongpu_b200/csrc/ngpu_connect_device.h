// Device-side connection builder (ngpu_connect_device.cu): rule kernels that
// append to a device edge store, and the stable CSR build.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace ngpu {

// edges in insertion order (device arrays)
struct EdgeStore {
  uint32_t *src;
  uint32_t *tgt;
  uint8_t *port;
  uint8_t *syn;
  float *w;
  uint16_t *d;          // delay in steps (>= 1)
};

// one rule call: edge ia of the call is stored at index base + ia
struct RuleArgs {
  EdgeStore e;
  long long base;
  const int *src_arr;   // device node list or null (range from src0)
  int src0;
  const int *tgt_arr;
  int tgt0;
  const float *w_arr;   // device per-connection weights or null
  float w;
  const float *d_arr;   // device per-connection delays (ms) or null
  float delay;
  uint8_t port, syn;
  float dt;
  unsigned long long seed, call;
  unsigned *err;        // bit 0 delay < dt, bit 1 delay > 65535 steps
};

// node -> group tables for the delivery slot of every edge
struct SlotTables {
  const int *node_group;
  const long long *acc_base;
  const int *n_pad;
  const int *i_node_0;
  const int *n_port;
  int n_syn_groups;
};

void DevRuleOneToOne(const RuleArgs &a, long long n, cudaStream_t s);
void DevRuleAllToAll(const RuleArgs &a, long long ns, long long nt, cudaStream_t s);
void DevRuleFixedTotal(const RuleArgs &a, long long n, long long ns, long long nt,
                       cudaStream_t s);
// ints of scratch one thread needs for fixed_indegree / fixed_outdegree
long long DevRuleFixedDegreeScratchInts(long long n_pool, int K);
void DevRuleFixedDegree(const RuleArgs &a, long long n_outer, long long n_pool, int K, int indeg,
                        int *scratch, long long slice, int n_threads, cudaStream_t s);

// histogram of the delays (65536 bins)
void DevDelayHistogram(const uint16_t *d, long long n, unsigned *hist65536, cudaStream_t s);
// CSR by key source * nd + delay index: group offsets [n_keys + 1] and the
// per-edge target, port, synapse group and weight in CSR order
cudaError_t DevBuildCSR(const EdgeStore &e, long long n, const int *d_delay_index, int nd,
                        long long n_keys, unsigned long long *grp_off, uint32_t *c_tgt,
                        uint8_t *c_port, uint8_t *c_syn, float *c_w, cudaStream_t s);
// accumulator slot of every CSR edge; err bit 2 bad port, bit 3 bad group
void DevCsrSlots(const uint32_t *c_tgt, const uint8_t *c_port, const uint8_t *c_syn,
                 long long n, const SlotTables &t, uint32_t *slot, unsigned *err,
                 cudaStream_t s);
// incoming plastic edges per target node (CSR indices, CSR order)
cudaError_t DevPlasticLists(const uint32_t *c_tgt, const uint8_t *c_syn, long long n,
                            long long n_nodes, unsigned long long *rev_off,
                            uint32_t **rev_edge_out, long long *n_plastic, cudaStream_t s);

}  // namespace ngpu
