// Connections: specification objects, connection rules, the host CSR that
// becomes the device delivery graph, connection queries, synapse groups and
// the host random-array helpers.
//
// Reference behaviour followed (paths within golosio/NeuronGPU):
//   ConnSpec / SynSpec parameters      src/connect_rules.cpp:14-230, src/connect_spec.h
//   single connection, delay -> steps  src/connect.cu:26-62
//   rules                              src/connect_rules.h:48-400
//   connection ids and status          src/connect.h:124-188, src/connect.cu:139-170,
//                                      src/neurongpu.cu:1344-1400
//   synapse groups                     src/syn_model.cu:124-225, src/stdp.cu:53-69
//   random arrays                      src/neurongpu.cu:1101-1154
//
// Differences kept on purpose: random draws come from a counter-based
// generator keyed by the seed (not cuRAND), so a rule with a given seed makes
// the same graph for any thread count; fixed_indegree / fixed_outdegree draw
// an independent sample for every target / source (the reference reuses one
// block of draws for all thread batches, src/connect_rules.h:235-290).
#include <math.h>
#include <string.h>
#include <algorithm>
#include <numeric>
#include <unordered_set>

#include "ngpu_core.h"
#include "ngpu_rng.h"

#ifdef _OPENMP
#include <omp.h>
#endif

namespace ngpu {

// ---------------------------------------------------------------------------
// ConnSpec / SynSpec
// ---------------------------------------------------------------------------
int ConnSpec::SetParam(const std::string &name, int value) {
  if (name == "rule") {
    if (value < 0 || value > N_CONN_RULE) throw ngpu_exception("Unknown connection rule");
    rule_ = value;
  } else if (name == "indegree") {
    if (value < 0) throw ngpu_exception("Indegree must be >=0");
    indegree_ = value;
  } else if (name == "outdegree") {
    if (value < 0) throw ngpu_exception("Outdegree must be >=0");
    outdegree_ = value;
  } else if (name == "total_num") {
    if (value < 0) throw ngpu_exception("total_num must be >=0");
    total_num_ = value;
  } else {
    throw ngpu_exception("Unknown connection int parameter");
  }
  return 0;
}

bool ConnSpec::IsParam(const std::string &n) {
  return n == "rule" || n == "indegree" || n == "outdegree" || n == "total_num";
}

int SynSpec::SetParam(const std::string &name, int value) {
  if (name == "synapse_group") {
    if (value < 0) throw ngpu_exception("Unknown synapse group");
    syn_group_ = (unsigned char)value;
  } else if (name == "receptor") {
    if (value < 0) throw ngpu_exception("Port index must be >=0");
    port_ = (unsigned char)value;
  } else {
    throw ngpu_exception("Unknown synapse int parameter");
  }
  return 0;
}

int SynSpec::SetParam(const std::string &name, float value) {
  if (name == "weight") {
    weight_ = value;
  } else if (name == "delay") {
    if (value < 0) throw ngpu_exception("Delay must be >=0");
    delay_ = value;
  } else {
    throw ngpu_exception("Unknown synapse float parameter");
  }
  return 0;
}

int SynSpec::SetParam(const std::string &name, const float *arr) {
  if (name == "weight_array") weight_array_ = arr;
  else if (name == "delay_array") delay_array_ = arr;
  else throw ngpu_exception("Unknown synapse array parameter");
  return 0;
}

bool SynSpec::IsIntParam(const std::string &n) { return n == "synapse_group" || n == "receptor"; }
bool SynSpec::IsFloatParam(const std::string &n) { return n == "weight" || n == "delay"; }
bool SynSpec::IsFloatPtParam(const std::string &n) { return n == "weight_array" || n == "delay_array"; }

// ---------------------------------------------------------------------------
// edges
// ---------------------------------------------------------------------------
void NeuronGPU::AddEdge(int s, int t, unsigned char port, unsigned char syn, float w,
                        float delay) {
  if (delay < time_resolution_) throw ngpu_exception("Delay must be >= time resolution");
  float r = roundf(delay / time_resolution_);
  if (r > 65535.0f) throw ngpu_exception("Delay too large");
  e_src_.push_back((uint32_t)s);
  e_tgt_.push_back((uint32_t)t);
  e_port_.push_back(port);
  e_syn_.push_back(syn);
  e_w_.push_back(w);
  e_d_.push_back((uint16_t)r);
}

int NeuronGPU::Connect(int i_source, int i_target, unsigned char port,
                       unsigned char syn_group, float weight, float delay) {
  CheckUncalibrated("Connections cannot be created after calibration");
  const int N = (int)node_group_map_.size();
  if (i_source < 0 || i_source >= N || i_target < 0 || i_target >= N)
    throw ngpu_exception("Unrecognized node in connection");
  AddEdge(i_source, i_target, port, syn_group, weight, delay);
  host_csr_valid_ = false;
  return 0;
}

// Generic rule driver. Edges are appended in the reference's i_array order
// so weight_array / delay_array index the same connection.
int NeuronGPU::Connect(const int *src_arr, int i_src0, int n_source, const int *tgt_arr,
                       int i_tgt0, int n_target, ConnSpec &cs, SynSpec &ss) {
  CheckUncalibrated("Connections cannot be created after calibration");
  const long long N = (long long)node_group_map_.size();
  auto S = [&](long long k) -> int { return src_arr ? src_arr[k] : i_src0 + (int)k; };
  auto Tn = [&](long long k) -> int { return tgt_arr ? tgt_arr[k] : i_tgt0 + (int)k; };
  for (long long k = 0; k < n_source; k++)
    if (S(k) < 0 || S(k) >= N) throw ngpu_exception("Unrecognized source node");
  for (long long k = 0; k < n_target; k++)
    if (Tn(k) < 0 || Tn(k) >= N) throw ngpu_exception("Unrecognized target node");
  if (ss.syn_group_ > syn_groups_.size()) throw ngpu_exception("Unknown synapse group");
  auto W = [&](size_t ia) { return ss.weight_array_ ? ss.weight_array_[ia] : ss.weight_; };
  auto D = [&](size_t ia) { return ss.delay_array_ ? ss.delay_array_[ia] : ss.delay_; };
  const unsigned long long seed = rnd_seed_;
  const unsigned long long call = NextRngStream();
  size_t base = e_src_.size();
  auto reserve = [&](size_t n) {
    e_src_.resize(base + n); e_tgt_.resize(base + n); e_port_.resize(base + n);
    e_syn_.resize(base + n); e_w_.resize(base + n); e_d_.resize(base + n);
  };
  auto put = [&](size_t ia, int s, int t) {
    float delay = D(ia);
    if (delay < time_resolution_) throw ngpu_exception("Delay must be >= time resolution");
    float r = roundf(delay / time_resolution_);
    if (r > 65535.0f) throw ngpu_exception("Delay too large");
    size_t k = base + ia;
    e_src_[k] = (uint32_t)s; e_tgt_[k] = (uint32_t)t; e_port_[k] = ss.port_;
    e_syn_[k] = ss.syn_group_; e_w_[k] = W(ia); e_d_[k] = (uint16_t)r;
  };
  host_csr_valid_ = false;
  try {
    switch (cs.rule_) {
      case ONE_TO_ONE: {
        if (n_source != n_target)
          throw ngpu_exception("Number of source and target nodes must be equal for the one-to-one connection rule");
        reserve(n_source);
        for (long long k = 0; k < n_source; k++) put(k, S(k), Tn(k));
        break;
      }
      case ALL_TO_ALL: {
        size_t n = (size_t)n_source * n_target;
        reserve(n);
        for (long long it = 0; it < n_target; it++)
          for (long long is = 0; is < n_source; is++) put((size_t)it * n_source + is, S(is), Tn(it));
        break;
      }
      case FIXED_TOTAL_NUMBER: {
        size_t n = (size_t)cs.total_num_;
        reserve(n);
        if (n > 0 && (n_source <= 0 || n_target <= 0))
          throw ngpu_exception("Empty source or target list");
        for (size_t k = 0; k < n; k++) {
          Philox4 r = ng_random_block(seed, RNG_TAG_CONNECT, call, (int64_t)k, 0);
          int is = (int)(r.v[0] % (uint32_t)n_source);
          int it = (int)(r.v[1] % (uint32_t)n_target);
          put(k, S(is), Tn(it));
        }
        break;
      }
      case FIXED_INDEGREE:
      case FIXED_OUTDEGREE: {
        const bool indeg = cs.rule_ == FIXED_INDEGREE;
        const int K = indeg ? cs.indegree_ : cs.outdegree_;
        const long long n_outer = indeg ? n_target : n_source;
        const long long n_pool = indeg ? n_source : n_target;
        if (K > n_pool)
          throw ngpu_exception(indeg ? "Indegree larger than number of source nodes"
                                     : "Outdegree larger than number of target nodes");
        reserve((size_t)n_outer * K);
        bool err = false;
#pragma omp parallel for schedule(dynamic, 64)
        for (long long o = 0; o < n_outer; o++) {
          // sample K distinct pool indices for this target (source)
          std::vector<int> pick(K);
          if (n_pool < 5LL * K) {
            std::vector<int> perm(n_pool);
            std::iota(perm.begin(), perm.end(), 0);
            for (int i = 0; i < K; i++) {
              Philox4 r = ng_random_block(seed, RNG_TAG_SOURCE_SET, call, o, (uint32_t)i);
              long long j = i + (long long)(r.v[0] % (uint32_t)(n_pool - i));
              std::swap(perm[i], perm[j]);
              pick[i] = perm[i];
            }
          } else {
            // rejection of repeats with a small open-addressing set
            int cap = 16;
            while (cap < 2 * K) cap <<= 1;
            std::vector<int> table(cap, -1);
            uint32_t draw = 0;
            for (int i = 0; i < K; i++) {
              int j;
              for (;;) {
                Philox4 r = ng_random_block(seed, RNG_TAG_SOURCE_SET, call, o, draw++);
                j = (int)(r.v[0] % (uint32_t)n_pool);
                uint32_t hsh = ((uint32_t)j * 0x9E3779B1u) & (uint32_t)(cap - 1);
                bool dup = false;
                while (table[hsh] >= 0) {
                  if (table[hsh] == j) { dup = true; break; }
                  hsh = (hsh + 1) & (uint32_t)(cap - 1);
                }
                if (!dup) {
                  table[hsh] = j;
                  break;
                }
              }
              pick[i] = j;
            }
          }
          for (int i = 0; i < K; i++) {
            size_t ia = (size_t)o * K + i;
            float delay = D(ia);
            if (delay < time_resolution_) { err = true; continue; }
            size_t k = base + ia;
            e_src_[k] = (uint32_t)(indeg ? S(pick[i]) : S(o));
            e_tgt_[k] = (uint32_t)(indeg ? Tn(o) : Tn(pick[i]));
            e_port_[k] = ss.port_;
            e_syn_[k] = ss.syn_group_;
            e_w_[k] = W(ia);
            e_d_[k] = (uint16_t)std::min(65535.0f, roundf(delay / time_resolution_));
          }
        }
        if (err) throw ngpu_exception("Delay must be >= time resolution");
        break;
      }
      default:
        throw ngpu_exception("Unknown connection rule");
    }
  } catch (...) {
    e_src_.resize(base); e_tgt_.resize(base); e_port_.resize(base);
    e_syn_.resize(base); e_w_.resize(base); e_d_.resize(base);
    throw;
  }
  return 0;
}

// ---------------------------------------------------------------------------
// host CSR by (source, delay index); stable in insertion order
// ---------------------------------------------------------------------------
void NeuronGPU::BuildHostCSR() {
  if (host_csr_valid_) return;
  const uint64_t E = e_src_.size();
  const long long N = (long long)node_group_map_.size();
  int maxD = 0;
  for (uint64_t k = 0; k < E; k++) maxD = std::max<int>(maxD, e_d_[k]);
  std::vector<char> present(maxD + 1, 0);
  for (uint64_t k = 0; k < E; k++) present[e_d_[k]] = 1;
  delays_.clear();
  delay_index_.assign(maxD + 1, -1);
  for (int d = 1; d <= maxD; d++) {
    if (present[d]) {
      delay_index_[d] = (int)delays_.size();
      delays_.push_back(d);
    }
  }
  const int nd = (int)delays_.size();
  const uint64_t nkeys = (uint64_t)N * nd;
  h_grp_off_.assign(nkeys + 1, 0);
  // counts per (source, delay)
  for (uint64_t k = 0; k < E; k++) {
    uint64_t key = (uint64_t)e_src_[k] * nd + delay_index_[e_d_[k]];
    h_grp_off_[key + 1]++;
  }
  for (uint64_t k = 0; k < nkeys; k++) h_grp_off_[k + 1] += h_grp_off_[k];
  h_order_.assign(E, 0);
  // Stable scatter. The edge list is split into T contiguous chunks; each
  // chunk's edges of a key go after those of the earlier chunks, so the
  // result keeps insertion order for any T.
  int nthr = 1;
#ifdef _OPENMP
  nthr = omp_get_max_threads();
  if (E < 4000000) nthr = 1;
  while (nthr > 1 && (uint64_t)nthr * nkeys > (1ull << 30)) nthr /= 2;
#endif
  if (nthr <= 1) {
    std::vector<uint64_t> fill(h_grp_off_.begin(), h_grp_off_.end() - 1);
    for (uint64_t k = 0; k < E; k++) {
      uint64_t key = (uint64_t)e_src_[k] * nd + delay_index_[e_d_[k]];
      h_order_[fill[key]++] = k;
    }
  } else {
    std::vector<std::vector<uint32_t>> cnt(nthr);
#pragma omp parallel num_threads(nthr)
    {
      int tid = 0;
#ifdef _OPENMP
      tid = omp_get_thread_num();
#endif
      uint64_t lo = E * tid / nthr, hi = E * (tid + 1) / nthr;
      std::vector<uint32_t> &c = cnt[tid];
      c.assign(nkeys, 0);
      for (uint64_t k = lo; k < hi; k++)
        c[(uint64_t)e_src_[k] * nd + delay_index_[e_d_[k]]]++;
#pragma omp barrier
      // exclusive prefix over chunks, per key (offset inside the group)
      uint64_t k_lo = nkeys * tid / nthr, k_hi = nkeys * (tid + 1) / nthr;
      for (uint64_t key = k_lo; key < k_hi; key++) {
        uint32_t run = 0;
        for (int t = 0; t < nthr; t++) {
          uint32_t v = cnt[t][key];
          cnt[t][key] = run;
          run += v;
        }
      }
#pragma omp barrier
      for (uint64_t k = lo; k < hi; k++) {
        uint64_t key = (uint64_t)e_src_[k] * nd + delay_index_[e_d_[k]];
        h_order_[h_grp_off_[key] + c[key]++] = k;
      }
    }
  }
  host_csr_valid_ = true;
}

// ---------------------------------------------------------------------------
// connection queries
// ---------------------------------------------------------------------------
std::vector<ConnectionId> NeuronGPU::GetConnections(const int *src_arr, int i_src0,
                                                    int n_source, const int *tgt_arr,
                                                    int i_tgt0, int n_target,
                                                    int syn_group) {
  const int N = (int)node_group_map_.size();
  if (!calibrate_flag_) BuildHostCSR();
  const int nd = (int)delays_.size();
  if (src_arr == nullptr && n_source <= 0) { i_src0 = 0; n_source = N; }
  if (tgt_arr == nullptr && n_target <= 0) { i_tgt0 = 0; n_target = N; }
  std::vector<int> tsorted;
  if (tgt_arr) {
    tsorted.assign(tgt_arr, tgt_arr + n_target);
    std::sort(tsorted.begin(), tsorted.end());
  }
  std::vector<ConnectionId> out;
  for (int is = 0; is < n_source; is++) {
    int s = src_arr ? src_arr[is] : i_src0 + is;
    if (s < 0 || s >= N) throw ngpu_exception("Unrecognized source node");
    int ig = 0;
    for (int di = 0; di < nd; di++) {
      uint64_t b = h_grp_off_[(uint64_t)s * nd + di], e = h_grp_off_[(uint64_t)s * nd + di + 1];
      if (b == e) continue;
      for (uint64_t k = b; k < e; k++) {
        uint64_t o = h_order_[k];
        int t = (int)e_tgt_[o];
        bool ok;
        if (tgt_arr) ok = std::binary_search(tsorted.begin(), tsorted.end(), t);
        else ok = (t >= i_tgt0 && t < i_tgt0 + n_target);
        if (ok && syn_group >= 0 && e_syn_[o] != syn_group) ok = false;
        if (ok) {
          ConnectionId c;
          c.i_source_ = s; c.i_group_ = ig; c.i_conn_ = (int)(k - b);
          out.push_back(c);
        }
      }
      ig++;
    }
  }
  return out;
}

long long NeuronGPU::ExportConnections(int *src, int *tgt, int *port, int *syn,
                                       float *delay, float *weight) {
  const long long N = (long long)node_group_map_.size();
  if (!calibrate_flag_) BuildHostCSR();
  const int nd = (int)delays_.size();
  const long long M = (long long)e_src_.size();
  std::vector<float> dev_w;
  if (weight && calibrate_flag_ && M > 0) {
    dev_w.resize((size_t)M);
    NGPU_CUDA(cudaMemcpy(dev_w.data(), d_e_w_, sizeof(float) * M, cudaMemcpyDeviceToHost));
  }
#pragma omp parallel for schedule(dynamic, 1024)
  for (long long s = 0; s < N; s++) {
    for (int di = 0; di < nd; di++) {
      const uint64_t b = h_grp_off_[(uint64_t)s * nd + di];
      const uint64_t e = h_grp_off_[(uint64_t)s * nd + di + 1];
      for (uint64_t k = b; k < e; k++) {
        const uint64_t o = h_order_[k];
        if (src) src[k] = (int)s;
        if (tgt) tgt[k] = (int)e_tgt_[o];
        if (port) port[k] = e_port_[o];
        if (syn) syn[k] = e_syn_[o];
        if (delay) delay[k] = time_resolution_ * (float)delays_[di];
        if (weight) weight[k] = dev_w.empty() ? e_w_[o] : dev_w[k];
      }
    }
  }
  return M;
}

ConnectionStatus NeuronGPU::GetConnectionStatus(ConnectionId id) {
  const int N = (int)node_group_map_.size();
  if (!calibrate_flag_) BuildHostCSR();
  const int nd = (int)delays_.size();
  if (id.i_source_ < 0 || id.i_source_ >= N) throw ngpu_exception("Unrecognized source node");
  int ig = 0;
  for (int di = 0; di < nd; di++) {
    uint64_t b = h_grp_off_[(uint64_t)id.i_source_ * nd + di];
    uint64_t e = h_grp_off_[(uint64_t)id.i_source_ * nd + di + 1];
    if (b == e) continue;
    if (ig == id.i_group_) {
      if (id.i_conn_ < 0 || (uint64_t)id.i_conn_ >= e - b)
        throw ngpu_exception("Connection index out of range");
      uint64_t k = b + id.i_conn_;
      uint64_t o = h_order_[k];
      ConnectionStatus st;
      st.i_source = id.i_source_;
      st.i_target = (int)e_tgt_[o];
      st.port = e_port_[o];
      st.syn_group = e_syn_[o];
      st.delay = time_resolution_ * (float)delays_[di];
      st.weight = e_w_[o];
      if (calibrate_flag_) {
        // weights may have been changed by plasticity
        NGPU_CUDA(cudaMemcpy(&st.weight, d_e_w_ + k, sizeof(float), cudaMemcpyDeviceToHost));
      }
      return st;
    }
    ig++;
  }
  throw ngpu_exception("Connection group index out of range");
}

// ---------------------------------------------------------------------------
// synapse groups
// ---------------------------------------------------------------------------
int NeuronGPU::CreateSynGroup(const std::string &model) {
  CheckUncalibrated("Nodes cannot be created after calibration");
  SynGroupHost g;
  if (model == "test_syn_model") {
    g.type = 1;
    g.names = {"fact", "offset"};
    g.values = {0.1f, 0.0f};
  } else if (model == "stdp") {
    g.type = 2;
    g.names = {"tau_plus", "tau_minus", "lambda", "alpha", "mu_plus", "mu_minus", "Wmax"};
    g.values = {20.0f, 20.0f, 1.0e-4f, 1.0f, 1.0f, 1.0f, 100.0f};
  } else {
    throw ngpu_exception(std::string("Unknown synapse model name: ") + model);
  }
  if (syn_groups_.size() + 1 >= NGPU_MAX_SYN_GROUPS) throw ngpu_exception("Too many synapse groups");
  syn_groups_.push_back(g);
  return (int)syn_groups_.size();
}

static SynGroupHost &syn_at(std::vector<SynGroupHost> &v, int sg) {
  if (sg < 1 || sg > (int)v.size()) throw ngpu_exception("Unrecognized synapse group");
  return v[sg - 1];
}

int NeuronGPU::GetSynGroupNParam(int sg) { return (int)syn_at(syn_groups_, sg).names.size(); }
std::vector<std::string> NeuronGPU::GetSynGroupParamNames(int sg) { return syn_at(syn_groups_, sg).names; }
bool NeuronGPU::IsSynGroupParam(int sg, const std::string &n) {
  SynGroupHost &g = syn_at(syn_groups_, sg);
  return std::find(g.names.begin(), g.names.end(), n) != g.names.end();
}
int NeuronGPU::GetSynGroupParamIdx(int sg, const std::string &n) {
  SynGroupHost &g = syn_at(syn_groups_, sg);
  for (size_t i = 0; i < g.names.size(); i++) if (g.names[i] == n) return (int)i;
  throw ngpu_exception(std::string("Unrecognized parameter ") + n);
}
float NeuronGPU::GetSynGroupParam(int sg, const std::string &n) {
  SynGroupHost &g = syn_at(syn_groups_, sg);
  for (size_t i = 0; i < g.names.size(); i++) if (g.names[i] == n) return g.values[i];
  throw ngpu_exception(std::string("Unrecognized synapse parameter ") + n);
}
int NeuronGPU::SetSynGroupParam(int sg, const std::string &n, float v) {
  SynGroupHost &g = syn_at(syn_groups_, sg);
  for (size_t i = 0; i < g.names.size(); i++) {
    if (g.names[i] == n) {
      g.values[i] = v;
      if (calibrate_flag_ && (size_t)(sg - 1) < (size_t)NGPU_MAX_SYN_GROUPS && i < NGPU_MAX_SYN_PARAM) {
        syn_table_.param[sg - 1][i] = v;
        InvalidateGraphs();
      }
      return 0;
    }
  }
  throw ngpu_exception(std::string("Unrecognized synapse parameter ") + n);
}

// ---------------------------------------------------------------------------
// random arrays: caller owns the returned new[] arrays
// ---------------------------------------------------------------------------
unsigned int *NeuronGPU::RandomInt(size_t n) {
  unsigned long long st = NextRngStream();
  unsigned int *a = new unsigned int[n > 0 ? n : 1];
  for (size_t k = 0; k < n; k++) {
    Philox4 r = ng_random_block(rnd_seed_, RNG_TAG_ARRAY, st, (int64_t)(k >> 2), 0);
    a[k] = r.v[k & 3];
  }
  return a;
}

float *NeuronGPU::RandomUniform(size_t n) {
  unsigned long long st = NextRngStream();
  float *a = new float[n > 0 ? n : 1];
  for (size_t k = 0; k < n; k++) {
    Philox4 r = ng_random_block(rnd_seed_, RNG_TAG_ARRAY, st, (int64_t)(k >> 1), 0);
    int j = (int)(k & 1) * 2;
    a[k] = (float)ng_u01(r.v[j], r.v[j + 1]);
    if (a[k] >= 1.0f) a[k] = 0.99999994f;
  }
  return a;
}

// Box-Muller pairs from consecutive uniforms
static void normal_fill(float *a, size_t n, float mean, float stddev,
                        unsigned long long seed, unsigned long long st) {
  for (size_t k = 0; k < n; k += 2) {
    Philox4 r = ng_random_block(seed, RNG_TAG_ARRAY, st, (int64_t)(k >> 1), 0);
    double u1 = ng_u01(r.v[0], r.v[1]), u2 = ng_u01(r.v[2], r.v[3]);
    double rad = sqrt(-2.0 * log(u1));
    double z0 = rad * cos(6.283185307179586 * u2), z1 = rad * sin(6.283185307179586 * u2);
    a[k] = (float)(mean + stddev * z0);
    if (k + 1 < n) a[k + 1] = (float)(mean + stddev * z1);
  }
}

float *NeuronGPU::RandomNormal(size_t n, float mean, float stddev) {
  float *a = new float[n > 0 ? n : 1];
  normal_fill(a, n, mean, stddev, rnd_seed_, NextRngStream());
  return a;
}

// rejection of out-of-range values and optional rounding to a grid, as in
// src/neurongpu.cu:1116-1154
float *NeuronGPU::RandomNormalClipped(size_t n, float mean, float stddev, float vmin,
                                      float vmax, float vstep) {
  const float epsi = 1.0e-6f;
  if (vmax < vmin) throw ngpu_exception("Clipping range is empty");
  size_t n_alloc = (n / 4 + 1) * 4;
  float *a = new float[n_alloc];
  normal_fill(a, n_alloc, mean, stddev, rnd_seed_, NextRngStream());
  std::vector<float> extra;
  size_t ie = 0;
  int rounds = 0;
  for (size_t k = 0; k < n_alloc; k++) {
    while (a[k] < vmin || a[k] > vmax) {
      if (ie >= extra.size()) {
        if (++rounds > 100000) throw ngpu_exception("Clipped normal distribution has negligible mass in range");
        extra.assign(std::max<size_t>(n_alloc / 10 + 4, 1024), 0.0f);
        normal_fill(extra.data(), extra.size(), mean, stddev, rnd_seed_, NextRngStream());
        ie = 0;
      }
      a[k] = extra[ie++];
    }
  }
  if (vstep > stddev * epsi) {
    for (size_t k = 0; k < n_alloc; k++) a[k] = vmin + vstep * roundf((a[k] - vmin) / vstep);
  }
  return a;
}

}  // namespace ngpu
