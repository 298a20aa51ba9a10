// Connections: specification objects, the connection-rule driver (rules run
// on the GPU, ngpu_connect_device.cu, appending to a device edge store), the
// device CSR that becomes the delivery graph, connection queries (served
// from host copies of the CSR made on demand), synapse groups and the host
// random-array helpers.
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
// edges: device edge store in insertion order
// ---------------------------------------------------------------------------
void NeuronGPU::GrowRaw(long long need) {
  if (need <= raw_cap_) return;
  if (need >= 0x7fffffffLL) throw ngpu_exception("Too many connections (at most 2^31 - 1)");
  if (!stream_) NGPU_CUDA(cudaStreamCreate(&stream_));
  long long cap = std::max<long long>(need, std::max<long long>(1 << 16, raw_cap_ * 2));
  cap = std::min<long long>(cap, 0x7fffffffLL);
  EdgeStore e;
  NGPU_CUDA(cudaMalloc(&e.src, sizeof(uint32_t) * cap));
  NGPU_CUDA(cudaMalloc(&e.tgt, sizeof(uint32_t) * cap));
  NGPU_CUDA(cudaMalloc(&e.port, cap));
  NGPU_CUDA(cudaMalloc(&e.syn, cap));
  NGPU_CUDA(cudaMalloc(&e.w, sizeof(float) * cap));
  NGPU_CUDA(cudaMalloc(&e.d, sizeof(uint16_t) * cap));
  if (n_raw_ > 0) {
    NGPU_CUDA(cudaMemcpyAsync(e.src, d_raw_.src, sizeof(uint32_t) * n_raw_, cudaMemcpyDeviceToDevice, stream_));
    NGPU_CUDA(cudaMemcpyAsync(e.tgt, d_raw_.tgt, sizeof(uint32_t) * n_raw_, cudaMemcpyDeviceToDevice, stream_));
    NGPU_CUDA(cudaMemcpyAsync(e.port, d_raw_.port, n_raw_, cudaMemcpyDeviceToDevice, stream_));
    NGPU_CUDA(cudaMemcpyAsync(e.syn, d_raw_.syn, n_raw_, cudaMemcpyDeviceToDevice, stream_));
    NGPU_CUDA(cudaMemcpyAsync(e.w, d_raw_.w, sizeof(float) * n_raw_, cudaMemcpyDeviceToDevice, stream_));
    NGPU_CUDA(cudaMemcpyAsync(e.d, d_raw_.d, sizeof(uint16_t) * n_raw_, cudaMemcpyDeviceToDevice, stream_));
    NGPU_CUDA(cudaStreamSynchronize(stream_));
  }
  FreeRaw();
  d_raw_ = e;
  raw_cap_ = cap;
}

void NeuronGPU::FreeRaw() {
  auto F = [](void *p) { if (p) cudaFree(p); };
  F(d_raw_.src); F(d_raw_.tgt); F(d_raw_.port); F(d_raw_.syn); F(d_raw_.w); F(d_raw_.d);
  d_raw_ = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  raw_cap_ = 0;
}

// single connections buffered on the host go to the store in call order
void NeuronGPU::FlushPending() {
  const long long n = (long long)p_src_.size();
  if (n == 0) return;
  GrowRaw(n_raw_ + n);
  const long long b = n_raw_;
  NGPU_CUDA(cudaMemcpy(d_raw_.src + b, p_src_.data(), sizeof(uint32_t) * n, cudaMemcpyHostToDevice));
  NGPU_CUDA(cudaMemcpy(d_raw_.tgt + b, p_tgt_.data(), sizeof(uint32_t) * n, cudaMemcpyHostToDevice));
  NGPU_CUDA(cudaMemcpy(d_raw_.port + b, p_port_.data(), n, cudaMemcpyHostToDevice));
  NGPU_CUDA(cudaMemcpy(d_raw_.syn + b, p_syn_.data(), n, cudaMemcpyHostToDevice));
  NGPU_CUDA(cudaMemcpy(d_raw_.w + b, p_w_.data(), sizeof(float) * n, cudaMemcpyHostToDevice));
  NGPU_CUDA(cudaMemcpy(d_raw_.d + b, p_d_.data(), sizeof(uint16_t) * n, cudaMemcpyHostToDevice));
  n_raw_ += n;
  p_src_.clear(); p_tgt_.clear(); p_port_.clear(); p_syn_.clear(); p_w_.clear(); p_d_.clear();
}

void NeuronGPU::AddEdge(int s, int t, unsigned char port, unsigned char syn, float w,
                        float delay) {
  if (delay < time_resolution_) throw ngpu_exception("Delay must be >= time resolution");
  float r = roundf(delay / time_resolution_);
  if (r > 65535.0f) throw ngpu_exception("Delay too large");
  p_src_.push_back((uint32_t)s);
  p_tgt_.push_back((uint32_t)t);
  p_port_.push_back(port);
  p_syn_.push_back(syn);
  p_w_.push_back(w);
  p_d_.push_back((uint16_t)r);
  if (syn > 0) any_plastic_ = true;
  csr_valid_ = false;
}

int NeuronGPU::Connect(int i_source, int i_target, unsigned char port,
                       unsigned char syn_group, float weight, float delay) {
  CheckUncalibrated("Connections cannot be created after calibration");
  const int N = (int)node_group_map_.size();
  if (i_source < 0 || i_source >= N || i_target < 0 || i_target >= N)
    throw ngpu_exception("Unrecognized node in connection");
  AddEdge(i_source, i_target, port, syn_group, weight, delay);
  return 0;
}

namespace {
// device copy of a host array for the duration of one rule call
template <class T>
struct DevArray {
  T *p = nullptr;
  DevArray(const T *h, long long n, cudaStream_t s) {
    if (!h || n <= 0) return;
    if (cudaMalloc(&p, sizeof(T) * n) != cudaSuccess) throw ngpu_exception("cudaMalloc failed");
    if (cudaMemcpyAsync(p, h, sizeof(T) * n, cudaMemcpyHostToDevice, s) != cudaSuccess)
      throw ngpu_exception("cudaMemcpy failed");
  }
  ~DevArray() { if (p) cudaFree(p); }
};
}  // namespace

// Generic rule driver: the rule kernels append to the device edge store;
// edge ia of a call lands at store index base + ia, in the reference's
// i_array order, so weight_array / delay_array index the same connection.
int NeuronGPU::Connect(const int *src_arr, int i_src0, int n_source, const int *tgt_arr,
                       int i_tgt0, int n_target, ConnSpec &cs, SynSpec &ss) {
  CheckUncalibrated("Connections cannot be created after calibration");
  const long long N = (long long)node_group_map_.size();
  for (long long k = 0; k < n_source; k++) {
    int v = src_arr ? src_arr[k] : i_src0 + (int)k;
    if (v < 0 || v >= N) throw ngpu_exception("Unrecognized source node");
  }
  for (long long k = 0; k < n_target; k++) {
    int v = tgt_arr ? tgt_arr[k] : i_tgt0 + (int)k;
    if (v < 0 || v >= N) throw ngpu_exception("Unrecognized target node");
  }
  if (ss.syn_group_ > syn_groups_.size()) throw ngpu_exception("Unknown synapse group");
  if (!stream_) NGPU_CUDA(cudaStreamCreate(&stream_));
  long long n_conn = 0;
  switch (cs.rule_) {
    case ONE_TO_ONE:
      if (n_source != n_target)
        throw ngpu_exception("Number of source and target nodes must be equal for the one-to-one connection rule");
      n_conn = n_source;
      break;
    case ALL_TO_ALL: n_conn = (long long)n_source * n_target; break;
    case FIXED_TOTAL_NUMBER:
      n_conn = cs.total_num_;
      if (n_conn > 0 && (n_source <= 0 || n_target <= 0))
        throw ngpu_exception("Empty source or target list");
      break;
    case FIXED_INDEGREE:
      if (cs.indegree_ > n_source) throw ngpu_exception("Indegree larger than number of source nodes");
      n_conn = (long long)n_target * cs.indegree_;
      break;
    case FIXED_OUTDEGREE:
      if (cs.outdegree_ > n_target) throw ngpu_exception("Outdegree larger than number of target nodes");
      n_conn = (long long)n_source * cs.outdegree_;
      break;
    default:
      throw ngpu_exception("Unknown connection rule");
  }
  const unsigned long long call = NextRngStream();
  if (n_conn <= 0) return 0;
  FlushPending();
  GrowRaw(n_raw_ + n_conn);
  DevArray<int> dsrc(src_arr, n_source, stream_), dtgt(tgt_arr, n_target, stream_);
  DevArray<float> dw(ss.weight_array_, n_conn, stream_), dd(ss.delay_array_, n_conn, stream_);
  unsigned *d_err = nullptr;
  NGPU_CUDA(cudaMalloc(&d_err, sizeof(unsigned)));
  NGPU_CUDA(cudaMemsetAsync(d_err, 0, sizeof(unsigned), stream_));
  RuleArgs a;
  a.e = d_raw_;
  a.base = n_raw_;
  a.src_arr = dsrc.p; a.src0 = i_src0;
  a.tgt_arr = dtgt.p; a.tgt0 = i_tgt0;
  a.w_arr = dw.p; a.w = ss.weight_;
  a.d_arr = dd.p; a.delay = ss.delay_;
  a.port = ss.port_; a.syn = ss.syn_group_;
  a.dt = time_resolution_;
  a.seed = rnd_seed_;
  a.call = call;
  a.err = d_err;
  int *scratch = nullptr;
  switch (cs.rule_) {
    case ONE_TO_ONE: DevRuleOneToOne(a, n_conn, stream_); break;
    case ALL_TO_ALL: DevRuleAllToAll(a, n_source, n_target, stream_); break;
    case FIXED_TOTAL_NUMBER: DevRuleFixedTotal(a, n_conn, n_source, n_target, stream_); break;
    default: {
      const bool indeg = cs.rule_ == FIXED_INDEGREE;
      const int K = indeg ? cs.indegree_ : cs.outdegree_;
      const long long n_outer = indeg ? n_target : n_source;
      const long long n_pool = indeg ? n_source : n_target;
      const long long slice = DevRuleFixedDegreeScratchInts(n_pool, K);
      // as many sampling threads as fit in 1 GB of scratch, at most 148 x 1024
      long long thr = std::min<long long>(n_outer, 148LL * 1024);
      thr = std::min<long long>(thr, std::max<long long>(1, (1LL << 28) / std::max<long long>(slice, 1)));
      NGPU_CUDA(cudaMalloc(&scratch, sizeof(int) * (size_t)(slice * thr)));
      DevRuleFixedDegree(a, n_outer, n_pool, K, indeg ? 1 : 0, scratch, slice, (int)thr, stream_);
      break;
    }
  }
  unsigned err = 0;
  cudaError_t ce = cudaGetLastError();
  if (ce == cudaSuccess) ce = cudaMemcpyAsync(&err, d_err, sizeof(unsigned), cudaMemcpyDeviceToHost, stream_);
  if (ce == cudaSuccess) ce = cudaStreamSynchronize(stream_);
  if (scratch) cudaFree(scratch);
  cudaFree(d_err);
  if (ce != cudaSuccess) throw ngpu_exception(std::string("CUDA error in Connect: ") + cudaGetErrorString(ce));
  if (err & 1u) throw ngpu_exception("Delay must be >= time resolution");
  if (err & 2u) throw ngpu_exception("Delay too large");
  n_raw_ += n_conn;
  if (ss.syn_group_ > 0) any_plastic_ = true;
  csr_valid_ = false;
  return 0;
}

// ---------------------------------------------------------------------------
// CSR by (source, delay index), stable in insertion order (device build)
// ---------------------------------------------------------------------------
void NeuronGPU::FreeCSR() {
  auto F = [](void *p) { if (p) cudaFree(p); };
  F(d_grp_off_); F(d_e_post_); F(d_c_port_); F(d_e_syn_); F(d_e_w_);
  d_grp_off_ = nullptr; d_e_post_ = nullptr; d_c_port_ = nullptr; d_e_syn_ = nullptr;
  d_e_w_ = nullptr;
  mirror_valid_ = false;
  csr_valid_ = false;
}

void NeuronGPU::BuildCSR() {
  if (csr_valid_) return;
  if (!stream_) NGPU_CUDA(cudaStreamCreate(&stream_));
  FlushPending();
  FreeCSR();
  const long long E = n_raw_;
  const long long N = (long long)node_group_map_.size();
  // distinct delays
  std::vector<unsigned> hist(65536, 0);
  if (E > 0) {
    unsigned *d_hist = nullptr;
    NGPU_CUDA(cudaMalloc(&d_hist, sizeof(unsigned) * 65536));
    DevDelayHistogram(d_raw_.d, E, d_hist, stream_);
    NGPU_CUDA(cudaMemcpyAsync(hist.data(), d_hist, sizeof(unsigned) * 65536, cudaMemcpyDeviceToHost, stream_));
    NGPU_CUDA(cudaStreamSynchronize(stream_));
    cudaFree(d_hist);
  }
  delays_.clear();
  delay_index_.assign(65536, -1);
  for (int d = 1; d < 65536; d++) {
    if (hist[d]) {
      delay_index_[d] = (int)delays_.size();
      delays_.push_back(d);
    }
  }
  const int nd = (int)delays_.size();
  const long long nkeys = N * nd;
  if (nkeys >= 0xFFFFFFFFLL) throw ngpu_exception("Too many (source, delay) groups");
  int *d_dix = nullptr;
  NGPU_CUDA(cudaMalloc(&d_dix, sizeof(int) * 65536));
  NGPU_CUDA(cudaMemcpy(d_dix, delay_index_.data(), sizeof(int) * 65536, cudaMemcpyHostToDevice));
  NGPU_CUDA(cudaMalloc(&d_grp_off_, sizeof(unsigned long long) * (size_t)(nkeys + 1)));
  const size_t ne = (size_t)(E > 0 ? E : 1);
  NGPU_CUDA(cudaMalloc(&d_e_post_, sizeof(unsigned) * ne));
  NGPU_CUDA(cudaMalloc(&d_c_port_, ne));
  NGPU_CUDA(cudaMalloc(&d_e_syn_, ne));
  NGPU_CUDA(cudaMalloc(&d_e_w_, sizeof(float) * ne));
  cudaError_t ce = DevBuildCSR(d_raw_, E, d_dix, nd, nkeys, d_grp_off_, d_e_post_, d_c_port_,
                               d_e_syn_, d_e_w_, stream_);
  if (ce == cudaSuccess) ce = cudaStreamSynchronize(stream_);
  cudaFree(d_dix);
  if (ce != cudaSuccess) throw ngpu_exception(std::string("CUDA error in the CSR build: ") + cudaGetErrorString(ce));
  h_grp_off_.resize((size_t)(nkeys + 1));
  NGPU_CUDA(cudaMemcpy(h_grp_off_.data(), d_grp_off_, sizeof(unsigned long long) * (size_t)(nkeys + 1),
                       cudaMemcpyDeviceToHost));
  mirror_valid_ = false;
  csr_valid_ = true;
}

// host copies of the CSR targets, ports and synapse groups (queries)
void NeuronGPU::EnsureMirror() {
  if (!calibrate_flag_) BuildCSR();
  if (mirror_valid_) return;
  const long long E = n_raw_;
  h_c_tgt_.resize((size_t)E);
  h_c_port_.resize((size_t)E);
  h_c_syn_.resize((size_t)E);
  if (E > 0) {
    NGPU_CUDA(cudaMemcpy(h_c_tgt_.data(), d_e_post_, sizeof(uint32_t) * E, cudaMemcpyDeviceToHost));
    NGPU_CUDA(cudaMemcpy(h_c_port_.data(), d_c_port_, E, cudaMemcpyDeviceToHost));
    NGPU_CUDA(cudaMemcpy(h_c_syn_.data(), d_e_syn_, E, cudaMemcpyDeviceToHost));
  }
  mirror_valid_ = true;
}

// ---------------------------------------------------------------------------
// connection queries
// ---------------------------------------------------------------------------
std::vector<ConnectionId> NeuronGPU::GetConnections(const int *src_arr, int i_src0,
                                                    int n_source, const int *tgt_arr,
                                                    int i_tgt0, int n_target,
                                                    int syn_group) {
  const int N = (int)node_group_map_.size();
  EnsureMirror();
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
        int t = (int)h_c_tgt_[k];
        bool ok;
        if (tgt_arr) ok = std::binary_search(tsorted.begin(), tsorted.end(), t);
        else ok = (t >= i_tgt0 && t < i_tgt0 + n_target);
        if (ok && syn_group >= 0 && h_c_syn_[k] != syn_group) ok = false;
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
  EnsureMirror();
  const int nd = (int)delays_.size();
  const long long M = n_raw_;
  if (weight && M > 0)
    NGPU_CUDA(cudaMemcpy(weight, d_e_w_, sizeof(float) * M, cudaMemcpyDeviceToHost));
#pragma omp parallel for schedule(dynamic, 1024)
  for (long long s = 0; s < N; s++) {
    for (int di = 0; di < nd; di++) {
      const uint64_t b = h_grp_off_[(uint64_t)s * nd + di];
      const uint64_t e = h_grp_off_[(uint64_t)s * nd + di + 1];
      for (uint64_t k = b; k < e; k++) {
        if (src) src[k] = (int)s;
        if (tgt) tgt[k] = (int)h_c_tgt_[k];
        if (port) port[k] = h_c_port_[k];
        if (syn) syn[k] = h_c_syn_[k];
        if (delay) delay[k] = time_resolution_ * (float)delays_[di];
      }
    }
  }
  return M;
}

ConnectionStatus NeuronGPU::GetConnectionStatus(ConnectionId id) {
  const int N = (int)node_group_map_.size();
  EnsureMirror();
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
      ConnectionStatus st;
      st.i_source = id.i_source_;
      st.i_target = (int)h_c_tgt_[k];
      st.port = h_c_port_[k];
      st.syn_group = h_c_syn_[k];
      st.delay = time_resolution_ * (float)delays_[di];
      // current device weight (plasticity may have changed it)
      NGPU_CUDA(cudaMemcpy(&st.weight, d_e_w_ + k, sizeof(float), cudaMemcpyDeviceToHost));
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
// random arrays: the caller owns the returned malloc'd arrays
// ---------------------------------------------------------------------------
unsigned int *NeuronGPU::RandomInt(size_t n) {
  unsigned long long st = NextRngStream();
  unsigned int *a = (unsigned int *)malloc(sizeof(unsigned int) * (n > 0 ? n : 1));
  for (size_t k = 0; k < n; k++) {
    Philox4 r = ng_random_block(rnd_seed_, RNG_TAG_ARRAY, st, (int64_t)(k >> 2), 0);
    a[k] = r.v[k & 3];
  }
  return a;
}

float *NeuronGPU::RandomUniform(size_t n) {
  unsigned long long st = NextRngStream();
  float *a = (float *)malloc(sizeof(float) * (n > 0 ? n : 1));
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
  float *a = (float *)malloc(sizeof(float) * (n > 0 ? n : 1));
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
  float *a = (float *)malloc(sizeof(float) * n_alloc);
  normal_fill(a, n_alloc, mean, stddev, rnd_seed_, NextRngStream());
  std::vector<float> extra;
  size_t ie = 0;
  int rounds = 0;
  for (size_t k = 0; k < n_alloc; k++) {
    while (a[k] < vmin || a[k] > vmax) {
      if (ie >= extra.size()) {
        if (++rounds > 100000) {
          free(a);
          throw ngpu_exception("Clipped normal distribution has negligible mass in range");
        }
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
