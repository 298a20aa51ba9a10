// NeuronGPU host driver: node groups, parameters, calibration and the
// simulation loop. Connection handling lives in ngpu_connect.cpp.
//
// Reference behaviour followed here (paths within golosio/NeuronGPU):
//   node creation and group table      src/neurongpu.cu:201-243, src/neuron_models.cu:44-149
//   calibration                        src/neurongpu.cu:277-333
//   Simulate / StartSimulation / Step  src/neurongpu.cu:340-605
//   parameter and variable access      src/base_neuron.cu:175-1266
//   multimeter records                 src/multimeter.cu:23-140
#include "ngpu_core.h"

#include <math.h>
#include <stdio.h>
#include <string.h>
#include <algorithm>
#include <functional>
#include <chrono>
#include <cstdlib>

#include "ngpu_rng.h"

namespace ngpu {

static const char *kFloatParamNames[] = {"time_resolution",
                                         "max_spike_num_fact",
                                         "max_spike_per_host_fact"};
static const char *kIntParamNames[] = {"rnd_seed", "verbosity_level",
                                       "max_spike_buffer_size",
                                       "remote_spike_height_flag"};

// ---------------------------------------------------------------------------
// NodeGroup name lookup
// ---------------------------------------------------------------------------
static int find_name(const std::vector<std::string> &v, const std::string &n) {
  for (size_t i = 0; i < v.size(); i++)
    if (v[i] == n) return (int)i;
  return -1;
}
int NodeGroup::ScalVarIdx(const std::string &n) const { return find_name(mi->scal_var, n); }
int NodeGroup::PortVarIdx(const std::string &n) const { return find_name(mi->port_var, n); }
int NodeGroup::ScalParamIdx(const std::string &n) const { return find_name(mi->scal_param, n); }
int NodeGroup::PortParamIdx(const std::string &n) const { return find_name(mi->port_param, n); }
int NodeGroup::GroupParamIdx(const std::string &n) const { return find_name(mi->group_param, n); }
int NodeGroup::IntVarIdx(const std::string &n) const { return find_name(int_var_names, n); }
int NodeGroup::ArrayParamIdx(const std::string &n) const { return find_name(mi->array_param, n); }

// ---------------------------------------------------------------------------
// construction
// ---------------------------------------------------------------------------
NeuronGPU::NeuronGPU() {
  memset(&syn_table_, 0, sizeof(syn_table_));
}

NeuronGPU::~NeuronGPU() {
  for (auto &r : records_) {
    if (r.fp) fclose(r.fp);
  }
  try {
    FreeDevice();
  } catch (...) {
  }
  for (NodeGroup *g : groups_) delete g;
}

void NeuronGPU::FreeDevice() {
  InvalidateGraphs();
  FreeRk5Batches();
  auto F = [](void *p) { if (p) cudaFree(p); };
  for (NodeGroup *g : groups_) {
    F(g->d_var); F(g->d_param); F(g->d_h); F(g->d_dx);
    F(g->d_spike_count); F(g->d_rec_times); F(g->d_n_rec);
    F(g->d_sg_off); F(g->d_sg_step); F(g->d_sg_next); F(g->d_sg_height);
    F(g->d_blk_evals);
    FreeRk5Queue(g->q);
    F(g->d_log_buf); F(g->d_log_count);
    g->d_log_buf = nullptr;
    g->d_log_count = nullptr;
    g->log_cap = 0;
    if (g->step_mode == STEP_LOG) g->step_mode = STEP_PLAIN;
    g->d_var = g->d_param = g->d_h = g->d_dx = nullptr;
  }
  F(d_ctx_); F(d_ctxs_); F(d_acc_); F(d_acc_stamp_);
  d_acc_stamp_ = nullptr;
  F(d_exported_);
  d_exported_ = nullptr;
  for (int *p : d_image_lut_) F(p);
  d_image_lut_.clear();
  d_ctxs_ = nullptr;
  n_ctxs_ = 0; F(d_ring_src_); F(d_ring_h_); F(d_ring_cnt_);
  F(d_last_spike_T_); F(d_last_rev_T_); F(d_last_post_T_); F(d_last_spike_h_);
  FreeRaw();
  F(d_grp_off_); F(d_e_slot_); F(d_e_w_); F(d_e_syn_); F(d_e_stamp_); F(d_c_port_);
  d_grp_off_ = nullptr; d_e_slot_ = nullptr; d_e_w_ = nullptr; d_e_syn_ = nullptr;
  d_e_stamp_ = nullptr; d_c_port_ = nullptr;
  F(d_e_post_); F(d_rev_off_); F(d_rev_edge_); F(d_delays_); F(d_delay_di_);
  F(d_rev_src_); F(d_rev_cnt_);
  d_rev_src_ = nullptr;
  d_rev_cnt_ = nullptr;
  rev_R_ = rev_C_ = 0;
  F(d_dc_off_); F(d_dc_gen_); F(d_dc_port_); F(d_dc_w_); F(d_dc_delay_);
  F(d_dc_stream_); F(d_gen_rate_); F(d_gen_origin_); F(d_gen_start_);
  F(d_gen_stop_); F(d_gen_lambda_); F(d_gen_explam_); F(d_gen_thr_); F(d_blk_events_); F(d_done_);
  F(d_rec_cols_); F(d_rec_buf_);
  F(d_mlp_img_);
  d_mlp_img_ = nullptr;
  for (cudaEvent_t e : kev_) cudaEventDestroy(e);
  kev_.clear();
  if (ev_start_) cudaEventDestroy(ev_start_);
  if (ev_stop_) cudaEventDestroy(ev_stop_);
  if (ev_c0_) cudaEventDestroy(ev_c0_);
  if (ev_c1_) cudaEventDestroy(ev_c1_);
  ev_start_ = ev_stop_ = ev_c0_ = ev_c1_ = nullptr;
  d_ctx_ = nullptr;
  if (ev_fork_) cudaEventDestroy(ev_fork_);
  if (ev_join_) cudaEventDestroy(ev_join_);
  ev_fork_ = ev_join_ = nullptr;
  if (dstream_) {
    cudaStreamDestroy(dstream_);
    dstream_ = nullptr;
  }
  if (stream_) {
    cudaStreamDestroy(stream_);
    stream_ = nullptr;
  }
}

void NeuronGPU::CheckUncalibrated(const std::string &msg) {
  if (calibrate_flag_) throw ngpu_exception(msg);
}

// ---------------------------------------------------------------------------
// kernel parameters (src/neurongpu.cu:59-85, 1643-1818)
// ---------------------------------------------------------------------------
int NeuronGPU::SetRandomSeed(unsigned long long seed) {
  rnd_seed_ = seed;
  kernel_seed_ = seed + 12345ULL;
  rng_calls_ = 0;
  return 0;
}

int NeuronGPU::SetTimeResolution(float t) {
  CheckUncalibrated("Time resolution cannot be changed after calibration");
  if (!(t > 0.0f)) throw ngpu_exception("Time resolution must be > 0");
  time_resolution_ = t;
  return 0;
}

std::vector<std::string> NeuronGPU::GetFloatParamNames() {
  return std::vector<std::string>(kFloatParamNames, kFloatParamNames + 3);
}
std::vector<std::string> NeuronGPU::GetIntParamNames() {
  return std::vector<std::string>(kIntParamNames, kIntParamNames + 4);
}
bool NeuronGPU::IsFloatParam(const std::string &n) {
  return find_name(GetFloatParamNames(), n) >= 0;
}
bool NeuronGPU::IsIntParam(const std::string &n) {
  return find_name(GetIntParamNames(), n) >= 0;
}
int NeuronGPU::GetFloatParamIdx(const std::string &n) {
  int i = find_name(GetFloatParamNames(), n);
  if (i < 0) throw ngpu_exception(std::string("Unrecognized kernel float parameter ") + n);
  return i;
}
int NeuronGPU::GetIntParamIdx(const std::string &n) {
  int i = find_name(GetIntParamNames(), n);
  if (i < 0) throw ngpu_exception(std::string("Unrecognized kernel int parameter ") + n);
  return i;
}
float NeuronGPU::GetFloatParam(const std::string &n) {
  switch (GetFloatParamIdx(n)) {
    case 0: return time_resolution_;
    case 1: return max_spike_num_fact_;
    default: return max_spike_per_host_fact_;
  }
}
int NeuronGPU::GetIntParam(const std::string &n) {
  switch (GetIntParamIdx(n)) {
    case 0: return (int)rnd_seed_;
    case 1: return verbosity_level_;
    case 2: return max_spike_buffer_size_;
    default: return remote_spike_height_flag_;
  }
}
int NeuronGPU::SetFloatParam(const std::string &n, float v) {
  switch (GetFloatParamIdx(n)) {
    case 0: return SetTimeResolution(v);
    case 1: max_spike_num_fact_ = v; return 0;
    default: max_spike_per_host_fact_ = v; return 0;
  }
}
int NeuronGPU::SetIntParam(const std::string &n, int v) {
  switch (GetIntParamIdx(n)) {
    case 0: return SetRandomSeed((unsigned long long)v);
    case 1: verbosity_level_ = v; return 0;
    case 2: max_spike_buffer_size_ = v; return 0;
    default:
      if (v != 0 && v != 1)
        throw ngpu_exception("Admissible values of remote_spike_height_flag are only 0 or 1");
      remote_spike_height_flag_ = v;
      return 0;
  }
}

// ---------------------------------------------------------------------------
// node creation
// ---------------------------------------------------------------------------
int NeuronGPU::Create(const std::string &model, int n_node, int n_port) {
  CheckUncalibrated("Nodes cannot be created after calibration");
  if (n_node <= 0) throw ngpu_exception("Number of nodes must be greater than zero.");
  if (n_port < 0) throw ngpu_exception("Number of ports must be >= zero.");
  int m = FindModel(model);
  if (m < 0) throw ngpu_exception(std::string("Unknown neuron model name: ") + model);
  const ModelInfo &mi = ModelCatalogue()[m];
  if (mi.fixed_n_port >= 0) n_port = mi.fixed_n_port;
  if (n_port > 128) throw ngpu_exception("Maximum number of ports 128 exceeded");
  if (mi.kind == MK_RK5 && n_port > 20)
    throw ngpu_exception("RK5 models support at most 20 receptor ports");
  if ((long long)node_group_map_.size() + n_node > 0x7FFFFFFFLL)
    throw ngpu_exception("Maximum number of nodes exceeded");
  if (cudaSuccess != cudaFree(0)) throw ngpu_exception("CUDA device not available");
  if (!stream_) NGPU_CUDA(cudaStreamCreate(&stream_));

  NodeGroup *g = new NodeGroup;
  g->model = m;
  g->mi = &mi;
  g->i_node_0 = (int)node_group_map_.size();
  g->n_node = n_node;
  g->n_port = n_port;
  g->n_pad = (n_node + 127) / 128 * 128;
  g->nvar = (int)(mi.scal_var.size() + mi.port_var.size() * n_port);
  g->nparam = (int)(mi.scal_param.size() + mi.port_param.size() * n_port);
  if (g->nparam > NGPU_MAX_PARAM || g->nvar > NGPU_MAX_VAR) {
    delete g;
    throw ngpu_exception("Too many ports for this model");
  }
  g->group_param = mi.group_param_def;
  try {
    if (g->nvar > 0)
      NGPU_CUDA(cudaMalloc(&g->d_var, sizeof(float) * (size_t)g->nvar * g->n_pad));
    if (g->nparam > 0)
      NGPU_CUDA(cudaMalloc(&g->d_param, sizeof(float) * (size_t)g->nparam * g->n_pad));
    if (mi.kind == MK_RK5) {
      NGPU_CUDA(cudaMalloc(&g->d_h, sizeof(float) * g->n_pad));
      NGPU_CUDA(cudaMalloc(&g->d_dx, sizeof(float) * g->n_pad));
    }
  } catch (...) {
    delete g;
    throw;
  }
  // defaults
  const int NSV = g->NSV(), NPV = g->NPV(), NSP = g->NSP(), NPP = g->NPP();
  for (int j = 0; j < NSV; j++)
    LaunchFillFloat(g->d_var + (size_t)j * g->n_pad, g->n_pad, mi.scal_var_def[j], stream_);
  for (int p = 0; p < n_port; p++)
    for (int k = 0; k < NPV; k++)
      LaunchFillFloat(g->d_var + (size_t)(NSV + p * NPV + k) * g->n_pad, g->n_pad,
                      mi.port_var_def[k], stream_);
  g->p_uniform.assign(g->nparam, 1);
  g->p_uval.assign(g->nparam, 0.0f);
  for (int j = 0; j < NSP; j++) g->p_uval[j] = mi.scal_param_def[j];
  for (int p = 0; p < n_port; p++)
    for (int k = 0; k < NPP; k++) g->p_uval[NSP + p * NPP + k] = mi.port_param_def[k];
  for (int j = 0; j < g->nparam; j++)
    LaunchFillFloat(g->d_param + (size_t)j * g->n_pad, g->n_pad, g->p_uval[j], stream_);
  if (mi.kind == MK_RK5) {
    float h0 = g->group_param[1] * 0.1f;
    LaunchFillFloat(g->d_h, g->n_pad, h0, stream_);
    LaunchFillFloat(g->d_dx, g->n_pad, 0.0f, stream_);
  }
  if (mi.kind == MK_SPIKE_GENERATOR) {
    g->sg_times.assign(n_node, std::vector<float>());
    g->sg_heights.assign(n_node, std::vector<float>());
  }
  NGPU_CUDA(cudaStreamSynchronize(stream_));
  groups_.push_back(g);
  node_group_map_.insert(node_group_map_.end(), n_node, (int)groups_.size() - 1);
  csr_valid_ = false;
  return g->i_node_0;
}

int NeuronGPU::CreatePoissonGenerator(int n_node, float rate) {
  CheckUncalibrated("Poisson generator cannot be created after calibration");
  for (NodeGroup *g : groups_)
    if (g->mi->kind == MK_POISSON_NODES)
      throw ngpu_exception("Number of poisson generators cannot be modified.");
  if (n_node <= 0) throw ngpu_exception("Number of nodes must be greater than zero.");
  static ModelInfo pn;
  if (pn.name.empty()) {
    pn.name = "";
    pn.kind = MK_POISSON_NODES;
    pn.rk5_model = -1;
    pn.fixed_n_port = 0;
    pn.in_var = -1; pn.in_step = 0; pn.w_param = false; pn.w_param_idx = -1;
    pn.refr_param = -1; pn.den_delay_param = -1;
  }
  if (!stream_) NGPU_CUDA(cudaStreamCreate(&stream_));
  NodeGroup *g = new NodeGroup;
  g->model = -1;
  g->mi = &pn;
  g->i_node_0 = (int)node_group_map_.size();
  g->n_node = n_node;
  g->n_port = 0;
  g->n_pad = (n_node + 127) / 128 * 128;
  // lambda as the reference computes it (src/neurongpu.cu:260)
  g->poisson_lambda = (float)(rate * time_resolution_ / 1000.0);
  groups_.push_back(g);
  node_group_map_.insert(node_group_map_.end(), n_node, (int)groups_.size() - 1);
  csr_valid_ = false;
  return g->i_node_0;
}

// ---------------------------------------------------------------------------
// group lookup
// ---------------------------------------------------------------------------
NodeGroup *NeuronGPU::GroupOf(int i_node, int n, int &i_local) {
  if (i_node < 0 || n <= 0 || (long long)i_node + n > (long long)node_group_map_.size())
    throw ngpu_exception("Unrecognized node in getting node sequence offset");
  int ig = node_group_map_[i_node];
  if (node_group_map_[i_node + n - 1] != ig)
    throw ngpu_exception("Nodes belong to different node groups in setting parameter");
  i_local = i_node - groups_[ig]->i_node_0;
  return groups_[ig];
}

NodeGroup *NeuronGPU::GroupOfList(const int *nodes, int n, std::vector<int> &local) {
  if (n <= 0) throw ngpu_exception("Number of nodes must be greater than zero");
  int in0 = nodes[0];
  if (in0 < 0 || in0 >= (int)node_group_map_.size())
    throw ngpu_exception("Unrecognized node in setting parameter");
  int ig = node_group_map_[in0];
  NodeGroup *g = groups_[ig];
  local.resize(n);
  for (int k = 0; k < n; k++) {
    int in = nodes[k];
    if (in < 0 || in >= (int)node_group_map_.size())
      throw ngpu_exception("Unrecognized node in setting parameter");
    if (node_group_map_[in] != ig)
      throw ngpu_exception("Nodes belong to different node groups in setting parameter");
    local[k] = in - g->i_node_0;
  }
  return g;
}

// ---------------------------------------------------------------------------
// parameter columns
// ---------------------------------------------------------------------------
void NeuronGPU::SetParamColumn(NodeGroup *g, int col, int i0, int n,
                               const int *nodes, float val, const float *vals,
                               int stride) {
  float *base = g->d_param + (size_t)col * g->n_pad;
  bool whole = (nodes == nullptr && i0 == 0 && n == g->n_node);
  const char old_uniform = g->p_uniform[col];
  const float old_uval = g->p_uval[col];
  if (vals == nullptr) {
    if (whole) {
      g->p_uniform[col] = 1;
      g->p_uval[col] = val;
    } else if (!(g->p_uniform[col] && g->p_uval[col] == val)) {
      g->p_uniform[col] = 0;
    }
  } else {
    g->p_uniform[col] = 0;
  }
  if (nodes == nullptr && vals == nullptr) {
    LaunchFillFloat(base + i0, n, val, stream_);
  } else if (nodes == nullptr) {
    std::vector<float> tmp(n);
    for (int k = 0; k < n; k++) tmp[k] = vals[(size_t)k * stride];
    NGPU_CUDA(cudaMemcpyAsync(base + i0, tmp.data(), sizeof(float) * n,
                              cudaMemcpyHostToDevice, stream_));
    NGPU_CUDA(cudaStreamSynchronize(stream_));
  } else {
    int *d_idx = nullptr;
    float *d_vals = nullptr;
    NGPU_CUDA(cudaMalloc(&d_idx, sizeof(int) * n));
    NGPU_CUDA(cudaMemcpyAsync(d_idx, nodes, sizeof(int) * n, cudaMemcpyHostToDevice, stream_));
    if (vals) {
      std::vector<float> tmp(n);
      for (int k = 0; k < n; k++) tmp[k] = vals[(size_t)k * stride];
      NGPU_CUDA(cudaMalloc(&d_vals, sizeof(float) * n));
      NGPU_CUDA(cudaMemcpyAsync(d_vals, tmp.data(), sizeof(float) * n,
                                cudaMemcpyHostToDevice, stream_));
    }
    LaunchScatterFloat(base, d_idx, n, val, d_vals, 1, stream_);
    NGPU_CUDA(cudaStreamSynchronize(stream_));
    cudaFree(d_idx);
    if (d_vals) cudaFree(d_vals);
  }
  NGPU_CUDA(cudaStreamSynchronize(stream_));
  // captured step graphs hold the uniform values (and which columns are
  // per-neuron) as kernel arguments; per-neuron columns are read from device
  // memory, so the graphs stay valid unless that information changed
  if (g->p_uniform[col] != old_uniform || (g->p_uniform[col] && g->p_uval[col] != old_uval))
    InvalidateGraphs();
}

void NeuronGPU::GetParamColumn(NodeGroup *g, float *col_base, int i0, int n,
                               const int *nodes, float *out, int stride) {
  (void)g;
  std::vector<float> tmp(n);
  if (nodes == nullptr) {
    NGPU_CUDA(cudaMemcpyAsync(tmp.data(), col_base + i0, sizeof(float) * n,
                              cudaMemcpyDeviceToHost, stream_));
  } else {
    int *d_idx = nullptr;
    float *d_out = nullptr;
    NGPU_CUDA(cudaMalloc(&d_idx, sizeof(int) * n));
    NGPU_CUDA(cudaMalloc(&d_out, sizeof(float) * n));
    NGPU_CUDA(cudaMemcpyAsync(d_idx, nodes, sizeof(int) * n, cudaMemcpyHostToDevice, stream_));
    LaunchGatherFloat(col_base, d_idx, n, d_out, 1, stream_);
    NGPU_CUDA(cudaMemcpyAsync(tmp.data(), d_out, sizeof(float) * n,
                              cudaMemcpyDeviceToHost, stream_));
    NGPU_CUDA(cudaStreamSynchronize(stream_));
    cudaFree(d_idx);
    cudaFree(d_out);
  }
  NGPU_CUDA(cudaStreamSynchronize(stream_));
  for (int k = 0; k < n; k++) out[(size_t)k * stride] = tmp[k];
}

static void check_local(NodeGroup *g, const std::vector<int> &loc) {
  for (int v : loc)
    if (v < 0 || v >= g->n_node) throw ngpu_exception("Neuron index out of range");
}

int NeuronGPU::SetNeuronParam(int i_node, int n, const std::string &name, float val) {
  int il;
  NodeGroup *g = GroupOf(i_node, n, il);
  if (g->mi->kind == MK_POISSON_NODES)
    throw ngpu_exception(std::string("Unrecognized scalar parameter ") + name);
  int j = g->ScalParamIdx(name);
  if (j < 0) throw ngpu_exception(std::string("Unrecognized scalar parameter ") + name);
  SetParamColumn(g, j, il, n, nullptr, val, nullptr, 1);
  return 0;
}

int NeuronGPU::SetNeuronParam(const int *nodes, int n, const std::string &name, float val) {
  std::vector<int> loc;
  NodeGroup *g = GroupOfList(nodes, n, loc);
  int j = g->ScalParamIdx(name);
  if (j < 0) throw ngpu_exception(std::string("Unrecognized scalar parameter ") + name);
  SetParamColumn(g, j, 0, n, loc.data(), val, nullptr, 1);
  return 0;
}

int NeuronGPU::SetNeuronParam(int i_node, int n, const std::string &name,
                              const float *arr, int size) {
  int il;
  NodeGroup *g = GroupOf(i_node, n, il);
  int k = g->PortParamIdx(name);
  if (k >= 0) {
    if (size != g->n_port)
      throw ngpu_exception("Parameter array size must be equal to the number of ports.");
    for (int p = 0; p < g->n_port; p++)
      SetParamColumn(g, g->NSP() + p * g->NPP() + k, il, n, nullptr, arr[p], nullptr, 1);
    return 0;
  }
  if (g->ArrayParamIdx(name) >= 0) {
    if (g->mi->kind != MK_SPIKE_GENERATOR)
      throw ngpu_exception(std::string("Unrecognized array parameter ") + name);
    CheckUncalibrated("Spike generator array parameters must be set before calibration");
    for (int i = il; i < il + n; i++) {
      if (name == "spike_times") g->sg_times[i].assign(arr, arr + size);
      else g->sg_heights[i].assign(arr, arr + size);
    }
    return 0;
  }
  throw ngpu_exception(std::string("Unrecognized array parameter ") + name);
}

int NeuronGPU::SetNeuronParam(const int *nodes, int n, const std::string &name,
                              const float *arr, int size) {
  std::vector<int> loc;
  NodeGroup *g = GroupOfList(nodes, n, loc);
  int k = g->PortParamIdx(name);
  if (k >= 0) {
    if (size != g->n_port)
      throw ngpu_exception("Parameter array size must be equal to the number of ports.");
    for (int p = 0; p < g->n_port; p++)
      SetParamColumn(g, g->NSP() + p * g->NPP() + k, 0, n, loc.data(), arr[p], nullptr, 1);
    return 0;
  }
  if (g->ArrayParamIdx(name) >= 0 && g->mi->kind == MK_SPIKE_GENERATOR) {
    CheckUncalibrated("Spike generator array parameters must be set before calibration");
    for (int i : loc) {
      if (name == "spike_times") g->sg_times[i].assign(arr, arr + size);
      else g->sg_heights[i].assign(arr, arr + size);
    }
    return 0;
  }
  throw ngpu_exception(std::string("Unrecognized array parameter ") + name);
}

int NeuronGPU::IsNeuronScalParam(int i_node, const std::string &n) {
  int il; NodeGroup *g = GroupOf(i_node, 1, il);
  return g->ScalParamIdx(n) >= 0;
}
int NeuronGPU::IsNeuronPortParam(int i_node, const std::string &n) {
  int il; NodeGroup *g = GroupOf(i_node, 1, il);
  return g->PortParamIdx(n) >= 0;
}
int NeuronGPU::IsNeuronArrayParam(int i_node, const std::string &n) {
  int il; NodeGroup *g = GroupOf(i_node, 1, il);
  return g->ArrayParamIdx(n) >= 0;
}
int NeuronGPU::IsNeuronGroupParam(int i_node, const std::string &n) {
  int il; NodeGroup *g = GroupOf(i_node, 1, il);
  return g->GroupParamIdx(n) >= 0 || (g->mi->kind == MK_RK5 && n == "rk5_eps");
}
int NeuronGPU::IsNeuronIntVar(int i_node, const std::string &n) {
  int il; NodeGroup *g = GroupOf(i_node, 1, il);
  return g->IntVarIdx(n) >= 0;
}
int NeuronGPU::IsNeuronScalVar(int i_node, const std::string &n) {
  int il; NodeGroup *g = GroupOf(i_node, 1, il);
  return g->ScalVarIdx(n) >= 0;
}
int NeuronGPU::IsNeuronPortVar(int i_node, const std::string &n) {
  int il; NodeGroup *g = GroupOf(i_node, 1, il);
  return g->PortVarIdx(n) >= 0;
}
int NeuronGPU::IsNeuronArrayVar(int i_node, const std::string &n) {
  int il; GroupOf(i_node, 1, il);
  (void)n;
  return 0;
}

int NeuronGPU::GetNeuronParamSize(int i_node, const std::string &n) {
  int il; NodeGroup *g = GroupOf(i_node, 1, il);
  if (g->ArrayParamIdx(n) >= 0) {
    return (int)(n == "spike_times" ? g->sg_times[il].size() : g->sg_heights[il].size());
  }
  if (g->ScalParamIdx(n) >= 0) return 1;
  if (g->PortParamIdx(n) >= 0) return g->n_port;
  throw ngpu_exception(std::string("Unrecognized parameter ") + n);
}

int NeuronGPU::GetNeuronVarSize(int i_node, const std::string &n) {
  int il; NodeGroup *g = GroupOf(i_node, 1, il);
  if (g->ScalVarIdx(n) >= 0 || g->IntVarIdx(n) >= 0) return 1;
  if (g->PortVarIdx(n) >= 0) return g->n_port;
  throw ngpu_exception(std::string("Unrecognized variable ") + n);
}

// Returned arrays are malloc'd and owned by the caller, as in
// src/base_neuron.cu:446-471.
float *NeuronGPU::GetNeuronParam(int i_node, int n, const std::string &name) {
  int il; NodeGroup *g = GroupOf(i_node, n, il);
  int j = g->ScalParamIdx(name);
  if (j >= 0) {
    float *out = (float *)malloc(sizeof(float) * n);
    GetParamColumn(g, g->d_param + (size_t)j * g->n_pad, il, n, nullptr, out, 1);
    return out;
  }
  int k = g->PortParamIdx(name);
  if (k >= 0) {
    float *out = (float *)malloc(sizeof(float) * (size_t)n * g->n_port);
    for (int p = 0; p < g->n_port; p++)
      GetParamColumn(g, g->d_param + (size_t)(g->NSP() + p * g->NPP() + k) * g->n_pad,
                     il, n, nullptr, out + p, g->n_port);
    return out;
  }
  if (g->ArrayParamIdx(name) >= 0) {
    if (n != 1) throw ngpu_exception("Cannot get array parameters for more than one node at a time");
    return GetArrayParam(i_node, name);
  }
  throw ngpu_exception(std::string("Unrecognized parameter ") + name);
}

float *NeuronGPU::GetNeuronParam(const int *nodes, int n, const std::string &name) {
  std::vector<int> loc;
  NodeGroup *g = GroupOfList(nodes, n, loc);
  int j = g->ScalParamIdx(name);
  if (j >= 0) {
    float *out = (float *)malloc(sizeof(float) * n);
    GetParamColumn(g, g->d_param + (size_t)j * g->n_pad, 0, n, loc.data(), out, 1);
    return out;
  }
  int k = g->PortParamIdx(name);
  if (k >= 0) {
    float *out = (float *)malloc(sizeof(float) * (size_t)n * g->n_port);
    for (int p = 0; p < g->n_port; p++)
      GetParamColumn(g, g->d_param + (size_t)(g->NSP() + p * g->NPP() + k) * g->n_pad,
                     0, n, loc.data(), out + p, g->n_port);
    return out;
  }
  if (g->ArrayParamIdx(name) >= 0) {
    if (n != 1) throw ngpu_exception("Cannot get array parameters for more than one node at a time");
    return GetArrayParam(nodes[0], name);
  }
  throw ngpu_exception(std::string("Unrecognized parameter ") + name);
}

float *NeuronGPU::GetArrayParam(int i_node, const std::string &name) {
  int il; NodeGroup *g = GroupOf(i_node, 1, il);
  if (g->ArrayParamIdx(name) < 0 || g->mi->kind != MK_SPIKE_GENERATOR)
    throw ngpu_exception(std::string("Unrecognized parameter ") + name);
  std::vector<float> &v = (name == "spike_times") ? g->sg_times[il] : g->sg_heights[il];
  float *out = (float *)malloc(sizeof(float) * (v.size() > 0 ? v.size() : 1));
  for (size_t k = 0; k < v.size(); k++) out[k] = v[k];
  return out;
}

int NeuronGPU::SetNeuronIntVar(int i_node, int n, const std::string &name, int val) {
  int il; NodeGroup *g = GroupOf(i_node, n, il);
  int j = g->IntVarIdx(name);
  if (j < 0) throw ngpu_exception(std::string("Unrecognized integer variable ") + name);
  int *base = (g->int_var_names[j] == "spike_count") ? g->d_spike_count : g->d_n_rec;
  LaunchFillInt(base + il, n, val, stream_);
  NGPU_CUDA(cudaStreamSynchronize(stream_));
  return 0;
}

int NeuronGPU::SetNeuronIntVar(const int *nodes, int n, const std::string &name, int val) {
  std::vector<int> loc;
  NodeGroup *g = GroupOfList(nodes, n, loc);
  int j = g->IntVarIdx(name);
  if (j < 0) throw ngpu_exception(std::string("Unrecognized integer variable ") + name);
  int *base = (g->int_var_names[j] == "spike_count") ? g->d_spike_count : g->d_n_rec;
  for (int v : loc) NGPU_CUDA(cudaMemcpy(base + v, &val, sizeof(int), cudaMemcpyHostToDevice));
  return 0;
}

int NeuronGPU::SetNeuronVar(int i_node, int n, const std::string &name, float val) {
  FlushInput();
  int il; NodeGroup *g = GroupOf(i_node, n, il);
  int j = g->ScalVarIdx(name);
  if (j < 0) throw ngpu_exception(std::string("Unrecognized scalar variable ") + name);
  LaunchFillFloat(g->d_var + (size_t)j * g->n_pad + il, n, val, stream_);
  NGPU_CUDA(cudaStreamSynchronize(stream_));
  return 0;
}

int NeuronGPU::SetNeuronVar(const int *nodes, int n, const std::string &name, float val) {
  FlushInput();
  std::vector<int> loc;
  NodeGroup *g = GroupOfList(nodes, n, loc);
  int j = g->ScalVarIdx(name);
  if (j < 0) throw ngpu_exception(std::string("Unrecognized scalar variable ") + name);
  int *d_idx;
  NGPU_CUDA(cudaMalloc(&d_idx, sizeof(int) * n));
  NGPU_CUDA(cudaMemcpy(d_idx, loc.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
  LaunchScatterFloat(g->d_var + (size_t)j * g->n_pad, d_idx, n, val, nullptr, 1, stream_);
  NGPU_CUDA(cudaStreamSynchronize(stream_));
  cudaFree(d_idx);
  return 0;
}

int NeuronGPU::SetNeuronVar(int i_node, int n, const std::string &name,
                            const float *arr, int size) {
  FlushInput();
  int il; NodeGroup *g = GroupOf(i_node, n, il);
  int k = g->PortVarIdx(name);
  if (k < 0) throw ngpu_exception(std::string("Unrecognized port variable ") + name);
  if (size != g->n_port)
    throw ngpu_exception("Variable array size must be equal to the number of ports.");
  for (int p = 0; p < g->n_port; p++)
    LaunchFillFloat(g->d_var + (size_t)(g->NSV() + p * g->NPV() + k) * g->n_pad + il, n,
                    arr[p], stream_);
  NGPU_CUDA(cudaStreamSynchronize(stream_));
  return 0;
}

int NeuronGPU::SetNeuronVar(const int *nodes, int n, const std::string &name,
                            const float *arr, int size) {
  FlushInput();
  std::vector<int> loc;
  NodeGroup *g = GroupOfList(nodes, n, loc);
  int k = g->PortVarIdx(name);
  if (k < 0) throw ngpu_exception(std::string("Unrecognized port variable ") + name);
  if (size != g->n_port)
    throw ngpu_exception("Variable array size must be equal to the number of ports.");
  int *d_idx;
  NGPU_CUDA(cudaMalloc(&d_idx, sizeof(int) * n));
  NGPU_CUDA(cudaMemcpy(d_idx, loc.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
  for (int p = 0; p < g->n_port; p++)
    LaunchScatterFloat(g->d_var + (size_t)(g->NSV() + p * g->NPV() + k) * g->n_pad, d_idx,
                       n, arr[p], nullptr, 1, stream_);
  NGPU_CUDA(cudaStreamSynchronize(stream_));
  cudaFree(d_idx);
  return 0;
}

int *NeuronGPU::GetNeuronIntVar(int i_node, int n, const std::string &name) {
  int il; NodeGroup *g = GroupOf(i_node, n, il);
  int j = g->IntVarIdx(name);
  if (j < 0) throw ngpu_exception(std::string("Unrecognized integer variable ") + name);
  int *base = (g->int_var_names[j] == "spike_count") ? g->d_spike_count : g->d_n_rec;
  int *out = (int *)malloc(sizeof(int) * n);
  NGPU_CUDA(cudaMemcpy(out, base + il, sizeof(int) * n, cudaMemcpyDeviceToHost));
  return out;
}

int *NeuronGPU::GetNeuronIntVar(const int *nodes, int n, const std::string &name) {
  std::vector<int> loc;
  NodeGroup *g = GroupOfList(nodes, n, loc);
  int j = g->IntVarIdx(name);
  if (j < 0) throw ngpu_exception(std::string("Unrecognized variable ") + name);
  int *base = (g->int_var_names[j] == "spike_count") ? g->d_spike_count : g->d_n_rec;
  int *out = (int *)malloc(sizeof(int) * n);
  if (n == 0) return out;
  // one copy of the span the list covers, then a host-side pick
  auto mm = std::minmax_element(loc.begin(), loc.end());
  std::vector<int> span((size_t)(*mm.second - *mm.first) + 1);
  NGPU_CUDA(cudaMemcpy(span.data(), base + *mm.first, sizeof(int) * span.size(),
                       cudaMemcpyDeviceToHost));
  for (int k = 0; k < n; k++) out[k] = span[loc[k] - *mm.first];
  return out;
}

float *NeuronGPU::GetNeuronVar(int i_node, int n, const std::string &name) {
  FlushInput();
  int il; NodeGroup *g = GroupOf(i_node, n, il);
  int j = g->ScalVarIdx(name);
  if (j >= 0) {
    float *out = (float *)malloc(sizeof(float) * n);
    GetParamColumn(g, g->d_var + (size_t)j * g->n_pad, il, n, nullptr, out, 1);
    return out;
  }
  int k = g->PortVarIdx(name);
  if (k >= 0) {
    float *out = (float *)malloc(sizeof(float) * (size_t)n * g->n_port);
    for (int p = 0; p < g->n_port; p++)
      GetParamColumn(g, g->d_var + (size_t)(g->NSV() + p * g->NPV() + k) * g->n_pad,
                     il, n, nullptr, out + p, g->n_port);
    return out;
  }
  throw ngpu_exception(std::string("Unrecognized variable ") + name);
}

float *NeuronGPU::GetNeuronVar(const int *nodes, int n, const std::string &name) {
  FlushInput();
  std::vector<int> loc;
  NodeGroup *g = GroupOfList(nodes, n, loc);
  int j = g->ScalVarIdx(name);
  if (j >= 0) {
    float *out = (float *)malloc(sizeof(float) * n);
    GetParamColumn(g, g->d_var + (size_t)j * g->n_pad, 0, n, loc.data(), out, 1);
    return out;
  }
  int k = g->PortVarIdx(name);
  if (k >= 0) {
    float *out = (float *)malloc(sizeof(float) * (size_t)n * g->n_port);
    for (int p = 0; p < g->n_port; p++)
      GetParamColumn(g, g->d_var + (size_t)(g->NSV() + p * g->NPV() + k) * g->n_pad,
                     0, n, loc.data(), out + p, g->n_port);
    return out;
  }
  throw ngpu_exception(std::string("Unrecognized variable ") + name);
}

float *NeuronGPU::GetArrayVar(int i_node, const std::string &name) {
  int il; GroupOf(i_node, 1, il);
  throw ngpu_exception(std::string("Unrecognized array variable ") + name);
}

int NeuronGPU::SetNeuronGroupParam(int i_node, int n, const std::string &name, float val) {
  int il; NodeGroup *g = GroupOf(i_node, n, il);
  if (il != 0 || n != g->n_node)
    throw ngpu_exception("Group parameters must be set for all the nodes of a group");
  if (g->mi->kind == MK_RK5 && name == "rk5_eps") {
    if (!(val > 0.0f)) throw ngpu_exception("rk5_eps must be > 0");
    g->rk5_eps = val;
    InvalidateGraphs();
    return 0;
  }
  int j = g->GroupParamIdx(name);
  if (j < 0) throw ngpu_exception(std::string("Unrecognized group parameter ") + name);
  g->group_param[j] = val;
  InvalidateGraphs();
  return 0;
}

float NeuronGPU::GetNeuronGroupParam(int i_node, const std::string &name) {
  int il; NodeGroup *g = GroupOf(i_node, 1, il);
  if (g->mi->kind == MK_RK5 && name == "rk5_eps") return g->rk5_eps;
  int j = g->GroupParamIdx(name);
  if (j < 0) throw ngpu_exception(std::string("Unrecognized group parameter ") + name);
  return g->group_param[j];
}

std::vector<std::string> NeuronGPU::GetIntVarNames(int i_node) {
  int il; return GroupOf(i_node, 1, il)->int_var_names;
}
std::vector<std::string> NeuronGPU::GetScalVarNames(int i_node) {
  int il; return GroupOf(i_node, 1, il)->mi->scal_var;
}
std::vector<std::string> NeuronGPU::GetPortVarNames(int i_node) {
  int il; return GroupOf(i_node, 1, il)->mi->port_var;
}
std::vector<std::string> NeuronGPU::GetScalParamNames(int i_node) {
  int il; return GroupOf(i_node, 1, il)->mi->scal_param;
}
std::vector<std::string> NeuronGPU::GetPortParamNames(int i_node) {
  int il; return GroupOf(i_node, 1, il)->mi->port_param;
}
std::vector<std::string> NeuronGPU::GetGroupParamNames(int i_node) {
  int il; return GroupOf(i_node, 1, il)->mi->group_param;
}
std::vector<std::string> NeuronGPU::GetArrayParamNames(int i_node) {
  int il; return GroupOf(i_node, 1, il)->mi->array_param;
}
std::vector<std::string> NeuronGPU::GetArrayVarNames(int i_node) {
  int il; GroupOf(i_node, 1, il);
  return std::vector<std::string>();
}

// ---------------------------------------------------------------------------
// recording
// ---------------------------------------------------------------------------
int NeuronGPU::CreateRecord(const std::string &file, const std::vector<std::string> &vars,
                            const int *nodes, const int *ports, int n) {
  if (calibrate_flag_ && !first_simulation_flag_)
    throw ngpu_exception("Records cannot be created after the simulation started");
  Record r;
  r.file_name = file;
  r.var_names = vars;
  for (int k = 0; k < n; k++) {
    int il;
    NodeGroup *g = GroupOf(nodes[k], 1, il);
    int port = ports ? ports[k] : 0;
    if (vars[k] != "spike") {
      if (g->ScalVarIdx(vars[k]) < 0 && g->PortVarIdx(vars[k]) < 0 &&
          g->ScalParamIdx(vars[k]) < 0 && g->PortParamIdx(vars[k]) < 0)
        throw ngpu_exception(std::string("Unrecognized variable ") + vars[k]);
      if ((g->PortVarIdx(vars[k]) >= 0 || g->PortParamIdx(vars[k]) >= 0) &&
          (port < 0 || port >= g->n_port))
        throw ngpu_exception("Port index out of range in record");
    }
    r.nodes.push_back(nodes[k]);
    r.ports.push_back(port);
  }
  records_.push_back(r);
  return (int)records_.size() - 1;
}

std::vector<std::vector<float>> *NeuronGPU::GetRecordData(int i_record) {
  if (i_record < 0 || i_record >= (int)records_.size())
    throw ngpu_exception("Record does not exist.");
  FlushRecords();
  return &records_[i_record].data;
}

int NeuronGPU::ActivateSpikeCount(int i_node, int n) {
  CheckUncalibrated("Spike count must be activated before calibration");
  int il; NodeGroup *g = GroupOf(i_node, n, il);
  if (il != 0 || n != g->n_node)
    throw ngpu_exception("Spike count must be activated for all and only the nodes of the same group");
  if (g->IntVarIdx("spike_count") >= 0) throw ngpu_exception("Spike count already activated");
  g->int_var_names.push_back("spike_count");
  NGPU_CUDA(cudaMalloc(&g->d_spike_count, sizeof(int) * g->n_pad));
  NGPU_CUDA(cudaMemset(g->d_spike_count, 0, sizeof(int) * g->n_pad));
  return 0;
}

int NeuronGPU::ActivateRecSpikeTimes(int i_node, int n, int max_n) {
  CheckUncalibrated("Spike time recording must be activated before calibration");
  int il; NodeGroup *g = GroupOf(i_node, n, il);
  if (il != 0 || n != g->n_node)
    throw ngpu_exception("Spike count must be activated for all and only the nodes of the same group");
  if (max_n <= 0) throw ngpu_exception("Maximum number of recorded spike times must be greater than 0");
  if (g->IntVarIdx("n_rec_spike_times") >= 0)
    throw ngpu_exception("Spike times recording already activated");
  g->int_var_names.push_back("n_rec_spike_times");
  g->max_rec = max_n;
  NGPU_CUDA(cudaMalloc(&g->d_n_rec, sizeof(int) * g->n_pad));
  NGPU_CUDA(cudaMemset(g->d_n_rec, 0, sizeof(int) * g->n_pad));
  NGPU_CUDA(cudaMalloc(&g->d_rec_times, sizeof(float) * (size_t)g->n_pad * max_n));
  return 0;
}

int NeuronGPU::GetNRecSpikeTimes(int i_node) {
  int il; NodeGroup *g = GroupOf(i_node, 1, il);
  if (g->d_n_rec == nullptr) throw ngpu_exception("Spike times recording was not activated");
  int v = 0;
  NGPU_CUDA(cudaMemcpy(&v, g->d_n_rec + il, sizeof(int), cudaMemcpyDeviceToHost));
  return v;
}

std::vector<float> NeuronGPU::GetRecSpikeTimes(int i_node) {
  int il; NodeGroup *g = GroupOf(i_node, 1, il);
  int n = GetNRecSpikeTimes(i_node);
  std::vector<float> v(n);
  if (n > 0)
    NGPU_CUDA(cudaMemcpy(v.data(), g->d_rec_times + (size_t)il * g->max_rec,
                         sizeof(float) * n, cudaMemcpyDeviceToHost));
  return v;
}

// ---------------------------------------------------------------------------
// argument builders
// ---------------------------------------------------------------------------
// propagator from an exponential current to the membrane potential
// (src/iaf_psc_exp_g.cu:68-88): the exact expression, or its limit when the
// two time constants (nearly) coincide
static double propagator_32(double tau_syn, double tau, double C, double h) {
  const double P32_linear = 1.0 / (2.0 * C * tau * tau) * h * h * (tau_syn - tau) * exp(-h / tau);
  const double P32_singular = h / C * exp(-h / tau);
  const double P32 = -tau / (C * (1.0 - tau / tau_syn)) * exp(-h / tau_syn)
                     * expm1(h * (1.0 / tau_syn - 1.0 / tau));
  const double dev = fabs(P32 - P32_singular);
  if (tau == tau_syn || (fabs(tau - tau_syn) < 0.1 && dev > 2.0 * fabs(P32_linear)))
    return P32_singular;
  return P32;
}

// constants of the non-RK5 models that the reference computes from the group
// parameters at every update, in the reference's float / double mix
// (src/iaf_psc_exp_g.cu:143-150, src/izhikevich.cu:140-146,
// src/izhikevich_psc_exp_2s.cu:145-152)
static void group_constants(const NodeGroup *g, float dt, float *gc) {
  const ModelInfo *mi = g->mi;
  for (int k = 0; k < 8; k++) gc[k] = 0.0f;
  if (mi->kind == MK_IAF_PSC_EXP_G) {
    // iaf_psc_exp_hc: iaf_psc_exp_g's defaults at dt = 0.1 ms, whatever the
    // time resolution (src/iaf_psc_exp_hc_params.h)
    float h = dt, tau_m = 10.0f, C_m = 250.0f, Theta = 15.0f, V_reset = 0.0f;
    float tau_syn = 0.5f, t_ref = 2.0f;
    if (mi->hard_coded) {
      h = 0.1f;
    } else {
      tau_m = g->group_param[0]; C_m = g->group_param[1];
      Theta = g->group_param[3]; V_reset = g->group_param[4];
      tau_syn = g->group_param[5]; t_ref = g->group_param[6];
    }
    const float P22 = (float)exp((double)(-h / tau_m));
    gc[0] = (float)exp((double)(-h / tau_syn));
    gc[1] = P22;
    gc[2] = (float)propagator_32(tau_syn, tau_m, C_m, h);
    gc[3] = (float)(tau_m / C_m * (1.0 - (double)P22));
    gc[4] = Theta;
    gc[5] = V_reset;
    gc[6] = (float)(int)round((double)(t_ref / h));
  } else if (mi->kind == MK_IZHIKEVICH || mi->kind == MK_IZH_PSC_EXP) {
    const float h = dt / (float)mi->n_sub;
    for (int k = 0; k < 5; k++) gc[k] = g->group_param[k];   // V_th, a, b, c, d
    const float t_ref = g->group_param[mi->kind == MK_IZHIKEVICH ? 5 : 6];
    gc[5] = (float)(int)round((double)(t_ref / h));
    gc[6] = h;
    if (mi->kind == MK_IZH_PSC_EXP) gc[7] = (float)exp((double)(-h / g->group_param[5]));
  }
}

GroupArgs NeuronGPU::MakeGroupArgs(NodeGroup *g) {
  GroupArgs a;
  memset(&a, 0, sizeof(a));
  a.n = g->n_node;
  a.n_pad = g->n_pad;
  a.i_node_0 = g->i_node_0;
  a.nvar = g->nvar;
  a.nparam = g->nparam;
  a.var = g->d_var;
  a.param = g->d_param;
  a.h = g->d_h;
  a.dx = g->d_dx;
  a.all_uniform = 1;
  for (int j = 0; j < g->nparam; j++) {
    bool per_neuron = !g->p_uniform[j] || j == g->mi->refr_param;
    if (per_neuron) a.pmask[j >> 5] |= (1u << (j & 31));
    if (!g->p_uniform[j] && j != g->mi->refr_param) a.all_uniform = 0;
    a.puni[j] = g->p_uval[j];
    // reciprocals for the RK5 right-hand sides (IEEE float division, the
    // same value the kernel forms for per-neuron parameters)
    volatile float one = 1.0f;
    a.pinv[j] = one / g->p_uval[j];
  }
  if (g->mi->kind == MK_RK5) {
    a.h_min = g->group_param[0] * time_resolution_;
    {
      // the reference's escape test h <= h_min * (1.0 + 1.0e-5) is a double
      // comparison of the float h: the same as h <= the largest float that
      // does not exceed the double threshold
      const double thr = (double)a.h_min * (1.0 + 1.0e-5);
      float f = (float)thr;
      if ((double)f > thr) f = nextafterf(f, 0.0f);
      a.h_min_thr = f;
    }
    a.eps = g->rk5_eps;
    volatile float one = 1.0f;
    a.inv_eps = one / g->rk5_eps;
  }
  a.dt = time_resolution_;
  a.max_substeps = rk5_max_substeps_;
  a.wait_test = wait_test_;
  // the dendritic delay in steps as the update kernels round it, formed once
  // here for a group-wide value (IEEE float division, then roundf)
  if (g->mi->den_delay_param >= 0) {
    volatile float den = g->p_uval[g->mi->den_delay_param];
    a.den_steps = (int)roundf(den / time_resolution_);
  }
  group_constants(g, time_resolution_, a.gc);
  a.variant = g->rk5_variant;
  a.dry = 0;
  a.den_delay_col = g->mi->den_delay_param;
  a.blk_evals = g->d_blk_evals;
  a.q = g->q;
  // the learned proposer runs in the queue's finishing launch: queue kept on
  if (g->queue_off && g->step_mode != STEP_LEARNED) a.q.cap = 0;
  a.step_mode = g->step_mode;
  a.mlp_margin = mlp_margin_;
  a.mlp = d_mlp_img_;
  a.log_buf = g->d_log_buf;
  a.log_count = g->d_log_count;
  a.log_cap = g->log_cap;
  if (a.step_mode == STEP_LEARNED && a.mlp == nullptr)
    throw ngpu_exception("the learned step proposer has no parameters (train or set them first)");
  a.sg_off = g->d_sg_off;
  a.sg_step = g->d_sg_step;
  a.sg_height = g->d_sg_height;
  a.sg_next = g->d_sg_next;
  return a;
}

InputArgs NeuronGPU::MakeInputArgs(NodeGroup *g) {
  InputArgs in;
  memset(&in, 0, sizeof(in));
  const ModelInfo *mi = g->mi;
  in.acc = d_acc_;
  in.acc_base = g->acc_base;
  in.acc_par = n_acc_ > 0 ? n_acc_ : 1;
  in.acc_slots = acc_slots_;
  in.acc_stamp = d_acc_stamp_;
  in.np = g->n_port;
  if (mi->kind == MK_RK5) {
    in.in_var = mi->in_var - (mi->port_var.empty() ? 0 : 0);
  }
  in.in_var = mi->in_var;
  in.in_step = mi->in_step;
  in.w_param = mi->w_param ? 1 : 0;
  in.w_col = mi->w_param ? (int)mi->scal_param.size() + mi->w_param_idx : 0;
  in.w_col_step = (int)mi->port_param.size();
  for (int q = 0; q < 4; q++) {
    if (mi->w_const.empty()) in.w_const[q] = 1.0f;
    else in.w_const[q] = mi->w_const[q < (int)mi->w_const.size() ? q : mi->w_const.size() - 1];
  }
  if (g->has_dc) {
    in.dc_off = g->d_dc_off;
    in.dc_gen = d_dc_gen_;
    in.dc_port = d_dc_port_;
    in.dc_weight = d_dc_w_;
    in.dc_delay = d_dc_delay_;
    in.dc_stream = d_dc_stream_;
    in.gen_rate = d_gen_rate_;
    in.gen_origin = d_gen_origin_;
    in.gen_start = d_gen_start_;
    in.gen_stop = d_gen_stop_;
    in.gen_lambda = d_gen_lambda_;
    in.gen_explam = d_gen_explam_;
    in.gen_thr = d_gen_thr_;
  }
  if (g->ud && g->ud_gen < (int)gen_lam_h_.size()) {
    const int k = g->ud_gen;
    in.ud = 1;
    in.ud_port = g->ud_port;
    in.ud_w = g->ud_w;
    in.ud_delay = g->ud_delay;
    in.ud_origin = gen_origin_h_[k];
    in.ud_start = gen_start_h_[k];
    in.ud_stop = gen_stop_h_[k];
    in.ud_lambda = gen_lam_h_[k];
    in.ud_explam = gen_explam_h_[k];
    in.ud_thr = d_gen_thr_ + (size_t)k * NGPU_CDF_LEN;
    for (int j = 0; j < 8; j++) in.ud_thr8[j] = gen_thr_h_[(size_t)k * NGPU_CDF_LEN + j];
    in.ud_stream0 = g->ud_stream0;
  }
  in.seed = kernel_seed_;
  return in;
}

// Whether Poisson direct connections into group g may draw
// NGPU_POISSON_INV_MAX or more expected spikes per step; the update kernels
// of RK5 neurons, simple-model neurons and parrots leave those to
// LaunchPoissonLarge. Generator rates change only
// between simulation calls and a change re-captures the step graphs, so the
// answer holds for every step of a captured graph.
bool NeuronGPU::HasLargePoisson(const NodeGroup *g) const {
  if (g->ud && g->ud_gen >= 0 && g->ud_gen < (int)gen_lam_h_.size())
    return gen_lam_h_[g->ud_gen] >= NGPU_POISSON_INV_MAX;
  if (!g->has_dc) return false;
  for (double lam : gen_lam_h_) {
    if (lam >= NGPU_POISSON_INV_MAX) return true;
  }
  return false;
}

PushArgs NeuronGPU::MakePushArgs(NodeGroup *g) {
  PushArgs pa;
  memset(&pa, 0, sizeof(pa));
  pa.ring_src = d_ring_src_;
  pa.ring_h = d_ring_h_;
  pa.ring_cnt = d_ring_cnt_;
  pa.ring_R = ring_R_;
  pa.ring_C = ring_C_;
  pa.last_spike_T = d_last_spike_T_;
  pa.last_spike_h = d_last_spike_h_;
  pa.last_rev_T = d_last_rev_T_;
  pa.spike_count = g->d_spike_count;
  pa.rec_times = g->d_rec_times;
  pa.n_rec = g->d_n_rec;
  pa.max_rec = g->max_rec;
  pa.rev_src = d_rev_src_;
  pa.rev_cnt = d_rev_cnt_;
  pa.rev_R = rev_R_;
  pa.rev_C = rev_C_;
  return pa;
}

DeliverArgs NeuronGPU::MakeDeliverArgs() {
  DeliverArgs d;
  memset(&d, 0, sizeof(d));
  d.grp_off = d_grp_off_;
  d.e_slot = d_e_slot_;
  d.e_w = d_e_w_;
  d.e_syn = plastic_ ? d_e_syn_ : nullptr;
  d.e_stamp = d_e_stamp_;
  d.e_post = d_e_post_;
  d.acc = d_acc_;
  d.acc_par = n_acc_ > 0 ? n_acc_ : 1;
  d.acc_slots = acc_slots_;
  d.acc_stamp = d_acc_stamp_;
  d.ring_src = d_ring_src_;
  d.ring_h = d_ring_h_;
  d.ring_cnt = d_ring_cnt_;
  d.ring_R = ring_R_;
  d.ring_C = ring_C_;
  d.nd = (int)delays_.size();
  d.delays = d_delays_;
  d.delay_di = d_delay_di_;
  d.last_rev_T = d_last_rev_T_;
  d.last_post_T = d_last_post_T_;
  d.rev_off = d_rev_off_;
  d.rev_edge = d_rev_edge_;
  d.dt = time_resolution_;
  d.blk_events = d_blk_events_;
  d.step_book = 1;
  d.advance_flags = 0;
  d.ring_cnt_w = d_ring_cnt_;
  d.done = d_done_;
  d.rev_src = d_rev_src_;
  d.rev_cnt = d_rev_cnt_;
  d.rev_R = rev_R_;
  d.rev_C = rev_C_;
  return d;
}

// ---------------------------------------------------------------------------
// calibration (src/neurongpu.cu:277-333)
// ---------------------------------------------------------------------------
int NeuronGPU::Calibrate() {
  CheckUncalibrated("Calibration can be made only once");
  if (groups_.empty()) throw ngpu_exception("No nodes were created");
  if (!stream_) NGPU_CUDA(cudaStreamCreate(&stream_));
  if (verbosity_level_ >= 1) printf("Calibrating ...\n");
  neural_time_ = t_min_;
  BuildCSR();
  BuildDevice();
  calibrate_flag_ = true;
  // the insertion-order edge store is no longer needed
  FreeRaw();
  return 0;
}

// per-group calibration: defaults of derived parameters (g0, I0, iaf
// propagators), initial step sizes and spike generator tables
static void calibrate_group(NodeGroup *g, float dt, cudaStream_t s) {
  const ModelInfo *mi = g->mi;
  if (mi->kind == MK_RK5) {
    GroupArgs a;
    memset(&a, 0, sizeof(a));
    a.n = g->n_node; a.n_pad = g->n_pad; a.param = g->d_param;
    LaunchCalibrateRk5(mi->rk5_model, a, g->n_port, s);
    float h0 = g->group_param[1] * dt;
    LaunchFillFloat(g->d_h, g->n_pad, h0, s);
    LaunchFillFloat(g->d_dx, g->n_pad, 0.0f, s);
    NGPU_CUDA(cudaStreamSynchronize(s));
    // derived parameters: uniform iff their inputs are uniform
    auto derive = [&](int out_col, std::vector<int> in_cols) {
      bool uni = true;
      for (int c : in_cols) uni = uni && g->p_uniform[c];
      g->p_uniform[out_col] = uni ? 1 : 0;
      if (uni) {
        float v;
        NGPU_CUDA(cudaMemcpy(&v, g->d_param + (size_t)out_col * g->n_pad, sizeof(float),
                             cudaMemcpyDeviceToHost));
        g->p_uval[out_col] = v;
      }
    };
    const int NSP = g->NSP(), NPP = g->NPP();
    g->p_uniform[mi->refr_param] = 1;
    g->p_uval[mi->refr_param] = 0.0f;
    for (int q = 0; q < g->n_port; q++) {
      int b = NSP + q * NPP;
      switch (mi->rk5_model) {
        case RK5_AEIF_COND_BETA:
        case RK5_IZHIKEVICH_COND_BETA: derive(b + 3, {b + 1, b + 2}); break;
        case RK5_AEIF_COND_ALPHA: derive(b + 2, {b + 1}); break;
        case RK5_AEIF_PSC_ALPHA: derive(b + 1, {b + 0}); break;
        default: break;
      }
    }
  } else if (mi->kind == MK_IAF_PSC_EXP) {
    GroupArgs a;
    memset(&a, 0, sizeof(a));
    a.n = g->n_node; a.n_pad = g->n_pad; a.param = g->d_param;
    LaunchCalibrateIaf(a, dt, s);
    NGPU_CUDA(cudaStreamSynchronize(s));
    bool uni = g->p_uniform[0] && g->p_uniform[1] && g->p_uniform[6] && g->p_uniform[7];
    for (int c = 10; c <= 15; c++) {
      g->p_uniform[c] = uni ? 1 : 0;
      if (uni) {
        float v;
        NGPU_CUDA(cudaMemcpy(&v, g->d_param + (size_t)c * g->n_pad, sizeof(float),
                             cudaMemcpyDeviceToHost));
        g->p_uval[c] = v;
      }
    }
  } else if (mi->kind == MK_SPIKE_GENERATOR) {
    // spike times -> step indices (src/spike_generator.cu:214-257)
    std::vector<int> off(g->n_node + 1, 0), step;
    std::vector<float> height;
    for (int i = 0; i < g->n_node; i++) {
      std::vector<float> &tv = g->sg_times[i];
      std::vector<float> &hv = g->sg_heights[i];
      if (!tv.empty() && !hv.empty() && hv.size() != tv.size())
        throw ngpu_exception("spike time array and spike height array must have the same size in spike generator");
      int prev = -0x7fffffff;
      for (size_t k = 0; k < tv.size(); k++) {
        int si = (int)round((tv[k] - 0.0f) / dt);
        if (k > 0 && si <= prev)
          throw ngpu_exception("Spike times must be ordered, and the difference between\nconsecutive spikes must be >= the time resolution");
        prev = si;
        step.push_back(si);
        height.push_back(hv.empty() ? 1.0f : hv[k]);
      }
      off[i + 1] = (int)step.size();
    }
    NGPU_CUDA(cudaMalloc(&g->d_sg_off, sizeof(int) * (g->n_node + 1)));
    NGPU_CUDA(cudaMalloc(&g->d_sg_next, sizeof(int) * (g->n_node + 1)));
    NGPU_CUDA(cudaMalloc(&g->d_sg_step, sizeof(int) * (step.size() + 1)));
    NGPU_CUDA(cudaMalloc(&g->d_sg_height, sizeof(float) * (height.size() + 1)));
    NGPU_CUDA(cudaMemcpy(g->d_sg_off, off.data(), sizeof(int) * off.size(), cudaMemcpyHostToDevice));
    NGPU_CUDA(cudaMemcpy(g->d_sg_next, off.data(), sizeof(int) * off.size(), cudaMemcpyHostToDevice));
    if (!step.empty()) {
      NGPU_CUDA(cudaMemcpy(g->d_sg_step, step.data(), sizeof(int) * step.size(), cudaMemcpyHostToDevice));
      NGPU_CUDA(cudaMemcpy(g->d_sg_height, height.data(), sizeof(float) * height.size(), cudaMemcpyHostToDevice));
    }
  }
}

void NeuronGPU::BuildDevice() {
  const long long N = (long long)node_group_map_.size();
  const int nd = (int)delays_.size();
  // accumulator slots
  n_acc_ = 0;
  for (NodeGroup *g : groups_) {
    g->acc_base = n_acc_;
    n_acc_ += (long long)g->n_port * g->n_pad;
  }
  if (n_acc_ > 0xFFFFFFFFLL) throw ngpu_exception("Too many (node, port) input slots");
  // accumulator ring (InputArgs::acc_par, acc_slots): two slots, or, for a
  // network that can run several steps per launch (RK5 neurons and Poisson
  // generators only, no plastic synapse), one slot per step of the longest
  // window + 1 (the delivery before a window fills the slots of all its
  // steps), and no more than the longest delay + 2; at most kWindowAccBytes
  {
    int maxD_acc = 1;
    for (int dly : delays_) maxD_acc = std::max(maxD_acc, dly);
    bool capable = !any_plastic_;
    for (NodeGroup *g : groups_)
      if (g->mi->kind != MK_RK5 && g->mi->kind != MK_POISSON_GENERATOR) capable = false;
    const int slots = std::min(maxD_acc + 2, kWindowMaxSteps + 1);
    const double bytes = (double)slots * 8.0 * (double)(n_acc_ > 0 ? n_acc_ : 1);
    acc_slots_ = (capable && bytes <= kWindowAccBytes) ? slots : 2;
  }
  const size_t acc_bytes = (size_t)acc_slots_ * sizeof(long long) * (n_acc_ > 0 ? n_acc_ : 1);
  NGPU_CUDA(cudaMalloc(&d_acc_, acc_bytes));
  NGPU_CUDA(cudaMemset(d_acc_, 0, acc_bytes));
  NGPU_CUDA(cudaMalloc(&d_acc_stamp_, sizeof(long long) * acc_slots_));
  NGPU_CUDA(cudaMemset(d_acc_stamp_, 0xFF, sizeof(long long) * acc_slots_));   // -1: no step
  // accumulator slot of every CSR edge (device), with the port and
  // synapse-group checks of src/connect.cu:26-62
  const uint64_t E = (uint64_t)n_raw_;
  plastic_ = any_plastic_;
  {
    std::vector<long long> acc_base(groups_.size());
    std::vector<int> n_pad(groups_.size()), i0(groups_.size()), n_port(groups_.size());
    for (size_t gi = 0; gi < groups_.size(); gi++) {
      acc_base[gi] = groups_[gi]->acc_base;
      n_pad[gi] = groups_[gi]->n_pad;
      i0[gi] = groups_[gi]->i_node_0;
      n_port[gi] = groups_[gi]->n_port;
    }
    const size_t G = groups_.size();
    int *d_map = nullptr, *d_npad = nullptr, *d_i0 = nullptr, *d_nport = nullptr;
    long long *d_base = nullptr;
    unsigned *d_err = nullptr;
    NGPU_CUDA(cudaMalloc(&d_map, sizeof(int) * (N > 0 ? N : 1)));
    NGPU_CUDA(cudaMalloc(&d_npad, sizeof(int) * G));
    NGPU_CUDA(cudaMalloc(&d_i0, sizeof(int) * G));
    NGPU_CUDA(cudaMalloc(&d_nport, sizeof(int) * G));
    NGPU_CUDA(cudaMalloc(&d_base, sizeof(long long) * G));
    NGPU_CUDA(cudaMalloc(&d_err, sizeof(unsigned)));
    NGPU_CUDA(cudaMemcpy(d_map, node_group_map_.data(), sizeof(int) * N, cudaMemcpyHostToDevice));
    NGPU_CUDA(cudaMemcpy(d_npad, n_pad.data(), sizeof(int) * G, cudaMemcpyHostToDevice));
    NGPU_CUDA(cudaMemcpy(d_i0, i0.data(), sizeof(int) * G, cudaMemcpyHostToDevice));
    NGPU_CUDA(cudaMemcpy(d_nport, n_port.data(), sizeof(int) * G, cudaMemcpyHostToDevice));
    NGPU_CUDA(cudaMemcpy(d_base, acc_base.data(), sizeof(long long) * G, cudaMemcpyHostToDevice));
    NGPU_CUDA(cudaMemset(d_err, 0, sizeof(unsigned)));
    NGPU_CUDA(cudaMalloc(&d_e_slot_, sizeof(unsigned) * (E > 0 ? E : 1)));
    SlotTables t;
    t.node_group = d_map; t.acc_base = d_base; t.n_pad = d_npad; t.i_node_0 = d_i0;
    t.n_port = d_nport; t.n_syn_groups = (int)syn_groups_.size();
    DevCsrSlots(d_e_post_, d_c_port_, d_e_syn_, (long long)E, t, d_e_slot_, d_err, stream_);
    unsigned err = 0;
    NGPU_CUDA(cudaMemcpyAsync(&err, d_err, sizeof(unsigned), cudaMemcpyDeviceToHost, stream_));
    NGPU_CUDA(cudaStreamSynchronize(stream_));
    cudaFree(d_map); cudaFree(d_npad); cudaFree(d_i0); cudaFree(d_nport); cudaFree(d_base);
    cudaFree(d_err);
    if (err & 4u) throw ngpu_exception("Port index out of range for a target node");
    if (err & 8u) throw ngpu_exception("Unrecognized synapse group");
  }
  std::vector<int> dl(delays_.begin(), delays_.end());
  NGPU_CUDA(cudaMalloc(&d_delays_, sizeof(int) * (nd > 0 ? nd : 1)));
  if (nd > 0) NGPU_CUDA(cudaMemcpy(d_delays_, dl.data(), sizeof(int) * nd, cudaMemcpyHostToDevice));
  if (nd > 0) {
    const int dmax = delays_.back();
    NGPU_CUDA(cudaMalloc(&d_delay_di_, sizeof(int) * (dmax + 1)));
    NGPU_CUDA(cudaMemcpy(d_delay_di_, delay_index_.data(), sizeof(int) * (dmax + 1),
                         cudaMemcpyHostToDevice));
  }
  if (nd > NGPU_MAX_DELAYS) throw ngpu_exception("Too many distinct delays");
  // STDP structures: stamps and per-target incoming plastic lists (the CSR
  // targets d_e_post_ and groups d_e_syn_ are shared with the queries)
  if (plastic_) {
    NGPU_CUDA(cudaMalloc(&d_e_stamp_, sizeof(int) * (E > 0 ? E : 1)));
    LaunchFillInt(d_e_stamp_, (long long)E, -(1 << 30), stream_);
    NGPU_CUDA(cudaMalloc(&d_rev_off_, sizeof(unsigned long long) * (N + 1)));
    long long n_plastic = 0;
    cudaError_t ce = DevPlasticLists(d_e_post_, d_e_syn_, (long long)E, N, d_rev_off_,
                                     &d_rev_edge_, &n_plastic, stream_);
    if (ce != cudaSuccess)
      throw ngpu_exception(std::string("CUDA error building the plastic lists: ") + cudaGetErrorString(ce));
  }
  // node-level arrays
  NGPU_CUDA(cudaMalloc(&d_last_spike_T_, sizeof(int) * N));
  NGPU_CUDA(cudaMalloc(&d_last_rev_T_, sizeof(int) * N));
  NGPU_CUDA(cudaMalloc(&d_last_post_T_, sizeof(int) * N));
  NGPU_CUDA(cudaMalloc(&d_last_spike_h_, sizeof(float) * N));
  LaunchFillInt(d_last_spike_T_, N, (int)0x80000000, stream_);
  LaunchFillInt(d_last_rev_T_, N, -(1 << 30), stream_);
  LaunchFillInt(d_last_post_T_, N, (int)0x80000000, stream_);
  LaunchFillFloat(d_last_spike_h_, N, 0.0f, stream_);
  has_out_.assign(N, 0);
  for (long long s = 0; s < N; s++)
    has_out_[s] = (h_grp_off_[(s + 1) * nd] > h_grp_off_[s * nd]) ? 1 : 0;
  // shortest delay of a connection whose source can spike (Poisson
  // generators reach their targets through the direct connections, not
  // through the spike ring): the bound of a window of steps
  {
    std::vector<unsigned char> is_gen(N, 0);
    for (NodeGroup *g : groups_)
      if (g->mi->kind == MK_POISSON_GENERATOR)
        for (int k = 0; k < g->n_node; k++) is_gen[g->i_node_0 + k] = 1;
    min_ring_delay_ = 0;
    for (int di = 0; di < nd && min_ring_delay_ == 0; di++) {
      for (long long s2 = 0; s2 < N; s2++) {
        if (!is_gen[s2] && h_grp_off_[s2 * nd + di + 1] > h_grp_off_[s2 * nd + di]) {
          min_ring_delay_ = delays_[di];      // delays_ is sorted
          break;
        }
      }
    }
  }
  BuildRemoteTables();
  // spike ring
  int maxD = 1;
  for (int d : delays_) maxD = std::max(maxD, d);
  // a host that exports spikes keeps them for an exchange interval at least
  if (n_exported_ > 0) maxD = std::max(maxD, kExchangeRingSteps);
  // a network that can run several steps per launch keeps every step of a
  // window (up to 16) in its own ring slot, also where its delays are short
  if (acc_slots_ > 2) maxD = std::max(maxD, 15);
  // max delay + 2 slots: the slot of step T + 1 is emptied during step T
  // while the delivery reads the slots of steps T - 1 ... T - max delay
  ring_R_ = maxD + 2;
  // spike-list capacity per step: nodes x max_spike_num_fact (with a margin
  // of 64 for a node spiking twice in one step at the default factor 1); a
  // factor below 1 is honoured as set, as the reference sizes its spike
  // array from it (src/neurongpu.cu:294), and a step with more spikes sets
  // DERR_RING_OVERFLOW
  {
    const double want = (double)N * (double)max_spike_num_fact_;
    const long long c = max_spike_num_fact_ >= 1.0f ? (long long)ceil(want) + 64
                                                    : std::max(1LL, (long long)ceil(want));
    ring_C_ = (int)std::min<long long>(0x7fffffffLL, c);
  }
  NGPU_CUDA(cudaMalloc(&d_ring_src_, sizeof(unsigned) * (size_t)ring_R_ * ring_C_));
  NGPU_CUDA(cudaMalloc(&d_ring_h_, sizeof(float) * (size_t)ring_R_ * ring_C_));
  NGPU_CUDA(cudaMalloc(&d_ring_cnt_, sizeof(int) * ring_R_));
  NGPU_CUDA(cudaMemset(d_ring_cnt_, 0, sizeof(int) * ring_R_));
  // Poisson direct connections: edges whose source is a poisson_generator
  // node, ordered by (source, delay group, insertion) as in
  // src/neurongpu.cu:1156-1192; grouped by target for the update kernels.
  gen_nodes_.clear();
  std::vector<int> gen_index(N, -1);
  for (NodeGroup *g : groups_) {
    if (g->mi->kind != MK_POISSON_GENERATOR) continue;
    for (int i = 0; i < g->n_node; i++) {
      gen_index[g->i_node_0 + i] = (int)gen_nodes_.size();
      gen_nodes_.push_back(g->i_node_0 + i);
    }
  }
  n_gen_ = (int)gen_nodes_.size();
  if (n_gen_ > 0) {
    struct DC { uint32_t tgt, gen; uint8_t port; float w, delay; uint64_t stream; };
    std::vector<DC> dcs;
    uint64_t stream = 0;
    for (int gi = 0; gi < n_gen_; gi++) {
      int s = gen_nodes_[gi];
      const uint64_t b0 = h_grp_off_[(uint64_t)s * nd], e0 = h_grp_off_[(uint64_t)(s + 1) * nd];
      const size_t m = (size_t)(e0 - b0);
      std::vector<uint32_t> tg(m);
      std::vector<uint8_t> pt(m);
      std::vector<float> wt(m);
      if (m > 0) {
        NGPU_CUDA(cudaMemcpy(tg.data(), d_e_post_ + b0, sizeof(uint32_t) * m, cudaMemcpyDeviceToHost));
        NGPU_CUDA(cudaMemcpy(pt.data(), d_c_port_ + b0, m, cudaMemcpyDeviceToHost));
        NGPU_CUDA(cudaMemcpy(wt.data(), d_e_w_ + b0, sizeof(float) * m, cudaMemcpyDeviceToHost));
      }
      for (int di = 0; di < nd; di++) {
        for (uint64_t k = h_grp_off_[(uint64_t)s * nd + di]; k < h_grp_off_[(uint64_t)s * nd + di + 1]; k++) {
          DC c;
          c.tgt = tg[k - b0]; c.gen = gi; c.port = pt[k - b0]; c.w = wt[k - b0];
          c.delay = time_resolution_ * (float)delays_[di];
          c.stream = stream++;
          dcs.push_back(c);
        }
      }
    }
    std::stable_sort(dcs.begin(), dcs.end(), [](const DC &a, const DC &b) { return a.tgt < b.tgt; });
    size_t M = dcs.size();
    std::vector<unsigned> off(N + 1, 0), gen(M);
    std::vector<unsigned char> port(M);
    std::vector<float> wv(M), dv(M);
    std::vector<unsigned long long> st(M);
    for (size_t k = 0; k < M; k++) {
      off[dcs[k].tgt + 1]++;
      gen[k] = dcs[k].gen; port[k] = dcs[k].port; wv[k] = dcs[k].w; dv[k] = dcs[k].delay;
      st[k] = dcs[k].stream;
    }
    for (long long i = 0; i < N; i++) off[i + 1] += off[i];
    NGPU_CUDA(cudaMalloc(&d_dc_off_, sizeof(unsigned) * (N + 1)));
    NGPU_CUDA(cudaMemcpy(d_dc_off_, off.data(), sizeof(unsigned) * (N + 1), cudaMemcpyHostToDevice));
    NGPU_CUDA(cudaMalloc(&d_dc_gen_, sizeof(unsigned) * (M + 1)));
    NGPU_CUDA(cudaMalloc(&d_dc_port_, M + 1));
    NGPU_CUDA(cudaMalloc(&d_dc_w_, sizeof(float) * (M + 1)));
    NGPU_CUDA(cudaMalloc(&d_dc_delay_, sizeof(float) * (M + 1)));
    NGPU_CUDA(cudaMalloc(&d_dc_stream_, sizeof(unsigned long long) * (M + 1)));
    if (M > 0) {
      NGPU_CUDA(cudaMemcpy(d_dc_gen_, gen.data(), sizeof(unsigned) * M, cudaMemcpyHostToDevice));
      NGPU_CUDA(cudaMemcpy(d_dc_port_, port.data(), M, cudaMemcpyHostToDevice));
      NGPU_CUDA(cudaMemcpy(d_dc_w_, wv.data(), sizeof(float) * M, cudaMemcpyHostToDevice));
      NGPU_CUDA(cudaMemcpy(d_dc_delay_, dv.data(), sizeof(float) * M, cudaMemcpyHostToDevice));
      NGPU_CUDA(cudaMemcpy(d_dc_stream_, st.data(), sizeof(unsigned long long) * M, cudaMemcpyHostToDevice));
    }
    for (NodeGroup *g : groups_) {
      g->has_dc = off[g->i_node_0 + g->n_node] > off[g->i_node_0];
      g->d_dc_off = d_dc_off_ + g->i_node_0;
      // uniform drive: one connection per node, identical except for the
      // random stream, which must run consecutively with the node index
      g->ud = false;
      if (g->has_dc && g->n_port > 0) {
        const size_t b0 = off[g->i_node_0];
        bool ok = true;
        for (int i = 0; i < g->n_node && ok; i++) {
          size_t b = off[g->i_node_0 + i];
          ok = (off[g->i_node_0 + i + 1] - b == 1) && gen[b] == gen[b0] &&
               port[b] == port[b0] && wv[b] == wv[b0] && dv[b] == dv[b0] &&
               st[b] == st[b0] + (unsigned long long)i;
        }
        if (ok) {
          g->ud = true;
          g->ud_gen = (int)gen[b0];
          g->ud_port = port[b0];
          g->ud_w = wv[b0];
          g->ud_delay = dv[b0];
          g->ud_stream0 = st[b0];
        }
      }
    }
    NGPU_CUDA(cudaMalloc(&d_gen_rate_, sizeof(float) * n_gen_));
    NGPU_CUDA(cudaMalloc(&d_gen_origin_, sizeof(float) * n_gen_));
    NGPU_CUDA(cudaMalloc(&d_gen_start_, sizeof(float) * n_gen_));
    NGPU_CUDA(cudaMalloc(&d_gen_stop_, sizeof(float) * n_gen_));
    NGPU_CUDA(cudaMalloc(&d_gen_lambda_, sizeof(double) * n_gen_));
    NGPU_CUDA(cudaMalloc(&d_gen_explam_, sizeof(double) * n_gen_));
    NGPU_CUDA(cudaMalloc(&d_gen_thr_, sizeof(unsigned) * n_gen_ * NGPU_CDF_LEN));
  }
  // counters, per-group device extras and calibration
  // one full wave of resident delivery blocks (grid-stride over the items)
  int n_sm = 148;
  {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
  }
  n_sm_ = n_sm;
  deliver_blocks_ = n_sm * DeliverBlocksPerSM();
  // a serial step's delivery runs alone: every resident block; so does the
  // delivery before a window, with its own register cap
  solo_deliver_blocks_ = n_sm * DeliverOccupancy();
  window_deliver_blocks_ = n_sm * DeliverWindowOccupancy();
  n_evt_blocks_ = std::max(std::max(deliver_blocks_, solo_deliver_blocks_), window_deliver_blocks_);
  NGPU_CUDA(cudaMalloc(&d_done_, sizeof(unsigned)));
  NGPU_CUDA(cudaMemset(d_done_, 0, sizeof(unsigned)));
  NGPU_CUDA(cudaMalloc(&d_blk_events_, sizeof(unsigned long long) * n_evt_blocks_));
  NGPU_CUDA(cudaMemset(d_blk_events_, 0, sizeof(unsigned long long) * n_evt_blocks_));
  int max_den_steps = 0;
  for (NodeGroup *g : groups_) {
    if (g->mi->kind == MK_RK5) {
      g->n_blocks = (g->n_node + 127) / 128;
      NGPU_CUDA(cudaMalloc(&g->d_blk_evals, sizeof(unsigned long long) * g->n_blocks));
      NGPU_CUDA(cudaMemset(g->d_blk_evals, 0, sizeof(unsigned long long) * g->n_blocks));
    }
    calibrate_group(g, time_resolution_, stream_);
    if (g->mi->den_delay_param >= 0 && g->nparam > g->mi->den_delay_param) {
      std::vector<float> dd(g->n_node);
      NGPU_CUDA(cudaMemcpy(dd.data(), g->d_param + (size_t)g->mi->den_delay_param * g->n_pad,
                           sizeof(float) * g->n_node, cudaMemcpyDeviceToHost));
      for (int i = 0; i < g->n_node; i++) {
        const int dsteps = (int)roundf(dd[i] / time_resolution_);
        if (dsteps > 0) has_out_[g->i_node_0 + i] = 1;
        max_den_steps = std::max(max_den_steps, dsteps);
      }
    }
  }
  // dendritic-delay ring: spikes reaching their own node's dendrites
  // (STDP post rule) up to max_den_steps steps later
  if (plastic_) {
    rev_R_ = max_den_steps + 1;
    rev_C_ = ring_C_;
    NGPU_CUDA(cudaMalloc(&d_rev_src_, sizeof(unsigned) * (size_t)rev_R_ * rev_C_));
    NGPU_CUDA(cudaMalloc(&d_rev_cnt_, sizeof(int) * rev_R_));
    NGPU_CUDA(cudaMemset(d_rev_cnt_, 0, sizeof(int) * rev_R_));
  }
  // synapse group table
  memset(&syn_table_, 0, sizeof(syn_table_));
  syn_table_.n = (int)syn_groups_.size();
  if (syn_table_.n > NGPU_MAX_SYN_GROUPS) throw ngpu_exception("Too many synapse groups");
  for (int k = 0; k < syn_table_.n; k++) {
    syn_table_.type[k] = syn_groups_[k].type;
    for (size_t j = 0; j < syn_groups_[k].values.size() && j < NGPU_MAX_SYN_PARAM; j++)
      syn_table_.param[k][j] = syn_groups_[k].values[j];
  }
  // recording columns
  n_rec_cols_ = 0;
  std::vector<RecCol> cols;
  for (Record &r : records_) {
    r.col0 = (int)cols.size();
    for (size_t k = 0; k < r.nodes.size(); k++) {
      int il;
      NodeGroup *g = GroupOf(r.nodes[k], 1, il);
      RecCol c;
      memset(&c, 0, sizeof(c));
      c.node = r.nodes[k];
      const std::string &v = r.var_names[k];
      if (v == "spike") {
        c.spike = 1;
        c.has_out = has_out_[c.node];
      } else {
        int col;
        float *base;
        if ((col = g->ScalVarIdx(v)) >= 0) base = g->d_var;
        else if ((col = g->PortVarIdx(v)) >= 0) { col = g->NSV() + r.ports[k] * g->NPV() + col; base = g->d_var; }
        else if ((col = g->ScalParamIdx(v)) >= 0) base = g->d_param;
        else { col = g->NSP() + r.ports[k] * g->NPP() + g->PortParamIdx(v); base = g->d_param; }
        c.ptr = base + (size_t)col * g->n_pad + il;
      }
      cols.push_back(c);
    }
    if (!r.file_name.empty()) {
      r.fp = fopen(r.file_name.c_str(), "w");
      if (!r.fp) throw ngpu_exception("Cannot open record file " + r.file_name);
    }
  }
  n_rec_cols_ = (int)cols.size();
  if (n_rec_cols_ > 0) {
    NGPU_CUDA(cudaMalloc(&d_rec_cols_, sizeof(RecCol) * n_rec_cols_));
    NGPU_CUDA(cudaMemcpy(d_rec_cols_, cols.data(), sizeof(RecCol) * n_rec_cols_, cudaMemcpyHostToDevice));
    rec_cap_rows_ = std::max<long long>(4 * graph_chunk_ + 8, 4096);
    NGPU_CUDA(cudaMalloc(&d_rec_buf_, sizeof(float) * (size_t)rec_cap_rows_ * (n_rec_cols_ + 1)));
  }
  // step context
  NGPU_CUDA(cudaMalloc(&d_ctx_, sizeof(StepCtx)));
  StepCtx c;
  memset(&c, 0, sizeof(c));
  c.acc_slots = acc_slots_;
  c.ring_R = ring_R_;
  ctx_set_slots(c);
  NGPU_CUDA(cudaMemcpy(d_ctx_, &c, sizeof(StepCtx), cudaMemcpyHostToDevice));
  NGPU_CUDA(cudaStreamSynchronize(stream_));
  NGPU_CUDA(cudaDeviceSynchronize());
}

void NeuronGPU::UploadGeneratorParams() {
  if (n_gen_ == 0) return;
  std::vector<float> rate(n_gen_), origin(n_gen_), start(n_gen_), stop(n_gen_);
  std::vector<double> lam(n_gen_), explam(n_gen_);
  std::vector<unsigned> thr((size_t)n_gen_ * NGPU_CDF_LEN);
  const float time_step = (float)(time_resolution_ / 1000.0);
  for (int k = 0; k < n_gen_; k++) {
    int node = gen_nodes_[k];
    NodeGroup *g = groups_[node_group_map_[node]];
    int il = node - g->i_node_0;
    float v[4];
    for (int j = 0; j < 4; j++)
      NGPU_CUDA(cudaMemcpy(&v[j], g->d_param + (size_t)j * g->n_pad + il, sizeof(float),
                           cudaMemcpyDeviceToHost));
    rate[k] = v[0]; origin[k] = v[1]; start[k] = v[2]; stop[k] = v[3];
    float lf = time_step * rate[k];      // float product, as in src/poiss_gen.cu:62
    lam[k] = (double)lf;
    explam[k] = exp(-(double)lf);
    // inversion thresholds of the direct-connection sampler
    ng_poisson_thresholds(lam[k], explam[k], thr.data() + (size_t)k * NGPU_CDF_LEN);
  }
  // unchanged generator parameters keep the captured step graphs valid
  if (gen_lam_h_ == lam && gen_origin_h_ == origin && gen_start_h_ == start &&
      gen_stop_h_ == stop)
    return;
  NGPU_CUDA(cudaMemcpy(d_gen_thr_, thr.data(), sizeof(unsigned) * thr.size(), cudaMemcpyHostToDevice));
  gen_thr_h_ = thr;
  gen_origin_h_ = origin;
  gen_start_h_ = start;
  gen_stop_h_ = stop;
  gen_lam_h_ = lam;
  gen_explam_h_ = explam;
  InvalidateGraphs();
  NGPU_CUDA(cudaMemcpy(d_gen_rate_, rate.data(), sizeof(float) * n_gen_, cudaMemcpyHostToDevice));
  NGPU_CUDA(cudaMemcpy(d_gen_origin_, origin.data(), sizeof(float) * n_gen_, cudaMemcpyHostToDevice));
  NGPU_CUDA(cudaMemcpy(d_gen_start_, start.data(), sizeof(float) * n_gen_, cudaMemcpyHostToDevice));
  NGPU_CUDA(cudaMemcpy(d_gen_stop_, stop.data(), sizeof(float) * n_gen_, cudaMemcpyHostToDevice));
  NGPU_CUDA(cudaMemcpy(d_gen_lambda_, lam.data(), sizeof(double) * n_gen_, cudaMemcpyHostToDevice));
  NGPU_CUDA(cudaMemcpy(d_gen_explam_, explam.data(), sizeof(double) * n_gen_, cudaMemcpyHostToDevice));
}

// ---------------------------------------------------------------------------
// simulation loop
// ---------------------------------------------------------------------------
void NeuronGPU::InvalidateGraphs() {
  for (auto &kv : graphs_) cudaGraphExecDestroy(kv.second);
  graphs_.clear();
  batch_tables_dirty_ = true;
}

void NeuronGPU::KEvent(int step_in_chunk, int j) {
  size_t idx = (size_t)step_in_chunk * 5 + j;
  while (kev_.size() <= idx) {
    cudaEvent_t e;
    NGPU_CUDA(cudaEventCreate(&e));
    kev_.push_back(e);
  }
  NGPU_CUDA(cudaEventRecordWithFlags(kev_[idx], stream_,
                                     capturing_ ? cudaEventRecordExternal : cudaEventRecordDefault));
}

// class times of the event groups k0 ... k0 + n - 1 (one group per step, or
// one per window at the window's first step)
// a window: its delivery (events 0 -> 1), its update launches (1 -> 2) and,
// after the chunk's last window, the delivery into the last step's slot
// (2 -> 3)
void NeuronGPU::AccumulateWindowTiming(int k0, bool last) {
  NGPU_CUDA(cudaStreamSynchronize(stream_));
  const int kind[3] = {1, 0, 1};
  for (int j = 0; j < (last ? 3 : 2); j++) {
    float ms = 0.0f;
    NGPU_CUDA(cudaEventElapsedTime(&ms, kev_[(size_t)k0 * 5 + j], kev_[(size_t)k0 * 5 + j + 1]));
    ktime_ms_[kind[j]] += ms;
    klaunch_[kind[j]] += 1;
  }
}

void NeuronGPU::AccumulateKernelTiming(int k0, int n, unsigned kinds) {
  NGPU_CUDA(cudaStreamSynchronize(stream_));
  for (int k = k0; k < k0 + n; k++) {
    for (int j = 0; j < 4; j++) {
      if (!(kinds & (1u << j))) continue;       // no launch between these events
      float ms = 0.0f;
      NGPU_CUDA(cudaEventElapsedTime(&ms, kev_[(size_t)k * 5 + j], kev_[(size_t)k * 5 + j + 1]));
      ktime_ms_[j] += ms;
      klaunch_[j] += 1;
    }
  }
}

int NeuronGPU::SetRk5MaxSubsteps(int n) {
  if (n < 1) throw ngpu_exception("the RK5 sub-step limit must be >= 1");
  rk5_max_substeps_ = n;
  InvalidateGraphs();           // the limit is a launch argument of the captured updates
  return 0;
}

int NeuronGPU::SetWaitTest(int mask) {
  if (mask < 0 || mask > (WAIT_TEST_FIRST | WAIT_TEST_SECOND))
    throw ngpu_exception("unknown wait-test bits");
  wait_test_ = mask;
  InvalidateGraphs();
  return 0;
}

int NeuronGPU::SetKernelTiming(int on) {
  ktime_ = on != 0;
  for (int j = 0; j < 4; j++) { ktime_ms_[j] = 0; klaunch_[j] = 0; }
  InvalidateGraphs();
  return 0;
}

int NeuronGPU::GetKernelTiming(int kind, double *total_ms, long long *launches) {
  if (kind < 0 || kind > 3) throw ngpu_exception("Unknown kernel class");
  *total_ms = ktime_ms_[kind];
  *launches = klaunch_[kind];
  return 0;
}

// one time step on stream_ (kernel launches only, no host synchronisation)
void NeuronGPU::EnsureCtxCopies(int n) {
  if (n <= n_ctxs_) return;
  const int want = std::max(n, graph_chunk_);
  if (d_ctxs_) cudaFree(d_ctxs_);
  d_ctxs_ = nullptr;
  n_ctxs_ = 0;
  NGPU_CUDA(cudaMalloc(&d_ctxs_, sizeof(StepCtx) * want));
  n_ctxs_ = want;
  InvalidateGraphs();           // captured graphs hold the old copies
}

void NeuronGPU::EnsureForkResources() {
  if (dstream_ != nullptr) return;
  const char *env = getenv("NGB200_FORK_DELIVERY");
  if (env != nullptr && atoi(env) == 0) return;
  // highest priority: when an update block retires, the SM takes a pending
  // delivery block first, so the (memory-bound) delivery overlaps the
  // (issue-bound) update instead of waiting for its last wave
  int least = 0, greatest = 0;
  NGPU_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
  const char *prio = getenv("NGB200_DELIVERY_PRIORITY");
  NGPU_CUDA(cudaStreamCreateWithPriority(&dstream_, cudaStreamDefault,
                                         (prio != nullptr && atoi(prio) == 0) ? least : greatest));
  NGPU_CUDA(cudaEventCreateWithFlags(&ev_fork_, cudaEventDisableTiming));
  NGPU_CUDA(cudaEventCreateWithFlags(&ev_join_, cudaEventDisableTiming));
}

// The RK5 group whose update grid carries the step's delivery: the first
// single-group RK5 update with the plain controller and a variant that can
// carry it (null: none, or switched off with NGB200_FUSE_DELIVERY=0).
NodeGroup *NeuronGPU::FusedDeliveryGroup() {
  const char *e = getenv("NGB200_FUSE_DELIVERY");
  if (e != nullptr && atoi(e) == 0) return nullptr;
  if (delivery_busy_) return nullptr;
  for (NodeGroup *g : groups_) {
    if (g->mi->kind != MK_RK5 || g->batch >= 0 || g->n_node <= 0) continue;
    if (g->step_mode != STEP_PLAIN || g->n_port < 1 || g->n_port > 4) continue;
    const GroupArgs a = MakeGroupArgs(g);
    if (!a.all_uniform || !Rk5FusesDelivery(g->rk5_variant)) continue;
    return g;
  }
  return nullptr;
}

// Delivery blocks (128 threads) in a fused update grid: two per SM, or
// NGB200_FUSED_DELIVERY_BLOCKS per SM.
int NeuronGPU::FusedDeliveryBlocks() {
  const char *e = getenv("NGB200_FUSED_DELIVERY_BLOCKS");
  const int per_sm = (e != nullptr && atoi(e) > 0) ? atoi(e) : 2;
  int dev = 0, n_sm = 0;
  NGPU_CUDA(cudaGetDevice(&dev));
  NGPU_CUDA(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev));
  // at most the delivery grid's size: the per-block event counters hold that many
  return std::min(std::max(1, n_sm) * per_sm, std::max(1, deliver_blocks_));
}

void NeuronGPU::EnqueueStep(int step_in_chunk) {
  // this step's copy of the step context (k_step_prologue)
  StepCtx *ctx = d_ctxs_ + step_in_chunk;
  DeliverArgs d = MakeDeliverArgs();
  const bool has_delivery = d.nd > 0;
  // The delivery of step T reads the spikes of steps before T and adds into
  // the accumulator half that the update of T + 1 folds, while the updates
  // of step T fold the other half: without plastic synapses the two touch
  // disjoint data, so the delivery runs on its own stream beside the node
  // updates, and the next step (or the chunk's epilogue) waits for both.
  // Preferably the delivery runs inside the grid of one RK5 group's update
  // (k_rk5_update_deliver): no second stream, no join, and consecutive
  // steps' updates keep their programmatic launch overlap.
  NodeGroup *fuse_g = (has_delivery && !plastic_ && !ktime_) ? FusedDeliveryGroup() : nullptr;
  const bool fork = has_delivery && !plastic_ && !ktime_ && dstream_ != nullptr &&
                    fuse_g == nullptr && !(delivery_busy_ && busy_mode_ == BUSY_SERIAL);
  if (fuse_g != nullptr) d.advance_flags = 0;
  if (fork) {
    NGPU_CUDA(cudaEventRecord(ev_fork_, stream_));
    NGPU_CUDA(cudaStreamWaitEvent(dstream_, ev_fork_, 0));
    d.advance_flags = 0;
    LaunchDeliver(d, syn_table_, ctx, deliver_blocks_, dstream_);
    NGPU_CUDA(cudaEventRecord(ev_join_, dstream_));
  }
  if (ktime_) KEvent(step_in_chunk, 0);
  for (NodeGroup *g : groups_) {
    const ModelInfo *mi = g->mi;
    switch (mi->kind) {
      case MK_RK5:
        if (g->batch >= 0) {
          // the whole batch is launched once, at its first group
          const Rk5BatchHost &b = batches_[g->batch];
          if (b.groups[0] == g) {
            for (NodeGroup *bg : b.groups) {
              if (HasLargePoisson(bg))
                LaunchPoissonLarge(MakeGroupArgs(bg), MakeInputArgs(bg), ctx, stream_);
            }
            LaunchRk5Batch(MakeRk5Batch(b), ctx, stream_);
          }
        } else {
          if (HasLargePoisson(g)) LaunchPoissonLarge(MakeGroupArgs(g), MakeInputArgs(g), ctx, stream_);
          if (g == fuse_g) {
            if (!LaunchRk5Update(mi->rk5_model, g->n_port, MakeGroupArgs(g), MakeInputArgs(g),
                                 MakePushArgs(g), ctx, stream_, &d, FusedDeliveryBlocks()))
              throw ngpu_exception("internal error: the delivery could not be fused into the update");
          } else {
            LaunchRk5Update(mi->rk5_model, g->n_port, MakeGroupArgs(g), MakeInputArgs(g),
                            MakePushArgs(g), ctx, stream_);
          }
        }
        break;
      case MK_IAF_PSC_EXP:
      case MK_IAF_PSC_EXP_G:
      case MK_IZHIKEVICH:
      case MK_IZH_PSC_EXP:
        if (g->in_simple_batch) {
          // the whole batch is launched once, at its first group
          if (simple_batch_.groups[0] == g) {
            for (NodeGroup *bg : simple_batch_.groups) {
              if (HasLargePoisson(bg))
                LaunchPoissonLarge(MakeGroupArgs(bg), MakeInputArgs(bg), ctx, stream_);
            }
            LaunchSimpleBatch(simple_batch_.d_segs, simple_batch_.d_blk_seg,
                              simple_batch_.n_blocks, ctx, stream_);
          }
          break;
        }
        if (HasLargePoisson(g)) LaunchPoissonLarge(MakeGroupArgs(g), MakeInputArgs(g), ctx, stream_);
        if (mi->kind == MK_IAF_PSC_EXP) {
          LaunchIafPscExpUpdate(MakeGroupArgs(g), MakeInputArgs(g), MakePushArgs(g), ctx, stream_);
        } else {
          LaunchSimpleNeuronUpdate(mi->kind, mi->n_sub, MakeGroupArgs(g), MakeInputArgs(g),
                                   MakePushArgs(g), ctx, stream_);
        }
        break;
      case MK_SPIKE_GENERATOR:
        if (g->d_sg_off) LaunchSpikeGeneratorUpdate(MakeGroupArgs(g), MakePushArgs(g), ctx, stream_);
        break;
      case MK_PARROT:
        if (HasLargePoisson(g)) LaunchPoissonLarge(MakeGroupArgs(g), MakeInputArgs(g), ctx, stream_);
        LaunchParrotUpdate(MakeGroupArgs(g), MakeInputArgs(g), MakePushArgs(g), ctx, stream_);
        break;
      case MK_SPIKE_DETECTOR:
        LaunchSpikeDetectorUpdate(MakeGroupArgs(g), MakeInputArgs(g), ctx, stream_);
        break;
      case MK_POISSON_NODES: {
        double lam = (double)g->poisson_lambda;
        LaunchPoissonNodesUpdate(MakeGroupArgs(g), MakePushArgs(g), lam, exp(-lam), kernel_seed_,
                                 ctx, stream_);
        break;
      }
      default:
        break;
    }
  }
  // multimeter columns: state after the update, before this step's input is
  // delivered (the reference records between the two, src/neurongpu.cu:488)
  if (n_rec_cols_ > 0) {
    LaunchRecord(d_rec_cols_, n_rec_cols_, d_rec_buf_, rec_cap_rows_, d_last_spike_T_,
                 d_last_spike_h_, 0, time_resolution_, ctx, stream_);
  }
  if (ktime_) KEvent(step_in_chunk, 1);
  if (fork) {
    NGPU_CUDA(cudaStreamWaitEvent(stream_, ev_join_, 0));
    return;
  }
  if (fuse_g != nullptr) return;
  if (plastic_ && rev_R_ > 1) LaunchRevArrive(d, ctx, stream_);
  // the delivery runs alone here (plastic networks, no second stream, the
  // instrumented run): every resident block (beside the updates it takes
  // at most 3 per SM)
  LaunchDeliver(d, syn_table_, ctx, solo_deliver_blocks_, stream_);
  if (ktime_) KEvent(step_in_chunk, 2);
  if (plastic_) {
    d.advance_flags = 1;        // the post rule's last block empties the dendritic slot
    LaunchStdpPost(d, syn_table_, ctx, 2 * n_sm_, stream_);
  }
  if (ktime_) KEvent(step_in_chunk, 3);
  if (!has_delivery) LaunchAdvance(d_ring_cnt_, ring_R_, ring_C_, 1, ctx, stream_);
  if (ktime_) KEvent(step_in_chunk, 4);
}

// Steps per launch. A spike emitted in step s with a delay of D steps is
// folded by the update of step s + D + 1, so with W <= shortest delay + 1 no
// spike of a window of W steps arrives inside it: one delivery before the
// window fills the accumulator slots its W steps fold (k_deliver_window),
// then one launch per RK5 group integrates its neurons through all W steps
// (k_rk5_window). Windows need: every node group an RK5 group (batched or
// not) with the plain controller, or a Poisson generator; no plastic
// synapse, multimeter record or large-rate Poisson pre-pass; the
// accumulator ring of the longest delay + 2 slots. A quiet network (below
// kFusedDeliveryMaxEvents delivered events per step) runs in windows; a
// busy one where its mode trial timed them fastest (LaunchStepsTimed). W
// is at most 16 and preferably divides the graph chunk; NGB200_WINDOW caps
// it (0: one step per launch). 0: no windows.
int NeuronGPU::WindowSteps() {
  if (delivery_busy_ && busy_mode_ != BUSY_WINDOW) return 0;
  return WindowEligible();
}

int NeuronGPU::WindowEligible() {
  const char *env = getenv("NGB200_WINDOW");
  int cap = kWindowMaxSteps;
  if (env != nullptr) cap = std::max(0, std::min(kWindowMaxSteps, atoi(env)));
  // (the delivery's scan of 32 slots' spike counts stays within int)
  if (cap < 2 || acc_slots_ <= 2 || d_acc_stamp_ == nullptr || plastic_ || n_rec_cols_ > 0 ||
      n_exported_ > 0 || has_images_ || ring_C_ >= (1 << 26))
    return 0;
  for (NodeGroup *g : groups_) {
    if (g->mi->kind == MK_POISSON_GENERATOR) continue;
    if (g->mi->kind != MK_RK5 || g->step_mode != STEP_PLAIN || g->n_port > 4 ||
        HasLargePoisson(g))
      return 0;
  }
  // no connection through the spike ring: any W; every step of a window
  // has its own ring slot
  const int minD = min_ring_delay_ > 0 ? min_ring_delay_ : 15;
  // (the accumulator ring, min(max delay + 2, 17) slots, then holds the
  // slots of every step of a window: W <= min(shortest delay + 1, 16))
  int W = std::min(std::min(cap, minD + 1), ring_R_ - 1);
  if (W < 2) return 0;
  // prefer a divisor of the chunk (equal windows in every chunk) if one of
  // at least W / 2 exists
  for (int w = W; 2 * w >= W; w--) {
    if (graph_chunk_ % w == 0) return w;
  }
  return W;
}

// The steps k0 ... k0 + w - 1 of a chunk of n_steps steps in windows of W
// steps: the delivery into the accumulator slots the window's steps fold
// (from the slot of the step before the window on; the chunk's first
// window starts at its own first step, as the step before filled its slot
// itself), with the spike count of the previous window's steps (the
// chunk's first window: of the step before it) and the emptying of the
// ring slots the window writes; then each RK5 group's window launch. After
// the chunk's last window, the delivery into the slot of its last step, the
// count of the window's other steps and the emptying of the next step's
// ring slot: a chunk ends as a chunk of one step per launch does (the slot
// of its last step filled, the spikes of the steps before that step
// counted, the next step's ring slot empty), so either kind may follow.
void NeuronGPU::EnqueueWindow(int k0, int w, int W, int n_steps) {
  StepCtx *ctxs = d_ctxs_ + k0;
  const DeliverArgs d = MakeDeliverArgs();
  // the first delay of a spiking source (the others are Poisson
  // generators', which reach their targets by direct connections)
  const int di0 = min_ring_delay_ > 0 ? delay_index_[min_ring_delay_] : d.nd;
  const int D_lo = min_ring_delay_, D_hi = d.nd > 0 ? delays_.back() : 0;
  const int v_lo = k0 == 0 ? 0 : -1;
  const long long c_lo = k0 == 0 ? -1 : -(long long)W;
  if (ktime_) KEvent(k0, 0);
  LaunchDeliverWindow(d, ctxs, v_lo, w - 1 - v_lo, di0, D_lo, D_hi, 0, w, c_lo, 0,
                      window_deliver_blocks_, stream_);
  if (ktime_) KEvent(k0, 1);
  for (NodeGroup *g : groups_) {
    if (g->mi->kind != MK_RK5) continue;
    if (g->batch >= 0) {
      // a batch is launched once, at its first group
      const Rk5BatchHost &bh = batches_[g->batch];
      if (bh.groups[0] == g) LaunchRk5BatchWindow(MakeRk5Batch(bh), ctxs, w, stream_);
      continue;
    }
    if (!LaunchRk5Window(g->mi->rk5_model, g->n_port, delivery_busy_, MakeGroupArgs(g),
                         MakeInputArgs(g), MakePushArgs(g), ctxs, w, stream_))
      throw ngpu_exception("internal error: no window kernel for this node group");
  }
  if (ktime_) KEvent(k0, 2);
  if (k0 + w == n_steps)
    LaunchDeliverWindow(d, ctxs, w - 1, 1, di0, D_lo, D_hi, w, 1, 0, w - 1,
                        window_deliver_blocks_, stream_);
  if (ktime_) {
    KEvent(k0, 3);
    KEvent(k0, 4);
  }
}

void NeuronGPU::LaunchSteps(int n_steps) {
  if (n_steps <= 0) return;
  EnsureForkResources();
  EnsureCtxCopies(n_steps);
  if (batch_tables_dirty_) RefreshRk5BatchTables();
  if (n_rec_cols_ > 0 && rec_rows_used_ + n_steps > rec_cap_rows_) FlushRecords();
  if (ktime_) {
    // create the event pool before any capture
    for (int k = (int)(kev_.size() / 5); k < n_steps; k++) {
      for (int j = 0; j < 5; j++) {
        cudaEvent_t e;
        NGPU_CUDA(cudaEventCreate(&e));
        kev_.push_back(e);
      }
    }
  }
  const int rec = n_rec_cols_ > 0 ? 1 : 0;
  const int W = WindowSteps();
  window_w_ = W;
  auto enqueue_chunk = [&]() {
    LaunchStepPrologue(d_ctx_, d_ctxs_, n_steps, rec, stream_);
    if (W > 0) {
      for (int k = 0; k < n_steps; k += W) EnqueueWindow(k, std::min(W, n_steps - k), W, n_steps);
    } else {
      for (int k = 0; k < n_steps; k++) EnqueueStep(k);
    }
    LaunchStepEpilogue(d_ctx_, d_ctxs_, n_steps, rec, stream_);
  };
  if (!use_graphs_) {
    enqueue_chunk();
  } else {
    auto it = graphs_.find(GraphKey(n_steps, W));
    if (it == graphs_.end()) {
      cudaGraph_t graph;
      NGPU_CUDA(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
      capturing_ = true;
      try {
        enqueue_chunk();
      } catch (...) {
        capturing_ = false;
        cudaStreamEndCapture(stream_, &graph);
        throw;
      }
      capturing_ = false;
      NGPU_CUDA(cudaStreamEndCapture(stream_, &graph));
      size_t n_nodes = 0;
      NGPU_CUDA(cudaGraphGetNodes(graph, nullptr, &n_nodes));
      std::vector<cudaGraphNode_t> nodes(n_nodes);
      if (n_nodes > 0) NGPU_CUDA(cudaGraphGetNodes(graph, nodes.data(), &n_nodes));
      long long n_kernels = 0;
      for (cudaGraphNode_t nd : nodes) {
        cudaGraphNodeType ty;
        NGPU_CUDA(cudaGraphNodeGetType(nd, &ty));
        if (ty == cudaGraphNodeTypeKernel) n_kernels++;
      }
      kernels_per_step_ = (double)n_kernels / n_steps;
      cudaGraphExec_t exec;
      NGPU_CUDA(cudaGraphInstantiate(&exec, graph, cudaGraphInstantiateFlagUseNodePriority));
      cudaGraphDestroy(graph);
      it = graphs_.emplace(GraphKey(n_steps, W), exec).first;
    }
    NGPU_CUDA(cudaGraphLaunch(it->second, stream_));
  }
  if (n_rec_cols_ > 0) rec_rows_used_ += n_steps;
  NGPU_CUDA(cudaGetLastError());
  if (ktime_) {
    if (W > 0) {
      for (int k = 0; k < n_steps; k += W) AccumulateWindowTiming(k, k + W >= n_steps);
    } else {
      const bool has_delivery = MakeDeliverArgs().nd > 0;
      AccumulateKernelTiming(0, n_steps, 1u | (has_delivery ? 2u : 8u) | (plastic_ ? 4u : 0u));
    }
  }
}

void NeuronGPU::WriteInitialRecord() {
  if (n_rec_cols_ == 0) return;
  if (rec_rows_used_ + 1 > rec_cap_rows_) FlushRecords();
  LaunchRecord(d_rec_cols_, n_rec_cols_, d_rec_buf_, rec_cap_rows_, d_last_spike_T_,
               d_last_spike_h_, 1, time_resolution_, d_ctx_, stream_);
  LaunchAdvance(d_ring_cnt_, ring_R_, ring_C_, 2, d_ctx_, stream_);
  rec_rows_used_ += 1;
}

void NeuronGPU::FlushRecords() {
  if (n_rec_cols_ == 0 || d_rec_buf_ == nullptr) return;
  NGPU_CUDA(cudaStreamSynchronize(stream_));
  if (rec_rows_used_ > 0) {
    const int nc = n_rec_cols_ + 1;
    std::vector<float> buf((size_t)rec_rows_used_ * nc);
    NGPU_CUDA(cudaMemcpy(buf.data(), d_rec_buf_, sizeof(float) * buf.size(), cudaMemcpyDeviceToHost));
    for (Record &r : records_) {
      const int ncol = (int)r.nodes.size();
      for (long long row = 0; row < rec_rows_used_; row++) {
        const float *src = &buf[(size_t)row * nc];
        std::vector<float> v(ncol + 1);
        v[0] = src[0];
        for (int k = 0; k < ncol; k++) v[k + 1] = src[1 + r.col0 + k];
        if (r.fp) {
          fprintf(r.fp, "%f", v[0]);
          for (int k = 0; k < ncol; k++) fprintf(r.fp, "\t%f", v[k + 1]);
          fprintf(r.fp, "\n");
        }
        r.data.push_back(std::move(v));
      }
      if (r.fp) fflush(r.fp);
    }
  }
  rec_rows_used_ = 0;
  long long zero = 0;
  NGPU_CUDA(cudaMemcpy((char *)d_ctx_ + offsetof(StepCtx, rec_row), &zero, sizeof(long long),
                       cudaMemcpyHostToDevice));
}

void NeuronGPU::CheckDeviceErrors() {
  StepCtx c;
  NGPU_CUDA(cudaStreamSynchronize(stream_));
  NGPU_CUDA(cudaMemcpy(&c, d_ctx_, sizeof(StepCtx), cudaMemcpyDeviceToHost));
  if (c.err) {
    unsigned e = c.err;
    unsigned zero = 0;
    NGPU_CUDA(cudaMemcpy((char *)d_ctx_ + offsetof(StepCtx, err), &zero, sizeof(unsigned),
                         cudaMemcpyHostToDevice));
    std::string m = "Simulation error:";
    if (e & DERR_RING_OVERFLOW) m += " more spikes in one step than the spike list can hold (increase max_spike_num_fact);";
    if (e & DERR_RK5_STUCK) m += " RK5 integration exceeded the substep limit;";
    if (e & DERR_REC_OVERFLOW) m += " recording buffer overflow;";
    if (e & DERR_PROPOSER_TIMEOUT) m += " a tensor-core wait of the step proposer timed out;";
    if (e & DERR_REV_OVERFLOW) m += " a dendritic delay exceeds the one at calibration (or too many dendritic arrivals in one step);";
    if (e & DERR_TILE_TIMEOUT) m += " a shared-memory prefetch of the RK5 update timed out;";
    if (e & DERR_TILE_DRAIN) {
      // a bulk copy may still have landed in the shared memory of a block
      // that had exited: nothing computed on this device is trusted after it
      device_lost_ = true;
      m += " a timed-out prefetch did not drain (device state lost; reset the simulator);";
    }
    throw ngpu_exception(m);
  }
}

int NeuronGPU::FlushInput() {
  if (!calibrate_flag_ || !input_pending_) return 0;
  for (NodeGroup *g : groups_) {
    if (g->n_port > 0 && g->mi->in_var >= 0)
      LaunchFoldInput(MakeGroupArgs(g), MakeInputArgs(g), d_ctx_, stream_);
  }
  LaunchClearPending(d_ctx_, stream_);
  NGPU_CUDA(cudaStreamSynchronize(stream_));
  input_pending_ = false;
  return 0;
}

// RK5 autotuner: times every kernel variant of a group on the live state in
// dry mode (full computation, no stores) and keeps the fastest. The variants
// differ only in their register cap (occupancy), not in arithmetic.
// sum of a device array of per-block counters
static unsigned long long sum_counters(const unsigned long long *d, int n) {
  if (d == nullptr || n <= 0) return 0;
  std::vector<unsigned long long> v(n);
  NGPU_CUDA(cudaMemcpy(v.data(), d, sizeof(unsigned long long) * n, cudaMemcpyDeviceToHost));
  unsigned long long t = 0;
  for (auto x : v) t += x;
  return t;
}

// median of three timed launches of f on stream s, after one untimed
static float median_launch_ms(cudaStream_t s, const std::function<void()> &f) {
  cudaEvent_t e0, e1;
  NGPU_CUDA(cudaEventCreate(&e0));
  NGPU_CUDA(cudaEventCreate(&e1));
  f();
  float t[3];
  for (int r = 0; r < 3; r++) {
    NGPU_CUDA(cudaEventRecord(e0, s));
    f();
    NGPU_CUDA(cudaEventRecord(e1, s));
    NGPU_CUDA(cudaEventSynchronize(e1));
    NGPU_CUDA(cudaEventElapsedTime(&t[r], e0, e1));
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  NGPU_CUDA(cudaGetLastError());
  std::sort(t, t + 3);
  return t[1];
}

void NeuronGPU::TuneRk5(NodeGroup *g) {
  g->tuned = true;
  const char *force = getenv("NGB200_RK5_VARIANT");
  GroupArgs a = MakeGroupArgs(g);
  int nv = Rk5VariantCount(g->n_port, a.all_uniform);
  if (nv <= 1) g->rk5_variant = 0;
  if (force != nullptr) {
    g->rk5_variant = std::max(0, std::min(nv - 1, atoi(force)));
    InvalidateGraphs();
    return;
  }
  const char *off = getenv("NGB200_AUTOTUNE");
  if ((off != nullptr && atoi(off) == 0) || nv <= 1 || g->n_node < 16384) return;
  InputArgs in = MakeInputArgs(g);
  PushArgs pa = MakePushArgs(g);
  a.dry = 1;
  in.dry = 1;
  a.blk_evals = nullptr;
  a.step_mode = STEP_PLAIN;       // the variants exist for the plain controller
  // every variant with and without the straggler queue (four dry steps back
  // to back, so that the queue's extra launch in the chain shows); the
  // queue goes off only if the best variant without it is at least 3 %
  // faster than the best with it
  const Rk5Queue q_on = g->q;
  auto run = [&] {
    for (int k = 0; k < 4; k++)
      LaunchRk5Update(g->mi->rk5_model, g->n_port, a, in, pa, d_ctx_, stream_);
  };
  int best_on = 0, best_off = -1;
  float ms_on = 1e30f, ms_off = 1e30f;
  for (int v = 0; v < nv; v++) {
    a.variant = v;
    a.q = q_on;
    const float t_on = median_launch_ms(stream_, run) / 4.0f;
    g->tune_ms[v] = t_on;
    if (t_on < ms_on) {
      ms_on = t_on;
      best_on = v;
    }
    if (q_on.cap > 0 && !g->queue_keep) {
      a.q.cap = 0;
      const float t_off = median_launch_ms(stream_, run) / 4.0f;
      if (t_off < ms_off) {
        ms_off = t_off;
        best_off = v;
      }
    }
  }
  g->queue_off = best_off >= 0 && ms_off < 0.97f * ms_on;
  g->rk5_variant = g->queue_off ? best_off : best_on;
  g->queue_checked = steps_total_;
  g->evals_mark = sum_counters(g->d_blk_evals, g->n_blocks);
  InvalidateGraphs();
}



// The straggler queue adds a launch (the finishing grid) to every step's
// chain of launches, which pays only while some neurons take extra
// sub-steps; the autotuner switches it off for a group or batch that runs
// at least 3 % faster without it (the network was quiet when it was timed).
// Every kQueueRecheckSteps steps such a group's stage evaluations per
// neuron-step are read from its per-block counters: one RK5 attempt per
// step is 6 evaluations, and above 6.06 (neurons have begun to take extra
// sub-steps) the queue goes back on for good and the group's variant is
// tuned again. The results are the same with and without the queue.
// The delivery inside an update grid saves the launch and the join of a
// separate delivery (about 1 us per step on a quiet network) but has fewer
// warps than the forked delivery on its own high-priority stream, which is
// faster once there is much to deliver (26 Hz on the 1e9-synapse network:
// 94 vs 111 us per step). Every kQueueRecheckSteps steps the delivered
// events per step are read from the delivery's per-block counters; above
// kFusedDeliveryMaxEvents the step graphs are rebuilt with the forked
// delivery, and back with the fused one when the rate falls below half of
// it. Both give the same results.
void NeuronGPU::RecheckDeliveryMode() {
  const long long ds = steps_total_ - deliver_checked_;
  // during the first kQueueRecheckSteps steps after every chunk, so that a
  // busy network leaves the quiet network's modes (windows, the delivery in
  // the update's grid) early; then every kQueueRecheckSteps steps
  const long long interval = steps_total_ <= kQueueRecheckSteps
                                 ? std::min<long long>(graph_chunk_, kQueueRecheckSteps)
                                 : kQueueRecheckSteps;
  if (ds < interval || d_blk_events_ == nullptr) return;
  const unsigned long long e = DeliveredEvents();
  const double per_step = (double)(e - events_mark_) / (double)ds;
  const bool busy = delivery_busy_ ? per_step > 0.5 * kFusedDeliveryMaxEvents
                                   : per_step > kFusedDeliveryMaxEvents;
  if (busy != delivery_busy_) {
    delivery_busy_ = busy;
    // a network that turns busy times its delivery modes, unless
    // NGB200_BUSY_MODE names one (0: forked, 1: serial, 2: windows where
    // the network can run them, else forked)
    busy_mode_ = BUSY_FORK;
    delivery_trial_ = busy ? 1 : 0;
    const char *force = getenv("NGB200_BUSY_MODE");
    if (force != nullptr) {
      const int m = atoi(force);
      if (m < BUSY_FORK || m > BUSY_WINDOW)
        throw ngpu_exception("NGB200_BUSY_MODE must be 0, 1 or 2");
      busy_mode_ = (m == BUSY_WINDOW && WindowEligible() == 0) ? (int)BUSY_FORK : m;
      delivery_trial_ = 0;
    }
    trial_chunk_ = 0;
    for (int m = 0; m < 3; m++) {
      trial_ms_[m] = 0.0;
      trial_steps_[m] = 0;
    }
    InvalidateGraphs();
  }
  events_mark_ = e;
  deliver_checked_ = steps_total_;
}

void NeuronGPU::RecheckRk5Queues() {
  const double kEvalsQuiet = 6.06;
  for (Rk5BatchHost &b : batches_) {
    const long long ds = steps_total_ - b.queue_checked;
    if (!b.tuned || !b.queue_off || ds < kQueueRecheckSteps) continue;
    long long n = 0;
    for (NodeGroup *g : b.groups) n += g->n_node;
    const unsigned long long e = sum_counters(b.d_blk_evals, b.n_blocks);
    if ((double)(e - b.evals_mark) > kEvalsQuiet * (double)n * (double)ds) {
      b.queue_off = false;
      b.queue_keep = true;
      b.tuned = false;
      InvalidateGraphs();
    }
    b.evals_mark = e;
    b.queue_checked = steps_total_;
  }
  for (NodeGroup *g : groups_) {
    const long long ds = steps_total_ - g->queue_checked;
    if (g->mi->kind != MK_RK5 || g->batch >= 0 || !g->tuned || !g->queue_off ||
        ds < kQueueRecheckSteps)
      continue;
    const unsigned long long e = sum_counters(g->d_blk_evals, g->n_blocks);
    if ((double)(e - g->evals_mark) > kEvalsQuiet * (double)g->n_node * (double)ds) {
      g->queue_off = false;
      g->queue_keep = true;
      g->tuned = false;
      InvalidateGraphs();
    }
    g->evals_mark = e;
    g->queue_checked = steps_total_;
  }
}

bool NeuronGPU::TunePending() {
  for (Rk5BatchHost &b : batches_)
    if (!b.tuned) return true;
  for (NodeGroup *g : groups_)
    if (g->mi->kind == MK_RK5 && g->batch < 0 && !g->tuned) return true;
  return false;
}

void NeuronGPU::TuneAll() {
  if (batch_tables_dirty_) RefreshRk5BatchTables();
  for (Rk5BatchHost &b : batches_)
    if (!b.tuned) TuneRk5Batch(b);
  for (NodeGroup *g : groups_)
    if (g->mi->kind == MK_RK5 && g->batch < 0 && !g->tuned) TuneRk5(g);
}

int NeuronGPU::GetRk5Tuning(int i_node, int *variant, float *ms) {
  int il;
  NodeGroup *g = GroupOf(i_node, 1, il);
  if (g->batch >= 0) {
    const Rk5BatchHost &b = batches_[g->batch];
    *variant = b.variant;
    for (int v = 0; v < NGPU_RK5_VARIANTS; v++) ms[v] = b.tune_ms[v];
    return 0;
  }
  *variant = g->rk5_variant;
  for (int v = 0; v < NGPU_RK5_VARIANTS; v++) ms[v] = g->tune_ms[v];
  return 0;
}

int NeuronGPU::SetRk5Batching(int on) {
  if (batches_built_)
    throw ngpu_exception("RK5 batching must be chosen before the first simulation");
  rk5_batching_ = on != 0;
  return 0;
}

int NeuronGPU::Rk5BatchOf(int i_node) {
  int il;
  NodeGroup *g = GroupOf(i_node, 1, il);
  return g->batch;
}

// Groups with the same RK5 model and port count form one batch (launched
// once per step through a segment table) when there are at least two of
// them; a single group keeps its own launch with constant-bank arguments.
void NeuronGPU::BuildRk5Batches() {
  batches_built_ = true;
  const char *env = getenv("NGB200_RK5_BATCH");
  if (!rk5_batching_ || (env != nullptr && atoi(env) == 0)) return;
  std::map<std::pair<int, int>, std::vector<NodeGroup *>> by_key;
  for (NodeGroup *g : groups_) {
    if (g->mi->kind != MK_RK5 || g->n_node <= 0) continue;
    if (!Rk5BatchSupported(g->mi->rk5_model, g->n_port)) continue;
    by_key[{g->mi->rk5_model, g->n_port}].push_back(g);
  }
  // simple models: one launch for all their groups
  {
    SimpleBatchHost &sb = simple_batch_;
    for (NodeGroup *g : groups_) {
      const ModelKind k = g->mi->kind;
      if (g->n_node > 0 && (k == MK_IAF_PSC_EXP || k == MK_IAF_PSC_EXP_G ||
                            k == MK_IZHIKEVICH || k == MK_IZH_PSC_EXP))
        sb.groups.push_back(g);
    }
    if (sb.groups.size() >= 2) {
      for (NodeGroup *g : sb.groups) {
        g->in_simple_batch = true;
        sb.n_blocks += (g->n_node + 127) / 128;
      }
      std::vector<int> map(sb.n_blocks);
      int blk = 0;
      for (size_t si = 0; si < sb.groups.size(); si++) {
        const int nb = (sb.groups[si]->n_node + 127) / 128;
        for (int j = 0; j < nb; j++) map[blk + j] = (int)si;
        blk += nb;
      }
      NGPU_CUDA(cudaMalloc(&sb.d_segs, sizeof(SegArgs) * sb.groups.size()));
      NGPU_CUDA(cudaMalloc(&sb.d_blk_seg, sizeof(int) * sb.n_blocks));
      NGPU_CUDA(cudaMemcpy(sb.d_blk_seg, map.data(), sizeof(int) * sb.n_blocks,
                           cudaMemcpyHostToDevice));
    } else {
      sb.groups.clear();
    }
  }
  for (auto &kv : by_key) {
    if (kv.second.size() < 2) continue;
    Rk5BatchHost b;
    b.model = kv.first.first;
    b.np = kv.first.second;
    b.groups = kv.second;
    for (NodeGroup *g : b.groups) b.n_blocks += (g->n_node + 127) / 128;
    const int k = (int)batches_.size();
    for (NodeGroup *g : b.groups) g->batch = k;
    NGPU_CUDA(cudaMalloc(&b.d_segs, sizeof(SegArgs) * b.groups.size()));
    NGPU_CUDA(cudaMalloc(&b.d_blk_seg, sizeof(int) * b.n_blocks));
    NGPU_CUDA(cudaMalloc(&b.d_blk_evals, sizeof(unsigned long long) * b.n_blocks));
    NGPU_CUDA(cudaMemset(b.d_blk_evals, 0, sizeof(unsigned long long) * b.n_blocks));
    std::vector<int> map(b.n_blocks);
    int blk = 0;
    for (size_t si = 0; si < b.groups.size(); si++) {
      const int nb = (b.groups[si]->n_node + 127) / 128;
      for (int j = 0; j < nb; j++) map[blk + j] = (int)si;
      blk += nb;
    }
    NGPU_CUDA(cudaMemcpy(b.d_blk_seg, map.data(), sizeof(int) * b.n_blocks,
                         cudaMemcpyHostToDevice));
    AllocRk5Queue(b.q, b.n_blocks, Rk5RecordFloats(b.model, b.np));
    batches_.push_back(b);
  }
  batch_tables_dirty_ = true;
}

// (Re)writes every batch's segment table from the groups' current
// arguments; captured graphs read the tables at run time, so they stay valid.
void NeuronGPU::RefreshRk5BatchTables() {
  batch_tables_dirty_ = false;
  if (!simple_batch_.groups.empty()) {
    SimpleBatchHost &sb = simple_batch_;
    std::vector<SegArgs> segs(sb.groups.size());
    int blk = 0;
    for (size_t si = 0; si < sb.groups.size(); si++) {
      NodeGroup *g = sb.groups[si];
      memset(&segs[si], 0, sizeof(SegArgs));
      segs[si].g = MakeGroupArgs(g);
      segs[si].in = MakeInputArgs(g);
      segs[si].pa = MakePushArgs(g);
      segs[si].blk0 = blk;
      segs[si].kind = g->mi->kind;
      segs[si].n_sub = g->mi->n_sub;
      blk += (g->n_node + 127) / 128;
    }
    NGPU_CUDA(cudaMemcpy(sb.d_segs, segs.data(), sizeof(SegArgs) * segs.size(),
                         cudaMemcpyHostToDevice));
  }
  for (Rk5BatchHost &b : batches_) {
    std::vector<SegArgs> segs(b.groups.size());
    int blk = 0;
    for (size_t si = 0; si < b.groups.size(); si++) {
      NodeGroup *g = b.groups[si];
      memset(&segs[si], 0, sizeof(SegArgs));
      segs[si].g = MakeGroupArgs(g);
      segs[si].g.blk_evals = nullptr;
      segs[si].in = MakeInputArgs(g);
      segs[si].pa = MakePushArgs(g);
      segs[si].blk0 = blk;
      blk += (g->n_node + 127) / 128;
    }
    NGPU_CUDA(cudaMemcpy(b.d_segs, segs.data(), sizeof(SegArgs) * segs.size(),
                         cudaMemcpyHostToDevice));
  }
}

Rk5Batch NeuronGPU::MakeRk5Batch(const Rk5BatchHost &b) {
  Rk5Batch r;
  r.model = b.model;
  r.np = b.np;
  r.uni = 1;
  for (NodeGroup *g : b.groups) {
    GroupArgs a = MakeGroupArgs(g);
    if (!a.all_uniform) r.uni = 0;
  }
  r.variant = r.uni ? b.variant : 0;
  r.dry = 0;
  r.mode = b.groups[0]->step_mode;
  for (NodeGroup *g : b.groups)
    if (g->step_mode != r.mode)
      throw ngpu_exception("all node groups of a batched RK5 launch must use the same step "
                           "mode (or switch batching off before the first simulation)");
  r.n_blocks = b.n_blocks;
  r.segs = b.d_segs;
  r.blk_seg = b.d_blk_seg;
  r.blk_evals = b.d_blk_evals;
  r.q = b.q;
  if (b.queue_off && r.mode != STEP_LEARNED) r.q.cap = 0;
  r.first = MakeGroupArgs(b.groups[0]);
  return r;
}

// autotuner of a batch: as TuneRk5, over the whole segment table
void NeuronGPU::TuneRk5Batch(Rk5BatchHost &b) {
  b.tuned = true;
  Rk5Batch r = MakeRk5Batch(b);
  // the batched kernel has the four register-cap variants (no tile kernel)
  const int nv = r.uni ? std::min(4, Rk5VariantCount(b.np, 1)) : 1;
  const char *force = getenv("NGB200_RK5_VARIANT");
  if (force != nullptr) {
    b.variant = std::max(0, std::min(nv - 1, atoi(force)));
    InvalidateGraphs();
    return;
  }
  long long n_total = 0;
  for (NodeGroup *g : b.groups) n_total += g->n_node;
  const char *off = getenv("NGB200_AUTOTUNE");
  if ((off != nullptr && atoi(off) == 0) || nv <= 1 || n_total < 16384) return;
  r.dry = 1;
  r.blk_evals = nullptr;
  r.mode = STEP_PLAIN;
  // every variant with and without the straggler queue, as TuneRk5
  const Rk5Queue q_on = b.q;
  auto run = [&] {
    for (int k = 0; k < 4; k++) LaunchRk5Batch(r, d_ctx_, stream_);
  };
  int best_on = 0, best_off = -1;
  float ms_on = 1e30f, ms_off = 1e30f;
  for (int v = 0; v < nv; v++) {
    r.variant = v;
    r.q = q_on;
    const float t_on = median_launch_ms(stream_, run) / 4.0f;
    b.tune_ms[v] = t_on;
    if (t_on < ms_on) {
      ms_on = t_on;
      best_on = v;
    }
    if (q_on.cap > 0 && !b.queue_keep) {
      r.q.cap = 0;
      const float t_off = median_launch_ms(stream_, run) / 4.0f;
      if (t_off < ms_off) {
        ms_off = t_off;
        best_off = v;
      }
    }
  }
  b.queue_off = best_off >= 0 && ms_off < 0.97f * ms_on;
  b.variant = b.queue_off ? best_off : best_on;
  b.queue_checked = steps_total_;
  b.evals_mark = sum_counters(b.d_blk_evals, b.n_blocks);
  InvalidateGraphs();
}

void NeuronGPU::AllocRk5Queue(Rk5Queue &q, long long n_tiles, int stride) {
  FreeRk5Queue(q);
  const char *env = getenv("NGB200_RK5_QUEUE");
  if ((env != nullptr && atoi(env) == 0) || n_tiles <= 0 || stride <= 0) return;
  // sub-queue j takes the tiles j, j + NGPU_QLANES, ...: at most
  // ceil(n_tiles / NGPU_QLANES) tiles of 128 neurons, each queued at most once
  const long long sub_cap = (n_tiles + NGPU_QLANES - 1) / NGPU_QLANES * 128;
  const long long cap = sub_cap * NGPU_QLANES;
  if (cap > 0x7fffffffLL) return;
  NGPU_CUDA(cudaMalloc(&q.hdr, sizeof(Rk5QueueHdr)));
  NGPU_CUDA(cudaMemset(q.hdr, 0, sizeof(Rk5QueueHdr)));
  NGPU_CUDA(cudaMalloc(&q.rec, sizeof(float) * (size_t)cap * stride));
  q.cap = (int)cap;
  q.sub_cap = (int)sub_cap;
  q.stride = stride;
  // finishing launch: up to three 128-thread blocks per SM (its kernel is
  // compiled for one block per SM's registers), never more blocks than the
  // update launch has evaluation counters for
  int dev = 0, n_sm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
  q.fin_blocks = (int)std::min<long long>(n_tiles, 3LL * n_sm);
}

void NeuronGPU::FreeRk5Queue(Rk5Queue &q) {
  if (q.hdr) cudaFree(q.hdr);
  if (q.rec) cudaFree(q.rec);
  q = Rk5Queue{};
}

void NeuronGPU::FreeRk5Batches() {
  if (simple_batch_.d_segs) cudaFree(simple_batch_.d_segs);
  if (simple_batch_.d_blk_seg) cudaFree(simple_batch_.d_blk_seg);
  for (NodeGroup *g : simple_batch_.groups) g->in_simple_batch = false;
  simple_batch_ = SimpleBatchHost{};
  for (Rk5BatchHost &b : batches_) {
    if (b.d_segs) cudaFree(b.d_segs);
    if (b.d_blk_seg) cudaFree(b.d_blk_seg);
    if (b.d_blk_evals) cudaFree(b.d_blk_evals);
    FreeRk5Queue(b.q);
  }
  for (NodeGroup *g : groups_) g->batch = -1;
  batches_.clear();
  batches_built_ = false;
}

int NeuronGPU::StartSimulation() {
  if (device_lost_)
    throw ngpu_exception("the device state was lost in an earlier step (DERR_TILE_DRAIN); "
                         "reset the simulator");
  if (!calibrate_flag_) Calibrate();
  FlushInput();
  if (first_simulation_flag_) {
    // ctx at t_min for the initial record
    StepCtx c;
    NGPU_CUDA(cudaMemcpy(&c, d_ctx_, sizeof(StepCtx), cudaMemcpyDeviceToHost));
    c.it = 0;
    c.t0 = neural_time_;
    c.T0 = (long long)round(neural_time_ / time_resolution_);
    ctx_set_slots(c);
    NGPU_CUDA(cudaMemcpy(d_ctx_, &c, sizeof(StepCtx), cudaMemcpyHostToDevice));
    WriteInitialRecord();
    first_simulation_flag_ = false;
  }
  if (verbosity_level_ >= 1) {
    printf("Simulating ...\n");
    printf("Neural activity simulation time: %.3lf\n", (double)sim_time_);
  }
  UploadGeneratorParams();
  if (!batches_built_) BuildRk5Batches();
  for (NodeGroup *g : groups_)
    if (g->mi->kind == MK_RK5 && g->batch < 0 && g->q.hdr == nullptr && g->n_node > 0)
      AllocRk5Queue(g->q, (g->n_node + 127) / 128, Rk5RecordFloats(g->mi->rk5_model, g->n_port));
  if (batch_tables_dirty_) RefreshRk5BatchTables();
  // a variant forced through NGB200_RK5_VARIANT applies from the first step
  if (steps_total_ >= kTuneSteps || getenv("NGB200_RK5_VARIANT") != nullptr) TuneAll();
  neur_t0_ = neural_time_;
  it_ = 0;
  Nt_ = (long long)round(sim_time_ / time_resolution_);
  StepCtx c;
  NGPU_CUDA(cudaStreamSynchronize(stream_));
  NGPU_CUDA(cudaMemcpy(&c, d_ctx_, sizeof(StepCtx), cudaMemcpyDeviceToHost));
  c.it = 0;
  c.t0 = neur_t0_;
  c.T0 = (long long)round(neur_t0_ / time_resolution_);
  c.poisson_pending = 0;
  ctx_set_slots(c);
  NGPU_CUDA(cudaMemcpy(d_ctx_, &c, sizeof(StepCtx), cudaMemcpyHostToDevice));
  return 0;
}

int NeuronGPU::SimulationStep() {
  if (first_simulation_flag_) StartSimulation();
  if (input_pending_ == false && it_ > 0) {
    // state was read in between: the fold already consumed the pending
    // input, so the device context says so (poisson_pending == 0)
  }
  LaunchSteps(1);
  it_++;
  steps_total_++;
  input_pending_ = true;
  neural_time_ = neur_t0_ + (double)time_resolution_ * (double)it_;
  return 0;
}

int NeuronGPU::EndSimulation() {
  FlushInput();
  FlushRecords();
  CheckDeviceErrors();
  if (verbosity_level_ >= 2) printf("%.3lf\n", neural_time_);
  return 0;
}

int NeuronGPU::Simulate() {
  // the spikes of a partitioned network cross hosts between runs of steps,
  // through the caller's collective: a plain Simulate would drop them
  if (n_hosts_ > 1 && (has_images_ || n_exported_ > 0))
    throw ngpu_exception("a network partitioned over hosts is simulated by the Python "
                         "layer's Simulate, or by NGB200_SimulateSteps with the spike "
                         "exchange (NGB200_PackRemoteSpikes / NGB200_UnpackRemoteSpikes)");
  StartSimulation();
  auto t_start = std::chrono::steady_clock::now();
  if (!ev_start_) {
    NGPU_CUDA(cudaEventCreate(&ev_start_));
    NGPU_CUDA(cudaEventCreate(&ev_stop_));
  }
  NGPU_CUDA(cudaEventRecord(ev_start_, stream_));
  long long done = 0;
  while (done < Nt_) {
    if (verbosity_level_ >= 2 && done % 100 == 0)
      printf("%.3lf\n", neur_t0_ + (double)time_resolution_ * (double)done);
    long long n = std::min<long long>(graph_chunk_, Nt_ - done);
    if (verbosity_level_ >= 2) n = std::min<long long>(n, 100 - done % 100);
    LaunchStepsTimed((int)n);
    done += n;
    it_ = done;
    input_pending_ = true;
    steps_total_ += n;
    if (steps_total_ >= kTuneSteps && TunePending()) TuneAll();
    RecheckRk5Queues();
    RecheckDeliveryMode();
  }
  neural_time_ = neur_t0_ + (double)time_resolution_ * (double)Nt_;
  NGPU_CUDA(cudaEventRecord(ev_stop_, stream_));
  NGPU_CUDA(cudaEventSynchronize(ev_stop_));
  float dev_ms = 0.0f;
  NGPU_CUDA(cudaEventElapsedTime(&dev_ms, ev_start_, ev_stop_));
  last_sim_device_ms_ = dev_ms;
  EndSimulation();
  last_sim_seconds_ = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
  return 0;
}

// LaunchSteps; while a busy network's mode trial runs, the candidate modes
// take turns (two chunks each, the second timed on the device)
void NeuronGPU::LaunchStepsTimed(int n_steps) {
  if (delivery_trial_ == 1 && steps_total_ >= kQueueRecheckSteps) delivery_trial_ = 2;
  if (delivery_trial_ != 2 || ktime_ || !delivery_busy_) {
    LaunchSteps(n_steps);
    return;
  }
  if (!ev_c0_) {
    NGPU_CUDA(cudaEventCreate(&ev_c0_));
    NGPU_CUDA(cudaEventCreate(&ev_c1_));
  }
  const int n_modes = WindowEligible() > 0 ? 3 : 2;
  const int mode = (int)((trial_chunk_ / 2) % n_modes);
  const bool timed = (trial_chunk_ & 1) != 0;
  trial_chunk_++;
  busy_mode_ = mode;
  NGPU_CUDA(cudaEventRecord(ev_c0_, stream_));
  LaunchSteps(n_steps);
  NGPU_CUDA(cudaEventRecord(ev_c1_, stream_));
  if (timed) {
    NGPU_CUDA(cudaEventSynchronize(ev_c1_));
    float ms = 0.0f;
    NGPU_CUDA(cudaEventElapsedTime(&ms, ev_c0_, ev_c1_));
    trial_ms_[mode] += ms;
    trial_steps_[mode] += n_steps;
  }
  bool done = true;
  for (int m = 0; m < n_modes; m++) done = done && trial_steps_[m] >= kDeliveryTrialSteps;
  if (done) {
    int best = 0;
    double best_t = 1e300;
    for (int m = 0; m < n_modes; m++) {
      const double t = trial_ms_[m] / (double)trial_steps_[m];
      if (t < best_t) {
        best_t = t;
        best = m;
      }
      if (verbosity_level_ >= 2)
        printf("busy mode %d: %.2f us per step\n", m, 1000.0 * t);
    }
    busy_mode_ = best;
    delivery_trial_ = 0;
  }
}

int NeuronGPU::SimulateSteps(long long n) {
  if (n < 0) throw ngpu_exception("the number of steps must be >= 0");
  if (first_simulation_flag_) StartSimulation();
  long long done = 0;
  while (done < n) {
    const long long k = std::min<long long>(graph_chunk_, n - done);
    LaunchStepsTimed((int)k);
    done += k;
    it_ += k;
    steps_total_ += k;
    input_pending_ = true;
    if (steps_total_ >= kTuneSteps && TunePending()) TuneAll();
    RecheckRk5Queues();
    RecheckDeliveryMode();
  }
  neural_time_ = neur_t0_ + (double)time_resolution_ * (double)it_;
  return 0;
}

// ---------------------------------------------------------------------------
// networks partitioned over hosts
// ---------------------------------------------------------------------------
int NeuronGPU::SetHost(int id, int n_hosts) {
  if (n_hosts < 1 || id < 0 || id >= n_hosts) throw ngpu_exception("Invalid host index or count");
  if (has_images_ || n_exported_ > 0)
    throw ngpu_exception("the host cannot change after remote connections were made");
  host_id_ = id;
  n_hosts_ = n_hosts;
  image_of_.assign(n_hosts, std::map<int, int>());
  return 0;
}

int NeuronGPU::RemoteCreate(int i_host, const std::string &model, int n_node, int n_port) {
  if (i_host < 0 || i_host >= n_hosts_) throw ngpu_exception("Invalid host index in RemoteCreate");
  if (i_host == host_id_) return Create(model, n_node, n_port);
  return -1;
}

int NeuronGPU::RemoteConnect(int i_source_host, const int *src_arr, int i_src0, int n_source,
                             int i_target_host, const int *tgt_arr, int i_tgt0, int n_target,
                             ConnSpec &cs, SynSpec &ss) {
  if (i_source_host < 0 || i_source_host >= n_hosts_ || i_target_host < 0 ||
      i_target_host >= n_hosts_)
    throw ngpu_exception("Invalid host index in RemoteConnect");
  CheckUncalibrated("Connections cannot be created after calibration");
  if (n_source <= 0 || n_target <= 0) throw ngpu_exception("Empty source or target in RemoteConnect");
  auto src_of = [&](int k) { return src_arr != nullptr ? src_arr[k] : i_src0 + k; };
  if (i_source_host == i_target_host) {
    // both ends on one host: an ordinary connection there
    if (host_id_ != i_source_host) return 0;
    return Connect(src_arr, i_src0, n_source, tgt_arr, i_tgt0, n_target, cs, ss);
  }
  if (host_id_ == i_source_host) {
    // the sources send their spikes to the other hosts
    const long long N = (long long)node_group_map_.size();
    if ((long long)exported_.size() < N) exported_.resize(N, 0);
    for (int k = 0; k < n_source; k++) {
      const int s = src_of(k);
      if (s < 0 || s >= N) throw ngpu_exception("Source node index out of range in RemoteConnect");
      if (!exported_[s]) {
        exported_[s] = 1;
        n_exported_++;
      }
    }
    return 0;
  }
  if (host_id_ != i_target_host) return 0;
  // target host: image nodes of the remote sources, made in order of first
  // appearance, then the connection from the images with the given rule
  if ((int)image_of_.size() < n_hosts_) image_of_.resize(n_hosts_);
  std::map<int, int> &img_of = image_of_[i_source_host];
  std::vector<int> fresh;
  std::map<int, int> fresh_index;
  for (int k = 0; k < n_source; k++) {
    const int s = src_of(k);
    if (s < 0) throw ngpu_exception("Source node index out of range in RemoteConnect");
    if (img_of.count(s) == 0 && fresh_index.count(s) == 0) {
      fresh_index[s] = (int)fresh.size();
      fresh.push_back(s);
    }
  }
  if (!fresh.empty()) {
    const int i0 = Create("remote_image", (int)fresh.size(), 0);
    for (size_t j = 0; j < fresh.size(); j++) img_of[fresh[j]] = i0 + (int)j;
  }
  std::vector<int> img(n_source);
  for (int k = 0; k < n_source; k++) img[k] = img_of[src_of(k)];
  has_images_ = true;
  return Connect(img.data(), 0, n_source, tgt_arr, i_tgt0, n_target, cs, ss);
}

// device tables of the exchange, built at calibration
void NeuronGPU::BuildRemoteTables() {
  const long long N = (long long)node_group_map_.size();
  const int nd = (int)delays_.size();
  if (n_exported_ > 0) {
    exported_.resize(N, 0);
    NGPU_CUDA(cudaMalloc(&d_exported_, N));
    NGPU_CUDA(cudaMemcpy(d_exported_, exported_.data(), N, cudaMemcpyHostToDevice));
  }
  d_image_lut_.assign(n_hosts_, nullptr);
  image_lut_n_.assign(n_hosts_, 0);
  for (int h = 0; h < (int)image_of_.size() && h < n_hosts_; h++) {
    if (image_of_[h].empty()) continue;
    const int n = image_of_[h].rbegin()->first + 1;
    std::vector<int> lut(n, -1);
    for (const auto &kv : image_of_[h]) lut[kv.first] = kv.second;
    NGPU_CUDA(cudaMalloc(&d_image_lut_[h], sizeof(int) * n));
    NGPU_CUDA(cudaMemcpy(d_image_lut_[h], lut.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
    image_lut_n_[h] = n;
  }
  // the exchange interval: the shortest delay of a connection from an image
  min_image_delay_ = 0;
  for (NodeGroup *g : groups_) {
    if (g->mi->kind != MK_IMAGE) continue;
    for (int di = 0; di < nd; di++) {
      if (min_image_delay_ > 0 && delays_[di] >= min_image_delay_) break;
      for (int k = 0; k < g->n_node; k++) {
        const long long s = g->i_node_0 + k;
        if (h_grp_off_[s * nd + di + 1] > h_grp_off_[s * nd + di]) {
          min_image_delay_ = delays_[di];
          break;
        }
      }
    }
  }
}

// The longest exchange interval this host allows: the shortest delay of a
// connection from an image node (no remote spike may be due before it
// arrives), and on an exporting host the steps its spike ring keeps; 0 if
// the host neither receives nor sends remote spikes.
int NeuronGPU::RemoteExchangeSteps() {
  if (!calibrate_flag_) Calibrate();
  int e = min_image_delay_;
  if (n_exported_ > 0) e = e > 0 ? std::min(e, ring_R_ - 2) : ring_R_ - 2;
  return e;
}

long long NeuronGPU::PackRemoteSpikes(int n_steps, unsigned *buf, long long cap) {
  if (n_steps < 0 || n_steps > ring_R_ - 2)
    throw ngpu_exception("the exchange interval must lie within the longest delay");
  if (buf == nullptr) throw ngpu_exception("null exchange buffer");
  if (d_exported_ == nullptr || n_steps == 0) {
    NGPU_CUDA(cudaMemsetAsync(buf, 0, 4 * sizeof(unsigned), stream_));
    NGPU_CUDA(cudaStreamSynchronize(stream_));
    return 0;
  }
  LaunchPackRemote(d_ring_cnt_, d_ring_src_, d_ring_h_, ring_R_, ring_C_, d_ctx_, n_steps,
                   d_exported_, buf, cap, stream_);
  // the count of every exported spike; above cap only cap were written and
  // the caller packs again into a larger buffer (the ring is unchanged)
  unsigned hdr[2] = {0, 0};
  NGPU_CUDA(cudaMemcpyAsync(hdr, buf, sizeof(hdr), cudaMemcpyDeviceToHost, stream_));
  NGPU_CUDA(cudaStreamSynchronize(stream_));
  return (long long)hdr[0];
}

int NeuronGPU::UnpackRemoteSpikes(int src_host, int n_steps, const unsigned *buf,
                                  long long count) {
  if (src_host < 0 || src_host >= n_hosts_) throw ngpu_exception("Invalid host index");
  if (n_steps < 0 || n_steps > ring_R_ - 2)
    throw ngpu_exception("the exchange interval must lie within the longest delay");
  if (src_host == host_id_ || count <= 0 || src_host >= (int)d_image_lut_.size() ||
      d_image_lut_[src_host] == nullptr)
    return 0;
  LaunchUnpackRemote(buf, count, d_image_lut_[src_host], image_lut_n_[src_host], d_ring_cnt_,
                     d_ring_src_, d_ring_h_, ring_R_, ring_C_, d_ctx_, n_steps, stream_);
  NGPU_CUDA(cudaGetLastError());
  return 0;
}

int NeuronGPU::PushSpikesToNodes(int n, const int *nodes) {
  (void)n; (void)nodes;
  throw ngpu_exception("PushSpikesToNodes is only available for external-neuron co-simulation, which this build does not provide");
}

unsigned long long NeuronGPU::StageEvaluations() {
  unsigned long long tot = 0;
  for (const Rk5BatchHost &b : batches_) {
    std::vector<unsigned long long> v(b.n_blocks);
    NGPU_CUDA(cudaMemcpy(v.data(), b.d_blk_evals, sizeof(unsigned long long) * b.n_blocks,
                         cudaMemcpyDeviceToHost));
    for (auto x : v) tot += x;
  }
  for (NodeGroup *g : groups_) {
    if (!g->d_blk_evals) continue;
    std::vector<unsigned long long> v(g->n_blocks);
    NGPU_CUDA(cudaMemcpy(v.data(), g->d_blk_evals, sizeof(unsigned long long) * g->n_blocks,
                         cudaMemcpyDeviceToHost));
    for (auto x : v) tot += x;
  }
  return tot;
}

unsigned long long NeuronGPU::DeliveredEvents() {
  if (!d_blk_events_) return 0;
  std::vector<unsigned long long> v(n_evt_blocks_);
  NGPU_CUDA(cudaMemcpy(v.data(), d_blk_events_, sizeof(unsigned long long) * n_evt_blocks_,
                       cudaMemcpyDeviceToHost));
  unsigned long long tot = 0;
  for (auto x : v) tot += x;
  return tot;
}

unsigned long long NeuronGPU::TotalSpikes() {
  if (!d_ctx_) return 0;
  StepCtx c;
  NGPU_CUDA(cudaMemcpy(&c, d_ctx_, sizeof(StepCtx), cudaMemcpyDeviceToHost));
  // the spikes of the last step are counted by the next step's bookkeeping
  // (the delivery of step T counts step T - 1): add that ring slot here
  unsigned long long n = c.n_spikes;
  if (d_ring_cnt_ != nullptr && ring_R_ > 0) {
    const long long T_last = c.T0 + c.it;
    int cnt = 0;
    NGPU_CUDA(cudaMemcpy(&cnt, d_ring_cnt_ + (int)(T_last % ring_R_), sizeof(int),
                         cudaMemcpyDeviceToHost));
    n += (unsigned long long)std::min(cnt, ring_C_);
  }
  return n;
}

}  // namespace ngpu

namespace ngpu {

// ---------------------------------------------------------------------------
// learned RK5 step proposer
// ---------------------------------------------------------------------------
std::vector<NodeGroup *> NeuronGPU::ProposerGroups(int i_node) {
  std::vector<NodeGroup *> out;
  if (i_node < 0) {
    for (NodeGroup *g : groups_)
      if (g->mi->kind == MK_RK5 && StepProposerSupported(g->mi->rk5_model, g->n_port))
        out.push_back(g);
    if (out.empty()) throw ngpu_exception("no node group supports the step proposer");
    return out;
  }
  int il;
  NodeGroup *g = GroupOf(i_node, 1, il);
  if (g->mi->kind != MK_RK5 || !StepProposerSupported(g->mi->rk5_model, g->n_port))
    throw ngpu_exception("the step proposer supports aeif_cond_beta and aeif_cond_alpha "
                         "groups with 1 or 2 receptor ports");
  out.push_back(g);
  return out;
}

int NeuronGPU::SetStepLog(int i_node, int capacity) {
  if (capacity < 0 || capacity > (1 << 26)) throw ngpu_exception("step log capacity out of range");
  for (NodeGroup *g : ProposerGroups(i_node)) {
    if (g->d_log_buf) cudaFree(g->d_log_buf);
    if (g->d_log_count) cudaFree(g->d_log_count);
    g->d_log_buf = nullptr;
    g->d_log_count = nullptr;
    g->log_cap = 0;
    if (capacity > 0) {
      NGPU_CUDA(cudaMalloc(&g->d_log_buf, sizeof(float) * 8 * (size_t)capacity));
      NGPU_CUDA(cudaMalloc(&g->d_log_count, sizeof(unsigned)));
      NGPU_CUDA(cudaMemset(g->d_log_count, 0, sizeof(unsigned)));
      g->log_cap = capacity;
      g->step_mode = STEP_LOG;
    } else if (g->step_mode == STEP_LOG) {
      g->step_mode = STEP_PLAIN;
    }
  }
  InvalidateGraphs();
  return 0;
}

long long NeuronGPU::GetStepLogCount(int i_node) {
  long long tot = 0;
  if (stream_) NGPU_CUDA(cudaStreamSynchronize(stream_));
  for (NodeGroup *g : ProposerGroups(i_node)) {
    if (!g->d_log_count) continue;
    unsigned c = 0;
    NGPU_CUDA(cudaMemcpy(&c, g->d_log_count, sizeof(unsigned), cudaMemcpyDeviceToHost));
    tot += c;
  }
  return tot;
}

int NeuronGPU::GetStepLog(int i_node, float *out, int max_rows) {
  int rows = 0;
  if (stream_) NGPU_CUDA(cudaStreamSynchronize(stream_));
  for (NodeGroup *g : ProposerGroups(i_node)) {
    if (!g->d_log_count || rows >= max_rows) continue;
    unsigned c = 0;
    NGPU_CUDA(cudaMemcpy(&c, g->d_log_count, sizeof(unsigned), cudaMemcpyDeviceToHost));
    int k = (int)std::min<long long>(std::min<long long>((long long)c, (long long)g->log_cap),
                                     (long long)(max_rows - rows));
    if (k > 0)
      NGPU_CUDA(cudaMemcpy(out + (size_t)rows * 8, g->d_log_buf, sizeof(float) * 8 * (size_t)k,
                           cudaMemcpyDeviceToHost));
    rows += k;
  }
  return rows;
}

void NeuronGPU::UploadMlpImage() {
  MlpImage img;
  MlpBuildImage(mlp_params_.data(), &img);
  if (!d_mlp_img_) NGPU_CUDA(cudaMalloc(&d_mlp_img_, sizeof(MlpImage)));
  NGPU_CUDA(cudaMemcpy(d_mlp_img_, &img, sizeof(MlpImage), cudaMemcpyHostToDevice));
  InvalidateGraphs();
}

// Trains the proposer on every logged sample of every group (GPU kernels,
// FP32 Adam); logging is switched off afterwards.
int NeuronGPU::TrainStepProposer(int steps, int blocks, float lr, unsigned long long seed,
                                 float *loss_first, float *loss_last) {
  if (steps <= 0 || blocks <= 0 || !(lr > 0.0f)) throw ngpu_exception("invalid training settings");
  if (!stream_) NGPU_CUDA(cudaStreamCreate(&stream_));
  NGPU_CUDA(cudaStreamSynchronize(stream_));
  std::vector<std::pair<NodeGroup *, int>> parts;
  long long n = 0;
  for (NodeGroup *g : groups_) {
    if (!g->d_log_count) continue;
    unsigned c = 0;
    NGPU_CUDA(cudaMemcpy(&c, g->d_log_count, sizeof(unsigned), cudaMemcpyDeviceToHost));
    int k = (int)std::min<long long>((long long)c, (long long)g->log_cap);
    if (k > 0) parts.push_back({g, k});
    n += k;
  }
  if (n < 64) throw ngpu_exception("too few logged RK5 steps to train the step proposer");
  float *d_data = nullptr;
  NGPU_CUDA(cudaMalloc(&d_data, sizeof(float) * 8 * (size_t)n));
  long long off = 0;
  double tsum = 0.0;
  std::vector<float> tmp;
  for (auto &pk : parts) {
    NGPU_CUDA(cudaMemcpy(d_data + off * 8, pk.first->d_log_buf, sizeof(float) * 8 * (size_t)pk.second,
                         cudaMemcpyDeviceToDevice));
    tmp.resize((size_t)pk.second * 8);
    NGPU_CUDA(cudaMemcpy(tmp.data(), pk.first->d_log_buf, sizeof(float) * 8 * (size_t)pk.second,
                         cudaMemcpyDeviceToHost));
    for (int r = 0; r < pk.second; r++) tsum += tmp[(size_t)r * 8 + 6];
    off += pk.second;
  }
  mlp_params_.assign(NGPU_MLP_NPARAM, 0.0f);
  MlpInitParams(mlp_params_.data(), seed, (float)(tsum / (double)n));
  float l0 = 0.0f, l1 = 0.0f;
  try {
    MlpTrain(d_data, (int)std::min<long long>(n, 0x7fffffffLL), mlp_params_.data(), steps, blocks,
             lr, seed, &l0, &l1, stream_);
  } catch (const std::exception &e) {
    cudaFree(d_data);
    throw ngpu_exception(e.what());
  }
  cudaFree(d_data);
  for (NodeGroup *g : groups_) {
    if (g->step_mode == STEP_LOG) g->step_mode = STEP_PLAIN;
  }
  UploadMlpImage();
  if (loss_first) *loss_first = l0;
  if (loss_last) *loss_last = l1;
  return (int)std::min<long long>(n, 0x7fffffffLL);
}

int NeuronGPU::SetStepProposer(int i_node, int on) {
  if (on && mlp_params_.empty())
    throw ngpu_exception("the learned step proposer has no parameters (train or set them first)");
  for (NodeGroup *g : ProposerGroups(i_node)) {
    g->step_mode = on ? STEP_LEARNED : (g->d_log_buf ? STEP_LOG : STEP_PLAIN);
  }
  InvalidateGraphs();
  return 0;
}

int NeuronGPU::SetStepProposerParams(const float *params) {
  mlp_params_.assign(params, params + NGPU_MLP_NPARAM);
  if (!stream_) NGPU_CUDA(cudaStreamCreate(&stream_));
  UploadMlpImage();
  return 0;
}

int NeuronGPU::GetStepProposerParams(float *params) {
  if (mlp_params_.empty()) throw ngpu_exception("the step proposer has no parameters");
  std::copy(mlp_params_.begin(), mlp_params_.end(), params);
  return 0;
}

int NeuronGPU::SetStepProposerMargin(float margin) {
  if (!(margin > -4.0f && margin < 8.0f)) throw ngpu_exception("margin out of range");
  mlp_margin_ = margin;
  InvalidateGraphs();
  return 0;
}

// test entry points: gradients of the training kernels and tensor-core
// inference on caller data (host arrays)
float NeuronGPU::MlpGradientsHost(const float *data, int n, const float *params, float *grad) {
  if (n <= 0) throw ngpu_exception("no samples");
  if (!stream_) NGPU_CUDA(cudaStreamCreate(&stream_));
  float *d = nullptr;
  NGPU_CUDA(cudaMalloc(&d, sizeof(float) * 8 * (size_t)n));
  NGPU_CUDA(cudaMemcpy(d, data, sizeof(float) * 8 * (size_t)n, cudaMemcpyHostToDevice));
  float loss = 0.0f;
  try {
    loss = MlpGradients(d, n, params, grad, stream_);
  } catch (const std::exception &e) {
    cudaFree(d);
    throw ngpu_exception(e.what());
  }
  cudaFree(d);
  return loss;
}

int NeuronGPU::MlpInferHost(const float *x6, int n, const float *params, float *out) {
  if (n <= 0) throw ngpu_exception("no samples");
  if (!stream_) NGPU_CUDA(cudaStreamCreate(&stream_));
  MlpImage img;
  MlpBuildImage(params, &img);
  MlpImage *d_img = nullptr;
  float *d_x = nullptr, *d_out = nullptr;
  unsigned *d_err = nullptr;
  NGPU_CUDA(cudaMalloc(&d_img, sizeof(MlpImage)));
  NGPU_CUDA(cudaMalloc(&d_x, sizeof(float) * 6 * (size_t)n));
  NGPU_CUDA(cudaMalloc(&d_out, sizeof(float) * (size_t)n));
  NGPU_CUDA(cudaMalloc(&d_err, sizeof(unsigned)));
  NGPU_CUDA(cudaMemset(d_err, 0, sizeof(unsigned)));
  NGPU_CUDA(cudaMemcpy(d_img, &img, sizeof(MlpImage), cudaMemcpyHostToDevice));
  NGPU_CUDA(cudaMemcpy(d_x, x6, sizeof(float) * 6 * (size_t)n, cudaMemcpyHostToDevice));
  MlpInfer(d_x, n, d_img, d_out, d_err, stream_);
  NGPU_CUDA(cudaStreamSynchronize(stream_));
  NGPU_CUDA(cudaGetLastError());
  unsigned err = 0;
  NGPU_CUDA(cudaMemcpy(out, d_out, sizeof(float) * (size_t)n, cudaMemcpyDeviceToHost));
  NGPU_CUDA(cudaMemcpy(&err, d_err, sizeof(unsigned), cudaMemcpyDeviceToHost));
  cudaFree(d_img);
  cudaFree(d_x);
  cudaFree(d_out);
  cudaFree(d_err);
  if (err) throw ngpu_exception("tensor-core completion wait timed out in the step proposer");
  return 0;
}

}  // namespace ngpu
