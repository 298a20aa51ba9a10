// NeuronGPU: host driver of the B200 simulation core.
//
// Public methods mirror the reference class NeuronGPU (src/neurongpu.h:94-679)
// so the C ABI (src/neurongpu_C.h) maps one to one; the internals (SoA state,
// CSR delivery graph, spike ring, device-side step counter, CUDA graphs) are
// this build's own.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

#include "ngpu_connect_device.h"
#include "ngpu_device.h"
#include "ngpu_kernels.h"
#include "ngpu_models.h"

namespace ngpu {

class ngpu_exception : public std::exception {
  std::string msg_;

 public:
  explicit ngpu_exception(const std::string &m) : msg_(m) {}
  const char *what() const noexcept override { return msg_.c_str(); }
};

#define NGPU_CUDA(call)                                                    \
  do {                                                                     \
    cudaError_t e_ = (call);                                               \
    if (e_ != cudaSuccess) {                                               \
      throw ngpu::ngpu_exception(std::string("CUDA error: ") +             \
                                 cudaGetErrorString(e_) + " at " +         \
                                 __FILE__ + ":" + std::to_string(__LINE__)); \
    }                                                                      \
  } while (0)

enum { ON_EXCEPTION_EXIT = 0, ON_EXCEPTION_HANDLE = 1 };

struct ConnectionId {
  int i_source_;
  int i_group_;
  int i_conn_;
};

struct ConnectionStatus {
  int i_source;
  int i_target;
  unsigned char port;
  unsigned char syn_group;
  float delay;
  float weight;
};

enum ConnRule {
  ONE_TO_ONE = 0, ALL_TO_ALL, FIXED_TOTAL_NUMBER, FIXED_INDEGREE,
  FIXED_OUTDEGREE, N_CONN_RULE
};

struct ConnSpec {
  int rule_ = ALL_TO_ALL;
  int total_num_ = 0;
  int indegree_ = 0;
  int outdegree_ = 0;
  void Init() { *this = ConnSpec(); }
  int SetParam(const std::string &name, int value);
  static bool IsParam(const std::string &name);
};

struct SynSpec {
  unsigned char syn_group_ = 0;
  unsigned char port_ = 0;
  float weight_ = 0.0f;
  float delay_ = 0.0f;
  const float *weight_array_ = nullptr;
  const float *delay_array_ = nullptr;
  void Init() { *this = SynSpec(); }
  int SetParam(const std::string &name, int value);
  int SetParam(const std::string &name, float value);
  int SetParam(const std::string &name, const float *arr);
  static bool IsIntParam(const std::string &name);
  static bool IsFloatParam(const std::string &name);
  static bool IsFloatPtParam(const std::string &name);
};

struct SynGroupHost {
  int type;                       // 1 test_syn_model, 2 stdp
  std::vector<std::string> names;
  std::vector<float> values;
};

// One node group (one Create call).
struct NodeGroup {
  int model = -1;                 // index into ModelCatalogue()
  const ModelInfo *mi = nullptr;
  int i_node_0 = 0, n_node = 0, n_port = 0, n_pad = 0;
  int nvar = 0, nparam = 0;
  float *d_var = nullptr, *d_param = nullptr, *d_h = nullptr, *d_dx = nullptr;
  std::vector<char> p_uniform;
  std::vector<float> p_uval;
  std::vector<float> group_param;
  float rk5_eps = 1.0e-6f;
  long long acc_base = 0;
  // spike count / spike-time recording
  int *d_spike_count = nullptr;
  float *d_rec_times = nullptr;
  int *d_n_rec = nullptr;
  int max_rec = 0;
  std::vector<std::string> int_var_names;
  // spike generator
  std::vector<std::vector<float>> sg_times, sg_heights;
  int *d_sg_off = nullptr, *d_sg_step = nullptr, *d_sg_next = nullptr;
  float *d_sg_height = nullptr;
  // Poisson direct connections into this group (CSR by local node)
  unsigned *d_dc_off = nullptr;
  bool has_dc = false;
  // uniform drive (one identical direct connection per node, see InputArgs)
  bool ud = false;
  int ud_gen = -1, ud_port = 0;
  float ud_w = 0.0f, ud_delay = 0.0f;
  unsigned long long ud_stream0 = 0;
  // CreatePoissonGenerator nodes
  float poisson_lambda = 0.0f;
  // per-block RK5 derivative evaluation counters
  unsigned long long *d_blk_evals = nullptr;
  int n_blocks = 0;
  // straggler queue of the group's own RK5 launch (unbatched groups)
  Rk5Queue q{};
  // autotuned RK5 kernel variant and the timings it was chosen from
  int rk5_variant = 1;
  bool tuned = false;
  float tune_ms[NGPU_RK5_VARIANTS] = {0};
  bool queue_off = false;       // the autotuner switched the straggler queue off
  long long queue_checked = 0;  // steps_total_ at the last choice or check
  unsigned long long evals_mark = 0;  // stage evaluations counted by then
  bool queue_keep = false;      // the queue came back on: later tunings keep it
  // index of the batched RK5 launch this group belongs to, or -1
  int batch = -1;
  // updated by the batched launch of simple models
  bool in_simple_batch = false;
  // RK5 step mode (StepMode) and the accepted-step log of STEP_LOG
  int step_mode = 0;
  float *d_log_buf = nullptr;
  unsigned *d_log_count = nullptr;
  int log_cap = 0;

  int ScalVarIdx(const std::string &n) const;
  int PortVarIdx(const std::string &n) const;
  int ScalParamIdx(const std::string &n) const;
  int PortParamIdx(const std::string &n) const;
  int GroupParamIdx(const std::string &n) const;
  int IntVarIdx(const std::string &n) const;
  int ArrayParamIdx(const std::string &n) const;
  int NSV() const { return (int)mi->scal_var.size(); }
  int NPV() const { return (int)mi->port_var.size(); }
  int NSP() const { return (int)mi->scal_param.size(); }
  int NPP() const { return (int)mi->port_param.size(); }
};

struct Record {
  std::string file_name;
  std::vector<std::string> var_names;
  std::vector<int> nodes, ports;
  std::vector<std::vector<float>> data;   // rows: t, v1, v2, ...
  FILE *fp = nullptr;
  int col0 = 0;                           // first column in device buffer
};

class NeuronGPU {
 public:
  NeuronGPU();
  ~NeuronGPU();

  // errors
  bool error_flag_ = false;
  std::string error_message_;
  unsigned char error_code_ = 0;
  int on_exception_ = ON_EXCEPTION_EXIT;
  void SetErrorFlag(bool f) { error_flag_ = f; }
  void SetErrorMessage(const std::string &m) { error_message_ = m; }
  void SetErrorCode(unsigned char c) { error_code_ = c; }
  char *GetErrorMessage() { return (char *)error_message_.c_str(); }
  unsigned char GetErrorCode() { return error_code_; }
  void SetOnException(int v) { on_exception_ = v; }
  int OnException() { return on_exception_; }

  // kernel parameters
  int SetRandomSeed(unsigned long long seed);
  int SetTimeResolution(float t);
  float GetTimeResolution() { return time_resolution_; }
  int SetMaxSpikeBufferSize(int n) { max_spike_buffer_size_ = n; return 0; }
  int GetMaxSpikeBufferSize() { return max_spike_buffer_size_; }
  int SetSimTime(float t) { sim_time_ = t; return 0; }
  int SetVerbosityLevel(int v) { verbosity_level_ = v; return 0; }
  std::vector<std::string> GetFloatParamNames();
  std::vector<std::string> GetIntParamNames();
  bool IsFloatParam(const std::string &n);
  bool IsIntParam(const std::string &n);
  int GetFloatParamIdx(const std::string &n);
  int GetIntParamIdx(const std::string &n);
  float GetFloatParam(const std::string &n);
  int GetIntParam(const std::string &n);
  int SetFloatParam(const std::string &n, float v);
  int SetIntParam(const std::string &n, int v);

  // nodes
  int Create(const std::string &model, int n_node, int n_port);
  int CreatePoissonGenerator(int n_node, float rate);
  int SetNeuronParam(int i_node, int n, const std::string &name, float val);
  int SetNeuronParam(const int *nodes, int n, const std::string &name,
                     float val);
  int SetNeuronParam(int i_node, int n, const std::string &name,
                     const float *arr, int size);
  int SetNeuronParam(const int *nodes, int n, const std::string &name,
                     const float *arr, int size);
  int SetNeuronIntVar(int i_node, int n, const std::string &name, int val);
  int SetNeuronIntVar(const int *nodes, int n, const std::string &name,
                      int val);
  int SetNeuronVar(int i_node, int n, const std::string &name, float val);
  int SetNeuronVar(const int *nodes, int n, const std::string &name,
                   float val);
  int SetNeuronVar(int i_node, int n, const std::string &name,
                   const float *arr, int size);
  int SetNeuronVar(const int *nodes, int n, const std::string &name,
                   const float *arr, int size);
  int IsNeuronScalParam(int i_node, const std::string &n);
  int IsNeuronPortParam(int i_node, const std::string &n);
  int IsNeuronArrayParam(int i_node, const std::string &n);
  int IsNeuronGroupParam(int i_node, const std::string &n);
  int IsNeuronIntVar(int i_node, const std::string &n);
  int IsNeuronScalVar(int i_node, const std::string &n);
  int IsNeuronPortVar(int i_node, const std::string &n);
  int IsNeuronArrayVar(int i_node, const std::string &n);
  int GetNeuronParamSize(int i_node, const std::string &n);
  int GetNeuronVarSize(int i_node, const std::string &n);
  float *GetNeuronParam(int i_node, int n, const std::string &name);
  float *GetNeuronParam(const int *nodes, int n, const std::string &name);
  float *GetArrayParam(int i_node, const std::string &name);
  int *GetNeuronIntVar(int i_node, int n, const std::string &name);
  int *GetNeuronIntVar(const int *nodes, int n, const std::string &name);
  float *GetNeuronVar(int i_node, int n, const std::string &name);
  float *GetNeuronVar(const int *nodes, int n, const std::string &name);
  float *GetArrayVar(int i_node, const std::string &name);
  int SetNeuronGroupParam(int i_node, int n, const std::string &name,
                          float val);
  float GetNeuronGroupParam(int i_node, const std::string &name);
  std::vector<std::string> GetIntVarNames(int i_node);
  std::vector<std::string> GetScalVarNames(int i_node);
  std::vector<std::string> GetPortVarNames(int i_node);
  std::vector<std::string> GetScalParamNames(int i_node);
  std::vector<std::string> GetPortParamNames(int i_node);
  std::vector<std::string> GetGroupParamNames(int i_node);
  std::vector<std::string> GetArrayParamNames(int i_node);
  std::vector<std::string> GetArrayVarNames(int i_node);

  // recording
  int CreateRecord(const std::string &file, const std::vector<std::string> &vars,
                   const int *nodes, const int *ports, int n);
  std::vector<std::vector<float>> *GetRecordData(int i_record);
  int ActivateSpikeCount(int i_node, int n);
  int ActivateRecSpikeTimes(int i_node, int n, int max_n);
  int GetNRecSpikeTimes(int i_node);
  std::vector<float> GetRecSpikeTimes(int i_node);

  // connections
  int Connect(int i_source, int i_target, unsigned char port,
              unsigned char syn_group, float weight, float delay);
  int Connect(const int *src_arr, int i_src0, int n_source,
              const int *tgt_arr, int i_tgt0, int n_target,
              ConnSpec &cs, SynSpec &ss);
  std::vector<ConnectionId> GetConnections(const int *src_arr, int i_src0,
                                           int n_source, const int *tgt_arr,
                                           int i_tgt0, int n_target,
                                           int syn_group);
  ConnectionStatus GetConnectionStatus(ConnectionId id);
  int CreateSynGroup(const std::string &model);
  int GetSynGroupNParam(int sg);
  std::vector<std::string> GetSynGroupParamNames(int sg);
  bool IsSynGroupParam(int sg, const std::string &n);
  int GetSynGroupParamIdx(int sg, const std::string &n);
  float GetSynGroupParam(int sg, const std::string &n);
  int SetSynGroupParam(int sg, const std::string &n, float v);

  // random arrays (host, counter-based)
  unsigned int *RandomInt(size_t n);
  float *RandomUniform(size_t n);
  float *RandomNormal(size_t n, float mean, float stddev);
  float *RandomNormalClipped(size_t n, float mean, float stddev, float vmin,
                             float vmax, float vstep);

  // simulation
  int Calibrate();
  int Simulate();
  int Simulate(float sim_time) { sim_time_ = sim_time; return Simulate(); }
  int StartSimulation();
  int SimulationStep();
  int EndSimulation();
  // n steps of a started simulation (graph chunks, as Simulate)
  int SimulateSteps(long long n);
  int PushSpikesToNodes(int n, const int *nodes);

  // A network partitioned over hosts (one GPU per host process), the
  // reference's RemoteCreate / RemoteConnect (src/connect_rules.h:406-800,
  // src/neurongpu.cu:1626-1642, 1820-1836) without MPI: every host runs the
  // same script; a remote connection is made on its target host from image
  // nodes of the remote sources (one per remote node, created by
  // RemoteConnect), and its source host marks the source nodes as exported.
  // The spikes of exported nodes are exchanged every RemoteExchangeSteps()
  // steps (the shortest delay of a connection from an image node) by the
  // caller's collective: PackRemoteSpikes after the steps, an all-gather of
  // the packed lists, UnpackRemoteSpikes of every other host's list, which
  // pushes each image node's spikes into the spike ring at the step the
  // remote node emitted them, so they are delivered as the reference's
  // per-step MPI exchange delivers them (src/neurongpu.cu:490-521).
  int SetHost(int id, int n_hosts);
  int HostId() const { return host_id_; }
  int NHosts() const { return n_hosts_; }
  // the group's first node on host i_host, -1 on the other hosts (their
  // callers learn it from the owner by a broadcast)
  int RemoteCreate(int i_host, const std::string &model, int n_node, int n_port);
  int RemoteConnect(int i_source_host, const int *src_arr, int i_src0, int n_source,
                    int i_target_host, const int *tgt_arr, int i_tgt0, int n_target,
                    ConnSpec &cs, SynSpec &ss);
  int RemoteExchangeSteps();
  // spikes of exported nodes in the last n_steps steps into buf (device, u32:
  // [count, overflow, 0, 0, then (step offset, node, height bits) per spike]);
  // returns the count, which exceeds cap when only cap entries fitted
  long long PackRemoteSpikes(int n_steps, unsigned *buf, long long cap);
  // the packed list of host src_host (device buffer, count entries)
  int UnpackRemoteSpikes(int src_host, int n_steps, const unsigned *buf, long long count);

  // statistics exposed through the extension entry points
  unsigned long long StageEvaluations();
  unsigned long long DeliveredEvents();
  unsigned long long TotalSpikes();
  double LastSimulateSeconds() { return last_sim_seconds_; }
  double LastSimulateDeviceMs() { return last_sim_device_ms_; }
  // kernel launches per time step in the last captured step graph
  double KernelsPerStep() { return kernels_per_step_; }
  // per-kernel-class device timing (CUDA events around every launch)
  int SetKernelTiming(int on);
  NodeGroup *FusedDeliveryGroup();
  int FusedDeliveryBlocks();
  // RK5 sub-steps a neuron may take in one time step before the update
  // gives up on it and reports DERR_RK5_STUCK (default NGPU_RK5_MAX_SUBSTEPS)
  int SetRk5MaxSubsteps(int n);
  int Rk5MaxSubsteps() const { return rk5_max_substeps_; }
  // test hook: WaitTest bits; the marked bounded waits of the RK5 kernels
  // give up after a single non-blocking test (0: normal waits)
  int SetWaitTest(int mask);
  int GetKernelTiming(int kind, double *total_ms, long long *launches);
  // RK5 kernel variant chosen for the group of i_node and its timings
  int GetRk5Tuning(int i_node, int *variant, float *ms);
  void TuneRk5(NodeGroup *g);
  // the autotuner runs once the network has integrated kTuneSteps steps, so
  // that it times the kernels on a settled state (the first steps start
  // from the initial step size and take several sub-steps per neuron)
  static const long long kTuneSteps = 200;
  long long steps_total_ = 0;
  bool TunePending();
  void TuneAll();
  // the autotuner chooses the variant and whether the straggler queue is
  // used together; groups and batches without the queue are checked every
  // kQueueRecheckSteps steps (RecheckRk5Queues)
  static const long long kQueueRecheckSteps = 1000;
  void RecheckRk5Queues();
  // delivery in the update grid or on its own stream, by the delivered rate
  static constexpr double kFusedDeliveryMaxEvents = 65536.0;
  void RecheckDeliveryMode();
  bool delivery_busy_ = false;
  // A busy network runs in the mode a trial on the live network timed
  // fastest (every mode gives the same results): one step per launch with
  // the delivery on its own stream beside the updates (BUSY_FORK) or after
  // them on every resident block (BUSY_SERIAL), or windows of steps
  // (BUSY_WINDOW, where the network can run them). From step
  // kQueueRecheckSteps on (past the start's transient) the candidates take
  // turns, two chunks each, of which the second is timed (the first
  // captures the mode's graph), until
  // each has kDeliveryTrialSteps timed steps, so that a drift of the
  // network's activity weighs on all alike.
  enum BusyMode { BUSY_FORK = 0, BUSY_SERIAL = 1, BUSY_WINDOW = 2 };
  static const long long kDeliveryTrialSteps = 300;
  int busy_mode_ = BUSY_FORK;
  int delivery_trial_ = 0;      // 0 none, 1 waiting for the trial's first step, 2 running
  long long trial_chunk_ = 0;
  double trial_ms_[3] = {0.0, 0.0, 0.0};
  long long trial_steps_[3] = {0, 0, 0};
  int WindowEligible();         // W of the network's structure, ignoring its activity
  cudaEvent_t ev_c0_ = nullptr, ev_c1_ = nullptr;
  void LaunchStepsTimed(int n_steps);
  long long deliver_checked_ = 0;
  unsigned long long events_mark_ = 0;
  // RK5 groups of one model and port count are integrated by one launch
  // per step (segment table) unless batching is switched off
  int SetRk5Batching(int on);
  int Rk5BatchOf(int i_node);
  // learned RK5 step proposer: accepted-step logging, GPU training, use
  int SetStepLog(int i_node, int capacity);
  long long GetStepLogCount(int i_node);
  int GetStepLog(int i_node, float *out, int max_rows);
  int TrainStepProposer(int steps, int blocks, float lr, unsigned long long seed,
                        float *loss_first, float *loss_last);
  int SetStepProposer(int i_node, int on);
  int SetStepProposerParams(const float *params);
  int GetStepProposerParams(float *params);
  int SetStepProposerMargin(float margin);
  float MlpGradientsHost(const float *data, int n, const float *params, float *grad);
  int MlpInferHost(const float *x6, int n, const float *params, float *out);
  int SetGraphChunk(int g) { graph_chunk_ = g > 0 ? g : 1; InvalidateGraphs(); return 0; }
  long long NNodes() { return (long long)node_group_map_.size(); }
  long long NConnections() { return n_raw_ + (long long)p_src_.size(); }
  // every connection in delivery order (source, delay group, insertion);
  // null outputs are skipped; weights are the device values once calibrated
  long long ExportConnections(int *src, int *tgt, int *port, int *syn,
                              float *delay, float *weight);
  int UseGraphs(int f) { use_graphs_ = f != 0; return 0; }
  // synchronous device copy of a raw column (tests, bench)
  cudaStream_t Stream() { return stream_; }
  int FlushInput();

  // public state read by the C layer
  ConnSpec conn_spec_;
  SynSpec syn_spec_;

 private:
  // kernel parameters
  float time_resolution_ = 0.1f;
  float sim_time_ = 1000.0f;
  float max_spike_num_fact_ = 1.0f;
  float max_spike_per_host_fact_ = 1.0f;
  int verbosity_level_ = 4;
  int max_spike_buffer_size_ = 20;
  int remote_spike_height_flag_ = 0;
  unsigned long long rnd_seed_ = 54321ULL;
  unsigned long long kernel_seed_ = 54321ULL + 12345ULL;
  unsigned long long rng_calls_ = 0;   // host RNG stream counter

  // structure
  std::vector<NodeGroup *> groups_;
  struct Rk5BatchHost {
    int model = 0, np = 0;
    std::vector<NodeGroup *> groups;
    int n_blocks = 0;
    int variant = 1;
    bool tuned = false;
    float tune_ms[NGPU_RK5_VARIANTS] = {0};
    bool queue_off = false;
    long long queue_checked = 0;
    unsigned long long evals_mark = 0;
    bool queue_keep = false;
    SegArgs *d_segs = nullptr;
    int *d_blk_seg = nullptr;
    unsigned long long *d_blk_evals = nullptr;
    Rk5Queue q{};
  };
  std::vector<Rk5BatchHost> batches_;
  // one batched launch for the groups of simple models (iaf_psc_exp,
  // iaf_psc_exp_g, izhikevich family) when there are at least two
  struct SimpleBatchHost {
    std::vector<NodeGroup *> groups;
    int n_blocks = 0;
    SegArgs *d_segs = nullptr;
    int *d_blk_seg = nullptr;
  } simple_batch_;
  bool batches_built_ = false;
  bool batch_tables_dirty_ = true;
  bool rk5_batching_ = true;
  void BuildRk5Batches();
  void RefreshRk5BatchTables();
  void TuneRk5Batch(Rk5BatchHost &b);
  Rk5Batch MakeRk5Batch(const Rk5BatchHost &b);
  void FreeRk5Batches();
  // straggler queues for a launch of n_tiles 128-neuron tiles, records of
  // stride floats (none when switched off with NGB200_RK5_QUEUE=0)
  void AllocRk5Queue(Rk5Queue &q, long long n_tiles, int stride);
  static void FreeRk5Queue(Rk5Queue &q);
  std::vector<float> mlp_params_;       // FP32 proposer parameters (empty: none)
  MlpImage *d_mlp_img_ = nullptr;
  float mlp_margin_ = 0.25f;
  int rk5_max_substeps_ = NGPU_RK5_MAX_SUBSTEPS;
  int wait_test_ = 0;
  bool device_lost_ = false;    // set by DERR_TILE_DRAIN; every later simulation call fails
  void UploadMlpImage();
  std::vector<NodeGroup *> ProposerGroups(int i_node);
  std::vector<int> node_group_map_;
  std::vector<SynGroupHost> syn_groups_;
  std::vector<Record> records_;

  // edges in insertion order: device edge store filled by the rule kernels
  // (freed at calibration), single connections buffered on the host
  EdgeStore d_raw_ = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  long long n_raw_ = 0, raw_cap_ = 0;
  std::vector<uint32_t> p_src_, p_tgt_;
  std::vector<uint8_t> p_port_, p_syn_;
  std::vector<float> p_w_;
  std::vector<uint16_t> p_d_;
  bool any_plastic_ = false;          // an edge with synapse group > 0 exists
  bool csr_valid_ = false;
  // CSR by source, then delay index, insertion order inside (device arrays
  // d_grp_off_, d_e_post_ = targets, d_c_port_, d_e_syn_, d_e_w_; host copy
  // of the group offsets; host mirrors of targets, ports and groups for the
  // connection queries, made on demand)
  std::vector<int> delays_;           // distinct delays (steps), sorted
  std::vector<int> delay_index_;      // D -> di (or -1)
  std::vector<uint64_t> h_grp_off_;   // [n_nodes*nd + 1]
  unsigned char *d_c_port_ = nullptr;
  std::vector<uint32_t> h_c_tgt_;
  std::vector<uint8_t> h_c_port_, h_c_syn_;
  bool mirror_valid_ = false;
  void GrowRaw(long long need);
  void FlushPending();
  void FreeRaw();
  void FreeCSR();
  void EnsureMirror();

  // device state
  bool calibrate_flag_ = false;
  bool first_simulation_flag_ = true;
  cudaStream_t stream_ = nullptr;
  // delivery beside the node updates (non-plastic networks): its stream and
  // the fork / join events of a step (NGB200_FORK_DELIVERY=0 keeps one stream)
  cudaStream_t dstream_ = nullptr;
  cudaEvent_t ev_fork_ = nullptr, ev_join_ = nullptr;
  void EnsureForkResources();
  // per-step copies of the step context for a chunk of steps
  StepCtx *d_ctxs_ = nullptr;
  int n_ctxs_ = 0;
  void EnsureCtxCopies(int n);
  StepCtx *d_ctx_ = nullptr;
  long long *d_acc_ = nullptr;
  long long n_acc_ = 0;
  // accumulator ring: 2 slots, or max delay + 2 for networks that can run
  // several steps per launch; per slot the last step added into it
  int acc_slots_ = 2;
  static constexpr double kWindowAccBytes = 8e9;
  static constexpr int kWindowMaxSteps = 16;    // steps per window at most
  long long *d_acc_stamp_ = nullptr;
  unsigned *d_ring_src_ = nullptr;
  float *d_ring_h_ = nullptr;
  int *d_ring_cnt_ = nullptr;
  int ring_R_ = 0, ring_C_ = 0;
  int *d_last_spike_T_ = nullptr, *d_last_rev_T_ = nullptr;
  int *d_last_post_T_ = nullptr;
  // dendritic-delay ring of plastic networks (rev_R_ = max delay steps + 1)
  unsigned *d_rev_src_ = nullptr;
  int *d_rev_cnt_ = nullptr;
  int rev_R_ = 0, rev_C_ = 0;
  float *d_last_spike_h_ = nullptr;
  unsigned long long *d_grp_off_ = nullptr;
  unsigned *d_e_slot_ = nullptr;
  float *d_e_w_ = nullptr;
  unsigned char *d_e_syn_ = nullptr;
  int *d_e_stamp_ = nullptr;
  unsigned *d_e_post_ = nullptr;
  unsigned long long *d_rev_off_ = nullptr;
  unsigned *d_rev_edge_ = nullptr;
  int *d_delays_ = nullptr;
  int *d_delay_di_ = nullptr;         // delay in steps -> index in delays_, or -1
  bool plastic_ = false;
  std::vector<unsigned char> has_out_;
  // Poisson direct connections (global arrays, CSR by target node)
  unsigned *d_dc_off_ = nullptr, *d_dc_gen_ = nullptr;
  unsigned char *d_dc_port_ = nullptr;
  float *d_dc_w_ = nullptr, *d_dc_delay_ = nullptr;
  unsigned long long *d_dc_stream_ = nullptr;
  int n_gen_ = 0;
  std::vector<int> gen_nodes_;        // generator index -> node
  float *d_gen_rate_ = nullptr, *d_gen_origin_ = nullptr;
  float *d_gen_start_ = nullptr, *d_gen_stop_ = nullptr;
  double *d_gen_lambda_ = nullptr, *d_gen_explam_ = nullptr;
  unsigned *d_gen_thr_ = nullptr;       // [gen][NGPU_CDF_LEN] inversion thresholds
  std::vector<unsigned> gen_thr_h_;
  std::vector<float> gen_origin_h_, gen_start_h_, gen_stop_h_;
  std::vector<double> gen_lam_h_, gen_explam_h_;
  // delivery counters
  unsigned long long *d_blk_events_ = nullptr;
  unsigned *d_done_ = nullptr;
  int deliver_blocks_ = 0;
  // recording
  RecCol *d_rec_cols_ = nullptr;
  int n_rec_cols_ = 0;
  float *d_rec_buf_ = nullptr;
  long long rec_cap_rows_ = 0;
  long long rec_rows_used_ = 0;
  SynGroupTable syn_table_;

  // session
  double neural_time_ = 0.0, neur_t0_ = 0.0, t_min_ = 0.0;
  long long it_ = 0, Nt_ = 0;
  bool input_pending_ = false;
  double last_sim_seconds_ = 0.0;
  double last_sim_device_ms_ = 0.0;
  double kernels_per_step_ = 0.0;
  cudaEvent_t ev_start_ = nullptr, ev_stop_ = nullptr;
  bool ktime_ = false;
  bool capturing_ = false;
  std::vector<cudaEvent_t> kev_;
  double ktime_ms_[4] = {0, 0, 0, 0};
  long long klaunch_[4] = {0, 0, 0, 0};
  void KEvent(int step_in_chunk, int j);
  // kinds: bit j set where the interval between the events j and j + 1 of
  // a step holds a launch (update, delivery, post rule, bookkeeping)
  void AccumulateKernelTiming(int k0, int n, unsigned kinds);
  void AccumulateWindowTiming(int k0, bool last);

  // graphs
  bool use_graphs_ = true;
  int graph_chunk_ = 100;
  // captured step graphs by (steps, busy mode, steps per window): a network
  // can change its mode without capturing again
  std::map<long long, cudaGraphExec_t> graphs_;
  long long GraphKey(int n_steps, int W) const {
    return (long long)n_steps | ((long long)(delivery_busy_ ? busy_mode_ + 1 : 0) << 32) |
           ((long long)W << 40);
  }
  void InvalidateGraphs();
  void LaunchSteps(int n_steps);
  void EnqueueStep(int step_in_chunk);
  // several steps per launch (windows of W steps, W <= shortest delay + 1)
  int WindowSteps();
  void EnqueueWindow(int k0, int w, int W, int n_steps);
  int min_ring_delay_ = 0;      // shortest delay (steps) of a spiking source's connection
  // partitioned networks: host of this instance, exported nodes, and per
  // source host the image node of every remote node (host and device)
  int host_id_ = 0, n_hosts_ = 1;
  std::vector<unsigned char> exported_;
  long long n_exported_ = 0;
  std::vector<std::map<int, int>> image_of_;
  unsigned char *d_exported_ = nullptr;
  std::vector<int *> d_image_lut_;
  std::vector<int> image_lut_n_;
  int min_image_delay_ = 0;     // shortest delay of a connection from an image node
  static const int kExchangeRingSteps = 32;   // spike-ring steps of an exporting host
  bool has_images_ = false;
  void BuildRemoteTables();
  int window_w_ = 0;            // W of the last chunk (0: one step per launch)
  int solo_deliver_blocks_ = 0; // grid of a delivery that runs alone (serial steps)
  int window_deliver_blocks_ = 0;   // grid of the delivery before a window (all resident)
  int n_sm_ = 148;              // multiprocessors of the device (queried at calibration)
  int n_evt_blocks_ = 0;        // delivery event counters (max of both grids)

  // helpers
  NodeGroup *GroupOf(int i_node, int n, int &i_local);
  NodeGroup *GroupOfList(const int *nodes, int n, std::vector<int> &local);
  void CheckUncalibrated(const std::string &msg);
  void BuildCSR();
  void BuildDevice();
  void UploadGeneratorParams();
  void FlushRecords();
  void WriteInitialRecord();
  GroupArgs MakeGroupArgs(NodeGroup *g);
  InputArgs MakeInputArgs(NodeGroup *g);
  bool HasLargePoisson(const NodeGroup *g) const;
  PushArgs MakePushArgs(NodeGroup *g);
  DeliverArgs MakeDeliverArgs();
  void SetParamColumn(NodeGroup *g, int col, int i0, int n, const int *nodes,
                      float val, const float *vals, int stride);
  void GetParamColumn(NodeGroup *g, float *col_base, int i0, int n,
                      const int *nodes, float *out, int stride);
  void CheckDeviceErrors();
  unsigned long long NextRngStream() { return rng_calls_++; }
  void AddEdge(int s, int t, unsigned char port, unsigned char syn, float w,
               float delay);
  void FreeDevice();
};

}  // namespace ngpu
