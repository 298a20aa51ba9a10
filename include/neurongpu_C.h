/* C ABI of the B200 simulation core.
 *
 * Every NeuronGPU_* entry point has the name, signature, argument meaning,
 * return convention and error behaviour of the reference's C interface
 * (golosio/NeuronGPU src/neurongpu_C.h; the line of each reference
 * declaration is given beside it), so the reference's ctypes layer
 * (pythonlib/neurongpu.py) or C++ programs linking -lneurongpu bind to this
 * library unchanged. Errors: each call clears the error state; on failure the
 * code is 2 (library error), 1 (allocation failure) or 255 (other), the
 * message is kept for NeuronGPU_GetErrorMessage, and the process exits with
 * that code unless NeuronGPU_SetOnException(1) was called. Arrays returned by
 * Get* calls are allocated by the library and owned by the caller.
 *
 * The NGB200_* entry points at the end have no counterpart in the reference:
 * they expose device counters and run-time controls of this build.
 */
#ifndef NEURONGPU_B200_C_H
#define NEURONGPU_B200_C_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

char *NeuronGPU_GetErrorMessage();                          /* neurongpu_C.h:22 */
unsigned char NeuronGPU_GetErrorCode();                     /* neurongpu_C.h:24 */
void NeuronGPU_SetOnException(int on_exception);            /* neurongpu_C.h:26 */
int NeuronGPU_SetRandomSeed(unsigned long long seed);       /* neurongpu_C.h:28 */
int NeuronGPU_SetTimeResolution(float time_res);            /* neurongpu_C.h:30 */
float NeuronGPU_GetTimeResolution();                        /* neurongpu_C.h:32 */
int NeuronGPU_SetMaxSpikeBufferSize(int max_size);          /* neurongpu_C.h:34 */
int NeuronGPU_GetMaxSpikeBufferSize();                      /* neurongpu_C.h:36 */
int NeuronGPU_SetSimTime(float sim_time);                   /* neurongpu_C.h:38 */
int NeuronGPU_SetVerbosityLevel(int verbosity_level);       /* neurongpu_C.h:40 */
int NeuronGPU_Create(char *model_name, int n_neuron, int n_port);   /* :42 */
int NeuronGPU_CreatePoissonGenerator(int n_node, float rate);       /* :44 */
int NeuronGPU_CreateRecord(char *file_name, char *var_name_arr[],
                           int *i_node_arr, int *port_arr, int n_node); /* :46 */
int NeuronGPU_GetRecordDataRows(int i_record);              /* neurongpu_C.h:50 */
int NeuronGPU_GetRecordDataColumns(int i_record);           /* neurongpu_C.h:52 */
float **NeuronGPU_GetRecordData(int i_record);              /* neurongpu_C.h:54 */
int NeuronGPU_SetNeuronScalParam(int i_node, int n_neuron, char *param_name,
                                 float val);                /* neurongpu_C.h:56 */
int NeuronGPU_SetNeuronArrayParam(int i_node, int n_neuron, char *param_name,
                                  float *param, int array_size);    /* :59 */
int NeuronGPU_SetNeuronPtScalParam(int *i_node, int n_neuron,
                                   char *param_name, float val);    /* :63 */
int NeuronGPU_SetNeuronPtArrayParam(int *i_node, int n_neuron,
                                    char *param_name, float *param,
                                    int array_size);                /* :66 */
int NeuronGPU_IsNeuronScalParam(int i_node, char *param_name);      /* :70 */
int NeuronGPU_IsNeuronPortParam(int i_node, char *param_name);      /* :72 */
int NeuronGPU_IsNeuronArrayParam(int i_node, char *param_name);     /* :74 */
int NeuronGPU_SetNeuronIntVar(int i_node, int n_neuron, char *var_name,
                              int val);                     /* neurongpu_C.h:77 */
int NeuronGPU_SetNeuronScalVar(int i_node, int n_neuron, char *var_name,
                               float val);                  /* neurongpu_C.h:80 */
int NeuronGPU_SetNeuronArrayVar(int i_node, int n_neuron, char *var_name,
                                float *var, int array_size);        /* :83 */
int NeuronGPU_SetNeuronPtIntVar(int *i_node, int n_neuron, char *var_name,
                                int val);                   /* neurongpu_C.h:87 */
int NeuronGPU_SetNeuronPtScalVar(int *i_node, int n_neuron, char *var_name,
                                 float val);                /* neurongpu_C.h:90 */
int NeuronGPU_SetNeuronPtArrayVar(int *i_node, int n_neuron, char *var_name,
                                  float *var, int array_size);      /* :93 */
int NeuronGPU_IsNeuronIntVar(int i_node, char *var_name);           /* :97 */
int NeuronGPU_IsNeuronScalVar(int i_node, char *var_name);          /* :99 */
int NeuronGPU_IsNeuronPortVar(int i_node, char *var_name);          /* :101 */
int NeuronGPU_IsNeuronArrayVar(int i_node, char *var_name);         /* :103 */
int NeuronGPU_GetNeuronParamSize(int i_node, char *param_name);     /* :105 */
int NeuronGPU_GetNeuronVarSize(int i_node, char *var_name);         /* :107 */
float *NeuronGPU_GetNeuronParam(int i_node, int n_neuron,
                                char *param_name);          /* neurongpu_C.h:109 */
float *NeuronGPU_GetNeuronPtParam(int *i_node, int n_neuron,
                                  char *param_name);        /* neurongpu_C.h:112 */
float *NeuronGPU_GetArrayParam(int i_node, char *param_name);       /* :115 */
int *NeuronGPU_GetNeuronIntVar(int i_node, int n_neuron,
                               char *param_name);           /* neurongpu_C.h:117 */
int *NeuronGPU_GetNeuronPtIntVar(int *i_node, int n_neuron,
                                 char *param_name);         /* neurongpu_C.h:120 */
float *NeuronGPU_GetNeuronVar(int i_node, int n_neuron,
                              char *param_name);            /* neurongpu_C.h:123 */
float *NeuronGPU_GetNeuronPtVar(int *i_node, int n_neuron,
                                char *param_name);          /* neurongpu_C.h:126 */
float *NeuronGPU_GetArrayVar(int i_node, char *var_name);           /* :129 */
int NeuronGPU_Calibrate();                                  /* neurongpu_C.h:131 */
int NeuronGPU_Simulate();                                   /* neurongpu_C.h:133 */
int NeuronGPU_StartSimulation();                            /* neurongpu_C.h:135 */
int NeuronGPU_SimulationStep();                             /* neurongpu_C.h:137 */
int NeuronGPU_EndSimulation();                              /* neurongpu_C.h:139 */
int NeuronGPU_ConnectMpiInit(int argc, char *argv[]);       /* neurongpu_C.h:141 */
int NeuronGPU_MpiId();                                      /* neurongpu_C.h:143 */
int NeuronGPU_MpiNp();                                      /* neurongpu_C.h:145 */
int NeuronGPU_ProcMaster();                                 /* neurongpu_C.h:147 */
int NeuronGPU_MpiFinalize();                                /* neurongpu_C.h:149 */
unsigned int *NeuronGPU_RandomInt(size_t n);                /* neurongpu_C.h:151 */
float *NeuronGPU_RandomUniform(size_t n);                   /* neurongpu_C.h:153 */
float *NeuronGPU_RandomNormal(size_t n, float mean, float stddev);  /* :155 */
float *NeuronGPU_RandomNormalClipped(size_t n, float mean, float stddev,
                                     float vmin, float vmax,
                                     float vstep);          /* neurongpu_C.h:157 */
int NeuronGPU_Connect(int i_source_node, int i_target_node,
                      unsigned char port, unsigned char syn_group,
                      float weight, float delay);           /* neurongpu_C.h:160 */
int NeuronGPU_ConnSpecInit();                               /* neurongpu_C.h:164 */
int NeuronGPU_SetConnSpecParam(char *param_name, int value);        /* :166 */
int NeuronGPU_ConnSpecIsParam(char *param_name);            /* neurongpu_C.h:168 */
int NeuronGPU_SynSpecInit();                                /* neurongpu_C.h:170 */
int NeuronGPU_SetSynSpecIntParam(char *param_name, int value);      /* :172 */
int NeuronGPU_SetSynSpecFloatParam(char *param_name, float value);  /* :174 */
int NeuronGPU_SetSynSpecFloatPtParam(char *param_name,
                                     float *array_pt);      /* neurongpu_C.h:176 */
int NeuronGPU_SynSpecIsIntParam(char *param_name);          /* neurongpu_C.h:178 */
int NeuronGPU_SynSpecIsFloatParam(char *param_name);        /* neurongpu_C.h:180 */
int NeuronGPU_SynSpecIsFloatPtParam(char *param_name);      /* neurongpu_C.h:182 */
int NeuronGPU_ConnectSeqSeq(int i_source, int n_source, int i_target,
                            int n_target);                  /* neurongpu_C.h:184 */
int NeuronGPU_ConnectSeqGroup(int i_source, int n_source, int *i_target,
                              int n_target);                /* neurongpu_C.h:187 */
int NeuronGPU_ConnectGroupSeq(int *i_source, int n_source, int i_target,
                              int n_target);                /* neurongpu_C.h:190 */
int NeuronGPU_ConnectGroupGroup(int *i_source, int n_source, int *i_target,
                                int n_target);              /* neurongpu_C.h:193 */
int NeuronGPU_RemoteConnectSeqSeq(int i_source_host, int i_source,
                                  int n_source, int i_target_host,
                                  int i_target, int n_target);      /* :196 */
int NeuronGPU_RemoteConnectSeqGroup(int i_source_host, int i_source,
                                    int n_source, int i_target_host,
                                    int *i_target, int n_target);   /* :200 */
int NeuronGPU_RemoteConnectGroupSeq(int i_source_host, int *i_source,
                                    int n_source, int i_target_host,
                                    int i_target, int n_target);    /* :204 */
int NeuronGPU_RemoteConnectGroupGroup(int i_source_host, int *i_source,
                                      int n_source, int i_target_host,
                                      int *i_target, int n_target); /* :208 */
char **NeuronGPU_GetIntVarNames(int i_node);                /* neurongpu_C.h:212 */
char **NeuronGPU_GetScalVarNames(int i_node);               /* neurongpu_C.h:214 */
int NeuronGPU_GetNIntVar(int i_node);                       /* neurongpu_C.h:216 */
int NeuronGPU_GetNScalVar(int i_node);                      /* neurongpu_C.h:218 */
char **NeuronGPU_GetPortVarNames(int i_node);               /* neurongpu_C.h:220 */
int NeuronGPU_GetNPortVar(int i_node);                      /* neurongpu_C.h:222 */
char **NeuronGPU_GetScalParamNames(int i_node);             /* neurongpu_C.h:224 */
int NeuronGPU_GetNScalParam(int i_node);                    /* neurongpu_C.h:226 */
char **NeuronGPU_GetPortParamNames(int i_node);             /* neurongpu_C.h:228 */
int NeuronGPU_GetNGroupParam(int i_node);                   /* neurongpu_C.h:230 */
char **NeuronGPU_GetGroupParamNames(int i_node);            /* neurongpu_C.h:232 */
int NeuronGPU_GetNPortParam(int i_node);                    /* neurongpu_C.h:234 */
char **NeuronGPU_GetArrayParamNames(int i_node);            /* neurongpu_C.h:236 */
int NeuronGPU_GetNArrayParam(int i_node);                   /* neurongpu_C.h:238 */
char **NeuronGPU_GetArrayVarNames(int i_node);              /* neurongpu_C.h:240 */
int NeuronGPU_GetNArrayVar(int i_node);                     /* neurongpu_C.h:242 */
int *NeuronGPU_GetSeqSeqConnections(int i_source, int n_source, int i_target,
                                    int n_target, int syn_group,
                                    int *n_conn);           /* neurongpu_C.h:244 */
int *NeuronGPU_GetSeqGroupConnections(int i_source, int n_source,
                                      int *i_target, int n_target,
                                      int syn_group, int *n_conn);  /* :247 */
int *NeuronGPU_GetGroupSeqConnections(int *i_source, int n_source,
                                      int i_target, int n_target,
                                      int syn_group, int *n_conn);  /* :251 */
int *NeuronGPU_GetGroupGroupConnections(int *i_source, int n_source,
                                        int *i_target, int n_target,
                                        int syn_group, int *n_conn); /* :255 */
int NeuronGPU_GetConnectionStatus(int i_source, int i_group, int i_conn,
                                  int *i_target, unsigned char *port,
                                  unsigned char *syn_group, float *delay,
                                  float *weight);           /* neurongpu_C.h:258 */
int NeuronGPU_CreateSynGroup(char *model_name);             /* neurongpu_C.h:263 */
int NeuronGPU_GetSynGroupNParam(int i_syn_group);           /* neurongpu_C.h:265 */
char **NeuronGPU_GetSynGroupParamNames(int i_syn_group);    /* neurongpu_C.h:267 */
int NeuronGPU_IsSynGroupParam(int i_syn_group, char *param_name);   /* :269 */
int NeuronGPU_GetSynGroupParamIdx(int i_syn_group, char *param_name); /* :271 */
float NeuronGPU_GetSynGroupParam(int i_syn_group, char *param_name);  /* :273 */
int NeuronGPU_SetSynGroupParam(int i_syn_group, char *param_name,
                               float val);                  /* neurongpu_C.h:275 */
int NeuronGPU_ActivateSpikeCount(int i_node, int n_node);   /* neurongpu_C.h:277 */
int NeuronGPU_ActivateRecSpikeTimes(int i_node, int n_node,
                                    int max_n_rec_spike_times);     /* :279 */
int NeuronGPU_GetNRecSpikeTimes(int i_node);                /* neurongpu_C.h:282 */
float *NeuronGPU_GetRecSpikeTimes(int i_node);              /* neurongpu_C.h:284 */
int NeuronGPU_PushSpikesToNodes(int n_spikes, int *node_id);        /* :286 */
int NeuronGPU_GetExtNeuronInputSpikes(int *n_spikes, int **node, int **port,
                                      float **spike_height,
                                      int include_zeros);   /* neurongpu_C.h:288 */
int NeuronGPU_SetNeuronGroupParam(int i_node, int n_node, char *param_name,
                                  float val);               /* neurongpu_C.h:292 */
int NeuronGPU_IsNeuronGroupParam(int i_node, char *param_name);     /* :295 */
float NeuronGPU_GetNeuronGroupParam(int i_node, char *param_name);  /* :297 */
int NeuronGPU_GetNFloatParam();                             /* neurongpu_C.h:299 */
char **NeuronGPU_GetFloatParamNames();                      /* neurongpu_C.h:301 */
int NeuronGPU_IsFloatParam(char *param_name);               /* neurongpu_C.h:303 */
int NeuronGPU_GetFloatParamIdx(char *param_name);           /* neurongpu_C.h:305 */
float NeuronGPU_GetFloatParam(char *param_name);            /* neurongpu_C.h:307 */
int NeuronGPU_SetFloatParam(char *param_name, float val);   /* neurongpu_C.h:309 */
int NeuronGPU_GetNIntParam();                               /* neurongpu_C.h:311 */
char **NeuronGPU_GetIntParamNames();                        /* neurongpu_C.h:313 */
int NeuronGPU_IsIntParam(char *param_name);                 /* neurongpu_C.h:315 */
int NeuronGPU_GetIntParamIdx(char *param_name);             /* neurongpu_C.h:317 */
int NeuronGPU_GetIntParam(char *param_name);                /* neurongpu_C.h:319 */
int NeuronGPU_SetIntParam(char *param_name, int val);       /* neurongpu_C.h:321 */
int NeuronGPU_RemoteCreate(int i_host, char *model_name, int n_neuron,
                           int n_port);                     /* neurongpu_C.h:323 */

/* ---- extensions of this build (no counterpart in the reference) ---- */

/* Destroys the simulation instance and frees its device memory, so one
 * process can build and run several independent networks in sequence. */
int NGB200_Reset();
/* RK5 right-hand-side evaluations performed so far (all RK5 groups). */
unsigned long long NGB200_StageEvaluations();
/* Synaptic events (spike x synapse) delivered so far. */
unsigned long long NGB200_DeliveredEvents();
/* Spikes emitted so far (all nodes). */
unsigned long long NGB200_TotalSpikes();

/* Networks partitioned over hosts, one GPU per host process. These replace
 * the reference's MPI transport (src/spike_mpi.cu:284-486, the per-step
 * exchange of src/neurongpu.cu:490-521); NeuronGPU_ConnectMpiInit takes the
 * host index and count from the job launcher's environment, and the remote
 * entry points above make image nodes on the target host and mark exported
 * nodes on the source host. The caller moves the spikes between hosts with
 * its own collective, every NGB200_RemoteExchangeSteps() steps:
 *   NGB200_SimulateSteps(E); count = NGB200_PackRemoteSpikes(E, buf, cap);
 *   all-gather the lists; NGB200_UnpackRemoteSpikes(h, E, list_h, count_h)
 *   for every other host h.
 * The Python layer's Simulate does this with torch.distributed. */
/* Sets this instance's host index and host count. */
int NGB200_SetHost(int id, int n_hosts);
/* Runs n_steps steps of a started simulation (NeuronGPU_StartSimulation). */
int NGB200_SimulateSteps(long long n_steps);
/* The longest exchange interval (steps) this host allows: the shortest delay
 * of a connection from an image node, and on a host that exports spikes the
 * steps its spike ring keeps (at least 32); 0 if it neither receives nor
 * sends remote spikes. The hosts exchange at the minimum over all hosts. */
int NGB200_RemoteExchangeSteps();
/* Packs the spikes of exported nodes emitted in the last n_steps steps into
 * the device buffer buf of 4 + 3 * cap 32-bit words: [count, overflow, 0, 0]
 * then (step offset, node, height bits) per spike. Returns the count; when
 * it exceeds cap only cap spikes were written: pack again into a larger
 * buffer (the spikes stay in the ring). Synchronises the simulation stream. */
long long NGB200_PackRemoteSpikes(int n_steps, void *buf, long long cap);
/* Pushes the spikes of host src_host's packed list (device buffer, count
 * entries) whose nodes have images here into the spike ring, at the steps
 * they were emitted; n_steps as in the matching pack. Queued on the
 * simulation stream. */
int NGB200_UnpackRemoteSpikes(int src_host, int n_steps, const void *buf, long long count);
/* The rate (synaptic events per second) at which this GPU delivers events
 * when nothing else limits the delivery: n_events edges (4-byte target slot,
 * 4-byte weight) added as 64-bit fixed-point values into n_slots randomly
 * addressed accumulators by the delivery kernel's inner loop, timed over
 * reps launches. The bench uses it as the bound of the delivery (mostly the
 * L2's 64-bit reductions). Allocates its own arrays; returns 0 on success. */
int NGB200_StreamingDeliveryRate(long long n_slots, long long n_events, int reps,
                                 double *events_per_s);
/* Selects simulation instance k (0 <= k < 16; created on first use): every
 * later call of this interface acts on it. Instance 0 is the default. */
int NGB200_SetInstance(int k);
int NGB200_GetInstance();
/* Host wall time of the last NeuronGPU_Simulate call, in seconds. */
double NGB200_LastSimulateSeconds();
/* Steps per captured CUDA graph (default 100); 0 launches without graphs. */
int NGB200_SetGraphChunk(int n_steps);
/* Total number of nodes and of connections. */
long long NGB200_NNodes();
long long NGB200_NConnections();
/* RK5 node groups of the same model and port count are integrated by one
 * kernel launch per time step through a device segment table (many
 * independent networks, e.g. a parameter sweep). on = 0 gives every group
 * its own launch; must be called before the first simulation. Default on.
 * No reference counterpart (the reference launches one kernel per node
 * group, src/neurongpu.cu:481-483). */
int NGB200_SetRk5Batching(int on);
/* Index of the batched RK5 launch the node's group belongs to, -1 if the
 * group has its own launch (valid after the first simulation). */
int NGB200_Rk5BatchOf(int i_node);
/* Learned RK5 step proposer (no reference counterpart; the reference sizes
 * every RK5 sub-step with the embedded-error controller of src/rk5.h:57-147
 * only). A 6 -> 32 -> 32 -> 1 MLP over (V, w, conductances, previous step)
 * proposes the next sub-step of aeif_cond_beta / aeif_cond_alpha neurons
 * (1 or 2 ports) whenever the controller's own guess is shorter than the rest
 * of the time step; the RK5 error test still accepts or rejects every step.
 * i_node selects the node's group; -1 selects every supported group. */
/* Log accepted sub-steps of the plain controller (capacity rows of 8 floats:
 * 6 features, target log2(h/dt), 0); capacity 0 stops logging. */
int NGB200_SetStepLog(int i_node, int capacity);
/* Number of sub-steps logged so far (may exceed the capacity). */
long long NGB200_GetStepLogCount(int i_node);
/* Copies up to max_rows logged rows; returns the number copied. */
int NGB200_GetStepLog(int i_node, float *out, int max_rows);
/* Trains the proposer on every logged row (GPU forward / backward kernels,
 * FP32 Adam, steps mini-batches of blocks x 64 rows); logging stops. Returns
 * the number of rows; losses are mean squared errors of log2(h/dt) averaged
 * over the first and the last 5% of the steps. */
int NGB200_TrainStepProposer(int steps, int blocks, float lr, unsigned long long seed,
                             float *loss_first, float *loss_last);
/* Uses (on != 0) or stops using the trained proposer for the group. */
int NGB200_SetStepProposer(int i_node, int on);
/* The 1313 FP32 parameters: W1[32][6], b1[32], W2[32][32], b2[32], w3[32], b3. */
int NGB200_SetStepProposerParams(const float *params);
int NGB200_GetStepProposerParams(float *params);
/* Proposed step = dt * 2^(output - margin); default margin 0.25. */
int NGB200_SetStepProposerMargin(float margin);
/* Test entry points: mean gradient (1313 floats) and loss of the training
 * kernels over n samples of 8 floats; tensor-core inference of n rows of 6
 * features with the given parameters. */
float NGB200_MlpGradients(const float *data, int n_samples, const float *params, float *grad);
int NGB200_MlpInfer(const float *x6, int n_rows, const float *params, float *out);
/* Every connection in one call, in delivery order (source, delay group,
 * insertion; the order of NeuronGPU_GetSeqSeqConnections over all nodes).
 * Each non-null array must hold NGB200_NConnections() elements; weights are
 * the current device values once the network is calibrated. Returns the
 * number of connections. No reference counterpart (the reference returns
 * connections one status call at a time, src/neurongpu_C.h:294-331). */
long long NGB200_GetAllConnections(int *src, int *tgt, int *port, int *syn,
                                   float *delay, float *weight);
/* Releases an array returned by one of the entry points that hand the
 * caller a fresh host array: NeuronGPU_GetNeuronParam / GetNeuronPtParam /
 * GetArrayParam / GetNeuronIntVar / GetNeuronVar / GetNeuronPtIntVar /
 * GetNeuronPtVar / GetArrayVar / GetRecSpikeTimes / GetRecordData (the row
 * table only) / Random* and the Get*Connections lists. The reference's
 * entry points (src/neurongpu_C.h:54, 109-129, 151-157, 244-255, 284) hand
 * out such arrays with no way to release them; calling this is optional,
 * null is ignored. */
void NGB200_FreeArray(void *p);
/* Device time (CUDA events on the simulation stream) of the step loop of the
 * last NeuronGPU_Simulate call, in ms. */
double NGB200_LastSimulateDeviceMs();
/* Kernel launches per time step in the most recently captured step graph
 * (0 before the first capture). No reference counterpart. */
double NGB200_KernelsPerStep();
/* Per-kernel-class timing: on != 0 records CUDA events around every kernel
 * class of every step (resets the totals). Classes: 0 node updates,
 * 1 spike delivery, 2 STDP post rule, 3 recording and step bookkeeping. */
int NGB200_SetKernelTiming(int on);
int NGB200_GetKernelTiming(int kind, double *total_ms, long long *launches);
/* RK5 sub-steps one neuron may take in one time step (default 200,000)
 * before its update gives up on the step and Simulate fails with "RK5
 * integration exceeded the substep limit" (the reference has no limit). */
int NGB200_SetRk5MaxSubsteps(int n_substeps);
/* Test hook for the time-out paths of the bounded device waits: mask bit 0
 * makes the shared-memory prefetch wait of the persistent RK5 update and the
 * first tensor-core wait of each step-proposer round give up after one
 * non-blocking test, bit 1 the second tensor-core wait of a round; 0 (the
 * default) restores normal waits. A wait that gives up sets its error bit,
 * which the next Simulate reports; the kernels still wait (bounded) for
 * their outstanding copies and tensor-core work before they exit. */
int NGB200_SetWaitTest(int mask);
/* Parity bookkeeping of a step-proposer round's completion barrier (host
 * copy of the device function): the parity kept after a round that started
 * at phase_in, whose first / second completion wait succeeded (ok1 / ok2). */
unsigned NGB200_ProposerPhaseAfter(unsigned phase_in, int ok1, int ok2);
/* RK5 kernel variant picked by the autotuner for the group of node i_node
 * (0 = no register cap, 1..3 = caps for 5, 6, 8 resident blocks per SM,
 * 4..5 = persistent kernel with shared-memory prefetch of the state, caps
 * for 5 and 6 blocks per SM, 6 = cap for 4 blocks per SM, 7..8 = persistent
 * kernel with caps for 4 and 3 blocks per SM) and, in ms[0..8], the median
 * device time (ms) of each variant's timing launch (0 for variants not
 * timed). The tuner runs
 * once a simulation has integrated 200 steps, for groups with >= 16384
 * neurons; the environment variable NGB200_RK5_VARIANT forces a variant from
 * the first step, NGB200_AUTOTUNE=0 disables tuning. */
int NGB200_GetRk5Tuning(int i_node, int *variant, float *ms);

/* Standalone synaptic delivery, the simulator's delivery kernel applied to a
 * caller-owned graph and spike batch (all pointers are device memory):
 *   grp_off[n_src*nd + 1]  edge range of (source s, delay index di) is
 *                          [grp_off[s*nd+di], grp_off[s*nd+di+1])
 *   e_slot[E], e_w[E]      accumulator index and weight of every synapse
 *   spike_src[k], spike_h[k], spike_di[k]   source, height and delay index
 *                          (0 <= di < nd, nd <= 1024) of spike k
 *   acc[]                  64-bit fixed-point accumulators (32 fractional
 *                          bits), zeroed by the caller; every synapse of
 *                          every spike adds round(h*w * 2^32)
 * Scratch device memory for the per-delay spike lists is allocated and
 * released inside the call; the call returns after the stream is drained.
 * Returns 0 on success, 1 bad arguments, 2 allocation failure, 3 CUDA
 * error, 4 a spike with an out-of-range delay index. */
int NGB200_DeliverSpikes(const unsigned long long *grp_off,
                         const unsigned *e_slot, const float *e_w, int nd,
                         const unsigned *spike_src, const float *spike_h,
                         const int *spike_di, int n_spikes, long long *acc,
                         void *stream);

/* NGB200_DeliverSpikes without any device allocation. This entry point has
 * no counterpart in the reference. It is for callers that cannot allocate
 * device memory while they run: a host program whose own allocator owns the
 * device memory, or a loop that must not stall, where a cudaMalloc / cudaFree
 * could fail or would synchronise the device and block the caller's other
 * streams. Same arguments and result as NGB200_DeliverSpikes. Its scratch is
 * a file-scope __device__ array of about 8 MiB that every GPU loading the
 * library keeps until the process exits; a batch may use at most
 * (nd + 1) * n_spikes <= 1048576 spike-list entries, larger batches are
 * rejected with return code 5 before any work is queued. The first call on a
 * device looks up the array's device address with that device current; make
 * that first call before any stream capture. The address is kept for the
 * life of the process: do not call this entry point after cudaDeviceReset
 * (the reset ends the context the address belongs to). All calls share the array:
 * each call clears its counters and error word first, and calls that
 * overlap on the GPU race on it. Returns after the stream is drained. */
int NGB200_DeliverSpikesNoAlloc(const unsigned long long *grp_off,
                                const unsigned *e_slot, const float *e_w,
                                int nd, const unsigned *spike_src,
                                const float *spike_h, const int *spike_di,
                                int n_spikes, long long *acc, void *stream);

#ifdef __cplusplus
}
#endif

#endif
