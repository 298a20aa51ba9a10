// extern "C" entry points over one process-wide NeuronGPU instance, with the
// reference's error convention (src/neurongpu_C.cpp:25-34,
// src/propagate_error.h:4-30): every call clears the error state, catches
// exceptions, records code 2 / 1 / 255 and exits unless the caller asked for
// errors to be returned (NeuronGPU_SetOnException(1)).
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <iostream>
#include <new>
#include <string>
#include <vector>

#include "../../include/neurongpu_C.h"
#include "ngpu_core.h"

using ngpu::ConnectionId;
using ngpu::ConnectionStatus;
using ngpu::NeuronGPU;

// Instances: one by default, as in the reference; NGB200_SetInstance selects
// another (several simulators in one process, e.g. the hosts of a
// partitioned network driven from one process).
static const int kMaxInstances = 16;
static NeuronGPU *g_inst[kMaxInstances] = {nullptr};
static int g_cur = 0;

static NeuronGPU *inst() {
  if (g_inst[g_cur] == nullptr) g_inst[g_cur] = new NeuronGPU();
  return g_inst[g_cur];
}

// host index and count of this process in a job launched one process per
// GPU: the launcher's environment (torchrun RANK / WORLD_SIZE, Open MPI,
// PMI), 0 of 1 without one
static void host_from_env(int *id, int *n) {
  const char *pairs[][2] = {{"RANK", "WORLD_SIZE"},
                            {"OMPI_COMM_WORLD_RANK", "OMPI_COMM_WORLD_SIZE"},
                            {"PMI_RANK", "PMI_SIZE"}};
  *id = 0;
  *n = 1;
  for (auto &p : pairs) {
    const char *r = getenv(p[0]), *s = getenv(p[1]);
    if (r != nullptr && s != nullptr) {
      *id = atoi(r);
      *n = atoi(s);
      return;
    }
  }
}

template <class R, class F>
static R guarded(R dflt, F f) {
  NeuronGPU *n = inst();
  n->SetErrorFlag(false);
  n->SetErrorMessage("");
  n->SetErrorCode(0);
  R ret = dflt;
  try {
    ret = f(n);
  } catch (ngpu::ngpu_exception &e) {
    n->SetErrorFlag(true);
    n->SetErrorMessage(e.what());
    n->SetErrorCode(2);
  } catch (std::bad_alloc &) {
    n->SetErrorFlag(true);
    n->SetErrorMessage("Memory allocation error.");
    n->SetErrorCode(1);
  } catch (std::exception &e) {
    n->SetErrorFlag(true);
    n->SetErrorMessage(std::string("Error in NeuronGPU function: ") + e.what());
    n->SetErrorCode(255);
  } catch (...) {
    n->SetErrorFlag(true);
    n->SetErrorMessage("Error in NeuronGPU function.");
    n->SetErrorCode(255);
  }
  if (n->GetErrorCode() != 0 && n->OnException() == ngpu::ON_EXCEPTION_EXIT) {
    std::cerr << n->GetErrorMessage();
    exit(n->GetErrorCode());
  }
  return ret;
}

static char **names_to_c(const std::vector<std::string> &v) {
  char **arr = (char **)malloc(sizeof(char *) * (v.size() > 0 ? v.size() : 1));
  for (size_t i = 0; i < v.size(); i++) {
    arr[i] = (char *)malloc(v[i].size() + 1);
    strcpy(arr[i], v[i].c_str());
  }
  return arr;
}

static int *conn_ids_to_c(const std::vector<ConnectionId> &v, int *n_conn) {
  *n_conn = (int)v.size();
  int *a = (int *)malloc(sizeof(int) * 3 * (v.size() > 0 ? v.size() : 1));
  for (size_t i = 0; i < v.size(); i++) {
    a[3 * i] = v[i].i_source_;
    a[3 * i + 1] = v[i].i_group_;
    a[3 * i + 2] = v[i].i_conn_;
  }
  return a;
}

extern "C" {

char *NeuronGPU_GetErrorMessage() { return inst()->GetErrorMessage(); }
unsigned char NeuronGPU_GetErrorCode() { return inst()->GetErrorCode(); }
void NeuronGPU_SetOnException(int on_exception) { inst()->SetOnException(on_exception); }

int NeuronGPU_SetRandomSeed(unsigned long long seed) {
  return guarded(0, [&](NeuronGPU *n) { return n->SetRandomSeed(seed); });
}
int NeuronGPU_SetTimeResolution(float t) {
  return guarded(0, [&](NeuronGPU *n) { return n->SetTimeResolution(t); });
}
float NeuronGPU_GetTimeResolution() {
  return guarded(0.0f, [&](NeuronGPU *n) { return n->GetTimeResolution(); });
}
int NeuronGPU_SetMaxSpikeBufferSize(int m) {
  return guarded(0, [&](NeuronGPU *n) { return n->SetMaxSpikeBufferSize(m); });
}
int NeuronGPU_GetMaxSpikeBufferSize() {
  return guarded(0, [&](NeuronGPU *n) { return n->GetMaxSpikeBufferSize(); });
}
int NeuronGPU_SetSimTime(float t) {
  return guarded(0, [&](NeuronGPU *n) { return n->SetSimTime(t); });
}
int NeuronGPU_SetVerbosityLevel(int v) {
  return guarded(0, [&](NeuronGPU *n) { return n->SetVerbosityLevel(v); });
}
int NeuronGPU_Create(char *model_name, int n_neuron, int n_port) {
  return guarded(0, [&](NeuronGPU *n) { return n->Create(model_name, n_neuron, n_port); });
}
int NeuronGPU_CreatePoissonGenerator(int n_node, float rate) {
  return guarded(0, [&](NeuronGPU *n) { return n->CreatePoissonGenerator(n_node, rate); });
}
int NeuronGPU_CreateRecord(char *file_name, char *var_name_arr[], int *i_node_arr,
                           int *port_arr, int n_node) {
  return guarded(0, [&](NeuronGPU *n) {
    std::vector<std::string> vars;
    for (int i = 0; i < n_node; i++) vars.push_back(var_name_arr[i]);
    return n->CreateRecord(file_name, vars, i_node_arr, port_arr, n_node);
  });
}
int NeuronGPU_GetRecordDataRows(int i_record) {
  return guarded(0, [&](NeuronGPU *n) { return (int)n->GetRecordData(i_record)->size(); });
}
int NeuronGPU_GetRecordDataColumns(int i_record) {
  return guarded(0, [&](NeuronGPU *n) {
    auto *d = n->GetRecordData(i_record);
    if (d->empty()) throw ngpu::ngpu_exception("Record has no data");
    return (int)d->at(0).size();
  });
}
float **NeuronGPU_GetRecordData(int i_record) {
  return guarded((float **)nullptr, [&](NeuronGPU *n) {
    auto *d = n->GetRecordData(i_record);
    float **rows = (float **)malloc(sizeof(float *) * (d->size() > 0 ? d->size() : 1));
    for (size_t i = 0; i < d->size(); i++) rows[i] = d->at(i).data();
    return rows;
  });
}
int NeuronGPU_SetNeuronScalParam(int i_node, int n_neuron, char *param_name, float val) {
  return guarded(0, [&](NeuronGPU *n) { return n->SetNeuronParam(i_node, n_neuron, param_name, val); });
}
int NeuronGPU_SetNeuronArrayParam(int i_node, int n_neuron, char *param_name, float *param,
                                  int array_size) {
  return guarded(0, [&](NeuronGPU *n) {
    return n->SetNeuronParam(i_node, n_neuron, param_name, param, array_size);
  });
}
int NeuronGPU_SetNeuronPtScalParam(int *i_node, int n_neuron, char *param_name, float val) {
  return guarded(0, [&](NeuronGPU *n) {
    return n->SetNeuronParam((const int *)i_node, n_neuron, param_name, val);
  });
}
int NeuronGPU_SetNeuronPtArrayParam(int *i_node, int n_neuron, char *param_name, float *param,
                                    int array_size) {
  return guarded(0, [&](NeuronGPU *n) {
    return n->SetNeuronParam((const int *)i_node, n_neuron, param_name, (const float *)param,
                             array_size);
  });
}
int NeuronGPU_IsNeuronScalParam(int i_node, char *p) {
  return guarded(0, [&](NeuronGPU *n) { return n->IsNeuronScalParam(i_node, p); });
}
int NeuronGPU_IsNeuronPortParam(int i_node, char *p) {
  return guarded(0, [&](NeuronGPU *n) { return n->IsNeuronPortParam(i_node, p); });
}
int NeuronGPU_IsNeuronArrayParam(int i_node, char *p) {
  return guarded(0, [&](NeuronGPU *n) { return n->IsNeuronArrayParam(i_node, p); });
}
int NeuronGPU_SetNeuronIntVar(int i_node, int n_neuron, char *v, int val) {
  return guarded(0, [&](NeuronGPU *n) { return n->SetNeuronIntVar(i_node, n_neuron, v, val); });
}
int NeuronGPU_SetNeuronScalVar(int i_node, int n_neuron, char *v, float val) {
  return guarded(0, [&](NeuronGPU *n) { return n->SetNeuronVar(i_node, n_neuron, v, val); });
}
int NeuronGPU_SetNeuronArrayVar(int i_node, int n_neuron, char *v, float *var, int size) {
  return guarded(0, [&](NeuronGPU *n) { return n->SetNeuronVar(i_node, n_neuron, v, var, size); });
}
int NeuronGPU_SetNeuronPtIntVar(int *i_node, int n_neuron, char *v, int val) {
  return guarded(0, [&](NeuronGPU *n) {
    return n->SetNeuronIntVar((const int *)i_node, n_neuron, v, val);
  });
}
int NeuronGPU_SetNeuronPtScalVar(int *i_node, int n_neuron, char *v, float val) {
  return guarded(0, [&](NeuronGPU *n) {
    return n->SetNeuronVar((const int *)i_node, n_neuron, v, val);
  });
}
int NeuronGPU_SetNeuronPtArrayVar(int *i_node, int n_neuron, char *v, float *var, int size) {
  return guarded(0, [&](NeuronGPU *n) {
    return n->SetNeuronVar((const int *)i_node, n_neuron, v, (const float *)var, size);
  });
}
int NeuronGPU_IsNeuronIntVar(int i_node, char *v) {
  return guarded(0, [&](NeuronGPU *n) { return n->IsNeuronIntVar(i_node, v); });
}
int NeuronGPU_IsNeuronScalVar(int i_node, char *v) {
  return guarded(0, [&](NeuronGPU *n) { return n->IsNeuronScalVar(i_node, v); });
}
int NeuronGPU_IsNeuronPortVar(int i_node, char *v) {
  return guarded(0, [&](NeuronGPU *n) { return n->IsNeuronPortVar(i_node, v); });
}
int NeuronGPU_IsNeuronArrayVar(int i_node, char *v) {
  return guarded(0, [&](NeuronGPU *n) { return n->IsNeuronArrayVar(i_node, v); });
}
int NeuronGPU_GetNeuronParamSize(int i_node, char *p) {
  return guarded(0, [&](NeuronGPU *n) { return n->GetNeuronParamSize(i_node, p); });
}
int NeuronGPU_GetNeuronVarSize(int i_node, char *v) {
  return guarded(0, [&](NeuronGPU *n) { return n->GetNeuronVarSize(i_node, v); });
}
float *NeuronGPU_GetNeuronParam(int i_node, int n_neuron, char *p) {
  return guarded((float *)nullptr, [&](NeuronGPU *n) { return n->GetNeuronParam(i_node, n_neuron, p); });
}
float *NeuronGPU_GetNeuronPtParam(int *i_node, int n_neuron, char *p) {
  return guarded((float *)nullptr, [&](NeuronGPU *n) {
    return n->GetNeuronParam((const int *)i_node, n_neuron, p);
  });
}
float *NeuronGPU_GetArrayParam(int i_node, char *p) {
  return guarded((float *)nullptr, [&](NeuronGPU *n) { return n->GetArrayParam(i_node, p); });
}
int *NeuronGPU_GetNeuronIntVar(int i_node, int n_neuron, char *p) {
  return guarded((int *)nullptr, [&](NeuronGPU *n) { return n->GetNeuronIntVar(i_node, n_neuron, p); });
}
int *NeuronGPU_GetNeuronPtIntVar(int *i_node, int n_neuron, char *p) {
  return guarded((int *)nullptr, [&](NeuronGPU *n) {
    return n->GetNeuronIntVar((const int *)i_node, n_neuron, p);
  });
}
float *NeuronGPU_GetNeuronVar(int i_node, int n_neuron, char *p) {
  return guarded((float *)nullptr, [&](NeuronGPU *n) { return n->GetNeuronVar(i_node, n_neuron, p); });
}
float *NeuronGPU_GetNeuronPtVar(int *i_node, int n_neuron, char *p) {
  return guarded((float *)nullptr, [&](NeuronGPU *n) {
    return n->GetNeuronVar((const int *)i_node, n_neuron, p);
  });
}
float *NeuronGPU_GetArrayVar(int i_node, char *v) {
  return guarded((float *)nullptr, [&](NeuronGPU *n) { return n->GetArrayVar(i_node, v); });
}
int NeuronGPU_Calibrate() { return guarded(0, [&](NeuronGPU *n) { return n->Calibrate(); }); }
int NeuronGPU_Simulate() { return guarded(0, [&](NeuronGPU *n) { return n->Simulate(); }); }
int NeuronGPU_StartSimulation() {
  return guarded(0, [&](NeuronGPU *n) { return n->StartSimulation(); });
}
int NeuronGPU_SimulationStep() {
  return guarded(0, [&](NeuronGPU *n) { return n->SimulationStep(); });
}
int NeuronGPU_EndSimulation() {
  return guarded(0, [&](NeuronGPU *n) { return n->EndSimulation(); });
}
// Without MPI: the host index and count come from the job launcher's
// environment; the spike exchange is driven by the caller's collective
// (NGB200_PackRemoteSpikes / NGB200_UnpackRemoteSpikes, the Python layer's
// Simulate uses torch.distributed).
int NeuronGPU_ConnectMpiInit(int, char *[]) {
  return guarded(0, [&](NeuronGPU *n) {
    int id = 0, np = 1;
    host_from_env(&id, &np);
    return n->SetHost(id, np);
  });
}
int NeuronGPU_MpiId() { return guarded(0, [&](NeuronGPU *n) { return n->HostId(); }); }
int NeuronGPU_MpiNp() { return guarded(0, [&](NeuronGPU *n) { return n->NHosts(); }); }
int NeuronGPU_ProcMaster() { return guarded(0, [&](NeuronGPU *n) { return n->HostId() == 0 ? 1 : 0; }); }
int NeuronGPU_MpiFinalize() { return guarded(0, [&](NeuronGPU *) { return 0; }); }
unsigned int *NeuronGPU_RandomInt(size_t n_) {
  return guarded((unsigned int *)nullptr, [&](NeuronGPU *n) { return n->RandomInt(n_); });
}
float *NeuronGPU_RandomUniform(size_t n_) {
  return guarded((float *)nullptr, [&](NeuronGPU *n) { return n->RandomUniform(n_); });
}
float *NeuronGPU_RandomNormal(size_t n_, float mean, float stddev) {
  return guarded((float *)nullptr, [&](NeuronGPU *n) { return n->RandomNormal(n_, mean, stddev); });
}
float *NeuronGPU_RandomNormalClipped(size_t n_, float mean, float stddev, float vmin, float vmax,
                                     float vstep) {
  return guarded((float *)nullptr, [&](NeuronGPU *n) {
    return n->RandomNormalClipped(n_, mean, stddev, vmin, vmax, vstep);
  });
}
int NeuronGPU_Connect(int i_source_node, int i_target_node, unsigned char port,
                      unsigned char syn_group, float weight, float delay) {
  return guarded(0, [&](NeuronGPU *n) {
    return n->Connect(i_source_node, i_target_node, port, syn_group, weight, delay);
  });
}
int NeuronGPU_ConnSpecInit() {
  return guarded(0, [&](NeuronGPU *n) { n->conn_spec_.Init(); return 0; });
}
int NeuronGPU_SetConnSpecParam(char *p, int value) {
  return guarded(0, [&](NeuronGPU *n) { return n->conn_spec_.SetParam(p, value); });
}
int NeuronGPU_ConnSpecIsParam(char *p) {
  return guarded(0, [&](NeuronGPU *) { return ngpu::ConnSpec::IsParam(p) ? 1 : 0; });
}
int NeuronGPU_SynSpecInit() {
  return guarded(0, [&](NeuronGPU *n) { n->syn_spec_.Init(); return 0; });
}
int NeuronGPU_SetSynSpecIntParam(char *p, int value) {
  return guarded(0, [&](NeuronGPU *n) { return n->syn_spec_.SetParam(std::string(p), value); });
}
int NeuronGPU_SetSynSpecFloatParam(char *p, float value) {
  return guarded(0, [&](NeuronGPU *n) { return n->syn_spec_.SetParam(std::string(p), value); });
}
int NeuronGPU_SetSynSpecFloatPtParam(char *p, float *array_pt) {
  return guarded(0, [&](NeuronGPU *n) {
    return n->syn_spec_.SetParam(std::string(p), (const float *)array_pt);
  });
}
int NeuronGPU_SynSpecIsIntParam(char *p) {
  return guarded(0, [&](NeuronGPU *) { return ngpu::SynSpec::IsIntParam(p) ? 1 : 0; });
}
int NeuronGPU_SynSpecIsFloatParam(char *p) {
  return guarded(0, [&](NeuronGPU *) { return ngpu::SynSpec::IsFloatParam(p) ? 1 : 0; });
}
int NeuronGPU_SynSpecIsFloatPtParam(char *p) {
  return guarded(0, [&](NeuronGPU *) { return ngpu::SynSpec::IsFloatPtParam(p) ? 1 : 0; });
}
int NeuronGPU_ConnectSeqSeq(int i_source, int n_source, int i_target, int n_target) {
  return guarded(0, [&](NeuronGPU *n) {
    return n->Connect(nullptr, i_source, n_source, nullptr, i_target, n_target, n->conn_spec_,
                      n->syn_spec_);
  });
}
int NeuronGPU_ConnectSeqGroup(int i_source, int n_source, int *i_target, int n_target) {
  return guarded(0, [&](NeuronGPU *n) {
    return n->Connect(nullptr, i_source, n_source, i_target, 0, n_target, n->conn_spec_,
                      n->syn_spec_);
  });
}
int NeuronGPU_ConnectGroupSeq(int *i_source, int n_source, int i_target, int n_target) {
  return guarded(0, [&](NeuronGPU *n) {
    return n->Connect(i_source, 0, n_source, nullptr, i_target, n_target, n->conn_spec_,
                      n->syn_spec_);
  });
}
int NeuronGPU_ConnectGroupGroup(int *i_source, int n_source, int *i_target, int n_target) {
  return guarded(0, [&](NeuronGPU *n) {
    return n->Connect(i_source, 0, n_source, i_target, 0, n_target, n->conn_spec_, n->syn_spec_);
  });
}
int NeuronGPU_RemoteConnectSeqSeq(int i_source_host, int i_source, int n_source,
                                  int i_target_host, int i_target, int n_target) {
  return guarded(0, [&](NeuronGPU *n) {
    return n->RemoteConnect(i_source_host, nullptr, i_source, n_source, i_target_host, nullptr,
                            i_target, n_target, n->conn_spec_, n->syn_spec_);
  });
}
int NeuronGPU_RemoteConnectSeqGroup(int i_source_host, int i_source, int n_source,
                                    int i_target_host, int *i_target, int n_target) {
  return guarded(0, [&](NeuronGPU *n) {
    return n->RemoteConnect(i_source_host, nullptr, i_source, n_source, i_target_host, i_target,
                            0, n_target, n->conn_spec_, n->syn_spec_);
  });
}
int NeuronGPU_RemoteConnectGroupSeq(int i_source_host, int *i_source, int n_source,
                                    int i_target_host, int i_target, int n_target) {
  return guarded(0, [&](NeuronGPU *n) {
    return n->RemoteConnect(i_source_host, i_source, 0, n_source, i_target_host, nullptr,
                            i_target, n_target, n->conn_spec_, n->syn_spec_);
  });
}
int NeuronGPU_RemoteConnectGroupGroup(int i_source_host, int *i_source, int n_source,
                                      int i_target_host, int *i_target, int n_target) {
  return guarded(0, [&](NeuronGPU *n) {
    return n->RemoteConnect(i_source_host, i_source, 0, n_source, i_target_host, i_target, 0,
                            n_target, n->conn_spec_, n->syn_spec_);
  });
}
char **NeuronGPU_GetIntVarNames(int i) {
  return guarded((char **)nullptr, [&](NeuronGPU *n) { return names_to_c(n->GetIntVarNames(i)); });
}
char **NeuronGPU_GetScalVarNames(int i) {
  return guarded((char **)nullptr, [&](NeuronGPU *n) { return names_to_c(n->GetScalVarNames(i)); });
}
int NeuronGPU_GetNIntVar(int i) {
  return guarded(0, [&](NeuronGPU *n) { return (int)n->GetIntVarNames(i).size(); });
}
int NeuronGPU_GetNScalVar(int i) {
  return guarded(0, [&](NeuronGPU *n) { return (int)n->GetScalVarNames(i).size(); });
}
char **NeuronGPU_GetPortVarNames(int i) {
  return guarded((char **)nullptr, [&](NeuronGPU *n) { return names_to_c(n->GetPortVarNames(i)); });
}
int NeuronGPU_GetNPortVar(int i) {
  return guarded(0, [&](NeuronGPU *n) { return (int)n->GetPortVarNames(i).size(); });
}
char **NeuronGPU_GetScalParamNames(int i) {
  return guarded((char **)nullptr, [&](NeuronGPU *n) { return names_to_c(n->GetScalParamNames(i)); });
}
int NeuronGPU_GetNScalParam(int i) {
  return guarded(0, [&](NeuronGPU *n) { return (int)n->GetScalParamNames(i).size(); });
}
char **NeuronGPU_GetPortParamNames(int i) {
  return guarded((char **)nullptr, [&](NeuronGPU *n) { return names_to_c(n->GetPortParamNames(i)); });
}
int NeuronGPU_GetNGroupParam(int i) {
  return guarded(0, [&](NeuronGPU *n) { return (int)n->GetGroupParamNames(i).size(); });
}
char **NeuronGPU_GetGroupParamNames(int i) {
  return guarded((char **)nullptr, [&](NeuronGPU *n) { return names_to_c(n->GetGroupParamNames(i)); });
}
int NeuronGPU_GetNPortParam(int i) {
  return guarded(0, [&](NeuronGPU *n) { return (int)n->GetPortParamNames(i).size(); });
}
char **NeuronGPU_GetArrayParamNames(int i) {
  return guarded((char **)nullptr, [&](NeuronGPU *n) { return names_to_c(n->GetArrayParamNames(i)); });
}
int NeuronGPU_GetNArrayParam(int i) {
  return guarded(0, [&](NeuronGPU *n) { return (int)n->GetArrayParamNames(i).size(); });
}
char **NeuronGPU_GetArrayVarNames(int i) {
  return guarded((char **)nullptr, [&](NeuronGPU *n) { return names_to_c(n->GetArrayVarNames(i)); });
}
int NeuronGPU_GetNArrayVar(int i) {
  return guarded(0, [&](NeuronGPU *n) { return (int)n->GetArrayVarNames(i).size(); });
}
int *NeuronGPU_GetSeqSeqConnections(int i_source, int n_source, int i_target, int n_target,
                                    int syn_group, int *n_conn) {
  return guarded((int *)nullptr, [&](NeuronGPU *n) {
    return conn_ids_to_c(n->GetConnections(nullptr, i_source, n_source, nullptr, i_target,
                                           n_target, syn_group), n_conn);
  });
}
int *NeuronGPU_GetSeqGroupConnections(int i_source, int n_source, int *i_target, int n_target,
                                      int syn_group, int *n_conn) {
  return guarded((int *)nullptr, [&](NeuronGPU *n) {
    return conn_ids_to_c(n->GetConnections(nullptr, i_source, n_source, i_target, 0, n_target,
                                           syn_group), n_conn);
  });
}
int *NeuronGPU_GetGroupSeqConnections(int *i_source, int n_source, int i_target, int n_target,
                                      int syn_group, int *n_conn) {
  return guarded((int *)nullptr, [&](NeuronGPU *n) {
    return conn_ids_to_c(n->GetConnections(i_source, 0, n_source, nullptr, i_target, n_target,
                                           syn_group), n_conn);
  });
}
int *NeuronGPU_GetGroupGroupConnections(int *i_source, int n_source, int *i_target,
                                        int n_target, int syn_group, int *n_conn) {
  return guarded((int *)nullptr, [&](NeuronGPU *n) {
    return conn_ids_to_c(n->GetConnections(i_source, 0, n_source, i_target, 0, n_target,
                                           syn_group), n_conn);
  });
}
int NeuronGPU_GetConnectionStatus(int i_source, int i_group, int i_conn, int *i_target,
                                  unsigned char *port, unsigned char *syn_group, float *delay,
                                  float *weight) {
  return guarded(0, [&](NeuronGPU *n) {
    ConnectionId id;
    id.i_source_ = i_source; id.i_group_ = i_group; id.i_conn_ = i_conn;
    ConnectionStatus st = n->GetConnectionStatus(id);
    *i_target = st.i_target;
    *port = st.port;
    *syn_group = st.syn_group;
    *delay = st.delay;
    *weight = st.weight;
    return 0;
  });
}
int NeuronGPU_CreateSynGroup(char *model_name) {
  return guarded(0, [&](NeuronGPU *n) { return n->CreateSynGroup(model_name); });
}
int NeuronGPU_GetSynGroupNParam(int sg) {
  return guarded(0, [&](NeuronGPU *n) { return n->GetSynGroupNParam(sg); });
}
char **NeuronGPU_GetSynGroupParamNames(int sg) {
  return guarded((char **)nullptr, [&](NeuronGPU *n) { return names_to_c(n->GetSynGroupParamNames(sg)); });
}
int NeuronGPU_IsSynGroupParam(int sg, char *p) {
  return guarded(0, [&](NeuronGPU *n) { return n->IsSynGroupParam(sg, p) ? 1 : 0; });
}
int NeuronGPU_GetSynGroupParamIdx(int sg, char *p) {
  return guarded(0, [&](NeuronGPU *n) { return n->GetSynGroupParamIdx(sg, p); });
}
float NeuronGPU_GetSynGroupParam(int sg, char *p) {
  return guarded(0.0f, [&](NeuronGPU *n) { return n->GetSynGroupParam(sg, p); });
}
int NeuronGPU_SetSynGroupParam(int sg, char *p, float val) {
  return guarded(0, [&](NeuronGPU *n) { return n->SetSynGroupParam(sg, p, val); });
}
int NeuronGPU_ActivateSpikeCount(int i_node, int n_node) {
  return guarded(0, [&](NeuronGPU *n) { return n->ActivateSpikeCount(i_node, n_node); });
}
int NeuronGPU_ActivateRecSpikeTimes(int i_node, int n_node, int max_n) {
  return guarded(0, [&](NeuronGPU *n) { return n->ActivateRecSpikeTimes(i_node, n_node, max_n); });
}
int NeuronGPU_GetNRecSpikeTimes(int i_node) {
  return guarded(0, [&](NeuronGPU *n) { return n->GetNRecSpikeTimes(i_node); });
}
float *NeuronGPU_GetRecSpikeTimes(int i_node) {
  return guarded((float *)nullptr, [&](NeuronGPU *n) {
    std::vector<float> v = n->GetRecSpikeTimes(i_node);
    float *a = (float *)malloc(sizeof(float) * (v.size() > 0 ? v.size() : 1));
    for (size_t i = 0; i < v.size(); i++) a[i] = v[i];
    return a;
  });
}
int NeuronGPU_PushSpikesToNodes(int n_spikes, int *node_id) {
  return guarded(0, [&](NeuronGPU *n) { return n->PushSpikesToNodes(n_spikes, node_id); });
}
int NeuronGPU_GetExtNeuronInputSpikes(int *, int **, int **, float **, int) {
  return guarded(0, [&](NeuronGPU *) -> int {
    throw ngpu::ngpu_exception("ext_neuron co-simulation is not available in this build");
  });
}
int NeuronGPU_SetNeuronGroupParam(int i_node, int n_node, char *p, float val) {
  return guarded(0, [&](NeuronGPU *n) { return n->SetNeuronGroupParam(i_node, n_node, p, val); });
}
int NeuronGPU_IsNeuronGroupParam(int i_node, char *p) {
  return guarded(0, [&](NeuronGPU *n) { return n->IsNeuronGroupParam(i_node, p); });
}
float NeuronGPU_GetNeuronGroupParam(int i_node, char *p) {
  return guarded(0.0f, [&](NeuronGPU *n) { return n->GetNeuronGroupParam(i_node, p); });
}
int NeuronGPU_GetNFloatParam() {
  return guarded(0, [&](NeuronGPU *n) { return (int)n->GetFloatParamNames().size(); });
}
char **NeuronGPU_GetFloatParamNames() {
  return guarded((char **)nullptr, [&](NeuronGPU *n) { return names_to_c(n->GetFloatParamNames()); });
}
int NeuronGPU_IsFloatParam(char *p) {
  return guarded(0, [&](NeuronGPU *n) { return n->IsFloatParam(p) ? 1 : 0; });
}
int NeuronGPU_GetFloatParamIdx(char *p) {
  return guarded(0, [&](NeuronGPU *n) { return n->GetFloatParamIdx(p); });
}
float NeuronGPU_GetFloatParam(char *p) {
  return guarded(0.0f, [&](NeuronGPU *n) { return n->GetFloatParam(p); });
}
int NeuronGPU_SetFloatParam(char *p, float val) {
  return guarded(0, [&](NeuronGPU *n) { return n->SetFloatParam(p, val); });
}
int NeuronGPU_GetNIntParam() {
  return guarded(0, [&](NeuronGPU *n) { return (int)n->GetIntParamNames().size(); });
}
char **NeuronGPU_GetIntParamNames() {
  return guarded((char **)nullptr, [&](NeuronGPU *n) { return names_to_c(n->GetIntParamNames()); });
}
int NeuronGPU_IsIntParam(char *p) {
  return guarded(0, [&](NeuronGPU *n) { return n->IsIntParam(p) ? 1 : 0; });
}
int NeuronGPU_GetIntParamIdx(char *p) {
  return guarded(0, [&](NeuronGPU *n) { return n->GetIntParamIdx(p); });
}
int NeuronGPU_GetIntParam(char *p) {
  return guarded(0, [&](NeuronGPU *n) { return n->GetIntParam(p); });
}
int NeuronGPU_SetIntParam(char *p, int val) {
  return guarded(0, [&](NeuronGPU *n) { return n->SetIntParam(p, val); });
}
int NeuronGPU_RemoteCreate(int i_host, char *model_name, int n_neuron, int n_port) {
  return guarded(0, [&](NeuronGPU *n) {
    return n->RemoteCreate(i_host, std::string(model_name), n_neuron, n_port);
  });
}

// ---- extensions ----
int NGB200_Reset() {
  return guarded(0, [&](NeuronGPU *n) {
    int on_exc = n->OnException();
    delete g_inst[g_cur];
    g_inst[g_cur] = new NeuronGPU();
    g_inst[g_cur]->SetOnException(on_exc);
    return 0;
  });
}
int NGB200_SetInstance(int k) {
  if (k < 0 || k >= kMaxInstances) return -1;
  g_cur = k;
  inst();
  return 0;
}
int NGB200_GetInstance() { return g_cur; }
int NGB200_SetHost(int id, int n_hosts) {
  return guarded(0, [&](NeuronGPU *n) { return n->SetHost(id, n_hosts); });
}
int NGB200_SimulateSteps(long long n_steps) {
  return guarded(0, [&](NeuronGPU *n) { return n->SimulateSteps(n_steps); });
}
int NGB200_RemoteExchangeSteps() {
  return guarded(0, [&](NeuronGPU *n) { return n->RemoteExchangeSteps(); });
}
long long NGB200_PackRemoteSpikes(int n_steps, void *buf, long long cap) {
  return guarded(-1LL, [&](NeuronGPU *n) {
    return n->PackRemoteSpikes(n_steps, (unsigned *)buf, cap);
  });
}
int NGB200_UnpackRemoteSpikes(int src_host, int n_steps, const void *buf, long long count) {
  return guarded(0, [&](NeuronGPU *n) {
    return n->UnpackRemoteSpikes(src_host, n_steps, (const unsigned *)buf, count);
  });
}
unsigned long long NGB200_StageEvaluations() {
  return guarded(0ULL, [&](NeuronGPU *n) { return n->StageEvaluations(); });
}
unsigned long long NGB200_DeliveredEvents() {
  return guarded(0ULL, [&](NeuronGPU *n) { return n->DeliveredEvents(); });
}
unsigned long long NGB200_TotalSpikes() {
  return guarded(0ULL, [&](NeuronGPU *n) { return n->TotalSpikes(); });
}
double NGB200_LastSimulateSeconds() {
  return guarded(0.0, [&](NeuronGPU *n) { return n->LastSimulateSeconds(); });
}
int NGB200_SetGraphChunk(int n_steps) {
  return guarded(0, [&](NeuronGPU *n) {
    if (n_steps <= 0) { n->UseGraphs(0); return 0; }
    n->UseGraphs(1);
    return n->SetGraphChunk(n_steps);
  });
}
long long NGB200_NNodes() {
  return guarded(0LL, [&](NeuronGPU *n) { return n->NNodes(); });
}
long long NGB200_NConnections() {
  return guarded(0LL, [&](NeuronGPU *n) { return n->NConnections(); });
}
int NGB200_SetRk5Batching(int on) {
  return guarded(0, [&](NeuronGPU *n) { return n->SetRk5Batching(on); });
}
int NGB200_Rk5BatchOf(int i_node) {
  return guarded(-1, [&](NeuronGPU *n) { return n->Rk5BatchOf(i_node); });
}
int NGB200_SetStepLog(int i_node, int capacity) {
  return guarded(0, [&](NeuronGPU *n) { return n->SetStepLog(i_node, capacity); });
}
long long NGB200_GetStepLogCount(int i_node) {
  return guarded(0LL, [&](NeuronGPU *n) { return n->GetStepLogCount(i_node); });
}
int NGB200_GetStepLog(int i_node, float *out, int max_rows) {
  return guarded(0, [&](NeuronGPU *n) { return n->GetStepLog(i_node, out, max_rows); });
}
int NGB200_TrainStepProposer(int steps, int blocks, float lr, unsigned long long seed,
                             float *loss_first, float *loss_last) {
  return guarded(0, [&](NeuronGPU *n) {
    return n->TrainStepProposer(steps, blocks, lr, seed, loss_first, loss_last);
  });
}
int NGB200_SetStepProposer(int i_node, int on) {
  return guarded(0, [&](NeuronGPU *n) { return n->SetStepProposer(i_node, on); });
}
int NGB200_SetStepProposerParams(const float *params) {
  return guarded(0, [&](NeuronGPU *n) { return n->SetStepProposerParams(params); });
}
int NGB200_GetStepProposerParams(float *params) {
  return guarded(0, [&](NeuronGPU *n) { return n->GetStepProposerParams(params); });
}
int NGB200_SetStepProposerMargin(float margin) {
  return guarded(0, [&](NeuronGPU *n) { return n->SetStepProposerMargin(margin); });
}
float NGB200_MlpGradients(const float *data, int n_samples, const float *params, float *grad) {
  return guarded(0.0f, [&](NeuronGPU *n) {
    return n->MlpGradientsHost(data, n_samples, params, grad);
  });
}
int NGB200_MlpInfer(const float *x6, int n_rows, const float *params, float *out) {
  return guarded(0, [&](NeuronGPU *n) { return n->MlpInferHost(x6, n_rows, params, out); });
}
long long NGB200_GetAllConnections(int *src, int *tgt, int *port, int *syn,
                                   float *delay, float *weight) {
  return guarded(0LL, [&](NeuronGPU *n) {
    return n->ExportConnections(src, tgt, port, syn, delay, weight);
  });
}
void NGB200_FreeArray(void *p) { free(p); }
double NGB200_KernelsPerStep() {
  return guarded(0.0, [&](NeuronGPU *n) { return n->KernelsPerStep(); });
}
double NGB200_LastSimulateDeviceMs() {
  return guarded(0.0, [&](NeuronGPU *n) { return n->LastSimulateDeviceMs(); });
}
int NGB200_SetKernelTiming(int on) {
  return guarded(0, [&](NeuronGPU *n) { return n->SetKernelTiming(on); });
}
int NGB200_GetKernelTiming(int kind, double *total_ms, long long *launches) {
  return guarded(0, [&](NeuronGPU *n) { return n->GetKernelTiming(kind, total_ms, launches); });
}
int NGB200_SetRk5MaxSubsteps(int n_substeps) {
  return guarded(0, [&](NeuronGPU *n) { return n->SetRk5MaxSubsteps(n_substeps); });
}
int NGB200_SetWaitTest(int mask) {
  return guarded(0, [&](NeuronGPU *n) { return n->SetWaitTest(mask); });
}
unsigned NGB200_ProposerPhaseAfter(unsigned phase_in, int ok1, int ok2) {
  return ngpu::proposer_phase_after(phase_in, ok1 != 0, ok2 != 0);
}

}  // extern "C"

extern "C" int NGB200_GetRk5Tuning(int i_node, int *variant, float *ms) {
  return guarded(0, [&](NeuronGPU *n) { return n->GetRk5Tuning(i_node, variant, ms); });
}
