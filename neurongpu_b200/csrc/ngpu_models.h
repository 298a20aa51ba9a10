// Neuron model catalogue: names, defaults and input mapping (host side) and
// the per-neuron right-hand sides used by the RK5 kernels (device side).
//
// The variable/parameter names, their order and their defaults follow the
// reference models so that scripts that address them by name keep working:
//   aeif_cond_beta     src/aeif_cond_beta_kernel.h:30-100, src/aeif_cond_beta.cu:25-87
//                      (also user_m1, user_m2: src/user_m1_kernel.h, src/user_m2_kernel.h)
//   aeif_cond_alpha    src/aeif_cond_alpha_kernel.h, src/aeif_cond_alpha.cu:25-70
//   aeif_psc_alpha     src/aeif_psc_alpha_kernel.h, src/aeif_psc_alpha.cu:25-70
//   aeif_psc_exp       src/aeif_psc_exp_kernel.h, src/aeif_psc_exp.cu:25-60
//   aeif_psc_delta     src/aeif_psc_delta_kernel.h, src/aeif_psc_delta.cu:25-60
//   izhikevich_cond_beta src/izhikevich_cond_beta_kernel.h, src/izhikevich_cond_beta.cu
//   iaf_psc_exp        src/iaf_psc_exp.h:20-90, src/iaf_psc_exp.cu:53-180
//   iaf_psc_exp_g      src/iaf_psc_exp_g.h:30-75, src/iaf_psc_exp_g.cu:39-149
//   iaf_psc_exp_hc     src/iaf_psc_exp_hc.h:30-50, src/iaf_psc_exp_hc.cu:33-107,
//                      src/iaf_psc_exp_hc_params.h (iaf_psc_exp_g's defaults at dt 0.1)
//   izhikevich         src/izhikevich.h:30-72, src/izhikevich.cu:38-136
//   izhikevich_psc_exp(_2s, _5s) src/izhikevich_psc_exp.h:30-76,
//                      src/izhikevich_psc_exp.cu:40-148, src/izhikevich_psc_exp_2s.cu:41-155
//   spike_generator    src/spike_generator.cu:24-60
//   parrot_neuron      src/parrot_neuron.cu:20-112
//   spike_detector     src/spike_detector.cu:20-106
//   poisson_generator  src/poiss_gen.cu:76-90, src/poiss_gen_variables.h
// The state itself is stored structure-of-arrays (one column per variable or
// parameter) rather than the reference's per-neuron array of structures.
#pragma once
#include <string>
#include <vector>
#include <math.h>

namespace ngpu {

enum ModelKind {
  MK_RK5 = 0,
  MK_IAF_PSC_EXP,
  MK_SPIKE_GENERATOR,
  MK_PARROT,
  MK_SPIKE_DETECTOR,
  MK_POISSON_GENERATOR,   // device Poisson source, delivered by direct connections
  MK_POISSON_NODES,       // CreatePoissonGenerator: nodes that push spike counts
  MK_IAF_PSC_EXP_G,       // iaf_psc_exp_g / iaf_psc_exp_hc: one port, group parameters
  MK_IZHIKEVICH,          // Euler Izhikevich, input added to V_m
  MK_IZH_PSC_EXP,         // Euler Izhikevich with an exponential current, n_sub Euler steps
  MK_IMAGE                // image of a node of another host (remote connections): no
                          // dynamics, its spikes are the remote node's, received by
                          // the host's spike exchange
};

enum Rk5Model {
  RK5_AEIF_COND_BETA = 0,
  RK5_AEIF_COND_ALPHA,
  RK5_AEIF_PSC_ALPHA,
  RK5_AEIF_PSC_EXP,
  RK5_AEIF_PSC_DELTA,
  RK5_IZHIKEVICH_COND_BETA,
  N_RK5_MODELS
};

struct ModelInfo {
  std::string name;
  ModelKind kind;
  int rk5_model;                // Rk5Model for MK_RK5, else -1
  int fixed_n_port;             // -1: user chooses
  std::vector<std::string> scal_var, port_var, scal_param, port_param;
  std::vector<std::string> group_param, array_param;
  std::vector<float> scal_var_def, port_var_def, scal_param_def,
      port_param_def, group_param_def;
  // input folding: port p adds (acc * weight(p)) into var in_var + p*in_step
  int in_var;                   // var index (scalar layout) of port-0 input
  int in_step;                  // var index stride between ports
  bool w_param;                 // weight taken from a per-port parameter
  int w_param_idx;              // port-param index of the weight
  std::vector<float> w_const;   // constant weight per port (w_param false)
  int refr_param;               // param index of refractory_step (-1: none)
  int den_delay_param;          // param index of den_delay (-1: none)
  int n_sub = 1;                // Euler sub-steps per time step (MK_IZH_PSC_EXP)
  int hard_coded = 0;           // iaf_psc_exp_hc: constants of iaf_psc_exp_g's defaults
};

inline const std::vector<ModelInfo> &ModelCatalogue() {
  static std::vector<ModelInfo> cat;
  if (!cat.empty()) return cat;
  const std::vector<std::string> aeif_sp = {
      "V_th", "Delta_T", "g_L", "E_L", "C_m", "a", "b", "tau_w", "I_e",
      "V_peak", "V_reset", "t_ref", "refractory_step", "den_delay"};
  const std::vector<float> aeif_sp_def = {
      -50.4f, 2.0f, 30.0f, -70.6f, 281.0f, 4.0f, 80.5f, 144.0f, 0.0f,
      0.0f, -60.0f, 0.0f, 0.0f, 0.0f};
  const std::vector<std::string> rk5_gp = {"h_min_rel", "h0_rel"};
  const std::vector<float> rk5_gp_def = {1.0e-3f, 1.0e-2f};
  {
    ModelInfo m;
    m.name = "aeif_cond_beta"; m.kind = MK_RK5; m.rk5_model = RK5_AEIF_COND_BETA;
    m.fixed_n_port = -1;
    m.scal_var = {"V_m", "w"}; m.scal_var_def = {-70.6f, 0.0f};
    m.port_var = {"g", "g1"}; m.port_var_def = {0.0f, 0.0f};
    m.scal_param = aeif_sp; m.scal_param_def = aeif_sp_def;
    m.port_param = {"E_rev", "tau_rise", "tau_decay", "g0"};
    m.port_param_def = {0.0f, 2.0f, 20.0f, 0.0f};
    m.group_param = rk5_gp; m.group_param_def = rk5_gp_def;
    m.in_var = 2 + 1; m.in_step = 2; m.w_param = true; m.w_param_idx = 3;
    m.refr_param = 12; m.den_delay_param = 13;
    cat.push_back(m);
    // user_m1 / user_m2: the reference ships these user-model templates as
    // renamed copies of aeif_cond_beta (src/user_m1_kernel.h,
    // src/user_m2_kernel.h and their .cu files differ from
    // src/aeif_cond_beta_kernel.h / .cu only in the names)
    for (const char *alias : {"user_m1", "user_m2"}) {
      ModelInfo u = m;
      u.name = alias;
      cat.push_back(u);
    }
  }
  {
    ModelInfo m;
    m.name = "aeif_cond_alpha"; m.kind = MK_RK5; m.rk5_model = RK5_AEIF_COND_ALPHA;
    m.fixed_n_port = -1;
    m.scal_var = {"V_m", "w"}; m.scal_var_def = {-70.6f, 0.0f};
    m.port_var = {"g", "g1"}; m.port_var_def = {0.0f, 0.0f};
    m.scal_param = aeif_sp; m.scal_param_def = aeif_sp_def;
    m.port_param = {"E_rev", "tau_syn", "g0"};
    m.port_param_def = {0.0f, 2.0f, 0.0f};
    m.group_param = rk5_gp; m.group_param_def = rk5_gp_def;
    m.in_var = 2 + 1; m.in_step = 2; m.w_param = true; m.w_param_idx = 2;
    m.refr_param = 12; m.den_delay_param = 13;
    cat.push_back(m);
  }
  {
    ModelInfo m;
    m.name = "aeif_psc_alpha"; m.kind = MK_RK5; m.rk5_model = RK5_AEIF_PSC_ALPHA;
    m.fixed_n_port = -1;
    m.scal_var = {"V_m", "w"}; m.scal_var_def = {-70.6f, 0.0f};
    m.port_var = {"I_syn", "I1_syn"}; m.port_var_def = {0.0f, 0.0f};
    m.scal_param = aeif_sp; m.scal_param_def = aeif_sp_def;
    m.port_param = {"tau_syn", "I0"};
    m.port_param_def = {0.2f, 0.0f};
    m.group_param = rk5_gp; m.group_param_def = rk5_gp_def;
    m.in_var = 2 + 1; m.in_step = 2; m.w_param = true; m.w_param_idx = 1;
    m.refr_param = 12; m.den_delay_param = 13;
    cat.push_back(m);
  }
  {
    ModelInfo m;
    m.name = "aeif_psc_exp"; m.kind = MK_RK5; m.rk5_model = RK5_AEIF_PSC_EXP;
    m.fixed_n_port = -1;
    m.scal_var = {"V_m", "w"}; m.scal_var_def = {-70.6f, 0.0f};
    m.port_var = {"I_syn"}; m.port_var_def = {0.0f};
    m.scal_param = aeif_sp; m.scal_param_def = aeif_sp_def;
    m.port_param = {"tau_syn"};
    m.port_param_def = {0.2f};
    m.group_param = rk5_gp; m.group_param_def = rk5_gp_def;
    m.in_var = 2; m.in_step = 1; m.w_param = false; m.w_param_idx = -1;
    m.refr_param = 12; m.den_delay_param = 13;
    cat.push_back(m);
  }
  {
    ModelInfo m;
    m.name = "aeif_psc_delta"; m.kind = MK_RK5; m.rk5_model = RK5_AEIF_PSC_DELTA;
    m.fixed_n_port = 1;
    m.scal_var = {"V_m", "w"}; m.scal_var_def = {-70.6f, 0.0f};
    m.scal_param = aeif_sp; m.scal_param_def = aeif_sp_def;
    m.group_param = rk5_gp; m.group_param_def = rk5_gp_def;
    // every port adds directly into V_m (src/aeif_psc_delta.cu:118-120)
    m.in_var = 0; m.in_step = 0; m.w_param = false; m.w_param_idx = -1;
    m.refr_param = 12; m.den_delay_param = 13;
    cat.push_back(m);
  }
  {
    ModelInfo m;
    m.name = "izhikevich_cond_beta"; m.kind = MK_RK5;
    m.rk5_model = RK5_IZHIKEVICH_COND_BETA; m.fixed_n_port = -1;
    m.scal_var = {"V_m", "u"}; m.scal_var_def = {-70.0f, -14.0f};
    m.port_var = {"g", "g1"}; m.port_var_def = {0.0f, 0.0f};
    m.scal_param = {"V_th", "a", "b", "c", "d", "I_e", "t_ref",
                    "refractory_step", "den_delay"};
    m.scal_param_def = {30.0f, 0.02f, 0.2f, -65.0f, 8.0f, 0.0f, 0.0f, 0.0f,
                        0.0f};
    m.port_param = {"E_rev", "tau_rise", "tau_decay", "g0"};
    m.port_param_def = {0.0f, 2.0f, 20.0f, 0.0f};
    m.group_param = rk5_gp; m.group_param_def = rk5_gp_def;
    m.in_var = 2 + 1; m.in_step = 2; m.w_param = true; m.w_param_idx = 3;
    m.refr_param = 7; m.den_delay_param = 8;
    cat.push_back(m);
  }
  {
    ModelInfo m;
    m.name = "iaf_psc_exp"; m.kind = MK_IAF_PSC_EXP; m.rk5_model = -1;
    m.fixed_n_port = 2;
    m.scal_var = {"I_syn_ex", "I_syn_in", "V_m_rel", "refractory_step"};
    m.scal_var_def = {0.0f, 0.0f, 0.0f, 0.0f};
    m.scal_param = {"tau_m", "C_m", "E_L", "I_e", "Theta_rel", "V_reset_rel",
                    "tau_ex", "tau_in", "t_ref", "den_delay", "P20", "P11ex",
                    "P11in", "P21ex", "P21in", "P22"};
    m.scal_param_def = {10.0f, 250.0f, -70.0f, 0.0f, 15.0f, 0.0f, 2.0f, 2.0f,
                        2.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
    m.in_var = 0; m.in_step = 1; m.w_param = false; m.w_param_idx = -1;
    m.w_const = {1.0f, 1.0f};
    m.refr_param = -1; m.den_delay_param = 9;
    cat.push_back(m);
  }
  {
    // refractory_step is a state variable here; one input port into I_syn
    for (int hc = 0; hc < 2; hc++) {
      ModelInfo m;
      m.name = hc ? "iaf_psc_exp_hc" : "iaf_psc_exp_g";
      m.kind = MK_IAF_PSC_EXP_G; m.rk5_model = -1; m.fixed_n_port = 1;
      m.scal_var = {"I_syn", "V_m_rel", "refractory_step"};
      m.scal_var_def = {0.0f, 0.0f, 0.0f};
      m.scal_param = {"I_e"}; m.scal_param_def = {0.0f};
      if (!hc) {
        m.group_param = {"tau_m", "C_m", "E_L", "Theta_rel", "V_reset_rel", "tau_syn", "t_ref"};
        m.group_param_def = {10.0f, 250.0f, -65.0f, 15.0f, 0.0f, 0.5f, 2.0f};
      }
      m.hard_coded = hc;
      m.in_var = 0; m.in_step = 0; m.w_param = false; m.w_param_idx = -1;
      m.w_const = {1.0f};
      m.refr_param = -1; m.den_delay_param = -1;
      cat.push_back(m);
    }
  }
  {
    ModelInfo m;
    m.name = "izhikevich"; m.kind = MK_IZHIKEVICH; m.rk5_model = -1; m.fixed_n_port = 1;
    m.scal_var = {"I_syn", "V_m", "u", "refractory_step"};
    m.scal_var_def = {0.0f, -70.0f, -70.0f * 0.2f, 0.0f};
    m.scal_param = {"I_e", "den_delay"}; m.scal_param_def = {0.0f, 0.0f};
    m.group_param = {"V_th", "a", "b", "c", "d", "t_ref"};
    m.group_param_def = {30.0f, 0.02f, 0.2f, -65.0f, 8.0f, 0.0f};
    m.in_var = 0; m.in_step = 0; m.w_param = false; m.w_param_idx = -1;
    m.w_const = {1.0f};
    m.refr_param = -1; m.den_delay_param = 1;
    cat.push_back(m);
  }
  {
    const char *names[3] = {"izhikevich_psc_exp", "izhikevich_psc_exp_2s", "izhikevich_psc_exp_5s"};
    const int subs[3] = {1, 2, 5};
    const float tau[3] = {0.5f, 2.0f, 2.0f};
    for (int k = 0; k < 3; k++) {
      ModelInfo m;
      m.name = names[k]; m.kind = MK_IZH_PSC_EXP; m.rk5_model = -1; m.fixed_n_port = 1;
      m.scal_var = {"I_syn", "V_m", "u", "refractory_step"};
      m.scal_var_def = {0.0f, -70.0f, -70.0f * 0.2f, 0.0f};
      m.scal_param = {"I_e", "den_delay"}; m.scal_param_def = {0.0f, 0.0f};
      m.group_param = {"V_th", "a", "b", "c", "d", "tau_syn", "t_ref"};
      m.group_param_def = {30.0f, 0.02f, 0.2f, -65.0f, 8.0f, tau[k], 0.0f};
      m.n_sub = subs[k];
      m.in_var = 0; m.in_step = 0; m.w_param = false; m.w_param_idx = -1;
      m.w_const = {1.0f};
      m.refr_param = -1; m.den_delay_param = 1;
      cat.push_back(m);
    }
  }
  {
    ModelInfo m;
    m.name = "spike_generator"; m.kind = MK_SPIKE_GENERATOR; m.rk5_model = -1;
    m.fixed_n_port = 0;
    m.array_param = {"spike_times", "spike_heights"};
    m.in_var = -1; m.in_step = 0; m.w_param = false; m.w_param_idx = -1;
    m.refr_param = -1; m.den_delay_param = -1;
    cat.push_back(m);
  }
  {
    ModelInfo m;
    m.name = "parrot_neuron"; m.kind = MK_PARROT; m.rk5_model = -1;
    m.fixed_n_port = 2;
    m.scal_var = {"input_spike_height", "dummy_input", "V"};
    m.scal_var_def = {0.0f, 0.0f, 0.0f};
    m.scal_param = {"hold_spike_height", "den_delay"};
    m.scal_param_def = {0.0f, 0.0f};
    // port 0 drives input_spike_height, port 1 the ignored dummy_input
    m.in_var = 0; m.in_step = 1; m.w_param = false; m.w_param_idx = -1;
    m.w_const = {1.0f, 0.0f};
    m.refr_param = -1; m.den_delay_param = 1;
    cat.push_back(m);
  }
  {
    ModelInfo m;
    m.name = "spike_detector"; m.kind = MK_SPIKE_DETECTOR; m.rk5_model = -1;
    m.fixed_n_port = 1;
    m.scal_var = {"input_spike_height", "spike_height"};
    m.scal_var_def = {0.0f, 0.0f};
    m.scal_param = {"hold_spike_height"};
    m.scal_param_def = {1.0f};
    m.in_var = 0; m.in_step = 0; m.w_param = false; m.w_param_idx = -1;
    m.w_const = {1.0f};
    m.refr_param = -1; m.den_delay_param = -1;
    cat.push_back(m);
  }
  {
    ModelInfo m;
    m.name = "poisson_generator"; m.kind = MK_POISSON_GENERATOR;
    m.rk5_model = -1; m.fixed_n_port = 0;
    m.scal_param = {"rate", "origin", "start", "stop"};
    m.scal_param_def = {0.0f, 0.0f, 0.0f, 1.0e30f};
    m.in_var = -1; m.in_step = 0; m.w_param = false; m.w_param_idx = -1;
    m.refr_param = -1; m.den_delay_param = -1;
    cat.push_back(m);
  }
  {
    // the reference's remote nodes (src/neurongpu.cu:1626-1642, a base
    // neuron group created at calibration): created by RemoteConnect on the
    // target host, one per remote source node
    ModelInfo m;
    m.name = "remote_image"; m.kind = MK_IMAGE;
    m.rk5_model = -1; m.fixed_n_port = 0;
    m.in_var = -1; m.in_step = 0; m.w_param = false; m.w_param_idx = -1;
    m.refr_param = -1; m.den_delay_param = -1;
    cat.push_back(m);
  }
  return cat;
}

inline int FindModel(const std::string &name) {
  const std::vector<ModelInfo> &cat = ModelCatalogue();
  for (size_t i = 0; i < cat.size(); i++) {
    if (cat[i].name == name) return (int)i;
  }
  return -1;
}

}  // namespace ngpu
