// FP64 CPU oracle of the per-time-step simulation core -- TEST
// INFRASTRUCTURE ONLY. It is used by tests/, by __graft_entry__.smoke() and by
// the cpu_baseline leg of bench.py as the checker; the product (libneurongpu)
// never links or calls it.
//
// It restates the reference algorithm (golosio/NeuronGPU) in double
// precision, one neuron at a time, with no GPU:
//   RK5 Cash-Karp step and adaptive controller   src/rk5.h:57-162, src/rk5.cu:23-60
//   AdEx conductance / current models            src/aeif_cond_beta_kernel.h:153-214,
//                                                src/aeif_cond_alpha_kernel.h,
//                                                src/aeif_psc_{alpha,exp,delta}_kernel.h
//   Izhikevich with beta conductances            src/izhikevich_cond_beta_kernel.h
//   conductance normalisation g0 / I0            src/aeif_cond_beta.cu:58-87,
//                                                src/aeif_cond_alpha.cu:63-68
//   iaf_psc_exp exact propagators                src/iaf_psc_exp.cu:53-119
//   iaf_psc_exp_g / _hc (one current, group params) src/iaf_psc_exp_g.cu:39-88,143-150
//   izhikevich (Euler, input added to V_m)        src/izhikevich.cu:38-72
//   izhikevich_psc_exp, _2s, _5s (Euler sub-steps) src/izhikevich_psc_exp_2s.cu:41-83
//   delay handling d_int = round(d/dt)-1 and the
//   buffer timing (spike of step k reaches the
//   input after step k+D)                         src/connect.cu:26-62,
//                                                src/spike_buffer.cu:143-302
//   input accumulation in double, folded after
//   the update (g1 += acc * g0)                  src/get_spike.cu:48-140
//   Poisson direct connections                   src/poiss_gen.cu:43-74,
//                                                src/neurongpu.cu:1156-1192
//   STDP pre and post rules                      src/stdp.cu:24-51, src/get_spike.cu:73-83,
//                                                src/rev_spike.cu:41-75
// Poisson counts use the same counter-based generator and inversion sampler
// as the CUDA core (neurongpu_b200/csrc/ngpu_rng.h), so the integer counts are
// identical for rate*dt < 10; everything else is independent code.
//
// Build: python oracle/build_oracle.py  ->  oracle/lib/libngpu_oracle.so
#include <math.h>
#include <stdint.h>
#include <string.h>
#include <algorithm>
#include <map>
#include <utility>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../neurongpu_b200/csrc/ngpu_rng.h"

#define NGPU_MAX_SYN_DT_ORACLE 16384   // STDP window in steps

namespace {

enum OModel {
  O_AEIF_COND_BETA = 0, O_AEIF_COND_ALPHA, O_AEIF_PSC_ALPHA, O_AEIF_PSC_EXP,
  O_AEIF_PSC_DELTA, O_IZH_COND_BETA, O_IAF_PSC_EXP, O_SPIKE_GENERATOR,
  O_PARROT, O_POISSON_GENERATOR, O_IAF_PSC_EXP_G, O_IZHIKEVICH, O_IZH_PSC_EXP
};
// simple (non-RK5, non-generator) neuron models updated in the parallel loop
static inline bool simple_model(int m) {
  return m == O_IAF_PSC_EXP || m == O_IAF_PSC_EXP_G || m == O_IZHIKEVICH || m == O_IZH_PSC_EXP;
}

typedef double real;

struct Group {
  int model, n, np, nvar, nparam, i0;
  std::vector<real> var, param;     // [i*nvar + j], [i*nparam + j]
  std::vector<real> h, x;
  real h_min_rel, h0_rel, eps;
  // spike generator
  std::vector<int> sg_off, sg_step, sg_next;
  std::vector<real> sg_height;
  long long evals = 0;
  bool step_search = false;     // exact step search instead of the controller (bound)
};

struct Edge {
  int src, tgt, port, syn, d;   // d = delay in steps (>= 1)
  real w;
  long long order;              // insertion index
  int stamp;                    // last pre-spike arrival step (plastic)
};

struct Oracle {
  real dt;
  uint64_t seed;
  std::vector<Group> groups;
  std::vector<int> node_group;
  std::vector<Edge> edges;        // sorted by (src, d, order) after prepare
  std::vector<size_t> out_off;    // per source
  std::vector<std::vector<size_t>> in_plastic;  // per target: edge idx
  struct SynG { int type; real p[8]; };
  std::vector<SynG> syn;
  // Poisson direct connections: per target list
  struct DC { int gen_node, port; real w, delay; uint64_t stream; };
  std::vector<std::vector<DC>> dc_of;
  std::vector<real> gen_rate, gen_origin, gen_start, gen_stop;  // per node
  // direct-connection sampler thresholds per generator node and the rate
  // per step they were formed for
  std::vector<std::vector<uint32_t>> gen_thr;
  // explicit random streams of the direct connections, in their (source,
  // delay, insertion) order; empty: the order index (test hook: a sample of
  // a larger network keeps that network's streams)
  std::vector<uint64_t> dc_stream_set;
  std::vector<double> gen_thr_lam;
  std::vector<real> acc;          // [node*maxport + port]
  int maxport = 1;
  std::vector<std::vector<std::pair<int, real>>> spikes_at;  // per step: (node, height)
  std::vector<long long> last_rev;    // per node: step its last spike reached the dendrites
  std::map<long long, std::vector<int>> rev_at;  // step -> nodes whose spike reaches them then
  long long T = 0;                    // time index of the last finished step
  bool prepared = false;
  // records
  std::vector<int> rec_node, rec_col;
  // spike log
  std::vector<long long> log_step;
  std::vector<int> log_node;
};

// --------------------------------------------------------------------------
// model right-hand sides (double)
// --------------------------------------------------------------------------
enum { A_V_th = 0, A_Delta_T, A_g_L, A_E_L, A_C_m, A_a, A_b, A_tau_w, A_I_e,
       A_V_peak, A_V_reset, A_t_ref, A_refr, A_den_delay, A_NSP };
enum { I_V_th = 0, I_a, I_b, I_c, I_d, I_I_e, I_t_ref, I_refr, I_den_delay, I_NSP };

static void deriv(int model, int np, const real *y, real *dy, const real *p) {
  if (model == O_IZH_COND_BETA) {
    real refr = p[I_refr];
    real V = refr > 0 ? p[I_c] : y[0];
    real I_syn = 0;
    for (int i = 0; i < np; i++) I_syn += y[2 + 2 * i] * (p[I_NSP + 4 * i] - V);
    dy[0] = refr > 0 ? 0 : 0.04 * V * V + 5.0 * V + 140.0 - y[1] + I_syn + p[I_I_e];
    dy[1] = p[I_a] * (p[I_b] * V - y[1]);
    for (int i = 0; i < np; i++) {
      dy[2 + 2 * i + 1] = -y[2 + 2 * i + 1] / p[I_NSP + 4 * i + 1];
      dy[2 + 2 * i] = y[2 + 2 * i + 1] - y[2 + 2 * i] / p[I_NSP + 4 * i + 2];
    }
    return;
  }
  real refr = p[A_refr];
  real V = refr > 0 ? p[A_V_reset] : std::min(y[0], (real)p[A_V_peak]);
  real I = 0;
  switch (model) {
    case O_AEIF_COND_BETA:
      for (int i = 0; i < np; i++) I += y[2 + 2 * i] * (p[A_NSP + 4 * i] - V);
      break;
    case O_AEIF_COND_ALPHA:
      for (int i = 0; i < np; i++) I += y[2 + 2 * i] * (p[A_NSP + 3 * i] - V);
      break;
    case O_AEIF_PSC_ALPHA:
      for (int i = 0; i < np; i++) I += y[2 + 2 * i];
      break;
    case O_AEIF_PSC_EXP:
      for (int i = 0; i < np; i++) I += y[2 + i];
      break;
    default:
      break;
  }
  real V_spike = p[A_Delta_T] == 0 ? 0 : p[A_Delta_T] * exp((V - p[A_V_th]) / p[A_Delta_T]);
  dy[0] = refr > 0 ? 0 : (-p[A_g_L] * (V - p[A_E_L] - V_spike) + I - y[1] + p[A_I_e]) / p[A_C_m];
  dy[1] = (p[A_a] * (V - p[A_E_L]) - y[1]) / p[A_tau_w];
  switch (model) {
    case O_AEIF_COND_BETA:
      for (int i = 0; i < np; i++) {
        dy[2 + 2 * i + 1] = -y[2 + 2 * i + 1] / p[A_NSP + 4 * i + 1];
        dy[2 + 2 * i] = y[2 + 2 * i + 1] - y[2 + 2 * i] / p[A_NSP + 4 * i + 2];
      }
      break;
    case O_AEIF_COND_ALPHA:
      for (int i = 0; i < np; i++) {
        real tau = p[A_NSP + 3 * i + 1];
        dy[2 + 2 * i + 1] = -y[2 + 2 * i + 1] / tau;
        dy[2 + 2 * i] = y[2 + 2 * i + 1] - y[2 + 2 * i] / tau;
      }
      break;
    case O_AEIF_PSC_ALPHA:
      for (int i = 0; i < np; i++) {
        real tau = p[A_NSP + 2 * i];
        dy[2 + 2 * i + 1] = -y[2 + 2 * i + 1] / tau;
        dy[2 + 2 * i] = y[2 + 2 * i + 1] - y[2 + 2 * i] / tau;
      }
      break;
    case O_AEIF_PSC_EXP:
      for (int i = 0; i < np; i++) dy[2 + i] = -y[2 + i] / p[A_NSP + i];
      break;
    default:
      break;
  }
}

// returns 1 if the neuron spiked
static int external_update(int model, real *y, real *p, bool end, real dt) {
  if (model == O_IZH_COND_BETA) {
    if (y[0] < -1.0e3 || y[1] < -1.0e6 || y[1] > 1.0e6) {
      y[0] = p[I_c]; y[1] = 0; return 0;
    }
    if (p[I_refr] > 0) {
      y[0] = p[I_c];
      if (end) p[I_refr] -= 1.0;
      return 0;
    }
    if (y[0] >= p[I_V_th]) {
      y[0] = p[I_c]; y[1] += p[I_d];
      real r = round(p[I_t_ref] / dt);
      p[I_refr] = r < 0 ? 0 : r;
      return 1;
    }
    return 0;
  }
  if (y[0] < -1.0e3 || y[1] < -1.0e6 || y[1] > 1.0e6) {
    y[0] = p[A_V_reset]; y[1] = 0; return 0;
  }
  if (p[A_refr] > 0) {
    y[0] = p[A_V_reset];
    if (end) p[A_refr] -= 1.0;
    return 0;
  }
  if (y[0] >= p[A_V_peak]) {
    y[0] = p[A_V_reset];
    y[1] += p[A_b];
    real r = round(p[A_t_ref] / dt);
    p[A_refr] = r < 0 ? 0 : r;
    return 1;
  }
  return 0;
}

// Cash-Karp coefficients
static const real c_a21 = 0.2, c_a31 = 3.0 / 40.0, c_a32 = 9.0 / 40.0, c_a41 = 0.3,
                  c_a42 = -0.9, c_a43 = 1.2, c_a51 = -11.0 / 54.0, c_a52 = 2.5,
                  c_a53 = -70.0 / 27.0, c_a54 = 35.0 / 27.0, c_a61 = 1631.0 / 55296.0,
                  c_a62 = 175.0 / 512.0, c_a63 = 575.0 / 13824.0,
                  c_a64 = 44275.0 / 110592.0, c_a65 = 253.0 / 4096.0,
                  c_a71 = 37.0 / 378.0, c_a73 = 250.0 / 621.0, c_a74 = 125.0 / 594.0,
                  c_a76 = 512.0 / 1771.0, c_e1 = 37.0 / 378.0 - 2825.0 / 27648.0,
                  c_e3 = 250.0 / 621.0 - 18575.0 / 48384.0,
                  c_e4 = 125.0 / 594.0 - 13525.0 / 55296.0, c_e5 = -277.0 / 14336.0,
                  c_e6 = 512.0 / 1771.0 - 0.25, c_coeff = 0.9, c_exp_inc = -0.2,
                  c_exp_dec = -0.25, c_err_min = 1.889568e-4, c_scal_min = 1.0e-1;

static void rk5_step(int model, int np, int nv, real &x, real *y, real &h, real h_min,
                     real h_max, const real *p, real eps, long long &evals) {
  real k1[64], k2[64], k3[64], k4[64], k5[64], k6[64], yn[64], ys[64];
  deriv(model, np, y, k1, p);
  evals++;
  for (int i = 0; i < nv; i++) ys[i] = fabs(y[i]) + fabs(k1[i] * h) + c_scal_min;
  real err = 0;
  for (int guard = 0;; guard++) {
    if (h > h_max) h = h_max;
    if (h < h_min) h = h_min;
    for (int i = 0; i < nv; i++) yn[i] = y[i] + h * c_a21 * k1[i];
    deriv(model, np, yn, k2, p);
    for (int i = 0; i < nv; i++) yn[i] = y[i] + h * (c_a31 * k1[i] + c_a32 * k2[i]);
    deriv(model, np, yn, k3, p);
    for (int i = 0; i < nv; i++) yn[i] = y[i] + h * (c_a41 * k1[i] + c_a42 * k2[i] + c_a43 * k3[i]);
    deriv(model, np, yn, k4, p);
    for (int i = 0; i < nv; i++)
      yn[i] = y[i] + h * (c_a51 * k1[i] + c_a52 * k2[i] + c_a53 * k3[i] + c_a54 * k4[i]);
    deriv(model, np, yn, k5, p);
    for (int i = 0; i < nv; i++)
      yn[i] = y[i] + h * (c_a61 * k1[i] + c_a62 * k2[i] + c_a63 * k3[i] + c_a64 * k4[i]
                          + c_a65 * k5[i]);
    deriv(model, np, yn, k6, p);
    for (int i = 0; i < nv; i++)
      yn[i] = y[i] + h * (c_a71 * k1[i] + c_a73 * k3[i] + c_a74 * k4[i] + c_a76 * k6[i]);
    evals += 5;
    err = 0;
    for (int i = 0; i < nv; i++) {
      real val = h * (c_e1 * k1[i] + c_e3 * k3[i] + c_e4 * k4[i] + c_e5 * k5[i] + c_e6 * k6[i]);
      val /= ys[i];
      err = std::max(err, fabs(val));
    }
    err /= eps;
    if (err <= 1.0 || h <= h_min * (1.0 + 1.0e-5) || guard > 256) break;
    real h_new = h * c_coeff * pow(err, c_exp_dec);
    h = std::max(h_new, 0.1 * h);
  }
  x += h;
  if (err > c_err_min) h = h * c_coeff * pow(err, c_exp_inc);
  else h = 5.0 * h;
  for (int i = 0; i < nv; i++) y[i] = yn[i];
}

// Scaled error of one Cash-Karp attempt with step h from y (no state
// change): the quantity the controller compares with 1 (the error scale
// formed with this h). Used by the exact step search.
static real rk5_trial_err(int model, int np, int nv, const real *y, const real *k1, real h,
                          const real *p, real eps, real *yout) {
  real k2[64], k3[64], k4[64], k5[64], k6[64], yn[64];
  for (int i = 0; i < nv; i++) yn[i] = y[i] + h * c_a21 * k1[i];
  deriv(model, np, yn, k2, p);
  for (int i = 0; i < nv; i++) yn[i] = y[i] + h * (c_a31 * k1[i] + c_a32 * k2[i]);
  deriv(model, np, yn, k3, p);
  for (int i = 0; i < nv; i++) yn[i] = y[i] + h * (c_a41 * k1[i] + c_a42 * k2[i] + c_a43 * k3[i]);
  deriv(model, np, yn, k4, p);
  for (int i = 0; i < nv; i++)
    yn[i] = y[i] + h * (c_a51 * k1[i] + c_a52 * k2[i] + c_a53 * k3[i] + c_a54 * k4[i]);
  deriv(model, np, yn, k5, p);
  for (int i = 0; i < nv; i++)
    yn[i] = y[i] + h * (c_a61 * k1[i] + c_a62 * k2[i] + c_a63 * k3[i] + c_a64 * k4[i]
                        + c_a65 * k5[i]);
  deriv(model, np, yn, k6, p);
  real err = 0;
  for (int i = 0; i < nv; i++) {
    yout[i] = y[i] + h * (c_a71 * k1[i] + c_a73 * k3[i] + c_a74 * k4[i] + c_a76 * k6[i]);
    real val = h * (c_e1 * k1[i] + c_e3 * k3[i] + c_e4 * k4[i] + c_e5 * k5[i] + c_e6 * k6[i]);
    real ys = fabs(y[i]) + fabs(k1[i] * h) + c_scal_min;
    err = std::max(err, fabs(val / ys));
  }
  return err / eps;
}

// One sub-step with the largest step in [h_min, h_max] that the error test
// accepts, found by bisection over log h (a proposer that knew the answer):
// only the accepted attempt's 6 evaluations are counted, so the group's
// evaluation count is a lower bound for any step-size proposer that keeps
// the same acceptance test.
static void rk5_step_search(int model, int np, int nv, real &x, real *y, real &h, real h_min,
                            real h_max, const real *p, real eps, long long &evals) {
  real k1[64], yn[64], yb[64];
  deriv(model, np, y, k1, p);
  real hs = h_max;
  if (rk5_trial_err(model, np, nv, y, k1, h_max, p, eps, yb) > 1.0) {
    real lo = log(h_min), hi = log(h_max);
    real best = h_min;
    rk5_trial_err(model, np, nv, y, k1, h_min, p, eps, yb);
    for (int it = 0; it < 40; it++) {
      const real mid = 0.5 * (lo + hi);
      const real hm = exp(mid);
      if (rk5_trial_err(model, np, nv, y, k1, hm, p, eps, yn) <= 1.0) {
        lo = mid;
        best = hm;
        for (int i = 0; i < nv; i++) yb[i] = yn[i];
      } else {
        hi = mid;
      }
    }
    hs = best;
  }
  evals += 6;
  x += hs;
  h = hs;
  for (int i = 0; i < nv; i++) y[i] = yb[i];
}

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

// input var index and weight of port q
static int in_var(const Group &g, int q) {
  switch (g.model) {
    case O_AEIF_COND_BETA: case O_AEIF_COND_ALPHA: case O_AEIF_PSC_ALPHA:
    case O_IZH_COND_BETA: return 2 + 2 * q + 1;
    case O_AEIF_PSC_EXP: return 2 + q;
    case O_AEIF_PSC_DELTA: return 0;
    case O_IAF_PSC_EXP: return q;
    case O_PARROT: return q;
    case O_IAF_PSC_EXP_G: case O_IZHIKEVICH: case O_IZH_PSC_EXP: return 0;
    default: return -1;
  }
}
static real in_weight(const Group &g, int i, int q) {
  const real *p = &g.param[(size_t)i * g.nparam];
  switch (g.model) {
    case O_AEIF_COND_BETA: return p[A_NSP + 4 * q + 3];
    case O_IZH_COND_BETA: return p[I_NSP + 4 * q + 3];
    case O_AEIF_COND_ALPHA: return p[A_NSP + 3 * q + 2];
    case O_AEIF_PSC_ALPHA: return p[A_NSP + 2 * q + 1];
    case O_PARROT: return q == 0 ? 1.0 : 0.0;
    default: return 1.0;
  }
}

static void syn_update(const Oracle &o, int sg, real &w, real Dt) {
  const Oracle::SynG &s = o.syn[sg - 1];
  if (s.type == 2) {
    real tau_plus = s.p[0], tau_minus = s.p[1], lambda = s.p[2], alpha = s.p[3];
    real mu_plus = s.p[4], mu_minus = s.p[5], Wmax = s.p[6];
    real w1;
    if (Dt >= 0) w1 = w + lambda * exp(-Dt / tau_plus) * Wmax * pow(1.0 - w / Wmax, mu_plus);
    else w1 = w - alpha * lambda * exp(Dt / tau_minus) * Wmax * pow(w / Wmax, mu_minus);
    w1 = w1 > 0 ? w1 : 0;
    w = w1 < Wmax ? w1 : Wmax;
  } else if (s.type == 1) {
    w += s.p[1] + s.p[0] * Dt;
  }
}

// dendritic delay of a node in steps (src/spike_buffer.cu:148-166)
static int den_steps(const Oracle &o, int node) {
  const Group &g = o.groups[o.node_group[node]];
  const real *p = &g.param[(size_t)(node - g.i0) * g.nparam];
  real d = 0.0;
  switch (g.model) {
    case O_AEIF_COND_BETA: case O_AEIF_COND_ALPHA: case O_AEIF_PSC_ALPHA:
    case O_AEIF_PSC_EXP: case O_AEIF_PSC_DELTA: d = p[A_den_delay]; break;
    case O_IZH_COND_BETA: d = p[I_den_delay]; break;
    case O_IAF_PSC_EXP: d = p[9]; break;
    case O_PARROT: d = p[1]; break;
    case O_IZHIKEVICH: case O_IZH_PSC_EXP: d = p[1]; break;
    default: return 0;
  }
  return (int)round((float)d / (float)o.dt);
}

// A spike of step T reaches the node's own dendrites (STDP post rule) in
// step T + den_delay: at once for den_delay 0 (src/spike_buffer.cu:164-167),
// otherwise when the spike buffer's age reaches it (src/spike_buffer.cu:
// 265-300), which sets the node's last post-spike time to that step before
// that step's deliveries.
static void push(Oracle &o, int node, real height, long long T) {
  o.spikes_at[(size_t)(T % o.spikes_at.size())].push_back(std::make_pair(node, height));
  const int den = den_steps(o, node);
  if (den == 0) o.last_rev[node] = T;
  else o.rev_at[T + den].push_back(node);
  o.log_step.push_back(T - 1);
  o.log_node.push_back(node);
}

static void prepare(Oracle &o) {
  const int N = (int)o.node_group.size();
  std::stable_sort(o.edges.begin(), o.edges.end(), [](const Edge &a, const Edge &b) {
    if (a.src != b.src) return a.src < b.src;
    return a.d < b.d;
  });
  o.out_off.assign(N + 1, 0);
  int maxD = 1;
  for (const Edge &e : o.edges) { o.out_off[e.src + 1]++; maxD = std::max(maxD, e.d); }
  for (int i = 0; i < N; i++) o.out_off[i + 1] += o.out_off[i];
  o.spikes_at.assign(maxD + 1, {});
  o.in_plastic.assign(N, {});
  for (size_t k = 0; k < o.edges.size(); k++) {
    if (o.edges[k].syn > 0) o.in_plastic[o.edges[k].tgt].push_back(k);
    o.edges[k].stamp = -(1 << 30);
  }
  o.maxport = 1;
  for (const Group &g : o.groups) o.maxport = std::max(o.maxport, g.np);
  o.acc.assign((size_t)N * o.maxport, 0.0);
  o.last_rev.assign(N, -(1LL << 40));
  // Poisson direct connections, stream ids in (source, delay, insertion) order
  o.dc_of.assign(N, {});
  uint64_t stream = 0;
  for (int s = 0; s < N; s++) {
    const Group &g = o.groups[o.node_group[s]];
    if (g.model != O_POISSON_GENERATOR) continue;
    for (size_t k = o.out_off[s]; k < o.out_off[s + 1]; k++) {
      const Edge &e = o.edges[k];
      Oracle::DC c;
      c.gen_node = s; c.port = e.port; c.w = e.w;
      c.delay = (real)((float)o.dt * (float)e.d);
      c.stream = stream < o.dc_stream_set.size() ? o.dc_stream_set[stream] : stream;
      stream++;
      o.dc_of[e.tgt].push_back(c);
    }
  }
  // calibration: refractory counters and normalisations
  for (Group &g : o.groups) {
    for (int i = 0; i < g.n; i++) {
      real *p = &g.param[(size_t)i * g.nparam];
      switch (g.model) {
        case O_AEIF_COND_BETA: case O_IZH_COND_BETA: {
          int nsp = g.model == O_AEIF_COND_BETA ? (int)A_NSP : (int)I_NSP;
          p[g.model == O_AEIF_COND_BETA ? (int)A_refr : (int)I_refr] = 0;
          for (int q = 0; q < g.np; q++) {
            real tr = p[nsp + 4 * q + 1], td = p[nsp + 4 * q + 2];
            real d1 = td - tr, d2 = 0;
            if (d1 != 0) {
              real tp = td * tr * log(td / tr) / d1;
              d2 = exp(-tp / td) - exp(-tp / tr);
            }
            p[nsp + 4 * q + 3] = d2 == 0 ? M_E / td : (1.0 / tr - 1.0 / td) / d2;
          }
          break;
        }
        case O_AEIF_COND_ALPHA:
          p[A_refr] = 0;
          for (int q = 0; q < g.np; q++) p[A_NSP + 3 * q + 2] = M_E / p[A_NSP + 3 * q + 1];
          break;
        case O_AEIF_PSC_ALPHA:
          p[A_refr] = 0;
          for (int q = 0; q < g.np; q++) p[A_NSP + 2 * q + 1] = M_E / p[A_NSP + 2 * q];
          break;
        case O_AEIF_PSC_EXP: case O_AEIF_PSC_DELTA:
          p[A_refr] = 0;
          break;
        case O_IAF_PSC_EXP: {
          real h = o.dt, tau_m = p[0], C_m = p[1], tau_ex = p[6], tau_in = p[7];
          p[15] = exp(-h / tau_m);
          p[11] = exp(-h / tau_ex);
          p[12] = exp(-h / tau_in);
          p[13] = propagator_32(tau_ex, tau_m, C_m, h);
          p[14] = propagator_32(tau_in, tau_m, C_m, h);
          p[10] = tau_m / C_m * (1.0 - p[15]);
          break;
        }
        default:
          break;
      }
      if (g.model <= O_IZH_COND_BETA) {
        g.h[i] = g.h0_rel * o.dt;
        g.x[i] = 0.0;
      }
    }
  }
  o.prepared = true;
}

// fold the pending input into state: accumulators plus Poisson draws of
// step T (the step that just ended)
static void fold(Oracle &o, long long T_pending, bool poisson) {
  const int N = (int)o.node_group.size();
  double t = (double)T_pending * (double)(float)o.dt;
  // inversion thresholds per generator node (kept while its rate is unchanged)
  if (poisson) {
    if (o.gen_thr.size() != o.gen_rate.size()) {
      o.gen_thr.assign(o.gen_rate.size(), std::vector<uint32_t>());
      o.gen_thr_lam.assign(o.gen_rate.size(), -1.0);
    }
    for (size_t k = 0; k < o.gen_rate.size(); k++) {
      if (o.gen_rate[k] == 0) continue;
      float lf = (float)((double)(float)o.dt / 1000.0) * (float)o.gen_rate[k];
      double lam = (double)lf;
      if (o.gen_thr_lam[k] != lam) {
        o.gen_thr[k].resize(NGPU_CDF_LEN);
        ngpu::ng_poisson_thresholds(lam, exp(-lam), o.gen_thr[k].data());
        o.gen_thr_lam[k] = lam;
      }
    }
  }
  // every node folds only its own accumulators and state
#pragma omp parallel for schedule(static)
  for (int n = 0; n < N; n++) {
    Group &g = o.groups[o.node_group[n]];
    int i = n - g.i0;
    if (poisson) {
      for (const Oracle::DC &c : o.dc_of[n]) {
        double t_rel = t - o.gen_origin[c.gen_node] - c.delay;
        if (t_rel >= o.gen_start[c.gen_node] && t_rel <= o.gen_stop[c.gen_node]) {
          float lf = (float)((double)(float)o.dt / 1000.0) * (float)o.gen_rate[c.gen_node];
          double lam = (double)lf;
          unsigned cnt = ngpu::ng_poisson_direct(lam, o.gen_thr[c.gen_node].data(),
                                                 o.seed + 12345ULL, c.stream, T_pending);
          if (cnt > 0) o.acc[(size_t)n * o.maxport + c.port] += (double)((float)c.w * (float)cnt);
        }
      }
    }
    for (int q = 0; q < g.np; q++) {
      double &a = o.acc[(size_t)n * o.maxport + q];
      if (a == 0.0) continue;
      int vi = in_var(g, q);
      if (vi >= 0) g.var[(size_t)i * g.nvar + vi] += a * in_weight(g, i, q);
      a = 0.0;
    }
  }
}

// One time step of a simple model; true if the neuron spikes.
//   iaf_psc_exp:   vars I_ex, I_in, V_m_rel, refr; params as the library
//   iaf_psc_exp_g: vars I_syn, V_m_rel, refr; params I_e, tau_m, C_m, E_L,
//                  Theta_rel, V_reset_rel, tau_syn, t_ref, h_prop (the step of
//                  the propagators: dt, or 0.1 ms for iaf_psc_exp_hc)
//   izhikevich:    vars I_syn, V_m, u, refr; params I_e, den_delay, V_th, a,
//                  b, c, d, t_ref
//   izhikevich_psc_exp: as izhikevich plus tau_syn before t_ref and n_sub
static bool simple_update(int model, real *y, const real *p, real dt) {
  if (model == O_IAF_PSC_EXP) {
    real &I_ex = y[0], &I_in = y[1], &V = y[2], &refr = y[3];
    if (refr > 0) refr -= 1;
    else V = V * p[15] + I_ex * p[13] + I_in * p[14] + p[3] * p[10];
    I_ex *= p[11];
    I_in *= p[12];
    if (V >= p[4]) {
      V = p[5];
      refr = round(p[8] / dt);
      return true;
    }
    return false;
  }
  if (model == O_IAF_PSC_EXP_G) {
    real &I = y[0], &V = y[1], &refr = y[2];
    const real h = p[8] > 0 ? p[8] : dt;
    const real tau_m = p[1], C_m = p[2], tau_syn = p[6];
    const real P22 = exp(-h / tau_m);
    if (refr > 0) refr -= 1;
    else V = V * P22 + I * propagator_32(tau_syn, tau_m, C_m, h) + p[0] * (tau_m / C_m * (1.0 - P22));
    I *= exp(-h / tau_syn);
    if (V >= p[4]) {
      V = p[5];
      refr = round(p[7] / h);
      return true;
    }
    return false;
  }
  // Izhikevich family
  real &I = y[0], &V = y[1], &u = y[2], &refr = y[3];
  const real V_th = p[2], a = p[3], b = p[4], c = p[5], d = p[6];
  real h = dt, t_ref = p[7];
  if (model == O_IZHIKEVICH) {
    if (refr > 0) {
      refr -= 1;
    } else {
      const real v = V, w = u;
      V += h * (0.04 * v * v + 5.0 * v + 140.0 - w + p[0]) + I;
      u += h * a * (b * v - w);
    }
    I = 0;
  } else {
    const int n_sub = (int)p[9];
    h = dt / n_sub;
    t_ref = p[8];
    const real C_syn = exp(-h / p[7]);
    if (refr > 0) {
      refr -= 1;
      for (int k = 0; k < n_sub; k++) I *= C_syn;
    } else {
      for (int k = 0; k < n_sub; k++) {
        const real v = V, w = u;
        V += h * (0.04 * v * v + 5.0 * v + 140.0 - w + I + p[0]);
        u += h * a * (b * v - w);
        I *= C_syn;
      }
    }
  }
  if (V >= V_th) {
    V = c;
    u += d;
    refr = round(t_ref / h);
    if (refr < 0) refr = 0;
    return true;
  }
  return false;
}

static void step(Oracle &o, int it_in_session) {
  const long long T = o.T + 1;            // time index after this step
  const double t0 = (double)o.T * (double)(float)o.dt;
  const double x1 = t0 + (double)(float)o.dt;
  o.spikes_at[(size_t)(T % o.spikes_at.size())].clear();
  (void)it_in_session;
  for (Group &g : o.groups) {
    // node updates are independent: RK5 and iaf groups are updated in
    // parallel, each thread collecting its spikes in node order; the lists
    // are merged in thread (= node) order, so the result does not depend on
    // the number of threads
    if (g.model <= O_IZH_COND_BETA || simple_model(g.model)) {
      int nthr = 1;
#ifdef _OPENMP
      nthr = omp_get_max_threads();
#endif
      std::vector<std::vector<std::pair<int, real>>> part(nthr);
      std::vector<long long> evals(nthr, 0);
#pragma omp parallel num_threads(nthr)
      {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        const int chunk = (g.n + nthr - 1) / nthr;
        const int i0 = std::min(g.n, tid * chunk), i1 = std::min(g.n, i0 + chunk);
        for (int i = i0; i < i1; i++) {
          real *y = &g.var[(size_t)i * g.nvar];
          real *p = &g.param[(size_t)i * g.nparam];
          int node = g.i0 + i;
          if (g.model <= O_IZH_COND_BETA) {
            real h_min = g.h_min_rel * o.dt;
            real &x = g.x[i];
            real &h = g.h[i];
            bool end = false;
            int guard = 0;
            while (!end && guard++ < 200000) {
              real hmax = x1 - x;
              if (g.step_search)
                rk5_step_search(g.model, g.model == O_AEIF_PSC_DELTA ? 0 : g.np, g.nvar, x, y, h,
                                h_min, hmax, p, g.eps, evals[tid]);
              else
                rk5_step(g.model, g.model == O_AEIF_PSC_DELTA ? 0 : g.np, g.nvar, x, y, h, h_min,
                         hmax, p, g.eps, evals[tid]);
              end = (x >= x1 - h_min);
              if (external_update(g.model, y, p, end, o.dt)) part[tid].push_back({node, 1.0});
            }
          } else if (simple_update(g.model, y, p, o.dt)) {
            part[tid].push_back({node, 1.0});
          }
        }
      }
      for (int t = 0; t < nthr; t++) {
        g.evals += evals[t];
        for (const auto &sp : part[t]) push(o, sp.first, sp.second, T);
      }
      continue;
    }
    for (int i = 0; i < g.n; i++) {
      real *y = &g.var[(size_t)i * g.nvar];
      real *p = &g.param[(size_t)i * g.nparam];
      int node = g.i0 + i;
      if (g.model <= O_IZH_COND_BETA) {
        real h_min = g.h_min_rel * o.dt;
        real &x = g.x[i];
        real &h = g.h[i];
        bool end = false;
        int guard = 0;
        while (!end && guard++ < 200000) {
          real hmax = x1 - x;
          if (g.step_search)
            rk5_step_search(g.model, g.model == O_AEIF_PSC_DELTA ? 0 : g.np, g.nvar, x, y, h,
                            h_min, hmax, p, g.eps, g.evals);
          else
            rk5_step(g.model, g.model == O_AEIF_PSC_DELTA ? 0 : g.np, g.nvar, x, y, h, h_min,
                     hmax, p, g.eps, g.evals);
          end = (x >= x1 - h_min);
          if (external_update(g.model, y, p, end, o.dt)) push(o, node, 1.0, T);
        }
      } else if (simple_model(g.model)) {
        if (simple_update(g.model, y, p, o.dt)) push(o, node, 1.0, T);
      } else if (g.model == O_SPIKE_GENERATOR) {
        int b = g.sg_next[i];
        if (b < g.sg_off[i + 1] && (long long)g.sg_step[b] == T - 1) {
          push(o, node, g.sg_height[b], T);
          g.sg_next[i] = b + 1;
        }
      } else if (g.model == O_PARROT) {
        real sh = y[0];
        y[2] = sh;
        if (sh != 0) {
          if (p[0] == 0) sh = 1;
          y[0] = 0;
          push(o, node, sh, T);
        }
      }
    }
  }
  // spikes reaching dendrites now (dendritic delay > 0)
  std::vector<int> arrivals;
  {
    auto it = o.rev_at.find(T);
    if (it != o.rev_at.end()) {
      arrivals = it->second;
      o.rev_at.erase(it);
      for (int n : arrivals) o.last_rev[n] = T;
    }
  }
  // delivery of spikes emitted D steps ago, with the STDP pre rule
  const size_t R = o.spikes_at.size();
  for (size_t D = 1; D < R; D++) {
    const auto &lst = o.spikes_at[(size_t)((((T - (long long)D) % (long long)R) + (long long)R) % (long long)R)];
    for (const auto &sp : lst) {
      int s = sp.first;
      for (size_t k = o.out_off[s]; k < o.out_off[s + 1]; k++) {
        Edge &e = o.edges[k];
        if (e.d != (int)D) continue;
        if (o.groups[o.node_group[s]].model == O_POISSON_GENERATOR) continue;
        o.acc[(size_t)e.tgt * o.maxport + e.port] += (double)((float)sp.second * (float)e.w);
        if (e.syn > 0) {
          e.stamp = (int)T;
          long long Dt = T - o.last_rev[e.tgt];
          if (Dt > 0 && Dt < NGPU_MAX_SYN_DT_ORACLE) {
            real w = e.w;
            syn_update(o, e.syn, w, -(double)(float)o.dt * (double)Dt);
            e.w = (real)(float)w;
          }
        }
      }
    }
  }
  // STDP post rule for neurons whose spike reaches their dendrites in this
  // step: spikes of this step without dendritic delay, then the arrivals
  {
    const auto &lst = o.spikes_at[(size_t)(T % (long long)R)];
    std::vector<int> cand;
    for (const auto &sp : lst)
      if (den_steps(o, sp.first) == 0) cand.push_back(sp.first);
    cand.insert(cand.end(), arrivals.begin(), arrivals.end());
    std::vector<int> seen;
    for (int n : cand) {
      if (std::find(seen.begin(), seen.end(), n) != seen.end()) continue;
      seen.push_back(n);
      for (size_t k : o.in_plastic[n]) {
        Edge &e = o.edges[k];
        long long Dt = T - e.stamp;
        if (Dt >= 0 && Dt < NGPU_MAX_SYN_DT_ORACLE) {
          real w = e.w;
          syn_update(o, e.syn, w, (double)(float)o.dt * (double)Dt);
          e.w = (real)(float)w;
        }
      }
    }
  }
  o.T = T;
}

}  // namespace


extern "C" {

void *orc_create(double dt, unsigned long long seed) {
  Oracle *o = new Oracle;
  o->dt = dt;
  o->seed = seed;
  return o;
}

void orc_free(void *h) { delete (Oracle *)h; }

// Connection rules (src/connect_rules.h:48-400) with the library's random
// streams: per call index `call`, fixed_total_number draws pair k from
// Philox(seed, CONNECT, call, k); fixed_indegree / fixed_outdegree draw K
// distinct pool members for every outer node o from
// Philox(seed, SOURCE_SET, call, o, draw) by partial Fisher-Yates (pool
// < 5 K) or rejection of repeats. Writes the source and target list indices
// of every connection in insertion order; returns their number.
long long orc_rule_edges(int rule, unsigned long long seed, unsigned long long call,
                         int n_source, int n_target, int param, int *out_s, int *out_t) {
  long long m = 0;
  switch (rule) {
    case 0:  // one_to_one
      for (int k = 0; k < n_source; k++) { out_s[m] = k; out_t[m] = k; m++; }
      break;
    case 1:  // all_to_all
      for (int it = 0; it < n_target; it++)
        for (int is = 0; is < n_source; is++) { out_s[m] = is; out_t[m] = it; m++; }
      break;
    case 2:  // fixed_total_number
      for (long long k = 0; k < param; k++) {
        ngpu::Philox4 r = ngpu::ng_random_block(seed, ngpu::RNG_TAG_CONNECT, call, (uint64_t)k, 0);
        out_s[m] = (int)(r.v[0] % (uint32_t)n_source);
        out_t[m] = (int)(r.v[1] % (uint32_t)n_target);
        m++;
      }
      break;
    case 3: case 4: {  // fixed_indegree, fixed_outdegree
      const bool indeg = rule == 3;
      const int K = param;
      const long long n_outer = indeg ? n_target : n_source;
      const long long n_pool = indeg ? n_source : n_target;
      std::vector<int> pick(K);
      for (long long o = 0; o < n_outer; o++) {
        if (n_pool < 5LL * K) {
          std::vector<int> perm(n_pool);
          for (long long j = 0; j < n_pool; j++) perm[j] = (int)j;
          for (int i = 0; i < K; i++) {
            ngpu::Philox4 r = ngpu::ng_random_block(seed, ngpu::RNG_TAG_SOURCE_SET, call,
                                                    (uint64_t)o, (uint32_t)i);
            long long j = i + (long long)(r.v[0] % (uint32_t)(n_pool - i));
            std::swap(perm[i], perm[j]);
            pick[i] = perm[i];
          }
        } else {
          int cap = 16;
          while (cap < 2 * K) cap <<= 1;
          std::vector<int> table(cap, -1);
          uint32_t draw = 0;
          for (int i = 0; i < K; i++) {
            int j;
            for (;;) {
              ngpu::Philox4 r = ngpu::ng_random_block(seed, ngpu::RNG_TAG_SOURCE_SET, call,
                                                      (uint64_t)o, draw++);
              j = (int)(r.v[0] % (uint32_t)n_pool);
              uint32_t h = ((uint32_t)j * 0x9E3779B1u) & (uint32_t)(cap - 1);
              bool dup = false;
              while (table[h] >= 0) {
                if (table[h] == j) { dup = true; break; }
                h = (h + 1) & (uint32_t)(cap - 1);
              }
              if (!dup) { table[h] = j; break; }
            }
            pick[i] = j;
          }
        }
        for (int i = 0; i < K; i++) {
          out_s[m] = indeg ? pick[i] : (int)o;
          out_t[m] = indeg ? (int)o : pick[i];
          m++;
        }
      }
      break;
    }
    default:
      return -1;
  }
  return m;
}

// host threads of the parallel node-update and fold loops (results do not
// depend on it)
void orc_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

int orc_get_threads() {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

// params: [n][nparam]; vars: [n][nvar]
int orc_add_group(void *h, int model, int n, int np, int nvar, int nparam,
                  const double *params, const double *vars, double h_min_rel,
                  double h0_rel, double eps) {
  Oracle *o = (Oracle *)h;
  Group g;
  g.model = model; g.n = n; g.np = np; g.nvar = nvar; g.nparam = nparam;
  g.i0 = (int)o->node_group.size();
  g.param.assign(params, params + (size_t)n * nparam);
  g.var.assign(vars, vars + (size_t)n * nvar);
  g.h.assign(n, 0); g.x.assign(n, 0);
  g.h_min_rel = h_min_rel; g.h0_rel = h0_rel; g.eps = eps;
  g.sg_off.assign(n + 1, 0);
  g.sg_next.assign(n + 1, 0);
  o->groups.push_back(g);
  o->node_group.insert(o->node_group.end(), n, (int)o->groups.size() - 1);
  o->gen_rate.resize(o->node_group.size(), 0);
  o->gen_origin.resize(o->node_group.size(), 0);
  o->gen_start.resize(o->node_group.size(), 0);
  o->gen_stop.resize(o->node_group.size(), 1e30);
  if (model == O_POISSON_GENERATOR) {
    for (int i = 0; i < n; i++) {
      o->gen_rate[g.i0 + i] = params[(size_t)i * nparam + 0];
      o->gen_origin[g.i0 + i] = params[(size_t)i * nparam + 1];
      o->gen_start[g.i0 + i] = params[(size_t)i * nparam + 2];
      o->gen_stop[g.i0 + i] = params[(size_t)i * nparam + 3];
    }
  }
  return g.i0;
}

// spike generator tables: off[n+1], step[], height[]
int orc_set_spikes(void *h, int group, const int *off, const int *steps, const double *heights) {
  Oracle *o = (Oracle *)h;
  Group &g = o->groups[group];
  g.sg_off.assign(off, off + g.n + 1);
  g.sg_next.assign(off, off + g.n + 1);
  g.sg_step.assign(steps, steps + off[g.n]);
  g.sg_height.assign(heights, heights + off[g.n]);
  return 0;
}

int orc_add_syn_group(void *h, int type, const double *p, int np) {
  Oracle *o = (Oracle *)h;
  Oracle::SynG s;
  s.type = type;
  memset(s.p, 0, sizeof(s.p));
  for (int i = 0; i < np && i < 8; i++) s.p[i] = p[i];
  o->syn.push_back(s);
  return (int)o->syn.size();
}

// delays in ms, converted like src/connect.cu:37 (d_int + 1 steps)
void orc_set_step_search(void *h, int group, int on) {
  Oracle *o = (Oracle *)h;
  o->groups[group].step_search = on != 0;
}

long long orc_group_evals(void *h, int group) { return ((Oracle *)h)->groups[group].evals; }

void orc_set_direct_streams(void *h, long long n, const unsigned long long *streams) {
  Oracle *o = (Oracle *)h;
  o->dc_stream_set.assign(streams, streams + n);
  o->prepared = false;
}

int orc_connect(void *h, long long n, const int *src, const int *tgt, const int *port,
                const int *syn, const float *w, const float *delay) {
  Oracle *o = (Oracle *)h;
  long long base = (long long)o->edges.size();
  for (long long k = 0; k < n; k++) {
    Edge e;
    e.src = src[k]; e.tgt = tgt[k]; e.port = port[k]; e.syn = syn[k];
    e.w = (real)w[k];
    e.d = (int)roundf(delay[k] / (float)o->dt);
    e.order = base + k;
    e.stamp = 0;
    o->edges.push_back(e);
  }
  return 0;
}

// Runs n_steps; rec_nodes/rec_vars select state values recorded after every
// step into out[(n_steps) x n_rec] (column = var index within the node).
int orc_simulate(void *h, int n_steps, int n_rec, const int *rec_nodes, const int *rec_vars,
                 double *out) {
  Oracle *o = (Oracle *)h;
  if (!o->prepared) prepare(*o);
  for (int s = 0; s < n_steps; s++) {
    if (o->T > 0 || s > 0) fold(*o, o->T, true);
    step(*o, s);
    for (int r = 0; r < n_rec; r++) {
      const Group &g = o->groups[o->node_group[rec_nodes[r]]];
      out[(size_t)s * n_rec + r] = g.var[(size_t)(rec_nodes[r] - g.i0) * g.nvar + rec_vars[r]];
    }
  }
  return 0;
}

// folds the input of the last step (call before reading final state)
int orc_flush(void *h) {
  Oracle *o = (Oracle *)h;
  if (o->T > 0) fold(*o, o->T, true);
  return 0;
}

long long orc_n_spikes(void *h) { return (long long)((Oracle *)h)->log_step.size(); }

int orc_get_spikes(void *h, long long *steps, int *nodes) {
  Oracle *o = (Oracle *)h;
  for (size_t k = 0; k < o->log_step.size(); k++) {
    steps[k] = o->log_step[k];
    nodes[k] = o->log_node[k];
  }
  return 0;
}

// weights in insertion order
int orc_get_weights(void *h, float *w) {
  Oracle *o = (Oracle *)h;
  for (const Edge &e : o->edges) w[e.order] = (float)e.w;
  return 0;
}

int orc_get_state(void *h, int node, double *var_out, double *param_out) {
  Oracle *o = (Oracle *)h;
  const Group &g = o->groups[o->node_group[node]];
  int i = node - g.i0;
  for (int j = 0; j < g.nvar; j++) var_out[j] = g.var[(size_t)i * g.nvar + j];
  if (param_out)
    for (int j = 0; j < g.nparam; j++) param_out[j] = g.param[(size_t)i * g.nparam + j];
  return 0;
}

long long orc_stage_evals(void *h) {
  long long t = 0;
  for (const Group &g : ((Oracle *)h)->groups) t += g.evals;
  return t;
}

}  // extern "C"
