// Device right-hand sides of the RK5 neuron models.
//
// Each model exposes, for a compile-time port bound NP and a runtime port
// count np <= NP:
//   deriv(y, dydx, p, q, refr, np) -- the model ODE
//   external(y, p, refr, end, dt)  -- post-substep update; returns 1 when the
//                                     neuron spiked
// p[j] is parameter j and q[j] its reciprocal 1/p[j]; both point either into
// the kernel's constant parameter block (group-uniform parameters) or to
// per-neuron register arrays. Divisions by parameters are written as
// multiplications by q[j], which the caller computes once per step (or the
// host once per launch) instead of once per right-hand-side evaluation.
// refr is the neuron's refractory counter (the reference keeps it in the
// parameter array as "refractory_step").
// Index layout of y and p (scalar entries first, then per-port blocks) is the
// reference's, e.g. src/aeif_cond_beta_kernel.h:30-72; the equations follow
// src/aeif_cond_beta_kernel.h:153-214 and the other *_kernel.h files.
#pragma once
#include <math.h>
#include "ngpu_f32x2.cuh"

namespace ngpu {

// Cash-Karp tableau and controller constants as single-precision values
// (the reference's __constant__ floats, src/rk5.cu:23-60).
namespace rk5c {
constexpr float c2 = 0.2f, c3 = 0.3f, c4 = 0.6f, c5 = 1.0f, c6 = 0.875f;
constexpr float a21 = 0.2f;
constexpr float a31 = (float)(3.0 / 40.0), a32 = (float)(9.0 / 40.0);
constexpr float a41 = 0.3f, a42 = -0.9f, a43 = 1.2f;
constexpr float a51 = (float)(-11.0 / 54.0), a52 = 2.5f,
                a53 = (float)(-70.0 / 27.0), a54 = (float)(35.0 / 27.0);
constexpr float a61 = (float)(1631.0 / 55296.0), a62 = (float)(175.0 / 512.0),
                a63 = (float)(575.0 / 13824.0),
                a64 = (float)(44275.0 / 110592.0),
                a65 = (float)(253.0 / 4096.0);
constexpr float a71 = (float)(37.0 / 378.0), a73 = (float)(250.0 / 621.0),
                a74 = (float)(125.0 / 594.0), a76 = (float)(512.0 / 1771.0);
constexpr float e1 = (float)(37.0 / 378.0 - 2825.0 / 27648.0);
constexpr float e3 = (float)(250.0 / 621.0 - 18575.0 / 48384.0);
constexpr float e4 = (float)(125.0 / 594.0 - 13525.0 / 55296.0);
constexpr float e5 = (float)(-277.00 / 14336.0);
constexpr float e6 = (float)(512.0 / 1771.0 - 0.25);
constexpr float coeff = 0.9f;
constexpr float exp_inc = -0.2f;
constexpr float exp_dec = -0.25f;
constexpr float err_min = 1.889568e-4f;
constexpr float scal_min = 1.0e-1f;
}  // namespace rk5c

// ---------------------------------------------------------------------------
// AdEx family: common scalar part (V_m, w; 14 scalar parameters)
// ---------------------------------------------------------------------------
enum AeifScal {
  A_V_th = 0, A_Delta_T, A_g_L, A_E_L, A_C_m, A_a, A_b, A_tau_w, A_I_e,
  A_V_peak, A_V_reset, A_t_ref, A_refr, A_den_delay, A_NSP
};

__device__ __forceinline__ int aeif_external(float *y, const float *p,
                                             float &refr, bool end, float dt) {
  float &V_m = y[0];
  float &w = y[1];
  if (V_m < -1.0e3f) {           // numerical instability guard
    V_m = p[A_V_reset];
    w = 0.0f;
    return 0;
  }
  if (w < -1.0e6f || w > 1.0e6f) {
    V_m = p[A_V_reset];
    w = 0.0f;
    return 0;
  }
  if (refr > 0.0f) {
    V_m = p[A_V_reset];
    if (end) refr -= 1.0f;
    return 0;
  }
  if (V_m >= p[A_V_peak]) {
    V_m = p[A_V_reset];
    w += p[A_b];
    float r = (float)(int)roundf(p[A_t_ref] / dt);
    refr = r < 0.0f ? 0.0f : r;
    return 1;
  }
  return 0;
}

// membrane and adaptation derivatives shared by the AdEx models
__device__ __forceinline__ void aeif_vw(const float *y, float *dydx,
                                        const float *p, const float *q,
                                        float refr, float V, float I_in,
                                        bool exp_guard) {
  float V_spike;
  if (exp_guard && p[A_Delta_T] == 0.0f) {
    V_spike = 0.0f;
  } else {
    // Delta_T e^((V - V_th) / Delta_T) as Delta_T 2^((V - V_th) log2(e) / Delta_T)
    V_spike = p[A_Delta_T] * ex2_approx((V - p[A_V_th]) * (q[A_Delta_T] * kLog2e));
  }
  dydx[0] = (refr > 0.0f) ? 0.0f
      : (-p[A_g_L] * (V - p[A_E_L] - V_spike) + I_in - y[1] + p[A_I_e])
        * q[A_C_m];
  dydx[1] = (p[A_a] * (V - p[A_E_L]) - y[1]) * q[A_tau_w];
}

template <int NP>
struct AeifCondBeta {
  enum { NSV = 2, NPV = 2, NSP = A_NSP, NPP = 4,
         NVAR = NSV + NPV * NP, NPARAM = NSP + NPP * NP };
  __device__ __forceinline__ static void deriv(const float *y, float *dydx,
                                               const float *p, const float *q,
                                               float refr, int np) {
    float V = (refr > 0.0f) ? p[A_V_reset] : fminf(y[0], p[A_V_peak]);
    float I_syn = 0.0f;
#pragma unroll
    for (int i = 0; i < NP; i++) {
      if (i < np) I_syn += y[NSV + NPV * i] * (p[NSP + NPP * i] - V);
    }
    aeif_vw(y, dydx, p, q, refr, V, I_syn, false);
#pragma unroll
    for (int i = 0; i < NP; i++) {
      if (i < np) {
        float g = y[NSV + NPV * i], g1 = y[NSV + NPV * i + 1];
        dydx[NSV + NPV * i + 1] = -g1 * q[NSP + NPP * i + 1];
        dydx[NSV + NPV * i] = g1 - g * q[NSP + NPP * i + 2];
      }
    }
  }
  __device__ __forceinline__ static int external(float *y, const float *p,
                                                 float &refr, bool end,
                                                 float dt) {
    return aeif_external(y, p, refr, end, dt);
  }
};

template <int NP>
struct AeifCondAlpha {
  enum { NSV = 2, NPV = 2, NSP = A_NSP, NPP = 3,
         NVAR = NSV + NPV * NP, NPARAM = NSP + NPP * NP };
  __device__ __forceinline__ static void deriv(const float *y, float *dydx,
                                               const float *p, const float *q,
                                               float refr, int np) {
    float V = (refr > 0.0f) ? p[A_V_reset] : fminf(y[0], p[A_V_peak]);
    float I_syn = 0.0f;
#pragma unroll
    for (int i = 0; i < NP; i++) {
      if (i < np) I_syn += y[NSV + NPV * i] * (p[NSP + NPP * i] - V);
    }
    aeif_vw(y, dydx, p, q, refr, V, I_syn, false);
#pragma unroll
    for (int i = 0; i < NP; i++) {
      if (i < np) {
        float g = y[NSV + NPV * i], g1 = y[NSV + NPV * i + 1];
        float itau = q[NSP + NPP * i + 1];
        dydx[NSV + NPV * i + 1] = -g1 * itau;
        dydx[NSV + NPV * i] = g1 - g * itau;
      }
    }
  }
  __device__ __forceinline__ static int external(float *y, const float *p,
                                                 float &refr, bool end,
                                                 float dt) {
    return aeif_external(y, p, refr, end, dt);
  }
};

template <int NP>
struct AeifPscAlpha {
  enum { NSV = 2, NPV = 2, NSP = A_NSP, NPP = 2,
         NVAR = NSV + NPV * NP, NPARAM = NSP + NPP * NP };
  __device__ __forceinline__ static void deriv(const float *y, float *dydx,
                                               const float *p, const float *q,
                                               float refr, int np) {
    float V = (refr > 0.0f) ? p[A_V_reset] : fminf(y[0], p[A_V_peak]);
    float I_tot = 0.0f;
#pragma unroll
    for (int i = 0; i < NP; i++) {
      if (i < np) I_tot += y[NSV + NPV * i];
    }
    aeif_vw(y, dydx, p, q, refr, V, I_tot, true);
#pragma unroll
    for (int i = 0; i < NP; i++) {
      if (i < np) {
        float I = y[NSV + NPV * i], I1 = y[NSV + NPV * i + 1];
        float itau = q[NSP + NPP * i];
        dydx[NSV + NPV * i + 1] = -I1 * itau;
        dydx[NSV + NPV * i] = I1 - I * itau;
      }
    }
  }
  __device__ __forceinline__ static int external(float *y, const float *p,
                                                 float &refr, bool end,
                                                 float dt) {
    return aeif_external(y, p, refr, end, dt);
  }
};

template <int NP>
struct AeifPscExp {
  enum { NSV = 2, NPV = 1, NSP = A_NSP, NPP = 1,
         NVAR = NSV + NPV * NP, NPARAM = NSP + NPP * NP };
  __device__ __forceinline__ static void deriv(const float *y, float *dydx,
                                               const float *p, const float *q,
                                               float refr, int np) {
    float V = (refr > 0.0f) ? p[A_V_reset] : fminf(y[0], p[A_V_peak]);
    float I_tot = 0.0f;
#pragma unroll
    for (int i = 0; i < NP; i++) {
      if (i < np) I_tot += y[NSV + i];
    }
    aeif_vw(y, dydx, p, q, refr, V, I_tot, true);
#pragma unroll
    for (int i = 0; i < NP; i++) {
      if (i < np) dydx[NSV + i] = -y[NSV + i] * q[NSP + i];
    }
  }
  __device__ __forceinline__ static int external(float *y, const float *p,
                                                 float &refr, bool end,
                                                 float dt) {
    return aeif_external(y, p, refr, end, dt);
  }
};

template <int NP>
struct AeifPscDelta {
  enum { NSV = 2, NPV = 0, NSP = A_NSP, NPP = 0, NVAR = 2, NPARAM = A_NSP };
  __device__ __forceinline__ static void deriv(const float *y, float *dydx,
                                               const float *p, const float *q,
                                               float refr, int np) {
    float V = (refr > 0.0f) ? p[A_V_reset] : fminf(y[0], p[A_V_peak]);
    aeif_vw(y, dydx, p, q, refr, V, 0.0f, true);
  }
  __device__ __forceinline__ static int external(float *y, const float *p,
                                                 float &refr, bool end,
                                                 float dt) {
    return aeif_external(y, p, refr, end, dt);
  }
};

// Izhikevich with beta-function conductances
enum IzhScal {
  I_V_th = 0, I_a, I_b, I_c, I_d, I_I_e, I_t_ref, I_refr, I_den_delay, I_NSP
};

template <int NP>
struct IzhCondBeta {
  enum { NSV = 2, NPV = 2, NSP = I_NSP, NPP = 4,
         NVAR = NSV + NPV * NP, NPARAM = NSP + NPP * NP };
  __device__ __forceinline__ static void deriv(const float *y, float *dydx,
                                               const float *p, const float *q,
                                               float refr, int np) {
    float V = (refr > 0.0f) ? p[I_c] : y[0];
    float I_syn = 0.0f;
#pragma unroll
    for (int i = 0; i < NP; i++) {
      if (i < np) I_syn += y[NSV + NPV * i] * (p[NSP + NPP * i] - V);
    }
    dydx[0] = (refr > 0.0f) ? 0.0f
        : 0.04f * V * V + 5.0f * V + 140.0f - y[1] + I_syn + p[I_I_e];
    dydx[1] = p[I_a] * (p[I_b] * V - y[1]);
#pragma unroll
    for (int i = 0; i < NP; i++) {
      if (i < np) {
        float g = y[NSV + NPV * i], g1 = y[NSV + NPV * i + 1];
        dydx[NSV + NPV * i + 1] = -g1 * q[NSP + NPP * i + 1];
        dydx[NSV + NPV * i] = g1 - g * q[NSP + NPP * i + 2];
      }
    }
  }
  __device__ __forceinline__ static int external(float *y, const float *p,
                                                 float &refr, bool end,
                                                 float dt) {
    float &V_m = y[0];
    float &u = y[1];
    if (V_m < -1.0e3f || u < -1.0e6f || u > 1.0e6f) {
      V_m = p[I_c];
      u = 0.0f;
      return 0;
    }
    if (refr > 0.0f) {
      V_m = p[I_c];
      if (end) refr -= 1.0f;
      return 0;
    }
    if (V_m >= p[I_V_th]) {
      V_m = p[I_c];
      u += p[I_d];
      float r = (float)(int)roundf(p[I_t_ref] / dt);
      refr = r < 0.0f ? 0.0f : r;
      return 1;
    }
    return 0;
  }
};

}  // namespace ngpu
