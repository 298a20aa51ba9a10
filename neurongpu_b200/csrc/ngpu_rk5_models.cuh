// Device right-hand sides of the RK5 neuron models.
//
// Each model exposes, for a compile-time port bound NP and a runtime port
// count np <= NP:
//   deriv(y, dydx, p, np)        -- the model ODE
//   external(y, p, end, dt)      -- post-substep update; returns the number
//                                   of spikes emitted (0 or 1)
// Index layout of y and p (scalar entries first, then per-port blocks) is
// the reference's, e.g. src/aeif_cond_beta_kernel.h:30-72.
#pragma once
#include <math.h>

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

__device__ __forceinline__ int aeif_external(float *y, float *p, bool end,
                                             float dt) {
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
  if (p[A_refr] > 0.0f) {
    V_m = p[A_V_reset];
    if (end) p[A_refr] -= 1.0f;
    return 0;
  }
  if (V_m >= p[A_V_peak]) {
    V_m = p[A_V_reset];
    w += p[A_b];
    float r = (float)(int)roundf(p[A_t_ref] / dt);
    p[A_refr] = r < 0.0f ? 0.0f : r;
    return 1;
  }
  return 0;
}

template <int NP>
struct AeifCondBeta {
  enum { NSV = 2, NPV = 2, NSP = A_NSP, NPP = 4,
         NVAR = NSV + NPV * NP, NPARAM = NSP + NPP * NP };
  __device__ __forceinline__ static void deriv(const float *y, float *dydx,
                                               const float *p, int np) {
    float refr = p[A_refr];
    float V = (refr > 0.0f) ? p[A_V_reset] : fminf(y[0], p[A_V_peak]);
    float I_syn = 0.0f;
#pragma unroll
    for (int i = 0; i < NP; i++) {
      if (i < np) I_syn += y[NSV + NPV * i] * (p[NSP + NPP * i] - V);
    }
    float V_spike = p[A_Delta_T] * expf((V - p[A_V_th]) / p[A_Delta_T]);
    dydx[0] = (refr > 0.0f) ? 0.0f
        : (-p[A_g_L] * (V - p[A_E_L] - V_spike) + I_syn - y[1] + p[A_I_e])
          / p[A_C_m];
    dydx[1] = (p[A_a] * (V - p[A_E_L]) - y[1]) / p[A_tau_w];
#pragma unroll
    for (int i = 0; i < NP; i++) {
      if (i < np) {
        float g = y[NSV + NPV * i], g1 = y[NSV + NPV * i + 1];
        dydx[NSV + NPV * i + 1] = -g1 / p[NSP + NPP * i + 1];
        dydx[NSV + NPV * i] = g1 - g / p[NSP + NPP * i + 2];
      }
    }
  }
  __device__ __forceinline__ static int external(float *y, float *p, bool end,
                                                 float dt) {
    return aeif_external(y, p, end, dt);
  }
};

template <int NP>
struct AeifCondAlpha {
  enum { NSV = 2, NPV = 2, NSP = A_NSP, NPP = 3,
         NVAR = NSV + NPV * NP, NPARAM = NSP + NPP * NP };
  __device__ __forceinline__ static void deriv(const float *y, float *dydx,
                                               const float *p, int np) {
    float refr = p[A_refr];
    float V = (refr > 0.0f) ? p[A_V_reset] : fminf(y[0], p[A_V_peak]);
    float I_syn = 0.0f;
#pragma unroll
    for (int i = 0; i < NP; i++) {
      if (i < np) I_syn += y[NSV + NPV * i] * (p[NSP + NPP * i] - V);
    }
    float V_spike = p[A_Delta_T] * expf((V - p[A_V_th]) / p[A_Delta_T]);
    dydx[0] = (refr > 0.0f) ? 0.0f
        : (-p[A_g_L] * (V - p[A_E_L] - V_spike) + I_syn - y[1] + p[A_I_e])
          / p[A_C_m];
    dydx[1] = (p[A_a] * (V - p[A_E_L]) - y[1]) / p[A_tau_w];
#pragma unroll
    for (int i = 0; i < NP; i++) {
      if (i < np) {
        float g = y[NSV + NPV * i], g1 = y[NSV + NPV * i + 1];
        float tau = p[NSP + NPP * i + 1];
        dydx[NSV + NPV * i + 1] = -g1 / tau;
        dydx[NSV + NPV * i] = g1 - g / tau;
      }
    }
  }
  __device__ __forceinline__ static int external(float *y, float *p, bool end,
                                                 float dt) {
    return aeif_external(y, p, end, dt);
  }
};

template <int NP>
struct AeifPscAlpha {
  enum { NSV = 2, NPV = 2, NSP = A_NSP, NPP = 2,
         NVAR = NSV + NPV * NP, NPARAM = NSP + NPP * NP };
  __device__ __forceinline__ static void deriv(const float *y, float *dydx,
                                               const float *p, int np) {
    float refr = p[A_refr];
    float V = (refr > 0.0f) ? p[A_V_reset] : fminf(y[0], p[A_V_peak]);
    float I_tot = 0.0f;
#pragma unroll
    for (int i = 0; i < NP; i++) {
      if (i < np) I_tot += y[NSV + NPV * i];
    }
    float V_spike = p[A_Delta_T] == 0.0f ? 0.0f
        : p[A_Delta_T] * expf((V - p[A_V_th]) / p[A_Delta_T]);
    dydx[0] = (refr > 0.0f) ? 0.0f
        : (-p[A_g_L] * (V - p[A_E_L] - V_spike) + I_tot - y[1] + p[A_I_e])
          / p[A_C_m];
    dydx[1] = (p[A_a] * (V - p[A_E_L]) - y[1]) / p[A_tau_w];
#pragma unroll
    for (int i = 0; i < NP; i++) {
      if (i < np) {
        float I = y[NSV + NPV * i], I1 = y[NSV + NPV * i + 1];
        float tau = p[NSP + NPP * i];
        dydx[NSV + NPV * i + 1] = -I1 / tau;
        dydx[NSV + NPV * i] = I1 - I / tau;
      }
    }
  }
  __device__ __forceinline__ static int external(float *y, float *p, bool end,
                                                 float dt) {
    return aeif_external(y, p, end, dt);
  }
};

template <int NP>
struct AeifPscExp {
  enum { NSV = 2, NPV = 1, NSP = A_NSP, NPP = 1,
         NVAR = NSV + NPV * NP, NPARAM = NSP + NPP * NP };
  __device__ __forceinline__ static void deriv(const float *y, float *dydx,
                                               const float *p, int np) {
    float refr = p[A_refr];
    float V = (refr > 0.0f) ? p[A_V_reset] : fminf(y[0], p[A_V_peak]);
    float I_tot = 0.0f;
#pragma unroll
    for (int i = 0; i < NP; i++) {
      if (i < np) I_tot += y[NSV + i];
    }
    float V_spike = p[A_Delta_T] == 0.0f ? 0.0f
        : p[A_Delta_T] * expf((V - p[A_V_th]) / p[A_Delta_T]);
    dydx[0] = (refr > 0.0f) ? 0.0f
        : (-p[A_g_L] * (V - p[A_E_L] - V_spike) + I_tot - y[1] + p[A_I_e])
          / p[A_C_m];
    dydx[1] = (p[A_a] * (V - p[A_E_L]) - y[1]) / p[A_tau_w];
#pragma unroll
    for (int i = 0; i < NP; i++) {
      if (i < np) dydx[NSV + i] = -y[NSV + i] / p[NSP + i];
    }
  }
  __device__ __forceinline__ static int external(float *y, float *p, bool end,
                                                 float dt) {
    return aeif_external(y, p, end, dt);
  }
};

template <int NP>
struct AeifPscDelta {
  enum { NSV = 2, NPV = 0, NSP = A_NSP, NPP = 0, NVAR = 2, NPARAM = A_NSP };
  __device__ __forceinline__ static void deriv(const float *y, float *dydx,
                                               const float *p, int np) {
    float refr = p[A_refr];
    float V = (refr > 0.0f) ? p[A_V_reset] : fminf(y[0], p[A_V_peak]);
    float V_spike = p[A_Delta_T] == 0.0f ? 0.0f
        : p[A_Delta_T] * expf((V - p[A_V_th]) / p[A_Delta_T]);
    dydx[0] = (refr > 0.0f) ? 0.0f
        : (-p[A_g_L] * (V - p[A_E_L] - V_spike) - y[1] + p[A_I_e]) / p[A_C_m];
    dydx[1] = (p[A_a] * (V - p[A_E_L]) - y[1]) / p[A_tau_w];
  }
  __device__ __forceinline__ static int external(float *y, float *p, bool end,
                                                 float dt) {
    return aeif_external(y, p, end, dt);
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
                                               const float *p, int np) {
    float refr = p[I_refr];
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
        dydx[NSV + NPV * i + 1] = -g1 / p[NSP + NPP * i + 1];
        dydx[NSV + NPV * i] = g1 - g / p[NSP + NPP * i + 2];
      }
    }
  }
  __device__ __forceinline__ static int external(float *y, float *p, bool end,
                                                 float dt) {
    float &V_m = y[0];
    float &u = y[1];
    if (V_m < -1.0e3f || u < -1.0e6f || u > 1.0e6f) {
      V_m = p[I_c];
      u = 0.0f;
      return 0;
    }
    if (p[I_refr] > 0.0f) {
      V_m = p[I_c];
      if (end) p[I_refr] -= 1.0f;
      return 0;
    }
    if (V_m >= p[I_V_th]) {
      V_m = p[I_c];
      u += p[I_d];
      float r = (float)(int)roundf(p[I_t_ref] / dt);
      p[I_refr] = r < 0.0f ? 0.0f : r;
      return 1;
    }
    return 0;
  }
};

}  // namespace ngpu
