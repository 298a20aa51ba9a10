// Training and inference kernels of the learned RK5 step proposer
// (6 -> 32 -> 32 -> 1 MLP, ReLU hidden layers, linear output).
//
// Training runs in FP32 on the CUDA cores with hand-written forward and
// backward passes: k_mlp_grad evaluates one mini-batch block of 64 samples
// (each thread one sample, activations and deltas staged in shared memory)
// and writes that block's gradient sums; k_mlp_reduce_adam reduces the blocks
// in a fixed order (deterministic) and applies one Adam step to the FP32
// master parameters. Loss: mean squared error of log2(h / dt).
//
// Inference for the RK5 kernels is the tensor-core path of
// ngpu_step_proposer.cuh; k_mlp_infer runs it stand-alone on given feature
// rows so that it can be checked against a CPU evaluation.
#include <math.h>
#include <stdint.h>
#include <string.h>
#include <algorithm>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>
#include "ngpu_kernels.h"
#include "ngpu_rng.h"
#include "ngpu_step_proposer.cuh"

namespace ngpu {

#define MLP_TB 64           // samples per training block
#define MLP_NP NGPU_MLP_NPARAM

__global__ void __launch_bounds__(MLP_TB)
k_mlp_grad(const float *__restrict__ data, int n, const float *__restrict__ P,
           unsigned long long seed, long long step, int sequential,
           float *__restrict__ partials) {
  __shared__ float sx[MLP_TB][7];
  __shared__ float sh1[MLP_TB][33];
  __shared__ float sh2[MLP_TB][33];
  __shared__ float sd1[MLP_TB][33];
  __shared__ float sd2[MLP_TB][33];
  __shared__ float sdo[MLP_TB];
  __shared__ float sl[MLP_TB];
  __shared__ float sP[MLP_NP];
  const int t = threadIdx.x;
  for (int k = t; k < MLP_NP; k += MLP_TB) sP[k] = P[k];
  __syncthreads();
  const long long gi = (long long)blockIdx.x * MLP_TB + t;
  bool valid;
  long long idx;
  if (sequential) {
    valid = gi < n;
    idx = valid ? gi : 0;
  } else {
    Philox4 r = ng_random_block(seed, RNG_TAG_MLP, (unsigned long long)gi,
                                (unsigned long long)step, 0);
    idx = (long long)((((unsigned long long)r.v[0] << 32) | r.v[1]) % (unsigned long long)n);
    valid = true;
  }
  float x[6];
#pragma unroll
  for (int f = 0; f < 6; f++) x[f] = data[idx * 8 + f];
  const float target = data[idx * 8 + 6];
  float z1[32], z2[32];
#pragma unroll
  for (int j = 0; j < 32; j++) {
    float a = sP[MLP_B1 + j];
#pragma unroll
    for (int f = 0; f < 6; f++) a = fmaf(sP[MLP_W1 + j * 6 + f], x[f], a);
    z1[j] = a;
  }
  float o = sP[MLP_B3];
#pragma unroll 4
  for (int j = 0; j < 32; j++) {
    float a = sP[MLP_B2 + j];
#pragma unroll
    for (int i = 0; i < 32; i++) a = fmaf(sP[MLP_W2 + j * 32 + i], fmaxf(z1[i], 0.0f), a);
    z2[j] = a;
    o = fmaf(sP[MLP_W3 + j], fmaxf(a, 0.0f), o);
  }
  const float e = o - target;
  const float d_o = valid ? 2.0f * e : 0.0f;
  float dz2[32];
#pragma unroll
  for (int j = 0; j < 32; j++) dz2[j] = (z2[j] > 0.0f) ? d_o * sP[MLP_W3 + j] : 0.0f;
#pragma unroll 4
  for (int i = 0; i < 32; i++) {
    float a = 0.0f;
#pragma unroll
    for (int j = 0; j < 32; j++) a = fmaf(sP[MLP_W2 + j * 32 + i], dz2[j], a);
    sd1[t][i] = (z1[i] > 0.0f) ? a : 0.0f;
  }
#pragma unroll
  for (int f = 0; f < 6; f++) sx[t][f] = x[f];
#pragma unroll
  for (int j = 0; j < 32; j++) {
    sh1[t][j] = fmaxf(z1[j], 0.0f);
    sh2[t][j] = fmaxf(z2[j], 0.0f);
    sd2[t][j] = dz2[j];
  }
  sdo[t] = d_o;
  sl[t] = valid ? e * e : 0.0f;
  __syncthreads();
  float *out = partials + (size_t)blockIdx.x * (MLP_NP + 1);
  for (int k = t; k < MLP_NP; k += MLP_TB) {
    float acc = 0.0f;
    if (k < MLP_B1) {
      const int j = k / 6, f = k % 6;
      for (int b = 0; b < MLP_TB; b++) acc = fmaf(sd1[b][j], sx[b][f], acc);
    } else if (k < MLP_W2) {
      const int j = k - MLP_B1;
      for (int b = 0; b < MLP_TB; b++) acc += sd1[b][j];
    } else if (k < MLP_B2) {
      const int j = (k - MLP_W2) / 32, i = (k - MLP_W2) % 32;
      for (int b = 0; b < MLP_TB; b++) acc = fmaf(sd2[b][j], sh1[b][i], acc);
    } else if (k < MLP_W3) {
      const int j = k - MLP_B2;
      for (int b = 0; b < MLP_TB; b++) acc += sd2[b][j];
    } else if (k < MLP_B3) {
      const int j = k - MLP_W3;
      for (int b = 0; b < MLP_TB; b++) acc = fmaf(sdo[b], sh2[b][j], acc);
    } else {
      for (int b = 0; b < MLP_TB; b++) acc += sdo[b];
    }
    out[k] = acc;
  }
  if (t == 0) {
    float l = 0.0f;
    for (int b = 0; b < MLP_TB; b++) l += sl[b];
    out[MLP_NP] = l;
  }
}

// fixed-order reduction of the block sums; Adam step when m != null,
// otherwise the mean gradient is written to grad
__global__ void k_mlp_reduce_adam(const float *__restrict__ partials, int nblk, float inv_batch,
                                  float *P, float *m, float *v, float *grad, int t, float lr,
                                  float *loss_out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k > MLP_NP) return;
  double s = 0.0;
  for (int b = 0; b < nblk; b++) s += (double)partials[(size_t)b * (MLP_NP + 1) + k];
  const float g = (float)(s * (double)inv_batch);
  if (k == MLP_NP) {
    if (loss_out) *loss_out = g;
    return;
  }
  if (grad) grad[k] = g;
  if (m) {
    const float b1 = 0.9f, b2 = 0.999f, eps = 1.0e-8f;
    const float mk = b1 * m[k] + (1.0f - b1) * g;
    const float vk = b2 * v[k] + (1.0f - b2) * g * g;
    m[k] = mk;
    v[k] = vk;
    const float mh = mk / (1.0f - powf(b1, (float)t));
    const float vh = vk / (1.0f - powf(b2, (float)t));
    P[k] -= lr * mh / (sqrtf(vh) + eps);
  }
}

__global__ void __launch_bounds__(128, 1)
k_mlp_infer(const float *__restrict__ x6, int n, const MlpImage *img, float *out,
            unsigned *err) {
  __shared__ ProposerSmem ps;
  const int i = blockIdx.x * 128 + threadIdx.x;
  const bool want = i < n;
  float f[6] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
  if (want) {
#pragma unroll
    for (int k = 0; k < 6; k++) f[k] = x6[(size_t)i * 6 + k];
  }
  proposer_alloc(ps);
  proposer_stage_weights(ps, img);
  float o = 0.0f;
  const bool ok = proposer_round(ps, want, f, o, err);
  if (want) out[i] = ok ? o : __int_as_float(0x7fc00000);
  proposer_teardown(ps, !ok);
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
static void check(cudaError_t e, const char *what) {
  if (e != cudaSuccess)
    throw std::runtime_error(std::string("CUDA error in ") + what + ": " + cudaGetErrorString(e));
}

static uint16_t to_bf16(float f) {
  uint32_t u;
  memcpy(&u, &f, 4);
  // round to nearest even on the 16 dropped bits
  const uint32_t r = u + 0x7FFFu + ((u >> 16) & 1u);
  return (uint16_t)(r >> 16);
}

void MlpBuildImage(const float *P, MlpImage *img) {
  memset(img, 0, sizeof(MlpImage));
  uint8_t *w1 = reinterpret_cast<uint8_t *>(img->w1);
  uint8_t *w2 = reinterpret_cast<uint8_t *>(img->w2);
  for (int nn = 0; nn < 32; nn++) {
    for (int k = 0; k < 16; k++) {
      float v = 0.0f;
      if (k < 6) v = P[MLP_W1 + nn * 6 + k];
      else if (k == 6) v = P[MLP_B1 + nn];
      const uint16_t b = to_bf16(v);
      memcpy(w1 + umma_kmajor_off(nn, k, 16), &b, 2);
    }
    for (int k = 0; k < 32; k++) {
      const uint16_t b = to_bf16(P[MLP_W2 + nn * 32 + k]);
      memcpy(w2 + umma_kmajor_off(nn, k, 32), &b, 2);
    }
    img->b2[nn] = P[MLP_B2 + nn];
    img->w3[nn] = P[MLP_W3 + nn];
  }
  img->b3 = P[MLP_B3];
}

void MlpInitParams(float *P, unsigned long long seed, float b3) {
  std::mt19937_64 gen(seed ^ 0x5DEECE66DULL);
  std::normal_distribution<float> nd(0.0f, 1.0f);
  for (int k = 0; k < MLP_NP; k++) P[k] = 0.0f;
  const float s1 = sqrtf(2.0f / 6.0f), s2 = sqrtf(2.0f / 32.0f), s3 = sqrtf(1.0f / 32.0f);
  for (int k = 0; k < 192; k++) P[MLP_W1 + k] = s1 * nd(gen);
  for (int k = 0; k < 1024; k++) P[MLP_W2 + k] = s2 * nd(gen);
  for (int k = 0; k < 32; k++) P[MLP_W3 + k] = s3 * nd(gen);
  P[MLP_B3] = b3;
}

float MlpGradients(const float *d_data, int n, const float *P_host, float *grad_host,
                   cudaStream_t s) {
  const int nblk = (n + MLP_TB - 1) / MLP_TB;
  float *d_P = nullptr, *d_part = nullptr, *d_grad = nullptr, *d_loss = nullptr;
  check(cudaMalloc(&d_P, sizeof(float) * MLP_NP), "MlpGradients");
  check(cudaMalloc(&d_part, sizeof(float) * (size_t)nblk * (MLP_NP + 1)), "MlpGradients");
  check(cudaMalloc(&d_grad, sizeof(float) * MLP_NP), "MlpGradients");
  check(cudaMalloc(&d_loss, sizeof(float)), "MlpGradients");
  check(cudaMemcpyAsync(d_P, P_host, sizeof(float) * MLP_NP, cudaMemcpyHostToDevice, s),
        "MlpGradients");
  k_mlp_grad<<<nblk, MLP_TB, 0, s>>>(d_data, n, d_P, 0ULL, 0, 1, d_part);
  k_mlp_reduce_adam<<<(MLP_NP + 1 + 255) / 256, 256, 0, s>>>(
      d_part, nblk, 1.0f / (float)n, nullptr, nullptr, nullptr, d_grad, 0, 0.0f, d_loss);
  float loss = 0.0f;
  check(cudaMemcpyAsync(grad_host, d_grad, sizeof(float) * MLP_NP, cudaMemcpyDeviceToHost, s),
        "MlpGradients");
  check(cudaMemcpyAsync(&loss, d_loss, sizeof(float), cudaMemcpyDeviceToHost, s), "MlpGradients");
  check(cudaStreamSynchronize(s), "MlpGradients");
  cudaFree(d_P);
  cudaFree(d_part);
  cudaFree(d_grad);
  cudaFree(d_loss);
  return loss;
}

void MlpTrain(const float *d_data, int n, float *P_host, int steps, int blocks, float lr,
              unsigned long long seed, float *loss_first, float *loss_last, cudaStream_t s) {
  if (n <= 0 || steps <= 0) throw std::runtime_error("no training samples or steps");
  float *d_P, *d_m, *d_v, *d_part, *d_loss;
  check(cudaMalloc(&d_P, sizeof(float) * MLP_NP), "MlpTrain");
  check(cudaMalloc(&d_m, sizeof(float) * MLP_NP), "MlpTrain");
  check(cudaMalloc(&d_v, sizeof(float) * MLP_NP), "MlpTrain");
  check(cudaMalloc(&d_part, sizeof(float) * (size_t)blocks * (MLP_NP + 1)), "MlpTrain");
  check(cudaMalloc(&d_loss, sizeof(float) * steps), "MlpTrain");
  check(cudaMemcpyAsync(d_P, P_host, sizeof(float) * MLP_NP, cudaMemcpyHostToDevice, s), "MlpTrain");
  check(cudaMemsetAsync(d_m, 0, sizeof(float) * MLP_NP, s), "MlpTrain");
  check(cudaMemsetAsync(d_v, 0, sizeof(float) * MLP_NP, s), "MlpTrain");
  const float inv = 1.0f / (float)(blocks * MLP_TB);
  for (int t = 1; t <= steps; t++) {
    // constant rate, then a tenth of it for the last fifth of the steps
    const float lr_t = (t > (steps * 4) / 5) ? 0.1f * lr : lr;
    k_mlp_grad<<<blocks, MLP_TB, 0, s>>>(d_data, n, d_P, seed, t, 0, d_part);
    k_mlp_reduce_adam<<<(MLP_NP + 1 + 255) / 256, 256, 0, s>>>(d_part, blocks, inv, d_P, d_m,
                                                              d_v, nullptr, t, lr_t,
                                                              d_loss + (t - 1));
  }
  check(cudaGetLastError(), "MlpTrain launch");
  std::vector<float> losses(steps);
  check(cudaMemcpyAsync(P_host, d_P, sizeof(float) * MLP_NP, cudaMemcpyDeviceToHost, s), "MlpTrain");
  check(cudaMemcpyAsync(losses.data(), d_loss, sizeof(float) * steps, cudaMemcpyDeviceToHost, s),
        "MlpTrain");
  check(cudaStreamSynchronize(s), "MlpTrain");
  // average over the first and the last 5% of the steps
  const int w = std::max(1, steps / 20);
  double a = 0.0, b = 0.0;
  for (int k = 0; k < w; k++) {
    a += losses[k];
    b += losses[steps - 1 - k];
  }
  *loss_first = (float)(a / w);
  *loss_last = (float)(b / w);
  cudaFree(d_P);
  cudaFree(d_m);
  cudaFree(d_v);
  cudaFree(d_part);
  cudaFree(d_loss);
}

void MlpInfer(const float *d_x6, int n, const MlpImage *d_img, float *d_out, unsigned *d_err,
              cudaStream_t s) {
  if (n <= 0) return;
  k_mlp_infer<<<(n + 127) / 128, 128, 0, s>>>(d_x6, n, d_img, d_out, d_err);
}

}  // namespace ngpu
