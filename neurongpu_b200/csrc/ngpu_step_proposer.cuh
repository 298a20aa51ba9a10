// Learned RK5 step proposer: a 6 -> 32 -> 32 -> 1 MLP that proposes the next
// RK5 step size of a neuron from its state (V, w, conductances) and its
// previous step size. The RK5 embedded error estimate still accepts or
// rejects every step (src/rk5.h:57-147), so the plain controller remains the
// fallback; the proposer only replaces the controller's initial guess of a
// sub-step when that guess is shorter than the rest of the time step.
//
// Inference runs on the 5th-generation tensor cores, one CTA of 128 neurons
// at a time: each thread writes its neuron's features as one BF16 row of a
// 128 x 16 operand tile in shared memory; one thread issues tcgen05.mma
// (kind::f16, BF16 inputs, FP32 accumulation in tensor memory) for the two
// hidden layers; every thread reads its own row back with tcgen05.ld (TMEM
// lane = neuron), applies bias and ReLU, and forms the scalar output with 32
// FMAs. The layer-1 bias is folded into the MMA as weight column 6 against a
// constant-one feature.
//
// Shared-memory operand tiles use the UMMA canonical K-major layout without
// swizzle: 8 x 16-byte core matrices (8 rows x 8 BF16), consecutive K chunks
// LBO = 128 bytes apart, consecutive 8-row groups SBO = 16 * K bytes apart.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "ngpu_device.h"
#include "ngpu_rk5_models.cuh"

namespace ngpu {

// ---------------------------------------------------------------------------
// features (model specific); the same function feeds logging and inference
// ---------------------------------------------------------------------------
template <class M>
struct ProposerFeatures {
  static constexpr bool supported = false;
  __device__ __forceinline__ static void get(const float *, const float *, float, float,
                                             float *) {}
};

// AdEx with conductance ports (beta and alpha synapses): V relative to the
// spike threshold in units of Delta_T, adaptation current, the decaying and
// the rising conductances of ports 0 and 1, and log2 of the previous step.
__device__ __forceinline__ void aeif_cond_features(const float *y, const float *p, int nports,
                                                   float h_prev, float dt, float *f) {
  const float dT = fmaxf(p[A_Delta_T], 0.5f);
  f[0] = fminf(fmaxf((y[0] - p[A_V_th]) / dT, -20.0f), 20.0f) * 0.1f;
  f[1] = y[1] * 0.01f;
  const float g_ex = y[2], g1_ex = y[3];
  const float g_in = nports > 1 ? y[4] : 0.0f, g1_in = nports > 1 ? y[5] : 0.0f;
  f[2] = log1pf(fmaxf(g_ex, 0.0f));
  f[3] = log1pf(fmaxf(g_in, 0.0f));
  f[4] = log1pf(fmaxf(g1_ex, 0.0f) + fmaxf(g1_in, 0.0f));
  f[5] = log2f(fmaxf(h_prev, 1.0e-12f) / dt) * 0.1f;
}

template <int NP>
struct ProposerFeatures<AeifCondBeta<NP>> {
  static constexpr bool supported = true;
  __device__ __forceinline__ static void get(const float *y, const float *p, float h_prev,
                                             float dt, float *f) {
    aeif_cond_features(y, p, NP, h_prev, dt, f);
  }
};
template <int NP>
struct ProposerFeatures<AeifCondAlpha<NP>> {
  static constexpr bool supported = true;
  __device__ __forceinline__ static void get(const float *y, const float *p, float h_prev,
                                             float dt, float *f) {
    aeif_cond_features(y, p, NP, h_prev, dt, f);
  }
};

// training target of an accepted sub-step: log2 of the step the plain
// controller estimates for the state it started from (0.9 h err^-1/5, at
// most 5 h; src/rk5.h:120-140), capped at the time step
__device__ __forceinline__ float proposer_target(float h_acc, float err, float dt) {
  float h_opt = (err > 1.889568e-4f) ? 0.9f * h_acc * exp2f(-0.2f * log2f(err)) : 5.0f * h_acc;
  h_opt = fminf(h_opt, dt);
  return fmaxf(log2f(h_opt / dt), -14.0f);
}

// ---------------------------------------------------------------------------
// tcgen05 / mbarrier helpers (inline PTX, sm_100a)
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// UMMA shared-memory descriptor, K-major, no swizzle (layout type 0),
// descriptor version 1, base offset 0
__device__ __forceinline__ uint64_t umma_desc_kmajor(uint32_t saddr, uint32_t lbo,
                                                     uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1u << 46;
  return d;
}

// instruction descriptor: D f32, A and B bf16, both K-major, M = 128, N = 32
constexpr uint32_t kMlpIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((32u >> 3) << 17) |
                               ((128u >> 4) << 24);

__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc,
                                          uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
      :
      : "r"(d_tmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void umma_commit(uint64_t *mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
               :
               : "r"(smem_u32(mbar))
               : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t *mbar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" : : "r"(smem_u32(mbar)), "r"(count)
               : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" : : : "memory");
}

// Bounded wait for the completion of the barrier phase with the given
// parity; false if it did not complete within max_iter tries. give_up: the
// wait's limit is reached at once (the wait-test hook of GroupArgs), with the
// operation it waits for still in flight, so that the time-out path runs
// deterministically (a single test could see a fast operation complete).
__device__ __forceinline__ bool mbar_wait(uint64_t *mbar, uint32_t parity, int max_iter,
                                          bool give_up = false) {
  const uint32_t a = smem_u32(mbar);
  if (give_up) return false;
  for (int k = 0; k < max_iter; k++) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void tmem_alloc32(uint32_t *dst_smem) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 32;"
               :
               : "r"(smem_u32(dst_smem))
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" : : : "memory");
}

__device__ __forceinline__ void tmem_dealloc32(uint32_t taddr) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 32;" : : "r"(taddr)
               : "memory");
}

__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" : : : "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" : : : "memory");
}
__device__ __forceinline__ void proxy_fence_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" : : : "memory");
}

// 32 consecutive FP32 columns of this thread's TMEM lane
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float *r) {
  uint32_t v[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
        "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]),
        "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]),
        "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]),
        "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]),
        "=r"(v[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" : : : "memory");
#pragma unroll
  for (int j = 0; j < 32; j++) r[j] = __uint_as_float(v[j]);
}

__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
  // round to nearest even; the first source operand goes to the upper half
  uint32_t r;
  asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(hi), "f"(lo));
  return r;
}

// byte offset of element (row, k) in a K-major no-swizzle tile with K columns
__host__ __device__ __forceinline__ uint32_t umma_kmajor_off(int row, int k, int K) {
  return (uint32_t)((row >> 3) * (16 * K) + (k >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2);
}

// ---------------------------------------------------------------------------
// per-CTA state of the proposer (static shared memory of the learned kernels)
// ---------------------------------------------------------------------------
struct __align__(1024) ProposerSmem {
  uint8_t a[128 * 16 * 2];      // features, 128 rows x K 16 (bf16)
  uint8_t hid[128 * 32 * 2];    // hidden layer 1, 128 rows x K 32 (bf16)
  uint8_t w1[32 * 16 * 2];      // B of layer 1: N 32 x K 16 (bias in column 6)
  uint8_t w2[32 * 32 * 2];      // B of layer 2: N 32 x K 32
  float b2[32];
  float w3[32];
  float b3;
  uint32_t tmem;                // TMEM base address of the 32 accumulator columns
  uint64_t mbar;
  uint32_t phase;               // parity of the barrier phase to wait for next
};

// Allocates the CTA's 32 TMEM columns (warp 0) and initialises the completion
// barrier; called by every thread at kernel start. The allocation is made
// and its permit relinquished up front in every CTA: a CTA that still holds
// the allocation permit would keep further CTAs of the kernel from starting
// on its SM.
__device__ __forceinline__ void proposer_alloc(ProposerSmem &s) {
  const int tid = threadIdx.x;
  if (tid == 0) {
    s.phase = 0;
    mbar_init(&s.mbar, 1);
  }
  // K columns 8..15 of the feature tile stay zero
  if (tid < 128) {
    *reinterpret_cast<uint4 *>(s.a + umma_kmajor_off(tid, 8, 16)) = make_uint4(0, 0, 0, 0);
  }
  if ((tid >> 5) == 0) tmem_alloc32(&s.tmem);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
}

// Stages the weights in shared memory (every thread; CTA-uniform branch,
// before the first proposal round of the launch).
__device__ __forceinline__ void proposer_stage_weights(ProposerSmem &s, const MlpImage *img) {
  const int tid = threadIdx.x;
  const uint32_t *src1 = img->w1;
  const uint32_t *src2 = img->w2;
  uint32_t *d1 = reinterpret_cast<uint32_t *>(s.w1);
  uint32_t *d2 = reinterpret_cast<uint32_t *>(s.w2);
  for (int k = tid; k < 32 * 16 / 2; k += blockDim.x) d1[k] = src1[k];
  for (int k = tid; k < 32 * 32 / 2; k += blockDim.x) d2[k] = src2[k];
  if (tid < 32) {
    s.b2[tid] = img->b2[tid];
    s.w3[tid] = img->w3[tid];
  }
  if (tid == 0) s.b3 = img->b3;
  proxy_fence_async_smem();
  __syncthreads();
}

// One proposal round for the whole CTA: every thread with want != 0 passes
// its features f[0..5]; out receives the network output (log2 of the
// proposed step over dt) for this thread's row. Must be called by all
// threads; returns false (CTA-uniformly) if a completion wait timed out.
// wait_test: WaitTest bits of the test hook (0 in normal runs).
__device__ __forceinline__ bool proposer_round(ProposerSmem &s, bool want, const float *f,
                                               float &out, unsigned *err_flags,
                                               int wait_test = 0) {
  const int tid = threadIdx.x;
  const int warp = tid >> 5;
  if (want) {
    uint4 v;
    v.x = pack_bf16x2(f[0], f[1]);
    v.y = pack_bf16x2(f[2], f[3]);
    v.z = pack_bf16x2(f[4], f[5]);
    v.w = pack_bf16x2(1.0f, 0.0f);          // constant-one feature carries the bias
    *reinterpret_cast<uint4 *>(s.a + umma_kmajor_off(tid, 0, 16)) = v;
  }
  proxy_fence_async_smem();
  tc_fence_before();
  __syncthreads();
  const uint32_t taddr = s.tmem;
  if (tid == 0) {
    tc_fence_after();
    umma_bf16(taddr, umma_desc_kmajor(smem_u32(s.a), 128, 256),
              umma_desc_kmajor(smem_u32(s.w1), 128, 256), kMlpIdesc, 0u);
    umma_commit(&s.mbar);
  }
  const uint32_t ph0 = s.phase;
  bool ok = __all_sync(0xffffffffu, mbar_wait(&s.mbar, ph0, NGPU_WAIT_ITERS,
                                             (wait_test & WAIT_TEST_FIRST) != 0));
  tc_fence_after();
  float r[32];
  const uint32_t lane_addr = taddr + ((uint32_t)(warp * 32) << 16);
  if (ok) {
    tmem_ld32(lane_addr, r);
#pragma unroll
    for (int c = 0; c < 4; c++) {
      uint4 v;
      v.x = pack_bf16x2(fmaxf(r[8 * c + 0], 0.0f), fmaxf(r[8 * c + 1], 0.0f));
      v.y = pack_bf16x2(fmaxf(r[8 * c + 2], 0.0f), fmaxf(r[8 * c + 3], 0.0f));
      v.z = pack_bf16x2(fmaxf(r[8 * c + 4], 0.0f), fmaxf(r[8 * c + 5], 0.0f));
      v.w = pack_bf16x2(fmaxf(r[8 * c + 6], 0.0f), fmaxf(r[8 * c + 7], 0.0f));
      *reinterpret_cast<uint4 *>(s.hid + umma_kmajor_off(tid, 8 * c, 32)) = v;
    }
  }
  proxy_fence_async_smem();
  tc_fence_before();
  const int ok1 = __syncthreads_and(ok);
  if (!ok1) {
    if (tid == 0) {
      atomicOr(err_flags, (unsigned)DERR_PROPOSER_TIMEOUT);
      s.phase = proposer_phase_after(ph0, false, false);
    }
    __syncthreads();
    return false;
  }
  if (tid == 0) {
    tc_fence_after();
    umma_bf16(taddr, umma_desc_kmajor(smem_u32(s.hid), 128, 512),
              umma_desc_kmajor(smem_u32(s.w2), 128, 512), kMlpIdesc, 0u);
    umma_bf16(taddr, umma_desc_kmajor(smem_u32(s.hid) + 256, 128, 512),
              umma_desc_kmajor(smem_u32(s.w2) + 256, 128, 512), kMlpIdesc, 1u);
    umma_commit(&s.mbar);
  }
  ok = __all_sync(0xffffffffu, mbar_wait(&s.mbar, ph0 ^ 1u, NGPU_WAIT_ITERS,
                                        (wait_test & WAIT_TEST_SECOND) != 0));
  tc_fence_after();
  float o = s.b3;
  if (ok) {
    tmem_ld32(lane_addr, r);
#pragma unroll
    for (int j = 0; j < 32; j++) o = fmaf(s.w3[j], fmaxf(r[j] + s.b2[j], 0.0f), o);
  }
  tc_fence_before();
  const int ok2 = __syncthreads_and(ok);
  if (tid == 0) s.phase = proposer_phase_after(ph0, true, ok2 != 0);
  if (!ok2) {
    if (tid == 0) atomicOr(err_flags, (unsigned)DERR_PROPOSER_TIMEOUT);
    __syncthreads();
    return false;
  }
  out = o;
  return true;
}

// Releases the CTA's tensor memory (all threads; warp 0 deallocates). After
// a timed-out wait the tensor-core work may still be in flight: wait for the
// outstanding completion (bounded) before the columns are released.
__device__ __forceinline__ void proposer_teardown(ProposerSmem &s, bool failed) {
  if (failed) mbar_wait(&s.mbar, s.phase, NGPU_WAIT_ITERS);
  tc_fence_before();
  __syncthreads();
  if ((threadIdx.x >> 5) == 0) {
    tc_fence_after();
    tmem_dealloc32(s.tmem);
  }
}

}  // namespace ngpu
