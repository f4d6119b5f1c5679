// g1_step.cu -- C-ABI of the plain G1 step (libg1cuda.so): the step and
// rollout entry points, their launch-shape dispatch and autotuner, the
// reference's reset kernel and the FP32 FMA microbenchmark.  The step
// kernels themselves are compiled per launch shape (g1_step_kernels.cuh).
//
//   reset_done_kernel        reference src/g1_kernel.cu:85-103, bit-exact
//   ffma_kernel              FP32 FMA throughput microbenchmark
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "g1_env.cuh"
#include "g1_host.h"
#include "g1_step_launch.h"

namespace g1b {

thread_local char g_err[512] = "";

// ------------------------------------------------------------- reset
// reference src/g1_kernel.cu:85-103: stand keyframe, +drop on z, joint noise
// noise * (2u - 1) from the per-env hash stream, qvel = 0, anchors free.
__global__ void reset_done_kernel(int nenv, float* qpos, float* qvel, float* anchor, const uint8_t* done,
                                  unsigned seed, float noise, float drop) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nenv || !done[e]) return;
  const size_t n = (size_t)nenv;
  unsigned s = hash32(seed ^ (unsigned)(e + 1));
#pragma unroll
  for (int i = 0; i < kNQ; ++i) {
    float v = model().stand[i];
    if (i == 2) v = __fadd_rn(v, drop);
    if (i >= 7) {
      s = hash32(s + 0x9E3779B9u);
      const float u = __uint2float_rn(s) * 2.3283064365386963e-10f;
      const float r = __fsub_rn(__fmul_rn(2.0f, u), 1.0f);
      v = __fmaf_rn(noise, r, v);
    }
    qpos[i * n + e] = v;
  }
#pragma unroll
  for (int i = 0; i < kNV; ++i) qvel[i * n + e] = 0.0f;
#pragma unroll
  for (int i = 0; i < 2 * kNC; ++i) anchor[i * n + e] = kAnchorFree;
}

// ----------------------------------------------------------- FFMA peak
__device__ float g_ffma_sink[1024];
__global__ void __launch_bounds__(256) ffma_kernel(int iters, float a, float b) {
  float x[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) x[k] = (float)(threadIdx.x + k) * 1e-3f;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 16; ++k) x[k] = fmaf(x[k], a, b);
  }
  float s = 0.0f;
#pragma unroll
  for (int k = 0; k < 16; ++k) s += x[k];
  if (s == 1234.5f) g_ffma_sink[blockIdx.x & 1023] = s;  // keeps the chains live
}

// Stand pose, zero velocity, free anchors, stand targets (autotuner state).
__global__ void init_stand_kernel(int nenv, float* qpos, float* qvel, float* anchor, float* ctrl) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nenv) return;
  const size_t n = (size_t)nenv;
  for (int i = 0; i < kNQ; ++i) qpos[i * n + e] = model().stand[i];
  for (int i = 0; i < kNV; ++i) qvel[i * n + e] = 0.0f;
  for (int i = 0; i < 2 * kNC; ++i) anchor[i * n + e] = kAnchorFree;
  for (int i = 0; i < kNU; ++i) ctrl[i * n + e] = model().stand[7 + i];
}

}  // namespace g1b

// =================================================================== host
using namespace g1b;

namespace {

std::mutex g_mu;
int g_mapping = 1;  // two threads per env
int g_block = 128;
int g_blocks_per_sm = 0;

struct LaunchShape {
  int mapping, block, bps;
};
LaunchShape current_shape() {
  std::lock_guard<std::mutex> lk(g_mu);
  return LaunchShape{g_mapping, g_block, g_blocks_per_sm};
}

int dispatch(const LaunchShape& L, bool rollout, const StateArgs& a, float* ctrl, int* rc, int nouter,
             int ninner, const StepConfig& cfg, const RolloutParams& rp, cudaStream_t s) {
  if (L.mapping == 2) {
    if (L.block == 64) return run_split3<64>(rollout, a, ctrl, rc, nouter, ninner, cfg, rp, s, L.bps);
    return run_split3<128>(rollout, a, ctrl, rc, nouter, ninner, cfg, rp, s, L.bps);
  }
  if (L.mapping == 1) {
    switch (L.block) {
      case 32: return run_split<32>(rollout, a, ctrl, rc, nouter, ninner, cfg, rp, s, L.bps);
      case 64: return run_split<64>(rollout, a, ctrl, rc, nouter, ninner, cfg, rp, s, L.bps);
      case 96: return run_split<96>(rollout, a, ctrl, rc, nouter, ninner, cfg, rp, s, L.bps);
      default: return run_split<128>(rollout, a, ctrl, rc, nouter, ninner, cfg, rp, s, L.bps);
    }
  }
  switch (L.block) {
    case 32: return run_single<32>(rollout, a, ctrl, rc, nouter, ninner, cfg, rp, s, L.bps);
    case 64: return run_single<64>(rollout, a, ctrl, rc, nouter, ninner, cfg, rp, s, L.bps);
    case 96: return run_single<96>(rollout, a, ctrl, rc, nouter, ninner, cfg, rp, s, L.bps);
    default: return run_single<128>(rollout, a, ctrl, rc, nouter, ninner, cfg, rp, s, L.bps);
  }
}

int dispatch_step(const StateArgs& a, const float* ctrl, int nsub, const StepConfig& cfg, cudaStream_t s) {
  RolloutParams rp{};
  return dispatch(current_shape(), false, a, const_cast<float*>(ctrl), nullptr, 1, nsub, cfg, rp, s);
}

int dispatch_rollout(const StateArgs& a, float* ctrl, int* rc, int npolicy, int decim, const StepConfig& cfg,
                     const RolloutParams& rp, cudaStream_t s) {
  return dispatch(current_shape(), true, a, ctrl, rc, npolicy, decim, cfg, rp, s);
}

}  // namespace

extern "C" {

const char* g1b_last_error(void) { return g_err; }

int g1b_sizes(int* nb, int* nq, int* nv, int* nu, int* nc) {
  if (nb) *nb = kNB;
  if (nq) *nq = kNQ;
  if (nv) *nv = kNV;
  if (nu) *nu = kNU;
  if (nc) *nc = kNC;
  return 4;
}

int g1b_default_config(g1b_config* out) {
  if (!out) return fail("null config");
  *out = default_cfg();
  return 0;
}

int g1b_step(int nenv, int nsub, const g1b_config* cfg, float* qpos, float* qvel, float* anchor,
             const float* ctrl, const float* mu, const float* dmass, const float* kp_scale,
             const float* kd_scale, float* foot_pos, float* foot_vel, float* contact_forces,
             void* stream) {
  if (int r = check_state(nenv, qpos, qvel, anchor, ctrl)) return r;
  if (nsub < 0) return fail("nsub must be >= 0");
  if (nsub == 0) return 0;
  const g1b_config c = cfg ? *cfg : default_cfg();
  StateArgs a{nenv, qpos, qvel, anchor, foot_pos, foot_vel, contact_forces, mu, dmass, kp_scale, kd_scale};
  return dispatch_step(a, ctrl, nsub, to_cfg(&c), (cudaStream_t)stream);
}

int g1b_rollout(int nenv, int npolicy, int decim, const g1b_config* cfg, const g1b_rollout_params* rp,
                float* qpos, float* qvel, float* anchor, float* ctrl, const float* mu, const float* dmass,
                int* reset_count, float* foot_pos, float* foot_vel, float* contact_forces, void* stream) {
  if (int r = check_state(nenv, qpos, qvel, anchor, ctrl)) return r;
  if (!rp) return fail("null rollout params");
  if (npolicy < 0 || decim < 0) return fail("npolicy and decim must be >= 0");
  if (npolicy == 0 || decim == 0) return 0;
  const g1b_config c = cfg ? *cfg : default_cfg();
  StateArgs a{nenv, qpos, qvel, anchor, foot_pos, foot_vel, contact_forces, mu, dmass, nullptr, nullptr};
  RolloutParams p{rp->seed, rp->step0, rp->target_frac, rp->reset_z, rp->z0_lo, rp->z0_hi, rp->redraw};
  return dispatch_rollout(a, ctrl, reset_count, npolicy, decim, to_cfg(&c), p, (cudaStream_t)stream);
}

// reference src/g1_kernel.cu:154-163; dt fixed at the reference default (1 ms)
void g1_cuda_step(int nenv, int nsub, float* qpos, float* qvel, float* anchor, const float* ctrl,
                  float* foot_pos, float* foot_vel, float* contact_forces, void* stream) {
  const g1b_config c = default_cfg();
  if (check_state(nenv, qpos, qvel, anchor, ctrl) || nsub <= 0) return;
  StateArgs a{nenv, qpos, qvel, anchor, foot_pos, foot_vel, contact_forces, nullptr, nullptr, nullptr, nullptr};
  dispatch_step(a, ctrl, nsub, to_cfg(&c), (cudaStream_t)stream);
}

// reference src/g1_kernel.cu:165-173
void g1_cuda_reset_done(int nenv, float* qpos, float* qvel, float* anchor, const uint8_t* done,
                        unsigned seed, float noise, float drop, void* stream) {
  if (nenv <= 0 || !qpos || !qvel || !anchor || !done) {
    fail("g1_cuda_reset_done: invalid arguments");
    return;
  }
  const int tpb = 128, nb = (nenv + tpb - 1) / tpb;
  reset_done_kernel<<<nb, tpb, 0, (cudaStream_t)stream>>>(nenv, qpos, qvel, anchor, done, seed, noise, drop);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) cuda_fail(e, "reset_done_kernel launch");
}

int g1b_set_launch(int mapping, int block, int blocks_per_sm) {
  if (mapping < 0 || mapping > 2)
    return fail("mapping must be 0 (thread per env), 1 (two threads per env) or 2 (three threads per env)");
  if (block != 32 && block != 64 && block != 96 && block != 128) return fail("block must be 32, 64, 96 or 128");
  if (mapping == 2 && block != 64 && block != 128) return fail("mapping 2 takes block 64 or 128");
  if (blocks_per_sm < 0) return fail("blocks_per_sm must be >= 0");
  std::lock_guard<std::mutex> lk(g_mu);
  g_mapping = mapping;
  g_block = block;
  g_blocks_per_sm = blocks_per_sm;
  return 0;
}

int g1b_get_launch(int* mapping, int* block, int* blocks_per_sm) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (mapping) *mapping = g_mapping;
  if (block) *block = g_block;
  if (blocks_per_sm) *blocks_per_sm = g_blocks_per_sm;
  return 0;
}

int g1b_autotune(int nenv, int nsub, void* stream, float* best_ms) {
  if (nenv <= 0 || nsub <= 0) return fail("autotune: nenv and nsub must be positive");
  cudaStream_t st = (cudaStream_t)stream;
  const size_t n = (size_t)nenv;
  float* buf = nullptr;  // qpos, qvel, anchor, ctrl of a temporary state
  const size_t floats = n * (kNQ + kNV + 2 * kNC + kNU);
  cudaError_t e = cudaMalloc(&buf, floats * sizeof(float));
  if (e != cudaSuccess) return cuda_fail(e, "autotune: cudaMalloc");
  float *qpos = buf, *qvel = qpos + n * kNQ, *anchor = qvel + n * kNV, *ctrl = anchor + n * 2 * kNC;
  StateArgs a{nenv, qpos, qvel, anchor, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  g1b_config c = default_cfg();
  c.dt = 2e-3f;
  const StepConfig cfg = to_cfg(&c);
  RolloutParams rp{};
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int blocks[4] = {32, 64, 96, 128};
  LaunchShape best{1, 128, 0};
  float best_t = 1e30f;
  int rc = 0;
  for (int mapping = 0; mapping < 3 && rc == 0; ++mapping) {
    for (int bi = 0; bi < 4 && rc == 0; ++bi) {
      const LaunchShape L{mapping, blocks[bi], 0};
      if (mapping == 2 && blocks[bi] != 64 && blocks[bi] != 128) continue;
      init_stand_kernel<<<(nenv + 127) / 128, 128, 0, st>>>(nenv, qpos, qvel, anchor, ctrl);
      rc = dispatch(L, false, a, ctrl, nullptr, 1, 1, cfg, rp, st);  // warm-up
      if (rc) break;
      cudaEventRecord(e0, st);
      rc = dispatch(L, false, a, ctrl, nullptr, 1, nsub, cfg, rp, st);
      cudaEventRecord(e1, st);
      if (rc) break;
      e = cudaEventSynchronize(e1);
      if (e != cudaSuccess) {
        rc = cuda_fail(e, "autotune");
        break;
      }
      float t = 0.0f;
      cudaEventElapsedTime(&t, e0, e1);
      if (t < best_t) {
        best_t = t;
        best = L;
      }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(buf);
  if (rc) return rc;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    g_mapping = best.mapping;
    g_block = best.block;
    g_blocks_per_sm = best.bps;
  }
  if (best_ms) *best_ms = best_t;
  return 0;
}

int g1b_ffma_peak(int iters, float* tflops, float* ms) {
  if (iters <= 0 || !tflops) return fail("ffma_peak: invalid arguments");
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  int occ = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, ffma_kernel, 256, 0);
  const int grid = sms * (occ > 0 ? occ : 1);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  ffma_kernel<<<grid, 256>>>(iters / 10 + 1, 1.0000001f, -1e-7f);  // warm-up
  cudaEventRecord(e0);
  ffma_kernel<<<grid, 256>>>(iters, 1.0000001f, -1e-7f);
  cudaEventRecord(e1);
  cudaError_t e = cudaEventSynchronize(e1);
  float t = 0.0f;
  cudaEventElapsedTime(&t, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (e != cudaSuccess) return cuda_fail(e, "ffma_kernel");
  const double flops = 2.0 * 16.0 * (double)iters * (double)grid * 256.0;
  *tflops = (float)(flops / (t * 1e-3) / 1e12);
  if (ms) *ms = t;
  return 0;
}

}  // extern "C"
