// g1_env.cuh -- per-env plumbing shared by the step, policy and adjoint
// kernels: the slot-major shared-memory scratch, the SoA state arguments,
// per-env parameters, the counter-based RNG and the target redraw.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "g1_phys.cuh"

namespace g1b {

// ------------------------------------------------------------ scratch
// Slot-major per-thread scratch: p[slot * BLOCK].  Every phase of the step
// writes and reads it at run-time slot indices from separate loops, so the
// values are not forwarded into long-lived registers.
template <int BLOCK>
struct SmemScratch {
  float* p;
  template <int K>
  __host__ __device__ __forceinline__ float get() const { return p[K * BLOCK]; }
  template <int K>
  __host__ __device__ __forceinline__ void put(float v) { p[K * BLOCK] = v; }
  __host__ __device__ __forceinline__ float get(int k) const { return p[k * BLOCK]; }
  __host__ __device__ __forceinline__ void put(int k, float v) { p[k * BLOCK] = v; }
};

template <int BLOCK>
constexpr size_t smem_bytes() { return (size_t)kNumSlotsSingle * BLOCK * sizeof(float); }
template <int ENVS>
constexpr size_t smem_bytes_split() { return (size_t)kNumSlotsSplit * ENVS * sizeof(float); }

struct StateArgs {
  int nenv;
  float* qpos;
  float* qvel;
  float* anchor;
  float* foot_pos;
  float* foot_vel;
  float* cf;
  const float* mu;
  const float* dmass;
  const float* kp_scale;
  const float* kd_scale;
};

template <class Scr>
__device__ __forceinline__ void load_state(const StateArgs& a, int e, EnvState& st, Scr& scr) {
  const size_t n = (size_t)a.nenv;
#pragma unroll
  for (int k = 0; k < 3; ++k) st.pos[k] = a.qpos[k * n + e];
#pragma unroll
  for (int k = 0; k < 4; ++k) st.quat[k] = a.qpos[(3 + k) * n + e];
#pragma unroll
  for (int k = 0; k < 3; ++k) st.vw[k] = a.qvel[k * n + e];
#pragma unroll
  for (int k = 0; k < 3; ++k) st.wb[k] = a.qvel[(3 + k) * n + e];
  load_joints(a.qpos + e, a.qvel + e, n, scr);
}

template <class Scr>
__device__ __forceinline__ void store_state(const StateArgs& a, int e, const EnvState& st, Scr& scr) {
  const size_t n = (size_t)a.nenv;
#pragma unroll
  for (int k = 0; k < 3; ++k) a.qpos[k * n + e] = st.pos[k];
#pragma unroll
  for (int k = 0; k < 4; ++k) a.qpos[(3 + k) * n + e] = st.quat[k];
#pragma unroll
  for (int k = 0; k < 3; ++k) a.qvel[k * n + e] = st.vw[k];
#pragma unroll
  for (int k = 0; k < 3; ++k) a.qvel[(3 + k) * n + e] = st.wb[k];
  store_joints(a.qpos + e, a.qvel + e, n, scr);
}

// The env's in-memory arrays (ctrl, anchors, outputs), offset to env e.
__device__ __forceinline__ EnvIO env_io(const StateArgs& a, const float* ctrl, int e) {
  EnvIO io;
  io.ctrl = ctrl + e;
  io.anchor = a.anchor + e;
  io.foot_pos = a.foot_pos ? a.foot_pos + e : nullptr;
  io.foot_vel = a.foot_vel ? a.foot_vel + e : nullptr;
  io.cf = a.cf ? a.cf + e : nullptr;
  io.stride = (size_t)a.nenv;
  io.astride = (size_t)a.nenv;
  return io;
}

__device__ __forceinline__ EnvParams load_params(const StateArgs& a, int e) {
  EnvParams ep;
  constexpr float mu0 = (float)g1m_contact_mu;
  ep.mu = a.mu ? __ldg(a.mu + e) : mu0;
  ep.dmass = a.dmass ? __ldg(a.dmass + e) : 0.0f;
  ep.kp_scale = a.kp_scale ? __ldg(a.kp_scale + e) : 1.0f;
  ep.kd_scale = a.kd_scale ? __ldg(a.kd_scale + e) : 1.0f;
  return ep;
}

// ------------------------------------------------------------- RNG
// 32-bit xorshift-multiply integer hash ("lowbias32", C. Wellons), the same
// function as the reference's g1_hash (src/g1_kernel.cu:54-58).
__host__ __device__ __forceinline__ unsigned hash32(unsigned x) {
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}
// Counter-based uniform in [0, 1) with 24 random bits (exact in float).
__device__ __forceinline__ float uniform24(unsigned seed, unsigned stream, unsigned counter) {
  unsigned h = hash32(seed ^ hash32(stream * 0x9E3779B9u + 0x7F4A7C15u));
  h = hash32(h ^ (counter * 0x85EBCA6Bu + 0xC2B2AE35u));
  return __uint2float_rn(h >> 8) * (1.0f / 16777216.0f);
}

struct RolloutParams {
  unsigned seed;
  int step0;
  float target_frac, reset_z, z0_lo, z0_hi;
  int redraw;
};

// targets = stand + (2u - 1) * frac * (hi - lo), one rounding per operation
template <int J>
__device__ __forceinline__ float draw_target(unsigned seed, int e, int step, float frac) {
  const float u = uniform24(seed, (unsigned)e, (unsigned)step * 64u + (unsigned)J);
  const float r = __fsub_rn(__fmul_rn(2.0f, u), 1.0f);
  constexpr float lo = (float)g1m_jnt_range[2 * J], hi = (float)g1m_jnt_range[2 * J + 1];
  constexpr float stand = (float)g1m_qpos_stand[7 + J];
  const float span = __fmul_rn(frac, __fsub_rn(hi, lo));
  return __fadd_rn(stand, __fmul_rn(r, span));
}
// writes the env's targets of joints J..J1-1 into its ctrl column (read back
// by the substeps)
template <int J, int J1 = kNU>
__device__ __forceinline__ void draw_targets(float* ct, size_t stride, unsigned seed, int e, int step,
                                             float frac) {
  ct[J * stride] = draw_target<J>(seed, e, step, frac);
  if constexpr (J + 1 < J1) draw_targets<J + 1, J1>(ct, stride, seed, e, step, frac);
}

// Base height of a reset env, U[z0_lo, z0_hi] from the env's reset stream.
__device__ __forceinline__ float reset_height(const RolloutParams& rp, int e, int stp) {
  const float u = uniform24(rp.seed ^ 0x5bd1e995u, (unsigned)e, (unsigned)stp);
  return __fadd_rn(rp.z0_lo, __fmul_rn(u, __fsub_rn(rp.z0_hi, rp.z0_lo)));
}

}  // namespace g1b
