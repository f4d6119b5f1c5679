// g1_policy.cu -- the policy-fused rollout kernel (g1_policy.cuh) and its
// C-ABI: observation, critic and actor MLPs on tcgen05, sampling, pushes,
// physics substeps, reward, termination and resets in one launch.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>

#include "g1_env.cuh"
#include "g1_host.h"
#include "g1_mlp.cuh"

namespace g1b {
#include "g1_policy.cuh"
}  // namespace g1b

using namespace g1b;

extern "C" {

int g1b_policy_default_params(g1b_task_params* out) {
  if (!out) return fail("policy_default_params: null output");
  g1b_task_params t;
  memset(&t, 0, sizeof(t));
  t.seed = 0;
  t.step0 = 0;
  // velocity command ranges of the policy-fused workload
  const float lo[3] = {-1.0f, -0.5f, -1.0f}, hi[3] = {1.0f, 0.5f, 1.0f};
  for (int i = 0; i < 3; ++i) {
    t.cmd_lo[i] = lo[i];
    t.cmd_hi[i] = hi[i];
  }
  t.cmd_steps_lo = 150;  // reference examples/train.py:297
  t.cmd_steps_hi = 250;
  t.push_steps_lo = 50;  // train.py:259
  t.push_steps_hi = 150;
  const float pv[6] = {0.5f, 0.5f, 0.4f, 0.52f, 0.52f, 0.78f};  // train.py:275-280
  for (int i = 0; i < 6; ++i) t.push_vel[i] = pv[i];
  t.max_episode = 1000;                     // train.py:261
  t.tilt_limit = 70.0f * 3.14159f / 180.0f;  // train.py:215
  t.reset_seed = 42;                        // src/g1sim.py:84 default seed, train.py:293 noise
  t.reset_noise = 0.1f;
  t.reset_drop = 0.02f;
  t.flags = G1B_SAMPLE | G1B_PUSH | G1B_RESET | G1B_COMMANDS;
  *out = t;
  return 0;
}

int g1b_policy_sizes(int* weight_bytes, int* bias_floats, int* obs_dim, int* act_dim) {
  if (weight_bytes) *weight_bytes = (int)PolicyChain::kWeightBytes;
  if (bias_floats) *bias_floats = PolicyChain::kBiasFloats;
  if (obs_dim) *obs_dim = kObs;
  if (act_dim) *act_dim = kNU;
  return 0;
}

int g1b_policy_rollout(int nenv, int npolicy, int decim, const g1b_config* cfg, const g1b_task_params* tp,
                       const g1b_policy* pol, float* qpos, float* qvel, float* anchor, float* ctrl,
                       const float* mu, const float* dmass, const g1b_task_state* ts, const g1b_rollout_out* out,
                       float* foot_pos, float* foot_vel, float* contact_forces, void* stream) {
  if (int rc = check_state(nenv, qpos, qvel, anchor, ctrl)) return rc;
  if (npolicy < 0 || decim <= 0) return fail("policy_rollout: npolicy must be >= 0 and decim positive");
  if (!cfg || !tp || !pol || !ts || !out) return fail("policy_rollout: cfg, params, policy, state, out required");
  if (!pol->weights || !pol->bias || !pol->log_std || !pol->obs_mean || !pol->obs_var)
    return fail("policy_rollout: every policy array is required");
  if ((((uintptr_t)pol->weights) | ((uintptr_t)pol->bias)) & 15)
    return fail("policy_rollout: weights and bias must be 16-byte aligned");
  if (!ts->commands || !ts->prev_action || !ts->cmd_timer || !ts->ep_len || !ts->push_timer)
    return fail("policy_rollout: every task-state array is required");
  if (!foot_pos || !foot_vel || !contact_forces)
    return fail("policy_rollout: foot_pos, foot_vel and contact_forces are required");
  if (tp->cmd_steps_hi <= tp->cmd_steps_lo || tp->push_steps_hi <= tp->push_steps_lo)
    return fail("policy_rollout: timer ranges must be non-empty");
  StateArgs a{nenv, qpos, qvel, anchor, foot_pos, foot_vel, contact_forces, mu, dmass, nullptr, nullptr};
  TaskParams p;
  p.seed = tp->seed;
  p.step0 = tp->step0;
  for (int i = 0; i < 3; ++i) {
    p.cmd_lo[i] = tp->cmd_lo[i];
    p.cmd_hi[i] = tp->cmd_hi[i];
  }
  p.cmd_steps_lo = tp->cmd_steps_lo;
  p.cmd_steps_hi = tp->cmd_steps_hi;
  p.push_steps_lo = tp->push_steps_lo;
  p.push_steps_hi = tp->push_steps_hi;
  for (int i = 0; i < 6; ++i) p.push_vel[i] = tp->push_vel[i];
  p.max_episode = tp->max_episode;
  p.tilt_limit = tp->tilt_limit;
  p.reset_seed = tp->reset_seed;
  p.reset_noise = tp->reset_noise;
  p.reset_drop = tp->reset_drop;
  p.flags = tp->flags;
  PolicyArgs pa{static_cast<const uint8_t*>(pol->weights), pol->bias, pol->log_std, pol->obs_mean, pol->obs_var};
  TaskArgs ta{ts->commands, ts->prev_action, ts->cmd_timer, ts->ep_len, ts->push_timer};
  OutArgs oa{out->obs,  out->actions, out->mean,  out->logp,     out->value,
             out->reward, out->done,  out->reset, out->last_obs, out->last_value};
  return launch<10, kPolicyEnvs>(policy_kernel, 2 * kPolicyEnvs, kPolicySmem, nenv, kPolicyEnvs, 1,
                                 static_cast<cudaStream_t>(stream), "policy_kernel", a, ctrl, npolicy, decim,
                                 to_cfg(cfg), p, pa, ta, oa);
}

int g1b_policy_status(int* code) {
  int v = 0;
  cudaError_t e = cudaMemcpyFromSymbol(&v, g_policy_error, sizeof(int));
  if (e != cudaSuccess) return cuda_fail(e, "policy_status");
  const int zero = 0;
  e = cudaMemcpyToSymbol(g_policy_error, &zero, sizeof(int));
  if (e != cudaSuccess) return cuda_fail(e, "policy_status");
  if (code) *code = v;
  return 0;
}

}  // extern "C"
