// g1_policy.cuh -- the policy-fused rollout kernel (included by g1_policy.cu
// inside namespace g1b, after g1_env.cuh and g1_mlp.cuh).
//
// One CTA owns 128 envs for the whole call (two threads per env, the split
// step's lower/upper-body roles).  Each policy step runs, inside the CTA:
//   observation (reference src/g1sim.py:132-170) -> normalisation
//   (examples/train.py:68-69) -> critic and actor MLPs 99-512-256-128-{1,29}
//   ELU on tcgen05 (BF16 tiles in shared memory, FP32 accumulators in tensor
//   memory, weights streamed from L2) -> Gaussian action sample and log-prob
//   (train.py:85-93) -> PD targets stand + action * scale (train.py:269) ->
//   push (train.py:272-281) -> decim physics substeps -> reward and
//   termination (train.py:143-218) -> timers, resets, command redraws
//   (train.py:285-316).
// The observation tile never leaves the SM: it is built from the state in
// registers and shared memory straight into the first layer's A operand.

// Task tables of the reference training script.
// examples/train.py:244-256 (posture std while walking / running)
__constant__ float c_std_walk[kNU] = {0.3f,  0.15f, 0.15f, 0.35f, 0.25f, 0.1f,  0.3f,  0.15f, 0.15f, 0.35f,
                                      0.25f, 0.1f,  0.2f,  0.08f, 0.1f,  0.15f, 0.15f, 0.1f,  0.15f, 0.3f,
                                      0.3f,  0.3f,  0.15f, 0.15f, 0.1f,  0.15f, 0.3f,  0.3f,  0.3f};
__constant__ float c_std_run[kNU] = {0.5f,  0.2f,  0.2f,  0.6f, 0.35f, 0.15f, 0.5f, 0.2f, 0.2f, 0.6f,
                                     0.35f, 0.15f, 0.3f,  0.08f, 0.2f, 0.5f,  0.2f, 0.15f, 0.35f, 0.3f,
                                     0.3f,  0.3f,  0.5f,  0.2f, 0.15f, 0.35f, 0.3f, 0.3f, 0.3f};
// src/g1sim.py:77-83 (0.25 * effort limit / stiffness per actuator)
__constant__ float c_action_scale[kNU] = {
    0.443200f, 0.274054f, 0.443200f, 0.274054f, 0.365131f, 0.365131f, 0.443200f, 0.274054f,
    0.443200f, 0.274054f, 0.365131f, 0.365131f, 0.443200f, 0.365131f, 0.365131f, 0.365131f,
    0.365131f, 0.365131f, 0.365131f, 0.365131f, 0.074501f, 0.074501f, 0.365131f, 0.365131f,
    0.365131f, 0.365131f, 0.365131f, 0.074501f, 0.074501f};

constexpr int kObs = 99;
constexpr int kObsPad = 112;

// Critic then actor, the layer order of one network pass.
struct PolicyNet {
  static constexpr int kL = 8;
  static constexpr tc::Layer layer[8] = {
      {kObsPad, 512, 16, tc::kElu}, {512, 256, 32, tc::kElu}, {256, 128, 64, tc::kElu}, {128, 16, 128, tc::kNone},
      {kObsPad, 512, 16, tc::kElu}, {512, 256, 32, tc::kElu}, {256, 128, 64, tc::kElu}, {128, 32, 128, tc::kNone}};
};
using PolicyChain = tc::Chain<PolicyNet>;
using PolicyRun = tc::Runner<PolicyNet>;

constexpr int kPolicyEnvs = 128;
constexpr uint32_t kPolicyActOff = (uint32_t)kSlotJointState * kPolicyEnvs * 4;  // after q, qd
constexpr uint32_t kPolicyStageOff = kPolicyActOff + PolicyChain::kActBytes;
// The step scratch, extended where the weight ring reaches past it.
constexpr size_t kPolicyScratch = (size_t)kNumSlots * kPolicyEnvs * sizeof(float);
constexpr size_t kPolicyRingEnd = (size_t)kPolicyStageOff + (size_t)tc::kStages * tc::kStageBytes;
constexpr size_t kPolicySmem = kPolicyScratch > kPolicyRingEnd ? kPolicyScratch : kPolicyRingEnd;
static_assert(kPolicySmem + 4096 <= 232448, "dynamic + static shared memory must fit one CTA");
static_assert((size_t)kNumSlotsSplit * kPolicyEnvs * sizeof(float) <= kPolicySmem,
              "the physics' anchor slots lie inside the allocation");
static_assert(kPolicyActOff % 16 == 0 && kPolicyStageOff % 16 == 0, "operand tiles need 16-byte alignment");

enum : int { kFlagSample = 1, kFlagPush = 2, kFlagReset = 4, kFlagCommands = 8 };

struct TaskParams {
  unsigned seed;
  int step0;
  float cmd_lo[3], cmd_hi[3];
  int cmd_steps_lo, cmd_steps_hi, push_steps_lo, push_steps_hi;
  float push_vel[6];
  int max_episode;
  float tilt_limit;
  unsigned reset_seed;
  float reset_noise, reset_drop;
  int flags;
};
struct PolicyArgs {
  const uint8_t* w;
  const float* b;
  const float* log_std;
  const float* obs_mean;
  const float* obs_var;
};
struct TaskArgs {
  float* cmd;
  float* prev_a;
  int* cmd_timer;
  int* ep_len;
  int* push_timer;
};
struct OutArgs {
  float* obs;
  float* act;
  float* mean;
  float* logp;
  float* value;
  float* reward;
  uint8_t* done;
  uint8_t* reset;
  float* last_obs;
  float* last_value;
};

__device__ int g_policy_error = 0;  // 1: a pipeline wait gave up (the CTA stopped early)

// RNG purposes (seed offsets) of the policy kernel's draws.
enum : unsigned { kRngEps1 = 1, kRngEps2 = 2, kRngPush = 3, kRngCmdReset = 4, kRngCmdTimer = 5, kRngTimers = 6 };
__device__ __forceinline__ float task_u(const TaskParams& tp, unsigned purpose, int e, int stp, int j) {
  return uniform24(tp.seed + purpose * 0x9E3779B9u, (unsigned)e, (unsigned)stp * 64u + (unsigned)j);
}
__device__ __forceinline__ int task_randint(float u, int lo, int hi) {
  const int r = lo + (int)(u * (float)(hi - lo));
  return r < hi ? r : hi - 1;
}

// v rotated by the inverse of unit quaternion q (reference src/g1sim.py:151-154).
__device__ __forceinline__ void quat_rot_inv(const float* q, const float* v, float* o) {
  const float ux = -q[1], uy = -q[2], uz = -q[3];
  const float a0 = __fsub_rn(__fmul_rn(uy, v[2]), __fmul_rn(uz, v[1]));
  const float a1 = __fsub_rn(__fmul_rn(uz, v[0]), __fmul_rn(ux, v[2]));
  const float a2 = __fsub_rn(__fmul_rn(ux, v[1]), __fmul_rn(uy, v[0]));
  const float b0 = __fsub_rn(__fmul_rn(uy, a2), __fmul_rn(uz, a1));
  const float b1 = __fsub_rn(__fmul_rn(uz, a0), __fmul_rn(ux, a2));
  const float b2 = __fsub_rn(__fmul_rn(ux, a1), __fmul_rn(uy, a0));
  o[0] = __fadd_rn(v[0], __fmul_rn(2.0f, __fadd_rn(__fmul_rn(q[0], a0), b0)));
  o[1] = __fadd_rn(v[1], __fmul_rn(2.0f, __fadd_rn(__fmul_rn(q[0], a1), b1)));
  o[2] = __fadd_rn(v[2], __fmul_rn(2.0f, __fadd_rn(__fmul_rn(q[0], a2), b2)));
}

// The 12 base terms of the observation: command, projected gravity, body
// linear velocity, body angular velocity.
__device__ __forceinline__ void obs_base(const EnvState& st, const float* cmd, float* o) {
  const float g[3] = {0.0f, 0.0f, -1.0f};
  o[0] = cmd[0];
  o[1] = cmd[1];
  o[2] = cmd[2];
  quat_rot_inv(st.quat, g, o + 3);
  quat_rot_inv(st.quat, st.vw, o + 6);
  o[9] = st.wb[0];
  o[10] = st.wb[1];
  o[11] = st.wb[2];
}

// Observation column c (12 <= c < 112) from the joint state and the last
// targets: joint position error, joint velocity, last action (= ctrl), pad.
template <class Scr>
__device__ __forceinline__ float obs_joint_col(int c, const Scr& scr, const float* ctrl_e, size_t n) {
  if (c < 41) return __fsub_rn(scr.get(hslot(c - 11, 0)), model().stand[7 + (c - 12)]);
  if (c < 70) return scr.get(hslot(c - 40, 1));
  if (c < kObs) return ctrl_e[(size_t)(c - 70) * n];
  return 0.0f;
}

// Writes columns [8 g0, 8 g1) of this env's observation row: normalised and
// BF16 into the A tile, raw FP32 into raw_row (nullable).  The normalisation
// (reference examples/train.py:68-69) multiplies by the reciprocal standard
// deviation computed once per CTA; norm: [0, 112) mean, [112, 224)
// 1 / sqrt(var + 1e-8), in shared memory.
template <int G0, int G1, class Scr>
__device__ __forceinline__ void build_obs_cols(uint8_t* tile, int row, const float* base12, const Scr& scr,
                                               const float* ctrl_e, size_t n, const float* norm,
                                               float* raw_row) {
#pragma unroll
  for (int g = G0; g < G1; ++g) {
    float v[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int c = 8 * g + i;
      float o = 0.0f;
      if (c < 12)
        o = base12[c < 12 ? c : 0];
      else
        o = obs_joint_col(c, scr, ctrl_e, n);
      if (c < kObs) {
        if (raw_row) raw_row[c] = o;
        const float z = __fmul_rn(__fsub_rn(o, norm[c]), norm[kObsPad + c]);
        v[i] = fminf(fmaxf(z, -5.0f), 5.0f);
      } else {
        v[i] = 0.0f;
      }
    }
    tc::st_row8(tile, row, 8 * g, v);
  }
}

// Reward and termination of one env after a policy step (reference
// examples/train.py:143-218).  o: the 12 base terms of the new
// observation; joint positions from the scratch; foot data of the last
// substep; ar: sum of squared action differences.
template <class Scr>
__device__ float task_reward(const float* o, const Scr& scr, const float* fp, const float* fv, const float* cf,
                             float ar, float tilt_limit, bool& done) {
  const float c0 = o[0], c1 = o[1], c2 = o[2];
  const float lv0 = o[6], lv1 = o[7], lv2 = o[8], av0 = o[9], av1 = o[10], av2 = o[11];
  const float xy = (c0 - lv0) * (c0 - lv0) + (c1 - lv1) * (c1 - lv1);
  const float r_lin = expf(-(xy + lv2 * lv2) / 0.25f);
  const float rp = av0 * av0 + av1 * av1;
  const float r_ang = expf(-((c2 - av2) * (c2 - av2) + rp) / 0.5f);
  const float r_orient = expf(-(o[3] * o[3] + o[4] * o[4]) / 0.2f);
  const float speed = sqrtf(c0 * c0 + c1 * c1) + fabsf(c2);
  const bool standing = speed < 0.05f, running = speed >= 1.5f;
  float pose = 0.0f, lim = 0.0f;
#pragma unroll 1
  for (int j = 0; j < kNU; ++j) {
    const float q = scr.get(hslot(j + 1, 0));
    const float err = q - model().stand[7 + j];
    const float sd = standing ? 0.05f : (running ? c_std_run[j] : c_std_walk[j]);
    pose += err * err / (sd * sd);
    const float lo = model().b[j + 1].lo, hi = model().b[j + 1].hi;
    const float rng = hi - lo;
    lim += fmaxf(q - (hi - 0.05f * rng), 0.0f) + fmaxf((lo + 0.05f * rng) - q, 0.0f);
  }
  const float r_pose = expf(-pose / (float)kNU);
  const float lsq = fv[0] * fv[0] + fv[1] * fv[1], rsq = fv[3] * fv[3] + fv[4] * fv[4];
  const float active = speed > 0.05f ? 1.0f : 0.0f;
  const float clearance =
      (fabsf(fp[2] - 0.1f) * sqrtf(lsq + 1e-6f) + fabsf(fp[5] - 0.1f) * sqrtf(rsq + 1e-6f)) * active;
  const float lc = (cf[0] + cf[1] + cf[2] + cf[3]) > 1.0f ? 1.0f : 0.0f;
  const float rc = (cf[4] + cf[5] + cf[6] + cf[7]) > 1.0f ? 1.0f : 0.0f;
  const float slip = (lsq * lc + rsq * rc) * active;
  const float tilt = fabsf(acosf(fminf(fmaxf(-o[5], -1.0f), 1.0f)));
  done = tilt > tilt_limit;
  return 2.0f * r_lin + 2.0f * r_ang + r_orient + r_pose - lim - 2.0f * clearance - 0.5f * slip - 0.05f * ar -
         0.05f * rp;
}

// Joint angle of reset (reference src/g1_kernel.cu:85-103): the per-env hash
// chain advanced once per joint; returns joints [J0, J1) into the scratch.
template <class Scr>
__device__ void reset_joints(Scr& scr, int e, unsigned seed, float noise, int j0, int j1) {
  unsigned s = hash32(seed ^ (unsigned)(e + 1));
#pragma unroll 1
  for (int j = 0; j < j1; ++j) {
    s = hash32(s + 0x9E3779B9u);
    if (j < j0) continue;
    const float u = __uint2float_rn(s) * 2.3283064365386963e-10f;
    const float r = __fsub_rn(__fmul_rn(2.0f, u), 1.0f);
    scr.put(hslot(j + 1, 0), __fmaf_rn(noise, r, model().stand[7 + j]));
    scr.put(hslot(j + 1, 1), 0.0f);
  }
}

// Sample actions for joints [J0, J1) from the actor output in v (column
// j - C0 of v is joint j), write targets and outputs; returns the partial
// log-probability and accumulates the squared action change.
template <int J0, int J1, int C0>
__device__ __forceinline__ float sample_actions(const float* v, const PolicyArgs& pa, const TaskParams& tp, int e,
                                                int stp, float* ctrl_e, size_t n, const TaskArgs& ta,
                                                float* act_row, float* mean_row, float& ar) {
  constexpr float kHalfLog2Pi = 0.91893853320467274f;
  const float* bias = pa.b + PolicyChain::bias_off(7);
  float lp = 0.0f;
#pragma unroll
  for (int j = J0; j < J1; ++j) {
    const float mu = v[j - C0] + __ldg(bias + j);
    const float ls = __ldg(pa.log_std + j);
    float a = mu, eps = 0.0f;
    if (tp.flags & kFlagSample) {
      const float u1 = 1.0f - task_u(tp, kRngEps1, e, stp, j);  // (0, 1]
      const float u2 = task_u(tp, kRngEps2, e, stp, j);
      eps = sqrtf(-2.0f * logf(u1)) * cospif(2.0f * u2);
      a = mu + expf(ls) * eps;
    }
    lp += -0.5f * eps * eps - ls - kHalfLog2Pi;
    if (act_row) act_row[j] = a;
    if (mean_row) mean_row[j] = mu;
    const float pv = ta.prev_a[(size_t)j * n + e];
    ar += (a - pv) * (a - pv);
    ta.prev_a[(size_t)j * n + e] = a;
    ctrl_e[(size_t)j * n] = __fadd_rn(model().stand[7 + j], __fmul_rn(a, c_action_scale[j]));
  }
  return lp;
}

// Shared state of a policy CTA besides the scratch.
struct PolicyShared {
  uint64_t bars[tc::kBarriers];
  uint32_t tmem;
  int abort;
  float xch[3][kPolicyEnvs];  // 0: logp of the upper joints, 1: their action change, 2: reset flag
  float norm[2 * kObsPad];     // observation mean, reciprocal standard deviation
};

// Observation rows of the CTA's tile into the A tile: role 0 writes columns
// 0-47 (base terms, joint errors, first joint rates), role 1 columns 48-111.
template <class Scr>
__device__ __forceinline__ void policy_obs_tile(uint8_t* tile, int role, int le, bool act_env, const EnvState& st,
                                                const Scr& scr, int e, size_t n, const float* ctrl,
                                                const float* norm, const TaskArgs& ta, float* raw_row) {
  if (act_env) {
    const float* ctrl_e = ctrl + e;
    float base12[12];
    if (role == 0) {
      const float cmd[3] = {ta.cmd[e], ta.cmd[n + e], ta.cmd[2 * n + e]};
      obs_base(st, cmd, base12);
      build_obs_cols<0, 6>(tile, le, base12, scr, ctrl_e, n, norm, raw_row);
    } else {
#pragma unroll
      for (int i = 0; i < 12; ++i) base12[i] = 0.0f;
      build_obs_cols<6, kObsPad / 8>(tile, le, base12, scr, ctrl_e, n, norm, raw_row);
    }
  } else {
    const float z[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int g = role == 0 ? 0 : 6; g < (role == 0 ? 6 : kObsPad / 8); ++g) tc::st_row8(tile, le, 8 * g, z);
  }
}

// Closes a layer for every thread: publish the tile, CTA barrier that also
// ORs the threads' failed-wait flags (so every thread leaves together).
// Returns false when the CTA must stop.
__device__ __forceinline__ bool policy_layer_done(PolicyShared& ps, bool ok) {
  tc::tile_written();
  if (__syncthreads_or(ok ? 0 : 1) == 0) return true;
  if (threadIdx.x == 0) {
    ps.abort = 1;
    atomicExch(&g_policy_error, 1);
  }
  return false;
}

// Hidden layer L of the pass: MMAs, then bias + ELU into the next A tile.
template <int L>
__device__ __forceinline__ bool policy_hidden(tc::Pipe& p, PolicyShared& ps, uint8_t* tile, const PolicyArgs& pa) {
  bool ok = PolicyRun::issue<L>(p, pa.w);
  ok = PolicyRun::wait_acc(p, pa.w) && ok;
  PolicyRun::epilogue<L, 2 * kPolicyEnvs>(p, tile, pa.b + PolicyChain::bias_off(L));
  return policy_layer_done(ps, ok);
}

// Copy nrows rows of `width` floats from shared staging to contiguous global
// rows, consecutive threads on consecutive floats (coalesced).
__device__ __forceinline__ void copy_rows(float* dst, const float* src, int nrows, int width) {
  const int total = nrows * width;
  for (int i = threadIdx.x; i < total; i += 2 * kPolicyEnvs) dst[i] = src[i];
}

// Shared staging of the raw observation rows [128][99] inside the activation
// region, past the observation tile (28,672 bytes).
constexpr uint32_t kRawObsOff = kPolicyActOff + 32768;
static_assert(32768 >= kObsPad / 8 * (kPolicyEnvs / 8) * 128, "observation tile below the raw staging");
static_assert(32768 + kPolicyEnvs * kObs * 4 <= PolicyChain::kActBytes, "raw staging inside the region");

// One network pass (critic, then actor) for the CTA's tile; every thread
// calls it.  Role 0 threads hold the base state.  raw_dst (nullable): global
// rows of this tile's raw observation (nrows of them), written once through
// shared staging.  value: the critic output (role 0); out32: actor pre-bias
// outputs, columns 0-15 (both roles) and 16-31 (role 1).  Returns false when
// the CTA must stop (a wait gave up).
template <class Scr>
__device__ bool policy_pass(tc::Pipe& p, PolicyShared& ps, uint8_t* smraw, int role, int le, bool act_env,
                            const EnvState& st, const Scr& scr, int e, size_t n, const float* ctrl,
                            const PolicyArgs& pa, const TaskArgs& ta, float* raw_dst, int nrows, float& value,
                            float (&out32)[32]) {
  uint8_t* tile = smraw + kPolicyActOff;
  float* raw_sm = reinterpret_cast<float*>(smraw + kRawObsOff);
  const uint32_t lane = p.tmem + ((uint32_t)((threadIdx.x >> 5) & 3) * 32u << 16);
  bool ok = PolicyRun::begin(p, pa.w);
  // critic
  policy_obs_tile(tile, role, le, act_env, st, scr, e, n, ctrl, ps.norm, ta, raw_dst ? raw_sm + le * kObs : nullptr);
  if (!policy_layer_done(ps, ok)) return false;
  ok = PolicyRun::issue<0>(p, pa.w);
  if (raw_dst) copy_rows(raw_dst, raw_sm, nrows, kObs);  // block-uniform; runs under the MMAs
  ok = PolicyRun::wait_acc(p, pa.w) && ok;
  if (raw_dst) __syncthreads();  // the epilogue below overwrites the staging
  PolicyRun::epilogue<0, 2 * kPolicyEnvs>(p, tile, pa.b + PolicyChain::bias_off(0));
  if (!policy_layer_done(ps, ok)) return false;
  if (!policy_hidden<1>(p, ps, tile, pa) || !policy_hidden<2>(p, ps, tile, pa)) return false;
  ok = PolicyRun::issue<3>(p, pa.w);
  ok = PolicyRun::wait_acc(p, pa.w) && ok;
  if (role == 0) {
    float v[16];
    tc::tmem_ld16(lane, v);
    value = v[0] + __ldg(pa.b + PolicyChain::bias_off(3));
  }
  if (!policy_layer_done(ps, ok)) return false;
  // actor (the observation tile is rebuilt: the hidden layers overwrote it)
  policy_obs_tile(tile, role, le, act_env, st, scr, e, n, ctrl, ps.norm, ta, nullptr);
  if (!policy_layer_done(ps, true)) return false;
  if (!policy_hidden<4>(p, ps, tile, pa) || !policy_hidden<5>(p, ps, tile, pa) || !policy_hidden<6>(p, ps, tile, pa))
    return false;
  ok = PolicyRun::issue<7>(p, pa.w);
  ok = PolicyRun::wait_acc(p, pa.w) && ok;
  {
    float v[16];
    tc::tmem_ld16(lane, v);
#pragma unroll
    for (int i = 0; i < 16; ++i) out32[i] = v[i];
    if (role == 1) {
      tc::tmem_ld16(lane + 16, v);
#pragma unroll
      for (int i = 0; i < 16; ++i) out32[16 + i] = v[i];
    }
  }
  return policy_layer_done(ps, ok);
}

// decim substeps of the two-role split step for one env (role 0: legs,
// pelvis, base; role 1: waist and arms), the arithmetic of split_kernel with
// its single call sites of the chain routines (bwd_role, fwd_role).  Kept out
// of line so that the physics has its own register allocation: the network
// and task state live around it is saved once per policy step instead of
// competing with every substep for the 255 registers.  Returns the base
// state (role 0; role 1's copy is the one it read).
__device__ __noinline__ EnvState policy_substeps(int role, bool act, EnvState st, EnvIO io, EnvParams ep,
                                                 StepConfig cfg, float* col, int decim) {
  SmemScratch<kPolicyEnvs> scr{col};
  // the contacts' anchors on chip for these substeps (the network phase's
  // weight ring holds their slots in between): loaded here, stored at the end
  float* const gan = io.anchor;
  const size_t gsd = io.astride;
  if (act && role == 0) {
    float* an = scr.p + kXAnchor * kPolicyEnvs;
#pragma unroll
    for (int i = 0; i < 2 * kNC; ++i) an[i * kPolicyEnvs] = gan[i * gsd];
    io.anchor = an;
    io.astride = kPolicyEnvs;
  }
  for (int s = 0; s < decim; ++s) {
    const bool last_sub = s == decim - 1;
    AI acc0;
    SV accP0;
    EnvState su;  // role 1: the base state at the start of the substep
    if (act) {
      if (role == 0) {
        fk_lower(st, io, ep, cfg, scr, last_sub);
      } else {
        load_base(scr, su);
        fk_upper(su, cfg, scr);
      }
      bwd_role(role, role == 0 ? st : su, io, ep, cfg, scr, acc0, accP0);
      if (role == 1) store_ai(scr, kXUp, acc0, accP0);
    }
    __syncthreads();
    SV a0;
    if (act && role == 0) {
      AI up;
      SV upP;
      load_ai(scr, kXUp, up, upP);
      ai_add(acc0, up);
      sv_acc(accP0, upP);
      a0 = base_solve(acc0, accP0);
      store_sv(scr, kXA0, a0);
    }
    __syncthreads();
    if (act) {
      if (role == 1) {
        a0 = load_sv(scr, kXA0);
        st = su;
      }
      fwd_role(role, st, a0, cfg, scr);
      if (role == 0) store_base(scr, st);
    }
    __syncthreads();
  }
  if (act && role == 0) {
#pragma unroll
    for (int i = 0; i < 2 * kNC; ++i) gan[i * gsd] = io.anchor[i * kPolicyEnvs];
  }
  return st;
}

__global__ void __launch_bounds__(2 * kPolicyEnvs, 1)
    policy_kernel(StateArgs a, float* ctrl, int npolicy, int decim, StepConfig cfg, TaskParams tp, PolicyArgs pa,
                  TaskArgs ta, OutArgs out) {
  extern __shared__ __align__(128) uint8_t smraw[];
  __shared__ PolicyShared ps;
  constexpr int ENVS = kPolicyEnvs;
  const int role = threadIdx.x >= ENVS ? 1 : 0;
  const int le = threadIdx.x - role * ENVS;
  SmemScratch<ENVS> scr{reinterpret_cast<float*>(smraw) + le};
  const int n = a.nenv;
  const size_t sd = (size_t)n;

  tc::Pipe p;
  p.act = tc::smem_u32(smraw + kPolicyActOff);
  p.stage = tc::smem_u32(smraw + kPolicyStageOff);
  p.bar = tc::smem_u32(ps.bars);
  tc::pipe_init(p);
  if (threadIdx.x == 0) ps.abort = 0;
  if (threadIdx.x < kObsPad) {
    const int c = threadIdx.x;
    ps.norm[c] = c < kObs ? __ldg(pa.obs_mean + c) : 0.0f;
    ps.norm[kObsPad + c] = c < kObs ? __fdiv_rn(1.0f, sqrtf(__fadd_rn(__ldg(pa.obs_var + c), 1e-8f))) : 0.0f;
  }
  if (threadIdx.x < 32) tc::tmem_alloc(tc::smem_u32(&ps.tmem), tc::kTmemCols);
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  p.tmem = ps.tmem;

  const int ntiles = (n + ENVS - 1) / ENVS;
  bool stop = false;
  for (int tile = blockIdx.x; tile < ntiles && !stop; tile += gridDim.x) {
    const int e = tile * ENVS + le;
    const bool act = e < n;
    EnvState st;
    EnvIO io;
    EnvParams ep;
    if (act) {
      io = env_io(a, ctrl, e);
      ep = load_params(a, e);
      if (role == 0) {
#pragma unroll
        for (int k = 0; k < 3; ++k) st.pos[k] = a.qpos[k * sd + e];
#pragma unroll
        for (int k = 0; k < 4; ++k) st.quat[k] = a.qpos[(3 + k) * sd + e];
#pragma unroll
        for (int k = 0; k < 3; ++k) st.vw[k] = a.qvel[k * sd + e];
#pragma unroll
        for (int k = 0; k < 3; ++k) st.wb[k] = a.qvel[(3 + k) * sd + e];
        load_joints(a.qpos + e, a.qvel + e, sd, scr, 1, 12);
      } else {
        load_joints(a.qpos + e, a.qvel + e, sd, scr, 13, kNJ);
      }
    }
    __syncthreads();
    for (int k = 0; k <= npolicy; ++k) {
      const bool final_eval = k == npolicy;
      if (final_eval && !out.last_obs && !out.last_value) break;
      const int stp = tp.step0 + k;
      const size_t row = final_eval ? (size_t)e : (size_t)k * sd + (size_t)e;
      float value = 0.0f;
      float v32[32];
      const size_t e0 = (size_t)tile * ENVS;
      const int nrows = n - (int)e0 < ENVS ? n - (int)e0 : ENVS;
      const size_t row0 = final_eval ? e0 : (size_t)k * sd + e0;  // first output row of the tile
      float* raw_dst = final_eval ? (out.last_obs ? out.last_obs + e0 * kObs : nullptr)
                                  : (out.obs ? out.obs + row0 * kObs : nullptr);
      if (!policy_pass(p, ps, smraw, role, le, act, st, scr, e, sd, ctrl, pa, ta, raw_dst, nrows, value, v32)) {
        stop = true;
        break;
      }
      if (final_eval) {
        if (act && role == 0 && out.last_value) out.last_value[e] = value;
        break;
      }
      // ---- action, log-probability, targets, push
      float lp = 0.0f, ar = 0.0f;
      // action and mean rows staged in shared memory, copied out coalesced
      float* act_sm = reinterpret_cast<float*>(smraw + kPolicyActOff);
      float* mean_sm = act_sm + ENVS * kNU;
      if (act) {
        float* act_row = out.act ? act_sm + le * kNU : nullptr;
        float* mean_row = out.mean ? mean_sm + le * kNU : nullptr;
        if (role == 0) {
          lp = sample_actions<0, 12, 0>(v32, pa, tp, e, stp, ctrl + e, sd, ta, act_row, mean_row, ar);
          if (out.value) out.value[row] = value;
          if (tp.flags & kFlagPush) {
            int pt = ta.push_timer[e] - 1;
            if (pt <= 0) {
#pragma unroll
              for (int i = 0; i < 6; ++i) {
                const float pv = tp.push_vel[i];
                const float dv = __fsub_rn(__fmul_rn(task_u(tp, kRngPush, e, stp, i), 2.0f * pv), pv);
                if (i < 3)
                  st.vw[i] = __fadd_rn(st.vw[i], dv);
                else
                  st.wb[i - 3] = __fadd_rn(st.wb[i - 3], dv);
              }
              pt = task_randint(task_u(tp, kRngPush, e, stp, 6), tp.push_steps_lo, tp.push_steps_hi);
            }
            ta.push_timer[e] = pt;
          }
          store_base(scr, st);
        } else {
          lp = sample_actions<12, kNU, 0>(v32, pa, tp, e, stp, ctrl + e, sd, ta, act_row, mean_row, ar);
          ps.xch[0][le] = lp;
          ps.xch[1][le] = ar;
        }
      }
      __syncthreads();
      if (act && role == 0) {
        ar += ps.xch[1][le];
        if (out.logp) out.logp[row] = lp + ps.xch[0][le];
      }
      if (out.act || out.mean) {  // block-uniform
        if (out.act) copy_rows(out.act + row0 * kNU, act_sm, nrows, kNU);
        if (out.mean) copy_rows(out.mean + row0 * kNU, mean_sm, nrows, kNU);
        __syncthreads();  // the substeps reuse the staging
      }
      // ---- physics: decim substeps of the split step
      st = policy_substeps(role, act, st, io, ep, cfg, reinterpret_cast<float*>(smraw) + le, decim);
      // ---- reward, termination, timers, reset, command redraw
      if (act && role == 0) {
        float cmd[3] = {ta.cmd[e], ta.cmd[sd + e], ta.cmd[2 * sd + e]};
        float o[12];
        obs_base(st, cmd, o);
        float fp[6], fv[6], cf[8];
#pragma unroll
        for (int i = 0; i < 6; ++i) {
          fp[i] = io.foot_pos[i * sd];
          fv[i] = io.foot_vel[i * sd];
        }
#pragma unroll
        for (int i = 0; i < 8; ++i) cf[i] = io.cf[i * sd];
        bool done = false;
        const float r = task_reward(o, scr, fp, fv, cf, ar, tp.tilt_limit, done);
        int el = ta.ep_len[e] + 1;
        int ct = ta.cmd_timer[e] - 1;
        const bool rs = (tp.flags & kFlagReset) && (done || el >= tp.max_episode);
        if (rs) {
#pragma unroll
          for (int i = 0; i < 3; ++i) st.pos[i] = model().stand[i];
          st.pos[2] = __fadd_rn(st.pos[2], tp.reset_drop);
#pragma unroll
          for (int i = 0; i < 4; ++i) st.quat[i] = model().stand[3 + i];
#pragma unroll
          for (int i = 0; i < 3; ++i) st.vw[i] = st.wb[i] = 0.0f;
          reset_joints(scr, e, tp.reset_seed, tp.reset_noise, 0, 12);
#pragma unroll
          for (int i = 0; i < 2 * kNC; ++i) a.anchor[(size_t)i * sd + e] = kAnchorFree;
#pragma unroll 1
          for (int j = 0; j < 12; ++j) ta.prev_a[(size_t)j * sd + e] = 0.0f;
          el = 0;
          ta.push_timer[e] = task_randint(task_u(tp, kRngTimers, e, stp, 0), tp.push_steps_lo, tp.push_steps_hi);
          if (tp.flags & kFlagCommands) {
#pragma unroll
            for (int i = 0; i < 3; ++i)
              cmd[i] = __fadd_rn(tp.cmd_lo[i],
                                 __fmul_rn(task_u(tp, kRngCmdReset, e, stp, i), __fsub_rn(tp.cmd_hi[i], tp.cmd_lo[i])));
            ct = task_randint(task_u(tp, kRngCmdReset, e, stp, 3), tp.cmd_steps_lo, tp.cmd_steps_hi);
          }
          store_base(scr, st);
        }
        if ((tp.flags & kFlagCommands) && ct <= 0) {
#pragma unroll
          for (int i = 0; i < 3; ++i)
            cmd[i] = __fadd_rn(tp.cmd_lo[i],
                               __fmul_rn(task_u(tp, kRngCmdTimer, e, stp, i), __fsub_rn(tp.cmd_hi[i], tp.cmd_lo[i])));
          ct = task_randint(task_u(tp, kRngCmdTimer, e, stp, 3), tp.cmd_steps_lo, tp.cmd_steps_hi);
        }
        if (tp.flags & kFlagCommands) {
#pragma unroll
          for (int i = 0; i < 3; ++i) ta.cmd[i * sd + e] = cmd[i];
        }
        ta.ep_len[e] = el;
        ta.cmd_timer[e] = ct;
        if (out.reward) out.reward[row] = r;
        if (out.done) out.done[row] = done ? 1 : 0;
        if (out.reset) out.reset[row] = rs ? 1 : 0;
        ps.xch[2][le] = rs ? 1.0f : 0.0f;
      }
      __syncthreads();
      if (act && role == 1 && ps.xch[2][le] != 0.0f) {
        reset_joints(scr, e, tp.reset_seed, tp.reset_noise, 12, kNJ);
#pragma unroll 1
        for (int j = 12; j < kNU; ++j) ta.prev_a[(size_t)j * sd + e] = 0.0f;
      }
      __syncthreads();
    }
    if (stop) break;
    if (act) {
      if (role == 0) {
#pragma unroll
        for (int k = 0; k < 3; ++k) a.qpos[k * sd + e] = st.pos[k];
#pragma unroll
        for (int k = 0; k < 4; ++k) a.qpos[(3 + k) * sd + e] = st.quat[k];
#pragma unroll
        for (int k = 0; k < 3; ++k) a.qvel[k * sd + e] = st.vw[k];
#pragma unroll
        for (int k = 0; k < 3; ++k) a.qvel[(3 + k) * sd + e] = st.wb[k];
        store_joints(a.qpos + e, a.qvel + e, sd, scr, 1, 12);
      } else {
        store_joints(a.qpos + e, a.qvel + e, sd, scr, 13, kNJ);
      }
    }
    __syncthreads();  // the next tile reuses the scratch
    if (stop) break;
  }
  __syncthreads();
  if (stop) PolicyRun::drain(p);
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  if (threadIdx.x < 32) tc::tmem_dealloc(p.tmem, tc::kTmemCols);
}
