// g1_step_kernels.cuh -- the plain step kernels and their launchers, one
// launch shape (BLOCK envs per CTA) per including translation unit
// (g1_step_k{32,64,96,128}.cu), so that the instances compile in parallel.
//
//   step_kernel<BLOCK>       one thread per env, nsub substeps of g1b::step;
//                            state loaded from SoA once, stored once
//                            (reference src/g1_kernel.cu:106-151)
//   rollout_kernel<BLOCK>    npolicy x (target redraw, decim substeps, reset
//                            check) per env, all in one launch
//   split_kernel<ENVS, R>    two threads per env (lower / upper body)
#pragma once
#include "g1_env.cuh"
#include "g1_host.h"
#include "g1_step_launch.h"

namespace g1b {

// --------------------------------------------------------------- step
// --------------------------------------------------------------- step
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) step_kernel(StateArgs a, const float* __restrict__ ctrl,
                                                     int nsub, StepConfig cfg) {
  extern __shared__ float sm[];
  SmemScratch<BLOCK> scr{sm + threadIdx.x};
  const int n = a.nenv;
  for (int e = blockIdx.x * BLOCK + threadIdx.x; e < n; e += gridDim.x * BLOCK) {
    EnvState st;
    load_state(a, e, st, scr);
    const EnvIO io = env_io(a, ctrl, e);
    const EnvParams ep = load_params(a, e);
    for (int s = 0; s < nsub; ++s) step(st, io, ep, cfg, scr, s == nsub - 1);
    store_state(a, e, st, scr);
  }
}

template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) rollout_kernel(StateArgs a, float* ctrl,
                                                        int* __restrict__ reset_count, int npolicy,
                                                        int decim, StepConfig cfg, RolloutParams rp) {
  extern __shared__ float sm[];
  SmemScratch<BLOCK> scr{sm + threadIdx.x};
  const int n = a.nenv;
  for (int e = blockIdx.x * BLOCK + threadIdx.x; e < n; e += gridDim.x * BLOCK) {
    EnvState st;
    load_state(a, e, st, scr);
    const EnvIO io = env_io(a, ctrl, e);
    const EnvParams ep = load_params(a, e);
    int resets = 0;
    for (int k = 0; k < npolicy; ++k) {
      const int stp = rp.step0 + k;
      if (rp.redraw) draw_targets<0>(ctrl + e, (size_t)n, rp.seed, e, stp, rp.target_frac);
      for (int s = 0; s < decim; ++s) step(st, io, ep, cfg, scr, k == npolicy - 1 && s == decim - 1);
      if (st.pos[2] < rp.reset_z) {
        const float z0 = reset_height(rp, e, stp);
#pragma unroll
        for (int i = 0; i < 3; ++i) st.pos[i] = model().stand[i];
        st.pos[2] = z0;
#pragma unroll
        for (int i = 0; i < 4; ++i) st.quat[i] = model().stand[3 + i];
#pragma unroll 1
        for (int i = 0; i < kNJ; ++i) {
          scr.put(hslot(i + 1, 0), model().stand[7 + i]);
          scr.put(hslot(i + 1, 1), 0.0f);
        }
#pragma unroll
        for (int i = 0; i < 3; ++i) st.vw[i] = st.wb[i] = 0.0f;
#pragma unroll
        for (int i = 0; i < 2 * kNC; ++i) a.anchor[(size_t)i * n + e] = kAnchorFree;
        ++resets;
      }
    }
    store_state(a, e, st, scr);
    if (reset_count) reset_count[e] += resets;
  }
}

// ------------------------------------------------------- split mapping
// Two threads per env: threads [0, ENVS) run the lower body (pelvis, legs,
// contacts, base solve and base integration), threads [ENVS, 2 ENVS) the
// upper body (waist, arms) of env tile * ENVS + (tid % ENVS).  The two roles
// run the backward and forward passes through shared call sites (bwd_role,
// fwd_role), so one compiled copy of the chain routines serves both.  Both halves
// use the env's slot column of the shared scratch and exchange, per
// substep, the upper body's projection into the pelvis, the base
// acceleration and the base state (three block barriers).  kRollout: the
// decimated rollout (target redraw, reset); otherwise ninner substeps.
template <int ENVS, bool kRollout>
__global__ void __launch_bounds__(2 * ENVS) split_kernel(StateArgs a, float* ctrl, int* reset_count,
                                                         int nouter, int ninner, StepConfig cfg,
                                                         RolloutParams rp) {
  extern __shared__ float sm[];
  const int role = threadIdx.x >= ENVS ? 1 : 0;  // warp-uniform (ENVS is a multiple of 32)
  const int le = threadIdx.x - role * ENVS;
  SmemScratch<ENVS> scr{sm + le};
  const int n = a.nenv;
  const size_t sd = (size_t)n;
  const int ntiles = (n + ENVS - 1) / ENVS;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
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
        store_base(scr, st);
        // the contacts (this role) use the anchors on chip for the whole tile
        float* an = scr.p + kXAnchor * ENVS;
#pragma unroll
        for (int i = 0; i < 2 * kNC; ++i) an[i * ENVS] = a.anchor[(size_t)i * sd + e];
        io.anchor = an;
        io.astride = ENVS;
      } else {
        load_joints(a.qpos + e, a.qvel + e, sd, scr, 13, kNJ);
      }
    }
    __syncthreads();
    int resets = 0;
    for (int k = 0; k < nouter; ++k) {
      const int stp = rp.step0 + k;
      if (kRollout && act && rp.redraw) {
        if (role == 0)
          draw_targets<0, 12>(ctrl + e, sd, rp.seed, e, stp, rp.target_frac);
        else
          draw_targets<12, kNU>(ctrl + e, sd, rp.seed, e, stp, rp.target_frac);
      }
      for (int s = 0; s < ninner; ++s) {
        const bool last_sub = (k == nouter - 1) && (s == ninner - 1);
        AI acc0;
        SV accP0;
        EnvState su;  // upper half: base state at the start of the substep
        if (act) {
          if (role == 0) {
            fk_lower(st, io, ep, cfg, scr, last_sub);
          } else {
            load_base(scr, su);
            fk_upper(su, cfg, scr);
          }
          // one call site for both roles (one copy of the chain routines)
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
            st = su;  // the upper role's copy of the base state (not integrated by it)
          }
          fwd_role(role, st, a0, cfg, scr);
          if (role == 0) store_base(scr, st);
        }
        __syncthreads();
      }
      if (kRollout) {
        if (act && role == 0) {
          const bool rs = st.pos[2] < rp.reset_z;
          if (rs) {
            const float z0 = reset_height(rp, e, stp);
#pragma unroll
            for (int i = 0; i < 3; ++i) st.pos[i] = model().stand[i];
            st.pos[2] = z0;
#pragma unroll
            for (int i = 0; i < 4; ++i) st.quat[i] = model().stand[3 + i];
#pragma unroll
            for (int i = 0; i < 3; ++i) st.vw[i] = st.wb[i] = 0.0f;
#pragma unroll 1
            for (int i = 1; i <= 12; ++i) {
              scr.put(hslot(i, 0), model().stand[6 + i]);
              scr.put(hslot(i, 1), 0.0f);
            }
#pragma unroll
            for (int i = 0; i < 2 * kNC; ++i) io.anchor[i * io.astride] = kAnchorFree;
            store_base(scr, st);
            ++resets;
          }
          scr.put(kXReset, rs ? 1.0f : 0.0f);
        }
        __syncthreads();
        if (act && role == 1 && scr.get(kXReset) != 0.0f) {
#pragma unroll 1
          for (int i = 13; i <= kNJ; ++i) {
            scr.put(hslot(i, 0), model().stand[6 + i]);
            scr.put(hslot(i, 1), 0.0f);
          }
        }
      }
    }
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
#pragma unroll
        for (int i = 0; i < 2 * kNC; ++i) a.anchor[(size_t)i * sd + e] = io.anchor[i * ENVS];
        if (kRollout && reset_count) reset_count[e] += resets;
      } else {
        store_joints(a.qpos + e, a.qvel + e, sd, scr, 13, kNJ);
      }
    }
    __syncthreads();  // the next tile reuses the scratch
  }
}


// ----------------------------------------------- three-role mapping
// Three threads per env: threads [0, ENVS) run the left leg, its contacts,
// the pelvis, the base solve and the base integration; [ENVS, 2 ENVS) the
// right leg and its contacts; [2 ENVS, 3 ENVS) the waist and the arms.  The
// legs' code is shared by two roles, and the critical path of a substep is
// the upper body's 17 hinges instead of the lower body's 12 hinges plus
// eight contacts.  Exchanged through the scratch per substep: the right
// leg's and the upper body's projections into the pelvis, the base
// acceleration and the base state (three block barriers, as the two-role
// kernel).  The arithmetic is that of split_kernel, operation for operation.
template <int ENVS, bool kRollout>
__global__ void __launch_bounds__(3 * ENVS) split3_kernel(StateArgs a, float* ctrl, int* reset_count,
                                                          int nouter, int ninner, StepConfig cfg,
                                                          RolloutParams rp) {
  extern __shared__ float sm[];
  const int role = threadIdx.x / ENVS;  // warp-uniform (ENVS is a multiple of 32)
  const int le = threadIdx.x - role * ENVS;
  SmemScratch<ENVS> scr{sm + le};
  const int n = a.nenv;
  const size_t sd = (size_t)n;
  const int ntiles = (n + ENVS - 1) / ENVS;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
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
        load_joints(a.qpos + e, a.qvel + e, sd, scr, 1, 6);
        store_base(scr, st);
      } else if (role == 1) {
        load_joints(a.qpos + e, a.qvel + e, sd, scr, 7, 12);
      } else {
        load_joints(a.qpos + e, a.qvel + e, sd, scr, 13, kNJ);
      }
    }
    __syncthreads();
    int resets = 0;
    for (int k = 0; k < nouter; ++k) {
      const int stp = rp.step0 + k;
      if (kRollout && act && rp.redraw) {
        if (role == 0)
          draw_targets<0, 6>(ctrl + e, sd, rp.seed, e, stp, rp.target_frac);
        else if (role == 1)
          draw_targets<6, 12>(ctrl + e, sd, rp.seed, e, stp, rp.target_frac);
        else
          draw_targets<12, kNU>(ctrl + e, sd, rp.seed, e, stp, rp.target_frac);
      }
      for (int s = 0; s < ninner; ++s) {
        const bool last_sub = (k == nouter - 1) && (s == ninner - 1);
        AI acc0;
        SV accP0;
        EnvState su;  // roles 1, 2: base state at the start of the substep
        if (act) {
          if (role < 2) {  // both leg roles through one call site
            if (role == 1) load_base(scr, su);
            const EnvState& sl = role == 0 ? st : su;
            fk_leg(sl, role, io, ep, cfg, scr, last_sub);
            AI ci;
            SV cp;
            bwd_leg(role, io, ep, cfg, scr, ci, cp);
            if (role == 0) {
              pelvis_acc(st, ep, cfg, acc0, accP0);
              ai_add(acc0, ci);
              sv_acc(accP0, cp);
            } else {
              store_ai(scr, kXLeg, ci, cp);
            }
          } else {
            load_base(scr, su);
            fk_upper(su, cfg, scr);
            AI up;
            SV upP;
            bwd_upper(io, ep, cfg, scr, up, upP);
            store_ai(scr, kXUp, up, upP);
          }
        }
        __syncthreads();
        SV a0;
        if (act && role == 0) {
          AI ci;
          SV cp;
          load_ai(scr, kXLeg, ci, cp);
          ai_add(acc0, ci);
          sv_acc(accP0, cp);
          load_ai(scr, kXUp, ci, cp);
          ai_add(acc0, ci);
          sv_acc(accP0, cp);
          a0 = base_solve(acc0, accP0);
          store_sv(scr, kXA0, a0);
        }
        __syncthreads();
        if (act) {
          if (role < 2) {
            if (role == 1) a0 = load_sv(scr, kXA0);
            fwd_leg(role == 0 ? st : su, role, a0, cfg, scr);
            if (role == 0) {
              integrate_base(st, a0, cfg);
              store_base(scr, st);  // roles 1 and 2 read it after the barrier below
            }
          } else {
            fwd_upper(su, load_sv(scr, kXA0), cfg, scr);
          }
        }
        __syncthreads();
      }
      if (kRollout) {
        if (act && role == 0) {
          const bool rs = st.pos[2] < rp.reset_z;
          if (rs) {
            const float z0 = reset_height(rp, e, stp);
#pragma unroll
            for (int i = 0; i < 3; ++i) st.pos[i] = model().stand[i];
            st.pos[2] = z0;
#pragma unroll
            for (int i = 0; i < 4; ++i) st.quat[i] = model().stand[3 + i];
#pragma unroll
            for (int i = 0; i < 3; ++i) st.vw[i] = st.wb[i] = 0.0f;
#pragma unroll 1
            for (int i = 1; i <= 12; ++i) {
              scr.put(hslot(i, 0), model().stand[6 + i]);
              scr.put(hslot(i, 1), 0.0f);
            }
#pragma unroll
            for (int i = 0; i < 2 * kNC; ++i) a.anchor[(size_t)i * sd + e] = kAnchorFree;
            store_base(scr, st);
            ++resets;
          }
          scr.put(kXReset, rs ? 1.0f : 0.0f);
        }
        __syncthreads();
        if (act && role == 2 && scr.get(kXReset) != 0.0f) {
#pragma unroll 1
          for (int i = 13; i <= kNJ; ++i) {
            scr.put(hslot(i, 0), model().stand[6 + i]);
            scr.put(hslot(i, 1), 0.0f);
          }
        }
      }
    }
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
        store_joints(a.qpos + e, a.qvel + e, sd, scr, 1, 6);
        if (kRollout && reset_count) reset_count[e] += resets;
      } else if (role == 1) {
        store_joints(a.qpos + e, a.qvel + e, sd, scr, 7, 12);
      } else {
        store_joints(a.qpos + e, a.qvel + e, sd, scr, 13, kNJ);
      }
    }
    __syncthreads();  // the next tile reuses the scratch
  }
}

// One entry per launch shape: mapping 0 = one thread per env (BLOCK threads,
// BLOCK envs per block), mapping 1 = two threads per env (BLOCK envs,
// 2 * BLOCK threads per block), mapping 2 = three threads per env (BLOCK
// envs, 3 * BLOCK threads per block).
template <int BLOCK>
int run_single_impl(bool rollout, const StateArgs& a, float* ctrl, int* rc, int nouter, int ninner,
               const StepConfig& cfg, const RolloutParams& rp, cudaStream_t s, int bps) {
  constexpr size_t smem = smem_bytes<BLOCK>();
  if (rollout)
    return launch<1, BLOCK>(rollout_kernel<BLOCK>, BLOCK, smem, a.nenv, BLOCK, bps, s, "rollout_kernel", a, ctrl, rc,
                            nouter, ninner, cfg, rp);
  return launch<0, BLOCK>(step_kernel<BLOCK>, BLOCK, smem, a.nenv, BLOCK, bps, s, "step_kernel", a,
                          (const float*)ctrl, ninner, cfg);
}
template <int ENVS>
constexpr size_t smem_bytes_split3() { return (size_t)kNumSlots3 * ENVS * sizeof(float); }

template <int ENVS>
int run_split3_impl(bool rollout, const StateArgs& a, float* ctrl, int* rc, int nouter, int ninner,
                    const StepConfig& cfg, const RolloutParams& rp, cudaStream_t s, int bps) {
  constexpr size_t smem = smem_bytes_split3<ENVS>();
  if (rollout)
    return launch<5, ENVS>(split3_kernel<ENVS, true>, 3 * ENVS, smem, a.nenv, ENVS, bps, s, "split3_kernel", a, ctrl,
                           rc, nouter, ninner, cfg, rp);
  return launch<4, ENVS>(split3_kernel<ENVS, false>, 3 * ENVS, smem, a.nenv, ENVS, bps, s, "split3_kernel", a, ctrl,
                         rc, 1, ninner, cfg, rp);
}

template <int ENVS>
int run_split_impl(bool rollout, const StateArgs& a, float* ctrl, int* rc, int nouter, int ninner,
              const StepConfig& cfg, const RolloutParams& rp, cudaStream_t s, int bps) {
  constexpr size_t smem = smem_bytes_split<ENVS>();
  if (rollout)
    return launch<3, ENVS>(split_kernel<ENVS, true>, 2 * ENVS, smem, a.nenv, ENVS, bps, s, "split_kernel", a, ctrl,
                           rc, nouter, ninner, cfg, rp);
  return launch<2, ENVS>(split_kernel<ENVS, false>, 2 * ENVS, smem, a.nenv, ENVS, bps, s, "split_kernel", a, ctrl,
                         rc, 1, ninner, cfg, rp);
}


}  // namespace g1b

// Explicit instances of this unit's launch shape (used inside namespace g1b).
#define G1B_STEP_INSTANCE(B)                                                                                 \
  template <>                                                                                                \
  int run_single<B>(bool rollout, const StateArgs& a, float* ctrl, int* rc, int nouter, int ninner,     \
                         const StepConfig& cfg, const RolloutParams& rp, cudaStream_t s, int bps) {          \
    return run_single_impl<B>(rollout, a, ctrl, rc, nouter, ninner, cfg, rp, s, bps);                        \
  }                                                                                                          \
  template <>                                                                                                \
  int run_split<B>(bool rollout, const StateArgs& a, float* ctrl, int* rc, int nouter, int ninner,      \
                        const StepConfig& cfg, const RolloutParams& rp, cudaStream_t s, int bps) {           \
    return run_split_impl<B>(rollout, a, ctrl, rc, nouter, ninner, cfg, rp, s, bps);                         \
  } 

// Instances of the three-role mapping (64 and 128 envs per CTA).
#define G1B_STEP3_INSTANCE(B)                                                                                \
  template <>                                                                                                \
  int run_split3<B>(bool rollout, const StateArgs& a, float* ctrl, int* rc, int nouter, int ninner,          \
                    const StepConfig& cfg, const RolloutParams& rp, cudaStream_t s, int bps) {               \
    return run_split3_impl<B>(rollout, a, ctrl, rc, nouter, ninner, cfg, rp, s, bps);                        \
  }
