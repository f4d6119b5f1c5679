// g1_kernels.cu -- sm_100a kernels and the C-ABI of libg1cuda.so.
//
// Kernels (one env per thread, grid-stride over envs so a grid sized to the
// resident capacity runs persistently):
//   step_kernel<BLOCK>     nsub substeps of g1b::step per env; state loaded
//                          from SoA once, kept in registers, stored once
//                          (reference src/g1_kernel.cu:106-151)
//   rollout_kernel<BLOCK>  npolicy x (target redraw, decim substeps, reset
//                          check) per env, all in one launch
//   reset_done_kernel      reference src/g1_kernel.cu:85-103, bit-exact
//   ffma_kernel            FP32 FMA throughput microbenchmark
// Per-hinge scratch of the step lives in dynamic shared memory laid out
// slot-major, sm[slot * BLOCK + threadIdx.x], so every access is
// bank-conflict free.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <atomic>
#include <mutex>

#include "../../include/g1sim_b200.h"
#include "g1_phys.cuh"
#include "g1_mlp.cuh"
#include "g1_tangent.cuh"

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
        const float u = uniform24(rp.seed ^ 0x5bd1e995u, (unsigned)e, (unsigned)stp);
        const float z0 = __fadd_rn(rp.z0_lo, __fmul_rn(u, __fsub_rn(rp.z0_hi, rp.z0_lo)));
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
// upper body (waist, arms) of env tile * ENVS + (tid % ENVS).  Both halves
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
            bwd_lower(st, io, ep, cfg, scr, acc0, accP0);
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
            fwd_upper(su, load_sv(scr, kXA0), cfg, scr);
          } else {
            fwd_lower_and_base(st, a0, cfg, scr);
            store_base(scr, st);
          }
        }
        __syncthreads();
      }
      if (kRollout) {
        if (act && role == 0) {
          const bool rs = st.pos[2] < rp.reset_z;
          if (rs) {
            const float u = uniform24(rp.seed ^ 0x5bd1e995u, (unsigned)e, (unsigned)stp);
            const float z0 = __fadd_rn(rp.z0_lo, __fmul_rn(u, __fsub_rn(rp.z0_hi, rp.z0_lo)));
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
        if (kRollout && reset_count) reset_count[e] += resets;
      } else {
        store_joints(a.qpos + e, a.qvel + e, sd, scr, 13, kNJ);
      }
    }
    __syncthreads();  // the next tile reuses the scratch
  }
}

template <int ENVS>
constexpr size_t smem_bytes_split() { return (size_t)kNumSlots * ENVS * sizeof(float); }

#include "g1_policy.cuh"
#include "g1_adjoint.cuh"
#include "g1_gemm.cuh"
#include "g1_surrogate.cuh"
__device__ int g_gemm_error = 0;

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

thread_local char g_err[512] = "";
std::mutex g_mu;
int g_mapping = 1;  // two threads per env
int g_block = 128;
int g_blocks_per_sm = 0;

int fail(const char* msg) {
  snprintf(g_err, sizeof(g_err), "%s", msg);
  return -1;
}
int cuda_fail(cudaError_t e, const char* where) {
  snprintf(g_err, sizeof(g_err), "%s: %s", where, cudaGetErrorString(e));
  return -2;
}

StepConfig to_cfg(const g1b_config* c) {
  StepConfig s;
  s.gravity_z = c->gravity_z;
  s.contact_kn = c->contact_kn;
  s.contact_dn = c->contact_dn;
  s.contact_kt = c->contact_kt;
  s.contact_dt = c->contact_dt;
  s.limit_kp = c->limit_kp;
  s.limit_kd = c->limit_kd;
  s.dt = c->dt;
  return s;
}

g1b_config default_cfg() {  // reference src/g1_types.h:44-55
  g1b_config c;
  c.gravity_z = -9.81f;
  c.contact_kn = 2e4f;
  c.contact_dn = 280.0f;
  c.contact_kt = 1e4f;
  c.contact_dt = 280.0f;
  c.limit_kp = 200.0f;
  c.limit_kd = 5.0f;
  c.dt = 1e-3f;
  return c;
}

// Grid for a grid-stride kernel: enough blocks to cover nenv, capped at the
// resident capacity (blocks_per_sm of them per SM, 0 = occupancy limit).
// The SM count and occupancy are queried once per kernel instance and device
// so that launches inside a stream capture issue nothing but the launch.
template <int KIND, int BLOCK, class K>
int grid_for(K kernel, int block, size_t smem, int nenv, int blocks_per_sm) {
  static std::atomic<int> cache[64][2];  // (sms, occupancy) per device, 0 = unknown
  int dev = 0;
  cudaGetDevice(&dev);
  dev &= 63;
  int sms = cache[dev][0].load(), occ = cache[dev][1].load();
  if (sms == 0 || occ == 0) {
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel, block, smem);
    if (occ < 1) occ = 1;
    cache[dev][0].store(sms);
    cache[dev][1].store(occ);
  }
  if (blocks_per_sm > 0 && blocks_per_sm < occ) occ = blocks_per_sm;
  const int need = (nenv + block - 1) / block;
  const int cap = sms * occ;
  return need < cap ? need : cap;
}

// Opt each kernel instance (KIND, BLOCK) into its dynamic shared memory once
// per device.
template <int KIND, int BLOCK, class K>
cudaError_t prepare(K kernel, size_t smem) {
  static std::atomic<unsigned long long> done_mask{0};
  int dev = 0;
  cudaGetDevice(&dev);
  const unsigned long long bit = 1ull << (dev & 63);
  if (done_mask.load() & bit) return cudaSuccess;
  const cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess) done_mask.fetch_or(bit);
  return e;
}

// Launch of one kernel instance: attribute opt-in, resident-capped grid.
template <int KIND, int BLOCK, class K, class... Args>
int launch(K kernel, int threads, size_t smem, int nwork, int items_per_block, int bps, cudaStream_t stream,
           const char* what, Args... args) {
  cudaError_t e = prepare<KIND, BLOCK>(kernel, smem);
  if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute");
  const int need = (nwork + items_per_block - 1) / items_per_block;
  int grid = grid_for<KIND, BLOCK>(kernel, threads, smem, need * threads, bps);
  if (grid > need) grid = need;
  kernel<<<grid, threads, smem, stream>>>(args...);
  e = cudaGetLastError();
  return e == cudaSuccess ? 0 : cuda_fail(e, what);
}

// One entry per launch shape: mapping 0 = one thread per env (BLOCK threads,
// BLOCK envs per block), mapping 1 = two threads per env (BLOCK envs,
// 2 * BLOCK threads per block).
template <int BLOCK>
int run_single(bool rollout, const StateArgs& a, float* ctrl, int* rc, int nouter, int ninner,
               const StepConfig& cfg, const RolloutParams& rp, cudaStream_t s, int bps) {
  constexpr size_t smem = smem_bytes<BLOCK>();
  if (rollout)
    return launch<1, BLOCK>(rollout_kernel<BLOCK>, BLOCK, smem, a.nenv, BLOCK, bps, s, "rollout_kernel", a, ctrl, rc,
                            nouter, ninner, cfg, rp);
  return launch<0, BLOCK>(step_kernel<BLOCK>, BLOCK, smem, a.nenv, BLOCK, bps, s, "step_kernel", a,
                          (const float*)ctrl, ninner, cfg);
}
template <int ENVS>
int run_split(bool rollout, const StateArgs& a, float* ctrl, int* rc, int nouter, int ninner,
              const StepConfig& cfg, const RolloutParams& rp, cudaStream_t s, int bps) {
  constexpr size_t smem = smem_bytes_split<ENVS>();
  if (rollout)
    return launch<3, ENVS>(split_kernel<ENVS, true>, 2 * ENVS, smem, a.nenv, ENVS, bps, s, "split_kernel", a, ctrl,
                           rc, nouter, ninner, cfg, rp);
  return launch<2, ENVS>(split_kernel<ENVS, false>, 2 * ENVS, smem, a.nenv, ENVS, bps, s, "split_kernel", a, ctrl,
                         rc, 1, ninner, cfg, rp);
}

struct LaunchShape {
  int mapping, block, bps;
};
LaunchShape current_shape() {
  std::lock_guard<std::mutex> lk(g_mu);
  return LaunchShape{g_mapping, g_block, g_blocks_per_sm};
}

int dispatch(const LaunchShape& L, bool rollout, const StateArgs& a, float* ctrl, int* rc, int nouter,
             int ninner, const StepConfig& cfg, const RolloutParams& rp, cudaStream_t s) {
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

int check_state(int nenv, const void* qpos, const void* qvel, const void* anchor, const void* ctrl) {
  if (nenv <= 0) return fail("nenv must be positive");
  if (!qpos || !qvel || !anchor || !ctrl) return fail("qpos, qvel, anchor and ctrl must be non-null");
  return 0;
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
  if (mapping != 0 && mapping != 1) return fail("mapping must be 0 (thread per env) or 1 (two threads per env)");
  if (block != 32 && block != 64 && block != 96 && block != 128) return fail("block must be 32, 64, 96 or 128");
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
  for (int mapping = 0; mapping < 2 && rc == 0; ++mapping) {
    for (int bi = 0; bi < 4 && rc == 0; ++bi) {
      const LaunchShape L{mapping, blocks[bi], 0};
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

}  // extern "C"

namespace {
template <class R>
int adjoint_impl(int nenv, const g1b_config* cfg, const g1b_adjoint_problem* pr, const R* qpos0, const R* qvel0,
                 const R* anchor0, const R* targets, const R* kp_scale, const R* kd_scale, R* loss, R* grad_targets,
                 R* grad_kp, R* grad_kd, R* grad_qpos0, R* grad_qvel0, R* scratch, void* stream) {
  if (nenv <= 0) return fail("adjoint: nenv must be positive");
  if (!cfg || !pr) return fail("adjoint: cfg and problem are required");
  if (pr->horizon <= 0 || pr->checkpoint <= 0) return fail("adjoint: horizon and checkpoint must be positive");
  if (!qpos0 || !qvel0 || !anchor0 || !targets || !loss || !grad_targets || !scratch)
    return fail("adjoint: state, targets, loss, grad_targets and scratch are required");
  AdjArgs<R> a;
  a.n = nenv;
  a.H = pr->horizon;
  a.C = pr->checkpoint < pr->horizon ? pr->checkpoint : pr->horizon;
  a.S = (a.H + a.C - 1) / a.C;
  a.cfg = tg::CfgT<R>{(R)cfg->gravity_z, (R)cfg->contact_kn, (R)cfg->contact_dn, (R)cfg->contact_kt,
                      (R)cfg->contact_dt,  (R)cfg->limit_kp,   (R)cfg->limit_kd,   (R)cfg->dt};
  a.qpos0 = qpos0;
  a.qvel0 = qvel0;
  a.anchor0 = anchor0;
  a.targets = targets;
  a.kp = kp_scale;
  a.kd = kd_scale;
  a.z_ref = (R)pr->z_ref;
  a.w_track = (R)pr->w_track;
  a.loss = loss;
  a.gtar = grad_targets;
  a.gkp = grad_kp;
  a.gkd = grad_kd;
  a.gq0 = grad_qpos0;
  a.gv0 = grad_qvel0;
  const size_t n = (size_t)nenv;
  a.ck = scratch;
  a.seg = a.ck + (size_t)(a.S + 1) * kAdjState * n;
  a.lam = a.seg + (size_t)a.C * kAdjState * n;
  a.G = a.lam + (size_t)kAdjState * n;
  const cudaError_t e = adj_launch<R>(a, static_cast<cudaStream_t>(stream));
  return e == cudaSuccess ? 0 : cuda_fail(e, "adjoint kernels");
}
}  // namespace

extern "C" {

int g1b_adjoint_scratch_size(int nenv, const g1b_adjoint_problem* pr, size_t* count) {
  if (nenv <= 0 || !pr || pr->horizon <= 0 || pr->checkpoint <= 0 || !count)
    return fail("adjoint_scratch_size: invalid arguments");
  const int C = pr->checkpoint < pr->horizon ? pr->checkpoint : pr->horizon;
  *count = adj_scratch_count<float>(nenv, pr->horizon, C);
  return 0;
}

int g1b_adjoint(int nenv, const g1b_config* cfg, const g1b_adjoint_problem* pr, const float* qpos0,
                const float* qvel0, const float* anchor0, const float* targets, const float* kp_scale,
                const float* kd_scale, float* loss, float* grad_targets, float* grad_kp, float* grad_kd,
                float* grad_qpos0, float* grad_qvel0, float* scratch, void* stream) {
  return adjoint_impl<float>(nenv, cfg, pr, qpos0, qvel0, anchor0, targets, kp_scale, kd_scale, loss, grad_targets,
                             grad_kp, grad_kd, grad_qpos0, grad_qvel0, scratch, stream);
}

int g1b_adjoint_f64(int nenv, const g1b_config* cfg, const g1b_adjoint_problem* pr, const double* qpos0,
                    const double* qvel0, const double* anchor0, const double* targets, const double* kp_scale,
                    const double* kd_scale, double* loss, double* grad_targets, double* grad_kp, double* grad_kd,
                    double* grad_qpos0, double* grad_qvel0, double* scratch, void* stream) {
  return adjoint_impl<double>(nenv, cfg, pr, qpos0, qvel0, anchor0, targets, kp_scale, kd_scale, loss,
                              grad_targets, grad_kp, grad_kd, grad_qpos0, grad_qvel0, scratch, stream);
}

}  // extern "C"

// ------------------------------------------- adjoint without allocation
// Some callers cannot call cudaMalloc (a real-time control loop that reserves
// all device memory at start-up, or a process whose device memory belongs to
// another allocator and that cannot hand this library a buffer).  For them,
// g1b_adjoint_noalloc runs the FP32 horizon adjoint with its workspace in
// this fixed device array instead of caller scratch.  Every device that
// loads the library holds the array until the process exits.
constexpr size_t kNoAllocScratchFloats = size_t(1) << 21;  // 8 MiB of float
static __device__ __align__(256) float g_noalloc_scratch[kNoAllocScratchFloats];

namespace {
// Device address of the array, looked up once per device (the host-side
// name of a __device__ array is not a device address).
std::mutex g_noalloc_mu;
float* g_noalloc_ptr[64] = {};

int noalloc_scratch(float** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "adjoint_noalloc: cudaGetDevice");
  if (dev < 0 || dev >= 64) return fail("adjoint_noalloc: device index out of range");
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "adjoint_noalloc: cudaGetSymbolAddress");
    g_noalloc_ptr[dev] = static_cast<float*>(p);
  }
  *out = g_noalloc_ptr[dev];
  return 0;
}
}  // namespace

extern "C" {

size_t g1b_adjoint_noalloc_capacity(void) { return kNoAllocScratchFloats; }

int g1b_adjoint_noalloc(int nenv, const g1b_config* cfg, const g1b_adjoint_problem* pr, const float* qpos0,
                        const float* qvel0, const float* anchor0, const float* targets, const float* kp_scale,
                        const float* kd_scale, float* loss, float* grad_targets, float* grad_kp, float* grad_kd,
                        float* grad_qpos0, float* grad_qvel0, void* stream) {
  if (nenv <= 0 || !pr || pr->horizon <= 0 || pr->checkpoint <= 0)
    return fail("adjoint_noalloc: nenv, horizon and checkpoint must be positive");
  const int C = pr->checkpoint < pr->horizon ? pr->checkpoint : pr->horizon;
  const size_t need = adj_scratch_count<float>(nenv, pr->horizon, C);
  if (need > kNoAllocScratchFloats) {
    snprintf(g_err, sizeof(g_err),
             "adjoint_noalloc: this problem needs %zu floats of workspace, more than the fixed %zu "
             "(reduce nenv, the horizon or the checkpoint interval, or call g1b_adjoint with scratch)",
             need, kNoAllocScratchFloats);
    return -1;
  }
  float* scratch = nullptr;
  if (int rc = noalloc_scratch(&scratch)) return rc;
  // Every workspace slot is written before it is read within one call, so
  // nothing left by an earlier call needs clearing.
  return adjoint_impl<float>(nenv, cfg, pr, qpos0, qvel0, anchor0, targets, kp_scale, kd_scale, loss, grad_targets,
                             grad_kp, grad_kd, grad_qpos0, grad_qvel0, scratch, stream);
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


// ------------------------------------------------- surrogate kernels
int g1b_gemm_bf16(int M, int N, int K, const void* A, int lda, const void* B, int ldb, float* C, int ldc,
                  const float* bias, int splits, void* stream) {
  if (M <= 0 || N <= 0 || K <= 0 || !A || !B || !C) return fail("gemm_bf16: invalid arguments");
  if (splits < 1) splits = 1;
  const int Nt = N <= kGemmMaxN ? N : kGemmMaxN;
  if (M % 128 || N % 16 || N % Nt || K % (kGemmKC * splits))
    return fail("gemm_bf16: needs M % 128 == 0, N % 16 == 0 (and N % 256 == 0 above 256), K % (64 splits) == 0");
  if (lda % 8 || ldb % 8 || ldc % 4 || (((uintptr_t)A | (uintptr_t)B) & 15) || (((uintptr_t)C) & 15))
    return fail("gemm_bf16: lda, ldb multiples of 8, ldc of 4, 16-byte aligned pointers");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int MT = M % 256 == 0 ? 2 : 1;  // two row tiles per CTA share each weight chunk
  const dim3 grid(M / (128 * MT), N / Nt, splits);
  int* err = nullptr;
  cudaError_t e = cudaGetSymbolAddress((void**)&err, g_gemm_error);
  if (e != cudaSuccess) return cuda_fail(e, "gemm_bf16: error flag");
  const __nv_bfloat16* a = static_cast<const __nv_bfloat16*>(A);
  const __nv_bfloat16* b = static_cast<const __nv_bfloat16*>(B);
  if (splits > 1) {
    e = cudaMemset2DAsync(C, (size_t)ldc * 4, 0, (size_t)N * 4, M, st);
    if (e != cudaSuccess) return cuda_fail(e, "gemm_bf16: clear C");
  }
#define G1_GEMM_LAUNCH(AT, M_T, KEY)                                                              \
  do {                                                                                           \
    if ((e = prepare<20, KEY>(gemm_bf16_kernel<AT, M_T>, gemm_smem<M_T>())) != cudaSuccess)      \
      return cuda_fail(e, "gemm_bf16: attributes");                                              \
    gemm_bf16_kernel<AT, M_T><<<grid, 128, gemm_smem<M_T>(), st>>>(a, lda, b, ldb, C, ldc, bias, Nt, \
                                                                  K / splits, err);              \
  } while (0)
  if (splits > 1) {
    if (MT == 2) G1_GEMM_LAUNCH(true, 2, 3); else G1_GEMM_LAUNCH(true, 1, 1);
  } else {
    if (MT == 2) G1_GEMM_LAUNCH(false, 2, 2); else G1_GEMM_LAUNCH(false, 1, 0);
  }
#undef G1_GEMM_LAUNCH
  e = cudaGetLastError();
  return e == cudaSuccess ? 0 : cuda_fail(e, "gemm_bf16_kernel");
}

int g1b_gemm_status(int* code) {
  int v = 0;
  cudaError_t e = cudaMemcpyFromSymbol(&v, g_gemm_error, sizeof(int));
  if (e != cudaSuccess) return cuda_fail(e, "gemm_status");
  const int zero = 0;
  e = cudaMemcpyToSymbol(g_gemm_error, &zero, sizeof(int));
  if (e != cudaSuccess) return cuda_fail(e, "gemm_status");
  if (code) *code = v;
  return 0;
}

static int grid_1d(size_t n, int block) {
  const size_t g = (n + block - 1) / block;
  return (int)(g < 148 * 16 ? g : 148 * 16);
}
static int launched(const char* what) {
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? 0 : cuda_fail(e, what);
}

int g1b_sur_act(int B, int D, const float* Z, void* H, void* Ht, void* stream) {
  if (B <= 0 || D <= 0 || !Z || !H) return fail("sur_act: invalid arguments");
  const dim3 grid((D + 31) / 32, (B + 31) / 32), block(32, 8);
  sur_act_kernel<<<grid, block, 0, static_cast<cudaStream_t>(stream)>>>(
      B, D, Z, static_cast<__nv_bfloat16*>(H), static_cast<__nv_bfloat16*>(Ht));
  return launched("sur_act_kernel");
}

int g1b_sur_act_bwd(int B, int D, const float* dH, const float* Z, void* dZ, void* dZt, float* db, void* stream) {
  if (B <= 0 || D <= 0 || !dH || !Z || !dZ || !dZt || !db) return fail("sur_act_bwd: invalid arguments");
  const dim3 grid((D + 31) / 32, (B + 31) / 32), block(32, 8);
  sur_act_bwd_kernel<<<grid, block, 0, static_cast<cudaStream_t>(stream)>>>(
      B, D, dH, Z, static_cast<__nv_bfloat16*>(dZ), static_cast<__nv_bfloat16*>(dZt), db);
  return launched("sur_act_bwd_kernel");
}

int g1b_sur_loss(int B, int D, const float* Y, const float* T, const float* w, void* dY, void* dYt, float* db,
                 float* loss, void* stream) {
  if (B <= 0 || D <= 0 || !Y || !T || !w || !dY || !dYt || !db || !loss) return fail("sur_loss: invalid arguments");
  const dim3 grid((D + 31) / 32, (B + 31) / 32), block(32, 8);
  sur_loss_kernel<<<grid, block, 0, static_cast<cudaStream_t>(stream)>>>(
      B, D, Y, T, w, static_cast<__nv_bfloat16*>(dY), static_cast<__nv_bfloat16*>(dYt), db, loss);
  return launched("sur_loss_kernel");
}

int g1b_sur_adam(int n, float* p, const float* g, float* m, float* v, float lr, float b1, float b2, float eps,
                 int step, void* stream) {
  if (n <= 0 || !p || !g || !m || !v || step < 1) return fail("sur_adam: invalid arguments");
  const float c1 = 1.0f - powf(b1, (float)step), c2 = 1.0f - powf(b2, (float)step);
  sur_adam_kernel<<<grid_1d((size_t)n, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(n, p, g, m, v, lr, b1, b2,
                                                                                         eps, c1, c2);
  return launched("sur_adam_kernel");
}

int g1b_sur_cast(int rows, int cols, const float* W, void* Wb, void* Wt, void* stream) {
  if (rows <= 0 || cols <= 0 || !W || !Wb || !Wt) return fail("sur_cast: invalid arguments");
  sur_cast_kernel<<<grid_1d((size_t)rows * cols, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      rows, cols, W, static_cast<__nv_bfloat16*>(Wb), static_cast<__nv_bfloat16*>(Wt));
  return launched("sur_cast_kernel");
}

int g1b_sur_features(int n, const float* qpos, const float* qvel, const float* ctrl, const float* cf,
                     const float* mean, const float* istd, void* X, void* Xt, float* F, void* stream) {
  if (n <= 0 || !qpos || !qvel || !ctrl || !mean || !istd || !X) return fail("sur_features: invalid arguments");
  sur_features_kernel<<<(n + 127) / 128, 128, 0, static_cast<cudaStream_t>(stream)>>>(
      n, qpos, qvel, ctrl, cf, mean, istd, static_cast<__nv_bfloat16*>(X), static_cast<__nv_bfloat16*>(Xt), F);
  return launched("sur_features_kernel");
}

int g1b_sur_integrate(int n, const float* Y, int ldy, const float* omean, const float* ostd, float dt, float* qpos,
                      float* qvel, void* stream) {
  if (n <= 0 || !Y || ldy < kNV || !omean || !ostd || !qpos || !qvel) return fail("sur_integrate: invalid arguments");
  sur_integrate_kernel<<<(n + 127) / 128, 128, 0, static_cast<cudaStream_t>(stream)>>>(n, Y, ldy, omean, ostd, dt,
                                                                                       qpos, qvel);
  return launched("sur_integrate_kernel");
}

}  // extern "C"
