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
constexpr size_t smem_bytes() { return (size_t)kNumSlots * BLOCK * sizeof(float); }

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
// writes the env's targets into its ctrl column (read back by the substeps)
template <int J>
__device__ __forceinline__ void draw_targets(float* ct, size_t stride, unsigned seed, int e, int step,
                                             float frac) {
  ct[J * stride] = draw_target<J>(seed, e, step, frac);
  if constexpr (J + 1 < kNU) draw_targets<J + 1>(ct, stride, seed, e, step, frac);
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

}  // namespace g1b

// =================================================================== host
using namespace g1b;

namespace {

thread_local char g_err[512] = "";
std::mutex g_mu;
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

template <int BLOCK>
int launch_step(const StateArgs& a, const float* ctrl, int nsub, const StepConfig& cfg,
                cudaStream_t stream, int blocks_per_sm) {
  constexpr size_t smem = smem_bytes<BLOCK>();
  auto k = step_kernel<BLOCK>;
  cudaError_t e = prepare<0, BLOCK>(k, smem);
  if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute(step)");
  const int grid = grid_for<0, BLOCK>(k, BLOCK, smem, a.nenv, blocks_per_sm);
  k<<<grid, BLOCK, smem, stream>>>(a, ctrl, nsub, cfg);
  e = cudaGetLastError();
  return e == cudaSuccess ? 0 : cuda_fail(e, "step_kernel launch");
}

template <int BLOCK>
int launch_rollout(const StateArgs& a, float* ctrl, int* rc, int npolicy, int decim,
                   const StepConfig& cfg, const RolloutParams& rp, cudaStream_t stream,
                   int blocks_per_sm) {
  constexpr size_t smem = smem_bytes<BLOCK>();
  auto k = rollout_kernel<BLOCK>;
  cudaError_t e = prepare<1, BLOCK>(k, smem);
  if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute(rollout)");
  const int grid = grid_for<1, BLOCK>(k, BLOCK, smem, a.nenv, blocks_per_sm);
  k<<<grid, BLOCK, smem, stream>>>(a, ctrl, rc, npolicy, decim, cfg, rp);
  e = cudaGetLastError();
  return e == cudaSuccess ? 0 : cuda_fail(e, "rollout_kernel launch");
}

int dispatch_step(const StateArgs& a, const float* ctrl, int nsub, const StepConfig& cfg,
                  cudaStream_t s) {
  int block, bps;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    block = g_block;
    bps = g_blocks_per_sm;
  }
  switch (block) {
    case 32: return launch_step<32>(a, ctrl, nsub, cfg, s, bps);
    case 64: return launch_step<64>(a, ctrl, nsub, cfg, s, bps);
    case 96: return launch_step<96>(a, ctrl, nsub, cfg, s, bps);
    default: return launch_step<128>(a, ctrl, nsub, cfg, s, bps);
  }
}

int dispatch_rollout(const StateArgs& a, float* ctrl, int* rc, int npolicy, int decim,
                     const StepConfig& cfg, const RolloutParams& rp, cudaStream_t s) {
  int block, bps;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    block = g_block;
    bps = g_blocks_per_sm;
  }
  switch (block) {
    case 32: return launch_rollout<32>(a, ctrl, rc, npolicy, decim, cfg, rp, s, bps);
    case 64: return launch_rollout<64>(a, ctrl, rc, npolicy, decim, cfg, rp, s, bps);
    case 96: return launch_rollout<96>(a, ctrl, rc, npolicy, decim, cfg, rp, s, bps);
    default: return launch_rollout<128>(a, ctrl, rc, npolicy, decim, cfg, rp, s, bps);
  }
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

int g1b_set_launch(int block, int blocks_per_sm) {
  if (block != 32 && block != 64 && block != 96 && block != 128) return fail("block must be 32, 64, 96 or 128");
  if (blocks_per_sm < 0) return fail("blocks_per_sm must be >= 0");
  std::lock_guard<std::mutex> lk(g_mu);
  g_block = block;
  g_blocks_per_sm = blocks_per_sm;
  return 0;
}

int g1b_get_launch(int* block, int* blocks_per_sm) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (block) *block = g_block;
  if (blocks_per_sm) *blocks_per_sm = g_blocks_per_sm;
  return 0;
}

int g1b_autotune(int nenv, int nsub, void* stream, float* best_ms) {
  (void)nenv;
  (void)nsub;
  (void)stream;
  (void)best_ms;
  return fail("autotune: not built yet");
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
