// g1_adjoint.cu -- horizon adjoint through the G1 step and its C-ABI.
//
// Problem (one env per thread, H steps of one substep each):
//   x_{t+1} = step(x_t, u_t, kp_scale, kd_scale),  x = (qpos 36, qvel 35, anchor 16)
//   L = sum_{t=1..H} (z_t - z_ref)^2 + w_track * |q_t - u_{t-1}|^2
// with z the base height qpos[2] and q the 29 joint angles qpos[7:36].
// Outputs L, dL/du_t (H x 29), dL/dkp_scale, dL/dkd_scale and dL/dx_0.
//
// One launch does the whole sweep for each env: the forward rollout keeps
// x_t every C steps in caller scratch; then, segment by segment from the
// last, the segment's states are recomputed from its checkpoint, and each
// step is reversed from the last: the primal of step t is recomputed into
// the on-chip tape and g1b::adj::reverse (g1_adj.cuh) turns lambda_{t+1}
// into lambda_t = (dx_{t+1}/dx_t)^T lambda_{t+1} + dL/dx_t, writing the
// targets' adjoint and accumulating the gain-scale adjoints.  The tape, the
// current state and lambda live in shared memory (slot-major per env), so
// the only device-memory traffic is the checkpoints, the segment states, the
// targets and the outputs.
//
// Scratch (caller-provided, R = float or double), SoA [slot][nenv]:
//   checkpoints (ceil(H / C) + 1) x 87, segment states C x 87.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>

#include "g1_adj.cuh"
#include "g1_host.h"

namespace g1b {

namespace {

using adj::kState;
using adj::kTapeSlots;

template <class R>
struct AdjArgs {
  int n, H, C, S;  // envs, horizon, checkpoint interval, segments
  adj::Cfg<R> cfg;
  R mu0;
  const R *qpos0, *qvel0, *anchor0, *targets, *kp, *kd;
  R z_ref, w_track;
  R *loss, *gtar, *gkp, *gkd, *gq0, *gv0;
  R *ck, *seg;
};

template <class R>
__host__ __device__ inline size_t adj_scratch_count(int n, int H, int C) {
  const int S = (H + C - 1) / C;
  return (size_t)n * ((size_t)(S + 1) + (size_t)C) * kState;
}

// one env's column of a slot-major shared array
template <class R, int STRIDE>
struct SCol {
  R* p;
  __device__ __forceinline__ R get(int k) const { return p[k * STRIDE]; }
  __device__ __forceinline__ void put(int k, R v) { p[k * STRIDE] = v; }
};
// one env's column of a device-memory SoA array [slot][n]
template <class R>
struct GCol {
  const R* p;
  size_t n;
  __device__ __forceinline__ R get(int k) const { return p[(size_t)k * n]; }
};
template <class R>
struct GColW {
  R* p;
  size_t n;
  __device__ __forceinline__ void put(int k, R v) { p[(size_t)k * n] = v; }
};

template <class R, class XS>
__device__ __forceinline__ void base_from(const XS& x, adj::Base<R>& st) {
  for (int k = 0; k < 3; ++k) st.pos[k] = x.get(k);
  for (int k = 0; k < 4; ++k) st.quat[k] = x.get(3 + k);
  for (int k = 0; k < 3; ++k) st.vw[k] = x.get(adj::kQV + k);
  for (int k = 0; k < 3; ++k) st.wb[k] = x.get(adj::kQV + 3 + k);
}
template <class R, class XS>
__device__ __forceinline__ void base_to(const adj::Base<R>& st, XS& x) {
  for (int k = 0; k < 3; ++k) x.put(k, st.pos[k]);
  for (int k = 0; k < 4; ++k) x.put(3 + k, st.quat[k]);
  for (int k = 0; k < 3; ++k) x.put(adj::kQV + k, st.vw[k]);
  for (int k = 0; k < 3; ++k) x.put(adj::kQV + 3 + k, st.wb[k]);
}
// 87 entries between a device-memory SoA block (env column e) and shared
template <class R, class XS>
__device__ __forceinline__ void x_load(XS& x, const R* g, size_t n, int e) {
#pragma unroll 1
  for (int k = 0; k < kState; ++k) x.put(k, g[(size_t)k * n + e]);
}
template <class R, class XS>
__device__ __forceinline__ void x_store(const XS& x, R* g, size_t n, int e) {
#pragma unroll 1
  for (int k = 0; k < kState; ++k) g[(size_t)k * n + e] = x.get(k);
}

// dL/dx_t of the terms at x_t (t >= 1), added into lam; up: targets of step t-1
template <class R, class XS, class LS>
__device__ __forceinline__ void loss_grad(const XS& x, const R* up, size_t n, int e, R z_ref, R w, LS& lam) {
  lam.put(2, lam.get(2) + R(2) * (x.get(2) - z_ref));
#pragma unroll 1
  for (int j = 0; j < adj::kNU; ++j) lam.put(7 + j, lam.get(7 + j) + R(2) * w * (x.get(7 + j) - up[(size_t)j * n + e]));
}

// One rolled-out substep.  The forward rollout and the segment
// recomputation both call this one compiled copy, so that a recomputed state
// equals the stored one bit for bit whatever the checkpoint interval.
template <class R, int ENVS>
__device__ __noinline__ void roll_step(adj::Base<R>& st, SCol<R, ENVS>& X, const GCol<R>& U, const adj::Par<R>& par,
                                       const adj::Cfg<R>& cfg, adj::Tape<R, ENVS>& tp) {
  adj::primal<true>(st, X, U, par, cfg, tp);
}

template <class R, int ENVS>
constexpr size_t adj_smem() {
  return (size_t)(kTapeSlots + 2 * kState) * ENVS * sizeof(R);
}

template <class R, int ENVS>
__global__ void __launch_bounds__(ENVS) adj_kernel(AdjArgs<R> a) {
  extern __shared__ __align__(16) unsigned char adj_sm[];
  const int e = blockIdx.x * ENVS + threadIdx.x;
  if (e >= a.n) return;  // no block-wide synchronisation below
  R* col = reinterpret_cast<R*>(adj_sm) + threadIdx.x;
  adj::Tape<R, ENVS> tp{col};
  SCol<R, ENVS> X{col + kTapeSlots * ENVS};
  SCol<R, ENVS> Lm{col + (kTapeSlots + kState) * ENVS};
  const size_t n = (size_t)a.n;
  const adj::Par<R> par{a.mu0, R(0), a.kp ? a.kp[e] : R(1), a.kd ? a.kd[e] : R(1)};
  adj::Base<R> st;
  // ---- forward rollout: loss, checkpoints
#pragma unroll 1
  for (int k = 0; k < adj::kNQ; ++k) X.put(k, a.qpos0[(size_t)k * n + e]);
#pragma unroll 1
  for (int k = 0; k < adj::kNV; ++k) X.put(adj::kQV + k, a.qvel0[(size_t)k * n + e]);
#pragma unroll 1
  for (int k = 0; k < 2 * adj::kNC; ++k) X.put(adj::kAN + k, a.anchor0[(size_t)k * n + e]);
  base_from<R>(X, st);
  R loss = R(0);
#pragma unroll 1
  for (int t = 0; t < a.H; ++t) {
    if (t % a.C == 0) {
      base_to<R>(st, X);
      x_store<R>(X, a.ck + (size_t)(t / a.C) * kState * n, n, e);
    }
    const R* ut = a.targets + (size_t)t * adj::kNU * n + e;
    const GCol<R> U{ut, n};
    roll_step<R, ENVS>(st, X, U, par, a.cfg, tp);
    const R dz = st.pos[2] - a.z_ref;
    R tr = R(0);
#pragma unroll 1
    for (int j = 0; j < adj::kNU; ++j) {
      const R d = X.get(7 + j) - U.get(j);
      tr += d * d;
    }
    loss += dz * dz + a.w_track * tr;
  }
  base_to<R>(st, X);
  x_store<R>(X, a.ck + (size_t)a.S * kState * n, n, e);
  a.loss[e] = loss;
#pragma unroll 1
  for (int k = 0; k < kState; ++k) Lm.put(k, R(0));
  loss_grad<R>(X, a.targets + (size_t)(a.H - 1) * adj::kNU * n, n, e, a.z_ref, a.w_track, Lm);
  R kpb = R(0), kdb = R(0);
  // ---- reverse sweep, segment by segment
#pragma unroll 1
  for (int s = a.S - 1; s >= 0; --s) {
    const int t0 = s * a.C;
    const int len = a.H - t0 < a.C ? a.H - t0 : a.C;
    x_load<R>(X, a.ck + (size_t)s * kState * n, n, e);
    base_from<R>(X, st);
#pragma unroll 1
    for (int i = 0; i < len; ++i) {
      base_to<R>(st, X);
      x_store<R>(X, a.seg + (size_t)i * kState * n, n, e);
      if (i + 1 == len) break;
      const GCol<R> U{a.targets + (size_t)(t0 + i) * adj::kNU * n + e, n};
      roll_step<R, ENVS>(st, X, U, par, a.cfg, tp);
    }
#pragma unroll 1
    for (int i = len - 1; i >= 0; --i) {
      const int t = t0 + i;
      x_load<R>(X, a.seg + (size_t)i * kState * n, n, e);
      base_from<R>(X, st);
      const R* ut = a.targets + (size_t)t * adj::kNU * n + e;
      const GCol<R> U{ut, n};
      adj::Base<R> st0 = st;
      adj::primal<false>(st0, X, U, par, a.cfg, tp);
      GColW<R> Ub{a.gtar + (size_t)t * adj::kNU * n + e, n};
      adj::reverse(st, X, U, Lm, Ub, par, a.cfg, kpb, kdb, tp);
      // dL/du_t also has the tracking term of x_{t+1}: -2 w (q_{t+1} - u_t)
      const R* x1 = (i + 1 < len) ? a.seg + (size_t)(i + 1) * kState * n : a.ck + (size_t)(s + 1) * kState * n;
      R* gt = a.gtar + (size_t)t * adj::kNU * n + e;
#pragma unroll 1
      for (int j = 0; j < adj::kNU; ++j)
        gt[(size_t)j * n] -= R(2) * a.w_track * (x1[(size_t)(7 + j) * n + e] - ut[(size_t)j * n]);
      if (t >= 1) loss_grad<R>(X, a.targets + (size_t)(t - 1) * adj::kNU * n, n, e, a.z_ref, a.w_track, Lm);
    }
  }
  if (a.gq0)
#pragma unroll 1
    for (int k = 0; k < adj::kNQ; ++k) a.gq0[(size_t)k * n + e] = Lm.get(k);
  if (a.gv0)
#pragma unroll 1
    for (int k = 0; k < adj::kNV; ++k) a.gv0[(size_t)k * n + e] = Lm.get(adj::kQV + k);
  if (a.gkp) a.gkp[e] = kpb;
  if (a.gkd) a.gkd[e] = kdb;
}

// envs per CTA: the tape, state and adjoint of each env take (1,124 + 174)
// slots of shared memory, 166 KB for 32 float envs or 16 double envs.
template <class R>
constexpr int adj_envs() { return sizeof(R) == 4 ? 32 : 16; }

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
  a.cfg = adj::Cfg<R>{(R)cfg->gravity_z, (R)cfg->contact_kn, (R)cfg->contact_dn, (R)cfg->contact_kt,
                      (R)cfg->contact_dt,  (R)cfg->limit_kp,   (R)cfg->limit_kd,   (R)cfg->dt};
  a.mu0 = (R)g1m_contact_mu;
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
  a.ck = scratch;
  a.seg = a.ck + (size_t)(a.S + 1) * kState * (size_t)nenv;
  constexpr int E = adj_envs<R>();
  constexpr size_t smem = adj_smem<R, E>();
  cudaError_t e = prepare<30 + (int)sizeof(R), E>(adj_kernel<R, E>, smem);
  if (e != cudaSuccess) return cuda_fail(e, "adjoint: cudaFuncSetAttribute");
  adj_kernel<R, E><<<(nenv + E - 1) / E, E, smem, static_cast<cudaStream_t>(stream)>>>(a);
  return launched("adj_kernel");
}

}  // namespace
}  // namespace g1b

using namespace g1b;

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
// Device address of the array on the current device.  The host-side name of
// a __device__ array is not a device address; the address is looked up on
// every call (a cheap query once the module is loaded), so it stays right
// after a cudaDeviceReset re-creates the context.
int noalloc_scratch(float** out) {
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess) return cuda_fail(e, "adjoint_noalloc: cudaGetSymbolAddress");
  *out = static_cast<float*>(p);
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

}  // extern "C"
