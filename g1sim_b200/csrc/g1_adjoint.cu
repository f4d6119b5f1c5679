// g1_adjoint.cu -- horizon adjoint entry points.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <mutex>

#include "g1_host.h"
#include "g1_tangent.cuh"

namespace g1b {
#include "g1_adjoint.cuh"
}  // namespace g1b

using namespace g1b;

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
