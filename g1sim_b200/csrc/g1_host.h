// g1_host.h -- host-side helpers shared by the translation units of
// libg1cuda.so: the per-thread error message behind g1b_last_error(), the
// step configuration, and the launch of a resident-capped grid.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <cstdio>

#include "../../include/g1sim_b200.h"
#include "g1_phys.cuh"

namespace g1b {

// Message of the calling thread's last failed entry point (g1_step.cu).
extern thread_local char g_err[512];

inline int fail(const char* msg) {
  snprintf(g_err, sizeof(g_err), "%s", msg);
  return -1;
}
template <class... Args>
inline int failf(const char* fmt, Args... args) {
  snprintf(g_err, sizeof(g_err), fmt, args...);
  return -1;
}
inline int cuda_fail(cudaError_t e, const char* where) {
  snprintf(g_err, sizeof(g_err), "%s: %s", where, cudaGetErrorString(e));
  return -2;
}
inline int launched(const char* what) {
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? 0 : cuda_fail(e, what);
}

inline StepConfig to_cfg(const g1b_config* c) {
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

inline g1b_config default_cfg() {  // reference src/g1_types.h:44-55
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

// Grid for a grid-stride kernel: enough blocks to cover nwork threads,
// capped at the resident capacity (blocks_per_sm of them per SM, 0 = the
// occupancy limit).  The SM count and occupancy are queried once per kernel
// instance (KIND, BLOCK; unique across the library) and device, so that
// launches inside a stream capture issue nothing but the launch.
template <int KIND, int BLOCK, class K>
int grid_for(K kernel, int block, size_t smem, int nwork, int blocks_per_sm) {
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
  const int need = (nwork + block - 1) / block;
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

// Launch of one kernel instance: attribute opt-in, resident-capped grid over
// ceil(nwork / items_per_block) blocks of `threads` threads.
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

inline int check_state(int nenv, const void* qpos, const void* qvel, const void* anchor, const void* ctrl) {
  if (nenv <= 0) return fail("nenv must be positive");
  if (!qpos || !qvel || !anchor || !ctrl) return fail("qpos, qvel, anchor and ctrl must be non-null");
  return 0;
}

}  // namespace g1b
