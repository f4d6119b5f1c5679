// ref_rollout.cpp -- CPU timing harness around the REFERENCE's own step
// (TEST / BASELINE INFRASTRUCTURE; built by oracle/Makefile target `ref`
// against the reference's headers, never shipped in the product).
//
// It runs the decimated workload of the 65,536-env benchmark on the host
// cores with the reference's g1_step (reference src/g1_core.h:225-232) in
// FP32 (G1_PRECISION=4), one env per OpenMP iteration with a thread-private
// G1Ws, exactly as the reference's fake-CUDA shim runs its kernel body:
//   dt = 2 ms, decimation substeps per policy step, PD targets redrawn per
//   policy step as stand + U(-frac, frac) * (hi - lo) with the counter RNG
//   that the CUDA path uses, reset to the stand pose when base z < reset_z.
// The reference has no per-env friction or base-mass parameters (they are
// compile-time constants, src/g1_model.h:80,351), so this harness runs every
// env with the nominal model; the work per substep is the same.
//
// Envs env0 .. env0 + count - 1 are processed in chunks across the threads
// until they are done or --seconds of wall time have passed (a bounded
// sample of the workload); it prints one JSON line with env-steps/s.  The
// CPU baseline runs one such process per host core, pinned to that core,
// each on its own slice of the envs.  Built at G1_PRECISION=4 (the
// reference's FP32 step) and at G1_PRECISION=8 (its FP64 host build).
#include "g1_core.h"

#include <omp.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>

static unsigned hash32(unsigned x) {  // same integer hash as the CUDA path
  x ^= x >> 16; x *= 0x7feb352du;
  x ^= x >> 15; x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}
static float uniform24(unsigned seed, unsigned stream, unsigned counter) {
  unsigned h = hash32(seed ^ hash32(stream * 0x9E3779B9u + 0x7F4A7C15u));
  h = hash32(h ^ (counter * 0x85EBCA6Bu + 0xC2B2AE35u));
  return (float)(h >> 8) * (1.0f / 16777216.0f);
}

int main(int argc, char** argv) {
  int nenv = 65536, nsteps = 1000, decim = 10, threads = 0, env0 = 0, count = -1;
  double seconds = 10.0, dt = 2e-3;
  unsigned seed = 0;
  for (int i = 1; i < argc; ++i) {
    if (!strcmp(argv[i], "--nenv")) nenv = atoi(argv[++i]);
    else if (!strcmp(argv[i], "--steps")) nsteps = atoi(argv[++i]);
    else if (!strcmp(argv[i], "--decim")) decim = atoi(argv[++i]);
    else if (!strcmp(argv[i], "--threads")) threads = atoi(argv[++i]);
    else if (!strcmp(argv[i], "--seconds")) seconds = atof(argv[++i]);
    else if (!strcmp(argv[i], "--seed")) seed = (unsigned)atoi(argv[++i]);
    else if (!strcmp(argv[i], "--env0")) env0 = atoi(argv[++i]);
    else if (!strcmp(argv[i], "--count")) count = atoi(argv[++i]);
  }
  if (count < 0) count = nenv - env0;
  const int env_end = env0 + count < nenv ? env0 + count : nenv;
  if (threads > 0) omp_set_num_threads(threads);
  int nthr = omp_get_max_threads();
  const int npolicy = nsteps / decim;
  G1Config cfg = g1_default_config();
  cfg.dt = G1Real(dt);
  const float frac = 0.3f, reset_z = 0.3f;

  long long envs_done = 0, resets = 0;
  double t0 = omp_get_wtime(), elapsed = 0;
  int chunk = nthr * 4;
  double zsum = 0;
  for (int base = env0; base < env_end; base += chunk) {
    int hi = base + chunk < env_end ? base + chunk : env_end;
    long long rs = 0;
    double zs = 0;
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : rs, zs)
    for (int e = base; e < hi; ++e) {
      G1Ws w;
      G1Real qp[G1_NQ], qv[G1_NV], ct[G1_NU], an[2 * G1_NC];
      unsigned u = seed ^ 0x3c6ef372u;
      for (int i = 0; i < G1_NQ; ++i) qp[i] = g1_qpos_stand[i];
      qp[2] = G1Real(0.75f + uniform24(u, (unsigned)e, 0u) * 0.1f);
      for (int i = 0; i < G1_NV; ++i) qv[i] = 0;
      for (int i = 0; i < 2 * G1_NC; ++i) an[i] = G1_ANCHOR_FREE;
      for (int k = 0; k < npolicy; ++k) {
        for (int j = 0; j < G1_NU; ++j) {
          float r = 2.0f * uniform24(seed, (unsigned)e, (unsigned)k * 64u + (unsigned)j) - 1.0f;
          float span = frac * (float)(g1_jnt_range[2 * j + 1] - g1_jnt_range[2 * j]);
          ct[j] = G1Real((float)g1_qpos_stand[7 + j] + r * span);
        }
        for (int s = 0; s < decim; ++s) g1_step(cfg, qp, qv, ct, an, w, nullptr);
        if (qp[2] < reset_z) {
          for (int i = 0; i < G1_NQ; ++i) qp[i] = g1_qpos_stand[i];
          qp[2] = G1Real(0.75f + uniform24(seed ^ 0x5bd1e995u, (unsigned)e, (unsigned)k) * 0.1f);
          for (int i = 0; i < G1_NV; ++i) qv[i] = 0;
          for (int i = 0; i < 2 * G1_NC; ++i) an[i] = G1_ANCHOR_FREE;
          rs += 1;
        }
      }
      zs += qp[2];
    }
    envs_done += hi - base;
    resets += rs;
    zsum += zs;
    elapsed = omp_get_wtime() - t0;
    if (elapsed >= seconds) break;
  }
  double env_steps = (double)envs_done * npolicy * decim;
  printf("{\"env_steps_per_s\": %.6g, \"env_steps\": %.6g, \"threads\": %d, \"envs\": %lld, "
         "\"env0\": %d, \"substeps\": %d, \"seconds\": %.4f, \"resets\": %lld, \"mean_z\": %.5f, "
         "\"dt\": %g, \"decim\": %d, \"precision\": %d}\n",
         env_steps / elapsed, env_steps, nthr, envs_done, env0, npolicy * decim, elapsed, resets,
         zsum / (double)(envs_done > 0 ? envs_done : 1), dt, decim, (int)sizeof(G1Real));
  return 0;
}
