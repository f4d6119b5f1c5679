/* g1sim_b200.h -- C-ABI of the B200-native batched G1 step (libg1cuda.so).
 *
 * Two groups of entry points:
 *
 *  1. Drop-in replacements of the reference's GPU ABI, same names, argument
 *     meaning and layouts (reference src/g1_kernel.cu:153-174, bound by
 *     reference src/g1sim.py:15-33):
 *        g1_cuda_step, g1_cuda_reset_done
 *     As in the reference they return nothing, step with dt = 1 ms and
 *     launch on the caller's stream; invalid arguments are reported through
 *     g1b_last_error() instead of being launched.
 *
 *  2. Extended entry points (int status: 0 ok, <0 error, message in
 *     g1b_last_error()): step configuration with dt, per-env friction /
 *     base-mass / servo-gain arrays, the decimated rollout with in-kernel
 *     target redraw and reset, graph-captured persistent execution and the
 *     launch autotuner.
 *
 * Conventions (reference src/g1sim.py:46-53): every array is device float32,
 * SoA with the env axis fastest, array[i * nenv + e]:
 *   qpos [36][nenv]  base pos (3, world), base quat (4, wxyz), 29 hinge angles
 *   qvel [35][nenv]  base lin vel (3, world), base ang vel (3, body), 29 rates
 *   anchor [16][nenv] contact anchors (x, y) per sphere, 1e30 = free
 *   ctrl [29][nenv]  PD position targets
 *   foot_pos, foot_vel [6][nenv]; contact_forces [8][nenv] (all nullable)
 * The caller owns every buffer; the step entry points allocate nothing.
 * Streams are CUDA runtime streams passed as void* (cudaStream_t).
 */
#ifndef G1SIM_B200_H
#define G1SIM_B200_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------ reference GPU ABI ---- */
/* reference src/g1_kernel.cu:154-163 (g1_cuda_step) */
void g1_cuda_step(int nenv, int nsub, float* qpos, float* qvel, float* anchor, const float* ctrl,
                  float* foot_pos, float* foot_vel, float* contact_forces, void* stream);
/* reference src/g1_kernel.cu:165-173 (g1_cuda_reset_done) */
void g1_cuda_reset_done(int nenv, float* qpos, float* qvel, float* anchor, const uint8_t* done,
                        unsigned seed, float noise, float drop, void* stream);

/* ------------------------------------------------- extended entry points */
/* Step configuration; mirrors the reference G1Config (src/g1_types.h:33-42). */
typedef struct g1b_config {
  float gravity_z, contact_kn, contact_dn, contact_kt, contact_dt, limit_kp, limit_kd, dt;
} g1b_config;

/* Decimated-rollout parameters (no reference counterpart: the reference
 * redraws targets and resets envs from Python, examples/train.py:306,336). */
typedef struct g1b_rollout_params {
  unsigned seed;      /* RNG seed of the target redraw and of resets */
  int step0;          /* global index of the first policy step of this call */
  float target_frac;  /* targets = stand + U(-frac, frac) * (hi - lo) */
  float reset_z;      /* reset an env whose base height is below this */
  float z0_lo, z0_hi; /* reset base height U[z0_lo, z0_hi] */
  int redraw;         /* 0: keep ctrl as given */
} g1b_rollout_params;

/* Sizes (reference src/host_lib.cpp:7-10); returns the precision, 4. */
int g1b_sizes(int* nb, int* nq, int* nv, int* nu, int* nc);
/* Reference defaults (src/g1_types.h:44-55), dt = 1 ms. */
int g1b_default_config(g1b_config* out);
const char* g1b_last_error(void);

/* nsub substeps of every env.  mu, dmass, kp_scale, kd_scale: per-env
 * [nenv] arrays, each nullable (defaults 1, 0, 1, 1 = the reference). */
int g1b_step(int nenv, int nsub, const g1b_config* cfg, float* qpos, float* qvel, float* anchor,
             const float* ctrl, const float* mu, const float* dmass, const float* kp_scale,
             const float* kd_scale, float* foot_pos, float* foot_vel, float* contact_forces,
             void* stream);

/* npolicy policy steps of decim substeps: targets redrawn at each policy
 * step (written back to ctrl), env reset in the kernel when its base height
 * is below reset_z; reset_count[nenv] (int, nullable) is incremented per
 * reset.  Outputs as in g1b_step, from the last substep. */
int g1b_rollout(int nenv, int npolicy, int decim, const g1b_config* cfg,
                const g1b_rollout_params* rp, float* qpos, float* qvel, float* anchor, float* ctrl,
                const float* mu, const float* dmass, int* reset_count, float* foot_pos,
                float* foot_vel, float* contact_forces, void* stream);

/* Launch shape of the step kernels.  mapping 0: one thread per env, block =
 * envs (= threads) per block; mapping 1 (default): two threads per env, the
 * lower body (pelvis, legs, contacts, base) and the upper body (waist, arms)
 * on separate warps, block = envs per block (2 * block threads).  block is
 * 32, 64, 96 or 128; blocks_per_sm caps the persistent grid (0 = all that
 * fit).  g1b_autotune times the candidates on the current device for a
 * workload of nenv envs and keeps the fastest; g1b_get_launch reports it. */
int g1b_set_launch(int mapping, int block, int blocks_per_sm);
int g1b_get_launch(int* mapping, int* block, int* blocks_per_sm);
int g1b_autotune(int nenv, int nsub, void* stream, float* best_ms);

/* FP32 FMA throughput microbenchmark (the FP32-pipe roofline denominator):
 * runs a dependent-chain-free FFMA kernel for `iters` iterations per thread
 * on the whole device; writes achieved TFLOP/s (2 flops per FFMA). */
int g1b_ffma_peak(int iters, float* tflops, float* ms);

#ifdef __cplusplus
}
#endif
#endif /* G1SIM_B200_H */
