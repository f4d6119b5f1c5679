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
 * on separate warps, block = envs per block (2 * block threads); mapping 2:
 * three threads per env (left leg with the pelvis and base, right leg, upper
 * body), block 64 or 128 (3 * block threads).  block is 32, 64, 96 or 128;
 * blocks_per_sm caps the persistent grid (0 = all that fit).  g1b_autotune
 * times the candidates on the current device for a workload of nenv envs
 * and keeps the fastest; g1b_get_launch reports it. */
int g1b_set_launch(int mapping, int block, int blocks_per_sm);
int g1b_get_launch(int* mapping, int* block, int* blocks_per_sm);
int g1b_autotune(int nenv, int nsub, void* stream, float* best_ms);

/* FP32 FMA throughput microbenchmark (the FP32-pipe roofline denominator):
 * runs a dependent-chain-free FFMA kernel for `iters` iterations per thread
 * on the whole device; writes achieved TFLOP/s (2 flops per FFMA). */
int g1b_ffma_peak(int iters, float* tflops, float* ms);

/* ------------------------------------------------ policy-fused rollout */
/* No reference counterpart as one call: the reference runs the same loop in
 * Python (examples/train.py:262-325: ActorCritic.act, PD targets, pushes,
 * G1Sim.step, get_obs, compute_reward_and_done, resets, command redraws).
 * Here one CTA keeps 128 envs on an SM for all npolicy policy steps; the
 * observation (src/g1sim.py:132-170) is built in shared memory, normalised
 * (examples/train.py:68-69) and fed to the critic and actor MLPs
 * (99-512-256-128-{1,29}, ELU; train.py:16-39) on the tensor cores (BF16
 * operands, FP32 accumulation), then decim substeps run in the same kernel.
 *
 * Network weights in the kernel's layout, packed by g1sim_b200/policy.py
 * from an ActorCritic state dict (train.py:16-47):
 *   weights   BF16, the critic's four layers then the actor's four, each
 *             W (out x in) zero-padded to N x K = 512x112, 256x512,
 *             128x256, {16 | 32}x128 and stored in K-chunks of 16 / 32 /
 *             64 / 128 columns, each chunk as [K/8][N/8][8][8]
 *   bias      FP32, per layer padded to N (critic 912, then actor 928)
 *   log_std   [29], the actor's `std` parameter (sigma = exp(log_std))
 *   obs_mean, obs_var [99]: normaliser statistics, constant during a call
 * All device pointers; weights and bias 16-byte aligned. */
typedef struct g1b_policy {
  const void* weights;
  const float* bias;
  const float* log_std;
  const float* obs_mean;
  const float* obs_var;
} g1b_policy;

/* Per-env task state, SoA [.][nenv], kept by the caller across calls
 * (examples/train.py:257-261: command_timeout, env_episode_length,
 * push_interval; prev_actions :264). */
typedef struct g1b_task_state {
  float* commands;    /* [3][nenv] vx, vy (m/s), yaw rate (rad/s) */
  float* prev_action; /* [29][nenv] raw action of the previous policy step */
  int* cmd_timer;     /* [nenv] policy steps until the command is redrawn */
  int* ep_len;        /* [nenv] policy steps since the last reset */
  int* push_timer;    /* [nenv] policy steps until the next push */
} g1b_task_state;

enum { G1B_SAMPLE = 1, G1B_PUSH = 2, G1B_RESET = 4, G1B_COMMANDS = 8 };

/* Task parameters; g1b_policy_default_params fills the reference values. */
typedef struct g1b_task_params {
  unsigned seed;                     /* RNG seed: action noise, pushes, commands */
  int step0;                         /* global index of the call's first policy step */
  float cmd_lo[3], cmd_hi[3];        /* command draw ranges */
  int cmd_steps_lo, cmd_steps_hi;    /* command redraw interval, U{lo..hi-1} (150, 250) */
  int push_steps_lo, push_steps_hi;  /* push interval (50, 150) */
  float push_vel[6];                 /* push U(-v, v) added to qvel[0:6] */
  int max_episode;                   /* timeout in policy steps (1000) */
  float tilt_limit;                  /* termination tilt in rad (70 deg) */
  unsigned reset_seed;               /* g1_cuda_reset_done seed, noise, drop (42, 0.1, 0.02) */
  float reset_noise, reset_drop;
  int flags;                         /* G1B_SAMPLE | G1B_PUSH | G1B_RESET | G1B_COMMANDS */
} g1b_task_params;

/* Outputs per policy step t of the call, [npolicy][nenv][...] row-major as
 * the reference RolloutBuffer (examples/train.py:94-101); each nullable.
 * last_obs [nenv][99] / last_value [nenv]: observation and critic value of
 * the state after the last step (the bootstrap value, train.py:327-328). */
typedef struct g1b_rollout_out {
  float* obs;        /* observation the action was taken on, raw */
  float* actions;    /* [29] sampled action (network units) */
  float* mean;       /* [29] actor output */
  float* logp;       /* log-probability of the action */
  float* value;      /* critic value */
  float* reward;     /* reward of the transition */
  uint8_t* done;     /* termination (tilt), as buffered by the reference */
  uint8_t* reset;    /* termination or timeout: the env was reset after the step */
  float* last_obs;
  float* last_value;
} g1b_rollout_out;

int g1b_policy_default_params(g1b_task_params* out);
/* Sizes of the packed network: weight bytes, bias floats, obs and action dims. */
int g1b_policy_sizes(int* weight_bytes, int* bias_floats, int* obs_dim, int* act_dim);
/* npolicy policy steps of decim substeps each, on the caller's stream.
 * foot_pos, foot_vel, contact_forces are required (the reward reads them)
 * and hold the last substep's values on return.  npolicy = 0 with
 * last_obs / last_value set evaluates the current state only. */
int g1b_policy_rollout(int nenv, int npolicy, int decim, const g1b_config* cfg, const g1b_task_params* tp,
                       const g1b_policy* pol, float* qpos, float* qvel, float* anchor, float* ctrl,
                       const float* mu, const float* dmass, const g1b_task_state* ts, const g1b_rollout_out* out,
                       float* foot_pos, float* foot_vel, float* contact_forces, void* stream);
/* Device-side status of the policy kernels since the last call (reads a
 * device flag, synchronising the device): 0 ok, 1 a tensor-core pipeline
 * wait timed out and the affected CTAs stopped early.  Clears the flag. */
int g1b_policy_status(int* code);

/* ------------------------------------------------------ horizon adjoint */
/* No reference counterpart: the reference has no derivatives.  Gradient of
 *   L = sum_{t=1..H} (qpos_t[2] - z_ref)^2 + w_track * |qpos_t[7:36] - u_{t-1}|^2
 * over H single-substep steps x_{t+1} = step(x_t, u_t, kp_scale, kd_scale)
 * (x = qpos, qvel, anchor; friction 1, no base-mass offset), with respect
 * to the PD targets u_t, the per-env gain scales and the initial state.
 * One launch per call: the forward rollout keeps a checkpoint every
 * `checkpoint` steps, then each segment is recomputed from its checkpoint
 * and reversed step by step with a hand-derived reverse-mode product of the
 * step (exact to rounding: the derivative of the step as computed,
 * one-sided at contact / clamp switches). */
typedef struct g1b_adjoint_problem {
  int horizon;     /* H */
  int checkpoint;  /* keep the state every `checkpoint` steps */
  float z_ref;     /* base-height reference (0.78) */
  float w_track;   /* weight of the joint tracking term (0.1) */
} g1b_adjoint_problem;
/* Scratch elements (float, or double for the _f64 variant) that g1b_adjoint
 * needs for nenv envs: (ceil(H/C) + 1 + C) * 87 * nenv. */
int g1b_adjoint_scratch_size(int nenv, const g1b_adjoint_problem* pr, size_t* count);
/* Arrays SoA with the env axis fastest: qpos0 [36][nenv], qvel0 [35][nenv],
 * anchor0 [16][nenv], targets / grad_targets [H][29][nenv], kp_scale,
 * kd_scale, loss, grad_kp, grad_kd [nenv] (scales nullable = 1, gain and
 * initial-state gradients nullable), grad_qpos0 [36][nenv], grad_qvel0
 * [35][nenv]; scratch: g1b_adjoint_scratch_size elements, caller-owned. */
int g1b_adjoint(int nenv, const g1b_config* cfg, const g1b_adjoint_problem* pr, const float* qpos0,
                const float* qvel0, const float* anchor0, const float* targets, const float* kp_scale,
                const float* kd_scale, float* loss, float* grad_targets, float* grad_kp, float* grad_kd,
                float* grad_qpos0, float* grad_qvel0, float* scratch, void* stream);
/* The same computation in FP64 on the device (validation build: every array
 * double, cfg converted). */
int g1b_adjoint_f64(int nenv, const g1b_config* cfg, const g1b_adjoint_problem* pr, const double* qpos0,
                    const double* qvel0, const double* anchor0, const double* targets, const double* kp_scale,
                    const double* kd_scale, double* loss, double* grad_targets, double* grad_kp, double* grad_kd,
                    double* grad_qpos0, double* grad_qvel0, double* scratch, void* stream);
/* No counterpart in the reference.  g1b_adjoint for callers that cannot
 * allocate device memory (a real-time loop that reserves everything at
 * start-up, or a host whose device memory is owned by another allocator
 * and that cannot pass a buffer): the same FP32 computation, with the
 * workspace in one fixed device array of g1b_adjoint_noalloc_capacity()
 * floats (8 MiB; at horizon 64 and checkpoint 8 that is up to 1,418 envs)
 * instead of caller scratch.  Larger problems are rejected with a message
 * in g1b_last_error().  The library allocates nothing: every device that
 * loads it holds the array until the process exits.  The first call on a
 * device looks up the array's device address (cudaGetSymbolAddress) with
 * that device current; make that first call before any stream capture.
 * All calls on a device share the one array: calls that overlap on the GPU
 * (other streams, other host threads) race and corrupt each other's
 * results; serialise them. */
size_t g1b_adjoint_noalloc_capacity(void);
int g1b_adjoint_noalloc(int nenv, const g1b_config* cfg, const g1b_adjoint_problem* pr, const float* qpos0,
                        const float* qvel0, const float* anchor0, const float* targets, const float* kp_scale,
                        const float* kd_scale, float* loss, float* grad_targets, float* grad_kp, float* grad_kd,
                        float* grad_qpos0, float* grad_qvel0, void* stream);

/* ------------------------------------------------- dynamics surrogate */
/* No reference counterpart (the learned surrogate of the workload
 * configuration).  BF16 tcgen05 GEMM, FP32 accumulation, persistent (one
 * CTA per SM), operands loaded by TMA:
 *   C[M x N] = A[M x K] . B[N x K]^T (+ bias[N]), A, B row-major with K
 *   contiguous; splits > 1 selects the K-split form for small outputs of
 *   long products: the (tile, 64-wide K chunk) pairs are shared evenly by
 *   the SMs and their partial tiles added into C atomically (C cleared
 *   first; the sum order, and so the last bits, vary from call to call).
 *   M % 128 == 0, N % 16 == 0 (N % 256 == 0 above 256), K % 64 == 0,
 *   lda / ldb multiples of 8 and >= K, ldc a multiple of 4 and >= N,
 *   16-byte aligned pointers. */
int g1b_gemm_bf16(int M, int N, int K, const void* A, int lda, const void* B, int ldb, float* C, int ldc,
                  const float* bias, int splits, void* stream);
/* C[M x N] += A[M x K] . B[N x K]^T, K shared evenly by the SMs (the split
 * form of g1b_gemm_bf16 without clearing C first): for gradients summed
 * into buffers the caller zeroes once for several products. */
int g1b_gemm_bf16_acc(int M, int N, int K, const void* A, int lda, const void* B, int ldb, float* C, int ldc,
                      void* stream);
/* C[M x N] += A[K x M]^T . B[K x N] with A and B row-major (K the rows):
 * the weight gradient dW += dZ^T . H read from the activations as the layers
 * store them (no transposed copies), K shared evenly by the SMs as in
 * g1b_gemm_bf16_acc.  M % 16 == 0, N % 64 == 0 (N % 256 == 0 above 256),
 * K % 64 == 0, lda >= M and ldb >= N multiples of 8, ldc a multiple of 4
 * and >= N, 16-byte aligned pointers. */
int g1b_gemm_bf16_atb_acc(int M, int N, int K, const void* A, int lda, const void* B, int ldb, float* C, int ldc,
                          void* stream);
/* One hidden layer of the surrogate in one GEMM with a fused epilogue
 * (same shape rules; ldh and ldz multiples of 8, ldt >= M):
 *   z = A . W^T + bias (W [N x K]); Z = z (FP16 [M][ldz], |z| clamped to
 *   65000, nullable), H = bf16(silu(z)) [M][ldh], Ht = H transposed
 *   [N][ldt] (nullable). */
int g1b_sur_linear_silu(int M, int N, int K, const void* A, int lda, const void* W, int ldw, const float* bias,
                        void* Z, int ldz, void* H, int ldh, void* Ht, int ldt, void* stream);
/* Its backward through the previous layer's activation: with Wt [N x K]
 * (the layer's weight transposed) and Z [M][ldz] (FP16) the previous
 * layer's pre-activation, g = (dZ . Wt^T) * silu'(Z); dH = bf16(g)
 * [M][ldh], dHt = dH transposed [N][ldt] (nullable), db[N] += column sums
 * of g (FP32, nullable).  dH must not alias dZ. */
int g1b_sur_linear_silu_bwd(int M, int N, int K, const void* dZ, int ldd, const void* Wt, int ldw, const void* Z,
                            int ldz, void* dH, int ldh, void* dHt, int ldt, float* db, void* stream);
/* Device status of the GEMM kernels since the last call (synchronises):
 * 0 ok, 1 a pipeline wait timed out.  Clears the flag. */
int g1b_gemm_status(int* code);
/* The optimiser step of the surrogate in one launch: Adam (b1, b2, eps;
 * the step count t and the learning rate read from device memory, t >= 1)
 * on every layer's FP32 weights and biases with their gradients gW
 * (leading rows x cols entries) and gb, then the BF16 copies Wb [rows][cols]
 * and Wt [cols][rows] of each updated weight.  At most 8 layers. */
typedef struct g1b_sur_layer {
  float *W, *b, *mW, *vW, *mb, *vb;
  const float *gW, *gb;
  void *Wb, *Wt;
  int rows, cols;
} g1b_sur_layer;
int g1b_sur_adam_cast(int nl, const g1b_sur_layer* layers, const int* step, const float* lr, float b1, float b2,
                      float eps, void* stream);
/* Element-wise kernels of the surrogate: weighted MSE and its gradient
 * dY [B][D] (BF16; dYt, its transpose [D][B], nullable; adds into db and
 * loss; D divides 256 and is a multiple of 8), BF16 weight copies. */
int g1b_sur_loss(int B, int D, const float* Y, const float* T, const float* w, void* dY, void* dYt, float* db,
                 float* loss, void* stream);
int g1b_sur_cast(int rows, int cols, const float* W, void* Wb, void* Wt, void* stream);
/* The surrogate's input features of n envs (159 used of 192: joint angles
 * and rates, base height, rotation, body-frame velocities, per foot sphere
 * its penetration depth, contact flag, offset from its anchor and world
 * velocity, targets, friction, base-mass offset, 1), normalised with
 * (mean, istd) into BF16 X [n][192] (Xt [192][n] and raw F [n][192]
 * nullable).  State SoA as in g1b_step; mu, dmass [n] nullable (1, 0). */
int g1b_sur_features(int n, const float* qpos, const float* qvel, const float* anchor, const float* ctrl,
                     const float* mu, const float* dmass, const float* mean, const float* istd, void* X, void* Xt,
                     float* F, void* stream);
/* Adjoint of the features: dX [n][ld] (FP32) is the adjoint of the
 * normalised inputs; adds the state adjoint into qpos_b [36][n], qvel_b
 * [35][n], anchor_b [16][n] (nullable) and the targets' into ctrl_b [29][n]. */
int g1b_sur_features_vjp(int n, const float* qpos, const float* qvel, const float* anchor, const float* istd,
                         const float* dX, int ld, float* qpos_b, float* qvel_b, float* anchor_b, float* ctrl_b,
                         void* stream);
/* The surrogate's state update in place (qacc = Y * ostd + omean, then the
 * step's semi-implicit Euler), and its adjoint at the state before the
 * update: lam_qpos / lam_qvel hold the adjoint of the updated state and are
 * replaced by the adjoint through the update; dY [n][ldd] gets the adjoint
 * of the normalised network output. */
int g1b_sur_integrate(int n, const float* Y, int ldy, const float* omean, const float* ostd, float dt, float* qpos,
                      float* qvel, void* stream);
int g1b_sur_integrate_vjp(int n, const float* qpos, const float* qvel, const float* Y, int ldy, const float* omean,
                          const float* ostd, float dt, float* lam_qpos, float* lam_qvel, float* dY, int ldd,
                          void* stream);
/* BF16 copy of `total` FP32 values (the seed of the network's input-gradient
 * products). */
int g1b_sur_seed(int total, const float* dY, void* dZ, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* G1SIM_B200_H */
