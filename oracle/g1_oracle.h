/* g1_oracle.h -- FP64 CPU oracle of the batched G1 step.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA path:
 * only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline /
 * --impl reference legs may load it.  The product (g1sim_b200/) never links
 * or calls it.
 *
 * It restates, in plain C99 doubles, the reference's host-compiled physics
 * (reference: src/spatial.h, src/g1_core.h, src/host_lib.cpp) and exports the
 * reference's host ABI names (src/host_lib.cpp:5-55) so that tests written
 * against the reference's libg1host.so read the same.  The g1o_* entry
 * points extend it with what the configurations need: a step config with dt,
 * per-env friction / base-mass offset / servo gain scales, SoA batches, the
 * in-kernel reset and the decimated rollout with target redraw.
 *
 * Parity pin: tests/golden/ holds vectors produced by the reference's own
 * host_lib.cpp compiled at G1_PRECISION=8 (oracle/Makefile, target ref);
 * tests/test_oracle_golden.py checks this oracle against them.
 */
#ifndef G1_ORACLE_H
#define G1_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* G1Config (reference: src/g1_types.h:33-42). */
typedef struct {
  double gravity_z, contact_kn, contact_dn, contact_kt, contact_dt;
  double limit_kp, limit_kd, dt;
} g1o_config;

/* Per-env parameters; the reference has none of these (its model constants
 * are compile-time).  Defaults {1, 0, 1, 1} reproduce the reference. */
typedef struct {
  double mu;        /* Coulomb friction coefficient (reference g1_contact_mu) */
  double dmass;     /* added to the pelvis mass (body 0) */
  double kp_scale;  /* multiplies every servo kp */
  double kd_scale;  /* multiplies every servo kv (and its implicit damping) */
} g1o_envparams;

/* Reference host ABI (src/host_lib.cpp:7-53). */
int g1_sizes(int* nb, int* nq, int* nv, int* nu, int* nc);
void g1_c_fk(const double* qpos, double* xpos, double* xmat);
void g1_c_fd(const double* qpos, const double* qvel, const double* tau, double* qacc);
void g1_c_step(double* qpos, double* qvel, const double* ctrl, int nsub, double dt,
               double* fn_out, double* anchor);

void g1o_default_config(g1o_config* cfg);
void g1o_default_envparams(g1o_envparams* ep);

/* One env, AoS doubles.  nsub substeps; fn_out[8], foot_pos[6], foot_vel[6]
 * come from the last substep (its pre-integration kinematics), all nullable. */
void g1o_step(const g1o_config* cfg, const g1o_envparams* ep, double* qpos, double* qvel,
              const double* ctrl, double* anchor, int nsub, double* fn_out,
              double* foot_pos, double* foot_vel);

/* SoA batch, array[i*nenv + e], the CUDA path's layout in doubles.
 * mu / dmass / kp_scale / kd_scale are per-env arrays, each nullable. */
void g1o_step_soa(int nenv, int nsub, const g1o_config* cfg, double* qpos, double* qvel,
                  double* anchor, const double* ctrl, const double* mu, const double* dmass,
                  const double* kp_scale, const double* kd_scale,
                  double* foot_pos, double* foot_vel, double* contact_forces);

/* Per-env distance of the next substep from the model's branch thresholds
 * (contact touchdown, force clamps, stick/slip, soft limits, torque clamp),
 * normalised by FP32 rounding there; < 1 means an FP32 step may take the
 * other branch.  Used by the parity tests to set such steps apart. */
void g1o_branch_margin_soa(int nenv, const g1o_config* cfg, const double* qpos,
                           const double* qvel, const double* anchor, const double* ctrl,
                           const double* mu, const double* dmass, double* margin);

/* Reset of the envs with done[e] != 0 (reference: src/g1_kernel.cu:85-103),
 * computed in float exactly as the CUDA kernel computes it, widened to
 * double on store.  SoA doubles. */
void g1o_reset_done_soa(int nenv, double* qpos, double* qvel, double* anchor,
                        const uint8_t* done, unsigned seed, float noise, float drop);

/* Counter-based RNG shared with the CUDA path (float uniform in [0,1)). */
unsigned g1o_hash(unsigned x);
float g1o_uniform(unsigned seed, unsigned stream, unsigned counter);

/* Decimated rollout with per-env randomisation (the 65,536-env workload):
 * npolicy policy steps of decim substeps.  At the start of policy step k the
 * PD targets are redrawn, ctrl[j] = stand[7+j] + (2u-1)*target_frac*(hi-lo)
 * with u = g1o_uniform(seed, e, (step0+k)*64 + j); after the decim substeps
 * an env whose base height is below reset_z is reset to the stand pose with
 * base height z0_lo + u*(z0_hi-z0_lo), u = g1o_uniform(seed ^ 0x5bd1e995,
 * e, step0+k), zero velocity and free anchors.  reset_count[e] (nullable)
 * counts the resets.  ctrl is written back (the last targets drawn). */
typedef struct {
  unsigned seed;
  int step0;           /* global index of the first policy step */
  float target_frac;   /* 0.3 */
  float reset_z;       /* 0.3 */
  float z0_lo, z0_hi;  /* 0.75, 0.85 */
  int redraw;          /* 0: keep ctrl fixed (no redraw) */
} g1o_rollout_params;

void g1o_rollout_soa(int nenv, int npolicy, int decim, const g1o_config* cfg,
                     const g1o_rollout_params* rp, double* qpos, double* qvel,
                     double* anchor, double* ctrl, const double* mu, const double* dmass,
                     int* reset_count);

/* Targets drawn for policy step `step` (float, bit-exact with the GPU). */
void g1o_draw_targets(int nenv, unsigned seed, int step, float target_frac, float* ctrl_f);

#ifdef __cplusplus
}
#endif
#endif
