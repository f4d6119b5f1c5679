// ref_kernel_shim.cpp -- exposes the REFERENCE's GPU ABI kernels, compiled for
// the CPU through the reference's own fake-CUDA shim, as a shared library for
// golden-vector generation (TEST INFRASTRUCTURE; oracle/Makefile target `ref`).
//
// The reference's FAKE_CUDA g1_cuda_step / g1_cuda_reset_done call the
// kernel body once (env 0 only); these wrappers launch it over the whole
// grid with the reference's own G1_LAUNCH macro (src/g1_kernel.cu:25-41).
#include "g1_kernel.cu"

extern "C" {
void ref_cuda_step(int nenv, int nsub, float* qpos, float* qvel, float* anchor,
                   const float* ctrl, float* foot_pos, float* foot_vel,
                   float* contact_forces) {
  int tpb = 128, nblocks = (nenv + tpb - 1) / tpb;
  G1Config cfg = g1_default_config();
  G1_LAUNCH(g1_step_kernel, nblocks, tpb, nenv, nsub, cfg, qpos, qvel, anchor, ctrl,
            foot_pos, foot_vel, contact_forces);
}
void ref_cuda_reset_done(int nenv, float* qpos, float* qvel, float* anchor,
                         const uint8_t* done, unsigned seed, float noise, float drop) {
  int tpb = 128, nblocks = (nenv + tpb - 1) / tpb;
  G1_LAUNCH(g1_reset_done_kernel, nblocks, tpb, nenv, qpos, qvel, anchor, done, seed,
            noise, drop);
}
}
