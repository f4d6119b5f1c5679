// g1_step3_k128.cu -- the three-role step kernels for 128 envs per CTA.
#include "g1_step_kernels.cuh"

namespace g1b {
G1B_STEP3_INSTANCE(128)
}  // namespace g1b
