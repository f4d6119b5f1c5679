// g1_step_k128.cu -- plain step kernels for the launch shape of 128 envs per CTA.
#include "g1_step_kernels.cuh"

namespace g1b {
G1B_STEP_INSTANCE(128)
}  // namespace g1b
