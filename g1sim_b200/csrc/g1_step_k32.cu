// g1_step_k32.cu -- plain step kernels for the launch shape of 32 envs per CTA.
#include "g1_step_kernels.cuh"

namespace g1b {
G1B_STEP_INSTANCE(32)
}  // namespace g1b
