// g1_step_k96.cu -- plain step kernels for the launch shape of 96 envs per CTA.
#include "g1_step_kernels.cuh"

namespace g1b {
G1B_STEP_INSTANCE(96)
}  // namespace g1b
