// g1_step_k64.cu -- plain step kernels for the launch shape of 64 envs per CTA.
#include "g1_step_kernels.cuh"

namespace g1b {
G1B_STEP_INSTANCE(64)
}  // namespace g1b
