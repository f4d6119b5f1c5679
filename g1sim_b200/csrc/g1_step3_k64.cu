// g1_step3_k64.cu -- the three-role step kernels for 64 envs per CTA.
#include "g1_step_kernels.cuh"

namespace g1b {
G1B_STEP3_INSTANCE(64)
}  // namespace g1b
