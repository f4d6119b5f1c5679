// g1_step_launch.h -- launchers of the plain step kernels, one explicit
// specialisation per launch shape in g1_step_k{32,64,96,128}.cu.
#pragma once
#include <cuda_runtime.h>

#include "g1_env.cuh"

namespace g1b {
// mapping 0: one thread per env (BLOCK threads and envs per CTA)
template <int BLOCK>
int run_single(bool rollout, const StateArgs& a, float* ctrl, int* rc, int nouter, int ninner,
               const StepConfig& cfg, const RolloutParams& rp, cudaStream_t s, int bps);
// mapping 1: two threads per env (ENVS envs, 2 ENVS threads per CTA)
template <int ENVS>
int run_split(bool rollout, const StateArgs& a, float* ctrl, int* rc, int nouter, int ninner,
              const StepConfig& cfg, const RolloutParams& rp, cudaStream_t s, int bps);
// mapping 2: three threads per env (ENVS envs, 3 ENVS threads per CTA)
template <int ENVS>
int run_split3(bool rollout, const StateArgs& a, float* ctrl, int* rc, int nouter, int ninner,
               const StepConfig& cfg, const RolloutParams& rp, cudaStream_t s, int bps);
template <> int run_split3<64>(bool, const StateArgs&, float*, int*, int, int, const StepConfig&, const RolloutParams&, cudaStream_t, int);
template <> int run_split3<128>(bool, const StateArgs&, float*, int*, int, int, const StepConfig&, const RolloutParams&, cudaStream_t, int);
template <> int run_single<32>(bool, const StateArgs&, float*, int*, int, int, const StepConfig&, const RolloutParams&, cudaStream_t, int);
template <> int run_single<64>(bool, const StateArgs&, float*, int*, int, int, const StepConfig&, const RolloutParams&, cudaStream_t, int);
template <> int run_single<96>(bool, const StateArgs&, float*, int*, int, int, const StepConfig&, const RolloutParams&, cudaStream_t, int);
template <> int run_single<128>(bool, const StateArgs&, float*, int*, int, int, const StepConfig&, const RolloutParams&, cudaStream_t, int);
template <> int run_split<32>(bool, const StateArgs&, float*, int*, int, int, const StepConfig&, const RolloutParams&, cudaStream_t, int);
template <> int run_split<64>(bool, const StateArgs&, float*, int*, int, int, const StepConfig&, const RolloutParams&, cudaStream_t, int);
template <> int run_split<96>(bool, const StateArgs&, float*, int*, int, int, const StepConfig&, const RolloutParams&, cudaStream_t, int);
template <> int run_split<128>(bool, const StateArgs&, float*, int*, int, int, const StepConfig&, const RolloutParams&, cudaStream_t, int);
}  // namespace g1b
