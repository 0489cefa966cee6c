// Launch entry points of the fused step kernel, one pair per (CTA size,
// precision, dynamic spacing) instance.  Each instance is compiled as its own
// translation unit (mf_kernels.cu with MF_NT / MF_P / MF_D defined) so that
// the twenty instances build in parallel; mf_api.cu dispatches to them.
#pragma once
#include <cuda_runtime.h>
#include "mf_step.cuh"

namespace mf {

#define MF_FOR_EACH_INSTANCE_D(X, D) \
  X(128, 0, D) X(128, 1, D) X(256, 0, D) X(256, 1, D) X(384, 0, D) X(384, 1, D) X(512, 0, D) X(512, 1, D) \
  X(1024, 0, D) X(1024, 1, D)
#define MF_FOR_EACH_INSTANCE(X) MF_FOR_EACH_INSTANCE_D(X, 0) MF_FOR_EACH_INSTANCE_D(X, 1)

// prepare: raise the instance's dynamic shared-memory limit (not capturable,
// so done before any graph capture); launch: <<<grid, NT, smem, st>>>.
#define MF_DECLARE_INSTANCE(NT, P, D)                                                       \
  cudaError_t prepare_##NT##_##P##_##D(size_t smem);                                       \
  cudaError_t launch_##NT##_##P##_##D(const StepArgs& a, int grid, int base, size_t smem, cudaStream_t st);
MF_FOR_EACH_INSTANCE(MF_DECLARE_INSTANCE)

// The caller-owned-state kernel (mf_state.cuh), float32 only: one instance per
// (CTA size, dynamic spacing), compiled in the float32 step kernel's unit.
struct StateIO;
#define MF_FOR_EACH_STATE_INSTANCE(X) \
  X(128, 0) X(256, 0) X(384, 0) X(512, 0) X(1024, 0) X(128, 1) X(256, 1) X(384, 1) X(512, 1) X(1024, 1)
#define MF_DECLARE_STATE_INSTANCE(NT, D)                     \
  cudaError_t prepare_state_##NT##_##D(size_t smem);         \
  cudaError_t launch_state_##NT##_##D(const StepArgs& a, const StateIO& io, int grid, size_t smem, cudaStream_t st);
MF_FOR_EACH_STATE_INSTANCE(MF_DECLARE_STATE_INSTANCE)

}  // namespace mf
