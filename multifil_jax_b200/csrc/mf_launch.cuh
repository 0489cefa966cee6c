// Launch entry points of the fused step kernel, one pair per (CTA size,
// precision) instance.  Each instance is compiled as its own translation unit
// (mf_kernels.cu with MF_NT / MF_P defined) so that the ten instances build in
// parallel; mf_api.cu dispatches to them.
#pragma once
#include <cuda_runtime.h>
#include "mf_step.cuh"

namespace mf {

#define MF_FOR_EACH_INSTANCE(X) \
  X(128, 0) X(128, 1) X(256, 0) X(256, 1) X(384, 0) X(384, 1) X(512, 0) X(512, 1) X(1024, 0) X(1024, 1)

// prepare: raise the instance's dynamic shared-memory limit (not capturable,
// so done before any graph capture); launch: <<<grid, NT, smem, st>>>.
#define MF_DECLARE_INSTANCE(NT, P)                                                          \
  cudaError_t prepare_##NT##_##P(size_t smem);                                             \
  cudaError_t launch_##NT##_##P(const StepArgs& a, int grid, int base, size_t smem, cudaStream_t st);
MF_FOR_EACH_INSTANCE(MF_DECLARE_INSTANCE)

}  // namespace mf
