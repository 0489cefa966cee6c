// One instance of the fused step kernel: step_kernel<MF_NT, MF_P, MF_D> and
// its launch entry points (declared in mf_launch.cuh).  Built once per
// instance:
//   nvcc ... -DMF_NT=256 -DMF_P=1 -DMF_D=0 -c mf_kernels.cu
#include "mf_kernel.cuh"
#include "mf_launch.cuh"
#include "mf_state.cuh"

#if !defined(MF_NT) || !defined(MF_P) || !defined(MF_D)
#error "compile with -DMF_NT=<CTA size> -DMF_P=<0|1> -DMF_D=<0|1>"
#endif

#define MF_PASTE(a, b, c, d) a##b##_##c##_##d
#define MF_NAME(a, b, c, d) MF_PASTE(a, b, c, d)

namespace mf {

cudaError_t MF_NAME(prepare_, MF_NT, MF_P, MF_D)(size_t smem) {
  auto* kernel = step_kernel<MF_NT, (MF_P != 0), (MF_D != 0)>;
  // Function attributes belong to the device's context, so what has been set
  // is remembered per device.
  constexpr int kDevices = 64;
  static size_t attr_bytes[kDevices] = {};
  static int sm_bytes[kDevices] = {}, set_pct[kDevices] = {};  // set_pct: carve-out + 1, 0 = never set
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kDevices) return cudaErrorInvalidDevice;
  if (smem > attr_bytes[dev]) {
    e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    attr_bytes[dev] = smem;
  }
  // Shared-memory carve-out: just what the register-limited occupancy needs
  // (static and driver-reserved bytes included), so the rest of the SM's
  // 256 KB stays L1, where the spilled registers live.
  if (!sm_bytes[dev]) {
    if (cudaDeviceGetAttribute(&sm_bytes[dev], cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) != cudaSuccess ||
        sm_bytes[dev] <= 0)
      sm_bytes[dev] = 233472;
  }
  const size_t need = (size_t)min_ctas(MF_NT) * (smem + kStaticSmem + 1024);
  int pct = (int)((need * 100 + sm_bytes[dev] - 1) / (size_t)sm_bytes[dev]);
  pct = pct > 100 ? 100 : pct;
  if (pct + 1 != set_pct[dev]) {
    e = cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, pct);
    if (e != cudaSuccess) return e;
    set_pct[dev] = pct + 1;
  }
  return cudaSuccess;
}

cudaError_t MF_NAME(launch_, MF_NT, MF_P, MF_D)(const StepArgs& a, int grid, int base, size_t smem, cudaStream_t st) {
  step_kernel<MF_NT, (MF_P != 0), (MF_D != 0)><<<grid, MF_NT, smem, st>>>(a, base);
  return cudaPeekAtLastError();
}

#if MF_P == 0
#define MF_SNAME(a, b, c) MF_SPASTE(a, b, c)
#define MF_SPASTE(a, b, c) a##b##_##c
// The caller-owned-state kernel of this CTA size and spacing mode: its shared
// memory limit is raised on first use per device.
cudaError_t MF_SNAME(prepare_state_, MF_NT, MF_D)(size_t smem) {
  constexpr int kDevices = 64;
  static size_t attr_bytes[kDevices] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kDevices) return cudaErrorInvalidDevice;
  if (smem > attr_bytes[dev]) {
    e = cudaFuncSetAttribute(state_kernel<MF_NT, (MF_D != 0)>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    attr_bytes[dev] = smem;
  }
  return cudaSuccess;
}

cudaError_t MF_SNAME(launch_state_, MF_NT, MF_D)(const StepArgs& a, const StateIO& io, int grid, size_t smem,
                                                  cudaStream_t st) {
  state_kernel<MF_NT, (MF_D != 0)><<<grid, MF_NT, smem, st>>>(a, io);
  return cudaPeekAtLastError();
}
#endif

}  // namespace mf
