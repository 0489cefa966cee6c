// One instance of the fused step kernel: step_kernel<MF_NT, MF_P, MF_D> and
// its launch entry points (declared in mf_launch.cuh).  Built once per
// instance:
//   nvcc ... -DMF_NT=256 -DMF_P=1 -DMF_D=0 -c mf_kernels.cu
#include "mf_kernel.cuh"
#include "mf_launch.cuh"

#if !defined(MF_NT) || !defined(MF_P) || !defined(MF_D)
#error "compile with -DMF_NT=<CTA size> -DMF_P=<0|1> -DMF_D=<0|1>"
#endif

#define MF_PASTE(a, b, c, d) a##b##_##c##_##d
#define MF_NAME(a, b, c, d) MF_PASTE(a, b, c, d)

namespace mf {

cudaError_t MF_NAME(prepare_, MF_NT, MF_P, MF_D)(size_t smem) {
  auto* kernel = step_kernel<MF_NT, (MF_P != 0), (MF_D != 0)>;
  static size_t attr_bytes = 0;
  if (smem > attr_bytes) {
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    attr_bytes = smem;
  }
  // Shared-memory carve-out: just what the register-limited occupancy needs
  // (static and driver-reserved bytes included), so the rest of the SM's
  // 256 KB stays L1, where the spilled registers live.
  static int sm_bytes = 0, last_pct = -1;
  if (!sm_bytes) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&sm_bytes, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) != cudaSuccess ||
        sm_bytes <= 0)
      sm_bytes = 233472;
  }
  const size_t need = (size_t)min_ctas(MF_NT) * (smem + kStaticSmem + 1024);
  int pct = (int)((need * 100 + sm_bytes - 1) / (size_t)sm_bytes);
  pct = pct > 100 ? 100 : pct;
  if (pct != last_pct) {
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, pct);
    if (e != cudaSuccess) return e;
    last_pct = pct;
  }
  return cudaSuccess;
}

cudaError_t MF_NAME(launch_, MF_NT, MF_P, MF_D)(const StepArgs& a, int grid, int base, size_t smem, cudaStream_t st) {
  step_kernel<MF_NT, (MF_P != 0), (MF_D != 0)><<<grid, MF_NT, smem, st>>>(a, base);
  return cudaPeekAtLastError();
}

}  // namespace mf
