// float instantiation of the 1D cluster kernel (one translation unit per
// precision, so they build in parallel with the single-CTA kernel).
#include "uppe1d_cluster.cuh"

namespace uppe {
template <int CS>
static cudaError_t launch_cs(const Batch1D& b, int nclusters, size_t smem, cudaStream_t s) {
  cudaError_t e = cudaFuncSetAttribute(k_uppe1d_cl<float, CS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  k_uppe1d_cl<float, CS><<<nclusters * CS, T1, smem, s>>>(b);
  return cudaGetLastError();
}
template <>
cudaError_t launch_uppe1d_cl<float>(const Batch1D& b, int nclusters, size_t smem, cudaStream_t s, int cs) {
  return cs == 8 ? launch_cs<8>(b, nclusters, smem, s) : launch_cs<4>(b, nclusters, smem, s);
}
template <int CS>
static int max_clusters_cs(size_t smem) {
  if (cudaFuncSetAttribute(k_uppe1d_cl<float, CS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return 0;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(CS);
  cfg.blockDim = dim3(T1);
  cfg.dynamicSmemBytes = smem;
  int n = 0;
  if (cudaOccupancyMaxActiveClusters(&n, k_uppe1d_cl<float, CS>, &cfg) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}
template <>
int uppe1d_cl_max_clusters<float>(size_t smem, int cs) {
  return cs == 8 ? max_clusters_cs<8>(smem) : max_clusters_cs<4>(smem);
}
}  // namespace uppe
