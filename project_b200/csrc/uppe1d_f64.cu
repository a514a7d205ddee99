// double instantiation of the 1D persistent kernel (compiled separately so the
// two precisions build in parallel).
#include "uppe1d_kernel.cuh"

namespace uppe {
template <>
cudaError_t launch_uppe1d<double>(const Batch1D& b, int nblocks, size_t smem, cudaStream_t s) {
  cudaError_t e = cudaFuncSetAttribute(k_uppe1d<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  k_uppe1d<double><<<nblocks, T1, smem, s>>>(b);
  return cudaGetLastError();
}
cudaError_t launch_uppe1d_adjoint(const Adj1D& a, size_t smem, cudaStream_t s) {
  cudaError_t e = cudaFuncSetAttribute(k_uppe1d_adjoint, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  k_uppe1d_adjoint<<<1, T1, smem, s>>>(a);
  return cudaGetLastError();
}
}  // namespace uppe
