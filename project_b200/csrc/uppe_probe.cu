// Access-pattern bandwidth probe: a measurement hook for bench.py.
//
// The 3+1D passes move whole fields between HBM and the SMs with three access
// patterns: the t-line kernel streams contiguous lines; the x passes read and
// write tiles of kW omega columns (8 kW contiguous bytes) from 256 rows that lie
// Ny * Nt elements apart; the y passes the same tiles from rows Nt elements apart.
// uppe_pattern_probe copies one 256 x 256 x Nt complex64 field with exactly one of
// those patterns (each thread loads its 16 rows, adds 1 to one component, stores
// them; no transform), so the time of a pass can be set against what its access
// pattern alone reaches on the device it runs on.
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include "../../include/uppe_b200.h"

extern char g_uppe_err[512];

namespace uppe {

template <int KW, bool XPAT>
__global__ void __launch_bounds__(KW * 16) k_probe_tile(const float2* __restrict__ in, float2* __restrict__ out,
                                                       int nt) {
  constexpr int N = 256;
  const int tid = threadIdx.x, w = tid % KW, j = tid / KW;
  const int ntile = nt / KW;
  const int o = blockIdx.x / ntile, w0 = (blockIdx.x % ntile) * KW;
  const long long stride = XPAT ? (long long)N * nt : nt;
  const long long base = (XPAT ? (long long)o * nt : (long long)o * N * nt) + w0 + w;
  float2 v[16];
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __ldg(in + base + (long long)(j + 16 * i) * stride);
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i].x += 1.f;
#pragma unroll
  for (int i = 0; i < 16; ++i) out[base + (long long)(j + 16 * i) * stride] = v[i];
}

__global__ void k_probe_seq(const float4* __restrict__ in, float4* __restrict__ out, long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    float4 v = in[i];
    v.x += 1.f;
    out[i] = v;
  }
}

template <int KW>
static void probe_tile(int xpat, const void* in, void* out, int nt, cudaStream_t s) {
  const unsigned nb = (unsigned)(256 * (nt / KW));
  if (xpat) k_probe_tile<KW, true><<<nb, KW * 16, 0, s>>>((const float2*)in, (float2*)out, nt);
  else k_probe_tile<KW, false><<<nb, KW * 16, 0, s>>>((const float2*)in, (float2*)out, nt);
}

}  // namespace uppe

extern "C" int uppe_pattern_probe(int pattern, int kw, const void* in, void* out, int nt, uppe_stream_t stream) {
  using namespace uppe;
  cudaStream_t s = (cudaStream_t)stream;
  if (!in || !out || in == out || nt < 64 || (nt & (nt - 1)) || pattern < 0 || pattern > 2 ||
      (pattern > 0 && kw != 8 && kw != 16 && kw != 32) || (reinterpret_cast<uintptr_t>(in) % 16) ||
      (reinterpret_cast<uintptr_t>(out) % 16)) {
    snprintf(g_uppe_err, sizeof(g_uppe_err), "uppe_pattern_probe: invalid arguments");
    return UPPE_ERR_ARG;
  }
  if (pattern == 0) {
    const long long n4 = 256LL * 256 * nt / 2;   // float4 = two complex64
    k_probe_seq<<<148 * 8, 512, 0, s>>>((const float4*)in, (float4*)out, n4);
  } else if (kw == 8) {
    probe_tile<8>(pattern == 1, in, out, nt, s);
  } else if (kw == 16) {
    probe_tile<16>(pattern == 1, in, out, nt, s);
  } else {
    probe_tile<32>(pattern == 1, in, out, nt, s);
  }
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    snprintf(g_uppe_err, sizeof(g_uppe_err), "uppe_pattern_probe: %s", cudaGetErrorString(e));
    return UPPE_ERR_CUDA;
  }
  return 0;
}
