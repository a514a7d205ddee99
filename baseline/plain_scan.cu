// Plain-GPU comparator only: the reference's plasma density integration
// (media_physics.py:11-67) written naively, one thread per (x, y) line, serial
// over t, strided (uncoalesced) access -- the same launch shape the reference
// uses through cp.RawKernel.
#include <cuda_runtime.h>

__global__ void plain_scan(const float* w_ion, const float* w_ava, double* rho, double* gen,
                           float rate_rec, float dt, float rho_nt, int nt, int nlines) {
  const int line = blockIdx.x * blockDim.x + threadIdx.x;
  if (line >= nlines) return;
  const long long off = (long long)line * nt;
  const double rnt = rho_nt, rr = rate_rec, tdt = dt;
  double r = 0.0;
  for (int t = 0; t < nt; ++t) {
    rho[off + t] = r;
    const double wp = w_ion[off + t], wa = w_ava[off + t];
    double depl = (rnt - r) / rnt;
    depl = depl < 0.0 ? 0.0 : depl;
    gen[off + t] = (wp * rnt + wa * r) * depl;
    const double src = wp * rnt * depl;
    const double g = wa * depl - rr;
    double gdt = g * tdt;
    gdt = gdt > 10.0 ? 10.0 : (gdt < -10.0 ? -10.0 : gdt);
    const double e = exp(gdt);
    const double sf = fabs(gdt) < 1e-5 ? tdt * (1.0 + 0.5 * gdt) : (e - 1.0) / g;
    r = r * e + src * sf;
    r = r > rnt ? rnt : (r < 0.0 ? 0.0 : r);
  }
}

extern "C" int plain_scan_launch(const void* w_ion, const void* w_ava, void* rho, void* gen,
                                 float rate_rec, float dt, float rho_nt, int nt, int nlines,
                                 void* stream) {
  plain_scan<<<(nlines + 255) / 256, 256, 0, (cudaStream_t)stream>>>(
      (const float*)w_ion, (const float*)w_ava, (double*)rho, (double*)gen, rate_rec, dt, rho_nt,
      nt, nlines);
  return (int)cudaGetLastError();
}
