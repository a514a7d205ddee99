// Allocation-free entry point for one 1D propagation.
//
// Some callers cannot allocate device memory: code that runs inside a host
// framework which owns the CUDA allocator and forbids cudaMalloc from plug-ins,
// real-time or embedded hosts that must not allocate after start-up, and
// callers that only hold device pointers handed to them by another runtime.
// For them this file provides uppe1d_propagate_noalloc: the same persistent
// kernel as uppe1d_propagate, but the per-call device state it needs (instance
// record, result record, work-queue counter, FFT twiddles and the seven stage
// arrays) lives in one file-scope __device__ array of fixed size instead of
// plan-owned allocations.  Every GPU that loads the library holds that array
// (UPPE_NOALLOC_SCRATCH_BYTES) until the process exits.
//
// Set-up: the first call on a device resolves the array's device address with
// cudaGetSymbolAddress while that device is current and caches it; make that
// first call before any stream capture.  All calls share the one array and it
// keeps the last call's contents, so calls that overlap on the GPU (different
// streams, or different host threads on the same device) race; serialise them.
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <string.h>

#include "uppe1d_kernel.cuh"

extern char g_uppe_err[512];

namespace {

using namespace uppe;

constexpr size_t kHeader = 1024;                     // Inst1D, Res1D, order, counter
constexpr size_t kInstOff = 0, kResOff = 512, kOrderOff = 768, kCounterOff = 772;
static_assert(sizeof(Inst1D) <= kResOff - kInstOff, "Inst1D does not fit its slot");
static_assert(sizeof(Res1D) <= kOrderOff - kResOff, "Res1D does not fit its slot");

// Largest line: 7 stage arrays + 2 N twiddles of N complex values.
static_assert(UPPE_NOALLOC_SCRATCH_BYTES ==
                  kHeader + 9ull * UPPE_NOALLOC_MAX_NT_C128 * 16ull,
              "scratch size and the complex128 limit disagree");
static_assert(9ull * UPPE_NOALLOC_MAX_NT_C64 * 8ull <= UPPE_NOALLOC_SCRATCH_BYTES - kHeader,
              "the complex64 limit does not fit the scratch array");

static __device__ __align__(256) unsigned char g_noalloc_scratch[UPPE_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
static void* g_scratch_addr[kMaxDevices];   // device address per device ordinal

// Packed per-pass line-FFT twiddles for n = 1, 2, 4, ..., nmax at offset n - 1 (slot j
// of size n holds exp(-2 pi i m / n), m = line_twiddle_source(n, j)), written
// straight into the static array (this kernel names it directly).
template <typename C>
__global__ void k_noalloc_twiddles(size_t byte_off, int nmax) {
  C* tw = reinterpret_cast<C*>(g_noalloc_scratch + byte_off);
  const int total = 2 * nmax - 1;
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < total; p += gridDim.x * blockDim.x) {
    const int n = 1 << (31 - __clz(p + 1));   // largest power of two <= p + 1
    const long long m = line_twiddle_source(n, p + 1 - n);
    double s, c;
    sincospi(-2.0 * (double)m / (double)n, &s, &c);
    tw[p].x = (decltype(tw[p].x))c;
    tw[p].y = (decltype(tw[p].y))s;
  }
}

// Instance record into its slot; the work order (instance 0) and the work-queue
// counter start at zero on every call.
__global__ void k_noalloc_header(Inst1D q) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  *reinterpret_cast<Inst1D*>(g_noalloc_scratch + kInstOff) = q;
  int* oc = reinterpret_cast<int*>(g_noalloc_scratch + kOrderOff);
  oc[0] = 0;
  oc[1] = 0;
}

int fail(int code, const char* msg) {
  snprintf(g_uppe_err, sizeof(g_uppe_err), "uppe1d_propagate_noalloc: %s", msg);
  return code;
}

// Device address of the scratch array on the current device (set-up on first use).
int scratch_address(unsigned char** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(UPPE_ERR_CUDA, cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return fail(UPPE_ERR_ARG, "device ordinal out of range");
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      snprintf(g_uppe_err, sizeof(g_uppe_err),
               "uppe1d_propagate_noalloc: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
      return UPPE_ERR_CUDA;
    }
    g_scratch_addr[dev] = p;
  }
  *out = static_cast<unsigned char*>(g_scratch_addr[dev]);
  return 0;
}

}  // namespace

#define NA_CK(x)                                                                          \
  do {                                                                                    \
    cudaError_t e_ = (x);                                                                 \
    if (e_ != cudaSuccess) {                                                              \
      snprintf(g_uppe_err, sizeof(g_uppe_err), "uppe1d_propagate_noalloc: %s: %s", #x,    \
               cudaGetErrorString(e_));                                                   \
      return UPPE_ERR_CUDA;                                                               \
    }                                                                                     \
  } while (0)

extern "C" int uppe1d_propagate_noalloc(const uppe1d_inst_desc* s, int precision, const double* D,
                                        const double* G, const double* H, int lut_n,
                                        const void* lut_log10I, const void* lut_W, void* field,
                                        uppe1d_result* result, cudaStream_t stream) {
  g_uppe_err[0] = 0;
  if (!s || !D || !G || !field) return fail(UPPE_ERR_ARG, "null instance, table or field pointer");
  if (precision != UPPE_C64 && precision != UPPE_C128) return fail(UPPE_ERR_ARG, "bad precision");
  const int dbl = precision == UPPE_C128;
  const int nmax = dbl ? UPPE_NOALLOC_MAX_NT_C128 : UPPE_NOALLOC_MAX_NT_C64;
  const int n = s->Nt;
  if (n < 64 || (n & (n - 1))) return fail(UPPE_ERR_SIZE, "Nt must be a power of two >= 64");
  if (n > nmax) {
    snprintf(g_uppe_err, sizeof(g_uppe_err),
             "uppe1d_propagate_noalloc: Nt=%d exceeds the static scratch limit (Nt <= %d for "
             "complex64, <= %d for complex128); use uppe1d_plan_create/uppe1d_propagate",
             n, UPPE_NOALLOC_MAX_NT_C64, UPPE_NOALLOC_MAX_NT_C128);
    return UPPE_ERR_SIZE;
  }
  if (!(s->L >= 0.0) || !(s->tol > 0.0) || !(s->max_step > 0.0) || !(s->min_step > 0.0))
    return fail(UPPE_ERR_ARG, "invalid L/tol/max_step/min_step");
  if (s->hist_cap != 0) return fail(UPPE_ERR_ARG, "no history in this entry point (hist_cap must be 0)");
  if (s->raman && !H) return fail(UPPE_ERR_ARG, "raman needs the H table");
  if (s->plasma && (!(s->A_eff > 0.0) || lut_n < 2 || !lut_log10I || !lut_W))
    return fail(UPPE_ERR_ARG, "plasma needs A_eff > 0 and the ionisation table");

  unsigned char* base = nullptr;
  if (int rc = scratch_address(&base)) return rc;
  const size_t csz = dbl ? 16 : 8;

  Inst1D q;
  memset(&q, 0, sizeof(q));
  q.Nt = n;
  q.log2n = 31 - __builtin_clz((unsigned)n);
  q.dt = s->dt; q.L = s->L; q.tol = s->tol; q.max_step = s->max_step; q.min_step = s->min_step;
  q.max_attempts = s->max_attempts > 0 ? s->max_attempts : UPPE_DEFAULT_MAX_ATTEMPTS;
  q.raman = s->raman; q.plasma = s->plasma; q.f_R = s->f_R; q.A_eff = s->A_eff;
  q.pc.Ui = s->Ui; q.pc.sigma_half = s->sigma_drude / 2.0; q.pc.w0tc = s->omega0_tau_c;
  q.pc.rr = (double)(float)s->rate_rec; q.pc.dt = (double)(float)s->dt;
  q.pc.rho_nt = (double)(float)s->rho_nt; q.pc.ava = s->ava_coef;
  q.omega0 = s->omega0;

  Batch1D b;
  memset(&b, 0, sizeof(b));
  b.inst = reinterpret_cast<const Inst1D*>(base + kInstOff);
  b.res = reinterpret_cast<Res1D*>(base + kResOff);
  b.order = reinterpret_cast<const int*>(base + kOrderOff);
  b.counter = reinterpret_cast<int*>(base + kCounterOff);
  b.ninst = 1;
  b.D = reinterpret_cast<const double2*>(D);
  b.G = G;
  b.H = reinterpret_cast<const double2*>(H);
  b.field = field;
  b.hist = nullptr;
  b.zhist = nullptr;
  b.tw = base + kHeader;
  b.scratch = base + kHeader + 2 * (size_t)n * csz;
  b.scratch_per_block = 7LL * n;
  b.lut.n = 0;
  b.lut.x = b.lut.w = nullptr;
  b.lut.zero_x = -INFINITY;   // no zero-run shortcut: identical results, no host scan
  if (s->plasma) {
    // inv_dx = 0 tells the kernel to take the grid constants from the table's
    // ends on the device, so nothing is read back to the host
    b.lut.x = lut_log10I;
    b.lut.w = lut_W;
    b.lut.n = lut_n;
    b.lut.x0 = 0.0;
    b.lut.inv_dx = 0.0;
  }

  // the instance record goes in as a kernel argument (by value): no copy from
  // host memory is left pending when this call returns
  k_noalloc_header<<<1, 32, 0, stream>>>(q);
  NA_CK(cudaGetLastError());
  if (dbl) k_noalloc_twiddles<double2><<<8, 256, 0, stream>>>(kHeader, n);
  else k_noalloc_twiddles<float2><<<8, 256, 0, stream>>>(kHeader, n);
  NA_CK(cudaGetLastError());
  const size_t smem = csz * (size_t)(n + n / 32) + sizeof(double) * (64 + T1);
  NA_CK(dbl ? launch_uppe1d<double>(b, 1, smem, stream) : launch_uppe1d<float>(b, 1, smem, stream));
  if (result) {
    Res1D r;
    NA_CK(cudaMemcpyAsync(&r, base + kResOff, sizeof(r), cudaMemcpyDeviceToHost, stream));
    NA_CK(cudaStreamSynchronize(stream));
    result->z = r.z; result->h = r.h; result->err = r.err;
    result->attempts = r.attempts; result->accepted = r.accepted;
    result->status = r.status; result->hist_count = 0;
    result->energy = r.energy; result->photons = r.photons; result->peak_ion = r.peak_ion;
  }
  return 0;
}
