// Host side of the 1D propagator: plan (tables, twiddles, scratch) and launch.
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <numeric>
#include <vector>

#include "uppe1d_cluster.cuh"

extern char g_uppe_err[512];

using namespace uppe;

struct uppe1d_plan {
  int dbl;
  size_t csz;
  int ninst;
  int nmax;
  long long ftotal;       // sum Nt
  long long htotal;       // sum hist_cap * Nt
  long long zhtotal;      // sum hist_cap
  int nblocks;
  int nsm;
  size_t smem;
  bool use_cl = false;    // lines run on thread-block clusters (uppe1d_cluster.cuh)
  int cs = kCS;           // CTAs per cluster (4, or 8 with UPPE_CLUSTER_CTAS=8)
  int ncl = 0;            // clusters of the persistent cluster launch
  size_t cl_smem = 0;
  // mixed launch: n8 eight-CTA clusters take the costliest lines while the ncl
  // four-CTA clusters run the rest, concurrently on a second stream
  bool mixed = false;
  int n8 = 0;
  size_t cl_smem8 = 0;
  const void* xtw8 = nullptr;
  int* counter_head = nullptr;
  cudaStream_t s2 = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  int last_ctas = 0;      // CTAs of the last propagation launch (activity record)
  Batch1D b;
  Inst1D* d_inst;
  std::vector<Inst1D> h_inst;
  std::vector<void*> allocs;
  Res1D* h_res;
  // program buffers (grown on demand by uppe1d_run_programs)
  void* d_prog = nullptr;
  size_t prog_bytes = 0;
  void* d_prog_scratch = nullptr;   // stage arrays when programs outnumber the plan's CTAs
  int prog_blocks = 0;
  std::vector<unsigned char> h_prog;
};

#define UPPE1_CK(x)                                                                \
  do {                                                                             \
    cudaError_t e_ = (x);                                                          \
    if (e_ != cudaSuccess) {                                                       \
      snprintf(g_uppe_err, sizeof(g_uppe_err), "%s:%d %s: %s", __FILE__, __LINE__, \
               #x, cudaGetErrorString(e_));                                        \
      return UPPE_ERR_CUDA;                                                        \
    }                                                                              \
  } while (0)

static int up1(uppe1d_plan* p, void** dst, const void* src, size_t bytes) {
  UPPE1_CK(cudaMalloc(dst, bytes));
  p->allocs.push_back(*dst);
  if (src) UPPE1_CK(cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice));
  return 0;
}

extern "C" int uppe1d_plan_destroy(uppe1d_plan* p) {
  if (!p) return 0;
  for (void* a : p->allocs) cudaFree(a);
  if (p->d_prog) cudaFree(p->d_prog);
  if (p->d_prog_scratch) cudaFree(p->d_prog_scratch);
  if (p->h_res) cudaFreeHost(p->h_res);
  if (p->s2) cudaStreamDestroy(p->s2);
  if (p->ev_fork) cudaEventDestroy(p->ev_fork);
  if (p->ev_join) cudaEventDestroy(p->ev_join);
  delete p;
  return 0;
}

extern "C" int uppe1d_plan_create(const uppe1d_desc* d, uppe1d_plan** out) {
  NvtxRange nvtx_range("uppe1d_plan_create");
  *out = nullptr;
  g_uppe_err[0] = 0;
  if (!d || d->n_inst <= 0 || !d->inst || !d->D || !d->G) return UPPE_ERR_ARG;
  if (d->precision != UPPE_C64 && d->precision != UPPE_C128) return UPPE_ERR_ARG;
  const int dbl = d->precision == UPPE_C128;
  const int nmax_allowed = 16384;   // complex128 beyond 8192 only on the cluster kernel (below)
  uppe1d_plan* p = new uppe1d_plan();
  p->dbl = dbl;
  p->csz = dbl ? 16 : 8;
  p->ninst = d->n_inst;
  p->h_inst.resize(d->n_inst);
  long long off = 0, hoff = 0, zoff = 0;
  int nmax = 0;
  bool any_raman = false;
  for (int i = 0; i < d->n_inst; ++i) {
    const uppe1d_inst_desc& s = d->inst[i];
    const int n = s.Nt;
    if (n < 64 || n > nmax_allowed || (n & (n - 1))) {
      snprintf(g_uppe_err, sizeof(g_uppe_err),
               "instance %d: Nt=%d unsupported (power of two in [64, %d] for this precision)", i, n,
               nmax_allowed);
      delete p;
      return UPPE_ERR_SIZE;
    }
    if (!(s.L >= 0.0) || !(s.tol > 0.0) || !(s.max_step > 0.0) || !(s.min_step > 0.0) ||
        s.hist_cap < 0 || (s.plasma && !(s.A_eff > 0.0))) {
      snprintf(g_uppe_err, sizeof(g_uppe_err), "instance %d: invalid L/tol/step/history/A_eff", i);
      delete p;
      return UPPE_ERR_ARG;
    }
    Inst1D& q = p->h_inst[i];
    q.Nt = n;
    q.log2n = 31 - __builtin_clz((unsigned)n);
    q.dt = s.dt; q.L = s.L; q.tol = s.tol; q.max_step = s.max_step; q.min_step = s.min_step;
    q.off = off; q.hist_off = hoff; q.zh_off = zoff; q.hist_cap = s.hist_cap;
    // a bounded run: the device loop always ends (default cap when none is given)
    q.max_attempts = s.max_attempts > 0 ? s.max_attempts : UPPE_DEFAULT_MAX_ATTEMPTS;
    q.raman = s.raman; q.plasma = s.plasma; q.f_R = s.f_R; q.A_eff = s.A_eff;
    q.pc.Ui = s.Ui; q.pc.sigma_half = s.sigma_drude / 2.0; q.pc.w0tc = s.omega0_tau_c;
    q.pc.rr = (double)(float)s.rate_rec; q.pc.dt = (double)(float)s.dt;
    q.pc.rho_nt = (double)(float)s.rho_nt; q.pc.ava = s.ava_coef;
    q.omega0 = s.omega0;
    any_raman |= s.raman != 0;
    off += n;
    hoff += (long long)s.hist_cap * n;
    zoff += s.hist_cap;
    nmax = std::max(nmax, n);
  }
  if (any_raman && !d->H) { delete p; return UPPE_ERR_ARG; }
  // The cluster kernel serves plans whose lines are all 2048..16384 points without
  // Raman or history and at least one of them long (>= 8192): one line then runs
  // on four SMs (eight for the costliest lines of a large batch, below).
  // UPPE_1D_CLUSTER=0 keeps the single-CTA kernel where it can serve.
  {
    bool ok = true, longer = false;
    for (int i = 0; i < d->n_inst; ++i) {
      const uppe1d_inst_desc& s = d->inst[i];
      if (s.raman || s.hist_cap > 0 || s.Nt < 2048) ok = false;
      if (s.Nt >= 8192) longer = true;
    }
    const char* env = getenv("UPPE_1D_CLUSTER");
    const bool off = env && env[0] == '0';
    p->use_cl = ok && longer && !(off && !(dbl && nmax > 8192));
    if (dbl && nmax > 8192 && !p->use_cl) {
      snprintf(g_uppe_err, sizeof(g_uppe_err),
               "complex128 lines of %d points run on the cluster kernel, which needs every line of the "
               "plan in [2048, 16384] points without Raman or history", nmax);
      delete p;
      return UPPE_ERR_SIZE;
    }
  }
  for (int i = 0; i < d->n_inst; ++i)
    if (d->inst[i].plasma && (d->lut_n < 2 || !d->lut_log10I || !d->lut_W)) { delete p; return UPPE_ERR_ARG; }
  p->ftotal = off; p->htotal = hoff; p->zhtotal = zoff; p->nmax = nmax;
  int rc;
#define TRY1(x) do { rc = (x); if (rc) { uppe1d_plan_destroy(p); return rc; } } while (0)
  void* ptr;
  TRY1(up1(p, &ptr, p->h_inst.data(), sizeof(Inst1D) * p->ninst)); p->d_inst = (Inst1D*)ptr;
  TRY1(up1(p, &ptr, d->D, 16 * (size_t)off)); p->b.D = (const double2*)ptr;
  TRY1(up1(p, &ptr, d->G, 8 * (size_t)off)); p->b.G = (const double*)ptr;
  p->b.H = nullptr;
  if (any_raman) { TRY1(up1(p, &ptr, d->H, 16 * (size_t)off)); p->b.H = (const double2*)ptr; }
  // order: longest instances first (largest Nt, then longest L)
  std::vector<int> order(p->ninst);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b2) {
    const double ca = d->inst[a].cost > 0.0 ? d->inst[a].cost : (double)p->h_inst[a].Nt * p->h_inst[a].L;
    const double cb = d->inst[b2].cost > 0.0 ? d->inst[b2].cost : (double)p->h_inst[b2].Nt * p->h_inst[b2].L;
    return ca > cb;
  });
  TRY1(up1(p, &ptr, order.data(), sizeof(int) * p->ninst)); p->b.order = (const int*)ptr;
  TRY1(up1(p, &ptr, nullptr, sizeof(int))); p->b.counter = (int*)ptr;
  TRY1(up1(p, &ptr, nullptr, sizeof(Res1D) * p->ninst)); p->b.res = (Res1D*)ptr;
  {
    cudaError_t e = cudaMallocHost(&p->h_res, sizeof(Res1D) * p->ninst);
    if (e != cudaSuccess) { uppe1d_plan_destroy(p); return UPPE_ERR_CUDA; }
  }
  // packed per-pass twiddles of the line FFT: for every N = 2^k <= nmax, N slots at
  // offset N - 1, slot j holding exp(-2 pi i m / N) for m = line_twiddle_source(N, j)
  {
    std::vector<unsigned char> tw(p->csz * (size_t)(2 * nmax));
    for (int n = 1; n <= nmax; n *= 2) {
      for (int j = 0; j < n; ++j) {
        const long long m = line_twiddle_source(n, j);
        const long double ang = -2.0L * 3.141592653589793238462643383279502884L * (long double)m / (long double)n;
        const double cr = (double)cosl(ang), ci = (double)sinl(ang);
        if (dbl) { ((double2*)tw.data())[n - 1 + j] = make_double2(cr, ci); }
        else { ((float2*)tw.data())[n - 1 + j] = make_float2((float)cr, (float)ci); }
      }
    }
    TRY1(up1(p, &ptr, tw.data(), tw.size())); p->b.tw = ptr;
  }
  if (d->lut_n >= 2 && d->lut_log10I && d->lut_W) {
    const int n = d->lut_n;
    std::vector<unsigned char> lx(n * (dbl ? 8 : 4)), lw(n * (dbl ? 8 : 4));
    for (int i = 0; i < n; ++i) {
      if (dbl) { ((double*)lx.data())[i] = d->lut_log10I[i]; ((double*)lw.data())[i] = d->lut_W[i]; }
      else { ((float*)lx.data())[i] = (float)d->lut_log10I[i]; ((float*)lw.data())[i] = (float)d->lut_W[i]; }
    }
    TRY1(up1(p, &ptr, lx.data(), lx.size())); p->b.lut.x = ptr;
    TRY1(up1(p, &ptr, lw.data(), lw.size())); p->b.lut.w = ptr;
    {
      std::vector<double> sl(n - 1);
      if (dbl) lut_slopes<double>(d->lut_log10I, d->lut_W, n, sl.data());
      else lut_slopes<float>(d->lut_log10I, d->lut_W, n, sl.data());
      TRY1(up1(p, &ptr, sl.data(), sl.size() * sizeof(double)));
      p->b.lut.slope = static_cast<const double*>(ptr);
    }
    p->b.lut.n = n;
    p->b.lut.x0 = d->lut_log10I[0];
    p->b.lut.inv_dx = (n - 1) / (d->lut_log10I[n - 1] - d->lut_log10I[0]);
    {
      // leading run of zero rates (as stored in the field precision)
      int j0 = -1;
      for (int i = 0; i < n; ++i) {
        const double wv = dbl ? d->lut_W[i] : (double)(float)d->lut_W[i];
        if (wv != 0.0) break;
        j0 = i;
      }
      p->b.lut.zero_x = j0 < 0 ? -INFINITY
                       : (dbl ? d->lut_log10I[j0] : (double)(float)d->lut_log10I[j0]);
      if (j0 == n - 1) p->b.lut.zero_x = INFINITY;
      p->b.lut.I_zero = lut_zero_intensity(p->b.lut.zero_x);
    }
  } else {
    p->b.lut.x = p->b.lut.w = nullptr;
    p->b.lut.slope = nullptr;
    p->b.lut.n = 0;
    p->b.lut.zero_x = INFINITY;
    p->b.lut.I_zero = INFINITY;
  }
  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  p->nsm = nsm;
  p->nblocks = std::min(p->ninst, nsm);
  p->b.scratch_per_block = 7LL * nmax;
  TRY1(up1(p, &ptr, nullptr, p->csz * (size_t)p->b.scratch_per_block * p->nblocks)); p->b.scratch = ptr;
  p->smem = p->csz * (size_t)(nmax + nmax / 32) + sizeof(double) * (64 + T1);
  p->b.inst = p->d_inst;
  p->b.ninst = p->ninst;
  p->b.xtw = nullptr;
  p->b.cl_scratch = nullptr;
  p->b.cl_scratch_bytes = 0;
  p->b.counter_head = nullptr;
  p->b.nhead = 0;
  p->b.cl_off = 0;
  p->b.busy_off = 0;
  if (p->use_cl) {
    // CTAs per line: UPPE_CLUSTER_CTAS=4 or 8 forces one size; otherwise a batch of
    // many lines with 16384-point ones runs its costliest lines on eight-CTA
    // clusters next to four-CTA clusters for the rest (mixed launch)
    const char* env_cs = getenv("UPPE_CLUSTER_CTAS");
    const int force = env_cs ? atoi(env_cs) : 0;
    p->cs = force == 8 ? 8 : 4;
    int n16 = 0;
    for (int i = 0; i < p->ninst; ++i) n16 += p->h_inst[i].Nt == 16384;
    p->mixed = force == 0 && nmax == 16384 && p->ninst >= 16;
    // cross-CTA twiddles W_N^(m r) (r = 1..cs-1, m < M = N/cs) for M = 2048/cs .. nmax/cs
    auto xtw_table = [&](int cs, const void** dst) -> int {
      const int mmax = nmax / cs;
      std::vector<unsigned char> xt(p->csz * (size_t)(cl_xtw_offset(mmax, cs) + (long long)(cs - 1) * mmax));
      for (int M = 2048 / cs; M <= mmax; M *= 2) {
        const long long o = cl_xtw_offset(M, cs);
        for (int r = 1; r < cs; ++r)
          for (int m = 0; m < M; ++m) {
            const long double ang = -2.0L * 3.141592653589793238462643383279502884L * (long double)(m * r) /
                                    (long double)(cs * M);
            const double cr = (double)cosl(ang), ci = (double)sinl(ang);
            const long long e = o + (long long)(r - 1) * M + m;
            if (dbl) ((double2*)xt.data())[e] = make_double2(cr, ci);
            else ((float2*)xt.data())[e] = make_float2((float)cr, (float)ci);
          }
      }
      void* q = nullptr;
      const int r = up1(p, &q, xt.data(), xt.size());
      *dst = q;
      return r;
    };
    TRY1(xtw_table(p->cs, &p->b.xtw));
    p->cl_smem = dbl ? cl_smem<double>(nmax, p->cs) : cl_smem<float>(nmax, p->cs);
    const int maxcl = dbl ? uppe1d_cl_max_clusters<double>(p->cl_smem, p->cs)
                          : uppe1d_cl_max_clusters<float>(p->cl_smem, p->cs);
    p->ncl = std::min(p->ninst, maxcl > 0 ? maxcl : nsm / p->cs);
    if (p->mixed) {
      p->cl_smem8 = dbl ? cl_smem<double>(nmax, 8) : cl_smem<float>(nmax, 8);
      const int max8 = dbl ? uppe1d_cl_max_clusters<double>(p->cl_smem8, 8)
                           : uppe1d_cl_max_clusters<float>(p->cl_smem8, 8);
      p->n8 = std::min(std::min(4, n16), max8);
      if (p->n8 <= 0) {
        p->mixed = false;
      } else {
        TRY1(xtw_table(8, &p->xtw8));
        p->ncl = std::max(1, std::min(p->ninst - p->n8, std::min(maxcl > 0 ? maxcl : nsm / 4,
                                                                   (nsm - 8 * p->n8) / 4)));
        TRY1(up1(p, &ptr, nullptr, sizeof(int))); p->counter_head = (int*)ptr;
        if (cudaStreamCreateWithFlags(&p->s2, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&p->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&p->ev_join, cudaEventDisableTiming) != cudaSuccess) {
          uppe1d_plan_destroy(p);
          return UPPE_ERR_CUDA;
        }
      }
    }
    p->b.cl_scratch_bytes = (long long)(dbl ? cl_scratch_bytes<double>(nmax) : cl_scratch_bytes<float>(nmax));
    TRY1(up1(p, &ptr, nullptr, (size_t)p->b.cl_scratch_bytes * (p->ncl + p->n8))); p->b.cl_scratch = ptr;
  }
  {
    // activity record: two timer values per CTA of the widest launch
    const int ctas = std::max(p->nblocks, p->cs * p->ncl + 8 * p->n8);
    TRY1(up1(p, &ptr, nullptr, 2 * sizeof(unsigned long long) * (size_t)ctas));
    p->b.busy = static_cast<unsigned long long*>(ptr);
  }
#undef TRY1
  *out = p;
  return 0;
}

__global__ void k_queue_head(int* counter, int* counter_head, int nhead) {
  *counter = nhead;
  *counter_head = 0;
}

// the propagation kernel of the plan: thread-block clusters per line (one size, or
// the mixed launch), or one CTA per line
static cudaError_t launch_lines(uppe1d_plan* p, const Batch1D& b, cudaStream_t s) {
  if (p->use_cl && p->mixed) {
    // eight-CTA clusters take queue positions [0, n8), on a second stream forked
    // from and joined back into s; the four-CTA clusters take the rest from n8
    p->last_ctas = 8 * p->n8 + 4 * p->ncl;
    k_queue_head<<<1, 1, 0, s>>>(b.counter, p->counter_head, p->n8);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaEventRecord(p->ev_fork, s);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(p->s2, p->ev_fork, 0);
    if (e != cudaSuccess) return e;
    Batch1D b8 = b;
    b8.xtw = p->xtw8; b8.counter_head = p->counter_head; b8.nhead = p->n8; b8.cl_off = 0; b8.busy_off = 0;
    e = p->dbl ? launch_uppe1d_cl<double>(b8, p->n8, p->cl_smem8, p->s2, 8)
               : launch_uppe1d_cl<float>(b8, p->n8, p->cl_smem8, p->s2, 8);
    if (e != cudaSuccess) return e;
    Batch1D b4 = b;
    b4.nhead = 0; b4.cl_off = p->n8; b4.busy_off = 8 * p->n8;
    e = p->dbl ? launch_uppe1d_cl<double>(b4, p->ncl, p->cl_smem, s, 4)
               : launch_uppe1d_cl<float>(b4, p->ncl, p->cl_smem, s, 4);
    if (e == cudaSuccess) e = cudaEventRecord(p->ev_join, p->s2);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(s, p->ev_join, 0);
    return e;
  }
  p->last_ctas = p->use_cl ? p->cs * p->ncl : p->nblocks;
  if (p->use_cl)
    return p->dbl ? launch_uppe1d_cl<double>(b, p->ncl, p->cl_smem, s, p->cs)
                  : launch_uppe1d_cl<float>(b, p->ncl, p->cl_smem, s, p->cs);
  return p->dbl ? launch_uppe1d<double>(b, p->nblocks, p->smem, s) : launch_uppe1d<float>(b, p->nblocks, p->smem, s);
}

// SM occupancy of the last propagation launch from the CTAs' timer records: the
// persistent CTAs (one per SM) stay busy until the work queue runs dry, so
// sum(exit - start) / (SMs x span) is the fraction of the GPU's SM-time spent on
// instances.  Synchronises the stream.
extern "C" int uppe1d_last_activity(uppe1d_plan* p, double* sm_busy, double* span_ms, cudaStream_t s) {
  if (!p || !sm_busy || !span_ms || p->last_ctas <= 0) return UPPE_ERR_ARG;
  std::vector<unsigned long long> t(2 * (size_t)p->last_ctas);
  UPPE1_CK(cudaMemcpyAsync(t.data(), p->b.busy, t.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
  UPPE1_CK(cudaStreamSynchronize(s));
  unsigned long long t0 = ~0ull, t1 = 0;
  double sum = 0.0;
  for (int c = 0; c < p->last_ctas; ++c) {
    const unsigned long long a = t[2 * c], e = t[2 * c + 1];
    if (e < a) return UPPE_ERR_ARG;   // a CTA that never recorded its exit
    t0 = std::min(t0, a);
    t1 = std::max(t1, e);
    sum += (double)(e - a);
  }
  const double span = (double)(t1 - t0);
  *span_ms = span * 1e-6;
  *sm_busy = span > 0.0 ? sum / (span * (double)p->nsm) : 0.0;
  return 0;
}

extern "C" long long uppe1d_field_elems(const uppe1d_plan* p) { return p ? p->ftotal : 0; }
extern "C" int uppe1d_uses_clusters(const uppe1d_plan* p) { return p && p->use_cl ? p->ncl : 0; }
extern "C" long long uppe1d_hist_elems(const uppe1d_plan* p) { return p ? p->htotal : 0; }
extern "C" long long uppe1d_hist_slots(const uppe1d_plan* p) { return p ? p->zhtotal : 0; }

extern "C" int uppe1d_propagate(uppe1d_plan* p, void* field, void* hist, double* zhist,
                                uppe1d_result* results, cudaStream_t s) {
  NvtxRange nvtx_range("uppe1d_propagate");
  if (!p || !field) return UPPE_ERR_ARG;
  if (p->htotal > 0 && (!hist || !zhist)) {
    snprintf(g_uppe_err, sizeof(g_uppe_err), "plan has history slots: hist and zhist are required");
    return UPPE_ERR_ARG;
  }
  Batch1D b = p->b;
  b.field = field;
  b.hist = hist;
  b.zhist = zhist;
  UPPE1_CK(cudaMemsetAsync(p->b.counter, 0, sizeof(int), s));
  UPPE1_CK(launch_lines(p, b, s));
  if (results) {
    UPPE1_CK(cudaMemcpyAsync(p->h_res, p->b.res, sizeof(Res1D) * p->ninst, cudaMemcpyDeviceToHost, s));
    UPPE1_CK(cudaStreamSynchronize(s));
    for (int i = 0; i < p->ninst; ++i) {
      const Res1D& r = p->h_res[i];
      results[i].z = r.z; results[i].h = r.h; results[i].err = r.err;
      results[i].attempts = r.attempts; results[i].accepted = r.accepted;
      results[i].status = r.status; results[i].hist_count = r.hist_count;
      results[i].energy = r.energy; results[i].photons = r.photons; results[i].peak_ion = r.peak_ion;
    }
  }
  return 0;
}

// ---- step log, replay and adjoint ------------------------------------------
static int run1(uppe1d_plan* p, Batch1D& b, uppe1d_result* results, cudaStream_t s) {
  UPPE1_CK(cudaMemsetAsync(p->b.counter, 0, sizeof(int), s));
  UPPE1_CK(launch_lines(p, b, s));
  if (results) {
    UPPE1_CK(cudaMemcpyAsync(p->h_res, p->b.res, sizeof(Res1D) * p->ninst, cudaMemcpyDeviceToHost, s));
    UPPE1_CK(cudaStreamSynchronize(s));
    for (int i = 0; i < p->ninst; ++i) {
      const Res1D& r = p->h_res[i];
      results[i].z = r.z; results[i].h = r.h; results[i].err = r.err;
      results[i].attempts = r.attempts; results[i].accepted = r.accepted;
      results[i].status = r.status; results[i].hist_count = r.hist_count;
      results[i].energy = r.energy; results[i].photons = r.photons; results[i].peak_ion = r.peak_ion;
    }
  }
  return 0;
}

extern "C" int uppe1d_propagate_logged(uppe1d_plan* p, void* field, double* hlog, int hlog_cap,
                                       uppe1d_result* results, cudaStream_t s) {
  NvtxRange nvtx_range("uppe1d_propagate_logged");
  if (!p || !field || !hlog || hlog_cap <= 0 || p->htotal > 0) return UPPE_ERR_ARG;
  Batch1D b = p->b;
  b.field = field;
  b.hlog = hlog;
  b.hlog_cap = hlog_cap;
  return run1(p, b, results, s);
}

extern "C" int uppe1d_propagate_schedule(uppe1d_plan* p, void* field, const double* hsched,
                                         int nsched, uppe1d_result* results, cudaStream_t s) {
  NvtxRange nvtx_range("uppe1d_propagate_schedule");
  if (!p || !field || !hsched || nsched < 0 || p->htotal > 0) return UPPE_ERR_ARG;
  Batch1D b = p->b;
  b.field = field;
  b.hsched = hsched;
  b.nsched = nsched;
  return run1(p, b, results, s);
}

static int prog_fail(const char* msg) {
  snprintf(g_uppe_err, sizeof(g_uppe_err), "uppe1d_run_programs: %s", msg);
  return UPPE_ERR_ARG;
}

extern "C" int uppe1d_run_programs(uppe1d_plan* p, int nprog, const long long* op_begin,
                                   const uppe1d_op* ops, void* fields, void* records,
                                   uppe1d_result* op_results, cudaStream_t s) {
  NvtxRange nvtx_range("uppe1d_run_programs");
  g_uppe_err[0] = 0;
  if (!p || nprog <= 0 || !op_begin || !ops || !fields) return prog_fail("null argument or nprog <= 0");
  if (op_begin[0] != 0) return prog_fail("op_begin[0] must be 0");
  const long long nops = op_begin[nprog];
  if (nops <= 0) return prog_fail("no operations");
  std::vector<Prog1D> progs(nprog);
  std::vector<Op1D> hops(nops);
  long long foff = 0, roff = 0;
  for (int q = 0; q < nprog; ++q) {
    Prog1D& g = progs[q];
    g.op_begin = op_begin[q];
    g.op_end = op_begin[q + 1];
    if (g.op_end < g.op_begin || g.op_end > nops) return prog_fail("op_begin must be non-decreasing");
    g.Nt = 0;
    int nrec = 0;
    for (long long o = g.op_begin; o < g.op_end; ++o) {
      const uppe1d_op& u = ops[o];
      if (u.inst >= p->ninst) return prog_fail("operation names an instance outside the plan");
      if (u.inst >= 0) {
        const Inst1D& in = p->h_inst[u.inst];
        if (in.hist_cap > 0) return prog_fail("program instances must have hist_cap = 0");
        if (p->dbl && in.Nt > 8192) return prog_fail("complex128 programs take lines of at most 8192 points");
        if (g.Nt == 0) { g.Nt = in.Nt; g.log2n = in.log2n; g.dt = in.dt; }
        else if (in.Nt != g.Nt || in.dt != g.dt)
          return prog_fail("the propagations of one program must share Nt and dt");
      } else if (!(u.amp >= 0.0) || !isfinite(u.gdd) || !isfinite(u.tod)) {
        return prog_fail("mirror needs amp >= 0 and finite gdd, tod");
      }
      hops[o].inst = u.inst < 0 ? -1 : u.inst;
      hops[o].record = u.record ? 1 : 0;
      hops[o].amp = u.amp; hops[o].gdd = u.gdd; hops[o].tod = u.tod;
      nrec += u.record ? 1 : 0;
    }
    if (g.Nt == 0) return prog_fail("a program needs at least one propagation");
    g.field_off = foff;
    g.rec_off = roff;
    foff += g.Nt;
    roff += (long long)nrec * g.Nt;
  }
  if (roff > 0 && !records) return prog_fail("operations record fields but records is NULL");
  // one device buffer: programs, operations, per-operation results, queue order
  const size_t bp = sizeof(Prog1D) * nprog, bo = sizeof(Op1D) * nops, br = sizeof(Res1D) * nops,
               bq = sizeof(int) * nprog;
  auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
  const size_t need = al(bp) + al(bo) + al(br) + al(bq);
  if (need > p->prog_bytes) {
    if (p->d_prog) UPPE1_CK(cudaFree(p->d_prog));
    p->d_prog = nullptr;
    p->prog_bytes = 0;
    UPPE1_CK(cudaMalloc(&p->d_prog, need));
    p->prog_bytes = need;
  }
  unsigned char* base = static_cast<unsigned char*>(p->d_prog);
  Prog1D* d_progs = reinterpret_cast<Prog1D*>(base);
  Op1D* d_ops = reinterpret_cast<Op1D*>(base + al(bp));
  Res1D* d_res = reinterpret_cast<Res1D*>(base + al(bp) + al(bo));
  int* d_order = reinterpret_cast<int*>(base + al(bp) + al(bo) + al(br));
  // longest programs first (cost ~ Nt log Nt x sum of L / max_step)
  std::vector<double> cost(nprog, 0.0);
  for (int q = 0; q < nprog; ++q)
    for (long long o = progs[q].op_begin; o < progs[q].op_end; ++o)
      if (hops[o].inst >= 0) {
        const Inst1D& in = p->h_inst[hops[o].inst];
        cost[q] += (double)in.Nt * in.log2n * fmax(1.0, in.L / in.max_step);
      }
  std::vector<int> order(nprog);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost[a] > cost[b]; });
  p->h_prog.resize(need);
  memcpy(p->h_prog.data(), progs.data(), bp);
  memcpy(p->h_prog.data() + al(bp), hops.data(), bo);
  memcpy(p->h_prog.data() + al(bp) + al(bo) + al(br), order.data(), bq);
  UPPE1_CK(cudaMemcpyAsync(base, p->h_prog.data(), need, cudaMemcpyHostToDevice, s));
  Batch1D b = p->b;
  int nb = std::min(p->nblocks, nprog);
  const int want = std::min(nprog, p->nsm);
  if (want > nb) {   // more programs than the plan's CTAs: scratch for one CTA per SM
    if (want > p->prog_blocks) {
      if (p->d_prog_scratch) UPPE1_CK(cudaFree(p->d_prog_scratch));
      p->d_prog_scratch = nullptr;
      p->prog_blocks = 0;
      UPPE1_CK(cudaMalloc(&p->d_prog_scratch, p->csz * (size_t)p->b.scratch_per_block * want));
      p->prog_blocks = want;
    }
    b.scratch = p->d_prog_scratch;
    nb = want;
  }
  b.field = fields;
  b.prog = d_progs;
  b.ops = d_ops;
  b.op_res = d_res;
  b.records = records;
  b.order = d_order;
  b.ninst = nprog;
  b.hlog = nullptr;
  b.hsched = nullptr;
  UPPE1_CK(cudaMemsetAsync(p->b.counter, 0, sizeof(int), s));
  p->last_ctas = nb;
  UPPE1_CK(p->dbl ? launch_uppe1d<double>(b, nb, p->smem, s) : launch_uppe1d<float>(b, nb, p->smem, s));
  if (op_results) {
    std::vector<Res1D> hr(nops);
    UPPE1_CK(cudaMemcpyAsync(hr.data(), d_res, br, cudaMemcpyDeviceToHost, s));
    UPPE1_CK(cudaStreamSynchronize(s));
    for (long long o = 0; o < nops; ++o) {
      const Res1D& r = hr[o];
      uppe1d_result& x = op_results[o];
      x.z = r.z; x.h = r.h; x.err = r.err; x.attempts = r.attempts; x.accepted = r.accepted;
      x.status = r.status; x.hist_count = r.hist_count;
      x.energy = r.energy; x.photons = r.photons; x.peak_ion = r.peak_ion;
    }
  }
  return 0;
}

extern "C" long long uppe1d_adjoint_work_elems(int Nt, int nsteps, int K) {
  if (Nt <= 0 || nsteps < 0 || K <= 0) return -1;
  const long long nseg = (nsteps + K - 1) / K;
  return (18LL + (nseg > 0 ? nseg : 1) + K) * Nt;
}

extern "C" int uppe1d_adjoint(uppe1d_plan* p, int inst, const double* hlog, int nsteps, int K,
                              const void* A0, const void* Abar, void* A0bar, void* gD, double* gG,
                              void* rhs, double* gPlasma, void* work, cudaStream_t s) {
  NvtxRange nvtx_range("uppe1d_adjoint");
  g_uppe_err[0] = 0;
  if (!p || inst < 0 || inst >= p->ninst || !hlog || nsteps < 0 || K <= 0 || !A0 || !Abar ||
      !A0bar || !gD || !gG || !rhs || !work)
    return UPPE_ERR_ARG;
  if (!p->dbl) {
    snprintf(g_uppe_err, sizeof(g_uppe_err), "uppe1d_adjoint: the adjoint needs a complex128 plan");
    return UPPE_ERR_ARG;
  }
  const Inst1D& q = p->h_inst[inst];
  if (q.Nt > 8192) {
    snprintf(g_uppe_err, sizeof(g_uppe_err), "uppe1d_adjoint: lines of at most 8192 points");
    return UPPE_ERR_SIZE;
  }
  if (q.raman || (q.plasma && q.pc.ava != 0.0)) {
    snprintf(g_uppe_err, sizeof(g_uppe_err),
             "uppe1d_adjoint: the Raman response and avalanche ionisation have no adjoint here");
    return UPPE_ERR_ARG;
  }
  if (q.plasma && !gPlasma) {
    snprintf(g_uppe_err, sizeof(g_uppe_err), "uppe1d_adjoint: a plasma instance needs gPlasma[3]");
    return UPPE_ERR_ARG;
  }
  Adj1D a;
  a.b = p->b;
  a.inst = inst;
  a.hlog = hlog;
  a.nsteps = nsteps;
  a.K = K;
  a.A0 = (const double2*)A0;
  a.Abar = (const double2*)Abar;
  a.A0bar = (double2*)A0bar;
  a.gD = (double2*)gD;
  a.gG = gG;
  a.rhs = (double2*)rhs;
  a.gPl = gPlasma;
  a.work = (double2*)work;
  UPPE1_CK(launch_uppe1d_adjoint(a, p->smem, s));
  return 0;
}

// ---------------------------------------------------------------------------
// Input pulse from a measured spectrum (erk43ip_method.py:599-764, FFT path):
// the spectral density S(f), given as a piecewise cubic over ascending
// breakpoints, is evaluated on the simulation grid f = w/(2 pi) + f0 (zero
// outside the breakpoints, clipped at 0), and A_w = sqrt(S) exp(i (gdd w^2/2 +
// tod w^3/6)) is written in fft order.
// ---------------------------------------------------------------------------
namespace uppe {
__global__ void k_spectrum_field(const double* br, const double* cf, int nb, int n, double dt, double f0,
                                 double gdd, double tod, double2* out) {
  const double val = 1.0 / (n * dt);                  // fftfreq(n, dt) = k * val
  const double twopi = 6.283185307179586476925286766559;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const double w = twopi * ((k < (n + 1) / 2 ? k : k - n) * val);
    const double f = w / twopi + f0;
    double S = 0.0;
    if (f >= br[0] && f <= br[nb - 1]) {
      int lo = 0, hi = nb - 2;                        // last interval with br[j] <= f
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (br[mid] <= f) lo = mid; else hi = mid - 1;
      }
      const double x = f - br[lo];
      const double* c = cf + 4 * (long long)lo;
      S = ((c[0] * x + c[1]) * x + c[2]) * x + c[3];
    }
    if (!(S > 0.0)) S = 0.0;                          // negative or NaN -> 0
    const double m = sqrt(S);
    double sn, cs;
    sincos(0.5 * gdd * w * w + (1.0 / 6.0) * tod * w * w * w, &sn, &cs);
    out[k] = make_double2(m * cs, m * sn);
  }
}
}  // namespace uppe

extern "C" int uppe_spectrum_field(const double* breaks, const double* coef, int nb, int Nt, double dt,
                                   double f0, double gdd, double tod, void* out, cudaStream_t s) {
  if (!breaks || !coef || !out || nb < 2 || Nt < 1 || !(dt > 0.0)) return UPPE_ERR_ARG;
  const int threads = 256;
  const int blocks = (Nt + threads - 1) / threads < 1024 ? (Nt + threads - 1) / threads : 1024;
  k_spectrum_field<<<blocks, threads, 0, s>>>(breaks, coef, nb, Nt, dt, f0, gdd, tod, (double2*)out);
  UPPE1_CK(cudaGetLastError());
  return 0;
}

// ---------------------------------------------------------------------------
// Input-pulse utilities on the device (the reference does these on the host with
// numpy/scipy: erk43ip_method.py:383-446, 492-598, 599-764).
//
// uppe_fft_c128: one complex128 line of N = 2^m points, radix-2 Stockham
// autosort passes in global memory (pass with half-length m and stride s:
// y[q + s 2p] = a + b, y[q + s (2p+1)] = (a - b) W_n^p, a = x[q + s p],
// b = x[q + s (p + m)]), twiddles from sincospi in FP64.  Optional input
// rotation by N/2 (ifftshift) in the first pass and output rotation (fftshift)
// with a scale in the last.  Input pulses are built once per run, so a simple
// bandwidth-light formulation serves; the propagators never call it.
// ---------------------------------------------------------------------------
namespace uppe {
__global__ void k_fft_pass(const double2* __restrict__ x, double2* __restrict__ y, int N, int n, int s,
                           int dir, int shift_in) {
  const int half = N / 2, m = n / 2;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < half; t += gridDim.x * blockDim.x) {
    const int p = t / s, q = t % s;
    int ia = q + s * p, ib = q + s * (p + m);
    if (shift_in) { ia = (ia + half) & (N - 1); ib = (ib + half) & (N - 1); }
    const double2 a = x[ia], b = x[ib];
    double sn, cs;
    sincospi((double)dir * 2.0 * (double)p / (double)n, &sn, &cs);
    const double dr = a.x - b.x, di = a.y - b.y;
    y[q + s * (2 * p)] = make_double2(a.x + b.x, a.y + b.y);
    y[q + s * (2 * p + 1)] = make_double2(dr * cs - di * sn, dr * sn + di * cs);
  }
}

__global__ void k_fft_out(const double2* __restrict__ x, double2* __restrict__ out, int N, double scale,
                          int shift_out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    const double2 v = x[i];
    out[shift_out ? (i + N / 2) & (N - 1) : i] = make_double2(v.x * scale, v.y * scale);
  }
}

// field[k] *= exp(i (gdd w^2 / 2 + tod w^3 / 6)), w = 2 pi fftfreq(N, dt)[k]
__global__ void k_spectral_phase(double2* f, int n, double dt, double gdd, double tod) {
  const double val = 1.0 / (n * dt);
  const double twopi = 6.283185307179586476925286766559;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const double w = twopi * ((k < (n + 1) / 2 ? k : k - n) * val);
    double sn, cs;
    sincos(0.5 * gdd * w * w + (1.0 / 6.0) * tod * w * w * w, &sn, &cs);
    const double2 v = f[k];
    f[k] = make_double2(v.x * cs - v.y * sn, v.x * sn + v.y * cs);
  }
}

// Direct (non-uniform) Fourier sum of the exact-transform path: one block per
// output time, a fixed-order block reduction (deterministic).
constexpr int kEftThreads = 256;
__global__ void __launch_bounds__(kEftThreads) k_exact_ft(const double* __restrict__ t, int Nt,
                                                          const double* __restrict__ om,
                                                          const double2* __restrict__ a, int Nf,
                                                          double2* __restrict__ out) {
  __shared__ double sr[kEftThreads], si[kEftThreads];
  for (int i = blockIdx.x; i < Nt; i += gridDim.x) {
    const double ti = t[i];
    double re = 0.0, im = 0.0;
    for (int k = threadIdx.x; k < Nf; k += kEftThreads) {
      double sn, cs;
      sincos(-om[k] * ti, &sn, &cs);
      const double2 v = a[k];
      re += v.x * cs - v.y * sn;
      im += v.x * sn + v.y * cs;
    }
    sr[threadIdx.x] = re;
    si[threadIdx.x] = im;
    __syncthreads();
    for (int o = kEftThreads / 2; o > 0; o >>= 1) {
      if (threadIdx.x < o) { sr[threadIdx.x] += sr[threadIdx.x + o]; si[threadIdx.x] += si[threadIdx.x + o]; }
      __syncthreads();
    }
    if (threadIdx.x == 0) out[(i + Nt / 2) % Nt] = make_double2(sr[0], si[0]);   // fftshift
    __syncthreads();
  }
}
}  // namespace uppe

static int grid_for(long long n) {
  const long long b = (n + 255) / 256;
  return (int)(b < 1 ? 1 : (b > 4096 ? 4096 : b));
}

extern "C" int uppe_fft_c128(const void* in, void* out, void* work, int N, int dir, double scale, int shift_in,
                             int shift_out, cudaStream_t s) {
  if (!in || !out || !work || N < 2 || (N & (N - 1)) || N > (1 << 24) || (dir != -1 && dir != 1))
    return UPPE_ERR_ARG;
  double2* w[2] = {static_cast<double2*>(work), static_cast<double2*>(work) + N};
  const double2* src = static_cast<const double2*>(in);
  int k = 0, si = shift_in;
  for (int n = N, st = 1; n > 1; n >>= 1, st <<= 1, k ^= 1) {
    k_fft_pass<<<grid_for(N / 2), 256, 0, s>>>(src, w[k], N, n, st, dir, si);
    src = w[k];
    si = 0;
  }
  k_fft_out<<<grid_for(N), 256, 0, s>>>(src, static_cast<double2*>(out), N, scale, shift_out);
  UPPE1_CK(cudaGetLastError());
  return 0;
}

extern "C" int uppe_spectral_phase(void* field, int N, double dt, double gdd, double tod, cudaStream_t s) {
  if (!field || N < 1 || !(dt > 0.0)) return UPPE_ERR_ARG;
  k_spectral_phase<<<grid_for(N), 256, 0, s>>>(static_cast<double2*>(field), N, dt, gdd, tod);
  UPPE1_CK(cudaGetLastError());
  return 0;
}

extern "C" int uppe_exact_ft(const double* t, int Nt, const double* omega, const void* amp, int Nf, void* out,
                             cudaStream_t s) {
  if (!t || !omega || !amp || !out || Nt < 1 || Nf < 1) return UPPE_ERR_ARG;
  k_exact_ft<<<Nt < 8192 ? Nt : 8192, kEftThreads, 0, s>>>(t, Nt, omega, static_cast<const double2*>(amp), Nf,
                                                           static_cast<double2*>(out));
  UPPE1_CK(cudaGetLastError());
  return 0;
}
