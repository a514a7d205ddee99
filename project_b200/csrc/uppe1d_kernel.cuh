#pragma once
// 1D ERK4(3)-IP UPPE/GNLSE propagator, batched and persistent, sm_100a.
//
// Replaces ERK43IP_UPPE.propagate / erk43_step / linear_operator /
// nonlinear_operator (src/1D-ERK4(3)IP UPPE gas/erk43ip_method.py:181-369).
//
// One launch propagates a whole batch: each CTA pulls instances from a device
// work queue (longest first) and runs the complete adaptive loop of one
// instance on the device -- no host round trip per step.  The state is held in
// the omega domain, so exp(h/2 D) is a diagonal factor computed on the fly from
// the FP64 D(omega) table, and each nonlinear evaluation is one inverse FFT,
// the pointwise Kerr (+ Raman, + plasma) term and one forward FFT, all on a line
// resident in shared memory (Stockham, Nt <= 16384 complex64 / 8192 complex128).
// The stage arrays live in a per-CTA global scratch that stays in L2.
// FSAL: alpha5 of an accepted step is the next step's N(A) (bit-identical to
// recomputing it, which the reference does whenever h changes).
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <numeric>
#include <vector>

#include "common.cuh"
#include "../../include/uppe_b200.h"

namespace uppe {

constexpr int T1 = 512;   // threads per CTA

struct Inst1D {
  int Nt, log2n;
  double dt, L, tol, max_step, min_step;
  long long off;         // element offset in the packed field/table arrays
  long long hist_off;    // element offset of the history slots
  long long zh_off;      // offset of the history z values
  int hist_cap;
  long long max_attempts;
  int raman, plasma;
  double f_R, A_eff;
  PlasmaConst pc;
  double omega0;         // carrier angular frequency (photon number)
};

struct Res1D {
  double z, h, err;
  long long attempts, accepted;
  int status, hist_count;
  double energy, photons, peak_ion;
};

// One operation of a propagation program: a propagation through plan instance
// `inst` (its tables, medium, L, tol, step limits), or, with inst < 0, a mirror
// A_w *= amp exp(i (gdd w^2 / 2 + tod w^3 / 6)); `record` stores the
// time-domain field after the operation.
struct Op1D {
  int inst, record;
  double amp, gdd, tod;
};
struct Prog1D {
  long long op_begin, op_end;   // operations [op_begin, op_end)
  long long field_off;          // element offset of the program's field
  long long rec_off;            // element offset of its recorded fields
  int Nt, log2n;
  double dt;
};
struct Batch1D {
  const Inst1D* inst;
  Res1D* res;
  const int* order;
  int* counter;
  int ninst;
  const double2* D;
  const double* G;
  const double2* H;
  void* field;
  void* hist;
  double* zhist;
  void* scratch;
  long long scratch_per_block;   // complex elements
  const void* tw;                // packed twiddles: size N at offset N-1
  Lut lut;
  double* hlog;                  // accepted step sizes, hlog_cap per instance (or null)
  int hlog_cap;
  const double* hsched;          // replay: nsched step sizes per instance, all accepted (or null)
  int nsched;
  const Prog1D* prog;            // programs (work items are programs when set)
  const Op1D* ops;
  Res1D* op_res;                 // one result per operation
  void* records;                 // recorded fields (or null)
  const void* xtw;               // cluster kernel: cross-CTA twiddles W_N^(m r) (or null)
  void* cl_scratch;              // cluster kernel: per-cluster scratch
  long long cl_scratch_bytes;
  unsigned long long* busy;      // per CTA: globaltimer at start and at exit (or null)
  // cluster kernel, eight-CTA launch next to a four-CTA one: its clusters take the
  // queue positions [0, nhead) from counter_head (the four-CTA clusters start at
  // nhead); cl_off and busy_off offset the cluster scratch index and the activity
  // slots of a launch
  int* counter_head;
  int nhead;
  int cl_off;
  int busy_off;
};

// activity record of a persistent CTA (ns of the global timer)
static __device__ __forceinline__ void mark_busy(unsigned long long* busy, int slot, int off = 0) {
  if (busy && threadIdx.x == 0) {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    busy[2 * (off + (int)blockIdx.x) + slot] = t;
  }
}

template <int N> struct Cfg1 {
  static constexpr int FT = N / 2 < T1 ? N / 2 : T1;   // FFT team size
  static constexpr int PAD = N + N / 32;
  static constexpr int CH = N >= T1 ? N / T1 : 1;      // density-scan chunk per thread
  static constexpr int NA = N / CH;                    // threads owning a chunk
};

static __device__ __forceinline__ int pad1(int n) { return n + (n >> 5); }

// The line FFT (one signal of N points, team of Cfg1<N>::FT threads) reads its
// twiddles from a per-pass table: pass (Ns, R) owns (R-1)*Ns consecutive slots
// after the passes before it, slot (r-1)*Ns + k holding exp(-2 pi i r k / (Ns R)).
// Adjacent lanes have adjacent k, so a warp's twiddle load is one contiguous run
// instead of 32 scattered lines of the plain exp(-2 pi i m / N) table; the values
// are the same entries of that table, so the transform is unchanged bit for bit.
// The slots sum to N - 1, so the tables pack like the plain ones (size N at N-1).
__host__ __device__ constexpr int line_fft_team(int n) { return n / 2 < T1 ? n / 2 : T1; }
__host__ __device__ constexpr int line_pick_radix(int rem, int e) {
  return (rem % 16 == 0 && e % 16 == 0) ? 16 : (rem % 8 == 0 && e % 8 == 0) ? 8
       : (rem % 4 == 0 && e % 4 == 0) ? 4 : 2;
}
// plain-table index m (exp(-2 pi i m / n)) held by slot `slot` of the size-n per-pass table
__host__ __device__ inline long long line_twiddle_source(int n, int slot) {
  if (n < 2) return 0;
  const int e = n / line_fft_team(n);
  int ns = 1, off = 0;
  while (ns < n) {
    const int r = line_pick_radix(n / ns, e);
    const int cnt = (r - 1) * ns;
    if (slot < off + cnt) {
      const int rr = (slot - off) / ns + 1, k = (slot - off) % ns;
      return (long long)(rr * k) * (n / (ns * r));
    }
    off += cnt;
    ns *= r;
  }
  return 0;   // slot n - 1 is padding
}

template <int N, int NTHR, int DIR, int Ns, int OFF, typename C>
__device__ __forceinline__ void stockham_line(C* s, const C* tw, int tid) {
  if constexpr (Ns < N) {
    constexpr int E = N / NTHR;
    static_assert(E >= 2, "need at least two elements per thread");
    constexpr int R = PickRadix<N / Ns, E>::v;
    static_assert(R == line_pick_radix(N / Ns, E), "pass list and twiddle layout disagree");
    constexpr int B = E / R;
    constexpr int M = N / R;
    C v[B][R];
    const bool act = tid < NTHR;
    if (act) {
#pragma unroll
      for (int b = 0; b < B; ++b) {
        const int j = tid + b * NTHR;
        const int k = j & (Ns - 1);
#pragma unroll
        for (int r = 0; r < R; ++r) v[b][r] = s[pad1(j + r * M)];
        if constexpr (Ns > 1) {
#pragma unroll
          for (int r = 1; r < R; ++r) {
            C w = tw[OFF + (r - 1) * Ns + k];
            if (DIR > 0) w.y = -w.y;
            v[b][r] = cmul(v[b][r], w);
          }
        }
        DFT<R, DIR, C>::run(v[b]);
      }
    }
    __syncthreads();
    if (act) {
#pragma unroll
      for (int b = 0; b < B; ++b) {
        const int j = tid + b * NTHR;
        const int k = j & (Ns - 1);
        const int base = (j / Ns) * Ns * R + k;
#pragma unroll
        for (int r = 0; r < R; ++r) s[pad1(base + r * Ns)] = v[b][r];
      }
    }
    __syncthreads();
    stockham_line<N, NTHR, DIR, Ns * R, OFF + (R - 1) * Ns, C>(s, tw, tid);
  }
}
// DIR=-1 forward, +1 inverse (unscaled) transform of the padded line s
template <int N, int DIR, typename C>
__device__ __forceinline__ void line_fft(C* s, const C* tw, int tid) {
  static_assert(Cfg1<N>::FT == line_fft_team(N), "team size and twiddle layout disagree");
  stockham_line<N, Cfg1<N>::FT, DIR, 1, 0, C>(s, tw, tid);
}

static __device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// deterministic block sum (fixed order)
static __device__ double block_sum(double v, double* red) {
  const int tid = threadIdx.x;
  v = warp_sum(v);
  if ((tid & 31) == 0) red[tid >> 5] = v;
  __syncthreads();
  if (tid < 32) {
    double t = tid < T1 / 32 ? red[tid] : 0.0;
    t = warp_sum(t);
    if (tid == 0) red[T1 / 32] = t;
  }
  __syncthreads();
  const double r = red[T1 / 32];
  __syncthreads();
  return r;
}

// exp(hh * D[w]) with D the FP64 dispersion table (erk43ip_method.py:194)
template <typename Rl> struct EFac;
template <> struct EFac<double> {
  __device__ __forceinline__ static double2 get(double2 D, double hh) {
    double s, c;
    sincos(hh * D.y, &s, &c);
    const double m = exp(hh * D.x);
    return make_double2(m * c, m * s);
  }
};
template <> struct EFac<float> {
  __device__ __forceinline__ static float2 get(double2 D, double hh) {
    const float2 e = cis_quadrant(hh * D.y);
    const float m = expf((float)(hh * D.x));
    return make_float2(m * e.x, m * e.y);
  }
};

enum In1 { IN_A = 0, IN_2, IN_3, IN_4, IN_5 };

template <typename Rl> struct Ctx1 {
  using C = typename CT<Rl>::T;
  // the padded line at the start of the dynamic shared memory, named as a shared
  // array so the stage functions (not inlined into the kernel) get shared-memory
  // accesses that the compiler may reorder around the global stage arrays
  __device__ __forceinline__ C* sm() const {
    extern __shared__ __align__(16) unsigned char smem[];
    return reinterpret_cast<C*>(smem);
  }
  double* red;
  double* starts;
  const C* tw;
  C *A, *K1, *T, *O, *A4, *A4P, *GA;
  const double2* D;
  const double* G;
  const double2* H;
  const Inst1D* in;
  Lut lut;
};

// Density at the start of each thread's chunk of the line (time-domain field in
// GA, or with FROM_S in the padded shared line): a block scan of the chunks'
// affine maps, or lane 0's exact serial update when a clamp binds.  Returns
// false when the whole line has W_ion = 0 and no avalanche (the density stays 0).
template <typename Rl, int N, bool FROM_S = false>
__device__ bool density_starts(Ctx1<Rl>& c, double& rho0) {
  using C = typename CT<Rl>::T;
  constexpr int CH = Cfg1<N>::CH, NA = Cfg1<N>::NA;
  const int tid = threadIdx.x;
  const PlasmaConst& m = c.in->pc;
  const double Aeff = c.in->A_eff;
  const AffineStep aff(m);
  bool any_w = false, ok = (m.ava == 0.0);
  double cm = 1.0, dm = 0.0;
  if (tid < NA) {
    for (int t = tid * CH; t < tid * CH + CH; ++t) {
      const C a = FROM_S ? c.sm()[pad1(t)] : c.GA[t];
      const Rl I = (Rl)(((double)a.x * a.x + (double)a.y * a.y) / Aeff);
      const double w = (double)(float)lut_eval<Rl>(c.lut, I);
      any_w |= (w != 0.0);
      const double cc = aff.e - w * aff.sf;
      ok &= (cc >= 0.0);
      dm = cc * dm + w * m.rho_nt * aff.sf;
      cm = cc * cm;
    }
  }
  const bool any_block = __syncthreads_or(any_w) || m.ava != 0.0;
  if (!any_block) return false;
  const bool all_ok = __syncthreads_and(ok);
  if (all_ok) {
    // block exclusive scan of affine maps (c1,d1) then (c2,d2) = (c1 c2, c2 d1 + d2)
    const int lane = tid & 31, warp = tid >> 5;
    double cc = cm, dd = dm;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const double cp = __shfl_up_sync(0xffffffffu, cc, off);
      const double dp = __shfl_up_sync(0xffffffffu, dd, off);
      if (lane >= off) { dd = cc * dp + dd; cc = cc * cp; }
    }
    double* wc = c.starts;            // warp totals
    double* wd = c.starts + T1 / 32;
    if (lane == 31) { wc[warp] = cc; wd[warp] = dd; }
    __syncthreads();
    if (tid == 0) {
      double C0 = 1.0, D0 = 0.0;      // exclusive prefix over warps (applied to rho = 0)
      for (int w = 0; w < T1 / 32; ++w) {
        const double c2 = wc[w], d2 = wd[w];
        wc[w] = C0; wd[w] = D0;
        D0 = c2 * D0 + d2;
        C0 = C0 * c2;
      }
    }
    __syncthreads();
    double ce = __shfl_up_sync(0xffffffffu, cc, 1);
    double de = __shfl_up_sync(0xffffffffu, dd, 1);
    if (lane == 0) { ce = 1.0; de = 0.0; }
    rho0 = ce * wd[warp] + de;
    __syncthreads();
  } else {
    if (tid == 0) {
      double rho = 0.0;
      for (int t = 0; t < N; ++t) {
        if (t % CH == 0) c.starts[t / CH] = rho;
        const C a = FROM_S ? c.sm()[pad1(t)] : c.GA[t];
        const double Id = ((double)a.x * a.x + (double)a.y * a.y) / Aeff;
        const double w = (double)(float)lut_eval<Rl>(c.lut, (Rl)Id);
        const double wa = (double)(float)(m.ava * (double)(Rl)Id);
        rho_step(rho, w, wa, m);
      }
    }
    __syncthreads();
    rho0 = tid < NA ? c.starts[tid] : 0.0;
    __syncthreads();
  }
  return true;
}

// plasma term P(t) = (loss + defocus)(t) * a(t) into the shared line, from the
// time-domain field in GA (media_physics.py:156-203 with I = |A|^2 / A_eff).
// The field is first copied into the shared line with coalesced loads, so the
// per-thread chunks of the scan read shared memory, and each thread overwrites
// only its own chunk.  Returns false (the shared line then holds the field) when
// the whole line has W_ion = 0 and no avalanche, i.e. the term is identically zero.
template <typename Rl, int N>
__device__ bool plasma_line(Ctx1<Rl>& c, double* ion_out) {
  using C = typename CT<Rl>::T;
  constexpr int CH = Cfg1<N>::CH, NA = Cfg1<N>::NA;
  const int tid = threadIdx.x;
  for (int t = tid; t < N; t += T1) c.sm()[pad1(t)] = c.GA[t];
  __syncthreads();
  double rho0 = 0.0;
  if (!density_starts<Rl, N, true>(c, rho0)) return false;
  const PlasmaConst& m = c.in->pc;
  const double Aeff = c.in->A_eff;
  const AffineStep aff(m);
  const bool no_ava = (m.ava == 0.0);
  double ion = 0.0;
  if (tid < NA) {
    double rho = rho0;
    for (int t = tid * CH; t < tid * CH + CH; ++t) {
      const C a = c.sm()[pad1(t)];
      const double Id = ((double)a.x * a.x + (double)a.y * a.y) / Aeff;
      const Rl I = (Rl)Id;
      const double w = (double)(float)lut_eval<Rl>(c.lut, I);
      const double wa = (double)(float)(m.ava * (double)I);
      const double rho_t = rho;
      ion = fmax(ion, rho_t);
      // without avalanche the exp-free step gives the same values (rho_step0)
      const double gen = no_ava ? rho_step0(rho, w, m, aff) : rho_step(rho, w, wa, m);
      const double loss = -(gen * m.Ui) / (2.0 * (double)I + 1e-30);
      const double cr = loss - m.sigma_half * rho_t;
      const double ci = -m.sigma_half * m.w0tc * rho_t;
      c.sm()[pad1(t)] = C{(Rl)(cr * a.x - ci * a.y), (Rl)(cr * a.y + ci * a.x)};
    }
  }
  if (ion_out) {   // block max of rho/rho_nt (every thread gets it)
    ion = warp_max(ion / m.rho_nt);
    if ((tid & 31) == 0) c.red[tid >> 5] = ion;
    __syncthreads();
    double mx = 0.0;
    for (int wv = 0; wv < T1 / 32; ++wv) mx = fmax(mx, c.red[wv]);
    *ion_out = fmax(*ion_out, mx);
  }
  __syncthreads();
  return true;
}

// One nonlinear evaluation N(u) in the omega domain (erk43ip_method.py:197-255
// plus the plasma term), with the stage input u formed on the fly.
// Returns sum |u|^2 for IN_5 (else 0).
template <typename Rl, int N>
__device__ __noinline__ double nl_eval(Ctx1<Rl>& c, int mode, double h, typename CT<Rl>::T* out,
                          typename CT<Rl>::T* hist_t, typename CT<Rl>::T* save_u = nullptr,
                          bool input_only = false, double* ion_out = nullptr) {
  using C = typename CT<Rl>::T;
  const int tid = threadIdx.x;
  const Rl hR = (Rl)h, h2 = (Rl)(h / 2), h6 = (Rl)(h / 6);
  double nrm = 0.0;
  // The stage loops load UB iterations' operands before any store, so a thread
  // waits on one round of L2 latency per UB elements (the stage arrays may alias
  // as far as the compiler knows, which would otherwise serialise them).
  constexpr int UB = 4;
  if (mode == IN_A) {
    for (int w = tid; w < N; w += T1) {
      const C u = c.A[w];
      c.sm()[pad1(w)] = u;
      if (save_u) save_u[w] = u;
    }
  } else if (mode == IN_5) {
    for (int w0 = tid; w0 < N; w0 += UB * T1) {
      C xt[UB], xp[UB];
#pragma unroll
      for (int q = 0; q < UB; ++q) {
        const int w = w0 + q * T1;
        if (w < N) { xt[q] = c.T[w]; xp[q] = c.A4P[w]; }
      }
#pragma unroll
      for (int q = 0; q < UB; ++q) {
        const int w = w0 + q * T1;
        if (w < N) {
          const C u = cadd(xt[q], cscale(xp[q], h6));
          c.A4[w] = u;
          nrm += (double)u.x * u.x + (double)u.y * u.y;
          c.sm()[pad1(w)] = u;
          if (save_u) save_u[w] = u;
        }
      }
    }
  } else {
    const C* X = mode == IN_2 ? c.K1 : c.O;
    for (int w0 = tid; w0 < N; w0 += UB * T1) {
      C xa[UB], xx[UB], xt[UB];
      double2 xd[UB];
#pragma unroll
      for (int q = 0; q < UB; ++q) {
        const int w = w0 + q * T1;
        if (w < N) {
          xa[q] = c.A[w];
          xx[q] = X[w];
          xd[q] = c.D[w];
          xt[q] = mode == IN_2 ? czero<C>() : c.T[w];
        }
      }
#pragma unroll
      for (int q = 0; q < UB; ++q) {
        const int w = w0 + q * T1;
        if (w < N) {
          const C E = EFac<Rl>::get(xd[q], 0.5 * h);
          const C v = cmul(xa[q], E);
          C u;
          if (mode == IN_2) {
            const C a1 = cmul(xx[q], E);
            c.T[w] = a1;
            u = cadd(v, cscale(a1, h2));
          } else if (mode == IN_3) {
            const C o = xx[q];
            c.T[w] = cadd(xt[q], cscale(o, (Rl)2));
            u = cadd(v, cscale(o, h2));
          } else {   // IN_4
            const C o = xx[q];
            const C ts = cadd(xt[q], cscale(o, (Rl)2));
            c.T[w] = cmul(cadd(v, cscale(ts, h6)), E);    // beta
            u = cmul(cadd(v, cscale(o, hR)), E);
          }
          c.sm()[pad1(w)] = u;
          if (save_u) save_u[w] = u;
        }
      }
    }
  }
  __syncthreads();
  if (input_only) return 0.0;     // stage input formed (and saved) only
  line_fft<N, +1>(c.sm(), c.tw, tid);
  const Rl invN = (Rl)(1.0 / N);
  const bool raman = c.in->raman, plasma = c.in->plasma;
  for (int t = tid; t < N; t += T1) {
    const C a = cscale(c.sm()[pad1(t)], invN);
    if (raman || plasma) c.GA[t] = a;
    if (hist_t) hist_t[t] = a;
    if (raman) {
      c.sm()[pad1(t)] = C{a.x * a.x + a.y * a.y, (Rl)0};
    } else {
      const Rl I = a.x * a.x + a.y * a.y;
      c.sm()[pad1(t)] = cscale(a, I);
    }
  }
  __syncthreads();
  if (raman) {
    // I_eff = (1 - f_R) I + f_R ifft(H_R fft(I))   (erk43ip_method.py:208-215)
    line_fft<N, -1>(c.sm(), c.tw, tid);
    for (int w = tid; w < N; w += T1) {
      const double2 Hw = c.H[w];
      c.sm()[pad1(w)] = cmul(c.sm()[pad1(w)], C{(Rl)Hw.x, (Rl)Hw.y});
    }
    __syncthreads();
    line_fft<N, +1>(c.sm(), c.tw, tid);
    const Rl fR = (Rl)c.in->f_R, g1 = (Rl)(1.0 - c.in->f_R);
    for (int t = tid; t < N; t += T1) {
      const C a = c.GA[t];
      const Rl I = a.x * a.x + a.y * a.y;
      const C Id = cscale(c.sm()[pad1(t)], invN);
      const C Ieff = C{g1 * I + fR * Id.x, fR * Id.y};
      c.sm()[pad1(t)] = cmul(a, Ieff);
    }
    __syncthreads();
  }
  line_fft<N, -1>(c.sm(), c.tw, tid);
  for (int w0 = tid; w0 < N; w0 += UB * T1) {
    double g[UB];
#pragma unroll
    for (int q = 0; q < UB; ++q) g[q] = w0 + q * T1 < N ? c.G[w0 + q * T1] : 0.0;
#pragma unroll
    for (int q = 0; q < UB; ++q) {
      const int w = w0 + q * T1;
      if (w < N) {
        const C p = c.sm()[pad1(w)];
        const Rl gr = (Rl)g[q];
        out[w] = C{-gr * p.y, gr * p.x};     // i gamma U(w) P_NL(w)
      }
    }
  }
  __syncthreads();
  if (plasma) {
    if (plasma_line<Rl, N>(c, ion_out)) {
      line_fft<N, -1>(c.sm(), c.tw, tid);
      for (int w0 = tid; w0 < N; w0 += UB * T1) {
        C o[UB];
#pragma unroll
        for (int q = 0; q < UB; ++q) if (w0 + q * T1 < N) o[q] = out[w0 + q * T1];
#pragma unroll
        for (int q = 0; q < UB; ++q) {
          const int w = w0 + q * T1;
          if (w < N) out[w] = cadd(o[q], c.sm()[pad1(w)]);
        }
      }
      __syncthreads();
    }
  }
  return mode == IN_5 ? block_sum(nrm, c.red) : 0.0;
}

// one erk43_step from the state (A, K1); leaves A4, a4' (A4P), a5 (O), beta (T);
// returns the error of erk43ip_method.py:279-284
template <typename Rl, int N>
__device__ __noinline__ double attempt1(Ctx1<Rl>& c, double h, typename CT<Rl>::T* hist_t,
                                        double* ion_cand = nullptr) {
  using C = typename CT<Rl>::T;
  const int tid = threadIdx.x;
  nl_eval<Rl, N>(c, IN_2, h, c.O, nullptr);     // alpha2
  nl_eval<Rl, N>(c, IN_3, h, c.O, nullptr);     // alpha3
  nl_eval<Rl, N>(c, IN_4, h, c.A4P, nullptr);   // alpha4'
  const double nrm = nl_eval<Rl, N>(c, IN_5, h, c.O, hist_t, nullptr, false, ion_cand);   // alpha5' = N(A4)
  double acc = 0.0;
  const Rl h30 = (Rl)(h / 30);
  for (int w = tid; w < N; w += T1) {
    if (sizeof(Rl) == 8) {
      const C a4 = c.A4P[w], a5 = c.O[w];
      const C A3 = cadd(c.T[w], cscale(cadd(cscale(a4, (Rl)2), cscale(a5, (Rl)3)), h30));
      const C d = csub(c.A4[w], A3);
      acc += (double)d.x * d.x + (double)d.y * d.y;
    } else {
      const C a4 = c.A4P[w], a5 = c.O[w];
      const double dx = (double)a4.x - a5.x, dy = (double)a4.y - a5.y;
      acc += dx * dx + dy * dy;
    }
  }
  double num = block_sum(acc, c.red);
  if (sizeof(Rl) != 8) num *= (h / 10.0) * (h / 10.0);
  double normA = sqrt(nrm / N);          // time-domain norm by Parseval
  if (normA < 1e-20) normA = 1.0;
  return sqrt(num / N) / normA;
}

// State of one adaptive run.
struct Run1 {
  double z, h, err;
  long long attempts, accepted;
  int status, hcount;
  double ion_peak;
};

// The adaptive loop (erk43ip_method.py:294-367) from the state (A, K1 = N(A)),
// evaluated identically by all threads; i indexes the step log (b.hlog).
template <typename Rl, int N>
__device__ __forceinline__ void adaptive_run(Ctx1<Rl>& c, const Batch1D& b, int i, const Inst1D& in,
                                             typename CT<Rl>::T* hist, double* zh, Run1& r) {
  using C = typename CT<Rl>::T;
  const int tid = threadIdx.x;
  double ion_peak = r.ion_peak, ion_cand = 0.0;
  const double L = in.L, tol = in.tol, max_step = in.max_step, min_step = in.min_step;
  double z = 0.0, h = max_step / 100, err = 0.0, err_prev = -1.0, zlast = 0.0;
  long long attempts = 0, accepted = 0;
  int status = 0, hcount = 1;
  auto cand = [&]() -> C* { return (hist && hcount < in.hist_cap) ? hist + (long long)hcount * N : nullptr; };
  auto accept = [&](double hh) {
    z += hh;
    ion_peak = fmax(ion_peak, ion_cand);    // the accepted state's density (FSAL evaluation)
    C* t0 = c.A; c.A = c.A4; c.A4 = t0;     // state <- A4
    C* t1 = c.K1; c.K1 = c.O; c.O = t1;     // k1 <- alpha5' (FSAL)
    if (b.hlog) {                           // step log for the adjoint
      if (accepted < b.hlog_cap) { if (tid == 0) b.hlog[(long long)i * b.hlog_cap + accepted] = hh; }
      else status |= 16;
    }
    accepted += 1;
    if (hcount < 1000 || (z - zlast) > L / 500) {   // :327
      if (hist && hcount < in.hist_cap) {
        if (tid == 0) zh[hcount] = z;
        hcount += 1;
        zlast = z;
      } else if (hist) {
        status |= 8;   // history capacity exhausted
      }
    }
  };
  if (b.hsched) {
    // replay of a fixed step sequence, every step accepted (no control)
    const double* hs = b.hsched + (long long)i * b.nsched;
    for (int k = 0; k < b.nsched; ++k) {
      const double hh = hs[k];
      ion_cand = 0.0;
      err = attempt1<Rl, N>(c, hh, cand(), &ion_cand);
      attempts += 1;
      if (!isfinite(err)) { status |= UPPE_STATUS_NONFINITE; break; }
      accept(hh);
    }
  }
  while (!b.hsched && z < L) {
    if (z + h > L) h = L - z;
    ion_cand = 0.0;
    err = attempt1<Rl, N>(c, h, cand(), &ion_cand);
    attempts += 1;
    if (!isfinite(h) || (!isfinite(err) && h <= min_step)) { status |= UPPE_STATUS_NONFINITE; break; }
    if (!isfinite(err)) {
      // the attempt overflowed (the state is untouched): retry with a tenth of the step
      status |= UPPE_STATUS_RETRIED;
      h = fmax(h * 0.1, min_step);
    } else if (err < tol) {
      accept(h);
      double factor = 0.95 * pow(tol / (err + 1e-30), 0.25);
      if (err_prev >= 0.0 && err_prev > 1e-30) factor *= pow(err_prev / (err + 1e-30), 0.1);
      err_prev = err;
      h = fmin(h * fmin(factor, 2.0), max_step);
    } else {
      const double factor = 0.95 * pow(tol / (err + 1e-30), 0.25);
      h = fmax(h * fmax(factor, 0.1), min_step);
      if (h <= min_step) {   // forced step (:345-367)
        ion_cand = 0.0;
        err = attempt1<Rl, N>(c, h, cand(), &ion_cand);
        attempts += 1;
        status |= UPPE_STATUS_MIN_STEP;
        if (!isfinite(err)) { status |= UPPE_STATUS_NONFINITE; break; }
        accept(h);
        err_prev = -1.0;
      }
    }
    if (in.max_attempts > 0 && attempts >= in.max_attempts && z < L) {
      status |= UPPE_STATUS_MAX_ATTEMPTS;
      break;
    }
  }
  r.z = z; r.h = h; r.err = err;
  r.attempts = attempts; r.accepted = accepted;
  r.status = status; r.hcount = hcount;
  r.ion_peak = ion_peak;
}

// energy sum |A|^2 dt and photon number (Parseval in omega), FP64, fixed order
template <typename Rl, int N>
__device__ __forceinline__ void energy_photons(Ctx1<Rl>& c, const Inst1D& in, double& en, double& ph) {
  using C = typename CT<Rl>::T;
  const int tid = threadIdx.x;
  en = 0.0;
  ph = 0.0;
  {
    const double dw = 6.283185307179586476925286766559 / (N * in.dt);
    for (int w = tid; w < N; w += T1) {
      const C v = c.A[w];
      const double a2 = (double)v.x * v.x + (double)v.y * v.y;
      en += a2;
      const double wa = in.omega0 + dw * (w < (N + 1) / 2 ? w : w - N);
      if (wa > 0.0) ph += a2 / (1.054571817e-34 * wa);
    }
    en = block_sum(en, c.red) * in.dt / N;
    ph = block_sum(ph, c.red) * in.dt / N;
  }
}

template <typename Rl, int N>
__device__ void run_instance(const Batch1D& b, int i, unsigned char* smem) {
  using C = typename CT<Rl>::T;
  const int tid = threadIdx.x;
  const Inst1D& in = b.inst[i];
  Ctx1<Rl> c;
  c.red = reinterpret_cast<double*>(smem + sizeof(C) * Cfg1<N>::PAD);
  c.starts = c.red + 64;
  c.tw = reinterpret_cast<const C*>(b.tw) + (N - 1);
  C* sc = reinterpret_cast<C*>(b.scratch) + (long long)blockIdx.x * b.scratch_per_block;
  c.A = sc; c.K1 = sc + N; c.T = sc + 2 * N; c.O = sc + 3 * N;
  c.A4 = sc + 4 * N; c.A4P = sc + 5 * N; c.GA = sc + 6 * N;
  c.D = b.D + in.off;
  c.G = b.G + in.off;
  c.H = b.H ? b.H + in.off : nullptr;
  c.in = &in;
  c.lut = b.lut;
  if (c.lut.n > 1 && c.lut.inv_dx == 0.0) {
    // a table passed without its grid constants (the allocation-free entry
    // point): the first-index guess comes from the table's ends, as plans set it
    const Rl* xp = reinterpret_cast<const Rl*>(c.lut.x);
    c.lut.x0 = (double)xp[0];
    c.lut.inv_dx = (c.lut.n - 1) / ((double)xp[c.lut.n - 1] - c.lut.x0);
  }
  C* field = reinterpret_cast<C*>(b.field) + in.off;
  C* hist = in.hist_cap > 0 ? reinterpret_cast<C*>(b.hist) + in.hist_off : nullptr;
  double* zh = in.hist_cap > 0 ? b.zhist + in.zh_off : nullptr;

  // A0 -> history slot 0, state = fft(A0)
  for (int t = tid; t < N; t += T1) {
    const C a = field[t];
    c.sm()[pad1(t)] = a;
    if (hist) hist[t] = a;
  }
  if (zh && tid == 0) zh[0] = 0.0;
  __syncthreads();
  line_fft<N, -1>(c.sm(), c.tw, tid);
  for (int w = tid; w < N; w += T1) c.A[w] = c.sm()[pad1(w)];
  __syncthreads();
  double ion_peak = 0.0;
  nl_eval<Rl, N>(c, IN_A, 0.0, c.K1, nullptr, nullptr, false, &ion_peak);   // k1 = N(A)

  Run1 run;
  run.ion_peak = ion_peak;
  adaptive_run<Rl, N>(c, b, i, in, hist, zh, run);
  const double z = run.z, h = run.h, err = run.err;
  const long long attempts = run.attempts, accepted = run.accepted;
  const int status = run.status, hcount = run.hcount;
  ion_peak = run.ion_peak;
  double en, ph;
  energy_photons<Rl, N>(c, in, en, ph);
  // final state back to the time domain
  for (int w = tid; w < N; w += T1) c.sm()[pad1(w)] = c.A[w];
  __syncthreads();
  line_fft<N, +1>(c.sm(), c.tw, tid);
  const Rl invN = (Rl)(1.0 / N);
  for (int t = tid; t < N; t += T1) field[t] = cscale(c.sm()[pad1(t)], invN);
  if (tid == 0) {
    Res1D r;
    r.z = z; r.h = h; r.err = err; r.attempts = attempts; r.accepted = accepted;
    r.status = status; r.hist_count = hist ? hcount : 0;
    r.energy = en; r.photons = in.omega0 > 0.0 ? ph : NAN; r.peak_ion = ion_peak;
    b.res[i] = r;
  }
  __syncthreads();
}


// One propagation program (a multipass cell: slices with their own tables,
// mirrors with loss and GDD/TOD) run by this CTA with the state kept on chip
// between operations (gas.py:104-147; test_gaussian_pulse GDD TOD 1mj copy.py:
// 196-290).  Each propagation starts like a fresh propagate() call: h0 =
// max_step/100, no controller memory, z from 0.
template <typename Rl, int N>
__device__ void run_program(const Batch1D& b, int p, unsigned char* smem) {
  using C = typename CT<Rl>::T;
  const int tid = threadIdx.x;
  const Prog1D& pg = b.prog[p];
  Ctx1<Rl> c;
  c.red = reinterpret_cast<double*>(smem + sizeof(C) * Cfg1<N>::PAD);
  c.starts = c.red + 64;
  c.tw = reinterpret_cast<const C*>(b.tw) + (N - 1);
  C* sc = reinterpret_cast<C*>(b.scratch) + (long long)blockIdx.x * b.scratch_per_block;
  c.A = sc; c.K1 = sc + N; c.T = sc + 2 * N; c.O = sc + 3 * N;
  c.A4 = sc + 4 * N; c.A4P = sc + 5 * N; c.GA = sc + 6 * N;
  c.lut = b.lut;
  C* field = reinterpret_cast<C*>(b.field) + pg.field_off;
  C* rec = b.records ? reinterpret_cast<C*>(b.records) + pg.rec_off : nullptr;
  const Rl invN = (Rl)(1.0 / N);
  for (int t = tid; t < N; t += T1) c.sm()[pad1(t)] = field[t];
  __syncthreads();
  line_fft<N, -1>(c.sm(), c.tw, tid);
  for (int w = tid; w < N; w += T1) c.A[w] = c.sm()[pad1(w)];
  __syncthreads();
  for (long long o = pg.op_begin; o < pg.op_end; ++o) {
    const Op1D op = b.ops[o];
    Res1D r;
    memset(&r, 0, sizeof(r));
    if (op.inst >= 0) {
      const Inst1D& in = b.inst[op.inst];
      c.D = b.D + in.off;
      c.G = b.G + in.off;
      c.H = b.H ? b.H + in.off : nullptr;
      c.in = &in;
      double ion = 0.0;
      nl_eval<Rl, N>(c, IN_A, 0.0, c.K1, nullptr, nullptr, false, &ion);   // k1 with these tables
      Run1 run;
      run.ion_peak = ion;
      adaptive_run<Rl, N>(c, b, -1, in, nullptr, nullptr, run);
      double en, ph;
      energy_photons<Rl, N>(c, in, en, ph);
      r.z = run.z; r.h = run.h; r.err = run.err; r.attempts = run.attempts;
      r.accepted = run.accepted; r.status = run.status; r.energy = en;
      r.photons = in.omega0 > 0.0 ? ph : NAN; r.peak_ion = run.ion_peak;
    } else {
      // mirror: loss and spectral phase on the omega-domain state
      const double dw = 6.283185307179586476925286766559 / (N * pg.dt);
      double en = 0.0;
      for (int w = tid; w < N; w += T1) {
        const double om = dw * (w < (N + 1) / 2 ? w : w - N);
        double sn, cs;
        sincos(0.5 * op.gdd * om * om + (1.0 / 6.0) * op.tod * om * om * om, &sn, &cs);
        const C a = c.A[w];
        const double ar = op.amp * ((double)a.x * cs - (double)a.y * sn);
        const double ai = op.amp * ((double)a.x * sn + (double)a.y * cs);
        c.A[w] = C{(Rl)ar, (Rl)ai};
        en += ar * ar + ai * ai;
      }
      r.energy = block_sum(en, c.red) * pg.dt / N;
      r.photons = NAN;
    }
    if (op.record && rec) {
      for (int w = tid; w < N; w += T1) c.sm()[pad1(w)] = c.A[w];
      __syncthreads();
      line_fft<N, +1>(c.sm(), c.tw, tid);
      for (int t = tid; t < N; t += T1) rec[t] = cscale(c.sm()[pad1(t)], invN);
      rec += N;
      r.hist_count = 1;
      __syncthreads();
    }
    if (tid == 0) b.op_res[o] = r;
    __syncthreads();
  }
  for (int w = tid; w < N; w += T1) c.sm()[pad1(w)] = c.A[w];
  __syncthreads();
  line_fft<N, +1>(c.sm(), c.tw, tid);
  for (int t = tid; t < N; t += T1) field[t] = cscale(c.sm()[pad1(t)], invN);
  __syncthreads();
}

template <typename Rl>
__global__ void __launch_bounds__(T1, 1) k_uppe1d(Batch1D b) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ int s_k;
  mark_busy(b.busy, 0);
  for (;;) {
    if (threadIdx.x == 0) s_k = atomicAdd(b.counter, 1);
    __syncthreads();
    const int k = s_k;
    __syncthreads();
    if (k >= b.ninst) { mark_busy(b.busy, 1); return; }
    const int i = b.order[k];
    if (b.prog) {
      switch (b.prog[i].log2n) {
        case 6: run_program<Rl, 64>(b, i, smem); break;
        case 7: run_program<Rl, 128>(b, i, smem); break;
        case 8: run_program<Rl, 256>(b, i, smem); break;
        case 9: run_program<Rl, 512>(b, i, smem); break;
        case 10: run_program<Rl, 1024>(b, i, smem); break;
        case 11: run_program<Rl, 2048>(b, i, smem); break;
        case 12: run_program<Rl, 4096>(b, i, smem); break;
        case 13: run_program<Rl, 8192>(b, i, smem); break;
        case 14: if (sizeof(Rl) == 4) run_program<Rl, 16384>(b, i, smem); break;
        default: break;
      }
      continue;
    }
    switch (b.inst[i].log2n) {
      case 6: run_instance<Rl, 64>(b, i, smem); break;
      case 7: run_instance<Rl, 128>(b, i, smem); break;
      case 8: run_instance<Rl, 256>(b, i, smem); break;
      case 9: run_instance<Rl, 512>(b, i, smem); break;
      case 10: run_instance<Rl, 1024>(b, i, smem); break;
      case 11: run_instance<Rl, 2048>(b, i, smem); break;
      case 12: run_instance<Rl, 4096>(b, i, smem); break;
      case 13: run_instance<Rl, 8192>(b, i, smem); break;
      case 14: if (sizeof(Rl) == 4) run_instance<Rl, 16384>(b, i, smem); break;
      default: break;
    }
  }
}

// ---------------------------------------------------------------------------
// Adjoint (reverse mode) of the ERK4(3)-IP step for Kerr + steepening with
// dispersion, loss and the plasma term (no Raman, no avalanche), complex128.
// Convention: for a real loss L and complex x, the cotangent xb satisfies
// dL = Re sum conj(xb) dx (the same as torch's complex gradients).  Frozen
// accepted step sizes.
// ---------------------------------------------------------------------------
// Reverse mode of the plasma term over the line (complex128): field a_t in GA,
// cotangent q_t of the term's time samples in the shared line.  Writes the field
// cotangent into acc and adds d/d(rho_nt, sigma_drude, omega0 tau_c) into gpl
// (thread 0).  The density cotangent obeys lam_t = A_t lam_{t+1} + B_t: each
// thread composes its chunk's maps, a block suffix scan gives every chunk its
// end value, and the chunk is walked back once more.  Returns false (nothing
// written) when the line does not ionise.
template <int N>
__device__ bool plasma_vjp1(Ctx1<double>& c, double2* acc, double* gpl) {
  using C = double2;
  constexpr int CH = Cfg1<N>::CH, NA = Cfg1<N>::NA;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  double rho0 = 0.0;
  if (!density_starts<double, N>(c, rho0)) return false;
  const PlasmaConst& m = c.in->pc;
  const double Aeff = c.in->A_eff, alpha = 1.0 / Aeff;
  const AffineStep aff(m);
  double cur[CH];
  double Ac = 1.0, Bc = 0.0;
  if (tid < NA) {
    double rho = rho0;
    for (int i = 0; i < CH; ++i) {
      const C a = c.GA[tid * CH + i];
      const double I = (a.x * a.x + a.y * a.y) / Aeff;
      cur[i] = rho;
      rho_step(rho, (double)(float)lut_eval<double>(c.lut, I), 0.0, m);
    }
    for (int i = CH - 1; i >= 0; --i) {
      const int t = tid * CH + i;
      const C a = c.GA[t], q = c.sm()[pad1(t)];
      const double I = (a.x * a.x + a.y * a.y) / Aeff;
      double A, B;
      plasma_rev<false>(m, aff, alpha, cur[i], (double)(float)lut_eval<double>(c.lut, I),
                        lut_slope<double>(c.lut, I), I, a.x, a.y, q.x, q.y, A, B);
      Bc = A * Bc + B;
      Ac = A * Ac;
    }
  }
  // inclusive suffix scan over the warp: (A, B) o (A', B') = (A A', A B' + B)
  double sa = Ac, sb = Bc;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const double an = __shfl_down_sync(0xffffffffu, sa, off);
    const double bn = __shfl_down_sync(0xffffffffu, sb, off);
    if (lane + off < 32) { sb = sa * bn + sb; sa = sa * an; }
  }
  double* wa = c.starts;              // warp composites, then the value at each warp's end
  double* wb = c.starts + T1 / 32;
  if (lane == 0) { wa[warp] = sa; wb[warp] = sb; }
  __syncthreads();
  if (tid == 0) {
    double lam = 0.0;                 // cotangent of the density after the last sample
    for (int w = T1 / 32 - 1; w >= 0; --w) {
      const double a2 = wa[w], b2 = wb[w];
      wb[w] = lam;
      lam = a2 * lam + b2;
    }
  }
  __syncthreads();
  double xa = __shfl_down_sync(0xffffffffu, sa, 1);
  double xb = __shfl_down_sync(0xffffffffu, sb, 1);
  if (lane == 31) { xa = 1.0; xb = 0.0; }
  double lam = xa * wb[warp] + xb;    // cotangent of the density at this chunk's end
  double g[3] = {0.0, 0.0, 0.0};
  if (tid < NA) {
    for (int i = CH - 1; i >= 0; --i) {
      const int t = tid * CH + i;
      const C a = c.GA[t], q = c.sm()[pad1(t)];
      const double I = (a.x * a.x + a.y * a.y) / Aeff;
      double A, B, oar, oai;
      plasma_rev<true>(m, aff, alpha, cur[i], (double)(float)lut_eval<double>(c.lut, I),
                       lut_slope<double>(c.lut, I), I, a.x, a.y, q.x, q.y, A, B, lam, &oar, &oai, g);
      acc[t] = C{oar, oai};
      lam = A * lam + B;
    }
  }
  for (int k = 0; k < 3; ++k) {
    const double tot = block_sum(g[k], c.red);
    if (tid == 0 && gpl) gpl[k] += tot;
  }
  return true;
}

// VJP of N(u) = i G F(|a|^2 a) + F(P(a)), a = F^* u / N, with cotangent nb:
//   p^b = F^*(-i G nb), ab = 2|a|^2 p^b + a^2 conj(p^b) + VJP_P(F^* nb), ub = F ab / N;
// accumulates gG[w] += Re(conj(nb) i F(|a|^2 a)).
template <int N>
__device__ __noinline__ void vjp_eval(Ctx1<double>& c, const double2* u, const double2* nb,
                                      double2* out, double* gG, double* gpl) {
  using C = double2;
  const int tid = threadIdx.x;
  const double invN = 1.0 / N;
  const bool pl = c.in->plasma;
  for (int w = tid; w < N; w += T1) c.sm()[pad1(w)] = u[w];
  __syncthreads();
  line_fft<N, +1>(c.sm(), c.tw, tid);
  for (int t = tid; t < N; t += T1) {
    const C a = cscale(c.sm()[pad1(t)], invN);
    c.GA[t] = a;
    if (!pl) c.sm()[pad1(t)] = cscale(a, a.x * a.x + a.y * a.y);
  }
  __syncthreads();
  bool pl_any = false;
  if (pl) {   // plasma term: q = F*(nb) (time domain), field cotangent into A4P
    for (int w = tid; w < N; w += T1) c.sm()[pad1(w)] = nb[w];
    __syncthreads();
    line_fft<N, +1>(c.sm(), c.tw, tid);
    pl_any = plasma_vjp1<N>(c, c.A4P, gpl);
    __syncthreads();
    for (int t = tid; t < N; t += T1) {
      const C a = c.GA[t];
      c.sm()[pad1(t)] = cscale(a, a.x * a.x + a.y * a.y);
    }
    __syncthreads();
  }
  line_fft<N, -1>(c.sm(), c.tw, tid);
  for (int w = tid; w < N; w += T1) {
    const C ph = c.sm()[pad1(w)];
    const C n = nb[w];
    gG[w] += -n.x * ph.y + n.y * ph.x;
    const double g = c.G[w];
    c.sm()[pad1(w)] = C{g * n.y, -g * n.x};          // -i G nb
  }
  __syncthreads();
  line_fft<N, +1>(c.sm(), c.tw, tid);
  for (int t = tid; t < N; t += T1) {
    const C a = c.GA[t];
    const C pb = c.sm()[pad1(t)];
    const double I2 = 2.0 * (a.x * a.x + a.y * a.y);
    const C a2 = cmul(a, a);
    C ab = cadd(cscale(pb, I2), cmul(a2, cconj(pb)));
    if (pl_any) ab = cadd(ab, c.A4P[t]);
    c.sm()[pad1(t)] = ab;
  }
  __syncthreads();
  line_fft<N, -1>(c.sm(), c.tw, tid);
  for (int w = tid; w < N; w += T1) out[w] = cscale(c.sm()[pad1(w)], invN);
  __syncthreads();
}

struct Adj1D {
  Batch1D b;            // tables, twiddles, instance records of the plan
  int inst;
  const double* hlog;   // accepted step sizes of the forward run
  int nsteps, K;        // steps, checkpoint interval
  const double2* A0;    // time-domain input field
  const double2* Abar;  // cotangent of the final state (omega domain)
  double2* A0bar;       // out: cotangent of fft(A0) (omega domain)
  double2* gD;          // out: dL/dD
  double* gG;           // out: dL/dG
  double2* rhs;         // out: D A_L + N(A_L) (for d/dL)
  double* gPl;          // out: d/d(rho_nt, sigma_drude, omega0 tau_c) (plasma instances)
  double2* work;        // 18 N + (ceil(nsteps/K) + K) N complex
};

template <int N>
__device__ void adjoint_instance(const Adj1D& a, unsigned char* smem) {
  using C = double2;
  const int tid = threadIdx.x;
  const Inst1D& in = a.b.inst[a.inst];
  Ctx1<double> c;
  c.red = reinterpret_cast<double*>(smem + sizeof(C) * Cfg1<N>::PAD);
  c.starts = c.red + 64;
  c.tw = reinterpret_cast<const C*>(a.b.tw) + (N - 1);
  C* w = a.work;
  c.A = w; c.K1 = w + N; c.T = w + 2 * N; c.O = w + 3 * N;
  c.A4 = w + 4 * N; c.A4P = w + 5 * N; c.GA = w + 6 * N;
  C *A2 = w + 7 * N, *A3 = w + 8 * N, *U2 = w + 9 * N, *U3 = w + 10 * N, *U4 = w + 11 * N;
  C *AB = w + 12 * N, *VB = w + 13 * N, *A1B = w + 14 * N, *A2B = w + 15 * N, *A3B = w + 16 * N;
  C *TMP = w + 17 * N;
  const int nseg = (a.nsteps + a.K - 1) / a.K;
  C* CK = w + 18 * N;
  C* SEG = CK + (long long)(nseg > 0 ? nseg : 1) * N;
  c.D = a.b.D + in.off;
  c.G = a.b.G + in.off;
  c.H = nullptr;
  c.in = &in;
  c.lut = a.b.lut;
  auto copy = [&](C* dst, const C* src) {
    for (int x = tid; x < N; x += T1) dst[x] = src[x];
    __syncthreads();
  };
  auto advance = [&](double hh) {      // one accepted forward step (state A, FSAL K1)
    attempt1<double, N>(c, hh, nullptr);
    C* t0 = c.A; c.A = c.A4; c.A4 = t0;
    C* t1 = c.K1; c.K1 = c.O; c.O = t1;
  };
  // forward replay with checkpoints every K steps
  for (int t = tid; t < N; t += T1) c.sm()[pad1(t)] = a.A0[t];
  __syncthreads();
  line_fft<N, -1>(c.sm(), c.tw, tid);
  for (int x = tid; x < N; x += T1) { c.A[x] = c.sm()[pad1(x)]; a.gD[x] = C{0, 0}; a.gG[x] = 0.0; }
  if (tid < 3 && a.gPl) a.gPl[tid] = 0.0;
  __syncthreads();
  copy(CK, c.A);
  nl_eval<double, N>(c, IN_A, 0.0, c.K1, nullptr);
  for (int j = 0; j < a.nsteps; ++j) {
    advance(a.hlog[j]);
    if ((j + 1) % a.K == 0 && j + 1 < a.nsteps) copy(CK + (long long)((j + 1) / a.K) * N, c.A);
  }
  // d/dL of the final state: D A_L + N(A_L) (K1 holds N(A_L) by FSAL)
  for (int x = tid; x < N; x += T1) a.rhs[x] = cadd(cmul(c.D[x], c.A[x]), c.K1[x]);
  copy(AB, a.Abar);
  C* O0 = c.O;
  for (int sg = nseg - 1; sg >= 0; --sg) {
    const int j0 = sg * a.K, j1 = min(a.nsteps, j0 + a.K);
    copy(c.A, CK + (long long)sg * N);
    copy(SEG, c.A);
    nl_eval<double, N>(c, IN_A, 0.0, c.K1, nullptr);
    for (int j = j0; j < j1 - 1; ++j) {
      advance(a.hlog[j]);
      copy(SEG + (long long)(j - j0 + 1) * N, c.A);
    }
    for (int j = j1 - 1; j >= j0; --j) {
      const double h = a.hlog[j];
      // recompute the step's stage inputs from its start state
      copy(c.A, SEG + (long long)(j - j0) * N);
      nl_eval<double, N>(c, IN_A, 0.0, c.K1, nullptr);            // k1
      nl_eval<double, N>(c, IN_2, h, A2, nullptr, U2);            // T = a1, a2
      C* Osave = c.O;
      c.O = A2;
      nl_eval<double, N>(c, IN_3, h, A3, nullptr, U3);            // T += 2 a2, a3
      c.O = A3;
      nl_eval<double, N>(c, IN_4, h, nullptr, nullptr, U4, true); // T = beta, u4
      c.O = Osave;
      // reverse of A' = beta + h/6 a4, beta = E (v + h/6 T)
      for (int x = tid; x < N; x += T1) {
        const C E = EFac<double>::get(c.D[x], 0.5 * h);
        const C ab = AB[x];
        a.gD[x] = cadd(a.gD[x], cscale(cmul(ab, cconj(c.T[x])), 0.5 * h));
        const C wb = cmul(cconj(E), ab);
        const C tb = cscale(wb, h / 6);
        VB[x] = wb;
        A1B[x] = tb;
        A2B[x] = cscale(tb, 2.0);
        A3B[x] = cscale(tb, 2.0);
        TMP[x] = cscale(ab, h / 6);                  // a4 bar
      }
      __syncthreads();
      vjp_eval<N>(c, U4, TMP, AB, a.gG, a.gPl);             // u4 bar -> AB
      for (int x = tid; x < N; x += T1) {            // u4 = E z, z = v + h a3
        const C E = EFac<double>::get(c.D[x], 0.5 * h);
        const C u4b = AB[x];
        a.gD[x] = cadd(a.gD[x], cscale(cmul(u4b, cconj(U4[x])), 0.5 * h));
        const C zb = cmul(cconj(E), u4b);
        VB[x] = cadd(VB[x], zb);
        A3B[x] = cadd(A3B[x], cscale(zb, h));
      }
      __syncthreads();
      vjp_eval<N>(c, U3, A3B, TMP, a.gG, a.gPl);            // u3 bar
      for (int x = tid; x < N; x += T1) {            // u3 = v + h/2 a2
        VB[x] = cadd(VB[x], TMP[x]);
        A2B[x] = cadd(A2B[x], cscale(TMP[x], h / 2));
      }
      __syncthreads();
      vjp_eval<N>(c, U2, A2B, TMP, a.gG, a.gPl);            // u2 bar
      for (int x = tid; x < N; x += T1) {            // u2 = v + h/2 a1, a1 = E k1
        const C E = EFac<double>::get(c.D[x], 0.5 * h);
        VB[x] = cadd(VB[x], TMP[x]);
        const C a1b = cadd(A1B[x], cscale(TMP[x], h / 2));
        const C a1 = cmul(E, c.K1[x]);
        a.gD[x] = cadd(a.gD[x], cscale(cmul(a1b, cconj(a1)), 0.5 * h));
        TMP[x] = cmul(cconj(E), a1b);                // k1 bar
      }
      __syncthreads();
      vjp_eval<N>(c, c.A, TMP, AB, a.gG, a.gPl);            // through k1 = N(A)
      for (int x = tid; x < N; x += T1) {            // v = E A
        const C E = EFac<double>::get(c.D[x], 0.5 * h);
        const C vb = VB[x];
        const C v = cmul(E, c.A[x]);
        a.gD[x] = cadd(a.gD[x], cscale(cmul(vb, cconj(v)), 0.5 * h));
        AB[x] = cadd(AB[x], cmul(cconj(E), vb));
      }
      __syncthreads();
    }
  }
  c.O = O0;
  copy(a.A0bar, AB);
}

static __global__ void __launch_bounds__(T1, 1) k_uppe1d_adjoint(Adj1D a) {
  extern __shared__ __align__(16) unsigned char smem[];
  switch (a.b.inst[a.inst].log2n) {
    case 6: adjoint_instance<64>(a, smem); break;
    case 7: adjoint_instance<128>(a, smem); break;
    case 8: adjoint_instance<256>(a, smem); break;
    case 9: adjoint_instance<512>(a, smem); break;
    case 10: adjoint_instance<1024>(a, smem); break;
    case 11: adjoint_instance<2048>(a, smem); break;
    case 12: adjoint_instance<4096>(a, smem); break;
    case 13: adjoint_instance<8192>(a, smem); break;
    default: break;
  }
}

cudaError_t launch_uppe1d_adjoint(const Adj1D& a, size_t smem, cudaStream_t s);

// launcher implemented once per precision (uppe1d_f32.cu / uppe1d_f64.cu)
template <typename Rl> cudaError_t launch_uppe1d(const Batch1D& b, int nblocks, size_t smem, cudaStream_t s);

}  // namespace uppe

