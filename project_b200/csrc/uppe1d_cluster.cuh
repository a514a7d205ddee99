#pragma once
// 1D ERK4(3)-IP propagation of one instance by a thread-block cluster of CS = 4
// or 8 CTAs (long lines, sm_100a distributed shared memory).
//
// The single-CTA kernel (uppe1d_kernel.cuh) runs a whole instance on one SM, so a
// batch takes as long as its longest line.  Here the CTAs of a cluster share one
// line of N = CS M points (written below for CS = 4; with eight CTAs the cross
// step is radix 8):
//   * time domain: CTA r holds samples n = r M + m (m < M) in its shared line;
//   * omega domain: CTA r holds the bins k = r + 4 j (j < M), at index j;
//   * a forward transform is one radix-4 step across the cluster (each CTA reads
//     sample m of all four lines through distributed shared memory, combines them
//     with W_4^(q r) and twiddles by W_N^(m r)) followed by a local M-point FFT;
//     the inverse is the local inverse FFT, the conjugate twiddle and the radix-4
//     step;  k = r + 4 j with X[r + 4 j] = sum_m W_M^(m j) W_N^(m r) sum_q
//     W_4^(q r) x[q M + m];
//   * sums (error norm, energy) are per-CTA block sums combined in rank order, so
//     all four CTAs take the same decisions; the density scan composes the four
//     CTAs' affine maps (or runs the exact serial update CTA by CTA when a clamp
//     binds).
// The stage arrays live in a per-cluster global scratch in CTA-major order (CTA
// r's bins at r M + j), with the D and G tables copied into the same order.  The
// arithmetic per element is that of the single-CTA kernel; the transforms split
// differently, so results agree to rounding, not bit for bit.
#include <cooperative_groups.h>

#include "uppe1d_kernel.cuh"

namespace uppe {
namespace cg = cooperative_groups;

constexpr int kCS = 4;   // CTAs per line by default (8 is the other supported size)

// offset (elements) of the cross-CTA twiddles W_N^(m r), r = 1..3, m < M = N/4,
// for every M = 512 .. 4096: 3 (M - 512), entry (r - 1) M + m
// (for CS CTAs per line: (CS - 1) entries per M, M = 2048 / CS .. 16384 / CS)
__host__ __device__ constexpr long long cl_xtw_offset(int M, int CS = kCS) {
  return (long long)(CS - 1) * (M - 2048 / CS);
}

template <typename Rl> struct ClCtx {
  using C = typename CT<Rl>::T;
  // the two line buffers at the start of the dynamic shared memory (PAD elements
  // each), addressed through the shared array itself so that accesses compile to
  // shared-memory instructions; cur selects the one that holds the line
  int cur;
  int pad;
  __device__ __forceinline__ C* sbase() const {
    extern __shared__ __align__(16) unsigned char smem[];
    return reinterpret_cast<C*>(smem);
  }
  __device__ __forceinline__ C* line() const { return sbase() + cur * pad; }
  __device__ __forceinline__ C* buf() const { return sbase() + (cur ^ 1) * pad; }
  double* red;           // shared: 64 doubles (block sums)
  double* starts;        // shared: density at the start of each chunk (T1)
  double* slot;          // shared: 8 doubles exchanged across the cluster
  const C* tw;           // per-pass table of the local M-point FFT
  const C* xtw;          // W_N^(m r), r = 1..3
  C *A, *K1, *T, *O, *A4, *A4P, *GA;   // this CTA's slices of the stage arrays
  const double2* D;      // this CTA's bins of D, G (CTA-major copies)
  const double* G;
  const Inst1D* in;
  Lut lut;
  int r;                 // rank in the cluster
};

// x * W_CS^e (DIR = -1: exp(-2 pi i e / CS); +1: exp(+2 pi i e / CS)), CS = 4 or 8
template <int DIR, int CS, typename C> __device__ __forceinline__ C wcs(C x, int e) {
  if constexpr (CS == 4) {
    switch (e & 3) {
      case 0: return x;
      case 1: return mul_pmi<DIR>(x);
      case 2: return C{-x.x, -x.y};
      default: return mul_pmi<-DIR>(x);
    }
  } else {
    switch (e & 7) {
      case 0: return x;
      case 1: return rot<8, 1, DIR>(x);
      case 2: return rot<8, 2, DIR>(x);
      case 3: return rot<8, 3, DIR>(x);
      case 4: return rot<8, 4, DIR>(x);
      case 5: return rot<8, 5, DIR>(x);
      case 6: return rot<8, 6, DIR>(x);
      default: return rot<8, 7, DIR>(x);
    }
  }
}

// radix-4 step across the cluster into buf, then swap line/buf.  DIR = -1: out[m]
// = W_N^(m r) sum_q W_4^(q r) line_q[m]; DIR = +1: out[m] = sum_q W_4^(-q r)
// line_q[m] (the caller has applied the conjugate twiddles to line_q).
template <typename Rl, int M, int DIR, int CS>
__device__ __forceinline__ void cl_cross(ClCtx<Rl>& c, cg::cluster_group& cl) {
  using C = typename CT<Rl>::T;
  cl.sync();                                   // every CTA's line is complete
  C* rem[CS];
#pragma unroll
  for (int q = 0; q < CS; ++q) rem[q] = cl.map_shared_rank(c.line(), q);
  const int r = c.r;
  // all of a thread's remote loads in flight together (M / T1 <= 8 iterations)
#pragma unroll
  for (int m = threadIdx.x; m < M; m += T1) {
    C acc = rem[0][pad1(m)];
#pragma unroll
    for (int q = 1; q < CS; ++q) acc = cadd(acc, wcs<DIR, CS>(rem[q][pad1(m)], q * r));
    if (DIR < 0 && r > 0) acc = cmul(acc, c.xtw[(r - 1) * M + m]);
    c.buf()[pad1(m)] = acc;
  }
  cl.sync();                                   // every CTA has read the lines
  c.cur ^= 1;
}

// time domain (CTA r: samples r M + m) -> omega domain (CTA r: bins r + 4 j)
template <typename Rl, int M, int CS>
__device__ __forceinline__ void cl_fft_fwd(ClCtx<Rl>& c, cg::cluster_group& cl) {
  cl_cross<Rl, M, -1, CS>(c, cl);
  line_fft<M, -1>(c.line(), c.tw, threadIdx.x);
}

// omega domain -> time domain, unnormalised
template <typename Rl, int M, int CS>
__device__ __forceinline__ void cl_fft_inv(ClCtx<Rl>& c, cg::cluster_group& cl) {
  using C = typename CT<Rl>::T;
  line_fft<M, +1>(c.line(), c.tw, threadIdx.x);
  if (c.r > 0) {
    for (int m = threadIdx.x; m < M; m += T1) c.line()[pad1(m)] = cmul(c.line()[pad1(m)], cconj(c.xtw[(c.r - 1) * M + m]));
  }
  cl_cross<Rl, M, +1, CS>(c, cl);
}

// sum over the cluster (every thread of every CTA gets the same value)
template <typename Rl, int CS>
__device__ __forceinline__ double cl_sum(ClCtx<Rl>& c, cg::cluster_group& cl, double v) {
  v = block_sum(v, c.red);
  if (threadIdx.x == 0) c.slot[0] = v;
  cl.sync();
  double s = 0.0;
#pragma unroll
  for (int q = 0; q < CS; ++q) s += *cl.map_shared_rank(&c.slot[0], q);
  cl.sync();
  return s;
}

template <typename Rl, int CS>
__device__ __forceinline__ double cl_max(ClCtx<Rl>& c, cg::cluster_group& cl, double v) {
  v = warp_max(v);
  if ((threadIdx.x & 31) == 0) c.red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double mx = 0.0;
    for (int w = 0; w < T1 / 32; ++w) mx = fmax(mx, c.red[w]);
    c.slot[1] = mx;
  }
  cl.sync();
  double mx = 0.0;
#pragma unroll
  for (int q = 0; q < CS; ++q) mx = fmax(mx, *cl.map_shared_rank(&c.slot[1], q));
  cl.sync();
  return mx;
}

// Plasma term P(t) = (loss + defocus)(t) a(t) of this CTA's block into the shared
// line from the time-domain field in GA (media_physics.py:156-203 with I =
// |A|^2 / A_eff).  The density at the block start comes from composing the
// preceding CTAs' affine maps; when a clamp binds anywhere the exact serial
// update runs CTA by CTA.  Returns false on every CTA when the whole line has
// W_ion = 0 and no avalanche.
template <typename Rl, int M, int CS>
__device__ bool cl_plasma(ClCtx<Rl>& c, cg::cluster_group& cl, double* ion_out) {
  using C = typename CT<Rl>::T;
  constexpr int CH = Cfg1<M>::CH, NA = Cfg1<M>::NA;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const PlasmaConst& m = c.in->pc;
  const double Aeff = c.in->A_eff;
  const AffineStep aff(m);
  for (int t = tid; t < M; t += T1) c.line()[pad1(t)] = c.GA[t];
  __syncthreads();
  bool any_w = false, ok = (m.ava == 0.0);
  double cm = 1.0, dm = 0.0;
  if (tid < NA) {
    for (int t = tid * CH; t < tid * CH + CH; ++t) {
      const C a = c.line()[pad1(t)];
      const Rl I = (Rl)(((double)a.x * a.x + (double)a.y * a.y) / Aeff);
      const double w = (double)(float)lut_eval<Rl>(c.lut, I);
      any_w |= (w != 0.0);
      const double cc = aff.e - w * aff.sf;
      ok &= (cc >= 0.0);
      dm = cc * dm + w * m.rho_nt * aff.sf;
      cm = cc * cm;
    }
  }
  // within the block: exclusive scan of the chunk maps (c1,d1) then (c2,d2) = (c1 c2, c2 d1 + d2)
  double cc = cm, dd = dm;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const double cp = __shfl_up_sync(0xffffffffu, cc, off);
    const double dp = __shfl_up_sync(0xffffffffu, dd, off);
    if (lane >= off) { dd = cc * dp + dd; cc = cc * cp; }
  }
  double* wc = c.starts;            // warp totals, then their exclusive prefixes
  double* wd = c.starts + T1 / 32;
  if (lane == 31) { wc[warp] = cc; wd[warp] = dd; }
  const bool blk_any = __syncthreads_or(any_w);
  const bool blk_ok = __syncthreads_and(ok);
  if (tid == 0) {
    double C0 = 1.0, D0 = 0.0;
    for (int w = 0; w < T1 / 32; ++w) {
      const double c2 = wc[w], d2 = wd[w];
      wc[w] = C0; wd[w] = D0;
      D0 = c2 * D0 + d2;
      C0 = C0 * c2;
    }
    c.slot[2] = C0;                 // the block's whole map
    c.slot[3] = D0;
    c.slot[4] = blk_any ? 1.0 : 0.0;
    c.slot[5] = blk_ok ? 1.0 : 0.0;
  }
  cl.sync();
  bool all_any = m.ava != 0.0, all_ok = true;
  double rho_in = 0.0;
#pragma unroll
  for (int q = 0; q < CS; ++q) {
    const double* sq = cl.map_shared_rank(c.slot, q);
    all_any |= sq[4] != 0.0;
    all_ok &= sq[5] != 0.0;
    if (q < c.r) rho_in = sq[2] * rho_in + sq[3];
  }
  cl.sync();
  if (!all_any) return false;
  double rho0 = 0.0;
  if (all_ok) {
    double ce = __shfl_up_sync(0xffffffffu, cc, 1);
    double de = __shfl_up_sync(0xffffffffu, dd, 1);
    if (lane == 0) { ce = 1.0; de = 0.0; }
    rho0 = ce * (wc[warp] * rho_in + wd[warp]) + de;
    __syncthreads();
  } else {
    // exact serial update: CTA q continues from CTA q-1's final density
    for (int q = 0; q < CS; ++q) {
      if (c.r == q && tid == 0) {
        double rho = q == 0 ? 0.0 : *cl.map_shared_rank(&c.slot[6], q - 1);
        for (int t = 0; t < M; ++t) {
          if (t % CH == 0) c.starts[t / CH] = rho;
          const C a = c.line()[pad1(t)];
          const double Id = ((double)a.x * a.x + (double)a.y * a.y) / Aeff;
          const double w = (double)(float)lut_eval<Rl>(c.lut, (Rl)Id);
          const double wa = (double)(float)(m.ava * (double)(Rl)Id);
          rho_step(rho, w, wa, m);
        }
        c.slot[6] = rho;
      }
      cl.sync();
    }
    rho0 = tid < NA ? c.starts[tid] : 0.0;
    __syncthreads();
  }
  const bool no_ava = (m.ava == 0.0);
  double ion = 0.0;
  if (tid < NA) {
    double rho = rho0;
    for (int t = tid * CH; t < tid * CH + CH; ++t) {
      const C a = c.line()[pad1(t)];
      const double Id = ((double)a.x * a.x + (double)a.y * a.y) / Aeff;
      const Rl I = (Rl)Id;
      const double w = (double)(float)lut_eval<Rl>(c.lut, I);
      const double wa = (double)(float)(m.ava * (double)I);
      const double rho_t = rho;
      ion = fmax(ion, rho_t);
      const double gen = no_ava ? rho_step0(rho, w, m, aff) : rho_step(rho, w, wa, m);
      const double loss = -(gen * m.Ui) / (2.0 * (double)I + 1e-30);
      const double cr = loss - m.sigma_half * rho_t;
      const double ci = -m.sigma_half * m.w0tc * rho_t;
      c.line()[pad1(t)] = C{(Rl)(cr * a.x - ci * a.y), (Rl)(cr * a.y + ci * a.x)};
    }
  }
  const double mx = cl_max<Rl, CS>(c, cl, ion / m.rho_nt);
  if (ion_out) *ion_out = fmax(*ion_out, mx);
  return true;
}

// N(u) for this CTA's bins (erk43ip_method.py:197-255 plus the plasma term),
// the stage input u formed on the fly; returns sum |u|^2 over the line for IN_5.
template <typename Rl, int M, int CS>
__device__ __noinline__ double cl_nl_eval(ClCtx<Rl>& c, cg::cluster_group& cl, int mode, double h,
                                          typename CT<Rl>::T* out, double* ion_out = nullptr) {
  using C = typename CT<Rl>::T;
  constexpr int N = CS * M;
  const int tid = threadIdx.x;
  const Rl hR = (Rl)h, h2 = (Rl)(h / 2), h6 = (Rl)(h / 6);
  double nrm = 0.0;
  if (mode == IN_A) {
    for (int w = tid; w < M; w += T1) c.line()[pad1(w)] = c.A[w];
  } else if (mode == IN_5) {
    for (int w = tid; w < M; w += T1) {
      const C u = cadd(c.T[w], cscale(c.A4P[w], h6));
      c.A4[w] = u;
      nrm += (double)u.x * u.x + (double)u.y * u.y;
      c.line()[pad1(w)] = u;
    }
  } else {
    const C* X = mode == IN_2 ? c.K1 : c.O;
    for (int w = tid; w < M; w += T1) {
      const C E = EFac<Rl>::get(c.D[w], 0.5 * h);
      const C v = cmul(c.A[w], E);
      const C xx = X[w];
      C u;
      if (mode == IN_2) {
        const C a1 = cmul(xx, E);
        c.T[w] = a1;
        u = cadd(v, cscale(a1, h2));
      } else if (mode == IN_3) {
        c.T[w] = cadd(c.T[w], cscale(xx, (Rl)2));
        u = cadd(v, cscale(xx, h2));
      } else {   // IN_4
        const C ts = cadd(c.T[w], cscale(xx, (Rl)2));
        c.T[w] = cmul(cadd(v, cscale(ts, h6)), E);    // beta
        u = cmul(cadd(v, cscale(xx, hR)), E);
      }
      c.line()[pad1(w)] = u;
    }
  }
  __syncthreads();
  cl_fft_inv<Rl, M, CS>(c, cl);
  const Rl invN = (Rl)(1.0 / N);
  const bool plasma = c.in->plasma;
  for (int t = tid; t < M; t += T1) {
    const C a = cscale(c.line()[pad1(t)], invN);
    if (plasma) c.GA[t] = a;
    const Rl I = a.x * a.x + a.y * a.y;
    c.line()[pad1(t)] = cscale(a, I);
  }
  __syncthreads();
  cl_fft_fwd<Rl, M, CS>(c, cl);
  for (int w = tid; w < M; w += T1) {
    const C p = c.line()[pad1(w)];
    const Rl gr = (Rl)c.G[w];
    out[w] = C{-gr * p.y, gr * p.x};     // i gamma U(w) P_NL(w)
  }
  __syncthreads();
  if (plasma && cl_plasma<Rl, M, CS>(c, cl, ion_out)) {
    __syncthreads();
    cl_fft_fwd<Rl, M, CS>(c, cl);
    for (int w = tid; w < M; w += T1) out[w] = cadd(out[w], c.line()[pad1(w)]);
    __syncthreads();
  }
  return mode == IN_5 ? cl_sum<Rl, CS>(c, cl, nrm) : 0.0;
}

// one erk43_step from (A, K1); the error of erk43ip_method.py:279-284
template <typename Rl, int M, int CS>
__device__ __noinline__ double cl_attempt(ClCtx<Rl>& c, cg::cluster_group& cl, double h, double* ion_cand) {
  using C = typename CT<Rl>::T;
  constexpr int N = CS * M;
  const int tid = threadIdx.x;
  cl_nl_eval<Rl, M, CS>(c, cl, IN_2, h, c.O);
  cl_nl_eval<Rl, M, CS>(c, cl, IN_3, h, c.O);
  cl_nl_eval<Rl, M, CS>(c, cl, IN_4, h, c.A4P);
  const double nrm = cl_nl_eval<Rl, M, CS>(c, cl, IN_5, h, c.O, ion_cand);
  double acc = 0.0;
  const Rl h30 = (Rl)(h / 30);
  for (int w = tid; w < M; w += T1) {
    const C a4 = c.A4P[w], a5 = c.O[w];
    if (sizeof(Rl) == 8) {
      const C A3 = cadd(c.T[w], cscale(cadd(cscale(a4, (Rl)2), cscale(a5, (Rl)3)), h30));
      const C d = csub(c.A4[w], A3);
      acc += (double)d.x * d.x + (double)d.y * d.y;
    } else {
      const double dx = (double)a4.x - a5.x, dy = (double)a4.y - a5.y;
      acc += dx * dx + dy * dy;
    }
  }
  double num = cl_sum<Rl, CS>(c, cl, acc);
  if (sizeof(Rl) != 8) num *= (h / 10.0) * (h / 10.0);
  double normA = sqrt(nrm / N);
  if (normA < 1e-20) normA = 1.0;
  return sqrt(num / N) / normA;
}

// The whole propagation of instance i by this cluster (erk43ip_method.py:288-369).
template <typename Rl, int M, int CS>
__device__ void cl_run_instance(const Batch1D& b, int i, unsigned char* smem, cg::cluster_group& cl) {
  using C = typename CT<Rl>::T;
  constexpr int N = CS * M;
  const int tid = threadIdx.x;
  const Inst1D& in = b.inst[i];
  ClCtx<Rl> c;
  c.r = (int)cl.block_rank();
  c.cur = 0;
  c.pad = Cfg1<M>::PAD;
  c.red = reinterpret_cast<double*>(reinterpret_cast<C*>(smem) + 2 * Cfg1<M>::PAD);
  c.starts = c.red + 64;
  c.slot = c.starts + T1;
  c.tw = reinterpret_cast<const C*>(b.tw) + (M - 1);
  c.xtw = reinterpret_cast<const C*>(b.xtw) + cl_xtw_offset(M, CS);
  // per-cluster scratch: 7 stage arrays of N (CTA r's slice at r M), then D and G copies
  const long long cid = b.cl_off + blockIdx.x / CS;
  unsigned char* base = reinterpret_cast<unsigned char*>(b.cl_scratch) + cid * b.cl_scratch_bytes;
  C* sc = reinterpret_cast<C*>(base) + (long long)c.r * M;
  c.A = sc; c.K1 = sc + N; c.T = sc + 2 * N; c.O = sc + 3 * N;
  c.A4 = sc + 4 * N; c.A4P = sc + 5 * N; c.GA = sc + 6 * N;
  double2* Dp = reinterpret_cast<double2*>(reinterpret_cast<C*>(base) + 7LL * N) + (long long)c.r * M;
  double* Gp = reinterpret_cast<double*>(reinterpret_cast<double2*>(reinterpret_cast<C*>(base) + 7LL * N) + N) +
               (long long)c.r * M;
  for (int j = tid; j < M; j += T1) {
    const long long k = in.off + c.r + (long long)CS * j;
    Dp[j] = b.D[k];
    Gp[j] = b.G[k];
  }
  c.D = Dp;
  c.G = Gp;
  c.in = &in;
  c.lut = b.lut;
  C* field = reinterpret_cast<C*>(b.field) + in.off + (long long)c.r * M;
  for (int t = tid; t < M; t += T1) c.line()[pad1(t)] = field[t];
  __syncthreads();
  cl_fft_fwd<Rl, M, CS>(c, cl);
  for (int w = tid; w < M; w += T1) c.A[w] = c.line()[pad1(w)];
  __syncthreads();
  double ion_peak = 0.0, ion_cand = 0.0;
  cl_nl_eval<Rl, M, CS>(c, cl, IN_A, 0.0, c.K1, &ion_peak);

  // the adaptive loop of run_instance (every CTA takes the same decisions)
  const double L = in.L, tol = in.tol, max_step = in.max_step, min_step = in.min_step;
  double z = 0.0, h = max_step / 100, err = 0.0, err_prev = -1.0;
  long long attempts = 0, accepted = 0;
  int status = 0;
  const bool lead = c.r == 0 && tid == 0;
  auto accept = [&](double hh) {
    z += hh;
    ion_peak = fmax(ion_peak, ion_cand);
    C* t0 = c.A; c.A = c.A4; c.A4 = t0;
    C* t1 = c.K1; c.K1 = c.O; c.O = t1;
    if (b.hlog) {
      if (accepted < b.hlog_cap) { if (lead) b.hlog[(long long)i * b.hlog_cap + accepted] = hh; }
      else status |= 16;
    }
    accepted += 1;
  };
  if (b.hsched) {
    const double* hs = b.hsched + (long long)i * b.nsched;
    for (int k = 0; k < b.nsched; ++k) {
      const double hh = hs[k];
      ion_cand = 0.0;
      err = cl_attempt<Rl, M, CS>(c, cl, hh, &ion_cand);
      attempts += 1;
      if (!isfinite(err)) { status |= UPPE_STATUS_NONFINITE; break; }
      accept(hh);
    }
  }
  while (!b.hsched && z < L) {
    if (z + h > L) h = L - z;
    ion_cand = 0.0;
    err = cl_attempt<Rl, M, CS>(c, cl, h, &ion_cand);
    attempts += 1;
    if (!isfinite(h) || (!isfinite(err) && h <= min_step)) { status |= UPPE_STATUS_NONFINITE; break; }
    if (!isfinite(err)) {
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
        err = cl_attempt<Rl, M, CS>(c, cl, h, &ion_cand);
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
  // energy and photon number (Parseval in omega) over this CTA's bins, then the cluster
  double en = 0.0, ph = 0.0;
  {
    const double dw = 6.283185307179586476925286766559 / (N * in.dt);
    for (int w = tid; w < M; w += T1) {
      const int k = c.r + CS * w;
      const C v = c.A[w];
      const double a2 = (double)v.x * v.x + (double)v.y * v.y;
      en += a2;
      const double wa = in.omega0 + dw * (k < (N + 1) / 2 ? k : k - N);
      if (wa > 0.0) ph += a2 / (1.054571817e-34 * wa);
    }
    en = cl_sum<Rl, CS>(c, cl, en) * in.dt / N;
    ph = cl_sum<Rl, CS>(c, cl, ph) * in.dt / N;
  }
  for (int w = tid; w < M; w += T1) c.line()[pad1(w)] = c.A[w];
  __syncthreads();
  cl_fft_inv<Rl, M, CS>(c, cl);
  const Rl invN = (Rl)(1.0 / N);
  for (int t = tid; t < M; t += T1) field[t] = cscale(c.line()[pad1(t)], invN);
  if (lead) {
    Res1D rr;
    rr.z = z; rr.h = h; rr.err = err; rr.attempts = attempts; rr.accepted = accepted;
    rr.status = status; rr.hist_count = 0;
    rr.energy = en; rr.photons = in.omega0 > 0.0 ? ph : NAN; rr.peak_ion = ion_peak;
    b.res[i] = rr;
  }
  __syncthreads();
}

// Persistent cluster kernel: each cluster takes instances from the work queue
// (longest expected first) and propagates them one at a time.
template <typename Rl, int CS>
__global__ void __cluster_dims__(CS, 1, 1) __launch_bounds__(T1, 1) k_uppe1d_cl(Batch1D b) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ int s_k;
  cg::cluster_group cl = cg::this_cluster();
  mark_busy(b.busy, 0, b.busy_off);
  for (;;) {
    if (cl.block_rank() == 0 && threadIdx.x == 0) {
      if (CS == 8 && b.nhead > 0) {
        // the eight-CTA clusters of a mixed launch take the head of the queue (the
        // costliest lines) and nothing else, so every line's cluster size, hence
        // its result, is fixed by the plan
        const int k = atomicAdd(b.counter_head, 1);
        s_k = k < b.nhead ? k : b.ninst;
      } else {
        s_k = atomicAdd(b.counter, 1);
      }
    }
    cl.sync();
    const int k = *cl.map_shared_rank(&s_k, 0);
    cl.sync();
    if (k >= b.ninst) { mark_busy(b.busy, 1, b.busy_off); return; }
    const int i = b.order[k];
    switch (b.inst[i].log2n) {
      case 11: cl_run_instance<Rl, 2048 / CS, CS>(b, i, smem, cl); break;
      case 12: cl_run_instance<Rl, 4096 / CS, CS>(b, i, smem, cl); break;
      case 13: cl_run_instance<Rl, 8192 / CS, CS>(b, i, smem, cl); break;
      case 14: cl_run_instance<Rl, 16384 / CS, CS>(b, i, smem, cl); break;
      default: break;
    }
  }
}

// shared memory of the cluster kernel for lines up to nmax points
template <typename Rl> inline size_t cl_smem(int nmax, int cs = kCS) {
  const int M = nmax / cs;
  return 2 * sizeof(typename CT<Rl>::T) * (size_t)(M + M / 32) + sizeof(double) * (64 + T1 + 8);
}
// per-cluster scratch bytes for lines up to nmax points
template <typename Rl> inline size_t cl_scratch_bytes(int nmax) {
  const size_t b = 7 * sizeof(typename CT<Rl>::T) * (size_t)nmax + 24 * (size_t)nmax;
  return (b + 255) & ~(size_t)255;
}

template <typename Rl> cudaError_t launch_uppe1d_cl(const Batch1D& b, int nclusters, size_t smem, cudaStream_t s,
                                                   int cs);
template <typename Rl> int uppe1d_cl_max_clusters(size_t smem, int cs);

}  // namespace uppe
