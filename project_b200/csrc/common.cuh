// Shared device helpers for the ERK4(3)-IP UPPE kernels (sm_100a).
//
// * complex arithmetic on float2 / double2,
// * radix-2/4/8/16 DFTs held in registers,
// * an in-place Stockham (self-sorting) FFT over signals resident in shared
//   memory, driven by a compile-time pass list.  All threads of a "team" (a warp
//   or a block) own E elements each; pass p reads its R inputs per butterfly into
//   registers, synchronises the team, writes the R outputs in Stockham order and
//   synchronises again, so no second buffer is needed.
//
// Conventions follow numpy/scipy: forward X_k = sum_n x_n exp(-2 pi i k n / N),
// inverse without the 1/N factor (callers fold it into a power-of-two scale).
#pragma once
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>
#include <stdint.h>

namespace uppe {

// NVTX range over a library call (host side; popped on every return path), so a
// profiler timeline shows propagate / adjoint / program calls by name
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

template <typename R> struct CT;
template <> struct CT<float>  { using T = float2; };
template <> struct CT<double> { using T = double2; };

template <typename C> __device__ __forceinline__ C cadd(C a, C b) { return {a.x + b.x, a.y + b.y}; }
template <typename C> __device__ __forceinline__ C csub(C a, C b) { return {a.x - b.x, a.y - b.y}; }
template <typename C> __device__ __forceinline__ C cmul(C a, C b) {
  return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}
template <typename C, typename R> __device__ __forceinline__ C cscale(C a, R s) { return {a.x * s, a.y * s}; }
template <typename C> __device__ __forceinline__ C cconj(C a) { return {a.x, -a.y}; }
// multiply by i (DIR=+1) or -i (DIR=-1)
template <int DIR, typename C> __device__ __forceinline__ C mul_pmi(C a) {
  return DIR > 0 ? C{-a.y, a.x} : C{a.y, -a.x};
}
template <typename C> __device__ __forceinline__ C czero() { return {0, 0}; }

// exp(DIR * 2 pi i k / R) as compile-time constants for R dividing 32: the angle
// index on the 32-grid is exact for every such R (cos and sin of 2 pi i / 32 for
// i = 0..8; the values of the 16-grid are the even entries)
template <int R, int K> struct Twid {
  static_assert(R > 0 && 32 % R == 0, "compile-time twiddles cover R | 32");
  static constexpr int k32 = (K * (32 / R)) % 32;   // angle index on the 32-grid
  __host__ __device__ static constexpr double c32(int i) {   // cos(2 pi i / 32), 0 <= i <= 8
    return i == 0 ? 1.0 : i == 1 ? 0.98078528040323044913 : i == 2 ? 0.92387953251128675613
         : i == 3 ? 0.83146961230254523708 : i == 4 ? 0.70710678118654752440 : i == 5 ? 0.55557023301960222474
         : i == 6 ? 0.38268343236508977173 : i == 7 ? 0.19509032201612826785 : 0.0;
  }
  // first half turn: i in [0, 16); cos = c32(i) on [0, 8], -c32(16 - i) above
  __host__ __device__ static constexpr double kc(int i) { return i <= 8 ? c32(i) : -c32(16 - i); }
  __host__ __device__ static constexpr double ks(int i) { return i <= 8 ? c32(8 - i) : c32(i - 8); }
  static constexpr double cv = k32 < 16 ? kc(k32) : -kc(k32 - 16);
  static constexpr double sv = k32 < 16 ? ks(k32) : -ks(k32 - 16);
};

// x * exp(DIR * 2 pi i K / R)
template <int R, int K, int DIR, typename C> __device__ __forceinline__ C rot(C x) {
  using Rl = decltype(x.x);
  constexpr int k = K % R;
  if constexpr (k == 0) {
    return x;
  } else if constexpr (4 * k == R) {
    return mul_pmi<DIR>(x);
  } else if constexpr (2 * k == R) {
    return C{-x.x, -x.y};
  } else if constexpr (4 * k == 3 * R) {
    return mul_pmi<-DIR>(x);
  } else {
    constexpr double cd = Twid<R, k>::cv, sd = DIR * Twid<R, k>::sv;
    const Rl c = (Rl)cd;
    const Rl s = (Rl)sd;
    return C{x.x * c - x.y * s, x.x * s + x.y * c};
  }
}

// In-register DFT of size R (R in {1,2,4,8,16,32}); DIR=-1 forward, +1 inverse.
template <int R, int DIR, typename C> struct DFT {
  __device__ __forceinline__ static void run(C* v) {
    C e[R / 2], o[R / 2];
#pragma unroll
    for (int i = 0; i < R / 2; ++i) { e[i] = v[2 * i]; o[i] = v[2 * i + 1]; }
    DFT<R / 2, DIR, C>::run(e);
    DFT<R / 2, DIR, C>::run(o);
    combine<0>(v, e, o);
  }
  template <int K> __device__ __forceinline__ static void combine(C* v, const C* e, const C* o) {
    if constexpr (K < R / 2) {
      C t = rot<R, K, DIR>(o[K]);
      v[K] = cadd(e[K], t);
      v[K + R / 2] = csub(e[K], t);
      combine<K + 1>(v, e, o);
    }
  }
};
template <int DIR, typename C> struct DFT<1, DIR, C> {
  __device__ __forceinline__ static void run(C*) {}
};
template <int DIR, typename C> struct DFT<2, DIR, C> {
  __device__ __forceinline__ static void run(C* v) {
    C a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  }
};
template <int DIR, typename C> struct DFT<4, DIR, C> {
  __device__ __forceinline__ static void run(C* v) {
    C t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]);
    C t2 = cadd(v[1], v[3]), t3 = mul_pmi<DIR>(csub(v[1], v[3]));
    v[0] = cadd(t0, t2);
    v[2] = csub(t0, t2);
    v[1] = cadd(t1, t3);
    v[3] = csub(t1, t3);
  }
};

// Largest radix in {16,8,4,2} dividing both the remaining length and E.
template <int REM, int E> struct PickRadix {
  static constexpr int v = (REM % 16 == 0 && E % 16 == 0) ? 16
                         : (REM % 8 == 0 && E % 8 == 0)   ? 8
                         : (REM % 4 == 0 && E % 4 == 0)   ? 4
                                                           : 2;
};

// Stockham passes over NSIG signals of length N in shared memory.
//   IDX(sig, n) -> shared-memory element index.
//   tw[m] = exp(-2 pi i m / N) (forward table, conjugated for DIR=+1).
//   Team of NTHR threads, thread id `tid`; E = N*NSIG/NTHR elements per thread.
//   Butterfly b of thread tid: bf = tid + b*NTHR; sig = bf % NSIG; j = bf / NSIG.
template <int N, int NSIG, int NTHR, int DIR, int Ns, typename C, typename IDX, typename SYNC>
__device__ __forceinline__ void stockham(C* s, const C* tw, int tid, IDX idx, SYNC sync) {
  if constexpr (Ns < N) {
    constexpr int E = N * NSIG / NTHR;
    static_assert(E >= 2, "need at least two elements per thread");
    constexpr int R = PickRadix<N / Ns, E>::v;
    constexpr int B = E / R;
    constexpr int M = N / R;   // butterflies per signal
    C v[B][R];
    // threads with tid >= NTHR (a team padded to a full warp/block) only synchronise
    const bool act = tid < NTHR;
    if (act) {
#pragma unroll
    for (int b = 0; b < B; ++b) {
      const int bf = tid + b * NTHR;
      const int sig = bf % NSIG, j = bf / NSIG;
      const int k = j & (Ns - 1);
#pragma unroll
      for (int r = 0; r < R; ++r) v[b][r] = s[idx(sig, j + r * M)];
      if constexpr (Ns > 1) {
#pragma unroll
        for (int r = 1; r < R; ++r) {
          C w = tw[(r * k) * (N / (Ns * R))];
          if (DIR > 0) w.y = -w.y;
          v[b][r] = cmul(v[b][r], w);
        }
      }
      DFT<R, DIR, C>::run(v[b]);
    }
    }
    sync();
    if (act) {
#pragma unroll
    for (int b = 0; b < B; ++b) {
      const int bf = tid + b * NTHR;
      const int sig = bf % NSIG, j = bf / NSIG;
      const int k = j & (Ns - 1);
      const int base = (j / Ns) * Ns * R + k;
#pragma unroll
      for (int r = 0; r < R; ++r) s[idx(sig, base + r * Ns)] = v[b][r];
    }
    }
    sync();
    stockham<N, NSIG, NTHR, DIR, Ns * R, C>(s, tw, tid, idx, sync);
  }
}

// exp(i ph) in FP32 from an FP64 phase: ph = q pi/2 + f with q = rint(2 ph / pi)
// and |f| <= pi/4 formed in FP64, f rounded to FP32 (absolute error <= 2^-25 rad
// there, against ~1.2e-7 for an argument near pi), sincosf of f, then the exact
// rotation by i^q.  The mixed-precision interaction-picture factors use it.
__device__ __forceinline__ float2 cis_quadrant(double ph) {
  const double q = rint(ph * 0.63661977236758134308);
  const double f = fma(-q, 1.5707963267948966192, ph);
  float s, c;
  sincosf((float)f, &s, &c);
  switch ((int)((long long)q & 3)) {
    case 0: return make_float2(c, s);
    case 1: return make_float2(-s, c);
    case 2: return make_float2(-c, -s);
    default: return make_float2(s, -c);
  }
}

// Non-negative double -> order-preserving 64-bit key for atomicMax (NaN > +inf).
__device__ __forceinline__ unsigned long long dkey(double v) {
  return (unsigned long long)__double_as_longlong(v);
}
__device__ __forceinline__ void atomic_max_nonneg(unsigned long long* dst, double v) {
  atomicMax(dst, dkey(v));
}

// max over the first WIDTH lanes of a warp (WIDTH = 32, or the whole block when
// it is smaller than a warp); only those lanes may call it.
template <int WIDTH = 32, typename R> __device__ __forceinline__ R warp_max(R v) {
  constexpr unsigned mask = WIDTH >= 32 ? 0xffffffffu : ((1u << WIDTH) - 1u);
#pragma unroll
  for (int o = (WIDTH >= 32 ? 16 : WIDTH / 2); o > 0; o >>= 1) {
    R u = __shfl_xor_sync(mask, v, o);
    v = (u > v || u != u) ? u : v;    // NaN propagates
  }
  return v;
}

// ---------------------------------------------------------------------------
// Ionisation LUT (media_physics.py:131-137): clip log10(I + 1e-30) to the grid,
// then numpy.interp semantics (j with xp[j] <= x < xp[j+1]; slope evaluated in
// FP64 as numpy does).
// ---------------------------------------------------------------------------
struct Lut {
  const void* x;    // grid, field precision
  const void* w;    // rates, field precision
  const double* slope;   // (w[j+1] - w[j]) / (x[j+1] - x[j]) in FP64 from the field-precision
                         // values, j < n - 1 (or null: computed per evaluation)
  int n;
  double x0, inv_dx;
  double zero_x;    // W is exactly 0 for clipped log10(I) <= zero_x (-inf if none)
  double I_zero;    // W is exactly 0 for I < I_zero (no log10 needed)
};

// 10^(zero_x - 1e-3): the 1e-3 margin in log10 exceeds the rounding of log10 /
// log10f at these magnitudes by orders, so I < I_zero implies clipped log10(I)
// <= zero_x and lut_eval returns exactly 0.
static inline double lut_zero_intensity(double zero_x) {
  if (zero_x == -INFINITY) return 0.0;
  if (zero_x == INFINITY) return INFINITY;
  return pow(10.0, zero_x - 1e-3);
}

template <typename Rl>
__device__ __forceinline__ Rl lut_eval(const Lut& L, Rl I) {
  const Rl* xp = reinterpret_cast<const Rl*>(L.x);
  const Rl* fp = reinterpret_cast<const Rl*>(L.w);
  const int n = L.n;
  if ((double)I < L.I_zero) return (Rl)0;
  Rl x = (sizeof(Rl) == 8) ? (Rl)log10((double)I + 1e-30) : (Rl)log10f((float)I + 1e-30f);
  const Rl x0 = __ldg(xp), x1 = __ldg(xp + n - 1);
  x = x < x0 ? x0 : (x > x1 ? x1 : x);
  // below the last leading zero of the table the interpolant is exactly 0
  if ((double)x <= L.zero_x) return (Rl)0;
  int j = (int)floor(((double)x - L.x0) * L.inv_dx);
  j = j < 0 ? 0 : (j > n - 1 ? n - 1 : j);
  while (j < n - 1 && __ldg(xp + j + 1) <= x) ++j;
  while (j > 0 && __ldg(xp + j) > x) --j;
  if (j >= n - 1) return __ldg(fp + n - 1);
  const Rl xj = __ldg(xp + j);
  if (xj == x) return __ldg(fp + j);
  const double slope = L.slope ? __ldg(L.slope + j)
                               : ((double)__ldg(fp + j + 1) - (double)__ldg(fp + j)) /
                                     ((double)__ldg(xp + j + 1) - (double)xj);
  return (Rl)(slope * ((double)x - (double)xj) + (double)__ldg(fp + j));
}

// the slope table of lut_eval: the same FP64 quotients, formed once on the host
// (IEEE division rounds identically there), from the table in the field precision
template <typename Rl>
static inline void lut_slopes(const double* x, const double* w, int n, double* out) {
  for (int j = 0; j + 1 < n; ++j)
    out[j] = ((double)(Rl)w[j + 1] - (double)(Rl)w[j]) / ((double)(Rl)x[j + 1] - (double)(Rl)x[j]);
}

// Plasma constants shared by the 1D and 3D nonlinear kernels.
struct PlasmaConst {
  double Ui;          // ionisation energy [J]
  double sigma_half;  // sigma_drude / 2
  double w0tc;        // omega0 * tau_c
  double rr, dt, rho_nt;   // float32-rounded, as the reference passes them (:185-187)
  double ava;         // W_ava = ava * I
};

// One step of the reference density update (media_physics.py:36-64): returns
// gen[t] and advances rho.
__device__ __forceinline__ double rho_step(double& rho, double w_pi, double w_av, const PlasmaConst& m) {
  double depl = (m.rho_nt - rho) / m.rho_nt;
  if (depl < 0.0) depl = 0.0;
  const double gen = (w_pi * m.rho_nt + w_av * rho) * depl;
  const double S = w_pi * m.rho_nt * depl;
  const double G = w_av * depl - m.rr;
  double gdt = G * m.dt;
  if (gdt > 10.0) gdt = 10.0;
  if (gdt < -10.0) gdt = -10.0;
  const double eg = exp(gdt);
  const double sf = (fabs(gdt) < 1e-5) ? m.dt * (1.0 + 0.5 * gdt) : (eg - 1.0) / G;
  double r = rho * eg + S * sf;
  if (r > m.rho_nt) r = m.rho_nt;
  if (r < 0.0) r = 0.0;
  rho = r;
  return gen;
}

// Affine form of the update while no clamp binds (w_av = 0):
// rho' = rho (e - w sf) + w rho_nt sf with e = exp(gdt0), gdt0 = clamp(-rr dt).
struct AffineStep {
  double e, sf;
  __device__ __forceinline__ explicit AffineStep(const PlasmaConst& m) {
    const double gdt0 = fmin(fmax(-m.rr * m.dt, -10.0), 10.0);
    e = exp(gdt0);
    sf = (fabs(gdt0) < 1e-5) ? m.dt * (1.0 + 0.5 * gdt0) : (e - 1.0) / (-m.rr);
  }
};

// rho_step for w_av = 0 with the update's constants taken from AffineStep (the
// same values: G = 0 * depl - rr = -rr exactly, so gdt, exp(gdt) and sf are
// AffineStep's e and sf): no exp per sample.
__device__ __forceinline__ double rho_step0(double& rho, double w_pi, const PlasmaConst& m,
                                            const AffineStep& aff) {
  double depl = (m.rho_nt - rho) / m.rho_nt;
  if (depl < 0.0) depl = 0.0;
  const double gen = w_pi * m.rho_nt * depl;
  double r = rho * aff.e + gen * aff.sf;
  if (r > m.rho_nt) r = m.rho_nt;
  if (r < 0.0) r = 0.0;
  rho = r;
  return gen;
}

// ---------------------------------------------------------------------------
// Reverse mode of the plasma term P(a) = c a (media_physics.py:165-203),
//   c = -Ui gen / (2 I + 1e-30) - (sigma/2)(1 + i omega0 tau_c) rho,
// with I = alpha |a|^2, W = lut(I), and the density update of rho_step for
// w_av = 0.  Cotangent convention: dL = Re sum conj(xb) dx.
// ---------------------------------------------------------------------------

// dW/dI of lut_eval: the slope of the bracketing interval over (I + 1e-30) ln 10;
// 0 where log10(I) is clipped to the table ends or below the table's zero run.
template <typename Rl>
__device__ __forceinline__ double lut_slope(const Lut& L, Rl I) {
  const Rl* xp = reinterpret_cast<const Rl*>(L.x);
  const Rl* fp = reinterpret_cast<const Rl*>(L.w);
  const int n = L.n;
  if ((double)I < L.I_zero) return 0.0;
  const Rl x = (sizeof(Rl) == 8) ? (Rl)log10((double)I + 1e-30) : (Rl)log10f((float)I + 1e-30f);
  const Rl x0 = __ldg(xp), x1 = __ldg(xp + n - 1);
  if (!(x > x0) || !(x < x1)) return 0.0;
  if ((double)x <= L.zero_x) return 0.0;
  int j = (int)floor(((double)x - L.x0) * L.inv_dx);
  j = j < 0 ? 0 : (j > n - 1 ? n - 1 : j);
  while (j < n - 1 && __ldg(xp + j + 1) <= x) ++j;
  while (j > 0 && __ldg(xp + j) > x) --j;
  if (j >= n - 1) return 0.0;
  const double slope = ((double)__ldg(fp + j + 1) - (double)__ldg(fp + j)) /
                       ((double)__ldg(xp + j + 1) - (double)__ldg(xp + j));
  return slope / (((double)I + 1e-30) * 2.302585092994046);
}

// One sample.  cur = density before the update, W / dW = rate and slope at I,
// (ar, ai) = field sample, (qr, qi) = cotangent of the term's sample.  Gives the
// reverse recurrence lam_t = A lam_{t+1} + B for lam = cotangent of the density.
// With OUT, lam_next = lam_{t+1} gives the field cotangent (oar, oai) and adds
// d/d(rho_nt, sigma_drude, omega0 tau_c) into g (when g is not null).
template <bool OUT>
__device__ __forceinline__ void plasma_rev(const PlasmaConst& m, const AffineStep& aff, double alpha,
                                           double cur, double W, double dW, double I, double ar,
                                           double ai, double qr, double qi, double& A, double& B,
                                           double lam_next = 0.0, double* oar = nullptr,
                                           double* oai = nullptr, double* g = nullptr) {
  const double den = 2.0 * I + 1e-30;
  const double kr = m.sigma_half, ki = m.sigma_half * m.w0tc;
  double depl = (m.rho_nt - cur) / m.rho_nt;
  const bool dpos = depl >= 0.0;
  if (!dpos) depl = 0.0;
  const double gen = W * m.rho_nt * depl;
  const double r = cur * aff.e + gen * aff.sf;
  const bool hi = r > m.rho_nt, lo = r < 0.0;
  const double sr = qr * ar + qi * ai, si = qr * ai - qi * ar;   // s = conj(q) a
  const double genb = -m.Ui / den * sr;
  const double rhob = -(kr * sr - ki * si);
  const double gw = dpos ? W : 0.0;                               // d gen / d rho_nt
  A = (hi || lo) ? 0.0 : (aff.e - gw * aff.sf);
  B = rhob - genb * gw;
  if constexpr (OUT) {
    const double lam_eff = (hi || lo) ? 0.0 : lam_next;
    const double Wb = dpos ? (genb + lam_eff * aff.sf) * (m.rho_nt * depl) : 0.0;
    const double Ib = 2.0 * m.Ui * gen / (den * den) * sr + Wb * dW;
    const double cr = -m.Ui * gen / den - kr * cur, ci = -ki * cur;
    *oar = cr * qr + ci * qi + 2.0 * alpha * Ib * ar;             // conj(c) q + 2 alpha Ib a
    *oai = cr * qi - ci * qr + 2.0 * alpha * Ib * ai;
    if (g) {
      g[0] += genb * gw + (hi ? lam_next : (lo ? 0.0 : lam_next * gw * aff.sf));
      const double gkr = -cur * sr, gki = cur * si;                // d/d kr, d/d ki
      g[1] += 0.5 * gkr + 0.5 * m.w0tc * gki;                      // kr = sigma/2, ki = sigma w0tc/2
      g[2] += m.sigma_half * gki;
    }
  }
}

}  // namespace uppe
