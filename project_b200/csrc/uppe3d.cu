// 3+1D envelope ERK4(3)-IP UPPE propagator, sm_100a.
//
// Replaces ERK43IP_UPPE_3D_Optimized (src/3+1D-UPPE-ERK4(3)IP-envelope/solver_3d.py)
// and the envelope medium's nonlinear response + plasma kernel
// (src/3+1D-UPPE-ERK4(3)IP-envelope/media_physics.py:11-67, 156-205).
//
// Field layout in HBM: [Nx][Ny][Nt], t (or omega) contiguous, complex64 or
// complex128.  The accepted state is kept in the (x, y, omega) domain
// ("Z" = fft_t of the reference's time-domain field), so the reference's
// per-attempt output transform ifft_t(ifft2(A4) * filter) * exp(-damp h) and the
// next attempt's fft2(fft_t(.)) collapse into one x-pass that writes
// ifft2(A4) * filter * absorber.  One ERK attempt is a fixed sequence of passes:
//
//   T   : t-lines      -- ifft_t, Kerr + steepening, ADK LUT, rho scan, plasma,
//                         fft_t (x2), shock/mask combine              (k_tpass)
//   X   : x-columns    -- fft / ifft along x                           (k_space)
//   Y   : y-columns    -- fft_y, ERK stage algebra with the interaction-
//                         picture factor exp(h/2 D) computed on the fly in
//                         FP64, ifft_y of the next stage input          (k_space)
//
// Eval 1 (only after an accepted step):  T(Z) X(NL,Z) Ymid1
// Evals 2-4:                             Xinv T Xfwd Ymid{2,3,4}
// Eval 5:                                Xinv(+Z candidate) T Xfwd Yfwd5 (error)
// then an error kernel and (in propagate mode) the step-size controller, all
// on the device; every kernel reads the device state and exits early when the
// propagation is done, so the whole attempt is one reusable CUDA graph.
#include <cuda.h>            // CUtensorMap (encoded through the runtime's driver entry point)
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "common.cuh"
#include "../../include/uppe_b200.h"

namespace uppe {

// ---------------------------------------------------------------------------
// device state and tables
// ---------------------------------------------------------------------------
struct State3D {
  double z, h, L, tol, max_step, min_step;
  double err, err_num, err_den;
  double A_scale, inv_A_scale;
  unsigned long long red_norm, red_diff;
  unsigned long long ion_bits;   // running max of rho/rho_nt over step-start and final states
  double* hlog;                  // accepted step sizes (for the adjoint), or null
  long long hlog_cap;
  long long attempts, accepted, max_attempts;
  int fail_count, zidx, fresh, done, status, last_accept;
};

struct Medium3D : PlasmaConst {
  double gk;          // (omega0/c) n2          -> Kerr = i gk I A
  double g4;          // (omega0/c) n4          -> HOKE = i g4 I^2 A
  int plasma;         // 0: plasma terms off
};

struct Tables3D {
  const double* aw;      // k^2 - kref^2            [Nt]
  const double* ksq;     // k^2                     [Nt]
  const double* kref;    // k0 + k1 omega           [Nt]
  const unsigned char* valid;   // omega_abs > 0    [Nt]
  const double* shock;   // (omega+omega0)/omega0 or 1   [Nt]
  const double* filt;    // anti-alias filter        [Nt]
  const double* q;       // kx^2 + ky^2   [Nx*Ny]
  const double* damp;    // absorber damp(x, y)      [Nx*Ny]
  const void* twx;       // exp(-2 pi i m/Nx) in the field precision
  const void* twy;
  const void* twt;
  Lut lut;               // ionisation table (field precision)
};

enum SpaceMode { XINV = 0, XINV_Z, XFWD, XFWD_Z, YMID1, YMID1R, YMID2, YMID3, YMID4, YFWD5,
                 YPLAIN_INV, YPLAIN_FWD };

struct Bufs3D {
  void* z[2];     // accepted state / candidate (x, y, omega)
  void* acur;     // fft2(Z) of the accepted state (kx, ky, omega)
  void* k1;       // N(A) of the accepted state
  void* tsum;     // term_sum, then beta
  void* a4p;      // alpha4'
  void* tmp[3];   // pass temporaries
};

struct Geom {
  int Nx, Ny, Nt;
  long long npts;
};

// ---------------------------------------------------------------------------
// interaction-picture factor exp(h2 * D(kx, ky, omega)), D as in
// solver_3d.py:56-87:  D = i (k^2 - kref^2 - kperp^2) / (kz + kref),
// kz = sqrt(k^2 - kperp^2) (complex), masked where omega_abs <= 0.
// The complex division follows numpy's algorithm (Smith's method).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void ip_operator(const Tables3D& tb, int iw, double q, double& Dr,
                                            double& Di) {
  if (!tb.valid[iw]) { Dr = 0.0; Di = 0.0; return; }
  const double num = tb.aw[iw] - q;
  const double arg = tb.ksq[iw] - q;
  double dr, di;
  if (arg >= 0.0) { dr = sqrt(arg) + tb.kref[iw]; di = 0.0; }
  else { dr = tb.kref[iw]; di = sqrt(-arg); }
  double rr, ri;   // num / (dr + i di)
  if (fabs(dr) >= fabs(di)) {
    const double rat = di / dr;
    const double scl = 1.0 / (dr + di * rat);
    rr = num * scl;
    ri = (-num * rat) * scl;
  } else {
    const double rat = dr / di;
    const double scl = 1.0 / (di + dr * rat);
    rr = (num * rat) * scl;
    ri = (-num) * scl;
  }
  Dr = -ri;   // 1j * (rr + i ri)
  Di = rr;
}

// Per-omega constants of the operator, loaded once per thread (each thread of a
// y-pass tile owns one omega column).
struct OmegaCol {
  double aw, ksq, kref;
  bool valid;
  __device__ __forceinline__ OmegaCol(const Tables3D& tb, int iw)
      : aw(tb.aw[iw]), ksq(tb.ksq[iw]), kref(tb.kref[iw]), valid(tb.valid[iw] != 0) {}
};

template <typename Rl> struct IPFactor;
template <> struct IPFactor<double> {
  // complex128: the reference's formula (solver_3d.py:80-87) and numpy's exp
  __device__ __forceinline__ static double2 get(const Tables3D& tb, const OmegaCol&, int iw,
                                                double q, double h2) {
    double Dr, Di;
    ip_operator(tb, iw, q, Dr, Di);
    const double ar = h2 * Dr, ai = h2 * Di;
    double s, c;
    sincos(ai, &s, &c);
    const double m = exp(ar);
    return make_double2(m * c, m * s);
  }
};
template <> struct IPFactor<float> {
  // Mixed precision.  D = i (k_z - k_ref): the same operator as the reference's
  // i (k^2 - k_ref^2 - k_perp^2)/(k_z + k_ref); in FP64 the direct difference
  // loses ~1e-16 * k ~ 1e-9 rad/m, far below FP32 resolution of the field, and
  // needs no division.  k_z comes from an FP32 square root refined by one FP64
  // Newton step (error ~1e-8 1/m).  The phase h/2*Im(D) is formed in FP64 and
  // reduced mod 2 pi before it is rounded to FP32; __sincosf then works on
  // [-pi, pi] (absolute error ~4e-7).  The accurate sincosf cut the error of one
  // attempt at 256x256x512 only from 4.0e-7 to 2.9e-7 (the FP32 transforms
  // dominate) for 13 % more y-pass time, so the fast form is kept here.
  __device__ __forceinline__ static float2 get(const Tables3D&, const OmegaCol& oc, int,
                                               double q, double h2) {
    if (!oc.valid) return make_float2(1.f, 0.f);
    const double arg = oc.ksq - q;
    double ph;
    float m = 1.f;
    if (arg >= 0.0) {
      const float kf = sqrtf((float)arg);
      const double k0 = (double)kf;
      const double kz = fma(fma(-k0, k0, arg), (double)(0.5f / kf), k0);
      ph = h2 * (kz - oc.kref);
    } else {   // evanescent: k_z = i sqrt(-arg) -> D = -sqrt(-arg) - i k_ref
      m = expf((float)(-h2 * sqrt(-arg)));
      ph = -h2 * oc.kref;
    }
    const double twopi = 6.283185307179586476925286766559;
    ph = fma(-twopi, rint(ph * (1.0 / twopi)), ph);
    float s, c;
    __sincosf((float)ph, &s, &c);
    return make_float2(m * c, m * s);
  }
};

template <typename C> __device__ __forceinline__ C ldg_c(const C* p) { return __ldg(p); }

// ---------------------------------------------------------------------------
// spatial passes: tile = W omega-columns x N rows (x or y), N-point FFT per column
// ---------------------------------------------------------------------------
constexpr int kW = 16;   // omega columns per tile

template <int N> struct SpaceCfg {
  static constexpr int E = N < 16 ? N : 16;
  static constexpr int NTHR = kW * N / E;
};

struct SpaceArgs {
  State3D* st;
  Tables3D tb;
  Bufs3D b;
  Geom g;
  const void* in;     // primary input (pass temporaries)
  void* out;          // primary output
  int mode;
  void* save_u;       // y passes: also store the stage input u (kx, ky, omega) here
  double scale;       // plain y passes: output scale
};

template <typename C> struct TileIdx {
  __device__ __forceinline__ int operator()(int sig, int n) const { return n * kW + sig; }
};
template <int KW> struct TileIdxK {
  __device__ __forceinline__ int operator()(int sig, int n) const { return n * KW + sig; }
};
struct BlockSync {
  __device__ __forceinline__ void operator()() const { __syncthreads(); }
};

template <typename C, int N, int NTHR>
__device__ __forceinline__ void load_tile(C* s, const C* __restrict__ g, long long base,
                                          long long stride, int tid) {
  // 16-byte vectors: VPR vectors per row of kW complex; all of a thread's loads
  // are issued before its shared-memory stores
  constexpr int VPR = kW * (int)sizeof(C) / 16;
  constexpr int NV = N * VPR / NTHR;
  static_assert(N * VPR % NTHR == 0, "tile/threads mismatch");
  const float4* __restrict__ gv = reinterpret_cast<const float4*>(g);
  float4* sv = reinterpret_cast<float4*>(s);
  float4 r[NV];
#pragma unroll
  for (int k = 0; k < NV; ++k) {
    const int v = tid + k * NTHR;
    const int n = v / VPR, c = v % VPR;
    r[k] = __ldg(gv + (base + n * stride) * (long long)sizeof(C) / 16 + c);
  }
#pragma unroll
  for (int k = 0; k < NV; ++k) sv[tid + k * NTHR] = r[k];
}
template <typename C, int N, int NTHR, int KW = kW>
__device__ __forceinline__ void store_tile(const C* s, C* __restrict__ g, long long base,
                                           long long stride, int tid) {
  constexpr int VPR = KW * (int)sizeof(C) / 16;
  float4* __restrict__ gv = reinterpret_cast<float4*>(g);
  const float4* sv = reinterpret_cast<const float4*>(s);
#pragma unroll 4
  for (int v = tid; v < N * VPR; v += NTHR) {
    const int n = v / VPR, c = v % VPR;
    gv[(base + n * stride) * (long long)sizeof(C) / 16 + c] = sv[n * VPR + c];
  }
}

template <typename Rl, int N>
__global__ void __launch_bounds__(SpaceCfg<N>::NTHR, (sizeof(Rl) == 4 && N == 256) ? 2 : 1)
k_space(SpaceArgs a) {
  using C = typename CT<Rl>::T;
  constexpr int NTHR = SpaceCfg<N>::NTHR;
  constexpr int E = SpaceCfg<N>::E;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* tw = reinterpret_cast<C*>(smem_raw);
  C* s = tw + N;
  C* s2 = s + N * kW;   // second tile (XFWD_Z, YMID1)
  const int tid = threadIdx.x;
  State3D* st = a.st;
  const int mode = a.mode;
  const bool xpass = mode <= XFWD_Z;
  {
    const C* gtw = reinterpret_cast<const C*>(xpass ? a.tb.twx : a.tb.twy);
    for (int i = tid; i < N; i += NTHR) tw[i] = gtw[i];
  }
  __syncthreads();
  if (st->done) return;
  if ((mode == XFWD_Z || mode == YMID1) && !st->fresh) return;
  if (mode == YMID1R && st->fresh) return;

  const int Nt = a.g.Nt, Ny = a.g.Ny;
  const int ntile = Nt / kW;
  const int o = blockIdx.x / ntile;          // y index (x pass) or kx index (y pass)
  const int w0 = (blockIdx.x % ntile) * kW;  // omega offset
  const long long stride = xpass ? (long long)Ny * Nt : (long long)Nt;
  const long long base = (xpass ? (long long)o * Nt : (long long)o * Ny * Nt) + w0;
  const double h = st->h;
  TileIdx<C> idx;
  BlockSync sync;
  const C* in = reinterpret_cast<const C*>(a.in);
  C* out = reinterpret_cast<C*>(a.out);

  if (xpass) {
    const bool inv = (mode == XINV || mode == XINV_Z);
    load_tile<C, N, NTHR>(s, in, base, stride, tid);
    __syncthreads();
    if (inv) stockham<N, kW, NTHR, +1, 1, C>(s, tw, tid, idx, sync);
    else stockham<N, kW, NTHR, -1, 1, C>(s, tw, tid, idx, sync);
    store_tile<C, N, NTHR>(s, out, base, stride, tid);
    if (mode == XINV_Z) {
      // candidate state Z = ifft2(A4) * filter(omega) * exp(-damp(x,y) h)
      C* zc = reinterpret_cast<C*>(a.b.z[st->zidx ^ 1]);
      const Rl nrm = (Rl)(1.0 / ((double)a.g.Nx * (double)a.g.Ny));
#pragma unroll
      for (int i = 0; i < E; ++i) {
        const int e = tid + i * NTHR;
        const int n = e / kW, w = e % kW;   // n = x index, o = y index
        const double dp = a.tb.damp[(long long)n * Ny + o];
        const Rl ab = dp == 0.0 ? (Rl)1 : (Rl)exp(-dp * h);   // exp(-0 h) = 1 exactly
        const Rl f = (Rl)a.tb.filt[w0 + w];
        C v = s[idx(w, n)];
        v = cscale(cscale(cscale(v, nrm), f), ab);
        zc[base + n * stride + w] = v;
      }
    }
    if (mode == XFWD_Z) {
      const C* zin = reinterpret_cast<const C*>(a.b.z[st->zidx]);
      C* zout = reinterpret_cast<C*>(a.b.tmp[2]);
      __syncthreads();
      load_tile<C, N, NTHR>(s, zin, base, stride, tid);
      __syncthreads();
      stockham<N, kW, NTHR, -1, 1, C>(s, tw, tid, idx, sync);
      store_tile<C, N, NTHR>(s, zout, base, stride, tid);
    }
    return;
  }

  if (mode == YPLAIN_INV || mode == YPLAIN_FWD) {   // plain y FFT (adjoint passes)
    load_tile<C, N, NTHR>(s, in, base, stride, tid);
    __syncthreads();
    if (mode == YPLAIN_INV) stockham<N, kW, NTHR, +1, 1, C>(s, tw, tid, idx, sync);
    else stockham<N, kW, NTHR, -1, 1, C>(s, tw, tid, idx, sync);
    if (a.scale != 1.0) {
      const Rl sc = (Rl)a.scale;
      for (int e = tid; e < N * kW; e += NTHR) s[e] = cscale(s[e], sc);
      __syncthreads();
    }
    store_tile<C, N, NTHR>(s, out, base, stride, tid);
    return;
  }
  // ---------------- y passes (stage algebra in the (kx, ky, omega) domain) ----
  C* __restrict__ acur = reinterpret_cast<C*>(a.b.acur);
  C* __restrict__ k1b = reinterpret_cast<C*>(a.b.k1);
  C* __restrict__ tsum = reinterpret_cast<C*>(a.b.tsum);
  C* __restrict__ a4p = reinterpret_cast<C*>(a.b.a4p);
  const double h2 = 0.5 * h;
  const Rl hR = (Rl)h, h2R = (Rl)(h / 2), h6R = (Rl)(h / 6);
  // stage operands of this thread's elements, prefetched before the tile FFT so
  // their latency overlaps it (element i: e = tid + i*NTHR)
  C opA[E], opB[E];
  auto eidx = [&](int i) {
    const int e = tid + i * NTHR;
    return base + (long long)(e / kW) * stride + (e % kW);
  };
  if (mode == YMID1R) {
#pragma unroll
    for (int i = 0; i < E; ++i) { opA[i] = __ldg(acur + eidx(i)); opB[i] = __ldg(k1b + eidx(i)); }
  } else if (mode == YMID2 || mode == YMID3) {
#pragma unroll
    for (int i = 0; i < E; ++i) { opA[i] = __ldg(acur + eidx(i)); opB[i] = __ldg(tsum + eidx(i)); }
  } else if (mode == YMID4) {
#pragma unroll
    for (int i = 0; i < E; ++i) opB[i] = __ldg(tsum + eidx(i));
  } else if (mode == YFWD5) {
#pragma unroll
    for (int i = 0; i < E; ++i) {
      opA[i] = __ldg(a4p + eidx(i));
      if (sizeof(Rl) == 8) opB[i] = __ldg(tsum + eidx(i));
    }
  }

  if (mode != YMID1R) {
    load_tile<C, N, NTHR>(s, in, base, stride, tid);
    if (mode == YMID1) load_tile<C, N, NTHR>(s2, reinterpret_cast<const C*>(a.b.tmp[2]), base, stride, tid);
    __syncthreads();
    stockham<N, kW, NTHR, -1, 1, C>(s, tw, tid, idx, sync);
    if (mode == YMID1) stockham<N, kW, NTHR, -1, 1, C>(s2, tw, tid, idx, sync);
  }

  double red = 0.0;
  // every element of this thread has omega column w0 + tid % kW (NTHR is a
  // multiple of kW), so the per-omega tables are read once
  const OmegaCol oc(a.tb, w0 + tid % kW);
#pragma unroll
  for (int i = 0; i < E; ++i) {
    const int e = tid + i * NTHR;
    const int n = e / kW, w = e % kW;     // n = ky, o = kx
    const long long gi = base + n * stride + w;
    const int iw = w0 + w;
    if (mode == YFWD5) {
      const C a5 = s[idx(w, n)];
      const C a4 = opA[i];
      double d;
      if (sizeof(Rl) == 8) {
        // literal |A4 - A3| as in solver_3d.py:145-151
        const C beta = opB[i];
        const C A4 = cadd(beta, cscale(a4, h6R));
        const Rl h30 = (Rl)(h / 30);
        const C A3 = cadd(beta, cscale(cadd(cscale(a4, (Rl)2), cscale(a5, (Rl)3)), h30));
        const C dd = csub(A4, A3);
        d = (double)dd.x * dd.x + (double)dd.y * dd.y;
      } else {
        const double dx = (double)a4.x - (double)a5.x, dy = (double)a4.y - (double)a5.y;
        d = dx * dx + dy * dy;
      }
      red = (d > red || d != d) ? d : red;   // max of the squares (root taken once below)
      continue;
    }
    if (mode == YMID4) {
      const C a4 = s[idx(w, n)];
      const C beta = opB[i];
      const C A4 = cadd(beta, cscale(a4, h6R));
      a4p[gi] = a4;
      const double m = (double)A4.x * A4.x + (double)A4.y * A4.y;
      red = (m > red || m != m) ? m : red;
      s[idx(w, n)] = A4;
      continue;
    }
    const double qv = a.tb.q[(long long)o * Ny + n];
    const C Ef = IPFactor<Rl>::get(a.tb, oc, iw, qv, h2);
    if (mode == YMID1 || mode == YMID1R) {
      C A, k1;
      if (mode == YMID1) {
        A = s2[idx(w, n)];
        k1 = s[idx(w, n)];
        acur[gi] = A;
        k1b[gi] = k1;
      } else {
        A = opA[i];
        k1 = opB[i];
      }
      const C v = cmul(A, Ef);
      const C a1 = cmul(k1, Ef);
      tsum[gi] = a1;
      s[idx(w, n)] = cadd(v, cscale(a1, h2R));
      if (a.save_u) reinterpret_cast<C*>(a.save_u)[gi] = s[idx(w, n)];   // u2
    } else if (mode == YMID2) {
      const C a2 = s[idx(w, n)];
      const C v = cmul(opA[i], Ef);
      const C ts = opB[i];
      tsum[gi] = cadd(ts, cscale(a2, (Rl)2));
      s[idx(w, n)] = cadd(v, cscale(a2, h2R));
      if (a.save_u) reinterpret_cast<C*>(a.save_u)[gi] = s[idx(w, n)];   // u3
    } else {   // YMID3
      const C a3 = s[idx(w, n)];
      const C v = cmul(opA[i], Ef);
      const C ts = cadd(opB[i], cscale(a3, (Rl)2));
      const C beta = cmul(cadd(v, cscale(ts, h6R)), Ef);
      tsum[gi] = beta;
      s[idx(w, n)] = cmul(cadd(v, cscale(a3, hR)), Ef);
      if (a.save_u) reinterpret_cast<C*>(a.save_u)[gi] = s[idx(w, n)];   // u4
    }
  }
  if (mode == YMID4 || mode == YFWD5) {
    red = warp_max<(NTHR < 32 ? NTHR : 32)>(red);
    // sqrt and the positive factor are monotone, so the root of the largest square
    // is the largest root, bit for bit
    const double rv = (mode == YMID4 || sizeof(Rl) == 8) ? sqrt(red) : (h / 10.0) * sqrt(red);
    if ((tid & 31) == 0) atomic_max_nonneg(mode == YMID4 ? &st->red_norm : &st->red_diff, rv);
    if (mode == YFWD5) return;
  }
  __syncthreads();
  stockham<N, kW, NTHR, +1, 1, C>(s, tw, tid, idx, sync);
  store_tile<C, N, NTHR>(s, out, base, stride, tid);
}

// ---------------------------------------------------------------------------
// x passes for square sizes N = R*R (16, 64, 256): register four-step FFT.
// Thread (w, j) of a tile (kW omega-columns, N rows) holds rows j + R*i, i < R,
// both in natural order and in the four-step output order (X[k1 + R k2] with
// k1 = j), so loads and stores go directly between registers and HBM (a
// half-warp covers 16 consecutive omega = 128 contiguous bytes per row).
// One FFT = R-point DFT in registers, twiddle, one shared-memory transpose,
// R-point DFT; the inverse is the same with conjugated roots.
// ---------------------------------------------------------------------------
template <int R, int DIR, typename C, int KW = kW>
__device__ __forceinline__ void fft_sq(C (&v)[R], C* T, const C* tw, int j, int w) {
  DFT<R, DIR, C>::run(v);
#pragma unroll
  for (int k = 1; k < R; ++k) {
    C t = tw[j * k];                 // exp(-2 pi i j k / N), j k < N
    if (DIR > 0) t.y = -t.y;
    v[k] = cmul(v[k], t);
  }
#pragma unroll
  for (int k = 0; k < R; ++k) T[(k * R + j) * KW + w] = v[k];
  __syncthreads();
#pragma unroll
  for (int k = 0; k < R; ++k) v[k] = T[(j * R + k) * KW + w];
  __syncthreads();
  DFT<R, DIR, C>::run(v);
}

// XM: the pass (XINV, XINV_Z, XFWD, XFWD_Z) as a compile-time constant, so that
// each instantiation holds only its own path (fewer live registers for the plain
// transforms, which are seven of an attempt's nine x passes).
// NTC > 0: the omega extent Nt (and Ny = Nx) as compile-time constants, so the
// row stride Ny Nt and the row offsets fold into the address arithmetic.
template <typename Rl, int R, int XM, int NTC = 0>
__global__ void __launch_bounds__(kW * R, (sizeof(Rl) == 4 && R == 16) ? 3 : 1)
k_xpass_sq(SpaceArgs a) {
  using C = typename CT<Rl>::T;
  constexpr int N = R * R;
  constexpr int NTHR = kW * R;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* tw = reinterpret_cast<C*>(smem_raw);
  C* T = tw + N;
  const int tid = threadIdx.x, w = tid % kW, j = tid / kW;
  State3D* st = a.st;
  constexpr int mode = XM;
  {
    const C* gtw = reinterpret_cast<const C*>(a.tb.twx);
    for (int i = tid; i < N; i += NTHR) tw[i] = gtw[i];
  }
  __syncthreads();
  if (st->done) return;
  if constexpr (mode == XFWD_Z) if (!st->fresh) return;
  const int Nt = NTC > 0 ? NTC : a.g.Nt, Ny = NTC > 0 ? N : a.g.Ny;
  const int ntile = Nt / kW;
  const int o = blockIdx.x / ntile;          // y index
  const int w0 = (blockIdx.x % ntile) * kW;  // omega offset
  const long long stride = (long long)Ny * Nt;
  const long long base = (long long)o * Nt + w0 + w;
  const double h = st->h;
  const C* __restrict__ in = reinterpret_cast<const C*>(a.in);
  C* __restrict__ out = reinterpret_cast<C*>(a.out);
  C v[R];
  auto gidx = [&](int i) { return base + (long long)(j + R * i) * stride; };
  constexpr bool inv = (mode == XINV || mode == XINV_Z);
#pragma unroll
  for (int i = 0; i < R; ++i) v[i] = __ldg(in + gidx(i));
  if constexpr (inv) fft_sq<R, +1>(v, T, tw, j, w);
  else fft_sq<R, -1>(v, T, tw, j, w);
#pragma unroll
  for (int i = 0; i < R; ++i) out[gidx(i)] = v[i];
  if constexpr (mode == XINV_Z) {
    // candidate state Z = ifft2(A4) * filter(omega) * exp(-damp(x,y) h); one
    // absorber factor per x of this y (exp(-0 h) = 1 exactly), kept in the
    // transpose buffer, which fft_sq has released
    Rl* absx = reinterpret_cast<Rl*>(T);
    for (int x = tid; x < N; x += NTHR) {
      const double dp = a.tb.damp[(long long)x * Ny + o];
      absx[x] = dp == 0.0 ? (Rl)1 : (Rl)exp(-dp * h);
    }
    __syncthreads();
    C* __restrict__ zc = reinterpret_cast<C*>(a.b.z[st->zidx ^ 1]);
    const Rl nrm = (Rl)(1.0 / ((double)a.g.Nx * (double)a.g.Ny));
    const Rl f = (Rl)a.tb.filt[w0 + w];
#pragma unroll
    for (int i = 0; i < R; ++i) {
      const int x = j + R * i;   // output row = x index, o = y index
      zc[gidx(i)] = cscale(cscale(cscale(v[i], nrm), f), absx[x]);
    }
  }
  if constexpr (mode == XFWD_Z) {
    const C* __restrict__ zin = reinterpret_cast<const C*>(a.b.z[st->zidx]);
    C* __restrict__ zout = reinterpret_cast<C*>(a.b.tmp[2]);
#pragma unroll
    for (int i = 0; i < R; ++i) v[i] = __ldg(zin + gidx(i));
    fft_sq<R, -1>(v, T, tw, j, w);
#pragma unroll
    for (int i = 0; i < R; ++i) zout[gidx(i)] = v[i];
  }
}

// ---------------------------------------------------------------------------
// t-line nonlinear pass (media_physics.py:156-205 + the plasma kernel :11-67)
// ---------------------------------------------------------------------------
enum TMode { T_GENERAL = 0, T_FROM_Z = 1 };

struct TArgs {
  int diag;           // 1: evaluate even when the run is done (final-state diagnostics)
  State3D* st;
  Tables3D tb;
  Medium3D md;
  Bufs3D b;
  Geom g;
  const void* in;
  void* out;
  int mode;
};

template <int NT> struct TCfg {
  static constexpr int PAD = NT + NT / 16;
  static constexpr int FT = NT / 2 < 32 ? NT / 2 : 32;   // FFT team (lanes >= FT idle)
};
// one padding element per 16: conflict-free for the per-lane chunk accesses
// (lane l at 17 l) and for the Stockham writes of 8-byte elements
__device__ __forceinline__ int tpad(int n) { return n + (n >> 4); }

template <typename C, int NT>
__device__ __forceinline__ void load_line(C* s, const C* __restrict__ src, int lane) {
  // 16-byte vector loads, all issued before the shared stores
  constexpr int EPV = 16 / (int)sizeof(C);          // elements per vector
  if constexpr (NT >= 32 * EPV) {
    constexpr int NV = NT / (32 * EPV);
    const float4* __restrict__ v = reinterpret_cast<const float4*>(src);
    float4 r[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) r[k] = __ldg(v + lane + 32 * k);
#pragma unroll
    for (int k = 0; k < NV; ++k) {
      const C* e = reinterpret_cast<const C*>(&r[k]);
#pragma unroll
      for (int q = 0; q < EPV; ++q) s[tpad((lane + 32 * k) * EPV + q)] = e[q];
    }
  } else {
    for (int n = lane; n < NT; n += 32) s[tpad(n)] = src[n];
  }
}
struct LineIdx {
  __device__ __forceinline__ int operator()(int, int n) const { return tpad(n); }
};
struct WarpSync {
  __device__ __forceinline__ void operator()() const { __syncwarp(); }
};

template <typename Rl, int NT, int WPB>
__global__ void __launch_bounds__(WPB * 32, (sizeof(Rl) == 4 && NT <= 512) ? 3 : 1)
k_tpass(TArgs a) {
  using C = typename CT<Rl>::T;
  constexpr int PAD = TCfg<NT>::PAD;
  constexpr int E = NT / 32;                  // samples per lane (one contiguous chunk)
  constexpr bool KEEP_W = E <= 16;            // keep the rates in registers
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* tw = reinterpret_cast<C*>(smem_raw);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  C* sK = tw + NT + warp * 2 * PAD;
  C* sP = sK + PAD;
  {
    const C* gtw = reinterpret_cast<const C*>(a.tb.twt);
    for (int i = threadIdx.x; i < NT; i += WPB * 32) tw[i] = gtw[i];
  }
  __syncthreads();
  State3D* st = a.st;
  if (st->done && !a.diag) return;
  if (a.mode == T_FROM_Z && !st->fresh) return;
  const long long line = (long long)blockIdx.x * WPB + warp;
  const long long nlines = (long long)a.g.Nx * a.g.Ny;
  if (line >= nlines) return;
  const C* in = a.mode == T_FROM_Z ? reinterpret_cast<const C*>(a.b.z[st->zidx])
                                   : reinterpret_cast<const C*>(a.in);
  C* out = reinterpret_cast<C*>(a.out);
  const Rl in_scale = (Rl)(a.mode == T_FROM_Z ? 1.0 / NT
                                               : 1.0 / ((double)NT * a.g.Nx * a.g.Ny));
  const Rl A_scaleR = (Rl)st->A_scale;
  const Medium3D& m = a.md;
  LineIdx idx;
  WarpSync wsync;

  // load (16-byte vectors, coalesced) and inverse FFT along t
  load_line<C, NT>(sK, in + line * NT, lane);
  __syncwarp();
  stockham<NT, 1, TCfg<NT>::FT, +1, 1, C>(sK, tw, lane, idx, wsync);

  // ---- nonlinear response on this lane's chunk t in [lane*E, lane*E+E) ----
  const int t0 = lane * E;
  float Wr[KEEP_W ? E : 1];
  bool any_w = false;
  if (m.plasma) {
#pragma unroll
    for (int i = 0; i < E; ++i) {
      const C Ap = cscale(cscale(sK[tpad(t0 + i)], in_scale), A_scaleR);
      const float w = (float)lut_eval<Rl>(a.tb.lut, Ap.x * Ap.x + Ap.y * Ap.y);
      any_w |= (w != 0.f);
      if constexpr (KEEP_W) Wr[i] = w;
    }
  }
  const bool plasma_line = m.plasma && (__any_sync(0xffffffffu, any_w) || m.ava != 0.0);
  double rho0 = 0.0;
  if (plasma_line) {
    // composed affine map of the chunk: rho' = rho (e - w sf) + w rho_nt sf,
    // valid while no clamp binds (w sf <= e, no avalanche)
    const AffineStep aff(m);
    bool ok = (m.ava == 0.0);
    double cmap = 1.0, dmap = 0.0;
#pragma unroll
    for (int i = 0; i < E; ++i) {
      double w;
      if constexpr (KEEP_W) {
        w = (double)Wr[i];
      } else {
        const C Ap = cscale(cscale(sK[tpad(t0 + i)], in_scale), A_scaleR);
        w = (double)(float)lut_eval<Rl>(a.tb.lut, Ap.x * Ap.x + Ap.y * Ap.y);
      }
      const double c = aff.e - w * aff.sf;
      ok &= (c >= 0.0);
      dmap = c * dmap + w * m.rho_nt * aff.sf;
      cmap = c * cmap;
    }
    if (__all_sync(0xffffffffu, ok)) {
      // exclusive scan of affine maps over lanes: (c1,d1) then (c2,d2) = (c1 c2, c2 d1 + d2)
      double c = cmap, d = dmap;
#pragma unroll
      for (int off = 1; off < 32; off <<= 1) {
        const double cp = __shfl_up_sync(0xffffffffu, c, off);
        const double dp = __shfl_up_sync(0xffffffffu, d, off);
        if (lane >= off) { d = c * dp + d; c = c * cp; }
      }
      const double excl = __shfl_up_sync(0xffffffffu, d, 1);
      rho0 = lane == 0 ? 0.0 : excl;
    } else {
      // a clamp binds on this line: lane 0 runs the exact serial update and
      // records the density at each chunk start
      double* starts = reinterpret_cast<double*>(sP);
      if (lane == 0) {
        double rho = 0.0;
        for (int t = 0; t < NT; ++t) {
          if (t % E == 0) starts[t / E] = rho;
          const C Ap = cscale(cscale(sK[tpad(t)], in_scale), A_scaleR);
          const Rl I = Ap.x * Ap.x + Ap.y * Ap.y;
          const double w = (double)(float)lut_eval<Rl>(a.tb.lut, I);
          const double wa = (double)(float)(m.ava * (double)I);
          rho_step(rho, w, wa, m);
        }
      }
      __syncwarp();
      rho0 = starts[lane];
      __syncwarp();
    }
  }
  // Kerr (+ plasma) terms; exact per-sample density update from the chunk start
  double ion = 0.0;
  {
    double rho = rho0;
#pragma unroll
    for (int i = 0; i < E; ++i) {
      const int t = t0 + i;
      const C av = cscale(sK[tpad(t)], in_scale);
      const C Ap = cscale(av, A_scaleR);
      const Rl I = Ap.x * Ap.x + Ap.y * Ap.y;
      Rl g = (Rl)m.gk * I;
      if (m.g4 != 0.0) g += (Rl)m.g4 * I * I;
      sK[tpad(t)] = C{-g * av.y, g * av.x};   // i g a
      if (plasma_line) {
        double w;
        if constexpr (KEEP_W) w = (double)Wr[i];
        else w = (double)(float)lut_eval<Rl>(a.tb.lut, I);
        const double wa = (double)(float)(m.ava * (double)I);
        const double rho_t = rho;
        ion = fmax(ion, rho_t);
        const double gen = rho_step(rho, w, wa, m);
        const double loss = -(gen * m.Ui) / (2.0 * (double)I + 1e-30);
        const double cr = loss - m.sigma_half * rho_t;
        const double ci = -m.sigma_half * m.w0tc * rho_t;
        sP[tpad(t)] = C{(Rl)cr * av.x - (Rl)ci * av.y, (Rl)cr * av.y + (Rl)ci * av.x};
      }
    }
  }
  if (plasma_line && a.mode == T_FROM_Z) {
    ion = warp_max(ion / m.rho_nt);
    if (lane == 0) atomic_max_nonneg(&st->ion_bits, ion);
  }
  __syncwarp();
  stockham<NT, 1, TCfg<NT>::FT, -1, 1, C>(sK, tw, lane, idx, wsync);
  if (plasma_line) stockham<NT, 1, TCfg<NT>::FT, -1, 1, C>(sP, tw, lane, idx, wsync);
  C* dst = out + line * NT;
#pragma unroll
  for (int i = 0; i < E; ++i) {
    const int wi = lane + 32 * i;
    const Rl sh = (Rl)a.tb.shock[wi];
    C v = cscale(sK[tpad(wi)], sh);
    if (plasma_line) v = cadd(v, sP[tpad(wi)]);
    if (!a.tb.valid[wi]) v = C{0, 0};
    dst[wi] = v;
  }
}

// ---------------------------------------------------------------------------
// y passes of the complex64 attempt with a TMA-fed stage tile (Ny <= 256).
// Persistent CTAs (two per SM) walk the (kx, omega-tile) list; the tile to be
// transformed (Ny rows x kW omega columns, 128-byte rows) arrives by
// cp.async.bulk.tensor into one of two shared-memory buffers while the CTA
// works on the other, and the operand fields of the stage algebra are loaded
// into registers before the wait, so the HBM stream overlaps the FFTs.  One
// instantiation per pass (MODE); same arithmetic, element by element, as the
// y-pass branch of k_space.
// ---------------------------------------------------------------------------
struct YMaps {
  CUtensorMap in;     // (omega, ky, kx) view of the pass input (tmp[1])
  CUtensorMap acur;   // the same view of A = fft2(Z) (YMID1R transforms no input)
  CUtensorMap z2;     // the same view of tmp[2] = fft_x(Z) (YMID1's second field)
  CUtensorMap tsum;   // the stage operands, prefetched into L2 one tile ahead
  CUtensorMap k1;
  CUtensorMap a4p;
};

__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}

// bounded wait on an mbarrier phase: false when the limit ran out
__device__ __forceinline__ bool mbar_wait(unsigned bar, unsigned parity) {
  for (int it = 0; it < (1 << 22); ++it) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok) : "r"(bar), "r"(parity) : "memory");
    if (ok) return true;
  }
  return false;
}

// LATE = 0: the stage operands of a tile are loaded into registers before its
// wait (two CTAs per SM); LATE = 1: they are loaded where they are used (from L2,
// where the previous tile prefetched them), which leaves room for three CTAs per
// SM.  Same arithmetic either way.
// KW omega columns per tile (16 or 8, 256 or 128 threads: the same radix plan per
// column, so both compute the same bits); MINB resident CTAs per SM.
template <int KW, int LATE> struct YTmaCfg {
  static constexpr int NTHR = 16 * KW;
  static constexpr int MINB = KW == 16 ? (LATE ? 3 : 2) : (LATE ? 6 : 4);
};
template <int N, int MODE, int LATE, int KW>
__global__ void __launch_bounds__(YTmaCfg<KW, LATE>::NTHR, YTmaCfg<KW, LATE>::MINB)
k_ypass_tma(SpaceArgs a, const __grid_constant__ YMaps maps) {
  using C = float2;
  using Rl = float;
  constexpr int NTHR = YTmaCfg<KW, LATE>::NTHR;
  constexpr int E = N * KW / NTHR;
  constexpr int TILE = N * KW;
  // the dynamic window starts at offset 0 (no static shared memory here); the
  // buffers are TILE * 8 = 128 N bytes apart, so each starts 128-byte aligned
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr bool TWO = MODE == YMID1;   // YMID1 also transforms fft_x(Z) (single-buffered tile)
  const int tid = threadIdx.x;
  C* buf[2] = {reinterpret_cast<C*>(smem_raw), reinterpret_cast<C*>(smem_raw) + TILE};
  C* bufA = buf[1] + TILE;
  C* tw = TWO ? bufA + TILE : buf[1] + TILE;
  unsigned long long* mbar = reinterpret_cast<unsigned long long*>(tw + N);   // [2]: bufA
  double* qrow = reinterpret_cast<double*>(mbar + 3);   // k_perp^2 of the tile's kx row [N]
  State3D* st = a.st;
  if (st->done) return;
  if (MODE == YMID1R && st->fresh) return;
  if (MODE == YMID1 && !st->fresh) return;
  const int Nt = a.g.Nt, Ny = a.g.Ny;
  const int ntw = Nt / KW;
  const int total = a.g.Nx * ntw;
  auto issue = [&](int tile, int b) {
    const int o = tile / ntw, w0 = (tile % ntw) * KW;
    const unsigned bar = smem_u32(&mbar[b]);
    const CUtensorMap* map = MODE == YMID1R ? &maps.acur : &maps.in;
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
                 :: "r"(bar), "r"((unsigned)(TILE * sizeof(C))) : "memory");
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
        :: "r"(smem_u32(buf[b])), "l"(reinterpret_cast<unsigned long long>(map)), "r"(w0), "r"(0), "r"(o),
           "r"(bar)
        : "memory");
  };
  // the next tile's stage operands into L2 (their loads below then hit L2)
  auto prefetch_ops = [&](int tile) {
    const int o = tile / ntw, w0 = (tile % ntw) * KW;
    auto pf = [&](const CUtensorMap* m) {
      asm volatile("cp.async.bulk.prefetch.tensor.3d.L2.global.tile [%0, {%1, %2, %3}];"
                   :: "l"(reinterpret_cast<unsigned long long>(m)), "r"(w0), "r"(0), "r"(o) : "memory");
    };
    if constexpr (MODE == YMID2 || MODE == YMID3) { pf(&maps.acur); pf(&maps.tsum); }
    else if constexpr (MODE == YMID4) pf(&maps.tsum);
    else if constexpr (MODE == YMID1R) pf(&maps.k1);
    else if constexpr (MODE == YFWD5) pf(&maps.a4p);
  };
  auto issueA = [&](int tile) {
    const int o = tile / ntw, w0 = (tile % ntw) * KW;
    const unsigned bar = smem_u32(&mbar[2]);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
                 :: "r"(bar), "r"((unsigned)(TILE * sizeof(C))) : "memory");
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
        :: "r"(smem_u32(bufA)), "l"(reinterpret_cast<unsigned long long>(&maps.z2)), "r"(w0), "r"(0), "r"(o),
           "r"(bar)
        : "memory");
  };
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_u32(&mbar[0])) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_u32(&mbar[1])) : "memory");
    if (TWO) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_u32(&mbar[2])) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  {
    const C* gtw = reinterpret_cast<const C*>(a.tb.twy);
    for (int i = tid; i < N; i += NTHR) tw[i] = gtw[i];
  }
  __syncthreads();
  if (tid == 0 && (int)blockIdx.x < total) {
    issue(blockIdx.x, 0);
    if (TWO) issueA(blockIdx.x);
  }

  C* __restrict__ acur = reinterpret_cast<C*>(a.b.acur);
  C* __restrict__ k1b = reinterpret_cast<C*>(a.b.k1);
  C* __restrict__ tsum = reinterpret_cast<C*>(a.b.tsum);
  C* __restrict__ a4p = reinterpret_cast<C*>(a.b.a4p);
  C* __restrict__ out = reinterpret_cast<C*>(a.out);
  C* __restrict__ su = reinterpret_cast<C*>(a.save_u);
  const double h = st->h;
  const double h2 = 0.5 * h;
  const Rl hR = (Rl)h, h2R = (Rl)(h / 2), h6R = (Rl)(h / 6);
  TileIdxK<KW> idx;
  BlockSync sync;
  double red = 0.0;
  int k = 0;
  for (int tile = blockIdx.x; tile < total; tile += gridDim.x, ++k) {
    const int b = k & 1;
    const bool next = tile + (int)gridDim.x < total;
    if (tid == 0 && next) {
      issue(tile + gridDim.x, b ^ 1);
      prefetch_ops(tile + gridDim.x);
    }
    const int o = tile / ntw, w0 = (tile % ntw) * KW;
    const long long base = (long long)o * Ny * Nt + w0;
    // operands of this thread's elements (e = tid + i*NTHR), in flight during the wait and FFT
    C opA[LATE ? 1 : E], opB[LATE ? 1 : E];
    auto load_ops = [&](int i, C& A_, C& B_) {
      const int e = tid + i * NTHR;
      const long long gi = base + (long long)(e / KW) * Nt + (e % KW);
      if constexpr (MODE == YMID2 || MODE == YMID3) { A_ = __ldg(acur + gi); B_ = __ldg(tsum + gi); }
      else if constexpr (MODE == YMID4) B_ = __ldg(tsum + gi);
      else if constexpr (MODE == YMID1R) B_ = __ldg(k1b + gi);
      else if constexpr (MODE == YFWD5) A_ = __ldg(a4p + gi);
    };
    constexpr int QN = (N + NTHR - 1) / NTHR;   // k_perp^2 values of the row per thread
    double qn[QN];
#pragma unroll
    for (int i = 0; i < QN; ++i) {
      const int n = tid + i * NTHR;
      qn[i] = (n < N && MODE != YMID4 && MODE != YFWD5) ? __ldg(a.tb.q + (long long)o * Ny + n) : 0.0;
    }
    if constexpr (!LATE) {
#pragma unroll
      for (int i = 0; i < E; ++i) load_ops(i, opA[i], opB[i]);
    }
#pragma unroll
    for (int i = 0; i < QN; ++i)
      if (tid + i * NTHR < N) qrow[tid + i * NTHR] = qn[i];   // read after the barrier below
    bool ok = mbar_wait(smem_u32(&mbar[b]), (unsigned)((k >> 1) & 1));
    if (TWO) ok = ok && mbar_wait(smem_u32(&mbar[2]), (unsigned)(k & 1));
    if (!__syncthreads_and(ok)) {     // a tile never arrived: stop the run with a status
      if (tid == 0) {
        atomicOr(&st->status, UPPE_STATUS_DEVICE_WAIT);
        st->done = 1;
        // every copy this CTA started must have landed before it exits: wait again,
        // bounded, on each barrier with a copy in flight
        mbar_wait(smem_u32(&mbar[b]), (unsigned)((k >> 1) & 1));
        if (next) mbar_wait(smem_u32(&mbar[b ^ 1]), (unsigned)(((k + 1) >> 1) & 1));
        if (TWO) mbar_wait(smem_u32(&mbar[2]), (unsigned)(k & 1));
      }
      return;
    }
    C* s = buf[b];
    if constexpr (MODE != YMID1R) stockham<N, KW, NTHR, -1, 1, C>(s, tw, tid, idx, sync);
    if constexpr (TWO) stockham<N, KW, NTHR, -1, 1, C>(bufA, tw, tid, idx, sync);
    const OmegaCol oc(a.tb, w0 + tid % KW);
#pragma unroll
    for (int i = 0; i < E; ++i) {
      const int e = tid + i * NTHR;
      const int n = e / KW, w = e % KW;     // n = ky, o = kx; s[e] = s[idx(w, n)]
      const long long gi = base + (long long)n * Nt + w;
      C oA = C{0, 0}, oB = C{0, 0};
      if constexpr (LATE) load_ops(i, oA, oB);
      else { oA = opA[i]; oB = opB[i]; }
      if constexpr (MODE == YFWD5) {
        const C a5 = s[e], a4 = oA;
        const double dx = (double)a4.x - (double)a5.x, dy = (double)a4.y - (double)a5.y;
        const double d = dx * dx + dy * dy;   // max of the squares; root once per warp
        red = (d > red || d != d) ? d : red;
        continue;
      }
      if constexpr (MODE == YMID4) {
        const C a4 = s[e];
        const C A4 = cadd(oB, cscale(a4, h6R));
        a4p[gi] = a4;
        const double m = (double)A4.x * A4.x + (double)A4.y * A4.y;
        red = (m > red || m != m) ? m : red;
        s[e] = A4;
        continue;
      }
      const C Ef = IPFactor<Rl>::get(a.tb, oc, w0 + w, qrow[n], h2);
      C u;
      if constexpr (MODE == YMID1R) {   // s = A tile, opB = k1
        const C v = cmul(s[e], Ef);
        const C a1 = cmul(oB, Ef);
        tsum[gi] = a1;
        u = cadd(v, cscale(a1, h2R));
      } else if constexpr (MODE == YMID1) {   // s = k1 = N(A), bufA = A
        const C A = bufA[e], k1 = s[e];
        acur[gi] = A;
        k1b[gi] = k1;
        const C v = cmul(A, Ef);
        const C a1 = cmul(k1, Ef);
        tsum[gi] = a1;
        u = cadd(v, cscale(a1, h2R));
      } else if constexpr (MODE == YMID2) {
        const C a2 = s[e];
        const C v = cmul(oA, Ef);
        tsum[gi] = cadd(oB, cscale(a2, (Rl)2));
        u = cadd(v, cscale(a2, h2R));
      } else {   // YMID3
        const C a3 = s[e];
        const C v = cmul(oA, Ef);
        const C ts = cadd(oB, cscale(a3, (Rl)2));
        tsum[gi] = cmul(cadd(v, cscale(ts, h6R)), Ef);
        u = cmul(cadd(v, cscale(a3, hR)), Ef);
      }
      s[e] = u;
      if (su) su[gi] = u;
    }
    if constexpr (MODE != YFWD5) {
      __syncthreads();
      // bufA is free once every thread has read its elements: fetch the next tile's
      if (TWO && tid == 0 && tile + (int)gridDim.x < total) issueA(tile + gridDim.x);
      stockham<N, KW, NTHR, +1, 1, C>(s, tw, tid, idx, sync);
      store_tile<C, N, NTHR, KW>(s, out, base, Nt, tid);
    }
    __syncthreads();   // buffer b is refilled at iteration k + 1
  }
  if constexpr (MODE == YMID4 || MODE == YFWD5) {
    red = warp_max<32>(red);
    // the root of the largest square is the largest root (sqrt and h/10 > 0 are monotone)
    const double rv = MODE == YMID4 ? sqrt(red) : (h / 10.0) * sqrt(red);
    if ((tid & 31) == 0) atomic_max_nonneg(MODE == YMID4 ? &st->red_norm : &st->red_diff, rv);
  }
}

template <int N, int KW = kW>
static size_t ytma_smem(int mode) {
  return sizeof(float2) * (size_t)((mode == YMID1 ? 3 : 2) * N * KW + N) + 3 * sizeof(unsigned long long) +
         N * sizeof(double);
}

// ---------------------------------------------------------------------------
// y passes of complex64 plans with Ny = 256 on the register four-step FFT of the
// x passes.  Thread (w, j) of a tile (kW omega columns x 256 ky rows) holds rows
// j + 16 i, i < 16, in registers from the load to the store: a 256-point
// transform is a 16-point DFT in registers, a twiddle, one shared-memory
// transpose and a second 16-point DFT, and bin X[j + 16 k] lands on the same
// thread in register k, so the stage algebra runs on the registers and the
// results go straight back to HBM (half a warp covers 16 consecutive omega =
// one 128-byte row).  Per element that is two shared-memory round trips against
// six for the tile passes of k_ypass_tma.  The DFTs, the twiddles and the order
// they are applied in are those of k_ypass_tma's two radix-16 Stockham passes,
// and the stage algebra is the same expression per element, so both kernels
// give the same bits.  LATE = 0 issues the stage-operand loads with the tile's
// (two CTAs per SM); LATE = 1 issues them element by element in the stage loop
// (three CTAs per SM).  One instantiation per pass.
// ---------------------------------------------------------------------------
// NTC > 0: the omega extent Nt as a compile-time constant (row offsets become
// immediates, which frees the registers of sixteen 64-bit addresses); 0: runtime.
template <int MODE, int LATE, int KW = kW, int NTC = 0>
__global__ void __launch_bounds__(KW * 16, (LATE ? 3 : 2) * (kW / KW))
k_ypass_rq(SpaceArgs a) {
  using C = float2;
  using Rl = float;
  constexpr int R = 16, N = R * R, NTHR = KW * R;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* tw = reinterpret_cast<C*>(smem_raw);
  C* T = tw + N;                                          // transpose buffer, N * KW
  double* qrow = reinterpret_cast<double*>(T + N * KW);   // k_perp^2 of the tile's kx row
  const int tid = threadIdx.x, w = tid % KW, j = tid / KW;
  State3D* st = a.st;
  if (st->done) return;
  if (MODE == YMID1R && st->fresh) return;
  if (MODE == YMID1 && !st->fresh) return;
  const int Nt = NTC > 0 ? NTC : a.g.Nt;
  const int ntile = Nt / KW;
  const int o = blockIdx.x / ntile;            // kx index
  const int w0 = (blockIdx.x % ntile) * KW;    // omega offset
  const long long base = (long long)o * N * Nt + w0 + w;
  auto gidx = [&](int i) { return base + (long long)(j + R * i) * Nt; };
  C* __restrict__ acur = reinterpret_cast<C*>(a.b.acur);
  C* __restrict__ k1b = reinterpret_cast<C*>(a.b.k1);
  C* __restrict__ tsum = reinterpret_cast<C*>(a.b.tsum);
  C* __restrict__ a4p = reinterpret_cast<C*>(a.b.a4p);
  C* __restrict__ out = reinterpret_cast<C*>(a.out);
  C* __restrict__ su = reinterpret_cast<C*>(a.save_u);
  const C* __restrict__ in = reinterpret_cast<const C*>(MODE == YMID1R ? a.b.acur : a.in);
  constexpr bool TWO = MODE == YMID1;          // YMID1 also transforms fft_x(Z) = tmp[2]
  C v[R], v2[TWO ? R : 1];
#pragma unroll
  for (int i = 0; i < R; ++i) v[i] = __ldg(in + gidx(i));
  if constexpr (TWO) {
    const C* __restrict__ z2 = reinterpret_cast<const C*>(a.b.tmp[2]);
#pragma unroll
    for (int i = 0; i < R; ++i) v2[i] = __ldg(z2 + gidx(i));
  }
  C opA[LATE ? 1 : R], opB[LATE ? 1 : R];
  auto load_ops = [&](int i, C& A_, C& B_) {
    const long long gi = gidx(i);
    if constexpr (MODE == YMID2 || MODE == YMID3) { A_ = __ldg(acur + gi); B_ = __ldg(tsum + gi); }
    else if constexpr (MODE == YMID4) B_ = __ldg(tsum + gi);
    else if constexpr (MODE == YMID1R) B_ = __ldg(k1b + gi);
    else if constexpr (MODE == YFWD5) A_ = __ldg(a4p + gi);
  };
  if constexpr (!LATE) {
#pragma unroll
    for (int i = 0; i < R; ++i) load_ops(i, opA[i], opB[i]);
  }
  {
    const C* gtw = reinterpret_cast<const C*>(a.tb.twy);
    for (int i = tid; i < N; i += NTHR) tw[i] = gtw[i];
    if (MODE != YMID4 && MODE != YFWD5)
      for (int i = tid; i < N; i += NTHR) qrow[i] = __ldg(a.tb.q + (long long)o * N + i);
  }
  __syncthreads();
  if constexpr (MODE != YMID1R) fft_sq<R, -1, C, KW>(v, T, tw, j, w);
  if constexpr (TWO) fft_sq<R, -1, C, KW>(v2, T, tw, j, w);
  const double h = st->h;
  const double h2 = 0.5 * h;
  const Rl hR = (Rl)h, h2R = (Rl)(h / 2), h6R = (Rl)(h / 6);
  const OmegaCol oc(a.tb, w0 + w);
  double red = 0.0;
#pragma unroll
  for (int i = 0; i < R; ++i) {
    const int n = j + R * i;                   // ky row of register i
    const long long gi = gidx(i);
    C oA = C{0, 0}, oB = C{0, 0};
    if constexpr (LATE) load_ops(i, oA, oB);
    else { oA = opA[i]; oB = opB[i]; }
    if constexpr (MODE == YFWD5) {
      const C a5 = v[i], a4 = oA;
      const double dx = (double)a4.x - (double)a5.x, dy = (double)a4.y - (double)a5.y;
      const double d = dx * dx + dy * dy;   // max of the squares; root once per warp
      red = (d > red || d != d) ? d : red;
      continue;
    }
    if constexpr (MODE == YMID4) {
      const C a4 = v[i];
      const C A4 = cadd(oB, cscale(a4, h6R));
      a4p[gi] = a4;
      const double m = (double)A4.x * A4.x + (double)A4.y * A4.y;
      red = (m > red || m != m) ? m : red;
      v[i] = A4;
      continue;
    }
    const C Ef = IPFactor<Rl>::get(a.tb, oc, w0 + w, qrow[n], h2);
    C u;
    if constexpr (MODE == YMID1R) {   // v = A, opB = k1
      const C vv = cmul(v[i], Ef);
      const C a1 = cmul(oB, Ef);
      tsum[gi] = a1;
      u = cadd(vv, cscale(a1, h2R));
    } else if constexpr (MODE == YMID1) {   // v = k1 = N(A), v2 = A
      const C A = v2[i], k1 = v[i];
      acur[gi] = A;
      k1b[gi] = k1;
      const C vv = cmul(A, Ef);
      const C a1 = cmul(k1, Ef);
      tsum[gi] = a1;
      u = cadd(vv, cscale(a1, h2R));
    } else if constexpr (MODE == YMID2) {
      const C a2 = v[i];
      const C vv = cmul(oA, Ef);
      tsum[gi] = cadd(oB, cscale(a2, (Rl)2));
      u = cadd(vv, cscale(a2, h2R));
    } else {   // YMID3
      const C a3 = v[i];
      const C vv = cmul(oA, Ef);
      const C ts = cadd(oB, cscale(a3, (Rl)2));
      tsum[gi] = cmul(cadd(vv, cscale(ts, h6R)), Ef);
      u = cmul(cadd(vv, cscale(a3, hR)), Ef);
    }
    v[i] = u;
    if (su) su[gi] = u;
  }
  if constexpr (MODE == YMID4 || MODE == YFWD5) {
    red = warp_max<32>(red);
    // the root of the largest square is the largest root (sqrt and h/10 > 0 are monotone)
    const double rv = MODE == YMID4 ? sqrt(red) : (h / 10.0) * sqrt(red);
    if ((tid & 31) == 0) atomic_max_nonneg(MODE == YMID4 ? &st->red_norm : &st->red_diff, rv);
  }
  if constexpr (MODE != YFWD5) {
    fft_sq<R, +1, C, KW>(v, T, tw, j, w);
#pragma unroll
    for (int i = 0; i < R; ++i) out[gidx(i)] = v[i];
  }
}

template <int KW = kW> static constexpr size_t yrq_smem() {
  return sizeof(float2) * (size_t)(256 + 256 * KW) + 256 * sizeof(double);
}

// ---------------------------------------------------------------------------
// The same y passes (complex64, Ny = 256) on persistent CTAs, one per SM, with
// every HBM operand of a tile on a TMA ring: the pass input tile and the stage
// operand tiles (A, k1, term sum, alpha4', fft_x(Z): the ones the MODE reads,
// 256 ky rows x kW omega columns each, by cp.async.bulk.tensor) and the FP64
// k_perp^2 row of the tile's kx (by cp.async.bulk) land on one mbarrier per ring
// slot, STAGES - 1 tiles ahead of the tile being transformed.  The SM therefore
// always has the next tiles' loads in flight while it runs the register
// four-step FFTs and the stage algebra of the current one, and holds no
// operand in registers across a wait.  Ring: two slots of three tiles (YMID2,
// YMID3: 2 x 96 KB) or three slots of two tiles (the other passes).  The input
// slot doubles as the transpose buffer once its tile is in registers.  Element
// by element the same arithmetic as k_ypass_rq, hence the same bits.
// ---------------------------------------------------------------------------
template <int MODE> struct YRing {
  static constexpr int NOP = (MODE == YMID2 || MODE == YMID3) ? 3 : 2;   // tiles per slot
  static constexpr int STAGES = NOP == 3 ? 2 : 3;
  static constexpr bool Q = MODE != YMID4 && MODE != YFWD5;               // needs k_perp^2
  static constexpr int TILE = 256 * kW;                                   // float2 per tile
  static constexpr size_t bytes() {
    return sizeof(float2) * (size_t)(STAGES * NOP * TILE + 256) + sizeof(double) * 256 * STAGES +
           sizeof(unsigned long long) * STAGES;
  }
};

template <int MODE>
__global__ void __launch_bounds__(kW * 16, 1)
k_ypass_ring(SpaceArgs a, const __grid_constant__ YMaps maps) {
  using C = float2;
  using Rl = float;
  using RG = YRing<MODE>;
  constexpr int R = 16, N = R * R, NTHR = kW * R, TILE = RG::TILE, NOP = RG::NOP, STAGES = RG::STAGES;
  constexpr bool TWO = MODE == YMID1;          // YMID1 also transforms fft_x(Z) = tmp[2]
  extern __shared__ __align__(128) unsigned char smem_raw[];
  C* ring = reinterpret_cast<C*>(smem_raw);                     // [STAGES][NOP][TILE]
  C* tw = ring + STAGES * NOP * TILE;
  double* qbuf = reinterpret_cast<double*>(tw + N);             // [STAGES][256]
  unsigned long long* mbar = reinterpret_cast<unsigned long long*>(qbuf + STAGES * 256);
  State3D* st = a.st;
  if (st->done) return;
  if (MODE == YMID1R && st->fresh) return;
  if (MODE == YMID1 && !st->fresh) return;
  const int tid = threadIdx.x, w = tid % kW, j = tid / kW;
  const int Nt = a.g.Nt;
  const int ntw = Nt / kW;
  const int total = a.g.Nx * ntw;
  // slot order per MODE: YMID1 {in, z2}, YMID1R {A, k1}, YMID2/3 {in, A, tsum},
  // YMID4 {in, tsum}, YFWD5 {in, a4p}
  const CUtensorMap* m0 = MODE == YMID1R ? &maps.acur : &maps.in;
  const CUtensorMap* m1 = MODE == YMID1 ? &maps.z2 : MODE == YMID1R ? &maps.k1
                        : (MODE == YMID2 || MODE == YMID3) ? &maps.acur : MODE == YMID4 ? &maps.tsum : &maps.a4p;
  const CUtensorMap* m2 = &maps.tsum;
  auto slot = [&](int b, int op) { return ring + (b * NOP + op) * TILE; };
  auto issue = [&](int tile, int b) {
    const int o = tile / ntw, w0 = (tile % ntw) * kW;
    const unsigned bar = smem_u32(&mbar[b]);
    const unsigned bytes = (unsigned)(NOP * TILE * sizeof(C)) + (RG::Q ? 256u * 8u : 0u);
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(bar), "r"(bytes) : "memory");
#pragma unroll
    for (int op = 0; op < NOP; ++op) {
      const CUtensorMap* m = op == 0 ? m0 : op == 1 ? m1 : m2;
      asm volatile(
          "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
          :: "r"(smem_u32(slot(b, op))), "l"(reinterpret_cast<unsigned long long>(m)), "r"(w0), "r"(0), "r"(o),
             "r"(bar)
          : "memory");
    }
    if constexpr (RG::Q) {
      // the 2 KB k_perp^2 row of this kx (16-byte aligned: row starts at o * 2048 bytes)
      asm volatile(
          "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
          :: "r"(smem_u32(qbuf + b * 256)),
             "l"((unsigned long long)__cvta_generic_to_global(a.tb.q + (long long)o * N)), "r"(256u * 8u), "r"(bar)
          : "memory");
    }
  };
  if (tid == 0) {
    for (int b = 0; b < STAGES; ++b)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_u32(&mbar[b])) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  {
    const C* gtw = reinterpret_cast<const C*>(a.tb.twy);
    for (int i = tid; i < N; i += NTHR) tw[i] = gtw[i];
  }
  __syncthreads();
  if (tid == 0) {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    for (int s = 0; s < STAGES - 1; ++s) {
      const int t = (int)blockIdx.x + s * (int)gridDim.x;
      if (t < total) issue(t, s);
    }
  }
  C* __restrict__ acur = reinterpret_cast<C*>(a.b.acur);
  C* __restrict__ k1b = reinterpret_cast<C*>(a.b.k1);
  C* __restrict__ tsum = reinterpret_cast<C*>(a.b.tsum);
  C* __restrict__ a4p = reinterpret_cast<C*>(a.b.a4p);
  C* __restrict__ out = reinterpret_cast<C*>(a.out);
  C* __restrict__ su = reinterpret_cast<C*>(a.save_u);
  const double h = st->h;
  const double h2 = 0.5 * h;
  const Rl hR = (Rl)h, h2R = (Rl)(h / 2), h6R = (Rl)(h / 6);
  double red = 0.0;
  int k = 0;
  for (int tile = blockIdx.x; tile < total; tile += gridDim.x, ++k) {
    const int b = k % STAGES;
    if (tid == 0) {   // refill the slot that the previous tile released
      const int t = tile + (STAGES - 1) * (int)gridDim.x;
      if (t < total) issue(t, (k + STAGES - 1) % STAGES);
    }
    const bool ok = mbar_wait(smem_u32(&mbar[b]), (unsigned)((k / STAGES) & 1));
    if (!__syncthreads_and(ok)) {     // a tile never arrived: stop the run with a status
      if (tid == 0) {
        atomicOr(&st->status, UPPE_STATUS_DEVICE_WAIT);
        st->done = 1;
        // every copy this CTA started must have landed before it exits: wait
        // again, bounded, on each slot with a copy in flight
        for (int s = 0; s < STAGES; ++s)
          if (tile + s * (int)gridDim.x < total)
            mbar_wait(smem_u32(&mbar[(k + s) % STAGES]), (unsigned)(((k + s) / STAGES) & 1));
      }
      return;
    }
    const int o = tile / ntw, w0 = (tile % ntw) * kW;
    const long long base = (long long)o * N * Nt + w0 + w;
    auto gidx = [&](int i) { return base + (long long)(j + R * i) * Nt; };
    auto sidx = [&](int i) { return (j + R * i) * kW + w; };
    C* s0 = slot(b, 0);
    const C* s1 = slot(b, 1);
    const C* s2 = slot(b, NOP - 1);
    const double* qrow = qbuf + b * 256;
    C v[R], v2[TWO ? R : 1];
#pragma unroll
    for (int i = 0; i < R; ++i) v[i] = s0[sidx(i)];
    if constexpr (TWO) {
#pragma unroll
      for (int i = 0; i < R; ++i) v2[i] = s1[sidx(i)];
    }
    __syncthreads();                  // the input tile is in registers: slot 0 is the transpose buffer
    if constexpr (MODE != YMID1R) fft_sq<R, -1>(v, s0, tw, j, w);
    if constexpr (TWO) fft_sq<R, -1>(v2, s0, tw, j, w);
    const OmegaCol oc(a.tb, w0 + w);
#pragma unroll
    for (int i = 0; i < R; ++i) {
      const int n = j + R * i;
      const long long gi = gidx(i);
      if constexpr (MODE == YFWD5) {
        const C a5 = v[i], a4 = s1[sidx(i)];
        const double dx = (double)a4.x - (double)a5.x, dy = (double)a4.y - (double)a5.y;
        const double d = dx * dx + dy * dy;   // max of the squares; root once per warp
        red = (d > red || d != d) ? d : red;
        continue;
      }
      if constexpr (MODE == YMID4) {
        const C a4 = v[i];
        const C A4 = cadd(s1[sidx(i)], cscale(a4, h6R));
        a4p[gi] = a4;
        const double m = (double)A4.x * A4.x + (double)A4.y * A4.y;
        red = (m > red || m != m) ? m : red;
        v[i] = A4;
        continue;
      }
      const C Ef = IPFactor<Rl>::get(a.tb, oc, w0 + w, qrow[n], h2);
      C u;
      if constexpr (MODE == YMID1R) {   // v = A, slot 1 = k1
        const C vv = cmul(v[i], Ef);
        const C a1 = cmul(s1[sidx(i)], Ef);
        tsum[gi] = a1;
        u = cadd(vv, cscale(a1, h2R));
      } else if constexpr (MODE == YMID1) {   // v = k1 = N(A), v2 = A
        const C A = v2[i], k1 = v[i];
        acur[gi] = A;
        k1b[gi] = k1;
        const C vv = cmul(A, Ef);
        const C a1 = cmul(k1, Ef);
        tsum[gi] = a1;
        u = cadd(vv, cscale(a1, h2R));
      } else if constexpr (MODE == YMID2) {   // slot 1 = A, slot 2 = term sum
        const C a2 = v[i];
        const C vv = cmul(s1[sidx(i)], Ef);
        tsum[gi] = cadd(s2[sidx(i)], cscale(a2, (Rl)2));
        u = cadd(vv, cscale(a2, h2R));
      } else {   // YMID3
        const C a3 = v[i];
        const C vv = cmul(s1[sidx(i)], Ef);
        const C ts = cadd(s2[sidx(i)], cscale(a3, (Rl)2));
        tsum[gi] = cmul(cadd(vv, cscale(ts, h6R)), Ef);
        u = cmul(cadd(vv, cscale(a3, hR)), Ef);
      }
      v[i] = u;
      if (su) su[gi] = u;
    }
    if constexpr (MODE != YFWD5) {
      fft_sq<R, +1>(v, s0, tw, j, w);
#pragma unroll
      for (int i = 0; i < R; ++i) out[gidx(i)] = v[i];
    }
    // slot b is refilled by the copy issued at iteration k + 1: order this
    // iteration's shared-memory accesses before that async-proxy write
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
  }
  if constexpr (MODE == YMID4 || MODE == YFWD5) {
    red = warp_max<32>(red);
    // the root of the largest square is the largest root (sqrt and h/10 > 0 are monotone)
    const double rv = MODE == YMID4 ? sqrt(red) : (h / 10.0) * sqrt(red);
    if ((tid & 31) == 0) atomic_max_nonneg(MODE == YMID4 ? &st->red_norm : &st->red_diff, rv);
  }
}

// ---------------------------------------------------------------------------
// Warp FFT of a 1024-point t-line (E = 32) held in registers.  Natural layout:
// lane l holds x[l + 32 m], m < E.  Four-step layout: lane L holds
// X[out_index(L, k)] = X[L + 32 k], k < E.  fwd_like: DFT_32 in registers,
// twiddle W_NT^(l k), transpose through a padded shared buffer S, DFT_32.
// bwd_like is the transposed sequence (four-step -> natural).  With DIR=-1
// fwd_like is the forward FFT; with DIR=+1 bwd_like is the unnormalised
// inverse.  tw is the four-step table tw[k*32 + l] = W_NT^(l k).
// ---------------------------------------------------------------------------
template <int E> struct WarpFFT {
  static_assert(E == 32, "the 512-point line has its own specialisation below");
  static constexpr int SP = 33;                      // padded row stride of S
  static constexpr int NT = 32 * E;
  static constexpr int SBUF = E * SP;
  __device__ __forceinline__ static int out_index(int lane, int k) { return lane + E * k; }
  // the twiddle table in shared memory from gtw[i] = W_NT^i
  template <typename C>
  __device__ __forceinline__ static void fill_twiddles(C* tw, const C* gtw, int tid, int nthr) {
    for (int i = tid; i < NT; i += nthr) tw[i] = gtw[(i & 31) * (i >> 5)];
  }
  template <int DIR, typename C>
  __device__ __forceinline__ static void fwd_like(C (&v)[E], C* S, const C* tw, int lane) {
    DFT<E, DIR, C>::run(v);
#pragma unroll
    for (int k = 1; k < E; ++k) {
      C t = tw[k * 32 + lane];
      if (DIR > 0) t.y = -t.y;
      v[k] = cmul(v[k], t);
    }
#pragma unroll
    for (int k = 0; k < E; ++k) S[k * SP + lane] = v[k];
    __syncwarp();
#pragma unroll
    for (int i = 0; i < E; ++i) v[i] = S[lane * SP + i];
    __syncwarp();
    DFT<E, DIR, C>::run(v);
  }
  template <int DIR, typename C>
  __device__ __forceinline__ static void bwd_like(C (&v)[E], C* S, const C* tw, int lane) {
    DFT<E, DIR, C>::run(v);
#pragma unroll
    for (int i = 0; i < E; ++i) S[lane * SP + i] = v[i];
    __syncwarp();
#pragma unroll
    for (int k = 0; k < E; ++k) v[k] = S[k * SP + lane];
    __syncwarp();
#pragma unroll
    for (int k = 1; k < E; ++k) {
      C t = tw[k * 32 + lane];
      if (DIR > 0) t.y = -t.y;
      v[k] = cmul(v[k], t);
    }
    DFT<E, DIR, C>::run(v);
  }
};

// ---------------------------------------------------------------------------
// Warp FFT of a 512-point t-line (E = 16) as three radix-8 stages, natural order
// in and out: lane l holds x[l + 32 m], m < 16, and afterwards X[l + 32 m].
// With n = j + 64 n3 (j < 64) and k = 8 q + r:
//   X[8 q + r] = sum_j W_64^(j q) W_512^(j r) sum_n3 x[j + 64 n3] W_8^(n3 r);
// lane l owns j = l and l + 32 (registers m = 2 n3 + p, j = l + 32 p), so stage
// 1 is two 8-point DFTs in registers and the W_512^(j r) twiddle.  With j = j1 + 8
// j2 and q = 8 s + t the 64-point transform over j is stage 2 (8-point DFTs over
// j2 of the groups (r, j1), twiddle W_64^(j1 t)) and stage 3 (8-point DFTs over
// j1 of the groups (r, t)), and k = 64 s + 8 t + r.  Lane L takes the groups with
// r = L % 8 and j1 (stage 2) or t (stage 3) = L / 8 + 4 g, g < 2, so stage 3
// leaves X[L + 32 (2 s + g)] in register 2 s + g: the natural layout, stored with
// 256-byte warp rows.  Two exchanges through S (padded row strides 66 and 72:
// conflict-free for the 64-bit accesses of both sides).  The same routine with
// DIR = +1 and conjugate twiddles is the unnormalised inverse, so bwd_like =
// fwd_like.  tw: W_512^(j r) at (r - 1) 64 + j, then W_64^(j1 t) at 448 + (t - 1) 8
// + j1.  Against the four-step form with a radix-2 lane-pair step this needs no
// shuffles and about a quarter fewer instructions per point.
// ---------------------------------------------------------------------------
template <> struct WarpFFT<16> {
  static constexpr int E = 16, NT = 512;
  static constexpr int P1 = 66, P2 = 72;             // row strides of the two exchanges
  static constexpr int SBUF = 8 * P2;
  __device__ __forceinline__ static int out_index(int lane, int k) { return lane + 32 * k; }
  template <typename C>
  __device__ __forceinline__ static void fill_twiddles(C* tw, const C* gtw, int tid, int nthr) {
    for (int i = tid; i < 448; i += nthr) tw[i] = gtw[(i & 63) * ((i >> 6) + 1)];
    for (int i = tid; i < 56; i += nthr) tw[448 + i] = gtw[8 * (i & 7) * ((i >> 3) + 1)];
  }
  template <int DIR, typename C>
  __device__ __forceinline__ static void fwd_like(C (&v)[E], C* S, const C* tw, int lane) {
    // stage 1: j = lane + 32 p, 8-point DFT over n3, twiddle W_512^(j r), Z[j][r] -> S[r P1 + j]
#pragma unroll
    for (int p = 0; p < 2; ++p) {
      C e[8];
#pragma unroll
      for (int n3 = 0; n3 < 8; ++n3) e[n3] = v[2 * n3 + p];
      DFT<8, DIR, C>::run(e);
      const int j = lane + 32 * p;
#pragma unroll
      for (int r = 1; r < 8; ++r) {
        C t = tw[(r - 1) * 64 + j];
        if (DIR > 0) t.y = -t.y;
        e[r] = cmul(e[r], t);
      }
#pragma unroll
      for (int r = 0; r < 8; ++r) S[r * P1 + j] = e[r];
    }
    __syncwarp();
    // stage 2: groups (r, j1 = L / 8 + 4 g): 8-point DFT over j2, twiddle W_64^(j1 t)
    const int r = lane & 7, jq = lane >> 3;
    C w[2][8];
#pragma unroll
    for (int g = 0; g < 2; ++g) {
#pragma unroll
      for (int j2 = 0; j2 < 8; ++j2) w[g][j2] = S[r * P1 + jq + 4 * g + 8 * j2];
    }
    __syncwarp();
#pragma unroll
    for (int g = 0; g < 2; ++g) {
      const int j1 = jq + 4 * g;
      DFT<8, DIR, C>::run(w[g]);
#pragma unroll
      for (int t = 1; t < 8; ++t) {
        C tt = tw[448 + (t - 1) * 8 + j1];
        if (DIR > 0) tt.y = -tt.y;
        w[g][t] = cmul(w[g][t], tt);
      }
      // element t of group (r, j1) at S[t P2 + 8 j1 + r] = S[t P2 + lane + 32 g]
#pragma unroll
      for (int t = 0; t < 8; ++t) S[t * P2 + lane + 32 * g] = w[g][t];
    }
    __syncwarp();
    // stage 3: groups (r, t = L / 8 + 4 g): 8-point DFT over j1 -> X[L + 32 g + 64 s]
#pragma unroll
    for (int g = 0; g < 2; ++g) {
      C u[8];
#pragma unroll
      for (int j1 = 0; j1 < 8; ++j1) u[j1] = S[(jq + 4 * g) * P2 + 8 * j1 + r];
      DFT<8, DIR, C>::run(u);
#pragma unroll
      for (int s = 0; s < 8; ++s) v[2 * s + g] = u[s];
    }
    __syncwarp();
  }
  template <int DIR, typename C>
  __device__ __forceinline__ static void bwd_like(C (&v)[E], C* S, const C* tw, int lane) {
    fwd_like<DIR>(v, S, tw, lane);
  }
};

// t-line nonlinear pass with the register warp FFT (NT = 512, and NT = 1024 in
// complex64).  Same physics and operation order as k_tpass; the frequency-domain
// line is read and written in the transform's output order, X[lane + 32 k] in
// register k (coalesced: a warp covers 32 consecutive omega), the time-domain
// samples stay in registers, and only lines that ionise go through shared memory
// in time order for the scan.
template <typename Rl, int E, int WPB>
__global__ void __launch_bounds__(WPB * 32, (sizeof(Rl) == 4 && E == 16) ? 3 : 1)
k_tpass_w(TArgs a) {
  using C = typename CT<Rl>::T;
  using W = WarpFFT<E>;
  constexpr int NT = 32 * E;
  constexpr int PAD = TCfg<NT>::PAD;
  constexpr int BUF = W::SBUF > PAD ? W::SBUF : PAD;    // transpose buffer / time-order line
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* tw = reinterpret_cast<C*>(smem_raw);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  C* S = tw + NT + warp * BUF;
  double* starts = reinterpret_cast<double*>(tw + NT + WPB * BUF) + warp * 32;
  // rates of the line in time order (one pad per 32: conflict-free both ways)
  float* sW0 = reinterpret_cast<float*>(reinterpret_cast<double*>(tw + NT + WPB * BUF) + WPB * 32);
  float* sW = sW0 + warp * (NT + NT / 32);
  // output factor per omega bin: shock factor (> 0) where omega_abs > 0, -1 where masked
  Rl* shm = reinterpret_cast<Rl*>(sW0 + WPB * (NT + NT / 32));
  auto wpad = [](int t) { return t + (t >> 5); };
  {
    // the transform's twiddle table (per-lane factors consecutive: conflict-free
    // loads) and the output factor per omega bin
    W::fill_twiddles(tw, reinterpret_cast<const C*>(a.tb.twt), threadIdx.x, WPB * 32);
    for (int i = threadIdx.x; i < NT; i += WPB * 32) shm[i] = a.tb.valid[i] ? (Rl)a.tb.shock[i] : (Rl)-1;
  }
  __syncthreads();
  State3D* st = a.st;
  if (st->done && !a.diag) return;
  if (a.mode == T_FROM_Z && !st->fresh) return;
  const long long line = (long long)blockIdx.x * WPB + warp;
  const long long nlines = (long long)a.g.Nx * a.g.Ny;
  if (line >= nlines) return;
  const C* __restrict__ src = (a.mode == T_FROM_Z ? reinterpret_cast<const C*>(a.b.z[st->zidx])
                                                 : reinterpret_cast<const C*>(a.in)) + line * NT;
  C* __restrict__ dst = reinterpret_cast<C*>(a.out) + line * NT;
  const Rl in_scale = (Rl)(a.mode == T_FROM_Z ? 1.0 / NT
                                               : 1.0 / ((double)NT * a.g.Nx * a.g.Ny));
  const Rl A_scaleR = (Rl)st->A_scale;
  const Medium3D& m = a.md;

  C v[E];
#pragma unroll
  for (int k = 0; k < E; ++k) v[k] = __ldg(src + W::out_index(lane, k));
  W::template bwd_like<+1>(v, S, tw, lane);          // time domain, natural layout
#pragma unroll
  for (int k = 0; k < E; ++k) v[k] = cscale(v[k], in_scale);

  bool any_w = false;
  if (m.plasma) {
    // the rates can be non-zero only where I >= I_zero (lut_eval returns 0 below):
    // a cheap test of the whole line first, the table and the rate stores only for
    // lines that pass it (the same rates and the same plasma_line decision)
    bool cand = m.ava != 0.0;
    // in the field precision against I_zero rounded down: I < izr implies I < I_zero
    const Rl izr = sizeof(Rl) == 8 ? (Rl)a.tb.lut.I_zero : (Rl)__double2float_rd(a.tb.lut.I_zero);
#pragma unroll
    for (int k = 0; k < E; ++k) {
      const C Ap = cscale(v[k], A_scaleR);
      cand |= !(Ap.x * Ap.x + Ap.y * Ap.y < izr);
    }
    if (__any_sync(0xffffffffu, cand)) {
#pragma unroll
      for (int k = 0; k < E; ++k) {
        const C Ap = cscale(v[k], A_scaleR);
        const float w = (float)lut_eval<Rl>(a.tb.lut, Ap.x * Ap.x + Ap.y * Ap.y);
        any_w |= (w != 0.f);
        sW[wpad(lane + 32 * k)] = w;
      }
    }
  }
  const bool plasma_line = m.plasma && (__any_sync(0xffffffffu, any_w) || m.ava != 0.0);
  C pv[E];
  if (plasma_line) {
    // time-ordered copy for the density scan: lane owns t in [lane E, lane E + E)
#pragma unroll
    for (int k = 0; k < E; ++k) S[tpad(lane + 32 * k)] = v[k];
    __syncwarp();
    const int t0 = lane * E;
    const AffineStep aff(m);
    bool ok = (m.ava == 0.0);
    double cmap = 1.0, dmap = 0.0;
    for (int i = 0; i < E; ++i) {
      const double w = (double)sW[wpad(t0 + i)];
      const double c = aff.e - w * aff.sf;
      ok &= (c >= 0.0);
      dmap = c * dmap + w * m.rho_nt * aff.sf;
      cmap = c * cmap;
    }
    double rho0;
    if (__all_sync(0xffffffffu, ok)) {
      double c = cmap, d = dmap;
#pragma unroll
      for (int off = 1; off < 32; off <<= 1) {
        const double cp = __shfl_up_sync(0xffffffffu, c, off);
        const double dp = __shfl_up_sync(0xffffffffu, d, off);
        if (lane >= off) { d = c * dp + d; c = c * cp; }
      }
      const double excl = __shfl_up_sync(0xffffffffu, d, 1);
      rho0 = lane == 0 ? 0.0 : excl;
    } else {
      if (lane == 0) {
        double rho = 0.0;
        for (int t = 0; t < NT; ++t) {
          if (t % E == 0) starts[t / E] = rho;
          const C Ap = cscale(S[tpad(t)], A_scaleR);
          const Rl I = Ap.x * Ap.x + Ap.y * Ap.y;
          const double w = (double)sW[wpad(t)];
          const double wa = (double)(float)(m.ava * (double)I);
          rho_step(rho, w, wa, m);
        }
      }
      __syncwarp();
      rho0 = starts[lane];
    }
    __syncwarp();
    double rho = rho0, ion = 0.0;
    for (int i = 0; i < E; ++i) {
      const int t = t0 + i;
      const C av = S[tpad(t)];
      const C Ap = cscale(av, A_scaleR);
      const Rl I = Ap.x * Ap.x + Ap.y * Ap.y;
      const double w = (double)sW[wpad(t)];
      const double rho_t = rho;
      ion = fmax(ion, rho_t);
      const double gen = m.ava == 0.0 ? rho_step0(rho, w, m, aff)
                                      : rho_step(rho, w, (double)(float)(m.ava * (double)I), m);
      // -(0 Ui) / x = -0 exactly: skip the division where nothing is generated
      const double loss = gen != 0.0 ? -(gen * m.Ui) / (2.0 * (double)I + 1e-30) : -0.0;
      const double cr = loss - m.sigma_half * rho_t;
      const double ci = -m.sigma_half * m.w0tc * rho_t;
      S[tpad(t)] = C{(Rl)cr * av.x - (Rl)ci * av.y, (Rl)cr * av.y + (Rl)ci * av.x};
    }
    if (a.mode == T_FROM_Z) {
      ion = warp_max(ion / m.rho_nt);
      if (lane == 0) atomic_max_nonneg(&st->ion_bits, ion);
    }
    __syncwarp();
#pragma unroll
    for (int k = 0; k < E; ++k) pv[k] = S[tpad(lane + 32 * k)];
    __syncwarp();
  }
  // Kerr term i (gk I + g4 I^2) a, in place
#pragma unroll
  for (int k = 0; k < E; ++k) {
    const C av = v[k];
    const C Ap = cscale(av, A_scaleR);
    const Rl I = Ap.x * Ap.x + Ap.y * Ap.y;
    Rl g = (Rl)m.gk * I;
    if (m.g4 != 0.0) g += (Rl)m.g4 * I * I;
    v[k] = C{-g * av.y, g * av.x};
  }
  W::template fwd_like<-1>(v, S, tw, lane);
  if (plasma_line) W::template fwd_like<-1>(pv, S, tw, lane);
#pragma unroll
  for (int k = 0; k < E; ++k) {
    const int wi = W::out_index(lane, k);
    const Rl sh = shm[wi];
    C o = cscale(v[k], sh);
    if (plasma_line) o = cadd(o, pv[k]);
    if (sh < (Rl)0) o = C{0, 0};
    dst[wi] = o;
  }
}

// initial transform: Z = fft_t(A0 / A_scale)
template <typename Rl, int NT, int WPB>
__global__ void __launch_bounds__(WPB * 32)
k_tload(TArgs a) {
  using C = typename CT<Rl>::T;
  constexpr int PAD = TCfg<NT>::PAD;
  constexpr int E = NT / 32;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* tw = reinterpret_cast<C*>(smem_raw);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  C* sK = tw + NT + warp * 2 * PAD;
  const C* gtw = reinterpret_cast<const C*>(a.tb.twt);
  for (int i = threadIdx.x; i < NT; i += WPB * 32) tw[i] = gtw[i];
  __syncthreads();
  const long long line = (long long)blockIdx.x * WPB + warp;
  if (line >= (long long)a.g.Nx * a.g.Ny) return;
  const C* src = reinterpret_cast<const C*>(a.in) + line * NT;
  const Rl inv = (Rl)a.st->inv_A_scale;
#pragma unroll
  for (int i = 0; i < E; ++i) sK[tpad(lane + 32 * i)] = cscale(src[lane + 32 * i], inv);
  __syncwarp();
  stockham<NT, 1, TCfg<NT>::FT, -1, 1, C>(sK, tw, lane, LineIdx(), WarpSync());
  C* dst = reinterpret_cast<C*>(a.b.z[0]) + line * NT;
#pragma unroll
  for (int i = 0; i < E; ++i) dst[lane + 32 * i] = sK[tpad(lane + 32 * i)];
}

// |A0| max reduction
template <typename Rl>
__global__ void k_absmax(const typename CT<Rl>::T* __restrict__ x, long long n, State3D* st) {
  double m = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const auto v = x[i];
    const double a = sqrt((double)v.x * v.x + (double)v.y * v.y);
    m = (a > m || a != a) ? a : m;
  }
  m = warp_max(m);
  if ((threadIdx.x & 31) == 0) atomic_max_nonneg(&st->red_norm, m);
}

__global__ void k_set_scale(State3D* st) {
  double s = __longlong_as_double((long long)st->red_norm);
  st->red_norm = 0ull;
  if (!(s >= 1e-30)) s = 1.0;   // solver_3d.py:166-168
  st->A_scale = s;
  st->inv_A_scale = 1.0 / s;
  st->ion_bits = 0ull;
  st->zidx = 0;
  st->fresh = 1;
  st->done = 0;
  st->status = 0;
}

// error of the attempt (solver_3d.py:151-153)
__global__ void k_err(State3D* st) {
  if (st->done) return;
  const double num = __longlong_as_double((long long)st->red_diff);
  const double den = __longlong_as_double((long long)st->red_norm);
  st->red_diff = 0ull;
  st->red_norm = 0ull;
  st->err_num = num;
  st->err_den = den;
  st->err = num / (den + 1e-20);
}

// adaptive controller (solver_3d.py:182-208), plus the finite-value check the
// reference lacks (a NaN error there never terminates)
__global__ void k_controller(State3D* st) {
  if (st->done) return;
  double err = st->err;
  double h = st->h;
  st->attempts += 1;
  const double tol = st->tol, min_step = st->min_step, max_step = st->max_step;
  if (!isfinite(h) || (!isfinite(err) && h <= min_step * 1.01)) {
    st->status |= UPPE_STATUS_NONFINITE;
    st->done = 1;
    st->last_accept = 0;
    return;
  }
  if (!isfinite(err)) {
    // the attempt overflowed (the accepted state is untouched): reject it and
    // retry with a tenth of the step; at min_step the run stops (above)
    st->status |= UPPE_STATUS_RETRIED;
    st->fresh = 0;
    st->last_accept = 0;
    h = fmax(h * 0.1, min_step);
  } else if (err < tol || h <= min_step * 1.01) {
    if (st->hlog && st->accepted < st->hlog_cap) st->hlog[st->accepted] = h;
    st->fail_count = (h <= min_step * 1.01 && err > tol) ? st->fail_count + 1 : 0;
    if (st->fail_count > 0) st->status |= UPPE_STATUS_MIN_STEP;
    st->z += h;
    st->zidx ^= 1;
    st->fresh = 1;
    st->accepted += 1;
    st->last_accept = 1;
    err = fmax(err, 1e-30);
    double factor = 0.95 * pow(tol / err, 0.2);
    if (st->fail_count > 0) factor = fmin(factor, 1.2);
    h = fmin(h * fmin(factor, 2.0), max_step);
  } else {
    st->fresh = 0;
    st->last_accept = 0;
    err = fmax(err, 1e-30);
    const double factor = 0.95 * pow(tol / err, 0.2);
    h = fmax(h * factor, min_step);
  }
  if (!(st->z < st->L)) {
    st->done = 1;
  } else {
    const double dist = st->L - st->z;
    if (h > dist) {
      h = dist;
      if (h < 1e-15) st->done = 1;
    }
  }
  if (st->max_attempts > 0 && st->attempts >= st->max_attempts && !st->done) {
    st->status |= UPPE_STATUS_MAX_ATTEMPTS;
    st->done = 1;
  }
  st->h = h;
}

// the tuner's state: zeroed fields at unit scale, fresh (every pass of an attempt runs)
__global__ void k_set_scale_one(State3D* st) {
  st->A_scale = 1.0;
  st->inv_A_scale = 1.0;
  st->ion_bits = 0ull;
  st->zidx = 0;
  st->fresh = 1;
  st->done = 0;
}

__global__ void k_set_h(State3D* st, double h) {
  st->h = h;
  st->done = 0;
}

__global__ void k_commit(State3D* st, int accept) {
  if (accept) {
    st->z += st->h;
    st->zidx ^= 1;
    st->fresh = 1;
    st->accepted += 1;
  } else {
    st->fresh = 0;
  }
  st->attempts += 1;
}

__global__ void k_begin(State3D* st, double L, double tol, double max_step, double min_step,
                        long long max_attempts) {
  st->z = 0.0;
  st->L = L;
  st->tol = tol;
  st->max_step = max_step;
  st->min_step = min_step;
  double h = fmin(max_step, L / 1000.0);   // solver_3d.py:173
  st->attempts = 0;
  st->accepted = 0;
  st->max_attempts = max_attempts;
  st->fail_count = 0;
  st->status = 0;
  st->done = 0;
  st->red_norm = 0ull;
  st->red_diff = 0ull;
  if (!(0.0 < L)) st->done = 1;
  else if (h > L) { h = L; if (h < 1e-15) st->done = 1; }
  st->h = h;
}

// spectrum output: fftshift_t(Z * A_scale)   (solver_3d.py:215-222)
template <typename Rl>
__global__ void k_spectrum(const typename CT<Rl>::T* __restrict__ z, typename CT<Rl>::T* __restrict__ out,
                           long long nlines, int Nt, const State3D* st) {
  const Rl s = (Rl)st->A_scale;
  const long long n = nlines * Nt;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const long long line = i / Nt;
    const int w = (int)(i % Nt);
    const int ws = (w + Nt / 2) % Nt;   // fftshift destination
    out[line * Nt + ws] = cscale(z[i], s);
  }
}

// time-domain field A_t = ifft_t(Z) * A_scale, for chaining segments
template <typename Rl, int NT, int WPB>
__global__ void __launch_bounds__(WPB * 32)
k_tstore(TArgs a) {
  using C = typename CT<Rl>::T;
  constexpr int PAD = TCfg<NT>::PAD;
  constexpr int E = NT / 32;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* tw = reinterpret_cast<C*>(smem_raw);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  C* sK = tw + NT + warp * 2 * PAD;
  const C* gtw = reinterpret_cast<const C*>(a.tb.twt);
  for (int i = threadIdx.x; i < NT; i += WPB * 32) tw[i] = gtw[i];
  __syncthreads();
  const long long line = (long long)blockIdx.x * WPB + warp;
  if (line >= (long long)a.g.Nx * a.g.Ny) return;
  const C* src = reinterpret_cast<const C*>(a.b.z[a.st->zidx]) + line * NT;
#pragma unroll
  for (int i = 0; i < E; ++i) sK[tpad(lane + 32 * i)] = src[lane + 32 * i];
  __syncwarp();
  stockham<NT, 1, TCfg<NT>::FT, +1, 1, C>(sK, tw, lane, LineIdx(), WarpSync());
  const Rl s = (Rl)(a.st->A_scale / NT);
  C* dst = reinterpret_cast<C*>(a.out) + line * NT;
#pragma unroll
  for (int i = 0; i < E; ++i) dst[lane + 32 * i] = cscale(sK[tpad(lane + 32 * i)], s);
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
template <int NT, typename Rl> struct TLaunch {
  static constexpr int WPB = (2 * TCfg<NT>::PAD * (int)sizeof(typename CT<Rl>::T) * 8 <= 72 * 1024) ? 8
                           : (2 * TCfg<NT>::PAD * (int)sizeof(typename CT<Rl>::T) * 4 <= 72 * 1024) ? 4
                           : (2 * TCfg<NT>::PAD * (int)sizeof(typename CT<Rl>::T) * 2 <= 110 * 1024) ? 2 : 1;
  static size_t smem() {
    return (size_t)(NT + WPB * 2 * TCfg<NT>::PAD) * sizeof(typename CT<Rl>::T);
  }
};

}  // namespace uppe

using namespace uppe;

struct uppe3d_plan {
  uppe3d_desc d;
  Geom g;
  int dbl;
  size_t csz;
  State3D* st;          // device
  State3D* st_host;     // pinned mirror
  Tables3D tb;
  Medium3D md;
  Bufs3D b;
  std::vector<void*> allocs;
  cudaGraphExec_t g_attempt = nullptr, g_step = nullptr;
  const double* wabs = nullptr;   // omega + omega0 per omega bin (photon number)
  void* save_u[3] = {nullptr, nullptr, nullptr};   // adjoint recompute: u2, u3, u4
  double pass_scale = 1.0;                          // plain y passes
  double* diag_buf = nullptr;     // per-block partial sums + 3 results
  cudaStream_t cap_stream = nullptr;
  bool ytma = false;              // TMA-fed y passes possible (complex64, 64 <= Ny <= 256)
  YMaps ymaps;                    // boxes of kW omega columns
  YMaps ymaps8;                   // boxes of 8 omega columns
  int nsm = 148;
  // launch configuration picked per shape by the tuner (uppe3d_tuning): every
  // candidate computes the same bits, only the time differs
  int y_tma = 1;                  // y passes on k_ypass_tma (1), k_ypass_rq (2), k_ypass_ring (3) or k_space (0)
  int y_ctas = 2;                 // k_ypass_tma CTAs per SM (1..6; k_ypass_rq: 2 or 3, fixed by LATE)
  int y_late = 0;                 // the y kernel loads the stage operands where used (1)
  int y_kw = kW;                  // k_ypass_tma omega columns per tile (16 or 8)
  int t_wpb = 8;                  // warps (t-lines) per block of k_tpass_w (4 or 8)
  float tune_ms[UPPE3D_TUNE_SLOTS] = {0};   // measured per-attempt pass times of the candidates
  int tuned = 0;                  // 1 timed here, 2 from the process cache, 0 defaults
};

#define UPPE_CK(x)                                                                 \
  do {                                                                             \
    cudaError_t e_ = (x);                                                          \
    if (e_ != cudaSuccess) {                                                       \
      snprintf(g_uppe_err, sizeof(g_uppe_err), "%s:%d %s: %s", __FILE__, __LINE__, \
               #x, cudaGetErrorString(e_));                                        \
      return UPPE_ERR_CUDA;                                                        \
    }                                                                              \
  } while (0)

char g_uppe_err[512];

extern "C" const char* uppe_last_error(void) { return g_uppe_err; }

static int is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

static int dev_upload(uppe3d_plan* p, void** dst, const void* src, size_t bytes) {
  UPPE_CK(cudaMalloc(dst, bytes));
  p->allocs.push_back(*dst);
  UPPE_CK(cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice));
  return 0;
}

template <typename Rl> static std::vector<unsigned char> twiddles(int N) {
  using C = typename CT<Rl>::T;
  std::vector<unsigned char> out(sizeof(C) * N);
  C* c = reinterpret_cast<C*>(out.data());
  for (int m = 0; m < N; ++m) {
    // exp(-2 pi i m / N), evaluated in extended precision and rounded once
    const long double ang = -2.0L * 3.141592653589793238462643383279502884L * (long double)m / (long double)N;
    c[m].x = (Rl)(double)cosl(ang);
    c[m].y = (Rl)(double)sinl(ang);
  }
  return out;
}

// ---- template dispatch -----------------------------------------------------
template <int N> struct SqRoot {
  static constexpr int v = N == 16 ? 4 : N == 64 ? 8 : N == 256 ? 16 : 0;
};

template <typename Rl, int N>
static void launch_space_n(const SpaceArgs& a, long long nblocks, size_t smem, cudaStream_t s) {
  constexpr int R = SqRoot<N>::v;
  if constexpr (R > 0) {
    if (a.mode <= XFWD_Z) {   // x passes of square sizes: register four-step kernel
      using C = typename CT<Rl>::T;
      const size_t sm = sizeof(C) * (size_t)(N + N * kW);
      const unsigned nb = (unsigned)nblocks;
      if (sizeof(Rl) == 4 && N == 256 && a.g.Nt == 512 && a.g.Ny == 256) {   // 256 x 256 x 512 complex64
        switch (a.mode) {
          case XINV: k_xpass_sq<Rl, R, XINV, 512><<<nb, kW * R, sm, s>>>(a); break;
          case XINV_Z: k_xpass_sq<Rl, R, XINV_Z, 512><<<nb, kW * R, sm, s>>>(a); break;
          case XFWD: k_xpass_sq<Rl, R, XFWD, 512><<<nb, kW * R, sm, s>>>(a); break;
          default: k_xpass_sq<Rl, R, XFWD_Z, 512><<<nb, kW * R, sm, s>>>(a); break;
        }
        return;
      }
      switch (a.mode) {
        case XINV: k_xpass_sq<Rl, R, XINV><<<nb, kW * R, sm, s>>>(a); break;
        case XINV_Z: k_xpass_sq<Rl, R, XINV_Z><<<nb, kW * R, sm, s>>>(a); break;
        case XFWD: k_xpass_sq<Rl, R, XFWD><<<nb, kW * R, sm, s>>>(a); break;
        default: k_xpass_sq<Rl, R, XFWD_Z><<<nb, kW * R, sm, s>>>(a); break;
      }
      return;
    }
  }
  k_space<Rl, N><<<(unsigned)nblocks, SpaceCfg<N>::NTHR, smem, s>>>(a);
}

// the y passes of the attempt that k_ypass_tma and k_ypass_rq serve (input tmp[1])
static bool fused_ypass(const uppe3d_plan* p, int mode, const void* in) {
  return mode == YMID1R ||
         ((mode == YMID1 || mode == YMID2 || mode == YMID3 || mode == YMID4 || mode == YFWD5) && in == p->b.tmp[1]);
}
static bool use_ytma(const uppe3d_plan* p, int mode, const void* in) {
  return p->ytma && p->y_tma == 1 && fused_ypass(p, mode, in);
}
// k_ypass_rq: complex64, Ny = 256, and only where k_ypass_tma is available too
// (the two give the same bits; the plain tile kernel does not)
static bool yrq_ok(const uppe3d_plan* p) { return p->ytma && !p->dbl && p->g.Ny == 256; }
static bool use_yrq(const uppe3d_plan* p, int mode, const void* in) {
  return p->y_tma == 2 && yrq_ok(p) && fused_ypass(p, mode, in);
}
static bool use_ytq(const uppe3d_plan* p, int mode, const void* in) {
  return p->y_tma == 3 && yrq_ok(p) && fused_ypass(p, mode, in);
}

static void launch_ytq(const uppe3d_plan* p, const SpaceArgs& a, cudaStream_t s) {
  const long long total = (long long)p->g.Nx * (p->g.Nt / kW);
  const dim3 g((unsigned)(total < p->nsm ? total : p->nsm));
  constexpr unsigned T = kW * 16;
  const YMaps& mp = p->ymaps;
  switch (a.mode) {
    case YMID1: k_ypass_ring<YMID1><<<g, T, YRing<YMID1>::bytes(), s>>>(a, mp); break;
    case YMID1R: k_ypass_ring<YMID1R><<<g, T, YRing<YMID1R>::bytes(), s>>>(a, mp); break;
    case YMID2: k_ypass_ring<YMID2><<<g, T, YRing<YMID2>::bytes(), s>>>(a, mp); break;
    case YMID3: k_ypass_ring<YMID3><<<g, T, YRing<YMID3>::bytes(), s>>>(a, mp); break;
    case YMID4: k_ypass_ring<YMID4><<<g, T, YRing<YMID4>::bytes(), s>>>(a, mp); break;
    default: k_ypass_ring<YFWD5><<<g, T, YRing<YFWD5>::bytes(), s>>>(a, mp); break;
  }
}

template <int MODE> static cudaError_t set_yring_attr_m() {
  return cudaFuncSetAttribute(k_ypass_ring<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)YRing<MODE>::bytes());
}
static cudaError_t set_ytq_attr() {
  cudaError_t e = set_yring_attr_m<YMID1>();
  if (e == cudaSuccess) e = set_yring_attr_m<YMID1R>();
  if (e == cudaSuccess) e = set_yring_attr_m<YMID2>();
  if (e == cudaSuccess) e = set_yring_attr_m<YMID3>();
  if (e == cudaSuccess) e = set_yring_attr_m<YMID4>();
  if (e == cudaSuccess) e = set_yring_attr_m<YFWD5>();
  return e;
}

template <int LATE, int KW>
static void launch_yrq_l(const SpaceArgs& a, unsigned nblocks, cudaStream_t s) {
  constexpr unsigned T = KW * 16;
  constexpr size_t sm = yrq_smem<KW>();
  if (LATE == 0 && KW == kW && a.g.Nt == 512) {   // the tuned configuration at Nt = 512
    switch (a.mode) {
      case YMID1: k_ypass_rq<YMID1, 0, kW, 512><<<nblocks, T, sm, s>>>(a); break;
      case YMID1R: k_ypass_rq<YMID1R, 0, kW, 512><<<nblocks, T, sm, s>>>(a); break;
      case YMID2: k_ypass_rq<YMID2, 0, kW, 512><<<nblocks, T, sm, s>>>(a); break;
      case YMID3: k_ypass_rq<YMID3, 0, kW, 512><<<nblocks, T, sm, s>>>(a); break;
      case YMID4: k_ypass_rq<YMID4, 0, kW, 512><<<nblocks, T, sm, s>>>(a); break;
      default: k_ypass_rq<YFWD5, 0, kW, 512><<<nblocks, T, sm, s>>>(a); break;
    }
    return;
  }
  switch (a.mode) {
    case YMID1: k_ypass_rq<YMID1, LATE, KW><<<nblocks, T, sm, s>>>(a); break;
    case YMID1R: k_ypass_rq<YMID1R, LATE, KW><<<nblocks, T, sm, s>>>(a); break;
    case YMID2: k_ypass_rq<YMID2, LATE, KW><<<nblocks, T, sm, s>>>(a); break;
    case YMID3: k_ypass_rq<YMID3, LATE, KW><<<nblocks, T, sm, s>>>(a); break;
    case YMID4: k_ypass_rq<YMID4, LATE, KW><<<nblocks, T, sm, s>>>(a); break;
    default: k_ypass_rq<YFWD5, LATE, KW><<<nblocks, T, sm, s>>>(a); break;
  }
}

template <int N, int LATE, int KW>
static void launch_ytma_nl(const uppe3d_plan* p, const SpaceArgs& a, cudaStream_t s) {
  // persistent CTAs: never more per SM than the shared memory lets be resident
  const size_t sm = ytma_smem<N, KW>(a.mode);
  int per_sm = p->y_ctas;
  while (per_sm > 1 && sm * per_sm > 220 * 1024) --per_sm;
  const dim3 g((unsigned)(per_sm * p->nsm));
  const YMaps& mp = KW == kW ? p->ymaps : p->ymaps8;
  constexpr int T = YTmaCfg<KW, LATE>::NTHR;
  switch (a.mode) {
    case YMID1: k_ypass_tma<N, YMID1, LATE, KW><<<g, T, sm, s>>>(a, mp); break;
    case YMID1R: k_ypass_tma<N, YMID1R, LATE, KW><<<g, T, sm, s>>>(a, mp); break;
    case YMID2: k_ypass_tma<N, YMID2, LATE, KW><<<g, T, sm, s>>>(a, mp); break;
    case YMID3: k_ypass_tma<N, YMID3, LATE, KW><<<g, T, sm, s>>>(a, mp); break;
    case YMID4: k_ypass_tma<N, YMID4, LATE, KW><<<g, T, sm, s>>>(a, mp); break;
    default: k_ypass_tma<N, YFWD5, LATE, KW><<<g, T, sm, s>>>(a, mp); break;
  }
}

template <int N>
static void launch_ytma_n(const uppe3d_plan* p, const SpaceArgs& a, cudaStream_t s) {
  if (p->y_kw == 8) {
    if (p->y_late) launch_ytma_nl<N, 1, 8>(p, a, s);
    else launch_ytma_nl<N, 0, 8>(p, a, s);
  } else {
    if (p->y_late) launch_ytma_nl<N, 1, kW>(p, a, s);
    else launch_ytma_nl<N, 0, kW>(p, a, s);
  }
}

template <int N, int LATE, int KW>
static cudaError_t set_ytma_attr_l() {
  const int sm = (int)ytma_smem<N, KW>(YMID2);
  cudaError_t e = cudaFuncSetAttribute(k_ypass_tma<N, YMID1, LATE, KW>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)ytma_smem<N, KW>(YMID1));
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_ypass_tma<N, YMID1R, LATE, KW>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_ypass_tma<N, YMID2, LATE, KW>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_ypass_tma<N, YMID3, LATE, KW>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_ypass_tma<N, YMID4, LATE, KW>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_ypass_tma<N, YFWD5, LATE, KW>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
  return e;
}

template <int N>
static cudaError_t set_ytma_attr() {
  cudaError_t e = set_ytma_attr_l<N, 0, kW>();
  if (e == cudaSuccess) e = set_ytma_attr_l<N, 1, kW>();
  if (e == cudaSuccess) e = set_ytma_attr_l<N, 0, 8>();
  if (e == cudaSuccess) e = set_ytma_attr_l<N, 1, 8>();
  return e;
}

template <typename Rl>
static int launch_space(uppe3d_plan* p, int mode, const void* in, void* out, cudaStream_t s) {
  using C = typename CT<Rl>::T;
  SpaceArgs a;
  a.st = p->st; a.tb = p->tb; a.b = p->b; a.g = p->g; a.in = in; a.out = out; a.mode = mode;
  a.save_u = (mode == YMID1 || mode == YMID1R) ? p->save_u[0]
           : mode == YMID2 ? p->save_u[1] : mode == YMID3 ? p->save_u[2] : nullptr;
  a.scale = p->pass_scale;
  if (sizeof(Rl) == 4 && use_ytq(p, mode, in)) {
    launch_ytq(p, a, s);
    return 0;
  }
  if (sizeof(Rl) == 4 && use_yrq(p, mode, in)) {
    const unsigned nb = (unsigned)((long long)p->g.Nx * (p->g.Nt / p->y_kw));
    if (p->y_kw == 8) {
      if (p->y_late) launch_yrq_l<1, 8>(a, nb, s);
      else launch_yrq_l<0, 8>(a, nb, s);
    } else {
      if (p->y_late) launch_yrq_l<1, kW>(a, nb, s);
      else launch_yrq_l<0, kW>(a, nb, s);
    }
    return 0;
  }
  if (sizeof(Rl) == 4 && use_ytma(p, mode, in)) {
    switch (p->g.Ny) {
      case 64: launch_ytma_n<64>(p, a, s); break;
      case 128: launch_ytma_n<128>(p, a, s); break;
      case 256: launch_ytma_n<256>(p, a, s); break;
      default: return UPPE_ERR_SIZE;
    }
    return 0;
  }
  const bool xpass = mode <= XFWD_Z;
  const int N = xpass ? p->g.Nx : p->g.Ny;
  const long long nouter = xpass ? p->g.Ny : p->g.Nx;
  const long long nblocks = nouter * (p->g.Nt / kW);
  // the second tile is only used by the passes that transform two fields
  const int ntiles = (mode == YMID1 || mode == XFWD_Z) ? 2 : 1;
  const size_t smem = sizeof(C) * (size_t)(N + ntiles * N * kW);
  switch (N) {
#define UPPE_SP(n) case n: launch_space_n<Rl, n>(a, nblocks, smem, s); break;
    UPPE_SP(16) UPPE_SP(32) UPPE_SP(64) UPPE_SP(128) UPPE_SP(256) UPPE_SP(512)
#undef UPPE_SP
    default: return UPPE_ERR_SIZE;
  }
  return 0;
}

template <int NT, typename Rl> struct TWarp {
  static constexpr bool use = NT == 512 || (NT == 1024 && sizeof(Rl) == 4);
  static constexpr int E = NT / 32;
  static constexpr int BUF = WarpFFT<(E < 16 ? 16 : E)>::SBUF > TCfg<NT>::PAD
                                 ? WarpFFT<(E < 16 ? 16 : E)>::SBUF : TCfg<NT>::PAD;
  static size_t smem(int WPB) {
    return (size_t)(NT + WPB * BUF) * sizeof(typename CT<Rl>::T) + (size_t)WPB * 32 * sizeof(double) +
           (size_t)WPB * (NT + NT / 32) * sizeof(float) + (size_t)NT * sizeof(Rl);
  }
};

template <typename Rl, int NT, int KIND>
static void launch_t_n(const TArgs& a, long long nlines, int wpb, cudaStream_t s) {
  if constexpr (KIND == 0 && TWarp<NT, Rl>::use) {
    const unsigned nb = (unsigned)((nlines + wpb - 1) / wpb);
    const size_t sm = TWarp<NT, Rl>::smem(wpb);
    if (wpb == 4) k_tpass_w<Rl, NT / 32, 4><<<nb, 4 * 32, sm, s>>>(a);
    else k_tpass_w<Rl, NT / 32, 8><<<nb, 8 * 32, sm, s>>>(a);
    return;
  }
  constexpr int WPB = TLaunch<NT, Rl>::WPB;
  const unsigned nb = (unsigned)((nlines + WPB - 1) / WPB);
  const size_t smem = TLaunch<NT, Rl>::smem();
  if (KIND == 0) k_tpass<Rl, NT, WPB><<<nb, WPB * 32, smem, s>>>(a);
  else if (KIND == 1) k_tload<Rl, NT, WPB><<<nb, WPB * 32, smem, s>>>(a);
  else k_tstore<Rl, NT, WPB><<<nb, WPB * 32, smem, s>>>(a);
}

template <typename Rl, int KIND>
static int launch_t(uppe3d_plan* p, int mode, const void* in, void* out, cudaStream_t s, int diag = 0) {
  TArgs a;
  a.diag = diag;
  a.st = p->st; a.tb = p->tb; a.md = p->md; a.b = p->b; a.g = p->g;
  a.in = in; a.out = out; a.mode = mode;
  const long long nl = (long long)p->g.Nx * p->g.Ny;
  switch (p->g.Nt) {
#define UPPE_T(n) case n: launch_t_n<Rl, n, KIND>(a, nl, p->t_wpb, s); break;
    UPPE_T(32) UPPE_T(64) UPPE_T(128) UPPE_T(256) UPPE_T(512) UPPE_T(1024) UPPE_T(2048)
#undef UPPE_T
    default: return UPPE_ERR_SIZE;
  }
  return 0;
}

template <typename Rl, int N>
static cudaError_t set_space_attr() {
  constexpr int R = SqRoot<N>::v;
  if constexpr (R > 0) {
    const int sm = (int)(sizeof(typename CT<Rl>::T) * (N + N * kW));
    cudaError_t e = cudaFuncSetAttribute(k_xpass_sq<Rl, R, XINV>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_xpass_sq<Rl, R, XINV_Z>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_xpass_sq<Rl, R, XFWD>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_xpass_sq<Rl, R, XFWD_Z>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    if constexpr (sizeof(Rl) == 4 && N == 256) {
      if (e == cudaSuccess) e = cudaFuncSetAttribute(k_xpass_sq<Rl, R, XINV, 512>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
      if (e == cudaSuccess) e = cudaFuncSetAttribute(k_xpass_sq<Rl, R, XINV_Z, 512>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
      if (e == cudaSuccess) e = cudaFuncSetAttribute(k_xpass_sq<Rl, R, XFWD, 512>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
      if (e == cudaSuccess) e = cudaFuncSetAttribute(k_xpass_sq<Rl, R, XFWD_Z, 512>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    }
    if (e != cudaSuccess) return e;
  }
  const int smem = (int)(sizeof(typename CT<Rl>::T) * (N + 2 * N * kW));
  return cudaFuncSetAttribute(k_space<Rl, N>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
}
template <typename Rl, int NT>
static cudaError_t set_t_attr() {
  constexpr int WPB = TLaunch<NT, Rl>::WPB;
  const int smem = (int)TLaunch<NT, Rl>::smem();
  cudaError_t e = cudaFuncSetAttribute(k_tpass<Rl, NT, WPB>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e != cudaSuccess) return e;
  if constexpr (TWarp<NT, Rl>::use) {
    e = cudaFuncSetAttribute(k_tpass_w<Rl, NT / 32, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)TWarp<NT, Rl>::smem(4));
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(k_tpass_w<Rl, NT / 32, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)TWarp<NT, Rl>::smem(8));
    if (e != cudaSuccess) return e;
  }
  e = cudaFuncSetAttribute(k_tload<Rl, NT, WPB>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(k_tstore<Rl, NT, WPB>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
}
template <typename Rl>
static int set_attrs(const Geom& g) {
  cudaError_t e = cudaSuccess;
  for (int N : {g.Nx, g.Ny}) {
    switch (N) {
      case 16: e = set_space_attr<Rl, 16>(); break;
      case 32: e = set_space_attr<Rl, 32>(); break;
      case 64: e = set_space_attr<Rl, 64>(); break;
      case 128: e = set_space_attr<Rl, 128>(); break;
      case 256: e = set_space_attr<Rl, 256>(); break;
      case 512: e = set_space_attr<Rl, 512>(); break;
      default: return UPPE_ERR_SIZE;
    }
    if (e != cudaSuccess) break;
  }
  if (e == cudaSuccess) {
    switch (g.Nt) {
      case 32: e = set_t_attr<Rl, 32>(); break;
      case 64: e = set_t_attr<Rl, 64>(); break;
      case 128: e = set_t_attr<Rl, 128>(); break;
      case 256: e = set_t_attr<Rl, 256>(); break;
      case 512: e = set_t_attr<Rl, 512>(); break;
      case 1024: e = set_t_attr<Rl, 1024>(); break;
      case 2048: e = set_t_attr<Rl, 2048>(); break;
      default: return UPPE_ERR_SIZE;
    }
  }
  UPPE_CK(e);
  return 0;
}

// Launch recorder: in capture mode it only launches; in profile mode it brackets
// every launch with CUDA events on the launching stream and records the pass
// kind and the algorithmic bytes the launch moves.
struct Recorder {
  cudaStream_t s;
  bool prof = false;
  int fresh = 1;                 // known device state (profile mode only)
  double fbytes = 0.0;           // bytes of one field
  std::vector<cudaEvent_t> ev;
  std::vector<int> kind;
  std::vector<double> bytes;
  template <typename F> int operator()(int k, double nfields, bool active, F&& launch) {
    cudaEvent_t a = nullptr, b = nullptr;
    if (prof) { cudaEventCreate(&a); cudaEventCreate(&b); cudaEventRecord(a, s); }
    const int rc = launch();
    if (prof) {
      cudaEventRecord(b, s);
      ev.push_back(a); ev.push_back(b);
      kind.push_back(k);
      bytes.push_back(active ? nfields * fbytes : 0.0);
    }
    return rc;
  }
};

enum { KIND_T = 0, KIND_X = 1, KIND_Y = 2, KIND_SMALL = 3, KIND_YT = 4, KIND_YR = 5, KIND_YQ = 6 };

// the fixed pass sequence of one attempt (see the file header); the numbers are
// the fields each launch reads + writes (algorithmic bytes / field bytes)
template <typename Rl>
static int enqueue_attempt(uppe3d_plan* p, Recorder& r) {
  int rc = 0;
  cudaStream_t s = r.s;
  void* const* t = p->b.tmp;
  const bool f = r.fresh != 0;
  // the fused y passes: k_ypass_rq, k_ypass_tma or the plain tile kernel
  const int KY = (p->y_tma == 3 && yrq_ok(p)) ? KIND_YQ : (p->y_tma == 2 && yrq_ok(p)) ? KIND_YR
               : (p->ytma && p->y_tma == 1) ? KIND_YT : KIND_Y;
  // eval 1 (skipped on device unless the state is fresh)
  rc |= r(KIND_T, 2, f, [&] { return launch_t<Rl, 0>(p, T_FROM_Z, nullptr, t[0], s); });
  rc |= r(KIND_X, 4, f, [&] { return launch_space<Rl>(p, XFWD_Z, t[0], t[1], s); });
  rc |= r(KY, 6, f, [&] { return launch_space<Rl>(p, YMID1, t[1], t[0], s); });
  rc |= r(KY, 4, !f, [&] { return launch_space<Rl>(p, YMID1R, nullptr, t[0], s); });
  // eval 2..4
  const int mids[3] = {YMID2, YMID3, YMID4};
  const double midb[3] = {5, 5, 4};
  for (int k = 0; k < 3; ++k) {
    rc |= r(KIND_X, 2, true, [&] { return launch_space<Rl>(p, XINV, t[0], t[1], s); });
    rc |= r(KIND_T, 2, true, [&] { return launch_t<Rl, 0>(p, T_GENERAL, t[1], t[2], s); });
    rc |= r(KIND_X, 2, true, [&] { return launch_space<Rl>(p, XFWD, t[2], t[1], s); });
    rc |= r(KY, midb[k], true, [&] { return launch_space<Rl>(p, mids[k], t[1], t[0], s); });
  }
  // eval 5 (+ candidate state) and the error reduction
  rc |= r(KIND_X, 3, true, [&] { return launch_space<Rl>(p, XINV_Z, t[0], t[1], s); });
  rc |= r(KIND_T, 2, true, [&] { return launch_t<Rl, 0>(p, T_GENERAL, t[1], t[2], s); });
  rc |= r(KIND_X, 2, true, [&] { return launch_space<Rl>(p, XFWD, t[2], t[1], s); });
  rc |= r(KY, sizeof(Rl) == 8 ? 3 : 2, true,
          [&] { return launch_space<Rl>(p, YFWD5, t[1], nullptr, s); });
  rc |= r(KIND_SMALL, 0, true, [&] { k_err<<<1, 1, 0, s>>>(p->st); return 0; });
  return rc;
}

// (omega, ky, kx) tensor maps of the y passes' input field and of A for
// k_ypass_tma: 8-byte elements, box kW x Ny x 1 (128-byte rows; omega
// coordinates are multiples of kW, so every copy starts 16-byte aligned).
// Without the driver entry point the y passes stay on k_space.
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static int setup_ytma(uppe3d_plan* p) {
  void* fn = nullptr;
  cudaDriverEntryPointQueryResult q;
  if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
      q != cudaDriverEntryPointSuccess || !fn) {
    cudaGetLastError();
    return 0;
  }
  EncodeTiledFn encode = reinterpret_cast<EncodeTiledFn>(fn);
  const cuuint64_t dims[3] = {(cuuint64_t)p->g.Nt, (cuuint64_t)p->g.Ny, (cuuint64_t)p->g.Nx};
  const cuuint64_t strides[2] = {(cuuint64_t)p->g.Nt * 8, (cuuint64_t)p->g.Ny * p->g.Nt * 8};
  const cuuint32_t es[3] = {1, 1, 1};
  void* bufs[6] = {p->b.tmp[1], p->b.acur, p->b.tmp[2], p->b.tsum, p->b.k1, p->b.a4p};
  for (int set = 0; set < 2; ++set) {       // boxes of kW and of 8 omega columns (64-byte rows)
    YMaps& ym = set == 0 ? p->ymaps : p->ymaps8;
    const cuuint32_t box[3] = {(cuuint32_t)(set == 0 ? kW : 8), (cuuint32_t)p->g.Ny, 1};
    CUtensorMap* maps[6] = {&ym.in, &ym.acur, &ym.z2, &ym.tsum, &ym.k1, &ym.a4p};
    for (int i = 0; i < 6; ++i) {
      if (reinterpret_cast<uintptr_t>(bufs[i]) % 16) return 0;
      if (encode(maps[i], CU_TENSOR_MAP_DATA_TYPE_UINT64, 3, bufs[i], dims, strides, box, es,
                 CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                 CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return 0;
    }
  }
  int dev = 0;
  UPPE_CK(cudaGetDevice(&dev));
  UPPE_CK(cudaDeviceGetAttribute(&p->nsm, cudaDevAttrMultiProcessorCount, dev));
  switch (p->g.Ny) {
    case 64: UPPE_CK(set_ytma_attr<64>()); break;
    case 128: UPPE_CK(set_ytma_attr<128>()); break;
    case 256: UPPE_CK(set_ytma_attr<256>()); UPPE_CK(set_ytq_attr()); break;
    default: return 0;
  }
  p->ytma = true;
  return 0;
}

// ---------------------------------------------------------------------------
// Per-shape tuner.  Candidates: the y passes on k_ypass_tma with tiles of 16 omega
// columns (operands loaded early with one or two CTAs per SM, or late with two or
// three) or of 8 columns (early with four, late with six), and k_tpass_w with
// four or eight t-lines per block (same per-line code).  Every candidate computes
// the same bits, so the choice changes only the time.  Each candidate runs whole
// attempts launch by launch on zeroed fields with CUDA events around each launch;
// the y and t choices are independent (different launches), so they are timed
// separately.  The tile width changes which columns share a CTA, not the
// arithmetic of a column.  Choices are kept per (Nx, Ny, Nt, precision, SM count) for the
// life of the process; UPPE_TUNE=0 in the environment keeps the defaults.
// ---------------------------------------------------------------------------
struct TuneKey {
  int Nx, Ny, Nt, dbl, nsm;
  bool operator<(const TuneKey& o) const {
    return std::tie(Nx, Ny, Nt, dbl, nsm) < std::tie(o.Nx, o.Ny, o.Nt, o.dbl, o.nsm);
  }
};
struct TuneVal { int y_tma, y_ctas, y_late, y_kw, t_wpb; float ms[UPPE3D_TUNE_SLOTS]; };
static std::map<TuneKey, TuneVal> g_tune_cache;
static std::mutex g_tune_mu;

template <typename Rl>
// the fastest of `reps` attempts (y and t pass times separately), after one
// untimed attempt that takes the first launches of the candidate's kernels (module
// loading) out of the timing
static int time_attempts(uppe3d_plan* p, cudaStream_t s, int reps, float* y_ms, float* t_ms) {
  *y_ms = 3.4e38f;
  *t_ms = 3.4e38f;
  for (int r = -1; r < reps; ++r) {
    k_set_h<<<1, 1, 0, s>>>(p->st, 1e-3);
    Recorder rec;
    rec.s = s;
    rec.prof = true;
    rec.fresh = 1;
    rec.fbytes = (double)p->csz * (double)p->g.npts;
    int rc = enqueue_attempt<Rl>(p, rec);
    UPPE_CK(cudaStreamSynchronize(s));
    float ya = 0.f, ta = 0.f;
    for (size_t i = 0; i < rec.kind.size(); ++i) {
      float ms = 0.f;
      cudaEventElapsedTime(&ms, rec.ev[2 * i], rec.ev[2 * i + 1]);
      if (rec.kind[i] == KIND_Y || rec.kind[i] == KIND_YT || rec.kind[i] == KIND_YR || rec.kind[i] == KIND_YQ)
        ya += ms;
      if (rec.kind[i] == KIND_T) ta += ms;
    }
    for (auto e : rec.ev) cudaEventDestroy(e);
    if (rc) return rc;
    if (r >= 0) {
      *y_ms = fminf(*y_ms, ya);
      *t_ms = fminf(*t_ms, ta);
    }
  }
  return 0;
}

static int tune(uppe3d_plan* p) {
  const char* env = getenv("UPPE_TUNE");
  if (env && env[0] == '0') return 0;
  const TuneKey key{p->g.Nx, p->g.Ny, p->g.Nt, p->dbl, p->nsm};
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune_cache.find(key);
    if (it != g_tune_cache.end()) {
      p->y_tma = it->second.y_tma;
      p->y_ctas = it->second.y_ctas;
      p->y_late = it->second.y_late;
      p->y_kw = it->second.y_kw;
      p->t_wpb = it->second.t_wpb;
      memcpy(p->tune_ms, it->second.ms, sizeof(p->tune_ms));
      p->tuned = 2;
      return 0;
    }
  }
  cudaStream_t s;
  UPPE_CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  const size_t fbytes = p->csz * (size_t)p->g.npts;
  void* fields[] = {p->b.z[0], p->b.z[1], p->b.acur, p->b.k1, p->b.tsum, p->b.a4p,
                    p->b.tmp[0], p->b.tmp[1], p->b.tmp[2]};
  for (void* f : fields) UPPE_CK(cudaMemsetAsync(f, 0, fbytes, s));
  k_begin<<<1, 1, 0, s>>>(p->st, 1.0, 1e-5, 1e-2, 1e-9, 0);
  k_set_scale_one<<<1, 1, 0, s>>>(p->st);
  // the plain tile kernel rounds differently from the TMA-fed one, so it is a
  // candidate only where the TMA path is unavailable; the register four-step
  // kernels (plain loads or TMA-fed tiles) give the TMA-fed kernel's bits and
  // serve Ny = 256
  struct YC { int tma, ctas, late, kw; } yc[11] = {{1, 2, 0, kW}, {1, 1, 0, kW}, {1, 3, 1, kW}, {1, 2, 1, kW},
                                                 {1, 4, 0, 8}, {1, 6, 1, 8}, {2, 2, 0, kW}, {2, 3, 1, kW},
                                                 {3, 1, 0, kW}, {2, 4, 0, 8}, {2, 6, 1, 8}};
  const int ny = p->ytma ? (yrq_ok(p) ? 11 : 6) : 1;
  if (!p->ytma) yc[0] = YC{0, 2, 0, kW};
  const int tw_n = (p->g.Nt == 512 || (p->g.Nt == 1024 && !p->dbl)) ? 2 : 1;
  const int tw[2] = {8, 4};
  float best_y = 1e30f, best_t = 1e30f;
  int by = 0, bt = 0;
  int rc = 0;
  float y_ms, t_ms;
  p->y_tma = yc[0].tma; p->y_ctas = yc[0].ctas; p->y_late = yc[0].late; p->y_kw = yc[0].kw; p->t_wpb = tw[0];
  rc = p->dbl ? time_attempts<double>(p, s, 1, &y_ms, &t_ms) : time_attempts<float>(p, s, 1, &y_ms, &t_ms);
  for (int i = 0; i < ny && !rc; ++i) {        // y candidates with the default t-pass
    p->y_tma = yc[i].tma; p->y_ctas = yc[i].ctas; p->y_late = yc[i].late; p->y_kw = yc[i].kw;
    rc = p->dbl ? time_attempts<double>(p, s, 3, &y_ms, &t_ms) : time_attempts<float>(p, s, 3, &y_ms, &t_ms);
    p->tune_ms[i] = y_ms;
    if (y_ms < best_y) { best_y = y_ms; by = i; }
  }
  p->y_tma = yc[by].tma; p->y_ctas = yc[by].ctas; p->y_late = yc[by].late; p->y_kw = yc[by].kw;
  for (int i = 0; i < tw_n && !rc; ++i) {      // t candidates with the chosen y passes
    p->t_wpb = tw[i];
    rc = p->dbl ? time_attempts<double>(p, s, 3, &y_ms, &t_ms) : time_attempts<float>(p, s, 3, &y_ms, &t_ms);
    p->tune_ms[11 + i] = t_ms;
    if (t_ms < best_t) { best_t = t_ms; bt = i; }
  }
  p->t_wpb = tw[bt];
  cudaStreamDestroy(s);
  if (rc) return rc;
  p->tuned = 1;
  std::lock_guard<std::mutex> lk(g_tune_mu);
  TuneVal v{p->y_tma, p->y_ctas, p->y_late, p->y_kw, p->t_wpb, {0}};
  memcpy(v.ms, p->tune_ms, sizeof(v.ms));
  g_tune_cache[key] = v;
  return 0;
}

static int build_graphs(uppe3d_plan* p) {
  cudaStream_t s;
  UPPE_CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  for (int which = 0; which < 2; ++which) {
    cudaGraph_t graph;
    UPPE_CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    Recorder rec;
    rec.s = s;
    int rc = p->dbl ? enqueue_attempt<double>(p, rec) : enqueue_attempt<float>(p, rec);
    if (which == 1) k_controller<<<1, 1, 0, s>>>(p->st);
    UPPE_CK(cudaStreamEndCapture(s, &graph));
    if (rc) return rc;
    UPPE_CK(cudaGraphInstantiate(which ? &p->g_step : &p->g_attempt, graph, 0));
    UPPE_CK(cudaGraphDestroy(graph));
  }
  UPPE_CK(cudaStreamDestroy(s));
  return 0;
}

extern "C" int uppe3d_plan_create(const uppe3d_desc* d, uppe3d_plan** out) {
  NvtxRange nvtx_range("uppe3d_plan_create");
  *out = nullptr;
  g_uppe_err[0] = 0;
  if (!d) return UPPE_ERR_ARG;
  if (!is_pow2(d->Nx) || !is_pow2(d->Ny) || !is_pow2(d->Nt) || d->Nx < 16 || d->Ny < 16 ||
      d->Nx > 512 || d->Ny > 512 || d->Nt < 32 || d->Nt > 2048) {
    snprintf(g_uppe_err, sizeof(g_uppe_err),
             "unsupported grid %dx%dx%d: Nx, Ny must be powers of two in [16, 512] and Nt a "
             "power of two in [32, 2048]", d->Nx, d->Ny, d->Nt);
    return UPPE_ERR_SIZE;
  }
  if (d->precision != UPPE_C64 && d->precision != UPPE_C128) return UPPE_ERR_ARG;
  if (d->precision == UPPE_C128 && (d->Nx > 256 || d->Ny > 256)) {
    snprintf(g_uppe_err, sizeof(g_uppe_err),
             "complex128 plans support Nx, Ny <= 256 (shared-memory tile limit)");
    return UPPE_ERR_SIZE;
  }
  uppe3d_plan* p = new uppe3d_plan();
  p->d = *d;
  p->g.Nx = d->Nx; p->g.Ny = d->Ny; p->g.Nt = d->Nt;
  p->g.npts = (long long)d->Nx * d->Ny * d->Nt;
  p->dbl = d->precision == UPPE_C128;
  p->csz = p->dbl ? 16 : 8;
  int rc = 0;
#define UPPE_TRY(x) do { rc = (x); if (rc) { uppe3d_plan_destroy(p); return rc; } } while (0)
  {
    cudaError_t e = cudaMalloc(&p->st, sizeof(State3D));
    if (e != cudaSuccess) { snprintf(g_uppe_err, sizeof(g_uppe_err), "cudaMalloc state: %s", cudaGetErrorString(e)); delete p; return UPPE_ERR_CUDA; }
    p->allocs.push_back(p->st);
    e = cudaMallocHost(&p->st_host, sizeof(State3D));
    if (e != cudaSuccess) { snprintf(g_uppe_err, sizeof(g_uppe_err), "cudaMallocHost: %s", cudaGetErrorString(e)); uppe3d_plan_destroy(p); return UPPE_ERR_CUDA; }
    memset(p->st_host, 0, sizeof(State3D));
    e = cudaMemcpy(p->st, p->st_host, sizeof(State3D), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) { uppe3d_plan_destroy(p); return UPPE_ERR_CUDA; }
  }
  const int Nt = d->Nt, Nxy = d->Nx * d->Ny;
  void* ptr;
  UPPE_TRY(dev_upload(p, &ptr, d->aw, 8 * Nt)); p->tb.aw = (const double*)ptr;
  UPPE_TRY(dev_upload(p, &ptr, d->ksq, 8 * Nt)); p->tb.ksq = (const double*)ptr;
  UPPE_TRY(dev_upload(p, &ptr, d->kref, 8 * Nt)); p->tb.kref = (const double*)ptr;
  UPPE_TRY(dev_upload(p, &ptr, d->valid, Nt)); p->tb.valid = (const unsigned char*)ptr;
  UPPE_TRY(dev_upload(p, &ptr, d->shock, 8 * Nt)); p->tb.shock = (const double*)ptr;
  UPPE_TRY(dev_upload(p, &ptr, d->filt, 8 * Nt)); p->tb.filt = (const double*)ptr;
  UPPE_TRY(dev_upload(p, &ptr, d->kperp2, 8 * (size_t)Nxy)); p->tb.q = (const double*)ptr;
  UPPE_TRY(dev_upload(p, &ptr, d->damp, 8 * (size_t)Nxy)); p->tb.damp = (const double*)ptr;
  if (d->omega_abs) { UPPE_TRY(dev_upload(p, &ptr, d->omega_abs, 8 * Nt)); p->wabs = (const double*)ptr; }
  {
    cudaError_t e = cudaMalloc(&ptr, sizeof(double) * (2 * 592 + 3));
    if (e != cudaSuccess) { snprintf(g_uppe_err, sizeof(g_uppe_err), "cudaMalloc diag: %s", cudaGetErrorString(e)); uppe3d_plan_destroy(p); return UPPE_ERR_CUDA; }
    p->allocs.push_back(ptr);
    p->diag_buf = (double*)ptr;
  }
  {
    auto tx = p->dbl ? twiddles<double>(d->Nx) : twiddles<float>(d->Nx);
    auto ty = p->dbl ? twiddles<double>(d->Ny) : twiddles<float>(d->Ny);
    auto tt = p->dbl ? twiddles<double>(d->Nt) : twiddles<float>(d->Nt);
    UPPE_TRY(dev_upload(p, &ptr, tx.data(), tx.size())); p->tb.twx = ptr;
    UPPE_TRY(dev_upload(p, &ptr, ty.data(), ty.size())); p->tb.twy = ptr;
    UPPE_TRY(dev_upload(p, &ptr, tt.data(), tt.size())); p->tb.twt = ptr;
  }
  {
    const int n = d->lut_n;
    const int dbl = p->dbl;
    if (n < 2) { uppe3d_plan_destroy(p); return UPPE_ERR_ARG; }
    std::vector<unsigned char> lx(n * (p->dbl ? 8 : 4)), lw(n * (p->dbl ? 8 : 4));
    for (int i = 0; i < n; ++i) {
      if (p->dbl) { ((double*)lx.data())[i] = d->lut_log10I[i]; ((double*)lw.data())[i] = d->lut_W[i]; }
      else { ((float*)lx.data())[i] = (float)d->lut_log10I[i]; ((float*)lw.data())[i] = (float)d->lut_W[i]; }
    }
    UPPE_TRY(dev_upload(p, &ptr, lx.data(), lx.size())); p->tb.lut.x = ptr;
    UPPE_TRY(dev_upload(p, &ptr, lw.data(), lw.size())); p->tb.lut.w = ptr;
    {
      std::vector<double> sl(n - 1);
      if (dbl) lut_slopes<double>(d->lut_log10I, d->lut_W, n, sl.data());
      else lut_slopes<float>(d->lut_log10I, d->lut_W, n, sl.data());
      UPPE_TRY(dev_upload(p, &ptr, sl.data(), sl.size() * sizeof(double)));
      p->tb.lut.slope = static_cast<const double*>(ptr);
    }
    p->tb.lut.n = n;
    p->tb.lut.x0 = d->lut_log10I[0];
    p->tb.lut.inv_dx = (n - 1) / (d->lut_log10I[n - 1] - d->lut_log10I[0]);
    {
      // leading run of zero rates (as stored in the field precision)
      int j0 = -1;
      for (int i = 0; i < n; ++i) {
        const double wv = dbl ? d->lut_W[i] : (double)(float)d->lut_W[i];
        if (wv != 0.0) break;
        j0 = i;
      }
      p->tb.lut.zero_x = j0 < 0 ? -INFINITY
                       : (dbl ? d->lut_log10I[j0] : (double)(float)d->lut_log10I[j0]);
      if (j0 == n - 1) p->tb.lut.zero_x = INFINITY;
      p->tb.lut.I_zero = lut_zero_intensity(p->tb.lut.zero_x);
    }
  }
  p->md.gk = d->gamma_kerr;
  p->md.g4 = d->gamma_hoke;
  p->md.Ui = d->Ui;
  p->md.sigma_half = d->sigma_drude / 2.0;
  p->md.w0tc = d->omega0_tau_c;
  p->md.rr = (double)(float)d->rate_rec;
  p->md.dt = (double)(float)d->dt;
  p->md.rho_nt = (double)(float)d->rho_nt;
  p->md.ava = d->ava_coef;
  p->md.plasma = d->plasma_on;
  const size_t fbytes = p->csz * (size_t)p->g.npts;
  void** fields[] = {&p->b.z[0], &p->b.z[1], &p->b.acur, &p->b.k1, &p->b.tsum, &p->b.a4p,
                     &p->b.tmp[0], &p->b.tmp[1], &p->b.tmp[2]};
  for (void** f : fields) {
    cudaError_t e = cudaMalloc(f, fbytes);
    if (e != cudaSuccess) {
      snprintf(g_uppe_err, sizeof(g_uppe_err), "cudaMalloc of a %zu-byte field: %s", fbytes, cudaGetErrorString(e));
      uppe3d_plan_destroy(p);
      return UPPE_ERR_CUDA;
    }
    p->allocs.push_back(*f);
  }
  UPPE_TRY(p->dbl ? set_attrs<double>(p->g) : set_attrs<float>(p->g));
  {
    int dev = 0;
    UPPE_CK(cudaGetDevice(&dev));
    UPPE_CK(cudaDeviceGetAttribute(&p->nsm, cudaDevAttrMultiProcessorCount, dev));
  }
  if (!p->dbl && p->g.Ny >= 64 && p->g.Ny <= 256) UPPE_TRY(setup_ytma(p));
  UPPE_TRY(tune(p));
  UPPE_TRY(build_graphs(p));
#undef UPPE_TRY
  *out = p;
  return 0;
}

extern "C" int uppe3d_plan_destroy(uppe3d_plan* p) {
  if (!p) return 0;
  if (p->g_attempt) cudaGraphExecDestroy(p->g_attempt);
  if (p->g_step) cudaGraphExecDestroy(p->g_step);
  for (void* a : p->allocs) cudaFree(a);
  if (p->st_host) cudaFreeHost(p->st_host);
  delete p;
  return 0;
}

extern "C" int uppe3d_set_field(uppe3d_plan* p, const void* A0, cudaStream_t s) {
  if (!p || !A0) return UPPE_ERR_ARG;
  const long long n = p->g.npts;
  if (p->dbl) k_absmax<double><<<148 * 8, 256, 0, s>>>((const double2*)A0, n, p->st);
  else k_absmax<float><<<148 * 8, 256, 0, s>>>((const float2*)A0, n, p->st);
  k_set_scale<<<1, 1, 0, s>>>(p->st);
  int rc = p->dbl ? launch_t<double, 1>(p, 0, A0, nullptr, s) : launch_t<float, 1>(p, 0, A0, nullptr, s);
  if (rc) return rc;
  UPPE_CK(cudaGetLastError());
  return 0;
}

extern "C" int uppe3d_attempt(uppe3d_plan* p, double h, double* err, cudaStream_t s) {
  if (!p) return UPPE_ERR_ARG;
  k_set_h<<<1, 1, 0, s>>>(p->st, h);
  UPPE_CK(cudaGraphLaunch(p->g_attempt, s));
  UPPE_CK(cudaMemcpyAsync(p->st_host, p->st, sizeof(State3D), cudaMemcpyDeviceToHost, s));
  UPPE_CK(cudaStreamSynchronize(s));
  if (err) *err = p->st_host->err;
  return 0;
}

extern "C" int uppe3d_commit(uppe3d_plan* p, int accept, cudaStream_t s) {
  if (!p) return UPPE_ERR_ARG;
  k_commit<<<1, 1, 0, s>>>(p->st, accept);
  UPPE_CK(cudaGetLastError());
  return 0;
}

static void fill_result(const State3D* h, uppe3d_result* r) {
  r->z = h->z;
  r->h = h->h;
  r->err = h->err;
  r->attempts = h->attempts;
  r->accepted = h->accepted;
  r->fail_count = h->fail_count;
  r->status = h->status;
  r->A_scale = h->A_scale;
}

extern "C" int uppe3d_propagate(uppe3d_plan* p, double L, double tol, double max_step,
                                double min_step, long long max_attempts, uppe3d_result* res,
                                cudaStream_t s) {
  NvtxRange nvtx_range("uppe3d_propagate");
  if (!p || !(tol > 0.0) || !(max_step > 0.0) || !(min_step > 0.0) || !(L >= 0.0)) return UPPE_ERR_ARG;
  if (max_attempts <= 0) max_attempts = UPPE_DEFAULT_MAX_ATTEMPTS;
  k_begin<<<1, 1, 0, s>>>(p->st, L, tol, max_step, min_step, max_attempts);
  UPPE_CK(cudaGetLastError());
  int batch = 1;
  for (;;) {
    for (int i = 0; i < batch; ++i) UPPE_CK(cudaGraphLaunch(p->g_step, s));
    UPPE_CK(cudaMemcpyAsync(p->st_host, p->st, sizeof(State3D), cudaMemcpyDeviceToHost, s));
    UPPE_CK(cudaStreamSynchronize(s));
    if (p->st_host->done) break;
    if (batch < 16) batch *= 2;
  }
  if (res) fill_result(p->st_host, res);
  return 0;
}

extern "C" int uppe3d_run_steps(uppe3d_plan* p, int nsteps, cudaStream_t s) {
  if (!p) return UPPE_ERR_ARG;
  for (int i = 0; i < nsteps; ++i) UPPE_CK(cudaGraphLaunch(p->g_step, s));
  return 0;
}

extern "C" int uppe3d_begin(uppe3d_plan* p, double L, double tol, double max_step,
                            double min_step, long long max_attempts, cudaStream_t s) {
  if (!p || !(tol > 0.0) || !(max_step > 0.0) || !(min_step > 0.0) || !(L >= 0.0)) return UPPE_ERR_ARG;
  if (max_attempts <= 0) max_attempts = UPPE_DEFAULT_MAX_ATTEMPTS;
  k_begin<<<1, 1, 0, s>>>(p->st, L, tol, max_step, min_step, max_attempts);
  UPPE_CK(cudaGetLastError());
  return 0;
}

extern "C" int uppe3d_get_result(uppe3d_plan* p, uppe3d_result* res, cudaStream_t s) {
  if (!p || !res) return UPPE_ERR_ARG;
  UPPE_CK(cudaMemcpyAsync(p->st_host, p->st, sizeof(State3D), cudaMemcpyDeviceToHost, s));
  UPPE_CK(cudaStreamSynchronize(s));
  fill_result(p->st_host, res);
  return 0;
}

extern "C" int uppe3d_save_state(uppe3d_plan* p, void* field_out, uppe3d_state* out, cudaStream_t s) {
  if (!p || !field_out || !out) return UPPE_ERR_ARG;
  UPPE_CK(cudaMemcpyAsync(p->st_host, p->st, sizeof(State3D), cudaMemcpyDeviceToHost, s));
  UPPE_CK(cudaStreamSynchronize(s));
  const State3D& h = *p->st_host;
  UPPE_CK(cudaMemcpyAsync(field_out, p->b.z[h.zidx], p->csz * (size_t)p->g.npts, cudaMemcpyDeviceToDevice, s));
  out->z = h.z; out->h = h.h; out->L = h.L; out->tol = h.tol;
  out->max_step = h.max_step; out->min_step = h.min_step;
  out->err = h.err; out->A_scale = h.A_scale;
  memcpy(&out->peak_ion, &h.ion_bits, sizeof(double));
  out->attempts = h.attempts; out->accepted = h.accepted; out->max_attempts = h.max_attempts;
  out->fail_count = h.fail_count; out->status = h.status; out->done = h.done;
  return 0;
}

extern "C" int uppe3d_load_state(uppe3d_plan* p, const void* field_in, const uppe3d_state* in, cudaStream_t s) {
  if (!p || !field_in || !in || !(in->A_scale > 0.0) || !(in->tol > 0.0) || !(in->min_step > 0.0) ||
      !(in->max_step > 0.0))
    return UPPE_ERR_ARG;
  // the first stage of the next attempt is recomputed from the accepted state
  // (fresh), which gives the same bits as the stored one of the interrupted run
  State3D h;
  memset(&h, 0, sizeof(h));
  h.z = in->z; h.h = in->h; h.L = in->L; h.tol = in->tol;
  h.max_step = in->max_step; h.min_step = in->min_step;
  h.err = in->err; h.A_scale = in->A_scale; h.inv_A_scale = 1.0 / in->A_scale;
  memcpy(&h.ion_bits, &in->peak_ion, sizeof(double));
  h.attempts = in->attempts; h.accepted = in->accepted; h.max_attempts = in->max_attempts;
  h.fail_count = in->fail_count; h.status = in->status; h.done = in->done;
  h.zidx = 0;
  h.fresh = 1;
  h.hlog = nullptr;
  UPPE_CK(cudaMemcpyAsync(p->b.z[0], field_in, p->csz * (size_t)p->g.npts, cudaMemcpyDeviceToDevice, s));
  *p->st_host = h;
  UPPE_CK(cudaMemcpyAsync(p->st, p->st_host, sizeof(State3D), cudaMemcpyHostToDevice, s));
  UPPE_CK(cudaStreamSynchronize(s));   // st_host is reused by the next host read-back
  return 0;
}

extern "C" int uppe3d_resume(uppe3d_plan* p, uppe3d_result* res, cudaStream_t s) {
  NvtxRange nvtx_range("uppe3d_resume");
  if (!p) return UPPE_ERR_ARG;
  int batch = 1;
  for (;;) {
    UPPE_CK(cudaMemcpyAsync(p->st_host, p->st, sizeof(State3D), cudaMemcpyDeviceToHost, s));
    UPPE_CK(cudaStreamSynchronize(s));
    if (p->st_host->done) break;
    for (int i = 0; i < batch; ++i) UPPE_CK(cudaGraphLaunch(p->g_step, s));
    if (batch < 16) batch *= 2;
  }
  if (res) fill_result(p->st_host, res);
  return 0;
}

extern "C" int uppe3d_get_spectrum(uppe3d_plan* p, void* out, cudaStream_t s) {
  if (!p || !out) return UPPE_ERR_ARG;
  const long long nl = (long long)p->g.Nx * p->g.Ny;
  const void* z = nullptr;
  // the state index lives on the device; fetch it (tiny sync copy)
  UPPE_CK(cudaMemcpyAsync(p->st_host, p->st, sizeof(State3D), cudaMemcpyDeviceToHost, s));
  UPPE_CK(cudaStreamSynchronize(s));
  z = p->b.z[p->st_host->zidx];
  if (p->dbl) k_spectrum<double><<<148 * 8, 256, 0, s>>>((const double2*)z, (double2*)out, nl, p->g.Nt, p->st);
  else k_spectrum<float><<<148 * 8, 256, 0, s>>>((const float2*)z, (float2*)out, nl, p->g.Nt, p->st);
  UPPE_CK(cudaGetLastError());
  return 0;
}

extern "C" int uppe3d_get_field(uppe3d_plan* p, void* out, cudaStream_t s) {
  if (!p || !out) return UPPE_ERR_ARG;
  int rc = p->dbl ? launch_t<double, 2>(p, 0, nullptr, out, s) : launch_t<float, 2>(p, 0, nullptr, out, s);
  if (rc) return rc;
  UPPE_CK(cudaGetLastError());
  return 0;
}

extern "C" long long uppe3d_field_bytes(const uppe3d_plan* p) {
  return p ? (long long)(p->csz * p->g.npts) : 0;
}

extern "C" int uppe3d_tuning(const uppe3d_plan* p, int* cfg6, float* ms) {
  if (!p || !cfg6) return UPPE_ERR_ARG;
  cfg6[0] = p->y_tma >= 2 ? p->y_tma : (p->ytma && p->y_tma) ? 1 : 0;
  cfg6[1] = p->y_ctas;
  cfg6[2] = p->y_late;
  cfg6[3] = p->y_kw;
  cfg6[4] = p->t_wpb;
  cfg6[5] = p->tuned;
  if (ms) memcpy(ms, p->tune_ms, sizeof(p->tune_ms));
  return 0;
}

extern "C" int uppe3d_set_tuning(uppe3d_plan* p, int y_tma, int y_ctas, int y_late, int y_kw, int t_wpb) {
  if (!p || y_ctas < 1 || y_ctas > 6 || (y_kw != 8 && y_kw != kW) || (t_wpb != 4 && t_wpb != 8) ||
      y_tma < 0 || y_tma > 3 || (y_tma >= 2 && !yrq_ok(p)) || (y_tma == 3 && (y_late || y_kw != kW)))
    return UPPE_ERR_ARG;
  p->y_tma = y_tma;
  p->y_late = y_late ? 1 : 0;
  // k_ypass_rq / k_ypass_ring: CTAs per SM fixed by their launch bounds
  p->y_ctas = y_tma == 2 ? (p->y_late ? 3 : 2) * (kW / y_kw) : y_tma == 3 ? 1 : y_ctas;
  p->y_kw = y_kw;
  p->t_wpb = t_wpb;
  if (p->g_attempt) { cudaGraphExecDestroy(p->g_attempt); p->g_attempt = nullptr; }
  if (p->g_step) { cudaGraphExecDestroy(p->g_step); p->g_step = nullptr; }
  return build_graphs(p);
}

extern "C" int uppe3d_launches_per_step(const uppe3d_plan* p) {
  (void)p;
  return 22;   // 21 passes + error kernel per attempt, plus the controller
}

extern "C" int uppe3d_profile_attempt(uppe3d_plan* p, int cap, float* ms, int* kind,
                                      double* bytes, int* n, cudaStream_t s) {
  if (!p || !ms || !kind || !bytes || !n) return UPPE_ERR_ARG;
  UPPE_CK(cudaMemcpyAsync(p->st_host, p->st, sizeof(State3D), cudaMemcpyDeviceToHost, s));
  UPPE_CK(cudaStreamSynchronize(s));
  Recorder rec;
  rec.s = s;
  rec.prof = true;
  rec.fresh = p->st_host->fresh;
  rec.fbytes = (double)p->csz * (double)p->g.npts;
  int rc = p->dbl ? enqueue_attempt<double>(p, rec) : enqueue_attempt<float>(p, rec);
  k_controller<<<1, 1, 0, s>>>(p->st);
  UPPE_CK(cudaStreamSynchronize(s));
  const int m = (int)rec.kind.size();
  for (int i = 0; i < m && i < cap; ++i) {
    cudaEventElapsedTime(&ms[i], rec.ev[2 * i], rec.ev[2 * i + 1]);
    kind[i] = rec.kind[i];
    bytes[i] = rec.bytes[i];
  }
  for (auto e : rec.ev) cudaEventDestroy(e);
  *n = m < cap ? m : cap;
  return rc;
}

// ---- diagnostics: energy, photon number, peak ionisation fraction ------------
namespace uppe {
constexpr int kDiagBlocks = 592;
constexpr double kHbar = 1.054571817e-34;

template <typename Rl>
__global__ void __launch_bounds__(256) k_diag_partial(const typename CT<Rl>::T* __restrict__ z,
                                                      long long n, int Nt, const double* wabs,
                                                      double* partial) {
  double e = 0.0, ph = 0.0;
  for (long long i = blockIdx.x * 256LL + threadIdx.x; i < n; i += (long long)gridDim.x * 256) {
    const auto v = z[i];
    const double a2 = (double)v.x * v.x + (double)v.y * v.y;
    e += a2;
    if (wabs) {
      const double w = wabs[i % Nt];
      if (w > 0.0) ph += a2 / (kHbar * w);
    }
  }
  __shared__ double se[256], sp[256];
  se[threadIdx.x] = e;
  sp[threadIdx.x] = ph;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) { se[threadIdx.x] += se[threadIdx.x + o]; sp[threadIdx.x] += sp[threadIdx.x + o]; }
    __syncthreads();
  }
  if (threadIdx.x == 0) { partial[2 * blockIdx.x] = se[0]; partial[2 * blockIdx.x + 1] = sp[0]; }
}

__global__ void k_diag_final(const double* partial, int nb, const State3D* st, double scale,
                             double* out) {
  if (threadIdx.x != 0) return;
  double e = 0.0, ph = 0.0;
  for (int b = 0; b < nb; ++b) { e += partial[2 * b]; ph += partial[2 * b + 1]; }
  const double s2 = st->A_scale * st->A_scale * scale;
  out[0] = e * s2;
  out[1] = ph * s2;
  out[2] = __longlong_as_double((long long)st->ion_bits);
}
}  // namespace uppe

extern "C" int uppe3d_diagnostics(uppe3d_plan* p, double dx, double dy, double* out3, cudaStream_t s) {
  if (!p || !out3) return UPPE_ERR_ARG;
  // the final state's own density (the loop evaluated only step-start states)
  int rc = p->dbl ? launch_t<double, 0>(p, T_FROM_Z, nullptr, p->b.tmp[0], s, 1)
                  : launch_t<float, 0>(p, T_FROM_Z, nullptr, p->b.tmp[0], s, 1);
  if (rc) return rc;
  UPPE_CK(cudaMemcpyAsync(p->st_host, p->st, sizeof(State3D), cudaMemcpyDeviceToHost, s));
  UPPE_CK(cudaStreamSynchronize(s));
  const void* z = p->b.z[p->st_host->zidx];
  const long long n = p->g.npts;
  if (p->dbl) k_diag_partial<double><<<kDiagBlocks, 256, 0, s>>>((const double2*)z, n, p->g.Nt, p->wabs, p->diag_buf);
  else k_diag_partial<float><<<kDiagBlocks, 256, 0, s>>>((const float2*)z, n, p->g.Nt, p->wabs, p->diag_buf);
  // sum_t |A|^2 dt = (dt / Nt) sum_omega |fft_t A|^2
  const double scale = dx * dy * p->d.dt / (double)p->g.Nt;
  k_diag_final<<<1, 32, 0, s>>>(p->diag_buf, kDiagBlocks, p->st, scale, p->diag_buf + 2 * kDiagBlocks);
  UPPE_CK(cudaGetLastError());
  UPPE_CK(cudaMemcpyAsync(out3, p->diag_buf + 2 * kDiagBlocks, 3 * sizeof(double), cudaMemcpyDeviceToHost, s));
  UPPE_CK(cudaStreamSynchronize(s));
  if (!p->wabs) out3[1] = NAN;
  return 0;
}

// ---------------------------------------------------------------------------
// Beam diagnostics of the current state in one pass: the quantities that
// src/3+1D-ERK4(3)IP UPPE/sim.py:140-249 computes from a field copied back to
// the host.  Per omega: sum_xy |Z|^2 and sum_xy m Z (m: a fibre mode); per t,
// after the inverse t transform a = ifft_t(Z): sum_xy |a|^2 and sum_xy m a; per
// (x, y): sum_t |a|^2; the centre line (Nx/2, Ny/2) in both domains.  Z is the
// normalised state; the host applies A_scale, dx, dy, dt.  Per-block sums in
// shared memory, one global atomic per bin and block.
// ---------------------------------------------------------------------------
namespace uppe {
struct BeamDiagOut {
  double *spec, *cw, *pt, *ct, *zc, *ac, *flu;
};

template <int NT, typename Rl> struct BDLaunch {
  using C = typename CT<Rl>::T;
  static constexpr size_t per_warp = (size_t)TCfg<NT>::PAD * sizeof(C);
  static constexpr size_t fixed = NT * sizeof(C) + 6 * NT * sizeof(double);
  static constexpr int WPB = (fixed + 8 * per_warp <= 160 * 1024) ? 8 : (fixed + 4 * per_warp <= 160 * 1024) ? 4
                           : (fixed + 2 * per_warp <= 200 * 1024) ? 2 : 1;
  static size_t smem() { return fixed + WPB * per_warp; }
};

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  return v;
}

template <typename Rl, int NT, int WPB>
__global__ void __launch_bounds__(WPB * 32) k_beam_diag(const State3D* st, Bufs3D b, Geom g, const void* twt,
                                                      const double* mode, BeamDiagOut o) {
  using C = typename CT<Rl>::T;
  constexpr int PAD = TCfg<NT>::PAD;
  constexpr int E = NT / 32;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* tw = reinterpret_cast<C*>(smem_raw);
  double* acc = reinterpret_cast<double*>(tw + NT);   // [6][NT]: |Z|^2, mZ re/im, |a|^2, ma re/im
  C* sK = reinterpret_cast<C*>(acc + 6 * NT) + (threadIdx.x >> 5) * PAD;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int i = threadIdx.x; i < NT; i += WPB * 32) tw[i] = reinterpret_cast<const C*>(twt)[i];
  for (int i = threadIdx.x; i < 6 * NT; i += WPB * 32) acc[i] = 0.0;
  __syncthreads();
  const C* Z = reinterpret_cast<const C*>(b.z[st->zidx]);
  const long long nl = (long long)g.Nx * g.Ny;
  const long long centre = (long long)(g.Nx / 2) * g.Ny + g.Ny / 2;
  const double invN = 1.0 / NT;
  for (long long line = (long long)blockIdx.x * WPB + warp; line < nl; line += (long long)gridDim.x * WPB) {
    const double m = mode ? mode[line] : 0.0;
    const C* zl = Z + line * NT;
    for (int i = 0; i < E; ++i) {
      const int w = lane + 32 * i;
      const C v = zl[w];
      sK[tpad(w)] = v;
      const double vr = v.x, vi = v.y;
      atomicAdd(&acc[w], vr * vr + vi * vi);
      if (mode) { atomicAdd(&acc[NT + w], m * vr); atomicAdd(&acc[2 * NT + w], m * vi); }
      if (line == centre) { o.zc[2 * w] = vr; o.zc[2 * w + 1] = vi; }
    }
    __syncwarp();
    stockham<NT, 1, TCfg<NT>::FT, +1, 1, C>(sK, tw, lane, LineIdx(), WarpSync());
    double f = 0.0;
    for (int i = 0; i < E; ++i) {
      const int t = lane + 32 * i;
      const C v = sK[tpad(t)];
      const double ar = (double)v.x * invN, ai = (double)v.y * invN;
      const double pw = ar * ar + ai * ai;
      f += pw;
      atomicAdd(&acc[3 * NT + t], pw);
      if (mode) { atomicAdd(&acc[4 * NT + t], m * ar); atomicAdd(&acc[5 * NT + t], m * ai); }
      if (line == centre) { o.ac[2 * t] = ar; o.ac[2 * t + 1] = ai; }
    }
    f = warp_sum_d(f);
    if (lane == 0) o.flu[line] = f;
    __syncwarp();
  }
  __syncthreads();
  for (int i = threadIdx.x; i < NT; i += WPB * 32) {
    atomicAdd(&o.spec[i], acc[i]);
    atomicAdd(&o.pt[i], acc[3 * NT + i]);
    if (mode) {
      atomicAdd(&o.cw[2 * i], acc[NT + i]);
      atomicAdd(&o.cw[2 * i + 1], acc[2 * NT + i]);
      atomicAdd(&o.ct[2 * i], acc[4 * NT + i]);
      atomicAdd(&o.ct[2 * i + 1], acc[5 * NT + i]);
    }
  }
}
}  // namespace uppe

template <typename Rl, int NT>
static int beam_diag_n(uppe3d_plan* p, const double* mode, const BeamDiagOut& o, cudaStream_t s) {
  constexpr int WPB = BDLaunch<NT, Rl>::WPB;
  const size_t sm = BDLaunch<NT, Rl>::smem();
  UPPE_CK(cudaFuncSetAttribute(k_beam_diag<Rl, NT, WPB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  k_beam_diag<Rl, NT, WPB><<<148 * 2, WPB * 32, sm, s>>>(p->st, p->b, p->g, p->tb.twt, mode, o);
  UPPE_CK(cudaGetLastError());
  return 0;
}

extern "C" long long uppe3d_beam_diag_elems(const uppe3d_plan* p) {
  return p ? 10LL * p->g.Nt + (long long)p->g.Nx * p->g.Ny : 0;
}

extern "C" int uppe3d_beam_diagnostics(uppe3d_plan* p, const double* mode, double* out, cudaStream_t s) {
  if (!p || !out) return UPPE_ERR_ARG;
  const long long Nt = p->g.Nt;
  UPPE_CK(cudaMemsetAsync(out, 0, sizeof(double) * uppe3d_beam_diag_elems(p), s));
  BeamDiagOut o;
  o.spec = out; o.cw = out + Nt; o.pt = out + 3 * Nt; o.ct = out + 4 * Nt;
  o.zc = out + 6 * Nt; o.ac = out + 8 * Nt; o.flu = out + 10 * Nt;
  switch (p->g.Nt) {
#define UPPE_BD(n) case n: return p->dbl ? beam_diag_n<double, n>(p, mode, o, s) : beam_diag_n<float, n>(p, mode, o, s);
    UPPE_BD(32) UPPE_BD(64) UPPE_BD(128) UPPE_BD(256) UPPE_BD(512) UPPE_BD(1024) UPPE_BD(2048)
#undef UPPE_BD
    default: return UPPE_ERR_SIZE;
  }
}

// ---------------------------------------------------------------------------
// Mirrors on the current state (x, y, omega): amplitude, spectral phase and the
// curved-mirror phase -omega_abs r^2 / (c R) (src/3+1D-ERK4(3)IP UPPE/sim.py:83-96).
// ---------------------------------------------------------------------------
namespace uppe {
template <typename Rl>
__global__ void k_mirror3d(const State3D* st, Bufs3D b, long long n, int Nt, int Ny, double dt,
                           const double* r2, const double* wabs, double invcR, double amp, double gdd,
                           double tod) {
  using C = typename CT<Rl>::T;
  C* z = reinterpret_cast<C*>(b.z[st->zidx]);
  const double dw = 6.283185307179586476925286766559 / (Nt * dt);
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int w = (int)(i % Nt);
    const double om = dw * (w < (Nt + 1) / 2 ? w : w - Nt);
    double ph = 0.5 * gdd * om * om + (1.0 / 6.0) * tod * om * om * om;
    if (r2) ph -= wabs[w] * invcR * r2[i / Nt];
    double sn, cs;
    sincos(ph, &sn, &cs);
    const C a = z[i];
    z[i] = C{(Rl)(amp * ((double)a.x * cs - (double)a.y * sn)), (Rl)(amp * ((double)a.x * sn + (double)a.y * cs))};
  }
  (void)Ny;
}
}  // namespace uppe

extern "C" int uppe3d_mirror(uppe3d_plan* p, const double* r2, double R, double amp, double gdd, double tod,
                             cudaStream_t s) {
  if (!p || !(amp >= 0.0) || !isfinite(gdd) || !isfinite(tod)) return UPPE_ERR_ARG;
  if (r2 && (!p->wabs || !(R != 0.0) || !isfinite(R))) {
    snprintf(g_uppe_err, sizeof(g_uppe_err),
             "uppe3d_mirror: a curved mirror needs desc.omega_abs and a finite non-zero R");
    return UPPE_ERR_ARG;
  }
  const double invcR = r2 ? 1.0 / (299792458.0 * R) : 0.0;
  const long long n = p->g.npts;
  if (p->dbl)
    k_mirror3d<double><<<148 * 8, 256, 0, s>>>(p->st, p->b, n, p->g.Nt, p->g.Ny, p->d.dt, r2, p->wabs, invcR,
                                                amp, gdd, tod);
  else
    k_mirror3d<float><<<148 * 8, 256, 0, s>>>(p->st, p->b, n, p->g.Nt, p->g.Ny, p->d.dt, r2, p->wabs, invcR,
                                               amp, gdd, tod);
  UPPE_CK(cudaGetLastError());
  return 0;
}

// ---------------------------------------------------------------------------
// Adjoint (reverse mode) of the 3D ERK4(3)-IP propagation for the Kerr +
// self-steepening response with dispersion, diffraction, filter and absorber.
// The plasma terms (without avalanche) are differentiated along each t-line in
// k_tvjp.  Convention: dL = Re sum conj(xb) dx.
// ---------------------------------------------------------------------------
namespace uppe {

enum AdjPoint { AP_BOUND = 0, AP_R1, AP_R2, AP_R3, AP_R4, AP_R5 };

struct AdjPointArgs {
  Tables3D tb;
  Geom g;
  int mode;
  double h;
  void *ab, *vb, *a1b, *a2b, *a3b, *tmp;
  const void *acur, *beta, *u4, *zb;
};

// pointwise transposed stage algebra over all (kx, ky, omega) (AP_R*) and the step
// boundary multiply c(x, y, omega) = filter(omega) exp(-damp(x, y) h) / (Nx Ny) (AP_BOUND)
template <typename Rl>
__global__ void __launch_bounds__(256) k_adj_point(AdjPointArgs a) {
  using C = typename CT<Rl>::T;
  const long long n = (long long)a.g.Nx * a.g.Ny * a.g.Nt;
  const int Nt = a.g.Nt;
  const double h = a.h, h2 = 0.5 * h;
  C* ab = reinterpret_cast<C*>(a.ab);
  C* vb = reinterpret_cast<C*>(a.vb);
  C* a1b = reinterpret_cast<C*>(a.a1b);
  C* a2b = reinterpret_cast<C*>(a.a2b);
  C* a3b = reinterpret_cast<C*>(a.a3b);
  C* tmp = reinterpret_cast<C*>(a.tmp);
  const C* acur = reinterpret_cast<const C*>(a.acur);
  const C* beta = reinterpret_cast<const C*>(a.beta);
  const C* u4 = reinterpret_cast<const C*>(a.u4);
  const C* zb = reinterpret_cast<const C*>(a.zb);
  for (long long i = blockIdx.x * 256LL + threadIdx.x; i < n; i += (long long)gridDim.x * 256) {
    const int iw = (int)(i % Nt);
    const long long xy = i / Nt;
    if (a.mode == AP_BOUND) {
      const double c = a.tb.filt[iw] * exp(-a.tb.damp[xy] * h) / ((double)a.g.Nx * a.g.Ny);
      tmp[i] = cscale(zb[i], (Rl)c);
      continue;
    }
    const OmegaCol oc(a.tb, iw);
    const C E = IPFactor<Rl>::get(a.tb, oc, iw, a.tb.q[xy], h2);
    const C Ec = cconj(E);
    if (a.mode == AP_R1) {            // A' = beta + h/6 a4, beta = E (v + h/6 T)
      const C ab_ = ab[i];
      const C wb = cmul(Ec, ab_);
      const C tb = cscale(wb, (Rl)(h / 6));
      vb[i] = wb;
      a1b[i] = tb;
      a2b[i] = cscale(tb, (Rl)2);
      a3b[i] = cscale(tb, (Rl)2);
      tmp[i] = cscale(ab_, (Rl)(h / 6));
    } else if (a.mode == AP_R2) {     // u4 = E (v + h a3)
      const C zb_ = cmul(Ec, ab[i]);
      vb[i] = cadd(vb[i], zb_);
      a3b[i] = cadd(a3b[i], cscale(zb_, (Rl)h));
    } else if (a.mode == AP_R3) {     // u3 = v + h/2 a2
      vb[i] = cadd(vb[i], tmp[i]);
      a2b[i] = cadd(a2b[i], cscale(tmp[i], (Rl)(h / 2)));
    } else if (a.mode == AP_R4) {     // u2 = v + h/2 a1, a1 = E k1
      vb[i] = cadd(vb[i], tmp[i]);
      const C a1b_ = cadd(a1b[i], cscale(tmp[i], (Rl)(h / 2)));
      tmp[i] = cmul(Ec, a1b_);
    } else {                          // v = E A
      ab[i] = cadd(ab[i], cmul(Ec, vb[i]));
    }
  }
  (void)acur; (void)beta; (void)u4;
}

template <int NT, typename Rl> struct VLaunch {   // k_tvjp: three lines + 32 doubles per warp
  using C = typename CT<Rl>::T;
  static constexpr size_t per_warp = 3 * (size_t)TCfg<NT>::PAD * sizeof(C) + 32 * sizeof(double);
  static constexpr int WPB = (NT * sizeof(C) + 4 * per_warp <= 200 * 1024) ? 4
                           : (NT * sizeof(C) + 2 * per_warp <= 200 * 1024) ? 2 : 1;
  static size_t smem() { return NT * sizeof(C) + WPB * per_warp; }
};

// Reverse mode of the plasma term on one t-line held by a warp: the scaled field
// is sU * inv (time domain), the cotangent of the term's samples is in sQ; sQ is
// overwritten with the field cotangent.  Density chunk starts as in the forward
// t-pass (warp scan of affine maps, lane 0's serial update when a clamp binds);
// the density cotangent lam_t = A_t lam_{t+1} + B_t by a warp suffix scan.
template <typename Rl, int NT>
__device__ void tline_plasma_vjp(const TArgs& a, typename CT<Rl>::T* sU, typename CT<Rl>::T* sQ,
                                 double* starts, int lane, Rl inv) {
  using C = typename CT<Rl>::T;
  constexpr int E = NT / 32;
  const Medium3D& m = a.md;
  const AffineStep aff(m);
  const Rl AsR = (Rl)a.st->A_scale;
  const double alpha = a.st->A_scale * a.st->A_scale;
  const int t0 = lane * E;
  auto inten = [&](int t, C& av) {
    av = cscale(sU[tpad(t)], inv);
    const C Ap = cscale(av, AsR);
    return (Rl)(Ap.x * Ap.x + Ap.y * Ap.y);
  };
  bool ok = true;
  double cm = 1.0, dm = 0.0;
  for (int i = 0; i < E; ++i) {
    C av;
    const double w = (double)(float)lut_eval<Rl>(a.tb.lut, inten(t0 + i, av));
    const double cc = aff.e - w * aff.sf;
    ok &= (cc >= 0.0);
    dm = cc * dm + w * m.rho_nt * aff.sf;
    cm = cc * cm;
  }
  double rho0;
  if (__all_sync(0xffffffffu, ok)) {
    double cc = cm, dd = dm;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const double cp = __shfl_up_sync(0xffffffffu, cc, off);
      const double dp = __shfl_up_sync(0xffffffffu, dd, off);
      if (lane >= off) { dd = cc * dp + dd; cc = cc * cp; }
    }
    const double excl = __shfl_up_sync(0xffffffffu, dd, 1);
    rho0 = lane == 0 ? 0.0 : excl;
  } else {
    if (lane == 0) {
      double rho = 0.0;
      for (int t = 0; t < NT; ++t) {
        if (t % E == 0) starts[t / E] = rho;
        C av;
        rho_step(rho, (double)(float)lut_eval<Rl>(a.tb.lut, inten(t, av)), 0.0, m);
      }
    }
    __syncwarp();
    rho0 = starts[lane];
    __syncwarp();
  }
  double cur[E];
  {
    double rho = rho0;
    for (int i = 0; i < E; ++i) {
      C av;
      cur[i] = rho;
      rho_step(rho, (double)(float)lut_eval<Rl>(a.tb.lut, inten(t0 + i, av)), 0.0, m);
    }
  }
  double Ac = 1.0, Bc = 0.0;
  for (int i = E - 1; i >= 0; --i) {
    C av;
    const Rl I = inten(t0 + i, av);
    const C q = sQ[tpad(t0 + i)];
    double A, B;
    plasma_rev<false>(m, aff, alpha, cur[i], (double)(float)lut_eval<Rl>(a.tb.lut, I),
                      lut_slope<Rl>(a.tb.lut, I), (double)I, (double)av.x, (double)av.y, (double)q.x,
                      (double)q.y, A, B);
    Bc = A * Bc + B;
    Ac = A * Ac;
  }
  double sa = Ac, sb = Bc;   // inclusive suffix scan: (A, B) o (A', B') = (A A', A B' + B)
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const double an = __shfl_down_sync(0xffffffffu, sa, off);
    const double bn = __shfl_down_sync(0xffffffffu, sb, off);
    if (lane + off < 32) { sb = sa * bn + sb; sa = sa * an; }
  }
  double lam = __shfl_down_sync(0xffffffffu, sb, 1);
  if (lane == 31) lam = 0.0;
  for (int i = E - 1; i >= 0; --i) {
    C av;
    const Rl I = inten(t0 + i, av);
    const C q = sQ[tpad(t0 + i)];
    double A, B, oar, oai;
    plasma_rev<true>(m, aff, alpha, cur[i], (double)(float)lut_eval<Rl>(a.tb.lut, I),
                     lut_slope<Rl>(a.tb.lut, I), (double)I, (double)av.x, (double)av.y, (double)q.x,
                     (double)q.y, A, B, lam, &oar, &oai, nullptr);
    sQ[tpad(t0 + i)] = C{(Rl)oar, (Rl)oai};
    lam = A * lam + B;
  }
  __syncwarp();
}

// VJP of the t-line part: in U' = F*_xy u and X' = F*_xy nb (both (x, y, omega)),
// out = F_t(ab) / Ntot with a = F*_t U' / Ntot, kb = F*_t(mask shock X'),
// ab = 2|a|^2 conj(c) kb + c a^2 conj(kb), c = i gk A_scale^2.
// plus the plasma term's VJP on lines where it is non-zero.
template <typename Rl, int NT, int WPB>
__global__ void __launch_bounds__(WPB * 32) k_tvjp(TArgs a, const void* xin) {
  using C = typename CT<Rl>::T;
  constexpr int PAD = TCfg<NT>::PAD;
  constexpr int E = NT / 32;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* tw = reinterpret_cast<C*>(smem_raw);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  unsigned char* wbase = smem_raw + NT * sizeof(C) + warp * VLaunch<NT, Rl>::per_warp;
  C* sU = reinterpret_cast<C*>(wbase);
  C* sX = sU + PAD;
  C* sQ = sX + PAD;
  double* starts = reinterpret_cast<double*>(sQ + PAD);
  for (int i = threadIdx.x; i < NT; i += WPB * 32) tw[i] = reinterpret_cast<const C*>(a.tb.twt)[i];
  __syncthreads();
  const long long line = (long long)blockIdx.x * WPB + warp;
  if (line >= (long long)a.g.Nx * a.g.Ny) return;
  const C* uin = reinterpret_cast<const C*>(a.in) + line * NT;
  const C* xn = reinterpret_cast<const C*>(xin) + line * NT;
  C* out = reinterpret_cast<C*>(a.out) + line * NT;
  const double ntot = (double)NT * a.g.Nx * a.g.Ny;
  const Rl inv = (Rl)(1.0 / ntot);
  const Rl gp = (Rl)(a.md.gk * a.st->A_scale * a.st->A_scale);   // c = i gp
  for (int i = 0; i < E; ++i) {
    const int wi = lane + 32 * i;
    sU[tpad(wi)] = uin[wi];
    const Rl ms = a.tb.valid[wi] ? (Rl)a.tb.shock[wi] : (Rl)0;
    sX[tpad(wi)] = cscale(xn[wi], ms);
  }
  __syncwarp();
  stockham<NT, 1, TCfg<NT>::FT, +1, 1, C>(sU, tw, lane, LineIdx(), WarpSync());
  stockham<NT, 1, TCfg<NT>::FT, +1, 1, C>(sX, tw, lane, LineIdx(), WarpSync());
  bool pl = false;
  if (a.md.plasma) {   // the plasma term is non-zero only on lines where some W > 0
    const Rl AsR = (Rl)a.st->A_scale;
    bool any = false;
    for (int i = 0; i < E; ++i) {
      const C Ap = cscale(cscale(sU[tpad(lane * E + i)], inv), AsR);
      any |= (float)lut_eval<Rl>(a.tb.lut, Ap.x * Ap.x + Ap.y * Ap.y) != 0.f;
    }
    pl = __any_sync(0xffffffffu, any);
  }
  if (pl) {
    for (int i = 0; i < E; ++i) {
      const int wi = lane + 32 * i;
      sQ[tpad(wi)] = a.tb.valid[wi] ? xn[wi] : C{0, 0};
    }
    __syncwarp();
    stockham<NT, 1, TCfg<NT>::FT, +1, 1, C>(sQ, tw, lane, LineIdx(), WarpSync());
    tline_plasma_vjp<Rl, NT>(a, sU, sQ, starts, lane, inv);
  }
  for (int i = 0; i < E; ++i) {
    const int t = lane + 32 * i;
    const C av = cscale(sU[tpad(t)], inv);
    const C kb = sX[tpad(t)];
    const Rl I2 = (Rl)2 * (av.x * av.x + av.y * av.y);
    // 2|a|^2 conj(c) kb with conj(c) = -i gp ;  c a^2 conj(kb) with c = i gp
    const C t1 = cscale(C{kb.y, -kb.x}, gp * I2);
    const C a2 = cmul(av, av);
    const C t2p = cmul(a2, cconj(kb));
    const C t2 = cscale(C{-t2p.y, t2p.x}, gp);
    C r = cadd(t1, t2);
    if (pl) r = cadd(r, sQ[tpad(t)]);
    sU[tpad(t)] = r;
  }
  __syncwarp();
  stockham<NT, 1, TCfg<NT>::FT, -1, 1, C>(sU, tw, lane, LineIdx(), WarpSync());
  for (int i = 0; i < E; ++i) {
    const int wi = lane + 32 * i;
    out[wi] = cscale(sU[tpad(wi)], inv);
  }
}

// out = scale * (unnormalised FFT along t of in), DIR = -1 forward, +1 inverse
template <typename Rl, int NT, int WPB, int DIR>
__global__ void __launch_bounds__(WPB * 32) k_tline(TArgs a, double scale) {
  using C = typename CT<Rl>::T;
  constexpr int PAD = TCfg<NT>::PAD;
  constexpr int E = NT / 32;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* tw = reinterpret_cast<C*>(smem_raw);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  C* sK = tw + NT + warp * 2 * PAD;
  for (int i = threadIdx.x; i < NT; i += WPB * 32) tw[i] = reinterpret_cast<const C*>(a.tb.twt)[i];
  __syncthreads();
  const long long line = (long long)blockIdx.x * WPB + warp;
  if (line >= (long long)a.g.Nx * a.g.Ny) return;
  const C* src = reinterpret_cast<const C*>(a.in) + line * NT;
  C* dst = reinterpret_cast<C*>(a.out) + line * NT;
  for (int i = 0; i < E; ++i) sK[tpad(lane + 32 * i)] = src[lane + 32 * i];
  __syncwarp();
  stockham<NT, 1, TCfg<NT>::FT, DIR, 1, C>(sK, tw, lane, LineIdx(), WarpSync());
  const Rl sc = (Rl)scale;
  for (int i = 0; i < E; ++i) dst[lane + 32 * i] = cscale(sK[tpad(lane + 32 * i)], sc);
}

__global__ void k_set_state(State3D* st, int zidx, int fresh, double h) {
  st->zidx = zidx;
  st->fresh = fresh;
  st->h = h;
  st->done = 0;
}

__global__ void k_set_log(State3D* st, double* hlog, long long cap) {
  st->hlog = hlog;
  st->hlog_cap = cap;
}

}  // namespace uppe

template <typename Rl, int NT, int KIND>
static int adj_tlaunch_n(uppe3d_plan* p, const void* in, const void* xin, void* out, double scale,
                         cudaStream_t s) {
  TArgs a;
  memset(&a, 0, sizeof(a));
  a.st = p->st; a.tb = p->tb; a.md = p->md; a.b = p->b; a.g = p->g; a.in = in; a.out = out;
  constexpr int WPB = TLaunch<NT, Rl>::WPB;
  const long long nl = (long long)p->g.Nx * p->g.Ny;
  const unsigned nb = (unsigned)((nl + WPB - 1) / WPB);
  const size_t smem = TLaunch<NT, Rl>::smem();
  cudaError_t e;
  if (KIND == 0) {
    constexpr int VW = VLaunch<NT, Rl>::WPB;
    const size_t vsm = VLaunch<NT, Rl>::smem();
    const unsigned vnb = (unsigned)((nl + VW - 1) / VW);
    e = cudaFuncSetAttribute(k_tvjp<Rl, NT, VW>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)vsm);
    if (e == cudaSuccess) k_tvjp<Rl, NT, VW><<<vnb, VW * 32, vsm, s>>>(a, xin);
  } else if (KIND == 1) {
    e = cudaFuncSetAttribute(k_tline<Rl, NT, WPB, +1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) k_tline<Rl, NT, WPB, +1><<<nb, WPB * 32, smem, s>>>(a, scale);
  } else {
    e = cudaFuncSetAttribute(k_tline<Rl, NT, WPB, -1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) k_tline<Rl, NT, WPB, -1><<<nb, WPB * 32, smem, s>>>(a, scale);
  }
  if (e != cudaSuccess) return UPPE_ERR_CUDA;
  return cudaGetLastError() == cudaSuccess ? 0 : UPPE_ERR_CUDA;
}

template <typename Rl, int KIND>
static int adj_tlaunch(uppe3d_plan* p, const void* in, const void* xin, void* out, double scale,
                       cudaStream_t s) {
  switch (p->g.Nt) {
#define UPPE_AT(n) case n: return adj_tlaunch_n<Rl, n, KIND>(p, in, xin, out, scale, s);
    UPPE_AT(32) UPPE_AT(64) UPPE_AT(128) UPPE_AT(256) UPPE_AT(512) UPPE_AT(1024) UPPE_AT(2048)
#undef UPPE_AT
    default: return UPPE_ERR_SIZE;
  }
}

template <typename Rl>
static int adj_point(uppe3d_plan* p, int mode, double h, void* const* w, const void* zb, cudaStream_t s) {
  AdjPointArgs a;
  a.tb = p->tb; a.g = p->g; a.mode = mode; a.h = h;
  a.ab = w[0]; a.vb = w[1]; a.a1b = w[2]; a.a2b = w[3]; a.a3b = w[4]; a.tmp = w[5];
  a.acur = p->b.acur; a.beta = p->b.tsum; a.u4 = nullptr; a.zb = zb;
  k_adj_point<Rl><<<148 * 8, 256, 0, s>>>(a);
  return cudaGetLastError() == cudaSuccess ? 0 : UPPE_ERR_CUDA;
}

template <typename Rl>
static int adj_plain_y(uppe3d_plan* p, int mode, const void* in, void* out, double scale, cudaStream_t s) {
  p->pass_scale = scale;
  const int rc = launch_space<Rl>(p, mode, in, out, s);
  p->pass_scale = 1.0;
  return rc;
}

// VJP of N at u with cotangent nb -> out (all (kx, ky, omega)); uses tmp[0..2]
template <typename Rl>
static int adj_vjp(uppe3d_plan* p, const void* u, const void* nb, void* out, cudaStream_t s) {
  void* const* t = p->b.tmp;
  int rc = 0;
  rc |= adj_plain_y<Rl>(p, YPLAIN_INV, u, t[0], 1.0, s);
  rc |= launch_space<Rl>(p, XINV, t[0], t[1], s);              // U'
  rc |= adj_plain_y<Rl>(p, YPLAIN_INV, nb, t[0], 1.0, s);
  rc |= launch_space<Rl>(p, XINV, t[0], t[2], s);              // X'
  rc |= adj_tlaunch<Rl, 0>(p, t[1], t[2], t[0], 1.0, s);       // F_t(ab)/Ntot
  rc |= launch_space<Rl>(p, XFWD, t[0], t[1], s);
  rc |= adj_plain_y<Rl>(p, YPLAIN_FWD, t[1], out, 1.0, s);
  return rc;
}

template <typename Rl>
static int adjoint_impl(uppe3d_plan* p, const double* hl, int nsteps, int K, const void* A0,
                        const void* Zbar, void* A0bar, void* work, cudaStream_t s) {
  const size_t F = p->csz * (size_t)p->g.npts;
  unsigned char* wb = static_cast<unsigned char*>(work);
  void* W[6];                       // ab, vb, a1b, a2b, a3b, tmp
  for (int k = 0; k < 6; ++k) W[k] = wb + k * F;
  void* U2 = wb + 6 * F; void* U3 = wb + 7 * F; void* U4 = wb + 8 * F; void* ZB = wb + 9 * F;
  const int nseg = (nsteps + K - 1) / K;
  unsigned char* CK = wb + 10 * F;
  unsigned char* SEG = CK + (size_t)(nseg > 0 ? nseg : 1) * F;
  int rc = uppe3d_set_field(p, A0, s);
  if (rc) return rc;
  int zidx = 0;
  Recorder rec;
  rec.s = s;
  auto attempt = [&](double h) {
    k_set_h<<<1, 1, 0, s>>>(p->st, h);
    return enqueue_attempt<Rl>(p, rec);
  };
  // forward replay with checkpoints every K steps
  UPPE_CK(cudaMemcpyAsync(CK, p->b.z[zidx], F, cudaMemcpyDeviceToDevice, s));
  for (int j = 0; j < nsteps; ++j) {
    rc |= attempt(hl[j]);
    k_commit<<<1, 1, 0, s>>>(p->st, 1);
    zidx ^= 1;
    if ((j + 1) % K == 0 && j + 1 < nsteps)
      UPPE_CK(cudaMemcpyAsync(CK + (size_t)((j + 1) / K) * F, p->b.z[zidx], F, cudaMemcpyDeviceToDevice, s));
  }
  UPPE_CK(cudaMemcpyAsync(ZB, Zbar, F, cudaMemcpyDeviceToDevice, s));
  for (int sg = nseg - 1; sg >= 0; --sg) {
    const int j0 = sg * K, j1 = nsteps < j0 + K ? nsteps : j0 + K;
    UPPE_CK(cudaMemcpyAsync(p->b.z[0], CK + (size_t)sg * F, F, cudaMemcpyDeviceToDevice, s));
    UPPE_CK(cudaMemcpyAsync(SEG, p->b.z[0], F, cudaMemcpyDeviceToDevice, s));
    k_set_state<<<1, 1, 0, s>>>(p->st, 0, 1, hl[j0]);
    int zi = 0;
    for (int j = j0; j < j1 - 1; ++j) {
      rc |= attempt(hl[j]);
      k_commit<<<1, 1, 0, s>>>(p->st, 1);
      zi ^= 1;
      UPPE_CK(cudaMemcpyAsync(SEG + (size_t)(j - j0 + 1) * F, p->b.z[zi], F, cudaMemcpyDeviceToDevice, s));
    }
    for (int j = j1 - 1; j >= j0; --j) {
      const double h = hl[j];
      // recompute the step from its start state, saving u2, u3, u4
      UPPE_CK(cudaMemcpyAsync(p->b.z[0], SEG + (size_t)(j - j0) * F, F, cudaMemcpyDeviceToDevice, s));
      k_set_state<<<1, 1, 0, s>>>(p->st, 0, 1, h);
      p->save_u[0] = U2; p->save_u[1] = U3; p->save_u[2] = U4;
      rc |= enqueue_attempt<Rl>(p, rec);
      p->save_u[0] = p->save_u[1] = p->save_u[2] = nullptr;
      // boundary: A4 bar = F_xy(c Zbar) / (Nx Ny)
      rc |= adj_point<Rl>(p, AP_BOUND, h, W, ZB, s);
      rc |= launch_space<Rl>(p, XFWD, W[5], p->b.tmp[0], s);
      rc |= adj_plain_y<Rl>(p, YPLAIN_FWD, p->b.tmp[0], W[0], 1.0, s);
      // stages
      rc |= adj_point<Rl>(p, AP_R1, h, W, nullptr, s);
      rc |= adj_vjp<Rl>(p, U4, W[5], W[0], s);            // u4 bar -> ab
      rc |= adj_point<Rl>(p, AP_R2, h, W, nullptr, s);
      rc |= adj_vjp<Rl>(p, U3, W[4], W[5], s);            // u3 bar -> tmp
      rc |= adj_point<Rl>(p, AP_R3, h, W, nullptr, s);
      rc |= adj_vjp<Rl>(p, U2, W[3], W[5], s);            // u2 bar -> tmp
      rc |= adj_point<Rl>(p, AP_R4, h, W, nullptr, s);
      rc |= adj_vjp<Rl>(p, p->b.acur, W[5], W[0], s);     // through k1 = N(A) -> ab
      rc |= adj_point<Rl>(p, AP_R5, h, W, nullptr, s);
      // Zbar of the step start: A = F_xy Z -> Zbar = F*_xy(ab)
      rc |= adj_plain_y<Rl>(p, YPLAIN_INV, W[0], p->b.tmp[0], 1.0, s);
      rc |= launch_space<Rl>(p, XINV, p->b.tmp[0], ZB, s);
    }
  }
  // Z0 = F_t(A0 / A_scale) -> A0 bar = F*_t(Zbar) / A_scale (A_scale is read on the host)
  UPPE_CK(cudaMemcpyAsync(p->st_host, p->st, sizeof(State3D), cudaMemcpyDeviceToHost, s));
  UPPE_CK(cudaStreamSynchronize(s));
  rc |= adj_tlaunch<Rl, 1>(p, ZB, nullptr, A0bar, 1.0 / p->st_host->A_scale, s);
  UPPE_CK(cudaGetLastError());
  return rc;
}

extern "C" int uppe3d_transform_t(uppe3d_plan* p, const void* in, void* out, int dir, double scale,
                                  cudaStream_t s) {
  if (!p || !in || !out || (dir != -1 && dir != 1)) return UPPE_ERR_ARG;
  if (dir < 0) return p->dbl ? adj_tlaunch<double, 2>(p, in, nullptr, out, scale, s)
                             : adj_tlaunch<float, 2>(p, in, nullptr, out, scale, s);
  return p->dbl ? adj_tlaunch<double, 1>(p, in, nullptr, out, scale, s)
                : adj_tlaunch<float, 1>(p, in, nullptr, out, scale, s);
}

extern "C" long long uppe3d_adjoint_work_bytes(const uppe3d_plan* p, int nsteps, int K) {
  if (!p || nsteps < 0 || K <= 0) return -1;
  const long long nseg = (nsteps + K - 1) / K;
  return (10LL + (nseg > 0 ? nseg : 1) + K) * (long long)p->csz * p->g.npts;
}

extern "C" int uppe3d_set_step_log(uppe3d_plan* p, double* hlog, long long cap, cudaStream_t s) {
  if (!p || cap < 0) return UPPE_ERR_ARG;
  k_set_log<<<1, 1, 0, s>>>(p->st, hlog, hlog ? cap : 0);
  UPPE_CK(cudaGetLastError());
  return 0;
}

extern "C" int uppe3d_adjoint(uppe3d_plan* p, const double* hlog_host, int nsteps, int K, const void* A0,
                              const void* Zbar, void* A0bar, void* work, cudaStream_t s) {
  NvtxRange nvtx_range("uppe3d_adjoint");
  if (!p || !hlog_host || nsteps < 0 || K <= 0 || !A0 || !Zbar || !A0bar || !work) return UPPE_ERR_ARG;
  if (p->md.g4 != 0.0 || (p->md.plasma && p->md.ava != 0.0)) {
    snprintf(g_uppe_err, sizeof(g_uppe_err),
             "uppe3d_adjoint: the n4 term and avalanche ionisation have no adjoint here");
    return UPPE_ERR_ARG;
  }
  return p->dbl ? adjoint_impl<double>(p, hlog_host, nsteps, K, A0, Zbar, A0bar, work, s)
                : adjoint_impl<float>(p, hlog_host, nsteps, K, A0, Zbar, A0bar, work, s);
}

// ===========================================================================
// Real-field 3+1D ERK4(3)-IP UPPE (src/3+1D-UPPE-ERK4(3)IP-real-field/
// solver_3d.py, media_physics.py).  The accepted state is the real field
// E(x, y, t) / E_scale; spectra live in (kx, ky, omega >= 0) with Nt/2 + 1 bins
// stored in rows of Nw = Nt/2 + kW (the pad bins stay zero), so the plain x and
// y transform passes of the envelope solver serve them.  t-line kernels (one
// warp per (x, y) line, complex FFT in shared memory): real -> half spectrum,
// the nonlinear response (half spectrum -> real E via the Hermitian extension,
// PPT rate table, density + Drude current scan, Kerr + chi5 polarisation,
// P and J in one transform after per-line scaling, source coefficients
// P_c, J_c), and the output (filter, inverse transform, absorber).  Stage algebra: one spectral
// kernel with exp(s D) computed per element in FP64.
// ===========================================================================

namespace uppe {
struct RfConst {
  double I_coef, aval, chi3e, chi5e;           // I = I_coef E^2; W_ava = aval I; P = chi3e E^3 + chi5e E^5
  double fR;                                   // Raman fraction (0: none)
  double rr, dt, rho_nt, Ui, e2m, nu, exp_nu, step_J;   // density / Drude constants (float32-rounded inputs)
  double inv_rho_nt;                           // 1 / rho_nt (the depletion factor as a product)
  double E_scale;
};

struct RfTables {
  const double* kk;      // k(omega)^2 [Nr]
  const double* kref;    // k1 omega [Nr]
  const double* w;       // omega [Nr]
  const double* filt;    // [Nr]
  const double* kp2;     // k_perp^2 [Nx*Ny]
  const double* damp;    // [Nx*Ny]
  Lut lut;
  const void* ramH;      // Raman: H_k, k = 0..Nt, of the 2 Nt-point response (solver precision)
  const void* ramW;      // Raman: exp(-i pi k / Nt), k = 0..Nt/2
};

enum RfLine { RF_FROM_T = 0, RF_NL = 1, RF_OUT = 2 };

// the reference's density update for w_av = 0: Gamma = -rr exactly, so
// exp(Gamma dt) and the step factor are the constants e_r and sf0
__device__ __forceinline__ void rf_rho_step(double& rho, double wp, const RfConst& rc, double e_r, double sf0) {
  double dep = (rc.rho_nt - rho) * rc.inv_rho_nt;
  if (dep < 0.0) dep = 0.0;
  double r = rho * e_r + wp * rc.rho_nt * dep * sf0;
  if (r > rc.rho_nt) r = rc.rho_nt;
  if (r < 0.0) r = 0.0;
  rho = r;
}

// launch shape of k_rf_line: per warp a line buffer (PAD complex) and the real
// samples (NT; with the Raman response another NT for E_eff^2), up to 8 warps
// while two blocks fit an SM
template <int NT, typename Rl, bool RAMAN = false> struct RfLaunch {
  using C = typename CT<Rl>::T;
  static constexpr size_t per_warp = (size_t)TCfg<NT>::PAD * sizeof(C) + (RAMAN ? 2 : 1) * NT * sizeof(Rl);
  static constexpr size_t fixed = NT * sizeof(C);
  static constexpr int WPB = (fixed + 8 * per_warp <= 113 * 1024) ? 8 : (fixed + 4 * per_warp <= 113 * 1024) ? 4
                           : (fixed + 2 * per_warp <= 200 * 1024) ? 2 : 1;
  static size_t smem() { return fixed + WPB * per_warp; }
};

// The Raman term (media_physics.py:376-390): r = real(ifft(fft(x) H))[:NT] with x
// = E^2 zero-padded to M = 2 NT samples, i.e. the circular convolution of length
// M.  x is real, so one NT-point complex transform of z[m] = x[2m] + i x[2m+1]
// gives its spectrum (z = 0 for m >= NT/2): with W_k = exp(-i pi k / NT),
//   X_k = (Z_k + conj Z_(NT-k))/2 - (i/2) W_k (Z_k - conj Z_(NT-k)),  k = 0..NT,
// Y_k = X_k H_k is Hermitian, and the inverse packs back the same way:
//   Z'_k = (Y_k + conj Y_(NT-k)) + i conj(W_k) (Y_k - conj Y_(NT-k)),  k < NT,
// whose unnormalised inverse NT-point transform is M (r[2m] + i r[2m+1]).  Each
// lane handles the bin pairs (k, NT - k) it owns, so the update is in place.
template <typename Rl, int NT>
__device__ __forceinline__ void rf_raman(typename CT<Rl>::T* S, const Rl* R, Rl* Q, const typename CT<Rl>::T* tw,
                                         const RfTables& tb, const RfConst& rc, int lane) {
  using C = typename CT<Rl>::T;
  for (int m = lane; m < NT; m += 32) {
    C z = C{(Rl)0, (Rl)0};
    if (m < NT / 2) {
      const Rl e0 = R[2 * m], e1 = R[2 * m + 1];
      z = C{e0 * e0, e1 * e1};
    }
    S[tpad(m)] = z;
  }
  __syncwarp();
  stockham<NT, 1, TCfg<NT>::FT, -1, 1, C>(S, tw, lane, LineIdx(), WarpSync());
  const C* H = reinterpret_cast<const C*>(tb.ramH);
  const C* Wt = reinterpret_cast<const C*>(tb.ramW);
  const Rl half = (Rl)0.5;
  auto spec = [&](C Zk, C Zn, C w) {          // X_k from Z_k, Z_(NT-k), W_k
    const C ev = C{(Zk.x + Zn.x) * half, (Zk.y - Zn.y) * half};
    const C od = C{(Zk.y + Zn.y) * half, -(Zk.x - Zn.x) * half};   // (Z_k - conj Z_n) / (2i)
    return cadd(ev, cmul(w, od));
  };
  auto pack = [&](C Yk, C Yn, C w) {          // Z'_k from Y_k, Y_(NT-k), W_k
    const C s = C{Yk.x + Yn.x, Yk.y - Yn.y};
    const C d = C{Yk.x - Yn.x, Yk.y + Yn.y};
    const C wd = cmul(C{w.x, -w.y}, d);
    return C{s.x - wd.y, s.y + wd.x};
  };
  for (int k = lane; k <= NT / 2; k += 32) {
    if (k == 0) {
      const C Z0 = S[tpad(0)];
      const C Y0 = cscale(H[0], Z0.x + Z0.y);          // X_0 = Re Z_0 + Im Z_0
      const C YN = cscale(H[NT], Z0.x - Z0.y);         // X_NT = Re Z_0 - Im Z_0
      S[tpad(0)] = pack(Y0, YN, C{(Rl)1, (Rl)0});
      continue;
    }
    const int n = NT - k;
    const C Zk = S[tpad(k)], Zn = S[tpad(n)];
    const C wk = Wt[k];
    const C wn = C{-wk.x, wk.y};                       // W_(NT-k) = -conj(W_k)
    const C Yk = cmul(spec(Zk, Zn, wk), H[k]);
    const C Yn = cmul(spec(Zn, Zk, wn), H[n]);
    S[tpad(k)] = pack(Yk, Yn, wk);
    if (n != k) S[tpad(n)] = pack(Yn, Yk, wn);
  }
  __syncwarp();
  stockham<NT, 1, TCfg<NT>::FT, +1, 1, C>(S, tw, lane, LineIdx(), WarpSync());
  const Rl invM = (Rl)(1.0 / (2.0 * NT));
  const Rl a = (Rl)(1.0 - rc.fR), b = (Rl)rc.fR;
  for (int t = lane; t < NT; t += 32) {
    const C zr = S[tpad(t >> 1)];
    const Rl r = ((t & 1) ? zr.y : zr.x) * invM;
    const Rl E = R[t];
    Q[t] = a * (E * E) + b * r;
  }
  __syncwarp();
}

// one t-line per warp; S: line buffer (PAD complex), R: real samples (NT); with
// RAMAN, Q: E_eff^2 (NT)
template <typename Rl, int NT, int WPB, bool RAMAN>
__global__ void __launch_bounds__(WPB * 32, (WPB * 32 * 2 <= 1024) ? 2 : 1)
k_rf_line(int mode, RfTables tb, RfConst rc, Geom g, int Nw, const void* in, void* out, const void* twt,
          double in_scale, double h) {
  using C = typename CT<Rl>::T;
  using LS = RfLaunch<NT, Rl, RAMAN>;
  constexpr int PAD = TCfg<NT>::PAD;
  constexpr int NR = NT / 2 + 1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* tw = reinterpret_cast<C*>(smem_raw);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  C* S = reinterpret_cast<C*>(smem_raw + LS::fixed + warp * LS::per_warp);
  Rl* R = reinterpret_cast<Rl*>(S + PAD);
  Rl* Q = R + NT;
  for (int i = threadIdx.x; i < NT; i += WPB * 32) tw[i] = reinterpret_cast<const C*>(twt)[i];
  __syncthreads();
  const long long line = (long long)blockIdx.x * WPB + warp;
  if (line >= (long long)g.Nx * g.Ny) return;
  if (mode == RF_FROM_T) {   // real E_t -> bins 0..NT/2
    const Rl* e = reinterpret_cast<const Rl*>(in) + line * NT;
    for (int t = lane; t < NT; t += 32) S[tpad(t)] = C{e[t], (Rl)0};
    __syncwarp();
    stockham<NT, 1, TCfg<NT>::FT, -1, 1, C>(S, tw, lane, LineIdx(), WarpSync());
    C* o = reinterpret_cast<C*>(out) + line * Nw;
    for (int k = lane; k < Nw; k += 32) o[k] = k < NR ? S[tpad(k)] : C{0, 0};
    return;
  }
  // half spectrum (after the unnormalised inverse x, y transforms) -> Hermitian line
  const C* src = reinterpret_cast<const C*>(in) + line * Nw;
  const Rl sc = (Rl)in_scale;
  for (int k = lane; k < NR; k += 32) {
    C v = cscale(src[k], sc);
    if (mode == RF_OUT) v = cscale(v, (Rl)tb.filt[k]);
    // irfft takes the real parts of the DC and Nyquist bins
    if (k == 0 || k == NT / 2) v.y = (Rl)0;
    S[tpad(k)] = v;
    if (k > 0 && k < NT / 2) S[tpad(NT - k)] = C{v.x, -v.y};
  }
  __syncwarp();
  stockham<NT, 1, TCfg<NT>::FT, +1, 1, C>(S, tw, lane, LineIdx(), WarpSync());
  const Rl invN = (Rl)(1.0 / NT);
  if (mode == RF_OUT) {
    const double dp = tb.damp[line];
    const Rl ab = dp == 0.0 ? (Rl)1 : (Rl)exp(-dp * h);
    Rl* o = reinterpret_cast<Rl*>(out) + line * NT;
    for (int t = lane; t < NT; t += 32) o[t] = (S[tpad(t)].x * invN) * ab;
    return;
  }
  // ---- nonlinear response (media_physics.py:258-318 with the kernel :11-118) ----
  const Rl Es = (Rl)rc.E_scale;
  const Rl inv_Es = (Rl)1 / Es;
  for (int t = lane; t < NT; t += 32) R[t] = (S[tpad(t)].x * invN) * Es;   // physical field
  __syncwarp();
  if constexpr (RAMAN) rf_raman<Rl, NT>(S, R, Q, tw, tb, rc, lane);   // E_eff^2 into Q; S free again
  // density and Drude current (media_physics.py:11-118).  Without avalanche and
  // while no clamp binds the density update is affine in rho, and the free
  // current J' = J exp(-nu dt) + (e^2/m) rho E step_J always is: chunks of E
  // samples per lane, warp scans of the chunk maps, then each lane walks its
  // chunk.  Otherwise lane 0 runs the reference's serial loop.
  {
    constexpr int EC = NT / 32;
    const int t0 = lane * EC;
    const Rl Ic = (Rl)rc.I_coef, Av = (Rl)rc.aval;
    const double e_r = exp(fmin(fmax(-rc.rr * rc.dt, -10.0), 10.0));   // exp(gdt) with w_av = 0
    const double g0 = fmin(fmax(-rc.rr * rc.dt, -10.0), 10.0);
    const double sf0 = (fabs(g0) < 1e-5) ? rc.dt * (1.0 + 0.5 * g0) : (e_r - 1.0) / (-rc.rr);
    bool ok = rc.aval == 0.0;
    double cm = 1.0, dm = 0.0;
    for (int i = 0; i < EC; ++i) {   // rates cached in S.x (the samples now live in R)
      const Rl Ef = R[t0 + i];
      const float wf = (float)lut_eval<Rl>(tb.lut, Ic * (Ef * Ef));
      S[tpad(t0 + i)].x = (Rl)wf;
      const double wp = (double)wf;
      const double c = e_r - wp * sf0;
      ok &= (c >= 0.0);
      dm = c * dm + wp * rc.rho_nt * sf0;
      cm = c * cm;
    }
    // no clamp binds if every chunk map keeps rho in [0, rho_nt] (c >= 0 and the
    // composed value stays below rho_nt; checked on the scan result below)
    if (__all_sync(0xffffffffu, ok)) {
      double c = cm, d = dm;
#pragma unroll
      for (int off = 1; off < 32; off <<= 1) {
        const double cp = __shfl_up_sync(0xffffffffu, c, off);
        const double dp = __shfl_up_sync(0xffffffffu, d, off);
        if (lane >= off) { d = c * dp + d; c = c * cp; }
      }
      const double ex = __shfl_up_sync(0xffffffffu, d, 1);
      const double rho0 = lane == 0 ? 0.0 : ex;
      const double rho_end = __shfl_sync(0xffffffffu, d, 31);
      ok = rho_end <= rc.rho_nt;
      if (__all_sync(0xffffffffu, ok)) {
        // free-current chunk map: J_end = aJ J_start + bJ
        double rho = rho0, aJ = 1.0, bJ = 0.0;
        for (int i = 0; i < EC; ++i) {
          const Rl Ef = R[t0 + i];
          const double wp = (double)(float)S[tpad(t0 + i)].x;
          const double dJ = rc.e2m * rho * (double)(float)Ef * rc.step_J;
          bJ = bJ * rc.exp_nu + dJ;
          aJ = aJ * rc.exp_nu;
          rf_rho_step(rho, wp, rc, e_r, sf0);
        }
        double a = aJ, b = bJ;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
          const double ap = __shfl_up_sync(0xffffffffu, a, off);
          const double bp = __shfl_up_sync(0xffffffffu, b, off);
          if (lane >= off) { b = a * bp + b; a = a * ap; }
        }
        const double exJ = __shfl_up_sync(0xffffffffu, b, 1);
        double Jf = lane == 0 ? 0.0 : exJ;
        rho = rho0;
        for (int i = 0; i < EC; ++i) {
          const int t = t0 + i;
          const Rl Ef = R[t];
          const double E = (double)(float)Ef;
          const double wp = (double)(float)S[tpad(t)].x;
          double dep = (rc.rho_nt - rho) * rc.inv_rho_nt;
          if (dep < 0.0) dep = 0.0;
          const double gen = wp * rc.rho_nt * dep;            // w_av = 0
          const double Jl = fabs(E) > 1e-10 ? (gen * rc.Ui * E) / (E * E + 1e-20) : 0.0;
          const double nJ = Jf * rc.exp_nu + rc.e2m * rho * E * rc.step_J;
          S[tpad(t)].y = (Rl)(Jf + Jl) * inv_Es;
          rf_rho_step(rho, wp, rc, e_r, sf0);
          Jf = nJ;
        }
        goto scan_done;
      }
    }
    if (lane == 0) {   // the reference's serial loop
      double rho = 0.0, Jf = 0.0;
      for (int t = 0; t < NT; ++t) {
        const Rl Ef = R[t];
        const Rl I = Ic * (Ef * Ef);
        const double E = (double)(float)Ef;
        const double wp = (double)(float)lut_eval<Rl>(tb.lut, I);
        const double wa = (double)(float)(Av * I);
        double dep = (rc.rho_nt - rho) / rc.rho_nt;
        if (dep < 0.0) dep = 0.0;
        const double Se = wp * rc.rho_nt * dep;
        const double Ge = wa * dep - rc.rr;
        double gdt = Ge * rc.dt;
        if (gdt > 10.0) gdt = 10.0;
        if (gdt < -10.0) gdt = -10.0;
        const double eg = exp(gdt);
        const double sf = (fabs(gdt) < 1e-5) ? rc.dt * (1.0 + 0.5 * gdt) : (eg - 1.0) / Ge;
        double nr = rho * eg + Se * sf;
        if (nr > rc.rho_nt) nr = rc.rho_nt;
        if (nr < 0.0) nr = 0.0;
        const double gen = Se + wa * dep * rho;
        const double nJ = Jf * rc.exp_nu + rc.e2m * rho * E * rc.step_J;
        const double Jl = fabs(E) > 1e-10 ? (gen * rc.Ui * E) / (E * E + 1e-20) : 0.0;
        S[tpad(t)].y = (Rl)(Jf + Jl) / Es;       // J (solver precision) / E_scale
        rho = nr;
        Jf = nJ;
      }
    }
  scan_done:;
  }
  __syncwarp();
  const Rl c3 = (Rl)rc.chi3e, c5 = (Rl)rc.chi5e;
  for (int t = lane; t < NT; t += 32) {
    const Rl E = R[t];
    Rl P;
    if constexpr (RAMAN) P = (c3 * E) * Q[t];       // chi3_coef * E_t * E_eff_sq (:303-305)
    else P = ((c3 * E) * E) * E;
    if (rc.chi5e != 0.0) {
      const Rl E2 = E * E;
      P = P + ((c5 * E) * E2) * E2;
    }
    S[tpad(t)].x = P * inv_Es;
  }
  __syncwarp();
  // P and J (both real) share one complex transform, each scaled by its own line
  // maximum first: the polarisation can be many orders below the current, and an
  // unscaled packing would bury its spectrum in J's rounding
  Rl mp = (Rl)0, mj = (Rl)0;
  for (int t = lane; t < NT; t += 32) {
    const C pj = S[tpad(t)];
    mp = fmax(mp, fabs(pj.x));
    mj = fmax(mj, fabs(pj.y));
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    mp = fmax(mp, __shfl_xor_sync(0xffffffffu, mp, off));
    mj = fmax(mj, __shfl_xor_sync(0xffffffffu, mj, off));
  }
  const Rl sP = mp > (Rl)0 ? mp : (Rl)1, sJ = mj > (Rl)0 ? mj : (Rl)1;
  // divisions, not reciprocals: on weakly ionising lines the current's maximum is
  // a float32 subnormal whose reciprocal overflows
  for (int t = lane; t < NT; t += 32) {
    const C pj = S[tpad(t)];
    S[tpad(t)] = C{pj.x / sP, pj.y / sJ};
  }
  __syncwarp();
  stockham<NT, 1, TCfg<NT>::FT, -1, 1, C>(S, tw, lane, LineIdx(), WarpSync());    // F(P/sP + i J/sJ)
  C* o = reinterpret_cast<C*>(out) + line * Nw;
  const double kp2 = tb.kp2[line];
  const double cpl = 1.0 / (2.0 * 8.85418781e-12 * 299792458.0 * 299792458.0);
  for (int k = lane; k < Nw; k += 32) {
    if (k == 0 || k >= NR) { o[k] = C{0, 0}; continue; }   // DC source zeroed (solver_3d.py:95-97)
    const C z1 = S[tpad(k)], z2 = S[tpad((NT - k) % NT)];
    const double Pr = 0.5 * ((double)z1.x + z2.x) * sP, Pi = 0.5 * ((double)z1.y - z2.y) * sP;   // F(P)[k]
    const double Jr = 0.5 * ((double)z1.y + z2.y) * sJ, Ji = -0.5 * ((double)z1.x - z2.x) * sJ;  // F(J)[k]
    // kz: real root, or -i sqrt(|.|) for evanescent components; |kz| < 1e-10 -> 1e-10
    const double kz2 = tb.kk[k] - kp2;
    double kr, ki;
    if (kz2 >= 0.0) { kr = sqrt(kz2); ki = 0.0; } else { kr = 0.0; ki = -sqrt(-kz2); }
    if (sqrt(kr * kr + ki * ki) < 1e-10) { kr = 1e-10; ki = 0.0; }
    const double w = tb.w[k];
    const double den = kr * kr + ki * ki;
    const double ir = kr / den, ii = -ki / den;            // 1 / kz
    // Pc = -i w^2 cpl / kz ; Jc = -w cpl / kz
    const double pr = w * w * cpl * ii, pim = -w * w * cpl * ir;
    const double jr = -w * cpl * ir, ji = -w * cpl * ii;
    o[k] = C{(Rl)(pr * Pr - pim * Pi + jr * Jr - ji * Ji), (Rl)(pr * Pi + pim * Pr + jr * Ji + ji * Jr)};
  }
}

enum RfStage { RS_1 = 0, RS_2, RS_3, RS_4 };

struct RfBufs {
  void *ekw, *v, *a1, *ts, *el;   // E_kw and the stage accumulators (kx, ky, omega)
};

// Stage algebra of erk43_step (solver_3d.py:143-167) fused with the y transforms
// around it: the tile (Ny rows x kW omega columns at one kx) of x-transformed
// N(u) is transformed along y (giving the stage's N in (kx, ky, omega)), the
// stage algebra runs per element with exp((h/2) D), D = -i (kz - kref), formed in
// FP64, and the next stage input (or, in the last stage, the candidate E4) is
// transformed back along y and stored for the inverse x pass.  Per element:
//   RS_1: v = L(E_kw), a1 = L(k1), u = v + h/2 a1
//   RS_2: u = v + h/2 a2, ts = a1 + 2 a2, el = v + h/2 a1 + h/2 a2
//   RS_3: u = L(v + h a3), ts += 2 a3
//   RS_4: E4 = L(v + h/6 ts) + h/6 a4, E_low = L(el); max |E4 - E_low|, max |E4|
// Omega bins at or above Nt/2 + 1 (row padding) stay zero.
template <typename Rl, int N>
__global__ void __launch_bounds__(SpaceCfg<N>::NTHR, 1)
k_rf_ypass(int mode, RfTables tb, RfBufs b, int Nw, int NR, const void* in, void* out, const void* twy,
           double h, unsigned long long* red) {
  using C = typename CT<Rl>::T;
  constexpr int NTHR = SpaceCfg<N>::NTHR;
  constexpr int E = SpaceCfg<N>::E;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* tw = reinterpret_cast<C*>(smem_raw);
  C* s = tw + N;
  const int tid = threadIdx.x;
  for (int i = tid; i < N; i += NTHR) tw[i] = reinterpret_cast<const C*>(twy)[i];
  const int ntile = Nw / kW;
  const int o = blockIdx.x / ntile;            // kx index
  const int w0 = (blockIdx.x % ntile) * kW;    // omega offset
  const long long stride = Nw;
  const long long base = (long long)o * N * Nw + w0;
  TileIdx<C> idx;
  BlockSync sync;
  load_tile<C, N, NTHR>(s, reinterpret_cast<const C*>(in), base, stride, tid);
  __syncthreads();
  stockham<N, kW, NTHR, -1, 1, C>(s, tw, tid, idx, sync);
  C *ekw = (C*)b.ekw, *v = (C*)b.v, *a1 = (C*)b.a1, *ts = (C*)b.ts, *el = (C*)b.el;
  const Rl h2 = (Rl)(h / 2), h6 = (Rl)(h / 6), hR = (Rl)h;
  double mdiff = 0.0, mnorm = 0.0;
#pragma unroll
  for (int i = 0; i < E; ++i) {
    const int e = tid + i * NTHR;
    const int n = e / kW, w = e % kW;            // n = ky
    const int k = w0 + w;
    const long long gi = base + n * stride + w;
    if (k >= NR) { s[idx(w, n)] = C{(Rl)0, (Rl)0}; continue; }
    const double kz2 = tb.kk[k] - tb.kp2[(long long)o * N + n];
    const double sh = 0.5 * h;
    double mag = 1.0, ph;
    if (kz2 >= 0.0) ph = -(sqrt(kz2) - tb.kref[k]) * sh;
    else { mag = exp(-sqrt(-kz2) * sh); ph = tb.kref[k] * sh; }
    double sn, cs;
    sincos(ph, &sn, &cs);
    const C Ef = C{(Rl)(mag * cs), (Rl)(mag * sn)};
    const C a = s[idx(w, n)];                    // this stage's N in (kx, ky, omega)
    C u;
    if (mode == RS_1) {
      const C vv = cmul(ekw[gi], Ef), aa = cmul(a, Ef);
      v[gi] = vv;
      a1[gi] = aa;
      u = cadd(vv, cscale(aa, h2));
    } else if (mode == RS_2) {
      const C vv = v[gi], aa = a1[gi];
      u = cadd(vv, cscale(a, h2));
      ts[gi] = cadd(aa, cscale(a, (Rl)2));
      el[gi] = cadd(cadd(vv, cscale(aa, h2)), cscale(a, h2));
    } else if (mode == RS_3) {
      u = cmul(cadd(v[gi], cscale(a, hR)), Ef);
      ts[gi] = cadd(ts[gi], cscale(a, (Rl)2));
    } else {
      const C E4 = cadd(cmul(cadd(v[gi], cscale(ts[gi], h6)), Ef), cscale(a, h6));
      const C El = cmul(el[gi], Ef);
      const double dx = (double)E4.x - El.x, dy = (double)E4.y - El.y;
      // maxima of the squares; the roots are taken once per warp below
      const double d = dx * dx + dy * dy, m = (double)E4.x * E4.x + (double)E4.y * E4.y;
      mdiff = (d > mdiff || d != d) ? d : mdiff;
      mnorm = (m > mnorm || m != m) ? m : mnorm;
      u = E4;
    }
    s[idx(w, n)] = u;
  }
  if (mode == RS_4) {
    // blocks of fewer than 32 threads (Ny = 16) reduce over their own lanes only
    mdiff = sqrt(warp_max<(NTHR < 32 ? NTHR : 32)>(mdiff));
    mnorm = sqrt(warp_max<(NTHR < 32 ? NTHR : 32)>(mnorm));
    if ((threadIdx.x & 31) == 0) { atomic_max_nonneg(&red[0], mdiff); atomic_max_nonneg(&red[1], mnorm); }
  }
  __syncthreads();
  stockham<N, kW, NTHR, +1, 1, C>(s, tw, tid, idx, sync);
  store_tile<C, N, NTHR>(s, reinterpret_cast<C*>(out), base, stride, tid);
}

template <typename Rl, int N> static size_t rf_ypass_smem() {
  return sizeof(typename CT<Rl>::T) * (size_t)(N + N * kW);
}

template <typename Rl>
__global__ void k_rf_absmax(const Rl* e, long long n, unsigned long long* red) {
  double m = 0.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double a = fabs((double)e[i]);
    m = a > m ? a : m;
  }
  m = warp_max<32>(m);
  if ((threadIdx.x & 31) == 0) atomic_max_nonneg(red, m);
}

// float32 field arithmetic as the reference does it: E0 / float32(E_scale) and
// E * float32(E_scale)
__global__ void k_rf_div_f32(const float* in, float* out, long long n, float s) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = in[i] / s;
}
__global__ void k_rf_mul_f32(const float* in, float* out, long long n, float s) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = in[i] * s;
}

template <typename Rl>
__global__ void k_rf_scale(const Rl* in, Rl* out, long long n, double s) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = (Rl)((double)in[i] * s);
}
}  // namespace uppe

struct uppe_rf_plan {
  uppe_rf_desc d;
  int dbl, Nw;
  size_t csz, rsz;
  long long nspec, nreal;
  uppe3d_plan* xy;        // transform plan of the x and y passes (omega extent Nw)
  RfTables tb;
  RfConst rc;
  RfBufs b;
  void* state[2];         // accepted / candidate real field (normalised)
  void* tmp[2];           // spectral temporaries
  unsigned long long* red;
  unsigned long long* red_host;
  const void* twt;
  std::vector<void*> allocs;
  int cur = 0;
  double h_last = 0.0;
  bool raman = false;
};

static int rf_alloc(uppe_rf_plan* p, void** dst, size_t bytes, const void* src = nullptr) {
  UPPE_CK(cudaMalloc(dst, bytes));
  p->allocs.push_back(*dst);
  if (src) UPPE_CK(cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice));
  else UPPE_CK(cudaMemset(*dst, 0, bytes));
  return 0;
}

extern "C" int uppe_rf_plan_destroy(uppe_rf_plan* p) {
  if (!p) return 0;
  if (p->xy) uppe3d_plan_destroy(p->xy);
  for (void* a : p->allocs) cudaFree(a);
  if (p->red_host) cudaFreeHost(p->red_host);
  delete p;
  return 0;
}

template <typename Rl, int N> static cudaError_t rf_ypass_attr() {
  return cudaFuncSetAttribute(k_rf_ypass<Rl, N>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)rf_ypass_smem<Rl, N>());
}

template <typename Rl> static int rf_set_attrs(int Nx, int Ny, int Nt) {
  cudaError_t e = cudaSuccess;
  switch (Ny) {
    case 16: e = rf_ypass_attr<Rl, 16>(); break;
    case 32: e = rf_ypass_attr<Rl, 32>(); break;
    case 64: e = rf_ypass_attr<Rl, 64>(); break;
    case 128: e = rf_ypass_attr<Rl, 128>(); break;
    case 256: e = rf_ypass_attr<Rl, 256>(); break;
    case 512: e = rf_ypass_attr<Rl, 512>(); break;
    default: return UPPE_ERR_SIZE;
  }
  UPPE_CK(e);
  for (int N : {Nx, Ny}) {
    switch (N) {
      case 16: e = set_space_attr<Rl, 16>(); break;
      case 32: e = set_space_attr<Rl, 32>(); break;
      case 64: e = set_space_attr<Rl, 64>(); break;
      case 128: e = set_space_attr<Rl, 128>(); break;
      case 256: e = set_space_attr<Rl, 256>(); break;
      case 512: e = set_space_attr<Rl, 512>(); break;
      default: return UPPE_ERR_SIZE;
    }
    if (e != cudaSuccess) break;
  }
  UPPE_CK(e);
  (void)Nt;
  return 0;
}

extern "C" int uppe_rf_plan_create(const uppe_rf_desc* d, uppe_rf_plan** out) {
  *out = nullptr;
  g_uppe_err[0] = 0;
  if (!d) return UPPE_ERR_ARG;
  if (!is_pow2(d->Nx) || !is_pow2(d->Ny) || !is_pow2(d->Nt) || d->Nx < 16 || d->Ny < 16 || d->Nx > 512 ||
      d->Ny > 512 || d->Nt < 64 || d->Nt > 2048) {
    snprintf(g_uppe_err, sizeof(g_uppe_err), "unsupported real-field grid %dx%dx%d", d->Nx, d->Ny, d->Nt);
    return UPPE_ERR_SIZE;
  }
  if (d->precision != UPPE_C64 && d->precision != UPPE_C128) return UPPE_ERR_ARG;
  if (d->precision == UPPE_C128 && (d->Nx > 256 || d->Ny > 256)) return UPPE_ERR_SIZE;
  if (d->lut_n < 2 || !d->lut_log10I || !d->lut_W || !d->kk || !d->kref || !d->w || !d->filt || !d->kperp2 ||
      !d->damp)
    return UPPE_ERR_ARG;
  uppe_rf_plan* p = new uppe_rf_plan();
  p->d = *d;
  p->dbl = d->precision == UPPE_C128;
  p->csz = p->dbl ? 16 : 8;
  p->rsz = p->dbl ? 8 : 4;
  p->Nw = d->Nt / 2 + kW;
  const int Nr = d->Nt / 2 + 1;
  p->nspec = (long long)d->Nx * d->Ny * p->Nw;
  p->nreal = (long long)d->Nx * d->Ny * d->Nt;
  int rc = 0;
#define RF_TRY(x) do { rc = (x); if (rc) { uppe_rf_plan_destroy(p); return rc; } } while (0)
  // transform plan: geometry (Nx, Ny, Nw), twiddles, a device state that is never "done"
  {
    uppe3d_plan* q = new uppe3d_plan();
    p->xy = q;
    q->g.Nx = d->Nx; q->g.Ny = d->Ny; q->g.Nt = p->Nw;
    q->g.npts = p->nspec;
    q->dbl = p->dbl;
    q->csz = p->csz;
    cudaError_t e = cudaMalloc(&q->st, sizeof(State3D));
    if (e != cudaSuccess) { uppe_rf_plan_destroy(p); return UPPE_ERR_CUDA; }
    q->allocs.push_back(q->st);
    e = cudaMallocHost(&q->st_host, sizeof(State3D));
    if (e != cudaSuccess) { uppe_rf_plan_destroy(p); return UPPE_ERR_CUDA; }
    memset(q->st_host, 0, sizeof(State3D));
    e = cudaMemcpy(q->st, q->st_host, sizeof(State3D), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) { uppe_rf_plan_destroy(p); return UPPE_ERR_CUDA; }
    void* ptr = nullptr;
    auto tx = p->dbl ? twiddles<double>(d->Nx) : twiddles<float>(d->Nx);
    auto ty = p->dbl ? twiddles<double>(d->Ny) : twiddles<float>(d->Ny);
    auto tt = p->dbl ? twiddles<double>(d->Nt) : twiddles<float>(d->Nt);
    RF_TRY(dev_upload(q, &ptr, tx.data(), tx.size())); q->tb.twx = ptr;
    RF_TRY(dev_upload(q, &ptr, ty.data(), ty.size())); q->tb.twy = ptr;
    RF_TRY(dev_upload(q, &ptr, tt.data(), tt.size())); p->twt = ptr;
    RF_TRY(p->dbl ? rf_set_attrs<double>(d->Nx, d->Ny, d->Nt) : rf_set_attrs<float>(d->Nx, d->Ny, d->Nt));
  }
  void* ptr = nullptr;
  RF_TRY(rf_alloc(p, &ptr, 8 * Nr, d->kk)); p->tb.kk = (const double*)ptr;
  RF_TRY(rf_alloc(p, &ptr, 8 * Nr, d->kref)); p->tb.kref = (const double*)ptr;
  RF_TRY(rf_alloc(p, &ptr, 8 * Nr, d->w)); p->tb.w = (const double*)ptr;
  RF_TRY(rf_alloc(p, &ptr, 8 * Nr, d->filt)); p->tb.filt = (const double*)ptr;
  RF_TRY(rf_alloc(p, &ptr, 8 * (size_t)d->Nx * d->Ny, d->kperp2)); p->tb.kp2 = (const double*)ptr;
  RF_TRY(rf_alloc(p, &ptr, 8 * (size_t)d->Nx * d->Ny, d->damp)); p->tb.damp = (const double*)ptr;
  {
    const int n = d->lut_n;
    std::vector<unsigned char> lx(n * p->rsz), lw(n * p->rsz);
    for (int i = 0; i < n; ++i) {
      if (p->dbl) { ((double*)lx.data())[i] = d->lut_log10I[i]; ((double*)lw.data())[i] = d->lut_W[i]; }
      else { ((float*)lx.data())[i] = (float)d->lut_log10I[i]; ((float*)lw.data())[i] = (float)d->lut_W[i]; }
    }
    RF_TRY(rf_alloc(p, &ptr, lx.size(), lx.data())); p->tb.lut.x = ptr;
    RF_TRY(rf_alloc(p, &ptr, lw.size(), lw.data())); p->tb.lut.w = ptr;
    {
      std::vector<double> sl(n - 1);
      if (p->dbl) lut_slopes<double>(d->lut_log10I, d->lut_W, n, sl.data());
      else lut_slopes<float>(d->lut_log10I, d->lut_W, n, sl.data());
      RF_TRY(rf_alloc(p, &ptr, sl.size() * sizeof(double), sl.data()));
      p->tb.lut.slope = static_cast<const double*>(ptr);
    }
    p->tb.lut.n = n;
    const double x0 = p->dbl ? d->lut_log10I[0] : (double)(float)d->lut_log10I[0];
    const double x1 = p->dbl ? d->lut_log10I[n - 1] : (double)(float)d->lut_log10I[n - 1];
    p->tb.lut.x0 = x0;
    p->tb.lut.inv_dx = (n - 1) / (x1 - x0);
    int j0 = -1;
    for (int i = 0; i < n; ++i) {
      const double wv = p->dbl ? d->lut_W[i] : (double)(float)d->lut_W[i];
      if (wv != 0.0) break;
      j0 = i;
    }
    p->tb.lut.zero_x = j0 < 0 ? -INFINITY : (p->dbl ? d->lut_log10I[j0] : (double)(float)d->lut_log10I[j0]);
    if (j0 == n - 1) p->tb.lut.zero_x = INFINITY;
    p->tb.lut.I_zero = lut_zero_intensity(p->tb.lut.zero_x);
  }
  RfConst& c = p->rc;
  c.I_coef = d->I_coef; c.aval = d->aval_coef; c.chi3e = d->chi3e; c.chi5e = d->chi5e;
  c.rr = (double)(float)d->rate_rec; c.dt = (double)(float)d->dt; c.rho_nt = (double)(float)d->rho_nt;
  c.inv_rho_nt = 1.0 / c.rho_nt;
  c.Ui = (double)(float)d->Ui;
  const double e = (double)(float)d->e_charge, me = (double)(float)d->m_e, tc = (double)(float)d->tau_c;
  c.e2m = e * e / me;
  c.nu = 1.0 / tc;
  const double ndt = c.nu * c.dt;
  c.exp_nu = exp(-ndt);
  c.step_J = (fabs(ndt) < 1e-5) ? c.dt * (1.0 - 0.5 * ndt) : (1.0 - c.exp_nu) / c.nu;
  c.E_scale = 1.0;
  c.fR = 0.0;
  p->tb.ramH = p->tb.ramW = nullptr;
  if (d->raman_H) {
    // H_k as given; W_k = exp(-i pi k / Nt) in extended precision, rounded once
    const int Nt = d->Nt;
    std::vector<unsigned char> hb((Nt + 1) * p->csz), wb((Nt / 2 + 1) * p->csz);
    for (int k = 0; k <= Nt; ++k) {
      if (p->dbl) { ((double*)hb.data())[2 * k] = d->raman_H[2 * k]; ((double*)hb.data())[2 * k + 1] = d->raman_H[2 * k + 1]; }
      else { ((float*)hb.data())[2 * k] = (float)d->raman_H[2 * k]; ((float*)hb.data())[2 * k + 1] = (float)d->raman_H[2 * k + 1]; }
    }
    for (int k = 0; k <= Nt / 2; ++k) {
      const long double ang = -3.141592653589793238462643383279502884L * (long double)k / (long double)Nt;
      const double cr = (double)cosl(ang), ci = (double)sinl(ang);
      if (p->dbl) { ((double*)wb.data())[2 * k] = cr; ((double*)wb.data())[2 * k + 1] = ci; }
      else { ((float*)wb.data())[2 * k] = (float)cr; ((float*)wb.data())[2 * k + 1] = (float)ci; }
    }
    RF_TRY(rf_alloc(p, &ptr, hb.size(), hb.data())); p->tb.ramH = ptr;
    RF_TRY(rf_alloc(p, &ptr, wb.size(), wb.data())); p->tb.ramW = ptr;
    c.fR = d->raman_fR;
    p->raman = true;
  }
  void** spec[5] = {&p->b.ekw, &p->b.v, &p->b.a1, &p->b.ts, &p->b.el};
  for (int i = 0; i < 5; ++i) RF_TRY(rf_alloc(p, spec[i], p->csz * p->nspec));
  RF_TRY(rf_alloc(p, &p->tmp[0], p->csz * p->nspec));
  RF_TRY(rf_alloc(p, &p->tmp[1], p->csz * p->nspec));
  RF_TRY(rf_alloc(p, &p->state[0], p->rsz * p->nreal));
  RF_TRY(rf_alloc(p, &p->state[1], p->rsz * p->nreal));
  RF_TRY(rf_alloc(p, &ptr, 4 * sizeof(unsigned long long))); p->red = (unsigned long long*)ptr;
  if (cudaMallocHost(&p->red_host, 4 * sizeof(unsigned long long)) != cudaSuccess) { uppe_rf_plan_destroy(p); return UPPE_ERR_CUDA; }
#undef RF_TRY
  *out = p;
  return 0;
}

template <typename Rl, int NT, bool RAMAN>
static int rf_line_nr(uppe_rf_plan* p, int mode, const void* in, void* out, double in_scale, double h, cudaStream_t s) {
  using LS = RfLaunch<NT, Rl, RAMAN>;
  constexpr int WPB = LS::WPB;
  const size_t smem = LS::smem();
  UPPE_CK(cudaFuncSetAttribute(k_rf_line<Rl, NT, WPB, RAMAN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  Geom g;
  g.Nx = p->d.Nx; g.Ny = p->d.Ny; g.Nt = p->d.Nt; g.npts = p->nreal;
  const long long nl = (long long)g.Nx * g.Ny;
  k_rf_line<Rl, NT, WPB, RAMAN><<<(unsigned)((nl + WPB - 1) / WPB), WPB * 32, smem, s>>>(
      mode, p->tb, p->rc, g, p->Nw, in, out, p->twt, in_scale, h);
  UPPE_CK(cudaGetLastError());
  return 0;
}

template <typename Rl, int NT>
static int rf_line_n(uppe_rf_plan* p, int mode, const void* in, void* out, double in_scale, double h, cudaStream_t s) {
  // only the nonlinear response uses the Raman term
  if (p->raman && mode == RF_NL) return rf_line_nr<Rl, NT, true>(p, mode, in, out, in_scale, h, s);
  return rf_line_nr<Rl, NT, false>(p, mode, in, out, in_scale, h, s);
}

template <typename Rl>
static int rf_line(uppe_rf_plan* p, int mode, const void* in, void* out, double in_scale, double h, cudaStream_t s) {
  switch (p->d.Nt) {
#define UPPE_RL(n) case n: return rf_line_n<Rl, n>(p, mode, in, out, in_scale, h, s);
    UPPE_RL(64) UPPE_RL(128) UPPE_RL(256) UPPE_RL(512) UPPE_RL(1024) UPPE_RL(2048)
#undef UPPE_RL
    default: return UPPE_ERR_SIZE;
  }
}

// one stage: the stage input of this evaluation (already transformed back along y,
// in tmp[0]) -> inverse x pass -> nonlinear response per t-line (solver_3d.py:120-141)
// -> forward x pass -> y pass with the stage algebra, which leaves the next stage
// input (transformed back along y) in tmp[0]
template <typename Rl, int N>
static int rf_ypass_n(uppe_rf_plan* p, int mode, double h, cudaStream_t s) {
  const unsigned nb = (unsigned)((long long)p->d.Nx * (p->Nw / kW));
  k_rf_ypass<Rl, N><<<nb, SpaceCfg<N>::NTHR, rf_ypass_smem<Rl, N>(), s>>>(
      mode, p->tb, p->b, p->Nw, p->d.Nt / 2 + 1, p->tmp[1], p->tmp[0], p->xy->tb.twy, h, p->red);
  UPPE_CK(cudaGetLastError());
  return 0;
}

template <typename Rl>
static int rf_stage(uppe_rf_plan* p, int mode, double h, cudaStream_t s) {
  uppe3d_plan* q = p->xy;
  int rc = 0;
  rc |= launch_space<Rl>(q, XINV, p->tmp[0], p->tmp[1], s);
  rc |= rf_line<Rl>(p, RF_NL, p->tmp[1], p->tmp[0], 1.0 / ((double)p->d.Nx * p->d.Ny), 0.0, s);
  rc |= launch_space<Rl>(q, XFWD, p->tmp[0], p->tmp[1], s);
  if (rc) return rc;
  switch (p->d.Ny) {
#define UPPE_RY(n) case n: return rf_ypass_n<Rl, n>(p, mode, h, s);
    UPPE_RY(16) UPPE_RY(32) UPPE_RY(64) UPPE_RY(128) UPPE_RY(256) UPPE_RY(512)
#undef UPPE_RY
    default: return UPPE_ERR_SIZE;
  }
}

template <typename Rl>
static int rf_attempt(uppe_rf_plan* p, double h, double* err, cudaStream_t s) {
  uppe3d_plan* q = p->xy;
  int rc = 0;
  // E_kw = fft2(rfft(E_t)); the first stage's N(E_kw) starts from its inverse y transform
  rc |= rf_line<Rl>(p, RF_FROM_T, p->state[p->cur], p->tmp[0], 1.0, 0.0, s);
  rc |= launch_space<Rl>(q, XFWD, p->tmp[0], p->tmp[1], s);
  rc |= adj_plain_y<Rl>(q, YPLAIN_FWD, p->tmp[1], p->b.ekw, 1.0, s);
  rc |= adj_plain_y<Rl>(q, YPLAIN_INV, p->b.ekw, p->tmp[0], 1.0, s);
  rc |= rf_stage<Rl>(p, RS_1, h, s);                    // k1 -> u2
  rc |= rf_stage<Rl>(p, RS_2, h, s);                    // alpha2 -> u3
  rc |= rf_stage<Rl>(p, RS_3, h, s);                    // alpha3 -> u4
  UPPE_CK(cudaMemsetAsync(p->red, 0, 2 * sizeof(unsigned long long), s));
  rc |= rf_stage<Rl>(p, RS_4, h, s);                    // alpha4' -> E4, error
  // candidate: irfft(ifft2(E4) * filter) * exp(-damp h)
  rc |= launch_space<Rl>(q, XINV, p->tmp[0], p->tmp[1], s);
  rc |= rf_line<Rl>(p, RF_OUT, p->tmp[1], p->state[p->cur ^ 1], 1.0 / ((double)p->d.Nx * p->d.Ny), h, s);
  UPPE_CK(cudaMemcpyAsync(p->red_host, p->red, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
  UPPE_CK(cudaStreamSynchronize(s));
  double md, mn;
  memcpy(&md, &p->red_host[0], 8);
  memcpy(&mn, &p->red_host[1], 8);
  *err = md / (mn + 1e-20);
  p->h_last = h;
  return rc;
}

extern "C" int uppe_rf_set_field(uppe_rf_plan* p, const void* E0, double* E_scale, cudaStream_t s) {
  if (!p || !E0) return UPPE_ERR_ARG;
  UPPE_CK(cudaMemsetAsync(p->red, 0, sizeof(unsigned long long), s));
  if (p->dbl) k_rf_absmax<double><<<148 * 4, 256, 0, s>>>((const double*)E0, p->nreal, p->red);
  else k_rf_absmax<float><<<148 * 4, 256, 0, s>>>((const float*)E0, p->nreal, p->red);
  UPPE_CK(cudaMemcpyAsync(p->red_host, p->red, sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
  UPPE_CK(cudaStreamSynchronize(s));
  double m;
  memcpy(&m, &p->red_host[0], 8);
  if (!p->dbl) m = (double)(float)m;   // max|E0| of the float32 field, as float32 (solver_3d.py:180)
  double sc = m < 1e-30 ? 1.0 : m;
  p->rc.E_scale = sc;
  p->cur = 0;
  // E = E0 / E_scale in the field precision
  const double inv = p->dbl ? 1.0 / sc : 1.0;
  if (p->dbl) k_rf_scale<double><<<148 * 4, 256, 0, s>>>((const double*)E0, (double*)p->state[0], p->nreal, inv);
  else k_rf_div_f32<<<148 * 4, 256, 0, s>>>((const float*)E0, (float*)p->state[0], p->nreal, (float)sc);
  UPPE_CK(cudaGetLastError());
  if (E_scale) *E_scale = sc;
  return 0;
}

extern "C" int uppe_rf_attempt(uppe_rf_plan* p, double h, double* err, cudaStream_t s) {
  NvtxRange nvtx_range("uppe_rf_attempt");
  if (!p || !err || !(h > 0.0)) return UPPE_ERR_ARG;
  return p->dbl ? rf_attempt<double>(p, h, err, s) : rf_attempt<float>(p, h, err, s);
}

extern "C" int uppe_rf_commit(uppe_rf_plan* p, int accept, cudaStream_t s) {
  (void)s;
  if (!p) return UPPE_ERR_ARG;
  if (accept) p->cur ^= 1;
  return 0;
}

extern "C" int uppe_rf_get_field(uppe_rf_plan* p, void* out, cudaStream_t s) {
  if (!p || !out) return UPPE_ERR_ARG;
  if (p->dbl) k_rf_scale<double><<<148 * 4, 256, 0, s>>>((const double*)p->state[p->cur], (double*)out, p->nreal, p->rc.E_scale);
  else k_rf_mul_f32<<<148 * 4, 256, 0, s>>>((const float*)p->state[p->cur], (float*)out, p->nreal, (float)p->rc.E_scale);
  UPPE_CK(cudaGetLastError());
  return 0;
}

extern "C" int uppe_rf_get_spectrum(uppe_rf_plan* p, void* out, cudaStream_t s) {
  if (!p || !out) return UPPE_ERR_ARG;
  // rfft(E * E_scale) per line into rows of Nw bins (the candidate buffer is scratch here)
  int rc = uppe_rf_get_field(p, p->state[p->cur ^ 1], s);
  if (rc) return rc;
  return p->dbl ? rf_line<double>(p, RF_FROM_T, p->state[p->cur ^ 1], out, 1.0, 0.0, s)
                : rf_line<float>(p, RF_FROM_T, p->state[p->cur ^ 1], out, 1.0, 0.0, s);
}

extern "C" int uppe_rf_spec_bins(const uppe_rf_plan* p) { return p ? p->Nw : 0; }
