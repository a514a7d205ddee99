/* C ABI of the B200-native ERK4(3)-IP UPPE/GNLSE propagator (libuppe_b200.so).
 *
 * All field pointers are caller-owned DEVICE memory (e.g. torch tensors); every
 * call takes a CUDA stream; no C++ exception crosses this boundary.  Functions
 * return 0 on success or a negative UPPE_ERR_* code; uppe_last_error() gives a
 * one-line message.  Per-run solver conditions (non-finite error, forced steps
 * at min_step, attempt budget) are reported as UPPE_STATUS_* bits in the result.
 *
 * The reference is a Python research code with no FFI; each entry point below
 * names the reference function whose behaviour it replaces.
 */
#ifndef UPPE_B200_H
#define UPPE_B200_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* uppe_stream_t; /* == cudaStream_t */

enum { UPPE_C64 = 0, UPPE_C128 = 1 };

enum {
  UPPE_OK = 0,
  UPPE_ERR_ARG = -1,
  UPPE_ERR_SIZE = -2,
  UPPE_ERR_CUDA = -3
};

enum {
  UPPE_STATUS_NONFINITE = 1,     /* error or step size became NaN/inf: stopped   */
  UPPE_STATUS_MIN_STEP = 2,      /* a step was forced at min_step with err > tol */
  UPPE_STATUS_MAX_ATTEMPTS = 4,  /* attempt budget exhausted before z = L         */
  UPPE_STATUS_RETRIED = 64,      /* an attempt came out non-finite and was retried with
                                    a tenth of the step (the reference loops on h = NaN) */
  UPPE_STATUS_DEVICE_WAIT = 32   /* a bounded device wait ran out: run stopped     */
};

/* Attempt budget used when a caller passes max_attempts <= 0: every propagation
 * on the device is bounded.  min_step must be > 0. */
#define UPPE_DEFAULT_MAX_ATTEMPTS 2000000LL

/* Last error message of this library (thread-global, one line). */
const char* uppe_last_error(void);

/* ------------------------------------------------------------------ 3+1D ---- */
/* Grid, precomputed FP64 tables and medium constants of
 * ERK43IP_UPPE_3D_Optimized.__init__ (src/3+1D-UPPE-ERK4(3)IP-envelope/
 * solver_3d.py:8-98) and of the OpticalMedium plugin (media_physics.py:70-205).
 * Host pointers; copied into the plan. */
typedef struct {
  int Nx, Ny, Nt;          /* powers of two: Nx, Ny in [16,512], Nt in [32,2048] */
  int precision;           /* UPPE_C64 (mixed: FP64 phase/error/controller) or UPPE_C128 */
  double dt;               /* t[1]-t[0]                                            */
  const double* aw;        /* [Nt] k^2 - kref^2  (solver_3d.py:76-82)              */
  const double* ksq;       /* [Nt] k^2                                             */
  const double* kref;      /* [Nt] k0 + k1 omega (solver_3d.py:71-74)              */
  const unsigned char* valid; /* [Nt] omega + omega0 > 0 (solver_3d.py:53-54,86)   */
  const double* shock;     /* [Nt] (omega+omega0)/omega0 or 1 (media_physics.py:113-119) */
  const double* filt;      /* [Nt] anti-alias filter (solver_3d.py:47-50)          */
  const double* kperp2;    /* [Nx*Ny] kx^2+ky^2, index ix*Ny+iy (solver_3d.py:28-32) */
  const double* damp;      /* [Nx*Ny] absorber (solver_3d.py:89-98)                */
  int lut_n;               /* ionisation LUT (media_physics.py:121-137)            */
  const double* lut_log10I;/* [lut_n] uniform grid of log10(I [W/m^2])             */
  const double* lut_W;     /* [lut_n] rate [1/s]                                   */
  double gamma_kerr;       /* (omega0/c) n2        (media_physics.py:192)          */
  double gamma_hoke;       /* (omega0/c) n4        (media_physics.py:194-196)      */
  double Ui;               /* ionisation energy [J]                                */
  double sigma_drude;      /* [m^2]                                                */
  double omega0_tau_c;
  double rate_rec;         /* 1/tau_rec (rounded to float32 as in :185)            */
  double rho_nt;           /* neutral density (rounded to float32 as in :187)      */
  double ava_coef;         /* W_ava = ava_coef * I (0 for the gases)               */
  int plasma_on;           /* 0 disables the plasma terms                          */
  const double* omega_abs; /* [Nt] omega + omega0 (photon number; NULL: not computed) */
} uppe3d_desc;

typedef struct {
  double z;                /* distance reached                                     */
  double h;                /* next step size                                       */
  double err;              /* error of the last attempt                            */
  long long attempts;      /* ERK attempts (accepted + rejected)                   */
  long long accepted;
  int fail_count;          /* consecutive forced steps at min_step                 */
  int status;              /* UPPE_STATUS_* bits                                   */
  double A_scale;          /* max|A0| normalisation (solver_3d.py:166)             */
} uppe3d_result;

typedef struct uppe3d_plan uppe3d_plan;

/* Replaces ERK43IP_UPPE_3D_Optimized.__init__ (solver_3d.py:8-54): uploads the
 * tables, allocates the plan's field buffers and captures the CUDA graphs of one
 * ERK attempt.  No allocation happens in later calls. */
int uppe3d_plan_create(const uppe3d_desc* desc, uppe3d_plan** plan);
int uppe3d_plan_destroy(uppe3d_plan* plan);
/* Bytes of one complex field of the plan's grid and precision. */
long long uppe3d_field_bytes(const uppe3d_plan* plan);

/* Start of propagate (solver_3d.py:163-170): A_scale = max|A0|, state = A0/A_scale.
 * A0: device [Nx][Ny][Nt] time-domain field in the plan's precision. */
int uppe3d_set_field(uppe3d_plan* plan, const void* A0, uppe_stream_t stream);

/* One erk43_step (solver_3d.py:100-160) of size h from the current state; writes
 * the attempt's error (synchronises the stream). */
int uppe3d_attempt(uppe3d_plan* plan, double h, double* err, uppe_stream_t stream);
/* Accept (state <- attempt output, z += h) or reject the last attempt. */
int uppe3d_commit(uppe3d_plan* plan, int accept, uppe_stream_t stream);

/* The adaptive loop of propagate (solver_3d.py:172-208), run on the device:
 * step-size control and acceptance happen in device kernels; the host only
 * polls for completion.  max_attempts <= 0 means UPPE_DEFAULT_MAX_ATTEMPTS;
 * tol, max_step and min_step must be > 0. */
int uppe3d_propagate(uppe3d_plan* plan, double L, double tol, double max_step, double min_step,
                     long long max_attempts, uppe3d_result* result, uppe_stream_t stream);
/* Split form of uppe3d_propagate for timing: begin, then nsteps graph launches. */
int uppe3d_begin(uppe3d_plan* plan, double L, double tol, double max_step, double min_step,
                 long long max_attempts, uppe_stream_t stream);
int uppe3d_run_steps(uppe3d_plan* plan, int nsteps, uppe_stream_t stream);
int uppe3d_get_result(uppe3d_plan* plan, uppe3d_result* result, uppe_stream_t stream);

/* Continuation of an adaptive run (no reference counterpart; the reference's drivers
 * restart propagate from the last field, which resets the step size): the state
 * between two attempts.  uppe3d_save_state copies it out (field_out: device buffer
 * of uppe3d_field_bytes, the accepted state in the plan's layout, normalised by
 * A_scale); uppe3d_load_state puts it into a plan of the same grid, precision and
 * medium, after which uppe3d_resume (or uppe3d_run_steps) continues the run with the
 * same attempts, step sizes and fields as the uninterrupted run, bit for bit. */
typedef struct {
  double z, h, L, tol, max_step, min_step;
  double err;              /* error of the last attempt                            */
  double A_scale;
  double peak_ion;         /* running max of rho / rho_nt                           */
  long long attempts, accepted, max_attempts;
  int fail_count, status, done;
} uppe3d_state;
int uppe3d_save_state(uppe3d_plan* plan, void* field_out, uppe3d_state* state, uppe_stream_t stream);
int uppe3d_load_state(uppe3d_plan* plan, const void* field_in, const uppe3d_state* state, uppe_stream_t stream);
/* The adaptive loop of uppe3d_propagate from the plan's current state (after
 * uppe3d_load_state or uppe3d_begin + uppe3d_run_steps). */
int uppe3d_resume(uppe3d_plan* plan, uppe3d_result* result, uppe_stream_t stream);

/* End of propagate (solver_3d.py:215-222): out = fftshift_t(fft_t(A * A_scale)). */
int uppe3d_get_spectrum(uppe3d_plan* plan, void* out, uppe_stream_t stream);
/* Time-domain field A(x, y, t) of the current state (physical units), for
 * chaining segments as the reference's drivers do with the returned field. */
int uppe3d_get_field(uppe3d_plan* plan, void* out, uppe_stream_t stream);

/* -------------------------------------------------------------------- 1D ---- */
/* One propagation of ERK43IP_UPPE.propagate (src/1D-ERK4(3)IP UPPE gas/
 * erk43ip_method.py:288-369).  Many instances with different Nt and parameters
 * run in one persistent launch. */
typedef struct {
  int Nt;                  /* power of two: [64,16384]; complex128 above 8192 only when
                              every line of the plan is 2048..16384 points, without Raman
                              or history (the four-CTA cluster kernel)                 */
  double dt;               /* t[1]-t[0]                                                */
  double L, tol, max_step, min_step;   /* propagate() arguments (:288)                */
  long long max_attempts;  /* <= 0: UPPE_DEFAULT_MAX_ATTEMPTS                          */
  int raman;               /* Raman convolution with H_R (erk43ip_method.py:150-179, 208-215) */
  int plasma;              /* envelope plasma term with I = |A|^2 / A_eff              */
  double f_R;
  double A_eff;            /* [m^2] for the plasma intensity                          */
  double Ui, sigma_drude, omega0_tau_c, rate_rec, rho_nt, ava_coef;   /* plasma constants */
  int hist_cap;            /* history slots (the reference saves <= 1501); 0 = none   */
  double omega0;           /* carrier angular frequency (photon number; 0: not computed) */
  double cost;             /* expected cost for the work queue (longest first); <= 0: Nt L */
} uppe1d_inst_desc;

typedef struct {
  int n_inst;
  int precision;           /* UPPE_C64 (mixed: FP64 phase/error/controller) or UPPE_C128 */
  const uppe1d_inst_desc* inst;
  const double* D;         /* packed complex [sum Nt]: D(omega) = i(k - k0 - k1 w) - alpha/2 (:104-148) */
  const double* G;         /* packed [sum Nt]: gamma * (w_abs/w0)(n0/n(w)) or gamma (:244-255) */
  const double* H;         /* packed complex [sum Nt]: H_R(omega), required if any raman */
  int lut_n;               /* ionisation LUT for the plasma term                       */
  const double* lut_log10I;
  const double* lut_W;
} uppe1d_desc;

typedef struct {
  double z, h, err;
  long long attempts, accepted;
  int status;              /* UPPE_STATUS_* bits; 8 = history capacity reached          */
  int hist_count;          /* saved history slots (slot 0 = A0)                        */
  double energy;           /* sum |A|^2 dt of the final field [J]                      */
  double photons;          /* photon number of the final field (NaN if omega0 = 0)     */
  double peak_ion;         /* max rho/rho_nt over the initial and accepted states      */
} uppe1d_result;

typedef struct uppe1d_plan uppe1d_plan;

/* Replaces ERK43IP_UPPE.__init__ + the cached tables of linear_operator /
 * nonlinear_operator (erk43ip_method.py:21-70, 104-179): uploads the packed
 * FP64 tables and allocates the per-CTA scratch. */
int uppe1d_plan_create(const uppe1d_desc* desc, uppe1d_plan** plan);
int uppe1d_plan_destroy(uppe1d_plan* plan);
long long uppe1d_field_elems(const uppe1d_plan* plan);   /* sum Nt                   */
/* Clusters of the plan's four-CTA line kernel (0: one CTA per line).  A plan whose
 * lines are all 2048..16384 points without Raman or history, one of them at least
 * 8192, runs each line on a cluster of four SMs sharing it through distributed
 * shared memory (no reference counterpart: the reference runs one line at a time
 * on the CPU); a plan of 16 or more lines with 16384-point ones also runs its (up
 * to four) costliest lines on eight-SM clusters, concurrently, on a stream of its
 * own forked from and joined back into the caller's.  UPPE_1D_CLUSTER=0 keeps one
 * CTA per line where that can hold it; UPPE_CLUSTER_CTAS=4 or 8 forces one size. */
int uppe1d_uses_clusters(const uppe1d_plan* plan);
/* SM occupancy of the plan's last propagation launch (no reference counterpart):
 * each persistent CTA records the global timer when it starts and when the work
 * queue runs dry; sm_busy = sum over CTAs of (exit - start) / (SMs x span), span =
 * last exit - first start.  Synchronises the stream. */
int uppe1d_last_activity(uppe1d_plan* plan, double* sm_busy, double* span_ms, uppe_stream_t stream);
long long uppe1d_hist_elems(const uppe1d_plan* plan);    /* sum hist_cap * Nt        */
long long uppe1d_hist_slots(const uppe1d_plan* plan);    /* sum hist_cap             */
/* propagate (erk43ip_method.py:288-369) for every instance.  field: device,
 * packed time-domain A0 in, final A out; hist/zhist: device history fields and z
 * values (NULL when no instance keeps history); results: host array [n_inst]
 * (the call synchronises the stream when results is not NULL). */
int uppe1d_propagate(uppe1d_plan* plan, void* field, void* hist, double* zhist,
                     uppe1d_result* results, uppe_stream_t stream);

/* propagate with the accepted step sizes written to hlog (device, hlog_cap per
 * instance in instance order; result.accepted tells how many; status bit 16 when
 * the log overflowed).  The record the adjoint needs (no reference counterpart:
 * the reference has no differentiation). */
int uppe1d_propagate_logged(uppe1d_plan* plan, void* field, double* hlog, int hlog_cap,
                            uppe1d_result* results, uppe_stream_t stream);
/* Replay: every instance takes the nsched step sizes hsched[i*nsched + k] (device),
 * each accepted, no step control -- the frozen-schedule forward map that the adjoint
 * differentiates (used for finite-difference checks).  No reference counterpart. */
int uppe1d_propagate_schedule(uppe1d_plan* plan, void* field, const double* hsched, int nsched,
                              uppe1d_result* results, uppe_stream_t stream);
/* One operation of a propagation program.  inst >= 0: propagate through plan
 * instance inst (its D/G/H tables, medium, L, tol, max_step, min_step, max_attempts),
 * starting like a fresh propagate() call.  inst < 0: mirror, A_w *= amp exp(i (gdd w^2/2
 * + tod w^3/6)) with w = 2 pi fftfreq(Nt, dt) (test_gaussian_pulse GDD TOD 1mj copy.py:
 * 282-290; amp = sqrt(1 - loss)).  record != 0 stores the time-domain field after it. */
typedef struct {
  int inst;
  int record;
  double amp;
  double gdd;
  double tod;
} uppe1d_op;

/* Run nprog propagation programs (multipass cells, sliced capillaries with per-slice
 * gamma: gas.py:104-147, test_gaussian_pulse GDD TOD 1mj copy.py:196-290) in one
 * persistent launch, one CTA per program, the field kept on chip between operations.
 * Program p is ops[op_begin[p] .. op_begin[p+1]) (host arrays); all its propagation
 * instances share one Nt and dt, and it has at least one.  fields (device): the
 * programs' time-domain input fields packed back to back (Nt_p elements each),
 * overwritten with the outputs.  records (device, may be NULL): the recorded fields,
 * packed per program in operation order.  op_results (host, may be NULL): one per
 * operation (z, steps, status, energy after it; hist_count = 1 when recorded).
 * Replaces the reference's Python slice/pass loops around propagate(). */
int uppe1d_run_programs(uppe1d_plan* plan, int nprog, const long long* op_begin, const uppe1d_op* ops,
                        void* fields, void* records, uppe1d_result* op_results, uppe_stream_t stream);

/* ---- real-field 3+1D solver (src/3+1D-UPPE-ERK4(3)IP-real-field/solver_3d.py) ---- */
typedef struct {
  int Nx, Ny, Nt;          /* powers of two: Nx, Ny in [16, 512], Nt in [64, 2048]      */
  int precision;           /* UPPE_C64 (float32 fields) or UPPE_C128                    */
  double dt;
  const double* kk;        /* [Nt/2+1] k(omega)^2, omega = 2 pi rfftfreq (solver_3d.py:56-71) */
  const double* kref;      /* [Nt/2+1] k1 omega (:73-83)                               */
  const double* w;         /* [Nt/2+1] omega                                           */
  const double* filt;      /* [Nt/2+1] anti-alias filter (:50-52)                      */
  const double* kperp2;    /* [Nx*Ny] kx^2+ky^2, index ix*Ny+iy                        */
  const double* damp;      /* [Nx*Ny] absorber (:99-110)                               */
  int lut_n;               /* PPT rate table over log10(I [W/m^2]) (media_physics.py:167-183) */
  const double* lut_log10I;
  const double* lut_W;
  double I_coef;           /* 0.5 eps0 c n0: I_equiv = I_coef E^2 (:266)               */
  double aval_coef;        /* W_ava = aval_coef I_equiv (0 for the gases)              */
  double chi3e, chi5e;     /* eps0 chi3, eps0 chi5: P = chi3e E^3 + chi5e E^5 (:300-312) */
  double rate_rec, rho_nt, Ui, e_charge, m_e, tau_c;   /* density / Drude constants (:11-118) */
  /* Raman response of fused silica (media_physics.py:303-305, 362-390): NULL for none;
   * else H(omega_k), k = 0..Nt, of the 2 Nt-point response (interleaved re, im: 2 (Nt+1)
   * doubles) and its fraction: E_eff^2 = (1 - f_R) E^2 + f_R (the zero-padded E^2
   * convolved circularly over 2 Nt samples with the response), P = chi3e E E_eff^2. */
  const double* raman_H;
  double raman_fR;
} uppe_rf_desc;

typedef struct uppe_rf_plan uppe_rf_plan;
/* Replaces ERK43_RealField_UPPE_3D.__init__: uploads the tables, allocates the
 * spectral fields (rows of Nt/2 + 16 bins) and the two real state buffers. */
int uppe_rf_plan_create(const uppe_rf_desc* desc, uppe_rf_plan** plan);
int uppe_rf_plan_destroy(uppe_rf_plan* plan);
/* Start of propagate (:177-185): E_scale = max|E0|, state = E0 / E_scale.  E0: device
 * real field [Nx][Ny][Nt] in the plan's precision; E_scale (host, may be NULL) out. */
int uppe_rf_set_field(uppe_rf_plan* plan, const void* E0, double* E_scale, uppe_stream_t stream);
/* One erk43_step (:113-175) of size h from the accepted state into the candidate;
 * err = max|E4 - E_low| / max|E4| (synchronises the stream). */
int uppe_rf_attempt(uppe_rf_plan* plan, double h, double* err, uppe_stream_t stream);
/* Accept (state <- candidate) or reject the last attempt. */
int uppe_rf_commit(uppe_rf_plan* plan, int accept, uppe_stream_t stream);
/* Physical field E * E_scale of the state (device real [Nx][Ny][Nt]). */
int uppe_rf_get_field(uppe_rf_plan* plan, void* out, uppe_stream_t stream);
/* rfft_t(E * E_scale) (:226-233) into out (device complex [Nx][Ny][uppe_rf_spec_bins]);
 * bins >= Nt/2 + 1 are zero.  Uses the candidate buffer as scratch. */
int uppe_rf_get_spectrum(uppe_rf_plan* plan, void* out, uppe_stream_t stream);
int uppe_rf_spec_bins(const uppe_rf_plan* plan);

/* Spectral amplitude of an input pulse from a measured spectrum (the per-sample part
 * of generate_pulse_from_spectrum, erk43ip_method.py:599-764, FFT path): S(f) is the
 * piecewise cubic coef[4j..4j+3] (power form in f - breaks[j], highest first) on
 * ascending breaks[0..nb-1] (device arrays); out (device complex128 [Nt], fft order)
 * = sqrt(max(S(f_k), 0)) exp(i (gdd w_k^2/2 + tod w_k^3/6)) with w_k = 2 pi
 * fftfreq(Nt, dt)[k], f_k = w_k/(2 pi) + f0, S = 0 outside the breaks. */
int uppe_spectrum_field(const double* breaks, const double* coef, int nb, int Nt, double dt, double f0,
                        double gdd, double tod, void* out, uppe_stream_t stream);

/* One complex128 line transform on the device, N a power of two (2 .. 2^24):
 * out = scale * fftshift?(F(ifftshift?(in))) with F the forward (dir = -1) or
 * unnormalised inverse (dir = +1) DFT; shift_in / shift_out apply the
 * half-length rotations.  work: device, 2 N complex128; in may equal out.  The
 * numpy fft/ifft/fftshift calls of the reference's pulse builders
 * (erk43ip_method.py:415-429, 750-753). */
int uppe_fft_c128(const void* in, void* out, void* work, int N, int dir, double scale, int shift_in,
                  int shift_out, uppe_stream_t stream);
/* field (device complex128 [N], fft order) *= exp(i (gdd w^2/2 + tod w^3/6)), w = 2 pi
 * fftfreq(N, dt): the dispersion phase of generate_dispersed_pulse
 * (erk43ip_method.py:417-421). */
int uppe_spectral_phase(void* field, int N, double dt, double gdd, double tod, uppe_stream_t stream);
/* The direct Fourier sum of _exact_fourier_transform (erk43ip_method.py:583-596):
 * out[(i + Nt/2) mod Nt] = sum_k amp[k] exp(-i omega[k] t[i]) (the sum then the
 * fftshift), with amp[k] = Simpson weight x sqrt(S_k) x exp(i phase_k) on the dense
 * frequency grid (device arrays; amp complex128). */
int uppe_exact_ft(const double* t, int Nt, const double* omega, const void* amp, int Nf, void* out,
                  uppe_stream_t stream);

/* Workspace of uppe1d_adjoint, in complex128 elements. */
long long uppe1d_adjoint_work_elems(int Nt, int nsteps, int K);
/* Reverse-mode derivative of one instance's frozen-schedule propagation (complex128
 * plan; Kerr + self-steepening + dispersion + loss + the plasma term without
 * avalanche; no Raman).  Replays the forward with a checkpoint every K steps and
 * recomputes within segments.  Inputs (device): hlog[nsteps], A0 (time domain),
 * Abar = dL/dA_L in the omega domain (dL = Re sum conj(Abar) dA).  Outputs (device):
 * A0bar = dL/dfft(A0), gD = dL/dD, gG = dL/dG (the tables of uppe1d_desc), rhs =
 * D A_L + N(A_L) (so dL/dL = Re sum conj(Abar) rhs), gPlasma[3] = dL/d(rho_nt,
 * sigma_drude, omega0_tau_c) (required for plasma instances, else may be NULL).
 * No reference counterpart (the reference is not differentiable). */
int uppe1d_adjoint(uppe1d_plan* plan, int inst, const double* hlog, int nsteps, int K,
                   const void* A0, const void* Abar, void* A0bar, void* gD, double* gG, void* rhs,
                   double* gPlasma, void* work, uppe_stream_t stream);

/* Allocation-free single propagation, for callers that cannot allocate device
 * memory (a host framework that owns the CUDA allocator and forbids cudaMalloc
 * from plug-ins, a real-time host that must not allocate after start-up, or code
 * holding only device pointers lent by another runtime).  No counterpart in the
 * reference.  It runs the same kernel as uppe1d_propagate for one instance
 * without a plan: the caller passes the FP64 tables D, G (and H when raman, all
 * device memory, packed as in uppe1d_desc), the ionisation table in the field
 * precision (device, only when plasma) and the device field (A0 in, final A out,
 * time domain).  The per-call device state lives in one static device array of
 * UPPE_NOALLOC_SCRATCH_BYTES that every GPU loading the library keeps until exit;
 * Nt above UPPE_NOALLOC_MAX_NT_C64 / _C128 is rejected with UPPE_ERR_SIZE, and
 * hist_cap must be 0.  The ionisation grid must increase; its ends are read on
 * the device.  The first call on a device looks up the array's address (make it
 * before any stream capture).  Calls share the array: calls that overlap on the
 * GPU race.  Synchronises the stream only when result is not NULL (to copy the
 * result record back). */
#define UPPE_NOALLOC_MAX_NT_C64 16384
#define UPPE_NOALLOC_MAX_NT_C128 8192
#define UPPE_NOALLOC_SCRATCH_BYTES (1024ull + 9ull * UPPE_NOALLOC_MAX_NT_C128 * 16ull)
int uppe1d_propagate_noalloc(const uppe1d_inst_desc* inst, int precision, const double* D,
                             const double* G, const double* H, int lut_n,
                             const void* lut_log10I, const void* lut_W, void* field,
                             uppe1d_result* result, uppe_stream_t stream);

/* Diagnostics of the current 3D state: out3 = {pulse energy sum |A|^2 dx dy dt [J],
 * photon number sum_omega E_omega / (hbar omega_abs) (omega_abs > 0), peak ionisation
 * fraction max rho/rho_nt over the states at which steps started and the current
 * state}.  The reference prints no diagnostics; these are the quantities its
 * drivers compute from the returned field (src/3+1D-ERK4(3)IP UPPE/sim.py:140-249). */
int uppe3d_diagnostics(uppe3d_plan* plan, double dx, double dy, double* out3, uppe_stream_t stream);

/* Doubles in the output of uppe3d_beam_diagnostics: 10 Nt + Nx Ny. */
long long uppe3d_beam_diag_elems(const uppe3d_plan* plan);
/* Beam diagnostics of the current state in one device pass, the sums behind
 * src/3+1D-ERK4(3)IP UPPE/sim.py:140-249 (energy, P(t), fluence and beam moments,
 * full / centre / fibre-coupled spectra, centre and fibre-coupled intensity vs t).
 * out (device, uppe3d_beam_diag_elems doubles), all of the normalised state Z =
 * fft_t(A / A_scale) and a = ifft_t(Z): [0, Nt) sum_xy |Z|^2; [Nt, 3Nt) sum_xy m Z
 * (re, im interleaved); [3Nt, 4Nt) sum_xy |a|^2; [4Nt, 6Nt) sum_xy m a; [6Nt, 8Nt)
 * Z at (Nx/2, Ny/2); [8Nt, 10Nt) a there; then sum_t |a|^2 per (x, y), index
 * ix*Ny+iy.  mode: device [Nx*Ny] fibre mode, or NULL (its sums stay 0).  omega
 * in fft order. */
int uppe3d_beam_diagnostics(uppe3d_plan* plan, const double* mode, double* out, uppe_stream_t stream);

/* Mirror on the current state (x, y, omega): Z *= amp exp(i (gdd w^2/2 + tod w^3/6
 * - omega_abs r^2 / (c R))) with w = 2 pi fftfreq(Nt, dt), omega_abs = desc.omega_abs and
 * r2[ix*Ny+iy] = x^2 + y^2 (device; NULL for a flat mirror, R then ignored).  The curved
 * mirror of src/3+1D-ERK4(3)IP UPPE/sim.py:83-96 and the flat-mirror transmission
 * :331 (amp = sqrt(T)); uppe3d_get_field then returns the reflected field. */
int uppe3d_mirror(uppe3d_plan* plan, const double* r2, double R, double amp, double gdd, double tod,
                  uppe_stream_t stream);

/* Record the accepted step sizes of later uppe3d_propagate runs in hlog (device,
 * cap entries; NULL stops recording).  No reference counterpart (the adjoint's input). */
int uppe3d_set_step_log(uppe3d_plan* plan, double* hlog, long long cap, uppe_stream_t stream);
/* Workspace of uppe3d_adjoint in bytes. */
long long uppe3d_adjoint_work_bytes(const uppe3d_plan* plan, int nsteps, int K);
/* Reverse-mode derivative of the frozen-schedule 3D propagation (Kerr + self-steepening,
 * dispersion, diffraction, filter, absorber, the plasma terms without avalanche; no
 * n4 term).  hlog_host: the
 * nsteps accepted step sizes (host); A0: device input field (time domain, physical);
 * Zbar: device cotangent of the final state in the (x, y, omega) domain with the
 * state normalised by A_scale (dL = Re sum conj(Zbar) dZ); A0bar: device output,
 * cotangent of A0 (time domain).  Checkpoints every K steps, recomputes within
 * segments.  Overwrites the plan's state.  No reference counterpart. */
int uppe3d_adjoint(uppe3d_plan* plan, const double* hlog_host, int nsteps, int K, const void* A0,
                   const void* Zbar, void* A0bar, void* work, uppe_stream_t stream);

/* Line transform along t of a device field of the plan's grid and precision:
 * out = scale * fft_t(in) for dir = -1, out = scale * (unnormalised inverse) for
 * dir = +1; in and out may be the same buffer.  The reference applies cuFFT's
 * fft/ifft along t (solver_3d.py:101, 155, 216); this is the same transform with
 * the plan's own kernel, e.g. for the cotangent of a differentiable objective. */
int uppe3d_transform_t(uppe3d_plan* plan, const void* in, void* out, int dir, double scale,
                       uppe_stream_t stream);

/* Launch configuration chosen for the plan's shape by the tuner that runs in
 * uppe3d_plan_create (no reference counterpart: the reference leaves kernel
 * choice to cuFFT).  Candidates: y passes on the TMA-fed kernel with tiles of 16
 * omega columns (stage operands loaded before the tile's wait with 2 or 1 CTAs
 * per SM, or where they are used with 3 or 2) or of 8 columns (early with 4,
 * late with 6 CTAs per SM) -- complex64 plans with 64 <= Ny <= 256 -- then, for
 * Ny = 256, on the register four-step kernel (tiles of 16 columns: operands
 * loaded with the tile, 2 CTAs per SM, or where used, 3), on the register
 * four-step kernel with every operand tile on a TMA ring (persistent, 1 CTA per
 * SM) and on the register four-step kernel with tiles of 8 columns (early, 4 CTAs
 * per SM, or late, 6), and 8 or 4 t-lines per block of the warp t-line kernel.  All candidates compute identical bits (the plain tile
 * kernel, which rounds differently, serves the other shapes).  cfg6 = {y kernel
 * (1 TMA-fed, 2 register four-step, 3 register four-step on a TMA ring, 0 plain
 * tile), CTAs per SM, late operand loads, omega columns per tile, t-lines per
 * block, 1 timed / 2 from the process cache / 0 defaults (UPPE_TUNE=0)}; ms (may
 * be NULL, UPPE3D_TUNE_SLOTS floats): per-attempt time of the y passes for the
 * eleven y candidates in that order [0..10] and of the t passes for 8 and 4
 * lines per block [11..12], in ms (0 when not timed). */
#define UPPE3D_TUNE_SLOTS 13
int uppe3d_tuning(const uppe3d_plan* plan, int* cfg6, float* ms);
/* Force a launch configuration (y_tma 1 TMA-fed, 2 register four-step, 3
 * register four-step on a TMA ring -- 2 and 3: Ny = 256 complex64 only, 3 without
 * late loads and with 16 columns --, 0 the plain tile kernel; y_ctas 1..6, y_kw
 * 16 or 8, t_wpb 4 or 8) and re-capture the attempt graphs; for comparing the
 * candidates. */
int uppe3d_set_tuning(uppe3d_plan* plan, int y_tma, int y_ctas, int y_late, int y_kw, int t_wpb);

/* Access-pattern bandwidth probe (measurement hook; no reference counterpart):
 * one read and one write of a 256 x 256 x nt complex64 field (in, out: device,
 * distinct, 16-byte aligned; nt a power of two >= 64) with pattern 0 a sequential
 * stream, 1 the x-pass tiles (kw omega columns from 256 rows Ny*nt elements
 * apart), 2 the y-pass tiles (rows nt elements apart); kw 8, 16 or 32.  Each
 * element is loaded, has 1 added to its real part and is stored: the bandwidth
 * a pass's access pattern alone reaches, to set its achieved bandwidth against. */
int uppe_pattern_probe(int pattern, int kw, const void* in, void* out, int nt, uppe_stream_t stream);

/* Kernel launches of one propagate-mode attempt (graph nodes). */
int uppe3d_launches_per_step(const uppe3d_plan* plan);
/* Measurement hook: run one attempt (plus the controller) launch by launch,
 * bracketing each launch with CUDA events on `stream`.  Writes per launch its
 * time [ms], pass kind (0 t-line, 1 x-pass, 2 y-pass, 3 scalar, 4 TMA-fed y-pass, 5 register
 * four-step y-pass, 6 register four-step y-pass on TMA tiles) and algorithmic
 * bytes (0 for launches the device state made exit early). */
int uppe3d_profile_attempt(uppe3d_plan* plan, int cap, float* ms, int* kind, double* bytes,
                           int* n, uppe_stream_t stream);

#ifdef __cplusplus
}
#endif
#endif /* UPPE_B200_H */
