"""3+1D envelope ERK4(3)-IP UPPE propagator on the GPU (drop-in for
``ERK43IP_UPPE_3D_Optimized``, src/3+1D-UPPE-ERK4(3)IP-envelope/solver_3d.py).

The host computes the FP64 tables of ``__init__`` (solver_3d.py:8-98) exactly as
the reference does and hands them to ``libuppe_b200.so``; every per-step
operation (FFTs, interaction-picture factor, nonlinear response with the plasma
scan, ERK stages, error norm, step-size control) runs in the library's CUDA
kernels.  ``precision='double'`` is complex128 throughout; ``'single'`` is the
mixed mode: complex64 bulk with the FP64 interaction-picture phase (reduced mod
2 pi before rounding), FP64 density scan, FP64 error norm and controller.
"""
import ctypes

import numpy as np
import torch

from . import _lib


class ERK43IP_UPPE_3D_Optimized:
    def __init__(self, x_grid, y_grid, t_grid, medium, precision='single', device=None):
        lib = _lib.load()
        self._lib = lib
        self.medium = medium
        self.c, self.lambda0, self.omega0 = medium.c, medium.lambda0, medium.omega0
        self.precision = precision
        if precision == 'double':
            self.complex_dtype, self._prec = torch.complex128, _lib.UPPE_C128
        elif precision == 'single':
            self.complex_dtype, self._prec = torch.complex64, _lib.UPPE_C64
        else:
            raise ValueError("precision must be 'single' or 'double'")
        self.device = torch.device(device if device is not None else 'cuda')
        x = np.asarray(x_grid, dtype=np.float64)
        y = np.asarray(y_grid, dtype=np.float64)
        t = np.asarray(t_grid, dtype=np.float64)
        self.x, self.y, self.t = x, y, t
        self.Nx, self.Ny, self.Nt = len(x), len(y), len(t)
        self.dx, self.dy, self.dt = float(x[1] - x[0]), float(y[1] - y[0]), float(t[1] - t[0])
        self._tables()
        self._create_plan()
        self.A_scale = 1.0
        self.last_result = None

    def _tables(self):
        tb = tables3d(self.x, self.y, self.t, self.medium)
        for k, v in tb.items():
            setattr(self, k, v)

    def _create_plan(self):
        m = self.medium
        if m.lut_log10I is None:
            raise ValueError('the medium has no ionisation LUT')
        self._keep = [np.ascontiguousarray(a) for a in (
            self.a_w, self.k_sq, self.k_ref, self.valid, self.shock, self.filter,
            self.K2_perp.ravel(), self.damp.ravel(), m.lut_log10I, m.lut_W,
            self.omega + m.omega0)]
        ptr = [a.ctypes.data for a in self._keep]
        d = _lib.Desc3D()
        d.Nx, d.Ny, d.Nt, d.precision, d.dt = self.Nx, self.Ny, self.Nt, self._prec, self.dt
        (d.aw, d.ksq, d.kref, d.valid, d.shock, d.filt, d.kperp2, d.damp) = ptr[:8]
        d.lut_n = len(m.lut_log10I)
        d.lut_log10I, d.lut_W = ptr[8], ptr[9]
        d.gamma_kerr = (m.omega0 / m.c) * m.n2                               # media_physics.py:192
        d.gamma_hoke = (m.omega0 / m.c) * m.n4
        d.Ui = m.Ui
        d.sigma_drude = m.sigma_drude
        d.omega0_tau_c = m.omega0 * m.tau_c
        d.rate_rec = 1.0 / m.tau_rec
        d.rho_nt = m.rho_nt
        d.ava_coef = m.avalanche_coef
        d.plasma_on = 1 if m.plasma else 0
        d.omega_abs = ptr[10]
        plan = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            _lib.check(self._lib.uppe3d_plan_create(ctypes.byref(d), ctypes.byref(plan)),
                       'uppe3d_plan_create')
        self._plan = plan

    def __del__(self):
        plan = getattr(self, '_plan', None)
        if plan is not None and plan.value:
            self._lib.uppe3d_plan_destroy(plan)
            self._plan = None

    # ---- state ----------------------------------------------------------------
    def _as_device_field(self, A0):
        if isinstance(A0, torch.Tensor):
            A = A0.to(device=self.device, dtype=self.complex_dtype)
        else:
            A = torch.from_numpy(np.ascontiguousarray(A0)).to(self.device).to(self.complex_dtype)
        A = A.contiguous()
        if tuple(A.shape) != (self.Nx, self.Ny, self.Nt):
            raise ValueError(f'A0 must have shape {(self.Nx, self.Ny, self.Nt)}, got {tuple(A.shape)}')
        return A

    def set_field(self, A0, stream=None):
        """Load A0 (x, y, t): A_scale = max|A0|, state = A0/A_scale (solver_3d.py:163-170)."""
        A = self._as_device_field(A0)
        _lib.check(self._lib.uppe3d_set_field(self._plan, ctypes.c_void_p(A.data_ptr()),
                                              _lib.stream_ptr(stream)), 'uppe3d_set_field')
        return A

    def attempt(self, h, stream=None):
        """One erk43_step of size h from the current state; returns its error."""
        err = ctypes.c_double()
        _lib.check(self._lib.uppe3d_attempt(self._plan, float(h), ctypes.byref(err),
                                            _lib.stream_ptr(stream)), 'uppe3d_attempt')
        return err.value

    def commit(self, accept, stream=None):
        _lib.check(self._lib.uppe3d_commit(self._plan, 1 if accept else 0, _lib.stream_ptr(stream)),
                   'uppe3d_commit')

    def result(self, stream=None):
        r = _lib.Result3D()
        _lib.check(self._lib.uppe3d_get_result(self._plan, ctypes.byref(r), _lib.stream_ptr(stream)),
                   'uppe3d_get_result')
        return r

    def save_state(self, stream=None):
        """Continuation point of the adaptive run between two attempts: a dict with
        the loop state (z, h, counters, status, A_scale, ...) and a device copy of the
        accepted normalised state.  load_state + resume continue the run bit for bit."""
        st = _lib.State3D()
        buf = torch.empty((self.Nx, self.Ny, self.Nt), dtype=self.complex_dtype, device=self.device)
        _lib.check(self._lib.uppe3d_save_state(self._plan, ctypes.c_void_p(buf.data_ptr()), ctypes.byref(st),
                                               _lib.stream_ptr(stream)), 'uppe3d_save_state')
        return {'state': {k: getattr(st, k) for k, _ in _lib.State3D._fields_}, 'field': buf}

    def load_state(self, saved, stream=None):
        st = _lib.State3D(**saved['state'])
        buf = saved['field'].to(device=self.device, dtype=self.complex_dtype).contiguous()
        _lib.check(self._lib.uppe3d_load_state(self._plan, ctypes.c_void_p(buf.data_ptr()), ctypes.byref(st),
                                               _lib.stream_ptr(stream)), 'uppe3d_load_state')
        self.A_scale = st.A_scale

    def resume(self, return_gpu=False, stream=None):
        """Continue the adaptive run from the current state to its L; returns what
        propagate returns."""
        r = _lib.Result3D()
        _lib.check(self._lib.uppe3d_resume(self._plan, ctypes.byref(r), _lib.stream_ptr(stream)), 'uppe3d_resume')
        self.last_result = r
        A_w = self.spectrum(stream=stream)
        if return_gpu:
            return r.z, self.freq_axis_hz, A_w
        return r.z, self.freq_axis_hz, A_w.cpu().numpy()

    def spectrum(self, out=None, stream=None):
        """fftshift_t(fft_t(A * A_scale)) of the current state, on the device."""
        if out is None:
            out = torch.empty((self.Nx, self.Ny, self.Nt), dtype=self.complex_dtype, device=self.device)
        _lib.check(self._lib.uppe3d_get_spectrum(self._plan, ctypes.c_void_p(out.data_ptr()),
                                                 _lib.stream_ptr(stream)), 'uppe3d_get_spectrum')
        return out

    def field(self, out=None, stream=None):
        """Time-domain field A(x, y, t) of the current state (physical units)."""
        if out is None:
            out = torch.empty((self.Nx, self.Ny, self.Nt), dtype=self.complex_dtype, device=self.device)
        _lib.check(self._lib.uppe3d_get_field(self._plan, ctypes.c_void_p(out.data_ptr()),
                                              _lib.stream_ptr(stream)), 'uppe3d_get_field')
        return out

    def mirror(self, R=None, loss=0.0, gdd=0.0, tod=0.0, stream=None):
        """Reflect the current state: amplitude sqrt(1 - loss), spectral phase gdd w^2/2 +
        tod w^3/6 and, for a curved mirror of radius R, the phase -k(omega) r^2 / R
        (src/3+1D-ERK4(3)IP UPPE/sim.py:83-96, :331)."""
        r2 = None
        if R is not None:
            if getattr(self, '_r2', None) is None:
                x = torch.as_tensor(np.asarray(self.x, dtype=np.float64))
                y = torch.as_tensor(np.asarray(self.y, dtype=np.float64))
                self._r2 = (x[:, None] ** 2 + y[None, :] ** 2).reshape(-1).contiguous().to(self.device)
            r2 = ctypes.c_void_p(self._r2.data_ptr())
        _lib.check(self._lib.uppe3d_mirror(self._plan, r2, float(R) if R is not None else 0.0,
                                           float(np.sqrt(1.0 - loss)), float(gdd), float(tod),
                                           _lib.stream_ptr(stream)), 'uppe3d_mirror')

    def beam_diagnostics(self, w_mode=None, stream=None):
        """Diagnostics of the current state (src/3+1D-ERK4(3)IP UPPE/sim.py:140-249),
        the field-sized sums done on the device in one pass (uppe3d_beam_diagnostics)
        and only O(Nt + Nx Ny) arrays copied back.  w_mode: waist of the Gaussian
        fibre mode exp(-r^2 / w_mode^2) for the coupled spectrum and intensity.
        Returns a dict with the keys of the reference's DIAG record."""
        dev = self.device
        mode_ptr = None
        if w_mode is not None:
            key = float(w_mode)
            if getattr(self, '_mode_key', None) != key:
                x = torch.as_tensor(np.asarray(self.x, dtype=np.float64))
                y = torch.as_tensor(np.asarray(self.y, dtype=np.float64))
                self._mode = torch.exp(-(x[:, None] ** 2 + y[None, :] ** 2) / key ** 2).reshape(-1).contiguous().to(dev)
                self._mode_key = key
            mode_ptr = ctypes.c_void_p(self._mode.data_ptr())
        n = self._lib.uppe3d_beam_diag_elems(self._plan)
        out = torch.empty(n, dtype=torch.float64, device=dev)
        _lib.check(self._lib.uppe3d_beam_diagnostics(self._plan, mode_ptr, ctypes.c_void_p(out.data_ptr()),
                                                     _lib.stream_ptr(stream)), 'uppe3d_beam_diagnostics')
        o = out.cpu().numpy()
        Nt = self.Nt
        As2 = self.result(stream).A_scale ** 2
        cplx = lambda v: v[0::2] + 1j * v[1::2]
        spec, cw, pt, ct = o[:Nt], cplx(o[Nt:3 * Nt]), o[3 * Nt:4 * Nt], cplx(o[4 * Nt:6 * Nt])
        zc, ac, flu = cplx(o[6 * Nt:8 * Nt]), cplx(o[8 * Nt:10 * Nt]), o[10 * Nt:].reshape(self.Nx, self.Ny)
        dxdy = self.dx * self.dy
        P_t = pt * dxdy * As2
        fluence = flu * self.dt * As2
        moments = beam_moments(self.x, self.y, fluence)
        t = np.asarray(self.t, dtype=np.float64)
        I_center = np.abs(ac) ** 2 * As2
        I_smf = np.abs(ct) ** 2 * As2
        freq_abs = self.freq_axis_hz + self.c / self.lambda0
        wl_nm = np.zeros_like(freq_abs)
        ok = freq_abs > 1e9
        wl_nm[ok] = self.c / freq_abs[ok] * 1e9
        return {'energy_total': float(pt.sum() * dxdy * self.dt * As2),
                'x_mean_m': moments[0], 'y_mean_m': moments[1], 'wx_rms_m': moments[2], 'wy_rms_m': moments[3],
                't_s': t, 'P_t': P_t, 'it_peak': int(np.argmax(P_t)), 'fluence': fluence,
                'I_center_t': I_center, 'I_smf_t': I_smf,
                'fwhm_center_s': fwhm(t, I_center), 'fwhm_smf_s': fwhm(t, I_smf),
                'freq_abs_Hz': freq_abs, 'wl_nm': wl_nm,
                'spec_full_incoh': np.fft.fftshift(spec * As2),
                'spec_center': np.fft.fftshift(np.abs(zc) ** 2 * As2),
                'spec_smf': np.fft.fftshift(np.abs(cw) ** 2 * As2)}

    def diagnostics(self, stream=None):
        """{'energy' [J], 'photons', 'peak_ionization'} of the current state (device)."""
        out = (ctypes.c_double * 3)()
        _lib.check(self._lib.uppe3d_diagnostics(self._plan, self.dx, self.dy, out, _lib.stream_ptr(stream)),
                   'uppe3d_diagnostics')
        return {'energy': out[0], 'photons': out[1], 'peak_ionization': out[2]}

    def replay(self, A0, steps, stream=None):
        """Frozen-schedule forward map: every step in ``steps`` accepted."""
        self.set_field(A0, stream)
        for h in steps:
            self.attempt(float(h), stream)
            self.commit(True, stream)
        return self.field(stream=stream)

    # ---- the reference surface ---------------------------------------------------
    def propagate(self, A0, L, tol=1e-4, max_step=1e-2, min_step=1e-9, return_gpu=False,
                  max_attempts=0, stream=None, out=None, log_steps=False):
        """solver_3d.py:162-233 -> (z_reached, freq_axis_hz, A_w_final).

        ``out``: optional host tensor (e.g. pinned) that receives the spectrum.

        The adaptive loop runs on the device.  Unlike the reference (which never
        terminates once the error becomes NaN), a non-finite error stops the run
        with ``last_result.status & STATUS_NONFINITE`` set.
        """
        self.set_field(A0, stream)
        hlog = None
        if log_steps:   # accepted step sizes, for the adjoint
            cap = int(max_attempts) if max_attempts and max_attempts > 0 else 1 << 20
            hlog = torch.zeros(cap, dtype=torch.float64, device=self.device)
            _lib.check(self._lib.uppe3d_set_step_log(self._plan, ctypes.c_void_p(hlog.data_ptr()), cap,
                                                     _lib.stream_ptr(stream)), 'uppe3d_set_step_log')
        r = _lib.Result3D()
        _lib.check(self._lib.uppe3d_propagate(self._plan, float(L), float(tol), float(max_step),
                                              float(min_step), int(max_attempts), ctypes.byref(r),
                                              _lib.stream_ptr(stream)), 'uppe3d_propagate')
        self.last_result = r
        self.A_scale = r.A_scale
        if hlog is not None:
            self.last_steps = hlog[:int(r.accepted)].cpu().numpy()
            _lib.check(self._lib.uppe3d_set_step_log(self._plan, None, 0, _lib.stream_ptr(stream)),
                       'uppe3d_set_step_log')
        A_w = self.spectrum(stream=stream)
        if return_gpu:
            return r.z, self.freq_axis_hz, A_w
        if out is not None:      # caller-provided (e.g. pinned) host buffer
            out.copy_(A_w)
            return r.z, self.freq_axis_hz, out.numpy()
        return r.z, self.freq_axis_hz, A_w.cpu().numpy()


def tables3d(x, y, t, medium):
    """FP64 tables of ERK43IP_UPPE_3D_Optimized.__init__ (solver_3d.py:28-98)."""
    x = np.asarray(x, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    t = np.asarray(t, dtype=np.float64)
    Nx, Ny, Nt = len(x), len(y), len(t)
    dx, dy, dt = float(x[1] - x[0]), float(y[1] - y[0]), float(t[1] - t[0])
    kx = 2 * np.pi * np.fft.fftfreq(Nx, dx)                                  # :28
    ky = 2 * np.pi * np.fft.fftfreq(Ny, dy)                                  # :29
    # kperp^2 at field index (ix, iy).  The reference's meshgrid(ky, kx,
    # indexing='ij') (:30) puts ky on axis 0, which is the same array for the
    # square, equally spaced grids it supports.
    K2_perp = (kx[:, None] ** 2 + ky[None, :] ** 2).astype(np.float64)
    omega = 2 * np.pi * np.fft.fftfreq(Nt, dt)                               # :34
    m = medium
    w0, c = float(m.omega0), float(m.c)
    n_omega = np.asarray(m.refractive_index(omega + w0), dtype=np.float64)   # :61
    k_val = n_omega * (omega + w0) / c                                       # :62
    n_center = float(m.refractive_index(np.array([w0]))[0])                 # :64-65
    dw = w0 * 1e-3                                                           # :67
    n_plus = float(m.refractive_index(np.array([w0 + dw]))[0])              # :68-69
    k0 = n_center * w0 / c                                                   # :71
    k_plus = n_plus * (w0 + dw) / c                                          # :72
    k1 = (k_plus - k0) / dw                                                  # :73
    k_ref = k0 + k1 * omega                                                  # :74
    k_sq = k_val ** 2
    f = omega / (2 * np.pi)                                                  # :47
    f_max = float(np.max(np.abs(f))) + 1e-10                                 # :48
    X, Y = np.meshgrid(x, y, indexing='ij')                                  # :90
    R = np.sqrt(X ** 2 + Y ** 2)
    half_w = float(np.max(np.abs(x)))
    r_edge, r_start = 0.98 * half_w, 0.85 * half_w
    s = np.clip((R - r_start) / (r_edge - r_start + 1e-30), 0.0, 1.0)
    return {
        'K2_perp': K2_perp, 'omega': omega,
        'freq_axis_hz': np.fft.fftshift(omega) / (2 * np.pi),                # :36
        'k_sq': k_sq, 'k_ref': k_ref,
        'a_w': k_sq - k_ref ** 2,                                            # :82 first term
        'valid': ((omega + w0) > 0).astype(np.uint8),                        # :86, :53-54
        'shock': np.asarray(m.get_shock_operator(omega), dtype=np.float64),  # :44
        'filter': np.exp(-(f / (0.85 * f_max)) ** 16),                       # :49
        'damp': (120.0 * (s ** 10)).astype(np.float64),                      # :98
    }


def ip_operator_host(tb, kx_index=None):
    """numpy restatement of the device's D(kx, ky, omega) from the tables (for checks)."""
    q = tb['K2_perp'][:, :, None]
    num = tb['a_w'][None, None, :] - q
    kz = np.sqrt((tb['k_sq'][None, None, :] - q).astype(np.complex128))
    D = 1j * (num / (kz + tb['k_ref'][None, None, :]))
    return D * tb['valid'][None, None, :]


def beam_moments(x, y, fluence):
    """Centroid and rms widths of a fluence map F[ix, iy] (sim.py:145-157)."""
    X, Y = np.meshgrid(np.asarray(x, dtype=np.float64), np.asarray(y, dtype=np.float64), indexing='ij')
    dxdy = float(x[1] - x[0]) * float(y[1] - y[0])
    tot = float(np.sum(fluence)) * dxdy + 1e-30
    xm = float(np.sum(X * fluence)) * dxdy / tot
    ym = float(np.sum(Y * fluence)) * dxdy / tot
    x2 = float(np.sum((X - xm) ** 2 * fluence)) * dxdy / tot
    y2 = float(np.sum((Y - ym) ** 2 * fluence)) * dxdy / tot
    return xm, ym, float(np.sqrt(x2)), float(np.sqrt(y2))


def fwhm(t, I):
    """Full width at half maximum of I(t) (sim.py:159-182): walk out from the peak
    to the first samples below half, interpolate linearly on each side; NaN when
    undefined."""
    I = np.asarray(I, dtype=np.float64)
    t = np.asarray(t, dtype=np.float64)
    if I.size < 4:
        return float('nan')
    top = float(np.max(I))
    if not np.isfinite(top) or top <= 0:
        return float('nan')
    half = 0.5 * top
    k = int(np.argmax(I))
    lo = k
    while lo > 0 and I[lo] >= half:
        lo -= 1
    hi = k
    while hi < I.size - 1 and I[hi] >= half:
        hi += 1
    if hi <= lo + 1:
        return float('nan')

    def cross(i, j):
        return t[i] + (half - I[i]) * (t[j] - t[i]) / (I[j] - I[i] + 1e-30)

    left = cross(lo, lo + 1)
    right = cross(hi - 1, hi)
    w = right - left
    return float(w) if (w > 0 and np.isfinite(w)) else float('nan')
