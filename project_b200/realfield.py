"""Real-field 3+1D ERK4(3)-IP UPPE solver on the device.

Mirror of ``ERK43_RealField_UPPE_3D`` (``src/3+1D-UPPE-ERK4(3)IP-real-field/
solver_3d.py:7-241``) and its media (``media_physics.py``: PPT ionisation
:121-246, density + Drude current :11-118, response :258-318, gases and fused
silica :321-626).  The field is real (carrier included, CEP kept); the spectral
state covers omega >= 0 (rfft).  The step, the transforms and the medium
response run in ``libuppe_b200`` (``uppe_rf_*``); the adaptive loop is the
reference's, on the host, one error read-back per attempt.
"""
import ctypes

import numpy as np
import torch

from . import _lib

C0 = 299792458.0
E_CH = 1.60217663e-19
EPS0 = 8.85418781e-12
M_E = 9.1093837e-31


def ppt_rate(I, omega0, Ui, n0, Z=1.0, l=0, m=0):
    """Perelomov-Popov-Terent'ev ionisation rate [1/s] at intensity I [W/m^2]
    (media_physics.py:185-246: Keldysh parameter, effective principal quantum
    number, C_nl^2, f(l, m), g(gamma) and 15 above-threshold channels)."""
    from scipy.special import gamma as G
    I = np.maximum(np.asarray(I, dtype=np.float64), 1e4)
    Ea = np.sqrt(2 * I / (C0 * EPS0 * n0)) / 5.142206538e11
    wa = omega0 * 2.418884e-17
    U = Ui / (27.21138 * E_CH)
    gk = wa * np.sqrt(2 * U) / Ea
    ns = Z / np.sqrt(2 * U)
    cnl = 2 ** (2 * ns) / (ns * G(ns + l + 1) * G(ns - l))
    am = abs(m)
    flm = (2 * l + 1) * 0.5 * G(l + am + 1) / (2 ** am * G(am + 1) * G(l - am + 1))
    al = 2 * gk ** 2 / (1 + gk ** 2)
    g = 3 / (2 * gk) * ((1 + 1 / (2 * gk ** 2)) * np.arcsinh(gk) - np.sqrt(1 + gk ** 2) / (2 * gk))
    ex = -(2 * (2 * U) ** 1.5) / (3 * Ea) * g
    pre = U * cnl * flm * np.sqrt(6 / np.pi) * ((2 * (2 * U) ** 1.5) / Ea) ** (2 * ns - am - 1.5) * \
        (1 + gk ** 2) ** (am / 2 + 0.75 - ns)
    nu = (U / wa) * (1 + 1 / (2 * gk ** 2))
    k0 = np.ceil(nu)
    A = np.zeros_like(Ea)
    for k in range(15):
        A += np.exp(-al * (2 * (k0 + k - nu) * np.sqrt(1 + gk ** 2) / (gk ** 2 + 1e-20)))
    return pre * A * np.exp(ex) / 2.418884e-17


class RealFieldMedium:
    """Constants and tables of a real-field medium (media_physics.py:121-183)."""

    def __init__(self, center_wavelength, *, n0, n2, n4=0.0, Ui_eV, rho_nt, tau_rec, tau_c, avalanche=False):
        self.lambda0, self.c = center_wavelength, C0
        self.omega0 = 2 * np.pi * C0 / center_wavelength
        self.n0, self.n2, self.n4 = n0, n2, n4
        self.chi3 = (4.0 / 3.0) * C0 * EPS0 * n0 ** 2 * n2
        self.chi5 = (4.0 / 5.0) * C0 ** 2 * EPS0 ** 2 * n0 ** 3 * n4 if n4 else 0.0
        self.Ui = Ui_eV * E_CH
        self.rho_nt, self.tau_rec, self.tau_c = rho_nt, tau_rec, tau_c
        self.avalanche = avalanche
        self.log10_I = np.linspace(np.log10(1e8 * 1e4), np.log10(1e16 * 1e4), 2000)
        self.W = ppt_rate(10 ** self.log10_I, self.omega0, self.Ui, n0)

    def aval_coef(self):
        """W_ava = (sigma_drude / Ui) I (media_physics.py:247-252); 0 for the gases."""
        if not self.avalanche:
            return 0.0
        s = (E_CH ** 2 * self.tau_c) / (C0 * EPS0 * self.n0 * M_E * (1.0 + self.omega0 ** 2 * self.tau_c ** 2))
        return s / self.Ui


class CauchyGas(RealFieldMedium):
    """Rare gases and their Cauchy index 1 + (A + B/l^2 + C/l^4) P (e.g. :537-543)."""

    def __init__(self, center_wavelength, pressure_atm, A, B, Cc, n2_1atm, n4_1atm, Ui_eV, tau_c_1atm):
        P = pressure_atm
        self.pressure, self.cauchy = P, (A, B, Cc)
        super().__init__(center_wavelength, n0=1.0 + A * P, n2=n2_1atm * P, n4=n4_1atm * P ** 2, Ui_eV=Ui_eV,
                         rho_nt=2.45e25 * P, tau_rec=1.0e-9, tau_c=tau_c_1atm / P)

    def refractive_index(self, w):
        w = np.asarray(w, dtype=np.float64)
        ws = np.where(np.abs(w) < 1e-12, 1e-12, w)
        l2 = ((2 * np.pi * C0 / np.abs(ws)) * 1e6) ** 2
        A, B, Cc = self.cauchy
        return 1.0 + (A + B / l2 + Cc / l2 ** 2) * (self.pressure / 1.0)


def Helium(lam, pressure_atm=1.0):
    """:426-466"""
    return CauchyGas(lam, pressure_atm, 3.48e-5, 5.4e-8, 1.2e-10, 4.0e-25, -1.0e-38, 24.59, 500e-15)


def Neon(lam, pressure_atm=1.0):
    """:469-506"""
    return CauchyGas(lam, pressure_atm, 6.66e-5, 2.4e-8, 1.7e-10, 2.0e-24, -5.0e-38, 21.56, 350e-15)


def Argon(lam, pressure_atm=1.0):
    """:509-546"""
    return CauchyGas(lam, pressure_atm, 27.9e-5, 12.8e-8, 5.2e-10, 1.0e-23, -1.0e-36, 15.76, 190e-15)


def Krypton(lam, pressure_atm=1.0):
    """:549-586"""
    return CauchyGas(lam, pressure_atm, 41.9e-5, 21.3e-8, 8.4e-10, 2.8e-23, -2.5e-36, 14.00, 150e-15)


def Xenon(lam, pressure_atm=1.0):
    """:589-626"""
    return CauchyGas(lam, pressure_atm, 68.7e-5, 40.6e-8, 16.3e-10, 6.5e-23, -8.0e-36, 12.13, 120e-15)


class Air(RealFieldMedium):
    """:392-420: constant index, no avalanche."""

    def __init__(self, center_wavelength, pressure_atm=1.0):
        self.pressure = pressure_atm
        super().__init__(center_wavelength, n0=1.0 + 0.00027 * pressure_atm, n2=3.0e-23 * pressure_atm,
                         Ui_eV=12.1, rho_nt=2.7e25 * pressure_atm, tau_rec=1.0e-9, tau_c=350e-15 / pressure_atm)

    def refractive_index(self, w):
        return np.ones_like(np.asarray(w, dtype=np.float64)) * self.n0


class FusedSilica(RealFieldMedium):
    """:321-390: Sellmeier index (clipped to 0.2-6 um), avalanche on, and with
    use_raman the delayed response f_R = 0.18, tau1 = 12.2 fs, tau2 = 32 fs: the
    solver convolves E^2 with it on the device (k_rf_line)."""

    def __init__(self, center_wavelength, use_raman=False):
        super().__init__(center_wavelength, n0=1.45, n2=3.0e-20, Ui_eV=9.0, rho_nt=2.1e28, tau_rec=150e-15,
                         tau_c=3.0e-15, avalanche=True)
        self.B = (0.6961663, 0.4079426, 0.8974794)
        self.C = (0.0684043 ** 2, 0.1162414 ** 2, 9.896161 ** 2)
        self.use_raman = bool(use_raman)
        self.f_R, self.tau1, self.tau2 = 0.18, 12.2e-15, 32.0e-15

    def raman_response(self, Nt, dt, float_dtype):
        """init_raman (:362-374): h(t) = (t1^2 + t2^2)/(t1 t2^2) exp(-t/t2) sin(t/t1)
        on 2 Nt samples of the solver precision with h(0) = 0, H = fft(h) dt / |H(0)|;
        returns H_k for k = 0..Nt (the rest is the conjugate mirror)."""
        t = np.arange(2 * Nt, dtype=float_dtype) * dt
        a = (self.tau1 ** 2 + self.tau2 ** 2) / (self.tau1 * self.tau2 ** 2)
        h = a * np.exp(-t / self.tau2) * np.sin(t / self.tau1)
        h[0] = 0.0
        H = np.fft.fft(h) * dt
        norm = float(np.abs(H[0]))
        if norm > 1e-20:
            H = H / norm
        cd = np.complex64 if float_dtype == np.float32 else np.complex128
        return H.astype(cd)[:Nt + 1]

    def refractive_index(self, w):
        w = np.asarray(w, dtype=np.float64)
        ws = np.where(np.abs(w) < 1e-12, 1e-12, w)
        lam = np.clip(2 * np.pi * C0 / np.abs(ws), 0.2e-6, 6.0e-6)
        l2 = (lam * 1e6) ** 2
        n2 = np.ones_like(lam)
        for b, c in zip(self.B, self.C):
            n2 = n2 + b * l2 / (l2 - c)
        return np.sqrt(n2)


def rf_tables(x, y, t, medium):
    """Per-omega and per-(x, y) tables of solver_3d.py:28-110 (FP64)."""
    x, y, t = (np.asarray(v, dtype=np.float64) for v in (x, y, t))
    Nx, Ny, Nt = len(x), len(y), len(t)
    dx, dy, dt = x[1] - x[0], y[1] - y[0], t[1] - t[0]
    kx = 2 * np.pi * np.fft.fftfreq(Nx, dx)
    ky = 2 * np.pi * np.fft.fftfreq(Ny, dy)
    kp2 = (kx[:, None] ** 2 + ky[None, :] ** 2).reshape(-1)
    w = 2 * np.pi * np.fft.rfftfreq(Nt, dt)
    ws = np.where(w == 0, 1e-12, w)
    k = medium.refractive_index(ws) * ws / C0
    w0 = medium.omega0
    k0 = float(medium.refractive_index(np.array([w0]))[0]) * w0 / C0
    dw = w0 * 1e-3
    kp = float(medium.refractive_index(np.array([w0 + dw]))[0]) * (w0 + dw) / C0
    kref = ((kp - k0) / dw) * w
    f = w / (2 * np.pi)
    filt = np.exp(-(f / (0.85 * (np.max(f) + 1e-10))) ** 16)
    return {'kk': k ** 2, 'kref': kref, 'w': w, 'filt': filt, 'kperp2': kp2, 'freq_axis_hz': f}


class ERK43_RealField_UPPE_3D:
    """Mirror of ERK43_RealField_UPPE_3D (solver_3d.py:7-241); precision
    'single' (float32 fields, the reference's working precision) or 'double'."""

    def __init__(self, x_grid, y_grid, t_grid, medium, precision='single', device=None):
        self._lib = _lib.load()
        self.medium = medium
        self.c, self.lambda0, self.omega0 = medium.c, medium.lambda0, medium.omega0
        self.precision = precision
        self.float_dtype = torch.float32 if precision == 'single' else torch.float64
        self.device = torch.device(device if device is not None else 'cuda')
        fd = np.float32 if precision == 'single' else np.float64
        self.x, self.y, self.t = (np.asarray(v, dtype=np.float64) for v in (x_grid, y_grid, t_grid))
        self.Nx, self.Ny, self.Nt = len(self.x), len(self.y), len(self.t)
        self.dt = float(self.t[1] - self.t[0])
        tb = rf_tables(self.x, self.y, self.t, medium)
        self.freq_axis_hz = tb['freq_axis_hz']
        xs = self.x.astype(fd)
        ys = self.y.astype(fd)
        X, Y = np.meshgrid(xs, ys, indexing='ij')
        R = np.sqrt(X ** 2 + Y ** 2)
        hw = float(np.max(np.abs(xs)))
        s = np.clip((R - 0.85 * hw) / (0.98 * hw - 0.85 * hw + 1e-30), 0.0, 1.0)
        damp = (120.0 * s ** 10).astype(fd).astype(np.float64).reshape(-1)          # :99-110
        m = medium
        self._keep = {k: np.ascontiguousarray(v, dtype=np.float64) for k, v in tb.items()}
        self._keep['damp'] = np.ascontiguousarray(damp)
        self._keep['lx'] = np.ascontiguousarray(m.log10_I)
        self._keep['lw'] = np.ascontiguousarray(m.W)
        d = _lib.DescRF()
        d.Nx, d.Ny, d.Nt = self.Nx, self.Ny, self.Nt
        d.precision = _lib.UPPE_C64 if precision == 'single' else _lib.UPPE_C128
        d.dt = self.dt
        P = lambda k: self._keep[k].ctypes.data
        d.kk, d.kref, d.w, d.filt, d.kperp2, d.damp = P('kk'), P('kref'), P('w'), P('filt'), P('kperp2'), P('damp')
        d.lut_n, d.lut_log10I, d.lut_W = len(m.log10_I), P('lx'), P('lw')
        d.I_coef = 0.5 * EPS0 * C0 * m.n0
        d.aval_coef = m.aval_coef()
        d.chi3e, d.chi5e = EPS0 * m.chi3, EPS0 * m.chi5
        d.rate_rec, d.rho_nt, d.Ui = 1.0 / m.tau_rec, m.rho_nt, m.Ui
        d.e_charge, d.m_e, d.tau_c = E_CH, M_E, m.tau_c
        if getattr(m, 'use_raman', False):
            H = m.raman_response(self.Nt, self.dt, fd).astype(np.complex128)
            self._keep['ramH'] = np.ascontiguousarray(H.view(np.float64))
            d.raman_H, d.raman_fR = P('ramH'), m.f_R
        plan = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            _lib.check(self._lib.uppe_rf_plan_create(ctypes.byref(d), ctypes.byref(plan)), 'uppe_rf_plan_create')
        self._plan = plan
        self.E_scale = 1.0

    def __del__(self):
        plan = getattr(self, '_plan', None)
        if plan is not None and plan.value:
            self._lib.uppe_rf_plan_destroy(plan)
            self._plan = None

    def set_field(self, E0, stream=None):
        E = E0 if isinstance(E0, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(E0))
        E = E.to(device=self.device, dtype=self.float_dtype).contiguous()
        sc = ctypes.c_double()
        _lib.check(self._lib.uppe_rf_set_field(self._plan, ctypes.c_void_p(E.data_ptr()), ctypes.byref(sc),
                                               _lib.stream_ptr(stream)), 'uppe_rf_set_field')
        self.E_scale = sc.value
        return E

    def attempt(self, h, stream=None):
        err = ctypes.c_double()
        _lib.check(self._lib.uppe_rf_attempt(self._plan, float(h), ctypes.byref(err), _lib.stream_ptr(stream)),
                   'uppe_rf_attempt')
        return err.value

    def commit(self, accept, stream=None):
        _lib.check(self._lib.uppe_rf_commit(self._plan, 1 if accept else 0, _lib.stream_ptr(stream)), 'uppe_rf_commit')

    def field(self, stream=None):
        out = torch.empty((self.Nx, self.Ny, self.Nt), dtype=self.float_dtype, device=self.device)
        _lib.check(self._lib.uppe_rf_get_field(self._plan, ctypes.c_void_p(out.data_ptr()), _lib.stream_ptr(stream)),
                   'uppe_rf_get_field')
        return out

    def spectrum(self, stream=None):
        nw = self._lib.uppe_rf_spec_bins(self._plan)
        cd = torch.complex64 if self.precision == 'single' else torch.complex128
        out = torch.empty((self.Nx, self.Ny, nw), dtype=cd, device=self.device)
        _lib.check(self._lib.uppe_rf_get_spectrum(self._plan, ctypes.c_void_p(out.data_ptr()),
                                                  _lib.stream_ptr(stream)), 'uppe_rf_get_spectrum')
        return out[:, :, :self.Nt // 2 + 1]

    def propagate(self, E0, L, tol=1e-4, max_step=1e-2, min_step=1e-9, return_gpu=False, max_attempts=2_000_000):
        """solver_3d.py:177-241 -> (z, freq_axis_hz, rfft_t(E) of the final field).
        The loop (accept when err < tol or h at min_step, factor 0.9 (tol/err)^0.333,
        growth <= 2 and <= 1.2 after forced steps) runs on the host, one error read
        per attempt as in the reference; the attempt budget bounds it."""
        self.set_field(E0)
        z, h, fail, n = 0.0, min(max_step, L / 1000.0), 0, 0
        self.log = []
        while z < L and n < max_attempts:
            if h > L - z:
                h = L - z
                if h < 1e-15:
                    break
            err = self.attempt(h)
            n += 1
            self.log.append((h, err))
            if not np.isfinite(err):
                raise FloatingPointError(f'non-finite error at z = {z:.6e} m (h = {h:.3e} m)')
            if err < tol or h <= min_step * 1.01:
                fail = fail + 1 if (h <= min_step * 1.01 and err > tol) else 0
                self.commit(True)
                z += h
                err = max(err, 1e-30)
                f = 0.9 * (tol / err) ** 0.333
                if fail > 0:
                    f = min(f, 1.2)
                h = max(min(h * min(f, 2.0), max_step), min_step)
            else:
                self.commit(False)
                err = max(err, 1e-30)
                h = max(h * 0.9 * (tol / err) ** 0.333, min_step)
        Ew = self.spectrum()
        self.z = z
        if return_gpu:
            return z, self.freq_axis_hz, Ew
        return z, self.freq_axis_hz, Ew.cpu().numpy()
