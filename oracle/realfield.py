"""Restatement of the real-field 3+1D ERK4(3)-IP UPPE solver
(``src/3+1D-UPPE-ERK4(3)IP-real-field/solver_3d.py``) and its media
(``media_physics.py``: PPT ionisation table :121-246, density + Drude current
kernel :11-118, nonlinear response :258-318, gases and fused silica :321-626),
vectorised over (x, y) and serial over t where the reference kernel is.
Test infrastructure only; pinned to fixtures generated by running the
reference here (tests/golden/make_golden.py, single precision: the reference's
density kernel reads the field as float32).
"""
import numpy as np
from scipy.fft import fft, fft2, fftfreq, ifft, ifft2, irfft, rfft, rfftfreq
from scipy.special import gamma as G

C0 = 299792458.0
E_CH = 1.60217663e-19
EPS0 = 8.85418781e-12
M_E = 9.1093837e-31


class Medium:
    """OpticalMedium (:121-318) with the subclass constants passed in."""

    def __init__(self, lam, precision='single', *, n0, n2, n4=0.0, Ui_eV, rho_nt, tau_rec, tau_c,
                 dispersion, avalanche=False, Z=1.0, l=0, m=0):
        self.lambda0, self.c = lam, C0
        self.omega0 = 2 * np.pi * C0 / lam
        self.e_charge, self.eps0, self.m_e = E_CH, EPS0, M_E
        self.n0, self.n2, self.n4 = n0, n2, n4
        self.chi3 = (4.0 / 3.0) * C0 * EPS0 * n0 ** 2 * n2                      # e.g. :511
        self.chi5 = (4.0 / 5.0) * C0 ** 2 * EPS0 ** 2 * n0 ** 3 * n4 if n4 else 0.0
        self.Ui = Ui_eV * E_CH
        self.rho_nt, self.tau_rec, self.tau_c = rho_nt, tau_rec, tau_c
        self.Z, self.l, self.m = Z, l, m
        self.dispersion = dispersion
        self.avalanche = avalanche
        self.float_dtype = np.float64 if precision == 'double' else np.float32
        x = np.linspace(np.log10(1e8 * 1e4), np.log10(1e16 * 1e4), 2000)       # :167-175
        self.log10_I_cpu = x
        self.log10_I_gpu = x.astype(self.float_dtype)
        self.W_gpu = ppt_rate(10 ** x, self).astype(self.float_dtype)
        self.use_raman = False
        self.H_raman = None

    def init_raman(self, Nt, dt):
        """:362-374: h(t) = (t1^2 + t2^2)/(t1 t2^2) exp(-t/t2) sin(t/t1) on 2 Nt samples
        of the solver precision, h(0) = 0, H = fft(h) dt / |H[0]|."""
        if not self.use_raman:
            return
        t = np.arange(2 * Nt, dtype=self.float_dtype) * dt
        a = (self.tau1 ** 2 + self.tau2 ** 2) / (self.tau1 * self.tau2 ** 2)
        h = a * np.exp(-t / self.tau2) * np.sin(t / self.tau1)
        h[0] = 0.0
        H = fft(h) * dt
        norm = float(np.abs(H[0]))
        if norm > 1e-20:
            H = H / norm
        cd = np.complex128 if self.float_dtype == np.float64 else np.complex64
        self.H_raman = H.astype(cd)

    def raman_intensity(self, E):
        """:376-390: the E^2 history through the Raman response, a circular convolution
        of length 2 Nt of the zero-padded E^2 (real part, first Nt samples)."""
        Nt = E.shape[-1]
        pad = [(0, 0)] * (E.ndim - 1) + [(0, Nt)]
        Iw = fft(np.pad(E ** 2, pad, mode='constant'), axis=-1)
        return np.real(ifft(Iw * self.H_raman, axis=-1))[..., :Nt]

    def refractive_index(self, w):
        kind = self.dispersion[0]
        w64 = np.asarray(w, dtype=np.float64)
        if kind == 'const':                                                    # Air :414-416
            return np.ones_like(w64) * self.n0
        ws = np.where(np.abs(w64) < 1e-12, 1e-12, w64)
        if kind == 'cauchy':                                                   # gases, e.g. :537-543
            _, A, B, Cc, P = self.dispersion
            wl_sq = ((2 * np.pi * C0 / np.abs(ws)) * 1e6) ** 2
            return 1.0 + (A + B / wl_sq + Cc / wl_sq ** 2) * (P / 1.0)
        _, Bs, Cs, lo, hi = self.dispersion                                    # Sellmeier :350-360
        wl = np.clip(2 * np.pi * C0 / np.abs(ws), lo, hi)
        wl_sq = (wl * 1e6) ** 2
        n_sq = np.ones_like(wl)
        for b, c in zip(Bs, Cs):
            n_sq = n_sq + b * wl_sq / (wl_sq - c)
        return np.sqrt(n_sq)

    def ionization_rate(self, I):
        """:177-183"""
        logI = np.clip(np.log10(I + 1e-30), float(self.log10_I_gpu[0]), float(self.log10_I_gpu[-1]))
        return np.interp(logI.ravel(), self.log10_I_gpu, self.W_gpu).reshape(logI.shape)

    def avalanche_rate(self, I):
        """:247-252 (fused silica); zero for the gases (e.g. :418-420)."""
        if not self.avalanche:
            return np.zeros_like(I, dtype=self.float_dtype)
        s = (E_CH ** 2 * self.tau_c) / (C0 * EPS0 * self.n0 * M_E * (1.0 + self.omega0 ** 2 * self.tau_c ** 2))
        return (s / self.Ui) * I

    def response(self, E, dt):
        """:258-318 -> (P_NL, J) in the solver precision."""
        I = 0.5 * EPS0 * C0 * self.n0 * E ** 2
        Wi = np.ascontiguousarray(self.ionization_rate(I).astype(np.float32))
        Wa = np.ascontiguousarray(self.avalanche_rate(I).astype(np.float32))
        Nt = E.shape[-1]
        J, rho = density_current(E.reshape(-1, Nt).astype(np.float32), Wi.reshape(-1, Nt), Wa.reshape(-1, Nt),
                                 np.float32(1.0 / self.tau_rec), np.float32(dt), np.float32(self.rho_nt),
                                 np.float32(self.Ui), np.float32(E_CH), np.float32(M_E), np.float32(self.tau_c))
        c3 = EPS0 * self.chi3
        if self.use_raman and self.H_raman is not None:                        # :303-305
            Eeff = (1 - self.f_R) * (E ** 2) + self.f_R * self.raman_intensity(E)
            P = c3 * E * Eeff
        else:
            P = ((c3 * E) * E) * E
        if self.chi5 != 0.0:
            c5 = EPS0 * self.chi5
            E2 = E * E
            P = P + ((c5 * E) * E2) * E2
        return P.astype(self.float_dtype), J.reshape(E.shape).astype(self.float_dtype)


def ppt_rate(I, m):
    """PPT rate [1/s] of intensity I [W/m^2] (media_physics.py:185-246)."""
    Is = np.maximum(I, 1e4)
    E_au = np.sqrt(2 * Is / (C0 * EPS0 * m.n0)) / 5.142206538e11
    w_au = m.omega0 * 2.418884e-17
    U = m.Ui / (27.21138 * E_CH)
    gk = w_au * np.sqrt(2 * U) / E_au
    ns = m.Z / np.sqrt(2 * U)
    Cnl2 = 2 ** (2 * ns) / (ns * G(ns + m.l + 1) * G(ns - m.l))
    am = abs(m.m)
    flm = (2 * m.l + 1) * 0.5 * G(m.l + am + 1) / (2 ** am * G(am + 1) * G(m.l - am + 1))
    alpha = 2 * gk ** 2 / (1 + gk ** 2)
    g = 3 / (2 * gk) * ((1 + 1 / (2 * gk ** 2)) * np.arcsinh(gk) - np.sqrt(1 + gk ** 2) / (2 * gk))
    expo = -(2 * (2 * U) ** 1.5) / (3 * E_au) * g
    pre = U * Cnl2 * flm * np.sqrt(6 / np.pi) * ((2 * (2 * U) ** 1.5) / E_au) ** (2 * ns - am - 1.5) * \
        (1 + gk ** 2) ** (am / 2 + 0.75 - ns)
    nu = (U / w_au) * (1 + 1 / (2 * gk ** 2))
    K0 = np.ceil(nu)
    A = np.zeros_like(E_au)
    for k in range(15):
        A += np.exp(-alpha * (2 * (K0 + k - nu) * np.sqrt(1 + gk ** 2) / (gk ** 2 + 1e-20)))
    return pre * A * np.exp(expo) / 2.418884e-17


def density_current(E, Wi, Wa, rr, dt, rho_nt, Ui, e, me, tau_c):
    """media_physics.py:11-118: float32 inputs, float64 state; J = J_free + J_loss."""
    nl, Nt = E.shape
    J = np.zeros((nl, Nt))
    rho_o = np.zeros((nl, Nt))
    rho = np.zeros(nl)
    Jf = np.zeros(nl)
    rnt, rrd, dtd, Uid = float(rho_nt), float(rr), float(dt), float(Ui)
    nu = 1.0 / float(tau_c)
    e2m = float(e) * float(e) / float(me)
    for t in range(Nt):
        Et = E[:, t].astype(np.float64)
        wp = Wi[:, t].astype(np.float64)
        wa = Wa[:, t].astype(np.float64)
        dep = np.maximum((rnt - rho) / rnt, 0.0)
        S = wp * rnt * dep
        Gm = wa * dep - rrd
        gdt = np.clip(Gm * dtd, -10.0, 10.0)
        eg = np.exp(gdt)
        with np.errstate(divide='ignore', invalid='ignore'):
            sf = np.where(np.abs(gdt) < 1e-5, dtd * (1.0 + 0.5 * gdt), (eg - 1.0) / Gm)
        nrho = np.minimum(np.maximum(rho * eg + S * sf, 0.0), rnt)
        nrho = np.minimum(rho * eg + S * sf, rnt)
        nrho = np.maximum(nrho, 0.0)
        gen = S + wa * dep * rho
        drive = e2m * rho * Et
        ndt = nu * dtd
        en = np.exp(-ndt)
        sJ = dtd * (1.0 - 0.5 * ndt) if abs(ndt) < 1e-5 else (1.0 - en) / nu
        nJ = Jf * en + drive * sJ
        with np.errstate(divide='ignore', invalid='ignore'):
            Jl = np.where(np.abs(Et) > 1e-10, (gen * Uid * Et) / (Et * Et + 1e-20), 0.0)
        J[:, t] = Jf + Jl
        rho_o[:, t] = rho
        rho, Jf = nrho, nJ
    return J, rho_o


def argon(lam, P=1.0, precision='single'):
    """:509-547"""
    return Medium(lam, precision, n0=1.0 + 27.9e-5 * P, n2=1.0e-23 * P, n4=-1.0e-36 * P ** 2, Ui_eV=15.76,
                  rho_nt=2.45e25 * P, tau_rec=1e-9, tau_c=190e-15 / P,
                  dispersion=('cauchy', 27.9e-5, 12.8e-8, 5.2e-10, P))


def xenon(lam, P=1.0, precision='single'):
    """:589-626"""
    return Medium(lam, precision, n0=1.0 + 68.7e-5 * P, n2=6.5e-23 * P, n4=-8.0e-36 * P ** 2, Ui_eV=12.13,
                  rho_nt=2.45e25 * P, tau_rec=1e-9, tau_c=120e-15 / P,
                  dispersion=('cauchy', 68.7e-5, 40.6e-8, 16.3e-10, P))


def fused_silica(lam, precision='single', use_raman=False):
    """:321-390 (Raman fraction 0.18, tau1 12.2 fs, tau2 32 fs)"""
    m = Medium(lam, precision, n0=1.45, n2=3.0e-20, Ui_eV=9.0, rho_nt=2.1e28, tau_rec=150e-15, tau_c=3.0e-15,
               dispersion=('sellmeier', [0.6961663, 0.4079426, 0.8974794],
                           [0.0684043 ** 2, 0.1162414 ** 2, 9.896161 ** 2], 0.2e-6, 6.0e-6), avalanche=True)
    m.use_raman, m.f_R, m.tau1, m.tau2 = use_raman, 0.18, 12.2e-15, 32.0e-15
    return m


class Solver:
    """ERK43_RealField_UPPE_3D (solver_3d.py:7-241)."""

    def __init__(self, x, y, t, medium, precision='single'):
        self.medium = medium
        self.fd = np.float64 if precision == 'double' else np.float32
        self.cd = np.complex128 if precision == 'double' else np.complex64
        x, y, t = (np.asarray(v, dtype=np.float64) for v in (x, y, t))
        self.x, self.y, self.t = x.astype(self.fd), y.astype(self.fd), t.astype(self.fd)
        self.Nx, self.Ny, self.Nt = len(x), len(y), len(t)
        self.dx, self.dy, self.dt = float(x[1] - x[0]), float(y[1] - y[0]), float(t[1] - t[0])
        kx = 2 * np.pi * fftfreq(self.Nx, self.dx)
        ky = 2 * np.pi * fftfreq(self.Ny, self.dy)
        KX, KY = np.meshgrid(kx, ky, indexing='ij')
        self.K2 = (KX ** 2 + KY ** 2).astype(np.float64)                       # :31-32
        self.w = 2 * np.pi * rfftfreq(self.Nt, self.dt)                        # :35
        self.freq_axis_hz = self.w / (2 * np.pi)
        if hasattr(self.medium, 'init_raman'):                                 # :40-41
            self.medium.init_raman(self.Nt, self.dt)
        self._operators()
        X, Y = np.meshgrid(self.x, self.y, indexing='ij')                       # :101-110
        R = np.sqrt(X ** 2 + Y ** 2)
        hw = float(np.max(np.abs(self.x)))
        s = np.clip((R - 0.85 * hw) / (0.98 * hw - 0.85 * hw + 1e-30), 0.0, 1.0)
        self.damp = (120.0 * s ** 10)[:, :, None].astype(self.fd)
        fmax = float(np.max(self.freq_axis_hz)) + 1e-10                        # :50-52
        self.filt = np.exp(-(self.freq_axis_hz / (0.85 * fmax)) ** 16).astype(self.fd)[None, None, :].astype(self.cd)
        self.E_scale = 1.0

    def _operators(self):
        """:56-97"""
        m, w = self.medium, self.w
        ws = np.where(w == 0, 1e-12, w)
        k = m.refractive_index(ws) * ws / C0
        w0 = m.omega0
        k0 = float(m.refractive_index(np.array([w0]))[0]) * w0 / C0
        dw = w0 * 1e-3
        kp = float(m.refractive_index(np.array([w0 + dw]))[0]) * (w0 + dw) / C0
        kref = ((kp - k0) / dw) * w
        kz2 = (k ** 2)[None, None, :] - self.K2[:, :, None]
        kz = np.where(kz2 >= 0, np.sqrt(kz2.astype(np.complex128)), -1j * np.sqrt(np.abs(kz2)).astype(np.complex128))
        self.D = (-1j * (kz - kref[None, None, :])).astype(self.cd)
        kzs = np.where(np.abs(kz) < 1e-10, 1e-10, kz)
        self.Pc = (-1j * w ** 2 / (2 * EPS0 * C0 ** 2 * kzs)).astype(self.cd)
        self.Jc = (-w / (2 * EPS0 * C0 ** 2 * kzs)).astype(self.cd)
        self.Pc[:, :, 0] = 0.0
        self.Jc[:, :, 0] = 0.0

    def N(self, Ekw):
        """:120-141"""
        Et = irfft(ifft2(Ekw, axes=(0, 1)), n=self.Nt, axis=-1)
        P, J = self.medium.response(Et * self.E_scale, self.dt)
        Pw = rfft(P / self.E_scale, axis=-1)
        Jw = rfft(J / self.E_scale, axis=-1)
        return fft2(self.Pc * Pw + self.Jc * Jw, axes=(0, 1))

    def step(self, Et, h):
        """erk43_step (:113-175) -> (E4_t, err)."""
        L = lambda f, s: f * np.exp(s * self.D)
        Ekw = fft2(rfft(Et, axis=-1), axes=(0, 1))
        v = L(Ekw, h / 2)
        k1 = self.N(Ekw)
        a1 = L(k1, h / 2)
        a2 = self.N(v + (h / 2) * a1)
        a3 = self.N(v + (h / 2) * a2)
        a4 = self.N(L(v + h * a3, h / 2))
        ts = a1 + 2 * a2 + 2 * a3
        E4 = L(v + (h / 6) * ts, h / 2) + (h / 6) * a4
        El = L(v + (h / 2) * a1 + (h / 2) * a2, h / 2)
        err = float(np.max(np.abs(E4 - El)) / (np.max(np.abs(E4)) + 1e-20))
        E4w = ifft2(E4, axes=(0, 1)) * self.filt
        E4t = irfft(E4w, n=self.Nt, axis=-1)
        E4t = E4t * np.exp(-self.damp * h)
        return E4t, err

    def propagate(self, E0, L, tol=1e-4, max_step=1e-2, min_step=1e-9, schedule=None):
        """:177-241; schedule = [(h, accepted)] replays a recorded attempt sequence."""
        E0 = np.asarray(E0, dtype=self.fd)
        self.E_scale = float(np.max(np.abs(E0)))
        if self.E_scale < 1e-30:
            self.E_scale = 1.0
        E = (E0 / self.fd(self.E_scale)).astype(self.fd)
        z, log = 0.0, []
        if schedule is not None:
            for h, acc in schedule:
                En, err = self.step(E, h)
                log.append((h, err))
                if acc:
                    z, E = z + h, En
        else:
            h = min(max_step, L / 1000.0)
            fail = 0
            while z < L:
                if h > L - z:
                    h = L - z
                    if h < 1e-15:
                        break
                En, err = self.step(E, h)
                log.append((h, err))
                if not np.isfinite(err):   # the reference would loop forever on NaN
                    break
                if err < tol or h <= min_step * 1.01:
                    fail = fail + 1 if (h <= min_step * 1.01 and err > tol) else 0
                    z += h
                    E = En
                    err = max(err, 1e-30)
                    f = 0.9 * (tol / err) ** 0.333
                    if fail > 0:
                        f = min(f, 1.2)
                    h = max(min(h * min(f, 2.0), max_step), min_step)
                else:
                    err = max(err, 1e-30)
                    h = max(h * 0.9 * (tol / err) ** 0.333, min_step)
        self.last_state = E
        return z, self.freq_axis_hz, rfft(E * self.E_scale, axis=-1), log
