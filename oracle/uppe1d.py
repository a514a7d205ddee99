"""CPU oracle (test infrastructure only): numpy restatement of the reference 1D
ERK4(3)-IP UPPE/GNLSE solver.

Restates ``src/1D-ERK4(3)IP UPPE gas/erk43ip_method.py`` (class ``ERK43IP_UPPE``)
and the argon patch ``src/1D-ERK4(3)IP UPPE gas/gas.py:14-44`` operation by
operation.  The state is kept in the time domain as the reference does.

Extensions (N-new, parity unpinned by the reference):
  * ``taylor=(beta2, beta3)``: D(w) = i(b2 w^2/2 + b3 w^3/6) - alpha/2 and
    n(w) = n0 + c (b2 w^2/2 + b3 w^3/6) / w_abs for the UPPE factor;
  * ``plasma=dict(...)``: the envelope plasma term of media_physics.py:156-205
    (ADK LUT, the scan of media_physics.py:11-67, loss + defocusing) with the
    intensity I = |A|^2 / A_eff, added to N(A) in the time domain.
"""
import numpy as np
from scipy.fft import fft, ifft, fftfreq

from . import adk as _adk
from .uppe3d import plasma_scan

C0 = 299792458.0

SELLMEIER = {   # erk43ip_method.py:74-90
    'fused_silica': {'B': [0.6961663, 0.4079426, 0.8974794],
                     'C': [0.0684043 ** 2, 0.1162414 ** 2, 9.896161 ** 2],
                     'valid_range': (0.21e-6, 6.7e-6)},
    'sapphire': {'B': [1.4313493, 0.65054713, 5.3414021],
                 'C': [0.0726631 ** 2, 0.1193242 ** 2, 18.028251 ** 2],
                 'valid_range': (0.2e-6, 5.5e-6)},
    'yag': {'B': [2.282, 3.27644, 4.44174],
            'C': [0.01185 ** 2, 0.0282 ** 2, 282.734 ** 2],
            'valid_range': (0.4e-6, 5e-6)},
}


class Plasma1D:
    """Envelope plasma parameters for the 1D N-new plasma term (argon defaults)."""

    def __init__(self, A_eff, pressure_atm=1.0, Ui_eV=15.76, rho_nt=None, tau_rec=1e-9,
                 tau_c=None, center_wavelength=800e-9, adk_prefactor=2.5e15):
        e = 1.60217663e-19
        self.A_eff = A_eff
        self.Ui = Ui_eV * e
        self.rho_nt = 2.45e25 * pressure_atm if rho_nt is None else rho_nt
        self.tau_rec = tau_rec
        self.tau_c = 190e-15 / pressure_atm if tau_c is None else tau_c
        omega0 = 2 * np.pi * C0 / center_wavelength
        self.sigma = (e ** 2 * self.tau_c) / (C0 * 8.85418781e-12 * 1.0 * 9.1093837e-31
                                              * (1.0 + omega0 ** 2 * self.tau_c ** 2))
        self.omega0 = omega0
        self.log10_I, W = _adk.ionization_lut(self.Ui, n0=1.0, prefactor=adk_prefactor)
        self.W = W

    def term(self, A, dt):
        """Plasma(A) [1/m * A] following media_physics.py:165-203 with I = |A|^2/A_eff."""
        I = np.abs(A) ** 2 / self.A_eff
        log_I = np.clip(np.log10(I + 1e-30), self.log10_I[0], self.log10_I[-1])
        W_ion = np.interp(log_I, self.log10_I, self.W).astype(np.float32)
        W_ava = np.zeros_like(W_ion)
        rho, gen = plasma_scan(W_ion[None, :], W_ava[None, :], np.float32(1.0 / self.tau_rec),
                               np.float32(dt), np.float32(self.rho_nt))
        rho, gen = rho[0], gen[0]
        loss = -(gen * self.Ui) / (2.0 * I + 1e-30) * A
        defocus = -(self.sigma / 2.0) * (1.0 + 1j * self.omega0 * self.tau_c) * rho * A
        return loss + defocus, rho


class Solver1D:
    """Restatement of ``ERK43IP_UPPE`` (erk43ip_method.py:14-369) + gas patch."""

    def __init__(self, material='fused_silica', gamma=None, n2=None, beam_radius=None,
                 alpha=0.0, center_wavelength=1064e-9, use_raman=True, f_R=0.18,
                 tau1=12.2e-15, tau2=32e-15, use_self_steepening=True,
                 gas_P=101325.0, gas_T=293.15, taylor=None, plasma=None, n0=None):
        self.gas_P, self.gas_T = gas_P, gas_T                     # gas.py:16-17
        self.material = material
        self.alpha = alpha
        self.lambda0 = center_wavelength
        self.c = 299792458.0
        self.omega0 = 2 * np.pi * self.c / self.lambda0          # :33
        if gamma is not None:                                     # :36-51
            self.gamma = gamma
        elif n2 is not None and beam_radius is not None:
            self.beam_area = np.pi * beam_radius ** 2
            self.gamma = (2 * np.pi / self.lambda0) * (n2 / self.beam_area)
        else:
            self.gamma = 0.0
        self.use_raman, self.f_R, self.tau1, self.tau2 = use_raman, f_R, tau1, tau2
        self.use_self_steepening = use_self_steepening
        self.taylor = taylor
        self.plasma = plasma
        self.sellmeier = SELLMEIER.get(material, SELLMEIER['fused_silica'])   # :91
        if taylor is not None:
            self.n0 = 1.0 if n0 is None else n0
        else:
            self.n0 = self.refractive_index(np.array([self.lambda0]))[0]     # :70

    # erk43ip_method.py:93-102 and gas.py:20-40
    def refractive_index(self, wavelength):
        if self.material == 'argon_gas':
            P_ref, T_ref = 101325.0, 288.15
            lam_um = wavelength * 1e6
            sigma_sq = 1.0 / (lam_um ** 2)
            n0_minus_1 = ((1205582.27 / (130.0 - sigma_sq)) + (317222.05 / (38.9 - sigma_sq))) * 1e-8
            scale = (self.gas_P / P_ref) * (T_ref / self.gas_T)
            return 1.0 + n0_minus_1 * scale
        B, C = self.sellmeier['B'], self.sellmeier['C']
        wl_sq = (wavelength * 1e6) ** 2
        n_squared = np.ones_like(wavelength, dtype=float)
        for i in range(3):
            n_squared += (B[i] * wl_sq) / (wl_sq - C[i])
        return np.sqrt(n_squared)

    def dispersion(self, omega_grid):
        """erk43ip_method.py:104-148 -> (D, n_omega)."""
        if self.taylor is not None:                               # N-new Taylor medium
            b2, b3 = self.taylor
            poly = 0.5 * b2 * omega_grid ** 2 + (1.0 / 6.0) * b3 * omega_grid ** 3
            omega_abs = self.omega0 + omega_grid
            omega_safe = np.where(np.abs(omega_abs) < 1e-10, 1e-10, omega_abs)
            n_omega = self.n0 + self.c * poly / omega_safe
            return 1j * poly - self.alpha / 2, n_omega
        omega_abs = self.omega0 + omega_grid
        omega_safe = np.where(np.abs(omega_abs) < 1e-10, 1e-10, np.abs(omega_abs))
        wavelengths = 2 * np.pi * self.c / omega_safe
        # :117-118; for 'argon_gas' the coefficient lookup (:91) falls back to the
        # fused-silica entry, so its valid range clamps the gas wavelengths too
        lo, hi = self.sellmeier['valid_range']
        wavelengths = np.clip(wavelengths, lo, hi)
        n_omega = self.refractive_index(wavelengths)
        k_omega = n_omega * omega_abs / self.c
        d_omega = self.omega0 * 1e-5
        w_center = np.array([self.lambda0])
        w_plus = 2 * np.pi * self.c / (self.omega0 + d_omega)
        w_minus = 2 * np.pi * self.c / (self.omega0 - d_omega)
        n0 = self.refractive_index(w_center)[0]
        n_plus = self.refractive_index(np.array([w_plus]))[0]
        n_minus = self.refractive_index(np.array([w_minus]))[0]
        k0 = n0 * self.omega0 / self.c
        k_plus = n_plus * (self.omega0 + d_omega) / self.c
        k_minus = n_minus * (self.omega0 - d_omega) / self.c
        k1 = (k_plus - k_minus) / (2 * d_omega)
        D = 1j * (k_omega - k0 - k1 * omega_grid) - self.alpha / 2
        return D, n_omega

    def raman_response(self, omega_grid):
        """erk43ip_method.py:150-179"""
        N = len(omega_grid)
        if N > 1:
            d_omega = omega_grid[1] - omega_grid[0]
            dt = 2 * np.pi / (N * np.abs(d_omega))
        else:
            dt = 1e-15
        dt = max(dt, 1e-15)
        t = np.arange(N) * dt
        t1, t2 = max(self.tau1, 1e-20), max(self.tau2, 1e-20)
        h_t = (t1 ** 2 + t2 ** 2) / (t1 * t2 ** 2) * np.exp(-t / t2) * np.sin(t / t1)
        h_t[0] = 0.0
        H = fft(h_t) * dt
        if np.abs(H[0]) > 1e-15:
            H = H / H[0]
        else:
            H = np.ones_like(H, dtype=complex)
        return H

    def setup(self, omega, dt):
        self._D, self._n = self.dispersion(omega)
        self._H = self.raman_response(omega) if self.use_raman else None
        self._dt = dt
        n_w_safe = np.where(self._n < 1.0, 1.0, self._n)           # :244
        self._U = ((self.omega0 + omega) / self.omega0) * (self.n0 / n_w_safe)   # :248

    def linear_operator(self, A, h):
        """erk43ip_method.py:181-195"""
        return ifft(fft(A) * np.exp(h * self._D))

    def nonlinear_operator(self, A):
        """erk43ip_method.py:197-255 (+ N-new plasma term)."""
        Intensity = np.abs(A) ** 2
        if self.use_raman and self._H is not None:
            I_delayed = ifft(fft(Intensity) * self._H)
            I_eff = (1 - self.f_R) * Intensity + self.f_R * I_delayed
        else:
            I_eff = Intensity
        P_NL_time = A * I_eff
        if self.use_self_steepening:
            out = ifft(1j * self.gamma * self._U * fft(P_NL_time))
        else:
            out = 1j * self.gamma * P_NL_time
        if self.plasma is not None:
            out = out + self.plasma.term(A, self._dt)[0]
        return out

    def diagnostics(self, A, t):
        """energy sum |A|^2 dt and photon number sum_w E_w / (hbar w_abs), w_abs > 0."""
        N = len(t)
        dt = t[1] - t[0]
        Ew = np.abs(fft(A)) ** 2 * dt / N
        wa = 2 * np.pi * fftfreq(N, dt) + self.omega0
        return float(np.sum(np.abs(A) ** 2) * dt), float(np.sum(Ew[wa > 0] / (1.054571817e-34 * wa[wa > 0])))

    def ionization_fraction(self, A):
        if self.plasma is None:
            return 0.0
        rho = self.plasma.term(A, self._dt)[1]
        return float(rho.max()) / float(np.float32(self.plasma.rho_nt))

    def erk43_step(self, A, h):
        """erk43ip_method.py:256-286 (alpha1 always from N(A): the FSAL shortcut is
        bit-identical to it)."""
        L, N = self.linear_operator, self.nonlinear_operator
        v_ip = L(A, h / 2)
        alpha1 = L(N(A), h / 2)
        alpha2 = N(v_ip + h / 2 * alpha1)
        alpha3 = N(v_ip + h / 2 * alpha2)
        temp = L(v_ip + h * alpha3, h / 2)
        alpha4_prime = N(temp)
        beta = L(v_ip + h / 6 * (alpha1 + 2 * alpha2 + 2 * alpha3), h / 2)
        A4 = beta + h / 6 * alpha4_prime
        alpha5_prime = N(A4)
        A3 = beta + (h / 30) * (2 * alpha4_prime + 3 * alpha5_prime)
        norm_A = np.sqrt(np.sum(np.abs(A4) ** 2))
        if norm_A < 1e-20:
            norm_A = 1.0
        error = np.sqrt(np.sum(np.abs(A4 - A3) ** 2)) / norm_A
        return A4, error

    def propagate(self, A0, t, L, tol=1e-4, max_step=1e-2, min_step=1e-11, schedule=None,
                  max_attempts=None):
        """erk43ip_method.py:288-369.  Returns (z_hist, A_hist, omega, log)."""
        N = len(t)
        dt = t[1] - t[0]
        omega = 2 * np.pi * fftfreq(N, dt)
        self.setup(omega, dt)
        z = 0.0
        h = max_step / 100
        A = np.array(A0, dtype=complex)
        z_history, A_history = [0.0], [A.copy()]
        log = []

        def save():
            if len(z_history) < 1000 or (z - z_history[-1]) > L / 500:
                z_history.append(z)
                A_history.append(A.copy())

        if schedule is not None:
            for h_s, acc in schedule:
                A_new, err = self.erk43_step(A, h_s)
                log.append((z, h_s, err, bool(acc)))
                if acc:
                    z += h_s
                    A = A_new
                    save()
            return np.array(z_history), np.array(A_history), omega, log
        error_prev = None
        n = 0
        while z < L:
            if z + h > L:
                h = L - z
            A_new, error = self.erk43_step(A, h)
            n += 1
            if error < tol:
                log.append((z, h, error, True))
                z += h
                A = A_new
                save()
                factor = 0.95 * (tol / (error + 1e-30)) ** 0.25
                if error_prev is not None and error_prev > 1e-30:
                    factor *= (error_prev / (error + 1e-30)) ** 0.1
                error_prev = error
                h = min(h * min(factor, 2.0), max_step)
            else:
                log.append((z, h, error, False))
                factor = 0.95 * (tol / (error + 1e-30)) ** 0.25
                h = max(h * max(factor, 0.1), min_step)
                if h <= min_step:
                    A_new, error = self.erk43_step(A, h)
                    log.append((z, h, error, True))
                    z += h
                    A = A_new
                    error_prev = None
                    save()
            if max_attempts is not None and n >= max_attempts:
                break
        return np.array(z_history), np.array(A_history), omega, log
