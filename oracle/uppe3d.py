"""CPU oracle (test infrastructure only): numpy restatement of the reference 3+1D
envelope ERK4(3)-IP UPPE solver and its gas medium plugin.

Restates
  src/3+1D-UPPE-ERK4(3)IP-envelope/solver_3d.py   (ERK43IP_UPPE_3D_Optimized)
  src/3+1D-UPPE-ERK4(3)IP-envelope/media_physics.py (OpticalMedium, Argon, plasma kernel)
operation by operation, including the reference's dtype casts, so that in
``precision='double'`` the result equals the reference's up to FFT round-off.

Plugin substitutions (N-new, parity unpinned by the reference):
  * the ionisation LUT values come from ``oracle.adk`` (ADK) instead of the
    reference's broken Keldysh formula (``media_physics.py:139-146``);
  * ``n4 = 0`` (the reference's gas n4 values overflow the first step);
  * optional Taylor dispersion: n(w) = n0 + c*(b2*W^2/2 + b3*W^3/6)/w, W = w - w0.
"""
import numpy as np
import scipy.fft as sfft

from . import adk as _adk

C0 = 299792458.0


# ---------------------------------------------------------------------------
# medium (media_physics.py:70-205, Argon :396-432)
# ---------------------------------------------------------------------------
class GasMedium:
    """A gas medium with the OpticalMedium semantics of ``media_physics.py:70-205``.

    ``dispersion`` is ``('cauchy', A, B, C)`` (``media_physics.py:423-429``) or
    ``('taylor', n0, beta2, beta3)`` (N-new).
    """

    def __init__(self, center_wavelength, precision='single', use_shock=False, *,
                 pressure_atm=1.0, n2=None, n4=0.0, Ui_eV=15.76, rho_nt=None,
                 tau_rec=1.0e-9, tau_c=None, dispersion=None, adk_prefactor=2.5e15,
                 n0_drude=1.0):
        self.lambda0 = center_wavelength                       # :73
        self.c = 299792458.0                                   # :74
        self.omega0 = 2 * np.pi * self.c / self.lambda0        # :75
        self.use_shock = use_shock                             # :76
        self.e_charge = 1.60217663e-19                         # :79
        self.eps0 = 8.85418781e-12                             # :80
        self.m_e = 9.1093837e-31                               # :81
        self.n0 = 1.0                                          # :85 (Argon keeps the base n0)
        self.pressure = pressure_atm                           # :402
        P = pressure_atm
        self.cauchy_A, self.cauchy_B, self.cauchy_C = 27.9e-5, 12.8e-8, 5.2e-10   # :404-406
        self.n2 = 1.0e-23 * P if n2 is None else n2            # :408
        self.n4 = n4                                           # substitution: :409 -> 0
        self.Ui = Ui_eV * self.e_charge                        # :411
        self.rho_nt = 2.45e25 * P if rho_nt is None else rho_nt   # :412
        self.tau_rec = tau_rec                                 # :414
        self.tau_c = 190e-15 / P if tau_c is None else tau_c   # :415
        self.sigma_drude = (self.e_charge ** 2 * self.tau_c) / \
            (self.c * self.eps0 * n0_drude * self.m_e
             * (1.0 + self.omega0 ** 2 * self.tau_c ** 2))     # :417-419
        if precision == 'double':
            self.float_dtype, self.complex_dtype = np.float64, np.complex128   # :96-101
        else:
            self.float_dtype, self.complex_dtype = np.float32, np.complex64
        self.dispersion = dispersion if dispersion is not None else ('cauchy', self.cauchy_A,
                                                                     self.cauchy_B, self.cauchy_C)
        # LUT on the reference grid (:121-129), values from ADK (substitution)
        log10_I, W = _adk.ionization_lut(self.Ui, n0=self.n0, prefactor=adk_prefactor)
        self.log10_I_cpu = log10_I
        self.log10_I_gpu = log10_I.astype(self.float_dtype)   # :128
        self.W_gpu = W.astype(self.float_dtype)                # :129

    def refractive_index(self, omega_array):
        omega_64 = np.asarray(omega_array).astype(np.float64)
        omega_safe = np.where(np.abs(omega_64) < 1e-12, 1e-12, omega_64)   # :425
        if self.dispersion[0] == 'cauchy':
            _, A, B, Cc = self.dispersion
            wl_um = (2 * np.pi * self.c / np.abs(omega_safe)) * 1e6       # :426
            wl_sq = wl_um ** 2                                              # :427
            K = A + B / wl_sq + Cc / wl_sq ** 2                             # :428
            return 1.0 + K * (self.pressure / 1.0)                          # :429
        _, n0, b2, b3 = self.dispersion                                    # N-new Taylor
        W = omega_64 - self.omega0
        return n0 + self.c * (0.5 * b2 * W ** 2 + (1.0 / 6.0) * b3 * W ** 3) / omega_safe

    def get_shock_operator(self, omega_array):
        """media_physics.py:113-119"""
        if self.use_shock:
            factor = (omega_array + self.omega0) / self.omega0
        else:
            factor = np.ones_like(omega_array)
        return factor[np.newaxis, np.newaxis, :].astype(self.complex_dtype)

    def get_ionization_rate(self, Intensity):
        """media_physics.py:131-137 (clip + linear interpolation in log10 I)."""
        log_I = np.log10(Intensity + 1e-30)
        log_I = np.clip(log_I, float(self.log10_I_gpu[0]), float(self.log10_I_gpu[-1]))
        W_flat = np.interp(log_I.ravel(), self.log10_I_gpu, self.W_gpu)
        return W_flat.reshape(log_I.shape)

    def calc_nonlinear_response(self, A_t, dt):
        """media_physics.py:156-205 with the kernel launch of :176-189."""
        Intensity = np.abs(A_t) ** 2                                   # :165
        I_eff = Intensity                                              # :166 (no Raman in gases)
        W_ion = self.get_ionization_rate(Intensity).astype(np.float32)   # :169
        W_ava = np.zeros_like(Intensity, dtype=self.float_dtype).astype(np.float32)   # :170, :431-432
        Nt = Intensity.shape[-1]
        rho_t, gen_rate_out = plasma_scan(W_ion.reshape(-1, Nt), W_ava.reshape(-1, Nt),
                                          np.float32(1.0 / self.tau_rec), np.float32(dt),
                                          np.float32(self.rho_nt))
        rho_t = rho_t.reshape(Intensity.shape)
        gen_rate_out = gen_rate_out.reshape(Intensity.shape)
        gamma_kerr = 1j * (self.omega0 / self.c) * self.n2                 # :192
        Kerr_term = (gamma_kerr * I_eff * A_t).astype(self.complex_dtype)  # :193
        if self.n4 != 0.0:                                                  # :194-196
            gamma_hoke = 1j * (self.omega0 / self.c) * self.n4
            Kerr_term = Kerr_term + (gamma_hoke * I_eff * I_eff * A_t).astype(self.complex_dtype)
        Plasma_loss = - (gen_rate_out * self.Ui) / (2.0 * Intensity + 1e-30) * A_t   # :200
        Plasma_defocus = - (self.sigma_drude / 2.0) * \
            (1.0 + 1j * self.omega0 * self.tau_c) * rho_t * A_t                # :201-202
        Plasma_term = (Plasma_loss + Plasma_defocus).astype(self.complex_dtype)   # :203
        return Kerr_term, Plasma_term


def argon(center_wavelength, pressure_atm=1.0, precision='single', use_shock=False, **kw):
    """Argon with the constants of media_physics.py:396-432 (n4 -> 0, ADK LUT)."""
    return GasMedium(center_wavelength, precision, use_shock, pressure_atm=pressure_atm, **kw)


def plasma_scan(W_ion, W_ava, rate_rec, dt, rho_nt):
    """Restatement of the CUDA kernel ``media_physics.py:11-67``.

    Vectorised over lines (rows), serial over t.  Inputs float32, all
    arithmetic float64; ``rho[t]`` is the density BEFORE the update (:36).
    """
    W_ion = np.asarray(W_ion, dtype=np.float32)
    W_ava = np.asarray(W_ava, dtype=np.float32)
    nl, Nt = W_ion.shape
    rho = np.zeros((nl, Nt), dtype=np.float64)
    gen = np.zeros((nl, Nt), dtype=np.float64)
    cur = np.zeros(nl, dtype=np.float64)                   # :28
    rho_nt_d = float(np.float32(rho_nt))                   # :29
    rate_rec_d = float(np.float32(rate_rec))               # :30
    dt_d = float(np.float32(dt))                           # :31
    for t in range(Nt):                                    # :33
        rho[:, t] = cur                                    # :36
        w_pi = W_ion[:, t].astype(np.float64)              # :38
        w_av = W_ava[:, t].astype(np.float64)              # :39
        depletion = (rho_nt_d - cur) / rho_nt_d            # :41
        depletion = np.where(depletion < 0.0, 0.0, depletion)   # :42
        gen[:, t] = (w_pi * rho_nt_d + w_av * cur) * depletion  # :44-45
        S_eff = w_pi * rho_nt_d * depletion                # :47
        Gamma_eff = w_av * depletion - rate_rec_d          # :48
        gdt = Gamma_eff * dt_d                             # :50
        gdt = np.clip(gdt, -10.0, 10.0)                    # :51-52
        exp_gdt = np.exp(gdt)                              # :54
        with np.errstate(divide='ignore', invalid='ignore'):
            sf = np.where(np.abs(gdt) < 1e-5, dt_d * (1.0 + 0.5 * gdt),
                          (exp_gdt - 1.0) / Gamma_eff)     # :55-60
        cur = cur * exp_gdt + S_eff * sf                   # :62
        cur = np.minimum(cur, rho_nt_d)                    # :63
        cur = np.maximum(cur, 0.0)                         # :64
    return rho, gen


# ---------------------------------------------------------------------------
# solver (solver_3d.py)
# ---------------------------------------------------------------------------
class Solver3D:
    """Restatement of ``ERK43IP_UPPE_3D_Optimized`` (solver_3d.py:7-233)."""

    def __init__(self, x_grid, y_grid, t_grid, medium, precision='single'):
        self.medium = medium                                              # :9
        self.c, self.lambda0, self.omega0 = medium.c, medium.lambda0, medium.omega0
        if precision == 'double':                                         # :14-19
            self.float_dtype, self.complex_dtype = np.float64, np.complex128
        else:
            self.float_dtype, self.complex_dtype = np.float32, np.complex64
        x_grid, y_grid, t_grid = (np.asarray(a, dtype=np.float64) for a in (x_grid, y_grid, t_grid))
        self.x = x_grid.astype(self.float_dtype)                          # :21-23
        self.y = y_grid.astype(self.float_dtype)
        self.Nx, self.Ny, self.Nt = len(x_grid), len(y_grid), len(t_grid)   # :25
        self.dx = float(x_grid[1] - x_grid[0])                            # :26
        self.dy = float(y_grid[1] - y_grid[0])
        self.dt = float(t_grid[1] - t_grid[0])
        kx = 2 * np.pi * np.fft.fftfreq(self.Nx, self.dx)                 # :28
        ky = 2 * np.pi * np.fft.fftfreq(self.Ny, self.dy)                 # :29
        KY, KX = np.meshgrid(ky, kx, indexing='ij')                       # :30
        self.K2_perp_64 = (KX ** 2 + KY ** 2).astype(np.float64)          # :32
        omega = 2 * np.pi * np.fft.fftfreq(self.Nt, self.dt)              # :34
        self.omega = omega.astype(self.float_dtype)                       # :35
        self.freq_axis_hz = np.fft.fftshift(omega) / (2 * np.pi)          # :36
        self._precompute_dispersion_operator()                            # :41
        self._init_absorber()                                             # :42
        self.shock_operator = medium.get_shock_operator(self.omega)      # :44
        self.A_scale = 1.0                                                # :45
        freq_unshifted = self.omega / (2 * np.pi)                         # :47
        f_max = float(np.max(np.abs(freq_unshifted))) + 1e-10             # :48
        filter_w = np.exp(-(freq_unshifted / (0.85 * f_max)) ** 16).astype(self.float_dtype)  # :49
        self.anti_alias_filter = filter_w[np.newaxis, np.newaxis, :].astype(self.complex_dtype)  # :50
        self.omega_abs = self.omega + self.omega0                         # :53
        self.valid_freq_mask = (self.omega_abs > 0)[np.newaxis, np.newaxis, :].astype(self.float_dtype)  # :54

    def _precompute_dispersion_operator(self):
        """solver_3d.py:56-87"""
        omega_64 = self.omega.astype(np.float64)
        omega0_64, c_64 = float(self.omega0), float(self.c)
        n_omega = self.medium.refractive_index(omega_64 + omega0_64)
        k_val = n_omega * (omega_64 + omega0_64) / c_64
        n_center = float(self.medium.refractive_index(np.array([omega0_64]))[0])
        dw = omega0_64 * 1e-3
        n_plus = float(self.medium.refractive_index(np.array([omega0_64 + dw]))[0])
        k0 = n_center * omega0_64 / c_64
        k_plus = n_plus * (omega0_64 + dw) / c_64
        k1 = (k_plus - k0) / dw
        k_ref = k0 + k1 * omega_64
        k_sq = (k_val ** 2)[np.newaxis, np.newaxis, :]
        k_perp_sq = self.K2_perp_64[:, :, np.newaxis]
        k_ref_3d = k_ref[np.newaxis, np.newaxis, :]
        kz = np.sqrt((k_sq - k_perp_sq).astype(np.complex128))
        numerator = (k_sq - k_ref_3d ** 2) - k_perp_sq
        denominator = kz + k_ref_3d
        D_op_64 = 1j * (numerator / denominator)
        valid_mask = (omega_64 + omega0_64 > 0)[np.newaxis, np.newaxis, :]
        self.D_operator = (D_op_64 * valid_mask).astype(self.complex_dtype)

    def _init_absorber(self):
        """solver_3d.py:89-98"""
        X, Y = np.meshgrid(self.x, self.y, indexing='ij')
        R = np.sqrt(X ** 2 + Y ** 2)
        half_w = float(np.max(np.abs(self.x)))
        r_edge, r_start, p_space = 0.98 * half_w, 0.85 * half_w, 10
        s = (R - r_start) / (r_edge - r_start + 1e-30)
        s = np.clip(s, 0.0, 1.0)
        self.damp_space = (120.0 * (s ** p_space))[:, :, np.newaxis].astype(self.float_dtype)

    # -- one attempt ------------------------------------------------------
    def N_func(self, field_kw):
        """solver_3d.py:107-132"""
        A_t_local = sfft.ifftn(field_kw, axes=(0, 1, 2))
        A_physical = A_t_local * self.A_scale
        Kerr_phys, Plasma_phys = self.medium.calc_nonlinear_response(A_physical, self.dt)
        Kerr_t = Kerr_phys / self.A_scale
        Plasma_t = Plasma_phys / self.A_scale
        Kerr_w = sfft.fft(Kerr_t, axis=-1)
        Plasma_w = sfft.fft(Plasma_t, axis=-1)
        N_w_total = self.shock_operator * Kerr_w + Plasma_w
        N_w_total *= self.valid_freq_mask
        return sfft.fft2(N_w_total, axes=(0, 1))

    def erk43_step(self, A_t, h, tol=None):
        """solver_3d.py:100-160; returns (A4_t, err, err_num, err_den)."""
        A_w = sfft.fft(A_t, axis=-1)
        A_k_w = sfft.fft2(A_w, axes=(0, 1))
        E = np.exp((h / 2) * self.D_operator)

        def L_step(f):
            return f * E

        v_ip = L_step(A_k_w)
        k1 = self.N_func(A_k_w)
        alpha1_term = L_step(k1)
        alpha2 = self.N_func(v_ip + (h / 2) * alpha1_term)
        alpha3 = self.N_func(v_ip + (h / 2) * alpha2)
        temp_field = L_step(v_ip + h * alpha3)
        alpha4_prime = self.N_func(temp_field)
        term_sum = alpha1_term + 2 * alpha2 + 2 * alpha3
        beta = L_step(v_ip + (h / 6) * term_sum)
        A4_kw = beta + (h / 6) * alpha4_prime
        alpha5_prime = self.N_func(A4_kw)
        A3_kw = beta + (h / 30) * (2 * alpha4_prime + 3 * alpha5_prime)
        max_diff = np.max(np.abs(A4_kw - A3_kw))
        max_norm = np.max(np.abs(A4_kw))
        err = float(max_diff / (max_norm + 1e-20))
        A4_w = sfft.ifft2(A4_kw, axes=(0, 1))
        A4_w = A4_w * self.anti_alias_filter
        A4_t = sfft.ifft(A4_w, axis=-1)
        A4_t *= np.exp(-self.damp_space * h)
        return A4_t, err, float(max_diff), float(max_norm)

    # -- adaptive loop ----------------------------------------------------
    def propagate(self, A0, L, tol=1e-4, max_step=1e-2, min_step=1e-9, schedule=None,
                  max_attempts=None):
        """solver_3d.py:162-233.

        ``schedule`` (replay mode): a list of (h, accepted) pairs used instead of
        the controller, so a device run can be compared attempt by attempt.
        Returns (z, freq_axis_hz, A_w_final, log) with ``log`` the list of
        (z_before, h, err, accepted) per attempt.
        """
        A0 = np.asarray(A0).astype(self.complex_dtype)
        self.A_scale = float(np.max(np.abs(A0)))                           # :166
        if self.A_scale < 1e-30:
            self.A_scale = 1.0
        A = (A0 / self.complex_dtype(self.A_scale * 1.0 + 0.0j)).astype(self.complex_dtype)   # :170
        z = 0.0
        h = min(max_step, L / 1000.0)                                      # :173
        fail_count = 0
        log = []
        if schedule is not None:
            for h_s, acc in schedule:
                A_new, err, _, _ = self.erk43_step(A, h_s, tol)
                log.append((z, h_s, err, bool(acc)))
                if acc:
                    z += h_s
                    A = A_new
            return self._finish(A, z, log)
        n = 0
        while z < L:                                                       # :182
            dist_remaining = L - z
            if h > dist_remaining:
                h = dist_remaining
                if h < 1e-15:
                    break
            A_new, err, _, _ = self.erk43_step(A, h, tol)                 # :188
            n += 1
            if err < tol or h <= min_step * 1.01:                          # :190
                log.append((z, h, err, True))
                fail_count = fail_count + 1 if (h <= min_step * 1.01 and err > tol) else 0
                z += h
                A = A_new
                err = max(err, 1e-30)
                factor = 0.95 * (tol / err) ** 0.2
                if fail_count > 0:
                    factor = min(factor, 1.2)
                h = min(h * min(factor, 2.0), max_step)
            else:
                log.append((z, h, err, False))
                err = max(err, 1e-30)
                factor = 0.95 * (tol / err) ** 0.2
                h = max(h * factor, min_step)
            if max_attempts is not None and n >= max_attempts:
                break
        return self._finish(A, z, log)

    def ionization_fraction(self, A_t):
        """max rho/rho_nt of a normalised time-domain state (media_physics.py:165-189)."""
        m = self.medium
        A_phys = A_t * self.A_scale
        I = np.abs(A_phys) ** 2
        W_ion = m.get_ionization_rate(I).astype(np.float32)
        Nt = I.shape[-1]
        rho, _ = plasma_scan(W_ion.reshape(-1, Nt), np.zeros((W_ion.size // Nt, Nt), np.float32),
                             np.float32(1.0 / m.tau_rec), np.float32(self.dt), np.float32(m.rho_nt))
        return float(rho.max()) / float(np.float32(m.rho_nt))

    def diagnostics(self, A_t):
        """energy sum |A|^2 dx dy dt, photon number sum E_w/(hbar w_abs), w_abs > 0."""
        A = A_t * self.A_scale
        E = float(np.sum(np.abs(A) ** 2)) * self.dx * self.dy * self.dt
        Ew = np.sum(np.abs(sfft.fft(A, axis=-1)) ** 2, axis=(0, 1)) * self.dx * self.dy * self.dt / self.Nt
        wa = np.fft.fftfreq(self.Nt, self.dt) * 2 * np.pi + self.omega0
        ph = float(np.sum(Ew[wa > 0] / (1.054571817e-34 * wa[wa > 0])))
        return E, ph

    def _finish(self, A, z, log):
        """solver_3d.py:215-233"""
        self.last_state = A.copy()
        A = A * self.A_scale
        A_w_raw = sfft.fft(A, axis=-1)
        A_w_final = np.fft.fftshift(A_w_raw, axes=-1)
        return z, self.freq_axis_hz, A_w_final, log
