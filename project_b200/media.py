"""Medium plugins for the 3+1D envelope propagator (host side).

Mirrors the OpticalMedium protocol of
``src/3+1D-UPPE-ERK4(3)IP-envelope/media_physics.py:70-205``: a medium supplies
``c, lambda0, omega0``, ``refractive_index(omega_abs)`` (FP64), the shock
operator (``:113-119``), the Kerr/HOKE coefficients, the ionisation LUT on a
uniform log10(I) grid (``:121-137``) and the plasma constants.  The nonlinear
response itself (``calc_nonlinear_response``, ``:156-205``) and the density scan
(``:11-67``) run in the fused CUDA t-line kernel; a medium only provides data.

Differences from the reference, all deliberate:
  * the default ionisation table is the ADK rate of
    ``src/THz/2+1D-all field UPPE Argon.py:53-81`` on the reference's grid, since
    the reference's Keldysh tunnel term (``media_physics.py:139-146``) is broken
    (its ``+1e-20`` dominates the denominator, giving W >= 1e15 1/s everywhere);
    any (log10 I, W) table can be passed instead;
  * ``n4`` defaults to 0: the reference's gas n4 values overflow the first step.
"""
import numpy as np

C0 = 299792458.0
E_CHARGE = 1.60217663e-19
EPS0 = 8.85418781e-12
M_E = 9.1093837e-31
HBAR = 1.054571817e-34


def adk_rate(E_abs, Ui_J, Z=1, prefactor=2.5e15, threshold=5e7):
    """ADK rate W(E) [1/s] (``2+1D-all field UPPE Argon.py:53-81``)."""
    Uh = 13.6 * 1.60217663e-19
    n_eff = Z * np.sqrt(Uh / Ui_J)
    E_atomic = 5.142e11
    alpha = 4.0 * n_eff ** 2 * E_atomic * (Ui_J / Uh) ** 1.5 / 3.0
    beta = 2.0 * n_eff - 1.0
    E_abs = np.asarray(E_abs, dtype=np.float64)
    E_safe = np.maximum(E_abs, 1e-3)
    W = prefactor * (1.0 / E_safe) ** beta * np.exp(-alpha / E_safe)
    return W * (E_abs > threshold)


class OpticalMedium:
    """Base medium (``media_physics.py:70-119``)."""

    def __init__(self, center_wavelength, precision='single', use_shock=False):
        self.lambda0 = center_wavelength
        self.c = C0
        self.omega0 = 2 * np.pi * self.c / self.lambda0
        self.use_shock = use_shock
        self.precision = precision
        self.e_charge, self.eps0, self.m_e, self.hbar = E_CHARGE, EPS0, M_E, HBAR
        self.n0 = 1.0
        self.n2 = 0.0
        self.n4 = 0.0
        self.Ui = 0.0
        self.rho_nt = 0.0
        self.tau_c = 0.0
        self.tau_rec = 1e-9
        self.sigma_drude = 0.0
        self.avalanche_coef = 0.0    # W_ava = avalanche_coef * I
        self.plasma = True
        self.lut_log10I = None
        self.lut_W = None

    def refractive_index(self, omega_array):
        raise NotImplementedError

    def get_shock_operator(self, omega_array):
        """(omega + omega0)/omega0 with self-steepening, else 1 (FP64, [Nt])."""
        omega_array = np.asarray(omega_array, dtype=np.float64)
        if self.use_shock:
            return (omega_array + self.omega0) / self.omega0
        return np.ones_like(omega_array)

    def _lut_grid(self, I_min_W_cm2=1e8, I_max_W_cm2=1e16, points=2000):
        """The reference's LUT grid (``media_physics.py:121-126``)."""
        return np.linspace(np.log10(I_min_W_cm2 * 1e4), np.log10(I_max_W_cm2 * 1e4), points)

    def init_adk_lut(self, prefactor=2.5e15):
        log10_I = self._lut_grid()
        E = np.sqrt(2 * 10 ** log10_I / (self.c * self.eps0 * self.n0))
        self.set_ionization_lut(log10_I, adk_rate(E, self.Ui, prefactor=prefactor))

    def set_ionization_lut(self, log10_I, W):
        log10_I = np.asarray(log10_I, dtype=np.float64)
        d = np.diff(log10_I)
        if len(log10_I) < 2 or not np.all(d > 0) or np.ptp(d) > 1e-9 * abs(d.mean()):
            raise ValueError('the ionisation LUT needs a uniform, increasing log10(I) grid')
        self.lut_log10I = log10_I
        self.lut_W = np.asarray(W, dtype=np.float64)

    def sigma_from_tau_c(self, n0=1.0):
        return (self.e_charge ** 2 * self.tau_c) / (
            self.c * self.eps0 * n0 * self.m_e * (1.0 + self.omega0 ** 2 * self.tau_c ** 2))


class Argon(OpticalMedium):
    """Argon (``media_physics.py:396-432``).

    ``dispersion``: ``None`` for the reference's Cauchy n(lambda) (``:423-429``), or
    ``('taylor', n0, beta2, beta3)`` for n(w) = n0 + c (b2 W^2/2 + b3 W^3/6)/w with
    W = w - w0, which makes k(w) a Taylor polynomial around w0.
    """

    def __init__(self, center_wavelength, pressure_atm=1.0, precision='single', use_shock=False,
                 dispersion=None, n4=0.0, lut=None, adk_prefactor=2.5e15):
        super().__init__(center_wavelength, precision, use_shock)
        P = pressure_atm
        self.pressure = P
        self.cauchy_A, self.cauchy_B, self.cauchy_C = 27.9e-5, 12.8e-8, 5.2e-10
        self.n2 = 1.0e-23 * P
        self.n4 = n4
        self.Ui = 15.76 * self.e_charge
        self.rho_nt = 2.45e25 * P
        self.tau_rec = 1.0e-9
        self.tau_c = 190e-15 / P
        self.sigma_drude = self.sigma_from_tau_c(1.0)
        self.dispersion = dispersion
        if lut is None:
            self.init_adk_lut(adk_prefactor)
        else:
            self.set_ionization_lut(*lut)

    def refractive_index(self, omega_array):
        om = np.asarray(omega_array, dtype=np.float64)
        omega_safe = np.where(np.abs(om) < 1e-12, 1e-12, om)
        if self.dispersion is None:
            wl_um = (2 * np.pi * self.c / np.abs(omega_safe)) * 1e6
            wl_sq = wl_um ** 2
            K = self.cauchy_A + self.cauchy_B / wl_sq + self.cauchy_C / wl_sq ** 2
            return 1.0 + K * (self.pressure / 1.0)
        kind, n0, b2, b3 = self.dispersion
        if kind != 'taylor':
            raise ValueError(f'unknown dispersion model {kind!r}')
        W = om - self.omega0
        return n0 + self.c * (0.5 * b2 * W ** 2 + (1.0 / 6.0) * b3 * W ** 3) / omega_safe
