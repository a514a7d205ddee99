"""ADK ionisation rate and the ionisation look-up table (oracle, test infrastructure).

The reference's envelope medium builds a 2000-point LUT over log10(I)
(``media_physics.py:121-129``) from a Keldysh formula whose tunnel exponent is
broken (the ``+1e-20`` in the denominator of ``media_physics.py:143-144``
dominates, so W >= 1e15 s^-1 at every intensity).  The LUT values are therefore
replaced by the ADK rate that the reference uses for argon in
``src/THz/2+1D-all field UPPE Argon.py:53-81`` (N-new substitution, parity
unpinned), evaluated on the same log10(I) grid.  The field amplitude of an
envelope of intensity I is E = sqrt(2 I / (c eps0 n0)) (the same relation the
reference uses at ``media_physics.py:142``).
"""
import numpy as np

E_CHARGE = 1.60217663e-19      # media_physics.py:79
EPS0 = 8.85418781e-12          # media_physics.py:80
M_E = 9.1093837e-31            # media_physics.py:81
HBAR = 1.054571817e-34         # media_physics.py:82
C0 = 299792458.0               # media_physics.py:74


def adk_constants(Ui_J, Z=1, prefactor=2.5e15):
    """(alpha, beta, prefactor) of the ADK rate, ``2+1D-all field UPPE Argon.py:53-68``."""
    e = 1.60217663e-19                      # THz file :39
    Uh = 13.6 * e                           # :54
    n_eff = Z * np.sqrt(Uh / Ui_J)          # :55
    E_atomic = 5.142e11                     # :57
    alpha = 4.0 * n_eff ** 2 * E_atomic * (Ui_J / Uh) ** 1.5 / 3.0   # :60
    beta = 2.0 * n_eff - 1.0                # :61
    return alpha, beta, prefactor


def adk_rate(E_abs, Ui_J, prefactor=2.5e15, threshold=5e7):
    """W(E) = pre * E^-beta * exp(-alpha/E) * (E > 5e7), ``:70-81``."""
    alpha, beta, pre = adk_constants(Ui_J, prefactor=prefactor)
    E_abs = np.asarray(E_abs, dtype=np.float64)
    E_safe = np.maximum(E_abs, 1e-3)                       # :74
    W = pre * (1.0 / E_safe) ** beta * np.exp(-alpha / E_safe)   # :77
    W = W * (E_abs > threshold)                            # :80
    return W


def ionization_lut(Ui_J, n0=1.0, I_min_W_cm2=1e8, I_max_W_cm2=1e16, points=2000,
                   prefactor=2.5e15):
    """FP64 (log10 I, W) table on the reference's grid, ``media_physics.py:121-129``.

    Returns the float64 grid and rates; the reference then casts both to the
    solver's float dtype (``:128-129``), which the caller does.
    """
    I_min = I_min_W_cm2 * 1e4                                  # :123
    I_max = I_max_W_cm2 * 1e4                                  # :124
    log10_I = np.linspace(np.log10(I_min), np.log10(I_max), points)   # :125
    I_grid = 10 ** log10_I                                     # :126
    E = np.sqrt(2 * I_grid / (C0 * EPS0 * n0))                 # :142
    W = adk_rate(E, Ui_J, prefactor=prefactor)
    return log10_I, W
