"""Pulse analysis helpers of the 1D solver's drivers, on a (host) field.

``fwhm_precise`` follows ``ERK43IP_UPPE._calculate_fwhm_precise``
(``src/1D-ERK4(3)IP UPPE gas/erk43ip_method.py:448-490``) and
``analyze_spectral_phase`` follows ``ERK43IP_UPPE.analyze_spectral_phase``
(``:766-808``).  Both work on O(Nt) arrays after a propagation (the field-sized
sums of the 3D drivers run on the device: ``ERK43IP_UPPE_3D_Optimized.beam_diagnostics``).
"""
import numpy as np

C0 = 299792458.0


def fwhm_precise(x, y):
    """(x_left, x_right, width) of the half-maximum crossings of y(x), linearly
    interpolated at the first rising and last falling crossing; with fewer than
    two crossings, the outermost samples at or above half maximum; (None, None,
    None) when fewer than two samples reach it."""
    x = np.asarray(x)
    y = np.asarray(y)
    half = np.max(y) / 2
    up = (y >= half).astype(int)
    cross = np.nonzero(np.diff(up))[0]
    if len(cross) < 2:
        idx = np.nonzero(y >= half)[0]
        if len(idx) < 2:
            return None, None, None
        return x[idx[0]], x[idx[-1]], x[idx[-1]] - x[idx[0]]

    def at(i):
        return x[i] + (half - y[i]) * (x[i + 1] - x[i]) / (y[i + 1] - y[i])

    left, right = at(cross[0]), at(cross[-1])
    return left, right, right - left


def analyze_spectral_phase(A, t, omega0, fit_order=4, plot_threshold=0.01):
    """Spectral intensity and the residual spectral phase after a polynomial fit of
    order ``fit_order`` over the band where the normalised intensity exceeds
    ``plot_threshold``; the residual is zeroed at the spectral peak.  Returns a
    dict sorted by wavelength, or None when fewer than 5 samples are in band or
    the fit fails."""
    A = np.asarray(A)
    t = np.asarray(t, dtype=np.float64)
    N, dt = len(t), t[1] - t[0]
    w = np.fft.fftshift(2 * np.pi * np.fft.fftfreq(N, dt))
    S = np.fft.fftshift(np.fft.fft(A))
    I = np.abs(S) ** 2
    top = np.max(I)
    In = I / top if top > 0 else I
    phi = np.unwrap(np.angle(S))
    band = In > plot_threshold
    if np.sum(band) < 5:
        return None
    try:
        coef = np.polyfit(w[band], phi[band], fit_order)
    except Exception:
        return None
    res = phi - np.polyval(coef, w)
    res = res - res[np.argmax(In)]
    wa = w + omega0
    wa[wa < 1e-10] = 1e-10
    wl = 2 * np.pi * C0 / wa * 1e9
    order = np.argsort(wl)
    return {'wavelength_nm': wl[order], 'spectral_intensity': In[order], 'residual_phase': res[order],
            'mask': band[order]}
