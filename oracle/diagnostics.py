"""Restatement of the driver diagnostics of ``src/3+1D-ERK4(3)IP UPPE/sim.py``
(``_calc_energy`` :140-143, ``_calc_beam_moments`` :145-157,
``_fwhm_from_intensity`` :159-182, ``save_snapshot`` :190-241) on a physical
time-domain field A[x, y, t], for the parity tests.  Test infrastructure only.
"""
import numpy as np


def _fwhm(t, I):
    """sim.py:159-182"""
    I, t = np.asarray(I).astype(np.float64), np.asarray(t).astype(np.float64)
    if I.size < 4:
        return np.nan
    imax = np.max(I)
    if not np.isfinite(imax) or imax <= 0:
        return np.nan
    half = 0.5 * imax
    i_peak = int(np.argmax(I))
    il = i_peak
    while il > 0 and I[il] >= half:
        il -= 1
    ir = i_peak
    while ir < I.size - 1 and I[ir] >= half:
        ir += 1
    if ir <= il + 1:
        return np.nan

    def interp(i1, i2):
        y1, y2 = I[i1], I[i2]
        return t[i1] + (half - y1) * (t[i2] - t[i1]) / (y2 - y1 + 1e-30)

    t_left = interp(il, il + 1) if il + 1 < I.size else t[il]
    t_right = interp(ir - 1, ir) if ir - 1 >= 0 else t[ir]
    w = t_right - t_left
    return float(w) if (w > 0 and np.isfinite(w)) else np.nan


def beam_diagnostics(A, x, y, t, w_mode, lam):
    """sim.py:190-241 with field_clean * A_scale = A (physical units)."""
    x, y, t = (np.asarray(v, dtype=np.float64) for v in (x, y, t))
    dx, dy, dt = x[1] - x[0], y[1] - y[0], t[1] - t[0]
    I = np.abs(A).astype(np.float64) ** 2
    E_total = float(np.sum(I) * dx * dy * dt)                                  # :140-143
    P_t = np.sum(I, axis=(0, 1)) * dx * dy                                     # :203
    fluence = np.sum(I, axis=-1) * dt                                          # :206
    X, Y = np.meshgrid(x, y, indexing='ij')                                    # :145-157
    total = np.sum(fluence) * dx * dy + 1e-30
    xm = np.sum(X * fluence) * dx * dy / total
    ym = np.sum(Y * fluence) * dx * dy / total
    x2 = np.sum((X - xm) ** 2 * fluence) * dx * dy / total
    y2 = np.sum((Y - ym) ** 2 * fluence) * dx * dy / total
    field_w = np.fft.fftshift(np.fft.fft(A, axis=-1), axes=-1)                 # :218
    mode = np.exp(-(X ** 2 + Y ** 2) / w_mode ** 2)[:, :, None]                # :220
    coupled_w = np.sum(field_w * mode, axis=(0, 1))                            # :222
    ix0, iy0 = len(x) // 2, len(y) // 2
    coupled_t = np.sum(A * mode, axis=(0, 1))                                  # :237
    I_center_t = np.abs(A[ix0, iy0, :]) ** 2                                   # :236
    I_smf_t = np.abs(coupled_t) ** 2
    omega = 2 * np.pi * np.fft.fftfreq(len(t), dt)
    freq_abs = np.fft.fftshift(omega) / (2 * np.pi) + 299792458.0 / lam        # :227-229
    return {'energy_total': E_total, 'x_mean_m': xm, 'y_mean_m': ym, 'wx_rms_m': np.sqrt(x2),
            'wy_rms_m': np.sqrt(y2), 'P_t': P_t, 'it_peak': int(np.argmax(P_t)), 'fluence': fluence,
            'spec_smf': np.abs(coupled_w) ** 2, 'spec_full_incoh': np.sum(np.abs(field_w) ** 2, axis=(0, 1)),
            'spec_center': np.abs(field_w[ix0, iy0, :]) ** 2, 'I_center_t': I_center_t,
            'I_smf_t': I_smf_t, 'fwhm_center_s': _fwhm(t, I_center_t), 'fwhm_smf_s': _fwhm(t, I_smf_t),
            'freq_abs_Hz': freq_abs}
