"""Seeded synthetic inputs (oracle side, test infrastructure only).

None of these exist in the reference (N-new).  The formulas are defined here and
restated independently by ``project_b200.pulses``; tests check the two agree.

* ``gaussian_pulse``  -- erk43ip_method.py:375-381.
* ``dispersed_pulse`` -- erk43ip_method.py:383-446 (GDD/TOD spectral phase).
* ``photon_noise``    -- one photon per mode: a complex Gaussian per FFT bin with
  <|A_j|^2> = hbar*w_j*Nt/dt for absolute frequency w_j > 0 (zero otherwise), so
  that E = sum |A|^2 dt carries hbar*w_j per mode; added in the time domain.
* ``speckle``         -- amplitude factor (1 + amp*xi(x, y)) with xi a unit-variance
  Gaussian random field: white N(0,1) noise low-passed by exp(-(k_perp*l)^2/4),
  then normalised to zero mean and unit standard deviation.
"""
import numpy as np
from scipy.fft import fft, ifft, fftfreq, fftshift, ifftshift, fft2, ifft2

HBAR = 1.054571817e-34
C0 = 299792458.0


def gaussian_pulse(t, pulse_energy, pulse_fwhm, chirp=0.0):
    factor = np.sqrt(np.pi / (4 * np.log(2)))
    P0 = pulse_energy / (pulse_fwhm * factor)
    T0 = pulse_fwhm / (2 * np.sqrt(np.log(2)))
    return np.sqrt(P0) * np.exp(-(1 + 1j * chirp) * (t / T0) ** 2 / 2)


def dispersed_pulse(t, pulse_energy, pulse_fwhm, GDD=0.0, TOD=0.0):
    factor = np.sqrt(np.pi / (4 * np.log(2)))
    P0 = pulse_energy / (pulse_fwhm * factor)
    T0 = pulse_fwhm / (2 * np.sqrt(np.log(2)))
    A_tl = np.sqrt(P0) * np.exp(-(t / T0) ** 2 / 2)
    if GDD == 0 and TOD == 0:
        return A_tl.astype(complex)
    N = len(t)
    dt = t[1] - t[0]
    omega = 2 * np.pi * fftfreq(N, dt)
    A_freq = fft(ifftshift(A_tl))
    phase = 0.5 * GDD * omega ** 2 + (1.0 / 6.0) * TOD * omega ** 3
    return fftshift(ifft(A_freq * np.exp(1j * phase)))


def photon_noise(t, center_wavelength, seed):
    N = len(t)
    dt = t[1] - t[0]
    omega = 2 * np.pi * fftfreq(N, dt)
    w_abs = 2 * np.pi * C0 / center_wavelength + omega
    var = np.where(w_abs > 0, HBAR * w_abs * N / dt, 0.0)
    rng = np.random.Generator(np.random.PCG64(seed))
    xi = (rng.standard_normal(N) + 1j * rng.standard_normal(N)) / np.sqrt(2.0)
    return ifft(np.sqrt(var) * xi)


def speckle(x, y, corr_len, amp, seed):
    Nx, Ny = len(x), len(y)
    dx, dy = x[1] - x[0], y[1] - y[0]
    kx = 2 * np.pi * fftfreq(Nx, dx)
    ky = 2 * np.pi * fftfreq(Ny, dy)
    K2 = kx[:, None] ** 2 + ky[None, :] ** 2
    rng = np.random.Generator(np.random.PCG64(seed))
    w = rng.standard_normal((Nx, Ny))
    xi = np.real(ifft2(fft2(w) * np.exp(-K2 * corr_len ** 2 / 4)))
    xi = (xi - xi.mean()) / xi.std()
    return 1.0 + amp * xi


def gaussian_beam_3d(x, y, t, w0, pulse_energy, pulse_fwhm):
    """Collimated Gaussian beam exp(-r^2/w0^2) x Gaussian pulse, |A|^2 in W/m^2,
    normalised so that sum |A|^2 dx dy dt = pulse_energy."""
    X, Y = np.meshgrid(x, y, indexing='ij')
    T0 = pulse_fwhm / (2 * np.sqrt(np.log(2)))
    A = np.exp(-(X ** 2 + Y ** 2) / w0 ** 2)[:, :, None] * np.exp(-(t / T0) ** 2 / 2)[None, None, :]
    dx, dy, dt = x[1] - x[0], y[1] - y[0], t[1] - t[0]
    E = np.sum(np.abs(A) ** 2) * dx * dy * dt
    return (A * np.sqrt(pulse_energy / E)).astype(np.complex128)


def pulse_from_spectrum(t, wavelengths_nm, intensities, pulse_energy, GDD=0.0, TOD=0.0,
                        use_jacobian=True, interp_kind='cubic', center_wavelength=800e-9):
    """Restatement of ``generate_pulse_from_spectrum`` (erk43ip_method.py:599-764),
    FFT path: sort by wavelength, normalise, to frequency with the Jacobian
    lambda^2/c (renormalised), drop duplicate frequencies, interpolate onto the
    simulation grid (zero outside), sqrt, GDD/TOD phase, ifft, fftshift, energy
    normalisation by the trapezoidal rule."""
    from scipy.interpolate import interp1d
    c = 299792458.0
    t = np.asarray(t, dtype=np.float64)
    idx = np.argsort(wavelengths_nm)                                       # :676
    wl = np.asarray(wavelengths_nm, dtype=np.float64)[idx]
    I = np.asarray(intensities, dtype=np.float64)[idx]
    if np.max(I) > 0:                                                       # :681
        I = I / np.max(I)
    f = c / (wl * 1e-9)                                                     # :685
    if use_jacobian:                                                        # :687-693
        I = I * (wl * 1e-9) ** 2 / c
        if np.max(I) > 0:
            I = I / np.max(I)
    uf, ui = np.unique(f, return_index=True)                                # :698-701
    if len(uf) < len(f):
        f, I = uf, I[ui]
    if f[0] < f[-1]:                                                        # :704-706
        f, I = f[::-1], I[::-1]
    kind = 'linear' if interp_kind in ('cubic', 'quadratic') and len(f) < 4 else interp_kind
    g = interp1d(f, I, kind=kind, bounds_error=False, fill_value=0.0)      # :715
    N, dt = len(t), t[1] - t[0]
    w = 2 * np.pi * fftfreq(N, dt)                                          # :719
    S = g(w / (2 * np.pi) + c / center_wavelength)
    S[S < 0] = 0
    S[np.isnan(S)] = 0
    A = fftshift(ifft(np.sqrt(S) * np.exp(1j * (0.5 * GDD * w ** 2 + (1.0 / 6.0) * TOD * w ** 3))))
    E = np.trapz(np.abs(A) ** 2, t)                                         # :739
    if E > 0:
        A = A * np.sqrt(pulse_energy / E)
    return A
