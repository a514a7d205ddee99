"""Seeded synthetic inputs (host side, numpy).

Pulse builders follow the reference: ``generate_gaussian_pulse`` and
``generate_dispersed_pulse`` of ``src/1D-ERK4(3)IP UPPE gas/erk43ip_method.py:375-446``.
The noise and speckle models have no counterpart in the reference; their
definitions are:

* ``photon_noise``: one photon per mode.  For FFT bin j with absolute frequency
  w_j > 0, a complex Gaussian of variance hbar*w_j*Nt/dt is added to fft(A), so
  that with E = sum |A|^2 dt each mode carries hbar*w_j on average.
* ``speckle``: amplitude factor 1 + amp*xi(x, y), xi a zero-mean, unit-variance
  Gaussian random field obtained by filtering white N(0,1) noise with
  exp(-(k_perp*l)^2/4) (correlation length l).
All random draws use numpy's PCG64 generator with the given seed.
"""
import numpy as np

HBAR = 1.054571817e-34
C0 = 299792458.0


def gaussian_pulse(t, pulse_energy, pulse_fwhm, chirp=0.0):
    """erk43ip_method.py:375-381: sqrt(P0) exp(-(1 + i C)(t/T0)^2 / 2)."""
    t = np.asarray(t, dtype=np.float64)
    P0 = pulse_energy / (pulse_fwhm * np.sqrt(np.pi / (4 * np.log(2))))
    T0 = pulse_fwhm / (2 * np.sqrt(np.log(2)))
    return np.sqrt(P0) * np.exp(-(1 + 1j * chirp) * (t / T0) ** 2 / 2)


def dispersed_pulse(t, pulse_energy, pulse_fwhm, GDD=0.0, TOD=0.0):
    """erk43ip_method.py:383-446: transform-limited Gaussian with a spectral
    phase GDD w^2/2 + TOD w^3/6 applied about the window centre."""
    t = np.asarray(t, dtype=np.float64)
    P0 = pulse_energy / (pulse_fwhm * np.sqrt(np.pi / (4 * np.log(2))))
    T0 = pulse_fwhm / (2 * np.sqrt(np.log(2)))
    A = np.sqrt(P0) * np.exp(-(t / T0) ** 2 / 2)
    if GDD == 0 and TOD == 0:
        return A.astype(np.complex128)
    n = len(t)
    w = 2 * np.pi * np.fft.fftfreq(n, t[1] - t[0])
    spec = np.fft.fft(np.fft.ifftshift(A))
    spec = spec * np.exp(1j * (0.5 * GDD * w ** 2 + (1.0 / 6.0) * TOD * w ** 3))
    return np.fft.fftshift(np.fft.ifft(spec))


def photon_noise(t, center_wavelength, seed):
    t = np.asarray(t, dtype=np.float64)
    n = len(t)
    dt = t[1] - t[0]
    w_abs = 2 * np.pi * C0 / center_wavelength + 2 * np.pi * np.fft.fftfreq(n, dt)
    sigma = np.sqrt(np.where(w_abs > 0, HBAR * w_abs * n / dt, 0.0))
    rng = np.random.Generator(np.random.PCG64(seed))
    xi = (rng.standard_normal(n) + 1j * rng.standard_normal(n)) / np.sqrt(2.0)
    return np.fft.ifft(sigma * xi)


def speckle(x, y, corr_len, amp, seed):
    x = np.asarray(x, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    kx = 2 * np.pi * np.fft.fftfreq(len(x), x[1] - x[0])
    ky = 2 * np.pi * np.fft.fftfreq(len(y), y[1] - y[0])
    rng = np.random.Generator(np.random.PCG64(seed))
    white = rng.standard_normal((len(x), len(y)))
    filt = np.exp(-(kx[:, None] ** 2 + ky[None, :] ** 2) * corr_len ** 2 / 4)
    xi = np.real(np.fft.ifft2(np.fft.fft2(white) * filt))
    xi = (xi - xi.mean()) / xi.std()
    return 1.0 + amp * xi


def gaussian_beam(x, y, t, w0, pulse_energy, pulse_fwhm, dtype=np.complex128):
    """Collimated beam exp(-r^2/w0^2) x Gaussian pulse, |A|^2 in W/m^2, scaled so
    that sum |A|^2 dx dy dt equals the pulse energy."""
    x = np.asarray(x, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    t = np.asarray(t, dtype=np.float64)
    T0 = pulse_fwhm / (2 * np.sqrt(np.log(2)))
    sp = np.exp(-(x[:, None] ** 2 + y[None, :] ** 2) / w0 ** 2)
    tp = np.exp(-(t / T0) ** 2 / 2)
    E = np.sum(sp ** 2) * np.sum(tp ** 2) * (x[1] - x[0]) * (y[1] - y[0]) * (t[1] - t[0])
    s = np.sqrt(pulse_energy / E)
    return ((s * sp)[:, :, None] * tp[None, None, :]).astype(dtype)


def noll_nm(j):
    """(n, m) of Zernike polynomial number j in Noll's ordering (j >= 1)."""
    n, j1 = 0, j - 1
    while j1 > n:
        n += 1
        j1 -= n
    m = (-1) ** j * ((n % 2) + 2 * int((j1 + ((n + 1) % 2)) / 2))
    return n, m


def zernike(j, rho, theta):
    """Orthonormal Zernike polynomial Z_j (Noll) on the unit disk; rho is clipped to 1
    outside the aperture so the phase screen stays bounded there."""
    from math import factorial
    n, m = noll_nm(j)
    am = abs(m)
    r = np.minimum(np.asarray(rho, dtype=np.float64), 1.0)
    R = np.zeros_like(r)
    for k in range((n - am) // 2 + 1):
        R += ((-1) ** k * factorial(n - k)
              / (factorial(k) * factorial((n + am) // 2 - k) * factorial((n - am) // 2 - k))) * r ** (n - 2 * k)
    if m == 0:
        return np.sqrt(n + 1.0) * R
    ang = np.cos(m * theta) if m > 0 else np.sin(am * theta)
    return np.sqrt(2.0 * (n + 1.0)) * R * ang


def zernike_basis(x, y, aperture_radius, jmax=15):
    """[jmax, Nx, Ny] array of Z_1..Z_jmax over the (x, y) grid."""
    X, Y = np.meshgrid(np.asarray(x, dtype=np.float64), np.asarray(y, dtype=np.float64), indexing='ij')
    rho = np.sqrt(X ** 2 + Y ** 2) / aperture_radius
    th = np.arctan2(Y, X)
    return np.stack([zernike(j, rho, th) for j in range(1, jmax + 1)])


def spectrum_spline(wavelengths_nm, intensities, use_jacobian=True, interp_kind='cubic'):
    """Host part of generate_pulse_from_spectrum (erk43ip_method.py:674-716): sort,
    normalise, to frequency with the Jacobian lambda^2/c (renormalised), drop
    duplicate frequencies, and the interpolant of interp1d(kind) as a piecewise
    cubic: (breaks ascending [nb], coef [nb-1, 4] highest power first)."""
    from scipy.interpolate import PPoly, make_interp_spline
    idx = np.argsort(wavelengths_nm)
    wl = np.asarray(wavelengths_nm, dtype=np.float64)[idx]
    I = np.asarray(intensities, dtype=np.float64)[idx]
    if np.max(I) > 0:
        I = I / np.max(I)
    f = C0 / (wl * 1e-9)
    if use_jacobian:
        I = I * (wl * 1e-9) ** 2 / C0
        if np.max(I) > 0:
            I = I / np.max(I)
    uf, ui = np.unique(f, return_index=True)
    if len(uf) < len(f):
        f, I = uf, I[ui]
    order = np.argsort(f)                      # interp1d sorts its abscissae
    f, I = f[order], I[order]
    k = {'linear': 1, 'quadratic': 2, 'cubic': 3}[interp_kind]
    if k > 1 and len(f) < 4:
        k = 1
    pp = PPoly.from_spline(make_interp_spline(f, I, k=k))
    br, c = pp.x, pp.c                         # c[m, j]: power (k - m) on interval j
    keep = np.diff(br) > 0                     # drop the zero-length end intervals
    coef = np.zeros((int(keep.sum()), 4))
    coef[:, 4 - c.shape[0]:] = c[:, keep].T
    brk = np.concatenate([br[:-1][keep], [br[1:][keep][-1]]])
    return brk, coef


def pulse_from_spectrum(t, wavelengths_nm, intensities, pulse_energy, GDD=0.0, TOD=0.0,
                        use_jacobian=True, interp_kind='cubic', center_wavelength=800e-9,
                        device=None):
    """generate_pulse_from_spectrum (erk43ip_method.py:599-764, FFT path) with the
    per-sample work on the device (uppe_spectrum_field): the interpolated spectral
    density on the simulation grid, its square root and the GDD/TOD phase; then
    ifft, fftshift and the trapezoidal energy normalisation.  Returns a complex128
    torch tensor on the device."""
    import ctypes
    import torch
    from . import _lib
    lib = _lib.load()
    dev = torch.device(device if device is not None else 'cuda')
    t = np.asarray(t, dtype=np.float64)
    brk, coef = spectrum_spline(wavelengths_nm, intensities, use_jacobian, interp_kind)
    b = torch.from_numpy(np.ascontiguousarray(brk)).to(dev)
    c = torch.from_numpy(np.ascontiguousarray(coef)).to(dev)
    N, dt = len(t), float(t[1] - t[0])
    Aw = torch.empty(N, dtype=torch.complex128, device=dev)
    _lib.check(lib.uppe_spectrum_field(ctypes.c_void_p(b.data_ptr()), ctypes.c_void_p(c.data_ptr()), len(brk), N,
                                       dt, C0 / center_wavelength, float(GDD), float(TOD),
                                       ctypes.c_void_p(Aw.data_ptr()), _lib.stream_ptr()), 'uppe_spectrum_field')
    A = torch.fft.fftshift(torch.fft.ifft(Aw))
    P = (A.real ** 2 + A.imag ** 2)
    E = float(torch.trapezoid(P, torch.from_numpy(t).to(dev)))
    if E > 0:
        A = A * np.sqrt(pulse_energy / E)
    return A
