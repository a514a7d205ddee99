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


def _line_transform(x, direction, scale, shift_in=False, shift_out=False):
    """One complex128 device line through uppe_fft_c128 (N a power of two)."""
    import ctypes
    import torch
    from . import _lib
    lib = _lib.load()
    N = x.numel()
    if N < 2 or N & (N - 1):
        raise ValueError(f'the device line transform needs a power-of-two length, got {N}')
    x = x.to(torch.complex128).contiguous()
    out = torch.empty_like(x)
    work = torch.empty(2 * N, dtype=torch.complex128, device=x.device)
    _lib.check(lib.uppe_fft_c128(ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                 ctypes.c_void_p(work.data_ptr()), N, int(direction), float(scale),
                                 1 if shift_in else 0, 1 if shift_out else 0, _lib.stream_ptr()), 'uppe_fft_c128')
    return out


def dispersed_pulse_device(t, pulse_energy, pulse_fwhm, GDD=0.0, TOD=0.0, device=None):
    """generate_dispersed_pulse (erk43ip_method.py:383-446) on the device: the
    transform-limited Gaussian, ifftshift, fft, the phase GDD w^2/2 + TOD w^3/6,
    ifft and fftshift, all in the library's kernels (uppe_fft_c128,
    uppe_spectral_phase).  Returns a complex128 torch tensor on the device."""
    import ctypes
    import torch
    from . import _lib
    lib = _lib.load()
    dev = torch.device(device if device is not None else 'cuda')
    t = np.asarray(t, dtype=np.float64)
    P0 = pulse_energy / (pulse_fwhm * np.sqrt(np.pi / (4 * np.log(2))))
    T0 = pulse_fwhm / (2 * np.sqrt(np.log(2)))
    A = torch.from_numpy(np.sqrt(P0) * np.exp(-(t / T0) ** 2 / 2)).to(dev).to(torch.complex128)
    if GDD == 0 and TOD == 0:
        return A
    N = len(t)
    spec = _line_transform(A, -1, 1.0, shift_in=True)                         # fft(ifftshift(A))
    _lib.check(lib.uppe_spectral_phase(ctypes.c_void_p(spec.data_ptr()), N, float(t[1] - t[0]), float(GDD),
                                       float(TOD), _lib.stream_ptr()), 'uppe_spectral_phase')
    return _line_transform(spec, +1, 1.0 / N, shift_out=True)                 # fftshift(ifft(.))


def exact_fourier_pulse(t, wavelengths_nm, intensities, pulse_energy, GDD=0.0, TOD=0.0, use_jacobian=True,
                        interp_kind='cubic', center_wavelength=800e-9, device=None):
    """generate_pulse_from_spectrum(exact_fourier=True) (erk43ip_method.py:492-598,
    664-672, 734-741): the spectrum interpolated with interp1d onto a dense uniform
    frequency grid (min(4096, 4 n) points), its precise FWHM centre, the Simpson
    weights of scipy.integrate.simpson for that grid (the irregular-spacing form it
    applies when x is given, with the last-interval correction for an even count),
    then the direct sum over the dense grid for every t on the device
    (uppe_exact_ft) and the trapezoidal energy normalisation.  Returns
    (A, center_freq, delta_nu) with A a complex128 torch tensor on the device."""
    import ctypes
    import torch
    from scipy.interpolate import interp1d
    from . import _lib
    from .analysis import fwhm_precise
    lib = _lib.load()
    dev = torch.device(device if device is not None else 'cuda')
    t = np.asarray(t, dtype=np.float64)
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
    if f[0] < f[-1]:
        f, I = f[::-1], I[::-1]
    kind = 'linear' if interp_kind in ('cubic', 'quadratic') and len(f) < 4 else interp_kind
    fi = interp1d(f, I, kind=kind, bounds_error=False, fill_value=0.0)
    nd = min(4096, len(f) * 4)
    fd = np.linspace(f.min(), f.max(), nd)
    sd = fi(fd)
    sd[sd < 0] = 0
    fl, fr, dnu = fwhm_precise(fd, sd)
    if dnu:
        fc = (fl + fr) / 2
    else:
        fc = np.sum(fd * sd) / np.sum(sd) if np.sum(sd) > 0 else C0 / center_wavelength
    x = fd - fc
    om = 2 * np.pi * x
    phase = 0.5 * GDD * om ** 2 + (1.0 / 6.0) * TOD * om ** 3
    w = simpson_weights(x)
    amp = w * np.sqrt(sd) * np.exp(1j * phase)
    td = torch.from_numpy(t).to(dev)
    omd = torch.from_numpy(np.ascontiguousarray(om)).to(dev)
    ad = torch.from_numpy(np.ascontiguousarray(amp.astype(np.complex128))).to(dev)
    A = torch.empty(len(t), dtype=torch.complex128, device=dev)
    _lib.check(lib.uppe_exact_ft(ctypes.c_void_p(td.data_ptr()), len(t), ctypes.c_void_p(omd.data_ptr()),
                                 ctypes.c_void_p(ad.data_ptr()), nd, ctypes.c_void_p(A.data_ptr()),
                                 _lib.stream_ptr()), 'uppe_exact_ft')
    P = A.real ** 2 + A.imag ** 2
    E = float(torch.trapezoid(P, td))
    if E > 0:
        A = A * np.sqrt(pulse_energy / E)
    return A, fc, dnu


def simpson_weights(x):
    """Weights w with sum w_k y_k = scipy.integrate.simpson(y, x=x) for 1-D x (the
    composite rule for irregular spacing over pairs of intervals; for an even
    number of samples the rule covers the first n - 2 intervals and the last one
    gets the three-point correction of Cartwright's formula)."""
    x = np.asarray(x, dtype=np.float64)
    n = len(x)
    w = np.zeros(n)
    if n == 1:
        return w
    if n == 2:
        h = x[1] - x[0]
        w[:] = 0.5 * h
        return w
    h = np.diff(x)
    stop = n - 2 if n % 2 == 1 else n - 3
    for j in range(0, stop, 2):
        h0, h1 = h[j], h[j + 1]
        hs, hp = h0 + h1, h0 * h1
        r = h0 / h1 if h1 != 0 else 0.0
        w[j] += hs / 6.0 * (2.0 - (1.0 / r if r != 0 else 0.0))
        w[j + 1] += hs / 6.0 * (hs * (hs / hp if hp != 0 else 0.0))
        w[j + 2] += hs / 6.0 * (2.0 - r)
    if n % 2 == 0:
        h0, h1 = h[-2], h[-1]
        alpha = (2 * h1 ** 2 + 3 * h0 * h1) / (6 * (h1 + h0)) if (h1 + h0) != 0 else 0.0
        beta = (h1 ** 2 + 3.0 * h0 * h1) / (6 * h0) if h0 != 0 else 0.0
        eta = h1 ** 3 / (6 * h0 * (h0 + h1)) if h0 * (h0 + h1) != 0 else 0.0
        w[-1] += alpha
        w[-2] += beta
        w[-3] -= eta
    return w


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
    A = _line_transform(Aw, +1, 1.0 / N, shift_out=True)                      # fftshift(ifft(A_w))
    P = (A.real ** 2 + A.imag ** 2)
    E = float(torch.trapezoid(P, torch.from_numpy(t).to(dev)))
    if E > 0:
        A = A * np.sqrt(pulse_energy / E)
    return A
