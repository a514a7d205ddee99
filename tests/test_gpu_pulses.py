"""Device input-pulse builders and beam diagnostics against the reference's own
code run here (GPU).  Fixtures: tests/golden/make_golden.py (make_pulses,
make_beam_diag)."""
import numpy as np
import pytest

from conftest import golden, rel_l2

pytestmark = pytest.mark.gpu


def test_dispersed_pulse_device_matches_reference():
    from project_b200.pulses import dispersed_pulse_device
    g = golden('ref1d_pulses')
    for k in range(3):
        A = dispersed_pulse_device(g['t'], float(g['E']), float(g['fwhm']), float(g['gdd'][k]),
                                   float(g['tod'][k]))
        assert rel_l2(A.cpu().numpy(), g[f'D{k}']) < 1e-12


def test_exact_fourier_pulse_matches_reference():
    """generate_pulse_from_spectrum(exact_fourier=True) (erk43ip_method.py:492-598):
    the dense-grid direct sum runs on the device (uppe_exact_ft)."""
    from project_b200.pulses import exact_fourier_pulse
    g = golden('ref1d_pulses')
    for k in range(2):
        A, fc, dnu = exact_fourier_pulse(g['te'], g['wl'], g['I'], float(g['Ex']), float(g['x_gdd'][k]),
                                         float(g['x_tod'][k]), bool(g['x_jac'][k]), str(g['x_kinds'][k]))
        assert rel_l2(A.cpu().numpy(), g[f'X{k}']) < 1e-12


def test_line_transform_matches_numpy():
    import torch
    from project_b200.pulses import _line_transform
    rng = np.random.Generator(np.random.PCG64(9))
    for n in (2, 8, 1024, 16384):
        x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
        xd = torch.from_numpy(x).cuda()
        assert rel_l2(_line_transform(xd, -1, 1.0).cpu().numpy(), np.fft.fft(x)) < 1e-14
        assert rel_l2(_line_transform(xd, +1, 1.0 / n, shift_out=True).cpu().numpy(),
                      np.fft.fftshift(np.fft.ifft(x))) < 1e-14
        assert rel_l2(_line_transform(xd, -1, 2.0, shift_in=True).cpu().numpy(),
                      2.0 * np.fft.fft(np.fft.ifftshift(x))) < 1e-14


def test_beam_diagnostics_device_matches_reference_snapshot():
    """The device pass (uppe3d_beam_diagnostics) on the field of the reference's
    save_snapshot run (src/3+1D-ERK4(3)IP UPPE/sim.py:187-249), complex128 plan;
    the reference's own float32 sums set the 5e-6 tolerance."""
    import torch
    from project_b200.media import Argon
    from project_b200.solver3d import ERK43IP_UPPE_3D_Optimized
    g = golden('ref3d_beam_diag')
    lam = float(g['lam'])
    sol = ERK43IP_UPPE_3D_Optimized(g['x'], g['x'], g['t'], Argon(lam, 1.0, 'double', False), precision='double')
    A = g['field_norm'].astype(np.complex128) * float(g['A_scale'])
    sol.set_field(torch.from_numpy(A).cuda())
    o = sol.beam_diagnostics(w_mode=float(g['w0']))
    for k in ('energy_total', 'x_mean_m', 'y_mean_m', 'wx_rms_m', 'wy_rms_m', 'P_t', 'fluence', 'spec_smf',
              'spec_full_incoh', 'spec_center', 'I_center_t', 'I_smf_t', 'freq_abs_Hz'):
        a = np.asarray(o[k], dtype=np.float64)
        b = np.asarray(g['ref_' + k], dtype=np.float64)
        assert np.max(np.abs(a - b)) <= 5e-6 * max(np.max(np.abs(b)), 1e-300), k
    assert o['it_peak'] == int(g['ref_it_peak'])
