"""Host pieces of the input-pulse builders and the beam-diagnostics oracle against
fixtures from the reference's own code run here (tests/golden/make_golden.py:
make_pulses, make_beam_diag)."""
import numpy as np

from conftest import golden, rel_l2


def test_dispersed_pulse_host_matches_reference():
    """generate_dispersed_pulse (erk43ip_method.py:383-446), three GDD/TOD sets."""
    from project_b200.pulses import dispersed_pulse
    g = golden('ref1d_pulses')
    for k in range(3):
        A = dispersed_pulse(g['t'], float(g['E']), float(g['fwhm']), float(g['gdd'][k]), float(g['tod'][k]))
        assert rel_l2(A, g[f'D{k}']) < 1e-13


def test_simpson_weights_match_scipy():
    """The weights behind the exact-Fourier sum reproduce scipy.integrate.simpson
    (irregular-spacing rule; odd and even sample counts)."""
    from scipy.integrate import simpson
    from project_b200.pulses import simpson_weights
    rng = np.random.Generator(np.random.PCG64(5))
    for n in (2, 3, 4, 7, 10, 259, 1204):
        x = np.sort(rng.uniform(-1.0, 2.0, n))
        y = rng.standard_normal(n) + 1j * rng.standard_normal(n)
        assert abs(np.sum(simpson_weights(x) * y) - simpson(y, x=x)) <= 1e-13 * np.sum(np.abs(y))
        xu = np.linspace(3e12, 7e12, n)
        assert abs(np.sum(simpson_weights(xu) * y) - simpson(y, x=xu)) <= 1e-13 * abs(simpson(np.abs(y), x=xu))


def test_beam_diagnostics_oracle_matches_reference_snapshot():
    """oracle/diagnostics.py against MPC_Final_Runner.save_snapshot
    (src/3+1D-ERK4(3)IP UPPE/sim.py:187-249) run on the same seeded field.  The
    reference works on a complex64 field with some sums in float32, hence 5e-6."""
    from oracle import diagnostics as od
    g = golden('ref3d_beam_diag')
    A = g['field_norm'].astype(np.complex128) * float(g['A_scale'])
    o = od.beam_diagnostics(A, g['x'], g['x'], g['t'], float(g['w0']), float(g['lam']))
    for k in ('energy_total', 'x_mean_m', 'y_mean_m', 'wx_rms_m', 'wy_rms_m', 'P_t', 'fluence', 'spec_smf',
              'spec_full_incoh', 'spec_center', 'I_center_t', 'I_smf_t', 'freq_abs_Hz'):
        a = np.asarray(o[k], dtype=np.float64)
        b = np.asarray(g['ref_' + k], dtype=np.float64)
        assert np.max(np.abs(a - b)) <= 5e-6 * max(np.max(np.abs(b)), 1e-300), k
    assert o['it_peak'] == int(g['ref_it_peak'])
