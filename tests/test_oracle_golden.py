"""Pin the CPU oracle to golden vectors produced by the reference's own code
(tests/golden/make_golden.py).  CPU only."""
import numpy as np
import pytest

from conftest import golden, rel_l2
from oracle import uppe1d, uppe3d
from oracle.uppe3d import plasma_scan


def test_plasma_scan_matches_reference_kernel():
    g = golden('ref_plasma_kernel')
    rho, gen = plasma_scan(g['W_ion'], g['W_ava'], np.float32(g['rate_rec']),
                           np.float32(g['dt']), np.float32(g['rho_nt']))
    # lines without avalanche (all gases): bit-exact
    assert np.array_equal(rho[:20], g['rho'][:20])
    assert np.array_equal(gen[:20], g['gen'][:20])
    # avalanche lines: numpy's vector exp differs from libm exp by <= 1 ulp
    np.testing.assert_allclose(rho[20:], g['rho'][20:], rtol=1e-14)
    np.testing.assert_allclose(gen[20:], g['gen'][20:], rtol=0,
                               atol=1e-12 * np.abs(g['gen'][20:]).max())


def _argon1d():
    g = golden('ref1d_argon')
    s = uppe1d.Solver1D(material='argon_gas', n2=1.0e-23, beam_radius=0.65 * 125e-6,
                        center_wavelength=800e-9, alpha=0.5 * np.log(10) / 10,
                        use_raman=False, use_self_steepening=True)
    return g, s


def test_1d_argon_tables_bitexact():
    g, s = _argon1d()
    D, n = s.dispersion(g['omega'])
    assert np.array_equal(D, g['D'])
    assert np.array_equal(n, g['n_omega'])
    assert s.n0 == float(g['n0']) and s.gamma == float(g['gamma'])


def test_1d_argon_propagate_matches_reference():
    g, s = _argon1d()
    zh, Ah, om, log = s.propagate(g['A0'], g['t'], L=float(g['L']), tol=float(g['tol']))
    att = g['attempts']
    assert len(log) == len(att)
    np.testing.assert_allclose([r[1] for r in log], att[:, 0], rtol=1e-12)
    np.testing.assert_allclose([r[2] for r in log], att[:, 1], rtol=1e-8)
    assert len(zh) == int(g['n_hist'])
    assert rel_l2(Ah[-1], g['A_final']) < 1e-13


def test_1d_silica_raman_units_and_propagate():
    g = golden('ref1d_silica_raman')
    s = uppe1d.Solver1D(material='fused_silica', n2=2.6e-20, beam_radius=30e-6,
                        center_wavelength=1064e-9)
    t = g['t']
    om = 2 * np.pi * np.fft.fftfreq(len(t), t[1] - t[0])
    s.setup(om, t[1] - t[0])
    assert np.array_equal(s._D, g['D'])
    assert rel_l2(s._H, g['H_R']) < 1e-15
    assert rel_l2(s.nonlinear_operator(g['A_rand']), g['N_A']) < 1e-14
    assert rel_l2(s.linear_operator(g['A_rand'], float(g['h_L'])), g['L_A']) < 1e-14
    A4, err = s.erk43_step(g['A_rand'], float(g['step_h']))
    assert rel_l2(A4, g['step_A4']) < 1e-14
    assert abs(err - float(g['step_err'])) <= 1e-10 * float(g['step_err'])
    zh, Ah, _, log = s.propagate(g['A0'], t, L=float(g['L']), tol=float(g['tol']))
    assert len(log) == len(g['attempts'])
    assert rel_l2(Ah[-1], g['A_final']) < 1e-13


def test_1d_spm_nodispersion():
    g = golden('ref1d_spm')
    s = uppe1d.Solver1D(material='fused_silica', n2=2.6e-20, beam_radius=50e-6,
                        center_wavelength=800e-9, use_raman=False, use_self_steepening=False)
    s.dispersion = lambda om: (np.zeros_like(om, dtype=complex), np.ones_like(om))
    zh, Ah, _, log = s.propagate(g['A0'], g['t'], L=float(g['L']), tol=float(g['tol']))
    assert len(log) == len(g['attempts'])
    assert rel_l2(Ah[-1], g['A_final']) < 1e-13
    # known answer: pure SPM A(L) = A0 exp(i gamma |A0|^2 L)
    exact = g['A0'] * np.exp(1j * float(g['gamma']) * np.abs(g['A0']) ** 2 * float(g['L']))
    assert rel_l2(Ah[-1], exact) < 1e-7


CASES3D = ['ref3d_adk_taylor_double', 'ref3d_mpi_cauchy_double', 'ref3d_mpi_cauchy_single',
           'ref3d_noshock_double']


def make_oracle3d(g):
    prec = str(g['precision'])
    tay = g['taylor']
    disp = ('taylor', float(tay[0]), float(tay[1]), float(tay[2])) if str(g['lut']) == 'adk' and tay[0] != 0 else None
    med = uppe3d.argon(float(g['lam']), 1.0, prec, bool(g['shock']), dispersion=disp)
    med.W_gpu = g['W_lut'].astype(med.float_dtype)
    sol = uppe3d.Solver3D(g['x'], g['y'], g['t'], med, prec)
    return med, sol


@pytest.mark.parametrize('name', CASES3D)
def test_3d_matches_reference(name):
    g = golden(name)
    med, sol = make_oracle3d(g)
    double = str(g['precision']) == 'double'
    tol_unit = 1e-13 if double else 1e-6
    assert rel_l2(sol.D_operator, g['D']) < (1e-15 if double else 1e-7)
    K, P = med.calc_nonlinear_response(g['A0'], sol.dt)
    assert rel_l2(K, g['Kerr']) < tol_unit
    assert rel_l2(P, g['Plasma']) < tol_unit
    sol.A_scale = float(g['A_scale'])
    An = (g['A0'] / sol.complex_dtype(sol.A_scale + 0.0j)).astype(sol.complex_dtype)
    A4, err, _, _ = sol.erk43_step(An, float(g['step_h']))
    assert rel_l2(A4, g['step_A4_t']) < tol_unit
    assert abs(err - float(g['step_err'])) <= (1e-9 if double else 1e-3) * float(g['step_err'])
    z, freq, A_w, log = sol.propagate(g['A0'], float(g['L']), tol=float(g['tol']))
    att = g['attempts']
    assert len(log) == len(att)
    np.testing.assert_allclose([r[1] for r in log], att[:, 0], rtol=1e-9 if double else 1e-3)
    assert abs(z - float(g['z'])) < 1e-12
    assert np.array_equal(freq, g['freq'])
    assert rel_l2(A_w, g['A_w']) < (1e-12 if double else 1e-5)


def test_pulse_from_spectrum_oracle_matches_reference():
    """generate_pulse_from_spectrum (erk43ip_method.py:599-764) run here on a seeded
    spectrum, four option sets (cubic / linear / quadratic, Jacobian on/off, GDD/TOD,
    descending input order)."""
    from oracle.inputs import pulse_from_spectrum
    g = golden('ref1d_spectrum_pulse')
    for k in range(4):
        w, i = (g['wl'][::-1], g['I'][::-1]) if g['rev'][k] else (g['wl'], g['I'])
        A = pulse_from_spectrum(g['t'], w, i, float(g['E']), float(g['gdd'][k]), float(g['tod'][k]),
                                bool(g['jac'][k]), str(g['kinds'][k]))
        assert rel_l2(A, g[f'A{k}']) < 1e-13


@pytest.mark.parametrize('name', ['argon', 'silica', 'xenon', 'silica_raman'])
def test_realfield_oracle_matches_reference(name):
    """Real-field solver (src/3+1D-UPPE-ERK4(3)IP-real-field) run here: PPT table,
    density + Drude current response (with the fused-silica Raman convolution for
    silica_raman), one step, and the adaptive run."""
    from oracle import realfield as rf
    g = golden(f'refrf_{name}')
    m = {'argon': lambda: rf.argon(800e-9, 1.0), 'silica': lambda: rf.fused_silica(800e-9),
         'xenon': lambda: rf.xenon(800e-9, 2.0),
         'silica_raman': lambda: rf.fused_silica(800e-9, use_raman=True)}[name]()
    assert np.array_equal(m.W_gpu, g['lut_W'])
    dt = float(g['t'][1] - g['t'][0])
    m.init_raman(len(g['t']), dt)          # the reference's solver does this on construction
    P, J = m.response(g['E0'], dt)
    assert np.array_equal(P, g['P']) and np.array_equal(J, g['J'])
    s = rf.Solver(g['x'], g['x'], g['t'], m)
    z, f, Ew, log = s.propagate(g['E0'], float(g['L']), tol=float(g['tol']), max_step=float(g['L']) / 4,
                                min_step=1e-9)
    assert np.allclose(np.array(log), g['attempts'], rtol=1e-6, atol=0)
    assert rel_l2(Ew, g['Ew']) < 1e-6
