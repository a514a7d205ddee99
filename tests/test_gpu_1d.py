"""1D CUDA path vs the reference-generated goldens and the oracle (GPU)."""
import numpy as np
import pytest

from conftest import golden, rel_l2

pytestmark = pytest.mark.gpu


def argon_solver(precision='double', **kw):
    from project_b200.solver1d import ERK43IP_UPPE
    return ERK43IP_UPPE(material='argon_gas', n2=1.0e-23, beam_radius=0.65 * 125e-6,
                        center_wavelength=800e-9, alpha=0.5 * np.log(10) / 10, use_raman=False,
                        use_self_steepening=True, precision=precision, **kw)


def test_argon_capillary_matches_reference():
    g = golden('ref1d_argon')
    s = argon_solver()
    zh, Ah, om = s.propagate(g['A0'], g['t'], L=float(g['L']), tol=float(g['tol']))
    r = s.last_result
    assert r.status == 0
    assert r.attempts == len(g['attempts'])
    assert len(zh) == int(g['n_hist'])
    # err = |A4 - A3| / |A4| is a difference of nearly equal fields, accurate to
    # ~1e-10 relative in FP64, so free-running step sizes agree to ~1e-11
    np.testing.assert_allclose(zh, g['z_hist'], rtol=1e-9, atol=1e-15)
    assert rel_l2(Ah[-1], g['A_final']) < 1e-10
    assert np.array_equal(om, g['omega'])


def test_silica_raman_matches_reference():
    from project_b200.solver1d import ERK43IP_UPPE
    g = golden('ref1d_silica_raman')
    s = ERK43IP_UPPE(material='fused_silica', n2=2.6e-20, beam_radius=30e-6,
                     center_wavelength=1064e-9)
    zh, Ah, om = s.propagate(g['A0'], g['t'], L=float(g['L']), tol=float(g['tol']))
    assert s.last_result.attempts == len(g['attempts'])
    assert len(zh) == int(g['n_hist'])
    assert rel_l2(Ah[-1], g['A_final']) < 1e-10


def test_spm_known_answer():
    """Dispersion switched off (src/1D-ERK4(3)IP UPPE/test_3d-1d.py:52-61):
    A(L) = A0 exp(i gamma |A0|^2 L)."""
    from project_b200.solver1d import ERK43IP_UPPE
    g = golden('ref1d_spm')
    s = ERK43IP_UPPE(material='fused_silica', n2=2.6e-20, beam_radius=50e-6,
                     center_wavelength=800e-9, use_raman=False, use_self_steepening=False,
                     taylor=(0.0, 0.0))
    zh, Ah, om = s.propagate(g['A0'], g['t'], L=float(g['L']), tol=float(g['tol']))
    assert rel_l2(Ah[-1], g['A_final']) < 1e-10
    exact = g['A0'] * np.exp(1j * float(g['gamma']) * np.abs(g['A0']) ** 2 * float(g['L']))
    assert rel_l2(Ah[-1], exact) < 1e-7


def _plasma_pair(W0=3e12):
    from oracle import uppe1d as o1
    from project_b200.solver1d import ERK43IP_UPPE, GasPlasma1D
    Aeff = np.pi * (0.65 * 125e-6) ** 2
    op = o1.Plasma1D(Aeff, center_wavelength=800e-9)
    W = np.minimum(W0 * (10.0 ** op.log10_I / 5e17) ** 8, 1e20)
    op.W = W
    kw = dict(n2=1.0e-23, beam_radius=0.65 * 125e-6, center_wavelength=800e-9,
              alpha=0.11513, use_raman=False, use_self_steepening=True)
    osol = o1.Solver1D(material='argon_gas', taylor=(15e-30, 15e-45), plasma=op, **kw)
    psol = ERK43IP_UPPE(material='argon_gas', taylor=(15e-30, 15e-45),
                        plasma=GasPlasma1D(Aeff, lut=(op.log10_I, W)), **kw)
    return osol, psol


def test_plasma_1d_vs_oracle():
    from oracle.inputs import gaussian_pulse
    osol, psol = _plasma_pair()
    t = np.linspace(-0.5e-12, 0.5e-12, 1024)
    fwhm = 30e-15
    A0 = gaussian_pulse(t, 2e9 * fwhm * np.sqrt(np.pi / (4 * np.log(2))), fwhm)
    zo, Ao, _, log = osol.propagate(A0, t, L=0.05, tol=1e-6)
    zh, Ah, _ = psol.propagate(A0, t, L=0.05, tol=1e-6)
    assert psol.last_result.attempts == len(log)
    assert rel_l2(Ah[-1], Ao[-1]) < 1e-10
    # the plasma term changed the field (it is not negligible in this case)
    osol.plasma = None
    zn, An, _, _ = osol.propagate(A0, t, L=0.05, tol=1e-6)
    assert rel_l2(An[-1], Ao[-1]) > 1e-6


def test_mixed_precision_vs_fp64():
    g = golden('ref1d_argon')
    s = argon_solver(precision='single')
    zh, Ah, om = s.propagate(g['A0'], g['t'], L=float(g['L']), tol=float(g['tol']))
    assert abs(zh[-1] - g['z_hist'][-1]) < 1e-12
    assert rel_l2(s.last_final, g['A_final']) < 1e-4


def test_batched_instances_match_individual_oracle_runs():
    from oracle import uppe1d as o1
    from oracle.inputs import gaussian_pulse
    from project_b200.solver1d import BatchedPropagator
    rng = np.random.Generator(np.random.PCG64(2))
    insts, fields, refs = [], [], []
    for k in range(6):
        Nt = int(rng.choice([256, 512, 1024, 2048]))
        t = np.linspace(-0.5e-12, 0.5e-12, Nt)
        P = float(rng.uniform(0.2, 3.0))
        E = float(np.exp(rng.uniform(np.log(5e-6), np.log(60e-6))))
        kw = dict(n2=1.0e-23 * P, beam_radius=0.65 * 125e-6, center_wavelength=800e-9,
                  alpha=0.11513, use_raman=False, use_self_steepening=True)
        A0 = gaussian_pulse(t, E, 30e-15)
        L = 0.05
        osol = o1.Solver1D(material='argon_gas', taylor=(15e-30 * P, 15e-45 * P), **kw)
        _, Ao, _, _ = osol.propagate(A0, t, L=L, tol=1e-6)
        refs.append(Ao[-1])
        from project_b200.solver1d import ERK43IP_UPPE
        psol = ERK43IP_UPPE(material='argon_gas', taylor=(15e-30 * P, 15e-45 * P), **kw)
        insts.append(psol.instance(t, L, tol=1e-6))
        fields.append(A0)
    bp = BatchedPropagator(insts, precision='double')
    finals, _, res = bp.run(fields)
    for f, r0, r in zip(finals, refs, res):
        assert r.status == 0
        assert rel_l2(f, r0) < 1e-10


def test_diagnostics_vs_oracle():
    """Energy, photon number and peak ionisation fraction (initial and accepted states)."""
    from oracle.inputs import gaussian_pulse
    osol, psol = _plasma_pair()
    t = np.linspace(-0.5e-12, 0.5e-12, 1024)
    fwhm = 30e-15
    A0 = gaussian_pulse(t, 2e9 * fwhm * np.sqrt(np.pi / (4 * np.log(2))), fwhm)
    zo, Ao, _, log = osol.propagate(A0, t, L=0.05, tol=1e-6)
    peak = max(osol.ionization_fraction(a) for a in Ao)     # every accepted state is in the history
    Eo, pho = osol.diagnostics(Ao[-1], t)
    psol.propagate(A0, t, L=0.05, tol=1e-6)
    r = psol.last_result
    assert peak > 1e-8
    assert abs(r.energy - Eo) <= 1e-10 * Eo
    assert abs(r.photons - pho) <= 1e-10 * pho
    assert abs(r.peak_ion - peak) <= 1e-8 * peak


def test_pulse_from_spectrum_matches_reference():
    """The device spectrum-to-field builder vs generate_pulse_from_spectrum run here."""
    from project_b200.pulses import pulse_from_spectrum
    g = golden('ref1d_spectrum_pulse')
    for k in range(4):
        w, i = (g['wl'][::-1], g['I'][::-1]) if g['rev'][k] else (g['wl'], g['I'])
        A = pulse_from_spectrum(g['t'], w, i, float(g['E']), float(g['gdd'][k]), float(g['tod'][k]),
                                bool(g['jac'][k]), str(g['kinds'][k]))
        assert rel_l2(A.cpu().numpy(), g[f'A{k}']) < 1e-12
