"""Propagation programs (sliced gas cell, multipass cell with mirrors) on the
device vs the reference's driver loops restated over the oracle (GPU)."""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

LAM = 800e-9


def _mirror(A, t, loss, gdd, tod):
    """test_gaussian_pulse GDD TOD 1mj copy.py:282-290"""
    A = A * np.sqrt(1 - loss)
    w = 2 * np.pi * np.fft.fftfreq(len(t), t[1] - t[0])
    return np.fft.ifft(np.fft.fft(A) * np.exp(1j * (0.5 * gdd * w ** 2 + (1.0 / 6.0) * tod * w ** 3)))


def _oracle_run(prog, osolvers, A0, t):
    """The reference's loops: per slice solver.gamma = gamma; propagate; keep A_hist[-1]."""
    from project_b200.programs import Slice
    A, recs = A0.copy(), []
    for o in prog:
        if isinstance(o, Slice):
            os_ = osolvers[id(o.solver)]
            if o.gamma is not None:
                os_.gamma = o.gamma
            _, Ah, _, _ = os_.propagate(A, t, L=o.L, tol=o.tol, max_step=o.max_step, min_step=o.min_step)
            A = Ah[-1]
        else:
            A = _mirror(A, t, 1 - o.amp ** 2, o.gdd, o.tod)
        if o.record:
            recs.append(A.copy())
    return A, recs


def test_gas_cell_program_matches_oracle_loop():
    from oracle import uppe1d as o1
    from oracle.inputs import gaussian_pulse
    from project_b200.programs import ProgramRunner, gas_cell_program
    from project_b200.solver1d import ERK43IP_UPPE
    t = np.linspace(-0.5e-12, 0.5e-12, 1024)
    kw = dict(n2=1.0e-23, beam_radius=100e-6, center_wavelength=LAM, use_raman=False,
              use_self_steepening=True, taylor=(15e-30, 15e-45))
    sol = ERK43IP_UPPE(material='argon_gas', **kw)
    osol = o1.Solver1D(material='argon_gas', **kw)
    prog = gas_cell_program(sol, L_cell=0.4, n_slices=8, w0=100e-6, n2=1e-23, center_wavelength=LAM)
    A0 = gaussian_pulse(t, 60e-6, 30e-15)
    finals, recs, res = ProgramRunner([prog], t, 'double').run([A0])
    Ao, ro = _oracle_run(prog, {id(sol): osol}, A0, t)
    assert all(r.status == 0 for r in res[0])
    assert rel_l2(finals[0], Ao) < 1e-10
    assert len(recs[0]) == len(ro) == 8
    for a, b in zip(recs[0], ro):
        assert rel_l2(a, b) < 1e-10
    # the slices' gammas differ (focused beam), and the result differs from one slice
    assert len({round(s.gamma, 20) for s in prog}) > 2


def test_multipass_programs_batched_match_oracle_loops():
    """Two passes of air / crystal (with Raman) / air / mirror; three programs with
    different mirror GDD in one launch."""
    from oracle import uppe1d as o1
    from oracle.inputs import gaussian_pulse
    from project_b200.programs import Mirror, ProgramRunner, multipass_program
    from project_b200.solver1d import ERK43IP_UPPE
    t = np.linspace(-0.4e-12, 0.4e-12, 512)
    akw = dict(n2=0.0, beam_radius=200e-6, center_wavelength=LAM, use_raman=False,
               use_self_steepening=True, taylor=(20e-30, 0.0))
    ckw = dict(n2=2.6e-20, beam_radius=200e-6, center_wavelength=LAM, use_raman=True,
               use_self_steepening=True)
    air, crys = ERK43IP_UPPE(material='argon_gas', **akw), ERK43IP_UPPE(material='fused_silica', **ckw)
    oair, ocrys = o1.Solver1D(material='argon_gas', **akw), o1.Solver1D(material='fused_silica', **ckw)
    w0, zR = 200e-6, np.pi * (200e-6) ** 2 / LAM

    def w_at(z):
        return w0 * np.sqrt(1 + (z / zR) ** 2)

    progs = []
    for gdd in (-50e-30, -100e-30, -150e-30):
        progs.append(multipass_program(air, crys, n_passes=2, L_cavity=0.3, L_crystal=3e-3,
                                       crystal_offset=0.01, w_at=w_at, n2_air=0.0, n2_crystal=2.6e-20,
                                       center_wavelength=LAM, air_slices=2, crystal_slices=3,
                                       mirror=Mirror(loss=0.01, gdd=gdd, tod=-20e-45)))
    A0 = gaussian_pulse(t, 20e-6, 40e-15)
    finals, recs, res = ProgramRunner(progs, t, 'double').run([A0] * 3)
    for p in range(3):
        Ao, ro = _oracle_run(progs[p], {id(air): oair, id(crys): ocrys}, A0, t)
        assert rel_l2(finals[p], Ao) < 1e-10
        assert len(recs[p]) == len(ro)
        assert max(rel_l2(a, b) for a, b in zip(recs[p], ro)) < 1e-10
        # mirror energies: loss 1 %
        mres = [r for r, o in zip(res[p], progs[p]) if not hasattr(o, 'solver')]
        assert len(mres) == 2
    assert rel_l2(finals[0], finals[2]) > 1e-3


def test_program_mixed_precision_vs_fp64():
    from oracle.inputs import gaussian_pulse
    from project_b200.programs import ProgramRunner, gas_cell_program
    from project_b200.solver1d import ERK43IP_UPPE
    t = np.linspace(-0.5e-12, 0.5e-12, 2048)
    kw = dict(n2=1.0e-23, beam_radius=100e-6, center_wavelength=LAM, use_raman=False,
              use_self_steepening=True, taylor=(15e-30, 15e-45))
    sol = ERK43IP_UPPE(material='argon_gas', **kw)
    prog = gas_cell_program(sol, L_cell=0.4, n_slices=8, w0=100e-6, n2=1e-23, center_wavelength=LAM,
                            record=False)
    A0 = gaussian_pulse(t, 60e-6, 30e-15)
    fd, _, _ = ProgramRunner([prog], t, 'double').run([A0])
    fs, _, _ = ProgramRunner([prog], t, 'single').run([A0])
    assert rel_l2(fs[0], fd[0]) < 1e-4
