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


def test_sequence_3d_with_mirrors_matches_oracle_loop():
    """sim.py:304-331 pattern on a small grid: air / plate / curved mirror / plate /
    air / flat-mirror loss, two media (argon at 1 and 3 bar as stand-ins)."""
    import torch
    from oracle import uppe3d
    from oracle.inputs import gaussian_beam_3d
    from project_b200.media import Argon
    from project_b200.programs import Mirror3D, Segment3D, run_sequence_3d
    from project_b200.solver3d import ERK43IP_UPPE_3D_Optimized
    x = np.linspace(-1.5e-3, 1.5e-3, 16)
    t = np.linspace(-100e-15, 100e-15, 64)
    A0 = gaussian_beam_3d(x, x, t, 0.5e-3, 1e-4, 40e-15)
    sa = ERK43IP_UPPE_3D_Optimized(x, x, t, Argon(LAM, 1.0, 'double', True), precision='double')
    sf = ERK43IP_UPPE_3D_Optimized(x, x, t, Argon(LAM, 3.0, 'double', True), precision='double')
    oa = uppe3d.Solver3D(x, x, t, uppe3d.argon(LAM, 1.0, 'double', True), 'double')
    of = uppe3d.Solver3D(x, x, t, uppe3d.argon(LAM, 3.0, 'double', True), 'double')
    R, loss = 0.5, 0.05
    ops = [Segment3D(sa, 0.02, max_step=5e-3), Segment3D(sf, 0.01, tol=1e-5, max_step=2e-3),
           Mirror3D(R=R), Segment3D(sf, 0.01, tol=1e-5, max_step=2e-3), Segment3D(sa, 0.02, max_step=5e-3),
           Mirror3D(loss=loss)]
    A_dev, _ = run_sequence_3d(ops, torch.from_numpy(A0).cuda())
    # the reference loop over the oracle
    X, Y = np.meshgrid(x, x, indexing='ij')
    omega = 2 * np.pi * np.fft.fftfreq(len(t), t[1] - t[0])
    k = (2 * np.pi * 299792458.0 / LAM + omega) / 299792458.0
    mirror_phase = np.exp(-1j * k[None, None, :] * (X ** 2 + Y ** 2)[:, :, None] / R)
    A = A0.copy()
    for op in ops:
        if isinstance(op, Segment3D):
            os_ = oa if op.solver is sa else of
            _, _, A_w, _ = os_.propagate(A, op.L, tol=op.tol, max_step=op.max_step, min_step=op.min_step)
            A = np.fft.ifft(np.fft.ifftshift(A_w, axes=-1), axis=-1)
        elif op.R is not None:
            A = np.fft.ifft(np.fft.fft(A, axis=-1) * mirror_phase, axis=-1)
        else:
            A = A * np.sqrt(1 - op.loss)
    assert rel_l2(A_dev.cpu().numpy(), A) < 1e-10
