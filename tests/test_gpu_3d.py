"""3+1D CUDA path vs the oracle and the reference-generated goldens (GPU)."""
import numpy as np
import pytest

from conftest import golden, rel_l2

pytestmark = pytest.mark.gpu

CASES = ['ref3d_mpi_cauchy_double', 'ref3d_adk_taylor_double', 'ref3d_noshock_double']


def product_solver(g, precision=None):
    from project_b200.media import Argon
    from project_b200.solver3d import ERK43IP_UPPE_3D_Optimized
    prec = precision or str(g['precision'])
    tay = g['taylor']
    disp = ('taylor', float(tay[0]), float(tay[1]), float(tay[2])) if str(g['lut']) == 'adk' else None
    med = Argon(float(g['lam']), 1.0, prec, bool(g['shock']), dispersion=disp,
                lut=(g['log10_I'], g['W_lut']))
    return ERK43IP_UPPE_3D_Optimized(g['x'], g['y'], g['t'], med, precision=prec)


@pytest.mark.parametrize('name', CASES)
def test_single_attempt_matches_reference(name):
    g = golden(name)
    sol = product_solver(g)
    sol.set_field(g['A0'])
    err = sol.attempt(float(g['step_h']))
    assert abs(err - float(g['step_err'])) <= 1e-9 * float(g['step_err'])
    sol.commit(True)
    A4 = sol.field().cpu().numpy() / float(g['A_scale'])
    assert rel_l2(A4, g['step_A4_t']) < 1e-11


@pytest.mark.parametrize('name', CASES)
def test_replay_matches_reference(name):
    """Replay the reference's (h, accept) sequence: field parity at 1e-10 in c128."""
    g = golden(name)
    sol = product_solver(g)
    sol.set_field(g['A0'])
    tol = float(g['tol'])
    for h, err_ref in g['attempts']:
        err = sol.attempt(h)
        # errors at round-off level (~1e-16) carry no information beyond their size
        assert abs(err - err_ref) <= 1e-8 * err_ref + 1e-13 * tol
        sol.commit(err_ref < tol)
    A_w = sol.spectrum().cpu().numpy()
    assert rel_l2(A_w, g['A_w']) < 1e-10


@pytest.mark.parametrize('name', CASES)
def test_free_running_propagate(name):
    g = golden(name)
    sol = product_solver(g)
    z, freq, A_w = sol.propagate(g['A0'], float(g['L']), tol=float(g['tol']))
    r = sol.last_result
    assert r.status == 0
    assert r.attempts == len(g['attempts'])
    assert abs(z - float(g['z'])) < 1e-12
    assert np.array_equal(freq, g['freq'])
    assert rel_l2(A_w, g['A_w']) < 1e-9


def test_mixed_precision_vs_fp64_reference():
    """complex64 bulk + FP64 phase/error/controller against the complex128 reference run."""
    g = golden('ref3d_mpi_cauchy_double')
    sol = product_solver(g, precision='single')
    z, freq, A_w = sol.propagate(g['A0'], float(g['L']), tol=float(g['tol']))
    assert abs(z - float(g['z'])) < 1e-12
    assert rel_l2(A_w, g['A_w']) < 1e-4


def _oracle_case(N=32, Nt=64, W0=3e9, I_peak=5e16, precision='double', seed=3):
    from oracle import uppe3d
    from oracle.inputs import speckle
    x = np.linspace(-1.5e-3, 1.5e-3, N)
    t = np.linspace(-100e-15, 100e-15, Nt)
    lam = 800e-9
    med = uppe3d.argon(lam, 1.0, precision, True)
    # MPI-like test table, capped so that it stays finite in float32
    W = np.minimum(W0 * (10.0 ** med.log10_I_cpu / 5e16) ** 8, 1e20)
    med.W_gpu = W.astype(med.float_dtype)
    sol = uppe3d.Solver3D(x, x, t, med, precision)
    X, Y = np.meshgrid(x, x, indexing='ij')
    T0 = 40e-15 / (2 * np.sqrt(np.log(2)))
    A0 = np.sqrt(I_peak) * np.exp(-(X ** 2 + Y ** 2) / (0.5e-3) ** 2)[:, :, None] * \
        np.exp(-(t / T0) ** 2 / 2)[None, None, :]
    A0 = (A0 * speckle(x, x, 50e-6, 0.01, seed)[:, :, None]).astype(np.complex128)
    lut = (med.log10_I_cpu, W)
    return x, t, lam, A0, sol, lut


def test_strong_ionisation_clamped_scan():
    """Rates above 1/dt make the reference's density clamp bind: the kernel falls
    back to the exact serial scan for those lines."""
    from project_b200.media import Argon
    from project_b200.solver3d import ERK43IP_UPPE_3D_Optimized
    x, t, lam, A0, osol, lut = _oracle_case(W0=1e15, I_peak=5e16)
    osol.A_scale = float(np.max(np.abs(A0)))
    An = A0 / osol.A_scale
    A4o, erro, _, _ = osol.erk43_step(An, 1e-5)
    med = Argon(lam, 1.0, 'double', True, lut=lut)
    sol = ERK43IP_UPPE_3D_Optimized(x, x, t, med, precision='double')
    sol.set_field(A0)
    err = sol.attempt(1e-5)
    assert abs(err - erro) <= 1e-8 * erro
    sol.commit(True)
    assert rel_l2(sol.field().cpu().numpy() / osol.A_scale, A4o) < 1e-11


@pytest.mark.parametrize('N,Nt,precision', [(64, 128, 'double'), (64, 128, 'single'),
                                             (256, 64, 'single')])
def test_larger_grid_attempts_vs_oracle(N, Nt, precision):
    """Complex64 grids with Ny >= 64 run the TMA-fed y passes (k_ypass_tma)."""
    from project_b200.media import Argon
    from project_b200.solver3d import ERK43IP_UPPE_3D_Optimized
    x, t, lam, A0, osol, lut = _oracle_case(N=N, Nt=Nt)
    z, freq, Ao, log = osol.propagate(A0, 0.02, tol=1e-5, max_attempts=6)
    med = Argon(lam, 1.0, precision, True, lut=lut)
    sol = ERK43IP_UPPE_3D_Optimized(x, x, t, med, precision=precision)
    sol.set_field(A0)
    for z0, h, err_o, acc in log:
        err = sol.attempt(h)
        if precision == 'double':
            assert abs(err - err_o) <= 1e-8 * err_o + 1e-18
        else:   # FP32 fields: errors below ~1e-9 are rounding noise (tol is 1e-5)
            assert abs(err - err_o) <= 1e-3 * err_o + 1e-9
        sol.commit(acc)
    assert sol.result().status == 0
    assert rel_l2(sol.spectrum().cpu().numpy(), Ao) < (1e-10 if precision == 'double' else 1e-4)


@pytest.mark.parametrize('Nt,precision,W0', [(512, 'double', 3e9), (512, 'double', 1e15),
                                              (512, 'single', 3e9), (1024, 'single', 3e9)])
def test_long_lines_vs_oracle(Nt, precision, W0):
    """t-lines of 512 / 1024 samples (the register warp-FFT kernel): attempts from the
    oracle's schedule; W0 = 1e15 makes the density clamp bind (serial scan path)."""
    from project_b200.media import Argon
    from project_b200.solver3d import ERK43IP_UPPE_3D_Optimized
    x, t, lam, A0, osol, lut = _oracle_case(N=16, Nt=Nt, W0=W0, I_peak=5e16)
    z, freq, Ao, log = osol.propagate(A0, 0.01, tol=1e-5, max_attempts=4)
    med = Argon(lam, 1.0, precision, True, lut=lut)
    sol = ERK43IP_UPPE_3D_Optimized(x, x, t, med, precision=precision)
    sol.set_field(A0)
    for z0, h, err_o, acc in log:
        err = sol.attempt(h)
        if precision == 'double':
            assert abs(err - err_o) <= 1e-8 * err_o + 1e-18
        sol.commit(acc)
    tol = 1e-10 if precision == 'double' else 1e-4
    assert rel_l2(sol.spectrum().cpu().numpy(), Ao) < tol


@pytest.mark.parametrize('Nt,precision', [(512, 'single'), (1024, 'single'), (1024, 'double')])
def test_kerr_dominated_steps_vs_oracle(Nt, precision):
    """Steps whose change is mostly the Kerr term (1.8e16 W/m^2, 1.5 bar, w0 1 mm,
    h up to 2 mm): the nonlinear evaluation itself, including the 32-point register
    DFTs of the 1024-sample complex64 t-lines, must keep the per-step rounding
    level (complex64: rel-L2 ~3e-7 per step, a wrong transform shows as ~2e-5)."""
    from oracle import uppe3d
    from project_b200.media import Argon
    from project_b200.solver3d import ERK43IP_UPPE_3D_Optimized
    x = np.linspace(-2e-3, 2e-3, 32)
    t = np.linspace(-125e-15 * Nt / 512, 125e-15 * Nt / 512, Nt)
    lam = 800e-9
    om = uppe3d.argon(lam, 1.5, 'double', True)
    W = np.zeros_like(om.log10_I_cpu)
    om.W_gpu = W
    osol = uppe3d.Solver3D(x, x, t, om, 'double')
    X, Y = np.meshgrid(x, x, indexing='ij')
    T0 = 50e-15 / (2 * np.sqrt(np.log(2)))
    A0 = (np.sqrt(1.8e16) * np.exp(-(X ** 2 + Y ** 2) / 1e-6)[:, :, None]
          * np.exp(-(t / T0) ** 2 / 2)[None, None, :]).astype(np.complex128)
    osol.A_scale = float(np.max(np.abs(A0)))
    An = A0 / osol.A_scale
    sol = ERK43IP_UPPE_3D_Optimized(x, x, t, Argon(lam, 1.5, precision, True, lut=(om.log10_I_cpu, W)),
                                    precision=precision)
    sol.set_field(A0)
    for k, h in enumerate([2.5e-4, 5e-4, 1e-3, 2e-3]):
        An, err_o, _, _ = osol.erk43_step(An, h)
        sol.attempt(h)
        sol.commit(True)
        rel = rel_l2(sol.field().cpu().numpy() / osol.A_scale, An)
        assert rel < (1e-13 if precision == 'double' else 5e-7 * (k + 1)), (k, rel)


def test_diagnostics_vs_oracle():
    """Energy, photon number and peak ionisation fraction of a propagation with
    significant ionisation (MPI-like table), complex128, against the oracle."""
    from project_b200.media import Argon
    from project_b200.solver3d import ERK43IP_UPPE_3D_Optimized
    x, t, lam, A0, osol, lut = _oracle_case(N=16, Nt=64, W0=3e9, I_peak=5e16)
    z, freq, Ao, log = osol.propagate(A0, 0.01, tol=1e-5)
    # peak over the states at which steps started and the final state
    An = (A0 / osol.A_scale).astype(np.complex128)
    peak = osol.ionization_fraction(An)
    for z0, h, err, acc in log:
        if acc:
            An = osol.erk43_step(An, h)[0]
            peak = max(peak, osol.ionization_fraction(An))
    Eo, pho = osol.diagnostics(osol.last_state)
    sol = ERK43IP_UPPE_3D_Optimized(x, x, t, Argon(lam, 1.0, 'double', True, lut=lut), precision='double')
    sol.propagate(A0, 0.01, tol=1e-5)
    d = sol.diagnostics()
    assert peak > 1e-6
    assert abs(d['energy'] - Eo) <= 1e-10 * Eo
    assert abs(d['photons'] - pho) <= 1e-10 * pho
    assert abs(d['peak_ionization'] - peak) <= 1e-8 * peak


@pytest.mark.parametrize('precision,tol', [('double', 1e-10), ('single', 1e-4)])
def test_beam_diagnostics_vs_oracle(precision, tol):
    """sim.py:140-249 quantities from the device pass vs the oracle on the field."""
    from oracle.diagnostics import beam_diagnostics
    from project_b200.media import Argon
    from project_b200.solver3d import ERK43IP_UPPE_3D_Optimized
    x, t, lam, A0, osol, lut = _oracle_case(N=64, Nt=128)
    sol = ERK43IP_UPPE_3D_Optimized(x, x, t, Argon(lam, 1.0, precision, True, lut=lut), precision=precision)
    sol.propagate(A0, 0.01, tol=1e-5)
    d = sol.beam_diagnostics(w_mode=0.4e-3)
    A = sol.field().cpu().numpy().astype(np.complex128)
    o = beam_diagnostics(A, x, x, t, 0.4e-3, lam)
    for k in ('energy_total', 'x_mean_m', 'y_mean_m', 'wx_rms_m', 'wy_rms_m', 'fwhm_center_s', 'fwhm_smf_s'):
        scale = abs(o[k]) if k not in ('x_mean_m', 'y_mean_m') else o['wx_rms_m']
        assert abs(d[k] - o[k]) <= tol * scale + 1e-30, k
    for k in ('P_t', 'fluence', 'spec_smf', 'spec_full_incoh', 'spec_center', 'I_center_t', 'I_smf_t',
              'freq_abs_Hz'):
        assert rel_l2(d[k], o[k]) < tol, k
    assert d['it_peak'] == o['it_peak']


@pytest.mark.parametrize('precision', ['single', 'double'])
def test_state_continuation_is_bit_exact(precision):
    """save_state after a few attempts, load_state into a new plan, resume: the same
    attempts, step sizes, field and diagnostics as the uninterrupted run."""
    import torch
    from project_b200 import _lib
    from project_b200.media import Argon
    from project_b200.solver3d import ERK43IP_UPPE_3D_Optimized
    x, t, lam, A0, osol, lut = _oracle_case(N=32, Nt=64, W0=3e9, I_peak=5e16)
    mk = lambda: ERK43IP_UPPE_3D_Optimized(x, x, t, Argon(lam, 1.0, precision, True, lut=lut), precision=precision)
    L, tol = 0.02, 1e-5
    s1 = mk()
    z, _, Aref = s1.propagate(A0, L, tol=tol, return_gpu=True)
    r1 = s1.last_result
    s2 = mk()
    s2.set_field(A0)
    st = _lib.stream_ptr()
    _lib.check(s2._lib.uppe3d_begin(s2._plan, L, tol, 1e-2, 1e-9, 0, st), 'uppe3d_begin')
    _lib.check(s2._lib.uppe3d_run_steps(s2._plan, 5, st), 'uppe3d_run_steps')
    saved = s2.save_state()
    assert 0.0 < saved['state']['z'] < L and saved['state']['done'] == 0
    assert saved['state']['attempts'] == 5
    s3 = mk()
    s3.load_state(saved)
    z3, _, A3 = s3.resume(return_gpu=True)
    r3 = s3.last_result
    assert z3 == z and r3.attempts == r1.attempts and r3.accepted == r1.accepted and r3.status == r1.status
    assert r3.h == r1.h
    assert torch.equal(A3, Aref)
    assert s3.diagnostics()['peak_ionization'] == s1.diagnostics()['peak_ionization']
