"""Failure statuses of the device loops (GPU), every failure injected from the host.

The reference prints warnings, forces steps at min_step
(src/1D-ERK4(3)IP UPPE gas/erk43ip_method.py:345-367; solver_3d.py:190-191) and
never terminates once its error turns NaN.  Here every device loop is bounded and
reports UPPE_STATUS_* bits: an attempt that comes out non-finite is rejected and
retried with a tenth of the step (RETRIED) and the run stops once that happens at
min_step (NONFINITE); a step forced at min_step with err > tol is flagged
(MIN_STEP), and the attempt budget ends a run early (MAX_ATTEMPTS).
Nothing here faults or hangs a GPU: the inputs are finite-size host arrays with a
NaN or an overflowing Kerr coefficient.
"""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

NONFINITE, MIN_STEP, MAX_ATTEMPTS, RETRIED = 1, 2, 4, 64


def _grid3d():
    x = np.linspace(-1.5e-3, 1.5e-3, 32)
    t = np.linspace(-100e-15, 100e-15, 64)
    return x, x.copy(), t


def _beam(x, y, t, peak=5e16):
    X, Y = np.meshgrid(x, y, indexing='ij')
    T0 = 40e-15 / (2 * np.sqrt(np.log(2)))
    return (np.sqrt(peak) * np.exp(-(X ** 2 + Y ** 2) / 0.25e-6)[:, :, None]
            * np.exp(-(t / T0) ** 2 / 2)[None, None, :]).astype(np.complex128)


def _solver3d(precision, n2=None):
    from project_b200.media import Argon
    from project_b200.solver3d import ERK43IP_UPPE_3D_Optimized
    x, y, t = _grid3d()
    m = Argon(800e-9, 1.0, precision, True)
    if n2 is not None:
        m.n2 = n2
    return ERK43IP_UPPE_3D_Optimized(x, y, t, m, precision=precision), (x, y, t)


@pytest.mark.parametrize('precision', ['double', 'single'])
def test_3d_nan_input_stops_with_nonfinite(precision):
    sol, (x, y, t) = _solver3d(precision)
    A0 = _beam(x, y, t)
    A0[5, 7, 11] = np.nan
    z, _, _ = sol.propagate(A0, 0.05, tol=1e-5, max_attempts=1000)
    r = sol.last_result
    # every attempt from a NaN state is NaN: h falls by 10 per attempt from
    # L/1000 = 5e-5 to min_step = 1e-9, then the run stops
    assert r.status == NONFINITE | RETRIED
    assert r.attempts <= 7 and r.accepted == 0 and z == 0.0


@pytest.mark.parametrize('precision,n2', [('double', 1e290), ('single', 1e20)])
def test_3d_overflowing_kerr_stops_with_nonfinite(precision, n2):
    """gamma I beyond the field precision's range: the Kerr term overflows, the
    transforms turn it into NaN, the run stops instead of looping on h = NaN."""
    sol, (x, y, t) = _solver3d(precision, n2=n2)
    sol.propagate(_beam(x, y, t), 0.05, tol=1e-5, max_attempts=1000)
    r = sol.last_result
    assert r.status == NONFINITE | RETRIED
    assert r.attempts <= 7


def test_3d_attempt_budget():
    sol, (x, y, t) = _solver3d('single')
    z, _, _ = sol.propagate(_beam(x, y, t), 0.05, tol=1e-5, max_attempts=3)
    r = sol.last_result
    assert r.status == MAX_ATTEMPTS
    assert r.attempts == 3 and z < 0.05


def test_3d_forced_steps_at_min_step_are_flagged_and_bounded():
    """min_step = max_step with an unreachable tolerance: as in the reference
    (solver_3d.py:190-203), every step at h <= 1.01 min_step is accepted and the
    controller keeps shrinking h, so z never reaches L; the flag is set on the
    first forced step and the attempt budget ends the run with a finite field."""
    sol, (x, y, t) = _solver3d('double', n2=1e-19)     # ~40 rad of Kerr phase per mm
    z, _, A = sol.propagate(_beam(x, y, t), 0.004, tol=1e-14, max_step=1e-3, min_step=1e-3,
                            max_attempts=40)
    r = sol.last_result
    assert r.status == MIN_STEP | MAX_ATTEMPTS
    assert r.accepted == r.attempts == 40
    assert 0.0 < z < 0.004
    assert np.all(np.isfinite(A))


def _argon1d(precision, **kw):
    from project_b200.solver1d import ERK43IP_UPPE
    return ERK43IP_UPPE(material='argon_gas', n2=kw.pop('n2', 1.0e-23), beam_radius=0.65 * 125e-6,
                        center_wavelength=800e-9, alpha=0.11513, use_raman=False,
                        taylor=(15e-30, 15e-45), precision=precision, **kw)


def _pulse1d(Nt=1024):
    from oracle.inputs import gaussian_pulse
    t = np.linspace(-0.5e-12, 0.5e-12, Nt)
    fw = 30e-15
    return t, gaussian_pulse(t, 2e9 * fw * np.sqrt(np.pi / (4 * np.log(2))), fw)


@pytest.mark.parametrize('precision', ['double', 'single'])
def test_1d_nan_input_stops_with_nonfinite(precision):
    s = _argon1d(precision)
    t, A0 = _pulse1d()
    A0[100] = np.nan
    s.propagate(A0, t, 0.1, tol=1e-6, max_attempts=1000)
    # h falls by 10 per attempt from max_step/100 = 1e-4 to min_step = 1e-11
    assert s.last_result.status == NONFINITE | RETRIED
    assert s.last_result.attempts <= 9 and s.last_result.accepted == 0


@pytest.mark.parametrize('precision,n2', [('double', 1e290), ('single', 1e20)])
def test_1d_overflowing_kerr_stops_with_nonfinite(precision, n2):
    s = _argon1d(precision, n2=n2)
    t, A0 = _pulse1d()
    s.propagate(A0, t, 0.1, tol=1e-6, max_attempts=1000)
    assert s.last_result.status == NONFINITE | RETRIED
    assert s.last_result.attempts <= 9


def test_1d_attempt_budget_and_forced_steps_in_one_batch():
    """Three instances in one launch: normal, budget-limited, forced at min_step.
    Each gets its own status; the normal one matches its solo run."""
    from project_b200.solver1d import BatchedPropagator
    s = _argon1d('double')
    sk = _argon1d('double', n2=1e-21)          # ~0.8 rad of Kerr phase per millimetre
    t, A0 = _pulse1d()
    insts = [s.instance(t, 0.05, tol=1e-6),
             s.instance(t, 0.05, tol=1e-6, max_attempts=3),
             sk.instance(t, 0.004, tol=1e-12, max_step=1e-3, min_step=1e-3, max_attempts=100)]
    finals, _, res = BatchedPropagator(insts, precision='double').run([A0, A0, A0])
    assert res[0].status == 0
    assert res[1].status == MAX_ATTEMPTS and res[1].attempts == 3 and res[1].z < 0.05
    assert res[2].status == MIN_STEP and res[2].z >= 0.004 - 1e-12   # :345-367 forced steps reach L
    assert np.all(np.isfinite(finals[2]))
    solo, _, r0 = BatchedPropagator(insts[:1], precision='double').run([A0])
    assert r0[0].attempts == res[0].attempts
    assert rel_l2(finals[0], solo[0]) < 1e-14


def test_realfield_nan_input_raises():
    """The real-field loop runs on the host and raises on a non-finite error."""
    import torch
    from project_b200.realfield import Argon, ERK43_RealField_UPPE_3D
    N, Nt = 16, 128
    x = np.linspace(-0.4e-3, 0.4e-3, N)
    t = np.linspace(-100e-15, 100e-15, Nt)
    E0 = np.zeros((N, N, Nt), dtype=np.float32)
    E0[:, :, Nt // 2] = 1e9
    E0[3, 4, 5] = np.nan
    sol = ERK43_RealField_UPPE_3D(x, x, t, Argon(800e-9, 1.0), precision='single')
    with pytest.raises(FloatingPointError):
        sol.propagate(torch.from_numpy(E0), 1e-4, tol=1e-4, max_attempts=50)
