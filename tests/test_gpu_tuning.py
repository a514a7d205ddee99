"""Per-shape launch tuner of the 3+1D plan (GPU).

uppe3d_plan_create times the candidate launch configurations of the y passes
(TMA-fed kernel with tiles of 16 or 8 omega columns, early or late operand loads
and one to six CTAs per SM; for Ny = 256 also the register four-step kernels, with
plain loads or with every operand tile on a TMA ring) and
of the warp t-line kernel (four or eight lines per block) and keeps the fastest.  The
candidates are chosen so that they compute the same bits: these tests force each
one and compare the propagated fields bit for bit (the plain tile kernel, which
rounds differently, is used only where the TMA path is unavailable).
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _setup(precision='single', n=64, nt=512):
    from project_b200.media import Argon
    x = np.linspace(-1.5e-3, 1.5e-3, n)
    t = np.linspace(-100e-15, 100e-15, nt)
    X, Y = np.meshgrid(x, x, indexing='ij')
    T0 = 40e-15 / (2 * np.sqrt(np.log(2)))
    A0 = (np.sqrt(1e17) * np.exp(-(X ** 2 + Y ** 2) / 0.25e-6)[:, :, None]
          * np.exp(-(t / T0) ** 2 / 2)[None, None, :])
    lx = np.linspace(np.log10(1e12), np.log10(1e20), 2000)
    W = np.minimum(3e9 * (10.0 ** lx / 5e16) ** 8, 1e20)      # ionises at this peak intensity
    med = Argon(800e-9, 1.0, precision, True, lut=(lx, W))
    return x, t, med, A0


def _tuning(sol):
    from project_b200 import _lib
    cfg = (ctypes.c_int * 6)()
    ms = (ctypes.c_float * _lib.UPPE3D_TUNE_SLOTS)()
    _lib.check(sol._lib.uppe3d_tuning(sol._plan, cfg, ms), 'uppe3d_tuning')
    return list(cfg), list(ms)


YCANDS = [(1, 2, 0, 16), (1, 1, 0, 16), (1, 3, 1, 16), (1, 2, 1, 16), (1, 4, 0, 8), (1, 6, 1, 8)]
YCANDS_256 = YCANDS + [(2, 2, 0, 16), (2, 3, 1, 16), (3, 1, 0, 16), (2, 4, 0, 8), (2, 6, 1, 8)]   # + register 4-step


@pytest.mark.parametrize('n,nt', [(64, 512), (256, 128), (256, 512)])
def test_tuner_runs_and_every_candidate_gives_identical_fields(n, nt):
    import torch
    from project_b200 import _lib
    from project_b200.solver3d import ERK43IP_UPPE_3D_Optimized
    x, t, med, A0 = _setup(n=n, nt=nt)
    sol = ERK43IP_UPPE_3D_Optimized(x, x, t, med, precision='single')
    cfg, ms = _tuning(sol)
    assert cfg[5] in (1, 2)                       # timed here or taken from the process cache
    assert cfg[0] in (1, 2, 3) and 1 <= cfg[1] <= 6 and cfg[3] in (8, 16) and cfg[4] in (4, 8)
    ycands = YCANDS_256 if n == 256 else YCANDS
    if cfg[5] == 1:
        assert all(v > 0 for v in ms[:len(ycands)]) and ms[11] > 0
    if n != 256:
        assert cfg[0] == 1 and all(v == 0 for v in ms[6:11])
        assert sol._lib.uppe3d_set_tuning(sol._plan, 2, 2, 0, 16, 8) == -1   # Ny = 256 only
        assert sol._lib.uppe3d_set_tuning(sol._plan, 3, 2, 0, 16, 8) == -1
    ref = None
    for y_tma, y_ctas, y_late, y_kw in ycands:
        for wpb in ((4, 8) if nt == 512 else (8,)):
            _lib.check(sol._lib.uppe3d_set_tuning(sol._plan, y_tma, y_ctas, y_late, y_kw, wpb),
                       'uppe3d_set_tuning')
            assert _tuning(sol)[0][:5] == [y_tma, y_ctas, y_late, y_kw, wpb]
            z, _, A = sol.propagate(A0.astype(np.complex64), 0.02, tol=1e-4, return_gpu=True)
            assert sol.last_result.status == 0
            if ref is None:
                ref = (z, sol.last_result.attempts, A.clone(), sol.diagnostics()['peak_ionization'])
                assert ref[3] > 0                    # the plasma path ran
            else:
                assert z == ref[0] and sol.last_result.attempts == ref[1]
                assert torch.equal(A, ref[2]), (y_tma, y_ctas, y_late, y_kw, wpb)


def test_tuner_can_be_switched_off(monkeypatch):
    from project_b200.solver3d import ERK43IP_UPPE_3D_Optimized
    x, t, med, _ = _setup(n=32, nt=256)
    monkeypatch.setenv('UPPE_TUNE', '0')
    sol = ERK43IP_UPPE_3D_Optimized(x, x, t, med, precision='single')
    cfg, ms = _tuning(sol)
    assert cfg[5] == 0 and cfg[4] == 8
    assert all(v == 0 for v in ms)
