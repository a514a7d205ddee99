"""Mixed precision against complex128 at the full 256x256x512 workload (GPU).

The configured 3+1D run (argon 1 bar with GVD 20 fs^2/m, ADK plasma and
self-steepening; 6 mm x 400 fs; 2 mJ, 40 fs, w0 = 1 mm, 1 % speckle) propagated
over the same accepted steps in both precisions: the mixed path (complex64 bulk;
FP64 interaction-picture phase, density scan, error norm and controller), on the
kernels the bench times, against the complex128 device path, which the other
tests pin to the reference at small sizes (reference path solver_3d.py:100-160).
Bar: field rel-L2 <= 1e-4 (the step's tolerance in the mixed path), energy and
photon number to 1e-5, peak ionisation to 1e-2 relative.
"""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

N, NT = 256, 512


def _setup(precision):
    from project_b200.media import Argon
    from project_b200.pulses import gaussian_beam, speckle
    x = np.linspace(-3e-3, 3e-3, N)
    t = np.linspace(-200e-15, 200e-15, NT)
    m0 = Argon(800e-9, 1.0, precision, True)
    n0 = float(m0.refractive_index(np.array([m0.omega0]))[0])
    med = Argon(800e-9, 1.0, precision, True, dispersion=('taylor', n0, 20e-30, 0.0))
    A0 = gaussian_beam(x, x, t, 1e-3, 2e-3, 40e-15) * speckle(x, x, 50e-6, 0.01, seed=1)[:, :, None]
    return x, t, med, A0


def test_mixed_vs_complex128_at_256x256x512():
    import torch
    from project_b200.solver3d import ERK43IP_UPPE_3D_Optimized
    # the first steps of the configured run: h grows from L/1000 = 2 mm by the
    # controller's factors; 12 accepted steps reach 0.1 m
    steps = [2e-3, 2.4e-3, 2.88e-3, 3.456e-3, 4.147e-3, 4.977e-3, 5.972e-3, 7.166e-3, 8.6e-3, 1e-2, 1e-2, 1e-2]
    x, t, med32, A0 = _setup('single')
    s32 = ERK43IP_UPPE_3D_Optimized(x, x, t, med32, precision='single')
    A32 = s32.replay(A0.astype(np.complex64), steps).cpu().numpy()
    d32 = s32.diagnostics()
    del s32
    torch.cuda.empty_cache()
    _, _, med64, _ = _setup('double')
    s64 = ERK43IP_UPPE_3D_Optimized(x, x, t, med64, precision='double')
    A64 = s64.replay(A0.astype(np.complex128), steps).cpu().numpy()
    d64 = s64.diagnostics()
    del s64
    torch.cuda.empty_cache()
    rel = rel_l2(A32, A64)
    assert rel < 1e-4, rel
    assert abs(d32['energy'] - d64['energy']) <= 1e-5 * d64['energy']
    assert abs(d32['photons'] - d64['photons']) <= 1e-5 * d64['photons']
    if d64['peak_ionization'] > 0:
        assert abs(d32['peak_ionization'] - d64['peak_ionization']) <= 1e-2 * d64['peak_ionization']
