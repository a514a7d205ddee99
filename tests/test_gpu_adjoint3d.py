"""Device adjoint of the 3+1D propagation vs a complex128 torch autograd reference
and vs central differences of the frozen-schedule forward map (GPU)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _setup(N=16, Nt=64, precision='double', energy=2.0e-4, plasma=False, W0=1e9):
    """Argon at 1.5 bar; with ``plasma`` an MPI-like test table W = W0 (I / 4e15 W/m^2)^8
    (shared by the device medium and the oracle medium) makes the plasma terms
    matter at these energies."""
    from oracle import uppe3d
    from project_b200.adjoint import FilamentZernike
    from project_b200.media import Argon
    from project_b200.solver3d import ERK43IP_UPPE_3D_Optimized
    x = np.linspace(-2e-3, 2e-3, N)
    t = np.linspace(-150e-15, 150e-15, Nt)
    om = uppe3d.argon(800e-9, 1.5, 'double', True)
    lut = None
    if plasma:
        W = np.minimum(W0 * (10.0 ** om.log10_I_cpu / 4e15) ** 8, 1e20)
        om.W_gpu = W
        lut = (om.log10_I_cpu, W)
    med = Argon(800e-9, 1.5, precision, True, lut=lut)
    if not plasma:
        med.plasma = False
    sol = ERK43IP_UPPE_3D_Optimized(x, x, t, med, precision=precision)
    obj = FilamentZernike(sol, w0=0.8e-3, energy=energy, fwhm=50e-15, aperture_radius=2e-3)
    osol = uppe3d.Solver3D(x, x, t, om, 'double')
    return sol, obj, osol


@pytest.mark.parametrize('plasma', [False, True])
def test_adjoint3d_matches_torch_autograd_reference(plasma):
    import torch
    import torch_ref3d
    from project_b200.adjoint import Propagate3D, propagate_3d
    sol, obj, osol = _setup(plasma=plasma)
    rng = np.random.Generator(np.random.PCG64(4))
    c = torch.tensor(rng.normal(0, 0.1, 15), dtype=torch.float64, device='cuda', requires_grad=True)
    gdd = torch.tensor(200e-30, dtype=torch.float64, device='cuda', requires_grad=True)
    A0 = obj.input_field(c, gdd)
    w = torch.from_numpy(rng.uniform(0.5, 1.5, (16, 16, 64))).cuda()
    A = propagate_3d(A0, sol, 0.05, tol=1e-5)
    loss = (w * (A.real ** 2 + A.imag ** 2) ** 2).sum()
    gc, gg = torch.autograd.grad(loss, [c, gdd])
    hs = Propagate3D.last_steps
    assert len(hs) > 2
    c2 = c.detach().clone().requires_grad_(True)
    g2 = gdd.detach().clone().requires_grad_(True)
    A2 = torch_ref3d.propagate(obj.input_field(c2, g2), hs, torch_ref3d.make(osol, plasma))
    assert float((A2.detach() - A.detach()).abs().max() / A.detach().abs().max()) < 1e-10
    loss2 = (w * (A2.real ** 2 + A2.imag ** 2) ** 2).sum()
    gc2, gg2 = torch.autograd.grad(loss2, [c2, g2])
    assert float((gc - gc2).norm() / gc2.norm()) < 1e-8
    assert abs(float(gg - gg2)) <= 1e-8 * abs(float(gg2))
    if plasma:   # the plasma terms matter for these gradients
        c3 = c.detach().clone().requires_grad_(True)
        A3 = torch_ref3d.propagate(obj.input_field(c3, gdd.detach()), hs, torch_ref3d.make(osol, False))
        gc3, = torch.autograd.grad((w * (A3.real ** 2 + A3.imag ** 2) ** 2).sum(), [c3])
        assert float((gc3 - gc2).norm() / gc2.norm()) > 1e-2


def _filament_grad(precision, N=32, Nt=64, L=0.1, plasma=False):
    import torch
    from project_b200.adjoint import Propagate3D
    sol, obj, _ = _setup(N=N, Nt=Nt, precision=precision, energy=4e-4, plasma=plasma)
    rng = np.random.Generator(np.random.PCG64(4))
    c0 = rng.normal(0, 0.1, 15)
    c = torch.tensor(c0, dtype=torch.float64, device='cuda', requires_grad=True)
    gdd = torch.tensor(100e-30, dtype=torch.float64, device='cuda', requires_grad=True)
    loss = obj.loss(c, gdd, L, tol=1e-5)
    gc, gg = torch.autograd.grad(loss, [c, gdd])
    return sol, obj, c0, gc.cpu().numpy(), float(gg), np.array(Propagate3D.last_steps)


@pytest.mark.parametrize('plasma', [False, True])
def test_filament_gradients_vs_central_differences(plasma):
    import torch
    sol, obj, c0, gc, gg, hs = _filament_grad('double', plasma=plasma)

    def f(cv, gv):
        A0 = obj.input_field(torch.tensor(cv, dtype=torch.float64, device='cuda'),
                             torch.tensor(gv, dtype=torch.float64, device='cuda'))
        A = sol.replay(A0.to(sol.complex_dtype), hs)
        a = A[obj.ix, obj.iy, :].to(torch.complex128)
        return -float((a.real ** 2 + a.imag ** 2).sum()) * sol.dt

    eps = 1e-3
    for j in (3, 5, 11):
        cp, cm = c0.copy(), c0.copy()
        cp[j] += eps
        cm[j] -= eps
        fd = (f(cp, 100e-30) - f(cm, 100e-30)) / (2 * eps)
        assert abs(fd - gc[j]) <= 1e-4 * max(abs(fd), 1e-2 * np.abs(gc).max())
    eg = 5e-30
    fdg = (f(c0, 100e-30 + eg) - f(c0, 100e-30 - eg)) / (2 * eg)
    assert abs(fdg - gg) <= 1e-4 * abs(fdg)


@pytest.mark.parametrize('plasma', [False, True])
def test_filament_gradients_mixed_vs_fp64(plasma):
    """Mixed precision (complex64 bulk): the adjoint of the complex64 forward map
    against the FP64 gradient (each with its own free-running schedule)."""
    _, _, _, gd, ggd, _ = _filament_grad('double', plasma=plasma)
    _, _, _, gs, ggs, _ = _filament_grad('single', plasma=plasma)
    rc = np.linalg.norm(gs - gd) / np.linalg.norm(gd)
    rg = abs(ggs - ggd) / abs(ggd)
    print('mixed vs fp64 gradient: coeffs %.3e  gdd %.3e' % (rc, rg))
    assert rc < 1e-3 and rg < 1e-3
