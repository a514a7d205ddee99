"""Device adjoint of the 1D propagation vs a complex128 torch autograd reference
and vs central finite differences of the frozen-schedule forward map (GPU)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _case(Nt=1024, E=40e-6):
    import torch
    from oracle.inputs import gaussian_pulse
    from project_b200.adjoint import CapillaryCompression
    t = np.linspace(-0.5e-12, 0.5e-12, Nt)
    A0 = gaussian_pulse(t, E, 30e-15)
    cc = CapillaryCompression(t, A0, n_knots=16)
    return cc


def test_adjoint_matches_torch_autograd_reference():
    import torch
    import torch_ref1d
    from project_b200.adjoint import Propagate1D, propagate_1d
    cc = _case()
    rng = np.random.Generator(np.random.PCG64(7))
    knots = torch.tensor(rng.normal(0, 0.3, 16), dtype=torch.float64, device='cuda', requires_grad=True)
    P = torch.tensor(1.3, dtype=torch.float64, device='cuda', requires_grad=True)
    D, G = cc.tables(P)
    A0 = cc.input_field(knots)
    w = torch.from_numpy(rng.uniform(0.5, 1.5, cc.N)).cuda()
    A_L = propagate_1d(A0, D, G, 0.05, cc.template, cc.t, tol=1e-6)
    loss = (w * (A_L.real ** 2 + A_L.imag ** 2) ** 2).sum()
    gk, gP = torch.autograd.grad(loss, [knots, P])
    hs = Propagate1D.last_steps
    assert len(hs) > 3
    # reference: same frozen steps in torch autograd
    knots2 = knots.detach().clone().requires_grad_(True)
    P2 = P.detach().clone().requires_grad_(True)
    D2, G2 = cc.tables(P2)
    A_L2 = torch_ref1d.propagate(cc.input_field(knots2), D2, G2, hs)
    assert float((A_L2.detach() - A_L.detach()).abs().max() / A_L.detach().abs().max()) < 1e-10
    loss2 = (w * (A_L2.real ** 2 + A_L2.imag ** 2) ** 2).sum()
    gk2, gP2 = torch.autograd.grad(loss2, [knots2, P2])
    assert float((gk - gk2).norm() / gk2.norm()) < 1e-8
    assert abs(float(gP - gP2)) <= 1e-8 * abs(float(gP2))


def test_compression_gradients_vs_central_differences():
    """knots, pressure and length of the capillary-compression objective; the
    forward map for the differences replays the frozen step sequence (scaled
    for the length)."""
    import torch
    from project_b200.adjoint import Propagate1D, replay_1d
    cc = _case(E=60e-6)
    rng = np.random.Generator(np.random.PCG64(8))
    k0 = rng.normal(0, 0.2, 16)
    knots = torch.tensor(k0, dtype=torch.float64, device='cuda', requires_grad=True)
    P = torch.tensor(1.0, dtype=torch.float64, device='cuda', requires_grad=True)
    L = torch.tensor(0.2, dtype=torch.float64, requires_grad=True)
    loss = cc.loss(knots, P, L, tol=1e-7)
    gk, gP, gL = torch.autograd.grad(loss, [knots, P, L])
    hs = np.array(Propagate1D.last_steps)

    def f(kn, Pv, Lv):
        kt = torch.tensor(kn, dtype=torch.float64, device='cuda')
        D, G = cc.tables(torch.tensor(Pv, dtype=torch.float64, device='cuda'))
        A_L = replay_1d(cc.input_field(kt), D, G, cc.template, cc.t, hs * (Lv / 0.2))
        tl = torch.fft.ifft(torch.fft.fft(A_L).abs())
        return -float((tl.real ** 2 + tl.imag ** 2).max())

    eps = 1e-4
    for j in (3, 8, 12):
        kp, km = k0.copy(), k0.copy()
        kp[j] += eps
        km[j] -= eps
        fd = (f(kp, 1.0, 0.2) - f(km, 1.0, 0.2)) / (2 * eps)
        assert abs(fd - float(gk[j])) <= 1e-4 * max(abs(fd), 1e-3 * float(gk.abs().max()))
    fdP = (f(k0, 1.0 + eps, 0.2) - f(k0, 1.0 - eps, 0.2)) / (2 * eps)
    assert abs(fdP - float(gP)) <= 1e-4 * abs(fdP)
    fdL = (f(k0, 1.0, 0.2 * (1 + eps)) - f(k0, 1.0, 0.2 * (1 - eps))) / (2 * 0.2 * eps)
    assert abs(fdL - float(gL)) <= 1e-4 * abs(fdL)


def _plasma_case(Nt=1024, E=40e-6, W0=3e9):
    """Capillary with the plasma term; MPI-like test table W = W0 (I / 5e16 W/m^2)^8
    so that the term matters at these energies (no density clamp binds)."""
    from oracle.inputs import gaussian_pulse
    from project_b200.adjoint import CapillaryCompression
    t = np.linspace(-0.5e-12, 0.5e-12, Nt)
    A0 = gaussian_pulse(t, E, 30e-15)
    x = np.linspace(np.log10(1e8 * 1e4), np.log10(1e16 * 1e4), 2000)
    W = np.minimum(W0 * (10.0 ** x / 5e16) ** 8, 1e20)
    return CapillaryCompression(t, A0, n_knots=16, plasma=True, lut=(x, W))


def _torch_plasma(cc, P):
    import torch
    pp = cc.plasma_params(P)
    return dict(lx=torch.from_numpy(cc.plasma.lut[0]).cuda(), lw=torch.from_numpy(cc.plasma.lut[1]).cuda(),
                Ui=cc.plasma.Ui, rr=1.0 / cc.plasma.tau_rec, dt=float(cc.t[1] - cc.t[0]),
                rho_nt=pp[0], sigma=pp[1], w0tc=pp[2], A_eff=cc.A_eff)


def test_adjoint_plasma_matches_torch_autograd_reference():
    import torch
    import torch_ref1d
    from project_b200.adjoint import Propagate1D, propagate_1d
    cc = _plasma_case()
    rng = np.random.Generator(np.random.PCG64(7))
    knots = torch.tensor(rng.normal(0, 0.3, 16), dtype=torch.float64, device='cuda', requires_grad=True)
    P = torch.tensor(1.3, dtype=torch.float64, device='cuda', requires_grad=True)
    D, G = cc.tables(P)
    w = torch.from_numpy(rng.uniform(0.5, 1.5, cc.N)).cuda()
    A_L = propagate_1d(cc.input_field(knots), D, G, 0.05, cc.template, cc.t, tol=1e-6,
                       plasma_par=cc.plasma_params(P))
    loss = (w * (A_L.real ** 2 + A_L.imag ** 2) ** 2).sum()
    gk, gP = torch.autograd.grad(loss, [knots, P])
    hs = Propagate1D.last_steps
    knots2 = knots.detach().clone().requires_grad_(True)
    P2 = P.detach().clone().requires_grad_(True)
    D2, G2 = cc.tables(P2)
    A_L2 = torch_ref1d.propagate(cc.input_field(knots2), D2, G2, hs, _torch_plasma(cc, P2))
    assert float((A_L2.detach() - A_L.detach()).abs().max() / A_L.detach().abs().max()) < 1e-10
    loss2 = (w * (A_L2.real ** 2 + A_L2.imag ** 2) ** 2).sum()
    gk2, gP2 = torch.autograd.grad(loss2, [knots2, P2])
    assert float((gk - gk2).norm() / gk2.norm()) < 1e-8
    assert abs(float(gP - gP2)) <= 1e-8 * abs(float(gP2))
    # the plasma term matters for these gradients
    knots3 = knots.detach().clone().requires_grad_(True)
    A_L3 = torch_ref1d.propagate(cc.input_field(knots3), D2.detach(), G2.detach(), hs)
    gk3, = torch.autograd.grad((w * (A_L3.real ** 2 + A_L3.imag ** 2) ** 2).sum(), [knots3])
    assert float((gk3 - gk2).norm() / gk2.norm()) > 1e-2


def test_compression_gradients_with_plasma_vs_central_differences():
    """As above with the plasma term (pressure also scales rho_nt and 1/tau_c)."""
    import torch
    from project_b200.adjoint import Propagate1D, replay_1d
    cc = _plasma_case(W0=1e9)
    rng = np.random.Generator(np.random.PCG64(8))
    k0 = rng.normal(0, 0.2, 16)
    knots = torch.tensor(k0, dtype=torch.float64, device='cuda', requires_grad=True)
    P = torch.tensor(1.0, dtype=torch.float64, device='cuda', requires_grad=True)
    L = torch.tensor(0.2, dtype=torch.float64, requires_grad=True)
    loss = cc.loss(knots, P, L, tol=1e-7)
    gk, gP, gL = torch.autograd.grad(loss, [knots, P, L])
    hs = np.array(Propagate1D.last_steps)

    def f(kn, Pv, Lv):
        kt = torch.tensor(kn, dtype=torch.float64, device='cuda')
        Pt = torch.tensor(Pv, dtype=torch.float64, device='cuda')
        D, G = cc.tables(Pt)
        A_L = replay_1d(cc.input_field(kt), D, G, cc.template, cc.t, hs * (Lv / 0.2), cc.plasma_params(Pt))
        tl = torch.fft.ifft(torch.fft.fft(A_L).abs())
        return -float((tl.real ** 2 + tl.imag ** 2).max())

    # The rates are rounded to float32 (media_physics.py:169), so the forward map is
    # piecewise constant at the 6e-8 level in W, and the table is piecewise linear
    # in log10(I): differences carry noise ~ulp(W)/dW that grows as the step shrinks.
    # Larger steps and a 1e-3 bound here; the exact check is the autograd test above.
    eps = 1e-3
    for j in (3, 8, 12):
        kp, km = k0.copy(), k0.copy()
        kp[j] += eps
        km[j] -= eps
        fd = (f(kp, 1.0, 0.2) - f(km, 1.0, 0.2)) / (2 * eps)
        assert abs(fd - float(gk[j])) <= 1e-3 * max(abs(fd), 1e-3 * float(gk.abs().max()))
    fdP = (f(k0, 1.0 + eps, 0.2) - f(k0, 1.0 - eps, 0.2)) / (2 * eps)
    assert abs(fdP - float(gP)) <= 1e-3 * abs(fdP)
    fdL = (f(k0, 1.0, 0.2 * (1 + eps)) - f(k0, 1.0, 0.2 * (1 - eps))) / (2 * 0.2 * eps)
    assert abs(fdL - float(gL)) <= 1e-3 * abs(fdL)
