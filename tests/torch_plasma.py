"""complex128 torch restatement of the plasma term (media_physics.py:11-67 and
:156-203, avalanche off) for the autograd references.  The density recurrence
rho_{t+1} = rho_t (e - W_t sf) + W_t rho_nt sf is summed in closed form with
cumulative sums (valid while no clamp of the reference update binds, which
``density`` asserts).  Test infrastructure."""
import numpy as np
import torch


def f32(x):
    """Round to float32 and back, keeping the derivative of the identity."""
    if torch.is_tensor(x):
        return x + (x.to(torch.float32).to(torch.float64) - x).detach()
    return float(np.float32(x))


def lut_rate(I, lx, lw):
    """Linear interpolation in log10(I + 1e-30), clipped to the table (float32-rounded)."""
    x = torch.clamp(torch.log10(I + 1e-30), float(lx[0]), float(lx[-1]))
    j = (torch.searchsorted(lx, x.detach().contiguous(), right=True) - 1).clamp(0, len(lx) - 2)
    x0, x1, w0, w1 = lx[j], lx[j + 1], lw[j], lw[j + 1]
    return f32(w0 + (w1 - w0) / (x1 - x0) * (x - x0))


def density(W, rho_nt, rr, dt):
    """rho_t (density before sample t) along the last axis."""
    gdt = max(min(-rr * dt, 10.0), -10.0)
    e = np.exp(gdt)
    sf = dt * (1.0 + 0.5 * gdt) if abs(gdt) < 1e-5 else (e - 1.0) / (-rr)
    c = e - W * sf
    d = W * rho_nt * sf
    Lc = torch.cumsum(torch.log(c), -1)
    S = torch.cumsum(d * torch.exp(-Lc), -1)
    rho = torch.cat([torch.zeros_like(W[..., :1]), torch.exp(Lc[..., :-1]) * S[..., :-1]], -1)
    assert float(rho.detach().max()) < float(rho_nt.detach() if torch.is_tensor(rho_nt) else rho_nt)
    assert float(c.detach().min()) > 0
    return rho


def term(a, I, pl):
    """Plasma_t = (-gen Ui / (2 I + 1e-30) - sigma/2 (1 + i omega0 tau_c) rho) a.
    pl: dict with lx, lw (tables), Ui, rr, dt and rho_nt, sigma, w0tc (tensors)."""
    rho_nt = f32(pl['rho_nt'])
    W = lut_rate(I, pl['lx'], pl['lw'])
    rho = density(W, rho_nt, f32(pl['rr']), f32(pl['dt']))
    gen = W * rho_nt * ((rho_nt - rho) / rho_nt)
    loss = -(gen * pl['Ui']) / (2.0 * I + 1e-30)
    c = loss - (pl['sigma'] / 2) * (1.0 + 1j * pl['w0tc']) * rho
    return c * a, rho
