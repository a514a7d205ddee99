"""complex128 torch restatement of the 3+1D ERK4(3)-IP step in the (kx, ky, omega)
domain (solver_3d.py:100-160: Kerr + self-steepening, and the plasma term of
media_physics.py:156-203 when the medium has one), frozen step sequence;
autograd reference for the device adjoint.  Test infrastructure."""
import numpy as np
import torch

import torch_plasma


def make(osol, plasma=False):
    dev = 'cuda'
    D = torch.from_numpy(osol.D_operator).to(dev)
    mask = torch.from_numpy(osol.valid_freq_mask.astype('float64')).to(dev)
    shock = torch.from_numpy(osol.shock_operator.real.astype('float64')).to(dev)
    filt = torch.from_numpy(osol.anti_alias_filter.real.astype('float64')).to(dev)
    damp = torch.from_numpy(osol.damp_space.astype('float64')).to(dev)
    md = osol.medium
    gk = (md.omega0 / md.c) * md.n2
    pl = None
    if plasma:
        pl = dict(lx=torch.from_numpy(md.log10_I_gpu.astype(np.float64)).to(dev),
                  lw=torch.from_numpy(md.W_gpu.astype(np.float64)).to(dev), Ui=md.Ui,
                  rr=1.0 / md.tau_rec, dt=osol.dt, rho_nt=torch.tensor(md.rho_nt, dtype=torch.float64),
                  sigma=md.sigma_drude, w0tc=md.omega0 * md.tau_c)
    return dict(D=D, mask=mask, shock=shock, filt=filt, damp=damp, gk=gk, pl=pl)


def nonlinear(u, p, A_s):
    a = torch.fft.ifftn(u, dim=(0, 1, 2))
    I = A_s ** 2 * (a.real ** 2 + a.imag ** 2)
    Nw = p['shock'] * torch.fft.fft(1j * p['gk'] * I * a, dim=-1)
    if p['pl'] is not None:
        Nw = Nw + torch.fft.fft(torch_plasma.term(a, I, p['pl'])[0], dim=-1)
    return torch.fft.fft2(p['mask'] * Nw, dim=(0, 1))


def step(Z, h, p, A_s):
    A = torch.fft.fft2(Z, dim=(0, 1))
    E = torch.exp((h / 2) * p['D'])
    v = E * A
    a1 = E * nonlinear(A, p, A_s)
    a2 = nonlinear(v + (h / 2) * a1, p, A_s)
    a3 = nonlinear(v + (h / 2) * a2, p, A_s)
    a4 = nonlinear(E * (v + h * a3), p, A_s)
    beta = E * (v + (h / 6) * (a1 + 2 * a2 + 2 * a3))
    A4 = beta + (h / 6) * a4
    return torch.fft.ifft2(A4, dim=(0, 1)) * p['filt'] * torch.exp(-p['damp'] * h)


def propagate(A0, hs, p):
    A_s = float(A0.detach().abs().max())
    Z = torch.fft.fft(A0 / A_s, dim=-1)
    for h in hs:
        Z = step(Z, float(h), p, A_s)
    return torch.fft.ifft(Z, dim=-1) * A_s
