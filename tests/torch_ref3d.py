"""complex128 torch restatement of the 3+1D ERK4(3)-IP step in the (kx, ky, omega)
domain (solver_3d.py:100-160, Kerr + self-steepening, no plasma), frozen step
sequence; autograd reference for the device adjoint.  Test infrastructure."""
import torch


def make(osol):
    dev = 'cuda'
    D = torch.from_numpy(osol.D_operator).to(dev)
    mask = torch.from_numpy(osol.valid_freq_mask.astype('float64')).to(dev)
    shock = torch.from_numpy(osol.shock_operator.real.astype('float64')).to(dev)
    filt = torch.from_numpy(osol.anti_alias_filter.real.astype('float64')).to(dev)
    damp = torch.from_numpy(osol.damp_space.astype('float64')).to(dev)
    gk = (osol.medium.omega0 / osol.medium.c) * osol.medium.n2
    return dict(D=D, mask=mask, shock=shock, filt=filt, damp=damp, gk=gk)


def nonlinear(u, p, A_s):
    a = torch.fft.ifftn(u, dim=(0, 1, 2))
    K = 1j * p['gk'] * A_s ** 2 * (a.real ** 2 + a.imag ** 2) * a
    return torch.fft.fft2(p['mask'] * p['shock'] * torch.fft.fft(K, dim=-1), dim=(0, 1))


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
