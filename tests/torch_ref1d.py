"""complex128 torch restatement of the 1D ERK4(3)-IP step (omega-domain state,
frozen step sequence) used as an autograd reference for the device adjoint.
Test infrastructure: same algorithm as erk43ip_method.py:256-286 for Kerr +
self-steepening with dispersion and loss, plus the plasma term with
I = |A|^2 / A_eff when ``pl`` is given (torch_plasma.term)."""
import torch

import torch_plasma


def nonlinear(u, G, pl=None):
    a = torch.fft.ifft(u)
    I = a.real ** 2 + a.imag ** 2
    out = 1j * G * torch.fft.fft(I * a)
    if pl is not None:
        out = out + torch.fft.fft(torch_plasma.term(a, I / pl['A_eff'], pl)[0])
    return out


def step(A, h, D, G, pl=None):
    E = torch.exp((h / 2) * D)
    v = E * A
    a1 = E * nonlinear(A, G, pl)
    a2 = nonlinear(v + (h / 2) * a1, G, pl)
    a3 = nonlinear(v + (h / 2) * a2, G, pl)
    a4 = nonlinear(E * (v + h * a3), G, pl)
    beta = E * (v + (h / 6) * (a1 + 2 * a2 + 2 * a3))
    return beta + (h / 6) * a4


def propagate(A0_time, D, G, hs, pl=None):
    A = torch.fft.fft(A0_time)
    for h in hs:
        A = step(A, float(h), D, G, pl)
    return torch.fft.ifft(A)
