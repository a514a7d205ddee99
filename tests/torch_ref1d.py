"""complex128 torch restatement of the 1D ERK4(3)-IP step (omega-domain state,
frozen step sequence) used as an autograd reference for the device adjoint.
Test infrastructure: same algorithm as erk43ip_method.py:256-286 for Kerr +
self-steepening with dispersion and loss."""
import torch


def nonlinear(u, G):
    a = torch.fft.ifft(u)
    return 1j * G * torch.fft.fft((a.real ** 2 + a.imag ** 2) * a)


def step(A, h, D, G):
    E = torch.exp((h / 2) * D)
    v = E * A
    a1 = E * nonlinear(A, G)
    a2 = nonlinear(v + (h / 2) * a1, G)
    a3 = nonlinear(v + (h / 2) * a2, G)
    a4 = nonlinear(E * (v + h * a3), G)
    beta = E * (v + (h / 6) * (a1 + 2 * a2 + 2 * a3))
    return beta + (h / 6) * a4


def propagate(A0_time, D, G, hs):
    A = torch.fft.fft(A0_time)
    for h in hs:
        A = step(A, float(h), D, G)
    return torch.fft.ifft(A)
