"""Plain-GPU comparator: a direct torch (cuFFT) complex128 transliteration of the
reference's 3+1D step, ``solver_3d.py:100-160`` with ``media_physics.py:156-205``,
using the naive per-line density kernel in ``plain_scan.cu``.  Not the product."""
import ctypes
import os
import subprocess

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
SO = os.path.join(HERE, 'libplain_scan.so')


def build():
    src = os.path.join(HERE, 'plain_scan.cu')
    if os.path.exists(SO) and os.path.getmtime(SO) >= os.path.getmtime(src):
        return SO
    subprocess.check_call(['nvcc', '-gencode', 'arch=compute_100a,code=sm_100a', '-O3',
                           '-Xcompiler', '-fPIC', '-shared', '-o', SO, src])
    return SO


class PlainStep:
    def __init__(self, x, y, t, medium, device):
        self.dev = device
        self.lib = ctypes.CDLL(build())
        self.lib.plain_scan_launch.argtypes = [ctypes.c_void_p] * 4 + [ctypes.c_float] * 3 + \
            [ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
        m = medium
        Nx, Ny, Nt = len(x), len(y), len(t)
        self.dt = float(t[1] - t[0])
        dx, dy = float(x[1] - x[0]), float(y[1] - y[0])
        kx = 2 * np.pi * np.fft.fftfreq(Nx, dx)
        ky = 2 * np.pi * np.fft.fftfreq(Ny, dy)
        K2 = kx[:, None] ** 2 + ky[None, :] ** 2
        om = 2 * np.pi * np.fft.fftfreq(Nt, self.dt)
        w0, c = m.omega0, m.c
        n = m.refractive_index(om + w0)
        k = n * (om + w0) / c
        nc = float(m.refractive_index(np.array([w0]))[0])
        dw = w0 * 1e-3
        npl = float(m.refractive_index(np.array([w0 + dw]))[0])
        k0 = nc * w0 / c
        k1 = (npl * (w0 + dw) / c - k0) / dw
        kref = k0 + k1 * om
        ksq = (k ** 2)[None, None, :]
        kz = np.sqrt((ksq - K2[:, :, None]).astype(np.complex128))
        D = 1j * (((ksq - kref[None, None, :] ** 2) - K2[:, :, None]) / (kz + kref[None, None, :]))
        D = D * ((om + w0) > 0)[None, None, :]
        self.D = torch.from_numpy(D).to(device)
        self.shock = torch.from_numpy(m.get_shock_operator(om).astype(np.complex128)).to(device)
        self.mask = torch.from_numpy(((om + w0) > 0).astype(np.float64)).to(device)
        f = om / (2 * np.pi)
        fmax = float(np.max(np.abs(f))) + 1e-10
        self.filt = torch.from_numpy(np.exp(-(f / (0.85 * fmax)) ** 16)).to(device)
        X, Y = np.meshgrid(x, y, indexing='ij')
        R = np.sqrt(X ** 2 + Y ** 2)
        hw = float(np.max(np.abs(x)))
        s = np.clip((R - 0.85 * hw) / (0.13 * hw + 1e-30), 0, 1)
        self.damp = torch.from_numpy(120.0 * s ** 10)[:, :, None].to(device)
        self.lx = torch.from_numpy(m.lut_log10I).to(device)
        self.lw = torch.from_numpy(m.lut_W).to(device)
        self.gk = (m.omega0 / m.c) * m.n2
        self.Ui, self.sig, self.w0tc = m.Ui, m.sigma_drude, m.omega0 * m.tau_c
        self.rr, self.rnt = 1.0 / m.tau_rec, m.rho_nt
        self.A_scale = 1.0

    def interp(self, xq):
        xq = xq.clamp(float(self.lx[0]), float(self.lx[-1]))
        j = torch.searchsorted(self.lx, xq, right=True).clamp(1, len(self.lx) - 1) - 1
        x0, x1, y0, y1 = self.lx[j], self.lx[j + 1], self.lw[j], self.lw[j + 1]
        return y0 + (y1 - y0) / (x1 - x0) * (xq - x0)

    def N(self, fkw):
        A = torch.fft.ifftn(fkw, dim=(0, 1, 2)) * self.A_scale
        I = A.abs() ** 2
        W = self.interp(torch.log10(I + 1e-30)).to(torch.float32).contiguous()
        Wa = torch.zeros_like(W)
        rho = torch.empty(I.shape, dtype=torch.float64, device=self.dev)
        gen = torch.empty_like(rho)
        nt = I.shape[-1]
        self.lib.plain_scan_launch(W.data_ptr(), Wa.data_ptr(), rho.data_ptr(), gen.data_ptr(),
                                   self.rr, self.dt, self.rnt, nt, I.numel() // nt,
                                   torch.cuda.current_stream().cuda_stream)
        K = 1j * self.gk * I * A
        P = (-(gen * self.Ui) / (2.0 * I + 1e-30)) * A - (self.sig / 2.0) * (1 + 1j * self.w0tc) * rho * A
        Nw = self.shock * torch.fft.fft(K / self.A_scale, dim=-1) + torch.fft.fft(P / self.A_scale, dim=-1)
        return torch.fft.fft2(Nw * self.mask, dim=(0, 1))

    def step(self, A_t, h):
        Akw = torch.fft.fft2(torch.fft.fft(A_t, dim=-1), dim=(0, 1))
        E = torch.exp((h / 2) * self.D)
        v = Akw * E
        a1 = self.N(Akw) * E
        a2 = self.N(v + (h / 2) * a1)
        a3 = self.N(v + (h / 2) * a2)
        a4 = self.N((v + h * a3) * E)
        beta = (v + (h / 6) * (a1 + 2 * a2 + 2 * a3)) * E
        A4 = beta + (h / 6) * a4
        a5 = self.N(A4)
        A3 = beta + (h / 30) * (2 * a4 + 3 * a5)
        err = float((A4 - A3).abs().max() / (A4.abs().max() + 1e-20))
        out = torch.fft.ifft(torch.fft.ifft2(A4, dim=(0, 1)) * self.filt, dim=-1)
        return out * torch.exp(-self.damp * h), err


def time_step(x, y, t, A0, medium, device, reps=3):
    """Mean time of one complex128 plain-GPU ERK attempt at this grid."""
    st = PlainStep(x, y, t, medium, device)
    A = torch.from_numpy(A0.astype(np.complex128)).to(device)
    st.A_scale = float(A.abs().max())
    A = A / st.A_scale
    st.step(A, 2e-3)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        out, err = st.step(A, 2e-3)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    npts = A.numel()
    del st, A, out
    torch.cuda.empty_cache()
    return {'ms_per_attempt': ms, 'value': npts / (ms / 1e3), 'unit': 'pt-steps/s',
            'dtype': 'c128', 'what': 'torch/cuFFT complex128 transliteration of solver_3d.py:100-160 '
                                     'with a naive one-thread-per-line density kernel'}
