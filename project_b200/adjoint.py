"""Gradients of 1D propagations: a torch.autograd.Function over the device adjoint.

The forward runs ``ERK43IP_UPPE.propagate``'s adaptive loop on the device and
records the accepted step sizes; the backward runs the hand-written reverse-mode
kernel (``uppe1d_adjoint``) on that frozen step sequence: checkpoints every K
steps, recomputation within segments, transposed ERK4(3)-IP stages with the
conjugate interaction-picture factor, vector-Jacobian products of the Kerr +
self-steepening term.  Differentiable inputs: the time-domain input field, the
dispersion table D(omega) (so anything D depends on, e.g. pressure), the
nonlinear table G(omega) = gamma (w_abs/w0)(n0/n(w)), the length L (through
dA_L/dL = D A_L + N(A_L)) and, for plasma instances, the plasma parameters
(rho_nt, sigma_drude, omega0 tau_c).  complex128 only; the Raman response and
avalanche ionisation have no adjoint here.  torch.fft only converts cotangents
between the time and omega domains at the boundary.
"""
import ctypes

import numpy as np
import torch

from . import _lib
from .solver1d import BatchedPropagator

C0 = 299792458.0


class Propagate1D(torch.autograd.Function):
    @staticmethod
    def forward(ctx, A0, D, G, L, plasma_par, solver, t, tol, max_step, min_step, K):
        lib = _lib.load()
        inst = solver.instance(t, float(L), tol, max_step, min_step)
        inst['D'] = D.detach().cpu().numpy().astype(np.complex128)
        inst['G'] = G.detach().cpu().numpy().astype(np.float64)
        if inst['desc'].raman:
            raise NotImplementedError('the adjoint covers Kerr, self-steepening and plasma (no Raman)')
        _set_plasma(inst, plasma_par)
        bp = BatchedPropagator([inst], precision='double', device=A0.device)
        field = A0.detach().to(torch.complex128).contiguous().clone()
        cap = 2_000_000 if inst['desc'].max_attempts <= 0 else int(inst['desc'].max_attempts)
        cap = min(cap, 1 << 20)
        hlog = torch.zeros(cap, dtype=torch.float64, device=A0.device)
        res = (_lib.Result1D * 1)()
        _lib.check(lib.uppe1d_propagate_logged(bp._plan, ctypes.c_void_p(field.data_ptr()),
                                               ctypes.c_void_p(hlog.data_ptr()), cap, res,
                                               _lib.stream_ptr()), 'uppe1d_propagate_logged')
        r = res[0]
        if r.status & (_lib.STATUS_NONFINITE | 16):
            raise RuntimeError(f'forward propagation failed (status {r.status})')
        ctx.bp, ctx.hlog, ctx.nsteps, ctx.K = bp, hlog, int(r.accepted), int(K)
        Propagate1D.last_steps = hlog[:int(r.accepted)].cpu().numpy()
        ctx.result = r
        ctx.plasma = bool(inst['desc'].plasma)
        ctx.save_for_backward(A0.detach().to(torch.complex128).contiguous())
        return field

    @staticmethod
    def backward(ctx, gA):
        (A0,) = ctx.saved_tensors
        lib = _lib.load()
        N = A0.numel()
        dev = A0.device
        Abar = (torch.fft.fft(gA.to(torch.complex128)) / N).contiguous()
        work = torch.empty(lib.uppe1d_adjoint_work_elems(N, ctx.nsteps, ctx.K), dtype=torch.complex128,
                           device=dev)
        A0bar = torch.empty(N, dtype=torch.complex128, device=dev)
        gD = torch.empty(N, dtype=torch.complex128, device=dev)
        gG = torch.empty(N, dtype=torch.float64, device=dev)
        rhs = torch.empty(N, dtype=torch.complex128, device=dev)
        gPl = torch.zeros(3, dtype=torch.float64, device=dev)
        P = lambda x: ctypes.c_void_p(x.data_ptr())
        _lib.check(lib.uppe1d_adjoint(ctx.bp._plan, 0, P(ctx.hlog), ctx.nsteps, ctx.K, P(A0), P(Abar),
                                      P(A0bar), P(gD), P(gG), P(rhs), P(gPl), P(work), _lib.stream_ptr()),
                   'uppe1d_adjoint')
        gA0 = torch.fft.ifft(A0bar) * N
        gL = (torch.conj(Abar) * rhs).real.sum()
        return gA0, gD, gG, gL, (gPl if ctx.plasma else None), None, None, None, None, None, None


def _set_plasma(inst, plasma_par):
    """Plasma parameters (rho_nt, sigma_drude, omega0 tau_c) of a plasma instance."""
    if plasma_par is None:
        return
    if not inst['desc'].plasma:
        raise ValueError('plasma parameters given for an instance without the plasma term')
    v = [float(x) for x in plasma_par.detach().cpu()]
    inst['desc'].rho_nt, inst['desc'].sigma_drude, inst['desc'].omega0_tau_c = v


def replay_1d(A0, D, G, solver, t, hs, plasma_par=None):
    """Forward map with a frozen step sequence hs (every step accepted), on the device."""
    lib = _lib.load()
    inst = solver.instance(np.asarray(t, dtype=np.float64), float(np.sum(hs)), 1.0, 1.0, 1e-30)
    inst['D'] = D.detach().cpu().numpy().astype(np.complex128)
    inst['G'] = G.detach().cpu().numpy().astype(np.float64)
    _set_plasma(inst, plasma_par)
    bp = BatchedPropagator([inst], precision='double', device=A0.device)
    field = A0.detach().to(torch.complex128).contiguous().clone()
    hsd = torch.as_tensor(np.asarray(hs, dtype=np.float64), device=A0.device)
    res = (_lib.Result1D * 1)()
    _lib.check(lib.uppe1d_propagate_schedule(bp._plan, ctypes.c_void_p(field.data_ptr()),
                                             ctypes.c_void_p(hsd.data_ptr()), len(hs), res,
                                             _lib.stream_ptr()), 'uppe1d_propagate_schedule')
    return field


def propagate_1d(A0, D, G, L, solver, t, tol=1e-6, max_step=1e-2, min_step=1e-11, K=32,
                 plasma_par=None):
    """Differentiable final field A(L) (time domain) of a 1D propagation;
    plasma_par = (rho_nt, sigma_drude, omega0 tau_c) for a solver with a plasma term."""
    if not torch.is_tensor(L):
        L = torch.tensor(float(L), dtype=torch.float64)
    return Propagate1D.apply(A0, D, G, L, plasma_par, solver, np.asarray(t, dtype=np.float64), tol,
                             max_step, min_step, K)


# ---------------------------------------------------------------------------
# Capillary compression objective (spectral-phase knots, pressure, length)
# ---------------------------------------------------------------------------
def spline_basis(x_eval, x_knots):
    """Matrix B with phase(x_eval) = B @ knot_values for a natural cubic spline."""
    from scipy.interpolate import CubicSpline
    n = len(x_knots)
    B = np.zeros((len(x_eval), n))
    inside = (x_eval >= x_knots[0]) & (x_eval <= x_knots[-1])
    for j in range(n):
        e = np.zeros(n)
        e[j] = 1.0
        B[inside, j] = CubicSpline(x_knots, e, bc_type='natural')(x_eval[inside])
    return B


class CapillaryCompression:
    """Argon capillary (Taylor dispersion, loss, Kerr with self-steepening and,
    with ``plasma``, the ionisation/plasma term with I = |A|^2 / A_eff) whose
    input spectral phase is a cubic spline over n_knots knots spanning the band
    where the input spectrum exceeds 1 % of its peak.  Loss = -peak power of the
    output after ideal phase removal (the transform-limited output pulse).
    Pressure P scales beta2, beta3, n2, rho_nt (2.45e25 P) and 1/tau_c (190 fs / P)."""

    def __init__(self, t, A0_time, n_knots=64, lam=800e-9, radius=125e-6, beta2=15e-30, beta3=15e-45,
                 n2_per_bar=1e-23, loss_db_per_m=0.5, device='cuda', plasma=False, lut=None):
        from .solver1d import ERK43IP_UPPE, GasPlasma1D
        self.t = np.asarray(t, dtype=np.float64)
        self.N = len(self.t)
        self.dev = torch.device(device)
        dt = self.t[1] - self.t[0]
        self.omega = 2 * np.pi * np.fft.fftfreq(self.N, dt)
        self.omega0 = 2 * np.pi * C0 / lam
        self.alpha = loss_db_per_m * np.log(10) / 10
        self.A_eff = np.pi * (0.65 * radius) ** 2
        self.n2 = n2_per_bar
        self.beta2, self.beta3 = beta2, beta3
        self.lam = lam
        spec = np.fft.fft(np.asarray(A0_time, dtype=np.complex128))
        mag = np.abs(spec)
        band = self.omega[mag ** 2 >= 0.01 * (mag ** 2).max()]
        self.knots_x = np.linspace(band.min(), band.max(), n_knots)
        self.B = torch.from_numpy(spline_basis(self.omega, self.knots_x)).to(self.dev)
        self.spec0 = torch.from_numpy(spec).to(self.dev)
        # solver template: the tables are replaced by the differentiable ones below
        self.plasma = GasPlasma1D(self.A_eff, 1.0, lam, lut=lut) if plasma else None
        self.template = ERK43IP_UPPE(material='argon_gas', n2=n2_per_bar, beam_radius=0.65 * radius,
                                     center_wavelength=lam, alpha=self.alpha, use_raman=False,
                                     taylor=(beta2, beta3), precision='double', plasma=self.plasma)
        om = torch.from_numpy(self.omega).to(self.dev)
        self.poly = 0.5 * beta2 * om ** 2 + (1.0 / 6.0) * beta3 * om ** 3
        wa = self.omega0 + om
        self.w_safe = torch.where(wa.abs() < 1e-10, torch.full_like(wa, 1e-10), wa)
        self.wa = wa

    def tables(self, P):
        """D(omega), G(omega) at pressure P [bar] (beta2, beta3 and n2 scale with P),
        as solver1d builds them for a Taylor medium with n0 = 1."""
        D = 1j * (P * self.poly) - self.alpha / 2
        n = 1.0 + C0 * P * self.poly / self.w_safe
        n_safe = torch.where(n < 1.0, torch.ones_like(n), n)
        gamma = (2 * np.pi / self.lam) * (self.n2 * P / self.A_eff)
        G = gamma * (self.wa / self.omega0) * (1.0 / n_safe)
        return D.to(torch.complex128), G.to(torch.float64)

    def plasma_params(self, P):
        """(rho_nt, sigma_drude, omega0 tau_c) at pressure P (media_physics.py:412-419)."""
        if self.plasma is None:
            return None
        from .solver1d import E_CHARGE, EPS0, M_E
        tau_c = 190e-15 / P
        w = self.omega0
        sigma = (E_CHARGE ** 2 * tau_c) / (C0 * EPS0 * 1.0 * M_E * (1.0 + w ** 2 * tau_c ** 2))
        return torch.stack([2.45e25 * P, sigma, w * tau_c]).to(torch.float64)

    def input_field(self, knots):
        phase = self.B @ knots
        return torch.fft.ifft(self.spec0 * torch.exp(1j * phase))

    def loss(self, knots, P, L, tol=1e-6, K=32):
        D, G = self.tables(P)
        A_L = propagate_1d(self.input_field(knots), D, G, L, self.template, self.t, tol=tol, K=K,
                           plasma_par=self.plasma_params(P))
        tl = torch.fft.ifft(torch.fft.fft(A_L).abs())          # ideal phase removal
        return -(tl.real ** 2 + tl.imag ** 2).max()


# ---------------------------------------------------------------------------
# 3+1D: gradients of the final field with respect to the input field
# ---------------------------------------------------------------------------
class Propagate3D(torch.autograd.Function):
    """Final time-domain field A(x, y, t) of ERK43IP_UPPE_3D_Optimized.propagate as a
    differentiable function of the input field A0 (frozen accepted steps, device
    adjoint ``uppe3d_adjoint``: Kerr, self-steepening and the plasma terms)."""

    @staticmethod
    def forward(ctx, A0, solver, L, tol, max_step, min_step, K):
        solver.propagate(A0, L, tol=tol, max_step=max_step, min_step=min_step, return_gpu=True,
                         log_steps=True)
        out = solver.field().clone()
        ctx.solver, ctx.steps, ctx.K = solver, np.ascontiguousarray(solver.last_steps), int(K)
        ctx.save_for_backward(solver._as_device_field(A0))
        Propagate3D.last_steps = ctx.steps
        return out

    @staticmethod
    def backward(ctx, gA):
        (A0,) = ctx.saved_tensors
        sol = ctx.solver
        lib = _lib.load()
        Nt = sol.Nt
        A_scale = float(A0.abs().max())
        # Zbar = fft_t(gA) * A_scale / Nt with the plan's own t-line transform
        Zbar = gA.to(sol.complex_dtype).contiguous().clone()
        _lib.check(lib.uppe3d_transform_t(sol._plan, ctypes.c_void_p(Zbar.data_ptr()),
                                          ctypes.c_void_p(Zbar.data_ptr()), -1, A_scale / Nt,
                                          _lib.stream_ptr()), 'uppe3d_transform_t')
        nb = lib.uppe3d_adjoint_work_bytes(sol._plan, len(ctx.steps), ctx.K)
        work = torch.empty(nb, dtype=torch.uint8, device=A0.device)
        A0bar = torch.empty_like(A0)
        _lib.check(lib.uppe3d_adjoint(sol._plan, ctx.steps.ctypes.data, len(ctx.steps), ctx.K,
                                      ctypes.c_void_p(A0.data_ptr()), ctypes.c_void_p(Zbar.data_ptr()),
                                      ctypes.c_void_p(A0bar.data_ptr()), ctypes.c_void_p(work.data_ptr()),
                                      _lib.stream_ptr()), 'uppe3d_adjoint')
        Propagate3D.workspace_bytes = nb
        return A0bar, None, None, None, None, None, None


def propagate_3d(A0, solver, L, tol=1e-4, max_step=1e-2, min_step=1e-9, K=32):
    return Propagate3D.apply(A0, solver, L, tol, max_step, min_step, K)


class FilamentZernike:
    """3+1D filament objective: a Gaussian beam (w0, energy, FWHM) with a wavefront
    sum_j c_j Z_j (Noll j = 1..jmax over an aperture) and an input GDD applied along
    t; loss = - on-axis fluence of the output, sum_t |A(0, 0, t)|^2 dt."""

    def __init__(self, solver, w0, energy, fwhm, aperture_radius, jmax=15):
        from .pulses import gaussian_beam, zernike_basis
        self.sol = solver
        dev = solver.device
        self.env = torch.from_numpy(gaussian_beam(solver.x, solver.y, solver.t, w0, energy, fwhm)).to(dev)
        self.Z = torch.from_numpy(zernike_basis(solver.x, solver.y, aperture_radius, jmax)).to(dev)
        om = 2 * np.pi * np.fft.fftfreq(solver.Nt, solver.dt)
        self.w2 = torch.from_numpy(0.5 * om ** 2).to(dev)
        self.ix, self.iy = solver.Nx // 2, solver.Ny // 2

    def input_field(self, coeffs, gdd):
        phase = torch.einsum('j,jxy->xy', coeffs, self.Z)
        A = self.env * torch.exp(1j * phase)[:, :, None]
        return torch.fft.ifft(torch.fft.fft(A, dim=-1) * torch.exp(1j * gdd * self.w2), dim=-1)

    def loss(self, coeffs, gdd, L, tol=1e-4, K=32):
        A = propagate_3d(self.input_field(coeffs, gdd).to(self.sol.complex_dtype), self.sol, L, tol=tol, K=K)
        a = A[self.ix, self.iy, :].to(torch.complex128)
        return -(a.real ** 2 + a.imag ** 2).sum() * self.sol.dt
