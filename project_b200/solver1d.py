"""1D ERK4(3)-IP UPPE/GNLSE propagator on the GPU (drop-in for ``ERK43IP_UPPE``,
src/1D-ERK4(3)IP UPPE gas/erk43ip_method.py, with the argon patch of gas.py).

The host computes the reference's FP64 tables -- D(omega) (``:104-148``), the UPPE
factor (ω_abs/ω0)(n0/n(ω)) (``:226-250``) and the Raman response (``:150-179``) --
and ``libuppe_b200.so`` runs the whole adaptive loop of ``propagate``
(``:288-369``) in one persistent kernel launch: FFTs, the interaction-picture
factor, the nonlinear term, the error norm, the PI controller and the history
policy (``:327``) all execute on the device.  Many independent propagations run
in the same launch through :class:`BatchedPropagator`.

Extensions beyond the reference: ``taylor=(beta2, beta3)`` dispersion (D = i(b2 w^2/2 +
b3 w^3/6) - alpha/2), and ``plasma=GasPlasma1D(...)``: the envelope plasma term of
the 3+1D medium (ADK ionisation, density scan, loss and defocusing) with
intensity |A|^2 / A_eff.
"""
import ctypes

import numpy as np
import torch

from . import _lib
from .media import C0, E_CHARGE, EPS0, M_E, adk_rate

SELLMEIER = {   # erk43ip_method.py:74-90
    'fused_silica': {'B': [0.6961663, 0.4079426, 0.8974794],
                     'C': [0.0684043 ** 2, 0.1162414 ** 2, 9.896161 ** 2],
                     'valid_range': (0.21e-6, 6.7e-6)},
    'sapphire': {'B': [1.4313493, 0.65054713, 5.3414021],
                 'C': [0.0726631 ** 2, 0.1193242 ** 2, 18.028251 ** 2],
                 'valid_range': (0.2e-6, 5.5e-6)},
    'yag': {'B': [2.282, 3.27644, 4.44174],
            'C': [0.01185 ** 2, 0.0282 ** 2, 282.734 ** 2],
            'valid_range': (0.4e-6, 5e-6)},
}


class GasPlasma1D:
    """Plasma constants for the 1D envelope plasma term (argon defaults,
    media_physics.py:396-421), intensity I = |A|^2 / A_eff."""

    def __init__(self, A_eff, pressure_atm=1.0, center_wavelength=800e-9, Ui_eV=15.76,
                 rho_nt=None, tau_rec=1e-9, tau_c=None, lut=None, adk_prefactor=2.5e15):
        self.A_eff = A_eff
        self.Ui = Ui_eV * E_CHARGE
        self.rho_nt = 2.45e25 * pressure_atm if rho_nt is None else rho_nt
        self.tau_rec = tau_rec
        self.tau_c = 190e-15 / pressure_atm if tau_c is None else tau_c
        omega0 = 2 * np.pi * C0 / center_wavelength
        self.omega0 = omega0
        self.sigma = (E_CHARGE ** 2 * self.tau_c) / (C0 * EPS0 * 1.0 * M_E * (1.0 + omega0 ** 2 * self.tau_c ** 2))
        if lut is None:
            x = np.linspace(np.log10(1e8 * 1e4), np.log10(1e16 * 1e4), 2000)
            E = np.sqrt(2 * 10 ** x / (C0 * EPS0 * 1.0))
            lut = (x, adk_rate(E, self.Ui, prefactor=adk_prefactor))
        self.lut = (np.asarray(lut[0], dtype=np.float64), np.asarray(lut[1], dtype=np.float64))


class ERK43IP_UPPE:
    """Mirror of ``ERK43IP_UPPE`` (erk43ip_method.py:14-369) + the gas patch kwargs."""

    def __init__(self, material='fused_silica', gamma=None, n2=None, beam_radius=None,
                 alpha=0.0, center_wavelength=1064e-9, use_raman=True, f_R=0.18,
                 tau1=12.2e-15, tau2=32e-15, use_self_steepening=True, gas_P=101325.0,
                 gas_T=293.15, taylor=None, plasma=None, n0=None, precision='double', device=None):
        self.material = material
        self.alpha = alpha
        self.lambda0 = center_wavelength
        self.c = C0
        self.omega0 = 2 * np.pi * self.c / self.lambda0
        self.gas_P, self.gas_T = gas_P, gas_T
        if gamma is not None:                                                  # :36-51
            self.gamma, self.n2, self.beam_radius = gamma, 0.0, 0.0
        elif n2 is not None and beam_radius is not None:
            self.beam_radius, self.n2 = beam_radius, n2
            self.beam_area = np.pi * beam_radius ** 2
            self.gamma = (2 * np.pi / self.lambda0) * (n2 / self.beam_area)
        else:
            self.gamma, self.n2, self.beam_radius = 0.0, 0.0, 0.0
        self.use_raman, self.f_R, self.tau1, self.tau2 = use_raman, f_R, tau1, tau2
        self.use_self_steepening = use_self_steepening
        self.taylor = taylor
        self.plasma = plasma
        self.sellmeier_coeffs = SELLMEIER.get(material, SELLMEIER['fused_silica'])   # :61, :91
        self.precision = precision
        if precision not in ('single', 'double'):
            raise ValueError("precision must be 'single' or 'double'")
        self.device = torch.device(device if device is not None else 'cuda')
        if taylor is not None:
            self.n0 = 1.0 if n0 is None else n0
        else:
            self.n0 = float(self._compute_refractive_index(np.array([self.lambda0]))[0])   # :70

    # -- material model -------------------------------------------------------
    def _compute_refractive_index(self, wavelength):
        """Sellmeier n(lambda) (erk43ip_method.py:93-102); Peck & Fisher argon with
        ideal-gas scaling for material='argon_gas' (gas.py:20-37)."""
        wavelength = np.asarray(wavelength, dtype=np.float64)
        if self.material == 'argon_gas':
            lam_um = wavelength * 1e6
            sigma_sq = 1.0 / (lam_um ** 2)
            n0m1 = ((1205582.27 / (130.0 - sigma_sq)) + (317222.05 / (38.9 - sigma_sq))) * 1e-8
            return 1.0 + n0m1 * ((self.gas_P / 101325.0) * (288.15 / self.gas_T))
        B, Cc = self.sellmeier_coeffs['B'], self.sellmeier_coeffs['C']
        wl_sq = (wavelength * 1e6) ** 2
        n_sq = np.ones_like(wavelength, dtype=float)
        for i in range(3):
            n_sq += (B[i] * wl_sq) / (wl_sq - Cc[i])
        return np.sqrt(n_sq)

    def _compute_dispersion_operator(self, omega):
        """D(omega) and n(omega) (erk43ip_method.py:104-148)."""
        if self.taylor is not None:
            b2, b3 = self.taylor
            poly = 0.5 * b2 * omega ** 2 + (1.0 / 6.0) * b3 * omega ** 3
            wa = self.omega0 + omega
            n_omega = self.n0 + self.c * poly / np.where(np.abs(wa) < 1e-10, 1e-10, wa)
            return 1j * poly - self.alpha / 2, n_omega
        omega_abs = self.omega0 + omega
        omega_safe = np.where(np.abs(omega_abs) < 1e-10, 1e-10, np.abs(omega_abs))
        lo, hi = self.sellmeier_coeffs['valid_range']
        wl = np.clip(2 * np.pi * self.c / omega_safe, lo, hi)
        n_omega = self._compute_refractive_index(wl)
        k_omega = n_omega * omega_abs / self.c
        d_omega = self.omega0 * 1e-5
        n0 = self._compute_refractive_index(np.array([self.lambda0]))[0]
        n_p = self._compute_refractive_index(np.array([2 * np.pi * self.c / (self.omega0 + d_omega)]))[0]
        n_m = self._compute_refractive_index(np.array([2 * np.pi * self.c / (self.omega0 - d_omega)]))[0]
        k0 = n0 * self.omega0 / self.c
        k1 = (n_p * (self.omega0 + d_omega) / self.c - n_m * (self.omega0 - d_omega) / self.c) / (2 * d_omega)
        return 1j * (k_omega - k0 - k1 * omega) - self.alpha / 2, n_omega

    def _raman_response(self, omega):
        """H_R(omega) (erk43ip_method.py:150-179)."""
        N = len(omega)
        dt = 2 * np.pi / (N * np.abs(omega[1] - omega[0])) if N > 1 else 1e-15
        dt = max(dt, 1e-15)
        t = np.arange(N) * dt
        t1, t2 = max(self.tau1, 1e-20), max(self.tau2, 1e-20)
        h_t = (t1 ** 2 + t2 ** 2) / (t1 * t2 ** 2) * np.exp(-t / t2) * np.sin(t / t1)
        h_t[0] = 0.0
        H = np.fft.fft(h_t) * dt
        return H / H[0] if np.abs(H[0]) > 1e-15 else np.ones_like(H, dtype=complex)

    def tables(self, t):
        """Packed FP64 tables of one instance: (D, G, H or None, omega)."""
        t = np.asarray(t, dtype=np.float64)
        N = len(t)
        dt = t[1] - t[0]
        omega = 2 * np.pi * np.fft.fftfreq(N, dt)                                    # :292
        D, n_omega = self._compute_dispersion_operator(omega)
        if self.use_self_steepening:
            n_safe = np.where(n_omega < 1.0, 1.0, n_omega)                            # :244
            G = self.gamma * ((self.omega0 + omega) / self.omega0) * (self.n0 / n_safe)   # :248-250
        else:
            G = np.full(N, self.gamma)                                                # :255
        H = self._raman_response(omega) if self.use_raman else None
        return np.asarray(D, dtype=np.complex128), np.asarray(G, dtype=np.float64), H, omega

    def instance(self, t, L, tol=1e-4, max_step=1e-2, min_step=1e-11, hist_cap=0, max_attempts=0):
        t = np.asarray(t, dtype=np.float64)
        D, G, H, omega = self.tables(t)
        d = _lib.InstDesc1D()
        d.Nt, d.dt = len(t), float(t[1] - t[0])
        d.L, d.tol, d.max_step, d.min_step = float(L), float(tol), float(max_step), float(min_step)
        d.max_attempts = int(max_attempts)
        d.raman = 1 if self.use_raman else 0
        d.f_R = self.f_R
        d.hist_cap = int(hist_cap)
        d.omega0 = self.omega0
        p = self.plasma
        if p is not None:
            d.plasma = 1
            d.A_eff, d.Ui, d.sigma_drude = p.A_eff, p.Ui, p.sigma
            d.omega0_tau_c = p.omega0 * p.tau_c
            d.rate_rec, d.rho_nt, d.ava_coef = 1.0 / p.tau_rec, p.rho_nt, 0.0
        return {'desc': d, 'D': D, 'G': G, 'H': H, 'omega': omega,
                'lut': p.lut if p is not None else None}

    def propagate(self, A0, t, L, tol=1e-4, max_step=1e-2, min_step=1e-11, max_attempts=0):
        """erk43ip_method.py:288-369 -> (z_history, A_history, omega).

        History follows the reference policy (every accepted step while fewer than
        1000 are saved, afterwards when z advanced by more than L/500).  The final
        field and per-run diagnostics are in ``self.last_final`` / ``self.last_result``.
        """
        inst = self.instance(t, L, tol, max_step, min_step, hist_cap=1502, max_attempts=max_attempts)
        bp = BatchedPropagator([inst], precision=self.precision, device=self.device)
        finals, hist, results = bp.run([A0], with_history=True)
        r = results[0]
        self.last_result = r
        self.last_final = finals[0]
        zh, Ah = hist[0]
        return zh, Ah, inst['omega']


class BatchedPropagator:
    """Many 1D propagations (different Nt, media, pulses, lengths) in one persistent
    launch.  ``instances`` are dicts from :meth:`ERK43IP_UPPE.instance`."""

    def __init__(self, instances, precision='single', device=None):
        self._lib = _lib.load()
        self.device = torch.device(device if device is not None else 'cuda')
        self.instances = instances
        self.precision = precision
        self.cdtype = torch.complex64 if precision == 'single' else torch.complex128
        n = len(instances)
        self._descs = (_lib.InstDesc1D * n)(*[i['desc'] for i in instances])
        self._D = np.ascontiguousarray(np.concatenate([i['D'] for i in instances]))
        self._G = np.ascontiguousarray(np.concatenate([i['G'] for i in instances]))
        anyH = any(i['H'] is not None for i in instances)
        self._H = np.ascontiguousarray(np.concatenate(
            [i['H'] if i['H'] is not None else np.ones(i['desc'].Nt, complex) for i in instances])) if anyH else None
        luts = [i['lut'] for i in instances if i['lut'] is not None]
        if luts and any(not (np.array_equal(l[0], luts[0][0]) and np.array_equal(l[1], luts[0][1]))
                        for l in luts):
            raise ValueError('all plasma instances of a batch must share one ionisation LUT')
        self._lut = luts[0] if luts else None
        d = _lib.Desc1D()
        d.n_inst = n
        d.precision = _lib.UPPE_C64 if precision == 'single' else _lib.UPPE_C128
        d.inst = self._descs
        d.D, d.G = self._D.ctypes.data, self._G.ctypes.data
        d.H = self._H.ctypes.data if self._H is not None else None
        if self._lut is not None:
            self._lx = np.ascontiguousarray(self._lut[0])
            self._lw = np.ascontiguousarray(self._lut[1])
            d.lut_n, d.lut_log10I, d.lut_W = len(self._lx), self._lx.ctypes.data, self._lw.ctypes.data
        plan = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            _lib.check(self._lib.uppe1d_plan_create(ctypes.byref(d), ctypes.byref(plan)),
                       'uppe1d_plan_create')
        self._plan = plan
        self.offsets = np.concatenate([[0], np.cumsum([i['desc'].Nt for i in instances])])

    def __del__(self):
        plan = getattr(self, '_plan', None)
        if plan is not None and plan.value:
            self._lib.uppe1d_plan_destroy(plan)
            self._plan = None

    def pack(self, fields):
        """Host or device fields -> one packed device tensor."""
        parts = []
        for f, inst in zip(fields, self.instances):
            ft = f if isinstance(f, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(f))
            if ft.numel() != inst['desc'].Nt:
                raise ValueError('field length does not match Nt')
            parts.append(ft.reshape(-1).to(self.device, self.cdtype))
        return torch.cat(parts).contiguous()

    def run_packed(self, packed, hist=None, zhist=None, stream=None):
        """Propagate in place on a packed device field; returns the per-instance results."""
        res = (_lib.Result1D * len(self.instances))()
        _lib.check(self._lib.uppe1d_propagate(
            self._plan, ctypes.c_void_p(packed.data_ptr()),
            ctypes.c_void_p(hist.data_ptr() if hist is not None else 0),
            ctypes.c_void_p(zhist.data_ptr() if zhist is not None else 0),
            res, _lib.stream_ptr(stream)), 'uppe1d_propagate')
        return list(res)

    def run(self, fields, with_history=False, stream=None):
        packed = self.pack(fields)
        hist = zhist = None
        if with_history:
            nh = self._lib.uppe1d_hist_elems(self._plan)
            ns = self._lib.uppe1d_hist_slots(self._plan)
            hist = torch.zeros(max(nh, 1), dtype=self.cdtype, device=self.device)
            zhist = torch.zeros(max(ns, 1), dtype=torch.float64, device=self.device)
        results = self.run_packed(packed, hist, zhist, stream)
        out = packed.cpu().numpy()
        finals = [out[self.offsets[k]:self.offsets[k + 1]].copy() for k in range(len(self.instances))]
        hists = []
        if with_history:
            h = hist.cpu().numpy()
            zz = zhist.cpu().numpy()
            ho, zo = 0, 0
            for k, inst in enumerate(self.instances):
                n, cap = inst['desc'].Nt, inst['desc'].hist_cap
                cnt = results[k].hist_count
                hists.append((zz[zo:zo + cnt].copy(),
                              h[ho:ho + cap * n].reshape(cap, n)[:cnt].copy()))
                ho += cap * n
                zo += cap
        return finals, hists, results
