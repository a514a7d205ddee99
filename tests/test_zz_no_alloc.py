"""The allocation-free 1D entry point (uppe1d_propagate_noalloc) against the
plan-based one (uppe1d_propagate), through the C ABI (GPU).

The no-allocation entry point exists for callers that may not call cudaMalloc
themselves -- plug-ins inside a host framework that owns the device allocator,
real-time hosts that must not allocate once running, code that only holds
device pointers lent to it.  It keeps its per-call device state in a static
device array, so two calls in a row must not leak state into each other; this
file is collected last so a failure here does not stop the rest of the suite.
"""
import ctypes

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _instances():
    from oracle.inputs import gaussian_pulse
    from project_b200.solver1d import ERK43IP_UPPE
    # call 1: argon capillary, Taylor dispersion, self-steepening, Nt = 1024
    a = ERK43IP_UPPE(material='argon_gas', n2=1.0e-23, beam_radius=0.65 * 125e-6,
                     center_wavelength=800e-9, alpha=0.11513, use_raman=False,
                     taylor=(15e-30, 15e-45))
    ta = np.linspace(-0.5e-12, 0.5e-12, 1024)
    fw = 30e-15
    Aa = gaussian_pulse(ta, 2e9 * fw * np.sqrt(np.pi / (4 * np.log(2))), fw)
    # call 2: fused silica with Raman (different Nt and physics), Nt = 512
    b = ERK43IP_UPPE(material='fused_silica', n2=2.6e-20, beam_radius=30e-6,
                     center_wavelength=1064e-9)
    tb = np.linspace(-1.0e-12, 1.0e-12, 512)
    Ab = gaussian_pulse(tb, 20e-9, 100e-15)
    return [(a.instance(ta, 0.05, tol=1e-6), Aa), (b.instance(tb, 0.02, tol=1e-6), Ab)]


def test_noalloc_matches_plan_entry_point_on_two_calls():
    import torch
    from project_b200 import _lib
    from project_b200.solver1d import BatchedPropagator
    lib = _lib.load()
    for inst, A0 in _instances():
        finals, _, res = BatchedPropagator([inst], precision='double').run([A0])
        D = torch.from_numpy(np.ascontiguousarray(inst['D'])).cuda()
        G = torch.from_numpy(np.ascontiguousarray(inst['G'])).cuda()
        H = torch.from_numpy(np.ascontiguousarray(inst['H'])).cuda() if inst['H'] is not None else None
        field = torch.from_numpy(np.ascontiguousarray(A0)).cuda()
        r = _lib.Result1D()
        rc = lib.uppe1d_propagate_noalloc(
            ctypes.byref(inst['desc']), _lib.UPPE_C128, ctypes.c_void_p(D.data_ptr()),
            ctypes.c_void_p(G.data_ptr()), ctypes.c_void_p(H.data_ptr() if H is not None else 0),
            0, None, None, ctypes.c_void_p(field.data_ptr()), ctypes.byref(r), _lib.stream_ptr())
        assert rc == 0, lib.uppe_last_error()
        assert r.status == res[0].status == 0
        assert r.attempts == res[0].attempts and r.accepted == res[0].accepted
        assert abs(r.z - res[0].z) < 1e-12
        assert rel_l2(field.cpu().numpy(), finals[0]) < 1e-10


def _call_noalloc(inst, A0, precision):
    """One uppe1d_propagate_noalloc call through the C ABI; the ionisation table
    goes in as device arrays in the field precision, as the entry point expects."""
    import torch
    from project_b200 import _lib
    lib = _lib.load()
    D = torch.from_numpy(np.ascontiguousarray(inst['D'])).cuda()
    G = torch.from_numpy(np.ascontiguousarray(inst['G'])).cuda()
    H = torch.from_numpy(np.ascontiguousarray(inst['H'])).cuda() if inst['H'] is not None else None
    cdt = torch.complex128 if precision == _lib.UPPE_C128 else torch.complex64
    rdt = torch.float64 if precision == _lib.UPPE_C128 else torch.float32
    field = torch.from_numpy(np.ascontiguousarray(A0)).to(cdt).cuda()
    lut_n, lx, lw = 0, None, None
    if inst['lut'] is not None:
        lx = torch.from_numpy(np.ascontiguousarray(inst['lut'][0])).to(rdt).cuda()
        lw = torch.from_numpy(np.ascontiguousarray(inst['lut'][1])).to(rdt).cuda()
        lut_n = lx.numel()
    r = _lib.Result1D()
    rc = lib.uppe1d_propagate_noalloc(
        ctypes.byref(inst['desc']), precision, ctypes.c_void_p(D.data_ptr()),
        ctypes.c_void_p(G.data_ptr()), ctypes.c_void_p(H.data_ptr() if H is not None else 0),
        lut_n, ctypes.c_void_p(lx.data_ptr() if lx is not None else 0),
        ctypes.c_void_p(lw.data_ptr() if lw is not None else 0), ctypes.c_void_p(field.data_ptr()),
        ctypes.byref(r), _lib.stream_ptr())
    assert rc == 0, lib.uppe_last_error()
    return field.cpu().numpy(), r


def _boosted_plasma_pair():
    """Argon capillary with the ADK table scaled up (W = 3e12 (I / 5e17 W/m^2)^8 1/s)
    so that a 2 GW pulse ionises measurably within a centimetre: the oracle's
    solver and the product's mirror with the same table."""
    from oracle import uppe1d as o1
    from project_b200.solver1d import ERK43IP_UPPE, GasPlasma1D
    Aeff = np.pi * (0.65 * 125e-6) ** 2
    op = o1.Plasma1D(Aeff, center_wavelength=800e-9)
    W = np.minimum(3e12 * (10.0 ** op.log10_I / 5e17) ** 8, 1e20)
    op.W = W
    kw = dict(n2=1.0e-23, beam_radius=0.65 * 125e-6, center_wavelength=800e-9,
              alpha=0.11513, use_raman=False, taylor=(15e-30, 15e-45))
    return (o1.Solver1D(material='argon_gas', plasma=op, **kw),
            ERK43IP_UPPE(material='argon_gas', plasma=GasPlasma1D(Aeff, lut=(op.log10_I, W)), **kw))


def _pulse(t):
    from oracle.inputs import gaussian_pulse
    fw = 30e-15
    return gaussian_pulse(t, 2e9 * fw * np.sqrt(np.pi / (4 * np.log(2))), fw)


def test_noalloc_complex64_at_its_limit_with_plasma_vs_plan_and_oracle(monkeypatch):
    """Complex64 at Nt = UPPE_NOALLOC_MAX_NT_C64 (the whole static array in use)
    with the plasma term on: the same attempts and field as the plan entry point
    running the same one-CTA kernel (a plan of one 16384-point line would
    otherwise take the cluster kernel) on two calls in a row, and the FP64
    oracle within the mixed-precision tolerance 1e-4."""
    monkeypatch.setenv('UPPE_1D_CLUSTER', '0')
    from project_b200 import _lib
    from project_b200.solver1d import BatchedPropagator
    osol, psol = _boosted_plasma_pair()
    t = np.linspace(-1e-12, 1e-12, _lib.UPPE_NOALLOC_MAX_NT_C64)
    A0 = _pulse(t)
    inst = psol.instance(t, 0.01, tol=1e-6)
    finals, _, res = BatchedPropagator([inst], precision='single').run([A0])
    for _ in range(2):                            # two calls in a row share the array
        f, r = _call_noalloc(inst, A0, _lib.UPPE_C64)
        assert r.status == res[0].status == 0
        assert r.attempts == res[0].attempts and r.accepted == res[0].accepted
        assert abs(r.z - res[0].z) < 1e-12
        assert rel_l2(f, finals[0]) < 1e-6
        assert r.peak_ion == res[0].peak_ion and r.peak_ion > 1e-8
    _, Ao, _, _ = osol.propagate(A0, t, L=0.01, tol=1e-6)
    assert rel_l2(f, Ao[-1]) < 1e-4


def test_noalloc_complex128_plasma_matches_plan_entry_point():
    from project_b200 import _lib
    from project_b200.solver1d import BatchedPropagator
    _, psol = _boosted_plasma_pair()
    t = np.linspace(-0.5e-12, 0.5e-12, 4096)
    A0 = _pulse(t)
    inst = psol.instance(t, 0.02, tol=1e-6)
    finals, _, res = BatchedPropagator([inst], precision='double').run([A0])
    f, r = _call_noalloc(inst, A0, _lib.UPPE_C128)
    assert r.status == res[0].status == 0
    assert r.attempts == res[0].attempts
    assert rel_l2(f, finals[0]) < 1e-12
    assert r.peak_ion == res[0].peak_ion and r.peak_ion > 1e-8


def test_noalloc_rejects_lines_beyond_the_static_limit():
    import torch
    from project_b200 import _lib
    lib = _lib.load()
    d = _lib.InstDesc1D()
    d.Nt, d.dt, d.L, d.tol, d.max_step, d.min_step = 16384, 1e-16, 0.1, 1e-6, 1e-2, 1e-11
    buf = torch.zeros(2 * 16384, dtype=torch.float64, device='cuda')
    p = ctypes.c_void_p(buf.data_ptr())
    rc = lib.uppe1d_propagate_noalloc(ctypes.byref(d), _lib.UPPE_C128, p, p, None, 0, None, None,
                                      p, None, _lib.stream_ptr())
    assert rc == -2
    assert b'static scratch limit' in lib.uppe_last_error()
