"""1D lines on thread-block clusters (GPU).

A plan whose lines are all 2048..16384 points (no Raman, no history) with at
least one of 8192 or more runs every line on a cluster of four CTAs (or eight;
a batch of 16 or more lines with 16384-point ones runs its costliest lines on
eight-CTA clusters next to four-CTA ones) sharing the line through distributed
shared memory (uppe1d_cluster.cuh).  Checks: the
reference-derived oracle in complex128 (attempt for attempt), the single-CTA
kernel on the same batch (UPPE_1D_CLUSTER=0) with the plasma term, complex128 at
16384 points (which only the cluster kernel holds), and the logged / replayed
step sequence.
"""
import os

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _argon(precision='double', plasma=None, P=1.0):
    from project_b200.solver1d import ERK43IP_UPPE
    return ERK43IP_UPPE(material='argon_gas', n2=1.0e-23 * P, beam_radius=0.65 * 125e-6,
                        center_wavelength=800e-9, alpha=0.11513, use_raman=False,
                        taylor=(15e-30 * P, 15e-45 * P), plasma=plasma, precision=precision)


def _pulse(t, E=64e-6):
    from oracle.inputs import gaussian_pulse
    return gaussian_pulse(t, E, 30e-15)


def _boosted():
    from oracle import uppe1d as o1
    from project_b200.solver1d import GasPlasma1D
    Aeff = np.pi * (0.65 * 125e-6) ** 2
    op = o1.Plasma1D(Aeff, center_wavelength=800e-9)
    W = np.minimum(3e12 * (10.0 ** op.log10_I / 5e17) ** 8, 1e20)
    op.W = W
    return op, GasPlasma1D(Aeff, lut=(op.log10_I, W))


def test_cluster_kernel_matches_oracle_in_complex128():
    from oracle import uppe1d as o1
    from project_b200.solver1d import BatchedPropagator
    s = _argon()
    insts, fields, refs = [], [], []
    for Nt, E, L in [(8192, 64e-6, 0.03), (2048, 30e-6, 0.05), (16384, 50e-6, 0.02)]:
        t = np.linspace(-1e-12, 1e-12, Nt)
        A0 = _pulse(t, E)
        insts.append(s.instance(t, L, tol=1e-6))
        fields.append(A0)
        o = o1.Solver1D(material='argon_gas', n2=1.0e-23, beam_radius=0.65 * 125e-6, center_wavelength=800e-9,
                        alpha=0.11513, use_raman=False, taylor=(15e-30, 15e-45))
        _, Ao, _, log = o.propagate(A0, t, L=L, tol=1e-6)
        refs.append((Ao[-1], len(log)))
    finals, _, res = BatchedPropagator(insts, precision='double').run(fields)
    for f, (Ar, na), r in zip(finals, refs, res):
        assert r.status == 0
        assert r.attempts == na
        assert rel_l2(f, Ar) < 1e-10


@pytest.mark.parametrize('precision,tol', [('double', 1e-11), ('single', 1e-4)])
def test_cluster_kernel_matches_single_cta_kernel_with_plasma(monkeypatch, precision, tol):
    from project_b200.solver1d import BatchedPropagator
    op, pl = _boosted()
    s = _argon(plasma=pl)
    insts, fields = [], []
    for Nt in (8192, 4096, 2048):
        t = np.linspace(-0.5e-12, 0.5e-12, Nt)
        insts.append(s.instance(t, 0.02, tol=1e-6))
        fields.append(_pulse(t))
    fc, _, rc = BatchedPropagator(insts, precision=precision).run(fields)
    monkeypatch.setenv('UPPE_1D_CLUSTER', '0')
    fs, _, rs = BatchedPropagator(insts, precision=precision).run(fields)
    for a, b, r1, r2 in zip(fc, fs, rc, rs):
        assert r1.status == r2.status == 0
        assert r1.peak_ion > 1e-8
        assert abs(r1.energy - r2.energy) <= 1e-6 * r2.energy
        assert rel_l2(a, b) < tol
        if precision == 'double':
            assert r1.attempts == r2.attempts
            assert abs(r1.peak_ion - r2.peak_ion) <= 1e-9 * r2.peak_ion


def test_complex128_at_16384_points_with_plasma_vs_oracle():
    """Only the cluster kernel holds a 16384-point complex128 line."""
    from project_b200.solver1d import BatchedPropagator
    op, pl = _boosted()
    from oracle import uppe1d as o1
    s = _argon(plasma=pl)
    t = np.linspace(-1e-12, 1e-12, 16384)
    A0 = _pulse(t)
    o = o1.Solver1D(material='argon_gas', n2=1.0e-23, beam_radius=0.65 * 125e-6, center_wavelength=800e-9,
                    alpha=0.11513, use_raman=False, taylor=(15e-30, 15e-45), plasma=op)
    _, Ao, _, log = o.propagate(A0, t, L=0.01, tol=1e-6)
    finals, _, res = BatchedPropagator([s.instance(t, 0.01, tol=1e-6)], precision='double').run([A0])
    assert res[0].status == 0 and res[0].attempts == len(log)
    assert rel_l2(finals[0], Ao[-1]) < 1e-10
    assert res[0].peak_ion > 1e-8


def test_cluster_logged_steps_replay_to_the_same_field():
    import ctypes
    import torch
    from project_b200 import _lib
    from project_b200.solver1d import BatchedPropagator
    s = _argon()
    insts, fields = [], []
    for Nt in (16384, 8192):
        t = np.linspace(-1e-12, 1e-12, Nt)
        insts.append(s.instance(t, 0.03, tol=1e-6))
        fields.append(_pulse(t))
    bp = BatchedPropagator(insts, precision='double')
    lib = _lib.load()
    packed = bp.pack(fields)
    work = packed.clone()
    cap = 512
    hlog = torch.zeros(2 * cap, dtype=torch.float64, device='cuda')
    res = (_lib.Result1D * 2)()
    _lib.check(lib.uppe1d_propagate_logged(bp._plan, ctypes.c_void_p(work.data_ptr()),
                                           ctypes.c_void_p(hlog.data_ptr()), cap, res, _lib.stream_ptr()), 'log')
    n = max(res[0].accepted, res[1].accepted)
    sched = torch.zeros(2, n, dtype=torch.float64, device='cuda')
    for k in range(2):
        sched[k, :res[k].accepted] = hlog[k * cap:k * cap + res[k].accepted]
    rep = packed.clone()
    r2 = (_lib.Result1D * 2)()
    _lib.check(lib.uppe1d_propagate_schedule(bp._plan, ctypes.c_void_p(rep.data_ptr()),
                                             ctypes.c_void_p(sched.data_ptr()), n, r2, _lib.stream_ptr()), 'sched')
    assert torch.equal(rep, work)


@pytest.mark.parametrize('cluster', ['1', '0'])
def test_activity_record_of_the_persistent_launch(monkeypatch, cluster):
    """uppe1d_last_activity: every persistent CTA records its start and exit, so the
    SM-busy fraction lies in (0, 1] and the span covers the launch."""
    import ctypes
    from project_b200 import _lib
    from project_b200.solver1d import BatchedPropagator
    monkeypatch.setenv('UPPE_1D_CLUSTER', cluster)
    s = _argon()
    insts, fields = [], []
    for Nt in (8192, 4096, 2048, 2048):
        t = np.linspace(-1e-12, 1e-12, Nt)
        insts.append(s.instance(t, 0.02, tol=1e-6))
        fields.append(_pulse(t))
    bp = BatchedPropagator(insts, precision='single')
    assert bool(bp._lib.uppe1d_uses_clusters(bp._plan)) == (cluster == '1')
    bp.run(fields)
    busy, span = ctypes.c_double(), ctypes.c_double()
    _lib.check(bp._lib.uppe1d_last_activity(bp._plan, ctypes.byref(busy), ctypes.byref(span), _lib.stream_ptr()),
               'uppe1d_last_activity')
    assert 0.0 < busy.value <= 1.0 and span.value > 0.0
    # four instances on a 148-SM GPU: at most 4 x (CTAs per cluster) of the SMs can be busy
    ctas = 8 if os.environ.get('UPPE_CLUSTER_CTAS') == '8' else 4
    assert busy.value <= 4 * ctas / 148 + 1e-9


def test_mixed_launch_runs_each_line_as_one_of_the_two_cluster_sizes(monkeypatch):
    """A batch of 16 or more lines with 16384-point ones runs its costliest lines on
    eight-CTA clusters next to four-CTA clusters for the rest (two concurrent
    launches; the eight-CTA clusters take the head of the cost-ordered queue).  The
    costliest four lines' results are then bit for bit those of the forced
    eight-CTA run and every other line's those of the forced four-CTA run."""
    import torch
    from project_b200.solver1d import BatchedPropagator
    s = _argon(precision='single')
    insts, fields = [], []
    for k, Nt in enumerate([16384, 8192, 4096, 2048] * 5):
        t = np.linspace(-1e-12, 1e-12, Nt)
        inst = s.instance(t, 0.02, tol=1e-6)
        inst['desc'].cost = float(Nt) * (1.0 + 0.01 * k)
        insts.append(inst)
        fields.append(_pulse(t, 40e-6 + 2e-6 * k))

    def run(cs):
        if cs:
            monkeypatch.setenv('UPPE_CLUSTER_CTAS', cs)
        else:
            monkeypatch.delenv('UPPE_CLUSTER_CTAS', raising=False)
        bp = BatchedPropagator(insts, precision='single')
        finals, _, res = bp.run(fields)
        assert all(r.status == 0 for r in res)
        return finals

    mixed, four, eight = run(''), run('4'), run('8')
    costs = [i['desc'].cost for i in insts]
    head = set(np.argsort(costs)[::-1][:4].tolist())      # four 16384-point lines
    for k, (m, a, b) in enumerate(zip(mixed, four, eight)):
        assert np.array_equal(m, b if k in head else a), k
        assert rel_l2(a, b) < 1e-4        # the two cluster sizes agree to rounding
    torch.cuda.synchronize()
