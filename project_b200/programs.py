"""Propagation programs: the drivers around the 1D ``propagate`` run on the device.

The reference drives its 1D solver from Python loops: a gas cell cut into slices
whose nonlinear coefficient follows the beam radius w(z) of a focused Gaussian
beam (``src/1D-ERK4(3)IP UPPE gas/gas.py:104-147``), and multipass cells where
each pass crosses air, a crystal and air again, then a mirror with loss, GDD and
TOD (``src/1D-ERK4(3)IP UPPE/test_gaussian_pulse GDD TOD 1mj copy.py:196-290``).
Here such a sequence is a *program* of operations (propagation slices and
mirrors) executed by ``uppe1d_run_programs``: one CTA per program, the field kept
on chip between operations, many programs (e.g. a sweep of pulse energies or
mirror GDDs) in one persistent launch.  Each slice starts like a fresh
``propagate`` call of the reference (h0 = max_step / 100, no controller memory).
"""
import ctypes

import numpy as np
import torch

from . import _lib
from .solver1d import BatchedPropagator

C0 = 299792458.0


class Slice:
    """Propagate ``L`` through ``solver``'s medium; ``gamma`` overrides the solver's
    nonlinear coefficient for this slice (the reference sets ``solver.gamma`` per
    slice, gas.py:124-126)."""

    def __init__(self, solver, L, tol=1e-4, max_step=1e-2, min_step=1e-11, gamma=None, record=False):
        self.solver, self.L, self.tol = solver, float(L), float(tol)
        self.max_step, self.min_step = float(max_step), float(min_step)
        self.gamma = None if gamma is None else float(gamma)
        self.record = bool(record)

    def key(self):
        return (id(self.solver), self.gamma, self.L, self.tol, self.max_step, self.min_step)


class Mirror:
    """Reflection: amplitude sqrt(1 - loss), spectral phase GDD w^2 / 2 + TOD w^3 / 6
    (test_gaussian_pulse GDD TOD 1mj copy.py:282-290)."""

    def __init__(self, loss=0.0, gdd=0.0, tod=0.0, record=False):
        self.amp = float(np.sqrt(1.0 - loss))
        self.gdd, self.tod = float(gdd), float(tod)
        self.record = bool(record)


def slice_instance(sl, t):
    """Plan instance of one slice: the solver's tables with G scaled to the slice's gamma."""
    s = sl.solver
    if sl.gamma is None:
        return s.instance(t, sl.L, sl.tol, sl.max_step, sl.min_step)
    g0 = s.gamma
    s.gamma = 1.0
    try:
        inst = s.instance(t, sl.L, sl.tol, sl.max_step, sl.min_step)
    finally:
        s.gamma = g0
    inst['G'] = inst['G'] * sl.gamma
    return inst


class ProgramRunner:
    """Runs programs (lists of Slice / Mirror) that share the time grid ``t``."""

    def __init__(self, programs, t, precision='double', device=None):
        self.t = np.asarray(t, dtype=np.float64)
        self.Nt = len(self.t)
        self.programs = programs
        keys, instances = {}, []
        ops = []
        op_begin = [0]
        for prog in programs:
            if not any(isinstance(o, Slice) for o in prog):
                raise ValueError('a program needs at least one Slice')
            for o in prog:
                op = _lib.Op1D()
                op.record = 1 if o.record else 0
                if isinstance(o, Slice):
                    k = o.key()
                    if k not in keys:
                        keys[k] = len(instances)
                        instances.append(slice_instance(o, self.t))
                    op.inst = keys[k]
                    op.amp = 1.0
                else:
                    op.inst, op.amp, op.gdd, op.tod = -1, o.amp, o.gdd, o.tod
                ops.append(op)
            op_begin.append(len(ops))
        self.bp = BatchedPropagator(instances, precision=precision, device=device)
        self._ops = (_lib.Op1D * len(ops))(*ops)
        self._begin = (ctypes.c_longlong * len(op_begin))(*op_begin)
        self.op_begin = op_begin
        self.nrec = [sum(1 for o in prog if o.record) for prog in programs]

    def run(self, fields, stream=None):
        """fields: one input field (time domain) per program.  Returns (finals,
        records, op_results): finals[p] the output field, records[p] an array
        [n_recorded, Nt] of the recorded fields, op_results[p] the per-operation
        results (z, steps, status, energy after the operation)."""
        lib = self.bp._lib
        dev, cd = self.bp.device, self.bp.cdtype
        packed = torch.cat([(f if isinstance(f, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(f)))
                            .reshape(-1).to(dev, cd) for f in fields]).contiguous()
        if packed.numel() != self.Nt * len(self.programs):
            raise ValueError('one field of Nt samples per program')
        nrec = sum(self.nrec)
        rec = torch.zeros(max(nrec, 1) * self.Nt, dtype=cd, device=dev)
        res = (_lib.Result1D * len(self._ops))()
        _lib.check(lib.uppe1d_run_programs(self.bp._plan, len(self.programs), self._begin, self._ops,
                                           ctypes.c_void_p(packed.data_ptr()),
                                           ctypes.c_void_p(rec.data_ptr() if nrec else 0), res,
                                           _lib.stream_ptr(stream)), 'uppe1d_run_programs')
        out = packed.cpu().numpy().reshape(len(self.programs), self.Nt)
        recs = rec.cpu().numpy()[:nrec * self.Nt].reshape(nrec, self.Nt)
        records, op_results, r0 = [], [], 0
        for p in range(len(self.programs)):
            records.append(recs[r0:r0 + self.nrec[p]].copy())
            r0 += self.nrec[p]
            op_results.append(list(res[self.op_begin[p]:self.op_begin[p + 1]]))
        return [o.copy() for o in out], records, op_results


def gas_cell_program(solver, L_cell, n_slices, w0, n2, center_wavelength, tol=1e-5, min_step=1e-8,
                     record=True):
    """gas.py:104-147: the cell [-L/2, L/2] cut into n_slices; slice i has the beam
    radius w = w0 sqrt(1 + (z_mid / zR)^2), zR = pi w0^2 / lambda, gamma =
    (2 pi / lambda) n2 / (pi w^2), max_step = dz / 10."""
    zR = np.pi * w0 ** 2 / center_wavelength
    edges = np.linspace(-L_cell / 2, L_cell / 2, n_slices + 1)
    prog = []
    for i in range(n_slices):
        dz = edges[i + 1] - edges[i]
        zm = 0.5 * (edges[i] + edges[i + 1])
        w = w0 * np.sqrt(1 + (zm / zR) ** 2)
        gamma = (2 * np.pi / center_wavelength) * (n2 / (np.pi * w ** 2))
        prog.append(Slice(solver, dz, tol=tol, max_step=dz / 10, min_step=min_step, gamma=gamma,
                          record=record))
    return prog


def multipass_program(air, crystal, n_passes, L_cavity, L_crystal, crystal_offset, w_at, n2_air,
                      n2_crystal, center_wavelength, air_slices, crystal_slices, mirror,
                      air_tol=1e-3, crystal_tol=1e-4):
    """test_gaussian_pulse GDD TOD 1mj copy.py:168-290: per pass, air from the left
    mirror to the crystal, the crystal, air to the right mirror (each cut into
    slices with gamma from the local beam radius w_at(z)), then ``mirror``.
    Records the field after each air segment and each crystal slice."""
    half = L_crystal / 2.0
    zf, zb = crystal_offset - half, crystal_offset + half
    zl, zr = -L_cavity / 2.0, L_cavity / 2.0
    if zf < zl or zb > zr:
        raise ValueError('the crystal does not fit inside the cavity')
    k = 2 * np.pi / center_wavelength

    def air_seg(z0, z1):
        out = []
        edges = np.linspace(z0, z1, air_slices + 1)
        dz = (z1 - z0) / air_slices
        for i in range(air_slices):
            w = w_at(0.5 * (edges[i] + edges[i + 1]))
            g = k * (n2_air / (np.pi * w ** 2)) if n2_air > 0 else 0.0
            out.append(Slice(air, dz, tol=air_tol, max_step=dz, gamma=g, record=(i == air_slices - 1)))
        return out

    prog = []
    for _ in range(n_passes):
        prog += air_seg(zl, zf)
        edges = np.linspace(zf, zb, crystal_slices + 1)
        dz = L_crystal / crystal_slices
        for i in range(crystal_slices):
            w = w_at(0.5 * (edges[i] + edges[i + 1]))
            prog.append(Slice(crystal, dz, tol=crystal_tol, max_step=dz,
                              gamma=k * (n2_crystal / (np.pi * w ** 2)), record=True))
        prog += air_seg(zb, zr)
        prog.append(mirror)
    return prog


# ---------------------------------------------------------------------------
# 3+1D: segment sequences through several media with mirrors
# ---------------------------------------------------------------------------
class Segment3D:
    """Propagate L through ``solver`` (an ERK43IP_UPPE_3D_Optimized on the shared grid)."""

    def __init__(self, solver, L, tol=1e-4, max_step=1e-2, min_step=1e-9):
        self.solver, self.L, self.tol = solver, float(L), float(tol)
        self.max_step, self.min_step = float(max_step), float(min_step)


class Mirror3D:
    """Reflection: sqrt(1 - loss), spectral phase and, with R, a curved mirror."""

    def __init__(self, R=None, loss=0.0, gdd=0.0, tod=0.0):
        self.R, self.loss, self.gdd, self.tod = R, float(loss), float(gdd), float(tod)


def run_sequence_3d(ops, A0, callback=None):
    """src/3+1D-ERK4(3)IP UPPE/sim.py:304-351 (run): segments through their media,
    mirrors applied to the state of the last solver used.  The field stays on the
    device between segments (each segment renormalises by its own max|A|, as each
    propagate call of the reference does).  Returns the final time-domain field
    (device) and the per-segment results; callback(k, op, solver) runs after each op."""
    A = A0
    last = None
    results = []
    for k, op in enumerate(ops):
        if isinstance(op, Segment3D):
            op.solver.propagate(A, op.L, tol=op.tol, max_step=op.max_step, min_step=op.min_step,
                                return_gpu=True)
            results.append(op.solver.last_result)
            last = op.solver
        else:
            if last is None:
                last = next(o.solver for o in ops if isinstance(o, Segment3D))
                last.set_field(A)
            last.mirror(op.R, op.loss, op.gdd, op.tod)
            results.append(None)
        A = last.field()
        if callback is not None:
            callback(k, op, last)
    return A, results


def mpc_cycles_3d(air, fs, cycles, d_air_1, d_fs, d_air_mid, d_air_last, R_concave, T_per_round,
                  n_plates=4, air_tol=1e-4, fs_tol=1e-5, fs_max_step=20e-6):
    """The multipass cycle of sim.py:304-331: forward (air, [fs, air] x n_plates with the
    last air gap d_air_last), curved mirror, the same backward, flat-mirror transmission
    T_per_round.  Air segments use max_step = min(d, 5 mm) (sim.py:125-127)."""
    def air_seg(d):
        return Segment3D(air, d, tol=air_tol, max_step=min(d, 5e-3))
    fwd = [air_seg(d_air_1)]
    for i in range(n_plates):
        fwd.append(Segment3D(fs, d_fs, tol=fs_tol, max_step=fs_max_step))
        fwd.append(air_seg(d_air_last if i == n_plates - 1 else d_air_mid))
    bwd = [(air_seg(o.L) if o.solver is air else Segment3D(fs, o.L, tol=fs_tol, max_step=fs_max_step))
           for o in fwd[::-1]]
    ops = []
    for _ in range(cycles):
        ops += fwd + [Mirror3D(R=R_concave)] + bwd + [Mirror3D(loss=1.0 - T_per_round)]
    return ops
