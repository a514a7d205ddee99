"""Host-side logic without a GPU: table construction, input generators, ADK,
batch partitioning (world size 2 over gloo)."""
import os

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import golden, rel_l2


def test_3d_tables_reproduce_reference_operator():
    from oracle import uppe3d
    from project_b200.media import Argon
    from project_b200.solver3d import ip_operator_host, tables3d
    for name, disp in (('ref3d_mpi_cauchy_double', None),
                       ('ref3d_adk_taylor_double', ('taylor', 1.000283, 20e-30, 0.0))):
        g = golden(name)
        med = Argon(float(g['lam']), 1.0, 'double', bool(g['shock']), dispersion=disp,
                    lut=(g['log10_I'], g['W_lut']))
        tb = tables3d(g['x'], g['y'], g['t'], med)
        D = ip_operator_host(tb)
        assert rel_l2(D, g['D']) < 1e-15
        om = uppe3d.argon(float(g['lam']), 1.0, 'double', bool(g['shock']), dispersion=disp)
        osol = uppe3d.Solver3D(g['x'], g['y'], g['t'], om, 'double')
        assert np.array_equal(tb['damp'], osol.damp_space[:, :, 0])
        assert np.array_equal(tb['filter'], osol.anti_alias_filter[0, 0].real)
        assert np.array_equal(tb['shock'], osol.shock_operator[0, 0].real)
        assert np.array_equal(tb['freq_axis_hz'], g['freq'])


def test_1d_tables_match_reference():
    from project_b200.solver1d import ERK43IP_UPPE
    g = golden('ref1d_argon')
    s = ERK43IP_UPPE(material='argon_gas', n2=1.0e-23, beam_radius=0.65 * 125e-6,
                     center_wavelength=800e-9, alpha=0.5 * np.log(10) / 10, use_raman=False)
    D, G, H, om = s.tables(g['t'])
    assert np.array_equal(D, g['D'])
    assert np.array_equal(om, g['omega'])
    assert s.gamma == float(g['gamma']) and s.n0 == float(g['n0'])
    g = golden('ref1d_silica_raman')
    s = ERK43IP_UPPE(material='fused_silica', n2=2.6e-20, beam_radius=30e-6, center_wavelength=1064e-9)
    D, G, H, om = s.tables(g['t'])
    assert np.array_equal(D, g['D'])
    assert rel_l2(H, g['H_R']) < 1e-15


def test_1d_uppe_factor_matches_oracle():
    from oracle import uppe1d as o1
    from project_b200.solver1d import ERK43IP_UPPE
    t = np.linspace(-0.5e-12, 0.5e-12, 512)
    kw = dict(material='argon_gas', n2=1e-23, beam_radius=80e-6, center_wavelength=800e-9)
    o = o1.Solver1D(use_raman=False, **kw)
    om = 2 * np.pi * np.fft.fftfreq(512, t[1] - t[0])
    o.setup(om, t[1] - t[0])
    D, G, H, _ = ERK43IP_UPPE(use_raman=False, **kw).tables(t)
    assert np.allclose(G, o.gamma * o._U, rtol=1e-15, atol=0)


def test_inputs_match_oracle_definitions():
    from oracle import inputs as oi
    from project_b200 import pulses as pp
    t = np.linspace(-0.5e-12, 0.5e-12, 1024)
    assert np.allclose(pp.gaussian_pulse(t, 1e-4, 30e-15), oi.gaussian_pulse(t, 1e-4, 30e-15), rtol=1e-14)
    assert rel_l2(pp.dispersed_pulse(t, 1e-4, 30e-15, GDD=200e-30, TOD=100e-45),
                  oi.dispersed_pulse(t, 1e-4, 30e-15, GDD=200e-30, TOD=100e-45)) < 1e-13
    assert rel_l2(pp.photon_noise(t, 800e-9, 0), oi.photon_noise(t, 800e-9, 0)) < 1e-13
    x = np.linspace(-3e-3, 3e-3, 64)
    assert rel_l2(pp.speckle(x, x, 50e-6, 0.01, 1), oi.speckle(x, x, 50e-6, 0.01, 1)) < 1e-13
    # one photon per mode: mean |A_j|^2 over many seeds ~ hbar w_j Nt / dt
    n = np.mean([np.abs(np.fft.fft(pp.photon_noise(t, 800e-9, s))) ** 2 for s in range(200)], axis=0)
    w = 2 * np.pi * 299792458.0 / 800e-9 + 2 * np.pi * np.fft.fftfreq(1024, t[1] - t[0])
    expect = np.where(w > 0, 1.054571817e-34 * w * 1024 / (t[1] - t[0]), 0)
    sel = w > 0
    assert abs(np.mean(n[sel] / expect[sel]) - 1) < 0.05
    sp = pp.speckle(x, x, 50e-6, 0.01, 1)
    assert abs(np.std(sp) - 0.01) < 1e-12 and abs(np.mean(sp) - 1) < 1e-12


def test_adk_matches_oracle():
    from oracle import adk as oa
    from project_b200.media import Argon, adk_rate
    E = np.logspace(6, 12, 200)
    Ui = 15.76 * 1.60217663e-19
    assert np.array_equal(adk_rate(E, Ui), oa.adk_rate(E, Ui))
    m = Argon(800e-9, 1.0, 'double', True)
    x, W = oa.ionization_lut(Ui)
    assert np.array_equal(m.lut_log10I, x) and np.array_equal(m.lut_W, W)


def test_partition_instances_is_balanced_cover():
    from project_b200.distributed import instance_cost, partition_instances
    rng = np.random.Generator(np.random.PCG64(2))
    Nt = rng.choice([2048, 4096, 8192, 16384], size=256)
    costs = [instance_cost(int(n), 1.0) for n in Nt]
    parts = partition_instances(costs, 8)
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(256))
    loads = [sum(costs[i] for i in p) for p in parts]
    assert max(loads) / (sum(loads) / 8) < 1.05


def test_instance_cost_grows_with_energy_and_pressure():
    """The sweep's cost model: per-attempt cost Nt log2 Nt times attempts that grow
    with pulse energy and pressure (the nonlinear phase sets the step size)."""
    from project_b200.distributed import instance_cost
    base = instance_cost(4096, 1.0, energy=100e-6, pressure=1.0)
    assert instance_cost(4096, 1.0, energy=400e-6, pressure=1.0) > base
    assert instance_cost(4096, 1.0, energy=100e-6, pressure=2.5) > base
    assert instance_cost(8192, 1.0, energy=100e-6, pressure=1.0) > 2 * base
    assert instance_cost(4096, 2.0, energy=100e-6, pressure=1.0) == 2 * base
    assert instance_cost(4096, 1.0) == instance_cost(4096, 1.0, energy=None, pressure=None)


def _worker(rank, world, port, q):
    import torch.distributed as dist
    from project_b200.distributed import gather_results, partition_instances
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    dist.init_process_group('gloo', rank=rank, world_size=world)
    costs = [float(c) for c in range(1, 11)]
    parts = partition_instances(costs, world)
    mine = parts[rank]
    local = [(i, {'z': 1.0, 'rank': rank}) for i in mine]
    merged = gather_results(local)
    if rank == 0:
        q.put((sorted(merged), [merged[i]['rank'] for i in range(10)], parts))
    dist.barrier()
    dist.destroy_process_group()


def test_sharded_batch_gather_gloo_world2():
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    keys, owners, parts = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert keys == list(range(10))
    for r, part in enumerate(parts):
        assert all(owners[i] == r for i in part)


def test_gas_cell_program_slices_follow_the_beam():
    """gas.py:104-126: slice widths, w(z_mid) and gamma = (2 pi / lambda) n2 / (pi w^2)."""
    from project_b200.programs import Slice, gas_cell_program

    class Dummy:
        pass
    lam, w0, n2 = 800e-9, 150e-6, 1e-23
    prog = gas_cell_program(Dummy(), L_cell=1.0, n_slices=50, w0=w0, n2=n2, center_wavelength=lam)
    assert len(prog) == 50 and all(isinstance(s, Slice) for s in prog)
    zR = np.pi * w0 ** 2 / lam
    edges = np.linspace(-0.5, 0.5, 51)
    for i, s in enumerate(prog):
        zm = 0.5 * (edges[i] + edges[i + 1])
        w = w0 * np.sqrt(1 + (zm / zR) ** 2)
        assert abs(s.L - 0.02) < 1e-15 and abs(s.max_step - 0.002) < 1e-15
        assert abs(s.gamma - (2 * np.pi / lam) * n2 / (np.pi * w ** 2)) <= 1e-12 * s.gamma
    # symmetric about the focus, largest at the centre
    g = np.array([s.gamma for s in prog])
    assert np.allclose(g, g[::-1], rtol=1e-12) and g.argmax() in (24, 25)


def test_fwhm_and_moments_match_the_driver_formulas():
    """project_b200.solver3d.fwhm / beam_moments vs the restated sim.py:145-182."""
    from oracle.diagnostics import _fwhm, beam_diagnostics
    from project_b200.solver3d import beam_moments, fwhm
    rng = np.random.Generator(np.random.PCG64(5))
    t = np.linspace(-200e-15, 200e-15, 256)
    for _ in range(20):
        w = rng.uniform(10e-15, 80e-15)
        I = np.exp(-((t - rng.uniform(-50e-15, 50e-15)) / w) ** 2) + 0.05 * rng.random(256)
        assert fwhm(t, I) == _fwhm(t, I)
    assert np.isnan(fwhm(t, np.zeros(256))) and np.isnan(_fwhm(t, np.zeros(256)))
    x = np.linspace(-1e-3, 1e-3, 32)
    A = (rng.standard_normal((32, 32, 16)) + 1j * rng.standard_normal((32, 32, 16)))
    o = beam_diagnostics(A, x, x, t[:16], 0.3e-3, 800e-9)
    m = beam_moments(x, x, o['fluence'])
    assert np.allclose(m, [o['x_mean_m'], o['y_mean_m'], o['wx_rms_m'], o['wy_rms_m']], rtol=1e-12, atol=1e-18)


@pytest.mark.parametrize('kind', ['cubic', 'quadratic', 'linear'])
def test_spectrum_spline_matches_interp1d(kind):
    """The piecewise cubic handed to the device equals interp1d(kind) of the
    Jacobian-scaled spectrum (erk43ip_method.py:674-716), zero outside."""
    from scipy.interpolate import interp1d
    from conftest import golden
    from project_b200.pulses import spectrum_spline
    g = golden('ref1d_spectrum_pulse')
    c = 299792458.0
    brk, coef = spectrum_spline(g['wl'][::-1], g['I'][::-1], True, kind)
    wl = np.sort(g['wl'])
    I = g['I'][np.argsort(g['wl'])]
    I = I / I.max()
    f = c / (wl * 1e-9)
    Ij = I * (wl * 1e-9) ** 2 / c
    Ij = Ij / Ij.max()
    x = np.linspace(brk[0] - 1e12, brk[-1] + 1e12, 4001)
    j = np.clip(np.searchsorted(brk, x, side='right') - 1, 0, len(brk) - 2)
    d = x - brk[j]
    v = ((coef[j, 0] * d + coef[j, 1]) * d + coef[j, 2]) * d + coef[j, 3]
    v[(x < brk[0]) | (x > brk[-1])] = 0
    r = interp1d(f, Ij, kind=kind, bounds_error=False, fill_value=0.0)(x)
    assert np.abs(v - r).max() < 1e-14


def test_analysis_helpers_match_reference():
    """fwhm_precise / analyze_spectral_phase vs the reference's methods run on a
    propagated field (erk43ip_method.py:448-490, 766-808)."""
    from conftest import golden
    from project_b200.analysis import analyze_spectral_phase, fwhm_precise
    g = golden('ref1d_analysis')
    t, A = g['t'], g['A']
    xl, xr, fw = fwhm_precise(t, np.abs(A) ** 2)
    assert np.allclose([xl, xr, fw], g['fwhm'], rtol=1e-12, atol=0)
    w0 = 2 * np.pi * 299792458.0 / 800e-9
    for tag, B, order, thr in (('p4', A, 4, 0.01),
                               ('p3', A * np.exp(1j * float(g['chirp']) * (t - 1e-13) ** 2), 3, 0.05)):
        r = analyze_spectral_phase(B, t, w0, order, thr)
        for k in ('wavelength_nm', 'spectral_intensity', 'mask'):
            assert np.array_equal(r[k], g[f'{tag}_{k}']) if k == 'mask' else np.allclose(r[k], g[f'{tag}_{k}'], rtol=1e-12)
        band = g[f'{tag}_mask']
        assert np.allclose(r['residual_phase'][band], g[f'{tag}_residual_phase'][band], rtol=1e-7, atol=1e-7)
