"""Property tests (hypothesis) of the host-side planners and table builders (CPU).

The work partitioner, the instance cost model, the quadrature weights of the
spectrum builder, the pulse / beam analysis helpers and the 3D table builder are
driven with random inputs and checked against invariants that hold for every
input (coverage, bounds, monotonicity, agreement with scipy)."""
import math

import numpy as np
import pytest
from hypothesis import given, settings, strategies as st

pytestmark = pytest.mark.filterwarnings('ignore::DeprecationWarning')

SET = settings(max_examples=60, deadline=None)


@SET
@given(costs=st.lists(st.floats(0.0, 1e6, allow_nan=False), min_size=1, max_size=300),
       world=st.integers(1, 8))
def test_partition_covers_every_instance_once_and_balances(costs, world):
    from project_b200.distributed import partition_instances
    parts = partition_instances(costs, world)
    assert len(parts) == world
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(len(costs)))
    assert parts == partition_instances(costs, world)          # deterministic
    loads = [sum(costs[i] for i in p) for p in parts]
    # any greedy list schedule: makespan <= mean load + largest job
    assert max(loads) <= sum(costs) / world + max(costs) + 1e-6 * (1 + sum(costs))
    if world >= len(costs):
        assert all(len(p) <= 1 for p in parts)


@SET
@given(nt=st.sampled_from([64, 256, 1024, 4096, 16384]), L=st.floats(1e-3, 10.0),
       E=st.floats(1e-7, 1e-2), P=st.floats(0.05, 10.0), f=st.floats(1.01, 4.0))
def test_instance_cost_positive_and_monotone(nt, L, E, P, f):
    from project_b200.distributed import instance_cost
    c = instance_cost(nt, L, energy=E, pressure=P)
    assert c > 0 and math.isfinite(c)
    assert instance_cost(nt, L * f, energy=E, pressure=P) >= c
    assert instance_cost(nt, L, energy=E * f, pressure=P) >= c
    assert instance_cost(nt, L, energy=E, pressure=P * f) >= c
    if nt < 16384:
        assert instance_cost(nt * 2, L, energy=E, pressure=P) > c
    assert instance_cost(nt, L) > 0                            # without energy / pressure


@SET
@given(n=st.integers(2, 40), seed=st.integers(0, 2 ** 31 - 1))
def test_simpson_weights_match_scipy(n, seed):
    from scipy.integrate import simpson
    from project_b200.pulses import simpson_weights
    rng = np.random.default_rng(seed)
    x = np.cumsum(rng.uniform(0.1, 2.0, n))
    y = rng.normal(size=n)
    ref = simpson(y, x=x)
    got = float(simpson_weights(x) @ y)
    assert abs(got - ref) <= 1e-10 * (1 + np.sum(np.abs(y)) * (x[-1] - x[0]))


@SET
@given(sigma=st.floats(0.05, 0.3), shift=st.floats(-0.3, 0.3), n=st.integers(64, 2048))
def test_fwhm_of_sampled_gaussians(sigma, shift, n):
    from project_b200.solver3d import fwhm
    t = np.linspace(-1.0, 1.0, n)
    I = np.exp(-0.5 * ((t - shift) / sigma) ** 2)
    w = fwhm(t, I)
    true = 2 * math.sqrt(2 * math.log(2)) * sigma
    dt = t[1] - t[0]
    assert abs(w - true) <= max(0.02 * true, 0.5 * dt)
    assert math.isnan(fwhm(t, -I)) and math.isnan(fwhm(t[:3], I[:3]))


@SET
@given(x0=st.floats(-0.3, 0.3), y0=st.floats(-0.3, 0.3), w=st.floats(0.05, 0.2))
def test_beam_moments_recover_centroid_and_width(x0, y0, w):
    from project_b200.solver3d import beam_moments
    x = np.linspace(-1.0, 1.0, 128)
    X, Y = np.meshgrid(x, x, indexing='ij')
    F = np.exp(-((X - x0) ** 2 + (Y - y0) ** 2) / (2 * w ** 2))
    xm, ym, sx, sy = beam_moments(x, x, F)
    assert abs(xm - x0) < 1e-3 and abs(ym - y0) < 1e-3
    assert abs(sx - w) < 0.02 * w and abs(sy - w) < 0.02 * w


@SET
@given(j=st.integers(1, 66))
def test_noll_indices_are_valid_and_unique(j):
    from project_b200.pulses import noll_nm
    n, m = noll_nm(j)
    assert abs(m) <= n and (n - abs(m)) % 2 == 0
    assert sum(1 for k in range(1, 67) if noll_nm(k) == (n, m)) == 1


@settings(max_examples=25, deadline=None)
@given(N=st.sampled_from([16, 32, 64]), Nt=st.sampled_from([32, 64, 128, 512]),
       half=st.floats(0.5e-3, 4e-3), span=st.floats(50e-15, 500e-15), P=st.floats(0.1, 5.0))
def test_tables3d_invariants(N, Nt, half, span, P):
    from project_b200.media import Argon
    from project_b200.solver3d import tables3d
    x = np.linspace(-half, half, N)
    t = np.linspace(-span, span, Nt)
    tb = tables3d(x, x, t, Argon(800e-9, P, 'double', False))
    assert np.array_equal(tb['K2_perp'], tb['K2_perp'].T)         # square grid
    assert tb['K2_perp'][0, 0] == 0.0 and np.all(tb['K2_perp'] >= 0)
    assert np.all((tb['filter'] > 0) & (tb['filter'] <= 1))
    assert tb['filter'][0] == 1.0
    assert np.all(tb['damp'] >= 0) and np.all(np.isfinite(tb['damp']))
    X, Y = np.meshgrid(x, x, indexing='ij')
    assert np.all(tb['damp'][np.sqrt(X ** 2 + Y ** 2) <= 0.85 * half] == 0)
    assert set(np.unique(tb['valid'])) <= {0, 1}
    v = tb['valid'] == 1
    assert np.all(np.isfinite(tb['k_sq'][v])) and np.all(tb['k_sq'][v] > 0)
