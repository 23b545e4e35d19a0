"""Host side of the sweeps (no GPU): the vectorised connectome generator has
the documented shapes, sweep points are reproducible, and the rate read-out
is the per-region mean."""
import numpy as np

from flysim_b200 import netgen, sweep


def test_connectome_fast_shapes():
    c = netgen.connectome_fast(n=6000, regions=20, seed=4)
    pre, post = c.pre.astype(np.int64), c.post.astype(np.int64)
    assert not np.any(pre == post)
    key = pre * c.n + post
    assert np.unique(key).size == key.size  # distinct (pre, post) pairs
    deg = np.bincount(pre, minlength=c.n)
    assert 100 < deg.mean() < 125  # lognormal mean 120, minus region-size caps
    intra = np.mean(c.region[pre] == c.region[post])
    assert 0.7 < intra < 0.82
    assert abs(c.excit.mean() - 0.7) < 0.03
    assert set(np.unique(c.delay_ms)) <= {1, 2, 3, 4, 5}
    c2 = netgen.connectome_fast(n=6000, regions=20, seed=4)
    assert np.array_equal(c.pre, c2.pre) and np.array_equal(c.weight, c2.weight)


def test_sweep_points_reproducible_and_in_range():
    a = sweep.sweep_points(64, seed=9)
    b = sweep.sweep_points(64, seed=9)
    assert a == b
    assert all(2000 <= p.n <= 20000 and 0.2 <= p.gaba_gain <= 1.5 and 1000 <= p.drive_hz <= 5000 for p in a)
    assert [p.seed for p in a] == list(range(9, 73))


def test_region_rates():
    region = np.array([0, 0, 1, 1, 1, 57])
    counts = np.array([2, 4, 3, 3, 3, 10])
    r = sweep.region_rates(counts, region, 2.0)
    assert r.shape == (sweep.REGIONS,)
    assert r[0] == 1.5 and r[1] == 1.5 and r[57] == 5.0 and r[5] == 0.0


def test_surrogate_parameterisation():
    from flysim_b200 import surrogate as S
    g = S.region_group()
    assert g.shape == (58,) and g.min() == 0 and g.max() == 29
    assert np.all(np.bincount(g)[:28] == 2) and np.all(np.bincount(g)[28:] == 1)
    p = S.sample_params(1000, np.random.default_rng(1))
    x = S.encode(p)
    assert x.shape == (1000, 32) and x.min() >= -1.0 and x.max() <= 1.0
    rates = np.abs(np.random.default_rng(2).normal(20, 30, (5, 58)))
    t = S.targets(rates)
    assert t.shape == (5, 59)
    assert np.allclose(S.decode_rates(t), rates, rtol=1e-5)
    assert np.all(t[:, -1] == (rates.mean(1) > S.HYPER_HZ))
    assert S.rate_error(rates, rates).max() == 0.0
