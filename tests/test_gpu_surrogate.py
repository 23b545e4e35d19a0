"""Surrogate pipeline on the GPU: the batched simulator with per-point drive
and gains equals the plain engine run per point (bit for bit), the gains act
in the expected direction, and a small end-to-end run (simulate, train on
the tensor cores, screen, verify) beats the method without the learned
network (a linear least-squares response) on the audit set and enriches
hyperactive points among its top candidates."""
import numpy as np
import pytest

from flysim_b200 import surrogate as S

pytestmark = pytest.mark.gpu


def test_batched_points_equal_plain_engine(built):
    sim = S.Simulator(neurons=1500, batch=4, seconds=0.3, tune=False)
    try:
        p = S.sample_params(4, np.random.default_rng(5))
        rb = sim.rates(p, seed0=7)
        for i in range(4):
            rs, _ = sim.single_rates(p[i], 7 + i)
            np.testing.assert_array_equal(rb[i], rs)
            assert rs.sum() > 0
    finally:
        sim.close()


def test_inhibitory_gain_lowers_rates(built):
    sim = S.Simulator(neurons=1500, batch=4, seconds=0.3, tune=False)
    try:
        p = np.tile(S.sample_params(1, np.random.default_rng(6)), (4, 1))
        p[:, S.GROUPS] = 1.0
        p[:, S.GROUPS + 1] = [0.2, 0.6, 1.0, 1.5]
        r = sim.rates(p, seed0=3).mean(1)
        assert r[0] > r[1] > r[2] > r[3], r
    finally:
        sim.close()


def test_small_pipeline_beats_linear_response(built):
    r = S.run(neurons=2000, seconds=0.5, n_train=8192, epochs=300, grid=20000, audit=256, looped_sample=1)
    assert r["audit_rate_error_mean"] < r["audit_rate_error_linear_mean"], r
    assert r["top_verified_hyper_fraction"] >= r["audit_hyper_fraction"], r
    assert r["audit_hyper_accuracy"] > 0.85, r
    assert r["speedup_vs_plain_looped"] > 1.0, r
