"""CPU checks of the float64 LTP restatement (tests/prod_model.py).

The production engine keeps one conductance per (post, receptor) and turns
each LTP weight change into a correction of that conductance; the
restatement keeps the reference's per-record gates instead
(code/EqsGnl2.cpp:404-502, :1005-1044).  With no record flagged for LTP the
two formulations must agree: the per-record restatement then equals the
aggregated one (prod_model.simulate) step by step, which pins it before the
GPU tests compare the engine against it with LTP on.
"""
import numpy as np

import flysim_b200 as fb
import ltp_nets
import prod_model


def test_per_record_restatement_equals_aggregated_without_ltp():
    for tm in (False, True):
        na = ltp_nets.ltp_net(fb, tm=tm, frac_ltp=0.0)
        sp_a, V_a = prod_model.simulate(na, 1500)
        sp_r, V_r, w = prod_model.simulate_ltp(na, 1500)
        assert sum(x.size for x in sp_a) > 200
        for t in range(1500):
            np.testing.assert_array_equal(sp_r[t], sp_a[t], err_msg="step %d" % t)
        assert np.abs(V_r - V_a).max() < 1e-9
        np.testing.assert_array_equal(w, np.asarray(na.syn["g"], np.float32))


def test_ltp_changes_only_flagged_records_both_ways():
    na = ltp_nets.ltp_net(fb)
    _, _, w = prod_model.simulate_ltp(na, 3000)
    g0 = np.asarray(na.syn["g"], np.float32)
    el = na.syn["ltp"].astype(bool)
    d = w - g0
    assert not np.any(d[~el])
    assert np.count_nonzero(d > 0) > 100 and np.count_nonzero(d < 0) > 100


def test_ltp_rule_forms():
    g = np.array([2.0, 2.0], np.float32)
    out = prod_model.ltp_rule(g, np.array([0.5, 0.5]), np.array([0.1, -0.1]))
    np.testing.assert_array_equal(out, np.array([2.05, 1.9], np.float32))


def test_aggregated_ltp_equals_per_record():
    # the production engine's form of LTP (one conductance per post and
    # receptor, a weight change dg corrected by df*dg*st, NMDA over the
    # current weights, its phase order) against the reference's per-record
    # form: the same spikes, potentials to float64 rounding, the same
    # float32 weights
    for tm in (False, True):
        na = ltp_nets.ltp_net(fb, tm=tm)
        sp_a, V_a, w_a = prod_model.simulate(na, 3000, ltp=True)
        sp_r, V_r, w_r = prod_model.simulate_ltp(na, 3000)
        assert sum(x.size for x in sp_r) > 200
        for t in range(3000):
            np.testing.assert_array_equal(sp_a[t], sp_r[t], err_msg="step %d" % t)
        assert np.abs(V_a - V_r).max() < 1e-9
        np.testing.assert_array_equal(w_a, w_r)
        assert np.count_nonzero(w_r != np.asarray(na.syn["g"], np.float32)) > 100
