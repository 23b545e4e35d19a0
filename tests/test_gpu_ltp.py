"""Long-term plasticity in the production modes (k_prod_ltp) on the GPU.

1. Semantics: recurrent E/I networks with LTP (both rules, LP spike delays
   0-3 steps, 70 % of the records flagged, with and without Tsodyks-Markram
   plasticity) against the float64 per-record restatement
   prod_model.simulate_ltp, the reference's own form of the synapses
   (code/EqsGnl2.cpp:404-502, :1005-1044): identical spikes, membrane
   potentials within 1e-4 mV (FP64) / 2e-3 mV (FP32), the final weights
   (fs_get_weights) bit for bit (LTP works in float in both modes, with
   one rounding per operation, as the reference does).
2. Invariants: a run cut into calls at arbitrary steps, and a run restored
   from a checkpoint, give the same bits as one call.
3. Limits: batches, the tile kernels and synaptic delays are refused.
4. Reference-format connectome networks read from their .conf with -LTP
   (2,000 neurons with the LTP keywords; the 20,000-neuron benchmark
   network with their defaults): FP32 against FP64 (identical raster for
   50 ms, or as long as the same network without LTP) and against the
   reference-order compat engine (population rates within 2 %, mean ISI CV
   within 5 %).
"""
import os

import numpy as np
import pytest

import ltp_nets
import prod_model

pytestmark = pytest.mark.gpu


def _first_diff(a, b):
    for t, (x, y) in enumerate(zip(a, b)):
        if not np.array_equal(x, y):
            return t
    return len(a)


@pytest.mark.parametrize("mode,tol,steps", [("fp64", 1e-4, 3000), ("fp32", 2e-3, 1500)])
@pytest.mark.parametrize("tm", [False, True])
def test_ltp_matches_restatement(built, mode, tol, steps, tm):
    na = ltp_nets.ltp_net(built, tm=tm)
    ref_sp, ref_V, ref_w = prod_model.simulate_ltp(na, steps)
    e = built.Engine(na.desc, mode)
    try:
        assert e.layout()["kernel"] == "ltp"
        e.reset(1)
        sp, V = e.step(steps, want_V=True)
        w = e.weights(na.n_syn)
    finally:
        e.close()
    assert sum(x.size for x in ref_sp) > 200
    t = _first_diff(sp, ref_sp)
    assert t == steps, "spikes differ at step %d" % t
    err = np.abs(V.astype(np.float64) - ref_V)
    assert err.max() < tol, "max |dV| %.3g mV at step %d neuron %d" % (
        err.max(), *np.unravel_index(err.argmax(), err.shape))
    g0 = np.asarray(na.syn["g"], np.float32)
    assert np.count_nonzero(ref_w != g0) > 100  # LTP did change weights
    el = na.syn["ltp"].astype(bool)
    np.testing.assert_array_equal(w[~el], g0[~el])
    np.testing.assert_array_equal(w, ref_w)


def test_ltp_call_split_and_checkpoint(built):
    # LTP weights survive fs_reset (the reference's VarInit leaves g alone,
    # code/EqsGnl2.cpp:339-401), so each run gets a fresh handle
    na = ltp_nets.ltp_net(built, seed=7)
    steps = 1200
    e = built.Engine(na.desc, "fp32")
    try:
        e.reset(3)
        sp1, V1 = e.step(steps, want_V=True)
        w1 = e.weights(na.n_syn)
    finally:
        e.close()
    assert not np.array_equal(w1, np.asarray(na.syn["g"], np.float32))
    # the same run in calls of uneven length, with a checkpoint half way
    e = built.Engine(na.desc, "fp32")
    try:
        e.reset(3)
        sp2, V2 = [], []
        blob = None
        for k in (1, 7, 300, 292, 1, 599):
            a, b = e.step(k, want_V=True)
            sp2 += a
            V2.append(b)
            if len(sp2) == 600:
                blob = e.checkpoint()
        assert _first_diff(sp1, sp2) == steps
        np.testing.assert_array_equal(V1, np.concatenate(V2))
        np.testing.assert_array_equal(w1, e.weights(na.n_syn))
    finally:
        e.close()
    # restored into a fresh handle at step 600, the rest repeats
    assert blob is not None
    f = built.Engine(na.desc, "fp32")
    try:
        f.reset(3)
        f.restore(blob)
        sp3, V3 = f.step(steps - 600, want_V=True)
        assert _first_diff(sp1[600:], sp3) == steps - 600
        np.testing.assert_array_equal(V1[600:], V3)
        np.testing.assert_array_equal(w1, f.weights(na.n_syn))
    finally:
        f.close()


def test_ltp_limits(built):
    na = ltp_nets.ltp_net(built, n=64)
    with pytest.raises(built.FsError, match="tile kernels"):
        built.Engine(na.desc, "fp32", tile_kernels=True)
    with pytest.raises(built.FsError, match="[Bb]atch"):
        built.Batch([na.desc, na.desc], "fp32")
    from flysim_b200 import network
    d = network.desc_from_arrays(na.n, na.dt, na.fields, na.syn["pre"], na.syn["post"], na.syn["rec"],
                                 na.syn["g"], np.full(na.n_syn, 3, np.uint16),
                                 act_ctr=built.DEFAULT_ACT | built.ACT["LTP"], ltp=na.syn["ltp"])
    with pytest.raises(built.FsError, match="delay"):
        built.Engine(d.desc, "fp32")
    # networks without LTP keep their kernels and refuse fs_get_weights
    d0 = network.desc_from_arrays(na.n, na.dt, na.fields, na.syn["pre"], na.syn["post"], na.syn["rec"],
                                  na.syn["g"])
    e = built.Engine(d0.desc, "fp32")
    try:
        assert e.layout()["kernel"] != "ltp"
        with pytest.raises(built.FsError):
            e.weights(na.n_syn)
    finally:
        e.close()


def test_ltp_connectome_conf_fp32_fp64_compat(built, tmp_path):
    # one-neuron populations (every link a single-target record) with the
    # LTP keywords, run with -LTP: the production LTP kernel against FP64
    # and against the reference-order compat engine, 2 s each.  FP32 and
    # FP64 rewrite the weights alike (float LTP arithmetic), so their
    # rasters part no sooner than without LTP (the same network, same modes)
    from flysim_b200 import netgen
    from test_gpu_production import _compare_modes
    # weak potentiation, stronger depression, twice the inhibition: the
    # rates rise from ~13 Hz under LTP but the network does not run away
    # (the reference's own run of it, the CPU oracle: 13.1 Hz in the first
    # 100 ms, 25 Hz in the last of 2 s)
    c = netgen.connectome(n=2000, regions=8, mean_degree=60, seed=11, delays=False, gaba_scale=2.0)
    conf, pro = str(tmp_path / "net.conf"), str(tmp_path / "net.pro")
    netgen.write_connectome(c, conf, with_delays=False, ltp=dict(tLP=30, SpiLPDy=0.1, PosISI=0.001, NegISI=-0.01))
    netgen.write_pro(pro, 2000.0, seeds=(3,), outputs=({"name": "Spikes.dat", "type": "Spike", "pop": "AllPopulation"},))
    groups = np.where(c.excit, 0, 1).astype(np.int64)
    res = {}
    for ltp in (False, True):
        m = built.Model(conf, pro, ltp=ltp)
        desc = m.desc()
        e = built.Engine(desc, "fp32")
        try:
            assert (e.layout()["kernel"] == "ltp") == ltp
        finally:
            e.close()
        res[ltp] = (_compare_modes(built, desc, 2000, groups, 20000, "fp32", "fp64"),
                    _compare_modes(built, desc, 2000, groups, 20000, "fp32", "compat"))
    (first, dr, dcv, rates), (_, dr_c, dcv_c, rates_c) = res[True]
    first_plain = res[False][0][0]
    info = dict(first=first, first_without_ltp=first_plain, rates=rates, dr=dr, dcv=dcv, rates_compat=rates_c,
                dr_compat=dr_c, dcv_compat=dcv_c, rates_without_ltp=res[False][0][3])
    print(info)
    assert first >= min(500, first_plain), info
    assert np.all(rates > 1.0) and dr.max() < 0.02 and dcv.max() < 0.05, info
    assert dr_c.max() < 0.02 and dcv_c.max() < 0.05, info


def test_ltp_connectome20k_d0_fp32_fp64_compat(built, tmp_path):
    # the reference-format 20k connectome (delays 0, read from its .conf)
    # run with -LTP and the keywords' default parameters: FP32 against FP64
    # (identical raster for 50 ms, rates within 2 %) and against the
    # reference-order compat engine (rates within 2 %, ISI CV within 5 %)
    from conftest import generated_case
    from flysim_b200 import netgen
    from test_gpu_production import _compare_modes
    conf, pro = generated_case("connectome20k_d0", tmp_path)
    m = built.Model(conf, pro, ltp=True)
    c = netgen.connectome(n=20000, regions=58, seed=1)
    groups = np.where(c.excit, 0, 1).astype(np.int64)
    desc = m.desc()
    first, dr, dcv, rates = _compare_modes(built, desc, 20000, groups, 20000, "fp32", "fp64")
    assert first >= 500, "rasters differ at step %d (< 50 ms)" % first
    assert np.all(rates > 1.0) and dr.max() < 0.02 and dcv.max() < 0.05, (rates, dr, dcv)
    _, dr, dcv, rates = _compare_modes(built, desc, 20000, groups, 20000, "fp32", "compat")
    assert dr.max() < 0.02 and dcv.max() < 0.05, (rates, dr, dcv)
