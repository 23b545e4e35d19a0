"""Production modes (FS_MODE_FP32 / FS_MODE_FP64) on the GPU.

1. Semantics: small deterministic networks (a neuron driven by noiseless
   injection projects through AMPA, GABA and NMDA synapses with delays of
   0-255 steps, with and without Tsodyks-Markram plasticity) against the
   float64 step-by-step restatement in tests/prod_model.py: identical spike
   steps, membrane potentials within 1e-4 mV (FP64) / 2e-3 mV (FP32).
2. FP32 against FP64 on the 20,000-neuron connectome network (58 regions,
   delays 1-5 ms, 10 s): identical raster over the first 50 ms, E and I
   population rates within 2 %, mean ISI CV within 5 %; the same on the
   two-population E/I network (800/200); and production FP32 against the
   reference-order compat path (whose random streams differ) within 2 % /
   5 % on that network.
3. Invariants: results do not depend on how the steps are split into calls,
   on the number of resident blocks, or on repeated runs.
"""
import os

import numpy as np
import pytest

import prod_model

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")

pytestmark = pytest.mark.gpu


def _small_net(fb, delays_lin, delays_gaba, delays_nmda, tm=False, dt=0.1):
    from flysim_b200 import network
    k_lin, k_gaba, k_nmda = len(delays_lin), len(delays_gaba), len(delays_nmda)
    n = 1 + k_lin + k_gaba + k_nmda + 1  # driver, targets, one unconnected control
    f = network.neuron_fields(n, dt, receptors={
        fb.FS_AMPA: dict(Tau=2.0, Vrev=0.0, FExt=0.0),
        fb.FS_GABA: dict(Tau=5.0, Vrev=-80.0, FExt=0.0),
        fb.FS_NMDA: dict(Tau=100.0, TauXT=2.0, Vrev=0.0, FExt=0.0),
    })
    f["act"][0] |= fb.ACT["INJ"]
    f["inj_mean"][0] = 0.8  # fires at about 100 Hz
    post = np.arange(1, n - 1, dtype=np.uint32)
    rec = np.array([fb.FS_AMPA] * k_lin + [fb.FS_GABA] * k_gaba + [fb.FS_NMDA] * k_nmda, np.uint8)
    g = np.array([6.0] * k_lin + [9.0] * k_gaba + [3.0] * k_nmda, np.float32)
    d = np.array(list(delays_lin) + list(delays_gaba) + list(delays_nmda), np.uint16)
    pre = np.zeros(post.size, np.uint32)
    tmd = dict(enabled=(np.arange(n) == 0).astype(np.uint8), U=0.2, tau_rec=200.0, tau_fac=600.0) if tm else None
    return network.desc_from_arrays(n, dt, f, pre, post, rec, g, d, tm=tmd)


SMALL = {
    "d0": ((0, 0, 0), (0,), (0, 0)),  # every delay 0: the single-step kernel (FP32)
    "dmin0": ((0, 7, 23), (3,), (0, 13)),
    "dmin10": ((10, 17, 49, 255), (12,), (10, 31)),
}


@pytest.mark.parametrize("mode,tol", [("fp64", 1e-4), ("fp32", 2e-3)])
@pytest.mark.parametrize("tm", [False, True])
@pytest.mark.parametrize("shape", sorted(SMALL))
def test_small_network_matches_restatement(built, shape, tm, mode, tol):
    na = _small_net(built, *SMALL[shape], tm=tm)
    steps = 3000
    ref_sp, ref_V, ref_I, ref_NS = prod_model.simulate(na, steps, extra=True)
    e = built.Engine(na.desc, mode)
    try:
        e.reset(1)
        sp, V, I, NS = e.step(steps, want_V=True, want_Irep=True, want_nstate=True)
    finally:
        e.close()
    # receptor currents (IsynSep output) and the LIF state word (dV overflow output)
    np.testing.assert_array_equal(NS, ref_NS)
    scale = np.abs(ref_I).max()
    assert np.abs(I.astype(np.float64) - ref_I).max() <= 1e-3 * scale, np.abs(I - ref_I).max() / scale
    assert sum(x.size for x in ref_sp) > 20
    for t in range(steps):
        np.testing.assert_array_equal(sp[t], ref_sp[t], err_msg="spikes differ at step %d" % t)
    err = np.abs(V.astype(np.float64) - ref_V)
    assert err.max() < tol, "max |dV| %.3g mV at step %d neuron %d" % (
        err.max(), *np.unravel_index(err.argmax(), err.shape))
    # every target felt its input, no earlier than its delay allows
    first_spike = next(t for t in range(steps) if ref_sp[t].size)
    moved = np.abs(ref_V - ref_V[:, -1:]) > 1e-9
    dl = np.asarray(na.syn["delay"], np.int64)
    for j, d in enumerate(dl):
        tj = int(np.argmax(moved[:, j + 1]))
        assert moved[:, j + 1].any() and tj >= first_spike + 1 + d


def test_delay_above_ring_limit_is_rejected(built):
    na = _small_net(built, (256,), (), ())
    with pytest.raises(built.FsError, match="255"):
        built.Engine(na.desc, "fp32")


def _raster(e, steps, cap=20_000_000):
    sp, _ = e.step(steps, spike_cap=cap)
    t = np.concatenate([np.full(a.size, i, np.int64) for i, a in enumerate(sp)])
    k = np.concatenate(sp).astype(np.int64)
    return sp, t, k


def _isi_cv(t, k, n, min_isi=4):
    o = np.lexsort((t, k))
    t, k = t[o], k[o]
    same = k[1:] == k[:-1]
    d = np.diff(t)[same].astype(np.float64)
    kk = k[1:][same]
    cnt = np.bincount(kk, minlength=n)
    s1, s2 = np.bincount(kk, d, n), np.bincount(kk, d * d, n)
    ok = cnt >= min_isi
    m = s1 / np.maximum(cnt, 1)
    v = s2 / np.maximum(cnt, 1) - m * m
    return np.where(ok, np.sqrt(np.maximum(v, 0)) / np.maximum(m, 1e-12), np.nan)


def _pop_stats(t, k, groups, n, seconds):
    ng = int(groups.max()) + 1
    rate = np.bincount(groups[k], minlength=ng) / np.bincount(groups, minlength=ng) / seconds
    cv = _isi_cv(t, k, n)
    mcv = np.array([np.nanmean(cv[groups == g]) for g in range(ng)])
    return rate, mcv


def _compare_modes(fb, desc, n, groups, steps, a, b, dt=0.1, same_stream=True):
    runs = {}
    for m in (a, b):
        e = fb.Engine(desc, m, chunk_steps=10000)
        try:
            e.reset(1)
            runs[m] = _raster(e, steps)
        finally:
            e.close()
    seconds = steps * dt * 1e-3
    ra, ca = _pop_stats(runs[a][1], runs[a][2], groups, n, seconds)
    rb, cb = _pop_stats(runs[b][1], runs[b][2], groups, n, seconds)
    first = next((i for i, (x, y) in enumerate(zip(runs[a][0], runs[b][0])) if not np.array_equal(x, y)), steps)
    return first, np.abs(ra / rb - 1), np.abs(ca / cb - 1), rb


def test_fp32_vs_fp64_connectome_20k(built):
    from flysim_b200 import netgen, network
    c = netgen.connectome(n=20000, regions=58, seed=1)
    na = network.connectome_net(c)
    groups = np.where(c.excit, 0, 1).astype(np.int64)
    first, dr, dcv, rates = _compare_modes(built, na.desc, na.n, groups, 100000, "fp32", "fp64")
    assert first >= 500, "rasters differ at step %d (< 50 ms)" % first
    assert np.all(rates > 1.0)
    assert dr.max() < 0.02, dr
    assert dcv.max() < 0.05, dcv


def test_fp32_vs_compat_connectome_20k_delays0(built, tmp_path):
    # the reference-format 20k connectome (delays 0, parsed from its .conf):
    # FP32 production (single-step kernel) against the reference-order compat
    # path, 2 s each with independent random streams: E and I rates within
    # 2 %, mean ISI CV within 5 %; FP32 against FP64 as on the delayed network
    from conftest import generated_case, model_for
    from flysim_b200 import netgen
    generated_case("connectome20k_d0", tmp_path)
    m = model_for(built, "connectome20k_d0", conf_dir=tmp_path)
    c = netgen.connectome(n=20000, regions=58, seed=1)
    groups = np.where(c.excit, 0, 1).astype(np.int64)
    desc = m.desc()
    _, dr, dcv, rates = _compare_modes(built, desc, 20000, groups, 20000, "fp32", "compat")
    assert np.all(rates > 1.0)
    assert dr.max() < 0.02 and dcv.max() < 0.05, (dr, dcv)
    first, dr, dcv, _ = _compare_modes(built, desc, 20000, groups, 20000, "fp32", "fp64")
    assert first >= 500, "rasters differ at step %d (< 50 ms)" % first
    assert dr.max() < 0.02 and dcv.max() < 0.05, (dr, dcv)


def test_two_population_fp32_vs_fp64_and_compat(built):
    m = built.Model(os.path.join(GOLDEN, "two_pop", "net.conf"), os.path.join(GOLDEN, "two_pop", "net.pro"))
    desc = m.desc()
    groups = np.r_[np.zeros(800, np.int64), np.ones(200, np.int64)]
    first, dr, dcv, rates = _compare_modes(built, desc, 1000, groups, 100000, "fp32", "fp64")
    assert first >= 500, "rasters differ at step %d (< 50 ms)" % first
    assert np.all(rates > 5.0)
    assert dr.max() < 0.02 and dcv.max() < 0.05, (dr, dcv)
    # production against the reference-order path (independent random streams)
    _, dr, dcv, _ = _compare_modes(built, desc, 1000, groups, 100000, "fp32", "compat")
    assert dr.max() < 0.02 and dcv.max() < 0.05, (dr, dcv)


def test_gap_junctions_fp32_fp64_and_compat(built, tmp_path):
    # E/I network with gap junctions (E-E and I-I): the production modes run
    # them with the reference's one-step lag (interval 1); the coupling must
    # matter (compat rates with and without it differ) and the production
    # rates and ISI CVs hold to compat and to each other
    from flysim_b200 import netgen
    pro = os.path.join(GOLDEN, "two_pop", "net.pro")
    groups = np.r_[np.zeros(800, np.int64), np.ones(200, np.int64)]
    rates = {}
    for gap in (0.0, 0.002):
        conf = str(tmp_path / ("g%s.conf" % gap))
        netgen.write_two_pop(conf, gap=gap)
        m = built.Model(conf, pro)
        e = built.Engine(m.desc(), "compat", chunk_steps=10000)
        try:
            e.reset(1)
            _, t, k = _raster(e, 20000)
        finally:
            e.close()
        rates[gap] = _pop_stats(t, k, groups, 1000, 2.0)[0]
    assert rates[0.002][0] < 0.85 * rates[0.0][0], rates  # the gap coupling lowers the E rate
    desc = m.desc()
    first, dr, dcv, r = _compare_modes(built, desc, 1000, groups, 100000, "fp32", "fp64")
    assert first >= 500, "rasters differ at step %d (< 50 ms)" % first
    assert np.all(r > 5.0) and dr.max() < 0.02 and dcv.max() < 0.05, (r, dr, dcv)
    _, dr, dcv, _ = _compare_modes(built, desc, 1000, groups, 100000, "fp32", "compat")
    assert dr.max() < 0.02 and dcv.max() < 0.05, (dr, dcv)


def _conn_net(n=2000, seed=3):
    from flysim_b200 import netgen, network
    c = netgen.connectome(n=n, regions=max(2, n // 345), seed=seed)
    return network.connectome_net(c)


def test_results_do_not_depend_on_call_split_or_blocks(built):
    # calls of one step mid-run take the single-step NMDA pull, the others
    # the window pull: a step's sums must not depend on which one it falls in
    na = _conn_net()
    steps = 3000
    ref = None
    for bps, splits in ((0, [steps]), (1, [1, 7, 100, 892, 2000]), (2, [1500, 1500]),
                        (0, [503, 1, 1, 1, 14, 1, 479, 1, 999, 1000])):
        e = built.Engine(na.desc, "fp32", chunk_steps=256, blocks_per_sm=bps)
        try:
            e.reset(5)
            sp = []
            for k in splits:
                sp += e.step(k)[0]
            V = e.state()[0]
        finally:
            e.close()
        if ref is None:
            ref, Vref = sp, V
            assert sum(x.size for x in sp) > 100
        else:
            assert all(np.array_equal(x, y) for x, y in zip(ref, sp)), "blocks/SM %d, splits %s" % (bps, splits)
            assert np.array_equal(V.view(np.uint32), Vref.view(np.uint32)), "blocks/SM %d, splits %s" % (bps, splits)


@pytest.mark.parametrize("mode,tm", [("fp32", False), ("fp32", True), ("fp64", False)])
def test_checkpoint_resumes_bit_for_bit(built, mode, tm):
    # a drive event before the save, delays in flight in the ring, TM state:
    # a fresh handle restored from the checkpoint continues exactly as the
    # saved one, and the saved handle can be rewound to it
    from flysim_b200 import netgen, network
    c = netgen.connectome(n=2000, regions=5, seed=3)
    na = network.connectome_net(c, tm=tm)
    e = built.Engine(na.desc, mode, chunk_steps=256)
    f = built.Engine(na.desc, mode, chunk_steps=256)
    try:
        e.reset(7)
        e.step(1234)
        e.set_drive(0, 300, 0, 0.05)
        e.step(17)
        ck = e.checkpoint()
        a = e.step(1500)[0]
        Va = e.state()[0].copy()
        f.reset(99)  # another seed: the checkpoint carries the drive stream key
        f.restore(ck)
        assert f.stats()["steps"] == 1251
        b = f.step(1500)[0]
        assert sum(x.size for x in a) > 100
        assert all(np.array_equal(x, y) for x, y in zip(a, b))
        assert np.array_equal(f.state()[0].view(np.uint8), Va.view(np.uint8))
        assert f.stats()["spikes"] == e.stats()["spikes"]
        e.restore(ck)
        assert all(np.array_equal(x, y) for x, y in zip(a, e.step(1500)[0]))
    finally:
        e.close()
        f.close()
    # a checkpoint of another network, or a compat handle, is refused
    other = network.connectome_net(netgen.connectome(n=2100, regions=5, seed=4), tm=tm)
    g = built.Engine(other.desc, mode)
    try:
        with pytest.raises(built.FsError) as ex:
            g.restore(ck)
        assert ex.value.code == built.FS_ERR_ARG
    finally:
        g.close()


def test_bounded_wait_reports_timeout_and_device_stays_usable(built):
    # a grid barrier that a missing block never reaches: the wait gives up
    # after its poll limit, the host reads the error word as FS_ERR_TIMEOUT,
    # and the next engine runs normally
    rc = built.lib().fs_debug_barrier_timeout(1 << 14)
    assert rc == built.FS_ERR_TIMEOUT, rc
    assert built.lib().fs_debug_barrier_timeout(0) == built.FS_ERR_ARG
    na = _conn_net()
    e = built.Engine(na.desc, "fp32")
    try:
        e.reset(5)
        spk = e.step(3000)[0]
        assert sum(x.size for x in spk) > 100
    finally:
        e.close()


def _both_kernels(fb, desc, steps_split, events=None, seed=5, **kw):
    """Runs a delays-0 network on the single-step kernel and on the interval
    kernel; returns both runs' (spikes per step, final V, spike counts)."""
    out = []
    for interval in (False, True):
        e = fb.Engine(desc, "fp32", chunk_steps=700, interval_kernel=interval, **kw)
        try:
            assert e.layout()["single_step"] == (not interval)
            e.reset(seed)
            if events:
                events(e)
            sp = []
            for k in steps_split:
                sp += e.step(k)[0]
            out.append((sp, e.state()[0].copy(), e.spike_counts()))
        finally:
            e.close()
    return out


@pytest.mark.parametrize("variant", ["plain", "tm", "events"])
def test_single_step_kernel_equals_interval_kernel(built, variant):
    # the 20k connectome with delays 0: shared-memory NMDA copies, deliveries
    # by the targets' blocks and the ring hand-over between launches (calls
    # of 1 step, chunks of 700) against the interval kernel, bit for bit
    from flysim_b200 import netgen, network
    c = netgen.connectome(n=20000, regions=58, seed=1)
    na = network.connectome_net(c, with_delays=False, tm=(variant == "tm"))

    def events(e):
        e.set_drive(0, 5000, built.FS_NMDA, 0.02)
        e.set_drive(3000, 9000, built.FS_GABA, 0.05)
        e.set_injection(10000, 4000, 0.05, 0.3)
        e.set_act(10000, 4000, 0, built.ACT["INJ"])
    (a, Va, ca), (b, Vb, cb) = _both_kernels(built, na.desc, [1, 999, 1, 1500, 499],
                                             events=events if variant == "events" else None)
    assert sum(x.size for x in a) > 1000
    for t, (x, y) in enumerate(zip(a, b)):
        np.testing.assert_array_equal(x, y, err_msg="step %d" % t)
    assert np.array_equal(Va.view(np.uint32), Vb.view(np.uint32))
    np.testing.assert_array_equal(ca, cb)


@pytest.mark.parametrize("mode", ["fp32", "fp64"])
def test_tile_kernels_equal_interval_kernel(built, mode):
    # a 30k connectome with delays of 1-5 ms and Tsodyks-Markram plasticity
    # on the tile kernels (launch pairs over tiles of posts; FP32 stages each
    # tile's ring slots in shared memory) against the persistent interval
    # kernel, with calls that leave batches unaligned and partial: spikes,
    # membrane potentials and spike counts bit for bit
    from flysim_b200 import netgen, network
    c = netgen.connectome(n=30000, regions=58, seed=2)
    na = network.connectome_net(c, tm=True)
    runs = []
    for tiles in (False, True):
        e = built.Engine(na.desc, mode, chunk_steps=700, tile_kernels=tiles)
        try:
            assert e.layout()["kernel"] == ("tiles" if tiles else "interval")
            e.reset(4)
            sp = []
            for k in (1, 999, 7, 1493):
                sp += e.step(k)[0]
            runs.append((sp, e.state()[0].copy(), e.spike_counts()))
        finally:
            e.close()
    (a, Va, ca), (b, Vb, cb) = runs
    assert sum(x.size for x in a) > 1000
    for t, (x, y) in enumerate(zip(a, b)):
        np.testing.assert_array_equal(x, y, err_msg="step %d" % t)
    assert np.array_equal(Va.view(np.uint32), Vb.view(np.uint32))
    np.testing.assert_array_equal(ca, cb)


@pytest.mark.parametrize("case", ["two_pop", "two_pop_std", "two_pop_stp", "conn"])
def test_single_step_kernel_on_reference_networks(built, case):
    # networks read from the reference's own .conf format (delays 0, the
    # reference's STD / STP plasticity, group and one-neuron populations)
    from conftest import model_for
    m = model_for(built, case)
    (a, Va, ca), (b, Vb, cb) = _both_kernels(built, m.desc(), [1, 1200, 799])
    assert sum(x.size for x in a) > 20
    for t, (x, y) in enumerate(zip(a, b)):
        np.testing.assert_array_equal(x, y, err_msg="step %d" % t)
    assert np.array_equal(Va.view(np.uint32), Vb.view(np.uint32))
    np.testing.assert_array_equal(ca, cb)


@pytest.mark.parametrize("mode", ["fp64", "fp32"])
def test_gating_variables(built, mode):
    # GatingVariable output in the production modes: a single-target
    # record's gate is its presynaptic neuron's gate (NMDA: x and s).  (1)
    # Against the gate recurrences (code/EqsGnl2.cpp:404-502) run on the
    # host over the engine's own spike trains: st <- st + 1 on a spike of
    # the record's source, st * dfst(post) otherwise; NMDA x <- x + 1 or
    # x * dfxt(post), s <- dfst s + efst as x (1 - s).  (2) Against the
    # reference-order compat path on a deterministic drive (no Poisson input,
    # noiseless injection) for as long as the two runs' spikes agree.
    from conftest import model_for
    m = model_for(built, "conn")
    d = m.desc()
    lay = d.contents.compat.contents
    nv = d.contents.neurons
    n = nv.n
    sel, recs = [], []
    for r in range(5):
        L = lay.rec[r]
        for e in range(L.n_recs):
            if L.rec_pre[e] in (361, 367, 390, 5, 77):
                sel.append((r << 28) | e)
                recs.append((r, L.rec_src[e] if L.rec_src else L.rec_pre[e], L.rec_post[e]))
    assert len(sel) > 20 and any(r == built.FS_NMDA for r, _, _ in recs)
    steps = 2000
    out = {}
    for md in ("compat", mode):
        e = built.Engine(d, md, chunk_steps=700)
        try:
            e.reset(m.seed())
            for r in range(5):
                e.set_drive(0, n, r, 0.0)
            for k in range(0, n, 40):  # 0.75 .. 1.11 nA, well above threshold
                e.set_injection(k, min(40, n - k), 0.75 + 0.04 * ((k // 40) % 10), 0.0)
            e.set_act(0, n, 0, built.ACT["INJ"])  # as the protocol driver's injection event does
            out[md] = e.step_gv(steps, sel)
        finally:
            e.close()
    sb, gs_b, gx_b = out[mode]
    assert sum(x.size for x in sb) > 500
    # (1) the recurrences over the engine's own spikes, in float64
    spk = np.zeros((steps, n), bool)
    for t, x in enumerate(sb):
        spk[t, x] = True
    dfst = np.ctypeslib.as_array(nv.dfst, (5 * n,)).reshape(5, n).astype(np.float64)
    dfxt = np.ctypeslib.as_array(nv.nmda_dfxt, (n,)).astype(np.float64)
    efas = (np.ctypeslib.as_array(nv.nmda_efst, (n,)) * np.ctypeslib.as_array(nv.nmda_as, (n,))).astype(np.float64)
    ref_s = np.zeros((steps, len(sel)))
    ref_x = np.zeros((steps, len(sel)))
    for i, (r, src, post) in enumerate(recs):
        st = x = 0.0
        for t in range(steps):
            if r == built.FS_NMDA:
                x = x + 1.0 if spk[t, src] else x * dfxt[post]
                st = dfst[r, post] * st + efas[post] * x * (1.0 - st)
                ref_x[t, i] = x
            else:
                st = st + 1.0 if spk[t, src] else st * dfst[r, post]
            ref_s[t, i] = st
    assert np.abs(ref_s).max() > 0.5 and np.abs(ref_x).max() > 0.5
    # the output is float (FP64 state rounds once to it); FP32 state: each of
    # up to 2,000 decays rounds once (about 1e-4 in all)
    tol = 2e-7 if mode == "fp64" else 5e-4
    np.testing.assert_allclose(gs_b, ref_s, rtol=tol, atol=tol * np.abs(ref_s).max())
    np.testing.assert_allclose(gx_b, ref_x, rtol=tol, atol=tol * np.abs(ref_x).max())
    # (2) the compat path's records while the spike trains agree
    sa, gs_a, gx_a = out["compat"]
    first = next((t for t in range(steps) if not np.array_equal(sa[t], sb[t])), steps)
    np.testing.assert_allclose(gs_b[:first], gs_a[:first], rtol=5e-4, atol=5e-4 * np.abs(ref_s).max())
    np.testing.assert_allclose(gx_b[:first], gx_a[:first], rtol=5e-4, atol=5e-4 * np.abs(ref_x).max())


def test_checkpoint_refused_after_a_wait_gave_up(built):
    # the failure is made on the host: the handle's device error word is set
    # as a bounded wait that gave up sets it (no kernel is stopped or hung);
    # the state is then half an interval, so fs_sync reports the timeout and
    # fs_checkpoint_save saves nothing; a reset clears the word
    na = _conn_net()
    e = built.Engine(na.desc, "fp32")
    try:
        e.reset(5)
        e.run(500)
        e.inject_wait_failure()
        with pytest.raises(built.FsError) as ex:
            e.checkpoint()
        assert ex.value.code == built.FS_ERR_TIMEOUT
        with pytest.raises(built.FsError) as ex:
            e.sync()
        assert ex.value.code == built.FS_ERR_TIMEOUT
        e.reset(5)
        e.run(500)
        assert len(e.checkpoint()) > 0
    finally:
        e.close()


def test_checkpoint_needs_a_production_mode(built):
    m = built.Model(os.path.join(GOLDEN, "small", "net.conf"), os.path.join(GOLDEN, "small", "net.pro"))
    e = built.Engine(m.desc(), "compat")
    try:
        with pytest.raises(built.FsError) as ex:
            e.checkpoint()
        assert ex.value.code == built.FS_ERR_UNSUPPORTED
    finally:
        e.close()


def test_seed_and_key_change_the_drive(built):
    na = _conn_net()
    out = []
    for seed, key in ((5, 0), (6, 0), (5, 99)):
        e = built.Engine(na.desc, "fp32", philox_key=key)
        try:
            e.reset(seed)
            out.append(e.step(500)[0])
        finally:
            e.close()
    same = lambda a, b: all(np.array_equal(x, y) for x, y in zip(a, b))  # noqa: E731
    assert not same(out[0], out[1]) and not same(out[0], out[2])


def test_cli_production_modes_match_compat_statistics(built, tmp_path):
    """The drop-in command line in FS_MODE_FP32 / FP64 on a reference-format
    network (E=800 / I=200, 2 s): the same output files (line counts of the
    rate files), population spike counts within 3 % of the reference-order
    compat run."""
    import subprocess
    from flysim_b200 import netgen
    netgen.write_two_pop(str(tmp_path / "net.conf"))
    netgen.write_pro(str(tmp_path / "net.pro"), 2000.0, seeds=(3,), outputs=(
        {"name": "Spikes.dat", "type": "Spike", "pop": "AllPopulation"},))
    exe = os.path.join(ROOT, "flysim_b200", "_build", "flysim")
    counts = {}
    for mode in ("compat", "fp32", "fp64"):
        d = tmp_path / mode
        d.mkdir()
        for f in ("net.conf", "net.pro"):
            os.symlink(str(tmp_path / f), str(d / f))
        r = subprocess.run([exe, "-conf", "net.conf", "-pro", "net.pro", "-mode", mode], cwd=str(d),
                           capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr
        sp = np.loadtxt(str(d / "Spikes.dat"), ndmin=2)
        k = sp[:, 1].astype(np.int64)
        counts[mode] = np.array([np.count_nonzero(k < 800), np.count_nonzero(k >= 800)], np.float64)
    assert np.all(counts["compat"] > 1000), counts
    for mode in ("fp32", "fp64"):
        rel = np.abs(counts[mode] / counts["compat"] - 1)
        assert rel.max() < 0.03, (mode, counts)
