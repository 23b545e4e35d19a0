"""Batched engine (fs_batch_*): many independent production networks advanced
together by the tile kernels.  The bar is identity: every instance's per-neuron spike
counts equal those of the same network run alone on the plain engine (same
seed, same Philox key), whatever the block plan, the call split or the
tuner's choice."""
import numpy as np
import pytest

from flysim_b200 import netgen, network, sweep

pytestmark = pytest.mark.gpu


def _instances(specs):
    out = []
    for n, gain, drive, seed, delays in specs:
        c = netgen.connectome_fast(n=n, regions=max(2, n // 345), f_lo=drive, f_hi=drive, delays=delays, seed=seed)
        out.append((seed, network.connectome_net(c, gaba_gain=gain, with_delays=delays)))
    return out


SPECS = [  # neurons, inhibitory gain, drive Hz, seed, delays
    (2000, 1.0, 3500.0, 11, True),
    (3500, 0.3, 4000.0, 12, True),
    (700, 0.6, 4500.0, 13, False),  # delays 0: interval of one step
    (5000, 0.8, 3000.0, 14, True),
    (1200, 0.5, 5000.0, 15, True),
]


def _single(fb, na, seed, steps, mode="fp32"):
    e = fb.Engine(na.desc, mode, chunk_steps=10000)
    try:
        e.reset(seed)
        e.run(steps)
        e.sync()
        return e.spike_counts(), e.stats()["spikes"]
    finally:
        e.close()


@pytest.mark.parametrize("mode", ["fp32", "fp64"])
def test_batch_equals_single_runs(built, mode):
    inst = _instances(SPECS)
    steps = 3000
    b = built.Batch([na.desc for _, na in inst], mode=mode, chunk_steps=1000)
    try:
        b.reset([s for s, _ in inst])
        b.run(1000)
        b.run(2000)
        counts = [b.spike_counts(i) for i in range(len(inst))]
        totals = b.spike_totals()
        info = b.info()
    finally:
        b.close()
    assert info["graph"], "the batch launch was not captured into a CUDA graph"
    for i, (seed, na) in enumerate(inst):
        ref, tot = _single(built, na, seed, steps, mode)
        assert tot > 0
        np.testing.assert_array_equal(counts[i], ref, err_msg="instance %d" % i)
        assert int(totals[i]) == int(tot)


def test_tuner_and_plans_do_not_change_results(built):
    inst = _instances(SPECS[:4])
    res = []
    for tune in (False, True):
        b = built.Batch([na.desc for _, na in inst])
        try:
            plan = b.tune(100) if tune else None
            b.reset([s for s, _ in inst])
            b.run(2500)
            res.append([b.spike_counts(i) for i in range(len(inst))])
            if tune:
                assert plan["candidates"] == 6 and plan["blocks"] >= len(inst)
                assert plan["tile_posts"] in (64, 128, 256) and plan["edges_in_flight"] in (4, 8)
        finally:
            b.close()
    for r in res[1:]:
        for a, c in zip(res[0], r):
            np.testing.assert_array_equal(a, c)


def test_sweep_driver_matches_looped_engine(built):
    pts = sweep.sweep_points(count=6, seed=3, n_lo=1000, n_hi=3000)
    bl = [sweep.build_instance(p) for p in pts]
    a = sweep.run_batched(pts, seconds=0.2, built=bl)
    b = sweep.run_looped(pts, seconds=0.2, built=bl)
    for x, y in zip(a["counts"], b["counts"]):
        np.testing.assert_array_equal(x, y)
    assert a["region_rates"].shape == (6, sweep.REGIONS)
    np.testing.assert_array_equal(a["hyper"], b["hyper"])


def test_many_small_instances(built):
    # more instances than the GPU holds blocks: the tile kernels schedule
    # blocks freely, so 600 instances run; two of them equal their solo runs
    inst = _instances([(64 + 3 * i, 1.0, 3000.0, 100 + i, True) for i in range(600)])
    b = built.Batch([na.desc for _, na in inst], chunk_steps=1000)
    try:
        b.reset([s for s, _ in inst])
        b.run(1500)
        counts = [b.spike_counts(i) for i in (0, 599)]
        assert b.info()["blocks"] >= 600
    finally:
        b.close()
    for k, i in enumerate((0, 599)):
        ref, _ = _single(built, inst[i][1], inst[i][0], 1500)
        np.testing.assert_array_equal(counts[k], ref)
