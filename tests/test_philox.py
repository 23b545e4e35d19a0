"""The production modes' external drive, pinned bit for bit.

The reference draws its external input from one sequential std::mt19937
stream (EqsGnl2::BgInit, code/EqsGnl2.cpp:284-337) and its injection noise
from a ziggurat (code/StiExt.h:214-218).  The production modes replace both
with counter-based Philox-4x32-10 draws keyed by (step, neuron); the compat
mode keeps the reference's own streams.  The chain is checked link by link:

1. CPU: the restatement oracle/fs_philox.c against an independent Philox
   implementation, cuRAND's host generator (CURAND_RNG_PSEUDO_PHILOX4_32_10,
   run on the CPU): block k of a generator seeded with s is Philox with key
   (s_lo, s_hi) and counter ((k >> 16) mod 2^32, k >> 48, k mod 2^16, 0), which
   exercises both key words and counter words 0-2 (word 3 enters the first
   round exactly as word 1 does, with the other key word).
2. CPU: the restated drive draws have the probabilities and the normal law
   they claim (binomial and normal bounds).
3. GPU: the device Philox equals the restatement on arbitrary counters and
   keys, bit for bit; the engine's drive draws (fs_debug_drive, the function
   its kernels call) equal the restatement: hit bitmaps bit for bit, the
   injection current within 4 units of rounding of its state type (the
   device's log and cospi and glibc's log and cos may differ in the last bit
   of the double).
4. GPU: a network with external drive on every receptor and injection noise,
   run by the engine, equals the float64 step-by-step restatement
   (tests/prod_model.py) fed with those draws: identical spikes for 3,000
   steps, |dV| < 1e-4 mV (FP64) / 2e-3 mV (FP32).
"""
import ctypes as C
import ctypes.util
import os

import numpy as np
import pytest

import prod_model

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _curand():
    for p in ("/usr/local/cuda/lib64/libcurand.so.10", ctypes.util.find_library("curand")):
        if p:
            try:
                return C.CDLL(p)
            except OSError:
                pass
    return None


@pytest.fixture(scope="module")
def phil(oracle):
    oracle.oracle_philox4x32_10.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    oracle.oracle_drive_key.argtypes = [C.c_uint64, C.c_uint32, C.c_void_p]
    oracle.oracle_drive_draws.argtypes = [C.c_void_p, C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
                                          C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p,
                                          C.c_void_p]
    return oracle


def oracle_philox(L, ctr, key):
    ctr = np.ascontiguousarray(ctr, np.uint32).reshape(-1, 4)
    key = np.ascontiguousarray(key, np.uint32).reshape(-1, 2)
    out = np.zeros_like(ctr)
    for i in range(ctr.shape[0]):
        L.oracle_philox4x32_10(ctr[i].ctypes.data, key[i].ctypes.data, out[i].ctypes.data)
    return out


def oracle_key(L, user_key, seed):
    k = np.zeros(2, np.uint32)
    L.oracle_drive_key(user_key, seed, k.ctypes.data)
    return k


def oracle_draws(L, key, t0, nsteps, first, count, f, fp64):
    n = f["act"].size
    pb = np.ascontiguousarray(f["pb"], np.float32)
    act = np.ascontiguousarray(f["act"], np.uint32)
    mean = np.ascontiguousarray(f["inj_mean"], np.float32)
    std = np.ascontiguousarray(f["inj_std"], np.float32)
    hits = np.zeros((nsteps, count), np.uint8)
    gauss = np.zeros((nsteps, count), np.float64)
    L.oracle_drive_draws(key.ctypes.data, t0, nsteps, first, count, n, pb.ctypes.data, act.ctypes.data,
                         mean.ctypes.data, std.ctypes.data, 1 if fp64 else 0, hits.ctypes.data, gauss.ctypes.data)
    return hits, gauss


# ---- 1. restatement against cuRAND's host Philox (CPU) ----------------------
def _curand_blocks(L, seed, offset_blocks, k):
    g = C.c_void_p()
    assert L.curandCreateGeneratorHost(C.byref(g), 161) == 0  # CURAND_RNG_PSEUDO_PHILOX4_32_10
    try:
        assert L.curandSetPseudoRandomGeneratorSeed(g, C.c_ulonglong(seed)) == 0
        assert L.curandSetGeneratorOffset(g, C.c_ulonglong(4 * offset_blocks)) == 0
        out = np.zeros(4 * k, np.uint32)
        assert L.curandGenerate(g, out.ctypes.data_as(C.c_void_p), C.c_size_t(out.size)) == 0
    finally:
        L.curandDestroyGenerator(g)
    return out.reshape(k, 4)


@pytest.mark.parametrize("seed", [0, 1, 12345, 0xDEADBEEFCAFEBABE, 2 ** 64 - 1])
@pytest.mark.parametrize("offset", [0, 65536 - 100, 2 ** 32 + 3, 2 ** 48 + 2 ** 40 + 7])
def test_oracle_philox_matches_curand(phil, seed, offset):
    cr = _curand()
    if cr is None:
        pytest.skip("libcurand not found")
    k = 1024
    ref = _curand_blocks(cr, seed, offset, k)
    blk = np.arange(offset, offset + k, dtype=np.uint64)
    ctr = np.stack([(blk >> 16) & 0xFFFFFFFF, blk >> 48, blk & 0xFFFF, np.zeros_like(blk)], 1).astype(np.uint32)
    key = np.tile(np.array([seed & 0xFFFFFFFF, seed >> 32], np.uint32), (k, 1))
    np.testing.assert_array_equal(oracle_philox(phil, ctr, key), ref)


# ---- 2. the restated draws obey their laws (CPU) ----------------------------
def test_oracle_draw_statistics(phil, built):
    from flysim_b200 import network
    n, steps = 64, 4000
    f = network.neuron_fields(n, 0.1, receptors={
        built.FS_AMPA: dict(FExt=2400.0), built.FS_GABA: dict(FExt=800.0), built.FS_NMDA: dict(FExt=300.0),
        built.FS_ACH: dict(FExt=50.0), built.FS_GCL: dict(FExt=5000.0)})
    f["act"][: n // 2] |= built.ACT["INJ"]
    f["inj_mean"][:] = 0.25
    f["inj_std"][:] = 0.5
    key = oracle_key(phil, 0x123456789ABCDEF, 7)
    hits, gauss = oracle_draws(phil, key, 1000, steps, 0, n, f, fp64=True)
    pb = f["pb"].reshape(5, n)[:, 0].astype(np.float64)
    for r in range(5):
        m = steps * n
        k = np.count_nonzero(hits & (1 << r))
        assert abs(k - m * pb[r]) < 5 * np.sqrt(m * pb[r] * (1 - pb[r])) + 1, (r, k, m * pb[r])
    z = (gauss[:, : n // 2] - 0.25) / 0.5
    assert np.all(gauss[:, n // 2:] == 0)
    assert abs(z.mean()) < 5 / np.sqrt(z.size)
    assert abs(z.var() - 1) < 5 * np.sqrt(2 / z.size)
    # a step or neuron changes every draw; the same (key, step, neuron) repeats
    h2, g2 = oracle_draws(phil, key, 1000, steps, 0, n, f, fp64=True)
    assert np.array_equal(h2, hits) and np.array_equal(g2, gauss)
    h3, _ = oracle_draws(phil, key, 1001, steps, 0, n, f, fp64=True)
    assert np.array_equal(h3[:-1], hits[1:]) and not np.array_equal(h3, hits)


# ---- 3. device against the restatement (GPU) --------------------------------
@pytest.mark.gpu
def test_device_philox_matches_oracle(phil, built):
    rng = np.random.default_rng(11)
    k = 20000
    ctr = rng.integers(0, 2 ** 32, (k, 4), dtype=np.uint64).astype(np.uint32)
    key = rng.integers(0, 2 ** 32, (k, 2), dtype=np.uint64).astype(np.uint32)
    ctr[:16] = 0
    ctr[16:32] = 0xFFFFFFFF
    key[:8] = 0
    np.testing.assert_array_equal(built.debug_philox(ctr, key), oracle_philox(phil, ctr, key))


def _driven_net(fb, n=600, seed=5):
    from flysim_b200 import netgen, network
    c = netgen.connectome(n=n, regions=4, mean_degree=40, seed=seed)
    return c, network.connectome_net(c)


def _events(fb, e, f, n):
    """Drive and injection events as the protocol driver would apply them;
    f (the field arrays) is updated to the values the handle holds."""
    pb = f["pb"].reshape(5, n)
    for rec, lo, hi, hz in ((fb.FS_GABA, 0, n // 3, 900.0), (fb.FS_NMDA, n // 4, n // 2, 400.0),
                            (fb.FS_ACH, n // 2, n, 150.0), (fb.FS_GCL, 0, n // 5, 2000.0)):
        p = np.float32(hz) * np.float32(0.1) * np.float32(1e-3)
        e.set_drive(lo, hi - lo, rec, float(p))
        pb[rec, lo:hi] = p
    f["pb"] = pb.ravel()
    lo, hi = n // 3, (2 * n) // 3
    mean, std = np.float32(0.05), np.float32(0.4)
    e.set_injection(lo, hi - lo, float(mean), float(std))
    e.set_act(lo, hi - lo, 0, fb.ACT["INJ"])
    f["act"] = f["act"].copy()
    f["act"][lo:hi] |= fb.ACT["INJ"]
    f["inj_mean"] = f["inj_mean"].copy()
    f["inj_std"] = f["inj_std"].copy()
    f["inj_mean"][lo:hi] = mean
    f["inj_std"][lo:hi] = std


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["fp32", "fp64"])
def test_device_drive_matches_oracle(phil, built, mode):
    c, na = _driven_net(built)
    n = na.n
    f = {k: np.array(v, copy=True) for k, v in na.fields.items()}
    user_key, seed = 0xFEEDFACE12345678, 42
    e = built.Engine(na.desc, mode, philox_key=user_key)
    try:
        e.reset(seed)
        _events(built, e, f, n)
        key = oracle_key(phil, user_key, seed)
        for t0, steps, first, count in ((0, 300, 0, n), (2 ** 32 - 7, 20, 17, 300), (123456, 5, n - 1, 1)):
            hd, gd = e.drive_draws(t0, steps, first, count)
            ho, go = oracle_draws(phil, key, t0, steps, first, count, f, fp64=(mode == "fp64"))
            np.testing.assert_array_equal(hd, ho)
            assert np.count_nonzero(hd) > 0
            inj = (f["act"][first:first + count] & built.ACT["INJ"]) != 0
            assert np.all(gd[:, ~inj] == 0) and np.all(go[:, ~inj] == 0)
            if inj.any():
                # mean + std z: within 4 units of rounding of the larger of
                # its two terms (a result near 0 cancels; its own ulp is no
                # measure of the inputs' rounding)
                eps = np.finfo(np.float32 if mode == "fp32" else np.float64).eps
                mean = f["inj_mean"][first:first + count][inj].astype(np.float64)
                scale = np.maximum(np.abs(mean), np.abs(go[:, inj] - mean))
                assert np.all(np.abs(gd[:, inj] - go[:, inj]) <= 4 * eps * scale)
                if mode == "fp32":  # the float rounding hides the double's last bits
                    assert np.mean(gd[:, inj] == go[:, inj]) > 0.99
    finally:
        e.close()


# ---- 4. a driven, noisy network against the float64 restatement (GPU) -------
def _small_driven_net(fb):
    from flysim_b200 import network
    rng = np.random.default_rng(21)
    n = 48
    f = network.neuron_fields(n, 0.1, receptors={
        fb.FS_AMPA: dict(Tau=2.0, Vrev=0.0, FExt=1800.0, ExtEff=2.1),
        fb.FS_GABA: dict(Tau=5.0, Vrev=-80.0, FExt=400.0, ExtEff=1.5),
        fb.FS_NMDA: dict(Tau=100.0, TauXT=2.0, Vrev=0.0, FExt=200.0, ExtEff=0.4),
    })
    f["act"][::3] |= fb.ACT["INJ"]
    f["inj_mean"][::3] = 0.1
    f["inj_std"][::3] = 0.3
    m = 600
    pre = rng.integers(0, n, m).astype(np.uint32)
    post = rng.integers(0, n, m).astype(np.uint32)
    keep = pre != post
    pre, post = pre[keep], post[keep]
    rec = np.where(pre < 36, np.where(rng.random(pre.size) < 0.5, fb.FS_AMPA, fb.FS_NMDA), fb.FS_GABA).astype(np.uint8)
    g = np.where(rec == fb.FS_GABA, 3.0, np.where(rec == fb.FS_AMPA, 2.0, 0.5)).astype(np.float32)
    d = rng.integers(0, 30, pre.size).astype(np.uint16)
    return network.desc_from_arrays(n, 0.1, f, pre, post, rec, g, d)


@pytest.mark.gpu
@pytest.mark.parametrize("mode,tol", [("fp64", 1e-4), ("fp32", 2e-3)])
def test_driven_network_matches_restatement(built, mode, tol):
    na = _small_driven_net(built)
    steps = 3000
    e = built.Engine(na.desc, mode)
    try:
        e.reset(9)
        hits, gauss = e.drive_draws(0, steps)
        sp, V = e.step(steps, want_V=True)
    finally:
        e.close()
    ref_sp, ref_V = prod_model.simulate(na, steps, drive=(hits, gauss))
    assert sum(x.size for x in ref_sp) > 100
    for t in range(steps):
        np.testing.assert_array_equal(sp[t], ref_sp[t], err_msg="spikes differ at step %d" % t)
    err = np.abs(V.astype(np.float64) - ref_V)
    assert err.max() < tol, "max |dV| %.3g mV at step %d neuron %d" % (
        err.max(), *np.unravel_index(err.argmax(), err.shape))
