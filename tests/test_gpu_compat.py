"""GPU compat mode against the reference (needs a B200).

FS_MODE_COMPAT reproduces the reference's arithmetic and random streams, so
its output files must equal, byte for byte, the files the reference built
from its sources wrote (tests/golden), and its state must equal the CPU
oracle's after every step.
"""
import os
import subprocess

import numpy as np
import pytest

from conftest import (GOLDEN, ROOT, OracleEngine, compare_outputs, file_digest, first_diff, generated_case,
                      golden_cases, golden_log_digest, golden_outputs, model_for)

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", golden_cases())
def test_gpu_compat_matches_reference_files(built, case, tmp_path):
    m = model_for(built, case)
    m.run(str(tmp_path), mode="compat")
    bad = compare_outputs(case, str(tmp_path))
    msgs = [(f, first_diff(os.path.join(GOLDEN, case, f), os.path.join(str(tmp_path), f))) for f in bad]
    assert not bad, msgs


def test_gpu_compat_matches_reference_at_connectome_scale(built, tmp_path):
    # 20,000 one-neuron populations, ~4.1 M synapse entries, delays 0, 100 ms:
    # the reference's single-target path at the connectome configuration's
    # size, byte for byte (size and SHA-256 of the reference's files)
    case = "connectome20k_d0"
    generated_case(case, tmp_path)
    m = model_for(built, case, conf_dir=tmp_path)
    out = tmp_path / "out"
    out.mkdir()
    m.run(str(out), mode="compat")
    assert not compare_outputs(case, str(out))


@pytest.mark.parametrize("case,steps", [("two_pop", 600), ("misc", 400), ("conn_ltp", 300), ("two_pop_stp", 300)])
def test_gpu_state_equals_oracle_every_step(built, oracle, case, steps):
    m = model_for(built, case)
    d = m.desc()
    e = built.Engine(d, "compat")
    o = OracleEngine(built, oracle, d)
    seed = m.seed()
    e.reset(seed)
    o.reset(seed)
    try:
        for s in range(steps):
            sp_g, _ = e.step(1)
            sp_o = o.step(1)
            np.testing.assert_array_equal(sp_g[0], sp_o[0], err_msg="spikes differ at step %d" % s)
            if s % 25 == 0 or s == steps - 1:
                V, cnt, ns = e.state()
                G, isyn = e.syn_state()
                oV, ocnt, ons, oG, oisyn = o.state()
                assert V.tobytes() == oV.tobytes(), "V differs at step %d" % s
                assert np.array_equal(cnt, ocnt) and np.array_equal(ns, ons), "LIF state differs at step %d" % s
                assert G.tobytes() == oG.tobytes(), "conductances differ at step %d" % s
                assert isyn.tobytes() == oisyn.tobytes(), "Isyn differs at step %d" % s
    finally:
        o.close()
        e.close()


def test_device_expf_equals_glibc(built, oracle):
    # every 61st float in [-12.4, 12.4] plus all tabulated exceptions
    top = np.frombuffer(np.float32(12.4).tobytes(), np.uint32)[0]
    pos = np.arange(0, top, 61, dtype=np.uint32)
    xs = np.concatenate([pos, pos | np.uint32(0x80000000)]).view(np.float32)
    tab = np.fromfile(os.path.join(ROOT, "flysim_b200", "_build", "expf_glibc.bin"), np.uint32)
    n = int(tab[1])
    xs = np.concatenate([xs, tab[2:2 + n].view(np.float32)])
    for i in range(0, xs.size, 1 << 22):
        x = np.ascontiguousarray(xs[i:i + (1 << 22)])
        ref = np.zeros_like(x)
        oracle.oracle_expf(x.ctypes.data, ref.ctypes.data, x.size)
        dev = built.debug_expf(x)
        bad = np.nonzero(dev.view(np.uint32) != ref.view(np.uint32))[0]
        assert bad.size == 0, (x[bad[:5]], dev[bad[:5]], ref[bad[:5]])


def test_cli_is_a_drop_in(built, tmp_path):
    case = "small"
    for f in ("net.conf", "net.pro"):
        os.symlink(os.path.join(GOLDEN, case, f), str(tmp_path / f))
    exe = os.path.join(ROOT, "flysim_b200", "_build", "flysim")
    r = subprocess.run([exe, "-conf", "net.conf", "-pro", "net.pro"], cwd=str(tmp_path), capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert not compare_outputs(case, str(tmp_path))
    # the two logs the reference writes on every run
    for f in ("ConfsInfo.log", "network.log"):
        assert file_digest(str(tmp_path / f)) == golden_log_digest(case, f), f
    # through the binary network cache: stored, then read back, same files
    os.remove(str(tmp_path / "network.log"))
    for hit in (False, True):
        for f in golden_outputs(case):
            os.remove(str(tmp_path / f))
        r = subprocess.run([exe, "-conf", "net.conf", "-pro", "net.pro", "-cache", "net.cache", "-nolog"],
                           cwd=str(tmp_path), capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr
        assert ("network read from cache" in r.stdout) == hit
        assert not compare_outputs(case, str(tmp_path))
        assert not os.path.exists(str(tmp_path / "network.log"))
