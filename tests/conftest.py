import ctypes as C
import filecmp
import json
import os
import shutil
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def built():
    """Native library (and the oracle) built in-tree; where they already
    exist (a GPU machine that received the built files) they are used as
    they are."""
    from flysim_b200 import build
    lib = os.path.join(ROOT, "flysim_b200", "_build", "libflysim_b200.so")
    if not os.path.exists(lib) or os.environ.get("FS_REBUILD"):
        build.build()
    olib = os.path.join(ROOT, "oracle", "_build", "liboracle.so")
    if not os.path.exists(olib):
        build.build_oracle()
    import flysim_b200 as fb
    return fb


@pytest.fixture(scope="session")
def oracle(built):
    """The CPU oracle (test infrastructure) through its C interface."""
    L = C.CDLL(os.path.join(ROOT, "oracle", "_build", "liboracle.so"))
    L.oracle_engine.restype = C.POINTER(built.EngineVtbl)
    L.oracle_create.restype = C.c_void_p
    L.oracle_create.argtypes = [C.POINTER(built.NetDesc)]
    L.oracle_destroy.argtypes = [C.c_void_p]
    L.oracle_get_state.argtypes = [C.c_void_p] + [C.c_void_p] * 5
    L.oracle_expf.argtypes = [C.c_void_p, C.c_void_p, C.c_uint64]
    return L


def golden_cases():
    """Cases whose inputs are committed (generated cases are run by their
    own tests: their .conf is rewritten from gen.json first)."""
    return sorted(d for d in os.listdir(GOLDEN)
                  if os.path.isdir(os.path.join(GOLDEN, d)) and not os.path.exists(os.path.join(GOLDEN, d, "gen.json")))


def generated_case(case, dst):
    """Writes a generated case's net.conf (seeded generator call of gen.json,
    checked against the recorded SHA-256) and its net.pro into dst."""
    sys.path.insert(0, os.path.join(GOLDEN))
    import make_golden
    gen = json.load(open(os.path.join(GOLDEN, case, "gen.json")))
    conf = os.path.join(str(dst), "net.conf")
    make_golden.write_generated_conf(gen, conf)
    rec = make_golden.file_record(conf)
    assert rec["sha256"] == gen["conf"]["sha256"], "the generator no longer writes the recorded net.conf"
    shutil.copy(os.path.join(GOLDEN, case, "net.pro"), str(dst))
    return conf, os.path.join(str(dst), "net.pro")


def model_for(fb, case, conf_dir=None, **kw):
    """The case's model; conf_dir holds the inputs of a generated case."""
    d = os.path.join(GOLDEN, case)
    flags = json.load(open(os.path.join(d, "cmd.json")))
    opts = dict(stp="-STP" in flags, std="-STD" in flags, ltp="-LTP" in flags)
    val = {f: flags[i + 1] for i, f in enumerate(flags[:-1])}
    if "-rp" in val:
        opts["repeats"] = int(val["-rp"])
    if "-udfsed" in val:
        opts["user_seed"] = int(val["-udfsed"])
    if "-dt" in val:
        opts["dt"] = float(val["-dt"])
    for flag, key in (("-om", "out_mem"), ("-os", "out_spike"), ("-or", "out_rate")):
        if flag in val:
            opts[key] = val[flag]
    if "-t" in val:
        opts["threads"] = int(val["-t"])
    opts.update(kw)
    src = str(conf_dir) if conf_dir is not None else d
    return fb.Model(os.path.join(src, "net.conf"), os.path.join(src, "net.pro"), **opts)


def golden_digests(case):
    """Size and SHA-256 of each output of a case kept as digests, or None."""
    p = os.path.join(GOLDEN, case, "digests.json")
    return json.load(open(p)) if os.path.exists(p) else None


def golden_outputs(case):
    """The output files of a case (its inputs and the log digests excluded)."""
    dg = golden_digests(case)
    if dg is not None:
        return sorted(dg)
    d = os.path.join(GOLDEN, case)
    return sorted(f for f in os.listdir(d) if f not in ("net.conf", "net.pro", "cmd.json", "logs.json"))


def golden_log_digest(case, name):
    return json.load(open(os.path.join(GOLDEN, case, "logs.json")))[name]


def file_digest(path):
    import hashlib
    data = open(path, "rb").read()
    return {"bytes": len(data), "sha256": hashlib.sha256(data).hexdigest()}


def compare_outputs(case, out_dir):
    """Byte comparison of every output file of a golden case (size and
    SHA-256 for cases kept as digests)."""
    bad = []
    dg = golden_digests(case)
    if dg is not None:
        for f, rec in dg.items():
            b = os.path.join(out_dir, f)
            if not os.path.exists(b) or file_digest(b) != {"bytes": rec["bytes"], "sha256": rec["sha256"]}:
                bad.append(f)
        return bad
    for f in golden_outputs(case):
        a, b = os.path.join(GOLDEN, case, f), os.path.join(out_dir, f)
        if not os.path.exists(b) or not filecmp.cmp(a, b, shallow=False):
            bad.append(f)
    return bad


def first_diff(a, b):
    if not os.path.exists(a) or not os.path.exists(b):
        return None, None, None  # a digest-only case, or a missing output
    la, lb = open(a).read().splitlines(), open(b).read().splitlines()
    for i, (x, y) in enumerate(zip(la, lb)):
        if x != y:
            return i, x, y
    return min(len(la), len(lb)), None, None


class OracleEngine:
    """Python handle on the oracle's engine table (reset / drive / step)."""

    def __init__(self, fb, oracle_lib, desc):
        self.fb, self.L = fb, oracle_lib
        self.ctx = oracle_lib.oracle_create(desc)
        vt = oracle_lib.oracle_engine().contents
        self._reset = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_uint32, C.c_uint32)(vt.reset)
        self._step = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_uint32, C.POINTER(fb.StepOut))(vt.step)
        self.n = desc.contents.neurons.n

    def reset(self, seed):
        assert self._reset(self.ctx, seed, seed) == 0

    def step(self, k):
        import numpy as np
        counts = np.zeros(k, np.uint32)
        idx = np.zeros(max(1, k * self.n), np.uint32)
        so = self.fb.StepOut()
        so.spike_count = counts.ctypes.data_as(C.POINTER(C.c_uint32))
        so.spike_idx = idx.ctypes.data_as(C.POINTER(C.c_uint32))
        so.spike_cap = idx.size
        assert self._step(self.ctx, k, C.byref(so)) == 0
        offs = np.concatenate([[0], np.cumsum(counts.astype(np.int64))])
        return [idx[offs[i]:offs[i + 1]].copy() for i in range(k)]

    def state(self):
        import numpy as np
        V = np.zeros(self.n, np.float32)
        cnt = np.zeros(self.n, np.int32)
        ns = np.zeros(self.n, np.uint32)
        G = np.zeros(5 * self.n, np.float32)
        isyn = np.zeros(self.n, np.float32)
        self.L.oracle_get_state(self.ctx, V.ctypes.data, cnt.ctypes.data, ns.ctypes.data, G.ctypes.data,
                                isyn.ctypes.data)
        return V, cnt, ns, G.reshape(5, self.n), isyn

    def close(self):
        if self.ctx:
            self.L.oracle_destroy(self.ctx)
            self.ctx = None
