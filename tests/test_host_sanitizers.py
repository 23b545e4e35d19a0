"""The host code under AddressSanitizer, UndefinedBehaviorSanitizer and
ThreadSanitizer (CPU).

The flysim command line (flysim_b200/csrc/host: argv, .conf/.pro parser,
network builder, cache, protocol loop, output writers and logs) is compiled
with -fsanitize=address,undefined, with the CPU oracle (oracle/fs_oracle.cpp)
standing in for the GPU engine (tests/asan_oracle_engine.cpp), and run on
every golden case with the reference's own flags: no sanitizer report, and
every output file and both logs byte-identical to what the reference wrote;
under ThreadSanitizer on a few cases and on the set-up with four threads.
The sanitizers are the race and memory checks the GPU side cannot have on
this pool (compute-sanitizer is closed), applied to the code around it.
"""
import json
import os
import shutil
import subprocess

import pytest

from conftest import GOLDEN, ROOT, compare_outputs, file_digest, golden_cases

HOST = os.path.join(ROOT, "flysim_b200", "csrc", "host")
SAN = ["-fsanitize=address,undefined,float-cast-overflow", "-fno-sanitize-recover=all", "-fno-omit-frame-pointer", "-O1", "-g"]
TSAN = ["-fsanitize=thread", "-O1", "-g"]


def _build(tmp_path_factory, name, flags):
    if not shutil.which("g++"):
        pytest.skip("no g++")
    d = tmp_path_factory.mktemp(name)
    objs = []
    srcs = [os.path.join(HOST, f + ".cpp") for f in
            ("fs_cli", "fs_parse", "fs_build", "fs_cache", "fs_driver", "fs_model_api", "fs_netlog")]
    srcs += [os.path.join(ROOT, "oracle", "fs_oracle.cpp"), os.path.join(ROOT, "tests", "asan_oracle_engine.cpp")]
    for s in srcs:
        o = str(d / (os.path.basename(s) + ".o"))
        subprocess.run(["g++", "-std=c++17", *flags, "-I", os.path.join(ROOT, "include"), "-I", HOST, "-c", s, "-o", o],
                       check=True)
        objs.append(o)
    o = str(d / "fs_philox.o")
    subprocess.run(["gcc", *flags, "-I", os.path.join(ROOT, "include"), "-c",
                    os.path.join(ROOT, "oracle", "fs_philox.c"), "-o", o], check=True)
    objs.append(o)
    exe = str(d / name)
    subprocess.run(["g++", *flags, *objs, "-o", exe, "-lpthread"], check=True)
    return exe


@pytest.fixture(scope="module")
def flysim_asan(tmp_path_factory):
    return _build(tmp_path_factory, "flysim_asan", SAN)


@pytest.fixture(scope="module")
def flysim_tsan(tmp_path_factory):
    return _build(tmp_path_factory, "flysim_tsan", TSAN)


def _run_case(exe, case, tmp_path, env):
    src = os.path.join(GOLDEN, case)
    for f in ("net.conf", "net.pro"):
        shutil.copy(os.path.join(src, f), str(tmp_path / f))
    flags = json.load(open(os.path.join(src, "cmd.json")))
    r = subprocess.run([exe, "-conf", "net.conf", "-pro", "net.pro", *flags], cwd=str(tmp_path),
                       capture_output=True, text=True, timeout=900, env=dict(os.environ, **env))
    report = r.stderr[-4000:]
    assert r.returncode == 0, report
    assert "runtime error" not in r.stderr and "Sanitizer" not in r.stderr, report
    bad = compare_outputs(case, str(tmp_path))
    assert not bad, bad
    logs = json.load(open(os.path.join(src, "logs.json")))
    for name in ("ConfsInfo.log", "network.log"):
        assert file_digest(str(tmp_path / name)) == logs[name], name


# config1_1s is two_pop's network for a full second (a minute under the
# sanitizers); tests/test_oracle_ref.py runs it through the oracle
@pytest.mark.parametrize("case", [c for c in golden_cases() if c != "config1_1s"])
def test_cli_under_sanitizers_matches_reference(flysim_asan, case, tmp_path):
    _run_case(flysim_asan, case, tmp_path, {"ASAN_OPTIONS": "detect_leaks=1:halt_on_error=1",
                                            "UBSAN_OPTIONS": "halt_on_error=1:print_stacktrace=1"})


@pytest.mark.parametrize("case", ["conn", "repeats", "cli_flags"])
def test_cli_under_thread_sanitizer(flysim_tsan, case, tmp_path):
    # the formatter thread that writes a chunk's files while the engine
    # computes the next, the threaded network.log and the -t set-up
    _run_case(flysim_tsan, case, tmp_path, {"TSAN_OPTIONS": "halt_on_error=1:second_deadlock_stack=1"})


def test_threaded_setup_under_thread_sanitizer(flysim_tsan, tmp_path):
    # -t 4: the set-up's draws as the reference's four threads make them,
    # pinned by the network.log of the reference's -t 4 run
    src = os.path.join(GOLDEN, "conn")
    for f in ("net.conf", "net.pro"):
        shutil.copy(os.path.join(src, f), str(tmp_path / f))
    r = subprocess.run([flysim_tsan, "-conf", "net.conf", "-pro", "net.pro", "-t", "4"], cwd=str(tmp_path),
                       capture_output=True, text=True, timeout=900,
                       env=dict(os.environ, TSAN_OPTIONS="halt_on_error=1"))
    assert r.returncode == 0 and "Sanitizer" not in r.stderr, r.stderr[-4000:]
    logs = json.load(open(os.path.join(src, "logs.json")))
    assert file_digest(str(tmp_path / "network.log")) == logs["network.log -t 4"]


def test_engine_failure_mid_run_is_reported_cleanly(flysim_asan, tmp_path):
    # host-side fault injection: the second chunk's step call fails as a
    # device error would (FLYSIM_TEST_FAIL_STEP, tests/asan_oracle_engine.cpp).
    # The run stops with an error status and message, the formatter thread
    # joins, every output file is closed with the first chunk's steps in it
    # (a prefix of the reference's file), and nothing leaks
    src = os.path.join(GOLDEN, "two_pop")
    for f in ("net.conf", "net.pro"):
        shutil.copy(os.path.join(src, f), str(tmp_path / f))
    r = subprocess.run([flysim_asan, "-conf", "net.conf", "-pro", "net.pro"], cwd=str(tmp_path),
                       capture_output=True, text=True, timeout=900,
                       env=dict(os.environ, FLYSIM_TEST_FAIL_STEP="2", ASAN_OPTIONS="detect_leaks=1",
                                UBSAN_OPTIONS="halt_on_error=1"))
    assert r.returncode != 0
    assert "flysim:" in r.stderr and "Sanitizer" not in r.stderr, r.stderr[-4000:]
    got = open(str(tmp_path / "Spikes.dat"), "rb").read()
    ref = open(os.path.join(src, "Spikes.dat"), "rb").read()
    assert 0 < len(got) < len(ref) and ref.startswith(got)


def test_unwritable_output_is_an_error(flysim_asan, tmp_path):
    src = os.path.join(GOLDEN, "two_pop")
    for f in ("net.conf", "net.pro"):
        shutil.copy(os.path.join(src, f), str(tmp_path / f))
    r = subprocess.run([flysim_asan, "-conf", "net.conf", "-pro", "net.pro", "-os", "no_such_dir/Spikes.dat"],
                       cwd=str(tmp_path), capture_output=True, text=True, timeout=900,
                       env=dict(os.environ, ASAN_OPTIONS="detect_leaks=1", UBSAN_OPTIONS="halt_on_error=1"))
    assert r.returncode != 0
    assert "cannot open output file" in r.stderr and "Sanitizer" not in r.stderr, r.stderr[-4000:]


def _mutations(text, seed, k_trunc=6, k_del=6, k_num=12):
    """Deterministic damaged variants of an input file: truncations, a line
    deleted, a number replaced by garbage or an out-of-range value."""
    import random
    import re
    rng = random.Random(seed)
    lines = text.split("\n")
    out = [text[: len(text) * k // (k_trunc + 1)] for k in range(1, k_trunc + 1)]
    for _ in range(k_del):
        i = rng.randrange(len(lines))
        out.append("\n".join(lines[:i] + lines[i + 1:]))
    nums = list(re.finditer(r"-?\d+(\.\d+)?(e-?\d+)?", text))
    for _ in range(k_num):
        m = rng.choice(nums)
        out.append(text[: m.start()] + rng.choice(["abc", "", "-1", "0", "0.5", "nan", "-0.2", "inf9", "-7e20"])
                   + text[m.end():])
    return out


@pytest.mark.parametrize("case,which", [("small", "net.conf"), ("small", "net.pro"),
                                        ("keywords", "net.conf"), ("keywords", "net.pro")])
def test_damaged_inputs_run_or_fail_cleanly(flysim_asan, case, which, tmp_path):
    # every damaged .conf / .pro either runs or ends with an error message:
    # no sanitizer report, no signal (the reference crashes or runs undefined
    # on several of them: a negative N, a NaN connectivity, a zero
    # FiringRateWindow)
    src = os.path.join(GOLDEN, case)
    base = open(os.path.join(src, which)).read()
    env = dict(os.environ, ASAN_OPTIONS="detect_leaks=1", UBSAN_OPTIONS="halt_on_error=1:print_stacktrace=1")
    for v, text in enumerate(_mutations(base, seed=len(base))):
        d = tmp_path / str(v)
        d.mkdir()
        for f in ("net.conf", "net.pro"):
            shutil.copy(os.path.join(src, f), str(d / f))
        (d / which).write_text(text)
        r = subprocess.run([flysim_asan, "-conf", "net.conf", "-pro", "net.pro"], cwd=str(d), capture_output=True,
                           text=True, timeout=120, env=env)
        assert r.returncode >= 0, (v, r.stderr[-3000:])
        assert "Sanitizer" not in r.stderr and "runtime error" not in r.stderr, (v, r.stderr[-3000:])
        if r.returncode:
            assert "flysim:" in r.stderr, (v, r.stderr[-3000:])


def test_damaged_cache_is_rebuilt_under_sanitizers(flysim_asan, tmp_path):
    # a network cache with flipped bytes (header, payload, hash) or cut
    # short is never trusted: the run rebuilds from the text files and writes
    # the reference's outputs, with no sanitizer report
    case = "keywords"
    src = os.path.join(GOLDEN, case)
    env = dict(os.environ, ASAN_OPTIONS="detect_leaks=1", UBSAN_OPTIONS="halt_on_error=1:print_stacktrace=1")

    def run(d, cache):
        for f in ("net.conf", "net.pro"):
            shutil.copy(os.path.join(src, f), str(d / f))
        flags = json.load(open(os.path.join(src, "cmd.json")))
        r = subprocess.run([flysim_asan, "-conf", "net.conf", "-pro", "net.pro", "-cache", cache, *flags],
                           cwd=str(d), capture_output=True, text=True, timeout=300, env=env)
        assert r.returncode == 0 and "Sanitizer" not in r.stderr and "runtime error" not in r.stderr, \
            r.stderr[-3000:]
        assert not compare_outputs(case, str(d))
        return r.stdout

    cache = str(tmp_path / "net.cache")
    first = tmp_path / "first"
    first.mkdir()
    run(first, cache)
    good = open(cache, "rb").read()
    assert len(good) > 64
    cuts = [8, 20, len(good) // 2, len(good) - 3]
    flips = [0, 9, 13, 17, 30, len(good) // 3, len(good) // 2, len(good) - 12, len(good) - 1]
    damaged = [good[:c] for c in cuts] + [good[:i] + bytes([good[i] ^ 0x5A]) + good[i + 1:] for i in flips]
    for v, blob in enumerate(damaged):
        open(cache, "wb").write(blob)
        d = tmp_path / ("v%d" % v)
        d.mkdir()
        out = run(d, cache)
        assert "network read from cache" not in out, v
