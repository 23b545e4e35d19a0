"""Binary network cache and the reference's two log files (CPU only).

* ConfsInfo.log (Parser::ConfsInfo, code/parser.cpp:1488-1631) written from
  the parsed model and network.log (NetSimGnl2::logDataWrite,
  code/NetSimGnl2_info.cpp:93-546) written from the built network are
  byte-identical to the reference's for every golden case (size and SHA-256
  recorded in tests/golden/<case>/logs.json), network.log also for the
  reference run with -t 4, whose set-up draws depend on the thread count.
* A model read back from the cache drives the oracle to the same output files
  as the reference, byte for byte, and its counts and seeds equal a fresh load.
* Any change of the .conf, the .pro or a load option misses the cache; a
  damaged or truncated cache is rebuilt; an unwritable cache path still loads.
* A network without a fixed seed (no -udfsed, no RandomSeeds macro) draws a
  new seed on every load, as the reference does (code/NetSimGnl2_BulPp.cpp:
  80-88), and is never cached.
"""
import os
import shutil

import pytest

from conftest import (GOLDEN, golden_cases, model_for, compare_outputs, golden_log_digest, file_digest,
                      generated_case)


@pytest.mark.parametrize("case", golden_cases())
def test_confs_info_matches_reference(built, case, tmp_path):
    m = model_for(built, case)
    p = str(tmp_path / "ConfsInfo.log")
    m.confs_info(p)
    assert file_digest(p) == golden_log_digest(case, "ConfsInfo.log")


@pytest.mark.parametrize("case", golden_cases())
def test_network_log_matches_reference(built, case, tmp_path):
    m = model_for(built, case)
    p = str(tmp_path / "network.log")
    m.network_log(p)
    assert file_digest(p) == golden_log_digest(case, "network.log")


@pytest.mark.parametrize("case", golden_cases())
def test_threaded_setup_matches_reference(built, case, tmp_path):
    # -t 4 changes the reference's set-up draws (its run is not reproducible
    # with several threads, its set-up is); network.log lists every synapse
    m = model_for(built, case, threads=4)
    p = str(tmp_path / "network.log")
    m.network_log(p)
    assert file_digest(p) == golden_log_digest(case, "network.log -t 4")


def test_logs_match_reference_at_connectome_scale(built, tmp_path):
    # 20,000 one-neuron populations: a 329 MB ConfsInfo.log and a 93 MB
    # network.log listing ~4.1 M synapses, both equal to the reference's
    case = "connectome20k_d0"
    generated_case(case, tmp_path)
    m = model_for(built, case, conf_dir=tmp_path)
    for f, write in (("ConfsInfo.log", m.confs_info), ("network.log", m.network_log)):
        p = str(tmp_path / f)
        write(p)
        assert file_digest(p) == golden_log_digest(case, f), f
        os.remove(p)


def _copy_case(case, d):
    for f in ("net.conf", "net.pro"):
        shutil.copy(os.path.join(GOLDEN, case, f), d)
    return str(d / "net.conf"), str(d / "net.pro")


@pytest.mark.parametrize("case", ["misc", "conn_ltp", "repeats"])
def test_cached_model_reproduces_reference_outputs(built, oracle, case, tmp_path):
    cache = str(tmp_path / "net.cache")
    fresh = model_for(built, case)
    m1 = model_for(built, case, cache=cache)
    assert m1.cache_status == "stored" and os.path.getsize(cache) > 0
    m1.close()
    m = model_for(built, case, cache=cache)
    assert m.cache_status == "hit"
    assert m.info() == fresh.info()
    for r in range(1, 1 + (3 if case == "repeats" else 1)):
        assert m.seed(r) == fresh.seed(r)
    out = tmp_path / "out"
    out.mkdir()
    ctx = oracle.oracle_create(m.desc())
    try:
        m.run_with(oracle.oracle_engine(), ctx, str(out))
    finally:
        oracle.oracle_destroy(ctx)
    assert not compare_outputs(case, str(out))
    for f, write in (("ConfsInfo.log", m.confs_info), ("network.log", m.network_log)):
        p = str(tmp_path / f)
        write(p)
        assert file_digest(p) == golden_log_digest(case, f)


def test_cache_key_follows_files_and_options(built, tmp_path):
    conf, pro = _copy_case("two_pop", tmp_path)
    cache = str(tmp_path / "c.bin")
    assert built.Model(conf, pro, cache=cache).cache_status == "stored"
    assert built.Model(conf, pro, cache=cache).cache_status == "hit"
    # an option changes the key (and the network: -STD draws the user seed)
    assert built.Model(conf, pro, cache=cache, std=True).cache_status == "stored"
    assert built.Model(conf, pro, cache=cache, std=True).cache_status == "hit"
    assert built.Model(conf, pro, cache=cache, std=True, dt=0.05).cache_status == "stored"
    assert built.Model(conf, pro, cache=cache, out_spike="x.dat").cache_status == "stored"
    assert built.Model(conf, pro, cache=cache, out_spike="x.dat").cache_status == "hit"
    assert built.Model(conf, pro, cache=cache).cache_status == "stored"
    # one byte more in either file
    with open(pro, "a") as f:
        f.write("\n")
    assert built.Model(conf, pro, cache=cache).cache_status == "stored"
    with open(conf, "a") as f:
        f.write("\n")
    m = built.Model(conf, pro, cache=cache)
    assert m.cache_status == "stored"
    assert m.info()["synapses"] == model_for(built, "two_pop").info()["synapses"]


def test_damaged_cache_is_rebuilt(built, tmp_path):
    conf, pro = _copy_case("misc", tmp_path)
    cache = tmp_path / "c.bin"
    ref = built.Model(conf, pro, cache=str(cache))
    good = cache.read_bytes()
    # one flipped payload byte: the trailing hash no longer matches
    bad = bytearray(good)
    bad[len(bad) // 2] ^= 0x40
    cache.write_bytes(bytes(bad))
    m = built.Model(conf, pro, cache=str(cache))
    assert m.cache_status == "stored" and cache.read_bytes() == good
    # truncated, header only, and an absurd element count
    for cut in (len(good) - 9, 24, 40):
        cache.write_bytes(good[:cut])
        m = built.Model(conf, pro, cache=str(cache))
        assert m.cache_status == "stored" and m.info() == ref.info()
    huge = bytearray(good)
    # header 24 bytes, then 8 four-byte option fields, then the population count
    huge[56:64] = (2 ** 62).to_bytes(8, "little")
    cache.write_bytes(bytes(huge))
    assert built.Model(conf, pro, cache=str(cache)).cache_status == "stored"
    assert built.Model(conf, pro, cache=str(cache)).cache_status == "hit"


def test_unwritable_cache_still_loads(built, tmp_path):
    conf, pro = _copy_case("small", tmp_path)
    m = built.Model(conf, pro, cache=str(tmp_path / "no" / "such" / "dir" / "c.bin"))
    assert m.cache_status == "unwritable"
    assert m.info() == model_for(built, "small").info()
    assert "cannot write" in built.lib().fs_model_error().decode()
    assert built.Model(conf, pro).cache_status == "off"


def test_unseeded_network_is_never_cached(built, tmp_path):
    conf, pro = _copy_case("two_pop", tmp_path)
    text = open(pro).read()
    start, end = text.index("DefineMacro"), text.index("EndDefineMacro") + len("EndDefineMacro")
    with open(pro, "w") as f:
        f.write(text[:start] + text[end:])
    cache = tmp_path / "c.bin"
    seeds = set()
    for _ in range(3):
        m = built.Model(conf, pro, cache=str(cache))
        assert m.cache_status == "unseeded"
        seeds.add(m.seed(1))
        m.close()
    assert not cache.exists()
    # std::random_device: three equal 32-bit draws would be a frozen seed
    assert len(seeds) > 1
    # the same files with a macro seed are cached as before
    with open(pro, "w") as f:
        f.write(text)
    assert built.Model(conf, pro, cache=str(cache)).cache_status == "stored"
    assert built.Model(conf, pro, cache=str(cache)).cache_status == "hit"
