"""C ABI, host model and workload generator (CPU only: no compute calls)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from conftest import ROOT, GOLDEN, model_for


def header_functions():
    txt = open(os.path.join(ROOT, "include", "flysim_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(fs_[a-z_0-9]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol(built):
    L = C.CDLL(built.LIB_PATH)
    missing = [s for s in header_functions() if not hasattr(L, s)]
    assert not missing, missing
    assert len(header_functions()) >= 25
    assert built.lib().fs_abi_version() == built.ABI_VERSION == 2


def test_model_counts_match_reference_rules(built):
    m = model_for(built, "two_pop")
    info = m.info()
    # 800 E and 200 I, p = 0.2: ceil(800*0.2f) = 161 and ceil(200*0.2f) = 41
    # targets per link (float 0.2 > 1/5), 4 E links and 2 I links
    assert info["neurons"] == 1000
    assert info["synapses"] == 800 * (161 + 41) * 2 + 200 * (161 + 41)
    assert info["outputs"] == 3
    assert m.seed() == 7


def test_seed_rules(built):
    d = os.path.join(GOLDEN, "two_pop")
    # -STD shares the user-seed bit: the seed becomes the (unset) user seed 0
    m = built.Model(os.path.join(d, "net.conf"), os.path.join(d, "net.pro"), std=True)
    assert m.seed() == 0
    m = built.Model(os.path.join(d, "net.conf"), os.path.join(d, "net.pro"), user_seed=99)
    assert m.seed() == 99
    m = model_for(built, "repeats")
    assert [m.seed(r) for r in (1, 2)] == [5, 9]
    s3 = m.seed(3)
    assert s3 not in (5, 9) and s3 <= 2 ** 31 - 1


def test_parse_errors_are_reported(built, tmp_path):
    bad = tmp_path / "bad.conf"
    bad.write_text("NeuralPopulation: X\nN=abc\nEndNeuralPopulation\n")
    pro = os.path.join(GOLDEN, "two_pop", "net.pro")
    with pytest.raises(built.FsError) as e:
        built.Model(str(bad), pro)
    assert e.value.code == built.FS_ERR_PARSE
    with pytest.raises(built.FsError):
        built.Model(str(tmp_path / "missing.conf"), pro)


def test_desc_view_is_consistent(built):
    m = model_for(built, "conn")
    d = m.desc().contents
    n = d.neurons.n
    assert n == 400
    tot = 0
    for r in range(5):
        L = d.compat.contents.rec[r]
        if L.n_recs:
            rp = np.ctypeslib.as_array(L.rec_rowptr, (n + 1,))
            assert rp[-1] == L.n_recs and np.all(np.diff(rp.astype(np.int64)) >= 0)
            post = np.ctypeslib.as_array(L.rec_post, (L.n_recs,))
            assert np.all(np.diff(post.astype(np.int64)) >= 0)  # sorted by post
        tot += L.n_recs
    assert tot == d.syn.contents.n


def test_no_device_is_an_error_not_a_fallback(built):
    if built.device_count() > 0:
        pytest.skip("a GPU is visible")
    m = model_for(built, "small")
    with pytest.raises(built.FsError) as e:
        built.Engine(m.desc())
    assert e.value.code == built.FS_ERR_NODEVICE


def test_connectome_generator_shapes():
    from flysim_b200 import netgen
    c = netgen.connectome(n=3000, regions=12, seed=4)
    deg = np.bincount(c.pre, minlength=c.n)
    assert abs(deg.mean() - 120) < 12
    region = c.region
    intra = np.mean(region[c.pre] == region[c.post])
    assert 0.7 < intra < 0.9
    assert abs(c.excit.mean() - 0.7) < 0.05
    assert np.all(c.pre != c.post)
    assert np.all((c.delay_ms >= 1) & (c.delay_ms <= 5))
    assert 1000 <= c.freq_ext.min() and c.freq_ext.max() <= 4000


def test_array_network_matches_conf_builder(built, tmp_path):
    """The array-built production network has the same neurons and synapses as
    the .conf route (one population per neuron)."""
    from flysim_b200 import netgen, network
    c = netgen.connectome(n=120, regions=4, mean_degree=15, seed=9)
    conf = tmp_path / "c.conf"
    netgen.write_connectome(c, str(conf))
    pro = tmp_path / "c.pro"
    netgen.write_pro(str(pro), 10, seeds=(1,))
    m = built.Model(str(conf), str(pro))
    d = m.desc().contents
    s = d.syn.contents
    conf_syn = sorted(zip(np.ctypeslib.as_array(s.pre, (s.n,)).tolist(), np.ctypeslib.as_array(s.post, (s.n,)).tolist(),
                          np.ctypeslib.as_array(s.rec, (s.n,)).tolist(), np.ctypeslib.as_array(s.delay, (s.n,)).tolist()))
    na = network.connectome_net(c)
    arr_syn = sorted(zip(na.syn["pre"].tolist(), na.syn["post"].tolist(), na.syn["rec"].tolist(),
                         na.syn["delay"].tolist()))
    assert conf_syn == arr_syn
    g_conf = np.sort(np.ctypeslib.as_array(s.g, (s.n,)))
    g_arr = np.sort(na.syn["g"].astype(np.float32))
    np.testing.assert_allclose(g_conf, g_arr, rtol=1e-6)
    for k in ("Vth", "gl", "Cm", "RfPed", "SpiDy"):
        a = np.ctypeslib.as_array(getattr(d.neurons, k), (c.n,))
        np.testing.assert_array_equal(a, na.fields[k])
    pb = np.ctypeslib.as_array(d.neurons.pb, (5 * c.n,))
    np.testing.assert_allclose(pb, na.fields["pb"], rtol=1e-6)


def test_values_the_reference_leaves_undefined_are_parse_errors(built, tmp_path):
    # a negative population size, a NaN connectivity and a zero rate window:
    # the reference wraps an allocation, a target count or divides by zero;
    # here each is FS_ERR_PARSE naming the keyword
    d = os.path.join(GOLDEN, "keywords")
    conf, pro = open(os.path.join(d, "net.conf")).read(), open(os.path.join(d, "net.pro")).read()
    cases = [("net.conf", "N=30", "N=-1", "N"), ("net.conf", "Connectivity=0.3", "Connectivity=nan", "Connectivity")]
    if "FiringRateWindow=" in pro:
        import re
        w = re.search(r"FiringRateWindow=[0-9.]+", pro).group(0)
        cases.append(("net.pro", w, "FiringRateWindow=0", "FiringRateWindow"))
    for which, old, new, key in cases:
        text = {"net.conf": conf, "net.pro": pro}[which]
        assert old in text, old
        c, p = str(tmp_path / "c.conf"), str(tmp_path / "p.pro")
        open(c, "w").write(conf.replace(old, new, 1) if which == "net.conf" else conf)
        open(p, "w").write(pro.replace(old, new, 1) if which == "net.pro" else pro)
        with pytest.raises(built.FsError) as ei:
            built.Model(c, p)
        assert ei.value.code == built.FS_ERR_PARSE and key in str(ei.value), str(ei.value)


def test_header_is_plain_c_and_links(built, tmp_path):
    # the boundary is a C ABI: the header compiles as C99 with warnings as
    # errors, and a C program links against the library and calls it (no
    # GPU is needed for the version and the device count)
    import shutil
    import subprocess
    if not shutil.which("gcc"):
        pytest.skip("no gcc")
    src = tmp_path / "abi.c"
    src.write_text(
        '#include <stdio.h>\n#include "flysim_b200.h"\n'
        "int main(void) {\n"
        "  int n = -1;\n"
        "  int rc = fs_device_count(&n);\n"
        '  printf("%d %d %d\\n", fs_abi_version(), FS_ABI_VERSION, rc == FS_OK || rc == FS_ERR_NODEVICE);\n'
        "  return 0;\n}\n")
    lib_dir = os.path.join(ROOT, "flysim_b200", "_build")
    exe = str(tmp_path / "abi")
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror", "-I", os.path.join(ROOT, "include"),
                    str(src), "-o", exe, "-L", lib_dir, "-lflysim_b200", "-Wl,-rpath," + lib_dir], check=True)
    out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()
    assert out == ["2", "2", "1"], out


def test_array_network_with_ltp_matches_conf_builder(built, tmp_path):
    """connectome_net(..., ltp=...) gives the LTP parameters, activity bits
    and global flags the .conf route gives with -LTP and the keywords."""
    from flysim_b200 import netgen, network
    c = netgen.connectome(n=120, regions=4, mean_degree=15, seed=9, delays=False)
    kw = dict(tLP=30, SpiLPDy=0.2, PosISI=0.02, NegISI=-0.01)
    conf, pro = tmp_path / "c.conf", tmp_path / "c.pro"
    netgen.write_connectome(c, str(conf), with_delays=False, ltp=kw)
    netgen.write_pro(str(pro), 10, seeds=(1,))
    m = built.Model(str(conf), str(pro), ltp=True)
    d = m.desc().contents
    na = network.connectome_net(c, with_delays=False, ltp=kw)
    assert d.act_ctr == na.desc.act_ctr
    np.testing.assert_array_equal(np.ctypeslib.as_array(d.neurons.act, (c.n,)), na.fields["act"])
    for k in ("ltp_SpiLPDy", "ltp_PosISI", "ltp_NegISI"):
        np.testing.assert_array_equal(np.ctypeslib.as_array(getattr(d.neurons, k), (c.n,)), na.fields[k])
    np.testing.assert_allclose(np.ctypeslib.as_array(d.neurons.ltp_dfLP, (c.n,)), na.fields["ltp_dfLP"], rtol=1e-6)
