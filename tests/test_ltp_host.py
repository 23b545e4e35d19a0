"""Host side of long-term plasticity in the production modes (CPU only).

The reference's LTP rewrites only its single-target records (SynFst1 /
SynSlo1, code/EqsGnl2.cpp:1005-1044), not the gates of links from a
population to several targets.  The host builder marks exactly those
entries of the production synapse list (fs_syn_list.ltp), the binary
network cache keeps the marks, and the connectome writer's LTP keywords
reach every neuron's parameters (code/NetSimGnl2_BulPp.cpp:180-183).
"""
import ctypes as C
import os

import numpy as np

import flysim_b200 as fb
from flysim_b200 import netgen

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _syn(m):
    d = m.desc()
    d = d.contents if hasattr(d, "contents") else d
    s = d.syn.contents
    ltp = np.ctypeslib.as_array(s.ltp, (s.n,)).copy() if s.ltp else None
    rec = np.ctypeslib.as_array(s.rec, (s.n,)).copy()
    return d, ltp, rec


def _single_target_records(d):
    comp = d.compat.contents
    return sum(comp.rec[r].n_recs for r in range(fb.FS_NREC))


def test_ltp_marks_exactly_the_single_target_records():
    # the keywords case mixes a 30-neuron population (group gates) with
    # single-target links
    for case in ("keywords", "conn_ltp", "two_pop"):
        m = fb.Model(os.path.join(GOLDEN, case, "net.conf"), os.path.join(GOLDEN, case, "net.pro"), ltp=True)
        try:
            d, ltp, rec = _syn(m)
            assert ltp is not None and ltp.size == rec.size
            assert int(ltp.sum()) == _single_target_records(d), case
            assert d.act_ctr & fb.ACT["LTP"]
        finally:
            m.close()


def test_cache_keeps_the_ltp_marks(tmp_path):
    c = netgen.connectome(n=300, regions=3, mean_degree=20, seed=4, delays=False)
    conf, pro = str(tmp_path / "net.conf"), str(tmp_path / "net.pro")
    netgen.write_connectome(c, conf, with_delays=False, ltp=dict(tLP=30, SpiLPDy=0.2, PosISI=0.004, NegISI=-0.003))
    netgen.write_pro(pro, 100.0, seeds=(2,), outputs=())
    cache = str(tmp_path / "net.cache")
    got = []
    for expect in ("stored", "hit"):
        m = fb.Model(conf, pro, ltp=True, cache=cache)
        try:
            assert m.cache_status == expect
            d, ltp, rec = _syn(m)
            n = d.neurons.n
            got.append((ltp, rec,
                        np.ctypeslib.as_array(d.neurons.ltp_PosISI, (n,)).copy(),
                        np.ctypeslib.as_array(d.neurons.ltp_NegISI, (n,)).copy(),
                        np.ctypeslib.as_array(d.neurons.ltp_SpiLPDy, (n,)).copy(),
                        np.ctypeslib.as_array(d.neurons.ltp_dfLP, (n,)).copy()))
        finally:
            m.close()
    (l0, r0, pos, neg, spd, dflp), (l1, r1, *rest) = got
    np.testing.assert_array_equal(l0, l1)
    np.testing.assert_array_equal(r0, r1)
    assert l0.all()  # one-neuron populations: every entry is a single-target record
    assert np.all(pos == np.float32(0.004)) and np.all(neg == np.float32(-0.003))
    assert np.all(spd == 2)  # 0.2 ms at dt 0.1 ms (code/parser.cpp:565)
    np.testing.assert_allclose(dflp, np.exp(-0.1 / 30.0), rtol=1e-6)
    for a, b in zip((pos, neg, spd, dflp), rest):
        np.testing.assert_array_equal(a, b)
