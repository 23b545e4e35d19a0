"""The single-step kernel's plan, checked on the CPU (no device needed).

k_prod1 runs networks whose delays are all 0 with each block's tables in
shared memory.  fs_debug_single_step_plan builds the same plan fs_create
builds and verifies every index the kernel forms from it (post ranges in
whole warps of at most 512 posts, sorted tracked ids, linear rows and
entries, NMDA edge rows against the network's CSR, the tracked index and
source of every edge, shared-memory size) and that the plan holds each
synapse exactly once.
"""
import numpy as np
import pytest

from conftest import model_for


def _connectome(fb, n, delays=False, seed=1):
    from flysim_b200 import netgen, network
    c = netgen.connectome(n=n, regions=max(2, n // 345), seed=seed)
    return network.connectome_net(c, with_delays=delays)


@pytest.mark.parametrize("sm", [148, 132, 17])
def test_plan_of_the_20k_connectome(built, sm):
    na = _connectome(built, 20000)
    st = built.single_step_plan(na.desc, sm)
    nl = int(np.count_nonzero(na.syn["rec"] != built.FS_NMDA))
    nm = int(np.count_nonzero(na.syn["rec"] == built.FS_NMDA))
    if sm * 512 < 20000:
        assert st["qualifies"] == 0
        return
    assert st["qualifies"] == 1 and st["blocks"] == sm
    assert st["lin_entries"] == nl and st["nmda_edges"] == nm
    assert st["max_posts"] <= 512 and st["smem"] <= 200 * 1024


@pytest.mark.parametrize("case", ["two_pop", "two_pop_std", "conn", "small", "config1_1s"])
def test_plan_of_reference_networks(built, case):
    m = model_for(built, case)
    st = built.single_step_plan(m.desc(), 148)
    assert st["qualifies"] == 1
    assert st["max_posts"] <= 512


@pytest.mark.parametrize("n", [33, 700, 4735, 12345])
def test_plan_of_small_and_ragged_networks(built, n):
    # blocks cut at groups of four posts, up to one block per SM and the
    # 512-post maximum per block
    from flysim_b200 import netgen, network
    c = netgen.connectome_fast(n=n, regions=max(2, n // 345), delays=False, seed=13)
    na = network.connectome_net(c, with_delays=False)
    st = built.single_step_plan(na.desc, 148)
    assert st["qualifies"] == 1, built.lib().fs_last_error(None)
    assert st["blocks"] == min(148, (n + 3) // 4) and st["max_posts"] <= 512


def test_oversized_blocks_fall_back(built):
    # 148 x 512 posts of ~85 NMDA in-edges each do not fit in shared memory:
    # the plan is refused with its reason and the interval kernel runs
    from flysim_b200 import netgen, network
    c = netgen.connectome_fast(n=75776, regions=220, delays=False, seed=13)
    na = network.connectome_net(c, with_delays=False)
    assert built.single_step_plan(na.desc, 148)["qualifies"] == 0
    assert b"shared memory" in built.lib().fs_last_error(None)


def test_delayed_networks_do_not_qualify(built):
    na = _connectome(built, 2000, delays=True)
    assert built.single_step_plan(na.desc, 148)["qualifies"] == 0
