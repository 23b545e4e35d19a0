"""fs_debug_expf_noalloc (fixed static device scratch, no per-call device
allocation) against the allocating fs_debug_expf on the same inputs.

Both entry points run the same kernel, so the tolerance is 0 ulp (bitwise
equality).  Two calls in a row with different inputs check that the shared
scratch carries nothing stale from one call to the next.  The file is named
to be collected last so that it also runs after every other GPU test; it
passes alone as well (the first call does the per-device set-up).
"""
import os

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _inputs(seed: int, k: int) -> np.ndarray:
    # exponent arguments as the NMDA Mg block sees them (-0.062 * V for V in
    # [-100, 40] mV), a wide range, and tabulated glibc exceptions
    rng = np.random.default_rng(seed)
    tab = np.fromfile(os.path.join(ROOT, "flysim_b200", "_build", "expf_glibc.bin"), np.uint32)
    exc = tab[2:2 + int(tab[1])].view(np.float32)
    parts = [(-0.062 * rng.uniform(-100.0, 40.0, k // 2)).astype(np.float32),
             rng.uniform(-87.0, 88.0, k // 4).astype(np.float32),
             rng.choice(exc, k - k // 2 - k // 4)]
    x = np.concatenate(parts).astype(np.float32)
    rng.shuffle(x)
    return x


@pytest.mark.gpu
def test_noalloc_expf_matches_allocating_entry_twice(built):
    k = built.NOALLOC_MAX_K
    for seed in (11, 12):  # two calls in a row, different inputs
        x = _inputs(seed, k)
        ref = built.debug_expf(x)
        got = built.debug_expf_noalloc(x)
        bad = np.nonzero(got.view(np.uint32) != ref.view(np.uint32))[0]
        assert bad.size == 0, (x[bad[:5]], got[bad[:5]], ref[bad[:5]])
    # a short call after a full one: only its own k values come back
    x = _inputs(13, 1000)
    assert built.debug_expf_noalloc(x).tobytes() == built.debug_expf(x).tobytes()


@pytest.mark.gpu
def test_noalloc_expf_rejects_oversize(built):
    x = np.zeros(built.NOALLOC_MAX_K + 1, np.float32)
    with pytest.raises(RuntimeError, match="exceeds the fixed scratch"):
        built.debug_expf_noalloc(x)
    assert built.debug_expf_noalloc(np.zeros(0, np.float32)).size == 0
