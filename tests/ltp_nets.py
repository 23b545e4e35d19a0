"""Small networks with long-term plasticity for the LTP tests (test
infrastructure): recurrent E/I populations driven by noiseless injection, so
that the float64 restatement in tests/prod_model.py can follow them step by
step, with LTP parameters that exercise both rules (additive and
multiplicative), spike delays of the LP trace, and a mix of records that LTP
rewrites and records it leaves alone."""
import numpy as np


def ltp_net(fb, n=160, p=0.1, seed=5, tm=False, frac_ltp=0.7, dt=0.1):
    from flysim_b200 import network
    rng = np.random.default_rng(seed)
    f = network.neuron_fields(n, dt, receptors={
        fb.FS_AMPA: dict(Tau=2.0, Vrev=0.0, FExt=0.0),
        fb.FS_GABA: dict(Tau=5.0, Vrev=-80.0, FExt=0.0),
        fb.FS_NMDA: dict(Tau=100.0, TauXT=2.0, Vrev=0.0, FExt=0.0),
    })
    ne = int(0.8 * n)
    f["act"] |= fb.ACT["INJ"]
    on = rng.random(n) < 0.9
    f["act"][on] |= fb.ACT["LTP"]
    f["inj_mean"][:] = rng.uniform(0.40, 0.60, n).astype(np.float32)
    f["ltp_dfLP"][:] = np.exp(-np.float32(dt) / rng.uniform(20.0, 50.0, n).astype(np.float32)).astype(np.float32)
    f["ltp_PosISI"][:] = np.where(rng.random(n) < 0.5, 0.01, -0.01).astype(np.float32)
    f["ltp_NegISI"][:] = np.where(rng.random(n) < 0.5, 0.005, -0.01).astype(np.float32)
    f["ltp_SpiLPDy"][:] = rng.integers(0, 4, n).astype(np.int32)
    pre, post, rec, g = [], [], [], []
    for a in range(n):
        tg = np.nonzero(rng.random(n) < p)[0]
        for b in tg:
            if a < ne:
                pre += [a, a]
                post += [b, b]
                rec += [fb.FS_AMPA, fb.FS_NMDA]
                g += [rng.uniform(0.5, 2.0), rng.uniform(0.1, 0.4)]
            else:
                pre.append(a)
                post.append(b)
                rec.append(fb.FS_GABA)
                g.append(rng.uniform(2.0, 5.0))
    pre = np.asarray(pre, np.uint32)
    ltp = (rng.random(pre.size) < frac_ltp).astype(np.uint8)
    tmd = dict(enabled=(np.arange(n) < ne).astype(np.uint8), U=0.2, tau_rec=200.0, tau_fac=600.0) if tm else None
    return network.desc_from_arrays(n, dt, f, pre, np.asarray(post, np.uint32), np.asarray(rec, np.uint8),
                                    np.asarray(g, np.float32), None, tm=tmd,
                                    act_ctr=fb.DEFAULT_ACT | fb.ACT["LTP"], ltp=ltp)
