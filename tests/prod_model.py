"""Step-by-step float64 restatement of the production modes' semantics for
small networks (test infrastructure only; nothing in the product imports it).

Neuron model as the reference: exponential-Euler VmEul with the NMDA Mg
block, the dV clamp and the firing state machine (code/EqsGnl2.cpp:152-251).
Synapses as the production engine defines them:

* linear receptors: the gate of a presynaptic neuron obeys st <- st + inc on
  a spike and st <- st*df otherwise (code/EqsGnl2.cpp:866-917), so a spike at
  step t adds w*(inc + st(t-1)*(1-df)) to the post's conductance, which
  arrives in step t + 1 + delay and then decays by the post's df each step;
* NMDA: per-presynaptic x/s kinetics (code/EqsGnl2.cpp:493), the post reads
  w * s_pre(t - 1 - delay) in step t;
* Tsodyks-Markram facilitation/depression per presynaptic neuron (u, x kept
  in float32 between steps): on a spike u <- u + U(1-u), inc = u*x,
  x <- x - inc; otherwise u relaxes to U with tau_fac and x to 1 with tau_rec.

External drive and injection noise are random; they enter as inputs: the
`drive` argument gives, per step and neuron, the hit bitmap (bit r:
receptor r's external synapse hit) and the injection current, as the
engine's Philox draws produce them (fs_debug_drive, itself checked bit for
bit against the CPU restatement oracle/fs_philox.c).  The external gates
follow BgInit (code/EqsGnl2.cpp:284-337): a linear receptor's gate st <- st+1
on a hit, st*dfst otherwise, adding ext_g*st to its conductance; the NMDA
drive x <- x+1 on a hit, x*dfxt otherwise, s <- dfst*s + efst*as*x*(1-s),
adding ext_g*s.  Without `drive`, networks with drive or injection noise are
refused.
"""
from __future__ import annotations

import numpy as np

AMPA, GABA, ACH, GCL, NMDA = range(5)
ACT_INJ, ACT_NMDA = 128, 4
NS_FIRE, NS_SPIKE = 1, 2
NS_OVF, NS_UDF = 16, 32


ACT_EXT = (1, 2, 32, 64)  # AMPA, GABA, ACh, GluCl drive bits of ActCtr


def simulate(na, steps: int, extra: bool = False, drive=None, ltp: bool = False):
    """Returns (spikes: list of index arrays per step, V: [steps, n] float64)
    and, with `extra`, also the receptor currents Irep [steps, 5, n] (kept
    from the last integrated step while a neuron fires,
    code/EqsGnl2.cpp:196-206) and the LIF state word [steps, n].  drive =
    (hits uint8 [steps, n], injection current [steps, n]) of steps 0 ..
    steps-1 after a reset.

    ltp: long-term plasticity as the production engine applies it to its
    aggregated conductances (delays 0): step t's NMDA sums use the weights
    before step t - 1's LTP, then that LTP rewrites the weights and adds
    df*dg*st(t - 1) of each rewritten linear record to the conductance its
    post folds at step t + 1, then step t's spikes are pushed with the new
    weights.  The final weights (after the last step's LTP) are returned
    last."""
    f, s = na.fields, na.syn
    n = na.n
    if drive is None:
        assert not np.any(f["pb"]), "external drive is random: pass its draws"
        assert not np.any(f["inj_std"]), "injection noise is random: pass its draws"
    else:
        hits_in, gauss_in = drive
        assert hits_in.shape[0] >= steps and hits_in.shape[1] == n
    get = lambda k: np.asarray(f[k], np.float64)  # noqa: E731
    vrev = get("Vrev").reshape(5, n)
    dfs = get("dfst").reshape(5, n)
    vth, vreset, df, ef, dvm, cm = get("Vth"), get("Vreset"), get("df"), get("ef"), get("dVmax"), get("Cm")
    leak = get("gl") * get("El") * 1e3
    mg = get("nmda_mg")
    rf = np.asarray(f["RfPed"], np.int64)
    sd = np.asarray(f["SpiDy"], np.int64)
    act = np.asarray(f["act"], np.int64)
    inj = np.where(act & ACT_INJ, get("inj_mean"), 0.0)
    extg = get("ext_g").reshape(5, n)
    ndfxt = get("nmda_dfxt")
    nefas = get("nmda_efst") * get("nmda_as")
    est = np.zeros((4, n))
    ex, es = np.zeros(n), np.zeros(n)
    pre = np.asarray(s["pre"], np.int64)
    post = np.asarray(s["post"], np.int64)
    rec = np.asarray(s["rec"], np.int64)
    w = np.asarray(s["g"], np.float64)
    dl = np.asarray(s["delay"], np.int64) if s.get("delay") is not None else np.zeros(pre.size, np.int64)
    # presynaptic kinetics: the decay of a neuron's gate is its targets' df
    pdf = np.zeros((4, n))
    pdfxt, pdfst, pefas = np.zeros(n), np.zeros(n), np.zeros(n)
    for e in range(pre.size):
        a, b, r = pre[e], post[e], rec[e]
        if r != NMDA:
            pdf[r, a] = dfs[r, b]
        else:
            pdfxt[a] = f["nmda_dfxt"][b]
            pdfst[a] = dfs[NMDA, b]
            pefas[a] = np.float64(np.float32(f["nmda_efst"][b] * f["nmda_as"][b]))
    tm = na.tm
    tm_on = np.zeros(n, bool)
    if tm is not None:
        tm_on = np.asarray(tm["enabled"], bool)
        U = np.broadcast_to(np.asarray(tm.get("U", 0.2), np.float32), (n,)).astype(np.float64)
        dfr = np.exp(-np.float32(na.dt) / np.broadcast_to(np.asarray(tm.get("tau_rec", 200.0), np.float32), (n,)))
        dff = np.exp(-np.float32(na.dt) / np.broadcast_to(np.asarray(tm.get("tau_fac", 600.0), np.float32), (n,)))
        dfr, dff = dfr.astype(np.float32).astype(np.float64), dff.astype(np.float32).astype(np.float64)
        tu = U.astype(np.float32)
        tx = np.ones(n, np.float32)
    dmax = int(dl.max()) if dl.size else 0
    arrive = np.zeros((steps + dmax + 2, 4, n))
    s_hist = np.zeros((steps + 1, n))
    V = np.full(n, -70.0)
    cnt = np.zeros(n, np.int64)
    ns = np.zeros(n, np.int64)
    G = np.zeros((4, n))
    sp = np.zeros((4, n))
    xp = np.zeros(n)
    spre = np.zeros(n)
    nm = rec == NMDA
    if ltp:
        assert not np.any(dl), "LTP runs with delays 0"
        wf = np.asarray(s["g"], np.float32).copy()
        elig = np.ones(pre.size, bool) if s.get("ltp") is None else np.asarray(s["ltp"], bool)
        dflp = np.asarray(f["ltp_dfLP"], np.float32)
        lpos, lneg = np.asarray(f["ltp_PosISI"], np.float32), np.asarray(f["ltp_NegISI"], np.float32)
        spd = np.asarray(f["ltp_SpiLPDy"], np.int64)
        ltp_on = (act & ACT_LTP) != 0
        lp = np.zeros(n, np.float32)
        clp = np.zeros(n, np.int64)
        spk_prev = np.zeros(n, bool)
    spikes, Vout = [], np.zeros((steps, n))
    Irep = np.zeros((5, n))
    Iout = np.zeros((steps, 5, n)) if extra else None
    NSout = np.zeros((steps, n), np.int64) if extra else None
    for t in range(steps):
        if t >= 1:
            G = dfs[:4] * G + arrive[t - 1]
        g = np.zeros((5, n))
        g[:4] = G
        idx = t - 1 - dl[nm]
        sh = np.where(idx >= 0, s_hist[np.maximum(idx, 0), pre[nm]], 0.0)
        g[NMDA] = np.bincount(post[nm], w[nm] * sh, n)
        if ltp and spk_prev.any():
            # LTP of step t - 1 (LP and gates as they were after that step)
            w_old = wf.copy()
            wf = ltp_weights(wf, pre, post, elig, spk_prev, lp, lneg, lpos)
            w = wf.astype(np.float64)
            dg = w - w_old.astype(np.float64)
            lin = ~nm & (dg != 0)
            np.add.at(arrive[t], (rec[lin], post[lin]), dfs[rec[lin], post[lin]] * dg[lin] * sp[rec[lin], pre[lin]])
        isyn = inj
        if drive is not None:
            h = hits_in[t].astype(np.int64)
            for r in range(4):
                on = (act & ACT_EXT[r]) != 0
                est[r] = np.where(on, np.where(h & (1 << r), est[r] + 1.0, est[r] * dfs[r]), est[r])
                g[r] = np.where(on, g[r] + extg[r] * est[r], g[r])
            on = (act & ACT_NMDA) != 0
            ex = np.where(on, np.where(h & (1 << NMDA), ex + 1.0, ex * ndfxt), ex)
            es = np.where(on, dfs[NMDA] * es + nefas * ex * (1.0 - es), es)
            g[NMDA] = np.where(on, g[NMDA] + extg[NMDA] * es, g[NMDA])
            isyn = np.where(act & ACT_INJ, gauss_in[t], 0.0)
        fire_now = (ns & NS_FIRE) != 0
        v = V.copy()
        Ir = g * (vrev - v)
        Ir[NMDA] = g[NMDA] * (vrev[NMDA] - v) / (1.0 + mg * np.exp(-0.062 * v) / 3.57)
        I = Ir.sum(0) + isyn * 1e3 + leak
        I = 1e-3 * I / cm
        ovf, udf = I > dvm, I < -dvm
        ns = np.where(fire_now, ns, np.where(ovf, (ns | NS_OVF) & ~NS_UDF,
                                             np.where(udf, (ns & ~NS_OVF) | NS_UDF, ns & ~(NS_OVF | NS_UDF))))
        I = np.clip(I, -dvm, dvm)
        Irep = np.where(fire_now, Irep, Ir)
        Vi = df * v + ef * I
        crossed = ~fire_now & (Vi > vth)
        V = np.where(fire_now, V, Vi)
        ns = np.where(crossed, ns | NS_FIRE, ns)
        fire = fire_now | crossed
        ref = fire & (cnt < rf)
        V = np.where(ref, np.where(cnt == 0, 0.0, vreset), V)
        ns = np.where(ref, np.where(cnt == sd, ns | NS_SPIKE, ns & ~NS_SPIKE), ns)
        done = fire & ~ref
        cnt = np.where(ref, cnt + 1, np.where(done, 0, cnt))
        ns = np.where(done, ns & ~NS_FIRE, ns)
        if ltp:
            ns, lp, clp = lp_trace(ns, crossed, ltp_on, lp, clp, spd, dflp)
        Vout[t] = V
        if extra:
            Iout[t] = Irep
            NSout[t] = ns
        spk = (ns & NS_SPIKE) != 0
        spikes.append(np.nonzero(spk)[0].astype(np.uint32))
        inc = np.ones(n)
        if tm is not None:
            u, x = tu.astype(np.float64), tx.astype(np.float64)
            u_s = u + U * (1.0 - u)
            rel = u_s * x
            u_n = U + (u - U) * dff
            x_n = 1.0 + (x - 1.0) * dfr
            inc = np.where(tm_on & spk, rel, 1.0)
            tu = np.where(tm_on, np.where(spk, u_s, u_n), u).astype(np.float32)
            tx = np.where(tm_on, np.where(spk, x - rel, x_n), x).astype(np.float32)
        cinc = inc + sp * (1.0 - pdf)
        sp = np.where(spk, sp + inc, sp * pdf)
        xp = np.where(spk, xp + inc, xp * pdfxt)
        spre = pdfst * spre + pefas * xp * (1.0 - spre)
        s_hist[t] = spre
        if spk.any():
            for e in np.nonzero(spk[pre] & ~nm)[0]:
                arrive[t + dl[e], rec[e], post[e]] += w[e] * cinc[rec[e], pre[e]]
        if ltp:
            spk_prev = spk
    out = (spikes, Vout, Iout, NSout) if extra else (spikes, Vout)
    if ltp:
        if spk_prev.any():
            wf = ltp_weights(wf, pre, post, elig, spk_prev, lp, lneg, lpos)
        out = out + (wf,)
    return out


NS_LP_FIRE, NS_LP_SPIKE = 4, 8
ACT_LTP = 8192


def ltp_rule(g, lp, x):
    """One LTP update of float32 weights g (code/EqsGnl2.cpp:1005-1044):
    additive g + lp*x when x > 0, multiplicative g*(1 + lp*x) otherwise, in
    float32 with one rounding per operation, as the reference computes it
    (its g, LP and NegISI / PosISI are float)."""
    g, lp, x = (np.asarray(v, np.float32) for v in (g, lp, x))
    one = np.float32(1.0)
    return np.where(x > 0, g + lp * x, g * (one + lp * x)).astype(np.float32)


def ltp_weights(w, pre, post, elig, spk, lp, lneg, lpos):
    """The LTP of one step on float32 weights w (synapse-list order): the
    flagged records whose pre or post spiked, the presynaptic rule first
    (post's LP, pre's NegISI), then the postsynaptic one (pre's LP and
    PosISI)."""
    w = w.copy()
    sa, sb = spk[pre], spk[post]
    m = elig & (sa | sb)
    wn = w[m]
    a_, b_ = pre[m], post[m]
    wn = np.where(sa[m], ltp_rule(wn, lp[b_], lneg[a_]), wn)
    wn = np.where(sb[m], ltp_rule(wn, lp[a_], lpos[a_]), wn)
    w[m] = wn
    return w


def lp_trace(ns, crossed, ltp_on, lp, clp, spd, dflp):
    """LP_FIRE at a threshold crossing, then firLP and ltpEul
    (code/EqsGnl2.cpp:207-216, :254-280) for the neurons with LTP on; LP is
    float32 as in the reference."""
    ns = np.where(crossed & ltp_on, ns | NS_LP_FIRE, ns)
    lpf = ltp_on & ((ns & NS_LP_FIRE) != 0)
    hit = lpf & (clp == spd)
    ns = np.where(hit, (ns | NS_LP_SPIKE) & ~NS_LP_FIRE, np.where(ltp_on, ns & ~NS_LP_SPIKE, ns))
    clp = np.where(hit, 0, np.where(lpf, clp + 1, clp))
    lp = np.where(ltp_on, np.where((ns & NS_LP_SPIKE) != 0, lp + np.float32(1.0), dflp * lp), lp)
    return ns, lp.astype(np.float32), clp


def simulate_ltp(na, steps: int, drive=None):
    """Float64 restatement with long-term plasticity, in the reference's
    per-record form (code/EqsGnl2.cpp:404-502, :1005-1044) rather than the
    production engine's aggregated conductances: every synapse-list entry is a
    record with its own gate (linear: st <- st + inc on a presynaptic spike,
    st*df of its post otherwise; NMDA: its own x, s), the conductance a post
    sees at step t is sum(g*st) over its records after step t - 1's gather,
    and after each step's gather LTP rewrites g of the records flagged in the
    list (all when the list has no flags): on a presynaptic spike with the
    post's LP and the pre's NegISI, then on a postsynaptic spike with the
    pre's LP and PosISI.  The LP trace follows firLP / ltpEul
    (code/EqsGnl2.cpp:207-216, :254-280).  Delays must be 0.  Returns
    (spikes per step, V [steps, n], final weights in synapse-list order).
    The LP trace and the weight updates are float32, as in the reference
    and the engine (in both of its modes); everything else is float64."""
    f, s = na.fields, na.syn
    n = na.n
    if drive is None:
        assert not np.any(f["pb"]), "external drive is random: pass its draws"
        assert not np.any(f["inj_std"]), "injection noise is random: pass its draws"
    else:
        hits_in, gauss_in = drive
    get = lambda k: np.asarray(f[k], np.float64)  # noqa: E731
    vrev = get("Vrev").reshape(5, n)
    dfs = get("dfst").reshape(5, n)
    vth, vreset, df, ef, dvm, cm = get("Vth"), get("Vreset"), get("df"), get("ef"), get("dVmax"), get("Cm")
    leak = get("gl") * get("El") * 1e3
    mg = get("nmda_mg")
    rf = np.asarray(f["RfPed"], np.int64)
    sd = np.asarray(f["SpiDy"], np.int64)
    act = np.asarray(f["act"], np.int64)
    inj = np.where(act & ACT_INJ, get("inj_mean"), 0.0)
    extg = get("ext_g").reshape(5, n)
    ndfxt = get("nmda_dfxt")
    nefas = get("nmda_efst") * get("nmda_as")
    dflp = np.asarray(f["ltp_dfLP"], np.float32)
    lpos, lneg = np.asarray(f["ltp_PosISI"], np.float32), np.asarray(f["ltp_NegISI"], np.float32)
    spd = np.asarray(f["ltp_SpiLPDy"], np.int64)
    ltp_on = (act & ACT_LTP) != 0
    pre = np.asarray(s["pre"], np.int64)
    post = np.asarray(s["post"], np.int64)
    rec = np.asarray(s["rec"], np.int64)
    w = np.asarray(s["g"], np.float32).copy()
    if s.get("delay") is not None:
        assert not np.any(s["delay"]), "the LTP restatement has no delays"
    elig = np.ones(pre.size, bool) if s.get("ltp") is None else np.asarray(s["ltp"], bool)
    nm = rec == NMDA
    # per-record kinetics: the post's decay per receptor, NMDA the post's
    # x decay and efst*as (float32 product, as the engine forms it)
    rdf = dfs[np.minimum(rec, 4), post]
    rdfxt = np.asarray(f["nmda_dfxt"], np.float64)[post]
    refas = (np.asarray(f["nmda_efst"], np.float32) * np.asarray(f["nmda_as"], np.float32)).astype(np.float64)[post]
    tm = na.tm
    tm_on = np.zeros(n, bool)
    if tm is not None:
        tm_on = np.asarray(tm["enabled"], bool)
        U = np.broadcast_to(np.asarray(tm.get("U", 0.2), np.float32), (n,)).astype(np.float64)
        dfr = np.exp(-np.float32(na.dt) / np.broadcast_to(np.asarray(tm.get("tau_rec", 200.0), np.float32), (n,)))
        dff = np.exp(-np.float32(na.dt) / np.broadcast_to(np.asarray(tm.get("tau_fac", 600.0), np.float32), (n,)))
        dfr, dff = dfr.astype(np.float32).astype(np.float64), dff.astype(np.float32).astype(np.float64)
        tu = U.astype(np.float32)
        tx = np.ones(n, np.float32)
    st = np.zeros(pre.size)   # linear records' gates (unused for NMDA records)
    xr = np.zeros(pre.size)   # NMDA records' x, s
    sr = np.zeros(pre.size)
    H = np.zeros((5, n))      # conductances of the last gather
    est = np.zeros((4, n))
    ex, es = np.zeros(n), np.zeros(n)
    V = np.full(n, -70.0)
    cnt = np.zeros(n, np.int64)
    ns = np.zeros(n, np.int64)
    lp = np.zeros(n, np.float32)
    clp = np.zeros(n, np.int64)
    spikes, Vout = [], np.zeros((steps, n))
    for t in range(steps):
        g = H.copy()
        isyn = inj
        if drive is not None:
            h = hits_in[t].astype(np.int64)
            for r in range(4):
                on = (act & ACT_EXT[r]) != 0
                est[r] = np.where(on, np.where(h & (1 << r), est[r] + 1.0, est[r] * dfs[r]), est[r])
                g[r] = np.where(on, g[r] + extg[r] * est[r], g[r])
            on = (act & ACT_NMDA) != 0
            ex = np.where(on, np.where(h & (1 << NMDA), ex + 1.0, ex * ndfxt), ex)
            es = np.where(on, dfs[NMDA] * es + nefas * ex * (1.0 - es), es)
            g[NMDA] = np.where(on, g[NMDA] + extg[NMDA] * es, g[NMDA])
            isyn = np.where(act & ACT_INJ, gauss_in[t], 0.0)
        fire_now = (ns & NS_FIRE) != 0
        v = V.copy()
        Ir = g * (vrev - v)
        Ir[NMDA] = g[NMDA] * (vrev[NMDA] - v) / (1.0 + mg * np.exp(-0.062 * v) / 3.57)
        I = Ir.sum(0) + isyn * 1e3 + leak
        I = 1e-3 * I / cm
        I = np.clip(I, -dvm, dvm)
        Vi = df * v + ef * I
        crossed = ~fire_now & (Vi > vth)
        V = np.where(fire_now, V, Vi)
        ns = np.where(crossed, ns | NS_FIRE, ns)
        fire = fire_now | crossed
        ref = fire & (cnt < rf)
        V = np.where(ref, np.where(cnt == 0, 0.0, vreset), V)
        ns = np.where(ref, np.where(cnt == sd, ns | NS_SPIKE, ns & ~NS_SPIKE), ns)
        done = fire & ~ref
        cnt = np.where(ref, cnt + 1, np.where(done, 0, cnt))
        ns = np.where(done, ns & ~NS_FIRE, ns)
        ns, lp, clp = lp_trace(ns, crossed, ltp_on, lp, clp, spd, dflp)
        Vout[t] = V
        spk = (ns & NS_SPIKE) != 0
        spikes.append(np.nonzero(spk)[0].astype(np.uint32))
        inc = np.ones(n)
        if tm is not None:
            u, x = tu.astype(np.float64), tx.astype(np.float64)
            u_s = u + U * (1.0 - u)
            rel = u_s * x
            u_n = U + (u - U) * dff
            x_n = 1.0 + (x - 1.0) * dfr
            inc = np.where(tm_on & spk, rel, 1.0)
            tu = np.where(tm_on, np.where(spk, u_s, u_n), u).astype(np.float32)
            tx = np.where(tm_on, np.where(spk, x - rel, x_n), x).astype(np.float32)
        # gather of step t (code/EqsGnl2.cpp:404-502): every record's gate,
        # then sum(g * st) per post and receptor, over the weights before LTP
        sa = spk[pre]
        st = np.where(sa, st + inc[pre], st * rdf)
        xr = np.where(sa, xr + inc[pre], xr * rdfxt)
        sr = dfs[NMDA, post] * sr + refas * xr * (1.0 - sr)
        gate = np.where(nm, sr, st)
        H = np.zeros((5, n))
        np.add.at(H, (rec, post), w.astype(np.float64) * gate)
        # LTP of step t
        if spk.any():
            w = ltp_weights(w, pre, post, elig, spk, lp, lneg, lpos)
    return spikes, Vout, w
