"""Synthetic network.conf / network.pro writers for the benchmark and test
workloads.

The reference's real connectome inputs are not available, so seeded synthetic
networks with the documented shapes stand in for them:

* ``write_two_pop`` — two LIF populations E=800 / I=200, all-pairs connection
  probability 0.2, AMPA/NMDA from E and GABA from I, 2.4 kHz external Poisson
  drive on AMPA (the CPU-runnable plain method).
* ``connectome`` / ``write_connectome`` — a connectome-shaped network written
  the way the reference's brain models are (code/experiment/seizure): one
  population per neuron, one ``TargetPopulation`` block per synapse.  Neurons
  are split into regions; out-degrees are lognormal, most targets are drawn in
  the source's region, 70% of neurons are excitatory (AMPA + NMDA) and 30%
  inhibitory (GABA), weights are lognormal, drive frequency is per region and
  optional integer delays ride on the ``Delay`` keyword (ignored by the
  reference parser, which treats unknown keywords inside a target block as
  no-ops).

The files use only the reference's own keywords (code/parser.cpp:346-871,
:1069-1338) plus ``Delay``.
"""
from __future__ import annotations

import dataclasses
import os
from typing import Dict, List, Optional, Sequence

import numpy as np

REC_NAMES = {"AMPA": 0, "GABA": 1, "Ach": 2, "GluCl": 3, "NMDA": 4}


def _fmt(x: float) -> str:
    return ("%.9g" % float(x))


@dataclasses.dataclass
class Connectome:
    """A connectome-shaped synthetic network (arrays; one neuron per population)."""
    n: int
    region: np.ndarray        # [n] region id
    excit: np.ndarray         # [n] bool
    freq_ext: np.ndarray      # [n] Hz of AMPA drive
    pre: np.ndarray           # [C] presynaptic neuron of each connection
    post: np.ndarray          # [C]
    weight: np.ndarray        # [C] nS (AMPA or GABA efficacy; NMDA gets weight*k_nmda)
    delay_ms: np.ndarray      # [C] integer ms (0 = reference timing)
    k_nmda: float
    gaba_scale: float
    ext_eff: float

    @property
    def n_connections(self) -> int:
        return int(self.pre.size)

    @property
    def n_entries(self) -> int:
        """Synapse entries (one per (pre, post, receptor))."""
        return int(self.pre.size + np.count_nonzero(self.excit[self.pre]))


def connectome(n: int = 20000, regions: int = 58, mean_degree: float = 120.0,
               sigma_degree: float = 1.0, intra: float = 0.8, frac_exc: float = 0.7,
               w_median: float = 1.0, w_sigma: float = 0.8, ampa_scale: float = 0.25,
               k_nmda: float = 0.06, gaba_scale: float = 1.2, ext_eff: float = 1.0,
               f_lo: float = 1000.0, f_hi: float = 4000.0, delays: bool = True,
               d_lo: int = 1, d_hi: int = 5, seed: int = 1) -> Connectome:
    """Draws a connectome-shaped network.

    Out-degree ~ round(lognormal(ln(mean) - sigma^2/2, sigma)), so its mean is
    ``mean_degree``; a fraction ``intra`` of each neuron's targets lies in its
    own region; weights ~ lognormal(ln w_median, w_sigma) scaled per receptor.
    """
    rng = np.random.default_rng(seed)
    # region sizes: multinomial with uniform probabilities (each region >= 1)
    sizes = rng.multinomial(n - regions, np.full(regions, 1.0 / regions)) + 1
    region = np.repeat(np.arange(regions, dtype=np.int32), sizes)
    starts = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.int64)
    excit = rng.random(n) < frac_exc
    mu = np.log(mean_degree) - 0.5 * sigma_degree ** 2
    deg = np.rint(rng.lognormal(mu, sigma_degree, n)).astype(np.int64)
    deg = np.clip(deg, 0, n - 1)
    pre_l, post_l = [], []
    for i in range(n):
        k = int(deg[i])
        if k == 0:
            continue
        r = region[i]
        k_in = int(rng.binomial(k, intra))
        k_in = min(k_in, int(sizes[r]) - 1)
        k_out = min(k - k_in, n - int(sizes[r]))
        tin = rng.choice(int(sizes[r]) - 1, size=k_in, replace=False) + starts[r] if k_in else np.empty(0, np.int64)
        tin = tin + (tin >= i)  # skip self
        if k_out:
            # outside the region: sample from the complement
            tout = rng.choice(n - int(sizes[r]), size=k_out, replace=False)
            tout = tout + (tout >= starts[r]) * int(sizes[r])
        else:
            tout = np.empty(0, np.int64)
        t = np.sort(np.concatenate([tin, tout]))
        pre_l.append(np.full(t.size, i, np.int64))
        post_l.append(t)
    pre = np.concatenate(pre_l).astype(np.uint32)
    post = np.concatenate(post_l).astype(np.uint32)
    w = rng.lognormal(np.log(w_median), w_sigma, pre.size).astype(np.float32)
    w = np.where(excit[pre], w * ampa_scale, w * gaba_scale).astype(np.float32)
    if delays:
        d = rng.integers(d_lo, d_hi + 1, pre.size).astype(np.uint16)
    else:
        d = np.zeros(pre.size, np.uint16)
    freq_region = rng.uniform(f_lo, f_hi, regions)
    freq = freq_region[region].astype(np.float32)
    return Connectome(n=n, region=region, excit=excit, freq_ext=freq, pre=pre, post=post,
                      weight=w, delay_ms=d, k_nmda=float(k_nmda), gaba_scale=float(gaba_scale),
                      ext_eff=float(ext_eff))


def connectome_fast(n: int = 20000, regions: int = 58, mean_degree: float = 120.0,
                    sigma_degree: float = 1.0, intra: float = 0.8, frac_exc: float = 0.7,
                    w_median: float = 1.0, w_sigma: float = 0.8, ampa_scale: float = 0.25,
                    k_nmda: float = 0.06, gaba_scale: float = 1.2, ext_eff: float = 1.0,
                    f_lo: float = 1000.0, f_hi: float = 4000.0, delays: bool = True,
                    d_lo: int = 1, d_hi: int = 5, seed: int = 1) -> Connectome:
    """The distributions of :func:`connectome`, drawn vectorised (for sweeps
    of hundreds of instances).  Intra-region targets are distinct (a random
    key per (source, region member), smallest keys win); out-of-region
    targets are drawn with replacement and deduplicated, which at ~24 draws
    from ~n targets removes a negligible fraction.  Not draw-for-draw equal
    to :func:`connectome`."""
    rng = np.random.default_rng(seed)
    sizes = rng.multinomial(n - regions, np.full(regions, 1.0 / regions)) + 1
    region = np.repeat(np.arange(regions, dtype=np.int32), sizes)
    starts = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.int64)
    excit = rng.random(n) < frac_exc
    mu = np.log(mean_degree) - 0.5 * sigma_degree ** 2
    deg = np.clip(np.rint(rng.lognormal(mu, sigma_degree, n)).astype(np.int64), 0, n - 1)
    k_in = rng.binomial(deg, intra)
    rs = sizes[region]
    k_in = np.minimum(k_in, rs - 1)
    k_out = np.minimum(deg - k_in, n - rs)
    pre_l, post_l = [], []
    for r in range(regions):
        s, a = int(sizes[r]), int(starts[r])
        if s < 2:
            continue
        kk = k_in[a:a + s]
        if s > 2048:
            # large regions: targets drawn with replacement (self excluded)
            # and deduplicated below; at ~100 draws from thousands the loss
            # is a fraction of a percent
            src = np.repeat(np.arange(s), kk)
            u = rng.integers(0, s - 1, src.size)
            pre_l.append(src + a)
            post_l.append(u + (u >= src) + a)
            continue
        keys = rng.random((s, s))
        np.fill_diagonal(keys, 2.0)  # never self
        order = np.argsort(keys, axis=1)
        take = np.arange(s)[None, :] < kk[:, None]
        src = np.repeat(np.arange(s), kk)
        pre_l.append(src + a)
        post_l.append(order[take] + a)
    tot_out = int(k_out.sum())
    src = np.repeat(np.arange(n, dtype=np.int64), k_out)
    u = rng.integers(0, n - rs[src], tot_out)
    ra, rsz = starts[region[src]], rs[src]
    tgt = u + (u >= ra) * rsz
    pre_l.append(src)
    post_l.append(tgt)
    pre = np.concatenate(pre_l)
    post = np.concatenate(post_l)
    key = pre * n + post
    key.sort()
    key = key[np.concatenate([[True], key[1:] != key[:-1]])]
    pre = (key // n).astype(np.uint32)
    post = (key % n).astype(np.uint32)
    w = rng.lognormal(np.log(w_median), w_sigma, pre.size).astype(np.float32)
    w = np.where(excit[pre], w * ampa_scale, w * gaba_scale).astype(np.float32)
    d = (rng.integers(d_lo, d_hi + 1, pre.size) if delays else np.zeros(pre.size)).astype(np.uint16)
    freq_region = rng.uniform(f_lo, f_hi, regions)
    freq = freq_region[region].astype(np.float32)
    return Connectome(n=n, region=region, excit=excit, freq_ext=freq, pre=pre, post=post,
                      weight=w, delay_ms=d, k_nmda=float(k_nmda), gaba_scale=float(gaba_scale),
                      ext_eff=float(ext_eff))


_POP_HEADER = """NeuralPopulation: {name}
N=1
C=0.5
Taum=20
RestPot=-70
Threshold=-50
ResetPot=-55
RefractoryPeriod=2
SpikeDly=0

Receptor:AMPA
Tau=2
RevPot=0
FreqExt={freq}
MeanExtEff={ext}
EndReceptor

Receptor:GABA
Tau=5
RevPot=-70
FreqExt=0
EndReceptor

Receptor:NMDA
Tau=100
TauXT=2
RevPot=0
FreqExt=0
EndReceptor

"""


def write_connectome(c: Connectome, path: str, with_delays: bool = True, ltp: Optional[dict] = None) -> None:
    """Writes the network as one population per neuron (the reference's
    connectome format); each connection becomes one target block per
    receptor.  ``ltp`` (keys tLP, SpiLPDy, PosISI, NegISI) adds the
    long-term plasticity keywords to every population
    (code/parser.cpp:385-392, :559-575)."""
    order = np.argsort(c.pre, kind="stable")
    pre, post, w, d = c.pre[order], c.post[order], c.weight[order], c.delay_ms[order]
    bounds = np.searchsorted(pre, np.arange(c.n + 1))
    ltp_lines = "".join("LTP_%s=%s\n" % (k, _fmt(ltp[k])) for k in ("tLP", "SpiLPDy", "PosISI", "NegISI")) if ltp else ""
    with open(path, "w") as f:
        for i in range(c.n):
            head = _POP_HEADER.format(name="n%d" % i, freq=_fmt(c.freq_ext[i]), ext=_fmt(c.ext_eff))
            if ltp:
                head = head.replace("SpikeDly=0\n", "SpikeDly=0\n" + ltp_lines, 1)
            parts = [head]
            a, b = bounds[i], bounds[i + 1]
            exc = bool(c.excit[i])
            for e in range(a, b):
                dl = "Delay=%d\n" % int(d[e]) if (with_delays and d[e] > 0) else ""
                if exc:
                    parts.append("TargetPopulation: n%d\nTargetReceptor=AMPA\nMeanEff=%s\n%sEndTargetPopulation\n\n"
                                 % (post[e], _fmt(w[e]), dl))
                    parts.append("TargetPopulation: n%d\nTargetReceptor=NMDA\nMeanEff=%s\n%sEndTargetPopulation\n\n"
                                 % (post[e], _fmt(np.float32(w[e] * c.k_nmda)), dl))
                else:
                    parts.append("TargetPopulation: n%d\nTargetReceptor=GABA\nMeanEff=%s\n%sEndTargetPopulation\n\n"
                                 % (post[e], _fmt(w[e]), dl))
            parts.append("EndNeuralPopulation\n\n")
            f.write("".join(parts))


def write_two_pop(path: str, n_e: int = 800, n_i: int = 200, p: float = 0.2,
                  freq_ext: float = 2400.0, ampa: float = 0.05, nmda: float = 0.02,
                  gaba: float = 8.0, extra_pop: str = "", delay_ms: float = 0.0,
                  gap: float = 0.0, gap_p: float = 0.02) -> None:
    """E/I two-population network (the CPU-runnable plain method); gap > 0
    adds gap junctions E->E and I->I (MeanEff gap, Connectivity gap_p)."""
    dl = ("Delay=%s\n" % _fmt(delay_ms)) if delay_ms > 0 else ""
    recs = """Receptor:AMPA
Tau=2
RevPot=0
FreqExt={f}
MeanExtEff=2.1
EndReceptor

Receptor:GABA
Tau=5
RevPot=-70
EndReceptor

Receptor:NMDA
Tau=100
TauXT=2
RevPot=0
EndReceptor
""".format(f=_fmt(freq_ext))
    body = ""
    gl_e = (("E", "GAP", gap, gap_p),) if gap > 0 else ()
    gl_i = (("I", "GAP", gap, gap_p),) if gap > 0 else ()
    for name, n, links in (("E", n_e, tuple((t, r, e, p) for t, r, e in (("E", "AMPA", ampa), ("I", "AMPA", ampa),
                                                                       ("E", "NMDA", nmda), ("I", "NMDA", nmda))) + gl_e),
                           ("I", n_i, tuple((t, r, e, p) for t, r, e in (("E", "GABA", gaba), ("I", "GABA", gaba))) + gl_i)):
        body += """NeuralPopulation: {name}
N={n}
C=0.5
Taum=20
RestPot=-70
Threshold=-50
ResetPot=-55
RefractoryPeriod=2
SpikeDly=0

{recs}
""".format(name=name, n=n, recs=recs)
        for tgt, rec, eff, pc in links:
            body += ("TargetPopulation: {t}\nTargetReceptor={r}\nMeanEff={e}\nConnectivity={p}\n{dl}"
                     "EndTargetPopulation\n\n").format(t=tgt, r=rec, e=_fmt(eff), p=_fmt(pc),
                                                        dl=dl if rec != "GAP" else "")
        body += "EndNeuralPopulation\n\n"
    with open(path, "w") as f:
        f.write(body + extra_pop)


def write_pro(path: str, t_end_ms: float, seeds: Sequence[int] = (1,),
              outputs: Sequence[Dict] = ({"name": "Spikes.dat", "type": "Spike", "pop": "AllPopulation"},),
              events: Sequence[Dict] = (), groups: Dict[str, Sequence[str]] = None) -> None:
    """Protocol file: RandomSeeds macro (never -udfsed, which also turns STD
    on), events, EndTrial at ``t_end_ms``, outputs."""
    out = ["DefineMacro\n"]
    for g, members in (groups or {}).items():
        out.append("GroupName:%s\nGroupMembers:%s\nEndGroupMembers\n" % (g, ",".join(members)))
    if seeds:
        out.append("RandomSeeds: %s\nEndRandomSeeds\n" % " ".join(str(int(s)) for s in seeds))
    out.append("EndDefineMacro\n\n")
    for ev in events:
        out.append("EventTime %s\nType=%s\nLabel=#1#\nPopulation: %s\n" % (_fmt(ev["t"]), ev["type"], ev["pop"]))
        if ev["type"] == "ChangeExtFreq":
            out.append("Receptor: %s\nFreqExt=%s\n" % (ev.get("rec", "AMPA"), _fmt(ev["f"])))
        else:
            out.append("GaussMean=%s\nGaussSTD=%s\n" % (_fmt(ev["mean"]), _fmt(ev["std"])))
        out.append("EndEvent\n\n")
    out.append("EventTime %s\nType=EndTrial\nLabel=End_of_the_trial\nEndEvent\n\n" % _fmt(t_end_ms))
    out.append("OutControl\n")
    for o in outputs:
        out.append("FileName:%s\nType=%s\n" % (o["name"], o["type"]))
        if "win" in o:
            out.append("FiringRateWindow=%s\n" % _fmt(o["win"]))
        if "step" in o:
            out.append("PrintStep=%s\n" % _fmt(o["step"]))
        if o.get("sum"):
            out.append("SumAllPopulation:true\n")
        if o.get("align"):
            out.append("Align:true\n")
        pops = o.get("pop", "AllPopulation")
        for p in ([pops] if isinstance(pops, str) else pops):
            out.append("population:%s\n" % p)
        out.append("EndOutputFile\n\n")
    out.append("EndOutControl\n")
    with open(path, "w") as f:
        f.write("".join(out))
