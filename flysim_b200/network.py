"""Networks built directly from arrays (no .conf text), for the production
modes, the batched engine and the benchmarks.

Per-neuron constants follow the reference's set-up formulas
(code/NetSimGnl2_BulPp.cpp:159-278): gl = C/Taum, df = exp(-dt/Taum),
ef = Taum*(1-df), dfst = exp(-dt/Tau) per receptor, NMDA dfxt = exp(-dt/TauXT)
and efst = Tau*(1-dfst), dVmax = (Vth - Vrev_GABA)/ef, drive probability
pb = FreqExt*dt*1e-3, receptors a population does not declare get
Vrev 0 (AMPA/NMDA/ACh) or -90 (GABA/GluCl) and dfst 0.1.  The refractory
and spike-delay step counts use the reference parser's float expressions
(code/parser.cpp:508,513).
"""
from __future__ import annotations

import ctypes as C
import dataclasses
from typing import List, Optional

import numpy as np

from . import (ACT, DEFAULT_ACT, FS_AMPA, FS_GABA, FS_ACH, FS_GCL, FS_NMDA, FS_NREC, NetDesc, Neurons, SynList,
               TmParams)

_f = C.POINTER(C.c_float)
_u32 = C.POINTER(C.c_uint32)
_i32 = C.POINTER(C.c_int32)
_u8 = C.POINTER(C.c_uint8)
_u16 = C.POINTER(C.c_uint16)

F32 = np.float32


@dataclasses.dataclass
class NetArrays:
    """Numpy arrays behind a fs_net_desc (keeps them alive)."""
    n: int
    dt: float
    fields: dict
    syn: dict
    tm: Optional[dict]
    desc: NetDesc = None
    _keep: list = None

    @property
    def n_syn(self) -> int:
        return int(self.syn["pre"].size)


def _refractory_steps(ms: float, dt: float) -> int:
    return int(np.floor(F32(ms) / F32(dt)) + F32(dt))


def neuron_fields(n: int, dt: float, taum=20.0, cm=0.5, el=-70.0, vth=-50.0, vreset=-55.0, rf_ms=2.0,
                  spidy_ms=0.0, receptors=None, act=DEFAULT_ACT) -> dict:
    """SoA neuron parameters.  ``receptors`` maps a receptor index to a dict
    with Tau, Vrev, FExt (scalar or per-neuron array), ExtEff and, for NMDA,
    TauXT; receptors not listed get the reference's defaults."""
    dt = F32(dt)
    full = lambda v: np.broadcast_to(np.asarray(v, F32), (n,)).astype(F32)  # noqa: E731
    taum, cm, el, vth, vreset = full(taum), full(cm), full(el), full(vth), full(vreset)
    f = {}
    f["Vth"], f["El"], f["Cm"], f["Vreset"] = vth, el, cm, vreset
    f["gl"] = (cm / taum).astype(F32)
    f["df"] = np.exp(-dt / taum).astype(F32)
    f["ef"] = (taum * (F32(1) - f["df"])).astype(F32)
    f["RfPed"] = np.full(n, _refractory_steps(rf_ms, float(dt)), np.int32)
    f["SpiDy"] = np.full(n, int(np.floor(F32(spidy_ms) / dt)), np.int32)
    vrev = np.zeros((FS_NREC, n), F32)
    dfst = np.full((FS_NREC, n), F32(0.1), F32)
    vrev[FS_GABA] = -90.0
    vrev[FS_GCL] = -90.0
    ext_g = np.zeros((FS_NREC, n), F32)
    pb = np.zeros((FS_NREC, n), F32)
    nmda_dfxt = np.full(n, F32(0.1), F32)
    nmda_efst = np.full(n, F32(0.01), F32)
    for r, p in (receptors or {}).items():
        tau = full(p.get("Tau", 5.0))
        vrev[r] = full(p.get("Vrev", 0.0))
        dfst[r] = np.exp(-dt / tau).astype(F32)
        pb[r] = (full(p.get("FExt", 0.0)) * dt * F32(1e-3)).astype(F32)
        ext_g[r] = full(p.get("ExtEff", 2.1)) * full(p.get("ExtCon", 1.0))
        if r == FS_NMDA:
            nmda_dfxt = np.exp(-dt / full(p.get("TauXT", 2.0))).astype(F32)
            nmda_efst = (tau * (F32(1) - dfst[r])).astype(F32)
    f["dVmax"] = ((vth - vrev[FS_GABA]) / f["ef"]).astype(F32)
    f["Vrev"], f["dfst"], f["ext_g"], f["pb"] = vrev.ravel(), dfst.ravel(), ext_g.ravel(), pb.ravel()
    f["nmda_dfxt"], f["nmda_efst"] = nmda_dfxt, nmda_efst
    f["nmda_as"] = np.full(n, F32(0.6332), F32)
    f["nmda_mg"] = np.ones(n, F32)
    f["act"] = np.broadcast_to(np.asarray(act, np.uint32), (n,)).astype(np.uint32)
    f["inj_mean"] = np.zeros(n, F32)
    f["inj_std"] = np.zeros(n, F32)
    for k in ("stp_pv", "stp_dfD", "stp_efD", "stp_aF", "stp_dfF", "stp_efF", "stp_aCap", "stp_dfCap",
              "stp_aCar", "stp_dfCar", "stp_efCar", "ltp_dfLP", "ltp_PosISI", "ltp_NegISI"):
        f[k] = np.zeros(n, F32)
    f["ltp_SpiLPDy"] = np.zeros(n, np.int32)
    return f


def desc_from_arrays(n: int, dt: float, fields: dict, pre, post, rec, g, delay_steps=None,
                     tm: Optional[dict] = None, act_ctr: int = DEFAULT_ACT, ltp=None) -> NetArrays:
    """fs_net_desc over numpy arrays (production modes: flat synapse list).
    ``ltp``: per entry, whether long-term plasticity rewrites its weight
    (None: every entry, when act_ctr has the LTP bit)."""
    keep: List[np.ndarray] = []

    def p(a, ty, ct):
        a = np.ascontiguousarray(a, ty)
        keep.append(a)
        return a.ctypes.data_as(ct)

    nv = Neurons()
    nv.n = n
    for k in ("Vth", "El", "gl", "Cm", "Vreset", "df", "ef", "dVmax", "Vrev", "dfst", "nmda_dfxt", "nmda_efst",
              "nmda_as", "nmda_mg", "ext_g", "pb", "inj_mean", "inj_std", "stp_pv", "stp_dfD", "stp_efD",
              "stp_aF", "stp_dfF", "stp_efF", "stp_aCap", "stp_dfCap", "stp_aCar", "stp_dfCar", "stp_efCar",
              "ltp_dfLP", "ltp_PosISI", "ltp_NegISI"):
        setattr(nv, k, p(fields[k], np.float32, _f))
    for k in ("RfPed", "SpiDy", "ltp_SpiLPDy"):
        setattr(nv, k, p(fields[k], np.int32, _i32))
    nv.act = p(fields["act"], np.uint32, _u32)
    s = SynList()
    pre = np.ascontiguousarray(pre, np.uint32)
    s.n = pre.size
    s.pre = p(pre, np.uint32, _u32)
    s.post = p(post, np.uint32, _u32)
    s.rec = p(rec, np.uint8, _u8)
    s.g = p(g, np.float32, _f)
    s.delay = p(delay_steps if delay_steps is not None else np.zeros(pre.size, np.uint16), np.uint16, _u16)
    s.ltp = p(ltp, np.uint8, _u8) if ltp is not None else None
    d = NetDesc()
    d.dt = dt
    d.act_ctr = act_ctr
    d.neurons = nv
    d.compat = None
    d.syn = C.pointer(s)
    keep.append(s)
    if tm is not None:
        t = TmParams()
        t.enabled = p(tm["enabled"], np.uint8, _u8)
        t.U = p(np.broadcast_to(np.asarray(tm.get("U", 0.2), F32), (n,)), np.float32, _f)
        t.tau_rec = p(np.broadcast_to(np.asarray(tm.get("tau_rec", 200.0), F32), (n,)), np.float32, _f)
        t.tau_fac = p(np.broadcast_to(np.asarray(tm.get("tau_fac", 600.0), F32), (n,)), np.float32, _f)
        keep.append(t)
        d.tm = C.pointer(t)
    else:
        d.tm = None
    na = NetArrays(n=n, dt=dt, fields=fields,
                   syn=dict(pre=pre, post=np.asarray(post), rec=np.asarray(rec), g=np.asarray(g),
                            delay=np.asarray(delay_steps) if delay_steps is not None else None,
                            ltp=np.asarray(ltp, np.uint8) if ltp is not None else None),
                   tm=tm)
    na.desc = d
    na._keep = keep
    d._keep = keep
    return na


def connectome_net(c, dt: float = 0.1, with_delays: bool = True, tm: bool = False, ext_eff: Optional[float] = None,
                   gaba_gain: float = 1.0, ltp: Optional[dict] = None) -> NetArrays:
    """Production network of a :class:`flysim_b200.netgen.Connectome`: the same
    neurons and synapses as its .conf (one population per neuron).  ``ltp``
    (keys tLP, SpiLPDy in ms, PosISI, NegISI) switches long-term plasticity
    on for every neuron and synapse, as -LTP with those keywords in every
    population does (code/NetSimGnl2_BulPp.cpp:180-183, code/parser.cpp:559-575);
    its delays must then be 0."""
    n = c.n
    fields = neuron_fields(n, dt, receptors={
        FS_AMPA: dict(Tau=2.0, Vrev=0.0, FExt=c.freq_ext, ExtEff=c.ext_eff if ext_eff is None else ext_eff),
        FS_GABA: dict(Tau=5.0, Vrev=-70.0, FExt=0.0),
        FS_NMDA: dict(Tau=100.0, TauXT=2.0, Vrev=0.0, FExt=0.0),
    })
    exc = c.excit[c.pre]
    n_e = int(np.count_nonzero(exc))
    pre = np.concatenate([c.pre, c.pre[exc]])
    post = np.concatenate([c.post, c.post[exc]])
    rec = np.concatenate([np.where(exc, FS_AMPA, FS_GABA).astype(np.uint8), np.full(n_e, FS_NMDA, np.uint8)])
    w = c.weight.astype(F32)
    w_gaba = np.where(exc, w, w * F32(gaba_gain)).astype(F32)
    g = np.concatenate([w_gaba, (w[exc] * F32(c.k_nmda)).astype(F32)])
    if with_delays:
        dsteps = np.rint(c.delay_ms.astype(np.float64) / dt).astype(np.uint16)
        delay = np.concatenate([dsteps, dsteps[exc]])
    else:
        delay = np.zeros(pre.size, np.uint16)
    tmd = None
    if tm:
        tmd = dict(enabled=c.excit.astype(np.uint8), U=0.2, tau_rec=200.0, tau_fac=600.0)
    act_ctr = DEFAULT_ACT
    if ltp:
        d32 = F32(dt)
        fields["ltp_dfLP"][:] = np.exp(-d32 / F32(ltp["tLP"]))
        fields["ltp_SpiLPDy"][:] = int(np.floor(F32(ltp["SpiLPDy"]) / d32))
        fields["ltp_PosISI"][:] = F32(ltp["PosISI"])
        fields["ltp_NegISI"][:] = F32(ltp["NegISI"])
        fields["act"] |= ACT["LTP"]
        act_ctr |= ACT["LTP"]
    return desc_from_arrays(n, dt, fields, pre, post, rec, g, delay, tm=tmd, act_ctr=act_ctr)
