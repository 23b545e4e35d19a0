"""flysim_b200 — B200-native per-timestep integration for flysim networks.

Python mirror of the C ABI in include/flysim_b200.h (ctypes; no torch types).
The native library is built in-tree by :mod:`flysim_b200.build`; importing
this package never falls back to Python or CPU code — every call that needs
the engine goes to the CUDA library and fails loudly if it is missing.

Reference interface mirrored: the flysim command line (code/main.cpp) and its
NetSim seam (code/NetSim.h:80-109): load a .conf/.pro pair, run the protocol,
get the .pro's output files; or drive the step engine directly (reset, drive
and injection changes, steps) as NetSimGnl2::Run/DoEvt do.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Dict, Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
LIB_PATH = os.path.join(BUILD, "libflysim_b200.so")

FS_OK, FS_ERR_ARG, FS_ERR_CUDA, FS_ERR_NOMEM, FS_ERR_CAPACITY, FS_ERR_PARSE, FS_ERR_UNSUPPORTED, \
    FS_ERR_TIMEOUT, FS_ERR_IO, FS_ERR_NODEVICE = range(10)
FS_AMPA, FS_GABA, FS_ACH, FS_GCL, FS_NMDA, FS_NREC = 0, 1, 2, 3, 4, 5
FS_MODE_COMPAT, FS_MODE_FP32, FS_MODE_FP64 = 0, 1, 2
FS_RUN_INTERVAL_KERNEL, FS_RUN_TILE_KERNELS = 1, 2
MODES = {"compat": FS_MODE_COMPAT, "fp32": FS_MODE_FP32, "fp64": FS_MODE_FP64}
ACT = dict(AMPA=1, GABA=2, NMDA=4, GAP=8, ACH=32, GCL=64, INJ=128, LIF=256, LTP=8192, STD=16384, STP=32768)
NS_FIRE, NS_SPIKE = 1, 2
DEFAULT_ACT = ACT["AMPA"] | ACT["GABA"] | ACT["NMDA"] | ACT["ACH"] | ACT["GCL"] | ACT["GAP"] | ACT["LIF"]

_f = C.POINTER(C.c_float)
_u32 = C.POINTER(C.c_uint32)
_i32 = C.POINTER(C.c_int32)
_u8 = C.POINTER(C.c_uint8)
_u16 = C.POINTER(C.c_uint16)


class FsError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__("flysim_b200 error %d: %s" % (code, msg))
        self.code = code


class Neurons(C.Structure):
    _fields_ = [("n", C.c_uint32)] + [(k, _f) for k in ("Vth", "El", "gl", "Cm", "Vreset", "df", "ef", "dVmax")] + \
        [("RfPed", _i32), ("SpiDy", _i32), ("Vrev", _f), ("dfst", _f), ("nmda_dfxt", _f), ("nmda_efst", _f),
         ("nmda_as", _f), ("nmda_mg", _f), ("ext_g", _f), ("pb", _f), ("act", _u32), ("inj_mean", _f),
         ("inj_std", _f)] + \
        [(k, _f) for k in ("stp_pv", "stp_dfD", "stp_efD", "stp_aF", "stp_dfF", "stp_efF", "stp_aCap",
                           "stp_dfCap", "stp_aCar", "stp_dfCar", "stp_efCar")] + \
        [("ltp_dfLP", _f), ("ltp_PosISI", _f), ("ltp_NegISI", _f), ("ltp_SpiLPDy", _i32)]


class RecLayout(C.Structure):
    _fields_ = [("n_gates", C.c_uint32), ("gate_pre", _u32), ("gate_post0", _u32), ("gate_g", _f),
                ("gather_rowptr", _u32), ("gather_gate", _u32), ("n_recs", C.c_uint32), ("rec_pre", _u32),
                ("rec_post", _u32), ("rec_g", _f), ("rec_rowptr", _u32), ("rec_src", _u32)]


class CompatLayout(C.Structure):
    _fields_ = [("rec", RecLayout * FS_NREC), ("gap_rowptr", _u32), ("gap_other", _u32), ("gap_g", _f)]


class SynList(C.Structure):
    _fields_ = [("n", C.c_uint64), ("pre", _u32), ("post", _u32), ("rec", _u8), ("g", _f), ("delay", _u16),
                ("ltp", _u8)]


class TmParams(C.Structure):
    _fields_ = [("enabled", _u8), ("U", _f), ("tau_rec", _f), ("tau_fac", _f)]


class NetDesc(C.Structure):
    _fields_ = [("dt", C.c_float), ("act_ctr", C.c_uint32), ("neurons", Neurons),
                ("compat", C.POINTER(CompatLayout)), ("syn", C.POINTER(SynList)), ("tm", C.POINTER(TmParams))]


class RunOpts(C.Structure):
    _fields_ = [("mode", C.c_int), ("device", C.c_int), ("chunk_steps", C.c_uint32), ("philox_key", C.c_uint64),
                ("blocks_per_sm", C.c_uint32), ("flags", C.c_uint32)]


class StepOut(C.Structure):
    _fields_ = [("spike_count", _u32), ("spike_idx", _u32), ("spike_cap", C.c_uint64), ("spike_total", C.c_uint64),
                ("V", _f), ("Irep", _f), ("nstate", _u32), ("gv_sel", _u32), ("gv_n", C.c_uint32),
                ("gv_st", _f), ("gv_xt", _f)]


class ModelOpts(C.Structure):
    _fields_ = [("dt", C.c_float), ("flags", C.c_uint32), ("user_seed_set", C.c_int), ("user_seed", C.c_uint32),
                ("threads", C.c_int), ("repeats", C.c_int), ("out_mem", C.c_char_p), ("out_spike", C.c_char_p),
                ("out_rate", C.c_char_p)]


class BatchPlan(C.Structure):
    _fields_ = [("blocks", C.c_uint32), ("blocks_per_sm", C.c_uint32), ("candidates", C.c_uint32),
                ("tile_posts", C.c_uint32), ("edges_in_flight", C.c_uint32), ("sample_ms", C.c_double)]


class EngineVtbl(C.Structure):
    _fields_ = [("reset", C.c_void_p), ("set_drive", C.c_void_p), ("set_act", C.c_void_p),
                ("set_injection", C.c_void_p), ("step", C.c_void_p), ("error", C.c_void_p)]


_LIB: Optional[C.CDLL] = None
ABI_VERSION = 2  # FS_ABI_VERSION of include/flysim_b200.h the structures above follow


def lib() -> C.CDLL:
    """The native library (built in-tree).  Raises if it was not built."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise FsError(FS_ERR_IO, "native library missing: %s (run flysim_b200.build.build())" % LIB_PATH)
    L = C.CDLL(LIB_PATH)
    vp = C.c_void_p
    sig = {
        "fs_abi_version": (C.c_int, []),
        "fs_last_error": (C.c_char_p, [vp]),
        "fs_device_count": (C.c_int, [C.POINTER(C.c_int)]),
        "fs_create": (C.c_int, [C.POINTER(NetDesc), C.POINTER(RunOpts), C.POINTER(vp)]),
        "fs_destroy": (C.c_int, [vp]),
        "fs_reset": (C.c_int, [vp, C.c_uint32, C.c_uint32]),
        "fs_set_drive": (C.c_int, [vp, C.c_uint32, C.c_uint32, C.c_int, C.c_float]),
        "fs_set_act": (C.c_int, [vp, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32]),
        "fs_set_injection": (C.c_int, [vp, C.c_uint32, C.c_uint32, C.c_float, C.c_float]),
        "fs_step": (C.c_int, [vp, C.c_uint32, C.POINTER(StepOut)]),
        "fs_run": (C.c_int, [vp, C.c_uint32]),
        "fs_sync": (C.c_int, [vp]),
        "fs_run_timed": (C.c_int, [vp, C.c_uint32, C.POINTER(C.c_double)]),
        "fs_stats": (C.c_int, [vp, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
        "fs_kernel_time": (C.c_int, [vp, C.POINTER(C.c_double), C.POINTER(C.c_uint64)]),
        "fs_debug_expf": (C.c_int, [_f, _f, C.c_uint64]),
        "fs_debug_expf_noalloc": (C.c_int, [_f, _f, C.c_uint64]),
        "fs_get_state": (C.c_int, [vp, _f, _i32, _u32]),
        "fs_get_weights": (C.c_int, [vp, _f, C.c_uint64]),
        "fs_debug_barrier_timeout": (C.c_int, [C.c_uint32]),
        "fs_debug_philox": (C.c_int, [_u32, _u32, C.c_uint64, _u32]),
        "fs_engine_layout": (C.c_int, [vp, _u32, _u32, _u32, C.POINTER(C.c_int)]),
        "fs_debug_single_step_plan": (C.c_int, [C.POINTER(NetDesc), C.c_uint32, C.POINTER(C.c_uint64)]),
        "fs_debug_drive": (C.c_int, [vp, C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32,
                                     C.POINTER(C.c_uint8), C.POINTER(C.c_double)]),
        "fs_debug_inject_wait_failure": (C.c_int, [vp]),
        "fs_debug_phase_clock": (C.c_int, [vp, C.c_int]),
        "fs_debug_phase_times": (C.c_int, [vp, C.POINTER(C.c_uint64), C.c_uint32, _u32]),
        "fs_checkpoint_size": (C.c_int, [vp, C.POINTER(C.c_uint64)]),
        "fs_checkpoint_save": (C.c_int, [vp, C.c_void_p, C.c_uint64, C.POINTER(C.c_uint64)]),
        "fs_checkpoint_load": (C.c_int, [vp, C.c_void_p, C.c_uint64]),
        "fs_get_syn_state": (C.c_int, [vp, _f, _f]),
        "fs_model_load": (C.c_int, [C.c_char_p, C.c_char_p, C.POINTER(ModelOpts), C.POINTER(vp)]),
        "fs_model_load_cached": (C.c_int, [C.c_char_p, C.c_char_p, C.POINTER(ModelOpts), C.c_char_p,
                                          C.POINTER(vp), C.POINTER(C.c_int)]),
        "fs_model_confs_info": (C.c_int, [vp, C.c_char_p]),
        "fs_model_network_log": (C.c_int, [vp, C.c_char_p]),
        "fs_model_free": (C.c_int, [vp]),
        "fs_model_error": (C.c_char_p, []),
        "fs_model_desc": (C.c_int, [vp, C.POINTER(C.POINTER(NetDesc))]),
        "fs_model_info": (C.c_int, [vp, _u32, _u32, C.POINTER(C.c_uint64), _u32, _u32]),
        "fs_model_seed": (C.c_int, [vp, C.c_int, _u32]),
        "fs_model_run": (C.c_int, [vp, C.POINTER(RunOpts), C.c_char_p, C.POINTER(C.c_double)]),
        "fs_model_run_with": (C.c_int, [vp, C.POINTER(EngineVtbl), vp, C.c_char_p, C.c_uint32,
                                        C.POINTER(C.c_double)]),
        "fs_device_engine": (C.POINTER(EngineVtbl), []),
        "fs_spike_counts": (C.c_int, [vp, _u32]),
        "fs_batch_create": (C.c_int, [C.c_uint32, C.POINTER(C.POINTER(NetDesc)), C.POINTER(RunOpts), C.POINTER(vp)]),
        "fs_batch_destroy": (C.c_int, [vp]),
        "fs_batch_error": (C.c_char_p, [vp]),
        "fs_batch_reset": (C.c_int, [vp, _u32]),
        "fs_batch_tune": (C.c_int, [vp, C.c_uint32, C.POINTER(BatchPlan)]),
        "fs_batch_run": (C.c_int, [vp, C.c_uint32, C.POINTER(C.c_double)]),
        "fs_batch_info": (C.c_int, [vp, _u32, _u32, _u32, C.POINTER(C.c_int), C.POINTER(C.c_uint64)]),
        "fs_batch_spike_counts": (C.c_int, [vp, C.c_uint32, _u32]),
        "fs_batch_spike_totals": (C.c_int, [vp, C.POINTER(C.c_uint64)]),
        "fs_set_gains": (C.c_int, [vp, _f]),
        "fs_batch_set_gains": (C.c_int, [vp, C.c_uint32, _f]),
        "fs_batch_set_drive": (C.c_int, [vp, C.c_uint32, _f]),
        "fs_mlp_error": (C.c_char_p, []),
        "fs_mlp_create": (C.c_int, [_u32, C.c_uint32, C.c_int, C.c_uint64, C.POINTER(vp)]),
        "fs_mlp_destroy": (C.c_int, [vp]),
        "fs_mlp_param_count": (C.c_uint64, [vp]),
        "fs_mlp_get_params": (C.c_int, [vp, _f]),
        "fs_mlp_set_params": (C.c_int, [vp, _f]),
        "fs_mlp_forward": (C.c_int, [vp, _f, C.c_uint64, _f, C.POINTER(C.c_double)]),
        "fs_mlp_grad": (C.c_int, [vp, _f, _f, C.c_uint32, _f, _f]),
        "fs_mlp_train": (C.c_int, [vp, _f, _f, C.c_uint64, C.c_uint32, C.c_float, C.c_uint64, _f,
                                   C.POINTER(C.c_double)]),
        "fs_mlp_gemm": (C.c_int, [C.POINTER(C.c_uint16), C.POINTER(C.c_uint16), C.c_uint32, C.c_uint32, C.c_uint32,
                                  _f, C.c_int, _f]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    if L.fs_abi_version() != ABI_VERSION:
        raise FsError(FS_ERR_ARG, "native library ABI %d, these bindings need %d (rebuild it)"
                      % (L.fs_abi_version(), ABI_VERSION))
    _LIB = L
    return L


def exported_symbols() -> Sequence[str]:
    return [n for n in ("fs_abi_version", "fs_last_error", "fs_device_count", "fs_create", "fs_destroy",
                        "fs_reset", "fs_set_drive", "fs_set_act", "fs_set_injection", "fs_step", "fs_run",
                        "fs_run_timed",
                        "fs_sync", "fs_stats", "fs_kernel_time", "fs_debug_expf", "fs_debug_expf_noalloc",
                        "fs_get_state", "fs_get_weights", "fs_debug_barrier_timeout", "fs_engine_layout",
                        "fs_debug_single_step_plan", "fs_debug_philox",
                        "fs_debug_drive",
                        "fs_debug_inject_wait_failure", "fs_debug_phase_clock", "fs_debug_phase_times",
                        "fs_checkpoint_size", "fs_checkpoint_save", "fs_checkpoint_load",
                        "fs_get_syn_state", "fs_model_load", "fs_model_load_cached", "fs_model_confs_info", "fs_model_network_log",
                        "fs_model_free", "fs_model_error",
                        "fs_model_desc", "fs_model_info", "fs_model_seed", "fs_model_run",
                        "fs_model_run_with", "fs_device_engine", "fs_spike_counts", "fs_batch_create",
                        "fs_batch_destroy", "fs_batch_error", "fs_batch_reset", "fs_batch_tune", "fs_batch_run",
                        "fs_batch_info", "fs_batch_spike_counts", "fs_batch_spike_totals", "fs_set_gains",
                        "fs_batch_set_gains", "fs_batch_set_drive", "fs_mlp_error",
                        "fs_mlp_create", "fs_mlp_destroy", "fs_mlp_param_count", "fs_mlp_get_params",
                        "fs_mlp_set_params", "fs_mlp_forward", "fs_mlp_grad", "fs_mlp_train", "fs_mlp_gemm")]


def _check(rc: int, h=None):
    if rc != FS_OK:
        L = lib()
        msg = L.fs_last_error(h) if h is not None else L.fs_last_error(None)
        raise FsError(rc, (msg or b"").decode(errors="replace"))


def device_count() -> int:
    c = C.c_int(0)
    lib().fs_device_count(C.byref(c))
    return c.value


# ---------------------------------------------------------------------------
class Model:
    """A parsed and built network (Parser + SetPp of the reference).

    cache: path of a binary network cache; the model is read from it when it
    was written for the same .conf/.pro bytes and options, else parsed, built
    and stored there.  cache_status is then "hit", "stored", "unwritable" or
    "unseeded" (a network without a fixed seed draws a new one on every load,
    as the reference does, and is never cached); "off" without a cache."""

    CACHE_STATUS = {0: "off", 1: "hit", 2: "stored", 3: "unwritable", 4: "unseeded"}

    def __init__(self, conf: str, pro: str, dt: float = 0.1, stp: bool = False, std: bool = False,
                 ltp: bool = False, repeats: int = 1, threads: int = 1, user_seed: Optional[int] = None,
                 out_mem: Optional[str] = None, out_spike: Optional[str] = None, out_rate: Optional[str] = None,
                 cache: Optional[str] = None):
        L = lib()
        o = ModelOpts()
        o.dt = dt
        o.flags = (ACT["STP"] if stp else 0) | (ACT["STD"] if std else 0) | (ACT["LTP"] if ltp else 0)
        o.user_seed_set = 1 if user_seed is not None else 0
        o.user_seed = int(user_seed or 0)
        o.threads = threads
        o.repeats = repeats
        o.out_mem = out_mem.encode() if out_mem else None
        o.out_spike = out_spike.encode() if out_spike else None
        o.out_rate = out_rate.encode() if out_rate else None
        h = C.c_void_p()
        st = C.c_int(0)
        rc = L.fs_model_load_cached(conf.encode(), pro.encode(), C.byref(o), cache.encode() if cache else None,
                                    C.byref(h), C.byref(st))
        if rc != FS_OK:
            raise FsError(rc, L.fs_model_error().decode(errors="replace"))
        self._h = h
        self.dt = dt
        self.cache_status = self.CACHE_STATUS.get(st.value, str(st.value))

    def close(self):
        if getattr(self, "_h", None):
            lib().fs_model_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def desc(self) -> "C.POINTER(NetDesc)":
        p = C.POINTER(NetDesc)()
        _check(lib().fs_model_desc(self._h, C.byref(p)))
        return p

    def info(self) -> Dict[str, int]:
        a, b, d, e = C.c_uint32(), C.c_uint32(), C.c_uint32(), C.c_uint32()
        s = C.c_uint64()
        _check(lib().fs_model_info(self._h, C.byref(a), C.byref(b), C.byref(s), C.byref(d), C.byref(e)))
        return dict(neurons=a.value, populations=b.value, synapses=s.value, events=d.value, outputs=e.value)

    def confs_info(self, path: str) -> None:
        """Writes ConfsInfo.log (Parser::ConfsInfo, code/parser.cpp:1488-1631)."""
        rc = lib().fs_model_confs_info(self._h, path.encode())
        if rc != FS_OK:
            raise FsError(rc, lib().fs_model_error().decode(errors="replace"))

    def network_log(self, path: str) -> None:
        """Writes network.log (NetSimGnl2::logDataWrite, code/NetSimGnl2_info.cpp:93-546)."""
        rc = lib().fs_model_network_log(self._h, path.encode())
        if rc != FS_OK:
            raise FsError(rc, lib().fs_model_error().decode(errors="replace"))

    def seed(self, repeat: int = 1) -> int:
        v = C.c_uint32()
        _check(lib().fs_model_seed(self._h, repeat, C.byref(v)))
        return v.value

    def run(self, out_dir: str, mode: str = "compat", device: int = 0, chunk_steps: int = 0) -> float:
        """Runs the whole protocol on the GPU and writes the .pro's output files."""
        o = RunOpts(MODES[mode], device, chunk_steps, 0, 0)
        secs = C.c_double()
        rc = lib().fs_model_run(self._h, C.byref(o), out_dir.encode(), C.byref(secs))
        if rc != FS_OK:
            raise FsError(rc, lib().fs_model_error().decode(errors="replace"))
        return secs.value

    def run_with(self, vtbl, ctx, out_dir: str, chunk_steps: int = 1000) -> float:
        secs = C.c_double()
        rc = lib().fs_model_run_with(self._h, vtbl, ctx, out_dir.encode(), chunk_steps, C.byref(secs))
        if rc != FS_OK:
            raise FsError(rc, lib().fs_model_error().decode(errors="replace"))
        return secs.value


# ---------------------------------------------------------------------------
class Engine:
    """One network instance on one GPU (fs_create ... fs_destroy)."""

    def __init__(self, desc, mode: str = "compat", device: int = 0, chunk_steps: int = 0, philox_key: int = 0,
                 blocks_per_sm: int = 0, interval_kernel: bool = False, tile_kernels: bool = False):
        L = lib()
        self._keep = getattr(desc, "_keep", None)
        o = RunOpts(MODES[mode], device, chunk_steps, philox_key, blocks_per_sm,
                    (FS_RUN_INTERVAL_KERNEL if interval_kernel else 0) | (FS_RUN_TILE_KERNELS if tile_kernels else 0))
        h = C.c_void_p()
        dp = desc if isinstance(desc, C._Pointer) else C.pointer(desc)
        rc = L.fs_create(dp, C.byref(o), C.byref(h))
        if rc != FS_OK:
            raise FsError(rc, L.fs_last_error(None).decode(errors="replace"))
        self._h = h
        self.n = dp.contents.neurons.n
        self.mode = mode

    def close(self):
        if getattr(self, "_h", None):
            lib().fs_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def reset(self, seed: int, jcong_seed: Optional[int] = None):
        _check(lib().fs_reset(self._h, seed, seed if jcong_seed is None else jcong_seed), self._h)

    def set_drive(self, first: int, count: int, rec: int, pb: float):
        _check(lib().fs_set_drive(self._h, first, count, rec, pb), self._h)

    def set_act(self, first: int, count: int, clear_mask: int, set_mask: int):
        _check(lib().fs_set_act(self._h, first, count, clear_mask, set_mask), self._h)

    def set_injection(self, first: int, count: int, mean: float, std: float):
        _check(lib().fs_set_injection(self._h, first, count, mean, std), self._h)

    def step(self, nsteps: int, want_V: bool = False, spike_cap: Optional[int] = None, want_Irep: bool = False,
             want_nstate: bool = False):
        """Runs nsteps; returns (list of per-step spike index arrays, V or
        None), or with want_Irep / want_nstate (spikes, V, Irep [steps, 5, n]
        or None, LIF state words [steps, n] or None)."""
        counts = np.zeros(nsteps, np.uint32)
        cap = spike_cap if spike_cap is not None else max(1024, nsteps * self.n)
        idx = np.zeros(cap, np.uint32)
        V = np.zeros((nsteps, self.n), np.float32) if want_V else None
        I = np.zeros((nsteps, FS_NREC, self.n), np.float32) if want_Irep else None
        NS = np.zeros((nsteps, self.n), np.uint32) if want_nstate else None
        so = StepOut()
        so.spike_count = counts.ctypes.data_as(_u32)
        so.spike_idx = idx.ctypes.data_as(_u32)
        so.spike_cap = cap
        if V is not None:
            so.V = V.ctypes.data_as(_f)
        if I is not None:
            so.Irep = I.ctypes.data_as(_f)
        if NS is not None:
            so.nstate = NS.ctypes.data_as(_u32)
        _check(lib().fs_step(self._h, nsteps, C.byref(so)), self._h)
        offs = np.concatenate([[0], np.cumsum(counts.astype(np.int64))])
        spikes = [idx[offs[i]:offs[i + 1]].copy() for i in range(nsteps)]
        if want_Irep or want_nstate:
            return spikes, V, I, NS
        return spikes, V

    def step_gv(self, nsteps: int, gv_sel):
        """Runs nsteps with GatingVariable outputs for the selected
        single-target records (receptor << 28 | record index); returns
        (spikes per step, st [nsteps, k], xt [nsteps, k])."""
        sel = np.ascontiguousarray(gv_sel, np.uint32)
        k = sel.size
        counts = np.zeros(nsteps, np.uint32)
        cap = max(1024, nsteps * self.n)
        idx = np.zeros(cap, np.uint32)
        gst = np.zeros((nsteps, k), np.float32)
        gxt = np.zeros((nsteps, k), np.float32)
        so = StepOut()
        so.spike_count = counts.ctypes.data_as(_u32)
        so.spike_idx = idx.ctypes.data_as(_u32)
        so.spike_cap = cap
        so.gv_sel = sel.ctypes.data_as(_u32)
        so.gv_n = k
        so.gv_st = gst.ctypes.data_as(_f)
        so.gv_xt = gxt.ctypes.data_as(_f)
        _check(lib().fs_step(self._h, nsteps, C.byref(so)), self._h)
        offs = np.concatenate([[0], np.cumsum(counts.astype(np.int64))])
        return [idx[offs[i]:offs[i + 1]].copy() for i in range(nsteps)], gst, gxt

    def step_csr(self, nsteps: int, spike_cap: Optional[int] = None):
        """Runs nsteps; returns the spikes as the C ABI gives them: per-step
        counts (uint32 [nsteps]) and the neuron indices of all steps in step
        order (uint32 [sum(counts)]), with no per-step Python objects."""
        counts = np.zeros(nsteps, np.uint32)
        cap = spike_cap if spike_cap is not None else max(1024, nsteps * self.n)
        idx = np.empty(cap, np.uint32)
        so = StepOut()
        so.spike_count = counts.ctypes.data_as(_u32)
        so.spike_idx = idx.ctypes.data_as(_u32)
        so.spike_cap = cap
        _check(lib().fs_step(self._h, nsteps, C.byref(so)), self._h)
        return counts, idx[:int(counts.sum(dtype=np.int64))]

    def run(self, nsteps: int):
        _check(lib().fs_run(self._h, nsteps), self._h)

    def run_timed(self, nsteps: int) -> float:
        """Runs nsteps on the device; returns the device time in ms (CUDA events)."""
        ms = C.c_double()
        _check(lib().fs_run_timed(self._h, nsteps, C.byref(ms)), self._h)
        return ms.value

    def sync(self):
        _check(lib().fs_sync(self._h), self._h)

    def stats(self):
        a, b, c = C.c_uint64(), C.c_uint64(), C.c_uint64()
        _check(lib().fs_stats(self._h, C.byref(a), C.byref(b), C.byref(c)), self._h)
        return dict(steps=a.value, spikes=b.value, launches=c.value)

    def layout(self):
        """Launch layout (production modes): blocks, threads, interval and
        the kernels that run the network ("interval", "single_step",
        "tiles" or "ltp")."""
        b, t, i, k = C.c_uint32(), C.c_uint32(), C.c_uint32(), C.c_int()
        _check(lib().fs_engine_layout(self._h, C.byref(b), C.byref(t), C.byref(i), C.byref(k)), self._h)
        kind = {0: "interval", 1: "single_step", 2: "tiles", 3: "ltp"}[k.value]
        return dict(blocks=b.value, threads=t.value, interval=i.value, kernel=kind,
                    single_step=kind == "single_step")

    def kernel_time(self):
        ms, n = C.c_double(), C.c_uint64()
        _check(lib().fs_kernel_time(self._h, C.byref(ms), C.byref(n)), self._h)
        return ms.value, n.value

    def set_gains(self, gains):
        """Synaptic gain per receptor (production modes)."""
        g = np.ascontiguousarray(gains, np.float32)
        assert g.size == FS_NREC
        _check(lib().fs_set_gains(self._h, g.ctypes.data_as(_f)), self._h)

    def spike_counts(self) -> np.ndarray:
        """Per-neuron spike counts since the last reset (production modes)."""
        c = np.zeros(self.n, np.uint32)
        _check(lib().fs_spike_counts(self._h, c.ctypes.data_as(_u32)), self._h)
        return c

    def state(self):
        V = np.zeros(self.n, np.float32)
        cnt = np.zeros(self.n, np.int32)
        ns = np.zeros(self.n, np.uint32)
        _check(lib().fs_get_state(self._h, V.ctypes.data_as(_f), cnt.ctypes.data_as(_i32),
                                  ns.ctypes.data_as(_u32)), self._h)
        return V, cnt, ns

    def weights(self, n_syn: int) -> np.ndarray:
        """Synaptic weights in synapse-list order as long-term plasticity has
        made them (production modes, networks with LTP)."""
        g = np.zeros(n_syn, np.float32)
        _check(lib().fs_get_weights(self._h, g.ctypes.data_as(_f), C.c_uint64(n_syn)), self._h)
        return g

    def checkpoint(self) -> bytes:
        """The handle's state after its last step (production modes), for
        restore() on a handle of the same network and mode."""
        nb = C.c_uint64()
        _check(lib().fs_checkpoint_size(self._h, C.byref(nb)), self._h)
        buf = C.create_string_buffer(nb.value)
        _check(lib().fs_checkpoint_save(self._h, buf, nb.value, C.byref(nb)), self._h)
        return buf.raw[:nb.value]

    def restore(self, data: bytes):
        _check(lib().fs_checkpoint_load(self._h, data, len(data)), self._h)

    def drive_draws(self, t0: int, nsteps: int, first: int = 0, count: Optional[int] = None):
        """The production drive draws of steps [t0, t0 + nsteps) for neurons
        [first, first + count): (hits uint8 [nsteps, count], bit r = receptor
        r hit; injection current float64 [nsteps, count], 0 where off)."""
        count = self.n - first if count is None else count
        hits = np.zeros((nsteps, count), np.uint8)
        gauss = np.zeros((nsteps, count), np.float64)
        _check(lib().fs_debug_drive(self._h, t0, nsteps, first, count, hits.ctypes.data_as(C.POINTER(C.c_uint8)),
                                    gauss.ctypes.data_as(C.POINTER(C.c_double))), self._h)
        return hits, gauss

    def phase_clock(self, enable: bool = True):
        """Switches the persistent kernels' per-block phase clock on (zeroed)
        or off."""
        _check(lib().fs_debug_phase_clock(self._h, 1 if enable else 0), self._h)

    def phase_times(self) -> np.ndarray:
        """SM cycles per block and phase since the clock was switched on,
        [blocks, 16]."""
        nb = C.c_uint32()
        _check(lib().fs_debug_phase_times(self._h, None, 0, C.byref(nb)), self._h)
        out = np.zeros(nb.value * 16, np.uint64)
        _check(lib().fs_debug_phase_times(self._h, out.ctypes.data_as(C.POINTER(C.c_uint64)), out.size,
                                          C.byref(nb)), self._h)
        return out.reshape(nb.value, 16)

    def inject_wait_failure(self):
        """Sets the device error word as a bounded wait that gave up would."""
        _check(lib().fs_debug_inject_wait_failure(self._h), self._h)

    def syn_state(self):
        g = np.zeros(FS_NREC * self.n, np.float32)
        isyn = np.zeros(self.n, np.float32)
        _check(lib().fs_get_syn_state(self._h, g.ctypes.data_as(_f), isyn.ctypes.data_as(_f)), self._h)
        return g.reshape(FS_NREC, self.n), isyn


def device_engine_vtbl():
    return lib().fs_device_engine()


def single_step_plan(desc, sm_count: int = 148) -> dict:
    """Host-only check of the single-step kernel's plan for a network."""
    st = (C.c_uint64 * 8)()
    dp = desc if isinstance(desc, C._Pointer) else C.pointer(desc)
    _check(lib().fs_debug_single_step_plan(dp, sm_count, st))
    keys = ("qualifies", "blocks", "max_posts", "max_tracked", "max_edges", "smem", "lin_entries", "nmda_edges")
    return dict(zip(keys, [int(x) for x in st]))


def debug_philox(ctr: np.ndarray, key: np.ndarray) -> np.ndarray:
    """The device Philox-4x32-10 on counters ctr [k, 4] and keys key [k, 2]."""
    ctr = np.ascontiguousarray(ctr, np.uint32).reshape(-1, 4)
    key = np.ascontiguousarray(key, np.uint32).reshape(-1, 2)
    assert ctr.shape[0] == key.shape[0]
    out = np.zeros_like(ctr)
    _check(lib().fs_debug_philox(ctr.ctypes.data_as(_u32), key.ctypes.data_as(_u32), ctr.shape[0],
                                 out.ctypes.data_as(_u32)))
    return out


def debug_expf(x: np.ndarray) -> np.ndarray:
    x = np.ascontiguousarray(x, np.float32)
    y = np.zeros_like(x)
    _check(lib().fs_debug_expf(x.ctypes.data_as(_f), y.ctypes.data_as(_f), x.size))
    return y


class Batch:
    """Independent production networks advanced by one persistent launch
    (fs_batch_*): the generalisation of the reference's -rp repeat loop to
    instances of different size, parameters and seed."""

    def __init__(self, descs, mode: str = "fp32", device: int = 0, chunk_steps: int = 0, philox_key: int = 0,
                 blocks_per_sm: int = 0):
        L = lib()
        self._keep = [getattr(d, "_keep", None) for d in descs]
        self._descs = [d if isinstance(d, C._Pointer) else C.pointer(d) for d in descs]
        arr = (C.POINTER(NetDesc) * len(descs))(*self._descs)
        o = RunOpts(MODES[mode], device, chunk_steps, philox_key, blocks_per_sm)
        h = C.c_void_p()
        rc = L.fs_batch_create(len(descs), arr, C.byref(o), C.byref(h))
        if rc != FS_OK:
            raise FsError(rc, (L.fs_batch_error(None) or b"").decode(errors="replace"))
        self._h = h
        self.count = len(descs)
        self.n = [int(d.contents.neurons.n) for d in self._descs]

    def _ok(self, rc):
        if rc != FS_OK:
            raise FsError(rc, (lib().fs_batch_error(self._h) or b"").decode(errors="replace"))

    def reset(self, seeds=None):
        if seeds is None:
            self._ok(lib().fs_batch_reset(self._h, None))
        else:
            s = np.ascontiguousarray(seeds, np.uint32)
            assert s.size == self.count
            self._ok(lib().fs_batch_reset(self._h, s.ctypes.data_as(_u32)))

    def tune(self, sample_steps: int = 200) -> dict:
        p = BatchPlan()
        self._ok(lib().fs_batch_tune(self._h, sample_steps, C.byref(p)))
        return dict(blocks=p.blocks, blocks_per_sm=p.blocks_per_sm, candidates=p.candidates,
                    tile_posts=p.tile_posts, edges_in_flight=p.edges_in_flight, sample_ms=p.sample_ms)

    def run(self, nsteps: int) -> float:
        ms = C.c_double()
        self._ok(lib().fs_batch_run(self._h, nsteps, C.byref(ms)))
        return ms.value

    def info(self) -> dict:
        a, b, c, g, l_ = C.c_uint32(), C.c_uint32(), C.c_uint32(), C.c_int(), C.c_uint64()
        self._ok(lib().fs_batch_info(self._h, C.byref(a), C.byref(b), C.byref(c), C.byref(g), C.byref(l_)))
        return dict(count=a.value, blocks=b.value, blocks_per_sm=c.value, graph=bool(g.value), launches=l_.value)

    def spike_counts(self, i: int) -> np.ndarray:
        c = np.zeros(self.n[i], np.uint32)
        self._ok(lib().fs_batch_spike_counts(self._h, i, c.ctypes.data_as(_u32)))
        return c

    def set_gains(self, i: int, gains):
        g = np.ascontiguousarray(gains, np.float32)
        assert g.size == FS_NREC
        self._ok(lib().fs_batch_set_gains(self._h, i, g.ctypes.data_as(_f)))

    def set_drive(self, i: int, pb: np.ndarray):
        """Drive probabilities of instance i, pb[FS_NREC * n] (receptor-major)."""
        p = np.ascontiguousarray(pb, np.float32)
        assert p.size == FS_NREC * self.n[i]
        self._ok(lib().fs_batch_set_drive(self._h, i, p.ctypes.data_as(_f)))

    def spike_totals(self) -> np.ndarray:
        t = np.zeros(self.count, np.uint64)
        self._ok(lib().fs_batch_spike_totals(self._h, t.ctypes.data_as(C.POINTER(C.c_uint64))))
        return t

    def close(self):
        if getattr(self, "_h", None):
            lib().fs_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _mlp_ok(rc):
    if rc != FS_OK:
        raise FsError(rc, (lib().fs_mlp_error() or b"").decode(errors="replace"))


class Mlp:
    """The surrogate MLP (fs_mlp_*): BF16 tensor-core training and inference."""

    def __init__(self, dims, device: int = 0, seed: int = 1):
        d = np.ascontiguousarray(dims, np.uint32)
        h = C.c_void_p()
        _mlp_ok(lib().fs_mlp_create(d.ctypes.data_as(_u32), d.size, device, seed, C.byref(h)))
        self._h = h
        self.dims = [int(x) for x in dims]

    def param_count(self) -> int:
        return int(lib().fs_mlp_param_count(self._h))

    def get_params(self) -> np.ndarray:
        p = np.zeros(self.param_count(), np.float32)
        _mlp_ok(lib().fs_mlp_get_params(self._h, p.ctypes.data_as(_f)))
        return p

    def set_params(self, p: np.ndarray):
        p = np.ascontiguousarray(p, np.float32)
        assert p.size == self.param_count()
        _mlp_ok(lib().fs_mlp_set_params(self._h, p.ctypes.data_as(_f)))

    def forward(self, x: np.ndarray, with_time: bool = False):
        x = np.ascontiguousarray(x, np.float32)
        rows = x.shape[0]
        y = np.zeros((rows, self.dims[-1]), np.float32)
        ms = C.c_double()
        _mlp_ok(lib().fs_mlp_forward(self._h, x.ctypes.data_as(_f), rows, y.ctypes.data_as(_f), C.byref(ms)))
        return (y, ms.value) if with_time else y

    def grad(self, x: np.ndarray, t: np.ndarray):
        x = np.ascontiguousarray(x, np.float32)
        t = np.ascontiguousarray(t, np.float32)
        g = np.zeros(self.param_count(), np.float32)
        loss = C.c_float()
        _mlp_ok(lib().fs_mlp_grad(self._h, x.ctypes.data_as(_f), t.ctypes.data_as(_f), x.shape[0],
                                  g.ctypes.data_as(_f), C.byref(loss)))
        return g, loss.value

    def train(self, x: np.ndarray, t: np.ndarray, epochs: int, lr: float = 1e-3, seed: int = 1):
        x = np.ascontiguousarray(x, np.float32)
        t = np.ascontiguousarray(t, np.float32)
        losses = np.zeros(epochs, np.float32)
        ms = C.c_double()
        _mlp_ok(lib().fs_mlp_train(self._h, x.ctypes.data_as(_f), t.ctypes.data_as(_f), x.shape[0], epochs, lr,
                                   seed, losses.ctypes.data_as(_f), C.byref(ms)))
        return losses, ms.value

    def close(self):
        if getattr(self, "_h", None):
            lib().fs_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def mlp_gemm(a_bf16: np.ndarray, b_bf16: np.ndarray, bias=None, relu: bool = False) -> np.ndarray:
    """fs_mlp_gemm: c = a . b^T on the tensor cores (a, b as uint16 BF16 bits)."""
    a = np.ascontiguousarray(a_bf16, np.uint16)
    b = np.ascontiguousarray(b_bf16, np.uint16)
    m, k = a.shape
    n = b.shape[0]
    c = np.zeros((m, n), np.float32)
    bp = None if bias is None else np.ascontiguousarray(bias, np.float32)
    _mlp_ok(lib().fs_mlp_gemm(a.ctypes.data_as(C.POINTER(C.c_uint16)), b.ctypes.data_as(C.POINTER(C.c_uint16)),
                              m, n, k, None if bp is None else bp.ctypes.data_as(_f), int(relu),
                              c.ctypes.data_as(_f)))
    return c


NOALLOC_MAX_K = 262144  # FS_NOALLOC_MAX_K


def debug_expf_noalloc(x: np.ndarray) -> np.ndarray:
    """fs_debug_expf_noalloc: the device expf without per-call device
    allocation (at most NOALLOC_MAX_K values per call)."""
    x = np.ascontiguousarray(x, np.float32)
    y = np.zeros_like(x)
    _check(lib().fs_debug_expf_noalloc(x.ctypes.data_as(_f), y.ctypes.data_as(_f), x.size))
    return y


from .network import desc_from_arrays, NetArrays  # noqa: E402  (array-built networks)
