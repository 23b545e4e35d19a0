"""Parameter sweeps over independent network instances.

The reference runs a sweep as one process per point, or as `-rp` repeats of
one network (code/main.cpp:251-252); its seizure study scans an inhibitory
gain factor against the drive (experiment/seizure/readme:1-6).  Here every
sweep point is its own connectome-shaped network (size, inhibitory gain,
drive and seed drawn per point) and the whole sweep advances in one
persistent launch of the batched engine (:class:`flysim_b200.Batch`), with
the block plan chosen by its autotuner.  The per-point result is the firing
rate of each of the 58 regions, the network mean rate and a hyperactivity
flag.

    python -m flysim_b200.sweep [--count 256] [--seconds 2] [--looped]

prints one JSON line: sweep points per hour of the batched engine and, with
``--looped``, of the plain engine run once per point on the same points.
"""
from __future__ import annotations

import argparse
import dataclasses
import json
import time
from typing import List, Optional, Sequence

import numpy as np

from . import Batch, Engine, netgen, network

REGIONS = 58
HYPER_HZ = 40.0  # a point is hyperactive when its network mean rate exceeds this


@dataclasses.dataclass
class SweepPoint:
    n: int
    gaba_gain: float
    drive_hz: float
    seed: int


def sweep_points(count: int = 256, seed: int = 1, n_lo: int = 2000, n_hi: int = 20000, g_lo: float = 0.2,
                 g_hi: float = 1.5, f_lo: float = 1000.0, f_hi: float = 5000.0) -> List[SweepPoint]:
    """Points of the batched sweep: neurons ~ U[n_lo, n_hi], inhibitory gain
    ~ U[g_lo, g_hi] (scales every GABA weight), drive ~ U[f_lo, f_hi] Hz on
    every region, seeds seed .. seed+count-1."""
    rng = np.random.default_rng(seed + 7919)
    ns = rng.integers(n_lo, n_hi + 1, count)
    gs = rng.uniform(g_lo, g_hi, count)
    fs = rng.uniform(f_lo, f_hi, count)
    return [SweepPoint(int(ns[i]), float(gs[i]), float(fs[i]), seed + i) for i in range(count)]


def build_instance(pt: SweepPoint, dt: float = 0.1):
    """(connectome, production network arrays) of one point."""
    c = netgen.connectome_fast(n=pt.n, regions=REGIONS, f_lo=pt.drive_hz, f_hi=pt.drive_hz, seed=pt.seed)
    return c, network.connectome_net(c, dt=dt, gaba_gain=pt.gaba_gain)


def region_rates(counts: np.ndarray, region: np.ndarray, seconds: float) -> np.ndarray:
    size = np.bincount(region, minlength=REGIONS).astype(np.float64)
    spk = np.bincount(region, counts.astype(np.float64), REGIONS)
    return spk / np.maximum(size, 1.0) / seconds


def summarise(counts: Sequence[np.ndarray], conns, seconds: float) -> dict:
    rates = np.stack([region_rates(k, c.region, seconds) for k, c in zip(counts, conns)])
    mean = np.array([k.sum() / k.size / seconds for k in counts])
    return dict(region_rates=rates, mean_rate=mean, hyper=mean > HYPER_HZ)


def run_batched(points: Sequence[SweepPoint], seconds: float = 2.0, dt: float = 0.1, tune: bool = True,
                built=None, mode: str = "fp32") -> dict:
    """All points in one batch.  Timing covers upload, tuning, the run and
    the read-back (not the host-side network synthesis)."""
    conns, nets = zip(*(built or [build_instance(p, dt) for p in points]))
    steps = int(round(seconds * 1e3 / dt))
    t0 = time.perf_counter()
    b = Batch([na.desc for na in nets], mode=mode)
    plan = b.tune(100) if tune else None
    b.reset([p.seed for p in points])
    dev_ms = b.run(steps)
    counts = [b.spike_counts(i) for i in range(len(points))]
    wall = time.perf_counter() - t0
    info = b.info()
    b.close()
    out = summarise(counts, conns, seconds)
    out.update(wall_s=wall, device_ms=dev_ms, plan=plan, info=info, counts=counts)
    return out


def run_looped(points: Sequence[SweepPoint], seconds: float = 2.0, dt: float = 0.1, built=None,
               mode: str = "fp32") -> dict:
    """Each point on its own engine, one after the other (the plain simulator
    looped per instance)."""
    conns, nets = zip(*(built or [build_instance(p, dt) for p in points]))
    steps = int(round(seconds * 1e3 / dt))
    counts = []
    t0 = time.perf_counter()
    for p, na in zip(points, nets):
        e = Engine(na.desc, mode, chunk_steps=10000)
        e.reset(p.seed)
        e.run(steps)
        counts.append(e.spike_counts())
        e.close()
    wall = time.perf_counter() - t0
    out = summarise(counts, conns, seconds)
    out.update(wall_s=wall, counts=counts)
    return out


def main(argv: Optional[Sequence[str]] = None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--count", type=int, default=256)
    ap.add_argument("--seconds", type=float, default=2.0)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--looped", action="store_true", help="also time the plain engine looped per point")
    args = ap.parse_args(argv)
    pts = sweep_points(args.count, args.seed)
    t0 = time.perf_counter()
    built = [build_instance(p) for p in pts]
    synth = time.perf_counter() - t0
    bat = run_batched(pts, args.seconds, built=built)
    line = {"metric": "verified sweep points per hour (batched engine)", "count": args.count,
            "seconds_simulated": args.seconds, "neurons_total": int(sum(p.n for p in pts)),
            "batched_points_per_hour": 3600.0 * args.count / bat["wall_s"], "batched_wall_s": bat["wall_s"],
            "batched_device_ms": bat["device_ms"], "plan": bat["plan"], "info": bat["info"],
            "hyperactive": int(bat["hyper"].sum()), "synthesis_s": synth}
    if args.looped:
        loo = run_looped(pts, args.seconds, built=built)
        same = all(np.array_equal(a, b) for a, b in zip(bat["counts"], loo["counts"]))
        line.update(looped_points_per_hour=3600.0 * args.count / loo["wall_s"], looped_wall_s=loo["wall_s"],
                    speedup=loo["wall_s"] / bat["wall_s"], identical_spike_counts=bool(same))
    print(json.dumps(line))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
