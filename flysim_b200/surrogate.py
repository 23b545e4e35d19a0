"""Learned mean-field surrogate for parameter sweeps.

The reference explores parameter space by simulating every point (its
seizure study scans an inhibitory efficacy factor against the drive,
experiment/seizure/readme:1-6).  Here a small MLP, trained on the GPU with
the library's own tensor-core kernels (:class:`flysim_b200.Mlp`) on rates
that the batched engine simulated, predicts the outcome of a point; it
screens a large grid, and the simulator verifies the surrogate's top
candidates and a random audit set, which measures the surrogate's error.

Parameterisation (32 inputs): the drive of 30 region groups (regions 2g and
2g+1 for g < 28; regions 56 and 57 alone), uniform in [1, 5] kHz on AMPA;
the excitatory gain in [0.5, 1.5] (scales every AMPA and NMDA weight) and
the inhibitory gain in [0.2, 1.5] (scales every GABA weight).  Inputs are
scaled to [-1, 1].  Outputs (59): log(1 + rate) of each of the 58 regions
and a hyperactivity logit (network mean rate above 40 Hz).

Surrogate rate error of a point: sum_r |pred_r - sim_r| / sum_r sim_r over
the 58 region rates (a rate-weighted relative L1 error).

    python -m flysim_b200.surrogate [--neurons 5000] [--train 20000] ...

prints one JSON line with the errors, the verified hit rate and the sweep
throughput against the plain engine looped per point.
"""
from __future__ import annotations

import argparse
import json
import time
from typing import Optional, Sequence

import numpy as np

from . import FS_AMPA, FS_GABA, FS_NMDA, FS_NREC, Batch, Engine, Mlp, netgen, network

REGIONS = 58
GROUPS = 30
N_IN = GROUPS + 2
N_OUT = REGIONS + 1
DRIVE_HZ = (1000.0, 5000.0)
E_GAIN = (0.5, 1.5)
I_GAIN = (0.2, 1.5)
HYPER_HZ = 40.0
DIMS = (N_IN, 256, 256, 256, N_OUT)


def region_group() -> np.ndarray:
    """Drive group of each region."""
    r = np.arange(REGIONS)
    return np.where(r < 56, r // 2, 28 + (r - 56))


def sample_params(count: int, rng: np.random.Generator) -> np.ndarray:
    """Raw parameters [count x 32]: 30 group drives (Hz), E gain, I gain."""
    p = np.empty((count, N_IN))
    p[:, :GROUPS] = rng.uniform(*DRIVE_HZ, (count, GROUPS))
    p[:, GROUPS] = rng.uniform(*E_GAIN, count)
    p[:, GROUPS + 1] = rng.uniform(*I_GAIN, count)
    return p


def encode(p: np.ndarray) -> np.ndarray:
    lo = np.array([DRIVE_HZ[0]] * GROUPS + [E_GAIN[0], I_GAIN[0]])
    hi = np.array([DRIVE_HZ[1]] * GROUPS + [E_GAIN[1], I_GAIN[1]])
    return (2.0 * (p - lo) / (hi - lo) - 1.0).astype(np.float32)


def targets(rates: np.ndarray) -> np.ndarray:
    hyper = (rates.mean(1) > HYPER_HZ).astype(np.float32)
    return np.concatenate([np.log1p(rates), hyper[:, None]], 1).astype(np.float32)


def decode_rates(y: np.ndarray) -> np.ndarray:
    return np.expm1(np.maximum(y[:, :REGIONS], 0.0))


def rate_error(pred: np.ndarray, sim: np.ndarray) -> np.ndarray:
    """Rate-weighted relative L1 error per point."""
    return np.abs(pred - sim).sum(1) / np.maximum(sim.sum(1), 1e-9)


class Simulator:
    """One connectome-shaped network, simulated for many parameter points at
    once: a batch of `batch` instances of it whose drive and gains are set
    per point before every run."""

    def __init__(self, neurons: int = 5000, seed: int = 1, batch: int = 256, seconds: float = 1.0,
                 dt: float = 0.1, tune: bool = True):
        self.c = netgen.connectome_fast(n=neurons, regions=REGIONS, f_lo=3000.0, f_hi=3000.0, seed=seed)
        self.na = network.connectome_net(self.c, dt=dt)
        self.n = neurons
        self.dt = dt
        self.seconds = seconds
        self.steps = int(round(seconds * 1e3 / dt))
        self.batch = batch
        self.group_of_neuron = region_group()[self.c.region]
        self.pb0 = np.asarray(self.na.fields["pb"], np.float32).reshape(FS_NREC, neurons).copy()
        self.b = Batch([self.na.desc] * batch)
        self.plan = self.b.tune(100) if tune else None
        self.device_ms = 0.0
        self.points = 0

    def _set(self, i: int, p: np.ndarray):
        pb = self.pb0.copy()
        pb[FS_AMPA] = (p[:GROUPS][self.group_of_neuron] * self.dt * 1e-3).astype(np.float32)
        self.b.set_drive(i, pb.ravel())
        g = np.ones(FS_NREC, np.float32)
        g[FS_AMPA] = g[FS_NMDA] = p[GROUPS]
        g[FS_GABA] = p[GROUPS + 1]
        self.b.set_gains(i, g)

    def rates(self, params: np.ndarray, seed0: int = 1) -> np.ndarray:
        """Per-region rates (Hz) of every parameter point [count x 58]."""
        out = np.zeros((len(params), REGIONS))
        for s in range(0, len(params), self.batch):
            chunk = params[s:s + self.batch]
            for i in range(self.batch):
                self._set(i, chunk[min(i, len(chunk) - 1)])
            self.b.reset(np.arange(seed0 + s, seed0 + s + self.batch, dtype=np.uint32))
            self.device_ms += self.b.run(self.steps)
            for i in range(len(chunk)):
                k = self.b.spike_counts(i)
                out[s + i] = np.bincount(self.c.region, k.astype(np.float64), REGIONS) / \
                    np.bincount(self.c.region, minlength=REGIONS) / self.seconds
            self.points += len(chunk)
        return out

    def single_rates(self, p: np.ndarray, seed: int) -> tuple:
        """The same point on the plain engine (one network, fs_create ... fs_destroy):
        returns (region rates, wall seconds)."""
        t0 = time.perf_counter()
        e = Engine(self.na.desc, "fp32", chunk_steps=10000)
        pb = self.pb0.copy()
        pb[FS_AMPA] = (p[:GROUPS][self.group_of_neuron] * self.dt * 1e-3).astype(np.float32)
        # set the drive region by region, as a plain-engine user does
        for g in range(GROUPS):
            for r in np.flatnonzero(region_group() == g):
                idx = np.flatnonzero(self.c.region == r)
                e.set_drive(int(idx[0]), int(idx.size), FS_AMPA, float(pb[FS_AMPA][idx[0]]))
        gains = np.ones(FS_NREC, np.float32)
        gains[FS_AMPA] = gains[FS_NMDA] = p[GROUPS]
        gains[FS_GABA] = p[GROUPS + 1]
        e.set_gains(gains)
        e.reset(seed)
        e.run(self.steps)
        k = e.spike_counts()
        e.close()
        wall = time.perf_counter() - t0
        rates = np.bincount(self.c.region, k.astype(np.float64), REGIONS) / \
            np.bincount(self.c.region, minlength=REGIONS) / self.seconds
        return rates, wall

    def close(self):
        self.b.close()


def linear_baseline(x: np.ndarray, t: np.ndarray):
    """The method without the learned network: least squares from the
    inputs to the same targets (a linear response around the sampled
    region)."""
    A = np.concatenate([x, np.ones((len(x), 1), np.float32)], 1).astype(np.float64)
    coef, *_ = np.linalg.lstsq(A, t.astype(np.float64), rcond=None)
    return lambda z: np.concatenate([z, np.ones((len(z), 1), np.float32)], 1) @ coef


def fit(net: Mlp, x: np.ndarray, y: np.ndarray, rates: np.ndarray, epochs: int, seed: int = 1,
        epochs_per_round: int = 10, lr: float = 2e-3, patience: int = 6):
    """Adam on 90 % of the points: the learning rate is held at `lr` for the
    first third of the epochs (the loss sits on a plateau near the
    population-average response until the network separates the
    hyperactive regime), then annealed on a cosine.  After every round of
    `epochs_per_round` epochs the rate error on the held-out 10 % is
    measured and the best parameters are kept; once the learning rate has
    fallen below a quarter of `lr`, training stops after `patience` rounds
    without improvement (stopping earlier, while the rate is still high,
    ends before the anneal that gives most of the accuracy).  Returns
    (losses, device ms, best validation error)."""
    n = len(x)
    perm = np.random.default_rng(seed + 17).permutation(n)
    nv = max(1, n // 10)
    vi, ti = perm[:nv], perm[nv:]
    rounds = max(1, epochs // epochs_per_round)
    hold = rounds // 3
    best, best_p, stall = np.inf, None, 0
    losses, ms_total = [], 0.0
    for k in range(rounds):
        f = 1.0 if k < hold else 0.5 * (1.0 + np.cos(np.pi * (k - hold) / max(1, rounds - hold)))
        ls, ms = net.train(x[ti], y[ti], epochs=epochs_per_round, lr=float(lr * max(f, 0.01)), seed=seed + k)
        losses += list(ls)
        ms_total += ms
        err = float(rate_error(decode_rates(net.forward(x[vi])), rates[vi]).mean())
        if err < best:
            best, best_p, stall = err, net.get_params(), 0
        elif k >= hold and f < 0.25:
            stall += 1
            if stall >= patience:
                break
    net.set_params(best_p)
    return np.array(losses), ms_total, best


def run(neurons: int = 5000, seconds: float = 1.0, n_train: int = 20000, epochs: int = 600, grid: int = 1_000_000,
        top_frac: float = 0.01, audit: int = 1000, seed: int = 1, looped_sample: int = 8,
        log=None) -> dict:
    rng = np.random.default_rng(seed)
    T0 = time.perf_counter()
    sim = Simulator(neurons=neurons, seed=seed, seconds=seconds)
    t_setup = time.perf_counter() - T0
    # training data from the batched simulator
    t0 = time.perf_counter()
    p_train = sample_params(n_train, rng)
    r_train = sim.rates(p_train, seed0=1)
    t_data = time.perf_counter() - t0
    x_train, y_train = encode(p_train), targets(r_train)
    # train on the tensor cores
    t0 = time.perf_counter()
    net = Mlp(list(DIMS), seed=seed)
    losses, train_ms, val_err = fit(net, x_train, y_train, r_train, epochs, seed)
    t_train = time.perf_counter() - t0
    lin = linear_baseline(x_train, y_train)
    # screen the grid
    t0 = time.perf_counter()
    p_grid = sample_params(grid, rng)
    x_grid = encode(p_grid)
    y_grid, screen_ms = net.forward(x_grid, with_time=True)
    k_top = max(1, int(round(top_frac * grid)))
    top = np.argsort(-y_grid[:, -1], kind="stable")[:k_top]
    aud = rng.choice(grid, audit, replace=False)
    t_screen = time.perf_counter() - t0
    # verify: the top candidates and the audit set on the batched simulator
    t0 = time.perf_counter()
    pick = np.concatenate([top, aud])
    r_ver = sim.rates(p_grid[pick], seed0=10_000_000)
    t_verify = time.perf_counter() - t0
    total = time.perf_counter() - T0
    r_top, r_aud = r_ver[:k_top], r_ver[k_top:]
    # the simulator's own spread: the audit points again with other seeds
    r_aud2 = sim.rates(p_grid[aud], seed0=30_000_000)
    noise = rate_error(r_aud2, r_aud)
    pred_aud = decode_rates(y_grid[aud])
    pred_lin = decode_rates(lin(x_grid[aud]))
    err_mlp = rate_error(pred_aud, r_aud)
    err_lin = rate_error(pred_lin, r_aud)
    hyper_aud = r_aud.mean(1) > HYPER_HZ
    acc_mlp = float(np.mean((y_grid[aud, -1] > 0) == hyper_aud))
    acc_lin = float(np.mean((lin(x_grid[aud])[:, -1] > 0.5) == hyper_aud))
    # the plain engine looped per point, on a sample of the audit points
    looped = [sim.single_rates(p_grid[i], 20_000_000 + j)[1] for j, i in enumerate(aud[:looped_sample])]
    per_point_plain = float(np.mean(looped))
    res = {
        "neurons": neurons, "seconds_simulated": seconds, "train_points": n_train, "epochs": epochs,
        "grid": grid, "top": k_top, "audit": audit,
        "audit_rate_error_mean": float(err_mlp.mean()), "audit_rate_error_median": float(np.median(err_mlp)),
        "audit_rate_error_linear_mean": float(err_lin.mean()),
        "audit_mean_rate_error_mean": float(np.mean(np.abs(pred_aud.mean(1) - r_aud.mean(1)) /
                                                    np.maximum(r_aud.mean(1), 1e-9))),
        "audit_seed_to_seed_error_mean": float(noise.mean()),
        "audit_rate_error_vs_seed_mean_mean": float(rate_error(pred_aud, 0.5 * (r_aud + r_aud2)).mean()),
        "audit_hyper_accuracy": acc_mlp, "audit_hyper_accuracy_linear": acc_lin,
        "audit_hyper_fraction": float(hyper_aud.mean()),
        "top_verified_hyper_fraction": float(np.mean(r_top.mean(1) > HYPER_HZ)),
        "top_rate_error_mean": float(rate_error(decode_rates(y_grid[top]), r_top).mean()),
        "loss_first_last": [float(losses[0]), float(losses[-1])], "epochs_run": int(len(losses)),
        "validation_rate_error": val_err,
        "times_s": {"setup": t_setup, "train_data": t_data, "train": t_train, "screen": t_screen,
                    "verify": t_verify, "total": total},
        "device_ms": {"simulation": sim.device_ms, "train": train_ms, "screen": screen_ms},
        "plan": sim.plan,
        "plain_engine_s_per_point": per_point_plain,
        "plain_points_per_hour": 3600.0 / per_point_plain,
        "batched_sim_points_per_hour": 3600.0 * sim.points / max(t_data + t_verify, 1e-9),
        "surrogate_verified_points_per_hour": 3600.0 * grid / total,
    }
    res["speedup_vs_plain_looped"] = res["surrogate_verified_points_per_hour"] / res["plain_points_per_hour"]
    net.close()
    sim.close()
    return res


def main(argv: Optional[Sequence[str]] = None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--neurons", type=int, default=5000)
    ap.add_argument("--seconds", type=float, default=1.0)
    ap.add_argument("--train", type=int, default=20000)
    ap.add_argument("--epochs", type=int, default=600)
    ap.add_argument("--grid", type=int, default=1_000_000)
    ap.add_argument("--audit", type=int, default=1000)
    ap.add_argument("--seed", type=int, default=1)
    a = ap.parse_args(argv)
    print(json.dumps(run(a.neurons, a.seconds, a.train, a.epochs, a.grid, audit=a.audit, seed=a.seed)))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
