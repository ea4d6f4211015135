"""Learned surrogate of the aging observables, trained on the engine's own
runs, and the proposal loop that uses it.

The network (bd_surrogate_*, hand-written tcgen05 BF16 GEMMs) maps a setting
    (phi, T_final, log10 t_w, log10 t, k)
to 34 outputs: F_s(k; t_w, t_w + t) of the big particles, log10 MSD of the
big particles over the same window, and 32 samples of the total g(r) at time
t_w + t.  The reference has no learned component; the engine is both the
source of the training data and the arbiter of every proposal: a proposed
setting is always simulated before it is used.

Proposal task.  For a fixed (phi, t_w, t, k), find the quench temperature
T* at which F_s falls to a target value (0.5 by default): the temperature
at which the structure relaxes within the observation window.  Without the
surrogate the simulation budget goes on a uniform temperature grid; with it,
each new simulation goes where the current network puts the crossing.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

from . import configs as CF
from . import lib as B

N_OUT = 34
G_BINS = 32
G_RANGE = (0.8, 2.4)  # r window of the g(r) features, in units of the small reference sigma


# ------------------------------------------------------------------ data
def make_systems(settings, n_per_replica=1000, dt=1e-4, seed=1):
    """One replica per (phi, T_final) or (phi, T_final, N): 50:50 mixture
    quenched from T0 = 1.0 to T_final at t = 0 (instantaneous: tf = t0 +
    1e-30), N = n_per_replica unless the setting gives it."""
    out = []
    for i, st in enumerate(settings):
        phi, tfin = st[0], st[1]
        n = int(st[2]) if len(st) > 2 else n_per_replica
        nb = ns = n // 2
        side = float(np.float32(CF.side_from_phi(nb, ns, float(phi))))
        out.append(B.System(n_big=nb, n_sml=ns, side=side, sigma_big=float(CF.SIGMA_BIG),
                            sigma_sml=float(CF.SIGMA_SML), dt=dt, T0=1.0, Tf=float(tfin), t0=0.0, tf=1e-30,
                            protocol="linear", seed=seed * 7919 + i))
    return out


def relaxed_start(systems, seed, relax_steps=1500):
    """Uniform random positions relaxed together by capped-force steps."""
    pos = np.concatenate([CF.uniform_config(s.n_big, s.n_sml, s.side, seed + k) for k, s in enumerate(systems)])
    relax = [dataclasses.replace(s, dt=1e-4, protocol="const", T0=1.0, force_cap=100.0) for s in systems]
    e = B.Engine(relax, rng_stream=1)
    e.set_positions(pos)
    e.run(relax_steps)
    p, _ = e.get_positions()
    e.close()
    return p


def g_features(counts, systems):
    """Total g(r) at G_BINS points in G_RANGE from exact counts [R, 4, bins]
    (bins of width (G_RANGE[1]) / nbins starting at 0)."""
    nb = counts.shape[-1]
    width = G_RANGE[1] / nb
    r_lo = np.arange(nb) * width
    shell = 4.0 / 3.0 * math.pi * ((r_lo + width) ** 3 - r_lo ** 3)
    out = []
    for r, s in enumerate(systems):
        tot = counts[r].sum(0).astype(np.float64)
        rho = s.n / s.side ** 3
        g = tot / (s.n * rho * shell)
        out.append(g[nb - G_BINS:])
    return np.array(out)


def simulate(settings, t_ws, lags, ks, n_per_replica=1000, dt=1e-4, trans_steps=200, seed=1, relax_steps=1500):
    """Run one replica per setting through every (t_w, lag) and return
    (X [samples, 5], Y [samples, 34]).  t_ws and lags are in steps; ks are
    wave numbers.  One batched engine, one correlator pass per sample step
    and wave number."""
    systems = make_systems(settings, n_per_replica, dt, seed)
    pos = relaxed_start(systems, seed, relax_steps)
    e = B.Engine(systems, ni_start=-trans_steps)
    e.set_positions(pos)
    e.run(trans_steps)
    tw_steps = sorted(set(int(t) for t in t_ws))
    e.reserve_snapshots(len(tw_steps))
    events = {}
    for k, tw in enumerate(tw_steps):
        for l in lags:
            events.setdefault(tw + int(l), []).append((k, int(l)))
    stops = sorted(set(events) | set(tw_steps))
    nbins = int(round(G_BINS * G_RANGE[1] / (G_RANGE[1] - G_RANGE[0])))
    rows_x, rows_y = [], []
    ni = 0
    for stop in stops:
        if stop > ni:
            e.run(stop - ni)
            ni = stop
        if stop in tw_steps:
            e.snapshot(tw_steps.index(stop))
        if stop not in events:
            continue
        slots = [k for k, _ in events[stop]]
        gf = g_features(e.gder(nbins, G_RANGE[1]), systems)
        for q in ks:
            c = e.correlate(slots, float(q))
            for j, (k, lag) in enumerate(events[stop]):
                tw_t, lag_t = max(tw_steps[k], 1) * dt, lag * dt
                for r, st in enumerate(settings):
                    phi, tfin = st[0], st[1]
                    msd = max(float(c[j, r]["msd_big"]), 1e-12)
                    rows_x.append([phi, tfin, math.log10(tw_t), math.log10(lag_t), q])
                    rows_y.append(np.concatenate([[c[j, r]["fself_big"], math.log10(msd)], gf[r]]))
    e.close()
    return np.array(rows_x, np.float32), np.array(rows_y, np.float32)


# ------------------------------------------------------------------ model
@dataclasses.dataclass
class Scaler:
    mean: np.ndarray
    std: np.ndarray

    @classmethod
    def fit(cls, a):
        s = a.std(0)
        return cls(a.mean(0), np.where(s > 1e-8, s, 1.0))

    def fwd(self, a):
        return ((a - self.mean) / self.std).astype(np.float32)

    def inv(self, a):
        return a * self.std + self.mean


class SurrogateModel:
    """Normalisation + the GPU network."""

    def __init__(self, width=256, depth=4, batch=4096, seed=1):
        self.net = B.Surrogate(n_in=5, n_out=N_OUT, width=width, depth=depth, batch=batch, seed=seed)
        self.sx = self.sy = None

    def fit(self, X, Y, steps=2000, lr=1e-3):
        if self.sx is None:
            self.sx, self.sy = Scaler.fit(X), Scaler.fit(Y)
        self.net.set_data(self.sx.fwd(X), self.sy.fwd(Y))
        return self.net.train(steps, lr)

    def predict(self, X):
        return self.sy.inv(self.net.predict(self.sx.fwd(np.asarray(X, np.float32))))

    def close(self):
        self.net.close()


# ------------------------------------------------------------------ proposals
def crossing(ts, fs, target):
    """Linear interpolation of the first crossing of fs(ts) through target
    (fs decreasing in ts); nearest end when there is none."""
    ts, fs = np.asarray(ts, np.float64), np.asarray(fs, np.float64)
    o = np.argsort(ts)
    ts, fs = ts[o], fs[o]
    for i in range(len(ts) - 1):
        a, b = fs[i] - target, fs[i + 1] - target
        if a == 0:
            return float(ts[i])
        if a * b < 0:
            return float(ts[i] + (ts[i + 1] - ts[i]) * a / (a - b))
    return float(ts[np.argmin(np.abs(fs - target))])


def propose_temperature(model, phi, log_tw, log_t, k, target=0.5, t_range=(0.05, 1.0), grid=400):
    """Quench temperature at which the surrogate puts F_s = target."""
    ts = np.linspace(t_range[0], t_range[1], grid)
    X = np.stack([np.full(grid, phi), ts, np.full(grid, log_tw), np.full(grid, log_t), np.full(grid, k)], 1)
    fs = model.predict(X)[:, 0]
    return crossing(ts, -fs, -target)  # F_s decreases as T rises


def fs_at(settings, tw, lag, k, seeds, n_per_replica=1000, dt=1e-4):
    """Plain simulation (the arbiter): F_s(k; t_w, t_w + lag) per setting,
    averaged over seeds, plus the sample rows of the whole run (8 lags up to
    `lag`, three wave numbers around k) for training."""
    reps = [s for s in settings for _ in seeds]
    lags = sorted(set(np.unique(np.geomspace(max(1, lag // 64), lag, 8).astype(int)).tolist()) | {int(lag)})
    ks = [0.7 * k, k, 1.3 * k]
    X, Y = simulate(reps, [tw], lags, ks, n_per_replica=n_per_replica, dt=dt, seed=int(seeds[0]))
    sel = (np.abs(X[:, 3] - math.log10(lag * dt)) < 1e-6) & (np.abs(X[:, 4] - np.float32(k)) < 1e-5)
    rows = X[sel]
    fs = np.zeros(len(settings))
    for i, (phi, tfin) in enumerate(settings):
        m = np.abs(rows[:, 1] - np.float32(tfin)) < 1e-7
        fs[i] = Y[sel][m, 0].mean()
    return fs, X, Y


def line_crossing(ts, fs, target, center, half_width):
    """Least-squares line through the points within center +- half_width
    (at least the three nearest), solved for fs = target."""
    ts, fs = np.asarray(ts, np.float64), np.asarray(fs, np.float64)
    d = np.abs(ts - center)
    sel = d <= half_width
    if sel.sum() < 3:
        sel = np.zeros(len(ts), bool)
        sel[np.argsort(d)[:3]] = True
    b, a = np.polyfit(ts[sel], fs[sel], 1)
    return float((target - a) / b) if b != 0 else float(center)


def crossing_study(phi=0.52, tw=100, lag=3000, k=7.0, budget=6, seeds=(1, 2, 3, 4), t_range=(0.05, 1.0),
                   truth_points=24, pretrain=None, fit_steps=1500, n_per_replica=1000, dt=1e-4, target=0.5):
    """Locate T* with F_s(k; t_w, t_w + lag) = target with `budget` simulated
    temperatures, (a) by a uniform grid and linear interpolation between the
    bracketing grid points, (b) with the surrogate: half the budget on a
    coarse grid, then proposals at the network's crossing and around it
    (each simulated, added to the training set, the network refitted), the
    estimate a least-squares line through the simulated points near the
    proposals.  The truth is a dense plain sweep.  The simulations decide:
    both estimates use simulated values only."""
    log_tw, log_t = math.log10(max(tw, 1) * dt), math.log10(lag * dt)
    ts_truth = np.linspace(t_range[0], t_range[1], truth_points)
    f_truth, _, _ = fs_at([(phi, t) for t in ts_truth], tw, lag, k, seeds, n_per_replica, dt)
    t_star = crossing(ts_truth, f_truth, target)
    # uniform grid
    ts_grid = np.linspace(t_range[0], t_range[1], budget)
    f_grid, _, _ = fs_at([(phi, t) for t in ts_grid], tw, lag, k, seeds, n_per_replica, dt)
    t_grid = crossing(ts_grid, f_grid, target)
    # surrogate: coarse grid, then proposals
    n0 = max(2, budget // 2)
    ts_s = list(np.linspace(t_range[0], t_range[1], n0))
    f_s, X, Y = fs_at([(phi, t) for t in ts_s], tw, lag, k, seeds, n_per_replica, dt)
    f_s = list(f_s)
    if pretrain is not None:
        X, Y = np.concatenate([pretrain[0], X]), np.concatenate([pretrain[1], Y])
    model = SurrogateModel(seed=5)
    model.fit(X, Y, steps=fit_steps)
    spacing = (t_range[1] - t_range[0]) / (n0 - 1)
    offsets = [0.0, -0.25, 0.25, -0.5, 0.5]  # in units of the coarse spacing / 2
    proposals, center = [], None
    for i in range(budget - n0):
        c = propose_temperature(model, phi, log_tw, log_t, k, target, t_range)
        center = c if center is None else c
        tp = float(np.clip(c + offsets[i % len(offsets)] * spacing * 0.5, t_range[0], t_range[1]))
        proposals.append(tp)
        fp, Xp, Yp = fs_at([(phi, tp)], tw, lag, k, seeds, n_per_replica, dt)
        ts_s.append(tp)
        f_s.append(float(fp[0]))
        X, Y = np.concatenate([X, Xp]), np.concatenate([Y, Yp])
        model.fit(X, Y, steps=fit_steps // 2)
    model.close()
    t_sur = line_crossing(ts_s, f_s, target, center, 0.3 * spacing)
    return {"t_star": t_star, "grid": t_grid, "surrogate": t_sur, "err_grid": abs(t_grid - t_star),
            "err_surrogate": abs(t_sur - t_star), "proposals": proposals, "budget": budget,
            "f_truth": [float(v) for v in f_truth], "ts_truth": [float(v) for v in ts_truth]}


# ------------------------------------------------------------------ held-out error
TRAIN_TW = (10, 100, 300, 1000)                      # steps at dt = 1e-4
TRAIN_LAGS = tuple(int(v) for v in np.unique(np.geomspace(10, 3000, 12).astype(int)))
TRAIN_KS = (5.0, 6.0, 7.0, 8.0, 9.0)


def build_dataset(phis, temps, seeds, t_ws=TRAIN_TW, lags=TRAIN_LAGS, ks=TRAIN_KS, n_per_replica=1000,
                  dt=1e-4, seed=1):
    """Training rows from one batched run: every (phi, T_final) x seed is a
    replica; each contributes one row per (t_w, lag, k)."""
    settings = [(float(p), float(t)) for p in phis for t in temps for _ in range(seeds)]
    return simulate(settings, list(t_ws), list(lags), list(ks), n_per_replica=n_per_replica, dt=dt, seed=seed)


def seed_average(X, Y):
    """Rows with identical inputs (replicas of one setting) averaged."""
    keys, inv = np.unique(np.round(X.astype(np.float64), 6), axis=0, return_inverse=True)
    inv = inv.ravel()
    ys = np.zeros((len(keys), Y.shape[1]))
    np.add.at(ys, inv, Y)
    cnt = np.bincount(inv, minlength=len(keys))[:, None]
    return keys.astype(np.float32), (ys / cnt).astype(np.float32)


def held_out_fs_error(model, phis, temps, seeds=4, n_per_replica=1000, dt=1e-4, seed=777, t_ws=TRAIN_TW,
                      lags=TRAIN_LAGS, ks=TRAIN_KS):
    """Mean and max |F_s(predicted) - F_s(simulated)| over plain runs at
    settings the model has not seen (seed-averaged simulations)."""
    X, Y = build_dataset(phis, temps, seeds, t_ws=t_ws, lags=lags, ks=ks, n_per_replica=n_per_replica, dt=dt,
                         seed=seed)
    Xa, Ya = seed_average(X, Y)
    err = np.abs(model.predict(Xa)[:, 0] - Ya[:, 0])
    return float(err.mean()), float(err.max()), len(Xa)


# ------------------------------------------------------------------ batched-run data
# Training data from one ragged batch of replicas like the batched workload:
# N uniform in [500, 8000], phi uniform in [0.50, 0.60], T_final uniform in
# [0.05, 1.0], dt = 1e-5, instantaneous quench from T0 = 1.0; 16 waiting
# times log-spaced over two decades and 8 lags log-spaced over three decades
# (in steps), three wave numbers: 256 replicas give about 1e5 samples.
BATCH_DT = 1e-5
BATCH_TW = tuple(int(v) for v in np.unique(np.geomspace(100, 10000, 16).astype(int)))
BATCH_LAGS = tuple(int(v) for v in np.unique(np.geomspace(10, 10000, 8).astype(int)))
BATCH_KS = (5.0, 7.0, 9.0)


def ragged_settings(replicas, seed):
    """(phi, T_final, N) of `replicas` replicas drawn like the batched workload."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(replicas):
        n = int(rng.integers(500, 8001)) // 2 * 2
        out.append((float(rng.uniform(0.50, 0.60)), float(rng.uniform(0.05, 1.0)), n))
    return out


def build_batched_dataset(replicas=256, seed=11, t_ws=BATCH_TW, lags=BATCH_LAGS, ks=BATCH_KS, dt=BATCH_DT):
    """Training rows from one ragged batched run (one row per replica, t_w,
    lag and wave number)."""
    return simulate(ragged_settings(replicas, seed), list(t_ws), list(lags), list(ks), dt=dt, seed=seed)


def held_out_batched_fs_error(model, phis=(0.525, 0.575), temps=(0.2, 0.45, 0.7, 0.9), seeds=4, n=4000,
                              seed=777):
    """held_out_fs_error on plain runs of N = n at fixed (phi, T_final)
    settings, over the batched data's windows and wave numbers."""
    return held_out_fs_error(model, phis, temps, seeds=seeds, n_per_replica=n, dt=BATCH_DT, seed=seed,
                             t_ws=BATCH_TW, lags=BATCH_LAGS, ks=BATCH_KS)
