"""One-process aging workflow: every waiting time of the decade protocol in a
single run of the batched engine, with all (t_w, lag) correlations of a
sample step reduced in one pass.

The reference runs the protocol as a shell loop (run-fself.sh:149-197):

* decade 0 starts from ``configs/init_config_%d``, runs ``trans_time`` at the
  transient temperature, sets the origin at ni == 0 (main.cu:497-506), and
  samples on the log schedule ``sampling_indexes`` (main.cu:14-53);
* at samples 1, 11, 21, ... (``(counter - 1) % points_per_decade == 1``,
  main.cu:809-835) it writes the wrapped configuration to
  ``configs/decade%d/init_config_%d``;
* decade k restarts the program from that file, replays the transient and
  measures F_s / MSD against its own new origin; configurations are run one
  after another (main.cu:213) and averaged.

Here all configurations are replicas of one engine and every waiting time is
a displacement snapshot of the same trajectory: snapshot k is taken right
after the update at which the reference writes decade k's configuration,
and decade k's sample at lag index l is taken ``l + 1`` updates after it (the
reference samples after the update of step l, counting from its origin
step 0).  No transient is replayed at a waiting time: the system keeps
aging, which is what the waiting time is meant to measure.  Decade 0 is the
reference's own decade-0 run.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field

import numpy as np

from . import lib as B


def _roundf(x: float) -> int:
    """roundf: half away from zero."""
    return int(math.floor(x + 0.5)) if x >= 0 else -int(math.floor(-x + 0.5))


def sampling_indexes(minimal_decade: float, run_time: float, dt: float, per_decade: int = 10) -> list[int]:
    """Sample step indices of the log schedule (log_sampling + sampling_indexes,
    main.cu:14-53), in the reference's float arithmetic: index 0, then
    ``per_decade`` points per decade from ``minimal_decade`` up to ``run_time``."""
    f = np.float32
    last_power = _roundf(float(np.log10(f(run_time))))
    initial_power = _roundf(float(np.log10(f(minimal_decade))))
    r = f(np.power(f(10.0), f(1.0) / f(per_decade)))
    values, x = [], f(1.0)
    for _ in range(per_decade + 1):
        values.append(x)
        x = f(x * r)
    idx = [0]
    for ipow in range(initial_power, last_power):
        power = f(10.0 ** ipow)
        for j in range(per_decade):
            idx.append(_roundf(float(f(f(values[j] * power) / f(dt)))))
    return idx


def waiting_time_steps(idx: list[int], number_of_tws: int, per_decade: int = 10) -> list[int]:
    """Engine step counter (next update index) at each waiting time: 0 for
    decade 0 (the origin step), then one update after the sample at which the
    reference writes decade k's configuration (sample 1 + per_decade (k-1))."""
    tw = [0]
    for k in range(1, number_of_tws + 1):
        s = 1 + per_decade * (k - 1)
        if s >= len(idx):
            raise ValueError(f"decade {k}: sample {s} is past the end of the schedule ({len(idx)} samples)")
        tw.append(idx[s] + 1)
    return tw


@dataclass
class DecadeResult:
    """Replica-averaged observables of one waiting time, one row per sample."""
    t: np.ndarray            # time since the waiting time, dt (1 + l) (main.cu:520)
    fself_big: np.ndarray
    fself_sml: np.ndarray
    msd_big: np.ndarray
    msd_sml: np.ndarray
    alpha2_big: np.ndarray   # non-Gaussian parameter 3<r^4> / (5<r^2>^2) - 1
    alpha2_sml: np.ndarray
    energy_big: np.ndarray
    energy_sml: np.ndarray
    temperature: np.ndarray
    pressure: np.ndarray     # Z = 1 + W / (3 N T) (main.cu:801-806)
    per_replica: np.ndarray = field(repr=False)  # correlations [samples, R] (lib.CORR_DTYPE)
    gder: np.ndarray | None = None                # counts [samples, R, 4, nbins] or None


def _alpha2(r4, r2):
    with np.errstate(divide="ignore", invalid="ignore"):
        return np.where(r2 > 0, 3.0 * r4 / (5.0 * r2 * r2) - 1.0, 0.0)


def run_aging(engine: B.Engine, idx: list[int], tw_steps: list[int], q: float, dt: float,
              gder_bins: int = 0, gder_range: float = 0.0) -> list[DecadeResult]:
    """Runs `engine` (positions loaded, step counter <= 0) through every sample
    of every waiting time.  Returns one DecadeResult per waiting time."""
    info = engine.info()
    ni = int(info.next_step)
    if ni > 0:
        raise ValueError("the engine has passed its origin step")
    ntw = len(tw_steps)
    engine.reserve_snapshots(ntw)
    # events: engine step counter -> list of (decade, sample index)
    events: dict[int, list[tuple[int, int]]] = {}
    for k, tw in enumerate(tw_steps):
        for s, l in enumerate(idx):
            events.setdefault(tw + l + 1, []).append((k, s))
    snaps = {tw: k for k, tw in enumerate(tw_steps)}
    stops = sorted(set(events) | set(snaps))
    R = len(engine.systems)
    ns = len(idx)
    corr = [np.zeros((ns, R), B.CORR_DTYPE) for _ in range(ntw)]
    obs = [[None] * ns for _ in range(ntw)]
    grs = [np.zeros((ns, R, 4, gder_bins), np.uint64) for _ in range(ntw)] if gder_bins > 0 else None
    for stop in stops:
        if stop > ni:
            engine.run(stop - ni)
            ni = stop
        if stop in snaps:
            engine.snapshot(snaps[stop])
        if stop in events:
            ks = events[stop]
            c = engine.correlate([k for k, _ in ks], q)
            o = engine.observe()
            g = engine.gder(gder_bins, gder_range) if grs is not None else None
            for j, (k, s) in enumerate(ks):
                corr[k][s] = c[j]
                obs[k][s] = o
                if g is not None:
                    grs[k][s] = g
    n_tot = np.array([s.n for s in engine.systems], np.float64)
    out = []
    for k in range(ntw):
        cr = corr[k]
        rows = obs[k]
        t = np.array([np.float32(dt * (1.0 + np.float32(l))) for l in idx], np.float64)
        eb = np.array([[o["energy_big"] for o in row] for row in rows])
        es = np.array([[o["energy_sml"] for o in row] for row in rows])
        temp = np.array([[o["temperature"] for o in row] for row in rows])
        vir = np.array([[o["virial"] for o in row] for row in rows])
        z = 1.0 + vir / (3.0 * n_tot[None, :] * temp)
        out.append(DecadeResult(
            t=t,
            fself_big=cr["fself_big"].mean(1), fself_sml=cr["fself_sml"].mean(1),
            msd_big=cr["msd_big"].mean(1), msd_sml=cr["msd_sml"].mean(1),
            alpha2_big=_alpha2(cr["r4_big"], cr["msd_big"]).mean(1),
            alpha2_sml=_alpha2(cr["r4_sml"], cr["msd_sml"]).mean(1),
            energy_big=eb.mean(1), energy_sml=es.mean(1), temperature=temp[:, 0],
            pressure=z.mean(1), per_replica=cr, gder=grs[k] if grs is not None else None))
    return out


def write_decades(results: list[DecadeResult], outdir: str, gder_bins: int = 0, gder_range: float = 0.0,
                  systems=None):
    """Writes ``results/decade%d/{fself,msd_averaged,energies_averaged,pressure}.out``
    (and ``gder_%d.out`` when g(r) was sampled) in the reference's column
    layout and ``%f`` format (main.cu:886-980)."""
    for k, r in enumerate(results):
        d = os.path.join(outdir, f"decade{k}")
        os.makedirs(d, exist_ok=True)
        with open(os.path.join(d, "fself.out"), "w") as f:
            for i in range(len(r.t)):
                f.write("%f  %f\n" % (r.t[i], r.fself_big[i]))
        with open(os.path.join(d, "msd_averaged.out"), "w") as f:
            for i in range(len(r.t)):
                f.write("%f  %f  %f\n" % (r.t[i], r.msd_big[i], r.msd_sml[i]))
        with open(os.path.join(d, "energies_averaged.out"), "w") as f:
            for i in range(len(r.t)):
                f.write("%f  %f  %f  %f\n" % (r.t[i], r.energy_big[i], r.energy_sml[i], r.temperature[i]))
        with open(os.path.join(d, "pressure.out"), "w") as f:
            for i in range(len(r.t)):
                f.write("%f  %f\n" % (r.t[i], r.pressure[i]))
        with open(os.path.join(d, "nongaussian.out"), "w") as f:
            for i in range(len(r.t)):
                f.write("%f  %f  %f\n" % (r.t[i], r.alpha2_big[i], r.alpha2_sml[i]))
        if r.gder is not None and systems is not None:
            s0 = systems[0]
            counts = r.gder.sum(axis=1).astype(np.float64)  # over replicas
            bs = float(np.float32(gder_range) / np.float32(gder_bins))
            for i in range(len(r.t)):
                g = B.gder_normalize(counts[i], gder_bins, bs, s0.side, s0.n_big, s0.n_sml, s0.sigma_big,
                                     s0.sigma_sml, len(systems))
                with open(os.path.join(d, f"gder_{i}.out"), "w") as f:
                    for nb in range(gder_bins):
                        f.write("%f  %f  %f  %f  %f\n" % ((0.5 + nb) * bs, g[0][nb], g[1][nb], g[2][nb], g[3][nb]))


# ------------------------------------------------------------------ command line
def _read_protocol(fp):
    """The stdin protocol of main.cu:93-148 (log sampling)."""
    lines = [ln for ln in (raw.strip() for raw in fp) if ln]
    it = iter(lines)
    p = {"protocol": next(it).split()[0]}
    v = next(it).split()
    p["T0"], p["Tf"], p["t0"], p["tf"] = (float(x) for x in v[:4])
    p["period"] = float(v[4]) if p["protocol"] == "sine" else 1.0
    p["dt"] = float(next(it).split()[0])
    if next(it).split()[0] != "log":
        raise SystemExit("aging workflow: log sampling only (the waiting times are decades)")
    p["trans_time"], p["minimal_decade"], p["run_time"] = (float(x) for x in next(it).split()[:3])
    v = next(it).split()
    p["print_decades"], p["number_of_tws"], p["current_decade"] = (int(x) for x in v[:3])
    p["ntags_big"], p["ntags_sml"] = (int(x) for x in next(it).split()[:2])
    p["n_configs"] = int(next(it).split()[0])
    v = next(it).split()
    p["nbins_gder"], p["range_gder"] = int(v[0]), float(v[1])
    p["qmax"] = float(next(it).split()[0])
    p["idum"] = int(next(it).split()[0])
    return p


def main(argv=None):
    """Run every decade of run-fself.sh's loop in one process: reads the
    bd_aging_self.data protocol on stdin, the decade-0 configurations from
    ../configs/init_config_%d, and writes results/decade%d/ for decade 0 and
    every waiting time.  --no-gder skips the O(N^2) g(r) samples."""
    import argparse
    import sys

    from . import configs as CF
    ap = argparse.ArgumentParser(description=main.__doc__)
    ap.add_argument("--configs", default="../configs", help="directory of init_config_%%d")
    ap.add_argument("--results", default="results")
    ap.add_argument("--no-gder", action="store_true")
    ap.add_argument("--rng", default="philox", choices=["philox", "curand"])
    args = ap.parse_args(argv)
    p = _read_protocol(sys.stdin)
    cfgs = [CF.read_init_config(os.path.join(args.configs, f"init_config_{i + 1}")) for i in range(p["n_configs"])]
    for c in cfgs:  # wrap into the box as main.cu:387-393 does on reading
        side = np.float32(c["side"])
        x = c["pos"]
        x -= side * np.floor(x / side)
        x[(x < 0) | (x > side)] = 0.0
    systems = []
    for i, c in enumerate(cfgs):
        systems.append(B.System(n_big=c["n_big"], n_sml=c["n_sml"], side=c["side"], sigma_big=c["sigma_big"],
                                sigma_sml=c["sigma_sml"], dt=p["dt"], T0=p["T0"], Tf=p["Tf"], t0=p["t0"],
                                tf=p["tf"], period=p["period"], protocol=p["protocol"],
                                seed=(p["idum"] * 1000003 + i) if args.rng == "philox" else p["idum"]))
    ntrans = int(p["trans_time"] / p["dt"])
    eng = B.Engine(systems, rng=args.rng, qmax=p["qmax"], ni_start=-ntrans)
    eng.set_positions(np.concatenate([c["pos"] for c in cfgs]))
    idx = sampling_indexes(p["minimal_decade"], p["run_time"], p["dt"])
    tws = waiting_time_steps(idx, p["number_of_tws"])
    if ntrans > 0:
        eng.run(ntrans)
    nb = 0 if args.no_gder else p["nbins_gder"]
    res = run_aging(eng, idx, tws, p["qmax"], p["dt"], nb, p["range_gder"])
    write_decades(res, args.results, nb, p["range_gder"], systems)
    eng.close()
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
