"""Long-run statistical agreement of the engine with the reference's own CUDA
build: K independent noise seeds of each, from the same K start states, and
the observables the reference samples compared at matched times through the
seed-to-seed spread.

TEST INFRASTRUCTURE ONLY (used by tests/test_gpu_statistics.py and bench.py's
statistics leg, always as the checker).  The reference side runs the
reference's kernels built from its sources (_ref/libref.so,
ref_cuda_run_sampled / ref_cuda_gder: cell_locate_dev, get_forces_*_dev,
update_ermak_dev in the order of main.cu:494-588, get_gder_dev of
get_gder.cu:69-127); its MSD and F_s follow main.cu:776-797 and
fself.cu:3-21 (displacements rr_raw - rr_ini since ni = 0), its g(r) the
normalisation of main.cu:849-877.  The engine side is the batched engine
with Philox noise (one replica per start state) and its own observation pass
and exact g(r) counts.

For every observable and time: z = (mean_engine - mean_reference) /
sqrt(se_engine^2 + se_reference^2), se = seed-to-seed standard deviation /
sqrt(K).  g(r) is compared bin by bin the same way and summarised by the mean
of z^2 over the bins where either side varies (about 1 when the two agree).
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import time

import numpy as np

from . import oracle as O

OBS = ("msd_big", "msd_sml", "fself_big")


@dataclasses.dataclass
class Case:
    name: str
    n_big: int
    n_sml: int
    phi: float
    dt: float
    T0: float
    Tf: float
    tf: float               # linear protocol from t0 = 0 to tf (tf = 1e-30: instantaneous quench)
    q: float                # wave number of F_s
    sample_after: tuple     # steps from ni = 0 at which MSD and F_s are compared (the last one: g(r) too)
    nbins: int
    rng: float              # g(r) range (0: L / 2)
    ntags: int = 16


# BASELINE conditions: config 1 (N = 1000, phi = 0.50, T = 1, dt = 2e-5, k = 2 pi,
# g(r) 200 bins to L/2) and config 2 (N = 32768, phi = 0.58, quench 1.0 -> 0.1,
# dt = 1e-5, k = 7.0, g(r) 400 bins to r = 15)
SMALL = Case("small N=1000 phi=0.50 T=1.0 dt=2e-5", 500, 500, 0.50, 2e-5, 1.0, 1.0, 1.0, 2 * np.pi,
             (250, 1000, 2500, 5000, 10000), 200, 0.0)
AGING = Case("aging quench N=32768 phi=0.58 T 1.0->0.1 dt=1e-5", 16384, 16384, 0.58, 1e-5, 1.0, 0.1, 1e-30, 7.0,
             (100, 300, 1000, 2000), 400, 15.0)


def _zscores(a, b):
    """a, b: [K, ...] per-seed values of the engine and the reference."""
    k = a.shape[0]
    ma, mb = a.mean(0), b.mean(0)
    sa, sb = a.std(0, ddof=1) / np.sqrt(k), b.std(0, ddof=1) / np.sqrt(k)
    se = np.sqrt(sa * sa + sb * sb)
    z = np.where(se > 0, (ma - mb) / np.where(se > 0, se, 1.0), 0.0)
    return ma, mb, se, z


def run(case: Case, seeds: int = 8, relax_seed: int = 321, idum0: int = 9001):
    """Runs both sides; returns a dict of per-time means, standard errors and
    z-scores, the g(r) summary, and the wall time of each side."""
    from bd_aging_b200 import configs as CF
    from bd_aging_b200 import lib as B
    from bd_aging_b200 import make_configs as MC
    sb, ss = float(CF.SIGMA_BIG), float(CF.SIGMA_SML)
    nb, ns = case.n_big, case.n_sml
    n = nb + ns
    side = float(np.float32(CF.side_from_phi(nb, ns, case.phi)))
    rng_g = case.rng if case.rng > 0 else side / 2
    protocol = "const" if case.T0 == case.Tf else "linear"
    systems = [B.System(n_big=nb, n_sml=ns, side=side, sigma_big=sb, sigma_sml=ss, dt=case.dt, T0=case.T0,
                        Tf=case.Tf, t0=0.0, tf=case.tf, protocol=protocol, seed=idum0 + 17 * k)
               for k in range(seeds)]
    start = MC.relaxed_batch(systems, relax_seed, 2000).reshape(seeds, n, 3)
    steps = list(case.sample_after)
    # engine: all seeds as one batch
    t0 = time.perf_counter()
    e = B.Engine(systems, qmax=case.q)
    e.set_positions(start.reshape(-1, 3))
    eng = {o: np.zeros((seeds, len(steps))) for o in OBS}
    done = 0
    for j, st in enumerate(steps):
        e.run(st - done)
        done = st
        for k, ob in enumerate(e.observe()):
            for o in OBS:
                eng[o][k, j] = ob[o]
    counts = e.gder(case.nbins, rng_g)
    e.close()
    bin_size = float(np.float32(rng_g) / np.float32(case.nbins))
    g_eng = np.stack([B.gder_normalize(counts[k].astype(np.float64), case.nbins, bin_size, side, nb, ns, sb, ss, 1)
                      for k in range(seeds)])
    t_eng = time.perf_counter() - t0
    # reference CUDA build: one run per seed, same start states
    t0 = time.perf_counter()
    p = O.setup_params(side, nb, ns, sb, ss, ntags=(case.ntags, case.ntags), nbins=case.nbins, rng=rng_g,
                       dt=case.dt, T0=case.T0)
    L = O.ref_lib()
    ref = {o: np.zeros((seeds, len(steps))) for o in OBS}
    g_ref = np.zeros((seeds, 4, case.nbins), np.float32)
    sa = np.array(steps, np.int32)
    for k in range(seeds):
        raw = np.zeros((len(steps), n, 3), np.float32)
        fb, fs = np.zeros((nb, 3), np.float32), np.zeros((ns, 3), np.float32)
        ms = C.c_float(0)
        rc = L.ref_cuda_run_sampled(C.byref(p), start[k, :nb].copy(), start[k, nb:].copy(), 0, steps[-1],
                                    systems[k].seed, case.T0, case.Tf, 0.0, case.tf, case.dt, len(steps), sa, raw,
                                    fb, fs, C.byref(ms))
        if rc != 0:
            raise RuntimeError("reference CUDA run returned %d" % rc)
        for j in range(len(steps)):
            d = raw[j].astype(np.float64) - start[k].astype(np.float64)
            r2 = (d * d).sum(1)
            ref["msd_big"][k, j] = r2[:nb].mean()          # main.cu:776-786
            ref["msd_sml"][k, j] = r2[nb:].mean()          # main.cu:787-792
            qr = case.q * np.sqrt(r2[:nb])                  # fself.cu:3-21 (big particles)
            ref["fself_big"][k, j] = np.where(qr > 0, np.sin(qr) / np.where(qr > 0, qr, 1.0), 1.0).mean()
        gc = np.zeros(4 * case.nbins, np.float32)
        if L.ref_cuda_gder(C.byref(p), fb, fs, gc) != 0:
            raise RuntimeError("reference g(r) failed")
        out = np.zeros((4, case.nbins), np.float32)
        O.oracle_lib().or_ref_gder_normalize(gc.astype(np.float64), case.nbins, bin_size, side, nb, ns, sb, ss, 1,
                                             out)
        g_ref[k] = out
    t_ref = time.perf_counter() - t0
    res = {"case": case.name, "seeds": seeds, "times": [s * case.dt for s in steps], "engine_s": t_eng,
           "reference_s": t_ref, "observables": {}}
    zmax = 0.0
    for o in OBS:
        ma, mb, se, z = _zscores(eng[o], ref[o])
        res["observables"][o] = {"engine": ma.tolist(), "reference": mb.tolist(), "se": se.tolist(),
                                 "z": z.tolist()}
        zmax = max(zmax, float(np.abs(z).max()))
    ma, mb, se, z = _zscores(g_eng.astype(np.float64), g_ref.astype(np.float64))
    live = se > 0
    res["gder"] = {"nbins": case.nbins, "range": rng_g, "bins_compared": int(live.sum()),
                   "mean_z2": float((z[live] ** 2).mean()), "max_abs_z": float(np.abs(z[live]).max()),
                   "peak_bb": [float(ma[0].max()), float(mb[0].max())],
                   "peak_ss": [float(ma[3].max()), float(mb[3].max())],
                   "peak_z": [float(z[0][ma[0].argmax()]), float(z[3][ma[3].argmax()])]}
    res["max_abs_z"] = zmax
    return res
