#!/usr/bin/env python
"""Throughput of the Ermak-McCammon time step (cell list -> WCA pair forces ->
stochastic update) of the bidisperse WCA mixture, in particle-steps/s.

Workload (default "aging"): the aging quench of N = 32768 (16384 big sigma 1.4,
16384 small sigma 1.0 in WCA units), phi = 0.58, T 1.0 -> 0.1 instantaneous
jump, dt = 1e-5, run as R independent replicas in one batched engine
(batched vs plain is the metric; the plain single-replica engine is timed
beside it).  Inputs are synthetic: uniform random positions relaxed by 2000
capped-force steps on the GPU (the reference ships no configuration
generator).  One bench "step" = `--md-steps` time steps of every replica.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun each rank runs its own replicas (replicas only: the path does
not shard, there is no collective on the data path); value = all ranks'
particle-steps / max-over-ranks time.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particle-steps/s on 1 B200, batched vs plain, at matched g(r)/F_s error"
ALG_BYTES_PER_PARTICLE_STEP = 96  # FP32 position + remainder (24 B) and FP64 displacement (24 B), read + write
FLOP_PER_PAIR = 30                # FP32 work of one interacting pair force
FP32_PEAK_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="aging", choices=["aging", "batched", "large", "small", "surrogate"],
                    help="surrogate: training throughput of the learned surrogate only")
    ap.add_argument("--replicas", type=int, default=64)
    ap.add_argument("--md-steps", type=int, default=960)
    ap.add_argument("--no-extras", action="store_true", help="skip plain/e2e/reference-CUDA/CPU legs")
    ap.add_argument("--only-leg", default=None, choices=["correlator", "gder"],
                    help="after the timed steps run only this extra leg (for profiling)")
    ap.add_argument("--brick", type=int, nargs=3, default=None, help="cells per brick (default: engine's)")
    ap.add_argument("--threads", type=int, default=0, help="CTA size (default: engine's)")
    ap.add_argument("--relax-steps", type=int, default=2000,
                    help="capped-force relaxation steps; 0 starts from a jittered lattice instead")
    ap.add_argument("--mode", default="plain", choices=["plain", "persistent"],
                    help="one launch per time step, or persistent cluster launches of many steps")
    ap.add_argument("--cluster", type=int, default=0, help="CTAs per cluster in persistent mode")
    ap.add_argument("--autotune", action="store_true", help="time brick shapes during warm-up, keep the fastest")
    ap.add_argument("--skin", type=float, default=None,
                    help="neighbour-list skin (0: sweep every step; default: the library's)")
    ap.add_argument("--list-variant", type=int, default=None,
                    help="list-step launch variant (default: the library's; chosen by --autotune)")
    return ap.parse_args()


# ------------------------------------------------------------------ workloads
def workload_systems(name, replicas, rank):
    """Returns (systems, description dict). Seeds differ per rank."""
    from bd_aging_b200 import configs as CF
    from bd_aging_b200 import lib as B
    from bd_aging_b200 import ranks
    sb, ss = float(CF.SIGMA_BIG), float(CF.SIGMA_SML)
    rng = np.random.default_rng(1000 + rank)
    out = []
    if name == "aging":
        nb = ns = 16384
        side = float(np.float32(CF.side_from_phi(nb, ns, 0.58)))
        for r in range(replicas):
            out.append(B.System(n_big=nb, n_sml=ns, side=side, sigma_big=sb, sigma_sml=ss, dt=1e-5, T0=1.0, Tf=0.1,
                                t0=0.0, tf=1e-30, protocol="linear", seed=ranks.replica_seed(1, r, rank)))
        desc = {"workload": "aging quench N=32768 phi=0.58 T 1.0->0.1 dt=1e-5, %d replicas batched" % replicas,
                "n_per_replica": 32768, "replicas": replicas, "phi": 0.58}
    elif name == "batched":
        for r in range(256):
            n = int(rng.integers(500, 8001)) // 2 * 2
            phi = float(rng.uniform(0.50, 0.60))
            tfin = float(rng.uniform(0.05, 1.0))
            side = float(np.float32(CF.side_from_phi(n // 2, n // 2, phi)))
            out.append(B.System(n_big=n // 2, n_sml=n // 2, side=side, sigma_big=sb, sigma_sml=ss, dt=1e-5, T0=1.0,
                                Tf=tfin, t0=0.0, tf=1e-30, protocol="linear", seed=ranks.replica_seed(7, r, rank)))
        desc = {"workload": "256 ragged replicas N in [500,8000] phi in [0.50,0.60] T_final in [0.05,1.0] dt=1e-5",
                "replicas": 256}
    elif name == "large":
        nb = ns = 524288
        side = float(np.float32(CF.side_from_phi(nb, ns, 0.58)))
        out.append(B.System(n_big=nb, n_sml=ns, side=side, sigma_big=sb, sigma_sml=ss, dt=1e-5, T0=0.2,
                            protocol="const", seed=ranks.replica_seed(3, 0, rank)))
        desc = {"workload": "large single system N=1048576 phi=0.58 T=0.2 dt=1e-5", "replicas": 1}
    else:
        nb = ns = 500
        side = float(np.float32(CF.side_from_phi(nb, ns, 0.50)))
        out.append(B.System(n_big=nb, n_sml=ns, side=side, sigma_big=sb, sigma_sml=ss, dt=2e-5, T0=1.0,
                            protocol="const", seed=ranks.replica_seed(1, 0, rank)))
        desc = {"workload": "small N=1000 phi=0.50 T=1.0 dt=2e-5 single replica", "replicas": 1}
    return out, desc


def relaxed_positions(systems, seed, steps=2000):
    """Uniform random positions relaxed by `steps` capped-force steps on the
    GPU (Philox stream 1), all replicas at once; steps=0: jittered lattice."""
    from bd_aging_b200 import make_configs as MC
    return MC.relaxed_batch(systems, seed, steps)


# ------------------------------------------------------------------ clocks
class ClockSampler:
    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index),
                 "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for ln in open(self.path):
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for k, nm in enumerate(names):
                if r[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": float(rows[0][2]) if rows[0][2].replace(".", "").isdigit() else None,
                "reasons": sorted(reasons), "samples": len(rows)}


def measured_peak_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        return float(json.load(open(p))["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_traffic_per_particle_step(list_mode=False):
    """DRAM bytes per particle-step of the step kernel from the committed ncu
    summary (profiles/k_step_list_aging.md in neighbour-list mode, else
    profiles/k_step_aging.md; line 'dram_bytes_per_particle_step: X')."""
    p = os.path.join(ROOT, "profiles", "k_step_list_aging.md" if list_mode else "k_step_aging.md")
    if not os.path.exists(p):
        return None
    for ln in open(p):
        if ln.strip().startswith("dram_bytes_per_particle_step:"):
            try:
                return float(ln.split(":")[1].strip().split()[0])
            except ValueError:
                return None
    return None


# ------------------------------------------------------------------ legs
def cuda_time(engine, fn, iters):
    import torch
    s = torch.cuda.ExternalStream(engine.stream_handle())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(s)
    for _ in range(iters):
        fn()
    e1.record(s)
    e1.synchronize()
    return e0.elapsed_time(e1)  # ms


def cpu_baseline(pos=None, seconds=12.0):
    """Reference host implementation (oracle/_ref) on one N=32768 phi=0.58
    replica of the timed batch (its relaxed start state `pos`; a jittered
    lattice when none is given), single thread (the reference's *_hst
    functions keep state in static locals), bounded sample."""
    from oracle import oracle as O
    from bd_aging_b200 import configs as CF
    if not O.ref_available():
        return None
    nb = ns = 16384
    side = float(np.float32(CF.side_from_phi(nb, ns, 0.58)))
    if pos is None:
        pos = CF.lattice_config(nb, ns, side, 99, jitter=0.05)
    p = O.setup_params(side, nb, ns, float(CF.SIGMA_BIG), float(CF.SIGMA_SML), ntags=(16, 16), nbins=400,
                       rng=side / 2, dt=1e-5, T0=1.0)
    run = O.RefHostRun(p, pos)
    t = time.perf_counter()
    run.run(1, 1.0, 0.1, 0.0, 1e-30, 1e-5)
    one = max(time.perf_counter() - t, 1e-4)
    n = max(1, int(seconds / one))
    t = time.perf_counter()
    run.run(n, 1.0, 0.1, 0.0, 1e-30, 1e-5)
    el = time.perf_counter() - t
    return {"value": 32768 * n / el, "unit": "particle-steps/s", "cores": 1, "kind": "reference",
            "sample": "%d steps of replica 0 of the timed batch (N=32768 phi=0.58, relaxed start), reference "
                      "host loop (oracle/_ref)" % n}


def reference_cuda(steps=200):
    """The reference's own CUDA kernels (oracle/_ref/libref.so, built from the
    reference sources for sm_100a) in its main.cu step order, one N=32768
    phi=0.58 system, ntags 16."""
    from oracle import oracle as O
    from bd_aging_b200 import configs as CF
    import ctypes as C
    if not O.ref_available():
        return None
    nb = ns = 16384
    side = float(np.float32(CF.side_from_phi(nb, ns, 0.58)))
    pos = relaxed_positions_single(nb, ns, side)
    p = O.setup_params(side, nb, ns, float(CF.SIGMA_BIG), float(CF.SIGMA_SML), ntags=(16, 16), nbins=400,
                       rng=side / 2, dt=1e-5, T0=1.0)
    ob, os_ = np.zeros((nb, 3), np.float32), np.zeros((ns, 3), np.float32)
    wb, ws = np.zeros_like(ob), np.zeros_like(os_)
    ms = C.c_float(0)
    rc = O.ref_lib().ref_cuda_run(C.byref(p), pos[:nb].copy(), pos[nb:].copy(), 0, 20, 1, 1.0, 0.1, 0.0, 1e-30,
                                  1e-5, ob, os_, wb, ws, C.byref(ms))
    rc = O.ref_lib().ref_cuda_run(C.byref(p), pos[:nb].copy(), pos[nb:].copy(), 0, steps, 1, 1.0, 0.1, 0.0, 1e-30,
                                  1e-5, ob, os_, wb, ws, C.byref(ms))
    if rc != 0:
        return {"error": "reference CUDA run returned %d" % rc}
    return {"value": 32768 * steps / (ms.value / 1e3), "unit": "particle-steps/s", "steps": steps,
            "ms_per_step": ms.value / steps}


def gder_leg(eng, systems, nbins=400, rng=15.0, iters=3):
    """g(r) counts of every replica (bd_engine_gder, exact integers; the
    reference scripts' 400 bins to r = 15, run-fself.sh:46-47), by the
    engine's choice of method (the cell stencil wherever the box holds its
    region, else all pairs).  Rate: the N (N - 1) ordered pairs of each
    replica that the reference's all-pairs kernel tests, per second."""
    import torch
    eng.gder(nbins, rng)
    st = torch.cuda.ExternalStream(eng.stream_handle())
    t0 = time.perf_counter()
    for _ in range(iters):
        eng.gder(nbins, rng)
    st.synchronize()
    t = (time.perf_counter() - t0) / iters
    pairs = float(sum(s.n * (s.n - 1) for s in systems))
    return {"ms_per_call": t * 1e3, "nbins": nbins, "range": rng, "method": "auto", "ordered_pairs": pairs,
            "all_pairs_equivalent_per_s": pairs / t,
            "note": "wall time of the call (exact u64 counts copied back)"}


def correlator_leg(eng, P, slots=16, iters=20, q=6.19):
    """Waiting-time correlator on the bench batch: `slots` displacement
    snapshots, then all of them reduced against the current state in one
    call.  Traffic per call: current displacement + every snapshot (FP64 x 3)
    and the global index, (24 (slots + 1) + 4) bytes per particle."""
    eng.reserve_snapshots(slots)
    for k in range(slots):
        eng.snapshot(k)
        eng.run(1)
    sl = list(range(slots))
    eng.correlate(sl, q)
    ms = cuda_time(eng, lambda: eng.correlate(sl, q), iters)
    t = ms / 1e3 / iters
    traffic = (24 * (slots + 1) + 4) * P
    return {"slots": slots, "ms_per_call": t * 1e3, "evaluations_per_s": P * slots / t,
            "unit": "(particle, t_w) evaluations/s", "achieved_gbs": traffic / t / 1e9,
            "bytes_per_call": traffic, "note": "call time includes the host read-back of the sums"}


def precision_leg(n=8192, phi=0.58, steps=1000, temp=0.1, dt=1e-5, seed=5, q=7.0):
    """Observables after 10^3 steps of one replica (config-2 conditions after
    the quench: phi=0.58, T=0.1, dt=1e-5; N=8192 so the host FP64 run stays
    within seconds) from the engine and from host runs in FP64 and at the
    reference's FP32 precision, all with the engine's Philox noise and the
    same relaxed start.  Errors are relative to the FP64 run."""
    from bd_aging_b200 import configs as CF
    from bd_aging_b200 import lib as B
    from oracle import oracle as O
    sb, ss = float(CF.SIGMA_BIG), float(CF.SIGMA_SML)
    nb = ns = n // 2
    side = float(np.float32(CF.side_from_phi(nb, ns, phi)))
    relax = B.System(n_big=nb, n_sml=ns, side=side, sigma_big=sb, sigma_sml=ss, dt=1e-4, seed=99, T0=1.0,
                     protocol="const", force_cap=100.0)
    e = B.Engine([relax], rng_stream=1)
    e.set_positions(CF.uniform_config(nb, ns, side, seed))
    e.run(1500)
    pos, _ = e.get_positions()
    e.close()
    sysd = B.System(n_big=nb, n_sml=ns, side=side, sigma_big=sb, sigma_sml=ss, dt=dt, seed=seed, T0=temp,
                    protocol="const")
    e = B.Engine([sysd], qmax=q)
    e.set_positions(pos)
    e.run(steps)
    o = e.observe()[0]
    e.close()
    keys = ("msd_big", "msd_sml", "fself_big", "energy_big", "energy_sml", "virial")
    mb, ms = float(np.float32(1) / np.float32(sb)), float(np.float32(1) / np.float32(ss))
    args = (pos, nb, side, sb, ss, mb, ms, dt, temp, seed, steps, q)
    f64, _ = O.precision_run("fp64", *args)
    f32, _ = O.precision_run("fp32_reference", *args)
    return {"workload": "N=%d phi=%.2f T=%.2f dt=%g, %d steps, Philox noise" % (n, phi, temp, dt, steps),
            "fp64": {k: float(f64[k]) for k in keys},
            "engine_rel_err": {k: abs(o[k] - f64[k]) / abs(f64[k]) for k in keys},
            "fp32_reference_rel_err": {k: abs(f32[k] - f64[k]) / abs(f64[k]) for k in keys}}


SURROGATE_SIZES = [(256, 5)] + [(256, 256)] * 3 + [(34, 256)]       # live (N, K) per layer
SURROGATE_PADDED = [(256, 64)] + [(256, 256)] * 3 + [(128, 256)]    # as executed (K and N padded)


def surrogate_flops(sizes, batch):
    """Forward, weight-gradient and input-gradient GEMM FLOPs of one training step."""
    fwd = sum(2 * batch * n * k for n, k in sizes)
    dx = sum(2 * batch * n * k for n, k in sizes[1:])
    return 2 * fwd + dx


def surrogate_leg(steps=200, warmup=20, batch=4096):
    """Training steps of the surrogate (5 -> 256 x 4 -> 34, GELU, batch 4096,
    Adam) on a synthetic 1e5-sample set, each step one CUDA graph of
    gather, the fused forward and input-gradient kernel (the 5 forward and 4
    input-gradient GEMMs in one launch), 5 weight-gradient GEMMs, bias
    gradients and Adam."""
    from bd_aging_b200 import lib as B
    import torch
    rng = np.random.default_rng(0)
    x = rng.uniform(-1, 1, (100000, 5)).astype(np.float32)
    y = np.tanh(x @ rng.normal(size=(5, 34))).astype(np.float32)
    s = B.Surrogate(batch=batch, seed=1)
    s.set_data(x, y)
    s.train(warmup)
    st = torch.cuda.ExternalStream(s.stream_handle())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(st)
    loss = s.train(steps)
    e1.record(st)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / steps
    s.close()
    useful, executed = surrogate_flops(SURROGATE_SIZES, batch), surrogate_flops(SURROGATE_PADDED, batch)
    return {"ms_per_train_step": ms, "useful_tflops": useful / (ms / 1e3) / 1e12,
            "executed_tflops": executed / (ms / 1e3) / 1e12, "gflop_per_step_useful": useful / 1e9,
            "gflop_per_step_executed": executed / 1e9, "batch": batch, "final_loss": loss,
            "gemm_launches_per_step": 6, "gemms_per_step": 14}


def surrogate_quality_leg():
    """The surrogate trained on one ragged batched engine run (256 replicas,
    N in [500, 8000], phi in [0.50, 0.60], T_final in [0.05, 1.0], dt = 1e-5,
    16 waiting times x 8 lags x 3 wave numbers: about 1e5 samples, 4000 Adam
    steps) and its F_s error on plain N = 4000 runs at unseen settings
    (phi in {0.525, 0.575} x T_final in {0.2, 0.45, 0.7, 0.9}, 4 seeds each)."""
    from bd_aging_b200 import surrogate as S
    t0 = time.perf_counter()
    X, Y = S.build_batched_dataset(replicas=256, seed=11)
    t1 = time.perf_counter()
    model = S.SurrogateModel(seed=3)
    loss = model.fit(X, Y, steps=4000, lr=1e-3)
    t2 = time.perf_counter()
    mean_err, max_err, n = S.held_out_batched_fs_error(model)
    model.close()
    return {"train_samples": int(len(X)), "final_loss": loss, "held_out_points": n,
            "held_out_fs_mean_abs_err": mean_err, "held_out_fs_max_abs_err": max_err,
            "data": "256 ragged replicas, dt=1e-5, t_w 1e-3..1e-1, lags 1e-4..1e-1, k in {5, 7, 9}",
            "held_out": "plain N=4000 runs, phi {0.525, 0.575} x T_final {0.2, 0.45, 0.7, 0.9}, 4 seeds",
            "data_generation_s": t1 - t0, "training_s": t2 - t1}


def workload_leg(name, steps=3, warmup=2, md_steps=960, autotune=False):
    """Throughput of another BASELINE configuration on its own engine (same
    timing as the headline: CUDA events around `steps` runs of `md_steps` time
    steps after `warmup` runs, inputs resident).  "large" also reports the
    rate with its g(r) sample every 100 steps (config 4)."""
    from bd_aging_b200 import lib as B
    systems, desc = workload_systems(name, 64, 0)
    pos = relaxed_positions(systems, 777, 2000)
    P = sum(s.n for s in systems)
    eng = B.Engine(systems, graph_steps=96, autotune=int(autotune))
    eng.set_positions(pos)
    for _ in range(warmup):
        eng.run(md_steps)
    info0 = eng.info()
    ms = cuda_time(eng, lambda: eng.run(md_steps), steps)
    info = eng.info()
    out = dict(desc, value=P * md_steps * steps / (ms / 1e3), unit="particle-steps/s", particles=P,
               md_steps_per_bench_step=md_steps, ms_per_step=ms / steps, steps=steps, warmup=warmup,
               list_rebuild_steps_timed=int(info.list_rebuild_steps - info0.list_rebuild_steps),
               autotune=bool(autotune), brick=list(info.brick), list_variant=info.list_variant)
    if name == "large":  # g(r) every 100 steps, 400 bins to r = 15 (the cell stencil at this size)
        import torch
        eng.gder(400, 15.0)
        st = torch.cuda.ExternalStream(eng.stream_handle())
        t0 = time.perf_counter()
        eng.gder(400, 15.0)
        st.synchronize()
        tg = time.perf_counter() - t0
        t100 = 100 * (ms / 1e3) / (md_steps * steps)
        out["gder_ms_per_sample"] = tg * 1e3
        out["value_with_gder_every_100_steps"] = P * 100 / (t100 + tg)
    eng.close()
    return out


def statistics_leg(seeds=8):
    """Long-run agreement with the reference's own CUDA build at the aging
    workload's conditions (N = 32768, phi = 0.58, quench 1.0 -> 0.1, dt =
    1e-5, 2000 steps): 8 noise seeds of each from the same 8 relaxed states;
    MSD and F_s (k = 7) at 4 times and g(r) (400 bins to r = 15) compared
    through the seed-to-seed standard errors (oracle/statistics.py)."""
    from oracle import oracle as O
    from oracle import statistics as ST
    if not O.ref_available():
        return None
    r = ST.run(ST.AGING, seeds=seeds)
    obs = {o: {"t": r["times"][-1], "engine": v["engine"][-1], "reference": v["reference"][-1],
               "se": v["se"][-1], "max_abs_z_over_times": max(abs(z) for z in v["z"])}
           for o, v in r["observables"].items()}
    return {"workload": r["case"], "seeds": seeds, "observables": obs, "max_abs_z": r["max_abs_z"],
            "gder": r["gder"], "engine_s": r["engine_s"], "reference_s": r["reference_s"]}


_RELAXED_CACHE = {}


def relaxed_positions_single(nb, ns, side):
    from bd_aging_b200 import configs as CF
    from bd_aging_b200 import lib as B
    key = (nb, ns, side)
    if key not in _RELAXED_CACHE:
        s = B.System(n_big=nb, n_sml=ns, side=side, sigma_big=float(CF.SIGMA_BIG), sigma_sml=float(CF.SIGMA_SML),
                     dt=1e-5, T0=1.0, protocol="const", seed=1)
        _RELAXED_CACHE[key] = relaxed_positions([s], 4242)
    return _RELAXED_CACHE[key]


def run_surrogate_only(args):
    import torch
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    r = surrogate_leg(steps=max(1, args.steps) * 20, warmup=max(3, args.warmup))
    peak = None
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peak = json.load(f).get("bf16_tflops")
    except (OSError, ValueError):
        pass
    print(json.dumps({"metric": "surrogate training throughput", "value": r["useful_tflops"], "unit": "TFLOP/s",
                      "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
                      "dtype": "bf16 x bf16 -> f32", "data": "synthetic 1e5 x (5 -> 34)",
                      "config": {"workload": "MLP 5->256x4->34 GELU, batch 4096, Adam"},
                      "roofline": {"bound": "tensor", "achieved": r["executed_tflops"], "peak": peak,
                                   "unit": "TFLOP/s", "frac": (r["executed_tflops"] / peak) if peak else None},
                      "surrogate": r}))


def run_ours(args):
    if args.workload == "surrogate":
        return run_surrogate_only(args)
    import torch
    from bd_aging_b200 import lib as B
    from bd_aging_b200 import ranks
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    rank, world, local = ranks.init("nccl")
    systems, desc = workload_systems(args.workload, args.replicas, rank)
    pos = relaxed_positions(systems, 777 + rank, args.relax_steps)
    P = sum(s.n for s in systems)
    S = args.md_steps
    eng = B.Engine(systems, graph_steps=96, brick=args.brick, threads=args.threads, mode=args.mode,
                   cluster=args.cluster, autotune=int(args.autotune), neighbor_skin=args.skin,
                   list_variant=args.list_variant)
    eng.set_positions(pos)
    for _ in range(args.warmup):
        eng.run(S)
    info = eng.info()  # after warm-up: the autotuner may have changed the layout
    clocks = ClockSampler(local)
    clocks.start()
    ranks.barrier()
    ms = cuda_time(eng, lambda: eng.run(S), args.steps)
    ms = ranks.max_over_ranks(ms)
    ranks.barrier()
    ck = clocks.stop()
    rebuild_steps = eng.info().list_rebuild_steps - info.list_rebuild_steps
    # interacting partners per particle in the timed state (each ordered pair
    # once per particle), for the FP32 work of the pair forces
    nbr_count, _ = eng.census()
    pairs = float(nbr_count.astype(np.int64).sum())
    total_ps = P * S * args.steps * world
    value = total_ps / (ms / 1e3)
    launches = S * args.steps
    avg_launch_s = (ms / 1e3) / launches
    peak, peak_kind = measured_peak_hbm()
    achieved = ALG_BYTES_PER_PARTICLE_STEP * P / avg_launch_s / 1e9
    list_mode = info.neighbor_skin > 0
    tpp = profile_traffic_per_particle_step(list_mode)
    # kernels per time step: the list step plus its three rebuild kernels
    # (clear, bin, build; they exit at once when no list is stale), or the one
    # sweep kernel; per 96-step graph the counter kernel, plus the
    # noise-amplitude table in list mode (persistent mode: the persistent
    # kernel and the counter; per-replica list variants 3-5: the amplitude
    # table, the per-replica kernel, its flag kernel and the counter)
    per_replica = list_mode and info.list_variant >= 3
    per_step = 0 if per_replica else (4 if list_mode else (1 if args.mode == "plain" else 0))
    per_graph = 4 if per_replica else (2 if (list_mode or not per_step) else 1)
    gpu_launches = args.steps * (math.ceil(S / 96) * per_graph + per_step * S)
    line = {"metric": METRIC, "value": value, "unit": "particle-steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 forces, f32+compensation positions, f64 displacement",
            "data": "synthetic: uniform random positions relaxed by 2000 capped-force steps (GPU)",
            "config": dict(desc, md_steps_per_bench_step=S, mobility="reference 1/sigma",
                           l2="inputs larger than L2" if P * 112 > 126e6 else "state fits in L2",
                           brick=list(info.brick), threads=info.threads, cell_capacity=info.cell_capacity,
                           mode=args.mode, cluster=info.cluster if args.mode == "persistent" else None,
                           neighbor_skin=info.neighbor_skin, list_builds=info.list_builds,
                           list_variant=info.list_variant,
                           list_rebuild_steps_timed=int(rebuild_steps),
                           autotune=bool(args.autotune)),
            "gpu_launches": int(gpu_launches),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind,
                         "alg_bytes_per_launch": ALG_BYTES_PER_PARTICLE_STEP * P,
                         "traffic": (tpp * P) if tpp else None},
            "clocks": ck,
            # secondary roofline (pair forces on the FP32 pipes): 30 FLOP per
            # interacting ordered pair; nominal FP32 peak 148 SMs x 128 lanes
            # x 2 FLOP x 1.965 GHz
            "fp32": {"flop_per_launch": FLOP_PER_PAIR * pairs, "interacting_pairs_per_particle": pairs / P,
                     "achieved_tflops": FLOP_PER_PAIR * pairs / avg_launch_s / 1e12,
                     "peak_tflops": FP32_PEAK_TFLOPS, "peak_kind": "nominal",
                     "frac": FLOP_PER_PAIR * pairs / avg_launch_s / 1e12 / FP32_PEAK_TFLOPS}}
    if rank == 0 and world == 1 and args.only_leg:
        if args.only_leg == "correlator":
            line["correlator"] = correlator_leg(eng, P)
        else:
            line["gder"] = gder_leg(eng, systems)
    elif rank == 0 and world == 1 and not args.no_extras:
        # plain single-replica engine, same system
        s1 = systems[0]
        e1 = B.Engine([s1], graph_steps=96, brick=args.brick, threads=args.threads, neighbor_skin=args.skin)
        e1.set_positions(pos[: s1.n])
        e1.run(S)
        k1 = max(3, args.steps)
        ms1 = cuda_time(e1, lambda: e1.run(S), k1)
        plain = s1.n * S * k1 / (ms1 / 1e3)
        e1.close()
        line["plain"] = {"value": plain, "unit": "particle-steps/s", "replicas": 1}
        line["batched_over_plain"] = value / plain
        # end to end through the C ABI with pinned host buffers: positions in,
        # wrapped and unwrapped positions out, every step
        def pinned():
            return torch.empty((P, 3), dtype=torch.float32, pin_memory=True).numpy()
        in_pos, out_pos, out_raw = pinned(), pinned(), pinned()
        in_pos[:] = pos

        def e2e_step():
            eng.set_positions(in_pos)
            eng.run(S)
            eng.get_positions(out_pos, out_raw)
        e2e_step()
        ms2 = cuda_time(eng, e2e_step, max(2, args.steps // 2))
        k2 = max(2, args.steps // 2)
        line["e2e"] = {"value": P * S * k2 / (ms2 / 1e3), "unit": "particle-steps/s",
                       "h2d_bytes_per_step": P * 12, "d2h_bytes_per_step": P * 24}
        try:
            line["reference_cuda"] = reference_cuda()
            if line["reference_cuda"] and "value" in line["reference_cuda"]:
                line["batched_over_reference_cuda"] = value / line["reference_cuda"]["value"]
        except Exception as ex:  # reported, never fatal for the bench line
            line["reference_cuda"] = {"error": str(ex)[:200]}
        line["cpu_baseline"] = cpu_baseline(pos[:32768] if args.workload == "aging" else None)
        line["gder"] = gder_leg(eng, systems)
        line["correlator"] = correlator_leg(eng, P)
        eng.close()
        line["workloads"] = {}
        for wl in ("batched", "large", "small"):  # BASELINE configs 3, 4 and 1 beside the headline (config 2)
            try:
                line["workloads"][wl] = workload_leg(wl, autotune=(wl in ("batched", "small")))
            except Exception as ex:  # reported, never fatal for the bench line
                line["workloads"][wl] = {"error": str(ex)[:200]}
        line["precision"] = precision_leg()
        try:
            line["statistics"] = statistics_leg()
        except Exception as ex:  # reported, never fatal for the bench line
            line["statistics"] = {"error": str(ex)[:200]}
        line["surrogate"] = surrogate_leg()
        line["surrogate_quality"] = surrogate_quality_leg()
    eng.close()
    ranks.finalize()
    if rank == 0:
        print(json.dumps(line))


# ------------------------------------------------------------ reference arm
def _ref_worker(args_tuple):
    nsteps, reps, seed, pos = args_tuple
    sys.path.insert(0, ROOT)
    from oracle import oracle as O
    from bd_aging_b200 import configs as CF
    nb = ns = 16384
    side = float(np.float32(CF.side_from_phi(nb, ns, 0.58)))
    p = O.setup_params(side, nb, ns, float(CF.SIGMA_BIG), float(CF.SIGMA_SML), ntags=(16, 16), nbins=400,
                       rng=side / 2, dt=1e-5, T0=1.0)
    run = O.RefHostRun(p, pos, seed)
    t = time.perf_counter()
    for _ in range(reps):
        run.run(nsteps, 1.0, 0.1, 0.0, 1e-30, 1e-5)
    return time.perf_counter() - t


def reference_start_states(count):
    """The GPU arm's start states: replicas 0 .. count-1 of the aging batch
    (uniform random positions relaxed by 2000 capped-force steps, seed 777),
    made before any timing; without a GPU, jittered lattices."""
    from bd_aging_b200 import configs as CF
    try:
        import torch
        if torch.cuda.is_available():
            systems, _ = workload_systems("aging", max(64, count), 0)
            pos = relaxed_positions(systems, 777, 2000)
            return [pos[k * 32768:(k + 1) * 32768].copy() for k in range(count)], "relaxed"
    except Exception:
        pass
    side = float(np.float32(CF.side_from_phi(16384, 16384, 0.58)))
    return [CF.lattice_config(16384, 16384, side, 11 + k, jitter=0.05) for k in range(count)], "lattice"


def run_reference(args):
    """The reference's own CPU implementation (host functions compiled from its
    sources, oracle/_ref) on every host core: one independent N=32768 replica
    per process (its functions are not reentrant), each bench step a bounded
    sample of 2 time steps per replica.  The replicas start from the GPU arm's
    relaxed states (replicas 0 .. cores-1 of its batch)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle as O
    if not O.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libref.so not built"}))
        return
    import multiprocessing as mp
    try:
        cores = len(os.sched_getaffinity(0))
    except Exception:
        cores = os.cpu_count() or 1
    per = 2
    ctx = mp.get_context("spawn")
    with ctx.Pool(cores) as pool:  # started before the first GPU call
        states, kind = reference_start_states(cores)
        pool.map(_ref_worker, [(per, max(1, args.warmup // 3), 11 + k, states[k]) for k in range(cores)])
        t = time.perf_counter()
        pool.map(_ref_worker, [(per, args.steps, 11 + k, states[k]) for k in range(cores)])
        wall = time.perf_counter() - t
    total = 32768 * per * args.steps * cores
    value = total / wall
    line = {"metric": METRIC, "impl": "reference", "value": value, "unit": "particle-steps/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": wall * 1e3 / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": ("synthetic: the GPU arm's start states (uniform random positions relaxed by 2000 capped-force "
                     "steps, made before timing)" if kind == "relaxed" else "synthetic: jittered lattice"),
            "config": {"workload": "aging quench N=32768 phi=0.58 T 1.0->0.1 dt=1e-5, one replica per host core",
                       "replicas": cores, "md_steps_per_bench_step": per,
                       "replicas_note": "one replica per host core (the reference's host functions are not "
                                        "reentrant); the GPU arm batches 64"},
            "cpu_baseline": {"value": value, "unit": "particle-steps/s", "cores": cores, "kind": "reference",
                             "sample": "%d replicas x %d steps per bench step, reference host loop" % (cores, per)},
            "e2e": {"value": value, "unit": "particle-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
