"""Initial-configuration pipeline (the reference's set_init_config.bin /
eliminate_overlap.bin / bd_aging_configs.bin are not part of its repository,
run-fself.sh:84-86): uniform random positions at packing fraction phi, relaxed
by capped-force Brownian steps on the GPU with the same engine, written in the
reference's init_config format (main.cu:815-830).

    python -m bd_aging_b200.make_configs --n-big 500 --n-sml 500 --phi 0.5 \\
        --n-configs 5 --out configs/ [--relax-steps 2000] [--equil-steps 0] [--seed 1]

All configurations are relaxed together as one batch of replicas.
"""
from __future__ import annotations

import argparse
import dataclasses
import os

import numpy as np

from . import configs as CF
from . import lib as B


def relaxed_batch(systems, seed, steps=2000, force_cap=100.0, dt_relax=1e-4):
    """Start states of a batch of replicas: uniform random positions (replica
    k drawn with seed + k) relaxed together by `steps` capped-force steps
    (|F| <= force_cap, dt_relax, T = 1, Philox stream 1) on the GPU, or, with
    steps <= 0, jittered lattices.  Returns positions [sum N, 3]."""
    if steps <= 0:
        return np.concatenate([CF.lattice_config(s.n_big, s.n_sml, s.side, seed + k, jitter=0.05)
                               for k, s in enumerate(systems)])
    pos = np.concatenate([CF.uniform_config(s.n_big, s.n_sml, s.side, seed + k) for k, s in enumerate(systems)])
    relax = [dataclasses.replace(s, dt=dt_relax, protocol="const", T0=1.0, force_cap=force_cap) for s in systems]
    e = B.Engine(relax, rng_stream=1)
    e.set_positions(pos)
    e.run(steps)
    p, _ = e.get_positions()
    e.close()
    return p


def make(n_big, n_sml, phi, n_configs, seed=1, relax_steps=2000, equil_steps=0, temp=1.0, force_cap=100.0,
         dt_relax=1e-4, dt_equil=1e-5, mobility="reference"):
    """Returns (side, positions [n_configs, N, 3])."""
    side = float(np.float32(CF.side_from_phi(n_big, n_sml, phi)))
    base = B.System(n_big=n_big, n_sml=n_sml, side=side, sigma_big=float(CF.SIGMA_BIG),
                    sigma_sml=float(CF.SIGMA_SML), dt=dt_relax, T0=temp, protocol="const", seed=seed,
                    mobility=mobility, force_cap=force_cap)
    systems = [dataclasses.replace(base, seed=seed * 7919 + k) for k in range(n_configs)]
    pos = np.concatenate([CF.uniform_config(n_big, n_sml, side, seed * 104729 + k) for k in range(n_configs)])
    e = B.Engine(systems, rng_stream=1)
    e.set_positions(pos)
    if relax_steps:
        e.run(relax_steps)
    pos, _ = e.get_positions()
    e.close()
    if equil_steps:
        eq = [dataclasses.replace(s, dt=dt_equil, force_cap=0.0) for s in systems]
        e = B.Engine(eq, rng_stream=2)
        e.set_positions(pos)
        e.run(equil_steps)
        pos, _ = e.get_positions()
        e.close()
    return side, pos.reshape(n_configs, n_big + n_sml, 3)


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--n-big", type=int, required=True)
    ap.add_argument("--n-sml", type=int, required=True)
    ap.add_argument("--phi", type=float, required=True)
    ap.add_argument("--n-configs", type=int, default=1)
    ap.add_argument("--out", default="configs")
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--relax-steps", type=int, default=2000)
    ap.add_argument("--equil-steps", type=int, default=0)
    ap.add_argument("--temp", type=float, default=1.0)
    ap.add_argument("--mobility", default="reference", choices=["reference", "unit"])
    a = ap.parse_args()
    side, pos = make(a.n_big, a.n_sml, a.phi, a.n_configs, a.seed, a.relax_steps, a.equil_steps, a.temp,
                     mobility=a.mobility)
    os.makedirs(a.out, exist_ok=True)
    for k in range(a.n_configs):
        CF.write_init_config(os.path.join(a.out, "init_config_%d" % (k + 1)), pos[k], a.n_big, a.n_sml, side)
    print("wrote %d configurations (side %f) to %s" % (a.n_configs, side, a.out))


if __name__ == "__main__":
    main()
