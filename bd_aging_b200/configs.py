"""System geometry and the reference's configuration file format.

* Box side from packing fraction: phi = (pi/6) (N_A s_A^3 + N_B s_B^3) / L^3 with
  the WCA diameters sigma_A = 1.0 (small), sigma_B = 1.4 (big).  The reference's
  own generators are not part of its repository (run-fself.sh:84-86), so this
  convention is ours and is stated wherever a box is built from phi.
* The reference's "sigma" is the WCA cut distance s = 2^(1/6) sigma (its
  potential eps[(s/r)^12 - 2 (s/r)^6 + 1], potentials.cu:137-147, is standard
  WCA written in terms of the minimum), so sigma_big = 2^(1/6)*1.4 and
  sigma_sml = 2^(1/6)*1.0.
* init_config_%d files (main.cu:231-241, 377-394 read; main.cu:815-830 write):
  "phi_b phi_s", "side", "N_b N_s N_tot", "sigma_b sigma_s", "m_b m_s", blank,
  then "idx x y z" with big particles first.
"""
from __future__ import annotations

import math
import os

import numpy as np

TWO16 = 2.0 ** (1.0 / 6.0)
WCA_SIGMA_SML = 1.0
WCA_SIGMA_BIG = 1.4
SIGMA_SML = np.float32(TWO16 * WCA_SIGMA_SML)   # reference cut distance s_s
SIGMA_BIG = np.float32(TWO16 * WCA_SIGMA_BIG)   # reference cut distance s_b


def side_from_phi(n_big: int, n_sml: int, phi: float, d_big: float = WCA_SIGMA_BIG,
                  d_sml: float = WCA_SIGMA_SML) -> float:
    vol = (math.pi / 6.0) * (n_big * d_big ** 3 + n_sml * d_sml ** 3)
    return (vol / phi) ** (1.0 / 3.0)


def partial_phis(n_big: int, n_sml: int, side: float, d_big: float = WCA_SIGMA_BIG,
                 d_sml: float = WCA_SIGMA_SML):
    v = side ** 3
    return (math.pi / 6.0) * n_big * d_big ** 3 / v, (math.pi / 6.0) * n_sml * d_sml ** 3 / v


def lattice_config(n_big: int, n_sml: int, side: float, seed: int, jitter: float = 0.15) -> np.ndarray:
    """Seeded jittered simple-cubic lattice with randomly assigned species:
    overlap-free starting points for tests.  Returns float32 [N, 3], big first."""
    rng = np.random.default_rng(seed)
    n = n_big + n_sml
    m = int(math.ceil(n ** (1.0 / 3.0)))
    a = side / m
    g = np.stack(np.meshgrid(np.arange(m), np.arange(m), np.arange(m), indexing="ij"), -1).reshape(-1, 3)
    g = g[rng.permutation(len(g))[:n]]
    pos = (g + 0.5 + rng.uniform(-jitter, jitter, size=(n, 3))) * a
    pos = np.mod(pos, side).astype(np.float32)
    pos[pos >= np.float32(side)] = 0.0
    return pos


def uniform_config(n_big: int, n_sml: int, side: float, seed: int) -> np.ndarray:
    """Uniform random positions in [0, L)^3 (the first stage of the
    initial-configuration pipeline; overlaps are removed afterwards by
    capped-force relaxation on the GPU)."""
    rng = np.random.default_rng(seed)
    pos = rng.uniform(0.0, side, size=(n_big + n_sml, 3)).astype(np.float32)
    pos[pos >= np.float32(side)] = 0.0
    return pos


def write_init_config(path: str, pos: np.ndarray, n_big: int, n_sml: int, side: float,
                      sigma_big: float = float(SIGMA_BIG), sigma_sml: float = float(SIGMA_SML),
                      mass_big: float = 1.0, mass_sml: float = 1.0) -> None:
    """Write the reference init_config format (main.cu:815-830, %f fields)."""
    pb, ps = partial_phis(n_big, n_sml, side)
    with open(path, "w") as f:
        f.write("%f %f    phi b, s\n" % (pb, ps))
        f.write("%f    side\n" % side)
        f.write("%d %d %d    ngr b, s, tot\n" % (n_big, n_sml, n_big + n_sml))
        f.write("%f %f    sigma b, s\n" % (sigma_big, sigma_sml))
        f.write("%f %f    mass b, s\n" % (mass_big, mass_sml))
        f.write("\n")
        for i, (x, y, z) in enumerate(pos):
            f.write("%d %f %f %f\n" % (i, x, y, z))


def read_init_config(path: str):
    """Read an init_config file (main.cu:231-241, 377-394).  Returns a dict
    with phi_big, phi_sml, side, n_big, n_sml, n_tot, sigma_big, sigma_sml,
    mass_big, mass_sml and pos [N, 3] float32.  Raises FileNotFoundError
    (reference: exit -2) or ValueError on an index mismatch (reference:
    exit 1)."""
    if not os.path.exists(path):
        raise FileNotFoundError(path)
    with open(path) as f:
        lines = f.read().split("\n")
    h = [ln.split() for ln in lines[:5]]
    out = dict(phi_big=float(h[0][0]), phi_sml=float(h[0][1]), side=float(h[1][0]), n_big=int(h[2][0]),
               n_sml=int(h[2][1]), n_tot=int(h[2][2]), sigma_big=float(h[3][0]), sigma_sml=float(h[3][1]),
               mass_big=float(h[4][0]), mass_sml=float(h[4][1]))
    n = out["n_tot"]
    pos = np.zeros((n, 3), np.float32)
    for m in range(n):
        parts = lines[6 + m].split()
        if int(parts[0]) != m:
            raise ValueError("error: mm %d  nn %d no match" % (m, int(parts[0])))
        pos[m] = [np.float32(float(v)) for v in parts[1:4]]
    out["pos"] = pos
    return out
