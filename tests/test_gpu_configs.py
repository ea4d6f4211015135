"""The initial-configuration pipeline on the GPU (bd_aging_b200/make_configs.py;
the reference's generators are not in its repository, run-fself.sh:84-86):

* one capped-force step from a random placement with deep overlaps matches
  the oracle (forces of the reference's pair rule, the cap restated in
  oracle.c:or_eng_cap_forces, the engine update with the engine's Philox
  noise), in the neighbour-list step and in the 27-cell sweep;
* make() relaxes uniform random placements into states where no pair is
  closer than 0.75 of its WCA diameter (from under 0.2 before), written in
  the reference's init_config format (main.cu:231-241, 377-394);
* the reference's own executable (oracle/_ref, built from its sources) reads
  those files and runs on them."""
import os
import subprocess

import numpy as np
import pytest

from bd_aging_b200 import configs as CF
from bd_aging_b200 import lib as B
from bd_aging_b200 import make_configs as MC
from oracle import oracle as O

pytestmark = pytest.mark.gpu
SB, SS = float(CF.SIGMA_BIG), float(CF.SIGMA_SML)
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref", "bd_aging_self.bin")


def min_pair_ratio(pos, nb, side):
    """Smallest r_ij / sigma_ij over all pairs (minimum image, WCA diameters
    1.4 and 1.0 in BASELINE units), float64."""
    n = len(pos)
    p = pos.astype(np.float64)
    sig = np.where(np.arange(n) < nb, 1.4, 1.0)
    best = np.inf
    for i0 in range(0, n, 512):
        d = p[i0:i0 + 512, None, :] - p[None, :, :]
        d -= side * np.round(d / side)
        r = np.sqrt((d * d).sum(-1))
        s = 0.5 * (sig[i0:i0 + 512, None] + sig[None, :])
        idx = np.arange(i0, min(i0 + 512, n))
        r[idx - i0, idx] = np.inf
        best = min(best, float((r / s).min()))
    return best


@pytest.mark.parametrize("skin", [None, 0.0], ids=["list_step", "sweep_step"])
def test_capped_step_from_random_placement_matches_oracle(skin):
    nb = ns = 1500
    side = float(np.float32(CF.side_from_phi(nb, ns, 0.55)))
    pos = CF.uniform_config(nb, ns, side, 12)
    s = B.System(n_big=nb, n_sml=ns, side=side, sigma_big=SB, sigma_sml=SS, dt=1e-4, T0=1.0, protocol="const",
                 seed=77, force_cap=100.0)
    e = B.Engine([s], neighbor_skin=skin)
    e.set_positions(pos)
    e.run(1)
    hi, _ = e.get_positions()
    e.close()
    types = np.array([0] * nb + [1] * ns, np.int32)
    ff, _, _, _, _ = O.eng_forces(pos, types, side, SB, SS)
    raw_max = np.abs(ff).max()
    L = O.oracle_lib()
    L.or_eng_cap_forces(s.n, ff, 100.0)
    assert raw_max > 1e3 and np.abs(ff).max() <= 100.0 * (1 + 1e-6)  # the cap was active
    noise = O.eng_gauss3(s.seed, np.arange(s.n), 0).astype(np.float32)
    mob = np.array([np.float32(1) / np.float32(SB), np.float32(1) / np.float32(SS)], np.float32)
    amp = np.array([L.or_eng_amplitude(1.0, float(mob[0]), np.float32(s.dt)),
                    L.or_eng_amplitude(1.0, float(mob[1]), np.float32(s.dt))], np.float32)
    ohi, olo, odsp = pos.copy(), np.zeros_like(pos), np.zeros(pos.shape, np.float64)
    L.or_eng_update(s.n, ohi, olo, odsp, ff, types, side, s.dt, mob, amp, np.ascontiguousarray(noise))
    d = np.abs(hi - ohi)
    d = np.minimum(d, side - d)
    # capped displacements are up to 100 * mob * dt = 7e-3; rounding of the
    # force sums moves them by far less
    assert d.max() < 2e-5, d.max()


def test_make_configs_removes_overlaps_and_reference_reads_them(tmp_path):
    nb = ns = 500
    side0 = float(np.float32(CF.side_from_phi(nb, ns, 0.5)))
    start = CF.uniform_config(nb, ns, side0, 104729)  # make(seed=1)'s placement of configuration 1
    assert min_pair_ratio(start, nb, side0) < 0.2  # random placement: deep overlaps
    side, pos = MC.make(nb, ns, 0.5, 2, seed=1, relax_steps=2000)
    assert side == side0 and pos.shape == (2, 1000, 3)
    for k in range(2):
        assert np.all((pos[k] >= 0) & (pos[k] <= side))
        assert min_pair_ratio(pos[k], nb, side) > 0.75
    cfg = tmp_path / "configs"
    sim = tmp_path / "simulation"
    cfg.mkdir()
    (sim / "results").mkdir(parents=True)
    for k in range(2):
        CF.write_init_config(str(cfg / ("init_config_%d" % (k + 1))), pos[k], nb, ns, side)
    lines = (cfg / "init_config_1").read_text().splitlines()
    assert lines[2].split()[:3] == ["500", "500", "1000"] and lines[6].split()[0] == "0"
    if not os.path.exists(REF):
        pytest.skip("reference executable (oracle/_ref) not built")
    data = "linear\n1.0  1.0  0.0  1.0  1\n2e-5\nlinear\n0.0  0.004  2\n16  16\n2\n100  6.0\n6.28\n77\n"
    r = subprocess.run([REF], input=data, cwd=sim, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    e = np.loadtxt(sim / "results" / "energies_averaged.out", ndmin=2)
    assert e.shape == (2, 4) and np.all(np.isfinite(e))
    # relaxed states: the reference sees a finite, moderate potential energy per particle
    assert 0 <= e[0, 1] < 5.0 and 0 <= e[0, 2] < 5.0
