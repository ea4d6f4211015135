"""Host-side behaviour of the drop-in CLI (no GPU needed): the stdin protocol
is consumed in the reference's order and the reference's exit codes come back
for missing or malformed configuration files (main.cu:225-229, 383-386)."""
import os
import subprocess

import numpy as np
import pytest

from bd_aging_b200 import configs as CF

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "bd_aging_b200", "bd_aging_self")

DATA = "linear\n1.0  0.5  0.0  0.005  1\n1e-5\nlinear\n0.001  0.01  5\n16  16\n2\n100  6.0\n6.19\n4321\n"

pytestmark = pytest.mark.skipif(not os.path.exists(CLI), reason="CLI not built")


def run(cwd, data=DATA):
    return subprocess.run([CLI], input=data, cwd=cwd, capture_output=True, text=True, timeout=60)


def test_missing_config_exits_minus_two(tmp_path):
    sim = tmp_path / "simulation"
    sim.mkdir()
    r = run(sim)
    assert r.returncode == 254  # exit(-2)
    assert "Verify file path: ../configs/init_config_1" in r.stdout
    for prompt in ("temp_protocol ?", "dt ?", "ntags: big, sml ?", "idum ?", "Starts simulation_3D_2SP Device"):
        assert prompt in r.stdout


def test_log_sampling_reads_decade_directory(tmp_path):
    sim = tmp_path / "simulation"
    sim.mkdir()
    data = "linear\n1.0  0.5  0.0  0.005  1\n1e-4\nlog\n0.1  1e-3  10.0\n1  3  2\n8  8\n1\n50  5.0\n6.19\n7\n"
    r = run(sim, data)
    assert r.returncode == 254
    assert "log sampling selected" in r.stdout
    assert "Verify file path: ../configs/decade2/init_config_1" in r.stdout


def test_index_mismatch_exits_one(tmp_path):
    (tmp_path / "configs").mkdir()
    sim = tmp_path / "simulation"
    sim.mkdir()
    nb = ns = 20
    side = CF.side_from_phi(nb, ns, 0.3)
    pos = CF.lattice_config(nb, ns, side, 1)
    path = tmp_path / "configs" / "init_config_1"
    CF.write_init_config(str(path), pos, nb, ns, side)
    lines = path.read_text().splitlines()
    lines[6 + 5] = "99 " + " ".join(lines[6 + 5].split()[1:])
    path.write_text("\n".join(lines) + "\n")
    r = run(sim)
    assert r.returncode == 1
    assert "error: mm 5  nn 99 no match" in r.stdout


def test_config_round_trip(tmp_path):
    nb, ns = 30, 50
    side = CF.side_from_phi(nb, ns, 0.4)
    pos = CF.lattice_config(nb, ns, side, 2)
    p = str(tmp_path / "init_config_1")
    CF.write_init_config(p, pos, nb, ns, side)
    c = CF.read_init_config(p)
    assert (c["n_big"], c["n_sml"], c["n_tot"]) == (nb, ns, nb + ns)
    np.testing.assert_allclose(c["pos"], pos, atol=1e-6)
    assert abs(c["side"] - side) < 1e-6
