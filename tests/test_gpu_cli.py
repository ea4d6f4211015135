"""End-to-end drop-in check on the GPU: the reference executable built from
its sources (oracle/_ref/bd_aging_self.bin) and bd_aging_b200/bd_aging_self
run on identical inputs (same stdin, same init_config files, same idum, so
the same cuRAND noise) and their output files are compared."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from bd_aging_b200 import configs as CF

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "bd_aging_b200", "bd_aging_self")
REF = os.path.join(ROOT, "oracle", "_ref", "bd_aging_self.bin")
REF_LOG = os.path.join(ROOT, "oracle", "_ref", "bd_aging_self_log.bin")  # built with -DLOG_SAMPLE

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not (os.path.exists(CLI) and os.path.exists(REF)),
                                 reason="needs the CLI and the reference build")]

# run_time 0.0102 with dt 1e-5 gives niter = 1020, five samples (ngap 204)
DATA = "linear\n1.0  0.5  0.0  0.005  1\n1e-5\nlinear\n0.001  0.0102  5\n16  16\n2\n100  6.0\n6.19\n4321\n"
# run_time 0.01 gives niter = (int)(0.01/1e-5) = 999 and ngap 199: a sixth
# sample, which the reference rejects ("counter fuera de rango", exit 1)
BAD = DATA.replace("0.0102", "0.01")


def tree(base, nb, ns, phi, n_configs):
    (base / "configs").mkdir(parents=True)
    (base / "simulation" / "results").mkdir(parents=True)
    side = float(np.float32(CF.side_from_phi(nb, ns, phi)))
    for k in range(n_configs):
        CF.write_init_config(str(base / "configs" / ("init_config_%d" % (k + 1))),
                             CF.lattice_config(nb, ns, side, 40 + k, jitter=0.1), nb, ns, side)


def load(path):
    return np.loadtxt(str(path), ndmin=2)


def compare_observables(res_a, res_b):
    """Same cuRAND noise, same inputs: the runs differ by float rounding (the
    reference accumulates positions and observables in float, the engine
    carries a compensated remainder and sums in FP64).  Outputs are printed
    with %f (6 decimals), so one unit in the last place is 1e-6; measured
    differences are 1.5e-6 relative at most for energies and pressure, one
    printed unit for F_s and MSD."""
    ea, eb = load(res_a / "energies_averaged.out"), load(res_b / "energies_averaged.out")
    np.testing.assert_allclose(eb[:, 0], ea[:, 0], atol=1e-6)             # time
    np.testing.assert_allclose(eb[:, 3], ea[:, 3], atol=1e-6)             # temperature
    np.testing.assert_allclose(eb[:, 1:3], ea[:, 1:3], rtol=2e-5, atol=2e-6)
    pa, pb = load(res_a / "pressure.out"), load(res_b / "pressure.out")
    np.testing.assert_allclose(pb, pa, rtol=2e-5, atol=2e-6)
    fa, fb = load(res_a / "fself.out"), load(res_b / "fself.out")
    assert fa[0, 1] == 0.0 and fb[0, 1] == 0.0  # the reference's 1-based F_s index
    np.testing.assert_allclose(fb, fa, atol=2.5e-6)
    ma, mb = load(res_a / "msd_averaged.out"), load(res_b / "msd_averaged.out")
    np.testing.assert_allclose(mb[:, 0], ma[:, 0], atol=1e-6)
    np.testing.assert_allclose(mb[:, 1:], ma[:, 1:], rtol=1e-4, atol=2.5e-6)


def test_cli_outputs_match_reference_executable(tmp_path):
    a, b = tmp_path / "ref", tmp_path / "ours"
    tree(a, 500, 500, 0.45, 2)
    shutil.copytree(a, b)
    ra = subprocess.run([REF], input=DATA, cwd=a / "simulation", capture_output=True, text=True, timeout=600)
    rb = subprocess.run([CLI], input=DATA, cwd=b / "simulation", capture_output=True, text=True, timeout=600)
    assert ra.returncode == 0, ra.stdout[-2000:] + ra.stderr[-2000:]
    assert rb.returncode == 0, rb.stdout[-2000:] + rb.stderr[-2000:]
    assert "TERMINADO" in rb.stdout
    # bitacora: identical text (geometry, ranges, run lengths)
    assert (a / "simulation" / "bitacora").read_text() == (b / "simulation" / "bitacora").read_text()
    res_a, res_b = a / "simulation" / "results", b / "simulation" / "results"
    assert sorted(os.listdir(res_a)) == sorted(os.listdir(res_b))
    ea, eb = load(res_a / "energies_averaged.out"), load(res_b / "energies_averaged.out")
    np.testing.assert_allclose(eb[:, 0], ea[:, 0], atol=1e-6)            # time
    np.testing.assert_allclose(eb[:, 3], ea[:, 3], atol=1e-6)            # temperature
    compare_observables(res_a, res_b)
    for k in range(5):
        ga, gb = load(res_a / ("gder_%d.out" % k)), load(res_b / ("gder_%d.out" % k))
        np.testing.assert_allclose(gb[:, 0], ga[:, 0], atol=1e-6)
        # positions agree to ~1e-6, so a pair can still change bin at a bin edge
        diff = np.abs(gb[:, 1:] - ga[:, 1:])
        assert diff.mean() < 1e-3, diff.mean()
        assert not (diff > 0.05).any()


def test_cli_reproduces_reference_sample_counter_error(tmp_path):
    a, b = tmp_path / "ref", tmp_path / "ours"
    tree(a, 200, 200, 0.4, 1)
    shutil.copytree(a, b)
    data = BAD.replace("\n2\n100", "\n1\n100")
    ra = subprocess.run([REF], input=data, cwd=a / "simulation", capture_output=True, text=True, timeout=600)
    rb = subprocess.run([CLI], input=data, cwd=b / "simulation", capture_output=True, text=True, timeout=600)
    assert ra.returncode == rb.returncode == 1
    assert "ERROR: counter=6 fuera de rango" in ra.stderr
    assert "ERROR: counter=6 fuera de rango" in rb.stderr


# log sampling (LOG_SAMPLE build): 10 points per decade from 1e-4 to 1e-2
# (samples at ni = 0, 10, 13, ..., 794; 21 in all); decade 0 writes the
# configurations of decades 1 and 2 at samples 1 and 11 (main.cu:809-835),
# then decade 1 runs from the configurations each program wrote.  With no
# transient, the second configuration's first step shows the reference's
# carried-over temperature (temp_set is set to T0 once, main.cu:156).
LOG0 = "linear\n1.0  0.5  0.0  0.005  1\n1e-5\nlog\n0.0  1e-4  1e-2\n1  2  0\n16  16\n2\n100  6.0\n6.19\n4321\n"
LOG1 = LOG0.replace("\n1  2  0\n", "\n0  2  1\n")


def log_tree(base, nb, ns, phi, n_configs):
    for d in ("decade0", "decade1", "decade2"):
        (base / "configs" / d).mkdir(parents=True)
        (base / "simulation" / "results" / d).mkdir(parents=True)
    side = float(np.float32(CF.side_from_phi(nb, ns, phi)))
    for k in range(n_configs):
        CF.write_init_config(str(base / "configs" / "decade0" / ("init_config_%d" % (k + 1))),
                             CF.lattice_config(nb, ns, side, 40 + k, jitter=0.1), nb, ns, side)


def compare_results(res_a, res_b, nsamples):
    assert sorted(os.listdir(res_a)) == sorted(os.listdir(res_b))
    assert load(res_a / "energies_averaged.out").shape == load(res_b / "energies_averaged.out").shape == (nsamples, 4)
    compare_observables(res_a, res_b)
    for k in range(nsamples):
        ga, gb = load(res_a / ("gder_%d.out" % k)), load(res_b / ("gder_%d.out" % k))
        np.testing.assert_allclose(gb[:, 0], ga[:, 0], atol=1e-6)
        # positions agree to ~1e-6, so a pair can still change bin at a bin edge
        diff = np.abs(gb[:, 1:] - ga[:, 1:])
        assert diff.mean() < 1e-3, (k, diff.mean())
        assert not (diff > 0.05).any()


@pytest.mark.skipif(not os.path.exists(REF_LOG), reason="needs the reference LOG_SAMPLE build")
def test_cli_log_sampling_and_decade_configs_match_reference_executable(tmp_path):
    a, b = tmp_path / "ref", tmp_path / "ours"
    log_tree(a, 500, 500, 0.45, 2)
    shutil.copytree(a, b)
    for data in (LOG0, LOG1):
        ra = subprocess.run([REF_LOG], input=data, cwd=a / "simulation", capture_output=True, text=True,
                            timeout=600)
        rb = subprocess.run([CLI], input=data, cwd=b / "simulation", capture_output=True, text=True, timeout=600)
        assert ra.returncode == 0, ra.stdout[-2000:] + ra.stderr[-2000:]
        assert rb.returncode == 0, rb.stdout[-2000:] + rb.stderr[-2000:]
        assert (a / "simulation" / "bitacora").read_text() == (b / "simulation" / "bitacora").read_text()
    for d in ("decade0", "decade1"):
        compare_results(a / "simulation" / "results" / d, b / "simulation" / "results" / d, 21)
    assert os.listdir(a / "simulation" / "results" / "decade2") == []
    # decade configurations written by decade 0 at samples 1 (ni = 10) and 11 (ni = 100)
    for d in ("decade1", "decade2"):
        for k in (1, 2):
            fa, fb = a / "configs" / d / ("init_config_%d" % k), b / "configs" / d / ("init_config_%d" % k)
            la, lb = fa.read_text().splitlines(), fb.read_text().splitlines()
            assert la[:6] == lb[:6] and len(la) == len(lb) == 1006
            xa, xb = np.loadtxt(fa, skiprows=6), np.loadtxt(fb, skiprows=6)
            np.testing.assert_array_equal(xa[:, 0], xb[:, 0])
            # same cuRAND noise: positions agree to the printed precision
            np.testing.assert_allclose(xb[:, 1:], xa[:, 1:], atol=1.5e-5)
            assert np.abs(xb[:, 1:] - xa[:, 1:]).mean() < 2e-6
