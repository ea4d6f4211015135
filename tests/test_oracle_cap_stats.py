"""CPU checks of two oracle pieces the GPU tests rely on: the capped-force
rule of the initial relaxation (oracle.c:or_eng_cap_forces) against a numpy
float32 restatement, and the seed-to-seed z-scores of oracle/statistics.py
on synthetic samples with and without a true difference."""
import numpy as np

from oracle import oracle as O
from oracle import statistics as ST


def cap_numpy(ff, fcap):
    out = ff.copy()
    for m in range(len(out)):
        f = out[m]
        fmx = np.float32(max(abs(f[0]), abs(f[1]), abs(f[2])))
        if fmx > 0 and np.isfinite(fmx):
            g = (f / fmx).astype(np.float32)
            ng = np.sqrt(np.float32(np.float32(g[0] * g[0] + g[1] * g[1]) + np.float32(g[2] * g[2])))
            if np.float32(fmx * ng) > fcap:
                out[m] = (g * np.float32(fcap / ng)).astype(np.float32)
        elif not np.isfinite(fmx):
            out[m] = 0.0
    return out


def test_cap_forces_matches_numpy_and_caps_magnitude():
    rng = np.random.default_rng(3)
    ff = (rng.standard_normal((2000, 3)) * 10.0 ** rng.uniform(-2, 6, (2000, 1))).astype(np.float32)
    ff[5] = [np.inf, 1.0, 2.0]
    ff[6] = [0.0, 0.0, 0.0]
    ff[7] = [3e38, -3e38, 1.0]
    with np.errstate(over="ignore"):  # the 3e38 row overflows |F|, as it does in float arithmetic
        want = cap_numpy(ff, np.float32(100.0))
    got = ff.copy()
    O.oracle_lib().or_eng_cap_forces(len(got), got, 100.0)
    np.testing.assert_array_equal(got, want)
    mag = np.sqrt((got.astype(np.float64) ** 2).sum(1))
    assert mag.max() <= 100.0 * (1 + 1e-6)
    small = np.sqrt((ff.astype(np.float64) ** 2).sum(1)) < 99.0
    np.testing.assert_array_equal(got[small], ff[small])            # below the cap: unchanged
    assert np.all(got[5] == 0) and np.all(got[6] == 0)                # non-finite -> zero; zero stays
    big = ~small & np.isfinite(ff).all(1)
    cosang = (got[big].astype(np.float64) * ff[big]).sum(1) / (
        mag[big] * np.sqrt((ff[big].astype(np.float64) ** 2).sum(1)))
    assert cosang.min() > 1 - 1e-6                                    # direction kept


def test_zscores_separate_equal_from_shifted_samples():
    rng = np.random.default_rng(9)
    a = rng.normal(1.0, 0.1, size=(8, 50))
    b = rng.normal(1.0, 0.1, size=(8, 50))
    _, _, se, z = ST._zscores(a, b)
    assert np.all(se > 0) and np.mean(z * z) < 2.0
    c = rng.normal(1.3, 0.1, size=(8, 50))
    _, _, _, z2 = ST._zscores(a, c)
    assert np.all(np.abs(z2) > 3.0)
    _, _, se0, z0 = ST._zscores(np.ones((8, 3)), np.ones((8, 3)))   # no spread: z = 0, not nan
    assert np.all(se0 == 0) and np.all(z0 == 0)
