"""Host check of the list-mode displacement (k_list_dsp in csrc/nlist.cuh):
dsp = ((double)hi + (double)lo + (double)L * crossings) - origin.  The
compensated position hi + lo (FP32 with |lo| <= ulp(hi)) and L * crossings
are exact in FP64; their sum is exact while few crossings have accumulated
and otherwise rounds once (its 53 bits no longer reach the remainder's
lowest bits), and the subtraction of the origin rounds once: the result is
within two FP64 roundings of the exact value.  Checked against exact
rational arithmetic, with up to 40 crossings per axis."""
from fractions import Fraction

import numpy as np


def test_rebuilt_displacement_is_one_rounding_from_exact():
    g = np.random.default_rng(11)
    n = 20000
    L = np.float32(30.2731)
    hi = (g.random(n) * float(L)).astype(np.float32)
    # remainders up to one ulp of hi, as the compensated sum keeps them
    ulp = np.spacing(hi).astype(np.float64)
    lo = ((g.random(n) * 2 - 1) * ulp).astype(np.float32)
    img = g.integers(-40, 41, n)
    x0 = (g.random(n) * float(L)).astype(np.float64) + g.random(n) * 1e-9
    s1 = (hi.astype(np.float64) + lo.astype(np.float64)) + np.float64(L) * img.astype(np.float64)
    dsp = s1 - x0
    exact_sums = 0
    for k in range(0, n, 97):
        exact = Fraction(float(hi[k])) + Fraction(float(lo[k])) + Fraction(float(L)) * int(img[k]) - Fraction(x0[k])
        err = abs(Fraction(dsp[k]) - exact)
        bound = (Fraction(abs(float(np.spacing(s1[k])))) + Fraction(abs(float(np.spacing(dsp[k]))))) / 2
        assert err <= bound, (k, float(err), float(bound))
        if abs(int(img[k])) <= 2:  # a few crossings: the sum is exact, one rounding in all
            exact_sums += 1
            assert err <= Fraction(abs(float(np.spacing(dsp[k])))) / 2, (k, float(err))
    assert exact_sums > 5
