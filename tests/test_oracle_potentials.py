"""The pair potentials of potentials.cu that the reference defines but never
calls: the oracle's restatement against the reference's own host functions
(oracle/_ref) bit for bit, and the HSAY form (written as potentials.cu
intends) against a finite difference of its energy."""
import numpy as np
import pytest

from bd_aging_b200 import configs as CF
from oracle import oracle as O

SIG = [float(CF.SIGMA_BIG), 1.2, float(CF.SIGMA_SML)]
DIST_INV = np.float32(1.0) / np.linspace(0.8, 1.7, 61).astype(np.float32)


def _ref(fn, *args):
    import ctypes as C
    u, nf = C.c_float(0), C.c_float(0)
    getattr(O.ref_lib(), fn)(*args, C.byref(u), C.byref(nf))
    return u.value, nf.value


@pytest.mark.skipif(not O.ref_available(), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("sigma", SIG)
def test_pair_potentials_match_reference(sigma):
    for di in DIST_INV:
        di = float(di)
        assert O.pair_extra("wca", [0, 0, 0, 0], sigma, di) == _ref("ref_potential_wca_hst", sigma, di)
        pp = [2.5, 1.3, 0, 0]
        assert O.pair_extra("wca49_50", pp, sigma, di) == _ref("ref_potential_wca49_50_hst", sigma, di, 2.5, 1.3)
        pp = [2.5, 1.3, 0.4, 0.15]
        assert O.pair_extra("ao", pp, sigma, di) == _ref("ref_potential_wca49_50_AO_hst", sigma, di, 2.5, 1.3,
                                                          0.4, 0.15)


def test_hsay_force_is_the_energy_derivative():
    pp = [2.0, 2.5, 0, 0]
    for r in np.linspace(0.9, 2.4, 31) + 0.013:  # away from r = s, where the core's curvature jumps
        h = 1e-3
        up, _ = O.pair_extra("hsay", pp, 1.0, 1.0 / (r + h))
        um, _ = O.pair_extra("hsay", pp, 1.0, 1.0 / (r - h))
        _, nf = O.pair_extra("hsay", pp, 1.0, 1.0 / r)
        assert nf == pytest.approx((up - um) / (2 * h), rel=2e-3, abs=2e-3)
