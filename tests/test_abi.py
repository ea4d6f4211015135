"""C-ABI checks that need no GPU: the library loads, exports every function
declared in include/bd_aging.h, and its host-only functions agree with the
oracle / golden vectors."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from bd_aging_b200 import configs as CF
from bd_aging_b200 import lib as B
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for h in os.listdir(os.path.join(ROOT, "include")):
        if not h.endswith(".h"):
            continue
        txt = open(os.path.join(ROOT, "include", h)).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        names += re.findall(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\**\s*(bd_\w+)\s*\(", txt, flags=re.M)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    L = B.lib()
    names = declared_functions()
    assert len(names) > 20
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert L.bd_abi_version() == 2


def test_status_strings():
    L = B.lib()
    for code in range(10):
        assert L.bd_status_string(code)
    assert b"ntags" in L.bd_status_string(3)


@pytest.mark.parametrize("nb,ns,phi", [(150, 150, 0.45), (60, 240, 0.30), (16384, 16384, 0.58), (500, 500, 0.5)])
def test_setup_params_matches_reference_restatement(nb, ns, phi):
    side = CF.side_from_phi(nb, ns, phi)
    mine = B.setup_params(side, nb, ns, float(CF.SIGMA_BIG), float(CF.SIGMA_SML), ntags_big=16, ntags_sml=16,
                          nbins_gder=200, range_gder=side / 2, dt=1e-5, temp0=1.0)
    ref = O.setup_params(side, nb, ns, float(CF.SIGMA_BIG), float(CF.SIGMA_SML), ntags=(16, 16), nbins=200,
                         rng=side / 2, dt=1e-5, T0=1.0)
    assert bytes(mine) == bytes(ref)


def test_temperature_protocols_match_golden(golden):
    for row in golden["temp_linear"]:
        T0, Tf, t0, tf, t, ref = (np.float32(v) for v in row)
        mine = np.float32(B.calculate_temp_linear(T0, Tf, t0, tf, t))
        assert (np.isnan(ref) and np.isnan(mine)) or mine == ref
    for row in golden["temp_sine"]:
        T0, Tf, t0, tf, per, t, ref = (np.float32(v) for v in row)
        assert np.float32(B.calculate_temp_sine(T0, Tf, t0, tf, per, t)) == ref


def test_gder_normalize_matches_oracle():
    rng = np.random.default_rng(3)
    nbins = 50
    counts = rng.integers(0, 10 ** 6, size=(4, nbins)).astype(np.float64)
    side, nb, ns = 12.5, 500, 500
    mine = B.gder_normalize(counts, nbins, np.float32(side / 2 / nbins), side, nb, ns, float(CF.SIGMA_BIG),
                            float(CF.SIGMA_SML), 3)
    ref = np.zeros(4 * nbins, np.float32)
    O.oracle_lib().or_ref_gder_normalize(counts.ravel(), nbins, np.float32(side / 2 / nbins), side, nb, ns,
                                         float(CF.SIGMA_BIG), float(CF.SIGMA_SML), 3, ref)
    np.testing.assert_array_equal(mine.ravel(), ref)


def test_engine_rejects_bad_geometry_without_gpu():
    # argument validation happens before any device allocation
    s = B.System(n_big=10, n_sml=10, side=2.0, sigma_big=float(CF.SIGMA_BIG), sigma_sml=float(CF.SIGMA_SML),
                 dt=1e-5)
    with pytest.raises((B.BDError, RuntimeError)):
        B.Engine([s])


def test_list_variant_count_matches_implementation():
    """The public count of list-step launch variants (include/bd_aging.h) is
    the engine's (csrc/nlist.cuh), so the ABI accepts exactly the variants the
    engine launches."""
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    with open(os.path.join(root, "include", "bd_aging.h")) as f:
        public = int(re.search(r"#define BD_LIST_VARIANTS (\d+)", f.read()).group(1))
    with open(os.path.join(root, "bd_aging_b200", "csrc", "nlist.cuh")) as f:
        src = f.read()
    engine = int(re.search(r"constexpr int kListVariants = (\d+);", src).group(1))
    assert public == engine
    for v in range(engine):  # every variant has its launch parameters
        assert re.search(r"struct ListVariant<%d> \{" % v, src), v
