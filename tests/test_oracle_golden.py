"""Pin the CPU oracle against golden vectors produced by the reference itself
(tests/golden/make_golden.py runs the reference's host functions compiled from
its sources).  CPU only."""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle as O
from bd_aging_b200 import configs as CF

SYSTEMS = {"g1": (150, 150, 60, 0.5, 16), "g2": (60, 240, 40, 0.45, 16)}


def _params(golden, name):
    raw = golden[name + "_params"].tobytes()
    p = O.Parametros.from_buffer_copy(raw)
    return p


@pytest.mark.parametrize("name", list(SYSTEMS))
def test_params_restatement(golden, name):
    nb, ns, nbins, rfrac, ntags = SYSTEMS[name]
    ref = _params(golden, name)
    side = float(golden[name + "_side"])
    mine = O.setup_params(side, nb, ns, float(CF.SIGMA_BIG), float(CF.SIGMA_SML), ntags=(ntags, ntags),
                          nbins=nbins, rng=side * rfrac, dt=1e-4, T0=1.0)
    assert bytes(mine) == bytes(ref)


@pytest.mark.parametrize("name", list(SYSTEMS))
def test_cell_locate_bit_exact(golden, name):
    p = _params(golden, name)
    for sp in "bs":
        nocup, cell, bad = O.cell_locate(p, sp, golden[name + "_r" + sp])
        assert bad == 0
        np.testing.assert_array_equal(nocup, golden[name + "_nocup_" + sp])
        np.testing.assert_array_equal(cell, golden[name + "_cell_" + sp])


@pytest.mark.parametrize("name", list(SYSTEMS))
def test_forces_bit_exact(golden, name):
    p = _params(golden, name)
    out = O.ref_forces(p, golden[name + "_rb"], golden[name + "_rs"])
    for k in ("ff_b", "ff_s", "vir_b", "vir_s", "pot_b", "pot_s"):
        np.testing.assert_array_equal(out[k], golden[name + "_" + k], err_msg=k)


@pytest.mark.parametrize("name", list(SYSTEMS))
def test_update_bit_exact(golden, name):
    p = _params(golden, name)
    L = O.oracle_lib()
    for sp in "bs":
        rr = golden[name + "_r" + sp].copy()
        raw = rr.copy()
        L.or_ref_update_ermak(sp.encode(), rr, raw, golden[name + "_ff_" + sp].copy(),
                              golden[name + "_noise_" + sp], C.byref(p))
        np.testing.assert_array_equal(rr, golden[name + "_upd_rr_" + sp])
        np.testing.assert_array_equal(raw, golden[name + "_upd_raw_" + sp])


@pytest.mark.parametrize("name", list(SYSTEMS))
def test_gder_counts_exact(golden, name):
    p = _params(golden, name)
    counts = O.gder_counts(p, golden[name + "_rb"], golden[name + "_rs"])
    for k, pair in enumerate(("bb", "bs", "sb", "ss")):
        np.testing.assert_array_equal(counts[k].astype(np.float64), golden[name + "_gder_" + pair], err_msg=pair)
    # bs and sb are the same unordered pairs seen from either side
    np.testing.assert_array_equal(counts[1], counts[2])


def test_fself(golden):
    fs = np.zeros(4, np.float32)
    O.oracle_lib().or_ref_fself(golden["g1_fself_raw_b"], golden["g1_rb"], 150, fs, 2, np.float32(7.0))
    np.testing.assert_array_equal(fs, golden["g1_fself"])


def test_temperatures(golden):
    L = O.oracle_lib()
    for row in golden["temp_linear"]:
        T0, Tf, t0, tf, t, ref = (np.float32(v) for v in row)
        mine = np.float32(L.or_ref_temp_linear(T0, Tf, t0, tf, t))
        if np.isnan(ref):
            assert np.isnan(mine)
        else:
            assert mine == ref
    for row in golden["temp_sine"]:
        T0, Tf, t0, tf, per, t, ref = (np.float32(v) for v in row)
        assert np.float32(L.or_ref_temp_sine(T0, Tf, t0, tf, per, t)) == ref
    # the shipped run-fself.sh protocol (t0 = tf = 0) gives NaN at t == 0
    assert np.isnan(L.or_ref_temp_linear(1.0, 0.25, 0.0, 0.0, 0.0))


def test_sampling_indexes(golden):
    for k in range(4):
        md, rt, dt = golden["sampling_%d_args" % k]
        np.testing.assert_array_equal(O.sampling_indexes(md, rt, dt, 10), golden["sampling_%d" % k])


def test_rannew64(golden):
    L = O.oracle_lib()
    for k in range(2):
        st = (C.c_uint64 * 252)()
        buf = C.create_string_buffer(250 * 8 + 8 + 16)
        L.or_rannew64_seed(buf, C.c_long(int(golden["rannew64_%d_seed" % k][0])))
        vals = np.array([L.or_rannew64_next(buf) for _ in range(1000)])
        np.testing.assert_array_equal(vals, golden["rannew64_%d" % k])
        del st


@pytest.mark.parametrize("k", [0, 1])
def test_cv3d(golden, k):
    pos, xx = golden["cv3d_pos"], golden["cv3d_xx"]
    side = float(golden["cv3d_side"][0]) if k == 0 else -1.0
    a1, b1, bad1 = O.cv3d_add(16, 3.0, pos, xx, side)
    a2, b2, bad2 = O.cv3d_add(16, 3.0, pos[::-1].copy(), xx, side)
    assert bad1 == 0 and bad2 == 0
    vec = O.cv3d_solve(a1 + a2, b1 + b2)
    ref = golden["cv3d_%d_vec" % k]
    # the solve goes through an SVD: the reference's GSL routine is replaced by
    # a Jacobi SVD (shim) on one side and LAPACK on the other
    np.testing.assert_allclose(vec, ref, rtol=2e-3, atol=2e-3 * np.abs(ref).max())
