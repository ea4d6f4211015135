"""GPU parity of the reference-mirror entry points (C ABI) against the golden
vectors produced by the reference itself and against the oracle."""
import ctypes as C

import numpy as np
import pytest

from bd_aging_b200 import configs as CF
from bd_aging_b200 import lib as B
from oracle import oracle as O

pytestmark = pytest.mark.gpu
SYSTEMS = ("g1", "g2")


def dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda:0")


def host(t):
    import torch
    torch.cuda.synchronize()
    return t.cpu().numpy()


def params(golden, name):
    return B.Parametros.from_buffer_copy(golden[name + "_params"].tobytes())


def cells(p, sp, rr_d):
    import torch
    nc = p.ncell_big if sp == "b" else p.ncell_sml
    nt = p.ntags_big if sp == "b" else p.ntags_sml
    nocup = torch.zeros(nc ** 3, dtype=torch.int32, device="cuda:0")
    cell = torch.zeros(nc ** 3 * nt, dtype=torch.int32, device="cuda:0")
    B.cell_locate(sp, rr_d, nocup, cell, p)
    return nocup, cell


@pytest.mark.parametrize("name", SYSTEMS)
def test_cell_locate_bit_exact(golden, name):
    p = params(golden, name)
    for sp in "bs":
        nocup, cell = cells(p, sp, dev(golden[name + "_r" + sp]))
        np.testing.assert_array_equal(host(nocup), golden[name + "_nocup_" + sp])
        np.testing.assert_array_equal(host(cell), golden[name + "_cell_" + sp])


def forces_four_calls(p, rb, rs):
    import torch
    rb_d, rs_d = dev(rb), dev(rs)
    nob, cb = cells(p, "b", rb_d)
    nos, cs = cells(p, "s", rs_d)
    z = lambda n, k: torch.zeros((n, k) if k > 1 else n, dtype=torch.float32, device="cuda:0")
    ffb, ffs = z(len(rb), 3), z(len(rs), 3)
    vb, pb, vs, ps = z(len(rb), 1), z(len(rb), 1), z(len(rs), 1), z(len(rs), 1)
    B.get_forces_same("b", rb_d, ffb, vb, pb, nob, cb, p)
    B.get_forces_same("s", rs_d, ffs, vs, ps, nos, cs, p)
    B.get_forces_diff("b", "s", rb_d, ffb, rs_d, vb, pb, nos, cs, p)
    B.get_forces_diff("s", "b", rs_d, ffs, rb_d, vs, ps, nob, cb, p)
    return dict(ff_b=host(ffb), ff_s=host(ffs), vir_b=host(vb), vir_s=host(vs), pot_b=host(pb), pot_s=host(ps))


@pytest.mark.parametrize("name", SYSTEMS)
def test_forces_match_reference(golden, name):
    p = params(golden, name)
    out = forces_four_calls(p, golden[name + "_rb"], golden[name + "_rs"])
    for k, v in out.items():
        ref = golden[name + "_" + k]
        # same neighbour sets and sum order as the reference host code; the
        # pair arithmetic may be fused (FMA) on the device
        np.testing.assert_allclose(v, ref, rtol=2e-5, atol=2e-5 * np.abs(ref).max(), err_msg=k)


@pytest.mark.parametrize("name", SYSTEMS)
def test_update_noise_bit_exact(golden, name):
    p = params(golden, name)
    for sp in "bs":
        rr = dev(golden[name + "_r" + sp])
        raw = rr.clone()
        B.update_ermak_noise(sp, rr, raw, dev(golden[name + "_ff_" + sp]), dev(golden[name + "_noise_" + sp]), p)
        np.testing.assert_array_equal(host(rr), golden[name + "_upd_rr_" + sp])
        np.testing.assert_array_equal(host(raw), golden[name + "_upd_raw_" + sp])


@pytest.mark.parametrize("name", SYSTEMS)
def test_gder_counts_exact(golden, name):
    import torch
    p = params(golden, name)
    rb, rs = dev(golden[name + "_rb"]), dev(golden[name + "_rs"])
    for pair, (a, b, ra, rbb) in zip(("bb", "bs", "sb", "ss"), (("b", "b", rb, rb), ("b", "s", rb, rs),
                                                               ("s", "b", rs, rb), ("s", "s", rs, rs))):
        counts = torch.zeros(p.nbins_gder, dtype=torch.int64, device="cuda:0")
        B.get_gder(a, b, ra, rbb, counts, p)
        np.testing.assert_array_equal(host(counts).astype(np.float64), golden[name + "_gder_" + pair], err_msg=pair)


def test_gder_counts_exact_larger_system():
    import torch
    nb = ns = 2000
    side = CF.side_from_phi(nb, ns, 0.5)
    pos = CF.lattice_config(nb, ns, side, 5)
    p = O.setup_params(side, nb, ns, float(CF.SIGMA_BIG), float(CF.SIGMA_SML), nbins=300, rng=side / 2)
    ref = O.gder_counts(p, pos[:nb], pos[nb:])
    pp = B.Parametros.from_buffer_copy(bytes(p))
    rb, rs = dev(pos[:nb]), dev(pos[nb:])
    for k, (a, b, ra, rbb) in enumerate((("b", "b", rb, rb), ("b", "s", rb, rs), ("s", "b", rs, rb),
                                         ("s", "s", rs, rs))):
        counts = torch.zeros(300, dtype=torch.int64, device="cuda:0")
        B.get_gder(a, b, ra, rbb, counts, pp)
        np.testing.assert_array_equal(host(counts).astype(np.uint64), ref[k])


def test_fself_and_msd(golden):
    raw, r0 = golden["g1_fself_raw_b"], golden["g1_rb"]
    fs = np.zeros(4, np.float32)
    B.fself_isotropic(dev(raw), dev(r0), len(r0), fs, 2, np.float32(7.0))
    np.testing.assert_allclose(fs, golden["g1_fself"], rtol=2e-6, atol=2e-7)
    m = B.msd(dev(raw), dev(r0), len(r0))
    assert abs(m - O.oracle_lib().or_ref_msd(raw, r0, len(r0))) < 1e-5 * m


def test_cell_overflow_is_reported_not_written_out_of_bounds():
    import torch
    nb, ns = 64, 64
    side = CF.side_from_phi(nb, ns, 0.3)
    p = B.setup_params(side, nb, ns, float(CF.SIGMA_BIG), float(CF.SIGMA_SML), ntags_big=2, ntags_sml=2)
    rr = np.full((nb, 3), 0.1, np.float32)  # every big particle in cell 0
    nocup = torch.zeros(p.ncell_big ** 3, dtype=torch.int32, device="cuda:0")
    guard = torch.full((p.ncell_big ** 3 * 2 + 64,), -7, dtype=torch.int32, device="cuda:0")
    cell = guard[: p.ncell_big ** 3 * 2]
    with pytest.raises(B.BDError) as ei:
        B.cell_locate("b", dev(rr), nocup, cell, p)
    assert ei.value.code == 3
    assert (host(guard)[p.ncell_big ** 3 * 2:] == -7).all()


def test_invalid_species_rejected():
    p = B.setup_params(10.0, 10, 10, 1.5, 1.1)
    with pytest.raises(B.BDError):
        B.cell_locate("x", None, None, None, p)
