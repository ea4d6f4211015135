"""Cell-bounded g(r) (gder.cu) against the oracle's restatement of
get_gder.cu and against the engine's all-pairs kernel: exact integer counts."""
import numpy as np
import pytest

from bd_aging_b200 import configs as CF
from bd_aging_b200 import lib as B
from oracle import oracle as O

pytestmark = pytest.mark.gpu
SB, SS = float(CF.SIGMA_BIG), float(CF.SIGMA_SML)


def system(nb, ns, phi, seed, force_cap=0.0):
    side = float(np.float32(CF.side_from_phi(nb, ns, phi)))
    pos = CF.lattice_config(nb, ns, side, seed)
    return B.System(n_big=nb, n_sml=ns, side=side, sigma_big=SB, sigma_sml=SS, dt=1e-4, seed=seed, T0=1.0,
                    force_cap=force_cap), pos


@pytest.mark.parametrize("nb,ns,phi,nbins,range_", [(3000, 3000, 0.5, 120, 4.0), (5000, 2000, 0.58, 64, 2.5),
                                                    (2500, 4000, 0.45, 200, 5.0)])
def test_cells_match_oracle(nb, ns, phi, nbins, range_):
    # no force cap: the lattice start blows up, and particles of the blown-up
    # state that sit outside their cells send the replica to the all-pairs kernel
    s, pos = system(nb, ns, phi, 3)
    e = B.Engine([s])
    e.set_positions(pos)
    e.run(50)  # off the lattice
    got = e.gder(nbins, range_, method="cells")[0]
    snap, _ = e.get_positions()
    p = O.setup_params(s.side, s.n_big, s.n_sml, SB, SS, nbins=nbins, rng=range_)
    ref = O.gder_counts(p, snap[: s.n_big], snap[s.n_big:])
    np.testing.assert_array_equal(got, ref)
    assert got.sum() > 0


def test_cells_on_a_relaxed_state_match_oracle():
    s, pos = system(4000, 4000, 0.55, 8, force_cap=100.0)
    e = B.Engine([s])
    e.set_positions(pos)
    e.run(300)
    snap, _ = e.get_positions()
    assert np.all((snap >= 0) & (snap <= np.float32(s.side)))
    got = e.gder(150, 5.0, method="cells")[0]
    p = O.setup_params(s.side, s.n_big, s.n_sml, SB, SS, nbins=150, rng=5.0)
    np.testing.assert_array_equal(got, O.gder_counts(p, snap[: s.n_big], snap[s.n_big:]))


def test_cells_equal_all_pairs_on_a_mixed_batch():
    specs = [(20000, 20000, 0.58, 1), (600, 600, 0.5, 2), (12000, 4000, 0.52, 3)]
    systems, poss = zip(*[system(*sp, force_cap=100.0) for sp in specs])
    e = B.Engine(list(systems))
    e.set_positions(np.concatenate(poss))
    e.run(30)
    for nbins, range_ in ((200, 6.0), (97, 3.3)):
        auto = e.gder(nbins, range_)  # large replicas on cells, the small one on all pairs
        ref = e.gder(nbins, range_, method="all_pairs")
        np.testing.assert_array_equal(auto, ref)
    with pytest.raises(B.BDError) as ei:
        e.gder(100, 6.0, method="cells")  # the 1200-particle box is too small for that reach
    assert ei.value.code == B.BD_ERR_ARG


def test_cells_equal_all_pairs_at_quarter_million():
    s, pos = system(131072, 131072, 0.58, 9, force_cap=100.0)
    e = B.Engine([s])
    e.set_positions(pos)
    e.run(20)
    a = e.gder(400, 15.0, method="cells")
    b = e.gder(400, 15.0, method="all_pairs")
    np.testing.assert_array_equal(a, b)
    # every particle sees its own neighbourhood: bs and sb counts match
    np.testing.assert_array_equal(a[0, 1].sum(), a[0, 2].sum())


@pytest.mark.parametrize("method", ["cells", "all_pairs"])
def test_bin_edges_on_a_lattice_match_oracle(method):
    # A simple cubic lattice of spacing 0.5 (every coordinate exact in float):
    # distances 0.5 sqrt(n) put many pairs exactly on edges of the 0.01-wide
    # bins (n a perfect square) and the rest anywhere, so the bin rounding of
    # the reference (sqrt, then divide, both correctly rounded) is checked
    # where a one-ulp slip would move a count to the next bin.
    k = 24
    side = 0.5 * k
    g = (np.arange(k, dtype=np.float32) * np.float32(0.5)) + np.float32(0.25)
    pos = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3).astype(np.float32)
    nb = len(pos) // 2
    s = B.System(n_big=nb, n_sml=len(pos) - nb, side=side, sigma_big=0.3, sigma_sml=0.2, dt=1e-6, seed=1,
                 T0=0.0, protocol="const")
    e = B.Engine([s], neighbor_skin=0.0)
    e.set_positions(pos)
    nbins, range_ = 300, 3.0
    got = e.gder(nbins, range_, method=method)[0]
    snap, _ = e.get_positions()
    np.testing.assert_array_equal(snap, pos)
    p = O.setup_params(side, s.n_big, s.n_sml, 0.3, 0.2, nbins=nbins, rng=range_)
    ref = O.gder_counts(p, snap[: s.n_big], snap[s.n_big:])
    np.testing.assert_array_equal(got, ref)
    assert got.sum() > 0
