"""Host check of the list step's interior shortcut (list_forces_wca<false>
in csrc/nlist.cuh), restated in numpy float32.

A warp whose particles all lie at least `interior` = (largest cut + skin) +
skin + 0.01 from every face skips the minimum image.  A list partner was
within cut + skin at the build, and each end has moved at most skin/2 since,
so the partner's stored (wrapped) coordinate lies in the same image.  The
plain float difference is then what the reference's minimum image
(get_forces.cu:389-391, float) returns, and the zero position that list
padding gathers lies beyond every cut distance.  Checked on random particles,
partners and boxes, including partners placed at the largest allowed
distance."""
import numpy as np
import pytest

F = np.float32


def min_image_ref(d, L, Linv):
    """d - L floor(Linv d + 0.5), every operation rounded to float."""
    t = (Linv * d).astype(F)
    return (d - (L * np.floor((t + F(0.5)).astype(F))).astype(F)).astype(F)


@pytest.mark.parametrize("L,rcmax,skin", [(30.3, 1.5714, 0.25), (8.0, 1.5714, 0.25), (12.0, 1.8, 0.4),
                                           (100.0, 1.1225, 0.25)])
def test_interior_partners_need_no_minimum_image(L, rcmax, skin):
    L = F(L)
    Linv = F(1.0) / L
    interior = F(rcmax + 2.0 * skin + 0.01)
    if L - interior <= interior:
        pytest.skip("no interior region in this box")
    g = np.random.default_rng(int(L * 10))
    n = 400000
    pi = (interior + g.random((n, 3)) * (L - 2 * interior)).astype(F)
    # partner displacement: uniform direction, length up to the largest
    # distance a list partner can reach (cut + skin + skin), 10% at the limit
    dirs = g.normal(size=(n, 3))
    dirs /= np.linalg.norm(dirs, axis=1)[:, None]
    r = (rcmax + 2 * skin) * np.where(g.random(n) < 0.1, 1.0, g.random(n) ** (1 / 3))
    pj_true = pi.astype(np.float64) + dirs * r[:, None]
    pj = np.mod(pj_true, float(L)).astype(F)  # stored coordinates are wrapped into the box
    d = (pj - pi).astype(F)
    np.testing.assert_array_equal(min_image_ref(d, L, Linv), d)
    # and the plain difference is the true one (no wrap happened)
    np.testing.assert_allclose(d, (pj_true - pi).astype(F), atol=1e-5)
    # padding entries gather the zero position: from an interior particle it
    # is farther than every cut distance, so they need no index test there
    d0 = (F(0) - pi).astype(F)
    d2 = ((d0[:, 0] * d0[:, 0]).astype(F) + (d0[:, 1] * d0[:, 1]).astype(F)).astype(F) + (d0[:, 2] * d0[:, 2]).astype(F)
    assert np.all(d2.astype(F) >= F(rcmax) ** 2)
