"""Host check (float32 numpy) of the list step's minimum image for boundary
warps (csrc/nlist.cuh, min_image_pair): for a partner within 0.495 L of the
particle, the reference's k = floor(fl(d / L) + 1/2) (get_forces.cu, with
d = x_j - x_i of wrapped coordinates and 1/L a float division) equals
rint(fl(d / L)), so d - L k, with L k exact, is the reference's value.  The
engine keeps list partners within 0.492 L (skin at most 0.9 of the largest
cut, at least three cells of side cut + skin per box side)."""
import numpy as np


def test_rint_image_equals_reference_floor_image():
    rng = np.random.default_rng(17)
    for L in (5.5, 9.35, 12.515, 38.116, 121.01):
        L32 = np.float32(L)
        linv = np.float32(1.0) / L32
        n = 400000
        xi = (rng.uniform(0, 1, n) * L).astype(np.float32)
        off = (rng.uniform(-0.495, 0.495, n) * L).astype(np.float32)
        xj = (xi + off).astype(np.float32)
        xj = np.where(xj >= L32, xj - L32, np.where(xj < 0, xj + L32, xj)).astype(np.float32)
        d = (xj - xi).astype(np.float32)
        t = (linv * d).astype(np.float32)
        k_ref = np.floor((t + np.float32(0.5)).astype(np.float32))
        k_new = np.rint(t)
        np.testing.assert_array_equal(k_ref, k_new)
        img_ref = (d - (L32 * k_ref).astype(np.float32)).astype(np.float32)
        img_new = (d - L32 * k_new.astype(np.float32)).astype(np.float32)
        np.testing.assert_array_equal(img_ref, img_new)
        assert np.abs(img_new).max() <= 0.5 * L


def test_engine_geometry_keeps_partners_within_0492_L():
    """Largest list distance cut + 2 skin against the smallest box the engine
    accepts, 3 (cut + skin), for every skin up to 0.9 of the cut."""
    for cut in (0.5, 1.122462, 1.571447, 3.0):
        for skin in np.linspace(1e-3, 0.9 * cut, 50):
            assert (cut + 2 * skin) / (3 * (cut + skin)) < 0.492
