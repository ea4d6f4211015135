"""Host check of the g(r) threshold binning (gr_bin_thr / k_gr_thresholds in
csrc/common.cuh and csrc/engine.cu), restated in numpy float32.

The reference bins a pair at (int)(sqrt(d2) / bin_size), both correctly
rounded, when sqrt(d2) < range, and puts a bin equal to nbins in the last bin
(get_gder.cu:116-121).  The kernels instead look the bin up in a table of the
smallest d2 reaching each bin, found by bisection over float bit patterns,
starting from an estimate that may be off by one.  Here the same bisection
and lookup run on the host: estimates a few ulp off (as an approximate
reciprocal square root gives) must still land in the reference's bin, for
d2 spread over the range and packed around every threshold."""
import numpy as np
import pytest

F = np.float32


def ref_bin(d2, rng, nbins):
    """The reference rule, -1 outside the range."""
    bs = F(rng) / F(nbins)
    dist = np.sqrt(d2.astype(F))
    b = (dist / bs).astype(F).astype(np.int64)
    b = np.where(b == nbins, nbins - 1, b)
    return np.where(dist < F(rng), b, -1)


def thresholds(rng, nbins):
    """thr[k] = smallest float d2 with bin >= k (k = 1..nbins), thr[nbins+1] = smallest with sqrt >= range."""
    bs = F(rng) / F(nbins)
    thr = np.zeros(nbins + 2, F)

    def raw(x):
        return int(np.float32(np.sqrt(F(x)) / bs))

    for k in range(1, nbins + 2):
        lo, hi = 0, 0x7F800000
        while lo < hi:
            mid = lo + (hi - lo) // 2
            x = np.array([mid], np.uint32).view(F)[0]
            reach = raw(x) >= k if k <= nbins else not (np.sqrt(F(x)) < F(rng))
            if reach:
                hi = mid
            else:
                lo = mid + 1
        thr[k] = np.array([lo], np.uint32).view(F)[0]
    return thr


def thr_bin(d2, thr, rng, nbins, ulps):
    """gr_bin_thr with the estimate's square root perturbed by `ulps` ulp."""
    inv_bs = F(1.0) / (F(rng) / F(nbins))
    r = np.sqrt(d2.astype(np.float64)).astype(F)
    r = np.nextafter(r, np.where(ulps > 0, np.inf, -np.inf).astype(F)) if np.any(ulps) else r
    for _ in range(int(np.abs(ulps).max()) - 1 if np.any(ulps) else 0):
        r = np.nextafter(r, np.where(ulps > 0, np.inf, -np.inf).astype(F))
    b = np.maximum(F(0), (r * inv_bs).astype(F)).astype(np.int64)
    b = np.minimum(b, nbins)
    up = (b < nbins) & (d2 >= thr[np.minimum(b + 1, nbins + 1)])
    down = ~up & (b > 0) & (d2 < thr[b])
    b = b + up - down
    b = np.minimum(b, nbins - 1)
    return np.where(d2 < thr[nbins + 1], b, -1)


@pytest.mark.parametrize("rng,nbins", [(15.0, 400), (3.0, 300), (2.5, 64), (5.0, 200)])
def test_threshold_bins_equal_the_reference_rule(rng, nbins):
    thr = thresholds(rng, nbins)
    # the bin thresholds are monotone; the range threshold may sit below the
    # last one (a d2 whose bin would round to nbins is out of range first)
    assert np.all(np.diff(thr[1:nbins + 1]) >= 0)
    g = np.random.default_rng(nbins)
    uniform = (g.random(200000) * (1.05 * rng) ** 2).astype(F)
    # every threshold and its float neighbours, where one ulp moves the bin
    edges = thr[1:].view(np.uint32).astype(np.int64)
    near = (edges[:, None] + np.arange(-3, 4)[None, :]).ravel()
    near = near[(near >= 0) & (near < 0x7F800000)].astype(np.uint32).view(F)
    d2 = np.concatenate([uniform, near, np.array([0.0], F)])
    want = ref_bin(d2, rng, nbins)
    for ulps in (0, 2, -2, 4, -4):
        got = thr_bin(d2, thr, rng, nbins, np.full(d2.shape, ulps))
        np.testing.assert_array_equal(got, want, err_msg=f"estimate off by {ulps} ulp")
