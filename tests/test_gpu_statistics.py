"""Long-run statistical agreement with the reference: MSD (both species), F_s
(big particles) and g(r) of the engine against the reference's own CUDA
build (oracle/_ref, built from the reference sources), K = 8 independent
noise seeds each from the same 8 relaxed start states, at the conditions of
BASELINE config 1 (N = 1000, phi = 0.50, T = 1, dt = 2e-5, 10^4 steps) and
config 2 (N = 32768, phi = 0.58, quench T 1.0 -> 0.1, dt = 1e-5, 2000 steps).

Agreement means: at every sampled time, |mean_engine - mean_reference| is
below 3 standard errors of the difference, the standard errors taken from
the seed-to-seed spread of each side (oracle/statistics.py); g(r) per bin the
same way, with the mean of z^2 over the bins below 2 (1 is expected when the
two agree) and the first-peak heights within the same 3-sigma bound."""
import pytest

from oracle import oracle as O
from oracle import statistics as ST

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not O.ref_available(), reason="reference build (oracle/_ref) not present")]


@pytest.mark.parametrize("case", [ST.SMALL, ST.AGING], ids=["config1", "config2"])
def test_observables_agree_with_reference_within_error_bars(case):
    r = ST.run(case, seeds=8)
    for o, v in r["observables"].items():
        for j, z in enumerate(v["z"]):
            assert abs(z) < 3.0, "%s at t=%g: engine %g, reference %g, se %g (z %.2f)" % (
                o, r["times"][j], v["engine"][j], v["reference"][j], v["se"][j], z)
    g = r["gder"]
    assert g["bins_compared"] > case.nbins // 2
    assert g["mean_z2"] < 2.0, g
    assert max(abs(z) for z in g["peak_z"]) < 3.0, g
    # the observables moved: the comparison is not between two unchanged states
    assert r["observables"]["msd_big"]["engine"][-1] > 10 * r["observables"]["msd_big"]["se"][-1]
    assert r["observables"]["fself_big"]["engine"][-1] < 0.999
