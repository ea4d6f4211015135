"""GPU parity: Contracting_Vector3D against the reference's golden vectors and
the oracle, and a 1000-step trajectory of the engine in the reference's
cuRAND stream against the reference's own CUDA kernels (oracle/_ref, built
from the reference sources) on the same device."""
import ctypes as C

import numpy as np
import pytest

from bd_aging_b200 import configs as CF
from bd_aging_b200 import lib as B
from oracle import oracle as O

pytestmark = pytest.mark.gpu
SB, SS = float(CF.SIGMA_BIG), float(CF.SIGMA_SML)


def dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda:0")


@pytest.mark.parametrize("k", [0, 1])
def test_cv3d_matches_reference_golden(golden, k):
    pos, xx = golden["cv3d_pos"], golden["cv3d_xx"]
    side = float(golden["cv3d_side"][0]) if k == 0 else None
    cv = B.Contracting_Vector3D(16, 3.0)
    cv.add_statistics(dev(pos), dev(xx), len(pos), side)
    cv.add_statistics(dev(pos[::-1].copy()), dev(xx), len(pos), side)
    cv.calculate_vector()
    vec = cv.get_vector()
    ref = golden["cv3d_%d_vec" % k]
    np.testing.assert_allclose(vec, ref, rtol=2e-3, atol=2e-3 * np.abs(ref).max())


def test_cv3d_fp64_normal_equations_against_oracle():
    rng = np.random.default_rng(5)
    nb = ns = 600
    side = CF.side_from_phi(nb, ns, 0.5)
    pos = CF.lattice_config(nb, ns, side, 5)
    xx = rng.standard_normal((nb + ns, 3)).astype(np.float32)
    ata, atb, bad = O.cv3d_add(24, 3.5, pos, xx, side)
    assert bad == 0
    ref = O.cv3d_solve(ata.astype(np.float64), atb.astype(np.float64), dtype=np.float64)
    cv = B.Contracting_Vector3D(24, 3.5)
    cv.add_statistics(dev(pos), dev(xx), len(pos), side)
    cv.calculate_vector()
    np.testing.assert_allclose(cv.get_vector(), ref, rtol=1e-3, atol=1e-3 * np.abs(ref).max())


def test_cv3d_state_errors_replace_reference_throws():
    cv = B.Contracting_Vector3D(8, 2.0)
    with pytest.raises(B.BDError) as e1:
        cv.calculate_vector()  # Contracting_Vector3D.cu:168-169 throws
    assert e1.value.code == 5
    with pytest.raises(B.BDError) as e2:
        cv.get_vector()  # Contracting_Vector3D.cu:300-301 throws
    assert e2.value.code == 5


@pytest.mark.skipif(not O.ref_available(), reason="reference build (oracle/_ref) not present")
def test_trajectory_against_reference_cuda_kernels():
    nb = ns = 500
    side = float(np.float32(CF.side_from_phi(nb, ns, 0.5)))
    pos = CF.lattice_config(nb, ns, side, 3, jitter=0.1)
    idum, dt, steps = 12345, 1e-5, 1000
    p = O.setup_params(side, nb, ns, SB, SS, ntags=(16, 16), nbins=100, rng=side / 2, dt=dt, T0=1.0)
    ob, os_ = np.zeros((nb, 3), np.float32), np.zeros((ns, 3), np.float32)
    wb, ws = np.zeros_like(ob), np.zeros_like(os_)
    ms = C.c_float(0)
    rc = O.ref_lib().ref_cuda_run(C.byref(p), pos[:nb].copy(), pos[nb:].copy(), 0, steps, idum, 1.0, 1.0, 0.0, 1.0,
                                  dt, ob, os_, wb, ws, C.byref(ms))
    assert rc == 0
    s = B.System(n_big=nb, n_sml=ns, side=side, sigma_big=SB, sigma_sml=SS, dt=dt, T0=1.0, Tf=1.0, t0=0.0, tf=1.0,
                 protocol="linear", seed=idum)
    e = B.Engine([s], rng="curand")
    e.set_positions(pos)
    e.run(steps)
    hi, raw = e.get_positions()
    ref = np.concatenate([ob, os_])
    d = np.abs(hi - ref)
    d = np.minimum(d, side - d)
    # same noise stream; differences come from float rounding only: the
    # reference accumulates positions in float, the engine carries a
    # compensated remainder, and force sums run in another order
    assert d.max() < 1e-3, d.max()
    assert d.mean() < 5e-5, d.mean()
    draw = np.abs(raw - np.concatenate([wb, ws]))
    assert draw.max() < 1e-3 and draw.mean() < 5e-5
    # the motion itself is far larger than the disagreement
    assert np.abs(raw - pos).mean() > 100 * draw.mean()
