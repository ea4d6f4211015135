"""Precision of the engine's arithmetic (FP32 forces, FP32 + compensated
positions, FP64 displacements and reductions) against an FP64 host run of
the same dynamics with the same Philox noise, over 10^3 steps; the run at
the reference's precision (FP32 positions and unwrapped positions) is
measured beside it."""
import numpy as np
import pytest

from bd_aging_b200 import configs as CF
from bd_aging_b200 import lib as B
from oracle import oracle as O

pytestmark = pytest.mark.gpu
SB, SS = float(CF.SIGMA_BIG), float(CF.SIGMA_SML)


def precision_case(nb, ns, phi, steps=1000, temp=0.1, dt=1e-5, seed=5, q=7.0):
    side = float(np.float32(CF.side_from_phi(nb, ns, phi)))
    relax = B.System(n_big=nb, n_sml=ns, side=side, sigma_big=SB, sigma_sml=SS, dt=1e-4, seed=99, T0=1.0,
                     protocol="const", force_cap=100.0)
    e = B.Engine([relax], rng_stream=1)
    e.set_positions(CF.uniform_config(nb, ns, side, seed))
    e.run(1500)
    pos, _ = e.get_positions()
    e.close()
    s = B.System(n_big=nb, n_sml=ns, side=side, sigma_big=SB, sigma_sml=SS, dt=dt, seed=seed, T0=temp,
                 protocol="const")
    e = B.Engine([s], qmax=q)
    e.set_positions(pos)
    e.run(steps)
    o = e.observe()[0]
    eng = {k: o[k] for k in ("msd_big", "msd_sml", "fself_big", "energy_big", "energy_sml", "virial")}
    e.close()
    mb, ms = float(np.float32(1) / np.float32(SB)), float(np.float32(1) / np.float32(SS))
    args = (pos, nb, side, SB, SS, mb, ms, dt, temp, seed, steps, q)
    f64, _ = O.precision_run("fp64", *args)
    f32, _ = O.precision_run("fp32_reference", *args)
    err = {k: abs(eng[k] - f64[k]) / abs(f64[k]) for k in eng}
    err32 = {k: abs(f32[k] - f64[k]) / abs(f64[k]) for k in eng}
    return eng, f64, err, err32


def test_observables_against_fp64_over_1000_steps():
    eng, f64, err, err32 = precision_case(1024, 1024, 0.58)
    # stated tolerances (relative to the FP64 run)
    assert err["msd_big"] < 1e-4 and err["msd_sml"] < 1e-4, err
    assert err["fself_big"] < 1e-5, err
    assert err["energy_big"] < 1e-4 and err["energy_sml"] < 1e-4, err
    assert err["virial"] < 1e-4, err
    # the compensated positions and FP64 displacements keep the MSD closer to
    # FP64 than FP32 positions with an FP32 unwrapped copy do
    assert err["msd_big"] < err32["msd_big"], (err, err32)
