"""GPU parity of the per-particle rannew64 noise mode (rannew64.cu:55-126
streams, one per particle) against the oracle."""
import numpy as np
import pytest

from bd_aging_b200 import configs as CF
from bd_aging_b200 import lib as B
from oracle import oracle as O

pytestmark = pytest.mark.gpu
SB, SS = float(CF.SIGMA_BIG), float(CF.SIGMA_SML)


def test_rannew64_streams_through_ring_wrap():
    # dilute lattice: no pair inside its cut distance, so every displacement
    # is amp * xi and the FP64 displacement after K steps is the sum of the
    # stream's noise; 70 steps draw 280 uniforms, past the 250-word ring
    nb, ns, steps = 400, 600, 70
    side = float(np.float32(CF.side_from_phi(nb, ns, 0.01)))
    pos = CF.lattice_config(nb, ns, side, 4)
    s = B.System(n_big=nb, n_sml=ns, side=side, sigma_big=SB, sigma_sml=SS, dt=1e-4, seed=77, T0=0.8,
                 protocol="const")
    e = B.Engine([s], rng="rannew64")
    e.set_positions(pos)
    e.run(steps)
    got = e.get_displacements()
    noise = O.rannew64_particle_noise(77, nb + ns, steps)
    L = O.oracle_lib()
    mob = [np.float32(1) / np.float32(SB), np.float32(1) / np.float32(SS)]
    amp = np.array([L.or_eng_amplitude(0.8, float(mob[0]), np.float32(1e-4))] * nb +
                   [L.or_eng_amplitude(0.8, float(mob[1]), np.float32(1e-4))] * ns, np.float32)
    exp = np.zeros((nb + ns, 3), np.float64)
    for k in range(steps):
        exp += (amp[:, None] * noise[k]).astype(np.float32).astype(np.float64)
    # Box-Muller uses logf / sinf / cosf, which may differ from the host's in the last bit
    np.testing.assert_allclose(got, exp, rtol=2e-5, atol=2e-8)
    # a wrong ring pointer would give unrelated noise
    assert np.corrcoef(got.ravel(), exp.ravel())[0, 1] > 0.999999


def test_rannew64_dense_steps_match_oracle():
    nb, ns = 900, 1100
    side = float(np.float32(CF.side_from_phi(nb, ns, 0.5)))
    pos = CF.lattice_config(nb, ns, side, 12)
    s = B.System(n_big=nb, n_sml=ns, side=side, sigma_big=SB, sigma_sml=SS, dt=1e-5, seed=5, T0=0.6,
                 protocol="const")
    e = B.Engine([s], rng="rannew64")
    e.set_positions(pos)
    steps = 3
    noise = O.rannew64_particle_noise(5, nb + ns, steps)
    types = np.array([0] * nb + [1] * ns, np.int32)
    L = O.oracle_lib()
    mob = np.array([np.float32(1) / np.float32(SB), np.float32(1) / np.float32(SS)], np.float32)
    amp = np.array([L.or_eng_amplitude(0.6, float(mob[0]), np.float32(1e-5)),
                    L.or_eng_amplitude(0.6, float(mob[1]), np.float32(1e-5))], np.float32)
    ohi, olo, odsp = pos.copy(), np.zeros_like(pos), np.zeros(pos.shape, np.float64)
    for k in range(steps):
        ff, _, _, _, _ = O.eng_forces(ohi, types, side, SB, SS)
        L.or_eng_update(s.n, ohi, olo, odsp, ff, types, side, s.dt, mob, amp, np.ascontiguousarray(noise[k]))
    e.run(steps)
    hi, _ = e.get_positions()
    d = np.abs(hi - ohi)
    d = np.minimum(d, side - d)
    assert d.max() < 4e-6, d.max()


def test_rannew64_plain_persistent_and_batched_agree():
    specs = [(300, 500, 0.5, 1), (800, 400, 0.45, 2)]
    systems, poss = [], []
    for nb, ns, phi, seed in specs:
        side = float(np.float32(CF.side_from_phi(nb, ns, phi)))
        poss.append(CF.lattice_config(nb, ns, side, seed))
        systems.append(B.System(n_big=nb, n_sml=ns, side=side, sigma_big=SB, sigma_sml=SS, dt=1e-5, seed=seed,
                                T0=1.0, protocol="const"))
    pos = np.concatenate(poss)
    out = []
    for kw in (dict(neighbor_skin=0.0), dict(mode="persistent", cluster=2)):
        e = B.Engine(systems, rng="rannew64", **kw)
        e.set_positions(pos)
        e.run(130)
        out.append(e.get_positions()[0])
    np.testing.assert_array_equal(out[0], out[1])
    e1 = B.Engine([systems[1]], rng="rannew64", neighbor_skin=0.0)
    e1.set_positions(poss[1])
    e1.run(130)
    np.testing.assert_array_equal(e1.get_positions()[0], out[0][systems[0].n:])
