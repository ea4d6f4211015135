"""The engine with the other pair potentials of potentials.cu (standard WCA,
WCA 49-50, 49-50 + Asakura-Oosawa depletion, HSAY): energies and virial
against the oracle's all-pairs forces, one injected-noise step against the
oracle update (sweep path), the list path against the sweep path, and the
per-replica list launch against the per-step one."""
import numpy as np
import pytest

from bd_aging_b200 import configs as CF
from bd_aging_b200 import lib as B
from oracle import oracle as O

pytestmark = pytest.mark.gpu
SB, SS = float(CF.SIGMA_BIG), float(CF.SIGMA_SML)
CASES = [("wca", (0, 0, 0, 0)), ("wca49_50", (1.4, 0.8, 0, 0)), ("ao", (1.0, 0.9, 2.0, 0.2)),
         ("hsay", (2.0, 1.6, 0, 0))]
_RELAXED = {}


def relaxed(nb, ns, side, seed):
    """Lattice start relaxed by capped modified-WCA steps: no core overlaps, so
    the stiff 49-50 cores give moderate forces."""
    key = (nb, ns, side, seed)
    if key not in _RELAXED:
        s = B.System(n_big=nb, n_sml=ns, side=side, sigma_big=SB, sigma_sml=SS, dt=1e-4, seed=seed, T0=0.2,
                     protocol="const", force_cap=100.0)
        e = B.Engine([s], rng_stream=1)
        e.set_positions(CF.lattice_config(nb, ns, side, seed))
        e.run(600)
        _RELAXED[key] = e.get_positions()[0]
        e.close()
    return _RELAXED[key].copy()


def system(pot, pp, nb=1500, ns=1500, phi=0.3, seed=3, **kw):
    # phi = 0.3: the long AO / HSAY cut distances make large cells (capacity 24)
    side = float(np.float32(CF.side_from_phi(nb, ns, phi)))
    pos = relaxed(nb, ns, side, seed)
    s = B.System(n_big=nb, n_sml=ns, side=side, sigma_big=SB, sigma_sml=SS, dt=1e-5, seed=seed, T0=0.5,
                 protocol="const", potential=pot, pot_param=pp, **kw)
    return s, pos


def types_of(s):
    return np.array([0] * s.n_big + [1] * s.n_sml, np.int32)


@pytest.mark.parametrize("pot,pp", CASES)
def test_energy_and_virial_match_oracle(pot, pp):
    s, pos = system(pot, pp)
    e = B.Engine([s])
    e.set_positions(pos)
    ob = e.observe()[0]
    _, u, vir = O.eng_forces_pot(pos, types_of(s), s.side, SB, SS, pot, pp)
    u = u.astype(np.float64)
    assert ob["energy_big"] == pytest.approx(0.5 * u[:s.n_big].sum() / s.n_big, rel=1e-4, abs=1e-6)
    assert ob["energy_sml"] == pytest.approx(0.5 * u[s.n_big:].sum() / s.n_sml, rel=1e-4, abs=1e-6)
    assert ob["virial"] == pytest.approx(vir.astype(np.float64).sum(), rel=1e-4, abs=1e-3)


@pytest.mark.parametrize("pot,pp", CASES)
def test_injected_noise_step_matches_oracle(pot, pp):
    s, pos = system(pot, pp)
    e = B.Engine([s], rng="noise")
    e.set_positions(pos)
    noise = np.random.default_rng(2).standard_normal((s.n, 3)).astype(np.float32)
    e.set_noise(noise)
    e.run(1)
    hi, _ = e.get_positions()
    ff, _, _ = O.eng_forces_pot(pos, types_of(s), s.side, SB, SS, pot, pp)
    L = O.oracle_lib()
    mob = np.array([np.float32(1) / np.float32(SB), np.float32(1) / np.float32(SS)], np.float32)
    amp = np.array([L.or_eng_amplitude(0.5, float(mob[0]), np.float32(s.dt)),
                    L.or_eng_amplitude(0.5, float(mob[1]), np.float32(s.dt))], np.float32)
    ohi, olo, odsp = pos.copy(), np.zeros_like(pos), np.zeros(pos.shape, np.float64)
    L.or_eng_update(s.n, ohi, olo, odsp, ff, types_of(s), s.side, s.dt, mob, amp, noise)
    d = np.abs(hi - ohi)
    d = np.minimum(d, s.side - d)
    assert d.max() < 5e-6, d.max()


@pytest.mark.parametrize("pot,pp", CASES)
def test_list_path_tracks_sweep_path(pot, pp):
    s, pos = system(pot, pp)
    out = []
    for skin in (0.0, 0.25):
        e = B.Engine([s], neighbor_skin=skin)
        e.set_positions(pos)
        e.run(50)
        out.append(e.get_positions()[0])
    d = np.abs(out[0] - out[1])
    d = np.minimum(d, s.side - d)
    assert d.max() < 1e-4, d.max()


def test_per_replica_launch_matches_per_step_launch_across_potentials():
    """The per-replica launch variants (3 and 5: one block per replica that
    runs a whole graph batch and rebuilds its replica's lists itself) on a
    batch mixing potentials (the kernels' EXTRA instantiation) and a
    capped-force replica: the same bits, the same census and the same rebuild
    counts as the per-step kernels (variant 0), over 300 steps with
    rebuilds."""
    specs = [("wca_modified", (0, 0, 0, 0), 0.0), ("ao", (1.0, 0.9, 2.0, 0.2), 0.0), ("hsay", (2.0, 1.6, 0, 0), 0.0),
             ("wca", (0, 0, 0, 0), 100.0)]
    systems, poss = [], []
    for k, (pot, pp, cap) in enumerate(specs):
        nb = ns = 1500
        side = float(np.float32(CF.side_from_phi(nb, ns, 0.3)))
        poss.append(relaxed(nb, ns, side, 20 + k))
        systems.append(B.System(n_big=nb, n_sml=ns, side=side, sigma_big=SB, sigma_sml=SS, dt=4e-5, seed=20 + k,
                                T0=1.0, protocol="const", potential=pot, pot_param=pp, force_cap=cap))
    pos = np.concatenate(poss)
    out = {}
    for v in (0, 3, 5):
        e = B.Engine(systems, list_variant=v)
        e.set_positions(pos)
        e.run(300)  # three 96-step graphs and 12 single steps
        info = e.info()
        out[v] = (e.get_positions(), e.census(), (info.list_builds, info.list_rebuild_steps))
        e.close()
    (hi0, raw0), (cnt0, hsh0), builds0 = out[0]
    assert builds0[0] > len(systems) and builds0[1] > 1, builds0  # lists were rebuilt during the run
    for v in (3, 5):
        (hi, raw), (cnt, hsh), builds = out[v]
        np.testing.assert_array_equal(hi, hi0, err_msg="variant %d" % v)
        np.testing.assert_array_equal(raw, raw0, err_msg="variant %d" % v)
        np.testing.assert_array_equal(cnt, cnt0)
        np.testing.assert_array_equal(hsh, hsh0)
        assert builds == builds0, (v, builds, builds0)
