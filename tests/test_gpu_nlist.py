"""GPU parity of the neighbour-list mode (csrc/nlist.cuh): the interacting
pairs of every particle equal the oracle's all-pairs neighbour sets, also
after many device-triggered rebuilds; one step matches the oracle update
with the engine's Philox noise; list runs are deterministic (batched ==
plain, graph == single steps); observation passes read the current state."""
import numpy as np
import pytest

from bd_aging_b200 import configs as CF
from bd_aging_b200 import lib as B
from oracle import oracle as O

pytestmark = pytest.mark.gpu
SB, SS = float(CF.SIGMA_BIG), float(CF.SIGMA_SML)
SKIN = 0.3


def system(nb, ns, phi, seed, **kw):
    side = float(np.float32(CF.side_from_phi(nb, ns, phi)))
    pos = CF.lattice_config(nb, ns, side, seed)
    s = B.System(n_big=nb, n_sml=ns, side=side, sigma_big=SB, sigma_sml=SS, dt=kw.pop("dt", 1e-4), seed=seed,
                 force_cap=kw.pop("force_cap", 100.0), **kw)
    return s, pos


def types_of(s):
    return np.array([0] * s.n_big + [1] * s.n_sml, np.int32)


@pytest.mark.parametrize("nb,ns,phi,brick", [(150, 150, 0.45, None), (2000, 2000, 0.55, None),
                                             (2000, 2000, 0.55, (8, 4, 2)), (700, 300, 0.5, (3, 5, 2))])
def test_list_neighbour_sets_bit_exact(nb, ns, phi, brick):
    s, pos = system(nb, ns, phi, 21)
    e = B.Engine([s], brick=brick, neighbor_skin=SKIN)
    assert e.info().neighbor_skin == pytest.approx(SKIN)
    e.set_positions(pos)
    cnt, hsh = e.census()
    _, _, _, nbr, h = O.eng_forces(pos, types_of(s), s.side, SB, SS)
    np.testing.assert_array_equal(cnt, nbr)
    np.testing.assert_array_equal(hsh, h)


def test_list_sets_stay_exact_across_rebuilds():
    s, pos = system(1500, 1500, 0.5, 31, T0=1.0)
    e = B.Engine([s], neighbor_skin=SKIN)
    e.set_positions(pos)
    for k in range(3):
        e.run(400)
        hi, _ = e.get_positions()
        cnt, hsh = e.census()
        _, _, _, nbr, h = O.eng_forces(hi, types_of(s), s.side, SB, SS)
        np.testing.assert_array_equal(cnt, nbr)
        np.testing.assert_array_equal(hsh, h)
    assert e.info().list_builds >= 4  # the first build plus device-triggered ones


def test_list_one_step_matches_oracle():
    s, pos = system(1500, 1500, 0.52, 4, T0=0.7, protocol="const", force_cap=0.0, dt=1e-5)
    e = B.Engine([s], neighbor_skin=SKIN)
    e.set_positions(pos)
    e.run(1)
    hi, raw = e.get_positions()
    ff, _, _, _, _ = O.eng_forces(pos, types_of(s), s.side, SB, SS)
    noise = O.eng_gauss3(s.seed, np.arange(s.n), 0).astype(np.float32)
    L = O.oracle_lib()
    mob = np.array([np.float32(1) / np.float32(SB), np.float32(1) / np.float32(SS)], np.float32)
    amp = np.array([L.or_eng_amplitude(0.7, float(mob[0]), np.float32(s.dt)),
                    L.or_eng_amplitude(0.7, float(mob[1]), np.float32(s.dt))], np.float32)
    ohi, olo, odsp = pos.copy(), np.zeros_like(pos), np.zeros(pos.shape, np.float64)
    L.or_eng_update(s.n, ohi, olo, odsp, ff, types_of(s), s.side, s.dt, mob, amp, np.ascontiguousarray(noise))
    d = np.abs(hi - ohi)
    d = np.minimum(d, s.side - d)
    assert d.max() < 2e-5, d.max()


def test_list_batched_equals_plain_and_graph_equals_single_steps():
    specs = [(300, 300, 0.5, 1), (1000, 700, 0.55, 2), (150, 450, 0.45, 3)]
    systems, poss = zip(*[system(*sp, T0=1.0) for sp in specs])
    eb = B.Engine(list(systems), neighbor_skin=SKIN)
    eb.set_positions(np.concatenate(poss))
    eb.run(250)
    pb, rb = eb.get_positions()
    for k, (s, p) in enumerate(zip(systems, poss)):
        e1 = B.Engine([s], neighbor_skin=SKIN)
        e1.set_positions(p)
        for _ in range(5):
            e1.run(50)
        p1, r1 = e1.get_positions()
        sl = slice(eb.offsets[k], eb.offsets[k + 1])
        np.testing.assert_array_equal(pb[sl], p1)
        np.testing.assert_array_equal(rb[sl], r1)
    e2 = B.Engine(list(systems), neighbor_skin=SKIN)
    e2.set_positions(np.concatenate(poss))
    for _ in range(250):
        e2.run(1)
    np.testing.assert_array_equal(e2.get_positions()[0], pb)
    # rebuilds inside graphs (conditional nodes) happen at the same steps as
    # in single-step launches
    ib, i2 = eb.info(), e2.info()
    assert ib.list_rebuild_steps == i2.list_rebuild_steps > 3
    assert ib.list_builds == i2.list_builds


def test_list_graph_rebuilds_only_when_flagged():
    # a cold system whose particles stay within half the skin: one build, and
    # graph runs launch no rebuild bodies; a hot one rebuilds inside graphs
    s, pos = system(800, 800, 0.5, 12, T0=1e-4, protocol="const", dt=1e-6)
    e = B.Engine([s], neighbor_skin=SKIN, graph_steps=96)
    e.set_positions(pos)
    e.run(96 * 3)
    assert e.info().list_rebuild_steps == 1 and e.info().list_builds == 1
    s, pos = system(800, 800, 0.5, 12, T0=2.0, protocol="const", dt=2e-4)
    e = B.Engine([s], neighbor_skin=SKIN, graph_steps=96)
    e.set_positions(pos)
    e.run(96 * 3)
    hot = e.info().list_rebuild_steps
    assert hot > 6
    hi, _ = e.get_positions()
    cnt, hsh = e.census()
    _, _, _, nbr, h = O.eng_forces(hi, types_of(s), s.side, SB, SS)
    np.testing.assert_array_equal(cnt, nbr)
    np.testing.assert_array_equal(hsh, h)


def test_list_observables_match_oracle():
    s, pos = system(1200, 1800, 0.5, 8, T0=0.5)
    e = B.Engine([s], neighbor_skin=SKIN)
    e.set_positions(pos)
    e.run(120)
    ob = e.observe()[0]
    hi, raw = e.get_positions()
    _, pot, vir, _, _ = O.eng_forces(hi, types_of(s), s.side, SB, SS)
    assert ob["energy_big"] == pytest.approx(0.5 * pot[:s.n_big].astype(np.float64).sum() / s.n_big, rel=1e-5)
    assert ob["virial"] == pytest.approx(vir.astype(np.float64).sum(), rel=1e-5)
    d = raw[: s.n_big].astype(np.float64) - pos[: s.n_big]
    assert ob["msd_big"] == pytest.approx((d ** 2).sum(1).mean(), rel=1e-4)
    counts = e.gder(100, 4.0)[0]
    p = O.setup_params(s.side, s.n_big, s.n_sml, SB, SS, nbins=100, rng=4.0)
    np.testing.assert_array_equal(counts, O.gder_counts(p, hi[: s.n_big], hi[s.n_big:]))


def test_single_species_replicas_in_a_batch():
    specs = [(0, 800, 0.45, 41), (600, 0, 0.45, 42), (300, 300, 0.5, 43)]
    systems, poss = zip(*[system(*sp, T0=0.8) for sp in specs])
    e = B.Engine(list(systems))
    e.set_positions(np.concatenate(poss))
    e.reserve_snapshots(1)
    e.snapshot(0)
    e.run(200)
    obs = e.observe()
    c = e.correlate([0], 6.19)[0]
    hi, _ = e.get_positions()
    cnt, hsh = e.census()
    for k, s in enumerate(systems):
        sl = slice(e.offsets[k], e.offsets[k + 1])
        _, _, _, nbr, h = O.eng_forces(hi[sl], types_of(s), s.side, SB, SS)
        np.testing.assert_array_equal(cnt[sl], nbr)
        np.testing.assert_array_equal(hsh[sl], h)
        o = obs[k]
        assert all(np.isfinite(v) for v in o.values())
        if s.n_big == 0:
            assert o["msd_big"] == 0.0 and o["energy_big"] == 0.0 and c[k]["msd_big"] == 0.0
            assert c[k]["msd_sml"] > 0.0
        if s.n_sml == 0:
            assert o["msd_sml"] == 0.0 and c[k]["fself_sml"] == 0.0
            assert c[k]["msd_big"] > 0.0


def test_list_displacement_follows_face_crossings():
    # list mode keeps no per-step displacement: face crossings are counted and
    # the FP64 displacement is rebuilt from them.  Against the host's sum of
    # minimum-image position increments, step by step, in a hot dilute system
    # where many particles cross faces (and some cross back).
    s, pos = system(300, 300, 0.2, 19, T0=6.0, protocol="const", dt=2e-4)
    e = B.Engine([s], neighbor_skin=SKIN)
    assert e.info().neighbor_skin > 0
    e.set_positions(pos)
    prev = pos.astype(np.float64)
    acc = np.zeros_like(prev)
    crossed = np.zeros(prev.shape, bool)
    for _ in range(300):
        e.run(1)
        cur = e.get_positions()[0].astype(np.float64)
        d = cur - prev
        crossed |= np.abs(d) > 0.5 * s.side
        acc += d - s.side * np.round(d / s.side)
        prev = cur
    got = e.get_displacements()
    assert crossed.sum() > 50
    np.testing.assert_allclose(got, acc, rtol=0, atol=2e-5)
    # the unwrapped output is the origin plus the same displacement
    _, raw = e.get_positions()
    np.testing.assert_allclose(raw.astype(np.float64), pos.astype(np.float64) + got, rtol=0, atol=2e-5)


@pytest.mark.parametrize("nb,ns,phi,seed", [(4000, 4000, 0.5, 51), (400, 400, 0.5, 52)])
def test_list_forces_match_oracle_at_zero_temperature(nb, ns, phi, seed):
    # T = 0: one step moves every particle by F mob dt exactly (no noise), and
    # the FP64 displacement recovers that float increment.  Checks the list
    # kernel's pair arithmetic (paired f32x2 lanes, padded lists, warps with
    # and without the minimum image: the large box has interior warps, the
    # small one nearly none) against the oracle's forces.
    s, pos = system(nb, ns, phi, seed, T0=0.0, protocol="const", force_cap=0.0, dt=1e-6)
    # a relaxed start keeps the forces moderate
    e0 = B.Engine([B.System(n_big=nb, n_sml=ns, side=s.side, sigma_big=SB, sigma_sml=SS, dt=1e-5, seed=seed,
                            T0=0.0, protocol="const", force_cap=50.0)])
    e0.set_positions(pos)
    e0.run(200)
    start = e0.get_positions()[0]
    e = B.Engine([s], neighbor_skin=SKIN)
    e.set_positions(start)
    e.run(1)
    d = e.get_displacements()
    ff, _, _, _, _ = O.eng_forces(start, types_of(s), s.side, SB, SS)
    mob = np.where(types_of(s) == 0, np.float32(1) / np.float32(SB), np.float32(1) / np.float32(SS))
    f_eng = d / (mob[:, None].astype(np.float64) * s.dt)
    scale = np.abs(ff).max()
    assert scale > 1.0
    # float rounding of F mob dt and of the force sums (different pair order)
    np.testing.assert_allclose(f_eng, ff.astype(np.float64), rtol=2e-5, atol=2e-5 * scale)


def test_many_replicas_rebuild_only_the_flagged_ones():
    # 40 replicas (the rebuild kernels number the flagged replicas' particles,
    # cells and bricks with a scan over replicas, here over two warp chunks):
    # hot ones rebuild often, cold ones rarely.  Each replica ends bit-identical
    # to its own single-replica run, and every neighbour set is exact.
    temps = [2.0 if k % 3 == 0 else 1e-3 for k in range(40)]
    specs = [(60 + 7 * k, 90 - k, 0.45, 100 + k) for k in range(40)]
    systems, poss = zip(*[system(*sp, T0=t, protocol="const", dt=2e-4) for sp, t in zip(specs, temps)])
    eb = B.Engine(list(systems), neighbor_skin=SKIN)
    eb.set_positions(np.concatenate(poss))
    eb.run(120)
    pb, rb = eb.get_positions()
    assert eb.info().list_builds > 40 + 10  # the first builds plus hot-replica rebuilds
    cnt, hsh = eb.census()
    for k in (0, 1, 17, 39):
        s = systems[k]
        e1 = B.Engine([s], neighbor_skin=SKIN)
        e1.set_positions(poss[k])
        e1.run(120)
        p1, r1 = e1.get_positions()
        sl = slice(eb.offsets[k], eb.offsets[k + 1])
        np.testing.assert_array_equal(pb[sl], p1)
        np.testing.assert_array_equal(rb[sl], r1)
    for k, s in enumerate(systems):
        sl = slice(eb.offsets[k], eb.offsets[k + 1])
        _, _, _, nbr, h = O.eng_forces(pb[sl], types_of(s), s.side, SB, SS)
        np.testing.assert_array_equal(cnt[sl], nbr)
        np.testing.assert_array_equal(hsh[sl], h)


def test_more_replicas_than_the_rebuild_scheduler_takes():
    # above 1024 replicas the rebuild kernels walk every particle, cell and
    # brick instead of numbering the flagged ones; the lists must be the same
    nrep = 1030
    temps = [2.0 if k % 5 == 0 else 1e-3 for k in range(nrep)]
    systems, poss = zip(*[system(80, 80, 0.3, 500 + k, T0=t, protocol="const", dt=2e-4)
                          for k, t in enumerate(temps)])
    eb = B.Engine(list(systems), neighbor_skin=SKIN)
    eb.set_positions(np.concatenate(poss))
    eb.run(60)
    pb, _ = eb.get_positions()
    assert eb.info().list_builds > nrep + 20
    cnt, hsh = eb.census()
    for k in list(range(0, nrep, 97)) + [nrep - 1]:
        s = systems[k]
        sl = slice(eb.offsets[k], eb.offsets[k + 1])
        _, _, _, nbr, h = O.eng_forces(pb[sl], types_of(s), s.side, SB, SS)
        np.testing.assert_array_equal(cnt[sl], nbr)
        np.testing.assert_array_equal(hsh[sl], h)
    for k in (0, 1, nrep - 1):
        e1 = B.Engine([systems[k]], neighbor_skin=SKIN)
        e1.set_positions(poss[k])
        e1.run(60)
        np.testing.assert_array_equal(e1.get_positions()[0], pb[eb.offsets[k]:eb.offsets[k + 1]])
