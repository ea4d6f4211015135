"""GPU parity of the batched replica engine against the oracle: neighbour
sets (exact), one step with injected noise, observables, g(r) counts (exact),
batched == plain bit identity, error paths."""
import numpy as np
import pytest

from bd_aging_b200 import configs as CF
from bd_aging_b200 import lib as B
from oracle import oracle as O

pytestmark = pytest.mark.gpu
SB, SS = float(CF.SIGMA_BIG), float(CF.SIGMA_SML)


def system(nb, ns, phi, seed, **kw):
    side = float(np.float32(CF.side_from_phi(nb, ns, phi)))
    pos = CF.lattice_config(nb, ns, side, seed)
    s = B.System(n_big=nb, n_sml=ns, side=side, sigma_big=SB, sigma_sml=SS, dt=kw.pop("dt", 1e-4), seed=seed, **kw)
    return s, pos


def types_of(s):
    return np.array([0] * s.n_big + [1] * s.n_sml, np.int32)


@pytest.mark.parametrize("nb,ns,phi,brick", [(150, 150, 0.45, None), (60, 240, 0.30, (2, 2, 2)),
                                             (2000, 2000, 0.55, None), (2000, 2000, 0.55, (8, 4, 2)),
                                             (700, 300, 0.5, (3, 5, 2))])
def test_neighbour_sets_bit_exact(nb, ns, phi, brick):
    s, pos = system(nb, ns, phi, 21)
    e = B.Engine([s], brick=brick)
    e.set_positions(pos)
    cnt, hsh = e.census()
    _, _, _, nbr, h = O.eng_forces(pos, types_of(s), s.side, SB, SS)
    np.testing.assert_array_equal(cnt, nbr)
    np.testing.assert_array_equal(hsh, h)
    e.close()


def test_one_step_with_injected_noise_matches_oracle():
    s, pos = system(1500, 1500, 0.52, 4, T0=0.7)
    e = B.Engine([s], rng="noise")
    e.set_positions(pos)
    noise = np.random.default_rng(9).standard_normal((s.n, 3)).astype(np.float32)
    e.set_noise(noise)
    e.run(1)
    hi, raw = e.get_positions()
    ff, _, _, _, _ = O.eng_forces(pos, types_of(s), s.side, SB, SS)
    mob = np.array([np.float32(1) / np.float32(SB), np.float32(1) / np.float32(SS)], np.float32)
    L = O.oracle_lib()
    amp = np.array([L.or_eng_amplitude(0.7, float(mob[0]), np.float32(s.dt)),
                    L.or_eng_amplitude(0.7, float(mob[1]), np.float32(s.dt))], np.float32)
    ohi, olo, odsp = pos.copy(), np.zeros_like(pos), np.zeros(pos.shape, np.float64)
    L.or_eng_update(s.n, ohi, olo, odsp, ff, types_of(s), s.side, s.dt, mob, amp, noise)
    # forces are summed in another order (cells vs index), so positions agree
    # to float rounding of the drift term
    d = np.abs(hi - ohi)
    d = np.minimum(d, s.side - d)
    assert d.max() < 2e-6, d.max()
    np.testing.assert_allclose(raw, (pos.astype(np.float64) + odsp).astype(np.float32), atol=2e-6)


def test_observables_match_oracle():
    s, pos = system(1200, 1800, 0.5, 8, T0=0.5)
    e = B.Engine([s])
    e.set_positions(pos)
    ob = e.observe()[0]
    _, pot, vir, _, _ = O.eng_forces(pos, types_of(s), s.side, SB, SS)
    assert ob["energy_big"] == pytest.approx(0.5 * pot[:s.n_big].astype(np.float64).sum() / s.n_big, rel=1e-5)
    assert ob["energy_sml"] == pytest.approx(0.5 * pot[s.n_big:].astype(np.float64).sum() / s.n_sml, rel=1e-5)
    assert ob["virial"] == pytest.approx(vir.astype(np.float64).sum(), rel=1e-5)
    assert ob["msd_big"] == 0.0 and ob["fself_big"] == 1.0
    # after steps: MSD/F_s from the FP64 displacement equal the raw positions'
    e.run(50)
    ob = e.observe()[0]
    _, raw = e.get_positions()
    d = raw[: s.n_big].astype(np.float64) - pos[: s.n_big]
    assert ob["msd_big"] == pytest.approx((d ** 2).sum(1).mean(), rel=1e-4)


def test_gder_counts_exact_against_oracle():
    s, pos = system(900, 1100, 0.5, 13)
    e = B.Engine([s])
    e.set_positions(pos)
    nbins, rng_ = 150, s.side / 2
    got = e.gder(nbins, rng_)[0]
    p = O.setup_params(s.side, s.n_big, s.n_sml, SB, SS, nbins=nbins, rng=rng_)
    ref = O.gder_counts(p, pos[: s.n_big], pos[s.n_big:])
    np.testing.assert_array_equal(got, ref)


def test_batched_equals_plain_bit_identical():
    specs = [(300, 300, 0.5, 1), (1000, 700, 0.55, 2), (150, 450, 0.45, 3)]
    systems, poss = zip(*[system(*sp, T0=1.0) for sp in specs])
    eb = B.Engine(list(systems))
    eb.set_positions(np.concatenate(poss))
    eb.run(200)
    pb, rb = eb.get_positions()
    for k, (s, p) in enumerate(zip(systems, poss)):
        e1 = B.Engine([s])
        e1.set_positions(p)
        e1.run(200)
        p1, r1 = e1.get_positions()
        sl = slice(eb.offsets[k], eb.offsets[k + 1])
        np.testing.assert_array_equal(pb[sl], p1)
        np.testing.assert_array_equal(rb[sl], r1)


def test_graph_and_single_steps_agree():
    s, pos = system(800, 800, 0.5, 5)
    e1 = B.Engine([s], graph_steps=96)
    e1.set_positions(pos)
    e1.run(96 + 5)
    e2 = B.Engine([s], graph_steps=96)
    e2.set_positions(pos)
    for _ in range(101):
        e2.run(1)
    np.testing.assert_array_equal(e1.get_positions()[0], e2.get_positions()[0])


def test_cell_capacity_overflow_raises():
    s, pos = system(400, 400, 0.55, 6)
    with pytest.raises(B.BDError) as ei:
        e = B.Engine([s], cell_capacity=1)
        e.set_positions(pos)
        e.run(3)
    assert ei.value.code == 3


def test_set_positions_rejects_positions_outside_the_box():
    # the storage order is computed on the device; a position outside [0, L]
    # or NaN is an argument error that leaves the loaded state as it was
    s, pos = system(500, 500, 0.5, 8)
    e = B.Engine([s])
    e.set_positions(pos)
    before = e.get_positions()[0]
    for bad in (np.nan, -1e-3, s.side * 1.001):
        p2 = pos.copy()
        p2[777, 1] = bad
        with pytest.raises(B.BDError) as ei:
            e.set_positions(p2)
        assert ei.value.code == B.BD_ERR_ARG
    np.testing.assert_array_equal(e.get_positions()[0], before)
    e.run(10)  # still usable


def test_nan_temperature_of_instant_quench_is_reported():
    # t0 == tf == 0 (run-fself.sh:30-31) gives T = NaN at t == 0 in the
    # reference (set_temp.cu:10-11); the next update turns positions into NaN.
    s, pos = system(300, 300, 0.45, 7, T0=1.0, Tf=0.25, t0=0.0, tf=0.0, protocol="linear")
    e = B.Engine([s], ni_start=-10)
    e.set_positions(pos)
    with pytest.raises(B.BDError) as ei:
        e.run(12)
    assert ei.value.code == 9


def test_graph_relaunch_after_single_steps():
    # 101 steps leave the buffer rotation one phase on (96 in a graph + 5 single
    # steps); later graph launches must use the rotation they run in
    s, pos = system(500, 700, 0.5, 15)
    e1 = B.Engine([s], graph_steps=96)
    e1.set_positions(pos)
    e1.run(101)
    e1.run(204)
    e1.run(97)
    e2 = B.Engine([s], graph_steps=96)
    e2.set_positions(pos)
    for _ in range(402):
        e2.run(1)
    np.testing.assert_array_equal(e1.get_positions()[0], e2.get_positions()[0])


def _ragged(n=6, seed=40):
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        nb = int(rng.integers(100, 900))
        ns = int(rng.integers(100, 900))
        out.append(system(nb, ns, float(rng.uniform(0.45, 0.56)), seed + k, T0=float(rng.uniform(0.1, 1.0))))
    return zip(*out)


def test_persistent_cluster_mode_bit_identical_to_plain():
    systems, poss = _ragged()
    pos = np.concatenate(poss)
    ep = B.Engine(list(systems), mode="persistent", cluster=4)
    ep.set_positions(pos)
    ep.run(96 + 40)  # one persistent graph chunk + one direct persistent launch
    ep.run(77)
    e1 = B.Engine(list(systems), neighbor_skin=0.0)  # persistent mode sweeps every step
    e1.set_positions(pos)
    e1.run(213)
    np.testing.assert_array_equal(ep.get_positions()[0], e1.get_positions()[0])
    np.testing.assert_array_equal(ep.get_positions()[1], e1.get_positions()[1])


def test_autotuner_changes_speed_not_results():
    systems, poss = _ragged(4, 70)
    pos = np.concatenate(poss)
    for mode in ("plain", "persistent"):
        ea = B.Engine(list(systems), mode=mode, autotune=1)
        ea.set_positions(pos)
        ea.run(300)
        e1 = B.Engine(list(systems), neighbor_skin=ea.info().neighbor_skin)
        e1.set_positions(pos)
        e1.run(300)
        np.testing.assert_array_equal(ea.get_positions()[0], e1.get_positions()[0])


def test_list_autotuner_and_launch_variants_change_speed_not_results():
    """List mode: every list-step launch variant, and the autotuner's choice
    of variant and build brick (timed on the live batch), give the same bits
    as the default layout.  Variants 3-5 run each batch of steps in one
    launch, one block per replica that rebuilds its own lists: their
    rebuild decisions (counted per replica and per step) and their lists
    are those of the per-step kernels."""
    systems, poss = _ragged(4, 71)
    pos = np.concatenate(poss)
    ref = B.Engine(list(systems))
    assert ref.info().neighbor_skin > 0 and ref.info().list_variant == 0
    ref.set_positions(pos)
    ref.run(700)  # seven 96-step graphs and 28 single steps
    want = ref.get_positions()
    ref_info = ref.info()
    assert ref_info.list_builds > 4 and ref_info.list_rebuild_steps > 1
    cnt_ref, hsh_ref = ref.census()
    for v in (1, 2, 3, 4, 5):
        ev = B.Engine(list(systems), list_variant=v)
        assert ev.info().list_variant == v
        ev.set_positions(pos)
        ev.run(700)
        got = ev.get_positions()
        np.testing.assert_array_equal(got[0], want[0], err_msg="variant %d" % v)
        np.testing.assert_array_equal(got[1], want[1], err_msg="variant %d" % v)
        info = ev.info()
        assert (info.list_builds, info.list_rebuild_steps) == (ref_info.list_builds, ref_info.list_rebuild_steps), v
        cnt, hsh = ev.census()
        np.testing.assert_array_equal(cnt, cnt_ref)
        np.testing.assert_array_equal(hsh, hsh_ref)
        ev.close()
    ea = B.Engine(list(systems), autotune=1)
    ea.set_positions(pos)
    # inside the first call: 15 (brick, per-step variant) pairs over 2 + 12
    # steps, then the best against variants 3-5 over 2 + 96 steps each
    ea.run(700)
    info = ea.info()
    assert info.tuned_ms > 0 and 0 <= info.list_variant < 6
    got = ea.get_positions()
    np.testing.assert_array_equal(got[0], want[0])
    np.testing.assert_array_equal(got[1], want[1])
    with pytest.raises(B.BDError):
        B.Engine(list(systems), list_variant=6)


def test_first_step_temperature_carried_over():
    """A replica given T_first takes its first update at that temperature and
    then follows its protocol (the drop-in executable uses this for
    configurations after the first, which the reference starts at the
    temperature the previous configuration ended on, main.cu:156).  With the
    same injected noise, constant T0 = 1 with T_first = 0.25 gives, bit for
    bit, the run of a quench from 0.25 to 1 right after the first update, and
    differs from constant T = 1 after the first step."""
    import dataclasses
    s, pos = system(300, 300, 0.5, 5, T0=1.0, force_cap=100.0)
    noise = np.random.default_rng(3).standard_normal((2, s.n, 3)).astype(np.float32)
    runs = {}
    for name, desc in (("carried", dataclasses.replace(s, protocol="const", T_first=0.25)),
                       ("stepped", dataclasses.replace(s, protocol="linear", T0=0.25, Tf=1.0, t0=0.0, tf=1e-30)),
                       ("hot", dataclasses.replace(s, protocol="const"))):
        e = B.Engine([desc], rng="noise")
        e.set_positions(pos)
        out = []
        for k in range(2):
            e.set_noise(noise[k])
            e.run(1)
            out.append(e.get_positions()[0].copy())
        runs[name] = out
        e.close()
    for k in range(2):
        np.testing.assert_array_equal(runs["carried"][k], runs["stepped"][k])
    assert not np.array_equal(runs["carried"][0], runs["hot"][0])
