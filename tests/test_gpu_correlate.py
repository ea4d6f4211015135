"""GPU parity of the waiting-time correlator (snapshots + batched F_s / MSD /
<|dr|^4> reduction) against an FP64 numpy restatement of fself.cu:3-21 and
the MSD loop of main.cu:776-797, and of the one-process aging workflow
against the same trajectory stepped by hand."""
import os
import subprocess
import sys

import numpy as np
import pytest

from bd_aging_b200 import aging as A
from bd_aging_b200 import configs as CF
from bd_aging_b200 import lib as B

pytestmark = pytest.mark.gpu
SB, SS = float(CF.SIGMA_BIG), float(CF.SIGMA_SML)
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
Q = 6.19


def ragged(n=3, seed=11):
    rng = np.random.default_rng(seed)
    systems, poss = [], []
    for k in range(n):
        nb, ns = int(rng.integers(200, 1200)), int(rng.integers(200, 1200))
        side = float(np.float32(CF.side_from_phi(nb, ns, float(rng.uniform(0.35, 0.45)))))
        # force cap: the jittered lattice start has overlaps
        systems.append(B.System(n_big=nb, n_sml=ns, side=side, sigma_big=SB, sigma_sml=SS, dt=1e-4,
                                seed=seed * 100 + k, T0=1.0, Tf=0.2, t0=0.0, tf=0.005, protocol="linear",
                                force_cap=200.0))
        poss.append(CF.lattice_config(nb, ns, side, seed + k))
    return systems, np.concatenate(poss)


def expected(systems, d_now, d_then, q=Q):
    """numpy FP64: per replica (msd, r4, fs) of big and small."""
    out = []
    off = 0
    for s in systems:
        dr = d_now[off:off + s.n] - d_then[off:off + s.n]
        r2 = (dr * dr).sum(1)
        qr = q * np.sqrt(r2)
        fs = np.where(qr > 0, np.sin(qr) / np.where(qr > 0, qr, 1.0), 1.0)
        b = slice(0, s.n_big)
        m = slice(s.n_big, s.n)
        out.append(dict(msd_big=r2[b].mean(), r4_big=(r2[b] ** 2).mean(), fself_big=fs[b].mean(),
                        msd_sml=r2[m].mean(), r4_sml=(r2[m] ** 2).mean(), fself_sml=fs[m].mean()))
        off += s.n
    return out


def check(c_row, exp, rtol=1e-12):
    for r, e in enumerate(exp):
        for k, v in e.items():
            np.testing.assert_allclose(c_row[r][k], v, rtol=rtol, atol=1e-300, err_msg=f"replica {r} {k}")


def test_correlate_matches_numpy_fp64():
    systems, pos = ragged()
    e = B.Engine(systems, ni_start=-50)
    e.set_positions(pos)
    e.reserve_snapshots(3)
    e.run(50)
    e.snapshot(0)  # origin step: zero displacement
    e.run(37)
    e.snapshot(1)
    d1 = e.get_displacements()
    e.run(120)
    e.snapshot(2)
    d2 = e.get_displacements()
    e.run(55)
    d3 = e.get_displacements()
    c = e.correlate([0, 1, 2], Q)
    assert list(c["lag_steps"][:, 0]) == [212, 175, 55]
    check(c[0], expected(systems, d3, np.zeros_like(d3)))
    check(c[1], expected(systems, d3, d1))
    check(c[2], expected(systems, d3, d2))
    # one slot at a time gives the same bits
    for j in range(3):
        np.testing.assert_array_equal(e.correlate([j], Q)[0], c[j])


def test_origin_slot_equals_builtin_observables():
    systems, pos = ragged(2, 5)
    e = B.Engine(systems, ni_start=-20, qmax=Q)
    e.set_positions(pos)
    e.reserve_snapshots(1)
    e.run(20)
    e.snapshot(0)
    e.run(150)
    c = e.correlate([0], float(np.float32(Q)))[0]  # the built-in F_s uses qmax as a float
    o = e.observe()
    for r in range(len(systems)):
        np.testing.assert_allclose(c[r]["msd_big"], o[r]["msd_big"], rtol=1e-12)
        np.testing.assert_allclose(c[r]["msd_sml"], o[r]["msd_sml"], rtol=1e-12)
        np.testing.assert_allclose(c[r]["fself_big"], o[r]["fself_big"], rtol=1e-12)


def test_correlations_independent_of_batching_and_mode():
    systems, pos = ragged(3, 17)
    res = []
    for kw in (dict(neighbor_skin=0.0), dict(mode="persistent", cluster=2)):
        e = B.Engine(systems, **kw)
        e.set_positions(pos)
        e.reserve_snapshots(2)
        e.snapshot(0)
        e.run(40)
        e.snapshot(1)
        e.run(101)
        res.append(e.correlate([0, 1], Q))
    np.testing.assert_array_equal(res[0], res[1])
    off = np.cumsum([0] + [s.n for s in systems])
    for r, s in enumerate(systems):  # a replica alone gives the same bits
        e = B.Engine([s], neighbor_skin=0.0)
        e.set_positions(pos[off[r]:off[r + 1]])
        e.reserve_snapshots(2)
        e.snapshot(0)
        e.run(40)
        e.snapshot(1)
        e.run(101)
        np.testing.assert_array_equal(e.correlate([0, 1], Q)[:, 0], res[0][:, r])


def test_correlate_errors():
    systems, pos = ragged(1, 3)
    e = B.Engine(systems, ni_start=-10)
    e.set_positions(pos)
    e.reserve_snapshots(2)
    with pytest.raises(B.BDError) as ei:
        e.correlate([0], Q)  # never taken
    assert ei.value.code == B.BD_ERR_STATE
    with pytest.raises(B.BDError) as ei:
        e.correlate([2], Q)  # out of range
    assert ei.value.code == B.BD_ERR_ARG
    with pytest.raises(B.BDError) as ei:
        e.correlate([0], 0.0)
    assert ei.value.code == B.BD_ERR_ARG
    e.run(3)
    e.snapshot(0)  # before the origin step
    e.run(4)
    e.correlate([0], Q)  # still before it: valid
    e.run(10)
    with pytest.raises(B.BDError) as ei:
        e.correlate([0], Q)  # the origin was re-based since
    assert ei.value.code == B.BD_ERR_STATE
    e.snapshot(1)
    e.set_positions(pos)
    with pytest.raises(B.BDError) as ei:
        e.correlate([1], Q)  # positions replaced since
    assert ei.value.code == B.BD_ERR_STATE


def test_aging_workflow_matches_hand_stepped_trajectory():
    systems, pos = ragged(2, 23)
    dt = systems[0].dt
    idx = A.sampling_indexes(1e-3, 1e-1, dt)
    tws = A.waiting_time_steps(idx, 2)
    assert tws == [0, idx[1] + 1, idx[11] + 1]
    e = B.Engine(systems, ni_start=-30, qmax=Q)
    e.set_positions(pos)
    e.run(30)
    res = A.run_aging(e, idx, tws, Q, dt)
    # the same trajectory, stepped to every needed step by hand
    h = B.Engine(systems, ni_start=-30, qmax=Q)
    h.set_positions(pos)
    h.run(30)
    need = sorted(set(tws) | {tw + l + 1 for tw in tws for l in idx})
    disp, ni = {}, 0
    for s in need:
        h.run(s - ni)
        ni = s
        disp[s] = h.get_displacements()
    disp[0] = np.zeros_like(disp[need[-1]])
    for k, tw in enumerate(tws):
        for si in (0, 3, len(idx) - 1):
            exp = expected(systems, disp[tw + idx[si] + 1], disp[tw])
            check(res[k].per_replica[si], exp)
        np.testing.assert_allclose(res[k].t[1], np.float32(dt * (1 + np.float32(idx[1]))))
    assert res[0].fself_big[0] < 1.0 and 0.0 < res[2].msd_big[-1] < 1.0


def test_aging_command_line_writes_every_decade(tmp_path):
    nb = ns = 600
    side = float(np.float32(CF.side_from_phi(nb, ns, 0.3)))  # dilute: the lattice start has no hard overlaps
    cfgdir = tmp_path / "configs"
    sim = tmp_path / "simulation"
    cfgdir.mkdir()
    sim.mkdir()
    rng = np.random.default_rng(3)
    for i in range(2):
        p = CF.lattice_config(nb, ns, side, 40 + i, jitter=0.05)
        CF.write_init_config(str(cfgdir / f"init_config_{i + 1}"), p, nb, ns, side)
    data = "linear\n1.0 0.25 0.0 0.002 1\n1e-4\nlog\n0.001 1e-3 1e-1\n1 2 0\n8 8\n2\n50 4.0\n6.19\n%d\n" % int(
        rng.integers(1, 1 << 30))
    r = subprocess.run([sys.executable, "-m", "bd_aging_b200.aging"], input=data, text=True, cwd=sim,
                       env=dict(os.environ, PYTHONPATH=ROOT), capture_output=True, timeout=600)
    assert r.returncode == 0, r.stderr
    idx = A.sampling_indexes(1e-3, 1e-1, 1e-4)
    for k in range(3):
        d = sim / "results" / f"decade{k}"
        for name in ("fself.out", "msd_averaged.out", "energies_averaged.out", "pressure.out"):
            rows = (d / name).read_text().strip().split("\n")
            assert len(rows) == len(idx), (k, name)
        assert (d / f"gder_{len(idx) - 1}.out").exists()
        fs = np.loadtxt(d / "fself.out")
        assert np.all(fs[:, 1] <= 1.0) and np.all(fs[:, 1] > -0.5)
