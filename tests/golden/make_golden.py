"""Generate the golden vectors in tests/golden/ by running the REFERENCE ITSELF.

The reference has no tests or fixtures of its own.  Its host functions
(cell_locate_hst, get_forces_same_hst / get_forces_diff_hst, update_ermak_hst,
get_gder_hst, fself_isotropic, calculate_temp_linear / _sine,
sampling_indexes, rannew64, Contracting_Vector3D) are compiled from the
reference sources into oracle/_ref/libref.so by `make -C oracle ref` and
called here on seeded inputs; their outputs become the fixtures that pin the
CPU oracle (tests/test_oracle_golden.py).

Run:  python tests/golden/make_golden.py      (needs the reference sources)
"""
import ctypes as C
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import oracle as O  # noqa: E402
from bd_aging_b200 import configs as CF  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))

SYSTEMS = {
    # name: (n_big, n_sml, phi, seed, nbins, range_frac, ntags)
    "g1": (150, 150, 0.45, 11, 60, 0.5, 16),
    "g2": (60, 240, 0.30, 12, 40, 0.45, 16),
}


def ref_params(L, side, nb, ns, nbins, rng, ntags, dt=1e-4, T0=1.0):
    p = O.Parametros()
    L.ref_setup_params(C.byref(p), side, nb, ns, float(CF.SIGMA_BIG), float(CF.SIGMA_SML), 1.0, 1.0, ntags, ntags,
                       nbins, rng, dt, T0)
    return p


def system_golden(L, name, nb, ns, phi, seed, nbins, rfrac, ntags):
    side = np.float32(CF.side_from_phi(nb, ns, phi))
    pos = CF.lattice_config(nb, ns, float(side), seed)
    rb, rs = pos[:nb].copy(), pos[nb:].copy()
    p = ref_params(L, float(side), nb, ns, nbins, float(side) * rfrac, ntags)
    g = {"side": np.float32(side), "rb": rb, "rs": rs, "params": np.frombuffer(bytes(p), np.uint8).copy()}
    # cell lists (reference host order = ascending particle index)
    for sp, rr, nc in (("b", rb, p.ncell_big), ("s", rs, p.ncell_sml)):
        nocup = np.zeros(nc ** 3, np.int32)
        cell = np.full(nc ** 3 * ntags, -1, np.int32)
        L.ref_cell_locate_hst(sp.encode(), rr, nocup, cell, C.byref(p))
        g["nocup_" + sp] = nocup
        g["cell_" + sp] = cell
    # forces: the four-call sequence of main.cu:566-574 on cleared arrays
    ffb = np.zeros_like(rb); ffs = np.zeros_like(rs)
    vb = np.zeros(nb, np.float32); pb = np.zeros(nb, np.float32)
    vs = np.zeros(ns, np.float32); ps = np.zeros(ns, np.float32)
    L.ref_get_forces_same_hst(b"b", rb, ffb, vb, pb, g["nocup_b"], g["cell_b"], C.byref(p))
    L.ref_get_forces_same_hst(b"s", rs, ffs, vs, ps, g["nocup_s"], g["cell_s"], C.byref(p))
    L.ref_get_forces_diff_hst(b"b", b"s", rb, ffb, rs, vb, pb, g["nocup_s"], g["cell_s"], C.byref(p))
    L.ref_get_forces_diff_hst(b"s", b"b", rs, ffs, rb, vs, ps, g["nocup_b"], g["cell_b"], C.byref(p))
    g.update(ff_b=ffb, ff_s=ffs, vir_b=vb, vir_s=vs, pot_b=pb, pot_s=ps)
    # Ermak-McCammon update with injected float32-valued N(0,1) noise
    rng = np.random.default_rng(seed + 100)
    for sp, rr, ff in (("b", rb, ffb), ("s", rs, ffs)):
        noise = rng.standard_normal(3 * len(rr)).astype(np.float32)
        r1 = rr.copy(); raw = rr.copy()
        L.ref_update_ermak_hst(sp.encode(), r1, raw, ff.copy(), noise.astype(np.float64), len(noise), C.byref(p))
        g["noise_" + sp] = noise
        g["upd_rr_" + sp] = r1
        g["upd_raw_" + sp] = raw
    # g(r): per-block float histograms summed over blocks (main.cu:742-754)
    NH = 256
    for k, (a, b, ra, rbb) in enumerate((("b", "b", rb, rb), ("b", "s", rb, rs), ("s", "b", rs, rb),
                                         ("s", "s", rs, rs))):
        nblk = 1 + (len(ra) - 1) // NH
        h = np.zeros(nblk * nbins, np.float32)
        L.ref_get_gder_hst(a.encode(), b.encode(), ra, rbb, h, C.byref(p))
        g["gder_" + a + b] = h.reshape(nblk, nbins).sum(0, dtype=np.float64)
    # F_s / MSD inputs: a displaced copy as rr_raw, origin rr
    disp = rng.normal(0.0, 0.3, size=rb.shape).astype(np.float32)
    raw_b = (rb + disp).astype(np.float32)
    fs = np.zeros(4, np.float32)
    L.ref_fself_isotropic(raw_b, rb, nb, fs, 2, np.float32(7.0))
    g["fself_raw_b"] = raw_b
    g["fself"] = fs
    return g


def main():
    L = O.ref_lib()
    all_g = {}
    for name, spec in SYSTEMS.items():
        for k, v in system_golden(L, name, *spec).items():
            all_g[name + "_" + k] = v
    # temperature protocols (set_temp.cu), including t == t0 == tf (NaN)
    tl = []
    for (T0, Tf, t0, tf) in ((1.0, 0.25, 0.0, 0.0), (1.0, 0.1, 0.5, 2.0), (0.2, 1.0, 0.0, 1.0e-3)):
        for t in (-1.0, 0.0, 1e-4, 0.5, 1.0, 1.9999, 2.0, 5.0):
            tl.append((T0, Tf, t0, tf, t, L.ref_calculate_temp_linear(T0, Tf, t0, tf, t)))
    all_g["temp_linear"] = np.array(tl, np.float32)
    ts = []
    for (T0, Tf, t0, tf, per) in ((1.0, 0.5, 0.0, 10.0, 2.0), (0.3, 0.9, 1.0, 3.0, 0.7)):
        for t in (-1.0, 0.0, 0.1, 1.3, 2.5, 3.0, 9.0, 11.0):
            ts.append((T0, Tf, t0, tf, per, t, L.ref_calculate_temp_sine(T0, Tf, t0, tf, per, t)))
    all_g["temp_sine"] = np.array(ts, np.float32)
    # log sampling schedule (main.cu:14-53)
    for k, (md, rt, dt) in enumerate(((1e-3, 10.0, 1e-4), (1e-3, 1e3, 1e-5), (1e-2, 1e1, 2e-5), (1e-1, 1e3, 1e-5))):
        buf = np.zeros(4096, np.int32)
        n = L.ref_sampling_indexes(md, rt, dt, 10, buf, 4096)
        all_g["sampling_%d" % k] = buf[:n].copy()
        all_g["sampling_%d_args" % k] = np.array([md, rt, dt])
    # rannew64 (rannew64.cu): a negative idum (re)initialises the stream
    for k, seed in enumerate((12345, 987654321)):
        idum = C.c_long(-seed)
        vals = [L.ref_rannew64(C.byref(idum)) for _ in range(1000)]
        all_g["rannew64_%d" % k] = np.array(vals, np.float64)
        all_g["rannew64_%d_seed" % k] = np.array([seed], np.int64)
    # Contracting_Vector3D with and without periodic images (GSL SVD -> shim)
    rng = np.random.default_rng(77)
    nb, ns = 200, 200
    side = CF.side_from_phi(nb, ns, 0.4)
    pos = CF.lattice_config(nb, ns, side, 77)
    xx = rng.standard_normal((nb + ns, 3)).astype(np.float32)
    for k, sd in enumerate((side, -1.0)):
        h = L.ref_cv3d_create(16, 3.0)
        L.ref_cv3d_add_statistics(h, pos, xx, nb + ns, sd)
        L.ref_cv3d_add_statistics(h, pos[::-1].copy(), xx, nb + ns, sd)
        L.ref_cv3d_calculate_vector(h)
        v = np.zeros(16, np.float32)
        L.ref_cv3d_get_vector(h, v)
        L.ref_cv3d_destroy(h)
        all_g["cv3d_%d_vec" % k] = v
    all_g["cv3d_pos"] = pos
    all_g["cv3d_xx"] = xx
    all_g["cv3d_side"] = np.array([side], np.float32)
    np.savez_compressed(os.path.join(OUT, "reference_golden.npz"), **all_g)
    print("wrote", os.path.join(OUT, "reference_golden.npz"), len(all_g), "arrays")


if __name__ == "__main__":
    main()
