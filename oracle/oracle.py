"""ctypes access to the CPU oracle (liboracle.so) and to the reference built
from its own sources (_ref/libref.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's reference / cpu_baseline legs, always as the checker.  The product
package never imports this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_ORACLE = os.path.join(HERE, "liboracle.so")
LIB_REF = os.path.join(HERE, "_ref", "libref.so")

_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")


class Parametros(C.Structure):
    """Layout of the reference `parametros` (encabezados.h:40-75)."""

    _fields_ = [(n, C.c_float) for n in (
        "side", "dt", "mass_big", "mass_sml", "sigma_big", "sigma_sml", "cell_side_big",
        "cell_side_sml", "temp_set", "bin_size_dplt", "bin_size_gder", "range_dplt", "range_gder")] + \
        [(n, C.c_int) for n in (
            "ngrain_big", "ngrain_sml", "ngrain_tot", "ntags_big", "ntags_sml", "ncell_big", "ncell_med",
            "ncell_sml", "nrange_bb", "nrange_bs", "nrange_sb", "nrange_ss", "nbins_dplt", "nbins_gder",
            "nsearch_big", "not_finished", "NH", "WCA_flag")] + [("idum", C.c_long)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


def build_oracle() -> None:
    """Compile liboracle.so (plain C, gcc)."""
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)


_oracle = None
_ref = None


def oracle_lib():
    global _oracle
    if _oracle is None:
        if not os.path.exists(LIB_ORACLE):
            build_oracle()
        L = C.CDLL(LIB_ORACLE)
        P = C.POINTER(Parametros)
        L.or_ref_setup_params.argtypes = [P, C.c_float, C.c_int, C.c_int, C.c_float, C.c_float, C.c_float,
                                          C.c_float, C.c_int, C.c_int, C.c_int, C.c_float, C.c_double, C.c_float]
        L.or_ref_cell_locate.argtypes = [C.c_char, _f32p, _i32p, _i32p, P]
        L.or_ref_cell_locate.restype = C.c_int
        L.or_ref_forces_same.argtypes = [C.c_char, _f32p, _f32p, _f32p, _f32p, _i32p, _i32p, P]
        L.or_ref_forces_diff.argtypes = [C.c_char, C.c_char, _f32p, _f32p, _f32p, _f32p, _f32p, _i32p, _i32p, P]
        L.or_ref_update_ermak.argtypes = [C.c_char, _f32p, _f32p, _f32p, _f32p, P]
        L.or_ref_gder_counts.argtypes = [C.c_char, C.c_char, _f32p, _f32p, _u64p, P]
        L.or_ref_gder_normalize.argtypes = [_f64p, C.c_int, C.c_float, C.c_float, C.c_int, C.c_int, C.c_float,
                                            C.c_float, C.c_int, _f32p]
        L.or_ref_fself.argtypes = [_f32p, _f32p, C.c_int, _f32p, C.c_int, C.c_float]
        L.or_ref_msd.argtypes = [_f32p, _f32p, C.c_int]
        L.or_ref_msd.restype = C.c_float
        L.or_ref_energy.argtypes = [_f32p, C.c_int]
        L.or_ref_energy.restype = C.c_float
        L.or_ref_pressure_z.argtypes = [_f32p, C.c_int, _f32p, C.c_int, C.c_float]
        L.or_ref_pressure_z.restype = C.c_float
        for fn, n in (("or_ref_temp_linear", 5), ("or_ref_temp_sine", 6)):
            getattr(L, fn).argtypes = [C.c_float] * n
            getattr(L, fn).restype = C.c_float
        L.or_ref_time_of_step.argtypes = [C.c_double, C.c_int]
        L.or_ref_time_of_step.restype = C.c_float
        L.or_ref_sampling_indexes.argtypes = [C.c_float, C.c_float, C.c_float, C.c_int, _i32p, C.c_int]
        L.or_ref_sampling_indexes.restype = C.c_int
        L.or_rannew64_next.restype = C.c_double
        L.or_rannew64_particle_noise.argtypes = [C.c_longlong, C.c_int, C.c_int, _f32p]
        L.or_ref_colors.argtypes = [C.c_int, C.c_int, _f32p, _f32p, C.c_float, C.c_float, C.c_float, _i32p, _i32p]
        L.or_pair_extra.argtypes = [C.c_int, _f32p, C.c_float, C.c_float, C.POINTER(C.c_float), C.POINTER(C.c_float)]
        L.or_eng_forces_pot.argtypes = [C.c_int, _f32p, _i32p, C.c_float, _f32p, C.c_int, _f32p, _f32p, _f32p, _f32p]
        L.or_precision_run.argtypes = [C.c_int, C.c_int, C.c_int, _f32p, C.c_double, C.c_double, C.c_double,
                                       C.c_double, C.c_double, C.c_double, C.c_double, C.c_uint64, C.c_uint32,
                                       C.c_longlong, C.c_int, C.c_double, _f64p, _f64p]
        L.or_precision_run.restype = C.c_int
        L.or_ref_cv3d_add.argtypes = [C.c_int, C.c_float, _f32p, _f32p, C.c_int, C.c_float, _f32p, _f32p]
        L.or_ref_cv3d_add.restype = C.c_int
        L.or_philox4x32_10.argtypes = [_u32p, _u32p, _u32p]
        L.or_eng_gauss3.argtypes = [C.c_uint64, C.c_uint32, C.c_uint64, C.c_uint32, _f64p]
        L.or_eng_uniform_bits.argtypes = [C.c_uint64, C.c_uint32, C.c_uint64, C.c_uint32, _u32p]
        L.or_eng_forces.argtypes = [C.c_int, _f32p, _i32p, C.c_float, _f32p, _f32p, _f32p, _f32p, _i32p, _u64p]
        L.or_eng_update.argtypes = [C.c_int, _f32p, _f32p, _f64p, _f32p, _i32p, C.c_float, C.c_double, _f32p,
                                    _f32p, _f32p]
        L.or_eng_cap_forces.argtypes = [C.c_int, _f32p, C.c_float]
        L.or_eng_amplitude.argtypes = [C.c_float, C.c_float, C.c_float]
        L.or_eng_amplitude.restype = C.c_float
        L.or_eng_fself_msd.argtypes = [C.c_int, _f64p, C.c_double, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        _oracle = L
    return _oracle


def rannew64_particle_noise(seed: int, n: int, steps: int) -> np.ndarray:
    """N(0,1) noise [steps, n, 3] of the engine's per-particle rannew64 mode."""
    out = np.zeros((steps, n, 3), np.float32)
    oracle_lib().or_rannew64_particle_noise(int(seed), int(n), int(steps), out)
    return out


PRECISION_FIELDS = ("msd_big", "msd_sml", "fself_big", "energy_big", "energy_sml", "virial")


def precision_run(mode, pos, n_big, side, sig_big, sig_sml, mob_big, mob_sml, dt, temp, seed, steps, q,
                  stream=0, ni0=0):
    """mode "fp64" or "fp32_reference": observables after `steps` steps with
    the engine's Philox noise, and the FP64 displacement [n, 3]."""
    pos = np.ascontiguousarray(pos, np.float32)
    n = len(pos)
    obs = np.zeros(6, np.float64)
    dsp = np.zeros((n, 3), np.float64)
    rc = oracle_lib().or_precision_run({"fp64": 0, "fp32_reference": 1}[mode], n, n_big, pos, side, sig_big,
                                       sig_sml, mob_big, mob_sml, dt, temp, seed, stream, ni0, steps, q, obs, dsp)
    if rc:
        raise MemoryError("or_precision_run")
    return dict(zip(PRECISION_FIELDS, obs)), dsp


def colors(rb, rs, side, sigma_big, sigma_sml):
    """Colour ids (0 blue, 1 green, 2 red) of the big particles and the
    blue/green/red counts: restatement of colors.cu."""
    rb = np.ascontiguousarray(rb, np.float32)
    rs = np.ascontiguousarray(rs, np.float32)
    ids = np.zeros(len(rb), np.int32)
    counts = np.zeros(3, np.int32)
    oracle_lib().or_ref_colors(len(rb), len(rs), rb, rs, side, sigma_big, sigma_sml, ids, counts)
    return ids, counts


def ref_colors(rb, rs, p: Parametros):
    """The reference's own calculate_color over every big particle."""
    L = ref_lib()
    rb = np.ascontiguousarray(rb, np.float32)
    rs = np.ascontiguousarray(rs, np.float32)
    counts = np.zeros(3, np.int32)
    ids = np.array([L.ref_calculate_color(m, rb, rs, counts, C.byref(p)) for m in range(len(rb))], np.int32)
    return ids, counts


POT = {"wca_modified": 0, "wca": 1, "wca49_50": 2, "ao": 3, "hsay": 4}


def pair_extra(pot, pp, sigma, dist_inv):
    """(energy, normal force) of one pair with a potential of potentials.cu."""
    u, nf = C.c_float(0), C.c_float(0)
    oracle_lib().or_pair_extra(POT[pot], np.ascontiguousarray(pp, np.float32), sigma, dist_inv, C.byref(u),
                               C.byref(nf))
    return u.value, nf.value


def eng_forces_pot(pos, types, side, sigma_big, sigma_sml, pot, pp):
    n = len(pos)
    ff = np.zeros((n, 3), np.float32)
    potv = np.zeros(n, np.float32)
    vir = np.zeros(n, np.float32)
    oracle_lib().or_eng_forces_pot(n, np.ascontiguousarray(pos, np.float32), np.ascontiguousarray(types, np.int32),
                                   side, np.array([sigma_big, sigma_sml], np.float32), POT[pot],
                                   np.ascontiguousarray(pp, np.float32), ff, potv, vir)
    return ff, potv, vir


def ref_available() -> bool:
    return os.path.exists(LIB_REF)


def ref_lib():
    """The reference compiled from its own sources (oracle/Makefile `ref`)."""
    global _ref
    if _ref is None:
        L = C.CDLL(LIB_REF)
        P = C.POINTER(Parametros)
        L.ref_sizeof_parametros.restype = C.c_int
        L.ref_cell_locate_hst.argtypes = [C.c_char, _f32p, _i32p, _i32p, P]
        L.ref_get_forces_same_hst.argtypes = [C.c_char, _f32p, _f32p, _f32p, _f32p, _i32p, _i32p, P]
        L.ref_get_forces_diff_hst.argtypes = [C.c_char, C.c_char, _f32p, _f32p, _f32p, _f32p, _f32p, _i32p,
                                              _i32p, P]
        L.ref_update_ermak_hst.argtypes = [C.c_char, _f32p, _f32p, _f32p, _f64p, C.c_long, P]
        L.ref_get_gder_hst.argtypes = [C.c_char, C.c_char, _f32p, _f32p, _f32p, P]
        L.ref_fself_isotropic.argtypes = [_f32p, _f32p, C.c_int, _f32p, C.c_int, C.c_float]
        L.ref_calculate_temp_linear.argtypes = [C.c_float] * 5
        L.ref_calculate_temp_linear.restype = C.c_float
        L.ref_calculate_temp_sine.argtypes = [C.c_float] * 6
        L.ref_calculate_temp_sine.restype = C.c_float
        L.ref_sampling_indexes.argtypes = [C.c_double, C.c_double, C.c_double, C.c_int, _i32p, C.c_int]
        L.ref_sampling_indexes.restype = C.c_int
        L.ref_rannew64.argtypes = [C.POINTER(C.c_long)]
        L.ref_rannew64.restype = C.c_double
        L.ref_cv3d_create.argtypes = [C.c_int, C.c_float]
        L.ref_cv3d_create.restype = C.c_void_p
        L.ref_cv3d_add_statistics.argtypes = [C.c_void_p, _f32p, _f32p, C.c_int, C.c_float]
        L.ref_cv3d_calculate_vector.argtypes = [C.c_void_p]
        L.ref_cv3d_get_vector.argtypes = [C.c_void_p, _f32p]
        L.ref_cv3d_destroy.argtypes = [C.c_void_p]
        L.ref_setup_params.argtypes = [P, C.c_float, C.c_int, C.c_int, C.c_float, C.c_float, C.c_float, C.c_float,
                                       C.c_int, C.c_int, C.c_int, C.c_float, C.c_double, C.c_float]
        L.ref_cuda_forces.argtypes = [P, _f32p, _f32p, _f32p, _f32p, _f32p, _f32p, _f32p, _f32p]
        L.ref_cuda_forces.restype = C.c_int
        L.ref_cuda_run.argtypes = [P, _f32p, _f32p, C.c_int, C.c_int, C.c_int, C.c_float, C.c_float, C.c_float,
                                   C.c_float, C.c_double, _f32p, _f32p, _f32p, _f32p, C.POINTER(C.c_float)]
        L.ref_cuda_run.restype = C.c_int
        L.ref_cuda_run_sampled.argtypes = [P, _f32p, _f32p, C.c_int, C.c_int, C.c_int, C.c_float, C.c_float,
                                           C.c_float, C.c_float, C.c_double, C.c_int, _i32p, _f32p, _f32p, _f32p,
                                           C.POINTER(C.c_float)]
        L.ref_cuda_run_sampled.restype = C.c_int
        L.ref_cuda_gder.argtypes = [P, _f32p, _f32p, _f32p]
        L.ref_cuda_gder.restype = C.c_int
        L.ref_hst_run.argtypes = [P] + [_f32p] * 10 + [_i32p] * 4 + [C.c_long, C.c_long] + [C.c_float] * 4 + \
            [C.c_double, C.c_ulong]
        L.ref_hst_run.restype = C.c_int
        L.ref_calculate_color.argtypes = [C.c_int, _f32p, _f32p, _i32p, P]
        F = C.c_float
        FP = C.POINTER(C.c_float)
        L.ref_potential_wca_hst.argtypes = [F, F, FP, FP]
        L.ref_potential_wca49_50_hst.argtypes = [F, F, F, F, FP, FP]
        L.ref_potential_wca49_50_AO_hst.argtypes = [F, F, F, F, F, F, FP, FP]
        L.ref_calculate_color.restype = C.c_int
        _ref = L
    return _ref


# --------------------------------------------------------------- helpers
def setup_params(side, nb, ns, sigma_big, sigma_sml, ntags=(8, 8), nbins=200, rng=None, dt=1e-5, T0=1.0,
                 mass=(1.0, 1.0)) -> Parametros:
    """main.cu parameter set-up, restated (or_ref_setup_params)."""
    p = Parametros()
    oracle_lib().or_ref_setup_params(C.byref(p), side, nb, ns, sigma_big, sigma_sml, mass[0], mass[1], ntags[0],
                                     ntags[1], nbins, side / 2 if rng is None else rng, dt, T0)
    return p


def cell_locate(p: Parametros, species: str, rr: np.ndarray):
    b = species == "b"
    nc = p.ncell_big if b else p.ncell_sml
    nt = p.ntags_big if b else p.ntags_sml
    nocup = np.zeros(nc ** 3, np.int32)
    cell = np.full(nc ** 3 * nt, -1, np.int32)
    bad = oracle_lib().or_ref_cell_locate(species.encode(), np.ascontiguousarray(rr, np.float32), nocup, cell,
                                          C.byref(p))
    return nocup, cell, bad


def ref_forces(p: Parametros, rb: np.ndarray, rs: np.ndarray):
    """Forces/vir/pot of both species with the reference four-call sequence
    (main.cu:576-585) restated: returns dict of arrays."""
    L = oracle_lib()
    rb = np.ascontiguousarray(rb, np.float32)
    rs = np.ascontiguousarray(rs, np.float32)
    nob, cb, _ = cell_locate(p, "b", rb)
    nos, cs, _ = cell_locate(p, "s", rs)
    out = {k: np.zeros_like(v) for k, v in (("ff_b", rb), ("ff_s", rs))}
    out["vir_b"] = np.zeros(len(rb), np.float32); out["pot_b"] = np.zeros(len(rb), np.float32)
    out["vir_s"] = np.zeros(len(rs), np.float32); out["pot_s"] = np.zeros(len(rs), np.float32)
    L.or_ref_forces_same(b"b", rb, out["ff_b"], out["vir_b"], out["pot_b"], nob, cb, C.byref(p))
    L.or_ref_forces_same(b"s", rs, out["ff_s"], out["vir_s"], out["pot_s"], nos, cs, C.byref(p))
    L.or_ref_forces_diff(b"b", b"s", rb, out["ff_b"], rs, out["vir_b"], out["pot_b"], nos, cs, C.byref(p))
    L.or_ref_forces_diff(b"s", b"b", rs, out["ff_s"], rb, out["vir_s"], out["pot_s"], nob, cb, C.byref(p))
    return out


def gder_counts(p: Parametros, rb, rs):
    """[4, nbins] uint64 ordered-pair counts (bb, bs, sb, ss)."""
    L = oracle_lib()
    rb = np.ascontiguousarray(rb, np.float32)
    rs = np.ascontiguousarray(rs, np.float32)
    out = np.zeros((4, p.nbins_gder), np.uint64)
    for k, (a, b, ra, rbb) in enumerate((("b", "b", rb, rb), ("b", "s", rb, rs), ("s", "b", rs, rb),
                                         ("s", "s", rs, rs))):
        c = np.zeros(p.nbins_gder, np.uint64)
        L.or_ref_gder_counts(a.encode(), b.encode(), ra, rbb, c, C.byref(p))
        out[k] = c
    return out


def sampling_indexes(minimal_decade, run_time, dt, per_decade=10):
    buf = np.zeros(4096, np.int32)
    n = oracle_lib().or_ref_sampling_indexes(minimal_decade, run_time, dt, per_decade, buf, 4096)
    return buf[:n].copy()


def eng_gauss3(seed: int, ids, step: int, stream: int = 0) -> np.ndarray:
    L = oracle_lib()
    out = np.zeros((len(ids), 3), np.float64)
    tmp = np.zeros(3, np.float64)
    for k, i in enumerate(ids):
        L.or_eng_gauss3(seed, int(i), step, stream, tmp)
        out[k] = tmp
    return out


def eng_forces(pos, types, side, sigma_big, sigma_sml):
    L = oracle_lib()
    n = len(pos)
    pos = np.ascontiguousarray(pos, np.float32)
    ff = np.zeros((n, 3), np.float32)
    pot = np.zeros(n, np.float32)
    vir = np.zeros(n, np.float32)
    nbr = np.zeros(n, np.int32)
    h = np.zeros(n, np.uint64)
    L.or_eng_forces(n, pos, np.ascontiguousarray(types, np.int32), side,
                    np.array([sigma_big, sigma_sml], np.float32), ff, pot, vir, nbr, h)
    return ff, pot, vir, nbr, h


def cv3d_add(bins, rng_, rr, xx, side):
    """Contracting_Vector3D::add_statistics restated (float): returns
    (ata [3, bins, bins], atb [3, bins], overflow)."""
    ata = np.zeros((3, bins, bins), np.float32)
    atb = np.zeros((3, bins), np.float32)
    bad = oracle_lib().or_ref_cv3d_add(bins, rng_, np.ascontiguousarray(rr, np.float32),
                                       np.ascontiguousarray(xx, np.float32), len(rr), side, ata, atb)
    return ata, atb, bad


def cv3d_solve(ata, atb, dtype=np.float32):
    """Contracting_Vector3D::calculate_vector (Contracting_Vector3D.cu:166-297)
    restated with numpy's FP64 SVD in place of GSL's: per component
    x = V diag(w_inv) U^T b with w_inv = 0 where |w/w_max| <= 1e-6, the
    solution arithmetic in `dtype`, then the mean of the three components."""
    bins = ata.shape[-1]
    acc = np.zeros(bins, dtype)
    for c in range(3):
        u, w, vt = np.linalg.svd(np.asarray(ata[c], np.float64))
        u = u.astype(dtype); w = w.astype(dtype); v = vt.T.astype(dtype)
        wmax = np.abs(w).max() if w.size else 0
        with np.errstate(divide="ignore", invalid="ignore"):
            winv = np.where(np.abs(w / wmax) > 1e-6, 1.0 / w, 0.0).astype(dtype) if wmax > 0 else np.zeros_like(w)
        aux = (u.T @ np.asarray(atb[c], dtype)) * winv
        acc += v @ aux
    return (acc / 3).astype(dtype)


class RefHostRun:
    """The reference's host time loop (oracle/_ref ref_hst_run) on one system:
    CPU baseline and reference arm of bench.py."""

    def __init__(self, p: Parametros, pos: np.ndarray, seed: int = 1):
        self.p = p
        nb, ns = p.ngrain_big, p.ngrain_sml
        self.rb = np.ascontiguousarray(pos[:nb], np.float32).copy()
        self.rs = np.ascontiguousarray(pos[nb:], np.float32).copy()
        self.rawb, self.raws = self.rb.copy(), self.rs.copy()
        self.ffb, self.ffs = np.zeros_like(self.rb), np.zeros_like(self.rs)
        self.vb, self.pb = np.zeros(nb, np.float32), np.zeros(nb, np.float32)
        self.vs, self.ps = np.zeros(ns, np.float32), np.zeros(ns, np.float32)
        ncb3, ncs3 = p.ncell_big ** 3, p.ncell_sml ** 3
        self.nob, self.cb = np.zeros(ncb3, np.int32), np.zeros(ncb3 * p.ntags_big, np.int32)
        self.nos, self.cs = np.zeros(ncs3, np.int32), np.zeros(ncs3 * p.ntags_sml, np.int32)
        self.ni = 0
        self.seed = seed

    def run(self, nsteps, T0, Tf, t0, tf, dt):
        rc = ref_lib().ref_hst_run(C.byref(self.p), self.rb, self.rs, self.rawb, self.raws, self.ffb, self.ffs,
                                   self.vb, self.vs, self.pb, self.ps, self.nob, self.cb, self.nos, self.cs,
                                   nsteps, self.ni, T0, Tf, t0, tf, dt, self.seed)
        self.ni += nsteps
        return rc
