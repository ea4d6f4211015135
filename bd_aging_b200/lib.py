"""ctypes binding of libbd_aging_b200.so (include/bd_aging.h) and a Python
mirror of the reference's entry points.

Reference-mirror functions take CUDA tensors (torch) holding the reference's
float3 array-of-structs data ([N, 3] float32, contiguous) and raise BDError
where the reference would exit().  The Engine class wraps the batched replica
engine.  There is no CPU fallback: without the built library or a CUDA
device every call raises.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("BD_AGING_LIB") or os.path.join(HERE, "libbd_aging_b200.so")

BD_OK, BD_ERR_ARG, BD_ERR_CUDA, BD_ERR_CELL_OVERFLOW, BD_ERR_NOMEM, BD_ERR_STATE = 0, 1, 2, 3, 4, 5
BD_ERR_TIMEOUT, BD_ERR_FILE, BD_ERR_FORMAT, BD_ERR_NUMERIC = 6, 7, 8, 9
STATUS_NAMES = {0: "BD_OK", 1: "BD_ERR_ARG", 2: "BD_ERR_CUDA", 3: "BD_ERR_CELL_OVERFLOW", 4: "BD_ERR_NOMEM",
                5: "BD_ERR_STATE", 6: "BD_ERR_TIMEOUT", 7: "BD_ERR_FILE", 8: "BD_ERR_FORMAT", 9: "BD_ERR_NUMERIC"}
PROTOCOL = {"linear": 0, "sine": 1, "const": 2}
POTENTIAL = {"wca_modified": 0, "wca": 1, "wca49_50": 2, "ao": 3, "hsay": 4}
RNG = {"philox": 0, "curand": 1, "noise": 2, "rannew64": 3}
MODE = {"auto": 0, "plain": 1, "persistent": 2}
GDER = {"auto": 0, "all_pairs": 1, "cells": 2}


class BDError(RuntimeError):
    def __init__(self, code: int, where: str):
        self.code = code
        msg = _lib().bd_status_string(code).decode() if _LIB is not None else str(code)
        super().__init__("%s: %s (%s)" % (where, STATUS_NAMES.get(code, code), msg))


class Parametros(C.Structure):
    """bd_parametros == the reference `parametros` (encabezados.h:40-75)."""

    _fields_ = [(n, C.c_float) for n in (
        "side", "dt", "mass_big", "mass_sml", "sigma_big", "sigma_sml", "cell_side_big",
        "cell_side_sml", "temp_set", "bin_size_dplt", "bin_size_gder", "range_dplt", "range_gder")] + \
        [(n, C.c_int) for n in (
            "ngrain_big", "ngrain_sml", "ngrain_tot", "ntags_big", "ntags_sml", "ncell_big", "ncell_med",
            "ncell_sml", "nrange_bb", "nrange_bs", "nrange_sb", "nrange_ss", "nbins_dplt", "nbins_gder",
            "nsearch_big", "not_finished", "NH", "WCA_flag")] + [("idum", C.c_long)]


class SystemDesc(C.Structure):
    _fields_ = [("n_big", C.c_int), ("n_sml", C.c_int), ("side", C.c_float), ("sigma_big", C.c_float),
                ("sigma_sml", C.c_float), ("mob_big", C.c_float), ("mob_sml", C.c_float), ("dt", C.c_double),
                ("temp_protocol", C.c_int), ("T0", C.c_float), ("Tf", C.c_float), ("t0", C.c_float),
                ("tf", C.c_float), ("period", C.c_float), ("seed", C.c_ulonglong), ("force_cap", C.c_float),
                ("potential", C.c_int), ("pot_param", C.c_float * 4), ("first_temp_set", C.c_int),
                ("T_first", C.c_float)]


class EngineOpts(C.Structure):
    _fields_ = [("rng", C.c_int), ("cell_capacity", C.c_int), ("brick", C.c_int * 3), ("threads", C.c_int),
                ("mode", C.c_int), ("cluster", C.c_int), ("autotune", C.c_int), ("graph_steps", C.c_int),
                ("qmax", C.c_float), ("ni_start", C.c_longlong), ("rng_stream", C.c_uint),
                ("neighbor_skin", C.c_float), ("list_variant", C.c_int)]


class Observables(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("energy_big", "energy_sml", "virial", "msd_big", "msd_sml",
                                          "fself_big", "nbr_pairs", "temperature")]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class Correlation(C.Structure):
    _fields_ = [("lag_steps", C.c_longlong)] + [(n, C.c_double) for n in ("fself_big", "fself_sml", "msd_big",
                                                                         "msd_sml", "r4_big", "r4_sml")]


CORR_DTYPE = np.dtype([("lag_steps", np.int64), ("fself_big", np.float64), ("fself_sml", np.float64),
                       ("msd_big", np.float64), ("msd_sml", np.float64), ("r4_big", np.float64),
                       ("r4_sml", np.float64)])


class EngineInfo(C.Structure):
    _fields_ = [("nsys", C.c_int), ("n_particles", C.c_longlong), ("n_cells", C.c_longlong),
                ("brick", C.c_int * 3), ("threads", C.c_int), ("cell_capacity", C.c_int),
                ("staging_capacity", C.c_int), ("mode", C.c_int), ("cluster", C.c_int),
                ("smem_bytes", C.c_size_t), ("next_step", C.c_longlong), ("neighbor_skin", C.c_float),
                ("list_builds", C.c_longlong), ("list_rebuild_steps", C.c_longlong), ("list_variant", C.c_int),
                ("tuned_ms", C.c_float)]


_LIB = None
_vp = C.c_void_p


def _lib():
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("libbd_aging_b200.so is not built (python -m bd_aging_b200.build); "
                               "there is no CPU fallback")
        L = C.CDLL(LIB_PATH)
        P = C.POINTER(Parametros)
        sig = {
            "bd_status_string": ([C.c_int], C.c_char_p),
            "bd_abi_version": ([], C.c_int),
            "bd_setup_params": ([P, C.c_float, C.c_int, C.c_int, C.c_float, C.c_float, C.c_float, C.c_float,
                                 C.c_int, C.c_int, C.c_int, C.c_float, C.c_double, C.c_float], C.c_int),
            "bd_cell_locate": ([C.c_char, _vp, _vp, _vp, P, _vp], C.c_int),
            "bd_get_forces_same": ([C.c_char, _vp, _vp, _vp, _vp, _vp, _vp, P, _vp], C.c_int),
            "bd_get_forces_diff": ([C.c_char, C.c_char, _vp, _vp, _vp, _vp, _vp, _vp, _vp, P, _vp], C.c_int),
            "bd_rng_state_size": ([], C.c_size_t),
            "bd_setup_rng": ([_vp, C.c_ulonglong, C.c_int, _vp], C.c_int),
            "bd_update_ermak": ([C.c_char, _vp, _vp, _vp, _vp, P, _vp], C.c_int),
            "bd_update_ermak_noise": ([C.c_char, _vp, _vp, _vp, _vp, P, _vp], C.c_int),
            "bd_calculate_temp_linear": ([C.c_float] * 5, C.c_float),
            "bd_calculate_temp_sine": ([C.c_float] * 6, C.c_float),
            "bd_get_gder": ([C.c_char, C.c_char, _vp, _vp, _vp, P, _vp], C.c_int),
            "bd_gder_normalize": ([_vp, C.c_int, C.c_float, C.c_float, C.c_int, C.c_int, C.c_float, C.c_float,
                                   C.c_int, _vp], C.c_int),
            "bd_fself_isotropic": ([_vp, _vp, C.c_int, _vp, C.c_int, C.c_float, _vp], C.c_int),
            "bd_msd": ([_vp, _vp, C.c_int, _vp, _vp], C.c_int),
            "bd_color_statistics": ([_vp, _vp, _vp, _vp, C.POINTER(Parametros), _vp], C.c_int),
            "bd_cv3d_create": ([C.c_int, C.c_float, C.POINTER(_vp)], C.c_int),
            "bd_cv3d_add_statistics": ([_vp, _vp, _vp, C.c_int, C.c_float, _vp], C.c_int),
            "bd_cv3d_calculate_vector": ([_vp], C.c_int),
            "bd_cv3d_get_vector": ([_vp, _vp], C.c_int),
            "bd_cv3d_destroy": ([_vp], C.c_int),
            "bd_engine_opts_default": ([C.POINTER(EngineOpts)], None),
            "bd_engine_create": ([C.POINTER(SystemDesc), C.c_int, C.POINTER(EngineOpts), C.POINTER(_vp)], C.c_int),
            "bd_engine_destroy": ([_vp], C.c_int),
            "bd_engine_get_info": ([_vp, C.POINTER(EngineInfo)], C.c_int),
            "bd_engine_get_stream": ([_vp, C.POINTER(_vp)], C.c_int),
            "bd_engine_set_positions": ([_vp, _vp], C.c_int),
            "bd_engine_run": ([_vp, C.c_longlong], C.c_int),
            "bd_engine_observe": ([_vp, C.POINTER(Observables)], C.c_int),
            "bd_engine_get_positions": ([_vp, _vp, _vp], C.c_int),
            "bd_engine_gder": ([_vp, C.c_int, C.c_float, _vp], C.c_int),
            "bd_engine_gder_method": ([_vp, C.c_int, C.c_float, C.c_int, _vp], C.c_int),
            "bd_engine_set_noise": ([_vp, _vp], C.c_int),
            "bd_engine_census": ([_vp, _vp, _vp], C.c_int),
            "bd_engine_reserve_snapshots": ([_vp, C.c_int], C.c_int),
            "bd_engine_snapshot": ([_vp, C.c_int], C.c_int),
            "bd_engine_correlate": ([_vp, _vp, C.c_int, C.c_double, _vp], C.c_int),
            "bd_engine_get_displacements": ([_vp, _vp], C.c_int),
            "bd_surrogate_create": ([C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_ulonglong, _vp], C.c_int),
            "bd_surrogate_destroy": ([_vp], C.c_int),
            "bd_surrogate_get_stream": ([_vp, _vp], C.c_int),
            "bd_surrogate_param_count": ([_vp, _vp], C.c_int),
            "bd_surrogate_get_params": ([_vp, _vp], C.c_int),
            "bd_surrogate_set_params": ([_vp, _vp], C.c_int),
            "bd_surrogate_set_output_weights": ([_vp, _vp], C.c_int),
            "bd_surrogate_set_data": ([_vp, _vp, _vp, C.c_int], C.c_int),
            "bd_surrogate_train": ([_vp, C.c_int, C.c_float, _vp], C.c_int),
            "bd_surrogate_gradients": ([_vp, _vp, _vp, _vp, _vp], C.c_int),
            "bd_surrogate_predict": ([_vp, _vp, C.c_int, _vp], C.c_int),
            "bd_umma_gemm_bf16": ([_vp, _vp, C.c_int, C.c_int, C.c_int, _vp], C.c_int),
        }
        for name, (args, res) in sig.items():
            if hasattr(L, name):
                f = getattr(L, name)
                f.argtypes = args
                f.restype = res
        _LIB = L
    return _LIB


def lib():
    return _lib()


def _check(rc: int, where: str):
    if rc != BD_OK:
        raise BDError(rc, where)


def _ptr(t) -> int:
    """Device (or host numpy) pointer of a contiguous array."""
    if t is None:
        return None
    if isinstance(t, np.ndarray):
        assert t.flags["C_CONTIGUOUS"]
        return t.ctypes.data
    assert t.is_contiguous(), "tensor must be contiguous"
    return t.data_ptr()


def _stream(stream):
    if stream is None:
        return None
    return getattr(stream, "cuda_stream", stream)


def _species(c) -> bytes:
    if c not in ("b", "s"):
        raise BDError(1, "species must be 'b' or 's'")
    return c.encode()


# ------------------------------------------------- reference-mirror functions
def setup_params(side, ngrain_big, ngrain_sml, sigma_big, sigma_sml, mass_big=1.0, mass_sml=1.0, ntags_big=8,
                 ntags_sml=8, nbins_gder=200, range_gder=None, dt=1e-5, temp0=1.0) -> Parametros:
    """Parameter set-up of the reference driver (main.cu:155-163, 244-298)."""
    p = Parametros()
    rg = side / 2 if range_gder is None else range_gder
    _check(_lib().bd_setup_params(C.byref(p), side, ngrain_big, ngrain_sml, sigma_big, sigma_sml, mass_big, mass_sml,
                                  ntags_big, ntags_sml, nbins_gder, rg, dt, temp0), "bd_setup_params")
    return p


def cell_locate(type, rr, nocup, cell_vec, pars: Parametros, stream=None):
    """cell_locate_dev (cell_locate.cu:155-209) with its clears."""
    _check(_lib().bd_cell_locate(_species(type), _ptr(rr), _ptr(nocup), _ptr(cell_vec), C.byref(pars),
                                 _stream(stream)), "cell_locate")


def get_forces_same(type, rr, ff, vir, pot, nocup, cell_vec, pars: Parametros, stream=None):
    """get_forces_same_dev (get_forces.cu:297-424); adds into ff/vir/pot."""
    _check(_lib().bd_get_forces_same(_species(type), _ptr(rr), _ptr(ff), _ptr(vir), _ptr(pot), _ptr(nocup),
                                     _ptr(cell_vec), C.byref(pars), _stream(stream)), "get_forces_same")


def get_forces_diff(type, type_other, rr, ff, rr_other, vir, pot, nocup_other, cell_other, pars: Parametros,
                    stream=None):
    """get_forces_diff_dev (get_forces.cu:428-558); adds into ff/vir/pot."""
    _check(_lib().bd_get_forces_diff(_species(type), _species(type_other), _ptr(rr), _ptr(ff), _ptr(rr_other),
                                     _ptr(vir), _ptr(pot), _ptr(nocup_other), _ptr(cell_other), C.byref(pars),
                                     _stream(stream)), "get_forces_diff")


def rng_state_size() -> int:
    return int(_lib().bd_rng_state_size())


def setup_rng(states, seed: int, n: int, stream=None):
    """setup_rng_kernel (update_ermak.cu:85-89)."""
    _check(_lib().bd_setup_rng(_ptr(states), seed, n, _stream(stream)), "setup_rng")


def update_ermak(type, rr, rr_raw, ff, states, pars: Parametros, stream=None):
    """update_ermak_dev (update_ermak.cu:91-160) with the cuRAND stream."""
    _check(_lib().bd_update_ermak(_species(type), _ptr(rr), _ptr(rr_raw), _ptr(ff), _ptr(states), C.byref(pars),
                                  _stream(stream)), "update_ermak")


def update_ermak_noise(type, rr, rr_raw, ff, noise, pars: Parametros, stream=None):
    """update_ermak with injected N(0,1) values (3 per particle)."""
    _check(_lib().bd_update_ermak_noise(_species(type), _ptr(rr), _ptr(rr_raw), _ptr(ff), _ptr(noise),
                                        C.byref(pars), _stream(stream)), "update_ermak_noise")


def calculate_temp_linear(T0, Tf, t0, tf, t) -> float:
    return _lib().bd_calculate_temp_linear(T0, Tf, t0, tf, t)


def calculate_temp_sine(T0, Tf, t0, tf, period, t) -> float:
    return _lib().bd_calculate_temp_sine(T0, Tf, t0, tf, period, t)


def get_gder(type, type_other, rr, rr_other, counts, pars: Parametros, stream=None):
    """get_gder_dev (get_gder.cu:69-127): adds exact counts into `counts`
    (int64 CUDA tensor of nbins_gder entries)."""
    _check(_lib().bd_get_gder(_species(type), _species(type_other), _ptr(rr), _ptr(rr_other), _ptr(counts),
                              C.byref(pars), _stream(stream)), "get_gder")


def gder_normalize(counts, nbins, bin_size, side, ngrain_big, ngrain_sml, sigma_big, sigma_sml, n_configs):
    """g(r) normalisation of main.cu:849-877 (host): counts [4, nbins]."""
    c = np.ascontiguousarray(counts, np.float64)
    out = np.zeros((4, nbins), np.float32)
    _check(_lib().bd_gder_normalize(_ptr(c), nbins, bin_size, side, ngrain_big, ngrain_sml, sigma_big, sigma_sml,
                                    n_configs, _ptr(out)), "gder_normalize")
    return out


def fself_isotropic(rr_raw, rr0, ngrain, fself: np.ndarray, sample_number, qmax, stream=None):
    """fself_isotropic (fself.cu:3-21): adds into the host array fself."""
    assert fself.dtype == np.float32
    _check(_lib().bd_fself_isotropic(_ptr(rr_raw), _ptr(rr0), ngrain, _ptr(fself), sample_number, qmax,
                                     _stream(stream)), "fself_isotropic")


def msd(rr_raw, rr0, ngrain, stream=None) -> float:
    out = np.zeros(1, np.float32)
    _check(_lib().bd_msd(_ptr(rr_raw), _ptr(rr0), ngrain, _ptr(out), _stream(stream)), "msd")
    return float(out[0])


def color_statistics(rr_big, rr_sml, pars: Parametros, color_ids=None, stream=None):
    """calculate_color (colors.cu) for every big particle: device positions in,
    optional device int ids out (0 blue, 1 green, 2 red); returns the counts
    (blue, green, red)."""
    counts = np.zeros(3, np.int32)
    _check(_lib().bd_color_statistics(_ptr(rr_big), _ptr(rr_sml), _ptr(color_ids), _ptr(counts), C.byref(pars),
                                      _stream(stream)), "color_statistics")
    return counts


class Contracting_Vector3D:
    """Contracting_Vector3D (Contracting_Vector3D.cuh:39-75) on the GPU with
    FP64 normal equations."""

    def __init__(self, bins: int, range: float):
        h = _vp()
        _check(_lib().bd_cv3d_create(bins, range, C.byref(h)), "Contracting_Vector3D")
        self._h = h
        self.bins = bins

    def add_statistics(self, rr_vec, xx_vec, nparticles: int, side=None, stream=None):
        _check(_lib().bd_cv3d_add_statistics(self._h, _ptr(rr_vec), _ptr(xx_vec), nparticles,
                                             -1.0 if side is None else side, _stream(stream)), "add_statistics")

    def calculate_vector(self):
        _check(_lib().bd_cv3d_calculate_vector(self._h), "calculate_vector")

    def get_vector(self) -> np.ndarray:
        out = np.zeros(self.bins, np.float32)
        _check(_lib().bd_cv3d_get_vector(self._h, _ptr(out)), "get_vector")
        return out

    def __del__(self):
        if getattr(self, "_h", None) and _LIB is not None:
            _LIB.bd_cv3d_destroy(self._h)
            self._h = None


# ------------------------------------------------------------------ engine
@dataclass
class System:
    n_big: int
    n_sml: int
    side: float
    sigma_big: float
    sigma_sml: float
    dt: float
    T0: float = 1.0
    Tf: float = 1.0
    t0: float = 0.0
    tf: float = 0.0
    period: float = 1.0
    protocol: str = "const"
    seed: int = 1
    mobility: str = "reference"   # "reference": 1/sigma; "unit": D0 = 1
    force_cap: float = 0.0
    potential: str = "wca_modified"  # POTENTIAL keys; parameters in pot_param (bd_aging.h BD_POT_*)
    pot_param: tuple = (0.0, 0.0, 0.0, 0.0)
    T_first: float = None  # temperature of the first update (None: T0)

    def desc(self) -> SystemDesc:
        d = SystemDesc()
        d.n_big, d.n_sml, d.side = self.n_big, self.n_sml, self.side
        d.sigma_big, d.sigma_sml = self.sigma_big, self.sigma_sml
        if self.mobility == "reference":
            d.mob_big = float(np.float32(1.0) / np.float32(self.sigma_big))
            d.mob_sml = float(np.float32(1.0) / np.float32(self.sigma_sml))
        else:
            d.mob_big = d.mob_sml = 1.0
        d.dt = self.dt
        d.temp_protocol = PROTOCOL[self.protocol]
        d.T0, d.Tf, d.t0, d.tf, d.period = self.T0, self.Tf, self.t0, self.tf, self.period
        d.seed = self.seed
        d.force_cap = self.force_cap
        d.potential = POTENTIAL[self.potential]
        for k in range(4):
            d.pot_param[k] = float(self.pot_param[k]) if k < len(self.pot_param) else 0.0
        if self.T_first is not None:
            d.first_temp_set, d.T_first = 1, float(self.T_first)
        return d

    @property
    def n(self):
        return self.n_big + self.n_sml


class Engine:
    """Batched replica engine (bd_engine_*)."""

    def __init__(self, systems, rng="philox", mode="auto", brick=None, threads=0, cell_capacity=0,
                 graph_steps=96, qmax=2 * np.pi, ni_start=0, rng_stream=0, cluster=0, autotune=0,
                 neighbor_skin=None, list_variant=None):
        self.systems = list(systems)
        n = len(self.systems)
        arr = (SystemDesc * n)(*[s.desc() for s in self.systems])
        o = EngineOpts()
        _lib().bd_engine_opts_default(C.byref(o))
        o.rng = RNG[rng]
        o.mode = MODE[mode]
        o.cell_capacity = cell_capacity
        if brick:
            o.brick[0], o.brick[1], o.brick[2] = brick
        o.threads = threads
        o.graph_steps = graph_steps
        o.qmax = qmax
        o.ni_start = ni_start
        o.rng_stream = rng_stream
        o.cluster = cluster
        o.autotune = autotune
        if neighbor_skin is not None:  # None: the library default
            o.neighbor_skin = neighbor_skin
        if list_variant is not None:  # None: the library default (tuned when autotune is set)
            o.list_variant = list_variant
        h = _vp()
        _check(_lib().bd_engine_create(arr, n, C.byref(o), C.byref(h)), "bd_engine_create")
        self._h = h
        self.P = sum(s.n for s in self.systems)
        self.offsets = np.cumsum([0] + [s.n for s in self.systems])

    def info(self) -> EngineInfo:
        i = EngineInfo()
        _check(_lib().bd_engine_get_info(self._h, C.byref(i)), "info")
        return i

    def stream_handle(self) -> int:
        s = _vp()
        _check(_lib().bd_engine_get_stream(self._h, C.byref(s)), "get_stream")
        return s.value or 0

    def set_positions(self, pos: np.ndarray):
        pos = np.ascontiguousarray(pos, np.float32).reshape(self.P, 3)
        _check(_lib().bd_engine_set_positions(self._h, _ptr(pos)), "set_positions")

    def run(self, nsteps: int):
        _check(_lib().bd_engine_run(self._h, int(nsteps)), "run")

    def observe(self):
        out = (Observables * len(self.systems))()
        _check(_lib().bd_engine_observe(self._h, out), "observe")
        return [o.as_dict() for o in out]

    def get_positions(self, out_pos: np.ndarray = None, out_raw: np.ndarray = None):
        """Wrapped and unwrapped positions [P, 3] by reference index, written
        into out_pos / out_raw when given (C-contiguous float32, e.g. pinned)."""
        def buf(a):
            if a is None:
                return np.empty((self.P, 3), np.float32)
            if a.dtype != np.float32 or a.shape != (self.P, 3) or not a.flags.c_contiguous:
                raise ValueError("output buffers must be C-contiguous float32 [P, 3]")
            return a
        pos, raw = buf(out_pos), buf(out_raw)
        _check(_lib().bd_engine_get_positions(self._h, _ptr(pos), _ptr(raw)), "get_positions")
        return pos, raw

    def gder(self, nbins: int, range_: float, method: str = "auto") -> np.ndarray:
        """Exact g(r) counts [nsys, 4 (bb, bs, sb, ss), nbins]; method "auto",
        "all_pairs" or "cells" (same counts, different candidate search)."""
        out = np.zeros((len(self.systems), 4, nbins), np.uint64)
        _check(_lib().bd_engine_gder_method(self._h, nbins, range_, GDER[method], _ptr(out)), "gder")
        return out

    def set_noise(self, noise: np.ndarray):
        noise = np.ascontiguousarray(noise, np.float32).reshape(self.P, 3)
        _check(_lib().bd_engine_set_noise(self._h, _ptr(noise)), "set_noise")

    def census(self):
        cnt = np.zeros(self.P, np.int32)
        hsh = np.zeros(self.P, np.uint64)
        _check(_lib().bd_engine_census(self._h, _ptr(cnt), _ptr(hsh)), "census")
        return cnt, hsh

    def reserve_snapshots(self, nslots: int):
        _check(_lib().bd_engine_reserve_snapshots(self._h, int(nslots)), "reserve_snapshots")

    def snapshot(self, slot: int):
        """Record every particle's displacement now (waiting time t_w) in `slot`."""
        _check(_lib().bd_engine_snapshot(self._h, int(slot)), "snapshot")

    def correlate(self, slots, q: float) -> np.ndarray:
        """F_s(q), MSD and <|dr|^4> per species since each slot: array [len(slots), nsys]."""
        sl = np.ascontiguousarray(np.atleast_1d(slots), np.int32)
        out = np.zeros((len(sl), len(self.systems)), CORR_DTYPE)
        assert CORR_DTYPE.itemsize == C.sizeof(Correlation)
        _check(_lib().bd_engine_correlate(self._h, _ptr(sl), len(sl), float(q), _ptr(out)), "correlate")
        return out

    def get_displacements(self) -> np.ndarray:
        """FP64 displacement since the origin step, [P, 3] in the set_positions order."""
        out = np.zeros((self.P, 3), np.float64)
        _check(_lib().bd_engine_get_displacements(self._h, _ptr(out)), "get_displacements")
        return out

    def close(self):
        if getattr(self, "_h", None):
            _lib().bd_engine_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------------ surrogate
class Surrogate:
    """The learned surrogate (bd_surrogate_*): MLP n_in -> width x depth (GELU)
    -> n_out on tcgen05 BF16 GEMMs, FP32 Adam."""

    def __init__(self, n_in=5, n_out=34, width=256, depth=4, batch=4096, seed=1):
        L = _lib()
        h = _vp()
        _check(L.bd_surrogate_create(n_in, n_out, width, depth, batch, C.c_ulonglong(seed), C.byref(h)),
               "bd_surrogate_create")
        self._h = h
        self.n_in, self.n_out, self.width, self.depth, self.batch = n_in, n_out, width, depth, batch
        c = C.c_longlong(0)
        _check(L.bd_surrogate_param_count(h, C.byref(c)), "param_count")
        self.n_params = c.value

    def sizes(self):
        return [(self.width, self.n_in)] + [(self.width, self.width)] * (self.depth - 1) + \
            [(self.n_out, self.width)]

    def get_params(self) -> np.ndarray:
        out = np.zeros(self.n_params, np.float32)
        _check(_lib().bd_surrogate_get_params(self._h, _ptr(out)), "get_params")
        return out

    def set_params(self, p: np.ndarray):
        p = np.ascontiguousarray(p, np.float32)
        assert p.size == self.n_params
        _check(_lib().bd_surrogate_set_params(self._h, _ptr(p)), "set_params")

    def set_output_weights(self, w: np.ndarray):
        w = np.ascontiguousarray(w, np.float32)
        _check(_lib().bd_surrogate_set_output_weights(self._h, _ptr(w)), "set_output_weights")

    def set_data(self, x: np.ndarray, y: np.ndarray):
        x = np.ascontiguousarray(x, np.float32).reshape(-1, self.n_in)
        y = np.ascontiguousarray(y, np.float32).reshape(-1, self.n_out)
        _check(_lib().bd_surrogate_set_data(self._h, _ptr(x), _ptr(y), len(x)), "set_data")

    def train(self, steps: int, lr: float = 1e-3) -> float:
        loss = C.c_float(0)
        _check(_lib().bd_surrogate_train(self._h, int(steps), C.c_float(lr), C.byref(loss)), "train")
        return loss.value

    def gradients(self, x: np.ndarray, y: np.ndarray):
        x = np.ascontiguousarray(x, np.float32).reshape(self.batch, self.n_in)
        y = np.ascontiguousarray(y, np.float32).reshape(self.batch, self.n_out)
        g = np.zeros(self.n_params, np.float32)
        loss = C.c_float(0)
        _check(_lib().bd_surrogate_gradients(self._h, _ptr(x), _ptr(y), _ptr(g), C.byref(loss)), "gradients")
        return g, loss.value

    def predict(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, np.float32).reshape(-1, self.n_in)
        y = np.zeros((len(x), self.n_out), np.float32)
        _check(_lib().bd_surrogate_predict(self._h, _ptr(x), len(x), _ptr(y)), "predict")
        return y

    def stream_handle(self) -> int:
        s = _vp()
        _check(_lib().bd_surrogate_get_stream(self._h, C.byref(s)), "get_stream")
        return s.value or 0

    def close(self):
        if getattr(self, "_h", None):
            _lib().bd_surrogate_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def umma_gemm_bf16(a_bits: np.ndarray, b_bits: np.ndarray) -> np.ndarray:
    """C = A B^T through the surrogate's tcgen05 GEMM kernel (BF16 bits in, FP32 out)."""
    a_bits = np.ascontiguousarray(a_bits, np.uint16)
    b_bits = np.ascontiguousarray(b_bits, np.uint16)
    M, K = a_bits.shape
    N = b_bits.shape[0]
    c = np.zeros((M, N), np.float32)
    _check(_lib().bd_umma_gemm_bf16(_ptr(a_bits), _ptr(b_bits), M, N, K, _ptr(c)), "umma_gemm_bf16")
    return c
