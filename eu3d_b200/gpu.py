"""ctypes binding of the C ABI in include/eu3d_gpu.h.

``DeviceFlowfield`` is the Python face of one handle: a device-resident
flowfield plus its chemistry for one rank, with methods named after the
reference's Flowfield / Reaction / Euler members they stand in for.  The
library is the in-tree libeu3d_gpu.so; if it is missing or no CUDA device is
present the constructor raises -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

from . import build as _build

_dp = C.POINTER(C.c_double)

# constants mirrored from include/eu3d_quirks.h and include/eu3d_gpu.h
QUIRKS_REF = 0x1FF
QUIRKS_FIXED = 0x000
BC_RSBI, BC_ODM, BC_TRANSMISSIVE, BC_NONE = 0, 1, 2, 3
REACT_TRAPEZOID, REACT_IMEX, REACT_NONE, REACT_SURROGATE = 0, 1, 2, 3
DIFF_MUSCL1, DIFF_MUSCL2 = 0, 1
ADV_EE, ADV_TVD_RK3, ADV_SSPRK2 = 0, 1, 2

FIELDS = {"U": 0, "V": 1, "W": 2, "P": 3, "D": 4, "T": 5, "H": 6, "Gamma": 7, "E": 8, "Yi": 9, "CS": 10, "RHS": 11,
          "C": 12, "Mc": 13, "Di": 14, "Nchem": 15}
UPLOADABLE = ("U", "V", "W", "P", "D", "T", "H", "Gamma", "E", "Yi", "CS", "RHS")

EXPORTS = ["eu3d_last_error", "eu3d_create", "eu3d_destroy", "eu3d_upload_field", "eu3d_download_field",
           "eu3d_set_inflow", "eu3d_init_uniform", "eu3d_set_wedge", "eu3d_set_dt", "eu3d_set_time", "eu3d_get_dt", "eu3d_cfl",
           "eu3d_boundary", "eu3d_advection", "eu3d_update_after_adv", "eu3d_update_after_cs", "eu3d_react_imex",
           "eu3d_react_trapezoid", "eu3d_step", "eu3d_run", "eu3d_synchronize", "eu3d_get_status",
           "eu3d_reset_status", "eu3d_stream", "eu3d_profile_enable", "eu3d_profile_read", "eu3d_cfl_noalloc",
           "eu3d_gemm_bf16"]


class Eu3dError(RuntimeError):
    pass


class Desc(C.Structure):
    _fields_ = [("ni", C.c_int), ("nj", C.c_int), ("nk", C.c_int), ("bc", C.c_int),
                ("xnode", _dp), ("ynode", _dp), ("znode", _dp), ("NS", C.c_int), ("NR", C.c_int),
                ("stoi_f", _dp), ("stoi_b", _dp), ("react_tb", _dp), ("af", _dp), ("bf", _dp), ("eaf", _dp),
                ("coeff0", _dp), ("coeff1", _dp), ("mw", _dp), ("quirks", C.c_uint), ("flux_bits", C.c_int),
                ("device", C.c_int)]


class StepDesc(C.Structure):
    _fields_ = [("react", C.c_int), ("type", C.c_int), ("timeadv", C.c_int), ("diff", C.c_int),
                ("bc_kind", C.c_int), ("cfl", C.c_double), ("final_time", C.c_double)]


class Status(C.Structure):
    _fields_ = [("nonfinite_cells", C.c_longlong), ("newton_capped", C.c_longlong), ("substeps", C.c_longlong),
                ("nchem_max", C.c_int), ("substep_capped", C.c_int), ("surrogate_cells", C.c_longlong),
                ("surrogate_fallback", C.c_longlong), ("dt", C.c_double), ("time", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_LIB = None


def load_library(path: Optional[str] = None):
    """Load libeu3d_gpu.so (no build attempt): raises if it is absent."""
    global _LIB
    if _LIB is not None and path is None:
        return _LIB
    p = path or _build.LIB
    if not os.path.exists(p):
        raise Eu3dError(f"CUDA library {p} is missing: run `python -m eu3d_b200.build`")
    L = C.CDLL(p)
    L.eu3d_last_error.restype = C.c_char_p
    L.eu3d_create.argtypes = [C.POINTER(Desc), C.POINTER(C.c_void_p)]
    h = [C.c_void_p]
    L.eu3d_destroy.argtypes = h
    L.eu3d_upload_field.argtypes = h + [C.c_int, _dp]
    L.eu3d_download_field.argtypes = h + [C.c_int, _dp]
    L.eu3d_set_inflow.argtypes = h + [_dp] * 10
    L.eu3d_set_wedge.argtypes = h + [C.c_double, C.c_double, C.c_double, C.c_int]
    L.eu3d_init_uniform.argtypes = h + [C.c_double] * 5 + [_dp]
    L.eu3d_set_dt.argtypes = h + [C.c_double]
    L.eu3d_set_time.argtypes = h + [C.c_double]
    L.eu3d_get_dt.argtypes = h + [_dp]
    L.eu3d_cfl.argtypes = h + [C.c_double, C.c_double, _dp]
    L.eu3d_boundary.argtypes = h + [C.c_int]
    L.eu3d_advection.argtypes = h + [C.c_int, C.c_int]
    for fn in ("eu3d_update_after_adv", "eu3d_update_after_cs", "eu3d_react_imex", "eu3d_synchronize",
               "eu3d_reset_status"):
        getattr(L, fn).argtypes = h
    L.eu3d_react_trapezoid.argtypes = h + [C.c_int]
    L.eu3d_step.argtypes = h + [C.POINTER(StepDesc)]
    L.eu3d_run.argtypes = h + [C.POINTER(StepDesc), C.c_int, C.c_int]
    L.eu3d_get_status.argtypes = h + [C.POINTER(Status)]
    L.eu3d_stream.argtypes = h
    L.eu3d_stream.restype = C.c_void_p
    L.eu3d_cfl_noalloc.argtypes = [C.c_void_p] * 6 + [C.c_int] * 4 + [C.c_longlong] * 2 + [C.c_double] * 3 + \
        [C.c_int, C.c_double, C.c_double, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]
    L.eu3d_gemm_bf16.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int,
                                 C.c_void_p, C.c_void_p]
    L.eu3d_profile_enable.argtypes = h + [C.c_int]
    L.eu3d_profile_read.argtypes = h + [C.c_char_p, C.c_size_t, _dp, C.POINTER(C.c_longlong), C.c_int,
                                        C.POINTER(C.c_int)]
    for fn in EXPORTS:
        if fn not in ("eu3d_last_error", "eu3d_stream"):
            getattr(L, fn).restype = C.c_int
    if path is None:
        _LIB = L
    return L


def _check(rc: int):
    if rc != 0:
        msg = load_library().eu3d_last_error().decode(errors="replace")
        raise Eu3dError(f"eu3d error {rc}: {msg}")


class DeviceFlowfield:
    """One rank's flowfield on the GPU (Flowfield + Reaction of the reference).

    mech: readers.Mechanism; grid: readers.Grid; quirks: QUIRKS_REF or
    QUIRKS_FIXED (or any EU3D_Q_* set); flux_bits: 64 (FP64 flux, parity
    path) or 32 (FP32 reconstruction/AUSM, FP64 state).
    """

    def __init__(self, mech, grid, quirks: int = QUIRKS_FIXED, flux_bits: int = 64, device: int = 0):
        self.L = load_library()
        self.mech, self.grid = mech, grid
        self.NS = mech.NS
        self.NI, self.NJ, self.NK = grid.ni + 2 * grid.bc, grid.nj + 2 * grid.bc, grid.nk + 2 * grid.bc
        keep = []

        def p(a):
            a = np.ascontiguousarray(a, dtype=np.float64)
            keep.append(a)
            return a.ctypes.data_as(_dp)

        d = Desc(grid.ni, grid.nj, grid.nk, grid.bc, p(grid.xnode), p(grid.ynode), p(grid.znode), mech.NS, mech.NR,
                 p(mech.stoi_f), p(mech.stoi_b), p(mech.react_tb), p(mech.af), p(mech.bf), p(mech.eaf),
                 p(mech.c0), p(mech.c1), p(mech.mw), quirks, flux_bits, device)
        self.h = C.c_void_p()
        _check(self.L.eu3d_create(C.byref(d), C.byref(self.h)))
        self.quirks, self.flux_bits = quirks, flux_bits

    def close(self):
        if getattr(self, "h", None):
            self.L.eu3d_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ------------------------------------------------------------ transfer
    def shape(self, name):
        n = {"Yi": self.NS, "Mc": self.NS, "Di": self.NS, "CS": self.NS + 4, "RHS": self.NS + 4}.get(name, 1)
        return (self.NI, self.NJ, self.NK) if n == 1 else (self.NI, self.NJ, self.NK, n)

    def upload(self, name: str, a: np.ndarray):
        if name not in UPLOADABLE:
            raise Eu3dError(f"{name} cannot be uploaded")
        a = np.ascontiguousarray(a, dtype=np.float64)
        if a.shape != self.shape(name):
            raise Eu3dError(f"{name}: shape {a.shape} != {self.shape(name)}")
        _check(self.L.eu3d_upload_field(self.h, FIELDS[name], a.ctypes.data_as(_dp)))

    def download(self, name: str, out: Optional[np.ndarray] = None) -> np.ndarray:
        if out is None:
            out = np.empty(self.shape(name), dtype=np.float64)
        _check(self.L.eu3d_download_field(self.h, FIELDS[name], out.ctypes.data_as(_dp)))
        return out

    def upload_state(self, src, names=("U", "V", "W", "P", "D", "T", "H", "Gamma", "E", "Yi", "CS")):
        """Copy a host state (any object with .view(name), e.g. an oracle field)."""
        for n in names:
            self.upload(n, src.view(n))

    def set_inflow(self, U, V, W, P, D, T, H, E, G, Y):
        args = [np.ascontiguousarray(x, dtype=np.float64) for x in (U, V, W, P, D, T, H, E, G, Y)]
        _check(self.L.eu3d_set_inflow(self.h, *[x.ctypes.data_as(_dp) for x in args]))

    def init_uniform(self, P, T, U, V, W, Y):
        y = np.ascontiguousarray(Y, dtype=np.float64)
        _check(self.L.eu3d_init_uniform(self.h, P, T, U, V, W, y.ctypes.data_as(_dp)))

    def set_wedge(self, x0, y0, tan_angle, enabled=True):
        _check(self.L.eu3d_set_wedge(self.h, x0, y0, tan_angle, 1 if enabled else 0))

    # ---------------------------------------------------------- operations
    @property
    def dt(self) -> float:
        v = C.c_double()
        _check(self.L.eu3d_get_dt(self.h, C.byref(v)))
        return v.value

    @dt.setter
    def dt(self, v: float):
        _check(self.L.eu3d_set_dt(self.h, v))

    def set_time(self, t: float):
        _check(self.L.eu3d_set_time(self.h, t))

    def cfl(self, cfl: float, final_time: float) -> float:
        v = C.c_double()
        _check(self.L.eu3d_cfl(self.h, cfl, final_time, C.byref(v)))
        return v.value

    def boundary(self, kind: int):
        _check(self.L.eu3d_boundary(self.h, kind))

    def advection(self, timeadv: int = ADV_EE, diff: int = DIFF_MUSCL2):
        _check(self.L.eu3d_advection(self.h, timeadv, diff))

    def update_after_adv(self):
        _check(self.L.eu3d_update_after_adv(self.h))

    def update_after_cs(self):
        _check(self.L.eu3d_update_after_cs(self.h))

    def imex(self):
        _check(self.L.eu3d_react_imex(self.h))

    def trapezoid(self, type_: int):
        _check(self.L.eu3d_react_trapezoid(self.h, type_))

    def step(self, react=REACT_IMEX, type_=0, timeadv=ADV_EE, diff=DIFF_MUSCL2, bc_kind=BC_RSBI, cfl=0.0,
             final_time=1.0):
        s = StepDesc(react, type_, timeadv, diff, bc_kind, cfl, final_time)
        _check(self.L.eu3d_step(self.h, C.byref(s)))

    def run(self, nsteps, react=REACT_IMEX, type_=0, timeadv=ADV_EE, diff=DIFF_MUSCL2, bc_kind=BC_RSBI, cfl=0.0,
            final_time=1.0, check_time=False):
        s = StepDesc(react, type_, timeadv, diff, bc_kind, cfl, final_time)
        _check(self.L.eu3d_run(self.h, C.byref(s), nsteps, 1 if check_time else 0))

    def synchronize(self):
        _check(self.L.eu3d_synchronize(self.h))

    def status(self) -> dict:
        s = Status()
        _check(self.L.eu3d_get_status(self.h, C.byref(s)))
        return s.as_dict()

    def reset_status(self):
        _check(self.L.eu3d_reset_status(self.h))

    def profile(self, on: bool = True):
        _check(self.L.eu3d_profile_enable(self.h, 1 if on else 0))

    def profile_read(self) -> dict:
        """{kernel name: (total ms, launches)} since the previous read."""
        cap, mk = 4096, 64
        names = C.create_string_buffer(cap)
        ms = (C.c_double * mk)()
        cnt = (C.c_longlong * mk)()
        n = C.c_int()
        _check(self.L.eu3d_profile_read(self.h, names, cap, ms, cnt, mk, C.byref(n)))
        keys = names.value.decode().split("\n")
        return {keys[i]: (ms[i], cnt[i]) for i in range(n.value)}

    @property
    def stream(self) -> int:
        return self.L.eu3d_stream(self.h)
