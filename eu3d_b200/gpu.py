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
REACT_TRAPEZOID, REACT_IMEX, REACT_NONE, REACT_SURROGATE, REACT_ADAPTIVE = 0, 1, 2, 3, 4
DIFF_MUSCL1, DIFF_MUSCL2, DIFF_WENO = 0, 1, 2
ADV_EE, ADV_TVD_RK3, ADV_SSPRK2, ADV_SSPRK3 = 0, 1, 2, 3

FIELDS = {"U": 0, "V": 1, "W": 2, "P": 3, "D": 4, "T": 5, "H": 6, "Gamma": 7, "E": 8, "Yi": 9, "CS": 10, "RHS": 11,
          "C": 12, "Mc": 13, "Di": 14, "Nchem": 15}
UPLOADABLE = ("U", "V", "W", "P", "D", "T", "H", "Gamma", "E", "Yi", "CS", "RHS")

EXPORTS = ["eu3d_last_error", "eu3d_create", "eu3d_destroy", "eu3d_upload_field", "eu3d_download_field",
           "eu3d_set_inflow", "eu3d_init_uniform", "eu3d_set_wedge", "eu3d_set_dt", "eu3d_set_time", "eu3d_get_dt", "eu3d_cfl",
           "eu3d_boundary", "eu3d_advection", "eu3d_update_after_adv", "eu3d_update_after_cs", "eu3d_react_imex",
           "eu3d_react_trapezoid", "eu3d_step", "eu3d_run", "eu3d_synchronize", "eu3d_get_status",
           "eu3d_reset_status", "eu3d_stream", "eu3d_profile_enable", "eu3d_profile_read", "eu3d_cfl_noalloc",
           "eu3d_gemm_bf16", "eu3d_sur_create", "eu3d_sur_destroy", "eu3d_sur_reset_dataset",
           "eu3d_sur_dataset_size", "eu3d_sur_add_random", "eu3d_sur_add_snapshot", "eu3d_sur_label",
           "eu3d_sur_get_dataset", "eu3d_sur_set_norm", "eu3d_sur_get_norm", "eu3d_sur_set_params",
           "eu3d_sur_get_params", "eu3d_sur_train", "eu3d_sur_loss_grad", "eu3d_sur_predict", "eu3d_sur_infer",
           "eu3d_set_surrogate", "eu3d_set_surrogate_gate", "eu3d_react_surrogate", "eu3d_set_tuning",
           "eu3d_set_wait_limit", "eu3d_get_tuning", "eu3d_autotune",
           "eu3d_set_elements", "eu3d_set_adaptive", "eu3d_react_adaptive", "eu3d_halo_bytes", "eu3d_halo_pack",
           "eu3d_halo_unpack", "eu3d_cfl_local", "eu3d_dt_device", "eu3d_advance_time", "eu3d_wedge_fill",
           "eu3d_step_part", "eu3d_write_tecplot", "eu3d_write_wait", "eu3d_tecplot_write_host", "eu3d_dlb_plan",
           "eu3d_dlb_select_rows", "eu3d_chem_load", "eu3d_dlb_select", "eu3d_dlb_pack", "eu3d_dlb_guest",
           "eu3d_dlb_unpack", "eu3d_sur_load", "eu3d_sdlb_select", "eu3d_sdlb_pack", "eu3d_sdlb_guest",
           "eu3d_sdlb_unpack"]

PART_STAGE1, PART_STAGE2, PART_REACT, PART_STAGE3, PART_CHEM_PREDICT, PART_CHEM_WORK = 0, 1, 2, 3, 4, 5
PART_SUR_PREDICT, PART_SUR_WORK = 6, 7
DLB_OUT_FIELDS, DLB_BACK_FIELDS, DLB_MAX_TRANSFERS = 15, 32, 64
SDLB_OUT_FIELDS, SDLB_BACK_FIELDS = 16, 31

SUR_NPARAM = 37264
SUR_NORM_LEN = 80


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
                ("surrogate_fallback", C.c_longlong), ("dt", C.c_double), ("time", C.c_double),
                ("surrogate_audited", C.c_longlong), ("surrogate_audit_max_dT", C.c_double),
                ("surrogate_rejects", C.c_longlong * 4), ("wait_timeouts", C.c_longlong),
                ("surrogate_frozen", C.c_longlong), ("frozen_audited", C.c_longlong),
                ("frozen_audit_max_dT", C.c_double), ("drain_timeouts", C.c_longlong)]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_}
        d["surrogate_rejects"] = list(d["surrogate_rejects"])
        return d


class Tuning(C.Structure):
    _fields_ = [("flux_kz", C.c_int), ("chem_queue", C.c_int), ("queue_blocks", C.c_int), ("flux_stage", C.c_int),
                ("sur_fused", C.c_int), ("adapt_queue", C.c_int), ("cell_blocks", C.c_int),
                ("gate_fused", C.c_int)]

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
    _fp = C.POINTER(C.c_float)
    L.eu3d_sur_create.argtypes = h + [C.c_longlong, _dp, C.POINTER(C.c_void_p)]
    L.eu3d_sur_destroy.argtypes = h
    L.eu3d_sur_reset_dataset.argtypes = h
    L.eu3d_sur_dataset_size.argtypes = h + [C.POINTER(C.c_longlong)]
    L.eu3d_sur_add_random.argtypes = h + [C.c_longlong, _dp, C.POINTER(C.c_int), C.c_ulonglong]
    L.eu3d_sur_add_snapshot.argtypes = h + [C.c_void_p, C.c_longlong, C.c_longlong, C.c_longlong, C.c_double,
                                            C.c_double, C.c_double, C.c_double, C.c_ulonglong]
    L.eu3d_sur_label.argtypes = h + [C.c_int, C.c_int, C.c_double, C.POINTER(C.c_longlong)]
    L.eu3d_sur_get_dataset.argtypes = h + [C.c_longlong, C.c_longlong, _dp, _fp, _fp]
    L.eu3d_sur_set_norm.argtypes = h + [_fp]
    L.eu3d_sur_get_norm.argtypes = h + [_fp]
    L.eu3d_sur_set_params.argtypes = h + [_fp]
    L.eu3d_sur_get_params.argtypes = h + [_fp]
    L.eu3d_sur_train.argtypes = h + [C.c_int, C.c_int, C.c_float, C.c_float, C.c_int, C.c_ulonglong, _fp]
    L.eu3d_sur_loss_grad.argtypes = h + [_fp, _fp, C.c_int, _fp, _fp, _fp]
    L.eu3d_sur_predict.argtypes = h + [_fp, C.c_longlong, _fp]
    L.eu3d_sur_infer.argtypes = h + [C.c_void_p, C.c_longlong, C.c_void_p, C.c_void_p]
    L.eu3d_set_surrogate.argtypes = h + [C.c_void_p, C.c_int]
    L.eu3d_set_surrogate_gate.argtypes = h + [C.c_double, C.c_double, C.c_uint, C.c_int]
    L.eu3d_react_surrogate.argtypes = h
    L.eu3d_set_elements.argtypes = h + [_dp]
    L.eu3d_set_adaptive.argtypes = h + [C.c_double, C.c_double, C.c_int]
    L.eu3d_react_adaptive.argtypes = h
    L.eu3d_set_tuning.argtypes = h + [C.POINTER(Tuning)]
    L.eu3d_set_wait_limit.argtypes = h + [C.c_longlong]
    L.eu3d_get_tuning.argtypes = h + [C.POINTER(Tuning)]
    L.eu3d_autotune.argtypes = h + [C.POINTER(StepDesc), C.c_int, C.POINTER(Tuning), _dp]
    L.eu3d_halo_bytes.argtypes = h + [C.POINTER(C.c_longlong)]
    L.eu3d_halo_pack.argtypes = h + [C.c_int, C.c_int, C.c_void_p]
    L.eu3d_halo_unpack.argtypes = h + [C.c_int, C.c_void_p]
    L.eu3d_cfl_local.argtypes = h + [C.c_double, C.c_double]
    L.eu3d_dt_device.argtypes = h
    L.eu3d_advance_time.argtypes = h
    L.eu3d_wedge_fill.argtypes = h
    L.eu3d_step_part.argtypes = h + [C.POINTER(StepDesc), C.c_int]
    L.eu3d_write_tecplot.argtypes = h + [C.c_char_p, C.c_double, C.c_int]
    L.eu3d_write_wait.argtypes = h
    L.eu3d_tecplot_write_host.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_int, _dp, _dp, _dp, _dp,
                                          C.POINTER(C.c_int), C.c_double]
    _lp = C.POINTER(C.c_longlong)
    _ip = C.POINTER(C.c_int)
    L.eu3d_dlb_plan.argtypes = [_lp, C.c_int, C.c_int, _ip, _ip, _lp, _ip]
    L.eu3d_dlb_select_rows.argtypes = [_lp, C.c_longlong, C.c_int, _lp, _lp, _lp]
    L.eu3d_chem_load.argtypes = h + [_lp]
    L.eu3d_dlb_select.argtypes = h + [C.c_int, _lp, _lp, _lp]
    L.eu3d_dlb_pack.argtypes = h + [C.c_void_p]
    L.eu3d_dlb_guest.argtypes = h + [C.c_int, _lp, C.c_void_p, C.c_void_p]
    L.eu3d_dlb_unpack.argtypes = h + [C.c_void_p]
    L.eu3d_sur_load.argtypes = h + [_lp]
    L.eu3d_sdlb_select.argtypes = h + [C.c_int, _lp, _lp]
    L.eu3d_sdlb_pack.argtypes = h + [C.c_void_p]
    L.eu3d_sdlb_guest.argtypes = h + [C.c_int, _lp, C.c_void_p, C.c_void_p]
    L.eu3d_sdlb_unpack.argtypes = h + [C.c_void_p]
    L.eu3d_profile_enable.argtypes = h + [C.c_int]
    L.eu3d_profile_read.argtypes = h + [C.c_char_p, C.c_size_t, _dp, C.POINTER(C.c_longlong), C.c_int,
                                        C.POINTER(C.c_int)]
    for fn in EXPORTS:
        if fn not in ("eu3d_last_error", "eu3d_stream", "eu3d_dt_device"):
            getattr(L, fn).restype = C.c_int
    L.eu3d_dt_device.restype = C.c_void_p
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
        self.device = device
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

    @property
    def time(self) -> float:
        return self.status()["time"]

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

    def set_elements(self, atoms):
        """(3, NS) H, O, N atom counts per species (adaptive chemistry, surrogate)."""
        a = np.ascontiguousarray(atoms, dtype=np.float64)
        if a.shape != (3, self.NS):
            raise Eu3dError("atoms must be (3, NS)")
        _check(self.L.eu3d_set_elements(self.h, a.ctypes.data_as(_dp)))

    def set_adaptive(self, rel: float = 0.02, amp: float = 0.5, nmax: int = 1024):
        _check(self.L.eu3d_set_adaptive(self.h, rel, amp, nmax))

    def react_adaptive(self):
        _check(self.L.eu3d_react_adaptive(self.h))

    def set_surrogate(self, sur, audit_stride: int = 0):
        """Use a trained DeviceSurrogate (None: none) for REACT_SURROGATE steps."""
        _check(self.L.eu3d_set_surrogate(self.h, sur.s if sur is not None else None, audit_stride))
        self._sur = sur  # keeps the surrogate alive while attached

    def set_surrogate_gate(self, t_frozen: float, y_max: float = 0.0, species=(), audit_stride: int = 0):
        """Frozen-chemistry gate of REACT_SURROGATE steps: fluid cells below
        t_frozen [K] whose mass fractions summed over `species` (names) are at
        most y_max skip the network.  t_frozen = 0 turns it off."""
        mask = 0
        for n in species:
            mask |= 1 << self.mech.species.index(n)
        _check(self.L.eu3d_set_surrogate_gate(self.h, float(t_frozen), float(y_max), mask, int(audit_stride)))

    def react_surrogate(self):
        _check(self.L.eu3d_react_surrogate(self.h))

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

    def write_tecplot(self, path: str, wait_time: float = 0.0, background: bool = False):
        """The reference's Tecplot block result file of this handle (Euler::Output)."""
        _check(self.L.eu3d_write_tecplot(self.h, path.encode(), wait_time, 1 if background else 0))

    def write_wait(self):
        _check(self.L.eu3d_write_wait(self.h))

    # ---- x-slab decomposition (one handle per rank; eu3d_b200.slabs drives them)
    def halo_bytes(self) -> int:
        n = C.c_longlong()
        _check(self.L.eu3d_halo_bytes(self.h, C.byref(n)))
        return n.value

    def halo_pack(self, side: int, dst_ptr: int, overlap: int = 0):
        """Pack the two interior planes next to face `side` (0 low x, 1 high x;
        overlap 1: past a node shared with the neighbour) into the device
        buffer at dst_ptr (eu3d_halo_bytes bytes)."""
        _check(self.L.eu3d_halo_pack(self.h, side, overlap, C.c_void_p(dst_ptr)))

    def halo_unpack(self, side: int, src_ptr: int):
        """Fill the two ghost planes of face `side` from the device buffer at src_ptr."""
        _check(self.L.eu3d_halo_unpack(self.h, side, C.c_void_p(src_ptr)))

    # ---- load balancing of the adaptive trapezoid across ranks (eu3d_b200.slabs drives it)
    def chem_load(self) -> int:
        v = C.c_longlong()
        _check(self.L.eu3d_chem_load(self.h, C.byref(v)))
        return v.value

    def dlb_select(self, amounts):
        """Rows for this rank's transfers: (cells, moved load) per transfer."""
        n = len(amounts)
        a = np.ascontiguousarray(amounts, dtype=np.int64)
        cells = np.zeros(n, dtype=np.int64)
        moved = np.zeros(n, dtype=np.int64)
        lp = C.POINTER(C.c_longlong)
        _check(self.L.eu3d_dlb_select(self.h, n, a.ctypes.data_as(lp), cells.ctypes.data_as(lp),
                                      moved.ctypes.data_as(lp)))
        return cells, moved

    def dlb_pack(self, dst_ptr: int):
        _check(self.L.eu3d_dlb_pack(self.h, C.c_void_p(dst_ptr)))

    def dlb_guest(self, seg_cells, src_ptr: int, dst_ptr: int):
        s = np.ascontiguousarray(seg_cells, dtype=np.int64)
        _check(self.L.eu3d_dlb_guest(self.h, len(s), s.ctypes.data_as(C.POINTER(C.c_longlong)), C.c_void_p(src_ptr),
                                     C.c_void_p(dst_ptr)))

    def dlb_unpack(self, src_ptr: int):
        _check(self.L.eu3d_dlb_unpack(self.h, C.c_void_p(src_ptr)))

    # ---- load balancing of the learned chemistry's FP64 fallback across ranks
    def sur_load(self) -> int:
        """The fallback list length after PART_SUR_PREDICT (synchronises)."""
        v = C.c_longlong()
        _check(self.L.eu3d_sur_load(self.h, C.byref(v)))
        return v.value

    def sdlb_select(self, amounts):
        """Cells of this rank's transfers, taken from the end of its fallback list."""
        n = len(amounts)
        a = np.ascontiguousarray(amounts, dtype=np.int64)
        cells = np.zeros(n, dtype=np.int64)
        lp = C.POINTER(C.c_longlong)
        _check(self.L.eu3d_sdlb_select(self.h, n, a.ctypes.data_as(lp), cells.ctypes.data_as(lp)))
        return cells

    def sdlb_pack(self, dst_ptr: int):
        _check(self.L.eu3d_sdlb_pack(self.h, C.c_void_p(dst_ptr)))

    def sdlb_guest(self, seg_cells, src_ptr: int, dst_ptr: int):
        s = np.ascontiguousarray(seg_cells, dtype=np.int64)
        _check(self.L.eu3d_sdlb_guest(self.h, len(s), s.ctypes.data_as(C.POINTER(C.c_longlong)),
                                      C.c_void_p(src_ptr), C.c_void_p(dst_ptr)))

    def sdlb_unpack(self, src_ptr: int):
        _check(self.L.eu3d_sdlb_unpack(self.h, C.c_void_p(src_ptr)))

    def cfl_local(self, cfl: float, final_time: float):
        """This rank's CFL dt into the device scalar (time not advanced)."""
        _check(self.L.eu3d_cfl_local(self.h, cfl, final_time))

    @property
    def dt_device_ptr(self) -> int:
        """Device address of dt (one FP64), for an in-place all-reduce MIN."""
        return self.L.eu3d_dt_device(self.h)

    def advance_time(self):
        _check(self.L.eu3d_advance_time(self.h))

    def wedge_fill(self):
        _check(self.L.eu3d_wedge_fill(self.h))

    def step_part(self, part: int, react=REACT_IMEX, type_=0, timeadv=ADV_EE, diff=DIFF_MUSCL2, bc_kind=BC_RSBI,
                  cfl=0.0, final_time=1.0):
        s = StepDesc(react, type_, timeadv, diff, bc_kind, cfl, final_time)
        _check(self.L.eu3d_step_part(self.h, C.byref(s), part))

    def tuning(self) -> dict:
        t = Tuning()
        _check(self.L.eu3d_get_tuning(self.h, C.byref(t)))
        return t.as_dict()

    def set_tuning(self, flux_kz=None, chem_queue=None, queue_blocks=None, flux_stage=None, sur_fused=None,
                   adapt_queue=None, cell_blocks=None, gate_fused=None):
        t = Tuning(**self.tuning())
        if gate_fused is not None:
            t.gate_fused = 1 if gate_fused else 0
        if cell_blocks is not None:
            t.cell_blocks = int(cell_blocks)
        if adapt_queue is not None:
            t.adapt_queue = 1 if adapt_queue else 0
        if flux_kz is not None:
            t.flux_kz = flux_kz
        if chem_queue is not None:
            t.chem_queue = int(chem_queue)
        if queue_blocks is not None:
            t.queue_blocks = queue_blocks
        if flux_stage is not None:
            t.flux_stage = int(flux_stage)
        if sur_fused is not None:
            t.sur_fused = 1 if sur_fused else 0
        _check(self.L.eu3d_set_tuning(self.h, C.byref(t)))

    def autotune(self, steps=3, react=REACT_IMEX, type_=0, timeadv=ADV_EE, diff=DIFF_MUSCL2, bc_kind=BC_RSBI,
                 cfl=0.0, final_time=1.0):
        """Time the candidate launch settings on the current state (which is
        restored) and keep the fastest; returns (setting, ms per step)."""
        s = StepDesc(react, type_, timeadv, diff, bc_kind, cfl, final_time)
        t = Tuning()
        ms = C.c_double()
        _check(self.L.eu3d_autotune(self.h, C.byref(s), steps, C.byref(t), C.byref(ms)))
        return t.as_dict(), ms.value

    def set_wait_limit(self, tries: int = 1 << 19):
        """Bound of the TMA-fed flux kernel's copy waits (0: give up at once)."""
        _check(self.L.eu3d_set_wait_limit(self.h, int(tries)))

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


def _f32(a, shape=None):
    a = np.ascontiguousarray(a, dtype=np.float32)
    if shape is not None and a.shape != shape:
        raise Eu3dError(f"shape {a.shape} != {shape}")
    return a


class DeviceSurrogate:
    """The learned chemistry surrogate's device side (training set, labels,
    parameters, training and inference), bound to a DeviceFlowfield's device,
    mechanism and quirk policy."""

    def __init__(self, dev: DeviceFlowfield, capacity: int, atoms: np.ndarray):
        self.L = dev.L
        self.dev = dev
        self.NS = dev.NS
        a = np.ascontiguousarray(atoms, dtype=np.float64)
        if a.shape != (3, dev.NS):
            raise Eu3dError("atoms must be (3, NS): H, O, N counts per species")
        self.s = C.c_void_p()
        _check(self.L.eu3d_sur_create(dev.h, int(capacity), a.ctypes.data_as(_dp), C.byref(self.s)))
        self.capacity = int(capacity)

    def close(self):
        if getattr(self, "s", None):
            self.L.eu3d_sur_destroy(self.s)
            self.s = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ------------------------------------------------------------ dataset
    def reset_dataset(self):
        _check(self.L.eu3d_sur_reset_dataset(self.s))

    @property
    def size(self) -> int:
        n = C.c_longlong()
        _check(self.L.eu3d_sur_dataset_size(self.s, C.byref(n)))
        return n.value

    def add_random(self, n: int, env, species_index, seed: int):
        e = np.ascontiguousarray(env, dtype=np.float64)
        sp = (C.c_int * 9)(*[int(x) for x in species_index])
        _check(self.L.eu3d_sur_add_random(self.s, int(n), e.ctypes.data_as(_dp), sp, int(seed)))

    def add_snapshot(self, src: DeviceFlowfield, n: int, stride: int, offset: int, jitter_T: float,
                     jitter_lnp: float, lndt_lo: float, lndt_hi: float, seed: int):
        _check(self.L.eu3d_sur_add_snapshot(self.s, src.h, int(n), int(stride), int(offset), jitter_T, jitter_lnp,
                                            lndt_lo, lndt_hi, int(seed)))

    def label(self, kind: int = REACT_IMEX, cap: int = 4096, proj_eps: float = 1e-4) -> int:
        nv = C.c_longlong()
        _check(self.L.eu3d_sur_label(self.s, kind, cap, proj_eps, C.byref(nv)))
        return nv.value

    def dataset(self, first: int = 0, count: Optional[int] = None, states: bool = False):
        count = self.size - first if count is None else count
        X = np.empty((count, 12), np.float32)
        Lb = np.empty((count, 12), np.float32)
        S = np.empty((count, 12), np.float64) if states else None
        _check(self.L.eu3d_sur_get_dataset(self.s, first, count, S.ctypes.data_as(_dp) if states else None,
                                           X.ctypes.data_as(C.POINTER(C.c_float)),
                                           Lb.ctypes.data_as(C.POINTER(C.c_float))))
        return (X, Lb, S) if states else (X, Lb)

    # ------------------------------------------------------------- model
    def set_norm(self, norm):
        a = _f32(norm, (SUR_NORM_LEN,))
        _check(self.L.eu3d_sur_set_norm(self.s, a.ctypes.data_as(C.POINTER(C.c_float))))

    def get_norm(self) -> np.ndarray:
        a = np.empty(SUR_NORM_LEN, np.float32)
        _check(self.L.eu3d_sur_get_norm(self.s, a.ctypes.data_as(C.POINTER(C.c_float))))
        return a

    def set_params(self, p):
        a = _f32(p, (SUR_NPARAM,))
        _check(self.L.eu3d_sur_set_params(self.s, a.ctypes.data_as(C.POINTER(C.c_float))))

    def get_params(self) -> np.ndarray:
        a = np.empty(SUR_NPARAM, np.float32)
        _check(self.L.eu3d_sur_get_params(self.s, a.ctypes.data_as(C.POINTER(C.c_float))))
        return a

    def train(self, steps: int, batch: int, lr_max: float, lr_min: float, warmup: int, seed: int) -> np.ndarray:
        losses = np.zeros(max(steps, 1), np.float32)
        _check(self.L.eu3d_sur_train(self.s, steps, batch, lr_max, lr_min, warmup, int(seed),
                                     losses.ctypes.data_as(C.POINTER(C.c_float))))
        return losses[:steps]

    def loss_grad(self, X, Y):
        B = X.shape[0]
        X = _f32(X, (B, 16))
        Y = _f32(Y, (B, 16))
        loss = np.zeros(1, np.float32)
        grad = np.empty(SUR_NPARAM, np.float32)
        out = np.empty((B, 16), np.float32)
        fp = C.POINTER(C.c_float)
        _check(self.L.eu3d_sur_loss_grad(self.s, X.ctypes.data_as(fp), Y.ctypes.data_as(fp), B,
                                         loss.ctypes.data_as(fp), grad.ctypes.data_as(fp), out.ctypes.data_as(fp)))
        return float(loss[0]), grad, out

    def predict(self, X) -> np.ndarray:
        n = X.shape[0]
        X = _f32(X, (n, 16))
        out = np.empty((n, 16), np.float32)
        fp = C.POINTER(C.c_float)
        _check(self.L.eu3d_sur_predict(self.s, X.ctypes.data_as(fp), n, out.ctypes.data_as(fp)))
        return out

    def infer_device(self, x_ptr: int, n: int, out_ptr: int, stream: int = 0):
        _check(self.L.eu3d_sur_infer(self.s, x_ptr, n, out_ptr, stream or None))


def tecplot_path(numprocs: int, react: str, num: int, rank: int) -> str:
    """The reference's result-file name (Euler::Output, src/Euler.cpp:802-805):
    output_<numprocs>/results/Series<react><num>_<rank>.dat on one rank,
    output_<numprocs>/results<react><num>_<rank>.dat on several."""
    if numprocs == 1:
        return f"./output_{numprocs}/results/Series{react}{num}_{rank}.dat"
    return f"./output_{numprocs}/results{react}{num}_{rank}.dat"


def write_tecplot_host(path: str, grid, cols, lcol, wait_time: float = 0.0):
    """The Tecplot block file from host arrays: cols (13, n) T D P U V Ma Y1..Y7 and
    lcol (n,) counts, both in the file's cell order (k outer, i inner)."""
    L = load_library()
    n = grid.ni * grid.nj * grid.nk
    c = np.ascontiguousarray(cols, dtype=np.float64)
    lc = np.ascontiguousarray(lcol, dtype=np.int32)
    if c.shape != (13, n) or lc.shape != (n,):
        raise Eu3dError("cols must be (13, n) and lcol (n,)")
    xs = [np.ascontiguousarray(a, dtype=np.float64) for a in (grid.xnode, grid.ynode, grid.znode)]
    _check(L.eu3d_tecplot_write_host(path.encode(), grid.ni, grid.nj, grid.nk, grid.bc,
                                     *(a.ctypes.data_as(_dp) for a in xs), c.ctypes.data_as(_dp),
                                     lc.ctypes.data_as(C.POINTER(C.c_int)), wait_time))


def dlb_plan(loads):
    """DynamicLoadBalancer::DLBPriorityQueue (src/LoadBalance.cpp:8-59) through
    the library: [(sender, receiver, amount)] in the reference's order."""
    L = load_library()
    a = np.ascontiguousarray(loads, dtype=np.int64)
    n = len(a)
    cap = max(1, n * n)
    snd = np.zeros(cap, dtype=np.int32)
    rcv = np.zeros(cap, dtype=np.int32)
    amt = np.zeros(cap, dtype=np.int64)
    m = C.c_int()
    lp, ip = C.POINTER(C.c_longlong), C.POINTER(C.c_int)
    _check(L.eu3d_dlb_plan(a.ctypes.data_as(lp), n, cap, snd.ctypes.data_as(ip), rcv.ctypes.data_as(ip),
                           amt.ctypes.data_as(lp), C.byref(m)))
    return [(int(snd[t]), int(rcv[t]), int(amt[t])) for t in range(m.value)]


def load_degree(loads) -> float:
    """(max - mean) / max of the loads, the mean an integer one as the
    reference's Array::AveValue (src/Euler.cpp:394)."""
    a = [int(v) for v in loads]
    mx = max(a)
    return 0.0 if mx <= 0 else (mx - sum(a) // len(a)) / mx


def dlb_select_rows(rowload, amounts):
    """The row picker of eu3d_dlb_select: (row bounds, moved load per transfer)."""
    L = load_library()
    r = np.ascontiguousarray(rowload, dtype=np.int64)
    a = np.ascontiguousarray(amounts, dtype=np.int64)
    bounds = np.zeros(len(a) + 1, dtype=np.int64)
    moved = np.zeros(len(a), dtype=np.int64)
    lp = C.POINTER(C.c_longlong)
    _check(L.eu3d_dlb_select_rows(r.ctypes.data_as(lp), len(r), len(a), a.ctypes.data_as(lp),
                                  bounds.ctypes.data_as(lp), moved.ctypes.data_as(lp)))
    return bounds, moved
