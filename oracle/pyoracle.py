"""ctypes access to the oracle libraries (TEST INFRASTRUCTURE ONLY).

* ``Oracle`` wraps ``oracle/liboracle.so``, the plain-C restatement of the
  reference's hot path (eu3d_oracle.c).
* ``RefCase`` wraps ``oracle/_ref/libeu3d_ref.so``, the reference's own
  sources compiled unmodified with a friend-class harness (ref_harness.cpp).

Only tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of bench.py
import this module.  Both wrappers expose every field as a numpy view in the
reference layout: 3D (NI, NJ, NK), 4D (NI, NJ, NK, n) with the last index
fastest.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libeu3d_ref.so")
REF_FIXED_SO = os.path.join(HERE, "_ref", "libeu3d_ref_fixed.so")

MAXS, MAXR = 16, 24
_dp = C.POINTER(C.c_double)


def build_oracle(ref: bool = False) -> None:
    target = "all" if ref else "oracle"
    subprocess.run(["make", "-s", "-C", HERE, target], check=True)


class OrcMech(C.Structure):
    _fields_ = [("NS", C.c_int), ("NR", C.c_int),
                ("stoi_f", C.c_double * (MAXS * MAXR)), ("stoi_b", C.c_double * (MAXS * MAXR)),
                ("react_tb", C.c_double * (MAXS * MAXR)),
                ("af", C.c_double * MAXR), ("bf", C.c_double * MAXR), ("eaf", C.c_double * MAXR),
                ("c0", C.c_double * (9 * MAXS)), ("c1", C.c_double * (9 * MAXS)),
                ("mw", C.c_double * MAXS), ("ri", C.c_double * MAXS)]


_F3 = ["U", "V", "W", "P", "D", "T", "C", "Ma", "Wav", "Rgas", "Cp", "H", "E", "Gamma"]
_F4S = ["Mc", "Yi", "Di"]
_F4V = ["CS", "RHS", "Partion_T", "F", "G", "Q"]
_INFLOW = ["Uint", "Vint", "Wint", "Pint", "Dint", "Tint", "Hint", "Eint", "Gint", "Yint"]


class OrcField(C.Structure):
    _fields_ = ([("ni", C.c_int), ("nj", C.c_int), ("nk", C.c_int), ("bc", C.c_int), ("NS", C.c_int),
                 ("NI", C.c_int), ("NJ", C.c_int), ("NK", C.c_int), ("quirks", C.c_uint),
                 ("dt", C.c_double), ("time", C.c_double),
                 ("xnode", _dp), ("ynode", _dp), ("znode", _dp)]
                + [(n, _dp) for n in _F3] + [(n, _dp) for n in _F4S] + [(n, _dp) for n in _F4V]
                + [("CMS", _dp), ("MDd", _dp), ("Nchem", C.POINTER(C.c_int))]
                + [(n, _dp) for n in _INFLOW])


def mech_struct(mech) -> OrcMech:
    m = OrcMech()
    m.NS, m.NR = mech.NS, mech.NR
    NS, NR = mech.NS, mech.NR
    for name in ("stoi_f", "stoi_b", "react_tb"):
        a = np.asarray(getattr(mech, name), dtype=np.float64).reshape(NS * NR)
        C.memmove(getattr(m, name), a.ctypes.data, a.nbytes)
    for name in ("af", "bf", "eaf"):
        a = np.ascontiguousarray(getattr(mech, name), dtype=np.float64)
        C.memmove(getattr(m, name), a.ctypes.data, a.nbytes)
    for name in ("c0", "c1"):
        a = np.ascontiguousarray(getattr(mech, name), dtype=np.float64).reshape(9 * NS)
        C.memmove(getattr(m, name), a.ctypes.data, a.nbytes)
    mw = np.ascontiguousarray(mech.mw, dtype=np.float64)
    C.memmove(m.mw, mw.ctypes.data, mw.nbytes)
    # Ri = R / Mw, as ReactionInitial (src/Reaction.cpp:352-353)
    ri = np.array([8.31434 / x for x in mech.mw], dtype=np.float64)
    C.memmove(m.ri, ri.ctypes.data, ri.nbytes)
    return m


def _lib(path):
    lib = C.CDLL(path)
    return lib


class Oracle:
    """One oracle field (state of one rank) plus its mechanism."""

    _lib = None

    @classmethod
    def lib(cls):
        if cls._lib is None:
            if not os.path.exists(ORACLE_SO):
                build_oracle()
            L = _lib(ORACLE_SO)
            L.orc_field_alloc.argtypes = [C.POINTER(OrcField), C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]
            L.orc_field_free.argtypes = [C.POINTER(OrcField)]
            for fn in ("orc_getcpi",):
                getattr(L, fn).argtypes = [C.POINTER(OrcMech), C.c_double, C.c_double, C.c_int]
                getattr(L, fn).restype = C.c_double
            for fn in ("orc_gethi", "orc_getsi"):
                getattr(L, fn).argtypes = [C.POINTER(OrcMech), C.c_double, C.c_double, C.c_int, C.c_uint]
                getattr(L, fn).restype = C.c_double
            fm = [C.POINTER(OrcField), C.POINTER(OrcMech)]
            for fn in ("orc_update_after_adv", "orc_update_after_cs", "orc_get_partial_t", "orc_diagonalized",
                       "orc_update_imex", "orc_imex", "orc_prediction", "orc_explicit", "orc_prims_from_state"):
                getattr(L, fn).argtypes = fm
            L.orc_advection.argtypes = [C.POINTER(OrcField), C.c_int, C.c_int]
            L.orc_trapezoid.argtypes = fm + [C.c_int]
            L.orc_boundary.argtypes = fm + [C.c_int, _dp]
            L.orc_cfl.argtypes = [C.POINTER(OrcField), C.c_double, C.c_double]
            L.orc_step.argtypes = fm + [C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_int, _dp]
            L.orc_rsbi_initial.argtypes = fm + [C.c_double, C.c_double, C.c_double]
            L.orc_get_temp.argtypes = fm + [C.c_double, C.c_int, C.c_int, C.c_int, _dp]
            L.orc_get_temp.restype = C.c_double
            cls._lib = L
        return cls._lib

    def __init__(self, mech, grid, quirks: int):
        L = self.lib()
        self.mech = mech
        self.m = mech_struct(mech)
        self.f = OrcField()
        rc = L.orc_field_alloc(C.byref(self.f), grid.ni, grid.nj, grid.nk, grid.bc, mech.NS)
        if rc != 0:
            raise MemoryError("orc_field_alloc")
        self.f.quirks = quirks
        self.ni, self.nj, self.nk, self.bc, self.NS = grid.ni, grid.nj, grid.nk, grid.bc, mech.NS
        self.NI, self.NJ, self.NK = self.f.NI, self.f.NJ, self.f.NK
        self.view("xnode")[:] = grid.xnode
        self.view("ynode")[:] = grid.ynode
        self.view("znode")[:] = grid.znode

    def __del__(self):
        try:
            self.lib().orc_field_free(C.byref(self.f))
        except Exception:
            pass

    def view(self, name):
        NI, NJ, NK, NS = self.NI, self.NJ, self.NK, self.NS
        if name == "xnode":
            shape = (NI,)
        elif name == "ynode":
            shape = (NJ,)
        elif name == "znode":
            shape = (NK,)
        elif name in _F3:
            shape = (NI, NJ, NK)
        elif name in _F4S or name == "CMS":
            shape = (NI, NJ, NK, NS)
        elif name in _F4V or name == "MDd":
            shape = (NI, NJ, NK, NS + 4)
        elif name == "Nchem":
            return np.ctypeslib.as_array(self.f.Nchem, shape=(NI, NJ, NK))
        elif name == "Yint":
            shape = (self.nj, self.nk, NS)
        elif name in _INFLOW:
            shape = (self.nj, self.nk)
        else:
            raise KeyError(name)
        return np.ctypeslib.as_array(getattr(self.f, name), shape=shape)

    @property
    def dt(self):
        return self.f.dt

    @dt.setter
    def dt(self, v):
        self.f.dt = v

    @property
    def time(self):
        return self.f.time

    @time.setter
    def time(self, v):
        self.f.time = v

    def _fm(self):
        return C.byref(self.f), C.byref(self.m)

    def getcpi(self, T, R, sp):
        return self.lib().orc_getcpi(C.byref(self.m), T, R, sp)

    def gethi(self, T, R, sp):
        return self.lib().orc_gethi(C.byref(self.m), T, R, sp, self.f.quirks)

    def getsi(self, T, R, sp):
        return self.lib().orc_getsi(C.byref(self.m), T, R, sp, self.f.quirks)

    def advection(self, timeadv=0, diff=1):
        self.lib().orc_advection(C.byref(self.f), timeadv, diff)

    def update_after_adv(self):
        self.lib().orc_update_after_adv(*self._fm())

    def update_after_cs(self):
        self.lib().orc_update_after_cs(*self._fm())

    def partial_t(self):
        self.lib().orc_get_partial_t(*self._fm())

    def imex(self):
        self.lib().orc_imex(*self._fm())

    def trapezoid(self, type_):
        self.lib().orc_trapezoid(*self._fm(), type_)

    def prediction(self):
        self.lib().orc_prediction(*self._fm())

    def explicit(self):
        self.lib().orc_explicit(*self._fm())

    def boundary(self, kind, wedge=None):
        w = None if wedge is None else np.ascontiguousarray(wedge, dtype=np.float64)
        self._wedge_keep = w
        self.lib().orc_boundary(*self._fm(), kind, None if w is None else w.ctypes.data_as(_dp))

    def cfl(self, cfl, final_time):
        self.lib().orc_cfl(C.byref(self.f), cfl, final_time)

    def step(self, react, type_, timeadv, diff, cfl, final_time, bc_kind, wedge=None):
        w = None if wedge is None else np.ascontiguousarray(wedge, dtype=np.float64)
        self.lib().orc_step(*self._fm(), react, type_, timeadv, diff, cfl, final_time, bc_kind,
                            None if w is None else w.ctypes.data_as(_dp))

    def rsbi_initial(self, P_pre, T_pre, M_wave):
        self.lib().orc_rsbi_initial(*self._fm(), P_pre, T_pre, M_wave)

    def prims_from_state(self):
        self.lib().orc_prims_from_state(*self._fm())

    def get_temp(self, T, i, j, k, Y):
        y = np.ascontiguousarray(Y, dtype=np.float64)
        return self.lib().orc_get_temp(*self._fm(), T, i, j, k, y.ctypes.data_as(_dp))


class RefCase:
    """The reference's Flowfield + Reaction pair for one rank, through the
    friend-class harness.  Field names follow the reference's members;
    reaction-side arrays are prefixed ``R.``."""

    _libs = {}

    @classmethod
    def available(cls, fixed: bool = False) -> bool:
        return os.path.exists(REF_FIXED_SO if fixed else REF_SO)

    @classmethod
    def lib(cls, fixed: bool = False):
        path = REF_FIXED_SO if fixed else REF_SO
        if path not in cls._libs:
            L = _lib(path)
            L.ref_create.restype = C.c_void_p
            L.ref_create.argtypes = [C.c_int] * 4 + [_dp] * 3 + [C.c_int] * 3 + [_dp] * 9
            L.ref_destroy.argtypes = [C.c_void_p]
            L.ref_field.restype = _dp
            L.ref_field.argtypes = [C.c_void_p, C.c_char_p, C.POINTER(C.c_size_t)]
            L.ref_nchem.restype = C.POINTER(C.c_int)
            L.ref_nchem.argtypes = [C.c_void_p, C.POINTER(C.c_size_t)]
            for fn in ("ref_set_dt", "ref_set_time"):
                getattr(L, fn).argtypes = [C.c_void_p, C.c_double]
            for fn in ("ref_get_dt", "ref_get_time"):
                getattr(L, fn).argtypes = [C.c_void_p]
                getattr(L, fn).restype = C.c_double
            L.ref_cfl.argtypes = [C.c_void_p, C.c_double, C.c_double]
            L.ref_boundary.argtypes = [C.c_void_p, C.c_int]
            L.ref_advection.argtypes = [C.c_void_p, C.c_int, C.c_int]
            for fn in ("ref_update_after_adv", "ref_update_after_cs", "ref_explicit", "ref_partial_t",
                       "ref_imex", "ref_prediction"):
                getattr(L, fn).argtypes = [C.c_void_p]
            L.ref_trapezoid.argtypes = [C.c_void_p, C.c_int]
            L.ref_get_temp.argtypes = [C.c_void_p, C.c_double, C.c_int, C.c_int, C.c_int, _dp]
            L.ref_get_temp.restype = C.c_double
            L.ref_thermo.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_double, C.c_int]
            L.ref_thermo.restype = C.c_double
            L.ref_read_mechanism.argtypes = [C.c_char_p, C.c_char_p, C.POINTER(C.c_int)] + [_dp] * 9 + [C.c_int] * 2
            L.ref_read_mechanism.restype = C.c_int
            cls._libs[path] = L
        return cls._libs[path]

    def __init__(self, mech, grid, fixed: bool = False):
        """fixed=False: the reference as shipped; fixed=True: the same sources
        with the documented defects corrected (oracle/Makefile, ref_fixed)."""
        self.fixed = fixed
        L = self.lib(fixed)
        self.mech = mech
        self._keep = []

        def p(a):
            a = np.ascontiguousarray(a, dtype=np.float64)
            self._keep.append(a)
            return a.ctypes.data_as(_dp)

        NS, NR = mech.NS, mech.NR
        self._L = L
        self.h = L.ref_create(grid.ni, grid.nj, grid.nk, grid.bc, p(grid.xnode), p(grid.ynode), p(grid.znode),
                              NS, NR, mech.TB, p(mech.stoi_f.reshape(-1)), p(mech.stoi_b.reshape(-1)),
                              p(mech.react_tb.reshape(-1)), p(mech.af), p(mech.bf), p(mech.eaf),
                              p(mech.c0.reshape(-1)), p(mech.c1.reshape(-1)), p(mech.mw))
        self.ni, self.nj, self.nk, self.bc, self.NS = grid.ni, grid.nj, grid.nk, grid.bc, NS
        self.NI, self.NJ, self.NK = grid.ni + 2 * grid.bc, grid.nj + 2 * grid.bc, grid.nk + 2 * grid.bc

    def __del__(self):
        try:
            if self.h:
                self._L.ref_destroy(self.h)
        except Exception:
            pass

    def view(self, name):
        n = C.c_size_t(0)
        if name == "R.Nchem":
            ptr = self._L.ref_nchem(self.h, C.byref(n))
            return np.ctypeslib.as_array(ptr, shape=(self.NI, self.NJ, self.NK))
        ptr = self._L.ref_field(self.h, name.encode(), C.byref(n))
        if not ptr:
            raise KeyError(name)
        cells = self.NI * self.NJ * self.NK
        if name in ("Uint", "Vint", "Wint", "Pint", "Dint", "Tint", "Hint", "Eint", "Gint"):
            return np.ctypeslib.as_array(ptr, shape=(self.nj, self.nk))
        if name == "Yint":
            return np.ctypeslib.as_array(ptr, shape=(self.nj, self.nk, self.NS))
        if name == "R.MD":
            return np.ctypeslib.as_array(ptr, shape=(self.NI, self.NJ, self.NK, self.NS + 3, self.NS + 3))
        per = n.value // cells
        if per == 1:
            return np.ctypeslib.as_array(ptr, shape=(self.NI, self.NJ, self.NK))
        return np.ctypeslib.as_array(ptr, shape=(self.NI, self.NJ, self.NK, per))

    @property
    def dt(self):
        return self._L.ref_get_dt(self.h)

    @dt.setter
    def dt(self, v):
        self._L.ref_set_dt(self.h, v)

    @property
    def time(self):
        return self._L.ref_get_time(self.h)

    @time.setter
    def time(self, v):
        self._L.ref_set_time(self.h, v)

    def cfl(self, cfl, final_time):
        self._L.ref_cfl(self.h, cfl, final_time)

    def boundary(self, kind):
        self._L.ref_boundary(self.h, kind)

    def advection(self, timeadv=0, diff=1):
        self._L.ref_advection(self.h, timeadv, diff)

    def update_after_adv(self):
        self._L.ref_update_after_adv(self.h)

    def update_after_cs(self):
        self._L.ref_update_after_cs(self.h)

    def explicit(self):
        self._L.ref_explicit(self.h)

    def partial_t(self):
        self._L.ref_partial_t(self.h)

    def imex(self):
        self._L.ref_imex(self.h)

    def trapezoid(self, type_):
        self._L.ref_trapezoid(self.h, type_)

    def prediction(self):
        self._L.ref_prediction(self.h)

    def get_temp(self, T, i, j, k, Y):
        y = np.ascontiguousarray(Y, dtype=np.float64)
        return self._L.ref_get_temp(self.h, T, i, j, k, y.ctypes.data_as(_dp))

    def thermo(self, which, T, R, sp):
        return self._L.ref_thermo(self.h, which, T, R, sp)

    @classmethod
    def read_mechanism(cls, mech_path, thermo_path, cap_ns=MAXS, cap_nr=MAXR):
        L = cls.lib()
        hdr = (C.c_int * 3)()
        bufs = [np.zeros(cap_ns * cap_nr) for _ in range(3)] + [np.zeros(cap_nr) for _ in range(3)] + \
               [np.zeros(9 * cap_ns) for _ in range(2)] + [np.zeros(cap_ns)]
        rc = L.ref_read_mechanism(mech_path.encode(), thermo_path.encode(), hdr,
                                  *[b.ctypes.data_as(_dp) for b in bufs], cap_ns, cap_nr)
        if rc != 0:
            raise RuntimeError("ref_read_mechanism failed")
        NS, NR, TB = hdr[0], hdr[1], hdr[2]
        sf, sb, tb, af, bf, ea, c0, c1, mw = bufs
        return dict(NS=NS, NR=NR, TB=TB, stoi_f=sf[:NS * NR].reshape(NS, NR), stoi_b=sb[:NS * NR].reshape(NS, NR),
                    react_tb=tb[:NS * NR].reshape(NS, NR), af=af[:NR], bf=bf[:NR], eaf=ea[:NR],
                    c0=c0[:9 * NS].reshape(9, NS), c1=c1[:9 * NS].reshape(9, NS), mw=mw[:NS])


# state fields that define one rank's flow for the hot path
STATE3 = ["U", "V", "W", "P", "D", "T", "C", "Wav", "Rgas", "Cp", "H", "E", "Gamma"]
STATE4 = ["Mc", "Yi", "Di", "CS", "Partion_T"]


def copy_state(src, dst, names=None):
    """Copy the named fields (default: the full hot-path state) between two
    wrappers (Oracle or RefCase) that describe the same grid."""
    for n in (names or STATE3 + STATE4):
        dst.view(n)[...] = src.view(n)
