"""The C-ABI library builds, loads without a GPU and exports every entry point
that include/eu3d_gpu.h declares; the oracle library exports its functions.
No compute call is made here."""
import ctypes
import os
import re

import pytest

from eu3d_b200 import build, gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(eu3d_\w+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    build.build()
    return gpu.load_library()


def test_every_declared_symbol_is_exported(lib):
    names = declared("eu3d_gpu.h")
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_header():
    assert sorted(gpu.EXPORTS) == declared("eu3d_gpu.h")


def test_field_ids_match_header():
    text = open(os.path.join(ROOT, "include", "eu3d_gpu.h")).read()
    body = re.search(r"enum \{(.*?)\};", text, flags=re.S).group(1)
    body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
    ids = [t.strip().split("=")[0].strip() for t in body.split(",") if t.strip()]
    ids = [i for i in ids if i.startswith("EU3D_FIELD_") and i != "EU3D_FIELD_COUNT"]
    mine = sorted(gpu.FIELDS.items(), key=lambda kv: kv[1])
    assert len(ids) == len(mine)
    for (name, idx), hid in zip(mine, ids):
        assert gpu.FIELDS[name] == ids.index(hid)


def test_constants_match_quirk_header():
    text = open(os.path.join(ROOT, "include", "eu3d_quirks.h")).read()
    vals = dict(re.findall(r"#define (EU3D_\w+) (0x[0-9a-fA-F]+u?|\d+)", text))
    num = lambda s: int(s.rstrip("u"), 0)
    assert num(vals["EU3D_QUIRKS_REF"]) == gpu.QUIRKS_REF
    assert num(vals["EU3D_BC_ODM"]) == gpu.BC_ODM
    assert num(vals["EU3D_REACT_IMEX"]) == gpu.REACT_IMEX
    assert num(vals["EU3D_ADV_SSPRK2"]) == gpu.ADV_SSPRK2
    assert num(vals["EU3D_ADV_SSPRK3"]) == gpu.ADV_SSPRK3
    assert num(vals["EU3D_DIFF_WENO"]) == gpu.DIFF_WENO
    text = open(os.path.join(ROOT, "include", "eu3d_gpu.h")).read()
    parts = dict(re.findall(r"#define (EU3D_PART_\w+) (\d+)", text))
    assert {k: int(v) for k, v in parts.items()} == {
        "EU3D_PART_STAGE1": gpu.PART_STAGE1, "EU3D_PART_STAGE2": gpu.PART_STAGE2, "EU3D_PART_REACT": gpu.PART_REACT,
        "EU3D_PART_STAGE3": gpu.PART_STAGE3, "EU3D_PART_CHEM_PREDICT": gpu.PART_CHEM_PREDICT,
        "EU3D_PART_CHEM_WORK": gpu.PART_CHEM_WORK, "EU3D_PART_SUR_PREDICT": gpu.PART_SUR_PREDICT,
        "EU3D_PART_SUR_WORK": gpu.PART_SUR_WORK}
    dlb = dict(re.findall(r"#define (EU3D_DLB_\w+) (\d+)", text))
    assert (int(dlb["EU3D_DLB_OUT_FIELDS"]), int(dlb["EU3D_DLB_BACK_FIELDS"]), int(dlb["EU3D_DLB_MAX_TRANSFERS"])) == \
        (gpu.DLB_OUT_FIELDS, gpu.DLB_BACK_FIELDS, gpu.DLB_MAX_TRANSFERS)
    sdlb = dict(re.findall(r"#define (EU3D_SDLB_\w+) (\d+)", text))
    assert (int(sdlb["EU3D_SDLB_OUT_FIELDS"]), int(sdlb["EU3D_SDLB_BACK_FIELDS"])) == \
        (gpu.SDLB_OUT_FIELDS, gpu.SDLB_BACK_FIELDS)


def test_null_arguments_are_rejected_without_a_device(lib):
    h = ctypes.c_void_p()
    assert lib.eu3d_create(None, ctypes.byref(h)) == -1
    assert lib.eu3d_step(None, None) == -1
    assert b"null" in lib.eu3d_last_error()


def test_oracle_library_exports():
    from pyoracle import Oracle
    L = Oracle.lib()
    for fn in ("orc_advection", "orc_imex", "orc_trapezoid", "orc_boundary", "orc_cfl", "orc_step",
               "orc_update_after_cs", "orc_get_partial_t", "orc_diagonalized", "orc_prediction"):
        assert hasattr(L, fn)
