"""The result-file writer (Euler::Output, src/Euler.cpp:792-973).

* host writer (eu3d_tecplot_write_host) on the oracle's initial RSBI state of
  rank 0 vs the reference's own published file output_8/resultsIMEX0_0.dat
  (tests/golden/rsbi_t0_text.npz, made by tests/golden/make_golden.py --text):
  byte for byte (block by block first, for a readable failure);
* device writer (eu3d_write_tecplot, foreground and background) vs the host
  writer fed with the same handle's downloaded fields.
"""
import os
import zlib

import numpy as np
import pytest

from _cases import QUIRKS_REF, make_oracle, small_grid
from eu3d_b200 import gpu
from eu3d_b200.readers import make_grid
from pyoracle import Oracle

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")
NAMES = ["X", "Y", "Z", "T", "D", "P", "U", "V", "Ma", "Y1", "Y2", "Y3", "Y4", "Y5", "Y6", "Y7", "L", "WaitTime"]


def _library_or_skip():
    try:
        gpu.load_library()
    except Exception as e:  # the library is built by __graft_entry__.build()
        pytest.skip(f"libeu3d_gpu.so not loadable: {e}")


def blocks_of(text: str, n: int):
    lines = text.split("\n")
    assert lines[-1] == ""  # every value line ends in a newline
    head, body = lines[:3], lines[3:-1]
    assert len(body) == 18 * n
    return head, {name: body[b * n:(b + 1) * n] for b, name in enumerate(NAMES)}


def cell_order(a, bc):
    """interior of an (NI, NJ, NK) field in the file's order: k outer, i inner"""
    return np.transpose(a[bc:-bc, bc:-bc, bc:-bc], (2, 1, 0)).reshape(-1)


def oracle_columns(o, bc):
    cols = [cell_order(o.view(n), bc) for n in ("T", "D", "P", "U", "V", "Ma")]
    cols += [cell_order(o.view("Yi")[..., s], bc) for s in range(7)]
    return np.stack(cols), cell_order(o.view("Nchem"), bc).astype(np.int32)


def test_host_writer_matches_published_output(mech, tmp_path):
    _library_or_skip()
    raw = zlib.decompress(np.load(os.path.join(GOLD, "rsbi_t0_text.npz"))["rank0"].tobytes()).decode()
    g = make_grid(241, 0.0, 0.17, 81, 0.0, 0.08, 2, 0.0, 0.02, 2, blocks=(4, 2, 1), rank=(0, 0, 0))
    o = Oracle(mech, g, QUIRKS_REF)
    o.rsbi_initial(101325.0, 1000.0, 3.0)
    cols, lcol = oracle_columns(o, g.bc)
    path = str(tmp_path / "resultsIMEX0_0.dat")
    gpu.write_tecplot_host(path, g, cols, lcol, 0.0)
    mine = open(path).read()
    n = g.ni * g.nj * g.nk
    h_ref, b_ref = blocks_of(raw, n)
    h_mine, b_mine = blocks_of(mine, n)
    assert h_mine == h_ref
    for name in NAMES:
        assert b_mine[name] == b_ref[name], name
    assert mine == raw  # byte for byte


def test_host_writer_format(tmp_path):
    """std::ostream's default formatting: %.6g for doubles, %d for counts."""
    _library_or_skip()
    g = small_grid(3, 2, 2)
    n = 12
    t = [1000.0, 2679.0123, 1e-7, 123456.5, 1234567.0, -0.0]
    y7 = [0.1, 1.0 / 3.0, 2e300, 5e-324, -7.25, 100.0]
    cols = np.zeros((13, n))
    cols[0], cols[12] = t * 2, y7 * 2
    lcol = np.array([0, 1, 17, 250, 100000, -3] * 2, dtype=np.int32)
    path = str(tmp_path / "f.dat")
    gpu.write_tecplot_host(path, g, cols, lcol, 0.5)
    head, b = blocks_of(open(path).read(), n)
    assert head == ["Variables = X,Y,Z,T,D,P,U,V,Ma,Y1,Y2,Y3,Y4,Y5,Y6,Y7,L,WaitTime", "ZONE I=3\tJ=2\tK=2",
                    "datapacking=block"]
    assert b["T"] == ["1000", "2679.01", "1e-07", "123456", "1.23457e+06", "-0"] * 2
    assert b["Y7"] == ["0.1", "0.333333", "2e+300", "4.94066e-324", "-7.25", "100"] * 2
    assert b["L"] == ["0", "1", "17", "250", "100000", "-3"] * 2
    assert b["WaitTime"] == ["0.5"] * n
    assert b["X"] == ["%.6g" % g.xnode[g.bc + i] for i in (0, 1, 2)] * 4
    assert b["Y"] == ["%.6g" % g.ynode[g.bc + j] for j in (0, 0, 0, 1, 1, 1)] * 2
    assert b["Z"] == ["%.6g" % g.znode[g.bc + k] for k in [0] * 6 + [1] * 6]


def test_result_file_names():
    # the published t = 0 files of the 8-rank RSBI run are output_8/resultsIMEX0_<rank>.dat
    assert gpu.tecplot_path(8, "IMEX", 0, 5) == "./output_8/resultsIMEX0_5.dat"
    assert gpu.tecplot_path(1, "Trapezoid", 12, 0) == "./output_1/results/SeriesTrapezoid12_0.dat"


def test_host_writer_errors(tmp_path):
    _library_or_skip()
    g = small_grid(3, 2, 2)
    with pytest.raises(gpu.Eu3dError):
        gpu.write_tecplot_host(str(tmp_path / "f.dat"), g, np.zeros((12, 12)), np.zeros(12), 0.0)
    with pytest.raises(gpu.Eu3dError):
        gpu.write_tecplot_host(str(tmp_path / "no_such_dir" / "f.dat"), g, np.zeros((13, 12)), np.zeros(12), 0.0)


def _device_columns(d, bc):
    """what k_tecplot_gather computes, from the handle's downloaded fields"""
    U, V, W, P, D, G = (d.download(n) for n in ("U", "V", "W", "P", "D", "Gamma"))
    C = np.sqrt(G * P / D)
    Ma = np.sqrt(U * U + V * V + W * W) / C
    Y = d.download("Yi")
    cols = [cell_order(a, bc) for a in (d.download("T"), D, P, U, V, Ma)]
    cols += [cell_order(Y[..., s], bc) for s in range(7)]
    return np.stack(cols), cell_order(d.download("Nchem"), bc).astype(np.int32)


@pytest.mark.gpu
@pytest.mark.parametrize("flux_bits", [64, 32])
def test_device_writer_matches_host_writer(mech, tmp_path, flux_bits):
    g = small_grid(37, 11, 5)
    o, _ = make_oracle(mech, seed=7, grid=g, tlo=1500.0, thi=2200.0, radicals=1e-5)
    with gpu.DeviceFlowfield(mech, g, flux_bits=flux_bits) as d:
        d.upload_state(o)
        d.dt = 1e-8
        d.step(react=gpu.REACT_TRAPEZOID, type_=1)  # substep counts in L
        cols, lcol = _device_columns(d, g.bc)
        ref = str(tmp_path / "host.dat")
        gpu.write_tecplot_host(ref, g, cols, lcol, 1.25e-6)
        fg, bg = str(tmp_path / "fg.dat"), str(tmp_path / "bg.dat")
        d.write_tecplot(fg, 1.25e-6)
        d.write_tecplot(bg, 1.25e-6, background=True)
        d.step(react=gpu.REACT_TRAPEZOID, type_=1)  # steps on while the file is formatted
        d.write_wait()
    n = g.ni * g.nj * g.nk
    h_ref, b_ref = blocks_of(open(ref).read(), n)
    for path in (fg, bg):
        h, b = blocks_of(open(path).read(), n)
        assert h == h_ref
        for name in NAMES:
            if name == "Ma":  # sqrt/div order of the host check may differ in the last bit
                np.testing.assert_allclose(np.array(b[name], float), np.array(b_ref[name], float), rtol=6e-6)
            else:
                assert b[name] == b_ref[name], name
    assert np.all(lcol >= 1)


@pytest.mark.gpu
def test_device_writer_io_error(mech, tmp_path):
    g = small_grid(5, 4, 3)
    o, _ = make_oracle(mech, seed=3, grid=g)
    with gpu.DeviceFlowfield(mech, g) as d:
        d.upload_state(o)
        with pytest.raises(gpu.Eu3dError):
            d.write_tecplot(str(tmp_path / "missing" / "a.dat"))
        d.write_tecplot(str(tmp_path / "missing" / "b.dat"), background=True)
        with pytest.raises(gpu.Eu3dError):
            d.write_wait()
        d.write_tecplot(str(tmp_path / "ok.dat"))  # the handle stays usable
    assert os.path.getsize(tmp_path / "ok.dat") > 0
