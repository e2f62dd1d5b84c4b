"""Dynamic load balancing of the adaptive trapezoid across ranks (CPU).

* the planner (eu3d_dlb_plan, host code of the CUDA library) and its
  restatement (oracle/dlb_oracle.py) against the reference's own
  DynamicLoadBalancer::DLBPriorityQueue (src/LoadBalance.cpp:8-59): golden
  plans made by running it (tests/golden/dlb_plans.npz, make_golden.py --dlb),
  and live when the compiled reference is present;
* the row picker of eu3d_dlb_select (eu3d_dlb_select_rows);
* the protocol of eu3d_b200.slabs (loads, plan, counts, packets out and
  back) on host slabs with a stand-in chemistry: in one process and as three
  gloo ranks, equal to the unbalanced result bit for bit.
The device kernels are covered by tests/test_gpu_slabs.py.
"""
import ctypes as C
import os
import socket
import subprocess
import sys

import numpy as np
import pytest

from _dlb_host import HostListSlab, HostSlab, chem, make_slabs, predict, unbalanced_list
from dlb_oracle import dlb_plan as oracle_plan
from eu3d_b200 import gpu
from eu3d_b200.slabs import LoopbackTransport, SlabRun, StepSpec

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
REF_SO = os.path.join(ROOT, "oracle", "_ref", "libeu3d_ref.so")


def _library_or_skip():
    try:
        gpu.load_library()
    except Exception as e:
        pytest.skip(f"libeu3d_gpu.so not loadable: {e}")


def _golden():
    g = np.load(os.path.join(HERE, "golden", "dlb_plans.npz"))
    n = len([k for k in g.files if k.startswith("loads")])
    return [(g[f"loads{t}"], [tuple(int(x) for x in row) for row in g[f"plan{t}"]]) for t in range(n)]


def test_oracle_plan_matches_reference_fixture():
    for loads, plan in _golden():
        assert oracle_plan(loads) == plan, loads


def test_library_plan_matches_reference_fixture():
    _library_or_skip()
    for loads, plan in _golden():
        assert gpu.dlb_plan(loads) == plan, loads


def test_library_plan_matches_live_reference():
    _library_or_skip()
    if not os.path.exists(REF_SO):
        pytest.skip("compiled reference absent")
    L = C.CDLL(REF_SO)
    rng = np.random.default_rng(77)
    for _ in range(200):
        n = int(rng.integers(1, 17))
        loads = [int(v) for v in rng.integers(0, 10 ** 6, n)]
        buf = (C.c_int * 900)()
        m = L.ref_dlb_plan((C.c_int * n)(*loads), n, buf, 300)
        assert gpu.dlb_plan(loads) == [tuple(buf[3 * t:3 * t + 3]) for t in range(m)], loads


def test_plan_without_imbalance_is_empty():
    _library_or_skip()
    assert gpu.dlb_plan([5, 5, 5]) == [] and gpu.dlb_plan([9]) == []
    assert gpu.load_degree([5, 5, 5]) == 0.0
    assert gpu.load_degree([100, 0, 0, 0]) == 0.75  # integer mean 25, as AveValue


def test_select_rows():
    _library_or_skip()
    rng = np.random.default_rng(3)
    for _ in range(50):
        rowload = rng.integers(0, 50, int(rng.integers(1, 40)))
        amounts = rng.integers(0, 300, int(rng.integers(1, 5)))
        bounds, moved = gpu.dlb_select_rows(rowload, amounts)
        assert bounds[0] == 0 and np.all(np.diff(bounds) >= 0) and bounds[-1] <= len(rowload)
        for p, a in enumerate(amounts):
            assert moved[p] == rowload[bounds[p]:bounds[p + 1]].sum() <= a
            if bounds[p + 1] < len(rowload):  # greedy: the next row would not fit
                assert moved[p] + rowload[bounds[p + 1]] > a


def _expected(data, steps):
    out = []
    for v, s in data:
        v = v.copy()
        for _ in range(steps):
            v = np.where(s, v, chem(v, predict(v)))
        out.append(v)
    return out


def test_loopback_host_slabs_equal_unbalanced():
    _library_or_skip()
    data = make_slabs(3)
    slabs = [HostSlab(v, s, r, 3) for r, (v, s) in enumerate(data)]
    spec = StepSpec(react=gpu.REACT_TRAPEZOID, type_=1, dlb=True)
    SlabRun(slabs, LoopbackTransport()).run(2, spec)
    plan = slabs[0].last_plan
    assert plan and all(p[0] == 0 for p in plan)  # the hot rank gives
    for got, want in zip([s.vals for s in slabs], _expected(data, 2)):
        assert np.array_equal(got, want)
    moved = sum(s.counts[t] for s in slabs[:1] for t in s.mine)
    assert moved > 0


def test_balancing_off_below_tolerance():
    _library_or_skip()
    data = make_slabs(2)
    slabs = [HostSlab(v, s, r, 2) for r, (v, s) in enumerate(data)]
    spec = StepSpec(react=gpu.REACT_TRAPEZOID, type_=1, dlb=True, dlb_tol=0.99)
    SlabRun(slabs, LoopbackTransport()).run(1, spec)
    assert slabs[0].last_plan == []
    for got, want in zip([s.vals for s in slabs], _expected(data, 1)):
        assert np.array_equal(got, want)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_three_gloo_ranks_equal_unbalanced(tmp_path):
    _library_or_skip()
    port, world, steps = _free_port(), 3, 2
    outs = [str(tmp_path / f"rank{r}.npz") for r in range(world)]
    procs = [subprocess.Popen([sys.executable, os.path.join(HERE, "dlb_worker.py"), str(r), str(world), str(port),
                               outs[r], str(steps)], stdout=subprocess.PIPE, stderr=subprocess.STDOUT)
             for r in range(world)]
    for p in procs:
        out, _ = p.communicate(timeout=240)
        assert p.returncode == 0, out.decode(errors="replace")[-2000:]
    res = [np.load(o) for o in outs]
    for r, want in enumerate(_expected(make_slabs(world), steps)):
        assert np.array_equal(res[r]["vals"], want), r
    assert len(res[0]["plan"]) > 0
    assert all(np.array_equal(res[0]["plan"], x["plan"]) for x in res)


def test_loopback_fallback_list_slabs_equal_unbalanced():
    """The learned chemistry's kind of the protocol on host slabs: the hot
    rank's fallback list is the longest, its last slots travel (in an
    arbitrary list order, as the device's atomic appends leave it), and
    every cell ends as the unbalanced step leaves it."""
    _library_or_skip()
    data = make_slabs(3)
    slabs = [HostListSlab(v, s, r, 3) for r, (v, s) in enumerate(data)]
    spec = StepSpec(react=gpu.REACT_SURROGATE, dlb=True)
    assert spec.balanced() and spec.balance_kind() == "sur"
    SlabRun(slabs, LoopbackTransport()).run(2, spec)
    plan = slabs[0].last_plan
    assert plan and all(p[0] == 0 for p in plan)
    assert sum(slabs[0].counts[t] for t in slabs[0].mine) > 0
    for got, want in zip([s.vals for s in slabs], unbalanced_list(data, 2)):
        assert np.array_equal(got, want)


def test_three_gloo_ranks_fallback_list_equal_unbalanced(tmp_path):
    """The same as three gloo processes (torch.distributed collectives)."""
    _library_or_skip()
    port, world, steps = _free_port(), 3, 2
    outs = [str(tmp_path / f"rank{r}.npz") for r in range(world)]
    procs = [subprocess.Popen([sys.executable, os.path.join(HERE, "dlb_worker.py"), str(r), str(world), str(port),
                               outs[r], str(steps), "sur"], stdout=subprocess.PIPE, stderr=subprocess.STDOUT)
             for r in range(world)]
    for p in procs:
        out, _ = p.communicate(timeout=240)
        assert p.returncode == 0, out.decode(errors="replace")[-2000:]
    res = [np.load(o) for o in outs]
    for r, want in enumerate(unbalanced_list(make_slabs(world), steps)):
        assert np.array_equal(res[r]["vals"], want), r
    assert len(res[0]["plan"]) > 0


def test_entry_points_reject_bad_arguments():
    _library_or_skip()
    L = gpu.load_library()
    lp, ip = C.POINTER(C.c_longlong), C.POINTER(C.c_int)
    loads = np.array([100, 0, 0, 0], dtype=np.int64)
    m = C.c_int()
    snd = np.zeros(1, dtype=np.int32)
    rcv = np.zeros(1, dtype=np.int32)
    amt = np.zeros(1, dtype=np.int64)
    # three transfers do not fit a capacity of one; the count is still reported
    rc = L.eu3d_dlb_plan(loads.ctypes.data_as(lp), 4, 1, snd.ctypes.data_as(ip), rcv.ctypes.data_as(ip),
                         amt.ctypes.data_as(lp), C.byref(m))
    assert rc == -1 and m.value == 3
    assert L.eu3d_dlb_plan(None, 4, 1, None, None, None, C.byref(m)) == -1
    assert L.eu3d_dlb_plan(loads.ctypes.data_as(lp), 0, 1, None, None, None, C.byref(m)) == -1
    b = np.zeros(2, dtype=np.int64)
    assert L.eu3d_dlb_select_rows(None, 3, 1, None, b.ctypes.data_as(lp), None) == -1
    assert L.eu3d_dlb_select_rows(loads.ctypes.data_as(lp), 4, -1, None, b.ctypes.data_as(lp), None) == -1
    for fn in ("eu3d_chem_load", "eu3d_dlb_pack", "eu3d_dlb_unpack"):
        assert getattr(L, fn)(None, None) == -1, fn
    assert L.eu3d_dlb_select(None, 0, None, None, None) == -1
    assert L.eu3d_dlb_guest(None, 0, None, None, None) == -1
    assert b"null" in L.eu3d_last_error() or b"bad" in L.eu3d_last_error()
    # the learned chemistry's fallback balancing
    for fn in ("eu3d_sur_load", "eu3d_sdlb_pack", "eu3d_sdlb_unpack"):
        assert getattr(L, fn)(None, None) == -1, fn
    assert L.eu3d_sdlb_select(None, 0, None, None) == -1
    assert L.eu3d_sdlb_guest(None, 0, None, None, None) == -1


@pytest.mark.parametrize("nranks,seed", [(2, 1), (3, 2), (4, 3), (5, 4), (5, 5)])
def test_loopback_host_slabs_random_hot_spots(nranks, seed):
    """Random hot rows on random ranks: every plan the planner makes moves
    whole rows out and back without changing any cell's result."""
    _library_or_skip()
    rng = np.random.default_rng(seed)
    data = []
    for r in range(nranks):
        vals = rng.uniform(0.0, 0.75, (10, 6))
        hot = rng.random(10) < rng.uniform(0.0, 0.6)
        vals[hot] = rng.uniform(0.8, 1.0, (int(hot.sum()), 6))
        solid = rng.random((10, 6)) < 0.05
        data.append((vals, solid))
    slabs = [HostSlab(v, s, r, nranks) for r, (v, s) in enumerate(data)]
    spec = StepSpec(react=gpu.REACT_TRAPEZOID, type_=1, dlb=True)
    SlabRun(slabs, LoopbackTransport()).run(2, spec)
    for got, want in zip([s.vals for s in slabs], _expected(data, 2)):
        assert np.array_equal(got, want)
    plan = slabs[0].last_plan
    assert plan == oracle_plan(slabs[0].loads)
