"""Learned chemistry surrogate on the GPU: training gradients against the CPU
FP64 oracle, fused inference against the oracle's forward pass, FP64 labels
against the oracle's IMEX step, training progress, and the coupled step's
fallback and conservation properties.  Everything runs through the C ABI."""
import numpy as np
import pytest

from mlp_oracle import NPARAM, forward, loss_grad, unpack
from pyoracle import Oracle

from _cases import QUIRKS_FIXED, fill_state, interior, small_grid
from eu3d_b200 import gpu
from eu3d_b200 import surrogate as S
from eu3d_b200.readers import make_grid

pytestmark = pytest.mark.gpu

LAYERS = ("W1", "b1", "W2", "b2", "W3", "b3", "W4", "b4")


@pytest.fixture(scope="module")
def dev(mech):
    d = gpu.DeviceFlowfield(mech, small_grid(), QUIRKS_FIXED, flux_bits=64)
    yield d
    d.close()


def _params(seed, bias=0.05):
    p = S.init_params(seed).astype(np.float64)
    rng = np.random.default_rng(seed + 100)
    for b in ("b1", "b2", "b3", "b4"):
        o, n = S.OFF[b]
        p[o:o + n] = bias * rng.standard_normal(n)
    p[S.OFF["b4"][0] + 10:S.OFF["b4"][0] + 16] = 0
    return p.astype(np.float32)


def _batch(seed, B):
    rng = np.random.default_rng(seed)
    X = rng.standard_normal((B, 16)).astype(np.float32)
    X[:, 15] = 0
    Y = rng.standard_normal((B, 16)).astype(np.float32)
    Y[:, 10:15] = 0
    Y[:, 15] = (rng.uniform(size=B) > 0.1).astype(np.float32)
    return X, Y


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-30))


@pytest.mark.parametrize("B", [256, 1024])
def test_loss_grad_matches_oracle(dev, B):
    sur = gpu.DeviceSurrogate(dev, 0, S.atoms_matrix(dev.mech))
    p = _params(7)
    sur.set_params(p)
    X, Y = _batch(11, B)
    loss, g, out = sur.loss_grad(X, Y)
    loss_o, g_o, out_o = loss_grad(p.astype(np.float64), X.astype(np.float64), Y.astype(np.float64), quantize=True)
    assert abs(loss - loss_o) <= 2e-3 * loss_o
    assert np.max(np.abs(out[:, :10] - out_o[:, :10])) <= 2e-2 * np.max(np.abs(out_o[:, :10]))
    gd, god = unpack(g), unpack(g_o)
    for name in LAYERS:
        assert _rel(gd[name], god[name]) < 1.5e-2, (name, _rel(gd[name], god[name]))
    # against the unquantised FP64 gradient the BF16 pipeline stays close too
    _, g_f, _ = loss_grad(p.astype(np.float64), X.astype(np.float64), Y.astype(np.float64), quantize=False)
    assert _rel(g, g_f) < 5e-2
    sur.close()


def test_fused_inference_matches_oracle_and_training_forward(dev):
    sur = gpu.DeviceSurrogate(dev, 0, S.atoms_matrix(dev.mech))
    p = _params(3)
    sur.set_params(p)
    n = 1000  # not a multiple of 128: the last tile is partial
    X, Y = _batch(5, 1024)
    out = sur.predict(X[:n])
    ref, _ = forward(p.astype(np.float64), X[:n].astype(np.float64), quantize=True)
    scale = np.max(np.abs(ref[:, :10]))
    assert np.max(np.abs(out[:, :10] - ref[:, :10])) <= 2e-2 * scale
    _, _, out_train = sur.loss_grad(X, Y)
    assert np.max(np.abs(out[:, :10] - out_train[:n, :10])) <= 1e-2 * scale
    sur.close()


def _oracle_labels(mech, states, dt):
    """Closed-reactor IMEX labels on the oracle: one cell per sample."""
    n = states.shape[0]
    ni = 16
    g = make_grid(ni, 0.0, 1.0, n // ni, 0.0, 1.0, 2, 0.0, 1.0, 2, fixed_ghosts=True)
    o = Oracle(mech, g, QUIRKS_FIXED)
    NS = mech.NS
    Ti = np.full((o.NI, o.NJ, o.NK), 1000.0)
    Pi = np.full_like(Ti, 101325.0)
    Yi = np.broadcast_to(S.stoichiometric_h2_air(mech), (o.NI, o.NJ, o.NK, NS)).copy()
    sl = (slice(2, 2 + ni), slice(2, 2 + n // ni), slice(2, 4))
    st = states.reshape(ni, n // ni, 1, 12, order="F")
    st = np.repeat(st, 2, axis=2)
    Ti[sl] = st[..., 0]
    Pi[sl] = st[..., 1]
    Yi[sl] = st[..., 2:11]
    o.view("T")[...] = Ti
    o.view("P")[...] = Pi
    o.view("U")[...] = 0
    o.view("V")[...] = 0
    o.view("W")[...] = 0
    o.view("Yi")[...] = Yi
    o.prims_from_state()
    o.partial_t()
    o.view("RHS")[...] = 0
    o.dt = dt
    cs0 = o.view("CS").copy()
    D0 = cs0[..., :NS].sum(-1)
    Y0 = cs0[..., :NS] / D0[..., None]
    o.imex()
    cs1 = o.view("CS")
    dY = cs1[..., :NS] / cs1[..., :NS].sum(-1)[..., None] - Y0
    A = S.atoms_matrix(mech) / mech.mw
    w = Y0 + 1e-4
    r = dY @ A.T
    M = np.einsum("ek,...k,fk->...ef", A, w, A)
    lam = np.linalg.solve(M, r[..., None])[..., 0]
    dY = dY - w * (lam @ A)
    csp = cs0.copy()
    csp[..., :NS] = D0[..., None] * np.maximum(Y0 + dY, 0)
    o.view("CS")[...] = csp
    T_imex = o.view("T").copy()
    o.update_after_cs()
    dT = o.view("T") - Ti
    return dY[sl][:, :, 0].reshape(n, NS, order="F"), dT[sl][:, :, 0].reshape(n, order="F"), T_imex


def test_imex_labels_match_oracle(dev, mech):
    sur = gpu.DeviceSurrogate(dev, 256, S.atoms_matrix(mech))
    dt = 5e-8
    env = (900.0, 2800.0, np.log(0.3), np.log(10.0), np.log(dt), np.log(dt))
    sur.add_random(256, env, S.species_index(mech), 99)
    nv = sur.label(gpu.REACT_IMEX)
    X, Lb, states = sur.dataset(states=True)
    # the one-step IMEX update is not positivity preserving: samples whose
    # projected composition goes negative are dropped (weight 0)
    ok = Lb[:, 10] == 1
    assert nv == ok.sum() and nv >= 0.9 * 256
    assert np.allclose(np.exp(X[:, 11]), dt, rtol=1e-6)
    dY, dT, _ = _oracle_labels(mech, states, dt)
    neg = np.any(states[:, 2:11] + dY < -1e-7, axis=1)
    assert np.array_equal(neg, ~ok)
    # element conservation of the labels
    A = S.atoms_matrix(mech) / mech.mw
    assert np.max(np.abs(Lb[:, :9].astype(np.float64) @ A.T)) < 1e-7 * np.max(np.abs(A))
    Lv, dY, dT = Lb[ok], dY[ok], dT[ok]
    assert np.max(np.abs(Lv[:, :9] - dY)) <= 1e-6 * np.max(np.abs(dY)) + 1e-12
    assert np.max(np.abs(Lv[:, 9] - dT)) <= 1e-6 * np.max(np.abs(dT)) + 1e-5
    assert np.max(np.abs(dT)) > 1.0  # the set holds reacting states
    sur.close()


def test_training_reduces_loss_and_heldout_error(dev, mech):
    n = 1 << 16
    sur = gpu.DeviceSurrogate(dev, n, S.atoms_matrix(mech))
    env = (300.0, 3500.0, np.log(0.05), np.log(50.0), np.log(1e-9), np.log(1e-7))
    sur.add_random(n, env, S.species_index(mech), 5)
    assert sur.label(gpu.REACT_IMEX) > 0.95 * n
    X, Lb = sur.dataset()
    norm = S.make_norm(mech, X, Lb)
    sur.set_norm(norm)
    sur.set_params(S.init_params(1))
    hold = slice(0, 4096)
    before = S.evaluate(sur, X[hold], Lb[hold], norm)
    losses = sur.train(600, 2048, 2e-3, 1e-4, 50, 17)
    after = S.evaluate(sur, X[hold], Lb[hold], norm)
    assert np.all(np.isfinite(losses))
    assert np.mean(losses[-50:]) < 0.3 * np.mean(losses[:10])
    assert after["mse"] < 0.3 * before["mse"]
    sur.close()


def _hot_pair(mech, dt):
    g = small_grid()
    o = Oracle(mech, g, QUIRKS_FIXED)
    fill_state(o, 21, 1100.0, 2600.0)
    devs = []
    for _ in range(2):
        d = gpu.DeviceFlowfield(mech, g, QUIRKS_FIXED, flux_bits=64)
        d.upload_state(o)
        d.upload("RHS", np.zeros(d.shape("RHS")))
        d.dt = dt
        devs.append(d)
    return devs


def test_all_fallback_equals_adaptive(mech):
    """With an envelope that admits nothing, every cell takes the FP64
    adaptive step (the network's teacher) on the fallback queue: the result
    equals the adaptive path's."""
    a, b = _hot_pair(mech, 3e-8)
    sur = gpu.DeviceSurrogate(b, 0, S.atoms_matrix(mech))
    norm = S.make_norm(mech, *_fake_set(mech))
    norm[S.N_ENV:S.N_ENV + 2] = (1e8, 2e8)  # no temperature is inside
    sur.set_norm(norm)
    sur.set_params(S.init_params(0))
    b.set_surrogate(sur)
    a.set_elements(S.atoms_matrix(mech))
    a.react_adaptive()
    b.react_surrogate()
    st = b.status()
    n = b.grid.ni * b.grid.nj * b.grid.nk
    assert st["surrogate_fallback"] == n and st["surrogate_cells"] == 0
    for f in ("CS", "T", "P", "Yi"):
        x, y = interior(a.download(f)), interior(b.download(f))
        assert np.max(np.abs(x - y)) <= 1e-13 * np.max(np.abs(x)), f
    b.set_surrogate(None)
    sur.close()


def _fake_set(mech, n=2048):
    rng = np.random.default_rng(0)
    X = np.zeros((n, 12), np.float32)
    X[:, 0] = rng.uniform(300, 3500, n)
    X[:, 1] = rng.uniform(-3, 3.9, n)
    Y = S.stoichiometric_h2_air(mech) * rng.uniform(0.5, 1.5, (n, mech.NS)) + 10 ** rng.uniform(-12, -3, (n, mech.NS))
    X[:, 2:11] = np.log(Y / Y.sum(-1, keepdims=True) + 1e-12)
    X[:, 11] = rng.uniform(np.log(1e-9), np.log(1e-7), n)
    Lb = np.zeros((n, 12), np.float32)
    Lb[:, :10] = rng.standard_normal((n, 10)) * 1e-4
    Lb[:, 10] = 1
    return X, Lb


def test_accepted_cells_conserve_elements_mass_energy(mech):
    """Cells the surrogate accepts keep rho, rho E and the element masses (to
    the negative-fraction clip) through the chemistry increment."""
    (d,) = _hot_pair(mech, 3e-8)[:1]
    sur = gpu.DeviceSurrogate(d, 0, S.atoms_matrix(mech))
    norm = S.make_norm(mech, *_fake_set(mech))
    norm[S.N_ENV:S.N_ENV + 6] = (200.0, 4000.0, -10.0, 10.0, -30.0, 0.0)
    norm[S.N_RES_ABS] = 1e9  # accept whatever the untrained network says
    norm[S.N_RATIO_TOL] = 10.0
    norm[S.N_LIN:S.N_LIN + 10] = 1e3  # increments of order dt A(T) 1e3 sinh(out)
    norm[S.N_OUT_MEAN:S.N_OUT_MEAN + 10] = 0
    norm[S.N_OUT_STD:S.N_OUT_STD + 10] = 1
    sur.set_norm(norm)
    p = S.init_params(4) * 0.05  # small increments
    sur.set_params(p)
    d.set_surrogate(sur)
    cs0 = interior(d.download("CS"))
    d.react_surrogate()
    st = d.status()
    n = d.grid.ni * d.grid.nj * d.grid.nk
    assert st["surrogate_cells"] + st["surrogate_fallback"] == n
    assert st["surrogate_cells"] > 0.9 * n, st["surrogate_rejects"]
    cs1 = interior(d.download("CS"))
    NS = mech.NS
    rho0, rho1 = cs0[..., :NS].sum(-1), cs1[..., :NS].sum(-1)
    assert np.max(np.abs(rho1 / rho0 - 1)) < 1e-12
    assert np.max(np.abs(cs1[..., NS:] - cs0[..., NS:])) <= 1e-12 * np.max(np.abs(cs0[..., NS:]))
    A = S.atoms_matrix(mech) / mech.mw
    el0 = cs0[..., :NS] @ A.T
    el1 = cs1[..., :NS] @ A.T
    assert np.max(np.abs(el1 - el0) / np.maximum(el0, 1e-30)) < 1e-10
    assert np.max(np.abs(cs1[..., :NS] - cs0[..., :NS])) > 0  # something happened
    d.set_surrogate(None)
    sur.close()


def test_surrogate_argument_errors(dev, mech):
    sur = gpu.DeviceSurrogate(dev, 16, S.atoms_matrix(mech))
    env = (300.0, 3500.0, 0.0, 1.0, -20.0, -16.0)
    with pytest.raises(gpu.Eu3dError):
        sur.add_random(17, env, S.species_index(mech), 1)  # beyond capacity
    with pytest.raises(gpu.Eu3dError):
        sur.train(10, 256, 1e-3, 1e-4, 1, 0)  # empty set
    with pytest.raises(gpu.Eu3dError):
        sur.label(gpu.REACT_NONE)
    bad = np.zeros(S.NORM_LEN, np.float32)
    with pytest.raises(gpu.Eu3dError):
        sur.set_norm(bad)
    with pytest.raises(gpu.Eu3dError):
        dev.react_surrogate()  # nothing attached
    with pytest.raises(gpu.Eu3dError):
        dev.step(react=gpu.REACT_SURROGATE, bc_kind=gpu.BC_RSBI)
    sur.close()


# ------------------------------------------------------- adaptive integrator
def _post_shock_states(mech, n, seed, dt):
    """Unburnt-to-igniting H2-air states (radical pools up to ~1e-3) at dt."""
    rng = np.random.default_rng(seed)
    sp = mech.species
    st = np.zeros((n, 12))
    st[:, 0] = rng.uniform(1050.0, 1600.0, n)
    st[:, 1] = 101325.0 * rng.uniform(0.3, 3.0, n)
    X = np.zeros((n, mech.NS))
    X[:, sp.index("H2")] = 2.0
    X[:, sp.index("O2")] = 1.0
    X[:, sp.index("N2")] = 3.76
    for r in ("H", "O", "OH", "HO2", "H2O2", "H2O"):
        X[:, sp.index(r)] = 10 ** rng.uniform(-9, -3, n)
    Y = X * mech.mw
    st[:, 2:11] = Y / Y.sum(-1, keepdims=True)
    st[:, 11] = dt
    return st


def _field_of_states(mech, states):
    """An oracle field whose interior cells (16 x n/16 x 2) hold the states."""
    n = states.shape[0]
    ni = 16
    g = make_grid(ni, 0.0, 1.0, n // ni, 0.0, 1.0, 2, 0.0, 1.0, 2, fixed_ghosts=True)
    o = Oracle(mech, g, QUIRKS_FIXED)
    NS = mech.NS
    Ti = np.full((o.NI, o.NJ, o.NK), 1000.0)
    Pi = np.full_like(Ti, 101325.0)
    Yi = np.broadcast_to(S.stoichiometric_h2_air(mech), (o.NI, o.NJ, o.NK, NS)).copy()
    sl = (slice(2, 2 + ni), slice(2, 2 + n // ni), slice(2, 4))
    st = np.repeat(states.reshape(ni, n // ni, 1, 12, order="F"), 2, axis=2)
    Ti[sl], Pi[sl], Yi[sl] = st[..., 0], st[..., 1], st[..., 2:11]
    for k, v in (("T", Ti), ("P", Pi), ("Yi", Yi)):
        o.view(k)[...] = v
    for k in ("U", "V", "W"):
        o.view(k)[...] = 0
    o.prims_from_state()
    o.view("RHS")[...] = 0
    return o, g, sl


def test_adaptive_labels_match_oracle(dev, mech):
    from adaptive_oracle import increment
    dt = 5.5e-8
    n = 64
    states = _post_shock_states(mech, n, 3, dt)
    sur = gpu.DeviceSurrogate(dev, n, S.atoms_matrix(mech))
    # the dataset takes the states through a snapshot of a flowfield holding them
    o, g, sl = _field_of_states(mech, states)
    d = gpu.DeviceFlowfield(mech, g, QUIRKS_FIXED, flux_bits=64)
    d.upload_state(o)
    d.upload("RHS", np.zeros(d.shape("RHS")))
    sur.add_snapshot(d, n, 1, 0, 0.0, 0.0, np.log(dt), np.log(dt), 0)
    assert sur.label(gpu.REACT_ADAPTIVE, cap=4096) == n
    X, Lb, _ = sur.dataset(states=True)
    # snapshot rows follow the interior order (x fastest, then y, then z)
    dY, Tchem, nsub = increment(o, dt, S.atoms_matrix(mech), nmax=4096)
    dY = dY[:, :, 0].reshape(n, mech.NS, order="F")
    nsub = nsub[:, :, 0].reshape(n, order="F")
    assert np.max(np.abs(Lb[:, :9] - dY)) <= 1e-6 * np.max(np.abs(dY)) + 1e-12
    # substep counts agree (a rounding-level difference may move one boundary)
    assert np.max(np.abs(Lb[:, 11].astype(np.int64) - nsub)) <= 1 and nsub.max() > 1
    assert np.max(np.abs(Lb[:, 9])) > 0.05  # the states react within dt
    d.close()
    sur.close()


def test_adaptive_step_matches_oracle_and_survives_ignition(mech):
    """The coupled adaptive update (with a flux residual) against the oracle
    restatement for one step, then 0-D reactors run through ignition on the
    GPU stay finite and keep their element masses."""
    from adaptive_oracle import adaptive_step
    dt = 5.5e-8
    n = 64
    states = _post_shock_states(mech, n, 5, dt)
    o, g, sl = _field_of_states(mech, states)
    rng = np.random.default_rng(2)
    rhs = np.zeros_like(o.view("RHS"))
    rhs[sl] = 1e-4 * o.view("CS")[sl] * rng.standard_normal(o.view("CS")[sl].shape)
    o.view("RHS")[...] = rhs
    d = gpu.DeviceFlowfield(mech, g, QUIRKS_FIXED, flux_bits=64)
    d.upload_state(o)
    d.upload("RHS", rhs)
    d.set_elements(S.atoms_matrix(mech))
    d.dt = dt
    o.dt = dt
    d.react_adaptive()
    adaptive_step(o, dt, S.atoms_matrix(mech))
    for f in ("CS", "T"):
        x, y = d.download(f)[sl], o.view(f)[sl]
        assert np.max(np.abs(x - y)) <= 1e-8 * np.max(np.abs(y)), f
    # closed reactors through ignition
    d.upload("RHS", np.zeros(d.shape("RHS")))
    A = S.atoms_matrix(mech) / mech.mw
    el0 = d.download("CS")[sl][..., :9] @ A.T
    T0 = d.download("T")[sl].copy()
    for _ in range(300):
        d.react_adaptive()
    T = d.download("T")[sl]
    cs = d.download("CS")[sl]
    assert np.all(np.isfinite(T)) and np.all(cs[..., :9] >= 0)
    assert np.max(T - T0) > 1000.0  # some reactors ignited
    assert T.max() < 4000.0
    el1 = cs[..., :9] @ A.T
    assert np.max(np.abs(el1 / el0 - 1)) < 1e-9
    d.close()


@pytest.mark.parametrize("flux_bits", [32, 64])
def test_fused_apply_equals_two_kernels(mech, flux_bits):
    """The network and its apply in one kernel (sur_fused) give the same
    accept/reject decisions, counters and conserved state as the network
    kernel followed by k_sur_apply, on an ODW with accepted, rejected and
    audited cells (FP32 flux: the conserved state bit for bit).  The decode's
    outputs (T, E, P) agree to 1e-8: inlined into the network kernel, the
    FP32 unscaling and the FP64 Newton polynomials are contracted into FMAs
    differently, and a Newton start that differs in its last bit converges to
    within the 1e-6 K tolerance of a slightly different temperature."""
    from eu3d_b200.cases import odw_case, setup_odw
    case = odw_case(mech, 160, 64, 3, L=0.05)
    m0 = S.SurrogateModel.load(S.DEFAULT_MODEL)
    norm = m0.norm.copy()
    norm[S.N_ENV + 0] = 320.0  # the 300 K free stream leaves the envelope: it falls back
    model = S.SurrogateModel(m0.params, norm, m0.meta)
    out = []
    for fused in (0, 1):
        d = gpu.DeviceFlowfield(mech, case.grid, gpu.QUIRKS_FIXED, flux_bits=flux_bits)
        setup_odw(d, case)
        s = model.attach(d, 7)
        d.set_tuning(sur_fused=fused)
        assert d.tuning()["sur_fused"] == fused
        kw = dict(timeadv=gpu.ADV_SSPRK2, bc_kind=gpu.BC_ODM, cfl=0.0, final_time=1.0)
        d.dt = 4e-8
        d.run(40, react=gpu.REACT_IMEX, **kw)
        d.run(3, react=gpu.REACT_SURROGATE, **kw)
        d.synchronize()
        st = d.status()
        out.append(({f: d.download(f) for f in ("CS", "T", "E", "P", "Yi")}, st))
        d.set_surrogate(None)
        s.close()
        d.close()
    (a, sa), (b, sb) = out
    assert sa["surrogate_cells"] > 0 and sa["surrogate_fallback"] > 0 and sa["surrogate_audited"] > 0, sa
    for k in ("surrogate_cells", "surrogate_fallback", "surrogate_rejects", "surrogate_audited",
              "nonfinite_cells", "wait_timeouts"):
        assert sa[k] == sb[k], k
    # FP32 primitives round the decode's last-bit differences away before the
    # next flux; FP64 primitives carry them into the next steps' state
    for f in ("CS", "Yi"):
        if flux_bits == 32:
            assert np.array_equal(a[f], b[f]), f
        else:
            assert np.max(np.abs(a[f] - b[f])) <= 1e-10 * np.max(np.abs(a[f])), f
    for f in ("T", "E", "P"):
        assert np.max(np.abs(a[f] - b[f]) / np.maximum(np.abs(a[f]), 1e-300)) <= 1e-8, f
