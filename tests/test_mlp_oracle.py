"""The surrogate network's CPU oracle (oracle/mlp_oracle.py) pinned by finite
differences of its own loss, and the host-side normalisation round trip."""
import numpy as np

from mlp_oracle import NPARAM, bf16, forward, loss_grad

from eu3d_b200 import surrogate as S
from eu3d_b200.readers import load_h2_ja919


def _problem(seed, B=48):
    rng = np.random.default_rng(seed)
    p = rng.standard_normal(NPARAM) * 0.08
    X = rng.standard_normal((B, 16))
    Y = rng.standard_normal((B, 16))
    Y[:, 15] = rng.uniform(0.5, 1.0, B)
    return rng, p, X, Y


def test_oracle_gradient_matches_central_differences():
    rng, p, X, Y = _problem(0)
    loss, g, _ = loss_grad(p, X, Y, quantize=False)
    assert loss > 0
    # a spread of parameters from every tensor, plus the unused output columns
    idx = np.unique(np.concatenate([rng.choice(NPARAM, 60, replace=False),
                                    [0, 2047, 2048, 2175, 2176, 18687, 35000, NPARAM - 7, NPARAM - 1]]))
    h = 1e-6
    for i in idx:
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (loss_grad(pp, X, Y, quantize=False)[0] - loss_grad(pm, X, Y, quantize=False)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-7 * max(1.0, abs(g[i])) + 1e-9, (i, fd, g[i])
    # unused outputs 10..15 carry no gradient
    assert np.all(g[-6:] == 0)


def test_oracle_quantisation_is_bf16():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -2.5e-3, 3.0e5])
    q = bf16(x)
    assert q[0] == 1.0 and q[1] == 1.0 + 2 ** -7 or q[1] == 1.0  # ties to even
    assert np.all(np.abs(q - x) <= np.abs(x) * 2 ** -8)
    out_q, _ = forward(_problem(1)[1], _problem(1)[2], quantize=True)
    out_f, _ = forward(_problem(1)[1], _problem(1)[2], quantize=False)
    assert np.max(np.abs(out_q - out_f)) < 0.1 * np.max(np.abs(out_f))


def test_norm_roundtrip_and_features():
    mech = load_h2_ja919()
    rng = np.random.default_rng(3)
    n = 4000
    X = np.zeros((n, 12), np.float32)
    X[:, 0] = rng.uniform(300, 3500, n)
    X[:, 1] = rng.uniform(-3, 3.9, n)
    Y = rng.dirichlet(np.ones(9), n)
    X[:, 2:11] = Y
    X[:, 11] = rng.uniform(np.log(1e-9), np.log(1e-7), n)
    Lb = np.zeros((n, 12), np.float32)
    Lb[:, :10] = rng.standard_normal((n, 10)) * 1e-3 * np.exp(X[:, 11:12]) / 1e-8
    Lb[:, 10] = 1.0
    norm = S.make_norm(mech, X, Lb)
    t = S.targets(X, Lb, norm)
    back = S.unscale(t, X, norm)
    # float32 targets: compare relative to max(|label|, the asinh linear scale)
    sc = np.exp(X[:, 11].astype(np.float64)) * S.activity(X[:, 0], norm[S.N_TA], norm[S.N_TR])
    ref = np.maximum(np.abs(Lb[:, :10]), sc[:, None] * norm[S.N_LIN:S.N_LIN + 10])
    assert np.max(np.abs(back - Lb[:, :10]) / ref) < 2e-5
    f = S.features(X, norm)
    assert f.shape == (n, 16) and np.all(f[:, 15] == 0)
    # the residual columns restore the inputs to about 16 bits
    rec = S.bf16_round(f[:, 0]) + S.bf16_round(f[:, 12]) / 256
    assert np.max(np.abs(rec - f[:, 0])) < 2e-4 * np.max(np.abs(f[:, 0]))
    assert np.allclose(S.element_ratios(mech, S.stoichiometric_h2_air(mech)), [2.0, 3.76], rtol=1e-12)


def test_atoms_and_species_index():
    mech = load_h2_ja919()
    A = S.atoms_matrix(mech)
    sp = mech.species
    assert A[:, sp.index("H2O2")].tolist() == [2, 2, 0]
    assert A[:, sp.index("N2")].tolist() == [0, 0, 2]
    assert A[:, sp.index("HO2")].tolist() == [1, 2, 0]
    idx = S.species_index(mech)
    assert [sp[i] for i in idx] == list(S.RADICAL_ORDER)
    p = S.init_params(0)
    assert p.shape == (NPARAM,) and np.all(p[S.OFF["b1"][0]:S.OFF["b1"][0] + 128] == 0)
