"""The configuration set-ups of eu3d_b200.cases on the host: the 3D reactive
shock-bubble interaction (its shock jump, bubble, interface and seeded
perturbation) and the oblique-detonation inflow."""
import numpy as np

from eu3d_b200.cases import odw_case, radial_perturbation, rsbi_case


def test_rsbi_case(mech):
    n = 32
    c = rsbi_case(mech, n=n, seed=3)
    st, g = c.state, c.grid
    NI = n + 4
    assert st["CS"].shape == (NI, NI, NI, mech.NS + 4) and np.isfinite(st["CS"]).all()
    # FieldInitial's normal-shock jump for Mach 2, gamma 1.4
    assert np.isclose(c.post["P"] / 101325.0, 4.5) and np.isclose(c.post["T"], 300.0 * 1.6875)
    post = g.xnode < c.shock_x
    assert np.allclose(st["P"][post], c.post["P"]) and np.allclose(st["U"][post], c.post["U"])
    assert np.allclose(st["U"][~post], 0.0)
    # mass fractions sum to one; the centre is the bubble, the corners air
    assert np.allclose(st["Yi"].sum(-1), 1.0)
    h2 = mech.species.index("H2")
    m = NI // 2
    assert st["Yi"][m, m, m, h2] > 0.99 * st["Yi"][..., h2].max()
    assert st["Yi"][2, 2, 2, h2] < 1e-6  # the tanh tail, nine interface widths out
    # the interface sits within the perturbed shell R (1 +- 0.02) at tanh's midpoint
    x = g.xnode - c.centre[0]
    r = np.sqrt(x[:, None, None] ** 2 + (g.ynode - c.centre[1])[None, :, None] ** 2
                + (g.znode - c.centre[2])[None, None, :] ** 2)
    chi = st["Yi"][..., h2] / st["Yi"][..., h2].max()
    mid = np.abs(chi - 0.5) < 0.2
    assert mid.any()
    dx = g.xnode[1] - g.xnode[0]
    assert np.all(np.abs(r[mid] - c.radius) <= 0.02 * c.radius + 2.0 * dx)


def test_radial_perturbation_is_seeded_and_unit():
    th = np.linspace(0, np.pi, 60)[:, None]
    ph = np.linspace(0, 2 * np.pi, 120)[None, :]
    f1, f2, f3 = radial_perturbation(8, 1), radial_perturbation(8, 1), radial_perturbation(8, 2)
    a, b, c = f1(th, ph), f2(th, ph), f3(th, ph)
    assert np.array_equal(a, b) and not np.allclose(a, c)
    assert 0.9 < np.abs(a).max() <= 1.0 + 1e-9


def test_odw_inflow_perturbation(mech):
    c = odw_case(mech, 64, 32, 8, seed=5, pert=0.01)
    rho = c.inflow["D"]
    assert rho.shape == (32, 8)
    rel = rho / c.free["D"] - 1.0
    assert 0.005 < np.abs(rel).max() <= 0.0101
    assert np.allclose(c.inflow["P"], c.P)
