"""The front-position measure of the coupled accuracy checks
(eu3d_b200.validate.front_position), on synthetic temperature fields."""
import numpy as np

from eu3d_b200.validate import front_position


def test_front_position_interpolates_per_line():
    T = np.full((10, 3, 2), 300.0)
    T[6:] = 2000.0
    T[5] = 1000.0
    T[:, 2, 1] = 300.0           # no front on this line
    T[:, 0, 1] = 2000.0          # hot from the first cell: no position either
    f = front_position(T)
    assert f.shape == (3, 2)
    assert np.isclose(f[0, 0], 5.8) and np.isclose(f[1, 1], 5.8)
    assert np.isnan(f[2, 1]) and np.isnan(f[0, 1])


def test_front_position_2d_rows():
    T = np.linspace(300.0, 3000.0, 28)[:, None] * np.ones((1, 4))
    f = front_position(T)
    x = (1800.0 - 300.0) / (2700.0 / 27)
    assert np.allclose(f, x)
