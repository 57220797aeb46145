"""The wall parameters the device initial state evaluates (nozzle.wall_parameters) against the host's
wall_half_height, on every contour family: the device's formula restated in NumPy here, operation for
operation, must give the host's wall to the last bit or within a few units of the last place."""

from __future__ import annotations

import math

import numpy as np
import pytest

from conftest import pkg


def _hermite(s, y0, y1, m0, m1):
    s2 = s * s
    s3 = s2 * s
    return (2.0 * s3 - 3.0 * s2 + 1.0) * y0 + (s3 - 2.0 * s2 + s) * m0 + (-2.0 * s3 + 3.0 * s2) * y1 + (s3 - s2) * m1


def device_wall(W, x):
    """The kernel's wall_y (csrc/initial.cuh) from the packed parameters."""
    fam, length, x_th, span, y_th, y_in, y_ex, m0, m1, c1, c2, h = W[:12]
    off = W[12:20]
    xi = x / length
    conv = _hermite(np.clip(xi / x_th, 0.0, 1.0), y_in, y_th, 0.0, 0.0)
    s = np.clip((xi - x_th) / span, 0.0, 1.0)
    if fam == 0:
        div = y_th + (y_ex - y_th) * s
    elif fam == 1:
        div = _hermite(s, y_th, y_ex, m0, m1)
    elif fam == 2:
        u = 1.0 - s
        div = u**3 * y_th + 3.0 * u**2 * s * c1 + 3.0 * u * s**2 * c2 + s**3 * y_ex
    else:
        u = 1.0 - s
        bump = sum(math.comb(9, k + 1) * s ** (k + 1) * u ** (8 - k) * off[k] for k in range(8))
        div = _hermite(s, y_th, y_ex, 0.0, m1) + y_th * bump
    return np.where(xi <= x_th, conv, div)


@pytest.mark.parametrize("contour", ["conical", "bell", "smooth", "moc", "bezier", "bezier8"])
def test_wall_parameters_reproduce_the_host_wall(contour):
    nz = pkg("nozzle")
    offs = tuple(np.random.default_rng(1).normal(0.0, 0.02, 8)) if contour == "bezier8" else (0.0,) * 8
    geom = nz.Geometry(area_ratio=2.7, contour=contour, offsets=offs, theta_exit_deg=3.0, length=1.3)
    W = nz.wall_parameters(geom)
    assert W.shape == (pkg("capi").NZB_WALL_PARAMS,)
    x = np.concatenate([np.linspace(0.0, geom.length, 2001), [geom.throat_location(), 1e-7, geom.length - 1e-9]])
    ref = geom.wall(x)
    got = device_wall(W, x)
    assert np.abs(got - ref).max() <= 4 * np.finfo(float).eps * np.abs(ref).max()


def test_quasi1d_table_is_the_initial_states_solution():
    nz, cfg = pkg("nozzle"), pkg("config")
    geom = nz.Geometry(area_ratio=2.5, contour="bell")
    flow = cfg.FlowConditions(back_pressure_ratio=0.2)
    T = nz.quasi1d_table(geom, flow)
    sol = nz.solve_quasi1d(geom, flow)
    assert T.shape == (4, sol.x.size) and np.all(np.diff(T[0]) > 0)
    assert np.array_equal(T, np.stack([sol.x, sol.density, sol.velocity, sol.pressure]))
