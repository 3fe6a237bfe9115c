"""The synthetic acquisitions of the geometry and adjoint workloads
(tcoh_b200.scene), on CPU: the phase-grid interpolation against the
geometry oracle, the fractal heights, the box average."""

import numpy as np

import oracle

import tcoh_b200.scene as scene


def test_acquisition_geolocates_and_its_grid_phase_matches_the_oracle():
    n, rows, cols = 6, 40, 56
    geo, orbits = scene.acquisition(n, rows, cols, seed=3)
    h = scene.fbm_heights(rows, cols, hurst=0.8, hmax=1500.0, seed=4)
    g = dict(geo, hmin=float(h.min()), hmax=float(h.max()), h0=0.0)
    grid = oracle.geometry_grid(g, orbits)  # raises when a point cannot be located
    _gr, _gc, nh, hs = oracle.geometry_shape(g)
    assert nh == 3
    got = scene.grid_phases(grid, list(hs[:nh]), h)
    want = oracle.geometry_phases(g, grid, h)
    assert got.shape == want.shape == (n, rows, cols)
    assert np.abs(got - want).max() <= 1e-9 * max(1.0, np.abs(want).max())
    # the reference date sees no geometric phase of its own
    assert np.abs(got[geo["ref"]]).max() < 1e-6


def test_fbm_heights_span_and_determinism():
    a = scene.fbm_heights(64, 48, hurst=0.8, hmax=2000.0, seed=9)
    b = scene.fbm_heights(64, 48, hurst=0.8, hmax=2000.0, seed=9)
    assert np.array_equal(a, b)
    assert a.min() == 0.0 and abs(a.max() - 2000.0) < 1e-9


def test_box_average():
    rng = np.random.default_rng(0)
    f = rng.normal(size=(20, 30))
    sm = scene.smooth(f, 5)
    p = np.pad(f, 2, mode="edge")
    want = np.array([[p[r:r + 5, c:c + 5].mean() for c in range(30)] for r in range(20)])
    assert np.allclose(sm, want, atol=1e-12)
