"""The adjoint oracle (oracle/adjoint_oracle.py) pinned on CPU: its forward
against the C oracle, its gradient against central finite differences in
FP64 (a step of 1e-3 m in height, 1e-5 rad in phase)."""

import numpy as np
import pytest

import adjoint_oracle
import oracle
from conftest import Case


def setup(estimator, bias, seed=0):
    c = Case("topographic")
    geo, orbits, _heights = c.geometry()
    grid = oracle.geometry_grid(geo, orbits)
    _gr, _gc, nh, hs = oracle.geometry_shape(geo)
    re, im, elev, row0 = c.raw_strip()
    rng = np.random.default_rng(seed)
    dh = rng.normal(0.0, 5.0, elev.shape)
    psi = rng.normal(0.0, 0.3, re.shape)
    hr = c.window[1] // 2
    slc, amp, valid = oracle.prepare_strip(re, im, elev, row0, c.rows, hr, geo, grid)
    o = oracle.run_oracle(slc, amp, valid, c.rows, c.cols, min_shp=6, estimator=estimator,
                          bias=bias, shp_fp32=True, want_mask=True)
    args = dict(row0=row0, region_rows=c.rows, halo_cols=hr, mask=o["mask"], count=o["count"],
                window=c.window, min_looks=6, estimator=estimator, bias=bias, grid=grid,
                grid_heights=hs[:nh])
    return c, re, im, elev, dh, psi, args, o


@pytest.mark.parametrize("estimator,bias", [("evd", False), ("emi", True)])
def test_adjoint_oracle_forward_is_the_oracle(estimator, bias):
    """With no height error and no screen, the torch forward is the C
    oracle's coherence (samples rotated in double here, rounded to float
    there)."""
    c, re, im, elev, dh, psi, args, o = setup(estimator, bias)
    _L, gam, _gdh, _gpsi = adjoint_oracle.adjoint(re, im, elev, 0 * dh, 0 * psi, **args)
    assert np.array_equal(np.isnan(gam), np.isnan(o["coh"]))
    assert np.nanmax(np.abs(gam - o["coh"])) < 1e-5


@pytest.mark.parametrize("estimator,bias", [("evd", False), ("emi", True)])
def test_adjoint_oracle_matches_finite_differences(estimator, bias):
    c, re, im, elev, dh, psi, args, _o = setup(estimator, bias)
    _L, _gam, gdh, gpsi = adjoint_oracle.adjoint(re, im, elev, dh, psi, **args)

    def loss(d, p):
        return adjoint_oracle.adjoint(re, im, elev, d, p, **args)[0]

    for r, col in ((15, 12), (20, 5)):
        e = 1e-3
        d1, d2 = dh.copy(), dh.copy()
        d1[r, col] += e
        d2[r, col] -= e
        fd = (loss(d1, psi) - loss(d2, psi)) / (2 * e)
        assert gdh[r, col] == pytest.approx(fd, rel=1e-4, abs=1e-8)
    for k, r, col in ((2, 15, 12), (5, 25, 20)):
        e = 1e-5
        p1, p2 = psi.copy(), psi.copy()
        p1[k, r, col] += e
        p2[k, r, col] -= e
        fd = (loss(dh, p1) - loss(dh, p2)) / (2 * e)
        assert gpsi[k, r, col] == pytest.approx(fd, rel=1e-4, abs=1e-8)
