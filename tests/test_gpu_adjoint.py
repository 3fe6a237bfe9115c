"""Adjoint of the temporal coherence on the device (B200 only), against the
FP64 torch oracle (oracle/adjoint_oracle.py, itself pinned by finite
differences in tests/test_adjoint.py)."""

import numpy as np
import pytest

import adjoint_oracle
import oracle
import tcoh_b200
from conftest import TOLERANCE, Case

pytestmark = pytest.mark.gpu


def tc_geometry(geo):
    return tcoh_b200.Geometry(*(geo[name] for name, _ in tcoh_b200.Geometry._fields_))


def compare(got, want, rel=2e-3):
    """Gradients agree to rel of their largest magnitude."""
    scale = np.abs(want).max()
    assert scale > 0
    assert np.abs(got - want).max() <= rel * scale, (np.abs(got - want).max(), scale)


@pytest.mark.parametrize("name,estimator,bias", [("topographic", "evd", False),
                                                 ("topographic", "emi", True),
                                                 ("flat_earth_ref2", "emi", False)])
def test_adjoint_matches_the_oracle(name, estimator, bias):
    c = Case(name)
    geo, orbits, _heights = c.geometry()
    grid = oracle.geometry_grid(geo, orbits)
    _gr, _gc, nh, hs = oracle.geometry_shape(geo)
    re, im, elev, row0 = c.raw_strip()
    rng = np.random.default_rng(3)
    dh = rng.normal(0.0, 5.0, (re.shape[1], re.shape[2]))
    psi = rng.normal(0.0, 0.3, re.shape).astype(np.float32)
    hr = c.window[1] // 2
    slc, amp, valid = oracle.prepare_strip(re, im, elev, row0, c.rows, hr, geo, grid)
    o = oracle.run_oracle(slc, amp, valid, c.rows, c.cols, min_shp=6, estimator=estimator,
                          bias=bias, shp_fp32=True, want_mask=True)
    _L, gam, gdh, gpsi = adjoint_oracle.adjoint(
        re, im, elev, dh, psi.astype(np.float64), row0=row0, region_rows=c.rows, halo_cols=hr,
        mask=o["mask"], count=o["count"], window=c.window, min_looks=6, estimator=estimator,
        bias=bias, grid=grid, grid_heights=hs[:nh], h0=geo["h0"])
    s = tcoh_b200.make_settings(c.n, min_shp=6, estimator=estimator, bias=bias)
    with tcoh_b200.Backend(s, c.cols + 2 * hr) as be:
        be.set_geometry(tc_geometry(geo), grid)
        r = be.adjoint_raw(re, im, elev, dh, psi, row0, c.rows, c.rows, c.cols)
    assert np.array_equal(r["count"], o["count"])
    assert np.array_equal(np.isnan(r["coh"]), np.isnan(gam))
    assert np.nanmax(np.abs(r["coh"] - gam)) < TOLERANCE
    compare(r["grad_psi"], gpsi)
    if nh == 3:
        compare(r["grad_dh"], gdh)
    else:
        assert not r["grad_dh"].any()


def test_adjoint_without_geometry_is_the_screen_gradient():
    """No geometry attached: theta = psi alone; two calls in a row agree."""
    c = Case("pairs")
    re, im, _elev, row0 = c.raw_strip()
    rng = np.random.default_rng(5)
    psi = rng.normal(0.0, 0.5, re.shape).astype(np.float32)
    hr = c.window[1] // 2
    slc, amp, valid = oracle.prepare_strip(re, im, None, row0, c.rows, hr)
    o = oracle.run_oracle(slc, amp, valid, c.rows, c.cols, min_shp=5, shp_fp32=True,
                          want_mask=True)
    _L, gam, _gdh, gpsi = adjoint_oracle.adjoint(
        re, im, None, np.zeros(re.shape[1:]), psi.astype(np.float64), row0=row0,
        region_rows=c.rows, halo_cols=hr, mask=o["mask"], count=o["count"], window=c.window,
        min_looks=5, estimator="evd", bias=False)
    s = tcoh_b200.make_settings(c.n, min_shp=5)
    with tcoh_b200.Backend(s, c.cols + 2 * hr) as be:
        r1 = be.adjoint_raw(re, im, None, None, psi, row0, c.rows, c.rows, c.cols)
        r2 = be.adjoint_raw(re, im, None, None, psi, row0, c.rows, c.rows, c.cols)
    assert np.nanmax(np.abs(r1["coh"] - gam)) < TOLERANCE
    compare(r1["grad_psi"], gpsi)
    # the candidates' sums are accumulated atomically: equal up to their order
    assert np.abs(r1["grad_psi"] - r2["grad_psi"]).max() <= 1e-5 * np.abs(gpsi).max()
