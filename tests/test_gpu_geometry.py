"""Geometry and strip preparation on the device (B200 only): the FP64 phase
grid against the oracle's restatement of geometry.c / orbit.c, the raw-strip
preparation against main.c:52-127, and the reference's own geometry tests
(test_flat_earth_phase, test_topographic_phase) end to end."""

import numpy as np
import pytest

import oracle
import tcoh_b200
import tcoh_b200.synthetic as syn
from conftest import GEOMETRY_CASES, TOLERANCE, Case

pytestmark = pytest.mark.gpu


def tc_geometry(geo):
    return tcoh_b200.Geometry(*(geo[name] for name, _ in tcoh_b200.Geometry._fields_))


@pytest.mark.parametrize("name", GEOMETRY_CASES)
def test_phase_grid_matches_the_oracle(name):
    c = Case(name)
    geo, orbits, _heights = c.geometry()
    want = oracle.geometry_grid(geo, orbits)
    got = tcoh_b200.geometry_grid(tc_geometry(geo), orbits)
    assert got.shape == want.shape
    # phases of up to ~1e5 rad, both in double precision
    assert np.abs(got - want).max() < 1e-6


@pytest.mark.parametrize("name", GEOMETRY_CASES)
def test_flat_earth_and_topographic_phase_end_to_end(name):
    """The module's geometry path against reference.py fed with the exact
    phase of the orbit model (the reference's test criterion)."""
    c = Case(name)
    geo, orbits, heights = c.geometry()
    out = tcoh_b200.temporal_coherence(
        c.stack, min_shp=6, pairs=True, pairs_mode="all", elevation=heights,
        geometry=tc_geometry(geo), orbits=orbits)
    assert np.array_equal(out["count"], c.count)
    assert np.allclose(out["coh"], c.coh, rtol=0, atol=TOLERANCE, equal_nan=True)
    assert np.allclose(out["pairs"], c.pairs, rtol=0, atol=TOLERANCE, equal_nan=True)


@pytest.mark.parametrize("name", GEOMETRY_CASES)
def test_raw_strip_preparation_matches_the_oracle(name):
    """Device strip preparation (validity, sorted amplitudes, rotation)
    through tc_run_raw against the oracle's restatement of main.c:52-127 fed
    to the same backend: identical SHP counts, coherence within the
    tolerance (the rotated samples may differ in their last bit where the
    device's and the host's double cos / sin round differently)."""
    c = Case(name)
    geo, orbits, _heights = c.geometry()
    grid = oracle.geometry_grid(geo, orbits)
    re, im, elev, row0 = c.raw_strip()
    slc, amp, valid = oracle.prepare_strip(re, im, elev, row0, c.rows, c.window[1] // 2, geo,
                                           grid)
    s = tcoh_b200.make_settings(c.n, min_shp=6, pairs=True, pairs_all=True)
    with tcoh_b200.Backend(s, c.cols + 6) as be:
        want = be.run(slc, amp, valid, c.rows, c.cols)
        be.set_geometry(tc_geometry(geo), grid)
        got = be.run_raw(re, im, elev, row0, c.rows, c.rows, c.cols)
    assert np.array_equal(got["count"], want["count"])
    assert np.allclose(got["coh"], want["coh"], rtol=0, atol=1e-5, equal_nan=True)
    assert np.allclose(got["pairs"], want["pairs"], rtol=0, atol=1e-5, equal_nan=True)


@pytest.mark.parametrize("n", [6, 12, 30, 40])
def test_raw_strip_without_geometry_is_the_host_strip(n):
    """Without geometry the device preparation builds exactly the strip of
    the host reader: outputs equal bit for bit, NULLs, zero samples and
    NULL heights included."""
    rows, cols = 23, 19
    stack = syn.generate(n, rows, cols, seed=n + 7, nregions=2, null_frac=0.05)
    stack[1, 3, 4] = 0.0
    elevation = np.zeros((rows, cols))
    elevation[5, 6] = np.nan
    ha, hr = 4, 2
    re = np.ascontiguousarray(stack.real, np.float32)
    im = np.ascontiguousarray(stack.imag, np.float32)
    slc, amp, valid = tcoh_b200.read_strip(re, im, -ha, rows + 2 * ha, hr, elevation=elevation)
    rre = np.full((n, rows + 2 * ha, cols), np.nan, np.float32)
    rim = rre.copy()
    rre[:, ha:ha + rows] = re
    rim[:, ha:ha + rows] = im
    rel = np.zeros((rows + 2 * ha, cols))
    rel[ha:ha + rows] = elevation
    s = tcoh_b200.make_settings(n, window=(9, 5), min_shp=n, pairs=True)
    with tcoh_b200.Backend(s, cols + 2 * hr) as be:
        want = be.run(slc, amp, valid, rows, cols, phases=True, status=True)
        got = be.run_raw(rre, rim, rel, -ha, rows, rows, cols, phases=True, status=True)
    for key in ("coh", "count", "pairs", "phases", "status"):
        assert np.array_equal(got[key], want[key], equal_nan=True), key


def test_geometry_errors_are_reported():
    c = Case("flat_earth_ref0")
    geo, orbits, _heights = c.geometry()
    short = [(t[:5], p[:5], v[:5]) for t, p, v in orbits]
    with pytest.raises(tcoh_b200.BackendError, match="state vectors"):
        tcoh_b200.geometry_grid(tc_geometry(geo), short)
    # an orbit that ends before the scene: the ground point is outside it
    late = dict(geo, first_line_time=geo["first_line_time"] + 3600.0)
    with pytest.raises(tcoh_b200.BackendError, match="outside of an orbit|Geolocation failed"):
        tcoh_b200.geometry_grid(tc_geometry(late), orbits)
