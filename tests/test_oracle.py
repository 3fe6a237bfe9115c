"""The oracle against the reference: golden vectors from tests/reference.py
(the reference's FP64 oracle) and the reference kernel compiled as C."""

import numpy as np
import pytest

import oracle
from conftest import GOLDEN, TOLERANCE, Case


@pytest.mark.parametrize("shp_fp32", [False, True])
def test_oracle_matches_reference_py(golden_case, shp_fp32):
    c = golden_case
    slc, amp, valid = c.strip()
    npairs = c.n * (c.n - 1) // 2 if c.pairs is not None else 0
    o = oracle.run_oracle(slc, amp, valid, c.rows, c.cols, npairs=npairs, pairs_all=True,
                          shp_fp32=shp_fp32, **c.kwargs())
    assert np.array_equal(o["count"], c.count)
    assert np.array_equal(np.isnan(o["coh"]), np.isnan(c.coh))
    m = ~np.isnan(c.coh)
    # Samples rotated by a geometric phase are rounded to float (main.c:121-122).
    tol = 1e-7 if c.phase is not None else 1e-12
    assert np.allclose(o["coh"][m], c.coh[m], rtol=0, atol=tol)
    if npairs:
        assert np.array_equal(np.isnan(o["pairs"]), np.isnan(c.pairs))
        pm = ~np.isnan(c.pairs)
        assert np.allclose(o["pairs"][pm], c.pairs[pm], rtol=0, atol=tol)


def test_statistics_known_answers():
    # tests/i_sar_temporal_coherence_test.py:30-46 of the reference, whose
    # statistics reference.py checks against scipy.stats.
    d = np.load(GOLDEN + "/statistics.npz")
    for a, b, ad, ks in zip(d["a"], d["b"], d["ad"], d["ks"]):
        a32, b32 = np.sort(a.astype(np.float32)), np.sort(b.astype(np.float32))
        assert oracle.ad_statistic(a32, b32) == pytest.approx(ad, rel=1e-6)
        assert oracle.ks_accept(a32, b32, 0.05) == bool(ks)
    for n, sigma in zip(range(3, 65), d["ad_sigma"]):
        assert oracle.ad_sigma(n) == pytest.approx(sigma, rel=1e-12)
    for alpha, crit in zip((0.001, 0.003, 0.01, 0.05, 0.1, 0.2, 0.25), d["ad_critical"]):
        assert oracle.ad_critical(alpha) == pytest.approx(crit, rel=1e-12)
    assert oracle.ad_critical(0.05) == pytest.approx(1.961)
    assert oracle.ad_critical(0.01) == pytest.approx(3.752)


def test_scipy_statistics():
    stats = pytest.importorskip("scipy.stats")
    rng = np.random.default_rng(11)
    for n in (5, 12, 30):
        for _ in range(10):
            a = np.sort(rng.rayleigh(size=n)).astype(np.float32)
            b = np.sort(rng.rayleigh(scale=1.4, size=n)).astype(np.float32)
            import warnings

            with warnings.catch_warnings():
                warnings.simplefilter("ignore")
                want = stats.anderson_ksamp([a.astype(float), b.astype(float)], midrank=False).statistic
            assert oracle.ad_statistic(a, b) == pytest.approx(want, rel=1e-9)


def test_eigensolver():
    rng = np.random.default_rng(3)
    for n in (2, 5, 30, 64):
        x = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
        h = x @ x.conj().T
        w, v = oracle.hermitian_eigen(h)
        assert np.allclose(np.sort(w), np.linalg.eigvalsh(h), rtol=1e-12, atol=1e-10)
        assert np.allclose(h @ v, v * w[None, :], atol=1e-9 * np.abs(w).max())


@pytest.mark.skipif(not oracle.reference_available(), reason="oracle/_ref not built")
def test_reference_kernel_matches_reference_py(golden_case):
    c = golden_case
    slc, amp, valid = c.strip()
    npairs = c.n * (c.n - 1) // 2 if c.pairs is not None else 0
    r = oracle.run_reference(slc, amp, valid, c.rows, c.cols, npairs=npairs, pairs_all=True,
                             **c.kwargs())
    assert np.array_equal(r["count"], c.count)
    assert np.array_equal(np.isnan(r["coh"]), np.isnan(c.coh))
    m = ~np.isnan(c.coh)
    assert np.allclose(r["coh"][m], c.coh[m], rtol=0, atol=TOLERANCE)


@pytest.mark.skipif(not oracle.reference_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("n,test,alpha", [(10, "ks", 0.05), (10, "ad", 0.05), (30, "ad", 0.01),
                                          (12, "tlog", 0.05), (30, "tlog", 0.01)])
def test_oracle_float_shp_is_the_reference_kernel(n, test, alpha):
    """The oracle's float SHP statistics decide as the reference kernel."""
    import tcoh_b200.synthetic as syn

    stack = syn.generate(n, 40, 32, seed=n, g0_max=0.9)
    import tcoh_b200

    slc, amp, valid = tcoh_b200.read_strip(stack.real, stack.imag, -10, 60, 3)
    kw = dict(window=(21, 7), shp_test=test, alpha=alpha, min_shp=n, estimator="evd")
    r = oracle.run_reference(slc, amp, valid, 40, 32, **kw)
    o = oracle.run_oracle(slc, amp, valid, 40, 32, shp_fp32=True, **kw)
    assert np.array_equal(r["count"], o["count"])


@pytest.mark.skipif(not oracle.reference_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("n,test,estimator,bias", [(10, "ks", "evd", False),
                                                   (30, "ad", "emi", True),
                                                   (60, "ks", "emi", False)])
def test_specialised_reference_build_is_the_generic_one(n, test, estimator, bias):
    """The reference kernel built with one configuration's -D constants (as
    ocl.c:222-229 builds it; the CPU baseline runs it) gives the outputs of
    the generic build bit for bit."""
    import tcoh_b200
    import tcoh_b200.synthetic as syn

    kw = dict(window=(21, 7), shp_test=test, alpha=0.05, min_shp=10 if n == 10 else 20,
              estimator=estimator, bias=bias)
    cols = 1024 if n == 60 else 512
    if oracle.ref_build(n, (21, 7), cols + 6, npairs=0, pairs_all=False,
                        **{k: v for k, v in kw.items() if k != "window"}) != "specialised":
        pytest.skip("the specialised build of this configuration is absent")
    stack = syn.generate(n, 3, cols, seed=n, g0_max=0.99, spacing=6.0 if n == 60 else 12.0)
    slc, amp, valid = tcoh_b200.read_strip(stack.real, stack.imag, -10, 23, 3)
    spec = oracle.run_reference(slc, amp, valid, 3, cols, **kw)
    gen = oracle._ref_lib(False)  # the generic build, called directly
    k = oracle.kernel_constants(n, test, 0.05)
    coh = np.empty((3, cols), np.float32)
    count = np.empty((3, cols), np.int32)
    pairs = np.empty((1, 3, cols), np.float32)
    assert gen.ref_run(n, 21, 7, oracle.TESTS[test], int(estimator == "emi"), int(bias),
                       max(kw["min_shp"], n), k.ks_max, k.ad_norm, k.ad_sigma, k.ad_crit,
                       k.tlog_crit, 0, oracle._ptr(slc), oracle._ptr(amp), oracle._ptr(valid),
                       23, cols + 6, 3, cols, oracle._ptr(coh), oracle._ptr(count),
                       oracle._ptr(pairs), 0) == 0
    assert np.array_equal(spec["count"], count)
    assert np.array_equal(spec["coh"], coh, equal_nan=True)


@pytest.mark.parametrize("name", ["flat_earth_ref0", "flat_earth_ref2", "topographic"])
def test_geometry_oracle_matches_the_orbit_model(name):
    """The phase grid restated from geometry.c and orbit.c, interpolated at
    every cell, against the reference test's independent orbit model
    (tests/geometry_model.py, Stack.phases): the grid's interpolation error
    is a fraction of a milliradian on phases of tens of thousands of
    radians."""
    c = Case(name)
    geo, orbits, heights = c.geometry()
    grid = oracle.geometry_grid(geo, orbits)
    h = heights if heights is not None else np.full((c.rows, c.cols), geo["h0"])
    ph = oracle.geometry_phases(geo, grid, h)
    assert np.abs(np.angle(np.exp(1j * (ph - c.phase)))).max() < 1e-3


@pytest.mark.parametrize("name", ["flat_earth_ref0", "flat_earth_ref2", "topographic"])
def test_geometry_oracle_end_to_end(name):
    """test_flat_earth_phase / test_topographic_phase of the reference
    (tests/i_sar_temporal_coherence_test.py:389-458): the coherence with the
    orbit-derived, grid-interpolated phase removed matches reference.py fed
    with the exact model phase within the tolerance."""
    c = Case(name)
    geo, orbits, _heights = c.geometry()
    grid = oracle.geometry_grid(geo, orbits)
    re, im, elev, row0 = c.raw_strip()
    slc, amp, valid = oracle.prepare_strip(re, im, elev, row0, c.rows, c.window[1] // 2, geo, grid)
    npairs = c.n * (c.n - 1) // 2
    o = oracle.run_oracle(slc, amp, valid, c.rows, c.cols, npairs=npairs, pairs_all=True,
                          **c.kwargs())
    assert np.array_equal(o["count"], c.count)
    assert np.allclose(o["coh"], c.coh, rtol=0, atol=TOLERANCE, equal_nan=True)
    assert np.allclose(o["pairs"], c.pairs, rtol=0, atol=TOLERANCE, equal_nan=True)


def test_strip_preparation_oracle_matches_the_host_reader():
    """Without geometry, the C restatement of main.c:52-127 and the package's
    host reader build the same strip, bit for bit."""
    import tcoh_b200

    c = Case("nulls")
    re, im, _elev, row0 = c.raw_strip()
    slc, amp, valid = oracle.prepare_strip(re, im, None, row0, c.rows, c.window[1] // 2)
    hs, ha, hv = c.strip()
    assert np.array_equal(valid, hv)
    assert np.array_equal(amp, ha)
    assert np.array_equal(slc, hs)
