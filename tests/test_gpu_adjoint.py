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


@pytest.mark.parametrize("gram", ["tensor", "fp32"])
def test_adjoint_thirty_dates(gram):
    """N = 30 on a synthetic acquisition over fractal heights (0 - 400 m),
    through both forms of the scatter: the transposed tensor-core Gram
    (gram "tensor") and the CUDA-core one (gram "fp32"). Two tiles across and
    two down share candidates, so the atomic sums across tiles are covered."""
    import tcoh_b200.scene as scene
    import tcoh_b200.synthetic as syn

    n, rows, cols, window = 30, 32, 16, (21, 7)
    ha, hr = window[0] // 2, window[1] // 2
    geo, orbits = scene.acquisition(n, rows, cols, seed=21)
    h = scene.fbm_heights(rows, cols, hmax=400.0, seed=22)
    geo.update(hmin=float(h.min()), hmax=float(h.max()), h0=0.0)
    grid = oracle.geometry_grid(geo, orbits)
    _gr, _gc, nh, hs = oracle.geometry_shape(geo)
    assert nh == 3
    stack = syn.generate(n, rows, cols, nregions=3, g0_max=0.95, seed=23, null_frac=0.02)
    prow = rows + 2 * ha
    re = np.full((n, prow, cols), np.nan, np.float32)
    im = re.copy()
    re[:, ha:ha + rows] = stack.real
    im[:, ha:ha + rows] = stack.imag
    elev = np.full((prow, cols), np.nan)
    elev[ha:ha + rows] = h
    rng = np.random.default_rng(24)
    dh = rng.normal(0.0, 5.0, (prow, cols))
    psi = rng.normal(0.0, 0.3, re.shape).astype(np.float32)
    slc, amp, valid = oracle.prepare_strip(re, im, elev, -ha, rows, hr, geo, grid)
    o = oracle.run_oracle(slc, amp, valid, rows, cols, window=window, min_shp=10,
                          estimator="evd", shp_fp32=True, want_mask=True)
    _L, gam, gdh, gpsi = adjoint_oracle.adjoint(
        re, im, elev, dh, psi.astype(np.float64), row0=-ha, region_rows=rows, halo_cols=hr,
        mask=o["mask"], count=o["count"], window=window, min_looks=max(10, n), estimator="evd",
        bias=False, grid=grid, grid_heights=hs[:nh], h0=0.0)
    s = tcoh_b200.make_settings(n, window=window, min_shp=10)
    with tcoh_b200.Backend(s, cols + 2 * hr, gram=gram) as be:
        be.set_geometry(tc_geometry(geo), grid)
        r = be.adjoint_raw(re, im, elev, dh, psi, -ha, rows, rows, cols)
    assert np.array_equal(r["count"], o["count"])
    # a pixel needs max(min_shp, N) looks (main.c:585-587): some have fewer
    assert np.isnan(gam).any() and not np.isnan(gam).all()
    assert np.array_equal(np.isnan(r["coh"]), np.isnan(gam))
    assert np.nanmax(np.abs(r["coh"] - gam)) < TOLERANCE
    compare(r["grad_psi"], gpsi)
    compare(r["grad_dh"], gdh)


class CoherenceSum:
    """torch.autograd.Function over tc_adjoint_raw (test harness only): L =
    sum of gamma over the estimated pixels as a function of the height error
    dh and the phase screen psi; the backward returns the device adjoint."""

    @staticmethod
    def function(be, re, im, elev, row0, rows, cols):
        import torch

        class F(torch.autograd.Function):
            @staticmethod
            def forward(ctx, dh, psi):
                r = be.adjoint_raw(re, im, elev, dh.detach().numpy(),
                                   psi.detach().numpy().astype(np.float32), row0, rows, rows, cols)
                ctx.save_for_backward(torch.from_numpy(r["grad_dh"].astype(np.float64)),
                                      torch.from_numpy(r["grad_psi"].astype(np.float64)))
                return torch.tensor(np.nansum(r["coh"].astype(np.float64)), dtype=torch.float64)

            @staticmethod
            def backward(ctx, gl):
                gdh, gpsi = ctx.saved_tensors
                return gl * gdh, gl * gpsi

        return F.apply


def test_autograd_function_matches_finite_differences():
    """The Function's gradient against central differences of the device
    forward at N = 30: along its own direction to 1e-3 relative (steps of
    0.05 m and 0.01 rad in norm), and along random directions (steps of
    0.01 m and 0.0005 rad per cell) to 1e-3 of |grad| |direction|."""
    import torch

    import tcoh_b200.scene as scene
    import tcoh_b200.synthetic as syn

    n, rows, cols, window = 30, 32, 16, (21, 7)
    ha, hr = window[0] // 2, window[1] // 2
    geo, orbits = scene.acquisition(n, rows, cols, seed=31)
    h = scene.fbm_heights(rows, cols, hmax=800.0, seed=32)
    geo.update(hmin=float(h.min()), hmax=float(h.max()), h0=0.0)
    grid = oracle.geometry_grid(geo, orbits)
    stack = syn.generate(n, rows, cols, nregions=2, g0_max=0.95, seed=33, null_frac=0.0)
    prow = rows + 2 * ha
    re = np.full((n, prow, cols), np.nan, np.float32)
    im = re.copy()
    re[:, ha:ha + rows] = stack.real
    im[:, ha:ha + rows] = stack.imag
    elev = np.full((prow, cols), np.nan)
    elev[ha:ha + rows] = h
    rng = np.random.default_rng(34)
    x0 = {"dh": rng.normal(0.0, 5.0, (prow, cols)), "psi": rng.normal(0.0, 0.2, re.shape)}
    s = tcoh_b200.make_settings(n, window=window, min_shp=20)
    with tcoh_b200.Backend(s, cols + 2 * hr) as be:
        be.set_geometry(tc_geometry(geo), grid)
        f = CoherenceSum.function(be, re, im, elev, -ha, rows, cols)
        x = {k: torch.tensor(v, requires_grad=True) for k, v in x0.items()}
        loss = f(x["dh"], x["psi"])
        loss.backward()
        assert loss.item() > 0

        def along(name, d, eps):
            with torch.no_grad():
                lp = f(*(torch.tensor(x0[k] + (eps * d if k == name else 0.0)) for k in x0)).item()
                lm = f(*(torch.tensor(x0[k] - (eps * d if k == name else 0.0)) for k in x0)).item()
            return (lp - lm) / (2 * eps)

        for name, step, cell_step in (("dh", 0.05, 0.01), ("psi", 0.01, 5e-4)):
            g = x[name].grad.numpy()
            gn = np.linalg.norm(g)
            assert along(name, g / gn, step) == pytest.approx(gn, rel=1e-3)
            d = rng.normal(0.0, 1.0, g.shape)
            fd = along(name, d, cell_step)
            assert abs(fd - (g * d).sum()) <= 1e-3 * gn * np.linalg.norm(d), (name, fd, (g * d).sum())
