"""Parity of the CUDA path with the oracle, through the C-ABI (B200 only).

Bars (the reference's own, tests/i_sar_temporal_coherence_test.py:26-62):
SHP counts and NULL masks exactly equal, temporal coherence and pair
coherences within 1e-4 of the double-precision oracle.
"""

import numpy as np
import pytest

import oracle
import tcoh_b200
import tcoh_b200.synthetic as syn
from conftest import TOLERANCE, Case, golden_names

pytestmark = pytest.mark.gpu


def grams():
    out = ["fp32"]
    s = tcoh_b200.make_settings(6, min_shp=6)
    try:
        tcoh_b200.Backend(s, 30, gram="tensor").close()
        out.append("tensor")
    except tcoh_b200.BackendError:
        pass
    return out


GRAMS = ["fp32", "tensor"]


def backend_for(n, cols, gram, split_terms=3, chunk_pixels=0, **kw):
    if gram not in grams():
        pytest.skip("tensor-core Gram not built")
    pairs = kw.pop("pairs", False)
    pairs_all = kw.pop("pairs_all", False)
    s = tcoh_b200.make_settings(n, pairs=pairs, pairs_all=pairs_all, **kw)
    return tcoh_b200.Backend(s, cols + s.win_rg - 1, gram=gram, split_terms=split_terms,
                             chunk_pixels=chunk_pixels)


def assert_close(got, want, tol=TOLERANCE):
    assert np.array_equal(np.isnan(got), np.isnan(want))
    m = ~np.isnan(want)
    if m.any():
        err = np.abs(got[m].astype(np.float64) - want[m])
        assert err.max() <= tol, (err.max(), np.argmax(err))


@pytest.mark.parametrize("gram", GRAMS)
@pytest.mark.parametrize("name", golden_names())
def test_golden_cases(name, gram):
    c = Case(name)
    kw = c.kwargs()
    be = backend_for(c.n, c.cols, gram, window=kw["window"], shp_test=kw["shp_test"],
                     alpha=kw["alpha"], min_shp=kw["min_shp"], estimator=kw["estimator"],
                     bias=kw["bias"], pairs=c.pairs is not None, pairs_all=True)
    with be:
        slc, amp, valid = c.strip()
        r = be.run(slc, amp, valid, c.rows, c.cols, phases=True, status=True)
    assert np.array_equal(r["count"], c.count)
    assert_close(r["coh"], c.coh)
    if c.pairs is not None:
        assert_close(r["pairs"], c.pairs)


def test_strip_loop_with_small_memory():
    """test_strips of the reference: memory=1 forces several strips, whose
    seams must not show."""
    c = Case("strips")
    out = tcoh_b200.temporal_coherence(c.stack, window=(7, 5), min_shp=10, memory=1, gram="fp32")
    assert out["strip_rows"] < 30
    assert np.array_equal(out["count"], c.count)
    assert_close(out["coh"], c.coh)


def test_ocl_entry_points():
    """The drop-in path: ocl_open / ocl_run / ocl_close as main.c calls them."""
    c = Case("pairs")
    s = tcoh_b200.make_settings(c.n, min_shp=5, pairs=True, pairs_all=False)
    h, max_alloc = tcoh_b200.ocl_open(-1, -1, s, c.cols + 6)
    assert h and max_alloc > 1 << 30
    slc, amp, valid = c.strip()
    coh = np.empty((c.rows, c.cols), np.float32)
    count = np.empty((c.rows, c.cols), np.int32)
    pairs = np.empty((c.n - 1, c.rows, c.cols), np.float32)
    tcoh_b200.ocl_run(h, slc, amp, valid, slc.shape[0], c.rows, c.cols, coh, count, pairs)
    tcoh_b200.ocl_close(h)
    assert np.array_equal(count, c.count)
    assert_close(coh, c.coh)
    all_pairs = tcoh_b200.pair_list(c.n, True)
    for p, (i, j) in enumerate(tcoh_b200.pair_list(c.n, False)):
        assert_close(pairs[p], c.pairs[all_pairs.index((i, j))])


def wrap(a):
    return np.angle(np.exp(1j * a))


CASES = [
    # n, test, alpha, estimator, bias, window, g0_max
    (10, "ks", 0.05, "evd", False, (21, 7), 0.95),
    (10, "ad", 0.05, "emi", False, (21, 7), 0.95),
    (12, "tlog", 0.05, "evd", True, (21, 7), 0.95),
    (30, "ks", 0.05, "evd", False, (21, 7), 0.95),
    (30, "ad", 0.05, "emi", True, (21, 7), 0.99),
    (30, "tlog", 0.01, "emi", False, (11, 5), 0.9),
    (17, "ks", 0.1, "emi", True, (9, 9), 0.8),
    (33, "ks", 0.05, "evd", False, (21, 7), 0.95),
    (64, "ad", 0.05, "evd", False, (21, 7), 0.95),
    (64, "ks", 0.05, "emi", True, (15, 5), 0.99),
    (48, "ks", 0.05, "emi", False, (21, 7), 0.99),
]


@pytest.mark.parametrize("gram", GRAMS)
@pytest.mark.parametrize("case", CASES, ids=lambda c: "n%d-%s-%s%s-%dx%d" % (
    c[0], c[1], c[3], "-b" if c[4] else "", c[5][0], c[5][1]))
def test_synthetic_vs_oracle(case, gram):
    n, test, alpha, est, bias, win, g0 = case
    rows, cols = 37, 29  # ragged: not whole tiles
    stack = syn.generate(n, rows, cols, seed=n, g0_max=g0, nregions=3)
    ha, hr = win[0] // 2, win[1] // 2
    slc, amp, valid = tcoh_b200.read_strip(stack.real, stack.imag, -ha, rows + 2 * ha, hr)
    kw = dict(window=win, shp_test=test, alpha=alpha, min_shp=n, estimator=est, bias=bias)
    with backend_for(n, cols, gram, pairs=True, pairs_all=True, **kw) as be:
        r = be.run(slc, amp, valid, rows, cols, phases=True, status=True)
    o = oracle.run_oracle(slc, amp, valid, rows, cols, npairs=n * (n - 1) // 2, pairs_all=True,
                          shp_fp32=True, want_phases=True, **kw)
    # The SHP decisions are the reference kernel's, bit for bit.
    assert np.array_equal(r["count"], o["count"])
    # Pair coherences within 1e-4 everywhere (the reference's bar,
    # i_sar_temporal_coherence_test.py:53-62), bias-corrected ones just
    # above zero included: their float error grows as 1 / |T_c|, and the
    # pixels with such an entry (L m2 within 3e-5 of 1) come from the exact
    # tier's double sums.
    assert_close(r["pairs"], o["pairs"])
    assert np.array_equal(np.isnan(r["coh"]), np.isnan(o["coh"]))
    m = ~np.isnan(o["coh"])
    err = np.abs(r["coh"][m] - o["coh"][m])
    assert err.max() <= TOLERANCE, err.max()
    # Per-date phases, relative to the reference date. The reference writes
    # no phases (its tests check gamma and the pair coherences only), so
    # this bound is this backend's own: every phase of a pixel whose
    # coherence is at least 0.2 within 1e-3 rad of the oracle's, and 99 %
    # of all. Below 0.2 the eigenvector's phases are set by noise-level
    # differences between nearly equal eigenvalues and move by more.
    dph = np.abs(wrap(r["phases"][m].astype(np.float64) - o["phases"][m]))
    assert np.percentile(dph, 99) < 1e-3, np.percentile(dph, 99)
    strong = o["coh"][m] >= 0.2
    if strong.any():
        assert dph[strong].max() < 1e-3, dph[strong].max()


@pytest.mark.parametrize("gram", GRAMS)
def test_chunking_is_invisible(gram):
    n, rows, cols = 12, 70, 45
    stack = syn.generate(n, rows, cols, seed=5)
    slc, amp, valid = tcoh_b200.read_strip(stack.real, stack.imag, -10, rows + 20, 3)
    outs = []
    for chunk in (0, 128):
        with backend_for(n, cols, gram, chunk_pixels=chunk, min_shp=n) as be:
            outs.append(be.run(slc, amp, valid, rows, cols))
    assert np.array_equal(outs[0]["count"], outs[1]["count"])
    assert np.array_equal(outs[0]["coh"], outs[1]["coh"], equal_nan=True)


@pytest.mark.parametrize("test", ["ks", "ad", "tlog"])
@pytest.mark.parametrize("chunk", [0, 256])
def test_shp_with_tied_amplitudes(test, chunk):
    """Amplitudes rounded to a coarse grid, so that most pairs of
    series share values: each pair is tested once in a block of chunks and
    its other direction taken from the same test when the series share no
    value, walked again the other way when they do. The counts must still
    be the reference kernel's, bit for bit; with chunks of 256 pixels the
    300 rows make 19 chunks of 16 rows, two blocks of at most 16 chunks,
    so that pairs also cross a block edge."""
    n, rows, cols = 10, 300, 20
    stack = syn.generate(n, rows, cols, seed=11, null_frac=0.0)
    # amplitudes on multiples of 64 (about a tenth of their mean) and phases
    # on multiples of pi / 2, so that the float amplitudes sqrt(re^2 + im^2)
    # are those multiples exactly
    q = np.maximum(np.round(np.abs(stack) / 64.0) * 64.0, 64.0)
    quarter = np.round(np.angle(stack) / (np.pi / 2)).astype(int) % 4
    stack = (q * np.array([1, 1j, -1, -1j])[quarter]).astype(np.complex64)
    slc, amp, valid = tcoh_b200.read_strip(stack.real, stack.imag, -10, rows + 20, 3)
    kw = dict(window=(21, 7), shp_test=test, alpha=0.05, min_shp=n, estimator="evd")
    a = amp.reshape(-1, n)
    assert sum(np.intersect1d(a[1000], a[1000 + k]).size > 0 for k in range(1, 8)) > 4
    with backend_for(n, cols, "fp32", chunk_pixels=chunk, **kw) as be:
        r = be.run(slc, amp, valid, rows, cols)
    o = oracle.run_oracle(slc, amp, valid, rows, cols, shp_fp32=True, **kw)
    assert np.array_equal(r["count"], o["count"])
    assert_close(r["coh"], o["coh"])


@pytest.mark.parametrize("gram", GRAMS)
@pytest.mark.parametrize("rows,cols", [(1, 1), (1, 9), (17, 1), (3, 200)])
def test_tiny_and_ragged_regions(rows, cols, gram):
    n = 6
    stack = syn.generate(n, rows, cols, seed=rows * 100 + cols, null_frac=0.0)
    slc, amp, valid = tcoh_b200.read_strip(stack.real, stack.imag, -2, rows + 4, 1)
    kw = dict(window=(5, 3), min_shp=2)
    with backend_for(n, cols, gram, **kw) as be:
        r = be.run(slc, amp, valid, rows, cols)
    o = oracle.run_oracle(slc, amp, valid, rows, cols, shp_fp32=True, **kw)
    assert np.array_equal(r["count"], o["count"])
    assert_close(r["coh"], o["coh"])


@pytest.mark.parametrize("gram", GRAMS)
def test_all_null_strip(gram):
    n, rows, cols = 5, 20, 20
    re = np.full((n, rows, cols), np.nan, np.float32)
    slc, amp, valid = tcoh_b200.read_strip(re, re, -10, rows + 20, 3)
    with backend_for(n, cols, gram, min_shp=5, pairs=True) as be:
        r = be.run(slc, amp, valid, rows, cols)
    assert (r["count"] == -1).all() and np.isnan(r["coh"]).all() and np.isnan(r["pairs"]).all()


@pytest.mark.parametrize("estimator", ["evd", "emi"])
def test_coherent_and_incoherent_stacks(estimator):
    means = {}
    for g in ("95", "0"):
        c = Case("coherence%s_%s" % (g, estimator))
        out = tcoh_b200.temporal_coherence(c.stack, estimator=estimator)
        means[g] = np.nanmean(out["coh"])
    assert means["95"] > 0.9
    assert means["0"] < 0.5


def test_flat_earth_removal_restores_coherence():
    """Without the geometric correction the fringes decorrelate the windows
    (test_flat_earth_phase of the reference)."""
    c = Case("flat_earth_ref0")
    corrected = tcoh_b200.temporal_coherence(c.stack, min_shp=6, pairs=True, pairs_mode="all",
                                             phase=c.phase)
    raw = tcoh_b200.temporal_coherence(c.stack, min_shp=6, pairs=True, pairs_mode="all")
    p = tcoh_b200.pair_list(6, True).index((2, 3))
    assert np.nanmean(corrected["pairs"][p]) > np.nanmean(raw["pairs"][p]) + 0.1


def test_device_resident_strip():
    torch = pytest.importorskip("torch")
    n, rows, cols = 10, 33, 40
    stack = syn.generate(n, rows, cols, seed=9)
    slc, amp, valid = tcoh_b200.read_strip(stack.real, stack.imag, -10, rows + 20, 3)
    with backend_for(n, cols, "fp32", min_shp=n, pairs=True) as be:
        host = be.run(slc, amp, valid, rows, cols, phases=True)
        dev = torch.device("cuda:0")
        d_slc, d_amp, d_valid = (torch.from_numpy(a).to(dev) for a in (slc, amp, valid))
        coh = torch.empty((rows, cols), dtype=torch.float32, device=dev)
        count = torch.empty((rows, cols), dtype=torch.int32, device=dev)
        pairs = torch.empty((n - 1, rows, cols), dtype=torch.float32, device=dev)
        phases = torch.empty((rows, cols, n), dtype=torch.float32, device=dev)
        stream = torch.cuda.current_stream()
        be.run_device(d_slc, d_amp, d_valid, rows, cols, coh, count, pairs, phases, stream=stream)
        torch.cuda.synchronize()
    assert np.array_equal(count.cpu().numpy(), host["count"])
    assert np.array_equal(coh.cpu().numpy(), host["coh"], equal_nan=True)
    assert np.array_equal(pairs.cpu().numpy(), host["pairs"], equal_nan=True)
    assert np.array_equal(phases.cpu().numpy(), host["phases"], equal_nan=True)


@pytest.mark.parametrize("n,est,win", [(10, "evd", (21, 7)), (64, "evd", (21, 7)),
                                       (30, "evd", (11, 5))])
def test_tensor_gram_two_terms(n, est, win):
    """Two BF16 terms per product (16 significant bits): within the
    tolerance on well-conditioned estimators."""
    rows, cols = 37, 29
    stack = syn.generate(n, rows, cols, seed=n + 1, nregions=3)
    ha, hr = win[0] // 2, win[1] // 2
    slc, amp, valid = tcoh_b200.read_strip(stack.real, stack.imag, -ha, rows + 2 * ha, hr)
    kw = dict(window=win, shp_test="ks", min_shp=n, estimator=est)
    with backend_for(n, cols, "tensor", split_terms=2, **kw) as be:
        r = be.run(slc, amp, valid, rows, cols)
    o = oracle.run_oracle(slc, amp, valid, rows, cols, shp_fp32=True, **kw)
    assert np.array_equal(r["count"], o["count"])
    assert_close(r["coh"], o["coh"])


@pytest.mark.parametrize("win", [(33, 25), (63, 3), (1, 25)])
def test_tensor_gram_window_extremes(win):
    """The widest and tallest windows the tensor-core Gram takes: the union
    of a tile's windows spans up to 32 columns and 78 rows."""
    n, rows, cols = 8, 40, 27
    stack = syn.generate(n, rows, cols, seed=win[0] * 100 + win[1], nregions=2)
    ha, hr = win[0] // 2, win[1] // 2
    slc, amp, valid = tcoh_b200.read_strip(stack.real, stack.imag, -ha, rows + 2 * ha, hr)
    kw = dict(window=win, shp_test="ad", min_shp=n, estimator="evd")
    with backend_for(n, cols, "tensor", pairs=True, pairs_all=True, **kw) as be:
        r = be.run(slc, amp, valid, rows, cols)
    o = oracle.run_oracle(slc, amp, valid, rows, cols, shp_fp32=True, npairs=n * (n - 1) // 2,
                          pairs_all=True, **kw)
    assert np.array_equal(r["count"], o["count"])
    assert_close(r["coh"], o["coh"])
    assert_close(r["pairs"], o["pairs"])


def test_tensor_gram_rejects_windows_beyond_its_tiles():
    s = tcoh_b200.make_settings(8, window=(5, 27), min_shp=8)
    with pytest.raises(tcoh_b200.BackendError, match="tensor-core Gram not available"):
        tcoh_b200.Backend(s, 40, gram="tensor")
    with tcoh_b200.Backend(s, 40) as be:  # the default falls back to FP32
        assert be.gram == "fp32"
