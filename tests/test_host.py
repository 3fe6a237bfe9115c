"""Host-side logic and the C-ABI library, without a GPU."""

import ctypes
import subprocess
import sys

import numpy as np
import pytest

import oracle
import tcoh_b200
from conftest import ROOT, header_functions


def test_library_exports_every_declared_function():
    lib = tcoh_b200.library()
    declared = header_functions()
    assert {"ocl_list_devices", "ocl_open", "ocl_run", "ocl_close"} <= set(declared)
    for name in declared:
        assert hasattr(lib, name), name
    assert set(declared) == set(tcoh_b200.EXPORTS)


@pytest.mark.parametrize("n,ks", [(10, 6), (20, 8), (30, 10), (60, 14)])
def test_ks_threshold(n, ks):
    assert tcoh_b200.make_settings(n, min_shp=n).ks_max == ks


@pytest.mark.parametrize("test,alpha", [("ks", 0.05), ("ad", 0.05), ("ad", 0.003), ("tlog", 0.01)])
@pytest.mark.parametrize("n", [3, 6, 30, 64])
def test_constants_match_kernel_build(test, alpha, n):
    """tc_shp_constants gives the doubles of stats.c; written as float
    literals they are the oracle's kernel constants."""
    s = tcoh_b200.make_settings(n, shp_test=test, alpha=alpha, min_shp=n)
    k = oracle.kernel_constants(n, test, alpha)
    f = lambda v: np.float32(float("%.9e" % v))  # noqa: E731
    assert s.ks_max == k.ks_max
    assert f(s.ad_norm) == np.float32(k.ad_norm)
    assert f(s.ad_sigma) == np.float32(k.ad_sigma)
    assert f(s.ad_crit) == np.float32(k.ad_crit)
    assert f(s.tlog_crit) == np.float32(k.tlog_crit)


@pytest.mark.parametrize("kwargs,message", [
    ({"window": (20, 7)}, "odd"),
    ({"window": (3, 3), "min_shp": 20}, "fewer pixels"),
    ({"alpha": 1.5}, "alpha"),
])
def test_option_failures(kwargs, message):
    with pytest.raises(ValueError, match=message):
        tcoh_b200.make_settings(6, **kwargs)


def test_ad_alpha_range():
    with pytest.raises(tcoh_b200.BackendError, match="alpha"):
        tcoh_b200.make_settings(6, shp_test="ad", alpha=0.5)


def test_pair_order():
    assert tcoh_b200.pair_list(4, True) == [(0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3)]
    assert tcoh_b200.pair_list(4, False) == [(0, 1), (1, 2), (2, 3)]
    assert tcoh_b200.npairs_for(30, True, True) == 435


def test_read_strip_layout():
    rng = np.random.default_rng(0)
    n, rows, cols = 4, 6, 5
    re = np.round(rng.standard_normal((n, rows, cols)) * 10).astype(np.float32)
    im = np.round(rng.standard_normal((n, rows, cols)) * 10).astype(np.float32)
    re[1, 2, 3] = np.nan
    re[2, 4, 1] = 0
    im[2, 4, 1] = 0
    elev = np.zeros((rows, cols))
    elev[0, 0] = np.nan
    slc, amp, valid = tcoh_b200.read_strip(re, im, -1, rows + 2, 2, elevation=elev)
    assert slc.shape == (rows + 2, cols + 4, n, 2) and amp.shape == (rows + 2, cols + 4, n)
    # halo rows and columns are invalid and zero
    assert not valid[0].any() and not valid[-1].any() and not valid[:, :2].any()
    assert not slc[0].any() and not amp[:, -2:].any()
    assert valid[1 + 2, 2 + 3] == 0 and valid[1 + 4, 2 + 1] == 0 and valid[1, 2] == 0
    assert valid.sum() == rows * cols - 3
    y, x = 3, 4
    a = amp[1 + y, 2 + x]
    want = np.sort(np.sqrt(re[:, y, x] * re[:, y, x] + im[:, y, x] * im[:, y, x]))
    assert np.array_equal(a, want) and np.all(np.diff(a) >= 0)
    assert np.array_equal(slc[1 + y, 2 + x, :, 0], re[:, y, x])
    # invalid pixels carry no samples
    assert not slc[1 + 2, 2 + 3].any() and not amp[1 + 2, 2 + 3].any()


def test_read_strip_phase_rotation():
    re = np.array([[[3.0]], [[0.0]]], np.float32)
    im = np.array([[[4.0]], [[2.0]]], np.float32)
    ph = np.array([[[0.5]], [[-1.0]]])
    slc, amp, valid = tcoh_b200.read_strip(re, im, 0, 1, 0, phase=ph)
    z = (re + 1j * im)[:, 0, 0].astype(np.complex128) * np.exp(1j * ph[:, 0, 0])
    assert np.allclose(slc[0, 0, :, 0], z.real.astype(np.float32))
    assert np.allclose(slc[0, 0, :, 1], z.imag.astype(np.float32))
    assert np.array_equal(amp[0, 0], np.float32([2.0, 5.0]))


def test_strip_rows_memory_budget():
    # test_strips of the reference: memory=1 with 8 dates x 400 columns
    # forces strips of fewer than 30 rows.
    r = tcoh_b200.strip_rows_for(30, 400, 8, 7, 5, 0, 1, 1 << 40)
    assert 1 <= r < 30
    with pytest.raises(MemoryError):
        tcoh_b200.strip_rows_for(30, 4000000, 30, 21, 7, 0, 1, 1 << 40)
    assert tcoh_b200.strip_rows_for(30, 24, 6, 21, 7, 0, 300, 1 << 40) == 30


def test_open_without_gpu_reports_device_error():
    if tcoh_b200.device_count() > 0:
        pytest.skip("a GPU is present")
    s = tcoh_b200.make_settings(6, min_shp=6)
    with pytest.raises(tcoh_b200.BackendError, match="CUDA device"):
        tcoh_b200.Backend(s, 30)


def test_ocl_open_is_fatal_like_the_module():
    """ocl_* report errors as G_fatal_error does: message and exit status."""
    code = (
        "import sys; sys.path.insert(0, %r); import tcoh_b200 as t; "
        "s = t.make_settings(6, min_shp=6); t.ocl_open(1, 0, s, 30); print('returned')" % ROOT
    )
    p = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=120)
    assert p.returncode != 0
    assert "platform 1 not found" in p.stderr
    assert "returned" not in p.stdout


def test_settings_struct_layout():
    """struct settings as local_proto.h:34-49 lays it out (x86-64)."""
    S = tcoh_b200.Settings
    assert S.alpha.offset == 16 and S.ks_max.offset == 36 and S.ad_norm.offset == 40
    assert S.npairs.offset == 72 and S.phase_reference.offset == 80 and ctypes.sizeof(S) == 96


def test_synthetic_stack_is_deterministic():
    import tcoh_b200.synthetic as syn

    a = syn.generate(10, 32, 24, seed=3)
    b = syn.generate(10, 32, 24, seed=3)
    assert np.array_equal(a, b, equal_nan=True)
    assert a.dtype == np.complex64
    bad = np.isnan(a).any(axis=0) | (a == 0).any(axis=0)
    assert 0 < bad.sum() <= 8
    assert np.all(np.isnan(a) | (a.real == np.round(a.real)))


def test_adjoint_output_buffers_are_checked_before_the_call():
    """adjoint_raw's caller-supplied outputs must have the gradient shapes
    and types; a mismatch is reported before anything reaches the device."""
    n, prow, cols, rows = 4, 12, 8, 2
    re = np.zeros((n, prow, cols), np.float32)

    class NoDevice:
        handle = None

    bad = {"grad_psi": np.zeros((n, prow, cols + 1), np.float32)}
    with pytest.raises(ValueError, match="grad_psi"):
        tcoh_b200.Backend.adjoint_raw(NoDevice(), re, re, None, None, None, -5, rows, rows,
                                      cols, out=bad)
    bad = {"grad_dh": np.zeros((prow, cols), np.float64)}
    with pytest.raises(ValueError, match="grad_dh"):
        tcoh_b200.Backend.adjoint_raw(NoDevice(), re, re, None, None, None, -5, rows, rows,
                                      cols, out=bad)
