"""Failure paths of the backend, made on the host (no GPU fault).

The reference reports every OpenCL failure through G_fatal_error, which ends
the module (ocl.c:44-48); the drop-in ocl_* entry points keep that
convention through the handler set by tc_set_fatal_handler, and the tc_*
extensions return a code instead. Failures are injected on the host: an
argument the backend refuses, and TCOH_FAIL_AT_CHUNK=k, which makes a run
fail before launching its chunk k as a CUDA error would. The per-pixel
status bits report the non-fatal conditions: dates left unlinked by the
bias correction (NaN, as tcoh.cl:644-647), |T| inverted by its
pseudo-inverse, pixels recomputed in double precision.
"""

import os
import subprocess
import sys
import textwrap

import numpy as np
import pytest

import oracle
import tcoh_b200
import tcoh_b200.synthetic as syn
from conftest import ROOT, TOLERANCE, Case

HANDLER_SCRIPT = textwrap.dedent("""
    import ctypes, os, sys
    sys.path.insert(0, %(root)r)
    import numpy as np
    import tcoh_b200
    lib = tcoh_b200.library()
    HANDLER = ctypes.CFUNCTYPE(None, ctypes.c_char_p)

    def handler(msg):
        # a fatal handler must not return (G_fatal_error ends the module)
        print("HANDLER:" + msg.decode(), flush=True)
        os._exit(7)

    keep = HANDLER(handler)
    if %(custom)r:
        lib.tc_set_fatal_handler(keep)
    s = tcoh_b200.make_settings(6, window=(5, 3), min_shp=6)
    %(body)s
    print("RETURNED", flush=True)
""")


def run_script(body, custom=True, env=None):
    code = HANDLER_SCRIPT % dict(root=ROOT, custom=custom, body=textwrap.dedent(body).strip())
    e = dict(os.environ)
    e.update(env or {})
    return subprocess.run([sys.executable, "-c", code], capture_output=True, text=True,
                          timeout=300, env=e)


def test_ocl_open_failure_reaches_the_fatal_handler():
    """A platform the backend does not have: ocl_open calls the handler,
    which ends the process; ocl_open never returns."""
    p = run_script("""
        m = ctypes.c_size_t(0)
        lib.ocl_open(5, 0, ctypes.byref(s), 12, ctypes.byref(m))
    """)
    assert p.returncode == 7, p.stderr
    assert "HANDLER:CUDA backend: platform 5 not found" in p.stdout
    assert "RETURNED" not in p.stdout


def test_default_fatal_handler_reports_and_exits():
    """Without a handler and without GRASS, the message goes to stderr and
    the process exits with failure (as G_fatal_error would end it)."""
    p = run_script("""
        m = ctypes.c_size_t(0)
        lib.ocl_open(-1, 3, ctypes.byref(s), 12, ctypes.byref(m))
    """, custom=False)
    assert p.returncode == 1
    assert "ERROR: CUDA backend: Option device requires option platform" in p.stderr
    assert "RETURNED" not in p.stdout


def test_tc_open_returns_codes_instead():
    s = tcoh_b200.make_settings(6, window=(5, 3), min_shp=6)
    s.win_az = 4
    with pytest.raises(tcoh_b200.BackendError, match="Window sizes must be odd"):
        tcoh_b200.Backend(s, 12)


def small_strip(n=8, rows=40, cols=24, seed=3):
    stack = syn.generate(n, rows, cols, seed=seed, nregions=2)
    return tcoh_b200.read_strip(stack.real, stack.imag, -2, rows + 4, 1)


@pytest.mark.gpu
def test_injected_chunk_failure_returns_the_code(monkeypatch):
    n, rows, cols = 8, 40, 24
    slc, amp, valid = small_strip(n, rows, cols)
    s = tcoh_b200.make_settings(n, window=(5, 3), min_shp=n)
    monkeypatch.setenv("TCOH_FAIL_AT_CHUNK", "1")
    with tcoh_b200.Backend(s, cols + 2, chunk_pixels=128) as be:
        with pytest.raises(tcoh_b200.BackendError, match="injected failure before chunk 1"):
            be.run(slc, amp, valid, rows, cols)
    # the device stays usable: the same strip without the injection
    monkeypatch.delenv("TCOH_FAIL_AT_CHUNK")
    with tcoh_b200.Backend(s, cols + 2, chunk_pixels=128) as be:
        r = be.run(slc, amp, valid, rows, cols)
    o = oracle.run_oracle(slc, amp, valid, rows, cols, window=(5, 3), min_shp=n, shp_fp32=True)
    assert np.array_equal(r["count"], o["count"])
    m = ~np.isnan(o["coh"])
    assert np.abs(r["coh"][m] - o["coh"][m]).max() <= TOLERANCE


@pytest.mark.gpu
def test_injected_failure_in_ocl_run_calls_the_fatal_handler():
    p = run_script("""
        slc, amp, valid = [np.zeros(sh, dt) for sh, dt in (((14, 12, 6, 2), np.float32),
                                                          ((14, 12, 6), np.float32),
                                                          ((14, 12), np.uint8))]
        h, _ = tcoh_b200.ocl_open(-1, -1, s, 12)
        coh = np.empty((10, 10), np.float32)
        count = np.empty((10, 10), np.int32)
        tcoh_b200.ocl_run(h, slc, amp, valid, 14, 10, 10, coh, count, None)
    """, env={"TCOH_FAIL_AT_CHUNK": "0"})
    assert p.returncode == 7, p.stderr
    assert "HANDLER:CUDA backend: injected failure before chunk 0" in p.stdout
    assert "RETURNED" not in p.stdout


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["bias_evd", "bias_emi"])
def test_unlinked_dates_are_null_with_their_status(name):
    """Pixels whose bias-corrected coherences leave a date unlinked are NULL
    (tcoh.cl:644-647) and carry TC_STATUS_UNLINKED; no other pixel does."""
    c = Case(name)
    kw = c.kwargs()
    s = tcoh_b200.make_settings(c.n, **kw)
    with tcoh_b200.Backend(s, c.cols + kw["window"][1] - 1) as be:
        r = be.run(*c.strip(), c.rows, c.cols, status=True)
    looks_ok = r["count"] >= max(kw["min_shp"], c.n)
    unlinked = looks_ok & np.isnan(c.coh)
    assert unlinked.any(), "the golden case has unlinked pixels"
    assert np.array_equal((r["status"] & tcoh_b200.STATUS_UNLINKED) != 0, unlinked)
    assert np.isnan(r["coh"][unlinked]).all()


@pytest.mark.gpu
def test_singular_coherence_magnitudes_take_the_pseudo_inverse():
    """Two identical dates make |T| singular: EMI inverts it by its
    eigen-pseudo-inverse (TC_STATUS_EMI_PINV), with the oracle's floor
    (tests/reference.py:151-156), and agrees with the oracle."""
    n, rows, cols = 10, 24, 20
    stack = syn.generate(n, rows, cols, seed=11, nregions=2, g0_max=0.9, null_frac=0.0)
    stack[1] = stack[0]
    kw = dict(window=(9, 5), shp_test="ks", min_shp=n, estimator="emi")
    slc, amp, valid = tcoh_b200.read_strip(stack.real, stack.imag, -4, rows + 8, 2)
    s = tcoh_b200.make_settings(n, **kw)
    with tcoh_b200.Backend(s, cols + 4) as be:
        r = be.run(slc, amp, valid, rows, cols, status=True)
    o = oracle.run_oracle(slc, amp, valid, rows, cols, shp_fp32=True, **kw)
    assert np.array_equal(r["count"], o["count"])
    m = ~np.isnan(o["coh"])
    assert m.any()
    assert ((r["status"][m] & tcoh_b200.STATUS_EMI_PINV) != 0).mean() > 0.9
    assert np.abs(r["coh"][m] - o["coh"][m]).max() <= TOLERANCE
