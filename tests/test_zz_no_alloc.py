"""The allocation-free entry point tc_run_device_static (B200 only).

Some hosts of this library cannot allocate device memory while they run:
they manage every device buffer themselves (a fixed pool, a strict budget
on a shared GPU) or call from code where cudaMalloc is not allowed.
tc_run_device_static serves them: the caller passes the strip and the
outputs, and the path's intermediate buffers live in one static device
array of the library. These tests call it through the C-ABI and check its
outputs against the context-based entry point (tc_open + tc_run_ex with the
same FP32 coherence matrices), on consecutive calls that share, and so
reuse, that static scratch.

This file is collected last on purpose (pytest orders files by name).
"""

import numpy as np
import pytest

import tcoh_b200
import tcoh_b200.synthetic as syn
from conftest import TOLERANCE

pytestmark = pytest.mark.gpu

CASES = [
    dict(n=12, rows=40, cols=33, seed=1, shp_test="ad", estimator="emi", bias=True,
         window=(21, 7), pairs=True, pairs_all=True),
    dict(n=30, rows=50, cols=45, seed=2, shp_test="ks", estimator="evd", bias=False,
         window=(21, 7), pairs=True, pairs_all=False),
    dict(n=10, rows=35, cols=70, seed=3, shp_test="tlog", estimator="evd", bias=False,
         window=(9, 5), pairs=False, pairs_all=False),
    # Several sub-strips: the coherence sums of the whole strip alone take
    # 8 B x 465 entries x (7 x 38 tiles of 128 pixels) = 127 MB, twice the
    # 64 MiB array (which also holds 36 MB of EMI scratch), so the strip is
    # cut into at least three sub-strips, the last one of 100 mod 16 = 4
    # rows; the pair planes go through the strided copy into the caller's
    # [npairs][rows][cols].
    dict(n=30, rows=100, cols=300, seed=4, shp_test="ks", estimator="emi", bias=True,
         window=(21, 7), pairs=True, pairs_all=False),
]


def prepare(case):
    n, rows, cols = case["n"], case["rows"], case["cols"]
    stack = syn.generate(n, rows, cols, seed=case["seed"], nregions=3)
    ha, hr = case["window"][0] // 2, case["window"][1] // 2
    slc, amp, valid = tcoh_b200.read_strip(stack.real, stack.imag, -ha, rows + 2 * ha, hr)
    s = tcoh_b200.make_settings(n, window=case["window"], shp_test=case["shp_test"],
                                min_shp=n, estimator=case["estimator"], bias=case["bias"],
                                pairs=case["pairs"], pairs_all=case["pairs_all"])
    return s, slc, amp, valid


def run_static(torch, s, slc, amp, valid, rows, cols):
    dev = torch.device("cuda:0")
    n = s.ndates
    d_slc, d_amp, d_valid = (torch.from_numpy(a).to(dev) for a in (slc, amp, valid))
    coh = torch.full((rows, cols), 7.0, dtype=torch.float32, device=dev)
    count = torch.full((rows, cols), 7, dtype=torch.int32, device=dev)
    pairs = (torch.full((s.npairs, rows, cols), 7.0, dtype=torch.float32, device=dev)
             if s.npairs else None)
    phases = torch.full((rows, cols, n), 7.0, dtype=torch.float32, device=dev)
    status = torch.full((rows, cols), 7, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)
    tcoh_b200.run_device_static(s, slc.shape[1], d_slc, d_amp, d_valid, rows, cols, coh, count,
                                pairs, phases, status, stream=stream)
    torch.cuda.synchronize()
    out = {"coh": coh.cpu().numpy(), "count": count.cpu().numpy(),
           "phases": phases.cpu().numpy(), "status": status.cpu().numpy()}
    if pairs is not None:
        out["pairs"] = pairs.cpu().numpy()
    return out


def close(got, want, tol):
    assert np.array_equal(np.isnan(got), np.isnan(want))
    m = ~np.isnan(want)
    if m.any():
        assert np.abs(got[m].astype(np.float64) - want[m]).max() <= tol


def test_static_entry_point_matches_tc_run_ex_on_consecutive_calls():
    torch = pytest.importorskip("torch")
    # Each case after the first reuses the scratch the previous one left;
    # the first case comes back last.
    for case in CASES + [CASES[0]]:
        s, slc, amp, valid = prepare(case)
        rows, cols = case["rows"], case["cols"]
        with tcoh_b200.Backend(s, slc.shape[1], gram="fp32") as be:
            want = be.run(slc, amp, valid, rows, cols, phases=True, status=True)
        got = run_static(torch, s, slc, amp, valid, rows, cols)
        assert np.array_equal(got["count"], want["count"])
        close(got["coh"], want["coh"], TOLERANCE)
        assert np.array_equal(got["status"], want["status"])
        d = np.angle(np.exp(1j * (got["phases"].astype(np.float64) - want["phases"])))
        close(np.where(np.isnan(got["phases"]), np.nan, d),
              np.where(np.isnan(want["phases"]), np.nan, 0.0), TOLERANCE)
        if s.npairs:
            close(got["pairs"], want["pairs"], TOLERANCE)


def test_static_entry_point_rejects_strips_beyond_its_scratch():
    torch = pytest.importorskip("torch")
    s = tcoh_b200.make_settings(64, window=(21, 7), min_shp=64)
    cols = 20000
    tiny = torch.zeros(1, device="cuda:0")
    with pytest.raises(tcoh_b200.BackendError, match="MiB of scratch"):
        tcoh_b200.library()
        tcoh_b200._check(tcoh_b200.library().tc_run_device_static(
            tcoh_b200.ctypes.byref(s), cols + 6, tcoh_b200._ptr(tiny), tcoh_b200._ptr(tiny),
            tcoh_b200._ptr(tiny), 21, 1, cols, tcoh_b200._ptr(tiny), tcoh_b200._ptr(tiny),
            None, None, None, None))
