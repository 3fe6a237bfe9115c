#!/usr/bin/env python
"""Throughput of the phase-linking temporal coherence path on B200.

Metric: Mpixel/s of temporal coherence at N = 30 dates, 21 x 7 window,
within 1e-4 of the FP64 oracle. Workload (one step = one pass of the path
over one strip): a 4096 x 4096 stack of 30 complex64 dates, 32 Voronoi
regions with coherence up to 0.99, shp_test=ad, estimator=emi, -b (the
precision-form configuration of the reference's published settings),
seeded synthetic data.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

* value: device-resident strips, K steps timed with CUDA events on the
  launching stream (inputs of 6 GB, far above the 126 MB L2: no flush);
* e2e: the same metric through the C-ABI with host buffers (tc_run_ex, the
  ocl_run path): page-locked strip in, outputs out, copies inside the
  timed region;
* roofline of the dominant kernel from per-launch CUDA events;
* cpu_baseline: the reference kernel (tcoh.cl compiled as C, oracle/_ref)
  on all host cores over a crop of the same workload;
* accuracy: max / RMS |coh - oracle| on a crop (FP64 oracle, float SHP
  decisions), and the SHP decision flips of the float tests against the
  FP64 ones.

With N > 1 (torchrun), every rank processes its own full workload (weak
scaling, no collective on the data path); time is the max over ranks.
"""

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = dict(n=30, rows=4096, cols=4096, window=(21, 7), shp_test="ad", alpha=0.05,
                min_shp=20, estimator="emi", bias=True, nregions=32, g0_max=0.99, spacing=12.0)
# The other configurations of the path, as bench lines of their own (not the
# metric's): N=10 KS/EVD on 512 x 512 here; the scenes of N=30 with geometry
# and all pair coherences (4096 x 8192) and of N=60 with six-day dates
# (8192 x 16384) in SCENES below, processed in strips.
WORKLOADS = {
    "emi": WORKLOAD,
    "ks10": dict(n=10, rows=512, cols=512, window=(21, 7), shp_test="ks", alpha=0.05,
                 min_shp=10, estimator="evd", bias=False, nregions=8, g0_max=0.95, spacing=12.0),
}
METRIC = "Mpixel/s temporal coherence at N=30, 21x7 window, <=1e-4 vs FP64"


def metric_name(w):
    if w is WORKLOAD:
        return METRIC
    return "Mpixel/s temporal coherence at N=%d, %dx%d window, <=1e-4 vs FP64" % (
        w["n"], w["window"][0], w["window"][1])
# DRAM bytes (read + write) per pixel of one phase-linking launch: a
# constant, from the ncu capture of profiles/
# tc_link_half_kernel_emi_bias_n30_256x4096.md (dram__bytes_read.sum +
# dram__bytes_write.sum of one 65,536-pixel chunk at N=30, AD / EMI / bias
# correction: 245.2 MB read, the packed Gram, 465 x 8 B per pixel, read at
# most once, + 7.3 MB written), not a measurement of the run that reports it.
LINK_DRAM_BYTES_PER_PIXEL = 252.5e6 / 65536


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--rows", type=int, default=None, help="output rows (default: the workload's)")
    p.add_argument("--cols", type=int, default=None, help="output columns (default: the workload's)")
    p.add_argument("--gram", default="tensor", choices=["tensor", "fp32"],
                   help="arithmetic of the coherence matrices (the tensor cores, else plain FP32)")
    p.add_argument("--workload", default="emi",
                   choices=["emi", "adjoint", "geometry-pairs", "n60", "n60emi"] +
                   [k for k in WORKLOADS if k != "emi"],
                   help="emi: the metric's configuration (default); adjoint: forward + "
                        "adjoint with geometry, a height error and a phase screen, and 20 "
                        "steps of gradient ascent on the height error (2048 x 2048 unless "
                        "--rows / --cols); geometry-pairs: N=30 tlog with all pair "
                        "coherences and the phase removed on the device from orbits and an "
                        "elevation map, 4096 x 8192 in strips of 512 rows; n60, n60emi: N=60 "
                        "KS with EVD or EMI, 8192 x 16384 in strips of 1024 rows; ks10: "
                        "N=10 KS/EVD on 512 x 512")
    p.add_argument("--strip-rows", type=int, default=None,
                   help="output rows per strip of the scene workloads")
    p.add_argument("--accuracy-size", type=int, default=256,
                   help="side of the centred crop checked against the FP64 oracle")
    p.add_argument("--no-extras", action="store_true",
                   help="skip the e2e, plain-FP32, CPU and accuracy legs")
    return p.parse_args()


def workload_name(rows, cols, w=WORKLOAD):
    return "N=%d %dx%d %s/%s%s window %dx%d, %d regions, coherence <= %.2f" % (
        w["n"], rows, cols, w["shp_test"], w["estimator"], "/-b" if w["bias"] else "",
        w["window"][0], w["window"][1], w["nregions"], w["g0_max"])


# ---------------------------------------------------------------------------
# Inputs.

def device_strip(torch, stack, ha, hr):
    """Padded strip buffers (main.c:52-127 layout) built on the device."""
    n, rows, cols = stack.shape
    re, im = stack.real.contiguous(), stack.imag.contiguous()
    bad = torch.isnan(re) | torch.isnan(im) | ((re == 0) & (im == 0))
    valid = ~bad.any(dim=0)
    re = torch.where(valid[None], re, torch.zeros_like(re))
    im = torch.where(valid[None], im, torch.zeros_like(im))
    amp = torch.sqrt(re * re + im * im)
    amp, _ = torch.sort(amp, dim=0)
    P, Q = rows + 2 * ha, cols + 2 * hr
    dev = stack.device
    slc = torch.zeros((P, Q, n, 2), dtype=torch.float32, device=dev)
    slc[ha:ha + rows, hr:hr + cols, :, 0] = re.permute(1, 2, 0)
    slc[ha:ha + rows, hr:hr + cols, :, 1] = im.permute(1, 2, 0)
    del re, im
    a = torch.zeros((P, Q, n), dtype=torch.float32, device=dev)
    a[ha:ha + rows, hr:hr + cols] = amp.permute(1, 2, 0)
    del amp
    v = torch.zeros((P, Q), dtype=torch.uint8, device=dev)
    v[ha:ha + rows, hr:hr + cols] = valid.to(torch.uint8)
    return slc, a, v


# ---------------------------------------------------------------------------
# Clocks during the timed region.

class Clocks:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.out = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.out, stderr=subprocess.DEVNULL)
        except (OSError, ValueError):
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=10)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.out.close()
        rows = [r.split(", ") for r in open(self.path).read().strip().splitlines() if r.strip()]
        os.unlink(self.path)
        if not rows:
            return None
        import statistics

        sm = [float(r[1]) for r in rows if len(r) > 1 and r[1].strip().replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if len(r) > 2 and r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in rows:
            for k, name in enumerate(names):
                if len(r) > 5 + k and r[5 + k].strip() == "Active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(rows)}


# ---------------------------------------------------------------------------
# Algorithmic work per pixel (fixed by formula; extra work of an
# implementation does not count).

def flops_per_pixel(n, looks, emi):
    gram = 8.0 * looks * n * (n + 1) / 2
    norm_gamma = 10.0 * n * (n - 1) / 2 + 20.0 * n * (n - 1) / 2
    evd = 16.0 * n ** 3 / 3 + 8.0 * n ** 2 + 64 * 5 * n
    link = norm_gamma + evd + ((n ** 3 + 2.0 * n ** 2) if emi else 0.0)
    return gram, link


def shp_ops_per_pixel(n, test, area):
    if test == "ks":
        return area * 2.0 * n
    if test == "ad":
        return area * (2.0 * n - 1) * 7
    return area * 6.0 + n


# ---------------------------------------------------------------------------
# CPU legs.

def cpu_crop(slc, amp, valid, rows, cols, r0, nrows, ncols, ha, hr):
    """Sub-strip for output rows r0 .. r0+nrows-1, columns 0 .. ncols-1."""
    import numpy as np

    sl = slice(r0, r0 + nrows + 2 * ha)
    cs = slice(0, ncols + 2 * hr)
    return (np.ascontiguousarray(slc[sl, cs]), np.ascontiguousarray(amp[sl, cs]),
            np.ascontiguousarray(valid[sl, cs]))


def reference_rate(slc, amp, valid, rows, cols, kw, target_s=10.0, threads=0, ccols=512,
                   npairs=0, max_rows=None):
    """Mpixel/s of the reference kernel (tcoh.cl as C) on the host cores,
    on a crop of ccols columns of the strip, its rows sized for about
    target_s seconds (at most max_rows, by default half the strip)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    ha, hr = kw["window"][0] // 2, kw["window"][1] // 2
    kind = "reference" if oracle.reference_available() else "port"
    run = oracle.run_reference if kind == "reference" else oracle.run_oracle
    extra = dict(npairs=npairs, pairs_all=True) if npairs else {}
    ccols = min(cols, ccols)
    max_rows = max_rows or rows // 2
    # calibration on 4 rows
    crop = cpu_crop(slc, amp, valid, rows, cols, rows // 2 if rows >= 8 else 0, 4, ccols, ha, hr)
    t = time.perf_counter()
    run(*crop, 4, ccols, threads=threads, **extra, **kw)
    rate = 4 * ccols / max(time.perf_counter() - t, 1e-6)
    nrows = int(max(4, min(max_rows, rate * target_s / ccols)))
    r0 = min(rows // 4, rows - nrows)
    crop = cpu_crop(slc, amp, valid, rows, cols, r0, nrows, ccols, ha, hr)
    t = time.perf_counter()
    run(*crop, nrows, ccols, threads=threads, **extra, **kw)
    dt = time.perf_counter() - t
    cores = oracle.reference_threads() if kind == "reference" else (threads or os.cpu_count())
    out = {"value": nrows * ccols / dt / 1e6, "unit": "Mpixel/s", "cores": cores, "kind": kind,
           "sample": "%d x %d output pixels of the workload (rows %d.., %.1f s)" % (
               nrows, ccols, r0, dt)}
    if kind == "reference":
        # "specialised": tcoh.cl built with this configuration's -D constants,
        # as the reference's OpenCL backend builds it (ocl.c:222-229)
        out["build"] = oracle.ref_build(amp.shape[2], kw["window"], ccols + 2 * hr,
                                        kw["shp_test"], kw["alpha"], kw["estimator"],
                                        kw["bias"], kw["min_shp"], npairs, bool(npairs))
    return out


def accuracy(slc, amp, valid, coh_gpu, count_gpu, rows, cols, kw, size=256, flips_size=64):
    """crop_accuracy on a centred size x size crop of a strip."""
    size = min(size, rows, cols)
    ha, hr = kw["window"][0] // 2, kw["window"][1] // 2
    r0, c0 = (rows - size) // 2, (cols - size) // 2
    crop = cpu_crop(slc[:, c0:], amp[:, c0:], valid[:, c0:], rows, cols, r0, size, size, ha, hr)
    return crop_accuracy(crop, coh_gpu[r0:r0 + size, c0:c0 + size],
                         count_gpu[r0:r0 + size, c0:c0 + size], size, amp.shape[2], kw,
                         flips_size)


def crop_accuracy(crop, coh_gpu, count_gpu, size, n, kw, flips_size=64):
    """|coh - FP64 oracle| on a size x size padded crop (slc, amp, valid),
    the oracle with the float SHP decisions, so that both use the same
    masks: the timed run's coherence (coh_gpu, count_gpu over the crop),
    and all pair coherences, per-date phases and status bits of a run on
    the crop; plus the SHP decision flips of the float statistics against
    the FP64 ones on a flips_size x flips_size part of it."""
    import numpy as np

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    import tcoh_b200

    ha, hr = kw["window"][0] // 2, kw["window"][1] // 2
    s = tcoh_b200.make_settings(n, pairs=True, pairs_all=True, **kw)
    with tcoh_b200.Backend(s, size + 2 * hr) as be:
        r = be.run(*crop, size, size, phases=True, status=True)
    t = time.perf_counter()
    o = oracle.run_oracle(*crop, size, size, shp_fp32=True, npairs=s.npairs, pairs_all=True,
                          want_phases=True, **kw)
    t_oracle = time.perf_counter() - t
    g = coh_gpu.astype(np.float64)
    m = ~np.isnan(o["coh"]) & ~np.isnan(g)
    err = np.abs(g[m] - o["coh"][m])
    out = {
        "pixels": int(size * size), "estimated": int(m.sum()),
        "max_abs": float(err.max()) if err.size else None,
        "rms": float(np.sqrt(np.mean(err ** 2))) if err.size else None,
        "over_1e-4": int((err > 1e-4).sum()),
        "count_mismatch": int((count_gpu != o["count"]).sum()),
        "null_mask_mismatch": int((np.isnan(g) != np.isnan(o["coh"])).sum()),
        "crop_run_equals_timed_run": bool(np.array_equal(r["coh"], coh_gpu, equal_nan=True)),
        "fp64_tier_fraction": float(((r["status"][m] & tcoh_b200.STATUS_FP64) != 0).mean())
        if m.any() else None,
        "emi_pivoted_fraction": float(((r["status"][m] & tcoh_b200.STATUS_EMI_PIVOTED) != 0)
                                      .mean()) if m.any() else None,
        "emi_pinv_fraction": float(((r["status"][m] & tcoh_b200.STATUS_EMI_PINV) != 0).mean())
        if m.any() else None,
        "oracle_seconds": t_oracle,
    }
    pm = ~np.isnan(o["pairs"]) & ~np.isnan(r["pairs"])
    perr = np.abs(r["pairs"][pm].astype(np.float64) - o["pairs"][pm])
    ph = ~np.isnan(o["phases"]) & ~np.isnan(r["phases"])
    d = np.angle(np.exp(1j * (r["phases"][ph].astype(np.float64) - o["phases"][ph])))
    out["pairs"] = {"planes": int(s.npairs), "max_abs": float(perr.max()) if perr.size else None,
                    "rms": float(np.sqrt(np.mean(perr ** 2))) if perr.size else None,
                    "null_mask_mismatch": int((np.isnan(o["pairs"]) != np.isnan(r["pairs"])).sum())}
    out["phases_rad"] = {"max_abs": float(np.abs(d).max()) if d.size else None,
                         "rms": float(np.sqrt(np.mean(d ** 2))) if d.size else None,
                         "p999": float(np.quantile(np.abs(d), 0.999)) if d.size else None}
    if d.size:
        dd = np.zeros(o["phases"].shape)
        dd[ph] = np.abs(d)
        # the phases of coherent pixels (gamma >= 0.2; on incoherent ones the
        # eigenproblem is nearly degenerate and the phases ill-determined)
        coherent = np.nan_to_num(o["coh"]) >= 0.2
        out["phases_rad"]["max_abs_coherence_ge_0.2"] = float(dd[coherent].max()) \
            if coherent.any() else None
        worst = np.argsort(dd.ravel())[::-1][:5]
        out["phases_rad"]["worst"] = [
            {"row": int(i // (size * n)), "col": int(i // n % size), "date": int(i % n),
             "err": float(dd.ravel()[i]), "status": int(r["status"].ravel()[i // n]),
             "coh": float(g.ravel()[i // n])} for i in worst]
    fs = min(flips_size, size)
    fc = cpu_crop(*crop, size, size, 0, fs, fs, ha, hr)
    o64 = oracle.run_oracle(*fc, fs, fs, shp_fp32=False, **kw)
    out["shp_count_flips_float_vs_fp64"] = {
        "pixels": fs * fs, "flips": int((o["count"][:fs, :fs] != o64["count"]).sum())}
    # the pixels beyond the tolerance, for the record
    bad = np.argwhere(m & (np.abs(np.nan_to_num(g - o["coh"])) > 1e-4))
    out["over_1e-4_pixels"] = [
        {"row": int(y), "col": int(x), "err": float(abs(g[y, x] - o["coh"][y, x])),
         "gpu": float(g[y, x]), "oracle": float(o["coh"][y, x]), "status": int(r["status"][y, x]),
         "looks": int(count_gpu[y, x])} for y, x in bad[:12]]
    if os.environ.get("TCOH_BENCH_DUMP") and len(bad):
        np.savez_compressed(os.environ["TCOH_BENCH_DUMP"], slc=crop[0], amp=crop[1],
                            valid=crop[2], coh_gpu=g, coh_oracle=o["coh"], status=r["status"],
                            bad=bad, kw=json.dumps(kw))
    return out


# ---------------------------------------------------------------------------

def adjoint_workload(args):
    """Forward + adjoint throughput and a height-error ascent.

    N=30, 2048 x 2048 (unless --rows / --cols), synthetic distributed
    scatterers (32 regions, coherence <= 0.99), synthetic orbits and a
    fractal height field (0 - 2000 m); the simulated samples carry the
    geometric phase at the true heights h + dh_true (dh_true: N(0, 15 m)
    smoothed over 9 x 9 and rescaled to 15 m RMS) and a per-date fractal
    phase screen (0 - 2 rad). The module removes the phase at h + dh and the
    screen psi; starting from dh = psi = 0, each step is one forward +
    adjoint (tc_adjoint_raw, host buffers) and an Adam step. The variable is
    u with dh = S u, S the 9 x 9 box average (its gradient S dL/d(dh)):
    gamma only sees height differences inside a window, and a free per-pixel
    dh fits the speckle instead of the height error (plain Adam on dh raises
    gamma further while the height error grows). Reported: Mpixel/s of
    forward + adjoint, mean gamma and the RMS of dh - dh_true (mean removed:
    gamma does not see a height offset common to a window) before and after
    the ascent, and mean gamma at dh = dh_true."""
    import numpy as np
    import torch

    import tcoh_b200
    import tcoh_b200.scene as scene
    import tcoh_b200.synthetic as syn

    n = 30
    rows = args.rows or 2048
    cols = args.cols or 2048
    ha, hr = 10, 3
    geo, orbits = scene.acquisition(n, rows, cols, seed=11)
    h = scene.fbm_heights(rows, cols, hurst=0.8, hmax=2000.0, seed=12)
    rng = np.random.default_rng(13)
    dh_true = scene.smooth(rng.normal(0.0, 15.0, (rows, cols)), 9)
    dh_true *= 15.0 / dh_true.std()
    screen = np.stack([scene.fbm_heights(rows, cols, hurst=0.8, hmax=2.0, seed=100 + k)
                       for k in range(n)])
    g = tcoh_b200.make_geometry(heights=h, h0=0.0, **geo)
    grid = tcoh_b200.geometry_grid(g, orbits)
    levels = ([g.hmin, 0.5 * (g.hmin + g.hmax), g.hmax] if grid.shape[2] == 3
              else [0.5 * (g.hmin + g.hmax)])
    phase = scene.grid_phases(grid, levels, h + dh_true) + screen
    stack = syn.generate(n, rows, cols, nregions=32, g0_max=0.99, seed=14, null_frac=0.0)
    stack = (stack * np.exp(-1j * phase)).astype(np.complex64)
    del phase
    prow = rows + 2 * ha

    def pinned(shape, dtype):
        return torch.empty(shape, dtype=dtype, pin_memory=True).numpy()

    # the samples and the gradients live in page-locked host memory
    re = pinned((n, prow, cols), torch.float32)
    im = pinned((n, prow, cols), torch.float32)
    re[:] = np.nan
    im[:] = np.nan
    re[:, ha:ha + rows] = stack.real
    im[:, ha:ha + rows] = stack.imag
    del stack
    out = {"coh": pinned((rows, cols), torch.float32), "count": pinned((rows, cols), torch.int32),
           "grad_dh": pinned((prow, cols), torch.float32),
           "grad_psi": pinned((n, prow, cols), torch.float32)}
    elev = np.zeros((prow, cols))
    elev[ha:ha + rows] = h
    s = tcoh_b200.make_settings(n, window=(21, 7), shp_test="tlog", alpha=0.05, min_shp=20,
                                estimator="evd")
    be = tcoh_b200.Backend(s, cols + 2 * hr)
    be.set_geometry(g, grid)
    u = np.zeros((prow, cols))
    dh = u
    m_t, v_t = np.zeros_like(u), np.zeros_like(u)
    lr, b1, b2, box = 2.0, 0.9, 0.999, 9
    inner = (slice(ha, ha + rows), slice(None))

    def err(d):
        e = d[inner] - dh_true
        return float(np.sqrt(np.mean((e - e.mean()) ** 2)))

    r = be.adjoint_raw(re, im, elev, dh, None, -ha, rows, rows, cols, out=out)  # warm-up
    first = {"mean_gamma": float(np.nanmean(r["coh"])), "dh_rms_error_m": err(dh)}
    r = be.adjoint_raw(re, im, elev, np.pad(dh_true, ((ha, ha), (0, 0))), None, -ha, rows, rows,
                       cols, out=out)
    truth = float(np.nanmean(r["coh"]))
    times = []
    steps = 20
    for it in range(1, steps + 1):
        t = time.perf_counter()
        r = be.adjoint_raw(re, im, elev, dh, None, -ha, rows, rows, cols, out=out)
        times.append(time.perf_counter() - t)
        gu = scene.smooth(r["grad_dh"].astype(np.float64), box)
        m_t = b1 * m_t + (1 - b1) * gu
        v_t = b2 * v_t + (1 - b2) * gu * gu
        mh, vh = m_t / (1 - b1 ** it), v_t / (1 - b2 ** it)
        u = u + lr * mh / (np.sqrt(vh) + 1e-12)
        dh = scene.smooth(u, box)
    be.set_timing(True)
    r = be.adjoint_raw(re, im, elev, dh, None, -ha, rows, rows, cols, out=out)
    stages = {k: {"ms": v[0], "launches": v[1]} for k, v in be.stage_stats().items()}
    be.close()
    ms = 1e3 * float(np.median(times))
    line = {"metric": "Mpixel/s forward + adjoint of temporal coherence, N=30, 21x7 window",
            "value": rows * cols / (ms * 1e-3) / 1e6, "unit": "Mpixel/s", "n_gpus": 1,
            "steps": steps, "warmup": 1, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "N=30 %dx%d tlog/evd window 21x7, geometry with fBm heights "
                                   "0-2000 m, dh_true 15 m RMS, phase screen 0-2 rad" % (rows, cols),
                       "api": "tc_adjoint_raw (page-locked host buffers, strip preparation on the device)"},
            "stages": stages,
            "ascent": {"optimizer": "Adam on u, dh = %dx%d box average of u, lr %.1f m"
                                    % (box, box, lr), "steps": steps,
                       "mean_gamma_at_dh_true": truth, "before": first,
                       "after": {"mean_gamma": float(np.nanmean(r["coh"])),
                                 "dh_rms_error_m": err(dh)}}}
    print(json.dumps(line))


# ---------------------------------------------------------------------------
# Configurations 2 and 4 at their stated sizes: scenes in strips.

SCENES = {
    # N=30 tlog / EVD, all 435 pair coherences, the geometric phase removed
    # on the device from synthetic orbits and a fractal elevation map
    "geometry-pairs": dict(n=30, rows=4096, cols=8192, window=(21, 7), shp_test="tlog",
                           alpha=0.05, min_shp=20, estimator="evd", bias=False, nregions=32,
                           g0_max=0.99, spacing=12.0, pairs=True, geometry=True, strip_rows=512),
    # N=60 six-day dates, KS, EVD and EMI
    "n60": dict(n=60, rows=8192, cols=16384, window=(21, 7), shp_test="ks", alpha=0.05,
                min_shp=20, estimator="evd", bias=False, nregions=32, g0_max=0.99, spacing=6.0,
                pairs=False, geometry=False, strip_rows=1024),
    "n60emi": dict(n=60, rows=8192, cols=16384, window=(21, 7), shp_test="ks", alpha=0.05,
                   min_shp=20, estimator="emi", bias=False, nregions=32, g0_max=0.99,
                   spacing=6.0, pairs=False, geometry=False, strip_rows=1024),
}


def scene_workload(args, name):
    """A scene at its stated size, processed as main.c:724-825 does: strips
    of output rows, each read with WA/2 halo rows above and below (NULL
    outside the region), raw I/Q planes in, the strip preparation (validity,
    sorted amplitudes and, with geometry, the phase removal) on the device.

    * value: device-resident raw planes, tc_run_raw_device per strip timed
      with CUDA events (the synthetic generation of each strip, the scene's
      raster reading, is outside the timed region), summed over the strips;
    * e2e: page-locked host strip buffers reused from strip to strip,
      tc_run_raw per strip: raw rows copied in row blocks on a side stream
      while earlier chunks compute, outputs (with all the pair planes) back
      into reused host buffers as each chunk completes; wall clock.
    * accuracy on a centred 256 x 256 crop against the FP64 oracle, and the
      reference kernel on the host cores on a crop of 1024 columns."""
    import numpy as np
    import torch

    import tcoh_b200
    import tcoh_b200.scene as scene
    import tcoh_b200.synthetic as syn

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    w = SCENES[name]
    n, window = w["n"], w["window"]
    rows, cols = args.rows or w["rows"], args.cols or w["cols"]
    S = min(args.strip_rows or w["strip_rows"], rows)
    ha, hr = window[0] // 2, window[1] // 2
    kw = dict(window=window, shp_test=w["shp_test"], alpha=w["alpha"], min_shp=w["min_shp"],
              estimator=w["estimator"], bias=w["bias"])
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    g = grid = h = levels = None
    grid_ms = None
    if w["geometry"]:
        geo, orbits = scene.acquisition(n, rows, cols, seed=21)
        h = scene.fbm_heights(rows, cols, hurst=0.8, hmax=2000.0, seed=22)
        g = tcoh_b200.make_geometry(heights=h, h0=0.0, **geo)
        t = time.perf_counter()
        grid = tcoh_b200.geometry_grid(g, orbits)
        grid_ms = (time.perf_counter() - t) * 1e3
        levels = ([g.hmin, 0.5 * (g.hmin + g.hmax), g.hmax] if grid.shape[2] == 3
                  else [0.5 * (g.hmin + g.hmax)])
    s = tcoh_b200.make_settings(n, pairs=w["pairs"], pairs_all=True, **kw)
    be = tcoh_b200.Backend(s, cols + 2 * hr, device=0)
    if w["geometry"]:
        be.set_geometry(g, grid)
    strips = [(r0, min(rows, r0 + S)) for r0 in range(0, rows, S)]

    def region_rows(a, b):
        """Raw I/Q of region rows a .. b - 1 on the device (complex64), with
        the geometric phase the acquisition carries."""
        st = syn.generate(n, rows, cols, nregions=w["nregions"], g0_max=w["g0_max"],
                          spacing=w["spacing"], seed=31, device=dev, row_range=(a, b))
        if w["geometry"]:
            for q0 in range(a, b, 128):
                q1 = min(b, q0 + 128)
                phi = torch.from_numpy(scene.grid_phases(grid, levels, h[q0:q1], row0=q0)).to(dev)
                st[:, q0 - a:q1 - a] *= torch.exp(-1j * phi).to(torch.complex64)
        return st

    def strip_planes(r0, r1):
        """re, im (N, padded rows, cols) of the strip of output rows r0 .. r1
        - 1 on the device, NULL outside the region, and its elevation rows
        (host, None without geometry)."""
        prow = r1 - r0 + 2 * ha
        a, b = max(0, r0 - ha), min(rows, r1 + ha)
        st = region_rows(a, b)
        re = torch.full((n, prow, cols), float("nan"), dtype=torch.float32, device=dev)
        im = torch.full_like(re, float("nan"))
        o = a - (r0 - ha)
        re[:, o:o + b - a] = st.real
        im[:, o:o + b - a] = st.imag
        elev = None
        if w["geometry"]:
            elev = np.full((prow, cols), np.nan)
            elev[o:o + b - a] = h[a:b]
        return re, im, elev

    npairs = s.npairs
    coh = np.empty((rows, cols), np.float32)
    count = np.empty((rows, cols), np.int32)
    stream = torch.cuda.Stream(dev)
    d_coh = torch.empty((S, cols), dtype=torch.float32, device=dev)
    d_count = torch.empty((S, cols), dtype=torch.int32, device=dev)
    d_pairs = (torch.empty((npairs, S, cols), dtype=torch.float32, device=dev)
               if npairs else None)

    def strip_on_device(r0, r1):
        re, im, elev = strip_planes(r0, r1)
        el = torch.from_numpy(elev).to(dev) if elev is not None else None
        m = r1 - r0
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        be.run_raw_device(re, im, el, r0 - ha, rows, m, cols, d_coh[:m], d_count[:m],
                          pairs=d_pairs[:, :m] if npairs and m == S else
                          (torch.empty((npairs, m, cols), dtype=torch.float32, device=dev)
                           if npairs else None), stream=stream)
        e1.record(stream)
        e1.synchronize()
        coh[r0:r1] = d_coh[:m].cpu().numpy()
        count[r0:r1] = d_count[:m].cpu().numpy()
        return e0.elapsed_time(e1)

    # device-resident: one untimed strip, then the scene
    strip_on_device(*strips[len(strips) // 2])
    clocks = Clocks(0)
    clocks.start()
    ms_strips = [strip_on_device(r0, r1) for r0, r1 in strips]
    ck = clocks.stop()
    ms = float(sum(ms_strips))
    npix = rows * cols
    # per-stage device time on the middle strip
    be.set_timing(True)
    strip_on_device(*strips[len(strips) // 2])
    stages = be.stage_stats()
    be.set_timing(False)
    mid = strips[len(strips) // 2]
    cnt_mid = count[mid[0]:mid[1]]
    lbar = float(cnt_mid[cnt_mid >= 0].mean()) if (cnt_mid >= 0).any() else 0.0
    est = int((cnt_mid >= s.min_looks).sum())
    f_gram, f_link = flops_per_pixel(n, lbar, w["estimator"] == "emi")
    exact = w["estimator"] == "emi" and n > 32
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        pass
    fp32_peak = tcoh_b200.fp32_peak_tflops(0)
    fp64_peak = tcoh_b200.fp64_peak_tflops(0)
    bf16_peak = peaks.get("bf16_tflops_sustained", peaks.get("bf16_tflops", 1381.5))
    valid_mid = int((cnt_mid >= 0).sum())
    work = {
        "shp": (shp_ops_per_pixel(n, w["shp_test"], window[0] * window[1]) * valid_mid,
                "fp32", fp32_peak),
        "gram": (f_gram * valid_mid, "tensor", bf16_peak),
        # above 32 dates EMI runs the exact tier: FP64 sums and chain
        "link": ((f_link + f_gram) * est if exact else f_link * est,
                 "fp64" if exact else "fp32", fp64_peak if exact else fp32_peak),
    }
    kernels = {}
    for k, (flops, bound, peak) in work.items():
        t_ms, nl = stages[k]
        if t_ms <= 0 or nl == 0:
            continue
        achieved = flops / (t_ms * 1e-3) / 1e12
        kernels[k] = {"ms_middle_strip": t_ms, "launches": nl, "achieved_tflops": achieved,
                      "bound": bound, "peak_tflops": peak, "frac": achieved / peak}
    dom = max(kernels, key=lambda k: kernels[k]["ms_middle_strip"])
    d = kernels[dom]
    if stages["exact"][1]:
        # the exact tier on the pixels the float kernels queued for it
        kernels["exact"] = {"ms_middle_strip": stages["exact"][0], "launches": stages["exact"][1],
                            "bound": "fp64"}
    roofline = {"kernel": dom, "bound": d["bound"], "achieved": d["achieved_tflops"],
                "peak": d["peak_tflops"], "unit": "TFLOP/s", "frac": d["frac"],
                "traffic": None,
                "peak_source": {"fp32": "measured FP32 FMA microbenchmark (tc_fp32_peak)",
                                "fp64": "measured FP64 FMA microbenchmark (tc_fp64_peak)",
                                "tensor": "MEASURED_PEAKS.json bf16_tflops_sustained"}[d["bound"]]}
    line = {"metric": "Mpixel/s temporal coherence at N=%d, %dx%d window%s" % (
                n, window[0], window[1], ", all pair coherences, phase removed from orbits "
                "and elevation on the device" if w["geometry"] else ""),
            "value": npix / (ms * 1e-3) / 1e6, "unit": "Mpixel/s", "n_gpus": 1, "steps": 1,
            "warmup": 1, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "N=%d %dx%d %s/%s window %dx%d, %d regions, coherence <= "
                                   "%.2f%s%s, strips of %d rows" % (
                                       n, rows, cols, w["shp_test"], w["estimator"], window[0],
                                       window[1], w["nregions"], w["g0_max"],
                                       ", pairs=all (%d planes)" % npairs if npairs else "",
                                       ", fBm elevation 0-2000 m, synthetic orbits"
                                       if w["geometry"] else "", S),
                       "api": "tc_run_raw_device per strip",
                       "strips": len(strips),
                       "l2": "raw strips of %.1f GB > 126 MB L2, no flush" % (
                           n * (S + 2 * ha) * cols * 8 / 1e9)},
            "roofline": roofline, "stages_middle_strip": kernels,
            "mean_shp_count": lbar, "clocks": ck,
            "mean_coherence": float(np.nanmean(coh)) if np.isfinite(coh).any() else None}
    if grid_ms is not None:
        line["geometry_grid_ms"] = grid_ms
    if args.no_extras:
        be.close()
        print(json.dumps(line))
        return

    # end to end: page-locked strip buffers reused from strip to strip
    def pinned(shape, dtype):
        return torch.empty(shape, dtype=dtype, pin_memory=True).numpy()

    prow = S + 2 * ha
    h_re, h_im = pinned((n, prow, cols), torch.float32), pinned((n, prow, cols), torch.float32)
    h_el = pinned((prow, cols), torch.float64) if w["geometry"] else None
    out = {"coh": pinned((S, cols), torch.float32), "count": pinned((S, cols), torch.int32)}
    if npairs:
        out["pairs"] = pinned((npairs, S, cols), torch.float32)
    wall = 0.0
    h2d = d2h = 0
    for r0, r1 in strips:
        m = r1 - r0
        re, im, elev = strip_planes(r0, r1)
        p = m + 2 * ha
        full = m == S
        tre = h_re if full else pinned((n, p, cols), torch.float32)
        tim = h_im if full else pinned((n, p, cols), torch.float32)
        tel = (h_el if full else pinned((p, cols), torch.float64)) if w["geometry"] else None
        o = out if full else {"coh": pinned((m, cols), torch.float32),
                              "count": pinned((m, cols), torch.int32),
                              **({"pairs": pinned((npairs, m, cols), torch.float32)}
                                 if npairs else {})}
        tre[...] = re.cpu().numpy()
        tim[...] = im.cpu().numpy()
        if tel is not None:
            tel[...] = elev
        del re, im
        t = time.perf_counter()
        be.run_raw(tre, tim, tel, r0 - ha, rows, m, cols, out=o)
        wall += time.perf_counter() - t
        h2d += tre.nbytes + tim.nbytes + (tel.nbytes if tel is not None else 0)
        d2h += sum(v.nbytes for v in o.values())
        assert np.array_equal(o["count"], count[r0:r1])
    line["e2e"] = {"value": npix / wall / 1e6, "unit": "Mpixel/s", "h2d_bytes_per_step": int(h2d),
                   "d2h_bytes_per_step": int(d2h), "ms_per_step": wall * 1e3,
                   "api": "tc_run_raw per strip (page-locked strip buffers, reused)"}
    be.close()

    # accuracy on a centred crop, and the reference kernel on the host cores
    import oracle

    def prepared(r0, nr, c0, nc):
        """Padded strip (slc, amp, valid) of output rows r0 .. r0 + nr - 1
        and columns c0 .. c0 + nc - 1 of the scene, as main.c reads it."""
        st = region_rows(max(0, r0 - ha), min(rows, r0 + nr + ha)).cpu().numpy()
        if w["geometry"]:
            pr = nr + 2 * ha
            re_c = np.full((n, pr, cols), np.nan, np.float32)
            im_c = re_c.copy()
            el_c = np.full((pr, cols), np.nan)
            o = max(0, r0 - ha) - (r0 - ha)
            re_c[:, o:o + st.shape[1]] = st.real
            im_c[:, o:o + st.shape[1]] = st.imag
            el_c[o:o + st.shape[1]] = h[max(0, r0 - ha):min(rows, r0 + nr + ha)]
            sg = dict(geo, hmin=g.hmin, hmax=g.hmax, h0=0.0)
            full = oracle.prepare_strip(re_c, im_c, el_c, r0 - ha, rows, hr, sg, grid)
            cs = slice(c0, c0 + nc + 2 * hr)
            return tuple(np.ascontiguousarray(x[:, cs]) for x in full)
        # interior crops: the halo rows and columns are pixels of the scene
        assert r0 >= ha and r0 + nr + ha <= rows and c0 >= hr and c0 + nc + hr <= cols
        st = st[:, :, c0 - hr:c0 + nc + hr]
        return tcoh_b200.read_strip(np.ascontiguousarray(st.real), np.ascontiguousarray(st.imag),
                                    0, nr + 2 * ha, 0)

    size = min(args.accuracy_size, rows - 2 * ha, cols - 2 * hr)
    r0, c0 = (rows - size) // 2, (cols - size) // 2
    crop = prepared(r0, size, c0, size)
    line["accuracy"] = crop_accuracy(crop, coh[r0:r0 + size, c0:c0 + size],
                                     count[r0:r0 + size, c0:c0 + size], size, n, kw)
    # a 1024 x 1024 crop at 60 dates; 512 columns with the pair planes
    ccols = min(512 if npairs else 1024, cols - 2 * hr)
    nrows = min(1024, rows - 2 * ha)
    cr0, cc0 = (rows - nrows) // 2, (cols - ccols) // 2
    cpu = prepared(cr0, nrows, cc0, ccols)
    line["cpu_baseline"] = reference_rate(*cpu, nrows, ccols, kw, target_s=30.0, ccols=ccols,
                                          npairs=npairs, max_rows=nrows)
    print(json.dumps(line))

def main():
    args = parse()
    if args.workload == "adjoint" and args.impl != "reference":
        return adjoint_workload(args)
    if args.workload in SCENES and args.impl != "reference":
        return scene_workload(args, args.workload)
    if args.workload == "adjoint" or args.workload in SCENES:
        print(json.dumps({"impl": "reference", "unavailable": "the reference arm times the "
                          "metric's configuration (--workload emi)"}))
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    w = WORKLOADS[args.workload]
    rows, cols = args.rows or w["rows"], args.cols or w["cols"]
    ha, hr = w["window"][0] // 2, w["window"][1] // 2
    kw = dict(window=w["window"], shp_test=w["shp_test"], alpha=w["alpha"], min_shp=w["min_shp"],
              estimator=w["estimator"], bias=w["bias"])

    import numpy as np
    import torch

    import tcoh_b200
    import tcoh_b200.synthetic as syn

    if args.impl == "reference" and world > 1 and rank != 0:
        return
    dist = None
    if world > 1 and args.impl != "reference":
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)

    stack = syn.generate(w["n"], rows, cols, nregions=w["nregions"], g0_max=w["g0_max"],
                         spacing=w["spacing"], seed=1 + rank, device=dev)
    slc, amp, valid = device_strip(torch, stack, ha, hr)
    del stack
    torch.cuda.synchronize()
    P, Q = slc.shape[0], slc.shape[1]

    if args.impl == "reference":
        slc_h, amp_h, valid_h = slc.cpu().numpy(), amp.cpu().numpy(), valid.cpu().numpy()
        vals = []
        for i in range(args.warmup + args.steps):
            r = reference_rate(slc_h, amp_h, valid_h, rows, cols, kw, target_s=5.0)
            if i >= args.warmup:
                vals.append(r["value"])
        v = float(np.mean(vals))
        line = {"impl": "reference", "metric": metric_name(w), "value": v, "unit": "Mpixel/s",
                "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": workload_name(rows, cols, w), "parallelism": "host cores"},
                "cpu_baseline": dict(r, value=v),
                "e2e": {"value": v, "unit": "Mpixel/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    s = tcoh_b200.make_settings(w["n"], **kw)
    try:
        be = tcoh_b200.Backend(s, Q, device=local, gram=args.gram)
    except tcoh_b200.BackendError:
        if args.gram != "tensor":
            raise
        args.gram = "fp32"
        be = tcoh_b200.Backend(s, Q, device=local, gram=args.gram)
    coh = torch.empty((rows, cols), dtype=torch.float32, device=dev)
    count = torch.empty((rows, cols), dtype=torch.int32, device=dev)
    stream = torch.cuda.Stream(dev)

    def step(b=be):
        b.run_device(slc, amp, valid, rows, cols, coh, count, stream=stream)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = Clocks(local)
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize()
    ck = clocks.stop()
    ms = e0.elapsed_time(e1) / args.steps
    if dist:
        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        dist.barrier()

    # Per-stage device time of one more step (events around every launch),
    # with the per-pixel status bits of the whole strip.
    status = torch.empty((rows, cols), dtype=torch.uint8, device=dev)
    be.set_timing(True)
    be.run_device(slc, amp, valid, rows, cols, coh, count, status=status, stream=stream)
    torch.cuda.synchronize()
    stages = be.stage_stats()
    be.set_timing(False)
    status_h = status.cpu().numpy()
    del status
    launches = sum(v[1] for k, v in stages.items() if k != "copy")

    npix = rows * cols
    value = world * npix / (ms * 1e-3) / 1e6
    cnt = count.cpu().numpy()
    coh_h = coh.cpu().numpy()
    validpix = cnt >= 0
    estimated = cnt >= s.min_looks
    lbar = float(cnt[validpix].mean()) if validpix.any() else 0.0
    f_gram, f_link = flops_per_pixel(w["n"], lbar, w["estimator"] == "emi")
    fp32_peak = tcoh_b200.fp32_peak_tflops(local)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        pass
    # the Gram runs inside a step of about a second: the sustained figure
    bf16_peak = peaks.get("bf16_tflops_sustained", peaks.get("bf16_tflops", 1381.5))
    work = {
        "shp": (shp_ops_per_pixel(w["n"], w["shp_test"], w["window"][0] * w["window"][1]) *
                validpix.sum(), "fp32", fp32_peak),
        "gram": (f_gram * validpix.sum(), "tensor" if args.gram == "tensor" else "fp32",
                 bf16_peak if args.gram == "tensor" else fp32_peak),
        "link": (f_link * estimated.sum(), "fp32", fp32_peak),
    }
    kernels = {}
    for name, (flops, bound, peak) in work.items():
        t_ms, nl = stages[name]
        if t_ms <= 0 or nl == 0:
            continue
        per_launch_ms = t_ms / nl
        achieved = flops / nl / (per_launch_ms * 1e-3) / 1e12
        kernels[name] = {"ms_per_step": t_ms, "launches": nl, "achieved_tflops": achieved,
                         "bound": bound, "peak_tflops": peak, "frac": achieved / peak}
    dom = max(kernels, key=lambda k: kernels[k]["ms_per_step"])
    d = kernels[dom]
    if stages["exact"][1]:
        # the exact tier on the pixels the float kernels queued for it
        kernels["exact"] = {"ms_per_step": stages["exact"][0], "launches": stages["exact"][1],
                            "bound": "fp64"}
    roofline = {"kernel": dom, "bound": d["bound"], "achieved": d["achieved_tflops"],
                "peak": d["peak_tflops"], "unit": "TFLOP/s",
                "frac": d["frac"], "traffic": None,
                "algorithmic_bytes_per_launch": None,
                "peak_source": ("measured FP32 FMA microbenchmark (tc_fp32_peak)"
                                if d["bound"] == "fp32" else "MEASURED_PEAKS.json bf16_tflops_sustained")}

    if dom == "link" and w["n"] == 30 and w["estimator"] == "emi":
        px_launch = npix / d["launches"]
        roofline["traffic"] = LINK_DRAM_BYTES_PER_PIXEL * px_launch
        roofline["algorithmic_bytes_per_launch"] = (8.0 * w["n"] * (w["n"] + 1) / 2 + 4) * px_launch
        roofline["traffic_source"] = ("constant: ncu dram bytes of one 65,536-pixel launch "
                                      "(profiles/tc_link_half_kernel_emi_bias_n30_256x4096.md), "
                                      "scaled by the pixels per launch")
    line = {"metric": metric_name(w), "value": value, "unit": "Mpixel/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": workload_name(rows, cols, w), "gram": args.gram,
                       "pixels_per_step": npix, "parallelism": "dp%d (independent strips)" % world,
                       "l2": "inputs %.1f GB per step > 126 MB L2, no flush" % (
                           (slc.numel() * 4 + amp.numel() * 4 + valid.numel()) / 1e9)},
            "gpu_launches": launches * args.steps,
            "roofline": roofline,
            "stages": kernels,
            "mean_shp_count": lbar,
            "estimated_fraction": float(estimated.mean()),
            # pixels of the whole strip that the FP64 exact tier computed
            "fp64_tier_fraction": float(((status_h & tcoh_b200.STATUS_FP64) != 0)[estimated].mean())
            if estimated.any() else 0.0,
            "mean_coherence": float(np.nanmean(coh_h)) if np.isfinite(coh_h).any() else None,
            "clocks": ck}

    if not args.no_extras and rank == 0:
        # Plain FP32 form of the Gram on the same strip.
        if args.gram == "tensor":
            try:
                be32 = tcoh_b200.Backend(s, Q, device=local, gram="fp32")
                c32 = torch.empty_like(coh)
                n32 = torch.empty_like(count)

                def step32():
                    be32.run_device(slc, amp, valid, rows, cols, c32, n32, stream=stream)

                step32()
                torch.cuda.synchronize()
                e0.record(stream)
                for _ in range(3):
                    step32()
                e1.record(stream)
                e1.synchronize()
                ms32 = e0.elapsed_time(e1) / 3
                line["plain_fp32"] = {"value": npix / (ms32 * 1e-3) / 1e6, "ms_per_step": ms32,
                                      "tensor_over_plain": ms32 / ms}
                be32.close()
            except tcoh_b200.BackendError as e:
                line["plain_fp32"] = {"error": str(e)}
        # End to end through the C-ABI with page-locked host buffers.
        slc_h = torch.empty(slc.shape, dtype=torch.float32, pin_memory=True)
        amp_h = torch.empty(amp.shape, dtype=torch.float32, pin_memory=True)
        valid_h = torch.empty(valid.shape, dtype=torch.uint8, pin_memory=True)
        slc_h.copy_(slc)
        amp_h.copy_(amp)
        valid_h.copy_(valid)
        out = {"coh": torch.empty((rows, cols), dtype=torch.float32, pin_memory=True).numpy(),
               "count": torch.empty((rows, cols), dtype=torch.int32, pin_memory=True).numpy()}
        sn, an, vn = slc_h.numpy(), amp_h.numpy(), valid_h.numpy()
        be.run(sn, an, vn, rows, cols, out=out)
        ke = max(1, min(3, args.steps))
        t = time.perf_counter()
        for _ in range(ke):
            be.run(sn, an, vn, rows, cols, out=out)
        dt = (time.perf_counter() - t) / ke
        line["e2e"] = {"value": npix / dt / 1e6, "unit": "Mpixel/s",
                       "h2d_bytes_per_step": int(sn.nbytes + an.nbytes + vn.nbytes),
                       "d2h_bytes_per_step": int(out["coh"].nbytes + out["count"].nbytes),
                       "ms_per_step": dt * 1e3, "api": "tc_run_ex (the ocl_run path)"}
        # CPU baseline and accuracy on crops.
        line["cpu_baseline"] = reference_rate(sn, an, vn, rows, cols, kw, target_s=12.0)
        line["accuracy"] = accuracy(sn, an, vn, coh_h, cnt, rows, cols, kw,
                                    size=args.accuracy_size)
    be.close()
    if rank == 0:
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
