"""Host-side strip preparation and strip loop, as the module does around its
device backend.

The GRASS module keeps these in C (main.c); this file restates them for
hosts that drive the backend from Python (the test harness, the benchmark,
notebooks). Layouts are the ones ``ocl_run`` receives (main.c:28-34,
52-127):

    slc   float32 [padded_rows][padded_cols][N][2]   (re, im), phase-removed
    amp   float32 [padded_rows][padded_cols][N]      sorted ascending
    valid uint8   [padded_rows][padded_cols]

with padded_cols = cols + 2 * (WR // 2) and padded_rows = rows + 2 * (WA // 2)
(main.c:651-653, 788); halo cells outside the region are invalid and zero.
"""

import numpy as np


def pair_list(n, pairs_all):
    """Dates (i, j) of each pair plane, in the order of main.c:611-615 and
    tcoh.cl:522-523: (0,1), (0,2), ... for all pairs, (0,1), (1,2), ... for
    consecutive ones."""
    if pairs_all:
        return [(i, j) for i in range(n - 1) for j in range(i + 1, n)]
    return [(i, i + 1) for i in range(n - 1)]


def npairs_for(n, pairs, pairs_all):
    """Number of pair planes (main.c:608)."""
    if not pairs:
        return 0
    return n * (n - 1) // 2 if pairs_all else n - 1


def read_strip(re, im, row0, padded_rows, halo_cols, phase=None, elevation=None):
    """Padded strip of region rows row0 .. row0 + padded_rows - 1.

    re, im: float32 (N, rows, cols) samples of the region, NaN for NULL (the
    FCELL rows that Rast_get_f_row returns). phase: optional float64
    (N, rows, cols) geometric phase to remove (date k times exp(i phase_k)),
    evaluated at each pixel's height. elevation: optional float64 (rows,
    cols); a NaN height makes the pixel invalid (main.c:93-94).

    Restates main.c:52-127: a pixel is valid when every date is non-null and
    not exactly zero; amplitudes sqrtf(re^2 + im^2) are taken and sorted
    before the phase rotation, which is done in double precision and rounded
    to float.
    """
    re = np.asarray(re, dtype=np.float32)
    im = np.asarray(im, dtype=np.float32)
    n, nrows, ncols = re.shape
    padded_cols = ncols + 2 * halo_cols
    slc = np.zeros((padded_rows, padded_cols, n, 2), np.float32)
    amp = np.zeros((padded_rows, padded_cols, n), np.float32)
    valid = np.zeros((padded_rows, padded_cols), np.uint8)
    r0, r1 = max(row0, 0), min(row0 + padded_rows, nrows)
    if r1 <= r0:
        return slc, amp, valid
    sl = slice(r0, r1)
    rr, ri = re[:, sl], im[:, sl]
    null = np.isnan(rr) | np.isnan(ri) | ((rr == 0) & (ri == 0))
    ok = ~null.any(axis=0)
    if elevation is not None:
        ok &= ~np.isnan(np.asarray(elevation, dtype=np.float64)[sl])
    rr = np.where(ok, rr, np.float32(0))
    ri = np.where(ok, ri, np.float32(0))
    a = np.sqrt(rr * rr + ri * ri)  # float32 throughout, as sqrtf
    a = np.sort(a, axis=0)
    if phase is not None:
        ph = np.asarray(phase, dtype=np.float64)[:, sl]
        cs, sn = np.cos(ph), np.sin(ph)
        rd, idd = rr.astype(np.float64), ri.astype(np.float64)
        nr = (rd * cs - idd * sn).astype(np.float32)
        ni = (rd * sn + idd * cs).astype(np.float32)
        rr = np.where(ok, nr, np.float32(0))
        ri = np.where(ok, ni, np.float32(0))
    y0 = r0 - row0
    y1 = y0 + (r1 - r0)
    cs_ = slice(halo_cols, halo_cols + ncols)
    slc[y0:y1, cs_, :, 0] = np.moveaxis(rr, 0, -1)
    slc[y0:y1, cs_, :, 1] = np.moveaxis(ri, 0, -1)
    amp[y0:y1, cs_, :] = np.moveaxis(a, 0, -1)
    valid[y0:y1, cs_] = ok.astype(np.uint8)
    return slc, amp, valid


def strip_rows_for(nrows, ncols, n, win_az, win_rg, npairs, memory_mb, max_alloc):
    """Strip height of main.c:727-749 for the memory= budget (MB) and the
    backend's largest allocation."""
    padded_cols = ncols + 2 * (win_rg // 2)
    per_row = padded_cols * (12 * n + 1) + ncols * 4 * (2 + npairs)
    budget = int(memory_mb) * 1024 * 1024
    strip_rows = budget // per_row - (win_az - 1)
    if max_alloc > 0:
        dev_rows = max_alloc // (padded_cols * n * 8) - (win_az - 1)
        strip_rows = min(strip_rows, dev_rows)
        if npairs:
            strip_rows = min(strip_rows, max_alloc // (ncols * npairs * 4))
    if strip_rows < 1:
        raise MemoryError(
            "Not enough memory for one row of %d columns and %d dates; "
            "increase memory or reduce the region" % (ncols, n)
        )
    return min(strip_rows, nrows)
