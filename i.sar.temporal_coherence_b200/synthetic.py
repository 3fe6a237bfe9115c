"""Seeded synthetic distributed-scatterer stacks.

The benchmark workloads follow the reference's published configurations: an
image split into Voronoi regions, each with a Rayleigh amplitude scale sigma
~ U[0.5, 4] and an exponential coherence model

    Gamma_ij = (g0 - ginf) exp(-|t_i - t_j| / tau) + ginf   (i != j),  Gamma_ii = 1,

g0 ~ U[0.3, g0_max], ginf ~ U[0, 0.2], tau ~ U[24, 120] days; per pixel
s = sigma chol(Gamma) CN(0, I), times a smooth deterministic per-date phase
ramp; 0.5 % of the pixels get a NULL (NaN) or zero sample at one random
date; samples are scaled to 16-bit digital numbers (x 300, rounded) like the
reference's test stacks, so that equal amplitudes occur and the tie rules of
the SHP tests are exercised.

``generate`` works in numpy (small stacks) or in torch on a GPU (large
ones); both are deterministic for a given seed, but they draw differently.
The torch form draws every band of rows from a generator of its own, so
that a range of rows of a scene too large for the device (``row_range``)
is the same whether it is generated alone or with the whole scene.
"""

import numpy as np


def _regions(rng, nregions, rows, cols):
    seeds_y = rng.uniform(0, rows, nregions)
    seeds_x = rng.uniform(0, cols, nregions)
    return seeds_y, seeds_x


def region_params(rng, nregions, g0_max):
    return {
        "sigma": rng.uniform(0.5, 4.0, nregions),
        "g0": rng.uniform(0.3, g0_max, nregions),
        "ginf": rng.uniform(0.0, 0.2, nregions),
        "tau": rng.uniform(24.0, 120.0, nregions),
    }


def coherence_model(n, spacing, g0, ginf, tau):
    t = np.arange(n) * spacing
    g = (g0 - ginf) * np.exp(-np.abs(t[:, None] - t[None, :]) / tau) + ginf
    np.fill_diagonal(g, 1.0)
    return g


def generate(n, rows, cols, nregions=8, g0_max=0.95, spacing=12.0, seed=0, null_frac=0.005,
             device=None, scale=300.0, row_range=None):
    """Stack (n, rows, cols) complex64 (NaN = NULL), as numpy, or as a torch
    tensor on `device` when given; with row_range = (a, b) (torch only),
    rows a .. b - 1 of that scene, (n, b - a, cols)."""
    rng = np.random.default_rng(seed)
    sy, sx = _regions(rng, nregions, rows, cols)
    par = region_params(rng, nregions, g0_max)
    chol = np.stack([
        np.linalg.cholesky(coherence_model(n, spacing, par["g0"][r], par["ginf"][r], par["tau"][r]))
        for r in range(nregions)
    ])
    fy, fx = rng.uniform(0.5, 2.0), rng.uniform(0.5, 2.0)
    nnull = int(round(null_frac * rows * cols))
    null_pix = rng.choice(rows * cols, size=nnull, replace=False)
    null_date = rng.integers(0, n, nnull)
    null_zero = rng.random(nnull) < 0.5
    if device is None:
        if row_range is not None:
            raise ValueError("row_range needs the torch form (device)")
        return _generate_numpy(rng, n, rows, cols, sy, sx, par, chol, fy, fx, null_pix,
                               null_date, null_zero, scale)
    return _generate_torch(seed, n, rows, cols, sy, sx, par, chol, fy, fx, null_pix,
                           null_date, null_zero, scale, device, row_range)


def _ramp(n, rows, cols, fy, fx, y, x):
    k = np.arange(n, dtype=np.float64)[:, None]
    return 0.7 * k + 2.0 * np.pi * k / n * (fy * y[None, :] / rows + fx * x[None, :] / cols)


def _generate_numpy(rng, n, rows, cols, sy, sx, par, chol, fy, fx, null_pix, null_date,
                    null_zero, scale):
    y, x = np.divmod(np.arange(rows * cols), cols)
    region = np.argmin((y[:, None] - sy[None, :]) ** 2 + (x[:, None] - sx[None, :]) ** 2, axis=1)
    z = (rng.standard_normal((n, rows * cols)) + 1j * rng.standard_normal((n, rows * cols))) / np.sqrt(2)
    s = np.empty((n, rows * cols), np.complex128)
    for r in range(len(sy)):
        m = region == r
        s[:, m] = par["sigma"][r] * (chol[r] @ z[:, m])
    s *= np.exp(1j * _ramp(n, rows, cols, fy, fx, y, x))
    s = np.round(s * scale)
    s[null_date, null_pix] = np.where(null_zero, 0.0, np.nan)
    return s.reshape(n, rows, cols).astype(np.complex64)


def _generate_torch(seed, n, rows, cols, sy, sx, par, chol, fy, fx, null_pix, null_date,
                    null_zero, scale, device, row_range=None):
    import torch

    a, b = (0, rows) if row_range is None else (int(row_range[0]), int(row_range[1]))
    if not 0 <= a <= b <= rows:
        raise ValueError("row range %r of %d rows" % ((a, b), rows))
    g = torch.Generator(device=device)
    out = torch.empty((n, b - a, cols), dtype=torch.complex64, device=device)
    sy_t = torch.tensor(sy, device=device, dtype=torch.float32)
    sx_t = torch.tensor(sx, device=device, dtype=torch.float32)
    chol_t = torch.tensor(chol, device=device, dtype=torch.complex64)
    sigma = torch.tensor(par["sigma"], device=device, dtype=torch.float32)
    k = torch.arange(n, device=device, dtype=torch.float64)[:, None]
    band = max(1, (1 << 21) // max(cols, 1))
    for r0 in range(a // band * band, b, band):
        r1 = min(rows, r0 + band)
        g.manual_seed(int(seed) * 1000003 + r0 // band)
        yy, xx = torch.meshgrid(torch.arange(r0, r1, device=device, dtype=torch.float32),
                                torch.arange(cols, device=device, dtype=torch.float32),
                                indexing="ij")
        yy, xx = yy.reshape(-1), xx.reshape(-1)
        d = (yy[:, None] - sy_t[None, :]) ** 2 + (xx[:, None] - sx_t[None, :]) ** 2
        region = torch.argmin(d, dim=1)
        p = yy.numel()
        z = torch.complex(torch.randn((n, p), generator=g, device=device),
                          torch.randn((n, p), generator=g, device=device)) / np.sqrt(2.0)
        lz = torch.empty_like(z)
        for r in range(len(sy)):
            idx = (region == r).nonzero().squeeze(1)
            if idx.numel():
                lz[:, idx] = (chol_t[r] @ z[:, idx]) * sigma[r]
        ramp = 0.7 * k + 2.0 * np.pi * k / n * (fy * yy.double()[None, :] / rows +
                                                fx * xx.double()[None, :] / cols)
        s = lz * torch.polar(torch.ones_like(ramp), ramp).to(torch.complex64)
        s = torch.complex(torch.round(s.real * scale), torch.round(s.imag * scale))
        s = s.reshape(n, r1 - r0, cols)
        lo, hi = max(a, r0), min(b, r1)
        out[:, lo - a:hi - a] = s[:, lo - r0:hi - r0]
    keep = (null_pix >= a * cols) & (null_pix < b * cols)
    if keep.any():
        flat = out.view(n, -1)
        vals = torch.tensor(np.where(null_zero[keep], 0.0, np.nan), device=device,
                            dtype=torch.float32)
        flat[torch.tensor(null_date[keep], device=device),
             torch.tensor(null_pix[keep] - a * cols, device=device)] = torch.complex(vals, vals)
    return out
