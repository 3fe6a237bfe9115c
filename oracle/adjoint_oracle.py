"""FP64 oracle of the adjoint of the temporal coherence.

TEST INFRASTRUCTURE ONLY: the checker that the CUDA adjoint is compared
with; nothing in the product imports it.

The objective is the sum of gamma over the estimated pixels of a strip,
L = sum_p gamma_p, as a function of the per-sample phase

    theta_{q,k} = phi_k(q, h_q + dh_q) + psi_{q,k}

removed from the raw samples (s'_{q,k} = s_{q,k} exp(i theta_{q,k})):
phi is the flat-earth / topographic phase interpolated from the orbit grid
at the cell's height plus a height error dh (geometry.c:256-291), psi a
per-date phase screen. The forward restates reference.py (tests/reference.py
of the reference, lines 124-184) in torch complex128 -- coherence matrix,
bias correction, EVD (np.linalg.eigh -> torch.linalg.eigh), EMI (the
eigen-pseudo-inverse of |T| with absolute floor 1e-9), phases relative to
the median date, Pepe-Lanari goodness of fit -- on the SHP masks of the
C oracle (the masks depend on amplitudes only, not on theta), and torch's
autograd gives dL/d(dh) and dL/d(psi). tests/test_adjoint.py pins this
gradient with central finite differences in FP64.
"""

import numpy as np
import torch

STEP = 16


def _weights(heights, h):
    """Quadratic Lagrange weights of h over three levels (geometry.c:273-281),
    or 1 for a single level."""
    if len(heights) == 1:
        return [torch.ones_like(h)]
    x0, x1, x2 = (float(v) for v in heights)
    return [(h - x1) * (h - x2) / ((x0 - x1) * (x0 - x2)),
            (h - x0) * (h - x2) / ((x1 - x0) * (x1 - x2)),
            (h - x0) * (h - x1) / ((x2 - x0) * (x2 - x1))]


def grid_phase(grid, heights, row0, rows, cols, h, region_rows):
    """phi (N, rows, cols) at region rows row0 .. of a strip and heights h
    (torch, rows x cols), bilinear in position, quadratic in h (rows
    outside the region take the nearest region row; they are invalid)."""
    g = torch.as_tensor(grid, dtype=torch.float64)
    n = g.shape[3]
    rr = torch.arange(row0, row0 + rows).clamp(0, region_rows - 1)
    cc = torch.arange(cols)
    gr, gc = rr // STEP, cc // STEP
    fr = ((rr - gr * STEP).double() / STEP)[:, None]
    fc = ((cc - gc * STEP).double() / STEP)[None, :]
    w = _weights(heights, h)
    phi = torch.zeros((n, rows, cols), dtype=torch.float64)
    for hl in range(len(heights)):
        p00 = g[gr][:, gc, hl]          # rows, cols, n
        p01 = g[gr][:, gc + 1, hl]
        p10 = g[gr + 1][:, gc, hl]
        p11 = g[gr + 1][:, gc + 1, hl]
        v = ((1 - fr)[..., None] * ((1 - fc)[..., None] * p00 + fc[..., None] * p01) +
             fr[..., None] * ((1 - fc)[..., None] * p10 + fc[..., None] * p11))
        phi = phi + (w[hl][..., None] * v).permute(2, 0, 1)
    return phi


def _connected(t):
    n = t.shape[0]
    seen, todo = {0}, [0]
    while todo:
        i = todo.pop()
        for j in range(n):
            if j not in seen and t[i, j] != 0:
                seen.add(j)
                todo.append(j)
    return len(seen) == n


def gamma_sum(a, mask, count, window, min_looks, estimator, bias):
    """L = sum of gamma over the estimated pixels, and gamma (numpy, NaN for
    the others). a: complex128 (P, W, N) rotated samples of the padded strip
    (zero where invalid); mask (rows, cols, words) SHP bits; count (rows,
    cols)."""
    rows, cols = count.shape
    wa, wr = window
    n = a.shape[2]
    iu = torch.triu_indices(n, n, 1)
    npairs = 0.5 * n * (n - 1)
    total = torch.zeros((), dtype=torch.float64)
    gam = np.full((rows, cols), np.nan)
    for y in range(rows):
        for x in range(cols):
            looks = int(count[y, x])
            if looks < min_looks:
                continue
            bits = [b for b in range(wa * wr) if (int(mask[y, x, b >> 5]) >> (b & 31)) & 1]
            dy = torch.tensor([b // wr for b in bits])
            dx = torch.tensor([b % wr for b in bits])
            s = a[y + dy, x + dx]                       # looks, n
            cov = s.T @ s.conj()
            d = torch.sqrt(cov.diagonal().real / looks)
            t = cov / looks / torch.outer(d, d)
            if bias and looks > 1:
                m2 = (t.real ** 2 + t.imag ** 2)
                m2c = (looks * m2 - 1.0) / (looks - 1.0)
                ok = (m2 > 0) & (m2c > 0)
                f = torch.where(ok, torch.sqrt(torch.where(ok, m2c, 1.0) / torch.where(ok, m2, 1.0)),
                                torch.zeros_like(m2))
                t = t * f
            t = t - torch.diag(t.diagonal()) + torch.eye(n, dtype=t.dtype)
            if bias and not _connected(t.detach().numpy()):
                continue
            if estimator == "evd":
                _w, v = torch.linalg.eigh(t)
                u = v[:, -1]
            else:
                g = torch.abs(t)
                w, v = torch.linalg.eigh(g)
                keep = (w.abs() >= 1e-9).double()
                inv = (v * (keep / torch.where(keep > 0, w, torch.ones_like(w)))) @ v.T
                _w, v = torch.linalg.eigh(inv * t)
                u = v[:, 0]
            mag = torch.abs(u).detach()
            floor = 1e-3 * float(mag.max())
            ref = n // 2
            if float(mag[ref]) <= floor:
                ref = int(torch.argmax(mag))
            rel = u * u[ref].conj()
            big = mag > floor
            e = torch.where(big, rel / torch.where(big, torch.abs(rel), torch.ones_like(mag)),
                            torch.ones_like(rel))
            tij = t[iu[0], iu[1]]
            nz = torch.abs(tij).detach() > 0
            wij = torch.where(nz, tij / torch.where(nz, torch.abs(tij), torch.ones_like(tij.real)),
                              torch.ones_like(tij))
            ssum = (wij * e[iu[0]].conj() * e[iu[1]]).sum()
            g = torch.abs(ssum) / npairs
            gam[y, x] = float(g.detach())
            total = total + g
    return total, gam


def adjoint(re, im, heights, dh, psi, row0, region_rows, halo_cols, mask, count, window,
            min_looks, estimator, bias, grid=None, grid_heights=None, h0=0.0):
    """(L, gamma, dL/d(dh), dL/d(psi)) for one strip.

    re, im (N, P, cols) raw samples of region rows row0 .. (NaN = NULL);
    heights (P, cols) or None (h0 everywhere); dh (P, cols) and psi (N, P,
    cols) the variables; mask / count from the oracle on the same strip;
    grid / grid_heights the phase grid (None: no geometric phase, dL/d(dh)
    is zero)."""
    n, prow, cols = re.shape
    re64 = torch.as_tensor(np.nan_to_num(re).astype(np.float64))
    im64 = torch.as_tensor(np.nan_to_num(im).astype(np.float64))
    rr = torch.arange(row0, row0 + prow)
    inreg = ((rr >= 0) & (rr < region_rows))[None, :, None]
    valid = inreg & torch.as_tensor(np.all(np.isfinite(re) & np.isfinite(im) &
                                           ~((re == 0) & (im == 0)), axis=0))[None]
    if heights is not None:
        valid = valid & torch.as_tensor(np.isfinite(heights))[None]
    dh_t = torch.as_tensor(np.asarray(dh, np.float64)).clone().requires_grad_(True)
    psi_t = torch.as_tensor(np.asarray(psi, np.float64)).clone().requires_grad_(True)
    theta = psi_t
    if grid is not None:
        h = torch.as_tensor(np.nan_to_num(heights) if heights is not None
                            else np.full((prow, cols), h0), dtype=torch.float64)
        theta = theta + grid_phase(grid, grid_heights, row0, prow, cols, h + dh_t, region_rows)
    s = torch.complex(re64, im64) * torch.exp(1j * theta)
    s = torch.where(valid, s, torch.zeros_like(s))
    a = torch.zeros((prow, cols + 2 * halo_cols, n), dtype=torch.complex128)
    a[:, halo_cols:halo_cols + cols] = s.permute(1, 2, 0)
    total, gam = gamma_sum(a, mask, count, window, min_looks, estimator, bias)
    total.backward()
    g_dh = dh_t.grad.numpy() if dh_t.grad is not None else np.zeros_like(np.asarray(dh))
    return float(total.detach()), gam, g_dh, psi_t.grad.numpy()
