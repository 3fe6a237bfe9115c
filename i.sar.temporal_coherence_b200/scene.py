"""Seeded synthetic acquisition geometry for the geometry and adjoint
workloads: orbits, raster timing, a fractal height field, and the host-side
interpolation of a phase grid.

The orbits are circular and near-polar in an Earth-fixed frame (no Earth
rotation), one per date, all flying the same ground track north at the
same along-track times relative to the date's epoch and offset across
track by the date's perpendicular baseline; the radar looks right (towards
+y). Each date gets ten state vectors, 10 s apart, centred on its scene.
The reference image's raster timing places its rows x cols samples at the
centre of that span, from a near slant range. The values follow the
benchmark configurations: 700 km altitude, 7.6 km/s, baselines uniform in
+-150 m, C band (5.55 cm), 12-day spacing.
"""

import numpy as np

SPEED_OF_LIGHT = 299792458.0
EARTH_A = 6378137.0


def acquisition(n, rows, cols, ref=None, seed=0, spacing_days=12.0, baseline=150.0,
                wavelength=0.0555, altitude=700e3, speed=7600.0, near_range=850e3,
                azimuth_time_interval=2.0e-3, range_sampling_rate=64.345e6,
                latitude_deg=25.0, epoch0=1.7e9):
    """(geometry fields, orbits): a dict with the fields of struct
    tc_geometry except the height range, and per date (t, pos, vel) with ten
    state vectors."""
    rng = np.random.default_rng(seed)
    ref = n // 2 if ref is None else ref
    radius = EARTH_A + altitude
    omega = speed / radius
    lat0 = np.radians(latitude_deg)
    offsets = rng.uniform(-baseline, baseline, n)
    offsets[ref] = 0.0
    orbits = []
    for k in range(n):
        epoch = epoch0 + k * spacing_days * 86400.0
        t = epoch + 10.0 * (np.arange(10) - 4.5)
        theta = lat0 + omega * (t - epoch)
        pos = np.stack([radius * np.cos(theta), np.full_like(theta, offsets[k]),
                        radius * np.sin(theta)], axis=1)
        vel = np.stack([-radius * omega * np.sin(theta), np.zeros_like(theta),
                        radius * omega * np.cos(theta)], axis=1)
        orbits.append((t, pos, vel))
    epoch_ref = epoch0 + ref * spacing_days * 86400.0
    geo = dict(ndates=n, ref=ref,
               first_line_time=epoch_ref - 0.5 * rows * azimuth_time_interval,
               azimuth_time_interval=azimuth_time_interval,
               slant_range_time=2.0 * near_range / SPEED_OF_LIGHT,
               range_sampling_rate=range_sampling_rate, wavelength=wavelength,
               line0=0.0, sample0=0.0, rows=rows, cols=cols)
    return geo, orbits


def fbm_heights(rows, cols, hurst=0.8, hmax=2000.0, seed=0):
    """Fractal Brownian surface (spectral synthesis, power spectrum
    ~ |k|^-(2H + 2)) scaled to 0 .. hmax metres."""
    rng = np.random.default_rng(seed)
    ky = np.fft.fftfreq(rows)[:, None]
    kx = np.fft.rfftfreq(cols)[None, :]
    k = np.sqrt(ky * ky + kx * kx)
    k[0, 0] = 1.0
    amp = k ** (-(hurst + 1.0))
    amp[0, 0] = 0.0
    noise = rng.normal(size=(rows, cols // 2 + 1)) + 1j * rng.normal(size=(rows, cols // 2 + 1))
    h = np.fft.irfft2(noise * amp, s=(rows, cols))
    h -= h.min()
    return h * (hmax / max(h.max(), 1e-12))


def smooth(field, size):
    """Box average over size x size cells (edges replicated)."""
    pad = size // 2
    f = np.pad(field, pad, mode="edge")
    c = np.cumsum(np.cumsum(f, axis=0), axis=1)
    c = np.pad(c, ((1, 0), (1, 0)))
    rows, cols = field.shape
    s = c[size:size + rows, size:size + cols] - c[:rows, size:size + cols] - \
        c[size:size + rows, :cols] + c[:rows, :cols]
    return s / (size * size)


def grid_phases(grid, grid_heights, heights, row0=0):
    """The phase of every date at region rows row0 .. and the given heights
    (rows x cols), interpolated from a phase grid [grid_rows][grid_cols]
    [nheights][ndates] bilinearly in position and quadratically in height,
    as the device does (geometry.c:256-291). Returns (ndates, rows, cols)."""
    rows, cols = heights.shape
    step = 16
    rr = np.arange(row0, row0 + rows)
    cc = np.arange(cols)
    gr, gc = rr // step, cc // step
    fr = ((rr - gr * step) / step)[:, None, None]
    fc = ((cc - gc * step) / step)[None, :, None]
    h = np.asarray(heights, np.float64)
    if len(grid_heights) == 3:
        x0, x1, x2 = grid_heights
        w = [(h - x1) * (h - x2) / ((x0 - x1) * (x0 - x2)),
             (h - x0) * (h - x2) / ((x1 - x0) * (x1 - x2)),
             (h - x0) * (h - x1) / ((x2 - x0) * (x2 - x1))]
    else:
        w = [np.ones_like(h)]
    out = 0.0
    for hl, wh in enumerate(w):
        g = grid[:, :, hl, :]
        v = ((1 - fr) * ((1 - fc) * g[gr][:, gc] + fc * g[gr][:, gc + 1]) +
             fr * ((1 - fc) * g[gr + 1][:, gc] + fc * g[gr + 1][:, gc + 1]))
        out = out + wh[:, :, None] * v
    return np.moveaxis(out, 2, 0)
