"""Row bands for running the path on several GPUs, one process per GPU.

Output pixels are independent given WA/2 rows of halo above and below
(main.c:782-790 reads every strip with its halo), so a region splits into
contiguous bands of output rows, one per rank, each read with its own halo
rows. Nothing crosses ranks until the outputs are gathered: there is no
collective on the data path.
"""

from .strip import read_strip


def row_band(rows, world, rank):
    """Output rows [r0, r1) of `rank` among `world` ranks: contiguous bands
    in rank order whose sizes differ by at most one row. With more ranks
    than rows the surplus ranks get no rows: None, and they skip the strip
    (band_strip returns None for them too)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank %d of %d" % (rank, world))
    base, extra = divmod(int(rows), world)
    r0 = rank * base + min(rank, extra)
    r1 = r0 + base + (1 if rank < extra else 0)
    return (r0, r1) if r1 > r0 else None


def band_strip(re, im, band, window, phase=None, elevation=None):
    """(slc, amp, valid) of the padded strip of output rows band = (r0, r1)
    of a region (re, im: (N, rows, cols), NaN = NULL): the band's rows with
    WA/2 halo rows on each side, NULL outside the region, as read_strip
    lays them out for ocl_run. None for a rank without rows (band None)."""
    if band is None:
        return None
    r0, r1 = band
    ha, hr = window[0] // 2, window[1] // 2
    return read_strip(re, im, r0 - ha, (r1 - r0) + 2 * ha, hr, phase=phase, elevation=elevation)
