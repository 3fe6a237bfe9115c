"""Shared fixtures: the package (by its import name), the oracle, golden
cases and strip builders."""

import glob
import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle  # noqa: E402
import tcoh_b200  # noqa: E402

GOLDEN = os.path.join(ROOT, "tests", "golden")
# Largest difference to the double-precision reference
# (tests/i_sar_temporal_coherence_test.py:26-27 of the reference).
TOLERANCE = 1e-4


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 GPU and the built CUDA library")


GEOMETRY_CASES = ["flat_earth_ref0", "flat_earth_ref2", "topographic"]


def golden_names():
    return sorted(
        os.path.basename(f)[:-4]
        for f in glob.glob(os.path.join(GOLDEN, "*.npz"))
        if not f.endswith("statistics.npz")
    )


class Case:
    """A golden case: its stack (region cut), options and reference.py
    outputs."""

    def __init__(self, name):
        d = np.load(os.path.join(GOLDEN, name + ".npz"))
        self.name = name
        self.data = d
        self.options = json.loads(str(d["options"]))
        stack = d["stack"]
        if "region" in d:
            r0, r1, c0, c1 = d["region"]
            stack = stack[:, r0:r1, c0:c1]
        self.stack = stack
        self.n, self.rows, self.cols = stack.shape
        self.window = tuple(self.options.get("window", (21, 7)))
        self.phase = d["phase"] if "phase" in d else None
        self.coh = d["coh"]
        self.count = d["count"]
        self.pairs = d["pairs"] if "pairs" in d else None

    def kwargs(self):
        o = self.options
        return dict(
            window=self.window,
            shp_test=o.get("shp_test", "ks"),
            alpha=o.get("alpha", 0.05),
            min_shp=o.get("min_shp", 20),
            estimator=o.get("estimator", "evd"),
            bias=o.get("bias_correction", False),
        )

    def geometry(self):
        """For the geometry cases: the orbits (per date (t, pos, vel)), the
        geometry fields of struct tc_geometry / orc_geometry (region = the
        whole reference image) and the elevation map (None for flat earth),
        as the module reads them from each date's metadata (geometry.c:161-
        200, main.c:684-709)."""
        d = self.data
        orbits = [(d["orbit_t"][k], d["orbit_pos"][k], d["orbit_vel"][k]) for k in range(self.n)]
        heights = d["heights"]
        h0 = float(d["geo_terrain_height"])
        topo = bool(np.any(heights != h0))
        geo = dict(ndates=self.n, ref=int(d["geo_ref"]),
                   first_line_time=float(d["geo_first_line_time"]),
                   azimuth_time_interval=float(d["geo_azimuth_time_interval"]),
                   slant_range_time=float(d["geo_slant_range_time"]),
                   range_sampling_rate=float(d["geo_range_sampling_rate"]),
                   wavelength=float(d["geo_wavelength"]), line0=0.0, sample0=0.0,
                   rows=self.rows, cols=self.cols,
                   hmin=float(heights.min()) if topo else h0,
                   hmax=float(heights.max()) if topo else h0, h0=h0)
        return geo, orbits, (heights if topo else None)

    def raw_strip(self):
        """Raw I/Q planes (N, padded_rows, cols) of the region rows of the
        one strip, and its elevation rows, as main.c's read_strip reads
        them (rows outside the region are NULL)."""
        ha = self.window[0] // 2
        prow = self.rows + 2 * ha
        re = np.full((self.n, prow, self.cols), np.nan, np.float32)
        im = re.copy()
        re[:, ha:ha + self.rows] = self.stack.real
        im[:, ha:ha + self.rows] = self.stack.imag
        _geo, _orbits, heights = self.geometry() if "orbit_t" in self.data else (None, None, None)
        elev = None
        if heights is not None:
            elev = np.full((prow, self.cols), np.nan)
            elev[ha:ha + self.rows] = heights
        return re, im, elev, -ha

    def strip(self):
        """The whole region as one padded strip, as main.c reads it."""
        ha, hr = self.window[0] // 2, self.window[1] // 2
        return tcoh_b200.read_strip(self.stack.real, self.stack.imag, -ha,
                                    self.rows + 2 * ha, hr, phase=self.phase)


@pytest.fixture(params=golden_names())
def golden_case(request):
    return Case(request.param)


def header_functions():
    """Function names declared in include/*.h."""
    import re

    names = []
    for path in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(path).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"\b([a-z_][a-z0-9_]*)\s*\(", text)
    keywords = {"if", "while", "for", "sizeof", "return", "defined"}
    return sorted({n for n in names if n not in keywords and (n.startswith("tc_") or n.startswith("ocl_"))})
