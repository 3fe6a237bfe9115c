"""Generate the golden vectors of the phase-linking path from the reference.

Run in a container that has the reference checkout (it is read, never
copied), naming its directory:

    python tests/golden/make_golden.py --reference PATH_TO_REFERENCE

For every numeric case of the reference's own test-suite
(tests/i_sar_temporal_coherence_test.py), this imports the reference's
tests/reference.py (the FP64 plain-loop oracle), tests/conftest.py (for its
synthetic_stack fixture; the GRASS imports it makes are stubbed, since only
the numpy fixture is called) and tests/geometry_model.py, builds the same
inputs the reference tests build, runs reference.stack_coherence on them and
writes one compressed .npz per case here. The tests then check the repo's
oracle and the CUDA path against these files, on machines without the
reference.

Each file holds:
    stack      complex64 (N, rows, cols); NaN marks a NULL sample
    options    JSON of the stack_coherence keyword arguments
    coh        float64 (rows, cols)          reference.py output
    count      int32 (rows, cols)
    pairs      float64 (N*(N-1)/2, rows, cols) |T_ij| for all i < j, in the
               order (0,1), (0,2), ...  (only when the case uses pairs)
    phase      float64 (N, rows, cols) geometric phase applied by the test
    region     int32 [row0, row1, col0, col1] of the computed sub-region
plus, for the geometry cases, the annotation orbits and raster geometry
that the module reads from description.json (times in seconds since 1970,
as epoch.c:28-32 computes them).
"""

import argparse
import json
import os
import sys
import types
from datetime import datetime

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def load_reference(ref_dir):
    tests = os.path.join(ref_dir, "tests")
    # conftest.py imports grass.script at module level; only its pure numpy
    # helpers are used here.
    grass = types.ModuleType("grass")
    grass.script = types.ModuleType("grass.script")
    sys.modules.setdefault("grass", grass)
    sys.modules.setdefault("grass.script", grass.script)
    sys.path.insert(0, tests)
    import conftest  # noqa: E402
    import geometry_model  # noqa: E402
    import reference  # noqa: E402

    return reference, conftest, geometry_model


def utc_seconds(dt):
    """Seconds since 1970 as epoch.c:28-32 sums them."""
    days = (dt.date() - datetime(1970, 1, 1).date()).days
    second = float("{:02d}.{:06d}".format(dt.second, dt.microsecond))
    return days * 86400.0 + dt.hour * 3600.0 + dt.minute * 60.0 + second


def parse_iso(text):
    return datetime.fromisoformat(text).replace(tzinfo=None)


def save(name, stack, options, result, phase=None, region=None, extra=None):
    coh, count = result[0], result[1]
    out = {
        "stack": stack.astype(np.complex64),
        "options": np.array(json.dumps(options)),
        "coh": np.asarray(coh, dtype=np.float64),
        "count": np.asarray(count, dtype=np.int32),
    }
    assert np.array_equal(out["stack"].astype(np.complex128), stack, equal_nan=True)
    if len(result) > 2:
        pairs = result[2]
        n = pairs.shape[0]
        iu = [(i, j) for i in range(n - 1) for j in range(i + 1, n)]
        out["pairs"] = np.stack([pairs[i, j] for i, j in iu]).astype(np.float64)
    if phase is not None:
        out["phase"] = np.asarray(phase, dtype=np.float64)
    if region is not None:
        out["region"] = np.asarray(region, dtype=np.int32)
    for k, v in (extra or {}).items():
        out[k] = np.asarray(v)
    path = os.path.join(HERE, name + ".npz")
    np.savez_compressed(path, **out)
    print("wrote", path, {k: getattr(v, "shape", None) for k, v in out.items()})


def geometry_extra(geometry, geometry_model, ref, heights, h0=0.0):
    n = len(geometry.orbits)
    times, pos, vel = [], [], []
    for k in range(n):
        sv = geometry.state_vectors(k)
        times.append([utc_seconds(parse_iso(v["time"])) for v in sv])
        pos.append([v["position"] for v in sv])
        vel.append([v["velocity"] for v in sv])
    meta = geometry.metadata(ref)
    rg = meta["raster_geometry"]
    return {
        "orbit_t": np.array(times, dtype=np.float64),
        "orbit_pos": np.array(pos, dtype=np.float64),
        "orbit_vel": np.array(vel, dtype=np.float64),
        "geo_ref": np.int32(ref),
        "geo_first_line_time": np.float64(utc_seconds(parse_iso(rg["first_line_time"]))),
        "geo_azimuth_time_interval": np.float64(rg["azimuth_time_interval"]),
        "geo_slant_range_time": np.float64(rg["slant_range_time_first_sample"]),
        "geo_range_sampling_rate": np.float64(meta["swath"]["range_sampling_rate"]),
        "geo_wavelength": np.float64(meta["swath"]["wavelength"]),
        "geo_terrain_height": np.float64(h0),
        "heights": np.asarray(heights, dtype=np.float64),
    }


def main():
    parser = argparse.ArgumentParser()
    parser.add_argument("--reference", required=True,
                        help="directory of the reference checkout (i.sar.temporal_coherence)")
    args = parser.parse_args()
    reference, conftest, geometry_model = load_reference(args.reference)
    synthetic_stack = conftest.synthetic_stack
    sc = reference.stack_coherence

    # test_matches_reference (i_sar_temporal_coherence_test.py:65-83)
    stack = synthetic_stack(6, 0.7)
    for name, opts in (
        ("ks_evd_default", {}),
        ("ad_emi_9x5", {"shp_test": "ad", "estimator": "emi", "min_shp": 9, "window": [9, 5]}),
        ("tlog_7x5", {"shp_test": "tlog", "alpha": 0.01, "min_shp": 9, "window": [7, 5]}),
    ):
        kw = dict(opts)
        if "window" in kw:
            kw["window"] = tuple(kw["window"])
        save(name, stack, opts, sc(stack, **kw))

    # test_bias_correction and test_pairs_defined_when_dates_unlinked
    stack = synthetic_stack(6, 0.3, seed=3)
    for est in ("evd", "emi"):
        opts = {"bias_correction": True, "estimator": est, "window": [5, 3], "min_shp": 6}
        kw = dict(opts, window=(5, 3))
        save("bias_" + est, stack, opts, sc(stack, with_pairs=True, **kw))

    # test_strips
    stack = synthetic_stack(8, 0.6, rows=30, cols=400, seed=4)
    opts = {"window": [7, 5], "min_shp": 10}
    save("strips", stack, opts, sc(stack, window=(7, 5), min_shp=10))

    # test_coherent_and_incoherent_stacks
    for g in (0.95, 0.0):
        stack = synthetic_stack(10, g, seed=5)
        for est in ("evd", "emi"):
            opts = {"estimator": est}
            save("coherence{}_{}".format(int(g * 100), est), stack, opts, sc(stack, estimator=est))

    # test_nulls_and_zero_samples
    stack = synthetic_stack(5, 0.8, seed=6)
    stack[2, 10:13, 4:9] = np.nan
    stack[4, 20, 20] = 0
    save("nulls", stack, {"min_shp": 5}, sc(stack, min_shp=5))

    # test_region_subset: the module computes rows 5..24, cols 3..19 only
    stack = synthetic_stack(5, 0.8, seed=7)
    save("region_subset", stack, {"min_shp": 5}, sc(stack[:, 5:25, 3:20], min_shp=5),
         region=[5, 25, 3, 20])

    # test_pairs
    stack = synthetic_stack(5, 0.7, seed=20)
    save("pairs", stack, {"min_shp": 5}, sc(stack, min_shp=5, with_pairs=True))

    # test_flat_earth_phase and test_topographic_phase
    rows, cols = conftest.ROWS, conftest.COLS
    for ref in (0, 2):
        geometry = conftest.geometry_stack(6, ref=ref)
        heights = np.zeros((rows, cols))
        x = synthetic_stack(6, 0.8, rows=rows, cols=cols, seed=21)
        phase = geometry.phases(heights)
        stack = np.round(x * np.exp(-1j * phase))
        opts = {"min_shp": 6}
        save("flat_earth_ref{}".format(ref), stack, opts,
             sc(stack, min_shp=6, with_pairs=True, phase=phase), phase=phase,
             extra=geometry_extra(geometry, geometry_model, ref, heights))
    geometry = conftest.geometry_stack(6)
    y, xg = np.mgrid[0:rows, 0:cols]
    hill = 800.0 * np.exp(-((y - 15) ** 2 / 100.0 + (xg - 12) ** 2 / 50.0))
    x = synthetic_stack(6, 0.8, rows=rows, cols=cols, seed=21)
    phase = geometry.phases(hill)
    stack = np.round(x * np.exp(-1j * phase))
    save("topographic", stack, {"min_shp": 6},
         sc(stack, min_shp=6, with_pairs=True, phase=phase), phase=phase,
         extra=geometry_extra(geometry, geometry_model, 0, hill))

    # Known answers of the statistics (test_reference_statistics_match_scipy):
    # AD statistic and KS decision for 50 Rayleigh sample pairs, n = 12.
    rng = np.random.default_rng(1)
    n = 12
    sigma = reference.ad_sigma(n)
    a_s, b_s, ad, ks = [], [], [], []
    for _k in range(50):
        a, b = rng.rayleigh(size=n), rng.rayleigh(scale=1.5, size=n)
        a_s.append(a)
        b_s.append(b)
        ad.append(reference.ad_statistic(list(a), list(b), sigma))
        ks.append(reference.ks_accept(list(a), list(b), 0.05))
    np.savez_compressed(
        os.path.join(HERE, "statistics.npz"),
        a=np.array(a_s), b=np.array(b_s), ad=np.array(ad), ks=np.array(ks),
        ad_sigma=np.array([reference.ad_sigma(k) for k in range(3, 65)]),
        ad_critical=np.array([reference.ad_critical(al) for al in (0.001, 0.003, 0.01, 0.05, 0.1, 0.2, 0.25)]),
    )
    print("wrote statistics.npz")


if __name__ == "__main__":
    main()
