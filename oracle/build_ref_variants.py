"""Builds the reference kernel, specialised per configuration, for the timed
CPU baseline.

TEST INFRASTRUCTURE ONLY (bench.py's CPU legs, tests/): the product never
loads these libraries.

The reference's OpenCL backend compiles tcoh.cl once per run with every
configuration value as a -D constant (ocl.c:222-229: N, WA, WR, W, SHP_TEST,
EMI, BIAS, MIN_LOOKS, KS_MAX, AD_NORM, AD_SIGMA, AD_CRIT, TLOG_CRIT, NPAIRS,
PAIRS_ALL), so its private N x N arrays have a fixed size and its loops
constant trip counts. The generic oracle/_ref/libtcoh_ref*.so turn those
constants into run-time globals; the libraries built here are the faithful
form: the same tcoh.cl, compiled from the reference checkout where it lies
(never copied), with the same -D constants, one library per configuration
of the CPU baseline (the bench's workloads on crops of 512 output columns,
1024 at 60 dates).
oracle.run_reference picks the library of a strip's configuration when it
exists, else the generic one.

    python oracle/build_ref_variants.py --reference PATH_TO_REFERENCE
"""

import argparse
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import oracle  # noqa: E402

CFLAGS = ["-O3", "-fPIC", "-fopenmp", "-ffp-contract=off", "-fno-fast-math", "-std=gnu11"]

# (dates, window, output columns of the crop, test, alpha, estimator, bias,
#  min_shp, pair planes, all pairs): the bench's workloads.
VARIANTS = [
    (10, (21, 7), 512, "ks", 0.05, "evd", False, 10, 0, False),   # N=10 KS/EVD
    (30, (21, 7), 512, "ad", 0.05, "emi", True, 20, 0, False),    # the metric's: AD/EMI/-b
    (30, (21, 7), 512, "ad", 0.05, "evd", True, 20, 0, False),
    (30, (21, 7), 512, "tlog", 0.05, "evd", False, 20, 435, True),  # all pair planes
    (60, (21, 7), 1024, "ks", 0.05, "evd", False, 20, 0, False),  # N=60 KS, EVD and EMI
    (60, (21, 7), 1024, "ks", 0.05, "emi", False, 20, 0, False),  # (1024-column crops)
]


def defines(n, window, cols, test, alpha, estimator, bias, min_shp, npairs, pairs_all):
    """The -D options of ocl.c:222-229 for this configuration (float
    constants as "%.9e" literals with an f suffix, as ocl.c writes them)."""
    k = oracle.kernel_constants(n, test, alpha)
    wa, wr = window
    return [
        "-DN=%d" % n, "-DWA=%d" % wa, "-DWR=%d" % wr, "-DW=%d" % (cols + wr - 1),
        "-DSHP_TEST=%d" % oracle.TESTS[test], "-DEMI=%d" % int(estimator == "emi"),
        "-DBIAS=%d" % int(bias), "-DMIN_LOOKS=%d" % max(int(min_shp), n),
        "-DKS_MAX=%d" % k.ks_max, "-DAD_NORM=%.9ef" % k.ad_norm,
        "-DAD_SIGMA=%.9ef" % k.ad_sigma, "-DAD_CRIT=%.9ef" % k.ad_crit,
        "-DTLOG_CRIT=%.9ef" % k.tlog_crit, "-DNPAIRS=%d" % npairs,
        "-DPAIRS_ALL=%d" % int(pairs_all),
    ]


def build(reference, variant, out_dir):
    n, window, cols, test, alpha, estimator, bias, min_shp, npairs, pairs_all = variant
    name = oracle.ref_variant_name(n, window, cols + window[1] - 1, test, alpha, estimator, bias,
                                   min_shp, npairs, pairs_all)
    lib = os.path.join(out_dir, name)
    src = os.path.join(reference, "tcoh.cl")
    deps = [src, os.path.join(HERE, "ref_shim.h"), os.path.join(HERE, "ref_runner.c"),
            os.path.abspath(__file__)]
    if os.path.exists(lib) and all(os.path.getmtime(lib) >= os.path.getmtime(d) for d in deps):
        return lib
    d = ["-DTCOH_REF_SPECIALISED"] + defines(*variant)
    kobj, robj = lib[:-3] + "_kernel.o", lib[:-3] + "_runner.o"
    subprocess.run(["gcc"] + CFLAGS + ["-x", "c", "-include", os.path.join(HERE, "ref_shim.h")]
                   + d + ["-c", src, "-o", kobj], check=True)
    subprocess.run(["gcc"] + CFLAGS + d + ["-c", os.path.join(HERE, "ref_runner.c"), "-o", robj],
                   check=True)
    subprocess.run(["gcc"] + CFLAGS + ["-shared", "-o", lib, kobj, robj, "-lm"], check=True)
    os.remove(kobj)
    os.remove(robj)
    return lib


def main():
    p = argparse.ArgumentParser()
    p.add_argument("--reference", required=True,
                   help="directory of the reference checkout (holds tcoh.cl)")
    args = p.parse_args()
    out_dir = os.path.join(HERE, "_ref")
    os.makedirs(out_dir, exist_ok=True)
    for v in VARIANTS:
        build(args.reference, v, out_dir)


if __name__ == "__main__":
    main()
