"""ctypes bindings of the CPU checkers (test infrastructure only).

Imported by tests/, __graft_entry__.smoke() and bench.py's CPU baseline; the
product never imports this module.

    run_oracle(...)     double-precision restatement of tests/reference.py
                        (tcoh_oracle.c), optionally with the reference
                        kernel's float SHP statistics
    run_reference(...)  the reference kernel tcoh.cl itself, compiled as C
                        (oracle/_ref, built by oracle/Makefile from the
                        reference checkout; present only where it was built)
"""

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
TESTS = {"ks": 0, "ad": 1, "tlog": 2}


def build(reference_dir=None):
    """Compile liboracle.so, and oracle/_ref when the reference is present."""
    cmd = ["make", "-s", "-C", HERE]
    if reference_dir:
        cmd.append("REF=" + reference_dir)
    subprocess.run(cmd, check=True)


class _Settings(ctypes.Structure):
    _fields_ = [
        ("ndates", ctypes.c_int),
        ("win_az", ctypes.c_int),
        ("win_rg", ctypes.c_int),
        ("test", ctypes.c_int),
        ("alpha", ctypes.c_double),
        ("emi", ctypes.c_int),
        ("bias", ctypes.c_int),
        ("min_looks", ctypes.c_int),
        ("npairs", ctypes.c_int),
        ("pairs_all", ctypes.c_int),
        ("shp_fp32", ctypes.c_int),
    ]


class _KernelConstants(ctypes.Structure):
    _fields_ = [
        ("ks_max", ctypes.c_int),
        ("ad_norm", ctypes.c_float),
        ("ad_sigma", ctypes.c_float),
        ("ad_crit", ctypes.c_float),
        ("tlog_crit", ctypes.c_float),
    ]


_lib = None


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        _lib = ctypes.CDLL(path)
        _lib.orc_strip.restype = ctypes.c_int
        _lib.orc_ad_statistic.restype = ctypes.c_double
        _lib.orc_ad_sigma_of.restype = ctypes.c_double
        _lib.orc_ad_critical.restype = ctypes.c_double
        _lib.orc_normal_quantile.restype = ctypes.c_double
        _lib.orc_ad_critical.argtypes = [ctypes.c_double]
        _lib.orc_normal_quantile.argtypes = [ctypes.c_double]
    return _lib


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


def _settings(n, window, shp_test, alpha, estimator, bias, min_shp, npairs, pairs_all, shp_fp32):
    return _Settings(
        n, window[0], window[1], TESTS[shp_test], alpha, int(estimator == "emi"),
        int(bias), max(int(min_shp), n), npairs, int(pairs_all), int(shp_fp32),
    )


class _Orbit(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int), ("t", ctypes.c_void_p), ("pos", ctypes.c_void_p),
                ("vel", ctypes.c_void_p)]


class _Geometry(ctypes.Structure):
    _fields_ = [
        ("ndates", ctypes.c_int), ("ref", ctypes.c_int),
        ("first_line_time", ctypes.c_double), ("azimuth_time_interval", ctypes.c_double),
        ("slant_range_time", ctypes.c_double), ("range_sampling_rate", ctypes.c_double),
        ("wavelength", ctypes.c_double), ("line0", ctypes.c_double), ("sample0", ctypes.c_double),
        ("rows", ctypes.c_int), ("cols", ctypes.c_int),
        ("hmin", ctypes.c_double), ("hmax", ctypes.c_double), ("h0", ctypes.c_double),
    ]


def _geometry(geo):
    """geo: dict with the fields of orc_geometry."""
    return _Geometry(*(geo[name] for name, _ in _Geometry._fields_))


def _orbits(orbits):
    """orbits: list of (t [n], pos [n][3], vel [n][3]); returns the ctypes
    array and the arrays it points into (kept alive by the caller)."""
    keep = []
    arr = (_Orbit * len(orbits))()
    for k, (t, pos, vel) in enumerate(orbits):
        t = np.ascontiguousarray(t, np.float64)
        pos = np.ascontiguousarray(pos, np.float64)
        vel = np.ascontiguousarray(vel, np.float64)
        keep += [t, pos, vel]
        arr[k] = _Orbit(len(t), t.ctypes.data, pos.ctypes.data, vel.ctypes.data)
    return arr, keep


def geometry_shape(geo):
    """(grid_rows, grid_cols, nheights, heights[3]) of geometry.c:201-216."""
    gr, gc, nh = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    hs = np.zeros(3)
    g = _geometry(geo)
    lib().orc_geometry_shape(ctypes.byref(g), ctypes.byref(gr), ctypes.byref(gc),
                             ctypes.byref(nh), _ptr(hs))
    return gr.value, gc.value, nh.value, hs


def geometry_grid(geo, orbits):
    """The coarse phase grid [grid_rows][grid_cols][nheights][ndates]
    (geometry.c:161-254), FP64; raises if a point cannot be located."""
    gr, gc, nh, _ = geometry_shape(geo)
    grid = np.zeros((gr, gc, nh, geo["ndates"]))
    arr, keep = _orbits(orbits)
    g = _geometry(geo)
    rc = lib().orc_geometry_grid(ctypes.byref(g), arr, _ptr(grid))
    if rc != 0:
        raise ValueError("geometry grid failed (%d)" % rc)
    return grid


def geometry_phases(geo, grid, heights):
    """Interpolated phase (ndates, rows, cols) at every region cell and its
    height (geometry.c:256-291)."""
    grid = np.ascontiguousarray(grid, np.float64)
    heights = np.asarray(heights, np.float64)
    rows, cols = heights.shape
    g = _geometry(geo)
    out = np.zeros((geo["ndates"], rows, cols))
    ph = np.zeros(geo["ndates"])
    for r in range(rows):
        for c in range(cols):
            lib().orc_geometry_phases(ctypes.byref(g), _ptr(grid), r, c,
                                      ctypes.c_double(heights[r, c]), _ptr(ph))
            out[:, r, c] = ph
    return out


def prepare_strip(re, im, elevation, row0, region_rows, halo_cols, geo=None, grid=None):
    """main.c:52-127 on raw I/Q planes re, im (ndates, padded_rows, cols) of
    region rows row0 ..; returns (slc, amp, valid) of the padded strip."""
    re = np.ascontiguousarray(re, np.float32)
    im = np.ascontiguousarray(im, np.float32)
    n, prow, cols = re.shape
    w = cols + 2 * halo_cols
    slc = np.empty((prow, w, n, 2), np.float32)
    amp = np.empty((prow, w, n), np.float32)
    valid = np.empty((prow, w), np.uint8)
    elev = None if elevation is None else np.ascontiguousarray(elevation, np.float64)
    g = None if geo is None else ctypes.byref(_geometry(geo))
    grid = None if grid is None else np.ascontiguousarray(grid, np.float64)
    lib().orc_prepare_strip(n, _ptr(re), _ptr(im), _ptr(elev), row0, region_rows, prow, cols,
                            halo_cols, g, _ptr(grid), _ptr(slc), _ptr(amp), _ptr(valid))
    return slc, amp, valid


def kernel_constants(n, shp_test="ks", alpha=0.05):
    """The float constants that the reference kernel is built with."""
    s = _settings(n, (21, 7), shp_test, alpha, "evd", False, n, 0, False, True)
    k = _KernelConstants()
    lib().orc_kernel_constants_for(ctypes.byref(s), ctypes.byref(k))
    return k


def run_oracle(slc, amp, valid, rows, cols, window=(21, 7), shp_test="ks", alpha=0.05,
               min_shp=20, estimator="evd", bias=False, npairs=0, pairs_all=False,
               shp_fp32=False, want_phases=False, want_mask=False, threads=0):
    """Oracle over a padded strip (layouts of ocl_run). Returns a dict with
    coh (float64), count (int32), and pairs / phases / mask when asked."""
    slc = np.ascontiguousarray(slc, np.float32)
    amp = np.ascontiguousarray(amp, np.float32)
    valid = np.ascontiguousarray(valid, np.uint8)
    prow, pcol, n = amp.shape
    s = _settings(n, window, shp_test, alpha, estimator, bias, min_shp, npairs, pairs_all, shp_fp32)
    coh = np.empty((rows, cols), np.float64)
    count = np.empty((rows, cols), np.int32)
    pairs = np.empty((npairs, rows, cols), np.float64) if npairs else None
    phases = np.empty((rows, cols, n), np.float64) if want_phases else None
    words = (window[0] * window[1] + 31) // 32
    mask = np.empty((rows, cols, words), np.uint32) if want_mask else None
    rc = lib().orc_strip(
        ctypes.byref(s), _ptr(slc), _ptr(amp), _ptr(valid), prow, pcol, rows, cols,
        _ptr(coh), _ptr(count), _ptr(pairs), _ptr(phases), _ptr(mask), int(threads),
    )
    if rc != 0:
        raise ValueError("oracle rejected the strip shape or settings")
    out = {"coh": coh, "count": count}
    if npairs:
        out["pairs"] = pairs
    if want_phases:
        out["phases"] = phases
    if want_mask:
        out["mask"] = mask
    return out


def ad_statistic(a, b):
    a = np.ascontiguousarray(a, np.float32)
    b = np.ascontiguousarray(b, np.float32)
    return lib().orc_ad_statistic(_ptr(a), _ptr(b), len(a))


def ks_accept(a, b, alpha):
    a = np.ascontiguousarray(a, np.float32)
    b = np.ascontiguousarray(b, np.float32)
    return bool(lib().orc_ks_accept(_ptr(a), _ptr(b), len(a), ctypes.c_double(alpha)))


def ad_sigma(n):
    return lib().orc_ad_sigma_of(n)


def ad_critical(alpha):
    return lib().orc_ad_critical(alpha)


def hermitian_eigen(m):
    """Eigenvalues and eigenvectors of a Hermitian matrix by the oracle's
    double-precision Jacobi solver (unsorted)."""
    m = np.asarray(m, np.complex128)
    n = m.shape[0]
    ar = np.ascontiguousarray(m.real)
    ai = np.ascontiguousarray(m.imag)
    vr = np.zeros((n, n))
    vi = np.zeros((n, n))
    lib().orc_hermitian_eigen(n, _ptr(ar), _ptr(ai), _ptr(vr), _ptr(vi))
    return np.diag(ar).copy(), vr + 1j * vi


# ---------------------------------------------------------------------------
# The reference kernel compiled as C.

_ref = {}


def reference_available():
    return os.path.exists(os.path.join(HERE, "_ref", "libtcoh_ref.so"))


def ref_variant_name(n, window, padded_cols, shp_test, alpha, estimator, bias, min_shp,
                     npairs, pairs_all):
    """File name of the reference kernel built for one configuration with its
    -D constants (oracle/build_ref_variants.py)."""
    return "libtcoh_ref_n%d_%dx%d_W%d_%s_a%g_%s_b%d_m%d_p%d%s.so" % (
        n, window[0], window[1], padded_cols, shp_test, alpha, estimator, int(bias),
        max(int(min_shp), n), npairs, "all" if pairs_all else "")


def ref_build(n, window, padded_cols, shp_test, alpha, estimator, bias, min_shp, npairs,
              pairs_all):
    """"specialised" when the reference kernel built for this configuration
    exists (it is the one run_reference then runs), else "generic"."""
    name = ref_variant_name(n, window, padded_cols, shp_test, alpha, estimator, bias, min_shp,
                            npairs, pairs_all)
    return "specialised" if os.path.exists(os.path.join(HERE, "_ref", name)) else "generic"


def _ref_lib(pairs, variant=None):
    name = "libtcoh_ref_pairs.so" if pairs else "libtcoh_ref.so"
    if variant and os.path.exists(os.path.join(HERE, "_ref", variant)):
        name = variant
    if name not in _ref:
        path = os.path.join(HERE, "_ref", name)
        if not os.path.exists(path):
            raise FileNotFoundError(path + " (build with: make -C oracle REF=<reference>)")
        lib_ = ctypes.CDLL(path)
        lib_.ref_run.restype = ctypes.c_int
        lib_.ref_run.argtypes = [ctypes.c_int] * 8 + [ctypes.c_float] * 4 + [ctypes.c_int] + [
            ctypes.c_void_p] * 3 + [ctypes.c_int] * 4 + [ctypes.c_void_p] * 3 + [ctypes.c_int]
        lib_.ref_threads.restype = ctypes.c_int
        _ref[name] = lib_
    return _ref[name]


def reference_threads():
    return _ref_lib(False).ref_threads()


def run_reference(slc, amp, valid, rows, cols, window=(21, 7), shp_test="ks", alpha=0.05,
                  min_shp=20, estimator="evd", bias=False, npairs=0, pairs_all=False,
                  threads=0):
    """The reference kernel (tcoh.cl compiled as C) over a padded strip: the
    build specialised for this configuration (its -D constants compiled in,
    as ocl.c:222-229 builds it) when one exists, else the generic build."""
    slc = np.ascontiguousarray(slc, np.float32)
    amp = np.ascontiguousarray(amp, np.float32)
    valid = np.ascontiguousarray(valid, np.uint8)
    prow, pcol, n = amp.shape
    k = kernel_constants(n, shp_test, alpha)
    coh = np.empty((rows, cols), np.float32)
    count = np.empty((rows, cols), np.int32)
    pairs = np.empty((max(npairs, 1), rows, cols), np.float32)
    variant = ref_variant_name(n, window, pcol, shp_test, alpha, estimator, bias, min_shp,
                               npairs, pairs_all)
    rc = _ref_lib(npairs > 0, variant).ref_run(
        n, window[0], window[1], TESTS[shp_test], int(estimator == "emi"), int(bias),
        max(int(min_shp), n), k.ks_max, k.ad_norm, k.ad_sigma, k.ad_crit, k.tlog_crit,
        int(pairs_all), _ptr(slc), _ptr(amp), _ptr(valid), prow, pcol, rows, cols,
        _ptr(coh), _ptr(count), _ptr(pairs), int(threads),
    )
    if rc != 0:
        raise ValueError("reference runner rejected the strip shape")
    out = {"coh": coh, "count": count}
    if npairs:
        out["pairs"] = pairs
    return out
