"""B200 backend of i.sar.temporal_coherence: Python host side.

The product is libtcoh_b200.so (C-ABI in include/tcoh_b200.h, CUDA kernels
in csrc/). This module binds it with ctypes for hosts that are not the GRASS
module itself:

* ``ocl_list_devices``, ``ocl_open``, ``ocl_run``, ``ocl_close`` and the
  ``Settings`` structure mirror the module's backend interface
  (local_proto.h:34-49, 104-112; ocl.c) one to one;
* ``Backend`` is the same with return codes turned into exceptions, extra
  outputs (per-date phases, status) and device-resident strips;
* ``temporal_coherence`` runs the module's strip loop (main.c:724-825) over
  an in-memory stack, with its options (window=, shp_test=, alpha=,
  min_shp=, estimator=, -b, pairs=/pairs_mode=, memory=).

There is no CPU fallback: the library must be built (``make -C csrc``) and a
B200 (sm_100) GPU present, or the calls raise.
"""

import ctypes
import os

import numpy as np

from .strip import npairs_for, pair_list, read_strip, strip_rows_for

HERE = os.path.dirname(os.path.abspath(__file__))
LIBRARY = os.path.join(HERE, "libtcoh_b200.so")

SHP_TESTS = {"ks": 0, "ad": 1, "tlog": 2}
GRAM_TENSOR, GRAM_FP32 = 0, 1
STATUS_EMI_PINV, STATUS_UNLINKED, STATUS_ITER_CAP, STATUS_FP64, STATUS_EMI_PIVOTED = 1, 2, 4, 8, 16
STAGES = ("prep", "shp", "gram", "link", "copy", "adjoint", "exact")

# Exported symbols of include/tcoh_b200.h.
EXPORTS = (
    "ocl_list_devices", "ocl_open", "ocl_run", "ocl_close",
    "tc_last_error", "tc_set_fatal_handler", "tc_shp_constants", "tc_device_count",
    "tc_open", "tc_run_ex", "tc_run_device", "tc_set_timing", "tc_stage_stats",
    "tc_close", "tc_fp32_peak", "tc_fp64_peak", "tc_run_device_static", "tc_get_options",
    "tc_geometry_grid_shape", "tc_geometry_init", "tc_set_geometry", "tc_run_raw",
    "tc_run_raw_device", "tc_adjoint_raw",
)


class BackendError(RuntimeError):
    """A tc_* call failed; the message is tc_last_error()."""


class Settings(ctypes.Structure):
    """struct settings of local_proto.h:34-49."""

    _fields_ = [
        ("ndates", ctypes.c_int),
        ("win_az", ctypes.c_int),
        ("win_rg", ctypes.c_int),
        ("test", ctypes.c_int),
        ("alpha", ctypes.c_double),
        ("emi", ctypes.c_int),
        ("bias", ctypes.c_int),
        ("min_looks", ctypes.c_int),
        ("ks_max", ctypes.c_int),
        ("ad_norm", ctypes.c_double),
        ("ad_sigma", ctypes.c_double),
        ("ad_crit", ctypes.c_double),
        ("tlog_crit", ctypes.c_double),
        ("npairs", ctypes.c_int),
        ("pairs_all", ctypes.c_int),
        ("phase_reference", ctypes.c_char_p),
        ("orbit", ctypes.c_char_p),
    ]


class Options(ctypes.Structure):
    """struct tc_options."""

    _fields_ = [
        ("gram", ctypes.c_int),
        ("split_terms", ctypes.c_int),
        ("chunk_pixels", ctypes.c_int),
    ]


class Orbit(ctypes.Structure):
    """struct tc_orbit: one date's state vectors (orbit.c:52-57)."""

    _fields_ = [("n", ctypes.c_int), ("t", ctypes.c_void_p), ("pos", ctypes.c_void_p),
                ("vel", ctypes.c_void_p)]


class Geometry(ctypes.Structure):
    """struct tc_geometry: raster timing of the reference date and the
    region (geometry.c:161-216)."""

    _fields_ = [
        ("ndates", ctypes.c_int), ("ref", ctypes.c_int),
        ("first_line_time", ctypes.c_double), ("azimuth_time_interval", ctypes.c_double),
        ("slant_range_time", ctypes.c_double), ("range_sampling_rate", ctypes.c_double),
        ("wavelength", ctypes.c_double), ("line0", ctypes.c_double), ("sample0", ctypes.c_double),
        ("rows", ctypes.c_int), ("cols", ctypes.c_int),
        ("hmin", ctypes.c_double), ("hmax", ctypes.c_double), ("h0", ctypes.c_double),
    ]


def make_geometry(ndates, ref, rows, cols, first_line_time, azimuth_time_interval,
                  slant_range_time, range_sampling_rate, wavelength, line0=0.0, sample0=0.0,
                  heights=None, h0=0.0):
    """struct tc_geometry; the height range is that of `heights` (an
    elevation map, NaN ignored) or h0 (main.c:684-709)."""
    if heights is not None:
        h = np.asarray(heights, np.float64)
        hmin, hmax = float(np.nanmin(h)), float(np.nanmax(h))
    else:
        hmin = hmax = float(h0)
    return Geometry(ndates, ref, first_line_time, azimuth_time_interval, slant_range_time,
                    range_sampling_rate, wavelength, line0, sample0, rows, cols, hmin, hmax, h0)


def _orbit_array(orbits):
    keep, arr = [], (Orbit * len(orbits))()
    for k, (t, pos, vel) in enumerate(orbits):
        t = np.ascontiguousarray(t, np.float64)
        pos = np.ascontiguousarray(pos, np.float64)
        vel = np.ascontiguousarray(vel, np.float64)
        keep += [t, pos, vel]
        arr[k] = Orbit(len(t), t.ctypes.data, pos.ctypes.data, vel.ctypes.data)
    return arr, keep


def geometry_grid(geometry, orbits):
    """tc_geometry_init: the flat-earth / topographic phase grid
    [grid_rows][grid_cols][nheights][ndates] (float64), computed in double
    precision on the current device. orbits: per date (t, pos, vel)."""
    gr, gc, nh = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    hs = (ctypes.c_double * 3)()
    _check(library().tc_geometry_grid_shape(ctypes.byref(geometry), ctypes.byref(gr),
                                            ctypes.byref(gc), ctypes.byref(nh), hs))
    grid = np.empty((gr.value, gc.value, nh.value, geometry.ndates), np.float64)
    arr, keep = _orbit_array(orbits)
    _check(library().tc_geometry_init(ctypes.byref(geometry), arr, grid.ctypes.data))
    del keep
    return grid


_lib = None


def library():
    """The loaded libtcoh_b200.so (raises when it is not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIBRARY):
            raise OSError(
                "libtcoh_b200.so is not built: run make -C %s" % os.path.join(HERE, "csrc")
            )
        lib = ctypes.CDLL(LIBRARY)
        vp, i, sz = ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_size_t)
        lib.tc_last_error.restype = ctypes.c_char_p
        lib.tc_shp_constants.argtypes = [ctypes.POINTER(Settings)]
        lib.tc_device_count.restype = i
        lib.tc_open.argtypes = [i, ctypes.POINTER(Settings), i, ctypes.POINTER(Options),
                                ctypes.POINTER(vp), sz]
        lib.tc_run_ex.argtypes = [vp, vp, vp, vp, i, i, i, vp, vp, vp, vp, vp]
        lib.tc_run_device.argtypes = [vp, vp, vp, vp, i, i, i, vp, vp, vp, vp, vp, vp]
        lib.tc_set_timing.argtypes = [vp, i]
        lib.tc_stage_stats.argtypes = [vp, vp, vp, i]
        lib.tc_close.argtypes = [vp]
        lib.tc_get_options.argtypes = [vp, ctypes.POINTER(Options)]
        lib.tc_geometry_grid_shape.argtypes = [ctypes.POINTER(Geometry), vp, vp, vp, vp]
        lib.tc_geometry_init.argtypes = [ctypes.POINTER(Geometry), vp, vp]
        lib.tc_set_geometry.argtypes = [vp, ctypes.POINTER(Geometry), vp]
        lib.tc_run_raw.argtypes = [vp, vp, vp, vp, i, i, i, i, i, vp, vp, vp, vp, vp]
        lib.tc_run_raw_device.argtypes = [vp, vp, vp, vp, i, i, i, i, i, vp, vp, vp, vp, vp, vp]
        lib.tc_adjoint_raw.argtypes = [vp, vp, vp, vp, vp, vp, i, i, i, i, i, vp, vp, vp, vp]
        lib.tc_fp32_peak.argtypes = [i, ctypes.POINTER(ctypes.c_double)]
        lib.tc_fp64_peak.argtypes = [i, ctypes.POINTER(ctypes.c_double)]
        lib.tc_run_device_static.argtypes = [ctypes.POINTER(Settings), i, vp, vp, vp, i, i, i,
                                             vp, vp, vp, vp, vp, vp]
        lib.ocl_open.restype = vp
        lib.ocl_open.argtypes = [i, i, ctypes.POINTER(Settings), i, sz]
        lib.ocl_run.argtypes = [vp, vp, vp, vp, i, i, i, vp, vp, vp]
        lib.ocl_close.argtypes = [vp]
        for name in EXPORTS:
            getattr(lib, name)
        _lib = lib
    return _lib


def _check(rc):
    if rc != 0:
        raise BackendError(library().tc_last_error().decode(errors="replace"))


def _ptr(a):
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        return ctypes.c_void_p(a.data_ptr())
    return a.ctypes.data_as(ctypes.c_void_p)


def make_settings(n, window=(21, 7), shp_test="ks", alpha=0.05, min_shp=20,
                  estimator="evd", bias=False, pairs=False, pairs_all=False):
    """Settings as main.c:553-608 fills them, constants from stats.c."""
    if window[0] % 2 == 0 or window[1] % 2 == 0 or min(window) < 1:
        raise ValueError("Window sizes must be odd, got %d,%d" % tuple(window))
    if not 0 < alpha < 1:
        raise ValueError("Option alpha must be between 0 and 1")
    s = Settings()
    s.ndates = n
    s.win_az, s.win_rg = int(window[0]), int(window[1])
    s.test = SHP_TESTS[shp_test]
    s.alpha = alpha
    s.emi = int(estimator == "emi")
    s.bias = int(bool(bias))
    s.min_looks = max(int(min_shp), n)
    if s.win_az * s.win_rg < s.min_looks:
        raise ValueError(
            "The %dx%d window holds fewer pixels than the %d SHPs needed"
            % (s.win_az, s.win_rg, s.min_looks)
        )
    s.pairs_all = int(bool(pairs_all))
    s.npairs = npairs_for(n, pairs, pairs_all)
    s.phase_reference = b"none"
    s.orbit = None
    shp_constants(s)
    return s


def shp_constants(settings):
    """Fill ks_max, ad_* and tlog_crit (stats.c:61-95)."""
    _check(library().tc_shp_constants(ctypes.byref(settings)))
    return settings


def device_count():
    return library().tc_device_count()


def fp32_peak_tflops(device=0):
    """Measured FP32 FMA throughput (TFLOP/s) of the device."""
    v = ctypes.c_double(0.0)
    _check(library().tc_fp32_peak(device, ctypes.byref(v)))
    return v.value


def fp64_peak_tflops(device=0):
    """Measured FP64 FMA throughput (TFLOP/s) of the device."""
    v = ctypes.c_double(0.0)
    _check(library().tc_fp64_peak(device, ctypes.byref(v)))
    return v.value


# -- the reference interface (local_proto.h:104-112) -------------------------

def ocl_list_devices():
    library().ocl_list_devices()


def ocl_open(platform, device, settings, padded_cols):
    """Returns (handle, max_alloc); fatal errors end the process, as in the
    module."""
    m = ctypes.c_size_t(0)
    h = library().ocl_open(platform, device, ctypes.byref(settings), padded_cols, ctypes.byref(m))
    return h, m.value


def ocl_run(o, slc, amp, valid, padded_rows, rows, cols, coh, count, pairs):
    library().ocl_run(o, _ptr(slc), _ptr(amp), _ptr(valid), padded_rows, rows, cols,
                      _ptr(coh), _ptr(count), _ptr(pairs))


def ocl_close(o):
    library().ocl_close(o)


# -- extended interface ---------------------------------------------------------

def run_device_static(settings, padded_cols, slc, amp, valid, rows, cols, coh, count,
                      pairs=None, phases=None, status=None, stream=None):
    """tc_run_device_static: the path on device buffers the caller owns,
    without allocating device memory (see include/tcoh_b200.h). Arguments
    are CUDA tensors (or objects with data_ptr()); asynchronous on
    `stream` (a torch.cuda.Stream or raw handle; None is CUDA's default
    stream) on the current device."""
    if stream is not None and hasattr(stream, "cuda_stream"):
        stream = stream.cuda_stream
    _check(library().tc_run_device_static(
        ctypes.byref(settings), padded_cols, _ptr(slc), _ptr(amp), _ptr(valid), slc.shape[0],
        rows, cols, _ptr(coh), _ptr(count), _ptr(pairs), _ptr(phases), _ptr(status),
        ctypes.c_void_p(int(stream or 0)),
    ))

class Backend:
    """One device context for strips of a fixed width (tc_open)."""

    def __init__(self, settings, padded_cols, device=-1, gram=None, split_terms=3,
                 chunk_pixels=0):
        self.settings = settings
        self.n = settings.ndates
        self.padded_cols = padded_cols
        code = {None: -1, "fp32": GRAM_FP32, "tensor": GRAM_TENSOR}[gram]
        opt = Options(code, split_terms, chunk_pixels)
        h = ctypes.c_void_p()
        m = ctypes.c_size_t(0)
        _check(library().tc_open(device, ctypes.byref(settings), padded_cols, ctypes.byref(opt),
                                 ctypes.byref(h), ctypes.byref(m)))
        self.handle = h
        self.max_alloc = m.value
        _check(library().tc_get_options(h, ctypes.byref(opt)))
        self.gram = {GRAM_FP32: "fp32", GRAM_TENSOR: "tensor"}[opt.gram]
        self.split_terms = opt.split_terms

    def close(self):
        if self.handle:
            library().tc_close(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run(self, slc, amp, valid, rows, cols, phases=False, status=False, out=None):
        """One padded strip from host arrays; returns a dict of outputs
        (coh, count, and pairs / phases / status). `out` may hold
        preallocated (e.g. page-locked) output arrays under those keys."""
        slc = np.ascontiguousarray(slc, np.float32)
        amp = np.ascontiguousarray(amp, np.float32)
        valid = np.ascontiguousarray(valid, np.uint8)
        padded_rows = amp.shape[0]
        out = self._outputs(rows, cols, phases, status, out)
        _check(library().tc_run_ex(
            self.handle, _ptr(slc), _ptr(amp), _ptr(valid), padded_rows, rows, cols,
            _ptr(out["coh"]), _ptr(out["count"]), _ptr(out.get("pairs")),
            _ptr(out.get("phases")), _ptr(out.get("status")),
        ))
        return out

    def _outputs(self, rows, cols, phases, status, out):
        out = dict(out or {})
        out.setdefault("coh", np.empty((rows, cols), np.float32))
        out.setdefault("count", np.empty((rows, cols), np.int32))
        if self.settings.npairs:
            out.setdefault("pairs", np.empty((self.settings.npairs, rows, cols), np.float32))
        if phases:
            out.setdefault("phases", np.empty((rows, cols, self.n), np.float32))
        if status:
            out.setdefault("status", np.empty((rows, cols), np.uint8))
        return out

    def run_device(self, slc, amp, valid, rows, cols, coh, count, pairs=None, phases=None,
                   status=None, stream=None):
        """Device-resident strip: arguments are CUDA tensors (or objects
        with data_ptr()); asynchronous on `stream` (a torch.cuda.Stream or a
        raw cudaStream_t integer; None or 0 is CUDA's default stream)."""
        padded_rows = slc.shape[0]
        if stream is not None and hasattr(stream, "cuda_stream"):
            stream = stream.cuda_stream
        _check(library().tc_run_device(
            self.handle, _ptr(slc), _ptr(amp), _ptr(valid), padded_rows, rows, cols,
            _ptr(coh), _ptr(count), _ptr(pairs), _ptr(phases), _ptr(status),
            ctypes.c_void_p(int(stream or 0)),
        ))

    def set_timing(self, on):
        _check(library().tc_set_timing(self.handle, int(bool(on))))

    def stage_stats(self):
        """{stage: (device ms, launches)} of the last run with timing on."""
        k = len(STAGES)
        ms = (ctypes.c_float * k)()
        nl = (ctypes.c_int * k)()
        library().tc_stage_stats(self.handle, ms, nl, k)
        return {name: (ms[i], nl[i]) for i, name in enumerate(STAGES)}

    def set_geometry(self, geometry, grid):
        """tc_set_geometry: attach a phase grid (geometry_grid) for run_raw;
        None detaches it."""
        if grid is None:
            _check(library().tc_set_geometry(self.handle, None, None))
            self._grid = None
            return
        self._grid = np.ascontiguousarray(grid, np.float64)
        _check(library().tc_set_geometry(self.handle, ctypes.byref(geometry),
                                         self._grid.ctypes.data))

    def run_raw(self, re, im, elevation, row0, region_rows, rows, cols, phases=False,
                status=False, out=None):
        """tc_run_raw: one strip from raw I/Q rows re, im (N, padded_rows,
        cols) of region rows row0 .., elevation (padded_rows, cols) or None;
        the strip preparation (validity, sorted amplitudes, geometric phase)
        runs on the device. Returns the outputs as run() does."""
        re = np.ascontiguousarray(re, np.float32)
        im = np.ascontiguousarray(im, np.float32)
        elev = None if elevation is None else np.ascontiguousarray(elevation, np.float64)
        padded_rows = re.shape[1]
        out = self._outputs(rows, cols, phases, status, out)
        _check(library().tc_run_raw(
            self.handle, re.ctypes.data, im.ctypes.data, _ptr(elev), row0, region_rows,
            padded_rows, rows, cols, _ptr(out["coh"]), _ptr(out["count"]), _ptr(out.get("pairs")),
            _ptr(out.get("phases")), _ptr(out.get("status"))))
        return out

    def adjoint_raw(self, re, im, elevation, dh, psi, row0, region_rows, rows, cols, out=None):
        """tc_adjoint_raw: gamma of a raw strip (as run_raw) and the gradient
        of the sum of gamma over its estimated pixels with respect to a
        height error dh (padded_rows, cols) and a phase screen psi (N,
        padded_rows, cols) added to the removed phase (either None for
        zero). Returns a dict with coh, count, grad_dh and grad_psi; `out`
        may hold any of them as C-contiguous arrays of those shapes and types
        (for instance in page-locked memory, which the copies read and write
        at full speed)."""
        re = np.ascontiguousarray(re, np.float32)
        im = np.ascontiguousarray(im, np.float32)
        n, padded_rows, _ = re.shape
        elev = None if elevation is None else np.ascontiguousarray(elevation, np.float64)
        dh = None if dh is None else np.ascontiguousarray(dh, np.float64)
        psi = None if psi is None else np.ascontiguousarray(psi, np.float32)
        want = {"coh": ((rows, cols), np.float32), "count": ((rows, cols), np.int32),
                "grad_dh": ((padded_rows, cols), np.float32),
                "grad_psi": ((n, padded_rows, cols), np.float32)}
        out = dict(out or {})
        for name, (shape, dtype) in want.items():
            a = out.get(name)
            if a is None:
                out[name] = np.empty(shape, dtype)
            elif a.shape != shape or a.dtype != dtype or not a.flags.c_contiguous:
                raise ValueError("out[%r] must be a C-contiguous %s array of shape %s"
                                 % (name, np.dtype(dtype).name, shape))
        _check(library().tc_adjoint_raw(
            self.handle, re.ctypes.data, im.ctypes.data, _ptr(elev), _ptr(dh), _ptr(psi), row0,
            region_rows, padded_rows, rows, cols, _ptr(out["coh"]), _ptr(out["count"]),
            _ptr(out["grad_dh"]), _ptr(out["grad_psi"])))
        return out

    def run_raw_device(self, re, im, elevation, row0, region_rows, rows, cols, coh, count,
                       pairs=None, phases=None, status=None, stream=None):
        """tc_run_raw_device: run_raw on CUDA tensors, asynchronously."""
        if stream is not None and hasattr(stream, "cuda_stream"):
            stream = stream.cuda_stream
        _check(library().tc_run_raw_device(
            self.handle, _ptr(re), _ptr(im), _ptr(elevation), row0, region_rows, re.shape[1],
            rows, cols, _ptr(coh), _ptr(count), _ptr(pairs), _ptr(phases), _ptr(status),
            ctypes.c_void_p(int(stream or 0))))


def temporal_coherence(stack, window=(21, 7), shp_test="ks", alpha=0.05, min_shp=20,
                       estimator="evd", bias_correction=False, pairs=False,
                       pairs_mode="consecutive", phase=None, elevation=None, memory=300,
                       device=-1, gram=None, split_terms=3, with_phases=False,
                       with_status=False, backend=None, geometry=None, orbits=None):
    """Temporal coherence of a stack (N, rows, cols) complex, NaN = NULL, by
    the module's strip loop (main.c:724-825) over the B200 backend.

    phase: optional (N, rows, cols) geometric phase to remove (radians,
    date k is multiplied by exp(i phase_k)); elevation: optional (rows, cols)
    heights whose NaN cells are invalid. geometry (make_geometry) and orbits
    (per date (t, pos, vel)) instead of phase: the flat-earth / topographic
    phase is computed from the orbits (tc_geometry_init) and removed on the
    device at each cell's elevation (else geometry.h0), main.c:655-712.
    Returns (coh, count) with NaN / -1
    for NULL, plus pairs (npairs, rows, cols) when `pairs`, and phases /
    status arrays when asked, in a dict.
    """
    stack = np.asarray(stack)
    n, nrows, ncols = stack.shape
    pairs_all = pairs_mode == "all"
    s = make_settings(n, window, shp_test, alpha, min_shp, estimator, bias_correction,
                      pairs, pairs_all)
    halo_az, halo_rg = s.win_az // 2, s.win_rg // 2
    padded_cols = ncols + 2 * halo_rg
    own = backend is None
    be = backend or Backend(s, padded_cols, device=device, gram=gram, split_terms=split_terms)
    try:
        strip_rows = strip_rows_for(nrows, ncols, n, s.win_az, s.win_rg, s.npairs, memory,
                                    be.max_alloc)
        re = np.ascontiguousarray(stack.real, np.float32)
        im = np.ascontiguousarray(stack.imag, np.float32)
        coh = np.empty((nrows, ncols), np.float32)
        count = np.empty((nrows, ncols), np.int32)
        pl = np.empty((s.npairs, nrows, ncols), np.float32) if s.npairs else None
        ph = np.empty((nrows, ncols, n), np.float32) if with_phases else None
        stt = np.empty((nrows, ncols), np.uint8) if with_status else None
        raw = geometry is not None
        if raw:
            if phase is not None:
                raise ValueError("give either phase or geometry and orbits")
            be.set_geometry(geometry, geometry_grid(geometry, orbits))
            elev = None if elevation is None else np.asarray(elevation, np.float64)
        for row0 in range(0, nrows, strip_rows):
            rows = min(strip_rows, nrows - row0)
            padded_rows = rows + 2 * halo_az
            if raw:
                lo, hi = max(row0 - halo_az, 0), min(row0 - halo_az + padded_rows, nrows)
                rre = np.zeros((n, padded_rows, ncols), np.float32)
                rim = np.zeros((n, padded_rows, ncols), np.float32)
                off = lo - (row0 - halo_az)
                rre[:, off:off + hi - lo] = re[:, lo:hi]
                rim[:, off:off + hi - lo] = im[:, lo:hi]
                rel = None
                if elev is not None:
                    rel = np.zeros((padded_rows, ncols))
                    rel[off:off + hi - lo] = elev[lo:hi]
                r = be.run_raw(rre, rim, rel, row0 - halo_az, nrows, rows, ncols,
                               phases=with_phases, status=with_status)
            else:
                slc, amp, valid = read_strip(re, im, row0 - halo_az, padded_rows, halo_rg,
                                             phase=phase, elevation=elevation)
                r = be.run(slc, amp, valid, rows, ncols, phases=with_phases,
                           status=with_status)
            coh[row0:row0 + rows] = r["coh"]
            count[row0:row0 + rows] = r["count"]
            if s.npairs:
                pl[:, row0:row0 + rows] = r["pairs"]
            if with_phases:
                ph[row0:row0 + rows] = r["phases"]
            if with_status:
                stt[row0:row0 + rows] = r["status"]
    finally:
        if own:
            be.close()
    out = {"coh": coh, "count": count, "strip_rows": strip_rows}
    if s.npairs:
        out["pairs"] = pl
    if with_phases:
        out["phases"] = ph
    if with_status:
        out["status"] = stt
    return out
