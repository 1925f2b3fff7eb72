"""Python bindings (ctypes) of libbbkde.so, the B200 direct kernel-density library.

The product is the C ABI in include/bbkde.h and the C++ drop-in headers in
include/bbkde/; this module only binds the C ABI so that tests and bench.py can
drive it. There is no CPU fallback: if the CUDA library is missing or no device
is present, every call raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "lib", "libbbkde.so")

# Status codes (bbkde_status).
OK, OUT_OF_RANGE, INVALID_ARGUMENT, CUDA_ERROR, TIMEOUT, UNSUPPORTED, NO_DEVICE, \
    ALLOC_FAILED = range(8)

# Kernel kinds (bbkde_kernel_kind).
GAUSSIAN, EPANECHNIKOV, GAUSSIAN_PRODUCT_2D, EPANECHNIKOV_PRODUCT_2D, \
    GAUSSIAN_PRODUCT_CONV_2D, EPANECHNIKOV_PRODUCT_CONV_2D, GAUSSIAN_CONV_1D, \
    EPANECHNIKOV_CONV_1D = range(8)

FP32C, FP64 = 0, 1
REFERENCE, QUERY = 0, 1
FLAG_EXACT_GAUSS_CONV = 1

# Every symbol include/bbkde.h declares.
EXPORTED = [
    "bbkde_abi_version", "bbkde_status_string", "bbkde_ctx_create", "bbkde_ctx_destroy",
    "bbkde_ctx_last_error", "bbkde_ctx_set_stream", "bbkde_upload", "bbkde_size",
    "bbkde_download_attributes", "bbkde_eval_range", "bbkde_eval_range_device",
    "bbkde_adapt_density", "bbkde_unadapt_density", "bbkde_likelihood_cv",
    "bbkde_lsq_conv_cv", "bbkde_last_launch_stats", "bbkde_launch_count",
    "bbkde_device_info", "bbkde_ctx_set_launch_variant", "bbkde_launch_variants",
    "bbkde_eval_noalloc", "bbkde_cv_batch", "bbkde_surrogate_create", "bbkde_surrogate_destroy",
    "bbkde_surrogate_last_error", "bbkde_surrogate_num_params", "bbkde_surrogate_set_params",
    "bbkde_surrogate_get_params", "bbkde_surrogate_gradient", "bbkde_surrogate_train",
    "bbkde_surrogate_predict", "bbkde_surrogate_predict_device", "bbkde_surrogate_save",
    "bbkde_surrogate_load", "bbkde_surrogate_set_inference", "bbkde_eval_culled",
    "bbkde_eval_grid", "bbkde_lsq_numint_cv", "bbkde_surrogate_set_engine",
    "bbkde_adapt_density_tol", "bbkde_likelihood_cv_tol", "bbkde_lsq_conv_cv_tol",
    "bbkde_eval_tol", "bbkde_cv_batch_info", "bbkde_ctx_set_cv_plan",
]

# Surrogate inference engines (bbkde_surrogate_set_engine).
ENGINE_TCGEN05, ENGINE_MMA_SYNC = 0, 1

# Dense-grid modes (bbkde_grid_config.mode).
GRID_EXACT, GRID_SURROGATE, GRID_ANCHORED = 0, 1, 2
# Where the network runs in anchored mode (bbkde_grid_config.net_scope).
NET_RESCUE, NET_EVERYWHERE = 0, 1


class Dataset(C.Structure):
    _fields_ = [("n", C.c_int64), ("coords", C.POINTER(C.c_double)),
                ("weights", C.POINTER(C.c_double))]


class TrainConfig(C.Structure):
    _fields_ = [("steps", C.c_int64), ("batch", C.c_int64), ("lr", C.c_double),
                ("lr_final", C.c_double), ("beta1", C.c_double), ("beta2", C.c_double),
                ("eps", C.c_double), ("seed", C.c_uint64)]


class CullStats(C.Structure):
    _fields_ = [("kernel_ms", C.c_double), ("pairs", C.c_double), ("full_pairs", C.c_double),
                ("max_bound_ratio", C.c_double)]


class Grid(C.Structure):
    _fields_ = [("nx", C.c_int64), ("ny", C.c_int64), ("x0", C.c_double), ("x1", C.c_double),
                ("y0", C.c_double), ("y1", C.c_double)]


class GridConfig(C.Structure):
    _fields_ = [("mode", C.c_int), ("tile", C.c_int), ("probes", C.c_int),
                ("exact_culled", C.c_int), ("rel_tol", C.c_double), ("low_frac", C.c_double),
                ("cull_rel", C.c_double), ("interp", C.c_int), ("pair_form", C.c_int),
                ("net_scope", C.c_int), ("lattice_tile", C.c_int), ("tensor_cores", C.c_int)]


class GridStats(C.Structure):
    _fields_ = [("tiles", C.c_int64), ("tiles_low", C.c_int64), ("tiles_flagged", C.c_int64),
                ("tiles_surrogate", C.c_int64), ("exact_points", C.c_int64),
                ("pairs", C.c_double), ("max_probe_err", C.c_double),
                ("max_bound_ratio", C.c_double), ("ms_total", C.c_double),
                ("ms_predict", C.c_double), ("ms_probe", C.c_double),
                ("ms_fallback", C.c_double), ("probes_used", C.c_int64),
                ("lattice_tile_used", C.c_int64)]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class KernelDesc(C.Structure):
    _fields_ = [("kind", C.c_int32), ("dim", C.c_int32), ("h", C.c_double * 2),
                ("flags", C.c_int32), ("reserved", C.c_int32)]


def kernel_desc(kind: int, dim: int, h, flags: int = 0) -> KernelDesc:
    h = list(h) if hasattr(h, "__len__") else [h]
    if len(h) == 1:
        h = h * 2
    return KernelDesc(kind, dim, (C.c_double * 2)(*h[:2]), flags, 0)


class BBKDEError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"[{status}] {msg}")
        self.status = status


class OutOfRange(BBKDEError, IndexError):
    pass


class InvalidArgument(BBKDEError, ValueError):
    pass


_dp = C.POINTER(C.c_double)
_lib = None


def _ensure_built():
    if not os.path.exists(LIB_PATH):
        from . import build
        build.build()


def load_library(path: str = LIB_PATH):
    """Load libbbkde.so (building it first if absent) and declare its signatures."""
    global _lib
    if _lib is not None:
        return _lib
    if path == LIB_PATH:
        _ensure_built()
    if not os.path.exists(path):
        raise RuntimeError(f"libbbkde.so not found at {path}; run python -m bbrcit_kde_b200.build")
    lib = C.CDLL(path)
    vp = C.c_void_p
    i64 = C.c_int64
    lib.bbkde_abi_version.restype = C.c_int
    lib.bbkde_status_string.restype = C.c_char_p
    lib.bbkde_status_string.argtypes = [C.c_int]
    lib.bbkde_ctx_create.argtypes = [C.c_int, C.POINTER(vp)]
    lib.bbkde_ctx_destroy.argtypes = [vp]
    lib.bbkde_ctx_last_error.restype = C.c_char_p
    lib.bbkde_ctx_last_error.argtypes = [vp]
    lib.bbkde_ctx_set_stream.argtypes = [vp, vp]
    lib.bbkde_upload.argtypes = [vp, C.c_int, C.c_int, i64, _dp, _dp, _dp, _dp]
    lib.bbkde_size.restype = i64
    lib.bbkde_size.argtypes = [vp, C.c_int]
    lib.bbkde_download_attributes.argtypes = [vp, _dp, _dp]
    kd = C.POINTER(KernelDesc)
    lib.bbkde_eval_range.argtypes = [vp, kd, i64, i64, i64, i64, C.c_int, C.c_int, _dp, i64]
    lib.bbkde_eval_range_device.argtypes = [vp, kd, i64, i64, i64, i64, C.c_int, C.c_int, vp,
                                            i64]
    lib.bbkde_adapt_density.argtypes = [vp, kd, C.c_double, C.c_int, _dp, _dp, _dp, _dp]
    lib.bbkde_adapt_density_tol.argtypes = [vp, kd, C.c_double, C.c_double, C.c_double, _dp,
                                            _dp, _dp, _dp]
    lib.bbkde_likelihood_cv_tol.argtypes = [vp, kd, C.c_double, C.c_double, _dp]
    lib.bbkde_lsq_conv_cv_tol.argtypes = [vp, kd, C.c_double, C.c_double, _dp]
    lib.bbkde_unadapt_density.argtypes = [vp]
    lib.bbkde_likelihood_cv.argtypes = [vp, kd, C.c_int, _dp]
    lib.bbkde_lsq_conv_cv.argtypes = [vp, kd, C.c_int, _dp]
    lib.bbkde_last_launch_stats.argtypes = [vp, _dp, _dp, C.POINTER(i64)]
    lib.bbkde_launch_count.restype = i64
    lib.bbkde_launch_count.argtypes = [vp]
    lib.bbkde_ctx_set_launch_variant.argtypes = [vp, C.c_int]
    lib.bbkde_launch_variants.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    lib.bbkde_device_info.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    lib.bbkde_cv_batch.argtypes = [vp, C.c_int, C.c_int, C.POINTER(Dataset), C.c_int, _dp,
                                   C.c_int, _dp, C.c_int, _dp, _dp]
    fp = C.POINTER(C.c_float)
    lib.bbkde_surrogate_create.argtypes = [C.c_int, C.c_uint64, C.POINTER(vp)]
    lib.bbkde_surrogate_destroy.argtypes = [vp]
    lib.bbkde_surrogate_last_error.restype = C.c_char_p
    lib.bbkde_surrogate_last_error.argtypes = [vp]
    lib.bbkde_surrogate_num_params.restype = C.c_int
    lib.bbkde_surrogate_set_params.argtypes = [vp, fp, fp]
    lib.bbkde_surrogate_get_params.argtypes = [vp, fp, fp]
    lib.bbkde_surrogate_gradient.argtypes = [vp, i64, _dp, _dp, fp, _dp]
    lib.bbkde_surrogate_train.argtypes = [vp, i64, _dp, _dp, C.POINTER(TrainConfig), _dp]
    lib.bbkde_surrogate_predict.argtypes = [vp, i64, _dp, _dp]
    lib.bbkde_surrogate_predict_device.argtypes = [vp, i64, vp, vp]
    lib.bbkde_surrogate_save.argtypes = [vp, C.c_char_p]
    lib.bbkde_surrogate_load.argtypes = [vp, C.c_char_p]
    lib.bbkde_eval_noalloc.argtypes = [kd, i64, vp, vp, vp, vp, i64, vp, vp, C.c_int, vp, vp,
                                       C.c_char_p, i64]
    lib.bbkde_surrogate_set_inference.argtypes = [vp, C.c_int]
    lib.bbkde_surrogate_set_engine.argtypes = [vp, C.c_int]
    lib.bbkde_eval_culled.argtypes = [vp, kd, C.c_int, C.c_double, vp, C.c_int,
                                      C.POINTER(CullStats)]
    lib.bbkde_cv_batch_info.argtypes = [vp, C.POINTER(C.c_int64), C.POINTER(C.c_int64),
                                        C.POINTER(C.c_int), C.POINTER(C.c_int)]
    lib.bbkde_ctx_set_cv_plan.argtypes = [vp, C.c_int]
    lib.bbkde_eval_tol.argtypes = [vp, kd, C.c_int, C.c_double, C.c_double, vp, C.c_int,
                                   C.POINTER(CullStats)]
    lib.bbkde_eval_grid.argtypes = [vp, vp, kd, C.POINTER(Grid), C.POINTER(GridConfig), vp,
                                    C.POINTER(GridStats)]
    lib.bbkde_lsq_numint_cv.argtypes = [vp, kd, C.POINTER(Grid), C.c_int, _dp]
    _lib = lib
    return lib


def _p(a):
    return None if a is None else a.ctypes.data_as(_dp)


def _c(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float64)


class Context:
    """One bbkde_ctx (device buffers + stream) on one CUDA device."""

    def __init__(self, device: int = 0):
        self.lib = load_library()
        h = C.c_void_p()
        rc = self.lib.bbkde_ctx_create(device, C.byref(h))
        if rc != OK:
            raise BBKDEError(rc, "bbkde_ctx_create failed: " +
                             self.lib.bbkde_status_string(rc).decode())
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.lib.bbkde_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, rc: int):
        if rc == OK:
            return
        msg = (self.lib.bbkde_ctx_last_error(self.h) or b"").decode()
        if rc == OUT_OF_RANGE:
            raise OutOfRange(rc, msg)
        if rc == INVALID_ARGUMENT:
            raise InvalidArgument(rc, msg)
        raise BBKDEError(rc, msg)

    def set_stream(self, stream_ptr: int | None):
        self._check(self.lib.bbkde_ctx_set_stream(self.h, stream_ptr))

    def upload(self, role: int, coords, mass=None, abw=None, weight=None):
        coords = _c(coords)
        if coords.ndim == 1:
            coords = coords.reshape(-1, 1)
        n, dim = coords.shape
        mass, abw, weight = _c(mass), _c(abw), _c(weight)
        self._check(self.lib.bbkde_upload(self.h, role, dim, n, _p(coords), _p(mass), _p(abw),
                                          _p(weight)))

    def size(self, role: int) -> int:
        return int(self.lib.bbkde_size(self.h, role))

    def download_attributes(self):
        n = self.size(REFERENCE)
        mass, abw = np.empty(n), np.empty(n)
        self._check(self.lib.bbkde_download_attributes(self.h, _p(mass), _p(abw)))
        return mass, abw

    def eval_range(self, desc: KernelDesc, r_i, r_j, q_i, q_j, normalized=True,
                   precision=FP32C, block_size=0, out=None):
        n = q_j - q_i + 1 if q_j >= q_i else 0
        if out is None:
            out = np.empty(max(n, 1))
        self._check(self.lib.bbkde_eval_range(self.h, C.byref(desc), r_i, r_j, q_i, q_j,
                                              int(normalized), precision, _p(out), block_size))
        return out[:n]

    def eval_range_device(self, desc: KernelDesc, r_i, r_j, q_i, q_j, out_ptr: int,
                          normalized=True, precision=FP32C, block_size=0):
        self._check(self.lib.bbkde_eval_range_device(self.h, C.byref(desc), r_i, r_j, q_i, q_j,
                                                     int(normalized), precision, out_ptr,
                                                     block_size))

    def eval_all(self, desc: KernelDesc, normalized=True, precision=FP32C):
        nr, nq = self.size(REFERENCE), self.size(QUERY)
        return self.eval_range(desc, 0, nr - 1, 0, nq - 1, normalized, precision)

    def adapt_density(self, desc: KernelDesc, alpha: float, precision=FP32C, outputs=True):
        """Returns (abw, mass, pilot, g); with outputs=False nothing is copied to the
        host and the adapted attributes only live on the device."""
        if not outputs:
            self._check(self.lib.bbkde_adapt_density(self.h, C.byref(desc), alpha, precision,
                                                     None, None, None, None))
            return None
        n = self.size(REFERENCE)
        abw, mass, pilot, g = np.empty(max(n, 1)), np.empty(max(n, 1)), np.empty(max(n, 1)), \
            np.zeros(1)
        self._check(self.lib.bbkde_adapt_density(self.h, C.byref(desc), alpha, precision,
                                                 _p(abw), _p(mass), _p(pilot), _p(g)))
        return abw[:n], mass[:n], pilot[:n], float(g[0])

    def adapt_density_tol(self, desc: KernelDesc, alpha: float, rel_tol=1e-6, abs_tol=0.0,
                          outputs=True):
        """adapt_density with the pilot to max(rel_tol f, abs_tol) (culled self-sum);
        same returns."""
        if not outputs:
            self._check(self.lib.bbkde_adapt_density_tol(self.h, C.byref(desc), alpha, rel_tol,
                                                         abs_tol, None, None, None, None))
            return None
        n = self.size(REFERENCE)
        abw, mass, pilot, g = np.empty(max(n, 1)), np.empty(max(n, 1)), np.empty(max(n, 1)), \
            np.zeros(1)
        self._check(self.lib.bbkde_adapt_density_tol(self.h, C.byref(desc), alpha, rel_tol,
                                                     abs_tol, _p(abw), _p(mass), _p(pilot),
                                                     _p(g)))
        return abw[:n], mass[:n], pilot[:n], float(g[0])

    def unadapt_density(self):
        self._check(self.lib.bbkde_unadapt_density(self.h))

    def likelihood_cv(self, desc: KernelDesc, precision=FP32C) -> float:
        cv = np.zeros(1)
        self._check(self.lib.bbkde_likelihood_cv(self.h, C.byref(desc), precision, _p(cv)))
        return float(cv[0])

    def likelihood_cv_tol(self, desc: KernelDesc, rel_tol=1e-6, abs_tol=0.0) -> float:
        """Likelihood CV with the density sums to max(rel_tol f, abs_tol) (culled)."""
        cv = np.zeros(1)
        self._check(self.lib.bbkde_likelihood_cv_tol(self.h, C.byref(desc), rel_tol, abs_tol,
                                                     _p(cv)))
        return float(cv[0])

    def lsq_conv_cv_tol(self, desc: KernelDesc, rel_tol=1e-6, abs_tol=0.0) -> float:
        """LSQ convolution CV with the density sums to max(rel_tol f, abs_tol) (culled)."""
        cv = np.zeros(1)
        self._check(self.lib.bbkde_lsq_conv_cv_tol(self.h, C.byref(desc), rel_tol, abs_tol,
                                                   _p(cv)))
        return float(cv[0])

    def lsq_conv_cv(self, desc: KernelDesc, precision=FP32C) -> float:
        cv = np.zeros(1)
        self._check(self.lib.bbkde_lsq_conv_cv(self.h, C.byref(desc), precision, _p(cv)))
        return float(cv[0])

    def last_launch_stats(self):
        ms, pairs, launches = C.c_double(), C.c_double(), C.c_int64()
        self._check(self.lib.bbkde_last_launch_stats(self.h, C.byref(ms), C.byref(pairs),
                                                     C.byref(launches)))
        return ms.value, pairs.value, launches.value

    def launch_count(self) -> int:
        return int(self.lib.bbkde_launch_count(self.h))

    def cv_batch(self, kind: int, datasets, hx, hy, precision=FP64):
        """Likelihood and LSQ-convolution CV of every dataset over the hx x hy grid.

        datasets: list of (coords (n, 2), weights or None). Returns (lik, lsq) with
        shape (n_sets, len(hx), len(hy))."""
        keep = []
        arr = (Dataset * max(len(datasets), 1))()
        for i, (xy, w) in enumerate(datasets):
            xy = _c(xy).reshape(-1, 2)
            w = _c(w)
            keep += [xy, w]
            arr[i].n = xy.shape[0]
            arr[i].coords = _p(xy)
            arr[i].weights = _p(w) if w is not None else None
        hx, hy = _c(hx), _c(hy)
        n = len(datasets)
        lik = np.empty((max(n, 1), len(hx), len(hy)))
        lsq = np.empty_like(lik)
        self._check(self.lib.bbkde_cv_batch(self.h, kind, n, arr, len(hx), _p(hx), len(hy),
                                            _p(hy), precision, _p(lik), _p(lsq)))
        return lik[:n], lsq[:n]

    def cv_batch_info(self):
        """(likelihood pairs, convolution pairs in support, plan, number of plans) of
        the last cv_batch."""
        a, b, p, n = C.c_int64(0), C.c_int64(0), C.c_int(0), C.c_int(0)
        self._check(self.lib.bbkde_cv_batch_info(self.h, C.byref(a), C.byref(b), C.byref(p),
                                                 C.byref(n)))
        return a.value, b.value, p.value, n.value

    def set_cv_plan(self, plan: int):
        """Force a batched-CV work-item plan (-1: autotune)."""
        self._check(self.lib.bbkde_ctx_set_cv_plan(self.h, plan))

    def eval_culled(self, desc: KernelDesc, rel_tol=1e-7, normalized=True):
        """Culled direct evaluation of every query; returns (values, CullStats)."""
        n = self.size(QUERY)
        out = np.empty(max(n, 1))
        st = CullStats()
        self._check(self.lib.bbkde_eval_culled(self.h, C.byref(desc), int(normalized), rel_tol,
                                               out.ctypes.data, 0, C.byref(st)))
        return out[:n], st

    def eval_tol(self, desc: KernelDesc, rel_err=1e-6, abs_err=1e-8, normalized=True):
        """bbkde_eval_tol: every query within max(rel_err f, abs_err) / 2 of the full
        sum (the reference's eval(queries, rel_err, abs_err)); (values, CullStats)."""
        n = self.size(QUERY)
        out = np.empty(max(n, 1))
        st = CullStats()
        self._check(self.lib.bbkde_eval_tol(self.h, C.byref(desc), int(normalized), rel_err,
                                            abs_err, out.ctypes.data, 0, C.byref(st)))
        return out[:n], st

    def eval_grid(self, desc: KernelDesc, grid, out_ptr: int, surrogate=None,
                  mode=GRID_EXACT, tile=16, probes=5, exact_culled=True, rel_tol=5e-4,
                  low_frac=1e-4, cull_rel=1e-7, interp=1, pair_form=False,
                  net_scope=NET_RESCUE, lattice_tile=0, tensor_cores=0) -> GridStats:
        """Density on a dense grid into device memory out_ptr (nx * ny doubles).

        grid = (nx, ny, x0, x1, y0, y1). Returns the GridStats."""
        g = Grid(*grid)
        cfg = GridConfig(mode, tile, probes, int(exact_culled), rel_tol, low_frac, cull_rel,
                         interp, int(pair_form), net_scope, lattice_tile, tensor_cores)
        st = GridStats()
        sh = surrogate.h if surrogate is not None else None
        self._check(self.lib.bbkde_eval_grid(self.h, sh, C.byref(desc), C.byref(g), C.byref(cfg),
                                             out_ptr, C.byref(st)))
        return st

    def lsq_numint_cv(self, desc: KernelDesc, grid, precision=FP32C) -> float:
        """grid = (nx, ny, x0, x1, y0, y1)."""
        cv = np.zeros(1)
        g = Grid(*grid)
        self._check(self.lib.bbkde_lsq_numint_cv(self.h, C.byref(desc), C.byref(g), precision,
                                                 _p(cv)))
        return float(cv[0])

    def set_launch_variant(self, variant: int):
        """-1 = autotune (default); 0..n-1 forces a launch shape."""
        self._check(self.lib.bbkde_ctx_set_launch_variant(self.h, variant))

    def launch_variants(self):
        n, last = C.c_int(), C.c_int()
        self._check(self.lib.bbkde_launch_variants(self.h, C.byref(n), C.byref(last)))
        return n.value, last.value

    def device_info(self):
        sm, dev = C.c_int(), C.c_int()
        self._check(self.lib.bbkde_device_info(self.h, C.byref(sm), C.byref(dev)))
        return sm.value, dev.value


def eval_noalloc(desc: KernelDesc, n_ref: int, ref_x: int, ref_y: int | None, ref_mass: int,
                 ref_abw: int | None, n_query: int, query_x: int, query_y: int | None,
                 out: int, normalized: bool = True, stream: int | None = None):
    """bbkde_eval_noalloc on device pointers (ints). Returns (status, message).

    Allocates no device memory; the work is enqueued on `stream` and the call
    returns before it finishes (synchronise before reading `out`)."""
    lib = load_library()
    buf = C.create_string_buffer(512)
    rc = lib.bbkde_eval_noalloc(C.byref(desc), n_ref, ref_x, ref_y, ref_mass, ref_abw,
                                n_query, query_x, query_y, int(normalized), out, stream,
                                buf, len(buf))
    return rc, buf.value.decode()


def _fp(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_float))


class Surrogate:
    """The learned log-density network (2 -> 128 -> 128 -> 128 -> 1, SiLU)."""

    def __init__(self, device: int = 0, seed: int = 1):
        self.lib = load_library()
        h = C.c_void_p()
        rc = self.lib.bbkde_surrogate_create(device, seed, C.byref(h))
        if rc != OK:
            raise BBKDEError(rc, "bbkde_surrogate_create failed: " +
                             self.lib.bbkde_status_string(rc).decode())
        self.h = h
        self.n_params = int(self.lib.bbkde_surrogate_num_params())

    def close(self):
        if getattr(self, "h", None):
            self.lib.bbkde_surrogate_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc == OK:
            return
        msg = (self.lib.bbkde_surrogate_last_error(self.h) or b"").decode()
        if rc == INVALID_ARGUMENT:
            raise InvalidArgument(rc, msg)
        raise BBKDEError(rc, msg)

    def params(self):
        p = np.empty(self.n_params, dtype=np.float32)
        norm = np.empty(6, dtype=np.float32)
        self._check(self.lib.bbkde_surrogate_get_params(self.h, _fp(p), _fp(norm)))
        return p, norm

    def set_params(self, p, norm=None):
        p = np.ascontiguousarray(p, dtype=np.float32)
        norm = None if norm is None else np.ascontiguousarray(norm, dtype=np.float32)
        self._check(self.lib.bbkde_surrogate_set_params(self.h, _fp(p), _fp(norm)))

    def gradient(self, xy, target):
        xy, target = _c(xy).reshape(-1, 2), _c(target)
        g = np.empty(self.n_params, dtype=np.float32)
        loss = C.c_double()
        self._check(self.lib.bbkde_surrogate_gradient(self.h, xy.shape[0], _p(xy), _p(target),
                                                      _fp(g), C.byref(loss)))
        return g, loss.value

    def train(self, xy, target, steps=2000, batch=8192, lr=2e-3, lr_final=1e-5, seed=7):
        xy, target = _c(xy).reshape(-1, 2), _c(target)
        cfg = TrainConfig(steps, batch, lr, lr_final, 0.0, 0.0, 0.0, seed)
        loss = C.c_double()
        self._check(self.lib.bbkde_surrogate_train(self.h, xy.shape[0], _p(xy), _p(target),
                                                   C.byref(cfg), C.byref(loss)))
        return loss.value

    def predict(self, xy):
        xy = _c(xy).reshape(-1, 2)
        out = np.empty(xy.shape[0])
        self._check(self.lib.bbkde_surrogate_predict(self.h, xy.shape[0], _p(xy), _p(out)))
        return out

    def set_inference(self, split_activations: bool):
        """False: BF16 activations (as trained); True: two-term BF16 activations."""
        self._check(self.lib.bbkde_surrogate_set_inference(self.h, int(split_activations)))

    def set_engine(self, engine: int):
        """ENGINE_TCGEN05 (default) or ENGINE_MMA_SYNC."""
        self._check(self.lib.bbkde_surrogate_set_engine(self.h, engine))

    def save(self, path):
        self._check(self.lib.bbkde_surrogate_save(self.h, str(path).encode()))

    def load(self, path):
        self._check(self.lib.bbkde_surrogate_load(self.h, str(path).encode()))
