"""ctypes binding of the C ABI in include/wavesim_b200.h.

The shared library ``libwavesim_b200.so`` is built in-tree next to this file
(``python wavesim_b200/build.py`` or ``__graft_entry__.build()``).  There is
no fallback: if the library is missing, importing this module raises.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libwavesim_b200.so")

WS_OK = 0
WS_ERR_INVALID_ARGUMENT = 1
WS_ERR_UNSUPPORTED = 2
WS_ERR_CUDA = 3
WS_ERR_OUT_OF_MEMORY = 4
WS_ERR_NO_SOURCE = 5
WS_ERR_DIVERGED = 6
WS_ERR_NO_DEVICE = 7

WS_HOST = 0
WS_DEVICE = 1
WS_STOP_REFERENCE = 0
WS_STOP_FRESH = 1
WS_OUTPUT_EPRIME = 0
WS_OUTPUT_FIELD = 1

STATUS_NAMES = {
    0: "WS_OK", 1: "WS_ERR_INVALID_ARGUMENT", 2: "WS_ERR_UNSUPPORTED", 3: "WS_ERR_CUDA",
    4: "WS_ERR_OUT_OF_MEMORY", 5: "WS_ERR_NO_SOURCE", 6: "WS_ERR_DIVERGED", 7: "WS_ERR_NO_DEVICE",
}


class ws_complex(C.Structure):
    _fields_ = [("re", C.c_float), ("im", C.c_float)]


class ws_wiggle(C.Structure):
    _fields_ = [("pxe", C.c_void_p), ("pye", C.c_void_p), ("pze", C.c_void_p),
                ("gx", C.c_void_p), ("gy", C.c_void_p), ("gz", C.c_void_p)]


class ws_source_block(C.Structure):
    _fields_ = [("position", C.c_int64 * 4), ("size", C.c_int64 * 4), ("values", C.c_void_p)]


CALLBACK = C.CFUNCTYPE(None, C.c_char_p, C.POINTER(C.c_double), C.c_int64, C.c_double, C.c_void_p)


class ws_plane_wave(C.Structure):
    _fields_ = [("position", C.c_int64 * 4), ("size", C.c_int64 * 4), ("amplitude", ws_complex),
                ("phase", C.c_double * 3), ("phase0", C.c_double)]


class ws_solve_options(C.Structure):
    _fields_ = [("max_iterations", C.c_int64), ("energy_threshold", C.c_double),
                ("energy_interval", C.c_int64), ("stop_rule", C.c_int), ("output", C.c_int),
                ("stop_on_nonfinite", C.c_int), ("use_graph", C.c_int), ("callback_type", C.c_char_p),
                ("callback_interval", C.c_int64), ("callback", CALLBACK), ("user_data", C.c_void_p),
                ("initial_field", C.c_void_p), ("initial_memory", C.c_int), ("initial_is_eprime", C.c_int),
                ("warm_discard_ratio", C.c_double)]


# every entry point declared in include/wavesim_b200.h
EXPORTS = [
    "ws_default_options", "ws_version", "ws_last_error", "ws_size_supported", "ws_run_algorithm",
    "ws_run_algorithm_release",
    "ws_solver_create", "ws_solver_create_media", "ws_solver_solve", "ws_solver_solve_batch", "ws_solver_solve_plane_waves", "ws_solver_buffers",
    "ws_solver_time_kernels", "ws_solver_time_split",
    "ws_solver_launches_per_iteration", "ws_solver_fused", "ws_solver_set_wait_limit", "ws_solver_time_fused", "ws_solver_warm_report", "ws_solver_warm_residual", "ws_solver_autotune", "ws_solver_get_layout", "ws_solver_set_layout", "ws_solver_destroy",
    "ws_run_algorithm_noalloc", "ws_medium_reduce", "ws_build_gamma", "ws_setup_last_error",
    "ws_noalloc_scratch_bytes", "ws_noalloc_last_error",
    "ws_pstd_default_options", "ws_pstd_create", "ws_pstd_run", "ws_pstd_destroy",
]


AMPLITUDE = C.CFUNCTYPE(None, C.c_double, C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_void_p)


class ws_pstd_options(C.Structure):
    _fields_ = [("max_iterations", C.c_int64), ("energy_threshold", C.c_double), ("energy_interval", C.c_int64),
                ("iterations_per_cycle", C.c_double), ("amplitude", AMPLITUDE), ("user_data", C.c_void_p)]


class WaveSimError(RuntimeError):
    def __init__(self, status, message):
        self.status = status
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build the CUDA library first (python wavesim_b200/build.py)")
    lib = C.CDLL(LIB_PATH)
    P = C.c_void_p
    i64p = C.POINTER(C.c_int64)
    lib.ws_default_options.argtypes = [C.POINTER(ws_solve_options)]
    lib.ws_default_options.restype = None
    lib.ws_version.restype = C.c_char_p
    lib.ws_last_error.restype = C.c_char_p
    lib.ws_size_supported.argtypes = [i64p]
    lib.ws_size_supported.restype = C.c_int
    lib.ws_run_algorithm.argtypes = [i64p, P, C.c_int64, C.POINTER(ws_wiggle), C.c_int64,
                                     C.POINTER(ws_source_block), C.c_float, ws_complex, i64p, C.c_int64,
                                     C.c_double, C.c_char_p, C.c_int64, CALLBACK, P, C.c_int, P,
                                     C.POINTER(C.c_double), i64p]
    lib.ws_run_algorithm.restype = C.c_int
    lib.ws_solver_create.argtypes = [i64p, P, C.c_int64, C.POINTER(ws_wiggle), C.c_float, ws_complex, i64p,
                                     C.c_int, C.c_int, C.POINTER(C.c_void_p)]
    lib.ws_solver_create.restype = C.c_int
    lib.ws_solver_create_media.argtypes = [i64p, C.c_int64, P, C.c_int64, C.POINTER(ws_wiggle), C.c_float, ws_complex,
                                           i64p, C.c_int, C.c_int, C.POINTER(C.c_void_p)]
    lib.ws_solver_create_media.restype = C.c_int
    lib.ws_solver_solve.argtypes = [P, C.c_int64, C.POINTER(ws_source_block), C.c_int,
                                    C.POINTER(ws_solve_options), P, C.c_int, C.POINTER(C.c_double), i64p,
                                    C.POINTER(C.c_int)]
    lib.ws_solver_solve.restype = C.c_int
    lib.ws_solver_solve_batch.argtypes = [P, C.c_int64, i64p, C.POINTER(ws_source_block), C.c_int,
                                          C.POINTER(ws_solve_options), P, C.c_int, C.POINTER(C.c_double), C.c_int64,
                                          i64p, C.POINTER(C.c_int)]
    lib.ws_solver_solve_batch.restype = C.c_int
    lib.ws_solver_solve_plane_waves.argtypes = [P, C.c_int64, C.POINTER(ws_plane_wave), C.POINTER(ws_solve_options), P,
                                                C.c_int, C.POINTER(C.c_double), C.c_int64, i64p, C.POINTER(C.c_int)]
    lib.ws_solver_solve_plane_waves.restype = C.c_int
    lib.ws_solver_buffers.argtypes = [P, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p)]
    lib.ws_solver_buffers.restype = C.c_int
    lib.ws_solver_time_kernels.argtypes = [P, C.c_int, C.POINTER(C.c_float), C.POINTER(C.c_double)]
    lib.ws_solver_time_kernels.restype = C.c_int
    lib.ws_solver_set_wait_limit.argtypes = [P, C.c_int64]
    lib.ws_solver_set_wait_limit.restype = C.c_int
    lib.ws_solver_launches_per_iteration.argtypes = [P]
    lib.ws_solver_launches_per_iteration.restype = C.c_int
    lib.ws_solver_fused.argtypes = [P]
    lib.ws_solver_fused.restype = C.c_int
    lib.ws_solver_time_fused.argtypes = [P, C.c_int, C.POINTER(C.c_float), C.POINTER(C.c_double)]
    lib.ws_solver_time_split.argtypes = [P, C.c_int, C.POINTER(C.c_float), C.POINTER(C.c_double)]
    lib.ws_solver_time_split.restype = C.c_int
    lib.ws_solver_time_fused.restype = C.c_int
    lib.ws_solver_warm_report.argtypes = [P, C.c_int64, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                          C.POINTER(C.c_int)]
    lib.ws_solver_warm_report.restype = C.c_int
    lib.ws_solver_warm_residual.argtypes = [P, C.c_int64, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    lib.ws_solver_warm_residual.restype = C.c_int
    lib.ws_solver_autotune.argtypes = [P, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_float), C.POINTER(C.c_float)]
    lib.ws_solver_autotune.restype = C.c_int
    lib.ws_solver_get_layout.argtypes = [P, C.POINTER(C.c_int32)]
    lib.ws_solver_get_layout.restype = C.c_int
    lib.ws_solver_set_layout.argtypes = [P, C.POINTER(C.c_int32)]
    lib.ws_solver_set_layout.restype = C.c_int
    i64a = C.POINTER(C.c_int64)
    lib.ws_medium_reduce.argtypes = [P, C.c_int, C.c_int64, C.c_double, C.c_double, C.POINTER(C.c_double), P]
    lib.ws_medium_reduce.restype = C.c_int
    lib.ws_build_gamma.argtypes = [P, C.c_int, i64a, i64a, i64a, P, P, P, C.c_double, C.c_double, C.c_double, P, P]
    lib.ws_build_gamma.restype = C.c_int
    lib.ws_setup_last_error.restype = C.c_char_p
    lib.ws_solver_destroy.argtypes = [P]
    lib.ws_solver_destroy.restype = C.c_int
    lib.ws_run_algorithm_noalloc.argtypes = [i64p, P, C.c_int64, C.POINTER(ws_wiggle), P, C.c_float, ws_complex,
                                             i64p, C.c_int64, C.c_double, C.c_int64, P, P, i64p,
                                             C.POINTER(C.c_int), P]
    lib.ws_run_algorithm_noalloc.restype = C.c_int
    lib.ws_noalloc_scratch_bytes.restype = C.c_int64
    lib.ws_pstd_default_options.argtypes = [C.POINTER(ws_pstd_options)]
    lib.ws_pstd_default_options.restype = None
    lib.ws_pstd_create.argtypes = [i64p, P, P, P, P, P, P, i64p, C.c_int, C.POINTER(C.c_void_p)]
    lib.ws_pstd_create.restype = C.c_int
    lib.ws_pstd_run.argtypes = [P, C.c_int64, C.POINTER(ws_source_block), C.c_int, C.POINTER(ws_pstd_options), P,
                                C.POINTER(C.c_double), C.c_int64, i64p, C.POINTER(C.c_int)]
    lib.ws_pstd_run.restype = C.c_int
    lib.ws_pstd_destroy.argtypes = [P]
    lib.ws_pstd_destroy.restype = C.c_int
    lib.ws_gemm_bf16.argtypes = [P, P, P, P, P, C.c_int64, C.c_int64, C.c_int64, C.c_int64, C.c_int64, C.c_int64,
                                 C.c_int, P, P]
    lib.ws_gemm_bf16.restype = C.c_int
    lib.ws_net_last_error.restype = C.c_char_p
    lib.ws_noalloc_last_error.restype = C.c_char_p
    return lib


lib = _load()


def check(status):
    if status != WS_OK:
        raise WaveSimError(status, lib.ws_last_error().decode(errors="replace"))
    return status


def check_setup(status):
    if status != WS_OK:
        raise WaveSimError(status, lib.ws_setup_last_error().decode(errors="replace"))
    return status


def default_options():
    o = ws_solve_options()
    lib.ws_default_options(C.byref(o))
    return o


class HostStage:
    """A reusable page-locked (pinned) host buffer that a solver's outputs
    land in, so that the device-to-host copy runs at the bus speed instead of
    through the driver's pageable staging (64 MB of fields: about 1 ms
    against 25 ms on the B200 boxes), then copied into an ordinary numpy
    array for the caller.  The buffer grows as needed and is reused by every
    solve of its owner (one per WaveSim, so concurrent solvers do not share
    one); without CUDA it is plain host memory."""

    def __init__(self):
        self._t = None
        self._a = None

    def get(self, count):
        """A complex64 array of `count` elements (the pointer to hand to the C ABI)."""
        import numpy as np
        count = int(count)
        if self._a is None or self._a.size < count:
            self._t = None
            try:
                import torch
                if torch.cuda.is_available():
                    self._t = torch.empty(count, dtype=torch.complex64, pin_memory=True)
                    self._a = self._t.numpy()
            except ImportError:
                pass
            if self._t is None:
                self._a = np.empty(count, np.complex64)
        return self._a[:count]

    _pool = None
    _pool_lock = __import__("threading").Lock()

    @classmethod
    def take(cls, buf, shape, order="C"):
        """A new array of `shape` (order "F": column-major) holding buf's
        values; copies above 4 MB run in chunks on a few host threads (numpy
        releases the interpreter lock for them), which is 3-4x faster than
        one thread and the page faults of the new array."""
        import numpy as np
        out = np.empty(buf.size, np.complex64)
        n = buf.size
        if buf.nbytes > (4 << 20):
            with cls._pool_lock:  # solvers on several host threads share one pool
                if cls._pool is None:
                    from concurrent.futures import ThreadPoolExecutor
                    cls._pool = ThreadPoolExecutor(max_workers=max(1, min(8, os.cpu_count() or 1)))
            k = cls._pool._max_workers
            step = -(-n // k)

            def part(i):
                out[i * step:(i + 1) * step] = buf[i * step:(i + 1) * step]
            list(cls._pool.map(part, range(k)))
        else:
            out[:] = buf[:n]
        shape = tuple(int(v) for v in shape)
        return out.reshape(shape[::-1]).T if order == "F" else out.reshape(shape)
