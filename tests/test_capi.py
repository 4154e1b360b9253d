"""The C-ABI library loads and exports every entry point of include/wavesim_b200.h
(no compute call is made: this runs without a GPU)."""
import ctypes as C
import os
import re

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions(name="wavesim_b200.h"):
    text = open(os.path.join(ROOT, "include", name)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ws_[a-z_0-9]+)\s*\(", text)) - {"ws_callback_fn"})


def test_library_exports_header_symbols():
    from wavesim_b200 import _lib
    names = header_functions()
    assert names, "no functions parsed from the header"
    for n in names:
        assert hasattr(_lib.lib, n), n
    assert sorted(_lib.EXPORTS) == names


def test_library_exports_network_header_symbols():
    """include/wavesim_b200_net.h (the warm-start network kernels)."""
    from wavesim_b200 import _lib
    names = header_functions("wavesim_b200_net.h")
    assert len(names) > 10
    for n in names:
        assert hasattr(_lib.lib, n), n


def test_version_and_defaults():
    from wavesim_b200 import _lib
    assert b"sm_100a" in _lib.lib.ws_version()
    o = _lib.default_options()
    assert o.max_iterations == 100000 and o.energy_interval == 8 and o.energy_threshold == 1e-2
    assert o.stop_rule == _lib.WS_STOP_REFERENCE and o.use_graph == 1


def test_size_support():
    from wavesim_b200 import _lib
    ok = lambda *n: _lib.lib.ws_size_supported((C.c_int64 * 4)(*n))  # noqa: E731
    assert ok(512, 512, 1, 1) and ok(1024, 1024, 1, 1) and ok(256, 256, 256, 1) and ok(192, 192, 192, 3)
    assert ok(77, 45, 1, 1) and ok(320, 1, 1, 1) and ok(96, 96, 96, 1)
    assert not ok(17, 64, 1, 1)      # prime factor above 13
    assert not ok(64, 64, 64, 2)     # N(4) must be 1 or 3


def test_errors_without_device_are_reported():
    from wavesim_b200 import _lib
    N = (C.c_int64 * 4)(16, 16, 1, 1)
    g = np.zeros((16, 16), np.complex64)
    h = C.c_void_p()
    rc = _lib.lib.ws_solver_create(N, g.ctypes.data, 0, None, C.c_float(3.0), _lib.ws_complex(1, 1),
                                   (C.c_int64 * 8)(1, 16, 1, 16, 1, 1, 1, 1), 0, 0, C.byref(h))
    assert rc == _lib.WS_ERR_INVALID_ARGUMENT  # null wiggles rejected before any CUDA call
    assert _lib.lib.ws_last_error()
