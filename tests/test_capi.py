"""The C ABI library builds, loads without a GPU and exports every function include/*.h declares."""
import ctypes
import glob
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for h in sorted(glob.glob(os.path.join(ROOT, "include", "*.h"))):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"\b(swb_\w+)\s*\(", text)
    return sorted(set(names))


def test_header_declares_functions():
    names = declared_functions()
    assert "swb_create" in names and "swb_sweep" in names and len(names) >= 20


def test_library_exports_every_declared_symbol():
    import computational_physics_b200 as cp
    if not cp.native_available():
        from computational_physics_b200.build import build
        build()
    lib = ctypes.CDLL(cp.lib_path())
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_declares_every_symbol():
    from computational_physics_b200 import _native
    import computational_physics_b200  # noqa: F401  (its modules register their entry points)
    declared = set(_native.declared_symbols())
    missing = [n for n in declared_functions() if n not in declared]
    assert not missing, missing


def test_pure_host_entry_points_without_gpu():
    """Entry points that need no device: version, p_add, device count, argument errors."""
    import computational_physics_b200 as cp
    lib = cp.lib()
    assert lib.swb_version().decode().startswith("swb200")
    for T in (1.5, 2.2691853, 3.0):
        assert cp.p_add(T) == pytest.approx(1 - __import__("math").exp(-2 / T), rel=1e-6)
    n = cp.device_count()
    assert n >= 0
    h = ctypes.c_void_p()
    assert lib.swb_create(ctypes.byref(h), 15, 16, 16, 8, 16, 1, 0) == 1          # odd extent
    assert "evenly sized" in lib.swb_last_error().decode()
    assert lib.swb_create(ctypes.byref(h), 16, 16, 12, 8, 16, 1, 0) == 1          # tile width
    assert lib.swb_create(ctypes.byref(h), 16, 16, 16, 8, 12, 1, 0) == 1          # lcg width
    assert lib.swb_create(ctypes.byref(h), 2, 4_200_000, 8, 32, 16, 1, 0) == 1     # > 65535 block rows
    assert "block rows" in lib.swb_last_error().decode()
    assert not h.value


def test_accept_threshold_is_the_reference_float_test():
    """u < swb_accept_threshold(p) must equal (float)u * 2^-32 < p for every u; checked at the
    threshold's neighbourhood and on random draws for many p, with numpy's round-to-nearest."""
    import numpy as np
    import computational_physics_b200 as cp
    lib = cp.lib()
    rng = np.random.default_rng(7)
    scale = np.float32(2.0 ** -32)
    ps = np.concatenate([np.float32([0.0, 1.0, 0.5, 0.5857864618301392, 1e-7, 0.9999999]),
                         rng.random(200).astype(np.float32),
                         np.array([cp.p_add(float(t)) for t in np.linspace(0.3, 6, 100)], np.float32)])
    for p in ps:
        thr = int(lib.swb_accept_threshold(float(p)))
        us = np.concatenate([rng.integers(0, 2 ** 32, 2000, dtype=np.uint64),
                             np.arange(max(thr - 300, 0), min(thr + 300, 2 ** 32), dtype=np.uint64)]).astype(np.uint32)
        want = (us.astype(np.float32) * scale) < np.float32(p)
        got = us.astype(np.uint64) < thr
        assert np.array_equal(want, got), float(p)
