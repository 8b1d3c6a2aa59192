"""Loads ``lib/libswb200.so`` and declares the C ABI of ``include/swb200.h`` for ctypes."""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

P = ctypes.c_void_p
U32 = ctypes.c_uint32
U64 = ctypes.c_uint64
I32 = ctypes.c_int
F32 = ctypes.c_float


class NativeError(RuntimeError):
    """A call into libswb200.so failed (the message is swb_last_error())."""

    def __init__(self, status: int, message: str):
        super().__init__(f"swb200 status {status}: {message}")
        self.status = status


def lib_path() -> str:
    return os.path.join(_HERE, "lib", "libswb200.so")


def native_available() -> bool:
    return os.path.exists(lib_path())


_SIGNATURES = {
    "swb_version": ([], ctypes.c_char_p),
    "swb_last_error": ([], ctypes.c_char_p),
    "swb_device_count": ([P], I32),
    "swb_kernel_launches": ([], U64),
    "swb_create": ([P, U32, U32, U32, U32, U32, U32, I32], I32),
    "swb_destroy": ([P], I32),
    "swb_set_spins": ([P, P], I32),
    "swb_get_spins": ([P, P], I32),
    "swb_hot_start": ([P, U32], I32),
    "swb_cold_start": ([P, ctypes.c_uint8], I32),
    "swb_p_add": ([F32], F32),
    "swb_accept_threshold": ([F32], U32),
    "swb_sweep": ([P, F32, U32, U32], I32),
    "swb_sweep_recorded": ([P, F32, P, P, P], I32),
    "swb_sweep_dumped": ([P, F32, P, P, P], I32),
    "swb_geometry": ([P, P], I32),
    "swb_synchronize": ([P], I32),
    "swb_energy_magnetization": ([P, P, P, P], I32),
    "swb_accumulators": ([P, P], I32),
    "swb_reset_accumulators": ([P], I32),
    "swb_samples": ([P, P, U64, P], I32),
    "swb_rng_shape": ([P, P, P], I32),
    "swb_get_rng": ([P, P, P, P, P], I32),
    "swb_set_rng": ([P, P, P, P, P], I32),
    "swb_device_buffers": ([P, P, P], I32),
    "swb_launches_per_sweep": ([P, P], I32),
    "swb_update_host": ([P, F32, P, P, P], I32),
    "swb_sweep_timed": ([P, F32, U32, I32, P], I32),
    "swb_attach_spins": ([P, P], I32),
    "swb_device_alloc": ([I32, ctypes.c_size_t, P], I32),
    "swb_device_free": ([I32, P], I32),
    "swb_copy_to_device": ([I32, P, P, ctypes.c_size_t], I32),
    "swb_copy_to_host": ([I32, P, P, ctypes.c_size_t], I32),
    "swb_device_synchronize": ([I32], I32),
    "swb_device_sm_count": ([I32, P], I32),
    "swb_spins_energy_magnetization": ([I32, U32, U32, P, P, P, P], I32),
    "swb_host_alloc": ([P, ctypes.c_size_t], I32),
    "swb_host_free": ([P], I32),
    "swb_sweep_static": ([P, U32, U32, U32, U32, U32, F32, U32, P, P, P, P, I32], I32),
    "swb_lcg32_benchmark": ([U32, U32, U32, U64, U32, P, P, P, I32], I32),
}


def declared_symbols() -> list[str]:
    return list(_SIGNATURES)


def _declare(handle, signatures) -> None:
    for name, (args, res) in signatures.items():
        fn = getattr(handle, name, None)
        if fn is None:
            continue
        fn.argtypes = args
        fn.restype = res


def extra_signatures(sigs: dict) -> None:
    """Lets other modules of the package declare further entry points."""
    _SIGNATURES.update(sigs)
    if _LIB is not None:
        _declare(_LIB, sigs)


def lib():
    """The loaded native library; raises when it is missing (no fallback)."""
    global _LIB
    if _LIB is None:
        path = lib_path()
        if not os.path.exists(path):
            raise NativeError(-1, f"native library {path} is missing; run python -m computational_physics_b200.build")
        _LIB = ctypes.CDLL(path)
        _declare(_LIB, _SIGNATURES)
    return _LIB


def check(status: int) -> None:
    if status != 0:
        msg = lib().swb_last_error()
        raise NativeError(status, msg.decode() if msg else "")
