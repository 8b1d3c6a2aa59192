"""One 3D lattice on one GPU: the Swendsen-Wang sweep of the 3D Ising model (swb3_* of
include/swb200.h).  The reference names the 3D case only (ising/include/swendsen_wang_selflabeling.hpp:20-22);
the conventions are the 2D ones extended by a third direction (see the header)."""
from __future__ import annotations

import ctypes

import numpy as np

from ._native import I32, P, U32, U64, F32, check, extra_signatures, lib

__all__ = ["SwendsenWang3D"]

extra_signatures({
    "swb3_create": ([P, U32, U32, U32, U32, U32, U32, U32, U32, I32], I32),
    "swb3_destroy": ([P], I32),
    "swb3_geometry": ([P, P], I32),
    "swb3_set_spins": ([P, P], I32),
    "swb3_get_spins": ([P, P], I32),
    "swb3_hot_start": ([P, U32], I32),
    "swb3_sweep": ([P, F32, U32, U32], I32),
    "swb3_sweep_dumped": ([P, F32, P, P], I32),
    "swb3_sweep_timed": ([P, F32, U32, P], I32),
    "swb3_energy_magnetization": ([P, P, P, P], I32),
    "swb3_samples": ([P, P, U64, P, P], I32),
    "swb3_rng_shape": ([P, P, P], I32),
    "swb3_get_rng": ([P, P, P, P, P], I32),
})


def _ptr(a):
    return None if a is None else a.ctypes.data


class SwendsenWang3D:
    """A periodic L0 x L1 x L2 Ising lattice (arrays are [L2, L1, L0]) swept on a B200."""

    def __init__(self, L0: int, L1: int, L2: int, tile: tuple[int, int, int] = (16, 4, 4), lcg_width: int = 16,
                 seed_base: int = 1, device: int = 0):
        self.shape = (int(L2), int(L1), int(L0))
        self.tile = tuple(int(t) for t in tile)
        self.lcg_width = int(lcg_width)
        self._lib = lib()
        h = ctypes.c_void_p()
        check(self._lib.swb3_create(ctypes.byref(h), int(L0), int(L1), int(L2), *self.tile, self.lcg_width, seed_base,
                                    device))
        self._h = h

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.swb3_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def num_sites(self) -> int:
        return int(np.prod(self.shape))

    def geometry(self) -> dict:
        g = np.zeros(12, np.uint32)
        check(self._lib.swb3_geometry(self._h, _ptr(g)))
        keys = ("L0", "L1", "L2", "tile_x", "tile_y", "tile_z", "block_x", "block_y", "block_z", "blocks_x", "blocks_y",
                "blocks_z")
        return {k: int(v) for k, v in zip(keys, g)}

    def set_spins(self, spins: np.ndarray) -> None:
        s = np.ascontiguousarray(spins, dtype=np.uint8)
        if s.size != self.num_sites:
            raise ValueError(f"expected {self.num_sites} spins, got {s.size}")
        check(self._lib.swb3_set_spins(self._h, _ptr(s)))

    def get_spins(self) -> np.ndarray:
        out = np.empty(self.shape, np.uint8)
        check(self._lib.swb3_get_spins(self._h, _ptr(out)))
        return out

    def hot_start(self, seed: int = 1) -> None:
        check(self._lib.swb3_hot_start(self._h, seed))

    def update(self, temperature: float, n_sweeps: int = 1, measure_every: int = 0) -> None:
        check(self._lib.swb3_sweep(self._h, temperature, n_sweeps, measure_every))

    def update_dumped(self, temperature: float):
        """One sweep returning (bonds, labels) of this sweep (bonds: bit 0 +x, 1 +y, 2 +z)."""
        b = np.empty(self.shape, np.uint8)
        lab = np.empty(self.shape, np.uint32)
        check(self._lib.swb3_sweep_dumped(self._h, temperature, _ptr(b), _ptr(lab)))
        return b, lab

    def sweep_timed(self, temperature: float, n_sweeps: int) -> float:
        ms = ctypes.c_float()
        check(self._lib.swb3_sweep_timed(self._h, temperature, n_sweeps, ctypes.byref(ms)))
        return ms.value

    def energy_magnetization_sums(self) -> tuple[int, int]:
        e = ctypes.c_int64()
        m = ctypes.c_int64()
        check(self._lib.swb3_energy_magnetization(self._h, None, ctypes.byref(e), ctypes.byref(m)))
        return e.value, m.value

    def samples(self) -> tuple[np.ndarray, np.ndarray]:
        """(e, m) integer sums of every measured sweep, shape [k, 2], and the accumulators."""
        n = ctypes.c_uint64()
        acc = np.zeros(4, np.float64)
        check(self._lib.swb3_samples(self._h, None, 0, ctypes.byref(n), _ptr(acc)))
        out = np.empty((n.value, 2), np.int64)
        check(self._lib.swb3_samples(self._h, _ptr(out), n.value, ctypes.byref(n), _ptr(acc)))
        return out, acc

    def get_rng(self):
        nt = ctypes.c_uint32()
        w = ctypes.c_uint32()
        check(self._lib.swb3_rng_shape(self._h, ctypes.byref(nt), ctypes.byref(w)))
        st = np.empty((nt.value, w.value), np.uint32)
        a = np.empty_like(st)
        c = np.empty_like(st)
        it = np.empty(nt.value, np.uint32)
        check(self._lib.swb3_get_rng(self._h, _ptr(st), _ptr(a), _ptr(c), _ptr(it)))
        return st, a, c, it
