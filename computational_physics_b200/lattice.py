"""One lattice on one GPU: the Python face of the drop-in ``nvidia_gpu`` target.

Mirrors ``SwendsenWang_2D<LCG32, Target>`` (ising/include/swendsen_wang.hpp:26-102) and
``Lattice<2>`` (ising/include/lattice.hpp:21-95) over the C ABI of include/swb200.h.
"""
from __future__ import annotations

import ctypes

import numpy as np

from ._native import check, lib

__all__ = ["SwendsenWang2D", "p_add", "device_count", "kernel_launches"]


def _ptr(a):
    return None if a is None else a.ctypes.data


def p_add(temperature: float) -> float:
    """1 - exp(-2/T) in float (ising/src/swendsen_wang.cpp:100)."""
    return lib().swb_p_add(temperature)


def device_count() -> int:
    n = ctypes.c_int(0)
    check(lib().swb_device_count(ctypes.byref(n)))
    return n.value


def kernel_launches() -> int:
    return int(lib().swb_kernel_launches())


class _Pinned:
    def __init__(self, nbytes: int):
        self.ptr = ctypes.c_void_p()
        check(lib().swb_host_alloc(ctypes.byref(self.ptr), nbytes))
        self.nbytes = nbytes

    def __del__(self):
        try:
            lib().swb_host_free(self.ptr)
        except Exception:
            pass


def pinned_empty(shape, dtype=np.uint8) -> np.ndarray:
    """A numpy array in page-locked host memory (kept alive by the array)."""
    dtype = np.dtype(dtype)
    n = int(np.prod(shape)) * dtype.itemsize
    mem = _Pinned(n)
    buf = (ctypes.c_char * max(n, 1)).from_address(mem.ptr.value)
    buf._owner = mem  # the array keeps buf alive, buf keeps the allocation alive
    return np.frombuffer(buf, dtype=dtype, count=int(np.prod(shape))).reshape(shape)


class SwendsenWang2D:
    """A periodic L0 x L1 Ising lattice swept by the Swendsen-Wang algorithm on a B200.

    ``tile`` and ``lcg_width`` fix how the lcg32 random numbers are consumed, exactly as
    the reference CPU path with one stream per tile seeded ``seed_base + tile id``.
    """

    def __init__(self, L0: int, L1: int | None = None, tile: tuple[int, int] = (16, 8), lcg_width: int = 16,
                 seed_base: int = 1, device: int = 0):
        L1 = L0 if L1 is None else L1
        self.L0, self.L1 = int(L0), int(L1)
        self.tile = (int(tile[0]), int(tile[1]))
        self.lcg_width = int(lcg_width)
        self._lib = lib()
        h = ctypes.c_void_p()
        check(self._lib.swb_create(ctypes.byref(h), self.L0, self.L1, self.tile[0], self.tile[1], self.lcg_width,
                                   seed_base, device))
        self._h = h

    # -- lifetime
    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.swb_destroy(self._h)
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
        return self.L0 * self.L1

    # -- spins
    def set_spins(self, spins: np.ndarray) -> None:
        s = np.ascontiguousarray(spins, dtype=np.uint8)
        if s.size != self.num_sites:
            raise ValueError(f"expected {self.num_sites} spins, got {s.size}")
        check(self._lib.swb_set_spins(self._h, _ptr(s)))

    def get_spins(self) -> np.ndarray:
        out = np.empty((self.L1, self.L0), np.uint8)
        check(self._lib.swb_get_spins(self._h, _ptr(out)))
        return out

    def hot_start(self, seed: int = 1) -> None:
        check(self._lib.swb_hot_start(self._h, seed))

    def cold_start(self, value: int = 1) -> None:
        check(self._lib.swb_cold_start(self._h, value))

    # -- sweeps
    def update(self, temperature: float, n_sweeps: int = 1, measure_every: int = 0) -> None:
        check(self._lib.swb_sweep(self._h, temperature, n_sweeps, measure_every))

    def update_recorded(self, temperature: float):
        """One sweep returning (bonds, labels_assign, labels_final) of this sweep."""
        b = np.empty((self.L1, self.L0), np.uint8)
        la = np.empty((self.L1, self.L0), np.uint32)
        lf = np.empty((self.L1, self.L0), np.uint32)
        check(self._lib.swb_sweep_recorded(self._h, temperature, _ptr(b), _ptr(la), _ptr(lf)))
        return b, la, lf

    def update_dumped(self, temperature: float):
        """One sweep through the kernels a plain update runs, returning (bonds, labels_block,
        labels_final) of this sweep (labels_block: components over the bonds inside each
        assign block, see :meth:`geometry`)."""
        b = np.empty((self.L1, self.L0), np.uint8)
        lb = np.empty((self.L1, self.L0), np.uint32)
        lf = np.empty((self.L1, self.L0), np.uint32)
        check(self._lib.swb_sweep_dumped(self._h, temperature, _ptr(b), _ptr(lb), _ptr(lf)))
        return b, lb, lf

    def geometry(self) -> dict:
        """Tile and assign-block shape of the handle."""
        g = np.zeros(8, np.uint32)
        check(self._lib.swb_geometry(self._h, _ptr(g)))
        keys = ("L0", "L1", "tile_x", "tile_y", "block_x", "block_y", "blocks_x", "blocks_y")
        return {k: int(v) for k, v in zip(keys, g)}

    def update_host(self, temperature: float, spins_in: np.ndarray, spins_out: np.ndarray,
                    em: np.ndarray | None = None) -> None:
        check(self._lib.swb_update_host(self._h, temperature, _ptr(spins_in), _ptr(spins_out), _ptr(em)))

    def synchronize(self) -> None:
        check(self._lib.swb_synchronize(self._h))

    def sweep_timed(self, temperature: float, n_sweeps: int, per_kernel: bool = False) -> np.ndarray:
        """Device milliseconds of n_sweeps sweeps: [total, assign, merge, flip] (per-kernel
        entries only with per_kernel=True)."""
        ms = np.zeros(4, np.float32)
        check(self._lib.swb_sweep_timed(self._h, temperature, n_sweeps, int(per_kernel), _ptr(ms)))
        return ms

    # -- observables
    def energy_magnetization(self) -> tuple[float, float]:
        out = np.zeros(2, np.float64)
        check(self._lib.swb_energy_magnetization(self._h, _ptr(out), None, None))
        return float(out[0]), float(out[1])

    def energy_magnetization_sums(self) -> tuple[int, int]:
        e = ctypes.c_int64()
        m = ctypes.c_int64()
        check(self._lib.swb_energy_magnetization(self._h, None, ctypes.byref(e), ctypes.byref(m)))
        return e.value, m.value

    def accumulators(self) -> np.ndarray:
        out = np.zeros(4, np.float64)
        check(self._lib.swb_accumulators(self._h, _ptr(out)))
        return out

    def reset_accumulators(self) -> None:
        check(self._lib.swb_reset_accumulators(self._h))

    def samples(self) -> np.ndarray:
        """Integer sums (e, m) of every measured sweep since the last reset, shape [k, 2]."""
        n = ctypes.c_uint64()
        check(self._lib.swb_samples(self._h, None, 0, ctypes.byref(n)))
        out = np.empty((n.value, 2), np.int64)
        check(self._lib.swb_samples(self._h, _ptr(out), n.value, ctypes.byref(n)))
        return out

    # -- lcg32 streams
    def rng_shape(self) -> tuple[int, int]:
        nt = ctypes.c_uint32()
        w = ctypes.c_uint32()
        check(self._lib.swb_rng_shape(self._h, ctypes.byref(nt), ctypes.byref(w)))
        return nt.value, w.value

    def get_rng(self):
        nt, w = self.rng_shape()
        st = np.empty((nt, w), np.uint32); a = np.empty((nt, w), np.uint32); c = np.empty((nt, w), np.uint32)
        it = np.empty(nt, np.uint32)
        check(self._lib.swb_get_rng(self._h, _ptr(st), _ptr(a), _ptr(c), _ptr(it)))
        return st, a, c, it

    def set_rng(self, state, a, c, iteration) -> None:
        nt, w = self.rng_shape()
        arrs = [np.ascontiguousarray(x, np.uint32) for x in (state, a, c, iteration)]
        if arrs[0].size != nt * w or arrs[1].size != nt * w or arrs[2].size != nt * w or arrs[3].size != nt:
            raise ValueError("rng arrays have the wrong size")
        check(self._lib.swb_set_rng(self._h, *[_ptr(x) for x in arrs]))

    def snapshot(self) -> dict:
        """Spins, lcg32 streams and recorded observables: enough to resume this lattice
        bit-identically in another handle or process (see :mod:`computational_physics_b200.snapshot`)."""
        st, a, c, it = self.get_rng()
        return {"L0": self.L0, "L1": self.L1, "tile": self.tile, "lcg_width": self.lcg_width,
                "spins": self.get_spins(), "rng_state": st, "rng_a": a, "rng_c": c, "rng_iteration": it,
                "samples": self.samples(), "accumulators": self.accumulators()}

    def restore(self, snap: dict) -> None:
        """Loads a snapshot's spins and lcg32 streams (same extent, tile and lcg width)."""
        if (self.L0, self.L1, self.tile, self.lcg_width) != (snap["L0"], snap["L1"], tuple(snap["tile"]),
                                                            snap["lcg_width"]):
            raise ValueError("snapshot geometry does not match the lattice")
        self.set_spins(snap["spins"])
        self.set_rng(snap["rng_state"], snap["rng_a"], snap["rng_c"], snap["rng_iteration"])

    def device_buffers(self) -> tuple[int, int]:
        s = ctypes.c_void_p()
        l = ctypes.c_void_p()
        check(self._lib.swb_device_buffers(self._h, ctypes.byref(s), ctypes.byref(l)))
        return s.value, l.value

    def launches_per_sweep(self) -> int:
        n = ctypes.c_uint32()
        check(self._lib.swb_launches_per_sweep(self._h, ctypes.byref(n)))
        return n.value
