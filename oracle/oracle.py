"""Test infrastructure: ctypes wrappers around the CPU checkers (see package docstring)."""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_P = ctypes.c_void_p
_U = ctypes.c_uint32
_F = ctypes.c_float

__all__ = [
    "Oracle", "RefHarness", "oracle_lib_path", "ref_lib_path", "have_ref", "RngTiles",
    "num_tiles", "build_oracle",
]


def oracle_lib_path() -> str:
    return os.path.join(HERE, "liboracle.so")


def ref_lib_path(width: int = 16) -> str:
    return os.path.join(HERE, "_ref", f"libswref{width}.so")


def have_ref(width: int = 16) -> bool:
    return os.path.exists(ref_lib_path(width))


def build_oracle() -> None:
    """Compiles liboracle.so (needs only gcc)."""
    import subprocess
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)


def _ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data


def num_tiles(L0: int, L1: int, tx: int, ty: int) -> int:
    return ((L0 + tx - 1) // tx) * ((L1 + ty - 1) // ty)


@dataclass
class RngTiles:
    """Per-tile lcg32 streams in the reference's LCG32_State<W> terms (random/include/random/lcg32.hpp:27-58)."""
    W: int
    state: np.ndarray      # uint32 [n_tiles, W]
    a: np.ndarray          # uint32 [n_tiles, W]
    c: np.ndarray          # uint32 [n_tiles, W]
    iteration: np.ndarray  # uint32 [n_tiles]

    @classmethod
    def empty(cls, W: int, n_tiles: int) -> "RngTiles":
        z = lambda: np.zeros((n_tiles, W), np.uint32)
        return cls(W, z(), z(), z(), np.zeros(n_tiles, np.uint32))

    def copy(self) -> "RngTiles":
        return RngTiles(self.W, self.state.copy(), self.a.copy(), self.c.copy(), self.iteration.copy())

    def equal(self, other: "RngTiles") -> bool:
        return (self.W == other.W and np.array_equal(self.state, other.state) and np.array_equal(self.a, other.a)
                and np.array_equal(self.c, other.c) and np.array_equal(self.iteration, other.iteration))


class Oracle:
    """The C restatement (sw_oracle.c)."""

    def __init__(self, path: str | None = None):
        path = path or oracle_lib_path()
        if not os.path.exists(path):
            build_oracle()
        lib = ctypes.CDLL(path)
        lib.orc_hot_start.argtypes = [_U, _U, _U, _P]
        lib.orc_lcg32_init.argtypes = [_U, _U, _P, _P, _P, _P]
        lib.orc_lcg32_update.argtypes = [_U, _P, _P, _P, _P]
        lib.orc_lcg32_next_real.argtypes = [_U, _P, _P, _P, _P, _U, _P]
        lib.orc_p_add.argtypes = [_F]
        lib.orc_p_add.restype = _F
        lib.orc_rng_init_tiles.argtypes = [_U, _U, _U, _P, _P, _P, _P]
        lib.orc_sw_sweep.argtypes = [_U, _U, _U, _U, _U, _F, _P, _P, _P, _P, _P, _P, _P, _P]
        lib.orc_sw_sweep.restype = ctypes.c_int
        lib.orc_energy_magnetization.argtypes = [_U, _U, _P, _P, _P]
        lib.orc_block_labels.argtypes = [_U, _U, _U, _U, _P, _P]
        lib.orc3_sw_sweep.argtypes = [_U, _U, _U, _U, _U, _U, _U, _F, _P, _P, _P, _P, _P, _P, _P]
        lib.orc3_sw_sweep.restype = ctypes.c_int
        lib.orc3_energy_magnetization.argtypes = [_U, _U, _U, _P, _P, _P]
        self.lib = lib

    def hot_start(self, L0: int, L1: int, seed: int = 1) -> np.ndarray:
        s = np.empty(L0 * L1, np.uint8)
        self.lib.orc_hot_start(L0, L1, seed, _ptr(s))
        return s.reshape(L1, L0)

    def p_add(self, T: float) -> float:
        return self.lib.orc_p_add(T)

    def rng_init(self, W: int, n_tiles: int, seed_base: int = 1) -> RngTiles:
        r = RngTiles.empty(W, n_tiles)
        self.lib.orc_rng_init_tiles(W, n_tiles, seed_base, _ptr(r.state), _ptr(r.a), _ptr(r.c), _ptr(r.iteration))
        return r

    def next_real(self, W: int, seed: int, sizes) -> np.ndarray:
        st = np.zeros(W, np.uint32); a = np.zeros(W, np.uint32); c = np.zeros(W, np.uint32)
        it = np.zeros(1, np.uint32)
        self.lib.orc_lcg32_init(W, seed, _ptr(st), _ptr(a), _ptr(c), _ptr(it))
        out = []
        for n in sizes:
            buf = np.empty(n, np.float32)
            self.lib.orc_lcg32_next_real(W, _ptr(st), _ptr(a), _ptr(c), _ptr(it), n, _ptr(buf))
            out.append(buf)
        return np.concatenate(out) if out else np.zeros(0, np.float32)

    def sweep(self, spins: np.ndarray, tx: int, ty: int, rng: RngTiles, T: float | None = None,
              p_add: float | None = None, dumps: bool = False):
        """One sweep in place on ``spins`` ([L1, L0] uint8) and ``rng``.  With ``dumps`` returns
        (bonds, labels_assign, labels_final) of this sweep."""
        L1, L0 = spins.shape
        assert spins.dtype == np.uint8 and spins.flags.c_contiguous
        p = self.p_add(T) if p_add is None else p_add
        bonds = la = lf = None
        if dumps:
            bonds = np.empty((L1, L0), np.uint8)
            la = np.empty((L1, L0), np.uint32)
            lf = np.empty((L1, L0), np.uint32)
        rc = self.lib.orc_sw_sweep(L0, L1, tx, ty, rng.W, p, _ptr(spins), _ptr(rng.state), _ptr(rng.a),
                                   _ptr(rng.c), _ptr(rng.iteration), _ptr(bonds), _ptr(la), _ptr(lf))
        if rc != 0:
            raise ValueError(f"orc_sw_sweep failed with status {rc}")
        return (bonds, la, lf) if dumps else None

    def block_labels(self, bonds: np.ndarray, block_x: int, block_y: int) -> np.ndarray:
        """Minimum-index labels of the components over the bonds inside each block_x x
        block_y block (the GPU path's labels between its assign and merge phases)."""
        L1, L0 = bonds.shape
        b = np.ascontiguousarray(bonds, np.uint8)
        out = np.empty((L1, L0), np.uint32)
        self.lib.orc_block_labels(L0, L1, block_x, block_y, _ptr(b), _ptr(out))
        return out

    def sweep3(self, spins: np.ndarray, tile: tuple[int, int, int], rng: RngTiles, T: float | None = None,
               p_add: float | None = None, dumps: bool = False):
        """One 3D sweep in place on spins [L2, L1, L0] (uint8); with dumps returns (bonds, labels)."""
        L2, L1, L0 = spins.shape
        p = self.p_add(T) if p_add is None else p_add
        bonds = np.empty(spins.shape, np.uint8) if dumps else None
        lab = np.empty(spins.shape, np.uint32) if dumps else None
        rc = self.lib.orc3_sw_sweep(L0, L1, L2, tile[0], tile[1], tile[2], rng.W, p, _ptr(spins), _ptr(rng.state),
                                    _ptr(rng.a), _ptr(rng.c), _ptr(rng.iteration), _ptr(bonds), _ptr(lab))
        if rc != 0:
            raise ValueError(f"orc3_sw_sweep failed with status {rc}")
        return (bonds, lab) if dumps else None

    def energy_magnetization3(self, spins: np.ndarray) -> tuple[int, int]:
        L2, L1, L0 = spins.shape
        e = ctypes.c_int64()
        m = ctypes.c_int64()
        s = np.ascontiguousarray(spins, np.uint8)
        self.lib.orc3_energy_magnetization(L0, L1, L2, _ptr(s), ctypes.byref(e), ctypes.byref(m))
        return e.value, m.value

    def energy_magnetization(self, spins: np.ndarray) -> tuple[int, int]:
        L1, L0 = spins.shape
        e = ctypes.c_int64(); m = ctypes.c_int64()
        s = np.ascontiguousarray(spins, np.uint8)
        self.lib.orc_energy_magnetization(L0, L1, _ptr(s), ctypes.byref(e), ctypes.byref(m))
        return e.value, m.value


class RefHarness:
    """The unmodified reference CPU sources behind oracle/ref_harness.cpp."""

    def __init__(self, width: int = 16):
        lib = ctypes.CDLL(ref_lib_path(width))
        lib.ref_lcg32_width.restype = ctypes.c_int
        lib.ref_p_add.argtypes = [_F]
        lib.ref_p_add.restype = _F
        lib.ref_hot_start.argtypes = [_U, _U, _P]
        lib.ref_lcg32_init.argtypes = [_U, _P, _P, _P, _P]
        lib.ref_lcg32_next_real.argtypes = [_U, _P, _U, _P]
        lib.ref_energy_magnetization.argtypes = [_U, _U, _P, _P, _P]
        lib.ref_sw_run.argtypes = [_U, _U, _U, _U, _U, _F, _U, _P, _P, _P, _P, _P, _P, _P, _P]
        lib.ref_sw_run.restype = ctypes.c_int
        lib.ref_cpu_sweep_many.argtypes = [_U, _P, _P, _P, _U, _U]
        lib.ref_cpu_sweep_many.restype = ctypes.c_double
        self.lib = lib
        self.W = lib.ref_lcg32_width()

    def p_add(self, T: float) -> float:
        return self.lib.ref_p_add(T)

    def hot_start(self, L0: int, L1: int) -> np.ndarray:
        s = np.empty(L0 * L1, np.uint8)
        self.lib.ref_hot_start(L0, L1, _ptr(s))
        return s.reshape(L1, L0)

    def lcg32_init(self, seed: int):
        W = self.W
        st = np.zeros(W, np.uint32); a = np.zeros(W, np.uint32); c = np.zeros(W, np.uint32)
        it = np.zeros(1, np.uint32)
        self.lib.ref_lcg32_init(seed, _ptr(st), _ptr(a), _ptr(c), _ptr(it))
        return st, a, c, int(it[0])

    def next_real(self, seed: int, sizes) -> np.ndarray:
        sizes = np.asarray(sizes, np.uint32)
        out = np.empty(int(sizes.sum()), np.float32)
        self.lib.ref_lcg32_next_real(seed, _ptr(sizes), len(sizes), _ptr(out))
        return out

    def energy_magnetization(self, spins: np.ndarray) -> tuple[float, float]:
        L1, L0 = spins.shape
        e = ctypes.c_double(); m = ctypes.c_double()
        s = np.ascontiguousarray(spins, np.uint8)
        self.lib.ref_energy_magnetization(L0, L1, _ptr(s), ctypes.byref(e), ctypes.byref(m))
        return e.value, m.value

    def run(self, spins: np.ndarray, tx: int, ty: int, T: float, n_sweeps: int = 1, seed_base: int = 1):
        """n_sweeps reference sweeps on a copy of ``spins``; returns
        (spins_after, bonds, labels_assign, labels_final, RngTiles) of the last sweep."""
        L1, L0 = spins.shape
        s = np.ascontiguousarray(spins, np.uint8).copy()
        bonds = np.empty((L1, L0), np.uint8)
        la = np.empty((L1, L0), np.uint32)
        lf = np.empty((L1, L0), np.uint32)
        nt = num_tiles(L0, L1, tx, ty)
        r = RngTiles.empty(self.W, nt)
        rc = self.lib.ref_sw_run(L0, L1, tx, ty, seed_base, T, n_sweeps, _ptr(s), _ptr(bonds), _ptr(la), _ptr(lf),
                                 _ptr(r.state), _ptr(r.a), _ptr(r.c), _ptr(r.iteration))
        if rc != 0:
            raise ValueError(f"ref_sw_run failed with status {rc}")
        return s, bonds, la, lf, r

    def cpu_sweep_many(self, extents, temperatures, spins_list, n_sweeps: int, num_threads: int) -> float:
        """The reference's own threaded SwendsenWang_2D<LCG32, CPU>::Update over several lattices."""
        k = len(extents)
        ext = np.asarray(extents, np.uint32)
        temps = np.asarray(temperatures, np.float32)
        ptrs = (ctypes.c_void_p * k)(*[s.ctypes.data for s in spins_list])
        return self.lib.ref_cpu_sweep_many(k, _ptr(ext), _ptr(temps), ctypes.cast(ptrs, ctypes.c_void_p),
                                           n_sweeps, num_threads)
