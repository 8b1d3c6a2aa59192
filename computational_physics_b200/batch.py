"""Many lattices on one GPU: the batched Swendsen-Wang engine (one launch per sweep phase over
all lattices' blocks, one CUDA graph per round) behind the swb_batch_* C ABI."""
from __future__ import annotations

import ctypes

import numpy as np

from ._native import I32, P, U32, U64, F32, check, extra_signatures, lib

extra_signatures({
    "swb_batch_create": ([P, U32, U64, U32, I32], I32),
    "swb_batch_destroy": ([P], I32),
    "swb_batch_lattice_bytes": ([U32, U32, U32, U32, U32, P], I32),
    "swb_batch_add": ([P, U32, U32, U32, U32, U32, U32, F32, U32, P], I32),
    "swb_batch_remove": ([P, U32], I32),
    "swb_batch_hot_start": ([P, U32, U32], I32),
    "swb_batch_set_spins": ([P, U32, P], I32),
    "swb_batch_get_spins": ([P, U32, P], I32),
    "swb_batch_set_temperature": ([P, U32, F32], I32),
    "swb_batch_set_schedule": ([P, U32, U32, U32], I32),
    "swb_batch_status": ([P, U32, P, P], I32),
    "swb_batch_poll": ([P, P, P], I32),
    "swb_batch_sweep": ([P, U32, I32], I32),
    "swb_batch_mark": ([P, P], I32),
    "swb_batch_mark_query": ([P, U32, P, P], I32),
    "swb_batch_synchronize": ([P], I32),
    "swb_batch_sweep_timed": ([P, U32, I32, P], I32),
    "swb_batch_accumulators": ([P, U32, P], I32),
    "swb_batch_samples": ([P, U32, P, U64, P], I32),
    "swb_batch_samples_finished": ([P, U32, P, U64, P, P], I32),
    "swb_batch_get_rng": ([P, U32, P, P, P, P], I32),
    "swb_batch_set_rng": ([P, U32, P, P, P, P], I32),
    "swb_batch_info": ([P, U32, P], I32),
    "swb_batch_memory": ([P, P, P], I32),
    "swb_batch_update_host": ([P, U32, P, P, P], I32),
    "swb_batch_update_host_rounds": ([P, U32, P, P, P, U32], I32),
})

UNLIMITED = 0xFFFFFFFF

__all__ = ["BatchedSW", "HostIO", "lattice_bytes", "UNLIMITED"]


def _ptr(a):
    return None if a is None else a.ctypes.data


def lattice_bytes(L0: int, L1: int, tile=(16, 8), lcg_width: int = 16) -> int:
    v = ctypes.c_uint64()
    check(lib().swb_batch_lattice_bytes(L0, L1, tile[0], tile[1], lcg_width, ctypes.byref(v)))
    return v.value


class BatchedSW:
    """Independent periodic lattices of different sizes, tiles and temperatures, swept
    together.  Each lattice is bit-identical to a :class:`SwendsenWang2D` with the same
    extent, tile, lcg width and seed base."""

    def __init__(self, capacity: int = 1024, hbm_budget_bytes: int = 0, lcg_width: int = 16, device: int = 0):
        self._lib = lib()
        h = ctypes.c_void_p()
        check(self._lib.swb_batch_create(ctypes.byref(h), capacity, hbm_budget_bytes, lcg_width, device))
        self._h = h
        self.capacity = capacity
        self.lcg_width = lcg_width
        self.shapes: dict[int, tuple[int, int]] = {}

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.swb_batch_destroy(self._h)
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

    def add(self, L0: int, L1: int | None = None, temperature: float = 2.2691853, seed_base: int = 1,
            tile=(16, 8), block=(0, 0)) -> int:
        L1 = L0 if L1 is None else L1
        i = ctypes.c_uint32()
        check(self._lib.swb_batch_add(self._h, L0, L1, tile[0], tile[1], block[0], block[1], temperature,
                                      seed_base, ctypes.byref(i)))
        self.shapes[i.value] = (L1, L0)
        return i.value

    def remove(self, lid: int) -> None:
        check(self._lib.swb_batch_remove(self._h, lid))
        self.shapes.pop(lid, None)

    def hot_start(self, lid: int, seed: int = 1) -> None:
        check(self._lib.swb_batch_hot_start(self._h, lid, seed))

    def set_spins(self, lid: int, spins: np.ndarray) -> None:
        s = np.ascontiguousarray(spins, np.uint8)
        if s.size != int(np.prod(self.shapes[lid])):
            raise ValueError("wrong number of spins")
        check(self._lib.swb_batch_set_spins(self._h, lid, _ptr(s)))

    def get_spins(self, lid: int) -> np.ndarray:
        out = np.empty(self.shapes[lid], np.uint8)
        check(self._lib.swb_batch_get_spins(self._h, lid, _ptr(out)))
        return out

    def set_temperature(self, lid: int, temperature: float) -> None:
        check(self._lib.swb_batch_set_temperature(self._h, lid, temperature))

    def set_schedule(self, lid: int, sweeps: int = UNLIMITED, measure_every: int = 0) -> None:
        check(self._lib.swb_batch_set_schedule(self._h, lid, sweeps, measure_every))

    def status(self, lid: int) -> tuple[int, int]:
        left = ctypes.c_uint32()
        done = ctypes.c_uint32()
        check(self._lib.swb_batch_status(self._h, lid, ctypes.byref(left), ctypes.byref(done)))
        return left.value, done.value

    def poll(self) -> tuple[np.ndarray, np.ndarray]:
        """sweeps_left and sweeps_done of every slot (0 for free slots)."""
        left = np.zeros(self.capacity, np.uint32)
        done = np.zeros(self.capacity, np.uint32)
        check(self._lib.swb_batch_poll(self._h, _ptr(left), _ptr(done)))
        return left, done

    def sweep(self, rounds: int = 1, measure: bool = False) -> None:
        check(self._lib.swb_batch_sweep(self._h, rounds, int(measure)))

    def mark(self) -> int:
        """Records a point after the work submitted so far; see :meth:`mark_done`."""
        m = ctypes.c_uint32()
        check(self._lib.swb_batch_mark(self._h, ctypes.byref(m)))
        return m.value

    def mark_done(self, mark: int) -> float | None:
        """None while the device has not passed `mark`, else its device time in seconds since
        the first mark (non-blocking)."""
        done = ctypes.c_int()
        ms = ctypes.c_double()
        check(self._lib.swb_batch_mark_query(self._h, mark, ctypes.byref(done), ctypes.byref(ms)))
        return ms.value / 1e3 if done.value else None

    def synchronize(self) -> None:
        check(self._lib.swb_batch_synchronize(self._h))

    def sweep_timed(self, rounds: int, per_kernel: bool = False) -> np.ndarray:
        ms = np.zeros(4, np.float32)
        check(self._lib.swb_batch_sweep_timed(self._h, rounds, int(per_kernel), _ptr(ms)))
        return ms

    def accumulators(self, lid: int) -> np.ndarray:
        out = np.zeros(4, np.float64)
        check(self._lib.swb_batch_accumulators(self._h, lid, _ptr(out)))
        return out

    def samples(self, lid: int) -> np.ndarray:
        n = ctypes.c_uint64()
        check(self._lib.swb_batch_samples(self._h, lid, None, 0, ctypes.byref(n)))
        out = np.empty((n.value, 2), np.int64)
        check(self._lib.swb_batch_samples(self._h, lid, _ptr(out), n.value, ctypes.byref(n)))
        return out

    def samples_finished(self, lid: int, max_samples: int) -> np.ndarray:
        """The sample series of a lattice that has finished its sweep budget, read without
        waiting for the batch's other work (valid once a mark after its last sweep is passed)."""
        n = ctypes.c_uint64()
        out = np.empty((max_samples, 2), np.int64)
        check(self._lib.swb_batch_samples_finished(self._h, lid, _ptr(out), max_samples, ctypes.byref(n), None))
        return out[:min(n.value, max_samples)]

    def get_rng(self, lid: int):
        g = self.info(lid)
        nt, w = g["tiles"], self.lcg_width
        st = np.empty((nt, w), np.uint32); a = np.empty((nt, w), np.uint32); c = np.empty((nt, w), np.uint32)
        it = np.empty(nt, np.uint32)
        check(self._lib.swb_batch_get_rng(self._h, lid, _ptr(st), _ptr(a), _ptr(c), _ptr(it)))
        return st, a, c, it

    def set_rng(self, lid: int, state, a, c, iteration) -> None:
        nt, w = self.info(lid)["tiles"], self.lcg_width
        arrs = [np.ascontiguousarray(x, np.uint32) for x in (state, a, c, iteration)]
        if any(x.size != nt * w for x in arrs[:3]) or arrs[3].size != nt:
            raise ValueError("rng arrays have the wrong size")
        check(self._lib.swb_batch_set_rng(self._h, lid, *[_ptr(x) for x in arrs]))

    def snapshot(self, lid: int) -> dict:
        """Everything needed to resume lattice `lid` bit-identically elsewhere (another slot,
        batch or process): geometry, spins, lcg32 streams, sweeps done and the recorded
        observables.  See :mod:`computational_physics_b200.snapshot` for the file format."""
        g = self.info(lid)
        st, a, c, it = self.get_rng(lid)
        return {"L0": g["L0"], "L1": g["L1"], "tile": (g["tile_x"], g["tile_y"]), "lcg_width": self.lcg_width,
                "spins": self.get_spins(lid), "rng_state": st, "rng_a": a, "rng_c": c, "rng_iteration": it,
                "sweeps_done": self.status(lid)[1], "samples": self.samples(lid),
                "accumulators": self.accumulators(lid)}

    def restore(self, lid: int, snap: dict) -> None:
        """Loads a snapshot's spins and lcg32 streams into lattice `lid`, which must have the same
        extent, tile and lcg width.  Its sweeps then continue the snapshot's Markov chain exactly;
        the snapshot's samples and accumulators stay with the caller."""
        g = self.info(lid)
        if (g["L0"], g["L1"], (g["tile_x"], g["tile_y"]), self.lcg_width) != \
                (snap["L0"], snap["L1"], tuple(snap["tile"]), snap["lcg_width"]):
            raise ValueError("snapshot geometry does not match the lattice")
        self.set_spins(lid, snap["spins"])
        self.set_rng(lid, snap["rng_state"], snap["rng_a"], snap["rng_c"], snap["rng_iteration"])

    def info(self, lid: int) -> dict:
        v = np.zeros(8, np.uint32)
        check(self._lib.swb_batch_info(self._h, lid, _ptr(v)))
        keys = ("L0", "L1", "tile_x", "tile_y", "block_x", "block_y", "tiles", "blocks")
        return {k: int(x) for k, x in zip(keys, v)}

    def memory(self) -> tuple[int, int]:
        used = ctypes.c_uint64()
        budget = ctypes.c_uint64()
        check(self._lib.swb_batch_memory(self._h, ctypes.byref(used), ctypes.byref(budget)))
        return used.value, budget.value

    def update_host(self, ids, spins_in, spins_out) -> None:
        k = len(ids)
        idarr = np.asarray(ids, np.uint32)
        pin = (ctypes.c_void_p * k)(*[s.ctypes.data for s in spins_in])
        pout = (ctypes.c_void_p * k)(*[s.ctypes.data for s in spins_out])
        check(self._lib.swb_batch_update_host(self._h, k, _ptr(idarr), ctypes.cast(pin, ctypes.c_void_p),
                                              ctypes.cast(pout, ctypes.c_void_p)))

    def host_io(self, ids) -> "HostIO":
        """Pinned host buffers for update_host_io: one arena per direction, a (L1, L0) view per
        lattice of `ids`, and the pointer arrays the C ABI takes, built once."""
        return HostIO(self, ids)

    def update_host_io(self, io: "HostIO") -> None:
        """update_host with the buffers of `io` (io.inputs in, io.outputs out), one copy per
        direction through the arenas and no per-call pointer work in Python."""
        check(self._lib.swb_batch_update_host(self._h, io.count, io._ids.ctypes.data, io._pin, io._pout))

    def update_host_io_rounds(self, io: "HostIO", rounds: int) -> None:
        """`rounds` rounds of update_host_io with io.swap() after each, as one pipeline: every
        round copies all of io's lattices in and out, and a lattice group's next copy in starts
        as soon as its copy out has landed.  Afterwards io.inputs holds the last round's
        spins."""
        check(self._lib.swb_batch_update_host_rounds(self._h, io.count, io._ids.ctypes.data, io._pin, io._pout,
                                                     int(rounds)))
        if rounds % 2:
            io.swap()


class HostIO:
    """Host side of repeated host-buffer sweeps of a fixed set of lattices: ``inputs`` and
    ``outputs`` are (L1, L0) uint8 views into two pinned arenas, consecutive in memory so that
    each direction is one copy.  :meth:`swap` exchanges them, so a step's output is the next
    step's input."""

    def __init__(self, batch: BatchedSW, ids):
        from .lattice import pinned_empty
        self.ids = [int(i) for i in ids]
        self.count = len(self.ids)
        self._ids = np.asarray(self.ids, np.uint32)
        shapes = [batch.shapes[i] for i in self.ids]
        total = sum(a * b for a, b in shapes)
        self._arenas = [pinned_empty((max(total, 1),), np.uint8), pinned_empty((max(total, 1),), np.uint8)]
        views, ptrs = [[], []], [[], []]
        for side in (0, 1):
            off = 0
            for rows, cols in shapes:
                v = self._arenas[side][off:off + rows * cols].reshape(rows, cols)
                views[side].append(v)
                ptrs[side].append(v.ctypes.data)
                off += rows * cols
        self.inputs, self.outputs = views
        self._arrs = [(ctypes.c_void_p * self.count)(*ptrs[0]), (ctypes.c_void_p * self.count)(*ptrs[1])]
        self._pin, self._pout = (ctypes.cast(a, ctypes.c_void_p) for a in self._arrs)

    def swap(self) -> None:
        self.inputs, self.outputs = self.outputs, self.inputs
        self._pin, self._pout = self._pout, self._pin
