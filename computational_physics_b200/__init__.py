"""B200-native Swendsen-Wang engine for the 2D Ising model (and its 3D extension).

Python host mirror of the reference's interface (flwende/computational_physics):

* :class:`SwendsenWang2D` -- one lattice on one GPU, the drop-in for
  ``SwendsenWang_2D<LCG32, Target>::Update`` plus ``Lattice<2>``'s observables
  (ising/include/swendsen_wang.hpp:26-102, ising/include/lattice.hpp:21-95);
* :func:`p_add` -- the bond probability exactly as ising/src/swendsen_wang.cpp:100;
* :class:`SwendsenWang3D` -- the same sweep on a periodic 3D lattice.

Everything runs through the C ABI of ``include/swb200.h`` in ``lib/libswb200.so``
(hand-written CUDA for sm_100a).  There is no CPU fallback: importing works without a
GPU, but any compute call raises if the native library or a CUDA device is missing.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from ._native import NativeError, lib, lib_path, native_available  # noqa: F401
from .lattice import SwendsenWang2D, p_add, device_count, kernel_launches, pinned_empty  # noqa: F401
from .batch import BatchedSW, HostIO, lattice_bytes, UNLIMITED  # noqa: F401
from .lattice3 import SwendsenWang3D  # noqa: F401

__all__ = ["SwendsenWang2D", "SwendsenWang3D", "BatchedSW", "HostIO", "p_add", "device_count", "kernel_launches", "pinned_empty",
           "lattice_bytes", "UNLIMITED", "NativeError", "lib", "lib_path", "native_available"]
