"""Test infrastructure: the CPU checkers for the Swendsen-Wang hot path.

Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline / reference legs of
``bench.py`` import this package.  It wraps

* ``liboracle.so`` -- the C restatement of the reference algorithm (``sw_oracle.c``);
* ``_ref/libswref{16,8}.so`` -- the stage-dump harness linked with the unmodified
  reference CPU sources (present only where ``oracle/Makefile`` could build it);
* ``exact`` -- the exact finite-lattice internal energy and specific heat.
"""
from .oracle import *  # noqa: F401,F403
