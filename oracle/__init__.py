"""CPU oracle for the SPH step (TEST INFRASTRUCTURE).

A restatement of the reference's CPU algorithm for the hot path: per-particle kernels in plain C
with OpenMP (``oracle.c``) and the step drivers in NumPy (``sph.py``, ``steps.py``).  It is the
checker for the CUDA path in ``tests/`` and ``__graft_entry__.smoke()``, and the CPU baseline that
``bench.py`` times beside it.  The product package never imports it.

It is pinned to the reference by the golden fixtures in ``tests/golden/`` (made by running the
reference itself; see ``tests/golden/make_golden.py``).  The bremsstrahlung cooling law has no
counterpart in the reference: its oracle (``cooling.py``) is pinned by closed-form known answers
instead ("parity unpinned" against the reference for that law only).
"""
