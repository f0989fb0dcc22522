"""CPU FP64 oracle for the SSA forward/adjoint hot path (test infrastructure).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg may import this package.  It is the checker, never the product path.
"""
