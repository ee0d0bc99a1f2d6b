"""B200 batched dense-solve engine for the per-cell linear systems of the
Python/Sirocco radiative-transfer code (solve_matrix / invert_matrix).

The product is the C ABI in ``include/sirocco_solve.h``, implemented by the
CUDA library ``python_b200/libsirocco_solve.so``; ``python_b200.engine`` binds
it for Python callers and ``python_b200.workloads`` builds seeded batches.
"""
__all__ = ["engine", "workloads"]
