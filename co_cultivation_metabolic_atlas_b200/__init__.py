"""B200-native batched flux-balance LP engine.

Public pieces:

* ``LPEngine`` / ``SolveConfig`` / ``EngineOptions`` -- tensor-level batched
  solver over the C ABI of ``include/fbalp.h`` (persistent sm_100a kernels).
* ``B200LPBackend`` -- drop-in ``solve_batch(requests)`` service with the
  contract of the reference's batched GPU LP backend.
* ``normalize`` -- the ``linprog``-kwargs request normaliser.
* ``synthetic`` -- seeded synthetic species / community workloads.
"""

from .problem import normalize, request, split_bounds  # noqa: F401


def __getattr__(name):
    # GPU-facing classes import torch / the native library lazily.
    if name in ("LPEngine", "SolveConfig", "EngineOptions", "SolveResult", "prepare_matrix"):
        from . import engine
        return getattr(engine, name)
    if name == "B200LPBackend":
        from .backend import B200LPBackend
        return B200LPBackend
    raise AttributeError(name)
