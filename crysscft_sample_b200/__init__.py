"""B200-native pseudo-spectral propagator library for AB-diblock SCFT.

Drop-in GPU replacements for the reference's three diffusion solvers
(CrysPSSolverP1, CrysPSSolver3m, CrysPSSolverPmmm) and the SCFT iteration
that drives them, implemented as hand-written sm_100a CUDA kernels behind a
C ABI (include/crysscft_b200.h).
"""
from .fields import seed_fields, to_physical, from_physical  # noqa: F401

__all__ = ["seed_fields", "to_physical", "from_physical", "solvers", "scft"]


def __getattr__(name):
    # the CUDA-backed modules load the library on first use
    if name in ("solvers", "scft"):
        import importlib

        return importlib.import_module(f".{name}", __name__)
    raise AttributeError(name)
