"""Batching form: many independent AB-diblock SCFT instances advanced together on one
GPU (scft_batch_* in include/crysscft_b200.h).  One batch iteration is one CUDA-graph
launch in which the instances' contour kernels run concurrently; an autotuner picks
the number of worker streams and the contour-kernel form."""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib, fields
from ._lib import check

__all__ = ["BatchSCFT", "batch_config", "FORMS"]

FORMS = {0: "automatic", 1: "alternating layout", 2: "two-phase", 3: "per-axis kernels",
         4: "one persistent launch (team kernel)"}


def batch_config(n: int = 64, seed: int = 20261203, sizes=(16, 24, 32, 48, 64)):
    """The seeded batching workload: n PMMM instances with reduced grids drawn from
    `sizes`^3 (full grids twice that), chiN ~ U[14, 30], fA ~ U[0.2, 0.35],
    L ~ U[3.8, 5.5] Rg, BCC or FCC seed fields."""
    u = fields.uniform53(seed, 99, 5 * n).reshape(n, 5)
    out = []
    for i in range(n):
        nr = sizes[min(int(u[i, 0] * len(sizes)), len(sizes) - 1)]
        out.append({
            "N": (2 * nr,) * 3,
            "xN": 14.0 + 16.0 * u[i, 1],
            "fA": 0.2 + 0.15 * u[i, 2],
            "L": 3.8 + 1.7 * u[i, 3],
            "phase": "BCC" if u[i, 4] < 0.5 else "FCC",
            "seed": seed + 1000 + i,
        })
    return out


class BatchSCFT:
    """n instances of one solver kind; per-instance grid, cell, fA and chiN."""

    def __init__(self, kind: str, instances, ds: float = 0.01, acceptance: float = 0.1,
                 precision: str = "fp64", device: int = -1):
        L = _lib.load()
        n = len(instances)
        grid = (ctypes.c_size_t * (3 * n))(*[int(v) for it in instances for v in it["N"]])
        cell = np.array([[it["L"]] * 3 if np.ndim(it["L"]) == 0 else list(it["L"]) for it in instances],
                        dtype=np.float64).ravel()
        fA = np.array([it["fA"] for it in instances], dtype=np.float64)
        xN = np.array([it["xN"] for it in instances], dtype=np.float64)
        h = ctypes.c_void_p()
        check(L.scft_batch_create(_lib.KIND[kind.upper()], n, grid, _lib.dptr(cell), _lib.dptr(fA), _lib.dptr(xN),
                                  float(ds), float(acceptance), _lib.PRECISION[precision], int(device),
                                  ctypes.byref(h)))
        self._h = h
        self.kind = kind.upper()
        self.instances = instances
        self.n = n
        self.M = [self._space_size(i) for i in range(n)]

    def _space_size(self, i: int) -> int:
        """Physical grid size of instance i, as its solver reports it."""
        L = _lib.load()
        d, s, m = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_size_t()
        check(L.scft_batch_instance(self._h, int(i), ctypes.byref(d)))
        check(L.scft_diblock_get_solver(d, ctypes.byref(s)))
        check(L.scft_solver_get_space_size_phy(s, ctypes.byref(m)))
        return int(m.value)

    def close(self):
        if getattr(self, "_h", None):
            _lib.load().scft_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def seed_fields(self):
        """Seeded BCC/FCC fields of every instance (layout of the solver kind)."""
        for i, it in enumerate(self.instances):
            wA, wB = fields.seed_fields(it["N"], it["L"], it.get("phase", "BCC"), seed=it.get("seed", 20261203))
            self.set_fields(i, fields.to_physical(self.kind, wA), fields.to_physical(self.kind, wB))

    def set_fields(self, i: int, wA, wB):
        wA = np.ascontiguousarray(wA, dtype=np.float64).ravel()
        wB = np.ascontiguousarray(wB, dtype=np.float64).ravel()
        check(_lib.load().scft_batch_set_fields(self._h, int(i), _lib.dptr(wA), _lib.dptr(wB)))

    def get_fields(self, i: int, out=None):
        """phiA, phiB, wA, wB of instance i; `out` (four contiguous float64 arrays of the
        instance's physical grid size, e.g. page-locked ones) receives them instead of new arrays."""
        if out is None:
            out = [np.empty(self.M[i]) for _ in range(4)]
        else:
            out = list(out)
            if len(out) != 4 or any(a.dtype != np.float64 or a.size != self.M[i] or not a.flags.c_contiguous
                                    for a in out):
                raise ValueError("out must be four contiguous float64 arrays of the instance's grid size")
        check(_lib.load().scft_batch_get_fields(self._h, int(i), *[_lib.dptr(a) for a in out]))
        return dict(zip(("phiA", "phiB", "wA", "wB"), out))

    def iterate(self, n_iter: int):
        F = np.empty((n_iter, self.n))
        mi = np.empty((n_iter, self.n))
        check(_lib.load().scft_batch_iterate(self._h, int(n_iter), _lib.dptr(F), _lib.dptr(mi)))
        return {"F": F, "maxinc": mi}

    def launches_per_iteration(self) -> int:
        """Kernel launches one batch iteration issues in the current configuration."""
        k = ctypes.c_size_t()
        check(_lib.load().scft_batch_launches_per_iteration(self._h, ctypes.byref(k)))
        return k.value

    def configure(self, nstreams: int = 8, form: int = 4):
        """Worker streams and contour form (FORMS); 4 runs every instance's contour in one
        persistent launch."""
        check(_lib.load().scft_batch_configure(self._h, int(nstreams), int(form)))

    def set_team_sizes(self, sizes: dict):
        """Form 4: fixed team sizes {grid side: CTAs per chain}; other sides get the planner's choice."""
        sides = (ctypes.c_int * max(1, len(sizes)))(*[int(k) for k in sizes])
        vals = (ctypes.c_int * max(1, len(sizes)))(*[int(v) for v in sizes.values()])
        check(_lib.load().scft_batch_set_team_sizes(self._h, len(sizes), sides, vals))

    def team_plan(self) -> dict:
        """The form-4 plan: CTAs, team tasks, instances in the launch, planned makespan and
        its lower bound (us per iteration, cost model)."""
        g, t, k = ctypes.c_int(), ctypes.c_size_t(), ctypes.c_size_t()
        pl, lb = ctypes.c_double(), ctypes.c_double()
        check(_lib.load().scft_batch_team_plan(self._h, ctypes.byref(g), ctypes.byref(t), ctypes.byref(k),
                                               ctypes.byref(pl), ctypes.byref(lb)))
        return {"grid": g.value, "tasks": t.value, "instances": k.value, "planned_us": pl.value,
                "bound_us": lb.value}

    def configure(self, nstreams: int, form: int = 0):
        check(_lib.load().scft_batch_configure(self._h, int(nstreams), int(form)))

    def set_wait_limit(self, spins: int | None = None):
        """Poll limit of every bounded device wait of every instance (None: the default);
        the one-launch form uses the smallest limit of its instances."""
        L = _lib.load()
        for i in range(self.n):
            d = ctypes.c_void_p()
            check(L.scft_batch_instance(self._h, i, ctypes.byref(d)))
            check(L.scft_diblock_set_wait_limit(d, int(spins) if spins is not None else 20000000))

    def autotune(self, n_trial: int = 3):
        ns, form, ms = ctypes.c_size_t(), ctypes.c_int(), ctypes.c_double()
        check(_lib.load().scft_batch_autotune(self._h, int(n_trial), ctypes.byref(ns), ctypes.byref(form),
                                              ctypes.byref(ms)))
        return {"nstreams": ns.value, "form": FORMS[form.value], "ms_per_iteration": ms.value}
