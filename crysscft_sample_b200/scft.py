"""Python mirror of the reference's SCFT driver (src/crysSCFT_sample.cpp), backed by the
B200 library.

* ``solve_diffusion_equation`` — src/crysSCFT_sample.cpp:373-396, through
  ``scft_solver_propagate`` (host buffers) with the same arguments and the same
  slot convention (direction +1 fills slots 0..Ns, -1 fills Ns..0).
* ``DiblockSCFT`` — the device-resident AB-diblock iteration (the loop of
  ``diblock_scft_simple_iterate``, :440-508) behind ``scft_diblock_*``.
* ``diblock_scft_simple_iterate`` — the driver itself with the reference's
  arguments and printout (:426-531).
"""
from __future__ import annotations

import ctypes
import time

import numpy as np

from . import _lib
from ._lib import check

__all__ = ["solve_diffusion_equation", "DiblockSCFT", "diblock_scft_simple_iterate", "contour_counts"]


def contour_counts(fA: float, ds: float):
    """NsA = size_t(fA/ds), NsB = size_t((1-fA)/ds) (src/crysSCFT_sample.cpp:442-444)."""
    return int(fA / ds), int((1 - fA) / ds)


def solve_diffusion_equation(q, init, wds, solver, Ns: int, direction: int):
    """Fill q[(Ns+1)*M] (numpy float64) with the propagator; returns q."""
    if direction not in (1, -1):
        raise _lib.ScftError(1, "Wrong direction")
    M = solver.get_space_size_phy()
    q = np.asarray(q)
    if q.dtype != np.float64 or not q.flags["C_CONTIGUOUS"] or q.size < (Ns + 1) * M:
        raise ValueError("q must be a contiguous float64 array of (Ns+1)*space_size_phy")
    init = np.ascontiguousarray(init, dtype=np.float64).ravel()
    wds = np.ascontiguousarray(wds, dtype=np.float64).ravel()
    check(_lib.load().scft_solver_propagate(solver.handle, _lib.dptr(q), _lib.dptr(init), _lib.dptr(wds),
                                            int(Ns), int(direction)))
    return q


class DiblockSCFT:
    """AB-diblock SCFT with simple mixing, resident on the GPU.

    One ``iterate()`` step is one pass of the reference loop body
    (src/crysSCFT_sample.cpp:476-508): Boltzmann factors, the four propagator
    chains, Q, phi (trapezoid), free energy, field update.
    """

    def __init__(self, solver, fA: float, ds: float, xN: float, acceptance: float):
        self.solver = solver
        h = ctypes.c_void_p()
        check(_lib.load().scft_diblock_create(solver.handle, float(fA), float(ds), float(xN), float(acceptance),
                                              ctypes.byref(h)))
        self._h = h
        self.fA, self.ds, self.xN, self.acceptance = fA, ds, xN, acceptance
        a, b = ctypes.c_size_t(), ctypes.c_size_t()
        check(_lib.load().scft_diblock_get_contour_counts(self._h, ctypes.byref(a), ctypes.byref(b)))
        self.NsA, self.NsB = a.value, b.value
        self.M = solver.get_space_size_phy()
        self.iterations_done = 0       # iterations run through this object (checkpoints record it)
        self.mixing = ["simple"]        # or ["anderson", history, beta]

    def close(self):
        if getattr(self, "_h", None):
            _lib.load().scft_diblock_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def set_fields(self, wA, wB):
        wA = np.ascontiguousarray(wA, dtype=np.float64).ravel()
        wB = np.ascontiguousarray(wB, dtype=np.float64).ravel()
        if wA.size != self.M or wB.size != self.M:
            raise ValueError("fields must have space_size_phy elements")
        check(_lib.load().scft_diblock_set_fields(self._h, _lib.dptr(wA), _lib.dptr(wB)))

    def get_fields(self):
        out = [np.empty(self.M) for _ in range(4)]
        check(_lib.load().scft_diblock_get_fields(self._h, *[_lib.dptr(a) for a in out]))
        return dict(zip(("phiA", "phiB", "wA", "wB"), out))

    def iterate(self, n_iter: int):
        """Run n_iter iterations; returns per-iteration F, parts (n,4), maxinc, Q."""
        F, mi, Q = np.empty(n_iter), np.empty(n_iter), np.empty(n_iter)
        parts = np.empty((n_iter, 4))
        check(_lib.load().scft_diblock_iterate(self._h, int(n_iter), _lib.dptr(F), _lib.dptr(parts),
                                               _lib.dptr(mi), _lib.dptr(Q)))
        self.iterations_done += int(n_iter)
        return {"F": F, "parts": parts, "maxinc": mi, "Q": Q}

    def iterate_host(self, wA, wB, n_iter: int, phiA=None, phiB=None):
        """End-to-end form: host fields in (updated in place), phi and history out.  phiA /
        phiB may be given (e.g. page-locked arrays, for faster copies); else they are allocated."""
        phiA = np.empty(self.M) if phiA is None else phiA
        phiB = np.empty(self.M) if phiB is None else phiB
        for a in (wA, wB, phiA, phiB):
            if a.dtype != np.float64 or a.size != self.M or not a.flags.c_contiguous:
                raise ValueError("host fields must be contiguous float64 arrays of the physical grid size")
        F, mi, Q = np.empty(n_iter), np.empty(n_iter), np.empty(n_iter)
        parts = np.empty((n_iter, 4))
        check(_lib.load().scft_diblock_iterate_host(self._h, _lib.dptr(wA), _lib.dptr(wB), int(n_iter),
                                                    _lib.dptr(phiA), _lib.dptr(phiB), _lib.dptr(F),
                                                    _lib.dptr(parts), _lib.dptr(mi), _lib.dptr(Q)))
        self.iterations_done += int(n_iter)
        return {"F": F, "parts": parts, "maxinc": mi, "Q": Q, "phiA": phiA, "phiB": phiB}

    def device_fields(self):
        """Raw device pointers (int) of phiA, phiB, wA, wB."""
        ps = [ctypes.c_void_p() for _ in range(4)]
        check(_lib.load().scft_diblock_device_fields(self._h, *[ctypes.byref(p) for p in ps]))
        return tuple(p.value for p in ps)

    def stress(self):
        """Backward pass from the stored contour of the last iteration (FP64, or FP32 after a
        precision-form iteration): d ln Q / d L (3 axes), dF/dchiN, Q.  At the saddle point
        the stress is dF/dL = -dlnQ_dL."""
        g = np.zeros(3)
        dx, Q = ctypes.c_double(), ctypes.c_double()
        check(_lib.load().scft_diblock_stress(self._h, _lib.dptr(g), ctypes.byref(dx), ctypes.byref(Q)))
        return {"dlnQ_dL": g, "dF_dxN": dx.value, "Q": Q.value}

    def get_contour(self, chain: int, slot: int) -> np.ndarray:
        """Stored propagator slice of the last iteration (chain 0: q, chain 1: q+)."""
        out = np.empty(self.M)
        check(_lib.load().scft_diblock_get_contour(self._h, int(chain), int(slot), _lib.dptr(out)))
        return out

    def set_precision(self, precision: str):
        """"fp64" (plain form) or "fp32" (3xTF32 triplets, FP64 Q/phi/energy/mixing)."""
        check(_lib.load().scft_diblock_set_precision(self._h, _lib.PRECISION[precision]))

    def get_precision(self) -> str:
        v = ctypes.c_int()
        check(_lib.load().scft_diblock_get_precision(self._h, ctypes.byref(v)))
        return {0: "fp64", 1: "fp32"}[v.value]

    def set_mixing(self, kind: str = "simple", history: int = 10, beta: float = 0.5):
        """Field mixing of the following iterations: "simple" (the reference's
        calc_new_fields with the acceptance given at construction) or "anderson" (device-side
        Anderson mixing over the last `history` iterates, mixing parameter `beta`; the history
        starts empty)."""
        if kind == "simple":
            check(_lib.load().scft_diblock_set_mixing(self._h, 0, 0.0))
            self.mixing = ["simple"]
        elif kind == "anderson":
            check(_lib.load().scft_diblock_set_mixing(self._h, int(history), float(beta)))
            self.mixing = ["anderson", int(history), float(beta)]
        else:
            raise ValueError(f"unknown mixing {kind!r}")

    def set_wait_limit(self, spins: int = 20_000_000):
        """Poll limit of the contour kernels' bounded waits (see scft_diblock_set_wait_limit)."""
        check(_lib.load().scft_diblock_set_wait_limit(self._h, int(spins)))

    def set_phi_form(self, fused: bool = True):
        """Integrate phi inside the whole-contour kernel (True, the default) or in a separate
        pass over the stored contour (False); see scft_diblock_set_phi_form."""
        check(_lib.load().scft_diblock_set_phi_form(self._h, 1 if fused else 0))

    def residuals(self) -> np.ndarray:
        """rms residual sqrt(<r, r> / 2M) of each iteration of the last iterate() call."""
        n = ctypes.c_size_t()
        check(_lib.load().scft_diblock_get_residuals(self._h, None, 0, ctypes.byref(n)))
        out = np.empty(n.value)
        check(_lib.load().scft_diblock_get_residuals(self._h, _lib.dptr(out), n.value, ctypes.byref(n)))
        return out

    def save_checkpoint(self, path):
        """Binary checkpoint of this run (crysscft_sample_b200.checkpoint)."""
        from . import checkpoint

        checkpoint.save(self, path)

    def iterate_polished(self, n_iter: int, n_polish: int):
        """The precision form: n_iter - n_polish FP32 iterations, then n_polish FP64 ones."""
        self.set_precision("fp32")
        h1 = self.iterate(n_iter - n_polish) if n_iter > n_polish else None
        self.set_precision("fp64")
        h2 = self.iterate(n_polish)
        if h1 is None:
            return h2
        return {k: np.concatenate([h1[k], h2[k]]) for k in h2}

    def time_phases(self, n_iter: int):
        """ms per iteration: (total, propagator chains, Q + phi, the rest); advances the fields."""
        out = np.zeros(4)
        check(_lib.load().scft_diblock_time_phases(self._h, int(n_iter), _lib.dptr(out)))
        return tuple(out)

    def launches_per_iteration(self) -> int:
        v = ctypes.c_size_t()
        check(_lib.load().scft_diblock_launches_per_iteration(self._h, ctypes.byref(v)))
        return v.value


def relax_cell(solver, fA, ds, xN, acceptance, wA, wB, L0, n_outer=40, n_inner=20, step=1.0, tol=1e-6,
               cubic=True):
    """Variable-cell relaxation: n_inner SCFT iterations at the current cell, then a
    gradient step L <- L - step * dF/dL with the saddle-point stress dF/dL = -dlnQ/dL
    (cubic: one length, the sum over axes).  Stops when |dF/dL| < tol.  Returns the
    history of (L, F, dF/dL) and the final fields."""
    L = np.array(L0 if np.ndim(L0) else (L0, L0, L0), dtype=np.float64)
    run = None
    hist = []
    w = (np.asarray(wA, dtype=np.float64).ravel().copy(), np.asarray(wB, dtype=np.float64).ravel().copy())
    for _ in range(n_outer):
        solver.set_cell_para(tuple(L))
        if run is None:
            run = DiblockSCFT(solver, fA, ds, xN, acceptance)
        run.set_fields(*w)
        h = run.iterate(n_inner)
        s = run.stress()
        f = run.get_fields()
        w = (f["wA"], f["wB"])
        g = -s["dlnQ_dL"]
        if cubic:
            gc = float(g.sum())
            hist.append((float(L[0]), float(h["F"][-1]), gc))
            if abs(gc) < tol:
                break
            L = L - step * gc
        else:
            hist.append((L.copy(), float(h["F"][-1]), g.copy()))
            if np.abs(g).max() < tol:
                break
            L = L - step * g
    out = {"history": hist, "L": L}
    out.update(run.get_fields())
    run.close()
    return out


def converge(run, tol: float, max_iter: int = 2000, chunk: int = 25, history: int = 20, beta: float = 0.5):
    """Anderson-mixed iterations (history, beta) until the rms residual of an iteration is
    below tol or max_iter iterations ran; returns (iterations, last residual, last F)."""
    run.set_mixing("anderson", history, beta)
    done, res, F = 0, np.inf, np.nan
    while done < max_iter:
        h = run.iterate(min(chunk, max_iter - done))
        r = run.residuals()
        done += len(r)
        res, F = float(r[-1]), float(h["F"][-1])
        if not np.isfinite(res):
            raise _lib.ScftError(6, "SCFT diverged while converging")
        if res < tol:
            break
    return done, res, F


def relax_cubic_cell(solver, fA, ds, xN, acceptance, wA, wB, L0, tol=1e-8, scf_tol=1e-10, max_eval=40,
                     simple_start=100, history=20, beta=0.5, fp32_tol=None, step0=0.1, max_step=0.4):
    """Variable-cell relaxation of a cubic cell to a stress-free state: at each cell length L
    the SCFT equations are converged (simple mixing for `simple_start` iterations at the
    first cell, then Anderson mixing to an rms residual below scf_tol) and the stress
    dF/dL = -sum_a dlnQ/dL_a comes from the backward pass.  L first moves downhill (against
    the sign of dF/dL) with doubling steps until dF/dL changes sign, then the bracketed root
    is refined by regula falsi (Illinois): a minimum of F(L), not just any zero of the stress.
    fp32_tol: the precision form, converging each cell with FP32 triplets to fp32_tol first
    and polishing in FP64 to scf_tol.  Stops at |dF/dL| <= tol.  Returns the history rows
    (L, F, dF/dL, FP32 iterations, FP64 iterations), the final L, F, stress and fields."""
    run = DiblockSCFT(solver, fA, ds, xN, acceptance)
    state = {"w": (np.asarray(wA, dtype=np.float64).ravel().copy(),
                   np.asarray(wB, dtype=np.float64).ravel().copy()), "first": True}
    hist = []

    def evaluate(L):
        solver.set_cell_para((L, L, L))
        run.set_fields(*state["w"])
        n32 = 0
        if state["first"] and simple_start:
            run.set_precision("fp32" if fp32_tol else "fp64")
            run.set_mixing("simple")
            run.iterate(simple_start)
            n32 += simple_start if fp32_tol else 0
        state["first"] = False
        if fp32_tol:
            run.set_precision("fp32")
            n32 += converge(run, fp32_tol, history=history, beta=beta)[0]
        run.set_precision("fp64")
        n64, _, F = converge(run, scf_tol, history=history, beta=beta)
        g = -float(run.stress()["dlnQ_dL"].sum())
        f = run.get_fields()
        state["w"] = (f["wA"], f["wB"])
        hist.append((L, F, g, n32, n64))
        return g, F

    try:
        L, (g, F) = float(L0), evaluate(float(L0))
        lo = hi = None
        step = step0
        # bracket: walk downhill until the stress changes sign
        while abs(g) > tol and lo is None and len(hist) < max_eval:
            Ln = L - np.sign(g) * step
            gn, Fn = evaluate(Ln)
            if np.sign(gn) != np.sign(g) or abs(gn) <= tol:
                lo, hi = ((L, g), (Ln, gn)) if L < Ln else ((Ln, gn), (L, g))
                L, g, F = Ln, gn, Fn
                break
            L, g, F = Ln, gn, Fn
            step = min(2 * step, max_step)
        # refine: regula falsi with the Illinois modification on [lo, hi] (g(lo) < 0 < g(hi))
        side = 0
        while abs(g) > tol and lo is not None and len(hist) < max_eval:
            (La, ga), (Lb, gb) = lo, hi
            L = (La * gb - Lb * ga) / (gb - ga)
            g, F = evaluate(L)
            if g < 0:
                lo = (L, g)
                if side == -1:
                    hi = (hi[0], hi[1] / 2)
                side = -1
            else:
                hi = (L, g)
                if side == 1:
                    lo = (lo[0], lo[1] / 2)
                side = 1
        out = {"history": hist, "L": L, "F": F, "stress": g}
        out.update(run.get_fields())
        return out
    finally:
        run.close()


def diblock_scft_simple_iterate(Nx, Ny, Nz, fA, ds, xN, Lx, Ly, Lz, acceptance, Nstep, solvername, solver,
                                init_func, verbose: bool = True):
    """src/crysSCFT_sample.cpp:426-531 on the GPU: init_func(wA, wB) fills numpy arrays of
    space_size_phy; prints every 10 iterations and the last (:502-503).  Returns the
    history dict plus the final phi/w fields and the wall time of the loop."""
    M = solver.get_space_size_phy()
    wA = np.empty(M)
    wB = np.empty(M)
    init_func(wA, wB)
    solver.set_cell_para((Lx, Ly, Lz))
    solver.set_contour_step(ds)
    run = DiblockSCFT(solver, fA, ds, xN, acceptance)
    run.set_fields(wA, wB)
    if verbose:
        print("*" * 66)
        print(f"Start solving with solver {solvername}...")
    t0 = time.perf_counter()
    hist = run.iterate(Nstep)
    wall = time.perf_counter() - t0
    if verbose:
        for itr in range(Nstep):
            if itr % 10 == 0 or itr == Nstep - 1:
                eh, e0, e1, ek = hist["parts"][itr]
                print(f"iter {itr}: FreeEnergy = {hist['F'][itr]:.10g} ( {eh:.10g} + {e0:.10g} + {e1:.10g} + "
                      f"{ek:.10g} )  , MaxIncompressibility = {hist['maxinc'][itr]:.10g}")
        print(f"{wall:.6f} s are consumed by {Nstep} iterations")
        print("*" * 66)
    hist.update(run.get_fields())
    hist["wall_seconds"] = wall
    run.close()
    return hist
