"""Python mirror of the reference's diffusion-solver plugin interface, backed by the
B200 library's C ABI.

The classes keep the reference's names and methods (src/solver_base.h:8-51):
``set_cell_para``, ``set_contour_step``, ``diffusion``, ``get_iomat_for_diffusion``
and the size/cell/ds getters.  ``get_iomat_for_diffusion()`` returns a numpy view
of the solver-owned (pinned) host buffer, so driver code that writes the buffer,
calls ``diffusion()`` and reads it back works unchanged.  Device-side extras take
torch CUDA tensors.

Errors: where the reference prints "ERROR" and calls exit(1), these classes raise
``ScftError`` carrying the C status code.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import ScftError, check

__all__ = ["CrysPSSolverBase", "CrysPSSolverP1", "CrysPSSolver3m", "CrysPSSolverPmmm", "ScftError"]


class CrysPSSolverBase:
    """src/solver_base.h:8-51 — construct one of the subclasses."""

    _kind = None

    def __init__(self, grid_size_log, translational_part=None, precision: str = "fp64", device: int = -1):
        L = _lib.load()
        grid = (ctypes.c_size_t * 3)(*[int(v) for v in grid_size_log])
        g = None
        if translational_part is not None:
            self._g = np.ascontiguousarray(translational_part, dtype=np.float64)
            if self._g.size != 9:
                raise ValueError("translational_part needs 9 values")
            g = _lib.dptr(self._g)
        h = ctypes.c_void_p()
        check(L.scft_solver_create(_lib.KIND[self._kind], grid, g, _lib.PRECISION[precision], int(device),
                                   ctypes.byref(h)))
        self._h = h
        self.precision = precision
        self._grid_log = tuple(int(v) for v in grid_size_log)
        out = (ctypes.c_size_t * 3)()
        check(L.scft_solver_get_grid_size_phy(self._h, out))
        self._grid_phy = tuple(int(v) for v in out)
        self._space_phy = int(np.prod(self._grid_phy))
        p = ctypes.POINTER(ctypes.c_double)()
        check(L.scft_solver_get_iomat_for_diffusion(self._h, ctypes.byref(p)))
        self._iomat = np.ctypeslib.as_array(p, shape=(self._space_phy,))

    # -- lifetime --------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            _lib.load().scft_solver_destroy(self._h)
            self._h = None
            self._iomat = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    # -- virtuals of src/solver_base.h:16-20 --------------------------------
    def set_cell_para(self, cell_para):
        c = np.zeros(6)
        c[: len(cell_para)] = cell_para
        check(_lib.load().scft_solver_set_cell_para(self._h, _lib.dptr(c)))

    def set_contour_step(self, ds: float):
        check(_lib.load().scft_solver_set_contour_step(self._h, float(ds)))

    def diffusion(self):
        """One triplet on get_iomat_for_diffusion(), in place."""
        check(_lib.load().scft_solver_diffusion(self._h))

    # -- getters of src/solver_base.h:22-28 ---------------------------------
    def get_cell_para(self):
        c = np.zeros(6)
        check(_lib.load().scft_solver_get_cell_para(self._h, _lib.dptr(c)))
        return tuple(c)

    def get_grid_size_log(self):
        return self._grid_log

    def get_grid_size_phy(self):
        return self._grid_phy

    def get_space_size_log(self):
        return int(np.prod(self._grid_log))

    def get_space_size_phy(self):
        return self._space_phy

    def get_ds(self):
        v = ctypes.c_double()
        check(_lib.load().scft_solver_get_ds(self._h, ctypes.byref(v)))
        return v.value

    def get_iomat_for_diffusion(self) -> np.ndarray:
        return self._iomat

    # -- device-resident extras ---------------------------------------------
    def set_stream(self, stream=None):
        """Issue work on a torch.cuda.Stream (or raw cudaStream_t); None = the solver's own."""
        check(_lib.load().scft_solver_set_stream(self._h, _stream_ptr(stream)))

    def diffusion_device(self, t, stream=None):
        """One triplet in place on a torch float64 CUDA tensor of space_size_phy elements."""
        _check_tensor(t, self._space_phy)
        check(_lib.load().scft_solver_diffusion_device(self._h, ctypes.c_void_p(t.data_ptr()),
                                                       _stream_ptr(stream)))

    def propagate_device(self, q, init, wds, Ns: int, direction: int, stream=None):
        """solve_diffusion_equation on torch CUDA tensors (q: (Ns+1)*space_size_phy)."""
        _check_tensor(q, (Ns + 1) * self._space_phy)
        _check_tensor(init, self._space_phy)
        _check_tensor(wds, self._space_phy)
        check(_lib.load().scft_solver_propagate_device(
            self._h, ctypes.c_void_p(q.data_ptr()), ctypes.c_void_p(init.data_ptr()),
            ctypes.c_void_p(wds.data_ptr()), int(Ns), int(direction), _stream_ptr(stream)))


class CrysPSSolverP1(CrysPSSolverBase):
    """CrysPSSolverP1 (src/solver_p1.h:14-53): full grid, no symmetry."""

    _kind = "P1"

    def __init__(self, grid_size_log, precision: str = "fp64", device: int = -1):
        super().__init__(grid_size_log, None, precision, device)


class CrysPSSolver3m(CrysPSSolverBase):
    """CrysPSSolver3m (src/solver_3m.h:14-53): even sub-lattice of a field with three
    perpendicular mirror planes (the 2x2y2z algorithm)."""

    _kind = "3M"

    def __init__(self, grid_size_log, translational_part=(0.0,) * 9, precision: str = "fp64", device: int = -1):
        super().__init__(grid_size_log, translational_part, precision, device)


class CrysPSSolverPmmm(CrysPSSolverBase):
    """CrysPSSolverPmmm (src/solver_Pmmm.h:13-53): first octant, DCT-II/III; cubic cell."""

    _kind = "PMMM"

    def __init__(self, grid_size_log, precision: str = "fp64", device: int = -1, anisotropic: bool = False):
        super().__init__(grid_size_log, None, precision, device)
        self.anisotropic = bool(anisotropic)
        if anisotropic:
            # orthorhombic cell (Lx, Ly, Lz); the reference's PMMM solver is cubic
            check(_lib.load().scft_solver_set_pmmm_anisotropic(self._h, 1))


def make_solver(kind: str, grid_size_log, precision: str = "fp64", device: int = -1) -> CrysPSSolverBase:
    kind = kind.upper()
    cls = {"P1": CrysPSSolverP1, "3M": CrysPSSolver3m, "PMMM": CrysPSSolverPmmm}[kind]
    return cls(grid_size_log, precision=precision, device=device)


def operator_terms(kind: str, grid_size_log, cell, ds: float, translational_part=None):
    """The per-axis factors [(A_x, A_y, A_z), ...] of the triplet the solver builds
    (sum over terms of A_x (x) A_y (x) A_z on the physical grid).  Host-only: needs the
    library but no GPU.  `cell` is used as given (also for PMMM)."""
    L = _lib.load()
    kind = kind.upper()
    grid = (ctypes.c_size_t * 3)(*[int(v) for v in grid_size_log])
    g = None
    if translational_part is not None:
        gg = np.ascontiguousarray(translational_part, dtype=np.float64)
        if gg.size != 9:
            raise ValueError("translational_part needs 9 values")
        g = _lib.dptr(gg)
    c = np.ascontiguousarray(cell[:3], dtype=np.float64)
    nt = ctypes.c_size_t()
    check(L.scft_operator_terms(_lib.KIND[kind], grid, g, _lib.dptr(c), float(ds), ctypes.byref(nt), None, 0))
    n = [int(v) if kind == "P1" else int(v) // 2 for v in grid_size_log]
    buf = np.zeros(nt.value * sum(v * v for v in n))
    check(L.scft_operator_terms(_lib.KIND[kind], grid, g, _lib.dptr(c), float(ds), ctypes.byref(nt),
                                _lib.dptr(buf), buf.size))
    out, o = [], 0
    for _ in range(nt.value):
        fac = []
        for v in n:
            fac.append(buf[o:o + v * v].reshape(v, v))
            o += v * v
        out.append(tuple(fac))
    return out


def _check_tensor(t, n):
    import torch

    if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.float64 and t.is_contiguous()):
        raise ValueError("expected a contiguous float64 CUDA tensor")
    if t.numel() < n:
        raise ValueError(f"tensor has {t.numel()} elements, need {n}")


def _stream_ptr(stream):
    if stream is None:
        return None
    return ctypes.c_void_p(int(getattr(stream, "cuda_stream", stream)))
