"""ctypes binding of the reference built as a CPU library — TEST INFRASTRUCTURE ONLY.

``oracle/_ref/libscft_ref.so`` is the reference program's own
``src/crysSCFT_sample.cpp`` (with the three solver headers) compiled unmodified
by ``oracle/Makefile`` against the FFTW-API shim in ``oracle/fftw_shim``.
Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline legs of
``bench.py`` use this module, and only as the checker or the timed CPU arm.

Solver kinds follow the reference's three classes:
``P1`` (src/solver_p1.h), ``3M`` (src/solver_3m.h), ``PMMM`` (src/solver_Pmmm.h).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libscft_ref.so")
SHIM_PATH = os.path.join(_HERE, "_ref", "libfftw_shim.so")
KINDS = {"P1": 0, "3M": 1, "PMMM": 2}

_lib = None
_dp = ctypes.POINTER(ctypes.c_double)


GPU_DRIVER_PATH = os.path.join(_HERE, "_ref", "libref_gpu_driver.so")


def reference_src() -> str:
    """The reference's src/ directory: $CRYSSCFT_REFERENCE/src, by default a checkout named
    `reference` beside this repository."""
    root = os.environ.get("CRYSSCFT_REFERENCE") or os.path.join(os.path.dirname(os.path.dirname(_HERE)), "reference")
    return os.path.join(root, "src")


def build(ref_src: str | None = None) -> None:
    """Compile oracle/_ref/ from the reference sources (only where they exist); the
    reference-driver-over-GPU-adapters library too when the CUDA library is built."""
    ref_src = ref_src or reference_src()
    if not os.path.isdir(ref_src):
        return
    targets = ["all", "shim"]
    gpulib = os.path.join(os.path.dirname(_HERE), "crysscft_sample_b200", "_lib", "libcrysscft_b200.so")
    if os.path.exists(gpulib):
        targets.append("gpu_driver")
    subprocess.run(["make", "-s", "-C", _HERE, f"REF_SRC={ref_src}"] + targets, check=True)


def run_reference_driver_on_gpu(kind: str, grid_log, fA, ds, xN, L, acceptance, nstep, wA0, wB0, name: str) -> str:
    """The reference's unmodified diblock_scft_simple_iterate over the GPU solver adapters
    (include/crysscft_b200_solvers.hpp); returns what the driver prints."""
    check_grid(kind.upper(), grid_log)
    G = ctypes.CDLL(GPU_DRIVER_PATH)
    G.refgpu_run_driver.restype = ctypes.c_long
    G.refgpu_run_driver.argtypes = ([ctypes.c_int] + [ctypes.c_long] * 3 + [ctypes.c_double] * 7
                                    + [ctypes.c_long, _dp, _dp, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_long])
    buf = ctypes.create_string_buffer(1 << 16)
    wA0 = np.ascontiguousarray(wA0, dtype=np.float64).ravel()
    wB0 = np.ascontiguousarray(wB0, dtype=np.float64).ravel()
    nx, ny, nz = (int(v) for v in grid_log)
    G.refgpu_run_driver(KINDS[kind.upper()], nx, ny, nz, fA, ds, xN, L[0], L[1], L[2], acceptance, int(nstep),
                        _p(wA0), _p(wB0), name.encode(), buf, len(buf))
    return buf.value.decode()


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        L.ref_solver_create.restype = ctypes.c_void_p
        L.ref_solver_create.argtypes = [ctypes.c_int, ctypes.c_long, ctypes.c_long, ctypes.c_long, _dp]
        L.ref_solver_destroy.argtypes = [ctypes.c_void_p]
        L.ref_solver_set_cell_para.argtypes = [ctypes.c_void_p, _dp]
        L.ref_solver_set_contour_step.argtypes = [ctypes.c_void_p, ctypes.c_double]
        L.ref_solver_space_size_phy.restype = ctypes.c_long
        L.ref_solver_space_size_phy.argtypes = [ctypes.c_void_p]
        L.ref_solver_grid_size_phy.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_long)]
        L.ref_solver_diffusion.argtypes = [ctypes.c_void_p, _dp]
        L.ref_solve_diffusion_equation.restype = ctypes.c_double
        L.ref_solve_diffusion_equation.argtypes = [ctypes.c_void_p, _dp, _dp, _dp, ctypes.c_long, ctypes.c_int]
        L.ref_array_exp.argtypes = [_dp, _dp, ctypes.c_double, ctypes.c_double, ctypes.c_long]
        L.ref_calc_ksi.argtypes = [_dp, _dp, _dp, ctypes.c_long, ctypes.c_double]
        L.ref_integrate_phi.argtypes = [_dp, _dp, _dp, ctypes.c_double, ctypes.c_double, ctypes.c_long, ctypes.c_long]
        L.ref_calc_new_fields.argtypes = [_dp, _dp, _dp, _dp, _dp, ctypes.c_double, ctypes.c_double, ctypes.c_long]
        L.ref_array_average.restype = ctypes.c_double
        L.ref_array_average.argtypes = [_dp, ctypes.c_long]
        L.ref_energy_terms.argtypes = [ctypes.c_double, ctypes.c_double, _dp, _dp, _dp, _dp, _dp, ctypes.c_long, _dp, _dp]
        L.ref_scft_run.restype = ctypes.c_double
        L.ref_scft_run.argtypes = [ctypes.c_void_p] + [ctypes.c_double] * 7 + [ctypes.c_long] + [_dp] * 11
        L.ref_run_driver.restype = ctypes.c_long
        L.ref_run_driver.argtypes = ([ctypes.c_void_p, ctypes.c_long, ctypes.c_long, ctypes.c_long]
                                     + [ctypes.c_double] * 7 + [ctypes.c_long, _dp, _dp,
                                                                ctypes.c_char_p, ctypes.c_char_p, ctypes.c_long])
        L.ref_output_fields.argtypes = [_dp] * 4 + [ctypes.c_long, ctypes.c_char_p]
        L.ref_input_fields.argtypes = [_dp] * 4 + [ctypes.c_long, ctypes.c_char_p]
        L.ref_set_num_threads.argtypes = [ctypes.c_int]
        L.ref_get_max_threads.restype = ctypes.c_int
        _lib = L
    return _lib


def _p(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_dp)


def check_grid(kind: str, grid_log) -> None:
    """The reference constructors print "ERROR" and call exit(1) on these grids
    (src/solver_p1.h:101-108, src/solver_3m.h:81-92, src/solver_Pmmm.h:71-82);
    refuse them here so the calling process survives."""
    Nx, Ny, Nz = (int(v) for v in grid_log)
    if min(Nx, Ny, Nz) <= 0:
        raise ValueError("ERROR: Bad Grid Size")
    if kind == "P1":
        if Nz % 8:
            raise ValueError("ERROR: Bad Grid Size For Group Triclinic P1, alignment cannot be guaranteed")
    else:
        if Nx % 2 or Ny % 2 or Nz % 2:
            raise ValueError("ERROR: Grid Size Must Be Even")
        if (Nz // 2) % 8:
            raise ValueError("ERROR: Bad Grid Size, Alignment Cannot Be Guaranteed")


def set_num_threads(n: int) -> None:
    lib().ref_set_num_threads(int(n))


def max_threads() -> int:
    return int(lib().ref_get_max_threads())


class RefSolver:
    """One of the reference's CrysPSSolverBase implementations, driven through ctypes."""

    def __init__(self, kind: str, grid_log, translational_part=None):
        self.kind = kind.upper()
        check_grid(self.kind, grid_log)
        g = None
        if translational_part is not None:
            self._g = np.ascontiguousarray(translational_part, dtype=np.float64)
            g = _p(self._g)
        self.h = lib().ref_solver_create(KINDS[self.kind], int(grid_log[0]), int(grid_log[1]), int(grid_log[2]), g)
        self.grid_log = tuple(int(v) for v in grid_log)

    def close(self):
        if self.h:
            lib().ref_solver_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def space_size_phy(self) -> int:
        return int(lib().ref_solver_space_size_phy(self.h))

    @property
    def grid_size_phy(self):
        out = (ctypes.c_long * 3)()
        lib().ref_solver_grid_size_phy(self.h, out)
        return tuple(int(v) for v in out)

    def set_cell_para(self, cell):
        c = np.zeros(6)
        c[: len(cell)] = cell
        lib().ref_solver_set_cell_para(self.h, _p(c))

    def set_contour_step(self, ds: float):
        lib().ref_solver_set_contour_step(self.h, float(ds))

    def diffusion(self, q: np.ndarray) -> np.ndarray:
        io = np.ascontiguousarray(q, dtype=np.float64).copy()
        lib().ref_solver_diffusion(self.h, _p(io))
        return io

    def solve_diffusion_equation(self, init, wds, Ns: int, direction: int) -> np.ndarray:
        M = self.space_size_phy
        q = np.zeros((Ns + 1) * M)
        init = np.ascontiguousarray(init, dtype=np.float64).ravel()
        wds = np.ascontiguousarray(wds, dtype=np.float64).ravel()
        lib().ref_solve_diffusion_equation(self.h, _p(q), _p(init), _p(wds), int(Ns), int(direction))
        return q.reshape(Ns + 1, M)

    def scft_run(self, fA, ds, xN, L, acceptance, nstep, wA0, wB0):
        """The driver's iteration loop (src/crysSCFT_sample.cpp:440-508) on this solver."""
        M = self.space_size_phy
        out = {k: np.zeros(nstep) for k in ("F", "maxinc", "Q")}
        parts = np.zeros(4 * nstep)
        phiA, phiB, wA, wB = (np.zeros(M) for _ in range(4))
        tcpu = np.zeros(1)
        wA0 = np.ascontiguousarray(wA0, dtype=np.float64).ravel()
        wB0 = np.ascontiguousarray(wB0, dtype=np.float64).ravel()
        wall = lib().ref_scft_run(self.h, fA, ds, xN, L[0], L[1], L[2], acceptance, int(nstep),
                                  _p(wA0), _p(wB0), _p(out["F"]), _p(parts), _p(out["maxinc"]),
                                  _p(out["Q"]), _p(phiA), _p(phiB), _p(wA), _p(wB), _p(tcpu))
        out.update(parts=parts.reshape(nstep, 4), phiA=phiA, phiB=phiB, wA=wA, wB=wB,
                   wall_seconds=wall, triplet_cpu_seconds=float(tcpu[0]))
        return out

    def run_driver(self, fA, ds, xN, L, acceptance, nstep, wA0, wB0, name: str) -> str:
        """The reference's unmodified diblock_scft_simple_iterate; returns its stdout."""
        buf = ctypes.create_string_buffer(1 << 16)
        wA0 = np.ascontiguousarray(wA0, dtype=np.float64).ravel()
        wB0 = np.ascontiguousarray(wB0, dtype=np.float64).ravel()
        nx, ny, nz = self.grid_log
        lib().ref_run_driver(self.h, nx, ny, nz, fA, ds, xN, L[0], L[1], L[2], acceptance, int(nstep),
                             _p(wA0), _p(wB0), name.encode(), buf, len(buf))
        return buf.value.decode()


def parse_driver_log(text: str):
    """(iteration, F, maxinc) rows from print_energy lines (src/crysSCFT_sample.cpp:420-423)."""
    rows = []
    for line in text.splitlines():
        if line.startswith("iter ") and "FreeEnergy" in line:
            it = int(line.split()[1].rstrip(":"))
            F = float(line.split("FreeEnergy = ")[1].split()[0])
            mi = float(line.split("MaxIncompressibility = ")[1].split()[0])
            rows.append((it, F, mi))
    return rows
