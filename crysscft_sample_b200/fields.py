"""Seeded synthetic initial fields (the reference reads BCC_fields_test.txt, which is not
available, src/crysSCFT_sample.cpp:196).

w_A = +A S(r) + noise_A, w_B = -A S(r) + noise_B with
  BCC: S = cx cy + cy cz + cz cx,   FCC: S = cx cy cz,   c. = cos(2 pi . / L),
sampled at x_i = (i + 1/2) L/N, so that every field is mirror-symmetric between grid
points (f[i] = f[N-1-i] on each axis) and valid for all three solvers.  The
Gaussian noise (sigma) is drawn on the first octant only and mirrored.

Random numbers: a counter-based generator (SplitMix64 finaliser applied to
seed ^ stream ^ counter) and the Box-Muller transform, so the fields are
identical on every platform and numpy version.

Layout helpers follow main()'s conventions (src/crysSCFT_sample.cpp:202-258):
P1 uses the full grid, 3M the even sub-lattice f[2i,2j,2k], PMMM the first octant.
"""
from __future__ import annotations

import numpy as np

_M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def _splitmix64(x: np.ndarray) -> np.ndarray:
    with np.errstate(over="ignore"):
        z = x + np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def uniform53(seed: int, stream: int, n: int) -> np.ndarray:
    """n doubles in [0, 1) from (seed, stream, counter)."""
    with np.errstate(over="ignore"):
        key = _splitmix64(np.array([(seed * 0x100000001B3 + stream) & 0xFFFFFFFFFFFFFFFF], dtype=np.uint64))[0]
        ctr = np.arange(n, dtype=np.uint64) * np.uint64(0xD1B54A32D192ED03)
        bits = _splitmix64(ctr ^ key)
    return (bits >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def gaussian(seed: int, stream: int, n: int) -> np.ndarray:
    """n standard normals by Box-Muller."""
    m = (n + 1) // 2
    u1 = uniform53(seed, 2 * stream, m)
    u2 = uniform53(seed, 2 * stream + 1, m)
    r = np.sqrt(-2.0 * np.log1p(-u1))
    z = np.concatenate([r * np.cos(2 * np.pi * u2), r * np.sin(2 * np.pi * u2)])
    return z[:n]


def mirror_extend(octant: np.ndarray) -> np.ndarray:
    """Full grid from its first octant with f[i] = f[N-1-i] on every axis."""
    f = np.concatenate([octant, octant[::-1]], axis=0)
    f = np.concatenate([f, f[:, ::-1]], axis=1)
    return np.concatenate([f, f[:, :, ::-1]], axis=2)


def seed_fields(N, L, phase: str = "BCC", A: float = 2.0, sigma: float = 0.01, seed: int = 20261203):
    """Full-grid (N0, N1, N2) fields wA, wB (all N even)."""
    N = tuple(int(v) for v in N)
    L = tuple(float(v) for v in (L if np.ndim(L) else (L, L, L)))
    if any(v % 2 for v in N):
        raise ValueError("grid sizes must be even")
    oct_shape = tuple(v // 2 for v in N)
    # evaluated on the first octant and mirrored, so the symmetry holds bit for bit
    c = [np.cos(2 * np.pi * (np.arange(oct_shape[d]) + 0.5) / N[d]) for d in range(3)]
    cx, cy, cz = c[0][:, None, None], c[1][None, :, None], c[2][None, None, :]
    if phase.upper() == "BCC":
        S = cx * cy + cy * cz + cz * cx
    elif phase.upper() == "FCC":
        S = cx * cy * cz
    else:
        raise ValueError("phase must be BCC or FCC")
    S = np.broadcast_to(S, oct_shape)
    n = int(np.prod(oct_shape))
    nA = sigma * gaussian(seed, 0, n).reshape(oct_shape)
    nB = sigma * gaussian(seed, 1, n).reshape(oct_shape)
    wA = np.ascontiguousarray(mirror_extend(A * S + nA))
    wB = np.ascontiguousarray(mirror_extend(-A * S + nB))
    return wA, wB


def write_fields_text(path: str, phiA, phiB, wA, wB, precision: int = 6) -> None:
    """The reference's output_fields format (src/crysSCFT_sample.cpp:271-282): one line
    "phiA phiB wA wB" per grid point, x slowest, z fastest.  The reference streams doubles
    with the default ostream format (6 significant digits, %g style); pass precision=17
    for a lossless file."""
    cols = [np.asarray(a, dtype=np.float64).ravel() for a in (phiA, phiB, wA, wB)]
    fmt = f"%.{int(precision)}g"
    with open(path, "w") as f:
        for i in range(cols[0].size):
            f.write(" ".join(fmt % c[i] for c in cols) + "\n")


def read_fields_text(path: str, size: int):
    """The reference's input_fields (src/crysSCFT_sample.cpp:284-292): reads `size` points
    of "phiA phiB wA wB" (any whitespace); returns the four arrays."""
    with open(path) as f:
        vals = np.array(f.read().split()[: 4 * size], dtype=np.float64)
    if vals.size < 4 * size:
        raise ValueError(f"{path}: {vals.size // 4} points, expected {size}")
    v = vals.reshape(size, 4)
    return v[:, 0].copy(), v[:, 1].copy(), v[:, 2].copy(), v[:, 3].copy()


def to_physical(kind: str, full: np.ndarray) -> np.ndarray:
    """main()'s per-solver field extraction (src/crysSCFT_sample.cpp:202-258)."""
    kind = kind.upper()
    if kind == "P1":
        return np.ascontiguousarray(full)
    if kind == "3M":
        return np.ascontiguousarray(full[::2, ::2, ::2])
    n0, n1, n2 = (v // 2 for v in full.shape)
    return np.ascontiguousarray(full[:n0, :n1, :n2])


def m3_mirror(b: int, p, g, N):
    """The mirror normal to axis b of the 3m group with translations g
    (generate_m3_operation, src/solver_utilities.h:56-66: g[0..2] belong to the mirror
    normal to z, g[3..5] to y, g[6..8] to x), on integer grid coordinates p = (x, y, z):
    p_b -> -p_b - 1 + g_b N_b (the plane lies between grid points), p_a -> p_a + g_a N_a."""
    t = g[3 * (2 - b): 3 * (2 - b) + 3]
    out = []
    for a in range(3):
        s = int(round(t[a] * N[a]))
        out.append(((-p[a] - 1 + s) if a == b else (p[a] + s)) % N[a])
    return tuple(out)


def extend_3m(phy: np.ndarray, N, g=(0.0,) * 9) -> np.ndarray:
    """The full-grid field of the 3m group with translations g whose even sub-lattice
    f[2i, 2j, 2k] is `phy` (the 3m solver's physical grid): each of the eight group
    elements m_x^cx m_y^cy m_z^cz (z applied first) carries the even sub-lattice onto one
    parity class.  Raises if the translations do not tile the grid that way."""
    N = tuple(int(v) for v in N)
    phy = np.asarray(phy).reshape(tuple(v // 2 for v in N))
    idx = np.meshgrid(*[2 * np.arange(v // 2) for v in N], indexing="ij")
    full = np.empty(N, dtype=phy.dtype)
    seen = np.zeros(N, dtype=np.int8)
    for c in range(8):
        p = tuple(idx)
        for b, bit in ((2, 1), (1, 2), (0, 4)):
            if c & bit:
                p = m3_mirror(b, p, g, N)
        full[p] = phy
        seen[p] += 1
    if not np.all(seen == 1):
        raise ValueError("the mirror translations do not carry the even sub-lattice onto the other parity classes")
    return full


def from_physical(kind: str, phy: np.ndarray, N) -> np.ndarray:
    """Inverse of to_physical for mirror-symmetric fields."""
    kind = kind.upper()
    if kind == "P1":
        return np.asarray(phy).reshape(N)
    if kind == "PMMM":
        return mirror_extend(np.asarray(phy).reshape(tuple(v // 2 for v in N)))
    # 3M: even sub-lattice point 2i; its mirror partner N-1-2i is odd
    full = np.empty(N)
    ev = np.asarray(phy).reshape(tuple(v // 2 for v in N))
    idx = [np.empty(N[d], dtype=np.int64) for d in range(3)]
    for d in range(3):
        i = np.arange(N[d] // 2)
        idx[d][2 * i] = i
        idx[d][N[d] - 1 - 2 * i] = i
    full[...] = ev[np.ix_(idx[0], idx[1], idx[2])]
    return full
