"""CPU restatement of the reference's hot path in numpy — TEST INFRASTRUCTURE ONLY.

This module is the oracle: tests, ``__graft_entry__.smoke()`` and the CPU
baseline of ``bench.py`` use it as the checker; the product never imports it.
Transforms use numpy.fft / scipy.fft, whose unnormalised r2c, c2r, DCT-II and
DCT-III follow the same published definitions as FFTW 3.3.3's r2c, c2r,
REDFT10 and REDFT01 (FFTW manual section 4.8), which the reference calls.

Parity pin: every function here is checked in tests/test_oracle.py against
the reference itself compiled as ``oracle/_ref/libscft_ref.so`` (the
reference's own sources + an FFTW-API shim) and against the committed golden
vectors in tests/golden/.

Layout: every field is a C-ordered (nx, ny, nz) array (x slowest, z fastest),
as in the reference.
"""
from __future__ import annotations

import math

import numpy as np
import scipy.fft as sfft

PI = 3.1415926535897932384626  # src/solver_base.h:5


# --------------------------------------------------------------------------
# diffusion operators (the "triplet")
# --------------------------------------------------------------------------
def p1_kmat(N, L, ds):
    """K for the full-grid real FFT, src/solver_p1.h:142-172.

    kx = 2 pi min(i, N-i) / Lx (same for y), kz = 2 pi k / Lz for k <= Nz/2;
    K = exp(-ds (kx^2 + ky^2 + kz^2)) on the r2c half spectrum.
    """
    Nx, Ny, Nz = N
    Lx, Ly, Lz = L
    kx = np.array([2 * PI * (i if i < (Nx + 1) // 2 else Nx - i) / Lx for i in range(Nx)]) ** 2
    ky = np.array([2 * PI * (j if j < (Ny + 1) // 2 else Ny - j) / Ly for j in range(Ny)]) ** 2
    kz = np.array([2 * PI * k / Lz for k in range(Nz // 2 + 1)]) ** 2
    return np.exp(-ds * (kx[:, None, None] + ky[None, :, None] + kz[None, None, :]))


def p1_diffusion(q, K):
    """CrysPSSolverP1::diffusion, src/solver_p1.h:83-93 and xyz_routine :184-202:
    r2c -> multiply by K -> c2r (unnormalised) -> multiply by 1/(Nx Ny Nz)."""
    N = q.shape
    spec = np.fft.rfftn(q, axes=(0, 1, 2)) * K
    # irfftn normalises by 1/(Nx Ny Nz): the same as the unnormalised c2r followed by :87-92
    return np.fft.irfftn(spec, s=N, axes=(0, 1, 2))


def pmmm_kmat(n_log, L, ds):
    """K for the DCT solver, src/solver_Pmmm.h:159-186 (cubic: only L[0] is used, :101)."""
    Nx, Ny, Nz = n_log
    Lc = L[0]
    kx = np.array([2 * PI * i / Lc for i in range(Nx // 2)]) ** 2
    ky = np.array([2 * PI * j / Lc for j in range(Ny // 2)]) ** 2
    kz = np.array([2 * PI * k / Lc for k in range(Nz // 2)]) ** 2
    return np.exp(-(kx[:, None, None] + ky[None, :, None] + kz[None, None, :]) * ds)


def pmmm_diffusion(q, K, n_log):
    """CrysPSSolverPmmm::diffusion, src/solver_Pmmm.h:125-143 and xyz_routine :194-215:
    REDFT10 3-D -> multiply by K -> REDFT01 3-D -> multiply by 1/(Nx Ny Nz) (full logical size)."""
    step1 = sfft.dctn(q, type=2, axes=(0, 1, 2))
    step2 = step1 * K
    out = sfft.dctn(step2, type=3, axes=(0, 1, 2))
    return out * (1.0 / (n_log[0] * n_log[1] * n_log[2]))


def m3_operations(g, s):
    """generate_m3_operation, src/solver_utilities.h:56-66 (7 mirror combinations)."""
    P2 = 2.0 * PI
    return [
        (-P2 * g[0], -P2 * g[1], -P2 * (g[2] - 1.0 / s[2])),
        (-P2 * g[3], -P2 * (g[4] - 1.0 / s[1]), -P2 * g[5]),
        (-P2 * (g[0] + g[3]), -P2 * (-g[1] + g[4] - 1.0 / s[1]), -P2 * (g[2] + g[5] - 1.0 / s[2])),
        (-P2 * (g[6] - 1.0 / s[0]), -P2 * g[7], -P2 * g[8]),
        (-P2 * (g[6] - g[0] - 1.0 / s[0]), -P2 * (g[1] + g[7]), -P2 * (g[2] + g[8] - 1.0 / s[2])),
        (-P2 * (-g[3] + g[6] - 1.0 / s[0]), -P2 * (g[4] + g[7] - 1.0 / s[1]), -P2 * (g[5] + g[8])),
        (-P2 * (-g[0] - g[3] + g[6] - 1.0 / s[0]), -P2 * (-g[1] + g[4] + g[7] - 1.0 / s[1]),
         -P2 * (g[2] + g[5] + g[8] - 1.0 / s[2])),
    ]


def m3_twiddles(n_log, g):
    """R_mat_generator_full, src/solver_3m.h:172-182 with twiddle_factor,
    src/solver_utilities.h:27-53: r[0] = 1, r[p] = exp(i (x a + y b + z c))."""
    Nx, Ny, Nz = n_log
    h = (Nx // 2, Ny // 2, Nz // 2)
    x = np.arange(h[0])[:, None, None]
    y = np.arange(h[1])[None, :, None]
    z = np.arange(h[2])[None, None, :]
    r_re = [np.ones(h)]
    r_im = [np.zeros(h)]
    for (a, b, c) in m3_operations(g, n_log):
        ang = x * a + y * b + z * c
        r_re.append(np.cos(ang))
        r_im.append(np.sin(ang))
    return r_re, r_im


def m3_kmat(n_log, L, ds, g=(0.0,) * 9):
    """CrysPSSolver3m::K_mat_generator, src/solver_3m.h:184-255.

    Full-size K x 1/(NxNyNz); split into 8 octants (src/solver_utilities.h:74-98,
    part bit 4 = x high, 2 = y high, 1 = z high); three add/sub (Walsh-Hadamard)
    passes (:244-246); mul_add_sub_by_seq with the twiddles for the pairs
    {0,7},{6,1},{2,5},{4,3} (:248-250, src/solver_utilities.h:165-208).
    Returns k_re[8], k_im[8], each (Nx/2, Ny/2, Nz/2).
    """
    Nx, Ny, Nz = n_log
    Lx, Ly, Lz = L
    fx = (2.0 * PI / Lx) ** 2
    fy = (2.0 * PI / Ly) ** 2
    fz = (2.0 * PI / Lz) ** 2
    ix = np.arange(Nx); ix = np.where(ix > Nx // 2, Nx - ix, ix)
    iy = np.arange(Ny); iy = np.where(iy > Ny // 2, Ny - iy, iy)
    iz = np.arange(Nz); iz = np.where(iz > Nz // 2, Nz - iz, iz)
    kx = ix * ix * fx
    ky = iy * iy * fy
    kz = iz * iz * fz
    factor = 1.0 / (Nx * Ny * Nz)
    temp = np.exp(-(kx[:, None, None] + ky[None, :, None] + kz[None, None, :]) * ds) * factor
    hx, hy, hz = Nx // 2, Ny // 2, Nz // 2
    ks = []
    for part in range(8):
        bx, by, bz = (part >> 2) & 1, (part >> 1) & 1, part & 1
        ks.append(temp[bx * hx:bx * hx + hx, by * hy:by * hy + hy, bz * hz:bz * hz + hz].copy())
    for seq in ([(0, 4), (1, 5), (2, 6), (3, 7)], [(0, 2), (1, 3), (4, 6), (5, 7)],
                [(0, 1), (2, 3), (4, 5), (6, 7)]):
        for a, b in seq:
            t = ks[a] + ks[b]
            ks[b] = ks[a] - ks[b]
            ks[a] = t
    r_re, r_im = m3_twiddles(n_log, g)
    k_re = [None] * 8
    k_im = [None] * 8
    for a, b in ((0, 7), (6, 1), (2, 5), (4, 3)):
        dre0, dim0 = ks[a] * r_re[a], ks[a] * r_im[a]
        dre1, dim1 = ks[b] * r_re[b], ks[b] * r_im[b]
        k_re[a], k_re[b] = dre0 + dre1, dre0 - dre1
        k_im[a], k_im[b] = dim0 + dim1, dim0 - dim1
    return k_re, k_im


def m3_diffusion(q, k_re, k_im):
    """CrysPSSolver3m::xyz_routine, src/solver_3m.h:281-324: half-size r2c, the
    4-source recombination (:292-322), half-size c2r (unnormalised; 1/N^3 is in K)."""
    n = q.shape
    X = np.fft.rfftn(q, axes=(0, 1, 2))  # (n0, n1, n2//2+1)
    h = X.shape[2]
    xi = np.arange(n[0])
    yi = np.arange(n[1])
    mx = (n[0] - xi) % n[0]
    my = (n[1] - yi) % n[1]
    s000 = X
    s110 = X[mx][:, my]
    s010 = X[:, my]
    s100 = X[mx]
    kr = [k[:, :, :h] for k in k_re]
    ki = [k[:, :, :h] for k in k_im]
    re = (s000.real * kr[0] - s000.imag * ki[7] + s110.real * kr[6] - s110.imag * ki[1]
          + s010.real * kr[2] - s010.imag * ki[5] + s100.real * kr[4] - s100.imag * ki[3])
    im = (s000.real * ki[0] + s000.imag * kr[7] + s110.real * ki[6] + s110.imag * kr[1]
          + s010.real * ki[2] + s010.imag * kr[5] + s100.real * ki[4] + s100.imag * kr[3])
    Y = re + 1j * im
    return np.fft.irfftn(Y, s=n, axes=(0, 1, 2)) * (n[0] * n[1] * n[2])


class OracleSolver:
    """CrysPSSolverBase restated: kind in {"P1", "3M", "PMMM"}; q is the physical grid."""

    def __init__(self, kind, grid_log, translational_part=(0.0,) * 9):
        self.kind = kind.upper()
        self.grid_log = tuple(int(v) for v in grid_log)
        self.g = tuple(translational_part)
        if self.kind == "P1":
            self.grid_phy = self.grid_log
        else:
            self.grid_phy = tuple(v // 2 for v in self.grid_log)
        self.cell = (4.0, 4.0, 4.0)
        self.ds = None

    @property
    def space_size_phy(self):
        return int(np.prod(self.grid_phy))

    def set_cell_para(self, cell):
        if self.kind == "PMMM":  # src/solver_Pmmm.h:98-104: cubic, only cell[0]
            self.cell = (cell[0],) * 3
        else:
            self.cell = tuple(cell[:3])
        self.ds = None

    def set_contour_step(self, ds):
        self.ds = ds
        if self.kind == "P1":
            self.K = p1_kmat(self.grid_log, self.cell, ds)
        elif self.kind == "PMMM":
            self.K = pmmm_kmat(self.grid_log, self.cell, ds)
        else:
            self.K = m3_kmat(self.grid_log, self.cell, ds, self.g)

    def diffusion(self, q):
        q = np.asarray(q, dtype=np.float64).reshape(self.grid_phy)
        if self.kind == "P1":
            return p1_diffusion(q, self.K)
        if self.kind == "PMMM":
            return pmmm_diffusion(q, self.K, self.grid_log)
        return m3_diffusion(q, *self.K)


# --------------------------------------------------------------------------
# contour loop and SCFT iteration (src/crysSCFT_sample.cpp)
# --------------------------------------------------------------------------
def solve_diffusion_equation(solver, init, wds, Ns, direction):
    """src/crysSCFT_sample.cpp:373-396.  Returns q[(Ns+1), *grid]; direction +1 fills
    slots 0..Ns, -1 fills Ns..0.  Each step: multiply by wds, triplet, multiply by wds."""
    shp = solver.grid_phy
    q = np.empty((Ns + 1,) + shp)
    cur = np.array(init, dtype=np.float64).reshape(shp)
    slot = 0 if direction == 1 else Ns
    q[slot] = cur
    for _ in range(Ns):
        cur = cur * wds
        cur = solver.diffusion(cur)
        cur = cur * wds
        slot += direction
        q[slot] = cur
    return q


def integrate_phi(q, qc, f, Q, Ns):
    """Trapezoid rule, src/crysSCFT_sample.cpp:348-360."""
    phi = np.zeros(q.shape[1:])
    for s in range(Ns + 1):
        factor = 0.5 if (s == 0 or s == Ns) else 1.0
        factor *= f / (Ns * Q)
        phi += factor * q[s] * qc[s]
    return phi


def energy_terms(Q, xN, wA, wB, phiA, phiB, ksi):
    """print_energy, src/crysSCFT_sample.cpp:398-424: returns (F, (enthalpic,
    -ln Q, entropic_1, ksi term), max incompressibility)."""
    size = wA.size
    e0 = -math.log(Q)
    e1 = float(np.sum(-wA * phiA - wB * phiB)) / size
    eh = float(np.sum(xN * phiA * phiB)) / size
    temp = 1 - phiA - phiB
    ek = float(np.sum(-ksi * temp)) / size
    return e0 + e1 + eh + ek, (eh, e0, e1, ek), float(np.max(np.abs(temp)))


def contour_counts(fA, ds):
    """NsA = size_t(fA/ds), NsB = size_t((1-fA)/ds), truncating: src/crysSCFT_sample.cpp:442-444."""
    return int(fA / ds), int((1 - fA) / ds)


def scft_iterations(solver, fA, ds, xN, L, acceptance, nstep, wA0, wB0):
    """diblock_scft_simple_iterate's loop, src/crysSCFT_sample.cpp:440-508."""
    fB = 1 - fA
    NsA, NsB = contour_counts(fA, ds)
    shp = solver.grid_phy
    wA = np.array(wA0, dtype=np.float64).reshape(shp).copy()
    wB = np.array(wB0, dtype=np.float64).reshape(shp).copy()
    solver.set_cell_para(L)
    solver.set_contour_step(ds)
    hist = {"F": [], "parts": [], "maxinc": [], "Q": []}
    phiA = phiB = None
    for _ in range(nstep):
        ksi = 0.5 * (wA + wB - xN)                       # calc_ksi :341-346
        wAds = np.exp((-ds / 2) * wA)                    # array_exp :315-322
        wBds = np.exp((-ds / 2) * wB)
        ones = np.ones(shp)
        qA = solve_diffusion_equation(solver, ones, wAds, NsA, 1)
        qcB = solve_diffusion_equation(solver, ones, wBds, NsB, -1)
        qB = solve_diffusion_equation(solver, qA[NsA], wBds, NsB, 1)
        qcA = solve_diffusion_equation(solver, qcB[0], wAds, NsA, -1)
        Q = float(np.sum(qcA[0])) / qcA[0].size          # array_average :324-331
        phiA = integrate_phi(qA, qcA, fA, Q, NsA)
        phiB = integrate_phi(qB, qcB, fB, Q, NsB)
        F, parts, mi = energy_terms(Q, xN, wA, wB, phiA, phiB, ksi)
        hist["F"].append(F); hist["parts"].append(parts); hist["maxinc"].append(mi); hist["Q"].append(Q)
        wA = wA + acceptance * (xN * phiB + ksi - wA)    # calc_new_fields :362-371
        wB = wB + acceptance * (xN * phiA + ksi - wB)
    out = {k: np.array(v) for k, v in hist.items()}
    out.update(phiA=phiA, phiB=phiB, wA=wA, wB=wB)
    return out


# --------------------------------------------------------------------------
# Anderson mixing (no counterpart in the reference, which mixes simply,
# src/crysSCFT_sample.cpp:362-371); restated here as the checker of the
# library's device-side Anderson mixing.
# --------------------------------------------------------------------------
def anderson_step(w_hist, r_hist, beta):
    """One Anderson-mixing update from the iterates w_hist[0..k] and residuals
    r_hist[0..k] (index 0 the current iterate, j the j-th previous one; each entry the
    pair (A field, B field) flattened into one vector).  With D_j = r_0 - r_j it solves
    sum_j <D_i, D_j> c_j = <D_i, r_0> (i, j = 1..k; <a, b> = a . b) and returns
    w_bar + beta r_bar, w_bar = w_0 + sum_j c_j (w_j - w_0), r_bar = r_0 + sum_j c_j (r_j - r_0).
    A singular system (pivot below 1e-13 of the largest diagonal) falls back to the
    simple step w_0 + beta r_0 and asks for a history restart (second return value)."""
    k = len(w_hist) - 1
    r0, w0 = r_hist[0], w_hist[0]
    if k == 0:
        return w0 + beta * r0, False
    G = np.array([[float(np.dot(a, b)) for b in r_hist] for a in r_hist])
    U = np.empty((k, k))
    V = np.empty(k)
    for i in range(1, k + 1):
        V[i - 1] = G[0, 0] - G[0, i]
        for j in range(1, k + 1):
            U[i - 1, j - 1] = G[0, 0] - G[0, j] - G[i, 0] + G[i, j]
    c = _solve_pivoted(U, V)
    if c is None:
        return w0 + beta * r0, True
    wbar = w0 + sum(c[j - 1] * (w_hist[j] - w0) for j in range(1, k + 1))
    rbar = r0 + sum(c[j - 1] * (r_hist[j] - r0) for j in range(1, k + 1))
    return wbar + beta * rbar, False


def _solve_pivoted(U, V):
    """Gaussian elimination with partial pivoting, in the order the device kernel uses;
    None when a pivot is below 1e-13 of the largest |U_ii|."""
    U = U.copy()
    V = V.copy()
    k = len(V)
    scale = max(abs(U[i, i]) for i in range(k))
    for col in range(k):
        piv = col + int(np.argmax(np.abs(U[col:, col])))
        if not abs(U[piv, col]) > 1e-13 * scale:
            return None
        if piv != col:
            U[[col, piv]] = U[[piv, col]]
            V[[col, piv]] = V[[piv, col]]
        for r in range(col + 1, k):
            f = U[r, col] / U[col, col]
            U[r, col:] -= f * U[col, col:]
            V[r] -= f * V[col]
    c = np.zeros(k)
    for r in range(k - 1, -1, -1):
        c[r] = (V[r] - np.dot(U[r, r + 1:], c[r + 1:])) / U[r, r]
    return c


def scft_iterations_anderson(solver, fA, ds, xN, L, history, beta, nstep, wA0, wB0):
    """The iteration of scft_iterations with calc_new_fields replaced by Anderson mixing
    over the last `history` iterates (anderson_step); also returns the rms residual
    sqrt(<r, r> / (2 M)) of every iteration."""
    fB = 1 - fA
    NsA, NsB = contour_counts(fA, ds)
    shp = solver.grid_phy
    wA = np.array(wA0, dtype=np.float64).reshape(shp).copy()
    wB = np.array(wB0, dtype=np.float64).reshape(shp).copy()
    solver.set_cell_para(L)
    solver.set_contour_step(ds)
    hist = {"F": [], "maxinc": [], "Q": [], "residual": []}
    W, R = [], []
    phiA = phiB = None
    for _ in range(nstep):
        ksi = 0.5 * (wA + wB - xN)
        wAds = np.exp((-ds / 2) * wA)
        wBds = np.exp((-ds / 2) * wB)
        ones = np.ones(shp)
        qA = solve_diffusion_equation(solver, ones, wAds, NsA, 1)
        qcB = solve_diffusion_equation(solver, ones, wBds, NsB, -1)
        qB = solve_diffusion_equation(solver, qA[NsA], wBds, NsB, 1)
        qcA = solve_diffusion_equation(solver, qcB[0], wAds, NsA, -1)
        Q = float(np.sum(qcA[0])) / qcA[0].size
        phiA = integrate_phi(qA, qcA, fA, Q, NsA)
        phiB = integrate_phi(qB, qcB, fB, Q, NsB)
        F, parts, mi = energy_terms(Q, xN, wA, wB, phiA, phiB, ksi)
        r = np.concatenate([(xN * phiB + ksi - wA).ravel(), (xN * phiA + ksi - wB).ravel()])
        w = np.concatenate([wA.ravel(), wB.ravel()])
        hist["F"].append(F); hist["maxinc"].append(mi); hist["Q"].append(Q)
        hist["residual"].append(math.sqrt(float(np.dot(r, r)) / r.size))
        W.insert(0, w)
        R.insert(0, r)
        del W[history + 1:], R[history + 1:]
        wn, restart = anderson_step(W, R, beta)
        if restart:
            del W[1:], R[1:]
        wA = wn[:wA.size].reshape(shp)
        wB = wn[wA.size:].reshape(shp)
    out = {k: np.array(v) for k, v in hist.items()}
    out.update(phiA=phiA, phiB=phiB, wA=wA, wB=wB)
    return out


# --------------------------------------------------------------------------
# field-layout conventions of main(), src/crysSCFT_sample.cpp:202-258
# --------------------------------------------------------------------------
def extract_3m(full):
    """Solver3m uses the even sub-lattice f[2i, 2j, 2k] (src/crysSCFT_sample.cpp:219-235)."""
    return np.ascontiguousarray(full[::2, ::2, ::2])


def extract_pmmm(full):
    """SolverPmmmDCT uses the first octant f[i, j, k], i < N/2 (src/crysSCFT_sample.cpp:242-258)."""
    n0, n1, n2 = (v // 2 for v in full.shape)
    return np.ascontiguousarray(full[:n0, :n1, :n2])
