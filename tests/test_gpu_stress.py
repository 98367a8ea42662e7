"""Differentiation form: the adjoint (backward) pass for d ln Q / d L and dF/dchiN,
checked against central finite differences (h = 1e-5 L) and against the same
adjoint identity assembled on the CPU from the reference's own propagators."""
import numpy as np
import pytest

from crysscft_sample_b200 import fields, scft, solvers
from oracle import ref

pytestmark = pytest.mark.gpu


def _one_iteration(G, L, a, b, fA=0.25, ds=0.01, xN=20.0):
    G.set_cell_para(L)
    run = scft.DiblockSCFT(G, fA, ds, xN, 0.1)
    run.set_fields(a, b)
    h = run.iterate(1)
    return run, h


@pytest.mark.parametrize("kind,N,L", [("P1", (32, 24, 16), (4.2, 3.9, 4.6)), ("3M", (32, 32, 48), (4.2, 3.9, 4.6)),
                                      ("PMMM", (32, 32, 32), (4.2, 4.2, 4.2))])
def test_dlnQ_dL_matches_central_differences(gpu, kind, N, L):
    wA, wB = fields.seed_fields(N, L[0], "BCC")
    a, b = fields.to_physical(kind, wA), fields.to_physical(kind, wB)
    G = solvers.make_solver(kind, N)
    run, h = _one_iteration(G, L, a, b)
    g = run.stress()["dlnQ_dL"]
    run.close()
    axes = [0] if kind == "PMMM" else [0, 1, 2]  # the PMMM solver takes one cubic length
    for ax in axes:
        lnQ = []
        for sgn in (1, -1):
            Lp = np.array(L, dtype=float)
            hstep = 1e-5 * L[ax]
            if kind == "PMMM":
                Lp += sgn * hstep
            else:
                Lp[ax] += sgn * hstep
            r, hh = _one_iteration(G, tuple(Lp), a, b)
            lnQ.append(np.log(hh["Q"][0]))
            r.close()
        fd = (lnQ[0] - lnQ[1]) / (2 * hstep)
        want = g.sum() if kind == "PMMM" else g[ax]
        assert abs(fd - want) <= 1e-6 * abs(want) + 1e-10


def test_dlnQ_dL_matches_reference_propagators(gpu):
    """The identity with the reference's CPU propagators (solve_diffusion_equation) and
    numpy derivative operators, against the GPU backward pass."""
    kind, N, L, fA, ds = "3M", (16, 16, 16), (4.2, 3.9, 4.6), 0.25, 0.02
    wA, wB = fields.seed_fields(N, 4.2)
    a, b = fields.to_physical(kind, wA), fields.to_physical(kind, wB)
    G = solvers.make_solver(kind, N)
    run, h = _one_iteration(G, L, a, b, fA=fA, ds=ds)
    g = run.stress()["dlnQ_dL"]
    run.close()
    R = ref.RefSolver(kind, N)
    R.set_cell_para(L)
    R.set_contour_step(ds)
    NsA, NsB = int(fA / ds), int((1 - fA) / ds)
    wAds, wBds = np.exp(-ds / 2 * a.ravel()), np.exp(-ds / 2 * b.ravel())
    ones = np.ones(R.space_size_phy)
    qA = R.solve_diffusion_equation(ones, wAds, NsA, 1)
    qcB = R.solve_diffusion_equation(ones, wBds, NsB, -1)
    qB = R.solve_diffusion_equation(qA[NsA], wBds, NsB, 1)
    qcA = R.solve_diffusion_equation(qcB[0], wAds, NsA, -1)
    q = np.concatenate([qA, qB[1:]])
    qc = np.concatenate([qcA, qcB[1:]])
    Q = qc[0].mean()
    shp = R.grid_size_phy
    PI = np.pi

    def circ(Nn, Lc, deriv):
        k = np.arange(Nn)
        kk = np.minimum(k, Nn - k)
        gk = np.exp(-ds * (2 * PI * kk / Lc) ** 2)
        if deriv:
            gk = gk * 2 * ds * (2 * PI * kk) ** 2 / Lc ** 3
        return (gk[None, :] * np.cos(2 * PI * np.outer(k, k) / Nn)).sum(1) / Nn

    def op(d, deriv):
        c = circ(N[d], L[d], deriv)
        i = np.arange(N[d] // 2)
        return c[(2 * i[:, None] - 2 * i[None, :]) % N[d]] + c[(2 * i[:, None] + 2 * i[None, :] + 1 - N[d]) % N[d]]

    for ax in range(3):
        ops = [op(d, d == ax) for d in range(3)]
        acc = 0.0
        for t in range(NsA + NsB):
            D = wAds if t < NsA else wBds
            x = (D * q[t]).reshape(shp)
            y = np.einsum("ia,jb,kc,abc->ijk", *ops, x).ravel()
            acc += np.sum(qc[t + 1] * D * y)
        want = acc / q.shape[1] / Q
        assert abs(g[ax] - want) <= 1e-10 * abs(want) + 1e-13


def test_dF_dxN_matches_central_differences(gpu):
    kind, N, L = "PMMM", (32, 32, 32), (4.2, 4.2, 4.2)
    wA, wB = fields.seed_fields(N, 4.2)
    a, b = fields.to_physical(kind, wA), fields.to_physical(kind, wB)
    G = solvers.make_solver(kind, N)
    run, _ = _one_iteration(G, L, a, b, xN=20.0)
    got = run.stress()["dF_dxN"]
    run.close()
    h = 1e-4
    F = []
    for xN in (20.0 + h, 20.0 - h):
        r, hh = _one_iteration(G, L, a, b, xN=xN)
        F.append(hh["F"][0])
        r.close()
    assert abs((F[0] - F[1]) / (2 * h) - got) < 1e-8 * max(1.0, abs(got))


def test_cell_relaxation_reduces_stress(gpu):
    N = (32, 32, 32)
    wA, wB = fields.seed_fields(N, 4.0)
    G = solvers.CrysPSSolverPmmm(N)
    out = scft.relax_cell(G, 0.25, 0.01, 20.0, 0.1, fields.to_physical("PMMM", wA), fields.to_physical("PMMM", wB),
                          4.0, n_outer=6, n_inner=10, step=2.0, tol=0.0)
    g = [abs(hh[2]) for hh in out["history"]]
    assert g[-1] < g[0]


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_dlnQ_dL_at_128_bcc_matches_central_differences(gpu, precision):
    # the bench system (128^3 BCC, PMMM on 64^3, ds = 0.005); "fp32": FP32 iterations, then
    # the FP64 polish iteration whose stored contour the backward pass uses
    N, L, ds = (128, 128, 128), 4.2, 0.005
    wA, wB = fields.seed_fields(N, L, "BCC")
    a, b = fields.to_physical("PMMM", wA), fields.to_physical("PMMM", wB)
    G = solvers.make_solver("PMMM", N)
    G.set_cell_para((L, L, L))
    run = scft.DiblockSCFT(G, 0.25, ds, 20.0, 0.1)
    run.set_fields(a, b)
    if precision == "fp32":
        run.set_precision("fp32")
        run.iterate(5)
        run.set_precision("fp64")
    f = run.get_fields()
    run.set_fields(f["wA"], f["wB"])
    run.iterate(1)
    g = run.stress()["dlnQ_dL"].sum()
    run.close()
    lnQ = []
    hstep = 1e-5 * L
    for sgn in (1, -1):
        Lp = L + sgn * hstep
        G.set_cell_para((Lp, Lp, Lp))
        r = scft.DiblockSCFT(G, 0.25, ds, 20.0, 0.1)
        r.set_fields(f["wA"], f["wB"])
        lnQ.append(np.log(r.iterate(1)["Q"][0]))
        r.close()
    fd = (lnQ[0] - lnQ[1]) / (2 * hstep)
    assert abs(fd - g) <= 1e-6 * abs(g) + 1e-10
