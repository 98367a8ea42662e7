"""Anderson mixing (the library's replacement for calc_new_fields,
src/crysSCFT_sample.cpp:362-371, when enabled): the oracle's restatement is checked
on its own here — the pivoted solve, the update on a linear fixed-point problem, and
on the SCFT iteration that its fixed point is the simple-mixing fixed point."""
import numpy as np

from crysscft_sample_b200 import fields
from oracle import scft_oracle as O


def test_pivoted_solve_matches_lapack_and_flags_singular():
    rng = np.random.default_rng(3)
    for k in (1, 2, 5, 12):
        A = rng.standard_normal((k, k)) + k * np.eye(k)
        b = rng.standard_normal(k)
        assert np.allclose(O._solve_pivoted(A, b), np.linalg.solve(A, b), rtol=1e-12, atol=1e-12)
    S = np.ones((3, 3))
    assert O._solve_pivoted(S, np.ones(3)) is None


def test_empty_history_is_the_simple_step():
    rng = np.random.default_rng(4)
    w, r = rng.standard_normal(50), rng.standard_normal(50)
    out, restart = O.anderson_step([w], [r], 0.3)
    assert not restart and np.array_equal(out, w + 0.3 * r)


def test_anderson_solves_a_linear_fixed_point_fast():
    # w = A w + b with a contraction A of spectral radius 0.97 (40 modes): simple mixing
    # needs ~700 steps for 1e-9, Anderson over 20 iterates under 100
    rng = np.random.default_rng(5)
    n = 40
    Qm, _ = np.linalg.qr(rng.standard_normal((n, n)))
    A = Qm @ np.diag(np.linspace(-0.5, 0.97, n)) @ Qm.T
    b = rng.standard_normal(n)
    exact = np.linalg.solve(np.eye(n) - A, b)
    W, R, w = [], [], np.zeros(n)
    for it in range(100):
        r = A @ w + b - w
        W.insert(0, w)
        R.insert(0, r)
        del W[21:], R[21:]
        w, restart = O.anderson_step(W, R, 1.0)
        if restart:
            del W[1:], R[1:]
    assert np.abs(w - exact).max() < 1e-9


def test_scft_anderson_fixed_point_is_the_simple_mixing_fixed_point():
    N, L = (16, 16, 16), 4.2
    wA, wB = fields.seed_fields(N, L)
    a, b = fields.to_physical("PMMM", wA), fields.to_physical("PMMM", wB)
    pre = O.scft_iterations(O.OracleSolver("PMMM", N), 0.25, 0.01, 20.0, (L,) * 3, 0.1, 150, a, b)
    h = O.scft_iterations_anderson(O.OracleSolver("PMMM", N), 0.25, 0.01, 20.0, (L,) * 3, 32, 0.5, 160,
                                   pre["wA"], pre["wB"])
    assert h["residual"][-1] < 1e-10
    # simple mixing from the converged fields stays there
    s = O.scft_iterations(O.OracleSolver("PMMM", N), 0.25, 0.01, 20.0, (L,) * 3, 0.1, 3, h["wA"], h["wB"])
    assert np.all(np.abs(s["F"] - h["F"][-1]) < 1e-9 * abs(h["F"][-1]))
    assert s["maxinc"][-1] < 1e-6
