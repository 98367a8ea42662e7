"""CPU tests of the 3m solver with mirror translations (src/solver_3m.h:17, :172-255,
src/solver_utilities.h:56-66): the numpy restatement against the reference build for
non-zero translations, and the library's host-built operator (a sum of Kronecker
products, scft_operator_terms) against the reference triplet."""
import numpy as np
import pytest

from crysscft_sample_b200 import solvers
from crysscft_sample_b200._lib import ScftError
from oracle import ref
from oracle import scft_oracle as O

needs_ref = pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")

N = (16, 12, 16)
L = (4.2, 3.7, 5.1)
DS = 0.03

# (translations, expected number of Kronecker terms)
CASES = [
    ((0,) * 9, 1),
    ((0.5, 0, 0, 0, 0, 0, 0, 0, 0), 2),        # z mirror glides by x/2
    ((0, 0, 0, 0, 0, 0.5, 0, 0, 0), 2),        # y mirror glides by z/2
    ((0, 0, 0, 0, 1 / 3, 0, 0, 0, 0), 1),      # y mirror plane moved by 4 grid points
    ((0, 0.5, 0, 0.5, 0, 0, 0, 0, 0.5), 8),    # cyclic: each sign depends on another axis
    ((0.5, 0.5, 0.25, 0.5, 0, 0.5, 0, 0.5, 0.5), 8),
]


def _apply(terms, q):
    out = np.zeros_like(q)
    for Ax, Ay, Az in terms:
        out += np.einsum("ia,jb,kc,abc->ijk", Ax, Ay, Az, q)
    return out


@needs_ref
@pytest.mark.parametrize("g,_", CASES)
def test_restatement_matches_reference_with_translations(g, _):
    R = ref.RefSolver("3M", N, g)
    R.set_cell_para(L)
    R.set_contour_step(DS)
    S = O.OracleSolver("3M", N, g)
    S.set_cell_para(L)
    S.set_contour_step(DS)
    q = np.random.default_rng(11).standard_normal(R.space_size_phy)
    assert np.abs(R.diffusion(q) - S.diffusion(q).ravel()).max() < 2e-15


@needs_ref
@pytest.mark.parametrize("g,nterms", CASES)
def test_operator_terms_match_reference(g, nterms):
    terms = solvers.operator_terms("3M", N, L, DS, g)
    assert len(terms) == nterms
    R = ref.RefSolver("3M", N, g)
    R.set_cell_para(L)
    R.set_contour_step(DS)
    q = np.random.default_rng(12).standard_normal(R.grid_size_phy)
    want = R.diffusion(q.ravel())
    got = _apply(terms, q).ravel()
    assert np.abs(got - want).max() < 1e-14 * np.abs(want).max()


def test_zero_translation_is_the_plain_3m_operator():
    """g = 0 and g = None give one term: B(0) + B(1) of the mirror-folded circulant."""
    a = solvers.operator_terms("3M", N, L, DS, (0,) * 9)
    b = solvers.operator_terms("3M", N, L, DS, None)
    assert len(a) == len(b) == 1
    for x, y in zip(a[0], b[0]):
        assert np.array_equal(x, y)


@pytest.mark.parametrize("g,grid", [
    ((0.25, 0, 0, 0, 0, 0, 0, 0, 0), N),       # quarter-cell glide: not a group with the lattice
    ((0, 0, 1 / 16, 0, 0, 0, 0, 0, 0), N),     # plane offset of one grid point maps even -> even
    ((0, 0.5, 0, 0, 0, 0, 0, 0, 0), (16, 10, 16)),  # half cell of 5 points: parity changes
    ((0.3, 0, 0, 0, 0, 0, 0, 0, 0), N),        # not on the grid
])
def test_inconsistent_translations_are_rejected(g, grid):
    with pytest.raises(ScftError) as e:
        solvers.operator_terms("3M", grid, L, DS, g)
    assert e.value.status == 1  # SCFT_ERR_INVALID_ARG


@pytest.mark.parametrize("g,_", CASES)
def test_extension_is_symmetric(g, _):
    """extend_3m builds a field invariant under the three generating mirrors."""
    from crysscft_sample_b200 import fields

    rng = np.random.default_rng(13)
    phy = rng.standard_normal(tuple(v // 2 for v in N))
    full = fields.extend_3m(phy, N, g)
    assert np.array_equal(full[::2, ::2, ::2], phy)
    p = np.meshgrid(*[np.arange(v) for v in N], indexing="ij")
    for b in range(3):
        assert np.array_equal(full[fields.m3_mirror(b, p, g, N)], full)
    if not any(g):
        assert np.array_equal(full, fields.from_physical("3M", phy, N))


@needs_ref
@pytest.mark.parametrize("g,_", CASES)
def test_reference_3m_triplet_is_p1_on_the_extension(g, _):
    """The meaning of the translations: the reference's 3m triplet with g equals its P1
    triplet on the symmetric extension, restricted to the even sub-lattice."""
    from crysscft_sample_b200 import fields

    R3 = ref.RefSolver("3M", N, g)
    P1 = ref.RefSolver("P1", N)
    for R in (R3, P1):
        R.set_cell_para(L)
        R.set_contour_step(DS)
    phy = np.random.default_rng(14).standard_normal(R3.grid_size_phy)
    full = fields.extend_3m(phy, N, g)
    want = P1.diffusion(full.ravel()).reshape(N)[::2, ::2, ::2]
    assert np.abs(R3.diffusion(phy.ravel()) - want.ravel()).max() < 1e-14
