"""The slot partition of the fused phi sums, checked on the CPU.

The alternating contour kernels (csrc/contour_kernel.cuh, csrc/contour_kernel_f32.cuh) add
q(s) q+(s) for a slot s in the phase k that finishes it when the other chain stored s at
least two phases earlier on the same layout, except s = NsA; chain 0 runs forward from
slot 0, chain 1 backward from slot U.  Tiles are in 8-column panels: element
(z / 8) * 8n + row * 8 + z % 8, rows y in plane tile x and rows x in slab tile y.
phi_fused_finish_kernel (csrc/field_kernels.cuh) adds the four accumulators of each point
and slots 0, NsA, U/2 and U with the trapezoid weights.  This model of both must equal
integrate_phi (src/crysSCFT_sample.cpp:348-360) for every block split, and every slot must
be counted exactly once.
"""
import numpy as np
import pytest


def _active(k, c, U, NsA):
    slot0, dirs = (0, U), (1, -1)
    s = slot0[c] + dirs[c] * k
    kq = (s - slot0[1 - c]) * dirs[1 - c]
    return s, (k >= 1 and k <= U and 1 <= kq <= k - 2 and (k - kq) % 2 == 0 and s != NsA)


def _panel(n):
    # panel index of (row, z) in an n x n tile
    r, z = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    return (z // 8) * 8 * n + r * 8 + z % 8


def _fused_phi(q, qc, NsA, NsB):
    U = NsA + NsB
    n = q.shape[1]
    pi = _panel(n)
    acc = np.zeros((2, 2, 2, n, n * n))  # chain, block, layout, tile, panel element
    for c in range(2):
        for k in range(U + 1):
            s, act = _active(k, c, U, NsA)
            if not act:
                continue
            plane = k % 2 == 0
            blk = 0 if s < NsA else 1
            for p in range(n):
                prod = (q[s, p] * qc[s, p]) if plane else (q[s, :, p] * qc[s, :, p])
                acc[c, blk, 0 if plane else 1, p, pi.ravel()] += prod.ravel()
    special = [0, NsA, U // 2, U] if U // 2 != NsA else [0, NsA, U]
    x, y, z = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    zp = (z // 8) * 8 * n + z % 8
    a = np.zeros((n, n, n))
    b = np.zeros((n, n, n))
    for c in range(2):
        a += acc[c, 0, 0][x, zp + y * 8] + acc[c, 0, 1][y, zp + x * 8]
        b += acc[c, 1, 0][x, zp + y * 8] + acc[c, 1, 1][y, zp + x * 8]
    for s in special:
        w = q[s] * qc[s]
        if s <= NsA:
            a += (0.5 if s in (0, NsA) else 1.0) * w
        if s >= NsA:
            b += (0.5 if s in (NsA, U) else 1.0) * w
    return a, b


def _integrate_phi(q, qc, NsA, NsB):
    wA = np.ones(NsA + 1)
    wA[[0, -1]] = 0.5
    wB = np.ones(NsB + 1)
    wB[[0, -1]] = 0.5
    return (np.einsum("s,sxyz->xyz", wA, (q * qc)[: NsA + 1]),
            np.einsum("s,sxyz->xyz", wB, (q * qc)[NsA:]))


@pytest.mark.parametrize("n,NsA,NsB", [(8, 2, 8), (8, 5, 5), (8, 7, 3), (8, 1, 1), (8, 1, 3), (8, 3, 1),
                                        (16, 25, 75), (16, 50, 150)])
def test_partition_and_finish_equal_integrate_phi(n, NsA, NsB):
    rng = np.random.default_rng(n * 1000 + NsA)
    U = NsA + NsB
    q = rng.random((U + 1, n, n, n))
    qc = rng.random((U + 1, n, n, n))
    a, b = _fused_phi(q, qc, NsA, NsB)
    ra, rb = _integrate_phi(q, qc, NsA, NsB)
    assert np.abs(a - ra).max() <= 1e-12 * U
    assert np.abs(b - rb).max() <= 1e-12 * U


@pytest.mark.parametrize("U,NsA", [(200, 50), (100, 50), (100, 70), (2, 1), (10, 9)])
def test_every_slot_counted_once(U, NsA):
    counted = {}
    for c in range(2):
        for k in range(U + 1):
            s, act = _active(k, c, U, NsA)
            if act:
                counted[s] = counted.get(s, 0) + 1
    special = {0, NsA, U // 2, U}
    assert all(v == 1 for v in counted.values())
    assert set(counted) | special == set(range(U + 1))
    assert not (set(counted) & special)
    # each active phase reads a slot the other chain stored before the midpoint phase
    for c in range(2):
        for k in range(U + 1):
            s, act = _active(k, c, U, NsA)
            if act:
                kq = U - k
                assert kq <= U // 2 - 1
