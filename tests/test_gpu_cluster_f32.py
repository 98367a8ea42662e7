"""The FP32 contour kernel on thread-block clusters (64^3 physical grids, PMMM and P1).

It runs each propagator chain on one 16-CTA cluster with the exchange in distributed
shared memory and the axis products on tcgen05 tensor cores (two-part fp16 splits).  The
checks: its iterations track FP64 as closely as the 3xTF32 kernel it replaces (selected
with CRYSSCFT_FP32_CLUSTER=0), the two FP32 kernels agree with each other to FP32
accuracy, and the stored contour shows no drift (the tensor cores' round-toward-zero
accumulation is kept out of the large partial sums).
"""
import os

import numpy as np
import pytest

from crysscft_sample_b200 import fields, scft, solvers

pytestmark = pytest.mark.gpu


def _run(kind, N, nstep, precision, cluster=True, L=4.2, ds=0.005):
    old = os.environ.get("CRYSSCFT_FP32_CLUSTER")
    os.environ["CRYSSCFT_FP32_CLUSTER"] = "1" if cluster else "0"
    try:
        wA, wB = fields.seed_fields(N, L, "BCC")
        G = solvers.make_solver(kind, N)
        G.set_cell_para((L, L, L))
        run = scft.DiblockSCFT(G, 0.25, ds, 20.0, 0.1)
        run.set_fields(fields.to_physical(kind, wA), fields.to_physical(kind, wB))
        run.set_precision(precision)
        h = run.iterate(nstep)
        h.update(run.get_fields())
        return G, run, h
    finally:
        if old is None:
            del os.environ["CRYSSCFT_FP32_CLUSTER"]
        else:
            os.environ["CRYSSCFT_FP32_CLUSTER"] = old


@pytest.mark.parametrize("kind,N", [("PMMM", (128, 128, 128)), ("P1", (64, 64, 64))])
def test_cluster_kernel_tracks_fp64(gpu, kind, N):
    G1, r1, h64 = _run(kind, N, 4, "fp64")
    G2, r2, hc = _run(kind, N, 4, "fp32", cluster=True)
    G3, r3, ht = _run(kind, N, 4, "fp32", cluster=False)
    rel_c = np.abs(hc["F"] - h64["F"]) / np.abs(h64["F"])
    rel_t = np.abs(ht["F"] - h64["F"]) / np.abs(h64["F"])
    print(f"\n{kind} {N}: |dF/F| vs FP64, cluster kernel {rel_c.max():.3e}, 3xTF32 kernel {rel_t.max():.3e}")
    assert rel_c.max() < 3e-5
    assert rel_c.max() > 1e-12  # it really ran in FP32
    assert rel_c.max() < 10 * rel_t.max() + 1e-9
    assert np.abs(hc["phiA"] - h64["phiA"]).max() < 1e-4
    for r in (r1, r2, r3):
        r.close()
    for g in (G1, G2, G3):
        g.close()


def test_cluster_kernel_contour_has_no_drift(gpu):
    # the last stored slice of each chain (200 contour steps) against FP64: the mean relative
    # difference measures a systematic shrink or growth of the propagators; it must stay at
    # the level of the 3xTF32 kernel's (whose precision form meets |dF/F| <= 1e-8)
    N = (128, 128, 128)
    G1, r64, _ = _run("PMMM", N, 1, "fp64")
    G2, rc, _ = _run("PMMM", N, 1, "fp32", cluster=True)
    G3, rt, _ = _run("PMMM", N, 1, "fp32", cluster=False)
    U = r64.NsA + r64.NsB
    stats = {}
    for name, r in (("cluster", rc), ("3xTF32", rt)):
        out = []
        for chain, slot in ((0, U), (1, 0)):
            a = r64.get_contour(chain, slot)
            rel = (r.get_contour(chain, slot) - a) / a
            out.append((float(rel.mean()), float(np.abs(rel).max())))
        stats[name] = out
        print(f"\n{name}: contour slot 200 relative difference FP32 - FP64: mean {out[0][0]:.3e} / {out[1][0]:.3e}, "
              f"max {out[0][1]:.3e} / {out[1][1]:.3e}")
    for (mc, xc), (mt, xt) in zip(stats["cluster"], stats["3xTF32"]):
        assert abs(mc) < 1.5 * abs(mt) + 1e-6
        assert xc < 1e-4
    for r in (r64, rc, rt):
        r.close()
    for g in (G1, G2, G3):
        g.close()
