"""Drop-in check through the plug-in interface: the reference's own, unmodified
diblock_scft_simple_iterate and solve_diffusion_equation (compiled as
oracle/_ref/libref_gpu_driver.so) drive the GPU solvers through the
CrysPSSolverBase adapters of include/crysscft_b200_solvers.hpp, and print the same
free energies and incompressibilities as with the reference's CPU solvers."""
import os

import pytest

from crysscft_sample_b200 import fields
from oracle import ref

pytestmark = pytest.mark.gpu


@pytest.mark.skipif(not os.path.exists(ref.GPU_DRIVER_PATH), reason="oracle/_ref/libref_gpu_driver.so not built")
@pytest.mark.parametrize("kind", ["PMMM", "3M", "P1"])
def test_reference_driver_runs_gpu_solvers(gpu, kind, tmp_path):
    N, L = (16, 16, 16), 4.2
    wA, wB = fields.seed_fields(N, L)
    a, b = fields.to_physical(kind, wA), fields.to_physical(kind, wB)
    args = (0.25, 0.01, 20.0, (L, L, L), 0.1, 11, a, b)
    cpu = ref.parse_driver_log(ref.RefSolver(kind, N).run_driver(*args, str(tmp_path / "cpu")))
    gpu_log = ref.run_reference_driver_on_gpu(kind, N, *args, str(tmp_path / "gpu"))
    g = ref.parse_driver_log(gpu_log)
    assert [r[0] for r in g] == [0, 10]
    for (i1, F1, m1), (i2, F2, m2) in zip(cpu, g):
        assert i1 == i2
        assert abs(F1 - F2) <= 1e-9 * abs(F1)
        assert abs(m1 - m2) <= 1e-9 * abs(m1)
