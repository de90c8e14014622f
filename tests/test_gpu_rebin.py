"""The re-sort with check_cell_for_empty_parts on FP32 particle storage:
its sub-cell index comes from integer arithmetic on the FP32 bits
(particles.cu, sub_bucket<float>), the FP64 storage uses the reference's
unsigned(xi / h) form (TurekBenchmark/pfem2particle.cpp:723-772). On
coordinates that FP32 represents exactly, both must put every particle in
the same sub-cell: the same particles are kept and removed, the same
sub-cells reseeded, including points on and one ulp beside the sub-cell
faces and at 0 and 1.
"""
import numpy as np
import pytest

from pfem2_b200 import _abi as A
from pfem2_b200.solver import Solver
from tests.test_gpu_parity import spec_2d

pytestmark = pytest.mark.gpu


def boundary_points(q, rng, n_rand=6):
    """FP32 values in [0, 1]: the sub-cell faces k / q, their FP32
    neighbours, 0, 1 and a few random values"""
    v = [np.float32(0.0), np.float32(1.0)]
    for k in range(1, q):
        f = np.float32(k / q)
        v += [f, np.nextafter(f, np.float32(0)), np.nextafter(f, np.float32(1))]
    v += list(rng.random(n_rand).astype(np.float32))
    return np.array(v, np.float32)


def run(sp, q, cell, xi, u, stages):
    s = Solver(sp, precision=A.PREC_MIXED, fp32_stages=stages)
    s.seed_particles(q, 0, 0.0)
    s.set_particles([(cell, xi, u)])
    s.check_empty()
    st = s.stats()
    out = s.particles(), st["removed"], st["reseeded"]
    s.close()
    return out


@pytest.mark.parametrize("q", [(4, 4), (5, 3), (3, 7)])
def test_fp32_sub_cells_match_fp64(q):
    sp = spec_2d()
    rng = np.random.default_rng(7)
    px, py = boundary_points(q[0], rng), boundary_points(q[1], rng)
    nc = sp.mesh.n_cells
    cells, xs = [], []
    for c in range(nc):
        # 12 points per cell: pairs drawn from the boundary lists, so that
        # buckets overflow (MAX_PARTICLES_PER_CELL_PART = 3) and others stay empty
        i = rng.integers(0, len(px), 12)
        j = rng.integers(0, len(py), 12)
        cells.append(np.full(12, c, np.int32))
        xs.append(np.stack([px[i], py[j]], 1))
    cell = np.concatenate(cells)
    xi = np.concatenate(xs).astype(np.float64)  # exact: FP32 values
    u = rng.standard_normal(xi.shape).astype(np.float32).astype(np.float64)
    (c32, x32, u32), rem32, res32 = run(sp, q, cell, xi, u, A.FP32_PARTICLES)
    (c64, x64, u64), rem64, res64 = run(sp, q, cell, xi, u, 0)
    assert rem32 == rem64 and res32 == res64
    assert rem64 > 0 and res64 > 0
    assert np.array_equal(c32, c64)
    # kept particles are the same values; reseeded ones sit at the sub-cell
    # centres, computed in each storage type
    assert np.allclose(x32, x64, rtol=0, atol=1e-7)
    assert np.allclose(u32, u64, rtol=1e-6, atol=1e-6)
