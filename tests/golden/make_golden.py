"""Writes the golden fixtures of tests/test_golden.py (run from the repo root:
`python tests/golden/make_golden.py`).

The reference cannot be built here (it needs deal.II, Trilinos and MPI), so
these fixtures are outputs of the FP64 oracle (oracle/, the CPU restatement
of the reference's algorithm) on three small seeded workloads. They pin the
oracle over time (a CPU test re-runs it) and give the GPU path a fixed target
(a GPU test compares the library against them).
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle as O  # noqa: E402
from pfem2_b200 import _abi as A  # noqa: E402
from pfem2_b200 import cases  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))


def golden_cases():
    """name -> (spec, steps): the fixture workloads (tests import this)."""
    p2 = cases.poiseuille_2d(nx=32, ny=12)
    p2.case.dt = 0.01
    p2.case.vel_tol, p2.case.p_tol = 1e-13, 1e-12
    ch = cases.channel_disk(h=0.05)
    ch.case.dt = 0.004
    ch.case.vel_tol, ch.case.p_tol = 1e-12, 1e-11
    ch.jitter = 0.05
    p3 = cases.pipe_3d(ny=6, nz=6, nx=12)
    p3.case.dt = 0.02
    p3.case.vel_tol, p3.case.p_tol = 1e-13, 1e-12
    return {"poiseuille_2d": (p2, 3), "channel_disk_coarse": (ch, 2), "pipe_3d": (p3, 1)}


def run_oracle(sp, steps):
    o = O.Oracle(sp.mesh, sp.case, movement_steps=sp.movement_steps, max_per_part=sp.max_per_part)
    o.seed_particles(sp.q, seed=sp.seed, jitter=sp.jitter)
    loads = []
    for _ in range(steps):
        o.step(1)
        if sp.case.load_patch_id >= 0:
            loads.append(o.calculate_loads(sp.case.load_patch_id))
    dim = sp.mesh.dim
    out = {f"v{'xyz'[d]}": o.field(A.FIELD_VX + d) for d in range(dim)}
    out["p"] = o.field(A.FIELD_P)
    cell, _, _ = o.particles()
    out["cell_counts"] = np.bincount(np.asarray(cell), minlength=sp.mesh.n_cells).astype(np.int32)
    out["loads"] = np.array(loads, dtype=np.float64).reshape(len(loads), 5)
    return out


def main():
    for name, (sp, steps) in golden_cases().items():
        out = run_oracle(sp, steps)
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, steps=steps, **out)
        print(name, {k: v.shape for k, v in out.items()}, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
