"""The launch-shape autotuner (pfem2_b200/autotune.py) and the library's
tuning cache (pfem2_set_tuning / pfem2_get_tuning / PFEM2_TUNING_CACHE):
a tiny search writes an entry, a new context with the same key reads it
back and uses it, explicit fields win over the cache, and the particle
shapes leave the results bitwise unchanged.
"""
import numpy as np
import pytest

from pfem2_b200 import _abi as A
from pfem2_b200 import autotune
from pfem2_b200.solver import Solver
from tests.helpers import rel_l2
from tests.test_gpu_parity import spec_2d

pytestmark = pytest.mark.gpu


def run(sp, tuning=None, steps=3):
    s = Solver(sp, precision=A.PREC_MIXED, tuning=tuning)
    s.seed_particles(sp.q, 0, 0.1)
    for _ in range(steps):
        s.step()
    out = [s.field(f) for f in (A.FIELD_VX, A.FIELD_VY, A.FIELD_P)], s.particles(), s.tuning()
    s.close()
    return out


def test_tuner_writes_and_library_reads_cache(tmp_path, monkeypatch):
    sp = spec_2d(dt=0.01)
    cache = str(tmp_path / "tuning.txt")
    space = {"advect_blocks_per_sm": [2, 4], "advect_split": [1, 2], "rebin_blocks_per_sm": [2, 4]}
    res = autotune.tune([sp], space=space, steps=3, warmup=1, cache=cache, precision=A.PREC_MIXED)
    assert res["ms_per_step"] <= res["baseline_ms"]
    assert len(res["trials"]) >= 1 + sum(len(v) for v in space.values()) - len(space)
    entries = autotune.read_cache(cache)
    assert list(entries) == [res["key"]]
    tuned = entries[res["key"]][0]
    assert tuned == res["tuning"]
    monkeypatch.setenv("PFEM2_TUNING_CACHE", cache)
    s = Solver(sp, precision=A.PREC_MIXED)
    assert s.tuning_key() == res["key"]
    assert s.tuning() == tuned
    s.close()
    # an explicit field wins over the cache, the others still come from it
    s = Solver(sp, precision=A.PREC_MIXED, tuning={"advect_blocks_per_sm": 3})
    got = s.tuning()
    assert got["advect_blocks_per_sm"] == 3
    assert got["rebin_blocks_per_sm"] == tuned["rebin_blocks_per_sm"]
    s.close()
    # another key (FP64) finds no entry: automatic shapes
    s = Solver(sp, precision=A.PREC_FP64)
    assert s.tuning_key() != res["key"] and s.tuning()["advect_blocks_per_sm"] == 16
    s.close()


def test_particle_shapes_do_not_change_results():
    sp = spec_2d(dt=0.01)
    a = run(sp, {"advect_blocks_per_sm": 2, "advect_split": 1, "rebin_blocks_per_sm": 2})
    b = run(sp, {"advect_blocks_per_sm": 16, "advect_split": 2, "rebin_blocks_per_sm": 12})
    assert a[2]["advect_split"] == 1 and b[2]["advect_split"] == 2
    for x, y in zip(a[0], b[0]):
        assert np.array_equal(x, y)
    for x, y in zip(a[1], b[1]):
        assert np.array_equal(x, y)


def test_solver_shapes_within_tolerance():
    """velocity tile size and blocks per SM, pressure blocks per SM: same
    solution to the solver tolerance (1e-13 / 1e-12 absolute in this spec)"""
    sp = spec_2d(dt=0.01)
    a = run(sp, {"vel_tile_slices": 1, "p_blocks_per_sm": 1, "vel_blocks_per_sm": 1})
    b = run(sp, {"vel_tile_slices": 8, "p_blocks_per_sm": 2, "vel_blocks_per_sm": 2})
    assert a[2]["vel_tile_slices"] == 1 and b[2]["p_blocks_per_sm"] == 2
    assert a[2]["vel_blocks_per_sm"] == 1 and b[2]["vel_blocks_per_sm"] == 2
    for x, y in zip(a[0], b[0]):
        assert rel_l2(x, y) <= 1e-9


def test_bad_tuning_rejected():
    sp = spec_2d()
    for bad in ({"p_blocks_per_sm": 3}, {"vel_blocks_per_sm": 3}, {"advect_split": 5}):
        with pytest.raises(Exception):
            Solver(sp, tuning=bad)
