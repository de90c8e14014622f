"""CPU checks of the C ABI: the ctypes mirror matches include/pfem2.h field
for field, and libpfem2b.so loads and exports every declared entry point
(no compute calls: this runs without a GPU)."""
import ctypes as C
import os
import re
import subprocess
import tempfile

import pytest

from pfem2_b200 import _abi as A
from pfem2_b200 import solver

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "pfem2.h")

STRUCTS = {
    "pfem2_dirichlet": (A.Dirichlet, ["boundary_id", "kind", "axis", "value", "a", "b"]),
    "pfem2_case": (A.Case, ["mu", "rho", "dt", "n_dirichlet", "dirichlet", "open_boundary_mask",
                            "open_boundary_pressure_flux", "zero_after_projection_mask", "load_patch_id",
                            "probe_a", "probe_b", "outer_corrections", "load_diam", "load_umean", "vel_tol",
                            "p_tol", "max_iter", "vel_solver", "p_solver", "reassemble_every_step",
                            "wall_pushback", "vel_rtol", "p_rtol"]),
    "pfem2_mesh_view": (A.MeshView, ["n_vertices", "n_cells", "vertices", "cells", "face_boundary_id"]),
    "pfem2_config": (A.Config, ["dim", "precision", "device", "movement_steps", "max_particles_per_cell_part",
                                "particles_per_cell_max", "particle_capacity_factor", "far_mover_capacity",
                                "use_graph", "particles_only", "fp32_stages", "moving_mesh"]),
    "pfem2_tuning": (A.Tuning, A.TUNING_FIELDS),
    "pfem2_elasticity": (A.Elasticity, ["lambda", "mu", "fixed_mask", "body_id", "tol", "rtol", "max_iter"]),
    "pfem2_stats": (A.Stats, ["n_particles", "n_deleted_last_move", "n_removed_last_check",
                              "n_reseeded_last_check", "n_far_movers_last_move", "iters", "residual",
                              "refinements_p"]),
}


def test_struct_layout_matches_header():
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', "int main(void){"]
    for cname, (_, fields) in STRUCTS.items():
        lines.append(f'printf("{cname} sizeof %zu\\n", sizeof({cname}));')
        for f in fields:
            lines.append(f'printf("{cname} {f} %zu\\n", offsetof({cname}, {f}));')
    lines.append("return 0;}")
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "probe.c")
        exe = os.path.join(d, "probe")
        open(src, "w").write("\n".join(lines))
        subprocess.check_call(["/usr/bin/gcc", "-std=c11", "-o", exe, src])
        out = subprocess.check_output([exe]).decode().split("\n")
    got = {}
    for ln in out:
        if ln.strip():
            n, f, v = ln.split()
            got[(n, f)] = int(v)
    for cname, (cls, fields) in STRUCTS.items():
        assert got[(cname, "sizeof")] == C.sizeof(cls), cname
        for f in fields:
            py = {"lambda": "lam"}.get(f, f)
            assert got[(cname, f)] == getattr(cls, py).offset, (cname, f)


def declared_entry_points():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(pfem2_[a-z_0-9]+)\s*\(", txt)))


def test_exports_cover_header():
    names = declared_entry_points()
    assert set(names) == set(solver.EXPORTS)
    from pfem2_b200 import build as B
    B.build()
    lib = C.CDLL(solver.LIB_PATH)
    for n in names:
        assert hasattr(lib, n), n
    lib.pfem2_abi_version.restype = C.c_int32
    assert lib.pfem2_abi_version() == A.ABI_VERSION


def test_status_codes_match_header():
    txt = open(HEADER).read()
    for name, val in (("PFEM2_OK", A.OK), ("PFEM2_INVALID_ARG", A.INVALID_ARG), ("PFEM2_CUDA_ERROR", A.CUDA_ERROR),
                      ("PFEM2_NOT_CONVERGED", A.NOT_CONVERGED), ("PFEM2_TIMEOUT", A.TIMEOUT),
                      ("PFEM2_PARTICLE_OVERFLOW", A.PARTICLE_OVERFLOW), ("PFEM2_NO_DEVICE", A.NO_DEVICE),
                      ("PFEM2_BAD_STATE", A.BAD_STATE), ("PFEM2_MESH_ERROR", A.MESH_ERROR),
                      ("PFEM2_FIELD_NODE_WEIGHT", A.FIELD_NODE_WEIGHT), ("PFEM2_FIELD_P", A.FIELD_P)):
        m = re.search(rf"\b{name}\s*=\s*(\d+)", txt)
        assert m and int(m.group(1)) == val, name


def test_create_without_device_fails_loudly():
    """On a machine without a CUDA device the library refuses to run (no CPU fallback)."""
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a CUDA device is present")
    except ImportError:
        pass
    from pfem2_b200 import cases
    sp = cases.poiseuille_2d(nx=4, ny=2)
    with pytest.raises(solver.Pfem2Error) as e:
        solver.Solver(sp)
    assert e.value.status in (A.NO_DEVICE, A.CUDA_ERROR)


def test_cpp_shim_compiles_and_links():
    """the header-only pfem2Solver shim compiles against pfem2.h and links to libpfem2b.so"""
    from pfem2_b200 import build as B
    B.build()
    src = (
        '#include "pfem2_solver.hpp"\n'
        "int main(int argc, char**) {\n"
        "  if (argc > 5) { pfem2_config c{}; pfem2_mesh_view m{}; pfem2_case k{};\n"
        "    pfem2b::Solver s(c, m, k); s.seed_particles({4, 4}); s.correct_particles_velocities();\n"
        "    s.move_particles(); s.distribute_particle_velocities_to_grid(); s.fem_step();\n"
        "    std::ofstream f(\"forces.csv\"); s.calculate_loads(3, &f); s.step(); s.calculate_vorticity(); }\n"
        "  return pfem2_abi_version() == PFEM2_ABI_VERSION ? 0 : 1; }\n")
    with tempfile.TemporaryDirectory() as d:
        cpp = os.path.join(d, "drv.cpp")
        exe = os.path.join(d, "drv")
        open(cpp, "w").write(src)
        libdir = os.path.dirname(solver.LIB_PATH)
        subprocess.check_call(["g++", "-std=c++17", "-Wall", "-I", os.path.join(ROOT, "include"), cpp, "-o", exe,
                               "-L", libdir, "-lpfem2b", f"-Wl,-rpath,{libdir}"])
        assert subprocess.call([exe]) == 0


def test_abi_version_mirror_matches_header():
    hdr = open(os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "pfem2.h")).read()
    assert int(re.search(r"#define PFEM2_ABI_VERSION (\d+)", hdr).group(1)) == A.ABI_VERSION


def test_tuning_cache_reader_accepts_both_line_forms(tmp_path):
    """cache lines with five launch-shape values (no velocity blocks per SM)
    and with six read back the same way; the time is recognised by its
    decimal point"""
    from pfem2_b200 import autotune
    p = tmp_path / "c.txt"
    p.write_text("# comment\n"
                 "DEV 2 4 15 0 16 2 8 16 1 2.5656\n"
                 "DEV 2 -1 15 0 16 2 6 16 1 1 2.6834\n"
                 "DEV 3 4 20 0 8 1 4 8 2\n")
    c = autotune.read_cache(str(p))
    assert c["DEV 2 4 15 0"] == (dict(zip(A.TUNING_FIELDS, [16, 2, 8, 16, 1, 0])), 2.5656)
    assert c["DEV 2 -1 15 0"] == (dict(zip(A.TUNING_FIELDS, [16, 2, 6, 16, 1, 1])), 2.6834)
    assert c["DEV 3 4 20 0"] == (dict(zip(A.TUNING_FIELDS, [8, 1, 4, 8, 2, 0])), None)


def test_tuner_searches_coupled_knobs_together(monkeypatch):
    """the advection grid and its one- or two-phase form (and the velocity
    tile and blocks per SM) are tried over all their combinations, the other
    knobs one at a time; measured here with a stand-in for the GPU timing"""
    from pfem2_b200 import autotune

    space = {"advect_blocks_per_sm": [2, 16], "advect_split": [1, 2], "rebin_blocks_per_sm": [4, 8]}
    assert autotune._groups(space) == [("advect_blocks_per_sm", "advect_split"), ("rebin_blocks_per_sm",)]

    # a landscape with a coupled optimum: one pass is best at 2 blocks per
    # SM, two phases at 16 blocks per SM and overall
    cost = {(2, 1): 3.0, (16, 1): 4.0, (2, 2): 5.0, (16, 2): 1.0}
    tried = []

    def fake_measure(specs, tuning, steps, warmup, prepare=None, **kw):
        t = dict({"advect_blocks_per_sm": 2, "advect_split": 1, "rebin_blocks_per_sm": 8}, **(tuning or {}))
        tried.append((t["advect_blocks_per_sm"], t["advect_split"], t["rebin_blocks_per_sm"]))
        ms = cost[(t["advect_blocks_per_sm"], t["advect_split"])] + (0.1 if t["rebin_blocks_per_sm"] == 8 else 0.0)
        return ms, dict(t, vel_tile_slices=0, p_blocks_per_sm=0, vel_blocks_per_sm=0)

    class FakeSolver:
        def __init__(self, *a, **k):
            pass

        def tuning_key(self):
            return "DEV 2 4 15 0"

        def close(self):
            pass

    monkeypatch.setattr(autotune, "measure", fake_measure)
    monkeypatch.setattr(autotune, "Solver", FakeSolver)
    res = autotune.tune([None], space=space, steps=1, warmup=0)
    assert res["tuning"]["advect_blocks_per_sm"] == 16 and res["tuning"]["advect_split"] == 2
    assert res["tuning"]["rebin_blocks_per_sm"] == 4
    assert (16, 2, 8) in tried  # the coupled corner one knob at a time would not reach


@pytest.mark.parametrize("steps", [0, 65536])
def test_movement_steps_range_checked_before_device(steps):
    """movement_steps outside 1 .. 65535 is refused at pfem2_create, before
    the device is looked at (the advection queues store the sub-step index
    in 16 bits)"""
    from pfem2_b200 import cases
    sp = cases.poiseuille_2d(nx=4, ny=2)
    with pytest.raises(solver.Pfem2Error) as e:
        solver.Solver(sp, movement_steps=steps)
    assert e.value.status == A.INVALID_ARG
