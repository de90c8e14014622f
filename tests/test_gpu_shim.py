"""The header-only pfem2Solver shim (include/pfem2_solver.hpp) driving the
library from C++ the way a reference case driver does: the run() order
correct -> move -> distribute -> fem_step -> calculate_loads
(TurekBenchmarkCuda/TurekBenchmark.cc:962-981), a forces CSV line per step
as TurekBenchmark/pfem2particle.cpp:963-967 writes it. The compiled driver
must give the same fields, bit for bit, as the same member calls made from
Python through the C ABI.
"""
import ctypes as C
import os
import subprocess
import tempfile

import numpy as np
import pytest

from pfem2_b200 import _abi as A
from pfem2_b200 import cases
from pfem2_b200.solver import LIB_PATH, Solver

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
STEPS = 5

DRIVER = r"""
#include <cstdio>
#include <vector>
#include "pfem2_solver.hpp"

// argv: input (int32 nv, nc; f64 X[nv][2]; int32 cells[nc][4], fb[nc][4];
// the pfem2_case bytes), forces CSV, output (f64 Vx[nv], P[nv])
int main(int argc, char** argv) {
  if (argc != 4) return 2;
  FILE* f = std::fopen(argv[1], "rb");
  if (!f) return 3;
  int32_t n[2];
  if (std::fread(n, 4, 2, f) != 2) return 4;
  std::vector<double> X((size_t)n[0] * 2);
  std::vector<int32_t> cells((size_t)n[1] * 4), fb((size_t)n[1] * 4);
  pfem2_case k{};
  if (std::fread(X.data(), 8, X.size(), f) != X.size() || std::fread(cells.data(), 4, cells.size(), f) != cells.size() ||
      std::fread(fb.data(), 4, fb.size(), f) != fb.size() || std::fread(&k, sizeof(k), 1, f) != 1)
    return 5;
  std::fclose(f);
  pfem2_config c{};
  c.dim = 2;
  c.precision = PFEM2_PREC_FP64;
  c.movement_steps = 3;
  c.max_particles_per_cell_part = 3;
  c.use_graph = 1;
  pfem2_mesh_view m{n[0], n[1], X.data(), cells.data(), fb.data()};
  try {
    pfem2b::Solver s(c, m, k);
    s.seed_particles({4, 4}, 0, 0.1);
    std::ofstream forces(argv[2]);
    for (int step = 0; step < %STEPS%; ++step) {
      s.correct_particles_velocities();
      s.move_particles();
      s.distribute_particle_velocities_to_grid();
      s.fem_step();
      s.time += s.time_step;
      ++s.timestep_number;
      s.calculate_loads(0, &forces);
    }
    std::vector<double> vx = s.get_field(PFEM2_FIELD_VX), p = s.get_field(PFEM2_FIELD_P);
    FILE* o = std::fopen(argv[3], "wb");
    std::fwrite(vx.data(), 8, vx.size(), o);
    std::fwrite(p.data(), 8, p.size(), o);
    std::fclose(o);
  } catch (const pfem2b::Error& e) {
    std::fprintf(stderr, "%s\n", e.what());
    return 10 + (int)e.status;
  }
  return 0;
}
"""


def test_cpp_driver_runs_reference_loop():
    sp = cases.poiseuille_2d(nx=16, ny=6)
    m = sp.mesh
    with tempfile.TemporaryDirectory() as d:
        src, exe = os.path.join(d, "drv.cpp"), os.path.join(d, "drv")
        inp, csv, out = os.path.join(d, "in.bin"), os.path.join(d, "forces.csv"), os.path.join(d, "out.bin")
        open(src, "w").write(DRIVER.replace("%STEPS%", str(STEPS)))
        libdir = os.path.dirname(LIB_PATH)
        subprocess.check_call(["g++", "-std=c++17", "-O1", "-Wall", "-I", os.path.join(ROOT, "include"), src, "-o", exe,
                               "-L", libdir, "-lpfem2b", f"-Wl,-rpath,{libdir}"])
        with open(inp, "wb") as f:
            f.write(np.array([m.n_vertices, m.n_cells], np.int32).tobytes())
            f.write(np.ascontiguousarray(m.vertices, np.float64).tobytes())
            f.write(np.ascontiguousarray(m.cells, np.int32).tobytes())
            f.write(np.ascontiguousarray(m.face_bid, np.int32).tobytes())
            f.write(C.string_at(C.addressof(sp.case), C.sizeof(sp.case)))
        r = subprocess.run([exe, inp, csv, out], capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        lines = open(csv).read().strip().splitlines()
        assert len(lines) == STEPS
        rows = np.array([[float(x) for x in ln.split(",")] for ln in lines])
        assert rows.shape == (STEPS, 8) and np.all(np.isfinite(rows))
        assert np.allclose(rows[:, 0], sp.case.dt * np.arange(1, STEPS + 1))
        res = np.fromfile(out, np.float64).reshape(2, m.n_vertices)
    # the same member calls from Python
    g = Solver(sp, precision=A.PREC_FP64, use_graph=True)
    g.seed_particles((4, 4), 0, 0.1)
    for _ in range(STEPS):
        g.correct_particles_velocities()
        g.move_particles()
        g.distribute_particle_velocities_to_grid()
        g.fem_step()
    assert np.array_equal(res[0], g.field(A.FIELD_VX)) and np.array_equal(res[1], g.field(A.FIELD_P))
    assert np.abs(res[0]).max() > 0.5  # the inflow has entered
    g.close()
