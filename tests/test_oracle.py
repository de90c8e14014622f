"""CPU tests of the FP64 oracle: known answers of the restated deal.II
pieces, analytic Poiseuille solutions, and the particle bookkeeping rules of
the reference (seed, check_cell_for_empty_parts, point location)."""
import numpy as np
import pytest

import oracle as O
from pfem2_b200 import _abi as A
from pfem2_b200 import cases, meshes


def splitmix64_py(z):
    m = (1 << 64) - 1
    z = (z + 0x9E3779B97F4A7C15) & m
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & m
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & m
    return z ^ (z >> 31)


def uniform_py(seed, ordinal, axis):
    m = (1 << 64) - 1
    key = (seed * 0xD1B54A32D192ED03 + ordinal * 4 + axis) & m
    return (splitmix64_py(key) >> 11) * (1.0 / 9007199254740992.0)


def test_splitmix_stream_matches_python():
    # SplitMix64 published reference value for seed 0 (first output of the generator)
    assert splitmix64_py(0) == 0xE220A8397B1DCDAF
    for seed in (0, 1, 12345):
        for ordinal in (0, 1, 77, 10 ** 9):
            for axis in range(3):
                assert O.uniform(seed, ordinal, axis) == uniform_py(seed, ordinal, axis)


@pytest.mark.parametrize("dim", [2, 3])
def test_shape_functions(dim):
    rng = np.random.default_rng(0)
    for _ in range(20):
        xi = rng.uniform(0, 1, dim)
        N = O.shape_values(dim, xi)
        assert abs(N.sum() - 1.0) < 1e-15
    for v in range(1 << dim):
        xi = np.array([(v >> d) & 1 for d in range(dim)], dtype=float)
        N = O.shape_values(dim, xi)
        e = np.zeros(1 << dim)
        e[v] = 1
        assert np.array_equal(N, e)


def _small_case(mesh):
    return cases.make_case(0.01, 1.0, 0.01, [[] for _ in range(mesh.dim)], [], open_ids=())


@pytest.mark.parametrize("maker", ["channel", "pipe"])
def test_mapping_roundtrip(maker):
    mesh = meshes.channel_disk_mesh(h=0.05) if maker == "channel" else meshes.pipe_mesh(6, 6, 8)
    o = O.Oracle(mesh, _small_case(mesh))
    rng = np.random.default_rng(1)
    for c in rng.integers(0, mesh.n_cells, 50):
        xi = rng.uniform(0, 1, mesh.dim)
        x = o.map_to_real(int(c), xi)
        ok, xi2 = o.map_to_unit(int(c), x)
        assert ok and np.abs(xi2 - xi).max() < 1e-11


def test_measures_2d_rect():
    m = meshes.rect_mesh(8, 4, 0.0, 4.0, 0.0, 1.0)
    o = O.Oracle(m, _small_case(m))
    assert abs(o.measure() - 4.0) < 1e-13
    for b, (L, n) in {0: (1.0, (-1, 0)), 1: (1.0, (1, 0)), 2: (4.0, (0, -4)), 3: (4.0, (0, 4))}.items():
        s, nint = o.boundary_measure(b)
        assert abs(s - L) < 1e-13
        assert np.allclose(nint, np.array(n, float), atol=1e-12)


def test_measures_channel_disk():
    m = meshes.channel_disk_mesh(h=0.02, radius=0.1)
    o = O.Oracle(m, _small_case(m))
    # straight-sided polygon inscribed in the circle
    nfaces = int((m.face_bid == 3).sum())
    poly = 0.5 * nfaces * 0.1 ** 2 * np.sin(2 * np.pi / nfaces)
    assert abs(o.measure() - (4.0 - poly)) < 1e-3  # the O-grid polygon is not regular
    s, nint = o.boundary_measure(3)
    assert abs(s - 2 * np.pi * 0.1) < 2e-3
    assert np.abs(nint).max() < 1e-12  # closed curve


def test_measures_pipe():
    m = meshes.pipe_mesh(8, 8, 4, length=2.0, radius=0.5)
    o = O.Oracle(m, _small_case(m))
    assert abs(o.measure() - np.pi * 0.25 * 2.0) < 0.05
    s0, n0 = o.boundary_measure(0)
    s1, n1 = o.boundary_measure(1)
    assert abs(s0 - s1) < 1e-12 and abs(n0[0] + s0) < 1e-12 and abs(n1[0] - s1) < 1e-12


def test_matrices_known_answers():
    sp = cases.poiseuille_2d(nx=8, ny=4)
    o = O.Oracle(sp.mesh, sp.case)
    o.assemble_matrices()
    rp, ci, mass = o.matrix(4)
    isd, _ = o.dirichlet(0)
    # mass entries summed over free rows and free columns + Dirichlet diagonals
    rp, ci, K = o.matrix(3)
    pdir, _ = o.dirichlet(3)
    for i in range(len(rp) - 1):
        cols = ci[rp[i]:rp[i + 1]]
        if pdir[i] or pdir[cols].any():
            continue
        assert abs(K[rp[i]:rp[i + 1]].sum()) < 1e-13  # Laplacian rows sum to zero
    # symmetric after elimination
    for which in (0, 1, 3, 4, 5):
        rp, ci, V = o.matrix(which)
        d = {}
        for i in range(len(rp) - 1):
            for k in range(rp[i], rp[i + 1]):
                d[(i, ci[k])] = V[k]
        for (i, j), v in d.items():
            assert abs(v - d[(j, i)]) < 1e-14


def test_mass_matrix_sum_is_area():
    m = meshes.rect_mesh(6, 3, 0.0, 3.0, 0.0, 1.5)
    cs = cases.make_case(1.0, 1.0, 0.1, [[], []], [], open_ids=())
    o = O.Oracle(m, cs)
    o.assemble_matrices()
    _, _, M = o.matrix(4)
    assert abs(M.sum() - 4.5) < 1e-13


def test_poiseuille_steady_state_preserved():
    """The exact steady solution u = 4y(1-y), p linear with dp/dx = -8 nu Umax
    (tube_Poiseuille/tube (Vx-driven).cc inflow) is a near fixed point."""
    sp = cases.poiseuille_2d()
    o = O.Oracle(sp.mesh, sp.case, movement_steps=3, max_per_part=3)
    X = sp.mesh.vertices
    ue = 4 * X[:, 1] * (1 - X[:, 1])
    for f, v in ((A.FIELD_VX, ue), (A.FIELD_OLD_VX, ue), (A.FIELD_VY, 0 * ue), (A.FIELD_OLD_VY, 0 * ue),
                 (A.FIELD_P, -0.08 * (X[:, 0] - 4.0))):
        o.set_field(f, v)
    o.seed_particles(sp.q, sp.seed, sp.jitter)
    for _ in range(20):
        assert o.step(1) == 0
    vx = o.field(A.FIELD_VX)
    assert np.linalg.norm(vx - ue) / np.linalg.norm(ue) < 5e-3
    p = o.field(A.FIELD_P)
    sel = np.abs(X[:, 1] - 0.5) < 1e-9
    slope = np.polyfit(X[sel, 0], p[sel], 1)[0]
    assert abs(slope - sp.meta["dpdx"]) < 0.1 * abs(sp.meta["dpdx"])


def test_seed_positions_and_velocity():
    sp = cases.poiseuille_2d(nx=4, ny=2)
    o = O.Oracle(sp.mesh, sp.case)
    X = sp.mesh.vertices
    o.set_field(A.FIELD_VX, 2.0 + 3.0 * X[:, 0])  # linear fields are reproduced exactly
    o.set_field(A.FIELD_VY, -X[:, 1])
    o.seed_particles((3, 2), seed=0, jitter=0.0)
    cell, xi, u = o.particles()
    assert len(cell) == sp.mesh.n_cells * 6
    assert np.allclose(np.sort(np.unique(np.round(xi[:, 0], 12))), [1 / 6, 0.5, 5 / 6])
    x = o.positions()
    assert np.allclose(u[:, 0], 2.0 + 3.0 * x[:, 0], atol=1e-13)
    assert np.allclose(u[:, 1], -x[:, 1], atol=1e-13)


def test_check_empty_removal_and_reseed():
    """check_cell_for_empty_parts: count per sub-cell in order, drop beyond MAX,
    one new particle at the centre of each empty sub-cell (i, j order)."""
    sp = cases.poiseuille_2d(nx=2, ny=1)
    o = O.Oracle(sp.mesh, sp.case, movement_steps=1, max_per_part=3)
    # cell 0: 5 particles in sub-cell (0,0) of a 2x2 split, nothing else
    xi = np.array([[0.1, 0.1], [0.2, 0.1], [0.3, 0.2], [0.15, 0.4], [0.05, 0.05]])
    cell = np.zeros(5, np.int32)
    u = np.arange(10, dtype=float).reshape(5, 2)
    o.set_particles(cell, xi, u, q=(2, 2))
    o.check_empty()
    c2, xi2, u2 = o.particles()
    st = o.stats()
    assert st["removed"] == 2
    # 3 kept in cell 0, 3 new in cell 0, 4 new in cell 1
    assert list(c2) == [0] * 6 + [1] * 4
    assert np.allclose(xi2[:3], xi[:3]) and np.allclose(u2[:3], u[:3])
    assert np.allclose(xi2[3:6], [[0.25, 0.75], [0.75, 0.25], [0.75, 0.75]])
    assert np.allclose(xi2[6:], [[0.25, 0.25], [0.25, 0.75], [0.75, 0.25], [0.75, 0.75]])
    assert st["reseeded"] == 7


def test_point_location_neighbour_and_exit():
    """A particle crossing a face lands in the neighbour; one leaving the
    domain through the outlet is deleted (sort_particles_into_subdomains_and_cells)."""
    m = meshes.rect_mesh(4, 4, 0.0, 1.0, 0.0, 1.0, reorder=False)
    cs = cases.make_case(0.01, 1.0, 0.1, [[], []], [], open_ids=())
    o = O.Oracle(m, cs, movement_steps=1, max_per_part=10)
    X = m.vertices
    o.set_field(A.FIELD_VX, np.ones(len(X)))
    o.set_field(A.FIELD_VY, 0.5 * np.ones(len(X)))
    # cell 5 = (i=1, j=1); a particle near its upper-right corner moves diagonally
    cell = np.array([5, 3], np.int32)
    xi = np.array([[0.9, 0.9], [0.9, 0.5]])
    u = np.zeros((2, 2))
    o.set_particles(cell, xi, u, q=(1, 1))
    o.advect()
    c2, xi2, _ = o.particles()
    st = o.stats()
    # particle in cell 3 (i=3, j=0) leaves through x = 1 and is deleted
    assert st["deleted"] == 1
    # moved by (0.1, 0.05): from (0.475, 0.475) to (0.575, 0.525) -> cell (2, 2) = 10
    assert list(c2) == [10]
    assert np.allclose(xi2[0], [0.3, 0.1], atol=1e-12)


def test_loads_pressure_only():
    """Pressure p = x over the disk: Fx_p = area of the (polygonal) disk."""
    sp = cases.channel_disk(h=0.02)
    o = O.Oracle(sp.mesh, sp.case)
    X = sp.mesh.vertices
    o.set_field(A.FIELD_P, X[:, 0].copy())
    out = o.calculate_loads(3)
    nfaces = int((sp.mesh.face_bid == 3).sum())
    area = 0.5 * nfaces * 0.1 ** 2 * np.sin(2 * np.pi / nfaces)
    s = 2.0 / (1.0 * 1.0 ** 2 * 0.2)
    assert abs(out[1] - s * area) < 2e-3 * s
    assert abs(out[3]) < 1e-10 and abs(out[0]) < 1e-14


def test_vorticity_of_linear_fields():
    """calculate_vorticity (cylinderDyM/pfem2particle.cpp:1000-1050): Q1 cells
    reproduce a linear velocity field exactly, so every node recovers its
    vorticity dVy/dx - dVx/dy, also on the curved O-grid cells"""
    sp = cases.channel_disk(h=0.05)
    o = O.Oracle(sp.mesh, sp.case)
    X = sp.mesh.vertices
    o.set_field(A.FIELD_VX, 2.0 - 0.5 * X[:, 1] + 0.3 * X[:, 0])
    o.set_field(A.FIELD_VY, 1.5 * X[:, 0] - 0.3 * X[:, 1])
    w = o.calculate_vorticity()
    assert np.allclose(w, 2.0, rtol=0, atol=1e-10)


def test_vorticity_rejects_3d():
    sp = cases.pipe_3d(ny=4, nz=4, nx=8)
    o = O.Oracle(sp.mesh, sp.case)
    with pytest.raises(ValueError):
        o.calculate_vorticity()


def test_wall_pushback_known_answer():
    """wall push-back (nacaAirfoil/pfem2particle.cpp:919-952): a uniform
    particle velocity U projects to U at every node; then every particle of a
    wall cell keeps U (1 - sum of N_v over the cell's wall vertices) and the
    wall nodes are zero. Without the flag the particles keep U."""
    U = np.array([1.0, 0.5])
    for push in (0, 1):
        sp = cases.poiseuille_2d(nx=4, ny=2, zero_ids=(2, 3), wall_pushback=push)
        o = O.Oracle(sp.mesh, sp.case)
        o.seed_particles((2, 2), seed=0, jitter=0.0)
        cell, xi, u = o.particles()
        o.set_particles(cell, xi, np.tile(U, (len(cell), 1)), q=(2, 2))
        o.distribute_particle_velocities_to_grid()
        cell2, xi2, u2 = o.particles()
        X = sp.mesh.vertices
        wall = (np.abs(X[:, 1]) < 1e-12) | (np.abs(X[:, 1] - 1.0) < 1e-12)
        vx, vy = o.field(A.FIELD_VX), o.field(A.FIELD_VY)
        assert np.all(vx[wall] == 0.0) and np.all(vy[wall] == 0.0)
        assert np.allclose(vx[~wall], U[0]) and np.allclose(vy[~wall], U[1])
        cv = sp.mesh.cells
        for p in range(len(cell2)):
            x, y = xi2[p]
            N = np.array([(1 - x) * (1 - y), x * (1 - y), (1 - x) * y, x * y])
            f = 1.0 - push * N[wall[cv[cell2[p]]]].sum()
            assert np.allclose(u2[p], f * U, atol=1e-14)
