"""Flow cases: mesh + physics + boundary conditions of the PFEM2 workloads.

Each builder returns a CaseSpec: a Mesh, a filled `Case` struct (include/pfem2.h)
and the particle seeding parameters. The five workloads are restated from
their published descriptions; all data is synthetic and seeded.

  poiseuille_2d   2D channel [0,4]x[0,1], 64x16 Q1, parabolic inflow Umax=1,
                  nu=0.01, dt=0.005, 4x4 particles/cell with +-0.1 jitter, seed 0
                  (boundary handling as tube_Poiseuille/tube (Vx-driven).cc:317-331)
  channel_disk    2D channel with a disk r=0.1 at (0.5,0.5), ~50k cells, inflow
                  Umax=1.5, Re=100 (nu = U_mean D / Re, U_mean = 2/3 Umax = 1),
                  dt=0.002, 5x5 particles/cell (boundary ids and conditions as
                  cylinder2D/cylinder2D.cc:459-466,535-545,608-610 with no-slip walls)
  pipe_3d         3D pipe along x, 64x64x256 hex cells mapped from a square,
                  driven by dp/dx = -1 on the open ends (tubePoiseuille3D/tube.cc:509
                  with G = -1), nu=0.01, dt=0.001, 3x3x3 particles/cell
  ensemble        many channel_disk instances with log-uniform cell counts,
                  Reynolds numbers and uniform radii (seed 2)
"""
from dataclasses import dataclass, field

import numpy as np

from . import _abi as A
from . import meshes as M


@dataclass
class CaseSpec:
    name: str
    mesh: M.Mesh
    case: A.Case
    q: tuple
    seed: int
    jitter: float
    steps: int
    movement_steps: int = 3
    max_per_part: int = 3
    meta: dict = field(default_factory=dict)


def make_case(mu, rho, dt, vel_bcs, p_bcs, open_ids, open_flux=0.0, zero_ids=(), load_patch=-1,
              load_diam=1.0, load_umean=1.0, probes=(-1, -1), outer=1, vel_tol=1e-7, p_tol=1e-7,
              max_iter=10000, vel_solver=A.SOLVER_BICGSTAB, p_solver=A.SOLVER_CG, reassemble=0,
              wall_pushback=0):
    """vel_bcs: list (per velocity component) of lists of (bid, kind, value, axis, a, b);
    p_bcs: list of the same tuples for the pressure."""
    cs = A.Case()
    cs.mu, cs.rho, cs.dt = mu, rho, dt
    for f, lst in list(enumerate(vel_bcs)) + [(3, p_bcs)]:
        if len(lst) > A.PFEM2_MAX_BC:
            raise ValueError("too many Dirichlet conditions")
        cs.n_dirichlet[f] = len(lst)
        for k, (bid, kind, value, axis, a, b) in enumerate(lst):
            d = cs.dirichlet[f][k]
            d.boundary_id, d.kind, d.value, d.axis, d.a, d.b = bid, kind, value, axis, a, b
    mask = 0
    for b in open_ids:
        mask |= 1 << b
    cs.open_boundary_mask = mask
    cs.open_boundary_pressure_flux = open_flux
    zm = 0
    for b in zero_ids:
        zm |= 1 << b
    cs.zero_after_projection_mask = zm
    cs.load_patch_id = load_patch
    cs.load_diam, cs.load_umean = load_diam, load_umean
    cs.probe_a, cs.probe_b = probes
    cs.outer_corrections = outer
    cs.vel_tol, cs.p_tol = vel_tol, p_tol
    cs.max_iter = max_iter
    cs.vel_solver, cs.p_solver = vel_solver, p_solver
    cs.reassemble_every_step = reassemble
    cs.wall_pushback = wall_pushback
    return cs


def const(bid, v=0.0):
    return (bid, A.BC_CONSTANT, v, 0, 0.0, 0.0)


def parabola(bid, umax, axis, a, b):
    return (bid, A.BC_PARABOLA, umax, axis, a, b)


def poiseuille_2d(nx=64, ny=16, steps=200, jitter=0.1, seed=0, q=(4, 4), **kw):
    mesh = M.rect_mesh(nx, ny, 0.0, 4.0, 0.0, 1.0)
    nu = 0.01
    cs = make_case(
        mu=nu, rho=1.0, dt=0.005,
        vel_bcs=[[parabola(0, 1.0, 1, 0.0, 1.0), const(2), const(3)],
                 [const(0), const(2), const(3)]],
        p_bcs=[const(1)], open_ids=(0, 1),
        probes=(M.nearest_vertex(mesh, (1.0, 0.5)), M.nearest_vertex(mesh, (3.0, 0.5))),
        **kw)
    return CaseSpec("poiseuille_2d", mesh, cs, q, seed, jitter, steps,
                    meta={"umax": 1.0, "nu": nu, "dpdx": -8.0 * nu * 1.0})


def channel_disk(h=0.0088, radius=0.1, reynolds=100.0, umax=1.5, dt=0.002, steps=500, q=(5, 5),
                 seed=0, jitter=0.0, zero_ids=(), **kw):
    mesh = M.channel_disk_mesh(h=h, radius=radius)
    umean = 2.0 / 3.0 * umax
    diam = 2.0 * radius
    nu = umean * diam / reynolds
    cs = make_case(
        mu=nu, rho=1.0, dt=dt,
        vel_bcs=[[parabola(1, umax, 1, 0.0, 1.0), const(3), const(4)],
                 [const(1), const(3), const(4)]],
        p_bcs=[const(2)], open_ids=(1, 2), zero_ids=zero_ids, load_patch=3,
        load_diam=diam, load_umean=umean,
        probes=(M.nearest_vertex(mesh, (0.5 - radius, 0.5)), M.nearest_vertex(mesh, (0.5 + radius, 0.5))),
        **kw)
    return CaseSpec("channel_disk", mesh, cs, q, seed, jitter, steps,
                    meta={"reynolds": reynolds, "radius": radius, "nu": nu})


def pipe_3d(ny=64, nz=64, nx=256, steps=100, q=(3, 3, 3), dpdx=-1.0, seed=0, jitter=0.0, **kw):
    mesh = M.pipe_mesh(ny, nz, nx)
    nu = 0.01
    cs = make_case(
        mu=nu, rho=1.0, dt=0.001,
        vel_bcs=[[const(2)], [const(2)], [const(2)]],
        p_bcs=[const(1)], open_ids=(0, 1), open_flux=dpdx,
        probes=(M.nearest_vertex(mesh, (2.0, 0.0, 0.0)), -1),
        **kw)
    return CaseSpec("pipe_3d", mesh, cs, q, seed, jitter, steps, meta={"nu": nu, "dpdx": dpdx})


def cylinder2d_unv(path, mu=0.003333333, dt=0.02, u_in=1.0, steps=100, q=(2, 2), seed=0, jitter=0.0, **kw):
    """The reference's cylinder2D case on a mesh read from a UNV file
    (cylinder2D/cylinder2D.cc:266-277, 455-470, 530-545, 605-610 and
    input_data.prm): boundary group 1 = inlet (Vx = u_in, Vy = 0), 2 = outlet
    (p = 0), 3 = cylinder (no slip, the load patch), 4 = walls (Vy = 0);
    inlet and outlet are the open sections."""
    from pfem2_b200 import unv

    mesh = unv.read_unv(path)
    cyl = np.unique(mesh.cells[np.nonzero(mesh.face_bid == 3)[0]].ravel())
    on3 = set()
    for c, f in zip(*np.nonzero(mesh.face_bid == 3)):
        ax, side = f // 2, f % 2
        on3.update(int(mesh.cells[c][v]) for v in range(4) if ((v >> ax) & 1) == side)
    pts = mesh.vertices[sorted(on3)] if on3 else mesh.vertices[cyl]
    centre = pts.mean(axis=0)
    diam = 2.0 * float(np.mean(np.linalg.norm(pts - centre, axis=1)))
    cs = make_case(
        mu=mu, rho=1.0, dt=dt,
        vel_bcs=[[const(1, u_in), const(3)], [const(1), const(3), const(4)]],
        p_bcs=[const(2)], open_ids=(1, 2), load_patch=3, load_diam=diam, load_umean=u_in,
        probes=(M.nearest_vertex(mesh, (float(centre[0]) - diam, float(centre[1]))),
                M.nearest_vertex(mesh, (float(centre[0]) + diam, float(centre[1])))),
        **kw)
    return CaseSpec("cylinder2d_unv", mesh, cs, q, seed, jitter, steps, meta={"diam": diam, "centre": centre.tolist()})


def ensemble(n=64, seed=2, cells_lo=5000, cells_hi=60000, re_lo=20.0, re_hi=200.0, r_lo=0.05, r_hi=0.15,
             q=(5, 5), steps=500, **kw):
    """Instances of channel_disk with log-uniform cells / Re and uniform radius."""
    rng = np.random.default_rng(seed)
    target = np.exp(rng.uniform(np.log(cells_lo), np.log(cells_hi), n))
    re = np.exp(rng.uniform(np.log(re_lo), np.log(re_hi), n))
    rad = rng.uniform(r_lo, r_hi, n)
    specs = []
    for k in range(n):
        # cells ~ 4 / h^2 on the 4x1 channel
        h = float(np.sqrt(4.0 / target[k]))
        specs.append(channel_disk(h=h, radius=float(rad[k]), reynolds=float(re[k]), q=q, steps=steps, **kw))
    return specs


def frozen_stream_field(mesh, n_modes=32, seed=1, cfl=0.5):
    """Divergence-free nodal velocity u = (d psi/dy, -d psi/dx) of a random
    Fourier stream function psi = sum_k a_k sin(2 pi (kx x + ky y) + phi_k),
    a_k ~ N(0,1) |k|^-2, scaled so max|u| * dt / h = cfl with dt = 1 and h
    the mean cell size. Returns (ux, uy, dt)."""
    rng = np.random.default_rng(seed)
    X = mesh.vertices
    ux = np.zeros(len(X)); uy = np.zeros(len(X))
    for _ in range(n_modes):
        kx, ky = rng.integers(-8, 9, size=2)
        if kx == 0 and ky == 0:
            kx = 1
        kn = np.hypot(kx, ky)
        a = rng.normal() * kn ** -2.0
        ph = rng.uniform(0, 2 * np.pi)
        arg = 2 * np.pi * (kx * X[:, 0] + ky * X[:, 1]) + ph
        c = a * np.cos(arg) * 2 * np.pi
        ux += c * ky
        uy -= c * kx
    h = np.sqrt((X[:, 0].max() - X[:, 0].min()) * (X[:, 1].max() - X[:, 1].min()) / mesh.n_cells)
    umax = np.sqrt(ux ** 2 + uy ** 2).max()
    s = cfl * h / umax
    return ux * s, uy * s, 1.0


def stress_2d(n=2048, q=(4, 4), seed=1, cfl=0.5):
    """Particle-kernel stress workload: unit square n x n, q particles/cell
    uniform-random inside their sub-cells, frozen divergence-free field."""
    mesh = M.rect_mesh(n, n, 0.0, 1.0, 0.0, 1.0)
    ux, uy, dt = frozen_stream_field(mesh, seed=seed, cfl=cfl)
    cs = make_case(mu=0.01, rho=1.0, dt=dt, vel_bcs=[[], []], p_bcs=[], open_ids=())
    return CaseSpec("stress_2d", mesh, cs, q, seed, 0.5 / q[0], 1, meta={"ux": ux, "uy": uy})
