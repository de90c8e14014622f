"""Benchmark of the PFEM2 time step on B200 (one JSON line on rank 0).

Workload (default): the 2D channel with a disk obstacle, ~52k Q1 cells,
25 particles per cell (~1.3M particles), Re=100, dt=0.002: one `step` is one
whole PFEM2 time step (correct -> move/locate/reseed -> project -> fractional
-step FEM with the three Krylov solves) of the mixed-precision path, inputs
resident in HBM, every solve to |r| <= rtol |b|. The mixed path runs the
inner Krylov iterations in FP32 and refines them in FP64; the bench checks
that its fields stay within 1e-6 relative L2 of the FP64 path after the same
steps (`fixed_error`), and reports the FP64 path, the all-FP32 path and the
per-stage error of each FP32 stage beside it.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
  python bench.py --only stress|pipe|ensemble|budget|channel   (one leg, its own JSON)

Multi-GPU: a single mesh does not shard, so N ranks run N independent
replicas of the instance (weak scaling, no data-path collective); value is
the sum of the ranks' instance-timesteps/s over the max-over-ranks time.

--impl reference times the FP64 CPU restatement of the reference algorithm
(oracle/, OpenMP over the host cores) on a bounded sample of the same
workload; deal.II (the reference's own dependency) is not installed here.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--h", type=float, default=0.0088, help="cell size of the channel mesh (~52k cells)")
    ap.add_argument("--rtol", type=float, default=1e-8,
                    help="relative tolerance |r| <= rtol |b| of every solve, both paths")
    ap.add_argument("--no-fp64", action="store_true", help="skip the FP64 comparison leg")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--stress-n", type=int, default=2048, help="particle-stress mesh: n x n cells (0 = skip)")
    ap.add_argument("--ensemble-n", type=int, default=64, help="instances of the batched leg (0 = skip)")
    ap.add_argument("--pipe-n", type=int, default=64,
                    help="3D pipe leg: n x n x 4n hex cells, mixed and FP64 (0 = skip)")
    ap.add_argument("--pipe-rtol", type=float, default=1e-11, help="relative tolerance of the pipe leg's solves")
    ap.add_argument("--extra-steps", type=int, default=5, help="timed steps of the stress and ensemble legs")
    ap.add_argument("--only", default="all", choices=["all", "channel", "stress", "pipe", "ensemble", "budget"],
                    help="run one leg alone and print its JSON (for profilers); 'all' prints the bench line")
    return ap.parse_args()


def dist_info():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


METRIC = "timesteps/s (mixed-precision PFEM2 step at fixed error vs FP64; particle updates/s alongside)"

# the bar the mixed path is measured at: relative L2 of velocity and
# pressure against the FP64 path on the same workload, seed and steps
FIXED_ERROR = 1e-6


def tight(sp, rtol):
    """both paths solve to |r| <= rtol |b| (no absolute floor), so that
    their difference is the arithmetic, not the stopping rule"""
    sp.case.vel_tol = sp.case.p_tol = 0.0
    sp.case.vel_rtol = sp.case.p_rtol = rtol
    return sp


def workload(args):
    from pfem2_b200 import cases

    return tight(cases.channel_disk(h=args.h), args.rtol)


WORKLOAD_DESC = {
    "workload": "2D channel [0,4]x[0,1] with disk r=0.1 at (0.5,0.5), O-grid+blocks Q1 mesh, "
                "parabolic inflow Umax=1.5, Re=100, dt=0.002, 5x5 particles/cell",
}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except Exception:
            self.proc = None

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["active", "hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names[1:], parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d["hbm_gbs"], "measured"
    return 6650.0, "fallback"


def cg_bytes(s, iters, outer):
    """Algorithmic bytes of the pressure solves by the per-row figures of a
    CG iteration on a Q1 SpMV: (FP32 values, int32 columns) SpMV 9 nnz x 8 B
    + row pointer, x, y = 84 B/row in 2D (27 nnz: 228 B/row in 3D), two dot
    products 16 B/row, three axpy 36 B/row, a Jacobi step 8 B/row: 144 B/row
    in 2D, 288 B/row in 3D (twice the value bytes in FP64); an FP64 residual
    refinement reads the FP64 matrix once: 9 x 12 + 4 + 24 = 136 B/row in 2D,
    27 x 12 + 4 + 24 = 352 B/row in 3D."""
    info = s.sizes()
    n, rb = info["rows"], info["real_bytes"]
    nnz_row = 9 if s.dim == 2 else 27
    inner = nnz_row * (rb + 4) + 4 + 2 * rb + 2 * 2 * rb + 3 * 3 * rb + 2 * rb
    outerb = nnz_row * 12 + 4 + 24
    return n * (iters * inner + outer * outerb)


def pressure_solve_bytes(s, iters, outer):
    """Algorithmic bytes of the pressure solves with the multigrid operators.
    One inner CG iteration (inner type R: FP32 for the mixed path) reads
    every operator once with its column indices and streams the vectors:
        A   q = A (z + beta p)         nnz*(R+4) + n*(z, p in; p, q out)
        B   e, r' update; b1, b2       n*(e, p, q, r in; e, r' out) + (R01 + R02 + C3)*(R+4) + (n1 + n2)*R
        UZ  z = J0 r + Pt0 x1, coarse  nnz*(R+4) + P0*(R+4) + (J1+P1+J2+P2)*(R+4) + n*(r in, z out) + n2*R
    FP64 refinement sweep: nnz*(8+4) + n*(x64 + e + b + r64) bytes."""
    info = s.sizes()
    n, nnz, rb = info["rows"], info["nnz"], info["real_bytes"]
    mg = s.solver_sizes()
    ops = mg["r01"] + mg["r02"] + mg["c3"] + mg["p0"] + mg["j1"] + mg["p1"] + mg["j2"] + mg["p2"]
    inner = 2 * nnz * (rb + 4) + ops * (rb + 4) + 12 * n * rb + (mg["n1"] + 2 * mg["n2"]) * rb
    outerb = nnz * 12 + n * (8 + rb + 8 + 8)
    return iters * inner + outer * outerb


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def run_ours(args, rank, world, local):
    import torch

    from pfem2_b200 import _abi as A
    from pfem2_b200.solver import STAGE_NAMES, Solver

    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local}")
    if args.only != "all":
        out = {"stress": lambda: stress_leg(args, local, flush), "pipe": lambda: pipe_leg(args, local, flush),
               "ensemble": lambda: ensemble_leg(args, rank, world, local, flush, None),
               "budget": lambda: budget_leg(args, local),
               "channel": lambda: channel_leg(args, local, flush, A.PREC_MIXED, 0)}[args.only]()
        if rank == 0:
            print(json.dumps(out), flush=True)
        return
    sp = workload(args)
    s = Solver(sp, precision=A.PREC_MIXED, device=local, use_graph=True)
    s.seed_particles(sp.q, sp.seed, sp.jitter)
    stream = torch.cuda.ExternalStream(s.stream(), device=local)
    for _ in range(args.warmup):
        s.step()
    s.synchronize()
    s.enable_stage_timing(True)
    s.stage_times(reset=True)
    it_p = 0
    outer_p = 0
    np_sum = 0
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    l0 = s.launch_count()
    clocks = ClockSampler(local)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    clocks.start()
    for k in range(args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()  # > L2: every step starts cold (outside the timed events)
        ev[k][0].record(stream)
        s.step()
        ev[k][1].record(stream)
        st = s.stats()
        it_p += st["iters"][3]
        outer_p += st["refinements_p"]
        np_sum += st["n_particles"]
    torch.cuda.synchronize()
    clk = clocks.stop()
    launches = s.launch_count() - l0
    ms = float(sum(a.elapsed_time(b) for a, b in ev))
    stages = s.stage_times()
    if world > 1:
        t = torch.tensor([ms], device=f"cuda:{local}")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms = float(t.item())
    steps_per_s = args.steps / (ms / 1e3)
    value = steps_per_s * world
    pupd = np_sum / (ms / 1e3) * world

    # roofline of the dominant kernel, the pressure solve, from its live
    # iteration counts: the CG bytes per row of the scope table (primary) and
    # the byte model that also counts the multigrid operators (secondary)
    hbm, peak_kind = peaks()
    ps_ms = stages[STAGE_NAMES.index("pressure_solve")]
    cgb = cg_bytes(s, it_p, outer_p)
    mgb = pressure_solve_bytes(s, it_p, outer_p)
    gbs = (lambda b: b / (ps_ms / 1e3) / 1e9 if ps_ms > 0 else None)
    s.enable_stage_timing(False)

    # e2e: the same steps through the C ABI with a host read of the loads and
    # of the Vx, Vy, P fields every step (pfem2_step_and_read) into pinned
    # host buffers; the median of three runs of K steps, so that one
    # host-side stall does not stand for the whole measurement
    fields = (A.FIELD_VX, A.FIELD_VY, A.FIELD_P)
    loads = torch.zeros(5, dtype=torch.float64, pin_memory=True).numpy()
    out = torch.zeros(sp.mesh.n_vertices * len(fields), dtype=torch.float64, pin_memory=True).numpy()
    s.step_and_read(fields, loads, out)
    torch.cuda.synchronize()
    runs = []
    for _ in range(3):
        t0 = time.perf_counter()
        for _ in range(args.steps):
            s.step_and_read(fields, loads, out)
        runs.append(time.perf_counter() - t0)
    e2e_s = sorted(runs)[1]
    if world > 1:
        from pfem2_b200.sharding import max_over_ranks

        e2e_s = max_over_ranks(e2e_s)
    e2e = {"value": args.steps / e2e_s * world, "unit": "timesteps/s", "h2d_bytes_per_step": 0,
           "d2h_bytes_per_step": int(out.nbytes + loads.nbytes),
           "note": "the time stepper's state stays resident on the device: a step has no host inputs; "
                   "every step reads Vx, Vy, P and the loads back through pfem2_step_and_read"}
    s.close()

    # the FP64 path and the all-FP32 path on the same workload: speed, and
    # the field error of each path against FP64 after the same steps
    fp64 = cmp = None
    if not args.no_fp64:
        fp64 = channel_leg(args, local, flush, A.PREC_FP64, 0)
        fast = channel_leg(args, local, flush, A.PREC_MIXED, A.FP32_ALL)
        cmp = fixed_error(args, local)
        fast["rel_l2_vs_fp64"] = cmp.pop("fp32_all")

    stress = stress_leg(args, local, flush) if args.stress_n > 0 else None
    pipe = pipe_leg(args, local, flush) if args.pipe_n > 0 else None
    extras = extras_leg(args, local, flush)
    ensemble = None
    if args.ensemble_n > 0:
        ensemble = ensemble_leg(args, rank, world, local, flush, fp64)
    budget = budget_leg(args, local) if not args.no_fp64 else None

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        cpu = cpu_baseline(sp, threads=1, budget_s=20.0)

    cells = sp.mesh.n_cells
    res = {
        "metric": METRIC,
        "value": value,
        "unit": "timesteps/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64 fields, particles and assembly; f32 inner Krylov iterations refined in f64",
        "data": "synthetic (programmatic mesh, seeded particles)",
        "config": dict(WORKLOAD_DESC, cells=cells, vertices=sp.mesh.n_vertices,
                       particles=int(np_sum / args.steps), l2="flushed between timed steps (256 MB write)",
                       solver_stop=f"|r| <= {args.rtol:g} |b| in every solve (both paths)",
                       parallelism=f"replicas x{world}" if world > 1 else "single instance"),
        "fixed_error": cmp,
        "particle_updates_per_s": pupd,
        "cell_updates_per_s": cells * value,
        "stage_ms_per_step": {n: stages[i] / args.steps for i, n in enumerate(STAGE_NAMES)},
        "pressure_cg_iters_per_step": it_p / args.steps,
        "roofline": {"bound": "hbm", "kernel": "k_krylov<float, MG> (pressure solve: CG, multigrid preconditioner)",
                     "achieved": gbs(cgb), "peak": hbm, "peak_kind": peak_kind, "unit": "GB/s",
                     "frac": (gbs(cgb) / hbm) if gbs(cgb) else None,
                     "algorithmic_bytes_per_step": cgb / args.steps,
                     "bytes_model": "CG per row: SpMV 9 nnz x (4+4) + 12, 2 dots 16, 3 axpy 36, Jacobi 8 = 144 B "
                                    "x rows x live iterations, + FP64 refinements 136 B/row",
                     "traffic": KRYLOV_TRAFFIC_PER_LAUNCH,
                     "traffic_per_algorithmic_byte": KRYLOV_TRAFFIC_PER_LAUNCH / (cgb / args.steps) if cgb else None,
                     "traffic_source": KRYLOV_TRAFFIC_SOURCE,
                     "with_multigrid_operators": {"achieved": gbs(mgb), "frac": (gbs(mgb) / hbm) if gbs(mgb) else None,
                                                  "bytes_per_step": mgb / args.steps}},
        "e2e": e2e,
        "gpu_launches": int(launches),
        "clocks": clk,
        "fp64": fp64,
        "fp32_all": fast if not args.no_fp64 else None,
        "speedups": speedups(value, cells, fp64, ensemble),
        "particle_stress": stress,
        "pipe_3d": pipe,
        "vorticity_and_wall_pushback": extras,
        "ensemble": ensemble,
        "error_budget": budget,
        "cpu_baseline": cpu,
    }
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if rank == 0:
        print(json.dumps(res), flush=True)


# DRAM bytes (read + write) of one pressure-solve launch of the channel in
# the timed window (steps 5 and 6 after 4 warm-up steps, 31 and 30 CG
# iterations, rtol 1e-8): ncu dram__bytes_read.sum + dram__bytes_write.sum
# of `bench.py --only channel --steps 3 --warmup 4`, mean of the two
# launches. Under ncu every launch starts with a flushed L2, so this is one
# cold read of the solve's working set, which then stays in L2: it does
# not grow with the iteration count.
KRYLOV_TRAFFIC_PER_LAUNCH = 0.5 * ((27532032 + 54272) + (27526400 + 10240))
KRYLOV_TRAFFIC_SOURCE = ("ncu dram__bytes_read.sum + dram__bytes_write.sum of the k_krylov<float, MG> launches "
                         "of steps 5-6 (31 and 30 iterations) of `bench.py --only channel --steps 3 --warmup 4`; "
                         "per launch = per step")


def speedups(value, cells, fp64, ensemble):
    """like-for-like ratios in cell updates per second"""
    if not fp64:
        return None
    f = fp64["timesteps_per_s"] * cells
    out = {"mixed_over_fp64_single": value * cells / f}
    if ensemble:
        out["ensemble_mixed_over_fp64_single"] = ensemble["cell_updates_per_s"] / f
    return out


def channel_leg(args, local, flush, prec, stages):
    """the channel workload in one precision: K timed steps after W warm-up"""
    import torch

    from pfem2_b200.solver import STAGE_NAMES, Solver

    sp = workload(args)
    s = Solver(sp, precision=prec, fp32_stages=stages, device=local, use_graph=True)
    s.seed_particles(sp.q, sp.seed, sp.jitter)
    stream = torch.cuda.ExternalStream(s.stream(), device=local)
    for _ in range(args.warmup):
        s.step()
    s.synchronize()
    s.enable_stage_timing(True)
    s.stage_times(reset=True)
    ms, iters, viters = 0.0, [], []
    for _ in range(args.steps):
        ms += timed_steps(s, stream, flush, 1)
        st = s.stats()
        iters.append(st["iters"][3])
        viters.append([st["iters"][k] for k in (0, 1, 4, 5)])
    stages_ms = s.stage_times()
    out = {"timesteps_per_s": args.steps / (ms / 1e3), "ms_per_step": ms / args.steps,
           "fp32_stages": s.fp32_stages(),
           "stage_ms_per_step": {n: stages_ms[i] / args.steps for i, n in enumerate(STAGE_NAMES)},
           "pressure_cg_iters_per_step": iters,
           "velocity_iters_per_step": viters}
    s.close()
    return out


def fixed_error(args, local, steps=None):
    """relative L2 of Vx, Vy, P of the mixed path (and of the all-FP32 path)
    against the FP64 path after the bench's warm-up + timed steps"""
    from pfem2_b200 import _abi as A
    from pfem2_b200.solver import Solver

    n = steps or (args.warmup + args.steps)
    sp = workload(args)
    runs = {}
    for name, prec, stages in (("fp64", A.PREC_FP64, 0), ("mixed", A.PREC_MIXED, 0),
                               ("fp32_all", A.PREC_MIXED, A.FP32_ALL)):
        s = Solver(sp, precision=prec, fp32_stages=stages, device=local, use_graph=True)
        s.seed_particles(sp.q, sp.seed, sp.jitter)
        for _ in range(n):
            s.step()
        runs[name] = [s.field(f) for f in (A.FIELD_VX, A.FIELD_VY, A.FIELD_P)]
        s.close()
    err = {k: {f: rel_l2(a, b) for f, a, b in zip(("vx", "vy", "p"), runs[k], runs["fp64"])}
           for k in ("mixed", "fp32_all")}
    return {"bar": FIXED_ERROR, "steps_compared": n, "rel_l2_vs_fp64": err["mixed"],
            "met": max(err["mixed"].values()) <= FIXED_ERROR, "fp32_all": err["fp32_all"]}


def budget_leg(args, local, steps=25):
    """per-stage error budget: one FP32 stage at a time against FP64 on the
    channel (relative L2 of Vx, Vy, P after `steps` steps)"""
    from pfem2_b200 import _abi as A
    from pfem2_b200.solver import Solver

    sp = workload(args)
    sets = (("fp64", A.PREC_FP64, 0), ("krylov", A.PREC_MIXED, A.FP32_KRYLOV),
            ("particles", A.PREC_MIXED, A.FP32_PARTICLES), ("assembly", A.PREC_MIXED, A.FP32_ASSEMBLY),
            ("pressure_rhs", A.PREC_MIXED, A.FP32_PRESSURE_RHS), ("all", A.PREC_MIXED, A.FP32_ALL))
    runs = {}
    for name, prec, stages in sets:
        s = Solver(sp, precision=prec, fp32_stages=stages, device=local, use_graph=True)
        s.seed_particles(sp.q, sp.seed, sp.jitter)
        for _ in range(steps):
            s.step()
        runs[name] = [s.field(f) for f in (A.FIELD_VX, A.FIELD_VY, A.FIELD_P)]
        s.close()
    return {"workload": "the bench channel", "steps": steps,
            "fp32_stage_rel_l2_vs_fp64": {k: {f: rel_l2(a, b) for f, a, b in zip(("vx", "vy", "p"), v, runs["fp64"])}
                                          for k, v in runs.items() if k != "fp64"}}


def timed_steps(solver, stream, flush, steps):
    """per-step CUDA events on the library stream, L2 flushed between steps"""
    import torch

    tot = 0.0
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for _ in range(steps):
        with torch.cuda.stream(stream):
            flush.zero_()
        e0.record(stream)
        solver.step()
        e1.record(stream)
        e1.synchronize()
        tot += e0.elapsed_time(e1)
    return tot


def extras_leg(args, local, flush):
    """the kernels beyond the time step on the channel workload: the nodal
    vorticity (calculate_vorticity) and the wall push-back after the
    projection (its cost read from the projection stage, flag on vs off)"""
    import torch

    from pfem2_b200 import _abi as A
    from pfem2_b200 import cases
    from pfem2_b200.solver import STAGE_NAMES, Solver

    out = {}
    proj = {}
    for push in (0, 1):
        sp = cases.channel_disk(h=args.h, zero_ids=(3, 4), wall_pushback=push)
        s = Solver(sp, precision=A.PREC_MIXED, device=local, use_graph=True)
        s.seed_particles(sp.q, sp.seed, sp.jitter)
        stream = torch.cuda.ExternalStream(s.stream(), device=local)
        for _ in range(3):
            s.step()
        s.synchronize()
        s.enable_stage_timing(True)
        s.stage_times(reset=True)
        timed_steps(s, stream, flush, args.extra_steps)
        proj[push] = s.stage_times()[STAGE_NAMES.index("project_nodes")] / args.extra_steps
        if push == 1:
            # vorticity: K calls, CUDA events on the library stream
            s.enable_stage_timing(False)
            s.calculate_vorticity()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            k = 20
            with torch.cuda.stream(stream):
                flush.zero_()
            e0.record(stream)
            for _ in range(k):
                s.L.pfem2_calculate_vorticity(s.h)
            e1.record(stream)
            e1.synchronize()
            ms = e0.elapsed_time(e1) / k
            nv, nc = sp.mesh.n_vertices, sp.mesh.n_cells
            # algorithmic bytes: Vx, Vy and coordinates of every vertex (32 B),
            # the result (8 B), connectivity (16 B per cell)
            b = 40.0 * nv + 16.0 * nc
            hbm, kind = peaks()
            out["vorticity"] = {"ms": ms, "GB/s": b / (ms / 1e3) / 1e9, "frac": b / (ms / 1e3) / 1e9 / hbm,
                                "peak_kind": kind, "vertices": nv}
        s.close()
    out["wall_pushback"] = {"project_stage_ms_off": proj[0], "project_stage_ms_on": proj[1],
                            "walls": "disk and channel walls (boundary ids 3, 4)"}
    return out


def pipe_leg(args, local, flush):
    """3D pipe Poiseuille (hex mesh n x n x 4n, 3x3x3 particles per cell,
    dp/dn driven): the mixed path (FP32 inner solves refined in FP64) and the
    FP64 path on the same steps, one context after the other; the pressure
    solve's bytes by the CG per-row figure of the scope table (288 B/row in 3D)"""
    import torch

    from pfem2_b200 import _abi as A
    from pfem2_b200 import cases
    from pfem2_b200.solver import STAGE_NAMES, Solver

    n = args.pipe_n
    sp = tight(cases.pipe_3d(ny=n, nz=n, nx=4 * n), args.pipe_rtol)
    k, warm = args.extra_steps, 2
    out = {"workload": f"3D pipe Poiseuille, circular section mapped from a square, {n}x{n}x{4 * n} Q1 hex cells, "
                       f"nu=0.01, dt=0.001, dp/dn=1, 3x3x3 particles/cell",
           "cells": sp.mesh.n_cells, "vertices": sp.mesh.n_vertices, "steps": k, "warmup": warm,
           "solver_stop": f"|r| <= {args.pipe_rtol:g} |b|"}
    hbm, kind = peaks()
    fields = {}
    for name, prec in (("mixed", A.PREC_MIXED), ("fp64", A.PREC_FP64)):
        s = Solver(sp, precision=prec, device=local, use_graph=True)
        s.seed_particles(sp.q, sp.seed, sp.jitter)
        stream = torch.cuda.ExternalStream(s.stream(), device=local)
        for _ in range(warm):
            s.step()
        s.synchronize()
        s.enable_stage_timing(True)
        s.stage_times(reset=True)
        tot, e0, e1 = 0.0, torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        it_p = outer_p = 0
        for _ in range(k):
            with torch.cuda.stream(stream):
                flush.zero_()
            e0.record(stream)
            s.step()
            e1.record(stream)
            e1.synchronize()
            tot += e0.elapsed_time(e1)
            st = s.stats(check=False)
            it_p += st["iters"][3]
            outer_p += st["refinements_p"]
        ms = tot
        stages = s.stage_times()
        ps_ms = stages[STAGE_NAMES.index("pressure_solve")]
        cgb = cg_bytes(s, it_p, outer_p)
        out[name] = {"timesteps_per_s": k / (ms / 1e3), "ms_per_step": ms / k,
                     "stage_ms_per_step": {nm: stages[i] / k for i, nm in enumerate(STAGE_NAMES)},
                     "pressure_cg_iters_per_step": it_p / k, "particles": st["n_particles"],
                     "status": st["status"],
                     "pressure_solve_roofline": {"GB/s": cgb / (ps_ms / 1e3) / 1e9, "frac": cgb / (ps_ms / 1e3) / 1e9 / hbm,
                                                 "peak": hbm, "peak_kind": kind,
                                                 "bytes_per_step": cgb / k}}
        if name == "mixed":
            out["particle_updates_per_s"] = st["n_particles"] / (ms / k / 1e3)
        fields[name] = [s.field(f) for f in (A.FIELD_VX, A.FIELD_P)]
        s.close()
    out["mixed_vs_fp64_rel_l2"] = {nm: rel_l2(a, b) for nm, a, b in zip(("vx", "p"), fields["mixed"], fields["fp64"])}
    out["fixed_error_met"] = max(out["mixed_vs_fp64_rel_l2"].values()) <= FIXED_ERROR
    out["mixed_over_fp64"] = out["mixed"]["timesteps_per_s"] / out["fp64"]["timesteps_per_s"]
    return out


def stress_leg(args, local, flush):
    """particle kernels alone (advect + project + correct) on a frozen field:
    unit square n x n, 4x4 particles per cell uniform in their sub-cells,
    FP32 particle coordinates and velocities (PFEM2_FP32_PARTICLES)"""
    import torch

    from pfem2_b200 import _abi as A
    from pfem2_b200 import cases
    from pfem2_b200.solver import STAGE_NAMES, Solver

    n = args.stress_n
    sp = cases.stress_2d(n=n)
    s = Solver(sp, precision=A.PREC_MIXED, fp32_stages=A.FP32_ALL, device=local, use_graph=True,
               particles_only=True, capacity_factor=3.0)
    ux, uy = sp.meta["ux"], sp.meta["uy"]
    for f, v in ((A.FIELD_VX, ux), (A.FIELD_VY, uy), (A.FIELD_PRED_VX, ux), (A.FIELD_PRED_VY, uy)):
        s.set_field(f, v)
    s.seed_particles(sp.q, sp.seed, sp.jitter)
    stream = torch.cuda.ExternalStream(s.stream(), device=local)
    for _ in range(2):
        s.step()
    s.synchronize()
    s.enable_stage_timing(True)
    s.stage_times(reset=True)
    st0 = s.stats()
    ms = timed_steps(s, stream, flush, args.extra_steps)
    st = s.stats()
    stages = s.stage_times()
    k = args.extra_steps
    npart = 0.5 * (st0["n_particles"] + st["n_particles"])
    nc, nv = sp.mesh.n_cells, sp.mesh.n_vertices
    hbm, kind = peaks()
    # algorithmic bytes (FP32 SoA, the per-unit figures of the scope table):
    # advect with the correction fused: read cell + xi + u (20 B), write
    # xi + u + new cell (20 B) per particle, the nodal velocity and its
    # increment once (16 B per node); re-sort with check and projection
    # partials fused: read + write the particle state (2 x 20 B) plus keys
    # and offsets (8 B) per particle, 48 B of partials and a 4 B offset per
    # cell; node gather: the partials (48 B per cell) in, 12 B per node out
    b_adv = 40.0 * npart + 16.0 * nv
    b_reb = 48.0 * npart + 52.0 * nc
    b_nod = 48.0 * nc + 12.0 * nv
    adv_ms = stages[STAGE_NAMES.index("advect")] / k
    reb_ms = stages[STAGE_NAMES.index("rebin")] / k
    nod_ms = stages[STAGE_NAMES.index("project_nodes")] / k
    gbs = lambda b, t: b / (t / 1e3) / 1e9 if t > 0 else None
    out = {
        "workload": f"unit square {n}x{n} Q1, 4x4 particles/cell uniform in sub-cells (seed 1), frozen "
                    f"divergence-free field of 32 random stream-function modes, CFL 0.5; correct+advect+rebin+project",
        "cells": nc, "particles": int(npart), "ms_per_step": ms / k,
        "particle_updates_per_s": npart * k / (ms / 1e3),
        "advect": {"ms": adv_ms, "GB/s": gbs(b_adv, adv_ms), "frac": gbs(b_adv, adv_ms) / hbm if adv_ms else None},
        "rebin": {"ms": reb_ms, "GB/s": gbs(b_reb, reb_ms), "frac": gbs(b_reb, reb_ms) / hbm if reb_ms else None},
        "project_nodes": {"ms": nod_ms, "GB/s": gbs(b_nod, nod_ms), "frac": gbs(b_nod, nod_ms) / hbm if nod_ms else None},
        "bytes_per_step": {"advect": b_adv, "rebin": b_reb, "project_nodes": b_nod},
        "step_GB/s": gbs(b_adv + b_reb + b_nod, ms / k), "peak": hbm, "peak_kind": kind,
        "deleted_per_step": st["deleted"], "far_movers": st["far"],
    }
    s.close()
    return out


def ensemble_leg(args, rank, world, local, flush, fp64_single):
    """many independent channel instances of uneven size in one batch:
    every stage is one launch for all of them (mixed path, the bench's
    relative tolerance); with N ranks every rank runs its longest-processing-
    time share of the instances (no collective but the max-over-ranks time)"""
    import torch

    from pfem2_b200 import _abi as A
    from pfem2_b200 import cases, sharding
    from pfem2_b200.solver import STAGE_NAMES, Solver

    all_specs = [tight(sp, args.rtol) for sp in cases.ensemble(n=args.ensemble_n)]
    specs = all_specs
    if world > 1:
        _, specs = sharding.shard(all_specs, rank, world)
    s = Solver(specs, precision=A.PREC_MIXED, device=local, use_graph=True)
    s.seed_particles(specs[0].q, 2, 0.0)
    stream = torch.cuda.ExternalStream(s.stream(), device=local)
    for _ in range(3):
        s.step()
    s.synchronize()
    s.enable_stage_timing(True)
    s.stage_times(reset=True)
    ms = timed_steps(s, stream, flush, args.extra_steps)
    stages = s.stage_times()
    if world > 1:
        ms = sharding.max_over_ranks(ms)
    st = s.stats()
    cells = sum(sp.mesh.n_cells for sp in all_specs)
    inst_steps = len(all_specs) * args.extra_steps / (ms / 1e3)
    out = {
        "workload": f"{len(specs)} channel-with-disk instances, cells log-uniform 5k-60k, Re log-uniform 20-200, "
                    f"r uniform 0.05-0.15 (seed 2), 5x5 particles/cell, one batch",
        "instances": len(all_specs), "cells": cells, "particles_rank0": st["n_particles"],
        "sharding": f"lpt over {world} ranks" if world > 1 else "one batch",
        "ms_per_batch_step": ms / args.extra_steps, "instance_timesteps_per_s": inst_steps,
        "cell_updates_per_s": cells * args.extra_steps / (ms / 1e3),
        "max_pressure_cg_iters": st["iters"][3], "far_movers_last_step": st["far"],
        "stage_ms_per_step": {n: stages[i] / args.extra_steps for i, n in enumerate(STAGE_NAMES)},
    }
    s.close()
    return out


def cpu_baseline(sp, threads, budget_s):
    """FP64 CPU restatement of the reference (oracle/) on the same workload:
    time whole steps until the budget is used (>= 1 step)."""
    import oracle as O

    o = O.Oracle(sp.mesh, sp.case, movement_steps=sp.movement_steps, max_per_part=sp.max_per_part,
                 threads=threads)
    o.seed_particles(sp.q, sp.seed, sp.jitter)
    o.step(1)  # warm-up step (first-touch, assembly)
    n = 0
    t0 = time.perf_counter()
    while True:
        o.step(1)
        n += 1
        el = time.perf_counter() - t0
        if el > budget_s or n >= 50:
            break
    return {"value": n / el, "unit": "timesteps/s", "cores": threads, "kind": "port",
            "sample": f"{n} whole time steps of the same workload after 1 warm-up step, FP64, "
                      f"{threads} thread(s)"}


def run_reference(args, rank, world):
    if rank != 0:
        return
    sp = workload(args)
    threads = os.cpu_count() or 1
    import oracle as O

    o = O.Oracle(sp.mesh, sp.case, movement_steps=sp.movement_steps, max_per_part=sp.max_per_part,
                 threads=threads)
    o.seed_particles(sp.q, sp.seed, sp.jitter)
    warm = max(1, min(args.warmup, 2))
    for _ in range(warm):
        o.step(1)
    budget = 120.0
    n = 0
    t0 = time.perf_counter()
    while n < args.steps:
        o.step(1)
        n += 1
        if time.perf_counter() - t0 > budget:
            break
    el = time.perf_counter() - t0
    v = n / el
    res = {
        "impl": "reference",
        "metric": METRIC,
        "value": v, "unit": "timesteps/s", "n_gpus": world, "steps": n, "warmup": warm,
        "ms_per_step": el / n * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (programmatic mesh, seeded particles)",
        "config": dict(WORKLOAD_DESC, cells=sp.mesh.n_cells, parallelism="host cores"),
        "cpu_baseline": {"value": v, "unit": "timesteps/s", "cores": threads, "kind": "port",
                         "sample": f"{n} whole time steps (of {args.steps} requested, 120 s cap) after "
                                   f"{warm} warm-up steps (of {args.warmup} requested); deal.II, which the "
                                   f"reference needs, is not installed, so its FP64 CPU restatement runs",
                         "parallel_parts": "OpenMP over particle advection, right-hand sides, SpMV and the Krylov "
                                           "vector operations; the pressure's SSOR preconditioner is sequential "
                                           "(as deal.II's), which bounds the scaling (8-core host: 0.45 "
                                           "timesteps/s on 1 thread, 0.90 on 4, 0.95 on 8)"},
        "e2e": {"value": v, "unit": "timesteps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(res), flush=True)


# the launch shapes the autotuner chose for these workloads on a B200
# (pfem2_b200/autotune.py); a tuning cache named in the environment wins
TUNING_CACHE = os.path.join(ROOT, "pfem2_b200", "tuning", "b200.txt")


def main():
    os.environ.setdefault("PFEM2_TUNING_CACHE", TUNING_CACHE)
    args = parse()
    rank, world, local = dist_info()
    if args.impl == "reference":
        run_reference(args, rank, world)
    else:
        run_ours(args, rank, world, local)


if __name__ == "__main__":
    main()
