"""Run one of the PFEM2 workloads for a few steps (command line).

    python -m pfem2_b200.workloads --case channel --steps 5
    python -m pfem2_b200.workloads --case stress --n 1024 --steps 3
    python -m pfem2_b200.workloads --case pipe --steps 2
    python -m pfem2_b200.workloads --case ensemble --instances 8 --steps 2

Prints one JSON line with the step time (CUDA events on the library stream)
and the solver statistics. It is the program the ncu captures under
profiles/ run, and a quick way to try a workload.
"""
import argparse
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def build_solver(args):
    from pfem2_b200 import _abi as A
    from pfem2_b200 import cases
    from pfem2_b200.solver import Solver

    prec = A.PREC_FP64 if args.fp64 else A.PREC_MIXED
    if args.case == "channel":
        sp = cases.channel_disk()
        s = Solver(sp, precision=prec)
        s.seed_particles(sp.q, sp.seed, sp.jitter)
    elif args.case == "poiseuille":
        sp = cases.poiseuille_2d()
        s = Solver(sp, precision=prec)
        s.seed_particles(sp.q, sp.seed, sp.jitter)
    elif args.case == "pipe":
        sp = cases.pipe_3d(ny=args.n or 64, nz=args.n or 64, nx=4 * (args.n or 64))
        s = Solver(sp, precision=prec)
        s.seed_particles(sp.q, sp.seed, sp.jitter)
    elif args.case == "stress":
        sp = cases.stress_2d(n=args.n or 2048)
        s = Solver(sp, precision=prec, particles_only=True, capacity_factor=3.0)
        for f, v in ((A.FIELD_VX, sp.meta["ux"]), (A.FIELD_VY, sp.meta["uy"]), (A.FIELD_PRED_VX, sp.meta["ux"]),
                     (A.FIELD_PRED_VY, sp.meta["uy"])):
            s.set_field(f, v)
        s.seed_particles(sp.q, sp.seed, sp.jitter)
    elif args.case == "ensemble":
        specs = cases.ensemble(n=args.instances)
        s = Solver(specs, precision=prec)
        s.seed_particles(specs[0].q, 2, 0.0)
    else:
        raise SystemExit(f"unknown case {args.case}")
    return s


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--case", default="channel", choices=["channel", "poiseuille", "pipe", "stress", "ensemble"])
    ap.add_argument("--n", type=int, default=0)
    ap.add_argument("--instances", type=int, default=8)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=1)
    ap.add_argument("--fp64", action="store_true")
    ap.add_argument("--stages", action="store_true", help="also report the per-stage device time per step")
    args = ap.parse_args()
    import torch

    s = build_solver(args)
    stream = torch.cuda.ExternalStream(s.stream())
    for _ in range(args.warmup):
        s.step()
    s.synchronize()
    if args.stages:
        s.enable_stage_timing(True)
        s.stage_times(reset=True)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        s.step()
    e1.record(stream)
    e1.synchronize()
    st = s.stats(False)
    out = {"case": args.case, "steps": args.steps, "ms_per_step": e0.elapsed_time(e1) / args.steps,
           "n_particles": st["n_particles"], "iters": st["iters"], "status": st["status"]}
    if args.stages:
        from pfem2_b200.solver import STAGE_NAMES
        out["stage_ms_per_step"] = dict(zip(STAGE_NAMES, (t / args.steps for t in s.stage_times())))
    print(json.dumps(out))
    s.close()


if __name__ == "__main__":
    main()
