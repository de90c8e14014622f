"""Autotuner of the library's launch shapes (pfem2_tuning, include/pfem2.h).

The particle kernels and the persistent Krylov solver have shapes that the
best choice of depends on the GPU and the mesh size: the advection grid
(particles per block) and whether advection runs in one pass or in two
phases (stayers, then queued leavers), the re-sort grid, the velocity
solves' tile size (SELL slices per tile) and blocks per SM, and the blocks
per SM of a single pressure system's multigrid solve. `tune` times whole
steps (the device time of every stage,
CUDA events inside the library) for candidate shapes by coordinate descent
(coupled knobs, such as the advection grid and its one- or two-phase form,
over all their combinations) and appends the fastest to a cache file under the context's key: device
name, dim, FP32 stages, log2 cells, log2 instances (pfem2_tuning_key). A
later context with the same key reads the entry at pfem2_setup when the
environment variable PFEM2_TUNING_CACHE names the file; fields the caller
sets explicitly win over the cache.

    from pfem2_b200 import autotune, cases
    res = autotune.tune([cases.channel_disk()], cache="pfem2_tuning.txt")

The particle shapes never change results (bitwise); the solver shapes change
the order of partial sums (tile size) or the preconditioner (blocks per SM),
within the solver tolerance.
"""
import os

import numpy as np

from . import _abi as A
from .solver import Pfem2Error, Solver

DEFAULT_SPACE = {
    "advect_blocks_per_sm": [2, 4, 8, 16],
    "advect_split": [1, 2],
    "rebin_blocks_per_sm": [2, 4, 6, 8, 12],
    "vel_tile_slices": [4, 8, 16, 32],
    "p_blocks_per_sm": [1, 2],
    "vel_blocks_per_sm": [1, 2],
}


def measure(specs, tuning, steps=5, warmup=2, seed_q=None, prepare=None, **solver_kw):
    """median device time of a step (ms) with the given shapes, and the
    shapes the context resolved; (None, None) if the context refuses them"""
    try:
        s = Solver(specs, tuning=tuning, use_graph=True, **solver_kw)
    except Pfem2Error:
        return None, None
    try:
        if prepare:
            prepare(s)
        sp = specs[0] if isinstance(specs, (list, tuple)) else specs
        s.seed_particles(seed_q or sp.q, sp.seed, sp.jitter)
        for _ in range(warmup):
            s.step()
        s.synchronize()
        s.enable_stage_timing(True)
        times = []
        s.stage_times(reset=True)
        for _ in range(steps):
            s.step()
            times.append(float(np.sum(s.stage_times(reset=True))))
        resolved = s.tuning()
        s.stats()  # raises on a failed step
        return float(np.median(times)), resolved
    except Pfem2Error:
        return None, None
    finally:
        s.close()


def cache_line(key, tuning, ms):
    vals = " ".join(str(int(tuning[k])) for k in A.TUNING_FIELDS)
    return f"{key} {vals} {ms:.4f}\n"


def tune(specs, space=None, steps=5, warmup=2, cache=None, rounds=1, prepare=None, **solver_kw):
    """Coordinate descent over `space` (knob -> candidate values) starting from
    the automatic shapes. Returns {"key", "tuning", "ms_per_step",
    "baseline_ms", "trials"}; with `cache` the best entry is appended there."""
    space = DEFAULT_SPACE if space is None else space
    # the candidates are timed without an existing cache's entries
    saved = os.environ.pop("PFEM2_TUNING_CACHE", None)
    try:
        return _tune(specs, space, steps, warmup, cache, rounds, prepare, solver_kw)
    finally:
        if saved is not None:
            os.environ["PFEM2_TUNING_CACHE"] = saved


# knobs whose best values depend on each other are searched together (every
# combination), the others one at a time
COUPLED = [("advect_blocks_per_sm", "advect_split"), ("vel_tile_slices", "vel_blocks_per_sm")]


def _groups(space):
    groups, done = [], set()
    for grp in COUPLED:
        g = tuple(k for k in grp if k in space)
        if g:
            groups.append(g)
            done.update(g)
    groups += [(k,) for k in space if k not in done]
    return groups


def _tune(specs, space, steps, warmup, cache, rounds, prepare, solver_kw):
    import itertools

    t0, best = measure(specs, None, steps, warmup, prepare=prepare, **solver_kw)
    if t0 is None:
        raise RuntimeError("the automatic launch shapes failed")
    probe = Solver(specs, use_graph=True, **solver_kw)
    key = probe.tuning_key()
    probe.close()
    best = {k: v for k, v in best.items() if k in space or v}
    best_t = t0
    trials = [({k: best[k] for k in best}, t0)]
    for _ in range(rounds):
        for grp in _groups(space):
            for combo in itertools.product(*(space[k] for k in grp)):
                if all(best.get(k) == v for k, v in zip(grp, combo)):
                    continue
                cand = dict(best, **dict(zip(grp, combo)))
                t, resolved = measure(specs, cand, steps, warmup, prepare=prepare, **solver_kw)
                trials.append((cand, t))
                if t is not None and t < best_t:
                    best_t, best = t, {k: resolved[k] for k in best}
    full = {k: int(best.get(k, 0)) for k in A.TUNING_FIELDS}
    if cache:
        with open(cache, "a") as f:
            f.write(cache_line(key, full, best_t))
    return {"key": key, "tuning": full, "ms_per_step": best_t, "baseline_ms": t0, "trials": trials}


def read_cache(path):
    """{key: (tuning dict, ms)} of a cache file, the last entry per key"""
    out = {}
    if not os.path.exists(path):
        return out
    for ln in open(path):
        if ln.startswith("#") or not ln.strip():
            continue
        parts = ln.split()
        if len(parts) < 10:
            continue
        key = " ".join(parts[:5])
        vals, ms = [], None
        for x in parts[5:]:
            if "." in x:
                ms = float(x)
                break
            if len(vals) < len(A.TUNING_FIELDS):
                vals.append(int(x))
        vals += [0] * (len(A.TUNING_FIELDS) - len(vals))
        out[key] = (dict(zip(A.TUNING_FIELDS, vals)), ms)
    return out


def main(argv=None):
    """Tunes the launch shapes of named workloads and appends them to a
    cache file:  python -m pfem2_b200.autotune --cache FILE [--workloads ...]"""
    import argparse

    from . import cases

    ap = argparse.ArgumentParser(description=main.__doc__)
    ap.add_argument("--cache", required=True)
    ap.add_argument("--workloads", nargs="+", default=["channel_mixed", "channel_fp64"],
                    choices=["channel_mixed", "channel_fp64", "stress", "pipe_mixed", "ensemble"])
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--rtol", type=float, default=1e-8)
    args = ap.parse_args(argv)

    def tight(sp, rtol):
        sp.case.vel_tol = sp.case.p_tol = 0.0
        sp.case.vel_rtol = sp.case.p_rtol = rtol
        return sp

    particle_space = {k: DEFAULT_SPACE[k] for k in ("advect_blocks_per_sm", "advect_split", "rebin_blocks_per_sm")}
    for w in args.workloads:
        prepare = None
        if w.startswith("channel"):
            specs = [tight(cases.channel_disk(), args.rtol)]
            kw = {"precision": A.PREC_MIXED if w == "channel_mixed" else A.PREC_FP64}
            space = DEFAULT_SPACE
        elif w == "pipe_mixed":
            specs = [tight(cases.pipe_3d(), 1e-11)]
            kw = {"precision": A.PREC_MIXED}
            space = {"p_blocks_per_sm": [1, 2], "vel_tile_slices": [8, 16, 32], "vel_blocks_per_sm": [1, 2],
                     "advect_blocks_per_sm": [8, 16], "rebin_blocks_per_sm": [4, 8]}
        elif w == "ensemble":
            specs = [tight(sp, args.rtol) for sp in cases.ensemble()]
            kw = {"precision": A.PREC_MIXED}
            space = {k: v for k, v in DEFAULT_SPACE.items() if k != "p_blocks_per_sm"}
        else:
            sp = cases.stress_2d()
            specs = [sp]
            kw = {"precision": A.PREC_MIXED, "fp32_stages": A.FP32_ALL, "particles_only": True,
                  "capacity_factor": 3.0}
            space = particle_space

            def prepare(s, sp=sp):
                for f, v in ((A.FIELD_VX, sp.meta["ux"]), (A.FIELD_VY, sp.meta["uy"]),
                             (A.FIELD_PRED_VX, sp.meta["ux"]), (A.FIELD_PRED_VY, sp.meta["uy"])):
                    s.set_field(f, v)
        res = tune(specs, space=space, steps=args.steps, warmup=2, cache=args.cache, prepare=prepare, **kw)
        print(w, res["key"], res["tuning"], f"{res['baseline_ms']:.4f} -> {res['ms_per_step']:.4f} ms", flush=True)


if __name__ == "__main__":
    main()
