"""Shared helpers of the parity tests (oracle vs CUDA library)."""
import numpy as np


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    n = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (n if n > 0 else 1.0))


def near_face(xi, eps):
    xi = np.asarray(xi)
    return np.any(np.minimum(xi, 1.0 - xi) < eps, axis=-1)


def compare_particles(o, g, eps_face, xi_tol, u_tol):
    """o, g: (cell, xi, u) in storage order (sorted by cell, stable).

    Cells whose particle counts agree are compared element-wise. Particles of
    cells whose counts differ must all lie within eps_face (reference units)
    of a face of their cell: membership may flip only there.
    Returns a dict of statistics; raises AssertionError on a violation.
    """
    oc, ox, ou = o
    gc, gx, gu = g
    ncell = int(max(oc.max(initial=-1), gc.max(initial=-1))) + 1
    co = np.bincount(oc, minlength=ncell)
    cg = np.bincount(gc, minlength=ncell)
    so = np.concatenate([[0], np.cumsum(co)])
    sg = np.concatenate([[0], np.cumsum(cg)])
    same = co == cg
    idx_o = np.concatenate([np.arange(so[c], so[c + 1]) for c in np.nonzero(same)[0]]) if same.any() else np.zeros(0, int)
    idx_g = np.concatenate([np.arange(sg[c], sg[c + 1]) for c in np.nonzero(same)[0]]) if same.any() else np.zeros(0, int)
    dxi = np.abs(ox[idx_o] - gx[idx_g]).max(initial=0.0)
    du = np.abs(ou[idx_o] - gu[idx_g]).max(initial=0.0)
    bad_cells = np.nonzero(~same)[0]
    flips = 0
    max_flip_dist = 0.0
    for c in bad_cells:
        a = ox[so[c]:so[c + 1]]
        b = gx[sg[c]:sg[c + 1]]
        # every particle not matched by a near-identical partner must be near a face
        for arr, other in ((a, b), (b, a)):
            for p in arr:
                if other.size and np.abs(other - p).max(axis=1).min() < 10 * xi_tol:
                    continue
                assert near_face(p[None, :], eps_face)[0], f"membership differs away from faces in cell {c}: {p}"
                flips += 1
                max_flip_dist = max(max_flip_dist, float(np.min(np.minimum(p, 1.0 - p))))
    assert dxi <= xi_tol, f"max |xi diff| {dxi} > {xi_tol}"
    assert du <= u_tol, f"max |u diff| {du} > {u_tol}"
    return {"dxi": dxi, "du": du, "flip_cells": len(bad_cells), "flips": flips,
            "max_flip_dist": max_flip_dist, "n_o": len(oc), "n_g": len(gc)}


# Precision modes of the library under test:
#   fp64   everything FP64 (PFEM2_PREC_FP64)
#   mixed  the default mixed path: FP32 inner Krylov iterations refined in
#          FP64, everything else FP64 (fields within 1e-6 of fp64)
#   fp32   every stage that can run in FP32 does (particles, right-hand
#          sides, inner Krylov): the fast path, looser bars
MODES = ["fp64", "mixed", "fp32"]


def solver_kw(mode):
    from pfem2_b200 import _abi as A

    return {"fp64": {"precision": A.PREC_FP64, "fp32_stages": 0},
            "mixed": {"precision": A.PREC_MIXED, "fp32_stages": 0},
            "fp32": {"precision": A.PREC_MIXED, "fp32_stages": A.FP32_ALL}}[mode]
