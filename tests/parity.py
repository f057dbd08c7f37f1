"""Shared parity checks: per-rotation minimum energy and first argmin against an oracle.

Tolerances (the path's stated bar):
  * FP32 form: |E - E_ref| <= 1e-4 * max(|E_ref|, 1)   (relative, with a floor of 1 kcal/mol
    so that minima near zero are judged on the energy scale rather than on their own size)
  * argmin identical, except at a stated near-tie: the oracle's second-best translation lies
    within 1e-4 * max(|E_ref|, 1) of its best.
"""
from __future__ import annotations

import numpy as np

REL_TOL = 1e-4
FLOOR = 1.0


def rel_err(e, e_ref):
    e = np.asarray(e, np.float64)
    r = np.asarray(e_ref, np.float64)
    both_inf = np.isinf(e) & np.isinf(r) & (np.sign(e) == np.sign(r))
    err = np.abs(e - r) / np.maximum(np.abs(r), FLOOR)
    err[both_inf] = 0.0
    return err


def near_tie(emap: np.ndarray, tol_abs: float) -> bool:
    """True when the second smallest value of the window map is within tol_abs of the best."""
    flat = np.sort(emap.reshape(-1))
    return flat.size > 1 and (flat[1] - flat[0]) <= tol_abs


def check_search(minE, idx, ref_minE, ref_idx, emap_fn=None, rel_tol=REL_TOL):
    """Returns a dict of statistics; asserts the bar. emap_fn(r) gives the oracle's double
    energy map of rotation r (used only for rotations whose argmin differs)."""
    err = rel_err(minE, ref_minE)
    assert np.all(np.isfinite(err)), "non-finite error"
    worst = int(np.argmax(err))
    assert err.max() <= rel_tol, f"max rel err {err.max():.3e} at rotation {worst}: " \
        f"{minE[worst]} vs {ref_minE[worst]}"
    diff = np.where(np.any(np.asarray(idx) != np.asarray(ref_idx), axis=1))[0]
    ties = 0
    for r in diff:
        assert emap_fn is not None, f"argmin differs at rotation {r} and no map to judge ties"
        emap = emap_fn(int(r))
        tol = rel_tol * max(abs(float(ref_minE[r])), FLOOR)
        assert near_tie(emap, tol), f"argmin differs at rotation {r} without a near-tie: " \
            f"{idx[r]} vs {ref_idx[r]}"
        ties += 1
    return {"max_rel": float(err.max()), "median_rel": float(np.median(err)),
            "argmin_diff": int(diff.size), "near_ties": ties, "n": int(len(minE))}
