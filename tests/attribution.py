"""Attribution of every difference between a fast-policy device pass and the f64 oracle.

The fast policy forms window costs in f32 (homographies composed in f64,
f32 taps), so its costs differ from the reference's f64 costs by a bounded
error.  An output can then differ from the oracle's only where a cost-based
decision of the pass lay within that error of going the other way.  This
module checks exactly that, site by site, against the oracle's decision
records (``Oracle.explain_reference_patch``, ``ExplainRecord`` in
oracle/oracle.hpp):

* sweep: the chosen hypothesis index is compared site by site; a site whose
  hypothesis moved (or whose comparable second moved, which changes the
  margin) is a *moved hypothesis* and counts against the >= 99.9 % agreement
  rule; a site whose accept/reject status differs at the same hypothesis must
  have its best cost or its margin within ``band`` of the gate (the oracle's
  ``sweep_gap``);
* reciprocal check and fusion (dense_legacy.rs:777-884): at a site both
  sweeps accepted with the same hypothesis, a point present in one result
  only, or fused points that differ by more than 1e-5 relative, must come
  from a reciprocal decision within ``band`` of its threshold or a near tie
  in a source's single-view sweep (``recip_gap``): a *moved reciprocal
  hypothesis*;
* completion (dense_legacy.rs:519-737): a completion point present in one
  result only or differing must have a differing neighbour on the grid (its
  prediction reads the neighbours) or its own direct-cost or reciprocal gap
  within ``band``.

Everything else is unexplained and fails the test.  ``band`` is twice the
stated cost tolerance of the fast policy: a margin is a difference of two
costs, and a tie between two hypotheses flips when their errors differ.
"""
import numpy as np

POINT_TOL = 1e-5  # fused points agree to 1e-5 relative
# The fast policy's stated cost tolerance: |f32 window cost - f64 window cost|
# of the chosen hypotheses stays below it (the tests assert it); decisions are
# attributed within twice it.
COST_TOLERANCE = 1e-4


def _key(x, y):
    return (int(x), int(y))


def attribute(g, g_sweep, o, o_rec, prof, band, rows=None):
    """g / o: the device and oracle analyses of one pass (points in the
    reference's order: primaries, then completions); g_sweep: the device's
    per-site sweep records; o_rec: the oracle's decision records of the same
    pass.  rows=(a, b): the oracle ran grid rows a..b-1 only (primaries, no
    completion); the device's full pass is compared on those rows.  Returns a
    report; ``report["unexplained"]`` lists the sites no rule covers."""
    y_lo, y_hi = 0, 1 << 62
    if rows is not None:
        border, stride = int(g.stats["grid_border"]), int(g.stats["grid_stride"])
        y_lo, y_hi = border + rows[0] * stride, border + rows[1] * stride
        g_sweep = g_sweep[(g_sweep["y"] >= y_lo) & (g_sweep["y"] < y_hi)]
    thr_e, thr_m = prof.max_photometric_error, prof.min_ambiguity_margin
    prim = o_rec[o_rec["stage"] == 0]
    comp = o_rec[o_rec["stage"] > 0]
    orec = {_key(r["x"], r["y"]): r for r in prim}
    gsw = {_key(r["x"], r["y"]): r for r in g_sweep}
    rep = {"band": band, "sites": len(g_sweep), "sampled": 0, "moved": 0, "second_moved": 0,
           "gate_band": 0, "gate_band_over_1e-5": 0, "recip_moved": 0,
           "recip_moved_over_1e-5": 0, "completion_cascade": 0, "completion_band": 0,
           "points_compared": 0, "points_equal_bits": 0, "positions_equal_bits": 0,
           "max_cost_error": 0.0,
           "median_cost_error": 0.0, "max_confidence_delta": 0.0, "unexplained": []}
    unexplained = rep["unexplained"]
    # ---- sweep -------------------------------------------------------------
    contrast_mismatch = 0
    moved_sites = set()
    errs = []
    for k, gr in gsw.items():
        orr = orec.get(k)
        g_status = int(gr["status"])
        o_status = 1 if orr is None else min(int(orr["outcome"]), 4)
        if (g_status == 1) != (o_status == 1):
            contrast_mismatch += 1  # the contrast gate reads exact pixel values in both
            unexplained.append(("contrast", k))
            continue
        if g_status == 1:
            continue
        rep["sampled"] += 1
        if g_status >= 3 and o_status >= 3:
            if int(gr["plane"]) != int(orr["plane"]):
                rep["moved"] += 1
                moved_sites.add(k)
                continue
            errs.append(abs(float(gr["error"]) - float(orr["error"])))
            gm, om = float(gr["margin"]), float(orr["margin"])
            if np.isinf(gm) != np.isinf(om) or (np.isfinite(om) and abs(gm - om) > band):
                if g_status != o_status:
                    rep["second_moved"] += 1
                    moved_sites.add(k)
                continue
        if g_status != o_status:
            gap = float(orr["sweep_gap"])
            if gap <= band:
                rep["gate_band"] += 1
                rep["gate_band_over_1e-5"] += int(gap > 1e-5)
                moved_sites.add(k)
            else:
                unexplained.append(("sweep", k, g_status, o_status, gap))
    if errs:
        rep["max_cost_error"] = float(np.max(errs))
        rep["median_cost_error"] = float(np.median(errs))
    # ---- points --------------------------------------------------------------
    # accepted_points counts the completed points too (dense_legacy.rs sets it after
    # completion); the primaries come first
    n_gp = g.stats["accepted_points"] - g.stats["surface_completed_points"]
    n_op = (o.stats["accepted_points"] - o.stats["surface_completed_points"] if rows is None
            else len(o.points))

    def table(a, lo, hi):
        t = {}
        for i in range(lo, hi):
            s = a.grid_sites[i]
            if y_lo <= int(s["y"]) < y_hi:
                t[_key(s["x"], s["y"])] = i
        return t

    gpt, opt = table(g, 0, n_gp), table(o, 0, n_op)
    if rows is None:
        gct, oct_ = table(g, n_gp, len(g.points)), table(o, n_op, len(o.points))
    else:
        gct, oct_ = {}, {}  # the band ran no completion

    def differs(i, j):
        gp = np.array([g.points[i][c] for c in "xyz"], np.float64)
        op = np.array([o.points[j][c] for c in "xyz"], np.float64)
        rel = np.linalg.norm(gp - op) / max(np.linalg.norm(op), 1e-30)
        rep["points_compared"] += 1
        if g.points[i].tobytes() == o.points[j].tobytes():
            rep["points_equal_bits"] += 1
        if all(g.points[i][c].tobytes() == o.points[j][c].tobytes() for c in "xyz"):
            rep["positions_equal_bits"] += 1
        rep["max_confidence_delta"] = max(rep["max_confidence_delta"],
                                          abs(float(g.points[i]["confidence"]) -
                                              float(o.points[j]["confidence"])))
        return rel > POINT_TOL

    diff_sites = set(moved_sites)
    for k in set(gpt) | set(opt):
        if k in moved_sites:
            continue  # the sweep decided differently: already attributed
        if k in gpt and k in opt and not differs(gpt[k], opt[k]):
            continue
        diff_sites.add(k)
        orr = orec.get(k)
        gap = float(orr["recip_gap"]) if orr is not None else np.inf
        if gap <= band:
            rep["recip_moved"] += 1
            rep["recip_moved_over_1e-5"] += int(gap > 1e-5)
        else:
            unexplained.append(("reciprocal", k, k in gpt, k in opt, gap))
    # ---- completion ------------------------------------------------------------
    ocomp = {}
    for r in comp:  # the last pass's record of a site is the one that decided it
        ocomp[_key(r["x"], r["y"])] = r
    stride = int(g.stats["grid_stride"])
    pending = []
    for k in set(gct) | set(oct_):
        if k in gct and k in oct_ and not differs(gct[k], oct_[k]):
            continue
        pending.append(k)
    # a completion difference is explained by its own gap or by a neighbour
    # whose difference is itself explained (grounded in the primaries)
    explained = set(diff_sites)

    def neighbour_explained(k):
        x, y = k
        return any((x + dx * stride, y + dy * stride) in explained
                   for dy in (-1, 0, 1) for dx in (-1, 0, 1) if dx or dy)

    changed = True
    while changed and pending:
        changed = False
        rest = []
        for k in pending:
            r = ocomp.get(k)
            if r is not None and min(float(r["sweep_gap"]), float(r["recip_gap"])) <= band:
                rep["completion_band"] += 1
            elif neighbour_explained(k):
                rep["completion_cascade"] += 1
            else:
                rest.append(k)
                continue
            explained.add(k)
            changed = True
        pending = rest
    for k in pending:
        unexplained.append(("completion", k, k in gct, k in oct_))
    rep["moved_fraction"] = (rep["moved"] + rep["second_moved"]) / max(1, rep["sampled"])
    return rep
