"""Depth-grid verification on the CPU: the oracle through its C entry point
against the reference's own test plane, and the invariants of its outcome on
seeded clips."""
import numpy as np
import pytest

from v3d import types

from tests import depth_grid_scenes
from tests.oracle_ffi import Oracle


def test_reference_plane_through_the_c_entry_point():
    # colmap_surface.rs:633-730
    frame, other_color, first, second, depth, wrong = depth_grid_scenes.reference_plane()
    views = [(frame, depth, first), (frame, depth, second), (frame, wrong, second),
             (other_color, depth, second), (frame, depth, first)]
    o = Oracle()
    per_ref, funnel = o.verify_depth_grids(views, [0], [[1]], 4, 4, 20.0)
    assert len(per_ref[0]) == 20
    assert funnel == {"reference_samples": 24, "missing_reference_depth": 0,
                      "insufficient_parallax": 0, "behind_source": 0, "outside_source": 4,
                      "missing_source_depth": 0, "depth_disagreement": 0,
                      "color_disagreement": 0, "accepted": 20}
    coarse, _ = o.verify_depth_grids(views, [0], [[1]], 4, 8, 20.0)
    assert len(coarse[0]) == 4
    assert (coarse[0]["site_x"] % 8 == 0).all() and (coarse[0]["site_y"] % 8 == 0).all()
    for source, gate in [(2, "depth_disagreement"), (3, "color_disagreement"),
                         (4, "insufficient_parallax")]:
        per_ref, funnel = o.verify_depth_grids(views, [0], [[source]], 4, 4, 20.0)
        assert len(per_ref[0]) == 0 and funnel["accepted"] == 0
        assert funnel[gate] == 24 - funnel["outside_source"] - funnel["missing_reference_depth"]


@pytest.mark.parametrize("seed,stride,rstride", [(1, 2, 2), (2, 2, 4), (3, 4, 8)])
def test_oracle_outcome_invariants(seed, stride, rstride):
    views, refs, sources, focal = depth_grid_scenes.clip_views(seed, stride=stride)
    per_ref, f = Oracle().verify_depth_grids(views, refs, sources, stride, rstride, focal)
    gates = sum(v for k, v in f.items() if k != "reference_samples")
    assert gates == f["reference_samples"]
    assert f["accepted"] > 0 and f["depth_disagreement"] > 0 and f["missing_reference_depth"] > 0
    for r, samples in enumerate(per_ref):
        if len(samples) == 0:
            continue
        order = samples["site_y"].astype(np.int64) * 100000 + samples["site_x"]
        assert (np.diff(order) > 0).all()
        assert (samples["site_x"] % rstride == 0).all() and (samples["site_y"] % rstride == 0).all()
        assert (samples["source_mask"] > 0).all()
        assert (samples["source_mask"] < (1 << len(sources[r]))).all()
        assert (samples["confidence"] > 0.97).all() and (samples["confidence"] <= 1.0).all()


def _tris(rows):
    from v3d import types
    t = np.zeros(len(rows), dtype=types.TRIANGLE_DTYPE)
    for i, (a, b, c) in enumerate(rows):
        t[i] = (a, b, c, 1.0, 0)
    return t


def test_topology_reference_case_through_the_c_entry_point():
    # colmap_surface.rs:732-759
    o = Oracle()
    top = o.surface_topology(_tris([(0, 1, 2), (1, 3, 2), (4, 5, 6), (5, 7, 6)]), 8)
    assert top == {"islands": 2, "small_islands": 2, "small_island_triangles": 4,
                   "largest_island_triangles": 2, "boundary_edges": 8}
    top = o.surface_topology(_tris([(i, i + 1, i + 2) for i in range(32)]), 34)
    assert (top["islands"], top["small_islands"], top["largest_island_triangles"]) == (1, 0, 32)


def _recompose(views, refs, sources, stride, rstride, focal):
    """colmap_surface.rs:380-471 in Python over the oracle's verification
    and mesh calls: per reference the united samples are meshed as one patch
    and the vertices appended in the order the triangles first use them."""
    o = Oracle()
    per_ref, funnel = o.verify_depth_grids(views, refs, sources, stride, rstride, focal)
    cams = [cam for _, _, cam in views]
    h, w = views[0][0].shape[:2]
    pts, sites, tris, regions = [], [], [], []
    meshing = {"candidate_cells": 0, "rejected_discontinuities": 0, "rejected_degenerate": 0,
               "multiply_verified_samples": 0}
    for r, samples in enumerate(per_ref):
        meshing["multiply_verified_samples"] += int(
            sum(bin(int(m)).count("1") > 1 for m in samples["source_mask"]))
        if len(samples) == 0:
            continue
        p = np.zeros(len(samples), dtype=types.POINT_DTYPE)
        for f in ("x", "y", "z", "confidence", "r", "g", "b"):
            p[f] = samples[f]
        g = np.zeros(len(samples), dtype=types.SITE_DTYPE)
        g["x"], g["y"] = samples["site_x"], samples["site_y"]
        frame = int(views[refs[r]][2].frame_index)
        mesh = o.reconstruct_dense_mesh_with_control(
            p, g, {"attempted": True, "reference_frame": frame, "grid_stride": rstride}, cams, w,
            h, focal)
        for k in ("candidate_cells", "rejected_discontinuities", "rejected_degenerate"):
            meshing[k] += int(mesh.stats[k])
        start, index, frames = len(pts), {}, set()
        for t in mesh.triangles:
            corners = []
            for i in (int(t["a"]), int(t["b"]), int(t["c"])):
                if i not in index:
                    index[i] = len(pts)
                    pts.append(p[i])
                    sites.append(g[i])
                    m = int(samples["source_mask"][i])
                    frames |= {int(views[sources[r][j]][2].frame_index) for j in range(4) if m >> j & 1}
                corners.append(index[i])
            tris.append((*corners, float(t["confidence"])))
        if len(pts) > start:
            regions.append({"reference_frame": frame, "first_point": start,
                            "point_count": len(pts) - start, "source_frames": sorted(frames)})
    return pts, sites, tris, regions, funnel, meshing


@pytest.mark.parametrize("seed,stride,rstride", [(1, 2, 2), (2, 2, 4), (4, 3, 6)])
def test_oracle_verified_surface_equals_its_recomposition(seed, stride, rstride):
    views, refs, sources, focal = depth_grid_scenes.clip_views(seed, stride=stride)
    surf = Oracle().mesh_verified_depth_grids(views, refs, sources, stride, rstride, focal)
    pts, sites, tris, regions, funnel, meshing = _recompose(views, refs, sources, stride, rstride,
                                                           focal)
    assert surf.status == 0 and len(tris) > 0
    assert surf.diagnostics["verification"] == funnel
    for k, v in meshing.items():
        assert surf.diagnostics["meshing"][k] == v, k
    assert surf.diagnostics["meshing"]["exported_triangles"] == len(tris)
    assert surf.diagnostics["meshing"]["meshed_reference_views"] == len(regions)
    assert surf.regions == regions
    assert np.array(pts, dtype=surf.points.dtype).tobytes() == surf.points.tobytes()
    assert np.array(sites, dtype=surf.sites.dtype).tobytes() == surf.sites.tobytes()
    t = surf.triangles
    assert [(int(a), int(b), int(c), float(f)) for a, b, c, f in
            zip(t["a"], t["b"], t["c"], t["confidence"])] == tris
    assert surf.diagnostics["topology"] == Oracle().surface_topology(surf.triangles, len(pts))
    top = surf.diagnostics["topology"]
    assert top["islands"] >= len(regions)
    assert surf.diagnostics["dominant_rejection"] is not None


def test_oracle_verified_surface_without_triangles_is_skipped():
    frame, _, first, second, depth, wrong = depth_grid_scenes.reference_plane()
    views = [(frame, depth, first), (frame, wrong, second)]
    surf = Oracle().mesh_verified_depth_grids(views, [0], [[1]], 4, 4, 20.0)
    assert surf.status == 1 and len(surf.points) == 0
    assert surf.diagnostics["verification"]["depth_disagreement"] > 0


def test_verified_surface_bounds_hold_the_oracle_outputs():
    import ctypes as C
    from v3d import dense
    lib = dense.library()
    mp, mt = C.c_uint64(), C.c_uint64()
    lib.v3d_verified_surface_bounds(640, 360, 4, 3, C.byref(mp), C.byref(mt))
    gw, gh = 160, 90
    slots = 2 * (gw + 1) * (gh + 1) + (gw - 2) * gh + gw * (gh - 2)
    assert (mp.value, mt.value) == (3 * gw * gh, 3 * slots)
    lib.v3d_verified_surface_bounds(641, 361, 4, 1, C.byref(mp), C.byref(mt))
    assert mp.value == 161 * 91
    for seed, stride, rstride in [(1, 2, 2), (3, 4, 8)]:
        views, refs, sources, focal = depth_grid_scenes.clip_views(seed, stride=stride)
        surf = Oracle().mesh_verified_depth_grids(views, refs, sources, stride, rstride, focal)
        h, w = views[0][0].shape[:2]
        lib.v3d_verified_surface_bounds(w, h, rstride, len(refs), C.byref(mp), C.byref(mt))
        assert 0 < len(surf.points) <= mp.value and 0 < len(surf.triangles) <= mt.value
