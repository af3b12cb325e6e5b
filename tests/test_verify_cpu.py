"""Depth-grid verification on the CPU: the oracle through its C entry point
against the reference's own test plane, and the invariants of its outcome on
seeded clips."""
import numpy as np
import pytest

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
