"""Surface fusion on the CPU: the oracle against the reference's own fusion
tests, the host-side support membership against its reference test, and
invariants of the oracle's outcome on the seeded defect-laden scenes."""
import numpy as np
import pytest

from v3d import surface

from tests import fusion_scenes
from tests.oracle_ffi import Oracle


def test_support_membership_follows_camera_support_not_patch_identity():
    # surface_fusion.rs:891-915
    regions = [(0, [2, 1], 0, 2), (0, [1, 2], 2, 1), (3, [4], 3, 1), (None, [], 4, 1)]
    membership, groups = surface.support_membership(regions, 5)
    assert groups == 2
    assert membership.tolist() == [0, 0, 0, 1, -1]


def _oracle_fuse(points, triangles, membership, control=None):
    return Oracle().fuse_mutually_supported_vertices(points, triangles, membership, control)


def test_reference_scenes_on_the_oracle():
    # surface_fusion.rs:917-1027, through the same C entry point shape the device uses
    pts, tris, mem = fusion_scenes.reference_scene("aligns_mutually_nearest_vertices")
    out = _oracle_fuse(pts, tris, mem)
    assert out.stats["fused_pairs"] == 3
    assert out.stats["rejected_normal_pairs"] == 0
    assert out.stats["rejected_topology_pairs"] == 0
    for left, right in [(0, 3), (1, 4), (2, 5)]:
        assert abs(pts["z"][left] - 0.03) < 1e-6
        assert abs(pts["z"][left] - pts["z"][right]) < 1e-6
    pts, tris, mem = fusion_scenes.reference_scene("rejects_when_normals_disagree")
    out = _oracle_fuse(pts, tris, mem)
    assert out.stats["fused_pairs"] == 0 and out.stats["rejected_normal_pairs"] >= 2
    assert pts["z"][0] == 0.0 and pts["z"][3] == np.float32(0.05)
    pts, tris, mem = fusion_scenes.reference_scene("rejects_a_weakening_seam_move")
    out = _oracle_fuse(pts, tris, mem)
    assert out.stats["fused_pairs"] == 0 and out.stats["rejected_topology_pairs"] > 0
    pts, tris, mem = fusion_scenes.reference_scene("never_fuses_within_a_group")
    out = _oracle_fuse(pts, tris, mem)
    assert out.stats["fused_pairs"] == 0 and out.stats["candidate_pairs"] == 0


@pytest.mark.parametrize("seed,kw", [(1, {}), (2, {"half_shift": True}), (3, {"wall": True}),
                                     (4, {"groups": 5, "nx": 40, "ny": 30})])
def test_oracle_outcome_invariants(seed, kw):
    pts, tris, mem = fusion_scenes.layered_grids(seed, **kw)
    before = pts.copy()
    out = _oracle_fuse(pts, tris, mem)
    s = out.stats
    assert s["fused_pairs"] == len(out.pairs) > 0
    assert s["candidate_pairs"] >= s["rejected_normal_pairs"]
    flat = out.pairs.ravel()
    assert len(np.unique(flat)) == len(flat)              # a vertex fuses at most once
    assert (out.pairs[:, 0] < out.pairs[:, 1]).all()
    assert (mem[out.pairs[:, 0]] != mem[out.pairs[:, 1]]).all()
    assert set(out.moved_indices.tolist()) <= set(flat.tolist())
    assert (np.diff(out.moved_indices.astype(np.int64)) > 0).all()
    untouched = np.setdiff1d(np.arange(len(pts)), flat)
    assert pts[untouched].tobytes() == before[untouched].tobytes()
    for a, b in out.pairs:
        assert (pts["x"][a], pts["y"][a], pts["z"][a]) == (pts["x"][b], pts["y"][b], pts["z"][b])
    if kw.get("wall"):
        assert s["rejected_normal_pairs"] > 0


def test_oracle_cancellation_leaves_everything_unchanged():
    pts, tris, mem = fusion_scenes.layered_grids(5)
    before = pts.copy()
    out = _oracle_fuse(pts, tris, mem, control=lambda: True)
    assert all(v == 0 for v in out.stats.values())
    assert len(out.pairs) == 0 and len(out.moved_indices) == 0
    assert pts.tobytes() == before.tobytes()
