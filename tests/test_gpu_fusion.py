"""Cross-reference surface fusion on the device against the CPU oracle, bit for
bit: statistics, pairs, moved indices and every byte of the moved points, on
the reference's own fusion scenes, on seeded defect-laden grid meshes (random
shifts, exact half-spacing ties, a perpendicular wall, many groups, a large
case) and on the consolidated output of real reference patches."""
import numpy as np
import pytest

from v3d import dense, profiles, surface, synth

from tests import fusion_scenes
from tests.oracle_ffi import Oracle


def _compare(points, triangles, membership):
    ctx = dense.Context(0)
    g, o = points.copy(), points.copy()
    og = ctx.fuse_mutually_supported_vertices(g, triangles, membership)
    oo = Oracle().fuse_mutually_supported_vertices(o, triangles, membership)
    assert og.stats == oo.stats
    assert np.array_equal(og.pairs, oo.pairs)
    assert np.array_equal(og.moved_indices, oo.moved_indices)
    assert g.tobytes() == o.tobytes()
    return og, g


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(fusion_scenes.REFERENCE_SCENES))
def test_reference_scenes(name):
    pts, tris, mem = fusion_scenes.reference_scene(name)
    out, moved = _compare(pts, tris, mem)
    if name == "aligns_mutually_nearest_vertices":
        assert out.stats["fused_pairs"] == 3
        assert abs(moved["z"][0] - 0.03) < 1e-6
    elif name == "rejects_when_normals_disagree":
        assert out.stats["fused_pairs"] == 0 and out.stats["rejected_normal_pairs"] >= 2
    elif name == "rejects_a_weakening_seam_move":
        assert out.stats["fused_pairs"] == 0 and out.stats["rejected_topology_pairs"] > 0
    else:
        assert out.stats["candidate_pairs"] == 0


@pytest.mark.gpu
@pytest.mark.parametrize("seed,kw", [(1, {}), (2, {"half_shift": True}), (3, {"wall": True}),
                                     (4, {"groups": 5, "nx": 40, "ny": 30}),
                                     (6, {"defects": False, "separation": 0.0}),
                                     (7, {"groups": 2, "nx": 7, "ny": 5})])
def test_seeded_grids(seed, kw):
    pts, tris, mem = fusion_scenes.layered_grids(seed, **kw)
    out, _ = _compare(pts, tris, mem)
    assert out.stats["fused_pairs"] > 0


@pytest.mark.gpu
def test_large_scene_and_repeated_calls():
    pts, tris, mem = fusion_scenes.layered_grids(8, groups=4, nx=320, ny=240)
    first, g1 = _compare(pts, tris, mem)
    ctx = dense.Context(0)
    g2 = pts.copy()
    again = ctx.fuse_mutually_supported_vertices(g2, tris, mem)
    assert again.stats == first.stats and g2.tobytes() == g1.tobytes()
    assert first.stats["fused_pairs"] > 1000


@pytest.mark.gpu
def test_consolidated_reference_patches():
    clip = synth.make_clip(320, 180, 6, 15.0, 1.5, seed=21, noise_sigma=0.01)
    frames = clip.frames("f32")
    ctx = dense.Context(0)
    res = ctx.reconstruct_reference_patches_meshed(frames, clip.cameras, clip.sparse, clip.focal,
                                                   [0, 2, 4, 5], profile=profiles.zncc(2, 64, 4, 2))
    patches = [r for r in res if r is not None]
    assert len(patches) >= 2
    pts, tris, mem, groups = surface.consolidation_inputs(patches)
    assert groups == len(patches) and len(tris) > 1000
    out, _ = _compare(pts, tris, mem)
    assert out.stats["candidate_pairs"] > 0


@pytest.mark.gpu
def test_cancellation_returns_the_default_outcome():
    pts, tris, mem = fusion_scenes.layered_grids(9)
    before = pts.copy()
    out = dense.Context(0).fuse_mutually_supported_vertices(pts, tris, mem, control=lambda: True)
    assert all(v == 0 for v in out.stats.values())
    assert len(out.pairs) == 0 and len(out.moved_indices) == 0
    assert pts.tobytes() == before.tobytes()
