"""GPU reference-grid triangle gates against the oracle (bit-identical)."""
import numpy as np
import pytest

from tests import fixtures
from v3d import profiles, synth
from v3d.types import POINT_DTYPE, SITE_DTYPE

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from v3d import dense
    c = dense.Context(0)
    yield c
    c.close()


def same_mesh(g, o):
    assert g.stats == o.stats
    assert g.triangles.tobytes() == o.triangles.tobytes()
    assert g.reference_frames == o.reference_frames
    assert g.reference_patches == o.reference_patches


def mesh_point(x, y, depth, conf=0.8, w=68, h=48, f=60.0):
    return ((x - w * 0.5) / f * depth, (y - h * 0.5) / f * depth, depth, conf, 120, 140, 160, 0)


LEGACY_STATS = {"attempted": True, "reference_frame": 0, "grid_stride": 4, "grid_border": 3}

# mesh_legacy.rs:609-908: (points as (x, y, depth, conf), sites)
CASES = {
    "quad": ([(3, 3, 4, .8), (7, 3, 4, .7), (3, 7, 4, .9), (7, 7, 4, .6)],
             [(3, 3), (7, 3), (3, 7), (7, 7)]),
    "too_few_vertices": ([(3, 3, 4, .8), (7, 3, 4, .7), (6, 7, 4, .9)],
                         [(3, 3), (7, 3), (3, 7)]),
    "bridge": ([(3, 3, 4, .8), (11, 3, 4, .8), (3, 7, 4, .8), (11, 7, 4, .8), (7, 7, 4, .8)],
               [(3, 3), (11, 3), (3, 7), (11, 7), (7, 7)]),
    "bridge_discontinuity": ([(3, 3, 4, .8), (11, 3, 5, .8), (3, 7, 4, .8), (11, 7, 5, .8),
                              (7, 7, 4, .8)],
                             [(3, 3), (11, 3), (3, 7), (11, 7), (7, 7)]),
    "discontinuity": ([(3, 3, 4, .8), (7, 3, 4, .8), (3, 7, 4, .8), (7, 7, 7, .8)],
                      [(3, 3), (7, 3), (3, 7), (7, 7)]),
    "fusion_shift": ([(4.8, 3, 4, .8), (7, 3, 4, .8), (3, 7, 4, .8)], [(3, 3), (7, 3), (3, 7)]),
    "footprint": ([(5.4, 3, 4, .8), (7, 3, 4, .8), (3, 7, 4, .8), (7, 7, 4, .8)],
                  [(3, 3), (7, 3), (3, 7), (7, 7)]),
    "winding": ([(4.9, 1.1, 4, .8), (5.1, 4.9, 4, .8), (8.9, 5.1, 4, .8)],
                [(3, 3), (7, 3), (7, 7)]),
    "too_few_points": ([(3, 3, 4, .8), (7, 3, 4, .8)], [(3, 3), (7, 3), (3, 7), (7, 7)]),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_reference_mesh_cases(ctx, oracle, name):
    pts, sites = CASES[name]
    P = np.array([mesh_point(*p) for p in pts], dtype=POINT_DTYPE)
    S = np.array(sites, dtype=SITE_DTYPE)
    cams = [fixtures.camera(0, 0.0)]
    g = ctx.reconstruct_dense_mesh_with_control(P, S, LEGACY_STATS, cams, 68, 48, 60.0)
    o = oracle.reconstruct_dense_mesh_with_control(P, S, LEGACY_STATS, cams, 68, 48, 60.0)
    same_mesh(g, o)


def test_mesh_of_dense_patches(ctx, oracle):
    clip = synth.plain_small_clip(seed=7, width=240, height=136)
    frames = clip.frames("rgba8")
    prof = profiles.reference()
    d, _ = oracle.estimate_depth_points_limited(frames, clip.cameras, clip.sparse, clip.focal, 3,
                                                False, prof)
    assert len(d.points) > 50
    g = ctx.reconstruct_dense_mesh_with_control(d.points, d.grid_sites, d.stats, clip.cameras,
                                                clip.width, clip.height, clip.focal)
    o = oracle.reconstruct_dense_mesh_with_control(d.points, d.grid_sites, d.stats, clip.cameras,
                                                   clip.width, clip.height, clip.focal)
    same_mesh(g, o)
    assert g.stats["accepted_triangles"] > 0


@pytest.mark.parametrize("storage,exact", [("rgba8", True), ("f32", True), ("f32", False)])
def test_meshed_reference_patches_match_per_patch_mesh(ctx, oracle, storage, exact):
    """Device mesh of every patch in the batch == the legacy mesh of that patch."""
    from v3d import abi
    clip = synth.make_clip(192, 112, 7, 20.0, 1.5, seed=21, noise_sigma=0.01,
                           landmark_cameras=[1, 3, 5], landmarks_per_camera=300)
    frames = clip.frames(storage)
    if storage == "rgba8":
        prof = profiles.reference()
    else:
        prof = profiles.zncc(2, 32, 4, 2, precision=abi.PRECISION_EXACT64 if exact
                             else abi.PRECISION_FAST32)
    refs = [0, 3, 6]
    got = ctx.reconstruct_reference_patches_meshed(frames, clip.cameras, clip.sparse, clip.focal,
                                                   refs, profile=prof)
    plain = ctx.reconstruct_reference_patches(frames, clip.cameras, clip.sparse, clip.focal, refs,
                                              profile=prof)
    total = 0
    for (d, m), p in zip(got, plain):
        # the dense half is the plain call's result
        assert d.stats == p.stats and d.points.tobytes() == p.points.tobytes()
        o = oracle.reconstruct_dense_mesh_with_control(d.points, d.grid_sites, d.stats,
                                                       clip.cameras, clip.width, clip.height,
                                                       clip.focal)
        same_mesh(m, o)
        total += len(m.triangles)
    assert total > 0
