"""GPU parity of the dense pass against the CPU oracle, through the C ABI.

Exact policy (f64 taps with the reference's formulas): every output —
points, sites, attributes and every statistic — is bit-identical to the
oracle.  Fast policy (f32 taps through f64-composed homographies): the chosen
hypothesis agrees on >= 99.9 % of sites, the accept/reject mask differs only
where the gate quantity lies within 1e-5 of its threshold (or the hypothesis
moved), and fused points of sites both keep agree to 1e-5 relative.
"""
import numpy as np
import pytest

from tests import fixtures
from v3d import abi, profiles, synth

pytestmark = pytest.mark.gpu

FAST_TOL = 1e-5


@pytest.fixture(scope="module")
def ctx():
    from v3d import dense
    c = dense.Context(0)
    yield c
    c.close()


def assert_same_analysis(g, o):
    assert g.status == o.status
    gs, os_ = dict(g.stats), dict(o.stats)
    assert gs == os_
    assert g.points.tobytes() == o.points.tobytes()
    assert g.grid_sites.tobytes() == o.grid_sites.tobytes()
    assert g.point_attributes.tobytes() == o.point_attributes.tobytes()


def check_reference_assertions(r):
    """dense_legacy.rs:1277-1320 on a result."""
    s = r.stats
    assert s["attempted"] and s["skip_reason"] is None
    assert s["reciprocal_checked_points"] == (s["reciprocal_consistent_points"]
                                              + s["reciprocal_rejected_points"])
    assert (s["reciprocal_consistent_points"] + s["surface_completed_points"]
            == s["accepted_points"] + s["fusion_rejected_points"])
    assert s["surface_completion_proposals"] == (
        s["surface_completed_points"] + s["surface_completion_rejected_texture"]
        + s["surface_completion_rejected_cross_view"]
        + s["surface_completion_rejected_reciprocal"]
        + s["surface_completion_rejected_fusion"] + s["surface_completion_rejected_footprint"])


# ---- the reference's own test scenes, exact policy -------------------------

def test_textured_plane_exact(ctx, oracle):
    frames, cams, sparse = fixtures.three_view_scene(fixtures.SCENES["legacy_plane"])
    prof = profiles.reference()
    g = ctx.estimate_depth_points_with_control(frames, cams, sparse, fixtures.FOCAL, profile=prof)
    o = oracle.estimate_depth_points_with_control(frames, cams, sparse, fixtures.FOCAL,
                                                  profile=prof)
    assert_same_analysis(g, o)
    check_reference_assertions(g)
    assert g.stats["reference_frame"] == 0
    assert g.stats["source_frames"] == [1, 2]
    assert len(g.points) >= 12
    assert abs(float(np.median(np.sort(g.points["z"]))) - fixtures.DEPTH) < 0.55


def test_multi_reference_exact(ctx, oracle):
    frames, cams, sparse = fixtures.three_view_scene(fixtures.SCENES["multi_reference"])
    prof = profiles.reference()
    fine = oracle.has_distributed_landmarks(frames, cams, sparse, fixtures.FOCAL)
    for views in (1, 2, 3):
        g, go = ctx.estimate_depth_points_limited(frames, cams, sparse, fixtures.FOCAL, views,
                                                  fine, profile=prof)
        o, oo = oracle.estimate_depth_points_limited(frames, cams, sparse, fixtures.FOCAL, views,
                                                     fine, prof)
        assert go == oo
        assert_same_analysis(g, o)
    assert len(g.stats["reference_patches"]) >= 2


def test_surface_completion_scene_exact(ctx, oracle):
    frames, cams, sparse = fixtures.three_view_scene(fixtures.SCENES["completion"])
    prof = profiles.reference()
    g, _ = ctx.estimate_depth_points_limited(frames, cams, sparse, fixtures.FOCAL, 3, False,
                                             profile=prof)
    o, _ = oracle.estimate_depth_points_limited(frames, cams, sparse, fixtures.FOCAL, 3, False,
                                                prof)
    assert_same_analysis(g, o)
    assert g.stats["surface_completed_points"] > 0
    n = len(g.points) - g.stats["surface_completed_points"]
    done = g.points[n:]
    assert np.all(np.abs(done["z"].astype(np.float64) - 4.0) < 0.55)
    assert np.all((done["confidence"] >= 0.05) & (done["confidence"] <= 0.9))


def test_textureless_and_single_camera(ctx, oracle):
    flat = fixtures.flat_frame()
    cams = [fixtures.camera(0, 0.0), fixtures.camera(1, 0.2)]
    sparse = fixtures.plane_sparse_points()
    g = ctx.estimate_depth_points_with_control([flat, flat], cams, sparse, fixtures.FOCAL)
    o = oracle.estimate_depth_points_with_control([flat, flat], cams, sparse, fixtures.FOCAL,
                                                  profile=profiles.reference())
    assert_same_analysis(g, o)
    assert g.stats["attempted"] and len(g.points) == 0
    assert g.stats["surface_completion_proposals"] == 0
    g = ctx.estimate_depth_points_with_control([fixtures.plane_frame()], cams[:1], sparse,
                                               fixtures.FOCAL)
    assert g.status == abi.SKIPPED and not g.stats["attempted"]
    assert "two accepted registered cameras" in g.stats["skip_reason"]


def test_cancellation_skips_like_the_reference(ctx, oracle):
    frames, cams, sparse = fixtures.three_view_scene(fixtures.SCENES["legacy_plane"])
    for cancel_at in (1, 3):
        results = []
        for impl in (ctx, oracle):
            polls = []

            def control():
                polls.append(1)
                return len(polls) == cancel_at

            r = impl.estimate_depth_points_with_control(frames, cams, sparse, fixtures.FOCAL,
                                                        control=control,
                                                        profile=profiles.reference())
            results.append((r.stats["skip_reason"], len(polls)))
        assert results[0] == results[1]
        assert results[0][0] == "dense reconstruction canceled"


# ---- synthetic scenes --------------------------------------------------------

@pytest.fixture(scope="module")
def small_clip():
    return synth.make_clip(160, 96, 5, 15.0, 1.2, seed=11, noise_sigma=0.01,
                           landmark_cameras=[2], landmarks_per_camera=300)


@pytest.mark.parametrize("storage,cost", [("rgba8", "zsad"), ("f32", "zncc"), ("f16", "zncc"),
                                          ("bf16", "zncc")])
def test_synthetic_exact_bitwise(ctx, oracle, small_clip, storage, cost):
    clip = small_clip
    frames = clip.frames(storage)
    if cost == "zsad":
        prof = profiles.reference()
    else:
        prof = profiles.zncc(2, 32, 4, 2, precision=abi.PRECISION_EXACT64)
    g = ctx.reconstruct_reference_patches(frames, clip.cameras, clip.sparse, clip.focal, [2, 0],
                                          profile=prof)
    o = oracle.reconstruct_reference_patches(frames, clip.cameras, clip.sparse, clip.focal,
                                             [2, 0], prof)
    for a, b in zip(g, o):
        assert (a is None) == (b is None)
        if a is not None:
            assert_same_analysis(a, b)
    assert len(g[0].points) > 100


def _fast_vs_oracle_sweep(ctx, oracle, frames, cams, sparse, focal, prof):
    exact = profiles.with_precision(prof, abi.PRECISION_EXACT64)
    gs = ctx.debug_sweep(frames, cams, sparse, focal, profile=prof)
    os_ = oracle.debug_sweep(frames, cams, sparse, focal, profile=exact)
    assert len(gs) == len(os_)
    assert np.array_equal(gs["x"], os_["x"]) and np.array_equal(gs["y"], os_["y"])
    # the contrast gate reads exact pixel values in both policies
    assert np.array_equal(gs["status"] == 1, os_["status"] == 1)
    both = (gs["status"] >= 3) & (os_["status"] >= 3)
    agree = gs["plane"][both] == os_["plane"][both]
    frac = agree.mean()
    assert frac >= 0.999, frac
    # accept/reject differences only near a threshold, or where the hypothesis moved
    diff = (gs["status"] != os_["status"]) & (gs["status"] >= 2) & (os_["status"] >= 2)
    same_plane = gs["plane"] == os_["plane"]
    near = (np.abs(os_["error"] - prof.max_photometric_error) <= FAST_TOL) | \
           (np.abs(os_["margin"] - prof.min_ambiguity_margin) <= FAST_TOL)
    bad = diff & same_plane & ~near
    assert bad.sum() == 0, np.nonzero(bad)
    moved = diff & ~same_plane
    assert moved.sum() <= max(1, 0.001 * both.sum())
    # cost of the chosen hypothesis against the f64 oracle
    err = np.abs(gs["error"][both & (gs["plane"] == os_["plane"])] -
                 os_["error"][both & (gs["plane"] == os_["plane"])])
    return frac, float(err.max()) if err.size else 0.0


@pytest.mark.parametrize("storage", ["f32", "f16", "bf16"])
def test_fast_zncc_sweep_agreement(ctx, oracle, storage):
    clip = synth.plain_small_clip(seed=3, width=192, height=112)
    frames = clip.frames(storage)
    prof = profiles.zncc(2, 64, 4, 2)
    # the legacy pass picks the camera with the most visible landmarks as reference
    frac, cost_err = _fast_vs_oracle_sweep(ctx, oracle, frames, clip.cameras, clip.sparse,
                                           clip.focal, prof)
    assert cost_err < 5e-5, cost_err


def test_fast_zsad_sweep_agreement(ctx, oracle):
    clip = synth.plain_small_clip(seed=4, width=240, height=136)
    frames = clip.frames("rgba8")
    prof = profiles.reference(precision=abi.PRECISION_FAST32)
    frac, cost_err = _fast_vs_oracle_sweep(ctx, oracle, frames, clip.cameras, clip.sparse,
                                           clip.focal, prof)
    assert cost_err < 1e-3, cost_err  # 0-255 units


def _zsad(radius):
    prof = profiles.reference(precision=abi.PRECISION_FAST32)
    prof.patch_radius = radius
    prof.depth_hypotheses = 48
    prof.grid_stride = 2
    return prof


# radius 4 (9x9, 81 taps) needs three rounds of 32 lanes in the lane-parallel
# direct cost and window reductions
@pytest.mark.parametrize("prof_of,storage", [
    (lambda: profiles.zncc(2, 64, 4, 2), "f32"),
    (lambda: profiles.zncc(4, 64, 4, 2), "f32"),
    (lambda: _zsad(4), "rgba8"),
], ids=["zncc-r2", "zncc-r4", "zsad-r4"])
def test_fast_points(ctx, oracle, prof_of, storage):
    clip = synth.plain_small_clip(seed=5, width=192, height=112)
    frames = clip.frames(storage)
    prof = prof_of()
    exact = profiles.with_precision(prof, abi.PRECISION_EXACT64)
    g = ctx.reconstruct_reference_patches(frames, clip.cameras, clip.sparse, clip.focal, [2],
                                          profile=prof)[0]
    o = oracle.reconstruct_reference_patches(frames, clip.cameras, clip.sparse, clip.focal, [2],
                                             exact)[0]
    check_reference_assertions(g)
    gk = {(int(s["x"]), int(s["y"])): i for i, s in enumerate(g.grid_sites)}
    ok = {(int(s["x"]), int(s["y"])): i for i, s in enumerate(o.grid_sites)}
    common = sorted(set(gk) & set(ok))
    union = set(gk) | set(ok)
    assert len(common) >= 0.99 * len(union), (len(common), len(union))
    gp = np.stack([g.points[[gk[k] for k in common]][c] for c in "xyz"], -1).astype(np.float64)
    op = np.stack([o.points[[ok[k] for k in common]][c] for c in "xyz"], -1).astype(np.float64)
    rel = np.linalg.norm(gp - op, axis=1) / np.linalg.norm(op, axis=1)
    assert (rel <= FAST_TOL).mean() >= 0.995, (rel <= FAST_TOL).mean()


# ---- the reference profile at the configurations' frame sizes ---------------

@pytest.mark.parametrize("size", ["360x202", "640x360"])
def test_reference_profile_at_config_sizes(ctx, oracle, size):
    """The reference's own profile (3x3 ZSAD on u8 luma, 24 hypotheses, at most
    4 sources, grid_stride(): 4 at 360x202, 7 at 640x360; dense_legacy.rs:6-21,
    dense.rs:215-218) on RGBA frames of the small configuration's generator at
    its size and at the full clip's size: bit-identical to the oracle,
    statistics included."""
    w, h = map(int, size.split("x"))
    clip, refs = synth.plain_small_clip(seed=1, width=w, height=h), [0, 2, 4]
    frames = clip.frames("rgba8")
    prof = profiles.reference()
    g = ctx.reconstruct_reference_patches(frames, clip.cameras, clip.sparse, clip.focal, refs,
                                          profile=prof)
    o = oracle.reconstruct_reference_patches(frames, clip.cameras, clip.sparse, clip.focal, refs,
                                             prof, threads=3)
    for a, b in zip(g, o):
        assert (a is None) == (b is None)
        if a is not None:
            assert_same_analysis(a, b)
            check_reference_assertions(a)
    assert g[0] is not None and len(g[0].points) > 200
    assert g[0].stats["grid_stride"] == (4 if size == "360x202" else 7)
