"""Fast-policy parity at the benchmark's own parameters, through the C ABI.

The headline configuration (7x7 ZNCC, 128 hypotheses, 8 source views, grid
stride 2; f32 and f16 images) and the heavy one (9x9 ZNCC, 256 hypotheses, 16
source views; bf16 images) run the kernels the benchmark times
(k_sweep_tiled<T, 3|4>, k_recip_prepare / k_recip_sweep<T, 3|4, 1>).  Each is
compared with the f64 oracle on a clip of the same generator and camera
spacing that the oracle finishes in seconds, and on one full-size 640x360
reference over a band of its grid rows.

Tolerances (tests/attribution.py):
* the chosen hypothesis agrees on >= 99.9 % of the sampled sites;
* the cost of the chosen hypothesis is within COST_TOLERANCE (1e-4) of the
  f64 cost;
* every other difference is attributed: a status that differs at the same
  hypothesis has its cost or margin within 2 x COST_TOLERANCE of the gate; a
  point present in one result only, or fused points more than 1e-5 relative
  apart, come from a reciprocal decision within 2 x COST_TOLERANCE of its
  threshold or of a tie between two single-view hypotheses; a completion
  difference has such a gap or a differing neighbour.  No slack by percentage.
"""
import pytest

from tests.attribution import COST_TOLERANCE, attribute
from v3d import abi, profiles, synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from v3d import dense
    c = dense.Context(0)
    yield c
    c.close()


def headline_clip(width=320, height=180, seed=21):
    """The full clip's generator: 120 keyframes on a 40-degree arc are 0.336
    degrees apart; 9 such keyframes, the middle one the reference."""
    return synth.make_clip(width, height, 9, 2.7, 4.0, seed, noise_sigma=0.01, jitter_deg=2.0,
                           landmark_cameras=[4], landmarks_per_camera=400)


def heavy_clip(width=224, height=126, seed=25):
    """The heavy clip's generator (8 planes + 4 boxes, 5 % low texture, noise
    0.02) with 17 keyframes at the same spacing: 16 sources for the middle one."""
    return synth.make_clip(width, height, 17, 5.4, 4.0, seed, noise_sigma=0.02, jitter_deg=2.0,
                           extra_planes=4, boxes=4, low_texture_fraction=0.05,
                           landmark_cameras=[8], landmarks_per_camera=400)


def run(ctx, oracle, clip, storage, prof, rows=None):
    frames = clip.frames(storage)
    exact = profiles.with_precision(prof, abi.PRECISION_EXACT64)
    o, rec = oracle.explain_reference_patch(frames, clip.cameras, clip.sparse, clip.focal, None,
                                            exact, rows=rows)
    gs = ctx.debug_sweep(frames, clip.cameras, clip.sparse, clip.focal, profile=prof)
    g = ctx.estimate_depth_points_with_control(frames, clip.cameras, clip.sparse, clip.focal,
                                               profile=prof)
    return attribute(g, gs, o, rec, prof, 2 * COST_TOLERANCE, rows=rows), g


def check(rep, min_points):
    assert rep["unexplained"] == [], rep["unexplained"][:10]
    assert rep["moved_fraction"] <= 1e-3, rep
    assert rep["max_cost_error"] <= COST_TOLERANCE, rep["max_cost_error"]
    assert rep["points_compared"] >= min_points, rep
    # fused positions agree bit for bit unless a reciprocal hypothesis moved (the
    # confidence follows the f32 cost and margin, so whole records may differ)
    assert rep["positions_equal_bits"] >= rep["points_compared"] - rep["recip_moved"] - \
        rep["completion_band"] - rep["completion_cascade"]


@pytest.mark.parametrize("storage", ["f32", "f16"])
def test_headline_parameters(ctx, oracle, storage):
    rep, g = run(ctx, oracle, headline_clip(), storage, profiles.zncc(3, 128, 8, 2))
    assert g.stats["source_views"] == 8 and g.stats["depth_hypotheses"] == 128
    check(rep, 1500)


def test_heavy_parameters_bf16(ctx, oracle):
    rep, g = run(ctx, oracle, heavy_clip(), "bf16", profiles.zncc(4, 256, 16, 2))
    assert g.stats["source_views"] == 16 and g.stats["depth_hypotheses"] == 256
    check(rep, 300)


@pytest.mark.parametrize("storage", ["f32", "f16"])
def test_full_size_reference_rows(ctx, oracle, storage):
    """One 640x360 reference of the headline generator, grid rows 60..84 of 175."""
    clip = headline_clip(640, 360, seed=22)
    rep, g = run(ctx, oracle, clip, storage, profiles.zncc(3, 128, 8, 2), rows=(60, 84))
    assert rep["sampled"] > 5000
    check(rep, 500)
