"""The working-set budget (dense.rs:354-605) on the CPU.

* The reference's own budget tests (dense.rs:1269-1519) restated against the
  oracle, which runs the whole plan and pass in f64.
* The library's host-side estimate (v3d_estimate_working_set, no device
  needed) equals the oracle's field by field over frame sizes, formats and
  counts, sparse-stage options, view counts and both grids, saturation
  included.
"""
import numpy as np
import pytest

from tests import fixtures
from v3d import abi, dense, profiles
from v3d.types import FrameInput

MAX_REFERENCE_VIEWS = 3


def _scene(offsets):
    frames = [fixtures.plane_frame(center_x=c) for c in offsets]
    cams = [fixtures.camera(i, c) for i, c in enumerate(offsets)]
    return frames, cams, fixtures.plane_sparse_points()


def _points_bits(a):
    return [(p["x"].tobytes(), p["y"].tobytes(), p["z"].tobytes(), p["confidence"].tobytes())
            for p in a.points]


def test_budget_below_estimate_suppresses_only_dense_geometry(oracle):
    """dense.rs:1269-1294"""
    frames, cams, sparse = _scene((0.0, 0.24))
    r, plan = oracle.estimate_depth_points_with_budget_and_control(
        frames, cams, sparse, fixtures.FOCAL, 1, 320, 3, profiles.reference())
    assert not r.stats["attempted"]
    assert len(r.points) == 0 and len(r.grid_sites) == 0
    assert plan["working_set_estimate"]["total_bytes"] > 1
    assert plan["working_set_budget_bytes"] == 1
    assert "exceeds the configured" in r.stats["skip_reason"]
    assert r.stats["skip_reason"] == (
        "estimated dense working set of %d bytes exceeds the configured 1 byte budget even for "
        "one reference view" % plan["working_set_estimate"]["total_bytes"])


def test_a_tight_budget_keeps_the_leading_reference_patches_of_the_full_run(oracle):
    """dense.rs:1296-1355"""
    frames, cams, sparse = _scene((0.0, 0.24, -0.22))
    prof = profiles.reference()
    fine = oracle.has_distributed_landmarks(frames, cams, sparse, fixtures.FOCAL)
    full, _ = oracle.estimate_depth_points_limited(frames, cams, sparse, fixtures.FOCAL,
                                                   MAX_REFERENCE_VIEWS, fine, prof)
    assert len(full.stats["reference_patches"]) >= 2
    one = oracle.estimate_working_set(frames, 320, 3, 1, False)["total_bytes"]
    three = oracle.estimate_working_set(frames, 320, 3, MAX_REFERENCE_VIEWS, False)["total_bytes"]
    assert one < three
    lim, plan = oracle.estimate_depth_points_with_budget_and_control(
        frames, cams, sparse, fixtures.FOCAL, one, 320, 3, prof)
    assert lim.stats["attempted"]
    assert lim.stats["reference_view_limit"] == 1
    assert plan["working_set_estimate"]["total_bytes"] == one
    assert plan["full_working_set_bytes"] == three
    assert len(lim.stats["reference_patches"]) == 1
    kept = lim.stats["reference_patches"][0]
    lead = full.stats["reference_patches"][0]
    assert kept["reference_frame"] == lead["reference_frame"]
    expected = np.concatenate([
        full.points[lead["primary_start"]:lead["primary_start"] + lead["primary_points"]],
        full.points[lead["completion_start"]:lead["completion_start"] + lead["completed_points"]]])
    assert expected.tobytes() == lim.points.tobytes()
    two = oracle.estimate_working_set(frames, 320, 3, 2, False)["total_bytes"]
    wider, _ = oracle.estimate_depth_points_with_budget_and_control(
        frames, cams, sparse, fixtures.FOCAL, two, 320, 3, prof)
    assert wider.stats["reference_view_limit"] == 2
    assert len(wider.stats["reference_patches"]) == min(len(full.stats["reference_patches"]), 2)
    unlimited, _ = oracle.estimate_depth_points_with_budget_and_control(
        frames, cams, sparse, fixtures.FOCAL, three, 320, 3, prof)
    assert unlimited.stats["reference_view_limit"] is None


def test_budget_above_estimate_preserves_dense_output(oracle):
    """dense.rs:1357-1427"""
    frames, cams, sparse = _scene((0.0, 0.24, -0.22))
    prof = profiles.reference()
    fine = oracle.has_distributed_landmarks(frames, cams, sparse, fixtures.FOCAL)
    base, _ = oracle.estimate_depth_points_limited(frames, cams, sparse, fixtures.FOCAL,
                                                   MAX_REFERENCE_VIEWS, fine, prof)
    got, plan = oracle.estimate_depth_points_with_budget_and_control(
        frames, cams, sparse, fixtures.FOCAL, (1 << 64) - 1, 320, 3, prof)
    assert base.points.tobytes() == got.points.tobytes()
    assert base.grid_sites.tobytes() == got.grid_sites.tobytes()
    assert base.point_attributes.tobytes() == got.point_attributes.tobytes()
    w = plan["working_set_estimate"]
    parts = [w[n] for n in abi.WORKING_SET_FIELDS[:-1]]
    assert w["total_bytes"] == min(sum(parts), (1 << 64) - 1)
    assert w["retry_frame_bytes"] == w["frame_bytes"]
    assert w["remapped_frame_bytes"] == w["frame_bytes"]
    for n in ("retained_candidate_bytes", "mesh_builder_bytes", "surface_fusion_bytes",
              "sparse_pipeline_bytes"):
        assert w[n] > 0, n


def test_the_retained_candidate_is_charged_at_the_largest_prior_plan(oracle):
    """dense.rs:1429-1450"""
    frames, _, _ = _scene((0.0, 0.24, -0.22))
    ordinary = oracle.estimate_working_set(frames, 320, 3, MAX_REFERENCE_VIEWS, False)
    retry = oracle.estimate_working_set(frames, 1200, 3, 1, False)
    assert retry["sparse_pipeline_bytes"] > ordinary["sparse_pipeline_bytes"]
    assert retry["dense_sample_bytes"] < ordinary["dense_sample_bytes"]
    assert retry["retained_candidate_bytes"] == ordinary["retained_candidate_bytes"]
    assert ordinary["retained_candidate_bytes"] >= ordinary["topology_bytes"]


def test_a_limit_that_omits_no_reference_is_not_reported(oracle):
    """dense.rs:1452-1473"""
    frames, cams, sparse = _scene((0.0, 0.24))
    two = oracle.estimate_working_set(frames, 320, 3, 2, False)["total_bytes"]
    lim, plan = oracle.estimate_depth_points_with_budget_and_control(
        frames, cams, sparse, fixtures.FOCAL, two, 320, 3, profiles.reference())
    assert plan["full_working_set_bytes"] > two
    assert lim.stats["reference_view_limit"] is None


def test_feature_options_increase_the_retained_sparse_estimate(oracle):
    """dense.rs:1475-1487"""
    frames, _, _ = _scene((0.0, 0.24, -0.22))
    ordinary = oracle.estimate_working_set(frames, 320, 3, MAX_REFERENCE_VIEWS, False)
    heavy = oracle.estimate_working_set(frames, 640, 7, MAX_REFERENCE_VIEWS, False)
    assert heavy["sparse_pipeline_bytes"] > ordinary["sparse_pipeline_bytes"]
    assert heavy["total_bytes"] > ordinary["total_bytes"]


def _frames(sizes, fmt):
    out = []
    for w, h in sizes:
        if fmt == "rgba8":
            out.append(FrameInput(np.zeros((h, w, 4), np.uint8)))
        elif fmt == "f32":
            out.append(FrameInput(np.zeros((h, w), np.float32)))
        elif fmt == "f16":
            out.append(FrameInput(np.zeros((h, w), np.float16)))
        else:
            out.append(FrameInput(np.zeros((h, w), np.uint16), bf16=True))
    return out


@pytest.mark.parametrize("sizes", [[], [(68, 48)], [(68, 48)] * 3, [(640, 360)] * 7,
                                   [(1920, 1080), (640, 360), (16, 16)], [(5, 5), (7, 300)]])
@pytest.mark.parametrize("fmt", ["rgba8", "f32", "f16", "bf16"])
def test_library_estimate_equals_the_oracle(oracle, sizes, fmt):
    frames = _frames(sizes, fmt)
    for features, radius in ((0, 0), (320, 3), (1200, 7), (1 << 62, 3), (320, (1 << 31) - 1)):
        for views in (1, 2, 3):
            for fine in (False, True):
                got = dense.estimate_working_set(frames, features, radius, views, fine)
                want = oracle.estimate_working_set(frames, features, radius, views, fine)
                assert got == want, (sizes, fmt, features, radius, views, fine)
