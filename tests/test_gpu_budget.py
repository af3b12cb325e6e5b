"""The working-set budget plan on the GPU (dense.rs:355-420), through the C ABI.

v3d_estimate_depth_points_with_budget_and_control picks the same plan (grid,
reference-view count, estimate, full bytes, limit) as the oracle and returns a
bit-identical dense result under every budget of the reference's tests: one
byte (the budget skip and its message), exactly the one- and two-view
estimates, exactly the full estimate, and no limit.
"""
import pytest

from tests import fixtures
from v3d import abi, profiles

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from v3d import dense
    c = dense.Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("offsets", [(0.0, 0.24), (0.0, 0.24, -0.22)])
def test_budget_plans_equal_the_oracle(ctx, oracle, offsets):
    frames = [fixtures.plane_frame(center_x=c) for c in offsets]
    cams = [fixtures.camera(i, c) for i, c in enumerate(offsets)]
    sparse = fixtures.plane_sparse_points()
    prof = profiles.reference()
    sizes = [oracle.estimate_working_set(frames, 320, 3, v, False)["total_bytes"]
             for v in (1, 2, 3)]
    for budget in [1, sizes[0] - 1] + sizes + [(1 << 64) - 1]:
        g, gp = ctx.estimate_depth_points_with_budget_and_control(
            frames, cams, sparse, fixtures.FOCAL, budget, 320, 3, profile=prof)
        o, op = oracle.estimate_depth_points_with_budget_and_control(
            frames, cams, sparse, fixtures.FOCAL, budget, 320, 3, prof)
        assert gp == op, budget
        assert g.status == o.status
        assert dict(g.stats) == dict(o.stats), budget
        assert g.points.tobytes() == o.points.tobytes()
        assert g.grid_sites.tobytes() == o.grid_sites.tobytes()
        assert g.point_attributes.tobytes() == o.point_attributes.tobytes()
        if gp["reference_views"] == 0:
            assert g.status == abi.SKIPPED
            assert g.stats["skip_code"] == abi.SKIP_WORKING_SET_BUDGET
            assert "exceeds the configured %d byte budget" % budget in g.stats["skip_reason"]


def test_a_cancel_during_the_landmark_test_is_sticky(ctx, oracle):
    """The control polled by has_distributed_landmarks stays canceled for the pass."""
    frames, cams, sparse = fixtures.three_view_scene(fixtures.SCENES["multi_reference"])
    results = []
    for impl in ("gpu", "oracle"):
        polls = []

        def control():
            polls.append(1)
            return len(polls) == 1

        if impl == "gpu":
            r, p = ctx.estimate_depth_points_with_budget_and_control(
                frames, cams, sparse, fixtures.FOCAL, (1 << 64) - 1, 320, 3,
                profile=profiles.reference(), control=control)
        else:
            r, p = oracle.estimate_depth_points_with_budget_and_control(
                frames, cams, sparse, fixtures.FOCAL, (1 << 64) - 1, 320, 3,
                profiles.reference(), control=control)
        results.append((r.status, r.stats["skip_reason"], p, len(polls)))
    assert results[0] == results[1]
