"""The connected-surface merge on the device (v3d_merge_fused_patches_owned)
against the CPU oracle, bit for bit: every output point and triangle, every
derived vertex's lineage, every statistic (the trimmed-area share included)
and the Err message where the reference rejects the merge -- on the
reference's own fixtures and on seeded multi-reference patches fused by the
oracle's fusion."""
import numpy as np
import pytest

from v3d import dense

from tests import merge_fixtures as mf
from tests.oracle_ffi import Oracle


def _both(case, control_g=None, control_o=None):
    args = (case["points"], case["triangles"], case["membership"], case["pairs"], case["cameras"],
            case["origins"])
    ctx = dense.Context(0)
    try:
        g = ctx.merge_fused_patches_owned(*args, control=control_g)
    except dense.MergeRejected as e:
        g = e
    try:
        o = Oracle().merge_fused_patches_owned(*args, control=control_o)
    except dense.MergeRejected as e:
        o = e
    return g, o


def _same(g, o):
    if isinstance(o, Exception):
        assert isinstance(g, Exception) and str(g) == str(o)
        return
    assert not isinstance(g, Exception), str(g)
    assert g.stats == o.stats  # the f64 area share compares exactly
    assert g.points.tobytes() == o.points.tobytes()
    assert g.triangles.tobytes() == o.triangles.tobytes()
    assert g.derived_vertices.tobytes() == o.derived_vertices.tobytes()
    assert np.array_equal(g.uncalibrated_patch_pairs, o.uncalibrated_patch_pairs)
    assert np.array_equal(g.retained_by_group, o.retained_by_group)
    assert g.triangle_sources.tobytes() == o.triangle_sources.tobytes()


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(mf.reference_cases()))
def test_reference_fixtures(name):
    case = mf.reference_cases()[name]
    g, o = _both(case)
    _same(g, o)


@pytest.mark.gpu
@pytest.mark.parametrize("kw", [dict(n_patches=6, width=160, height=90, seed=7),
                                dict(n_patches=4, width=96, height=54, seed=7),
                                dict(n_patches=8, width=200, height=112, seed=11, arc_deg=20.0),
                                dict(n_patches=5, width=128, height=72, seed=3, scale_drift=0.03)])
def test_synthetic_patches(kw):
    case = mf.synthetic_case(Oracle(), **kw)
    g, o = _both(case)
    _same(g, o)
    if not isinstance(o, Exception):
        assert o.stats["removed_duplicate_triangles"] > 0


@pytest.mark.gpu
def test_cancellation_is_an_err():
    case = mf.partial_overlap(sloped=True)
    n = []

    def cancel():
        n.append(1)
        return len(n) >= 4
    g, _ = _both(case, control_g=cancel)
    assert isinstance(g, dense.MergeRejected) and "reconstruction canceled" in str(g)


@pytest.mark.gpu
def test_without_cameras_and_origins():
    case = mf.synthetic_case(Oracle(), n_patches=4, width=120, height=68, seed=5)
    case["cameras"] = []
    case["origins"] = None
    g, o = _both(case)
    _same(g, o)
