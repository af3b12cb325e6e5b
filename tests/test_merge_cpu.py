"""The connected-surface merge's CPU oracle (oracle/oracle_merge.cpp), pinned
by the reference's own tests of surface_merge.rs and its derived acceptance
tests, restated in oracle/oracle_merge_selftest.cpp; and the C surface the
device path shares with it (argument checks, the Err path, the outcome's
shape on the reference fixtures)."""
import numpy as np
import pytest

from v3d import abi, dense

from tests import merge_fixtures as mf
from tests.oracle_ffi import Oracle


def test_reference_tests_pass_on_the_oracle():
    checks, failure = Oracle().merge_selftest()
    assert failure == "" and checks > 6000, failure


def _run(case, control=None):
    return Oracle().merge_fused_patches_owned(case["points"], case["triangles"], case["membership"],
                                              case["pairs"], case["cameras"], case["origins"],
                                              control=control)


def test_trimmed_seam_through_the_c_surface():
    out = _run(mf.trimmed_seam())
    s = out.stats
    assert s["removed_duplicate_triangles"] == 4 and s["trimmed_seam_triangles"] == 4
    assert s["stitched_seam_triangles"] == 4 and s["patch_components"] == 1
    assert len(out.points) == 27 and len(out.derived_vertices) == 0
    assert list(out.retained_by_group) == [16, 12 - 4]


def test_partial_overlap_derives_vertices_with_lineage():
    case = mf.partial_overlap(sloped=True)
    out = _run(case)
    n = len(case["points"])
    assert len(out.points) == n + len(out.derived_vertices) and len(out.derived_vertices) > 0
    assert out.points[:n].tobytes() == case["points"].tobytes()
    for rec in out.derived_vertices:
        assert rec["point_index"] >= n
        w = rec["barycentric"]
        assert abs(w.sum() - 1.0) < 1e-7
    assert out.stats["conformed_triangles"] > 0


def test_cancellation_is_an_err_and_no_result():
    polls = []

    def cancel():
        polls.append(1)
        return len(polls) >= 5
    with pytest.raises(dense.MergeRejected, match="reconstruction canceled"):
        _run(mf.partial_overlap(sloped=True), control=cancel)


def test_no_pairs_keep_every_triangle():
    case = mf.trimmed_seam()
    case["pairs"] = np.zeros((0, 2), dtype=np.uint64)
    out = _run(case)
    assert out.stats["removed_duplicate_triangles"] == 0
    assert out.triangles.tobytes() == case["triangles"].tobytes()


def test_synthetic_patches_merge_into_one_surface():
    o = Oracle()
    case = mf.synthetic_case(o, n_patches=6, width=160, height=90)
    out = _run(case)
    s = out.stats
    assert s["fused_pairs"] > 0 and s["removed_duplicate_triangles"] > 0
    assert s["meshed_patches"] == 6 and s["clipped_overlap_triangles"] > 0
    assert len(out.triangles) < len(case["triangles"])


def test_a_seam_that_cannot_be_conformed_rejects_the_merge():
    # this seeded cut leaves one triangle that cannot be split at its clipped
    # seam vertices: the reference rejects the whole merge (surface_merge.rs:333-338)
    o = Oracle()
    case = mf.synthetic_case(o, n_patches=4, width=96, height=54)
    with pytest.raises(dense.MergeRejected, match="could not split 1 triangle"):
        _run(case)
