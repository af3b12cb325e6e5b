"""Host side of surface consolidation's first step: the inputs of
``Context.fuse_mutually_supported_vertices``.

``support_membership`` is evidence_support_membership
(crates/video-to-3d-core/src/surface_fusion.rs:316-345): every evidence region
with a reference frame joins the camera-support group of its (reference frame,
sorted source frames), groups numbered in first-seen order, and its points
take that group.  ``consolidation_inputs`` lays reference patches out the way
the consolidated dense buffer holds them (one region per patch, points
concatenated in patch order, triangle indices shifted to match).
"""
import numpy as np

from . import types


def support_membership(regions, point_count):
    """regions: iterable of (reference_frame or None, source_frames, start, count).
    Returns (membership int64 [point_count], -1 for none; number of groups)."""
    membership = np.full(point_count, -1, dtype=np.int64)
    groups = {}
    for reference_frame, source_frames, start, count in regions:
        if reference_frame is None:
            continue
        key = (int(reference_frame), tuple(sorted(int(s) for s in source_frames)))
        group = groups.setdefault(key, len(groups))
        end = start + count
        if start < 0 or end > point_count or end < start:
            continue
        membership[start:end] = group
    return membership, len(groups)


def consolidation_inputs(patches):
    """patches: (DenseAnalysis, MeshAnalysis) per reference patch, in order.
    Returns (points POINT_DTYPE, triangles TRIANGLE_DTYPE, membership int64,
    number of support groups)."""
    points, tris, regions = [], [], []
    base = 0
    for dense, mesh in patches:
        n = len(dense.points)
        points.append(np.asarray(dense.points, dtype=types.POINT_DTYPE))
        t = np.array(mesh.triangles, dtype=types.TRIANGLE_DTYPE, copy=True)
        for k in ("a", "b", "c"):
            t[k] += np.uint64(base)
        tris.append(t)
        regions.append((dense.stats.get("reference_frame"), dense.stats.get("source_frames", []),
                        base, n))
        base += n
    pts = np.concatenate(points) if points else np.zeros(0, dtype=types.POINT_DTYPE)
    tri = np.concatenate(tris) if tris else np.zeros(0, dtype=types.TRIANGLE_DTYPE)
    membership, groups = support_membership(regions, len(pts))
    return np.ascontiguousarray(pts), np.ascontiguousarray(tri), membership, groups
