"""Scenes of the reference's own dense tests, rebuilt in Python.

camera/texture/plane_frame/plane_sparse_points follow
crates/video-to-3d-core/src/dense_legacy.rs:1189-1238 (the same helpers are
in dense.rs:1159-1208 and surface_completion_tests.rs:4-53): a 68x48 view of a
textured plane at depth 4 seen by cameras translated along x.
"""
import math

import numpy as np

from v3d.types import FrameInput, RegisteredCamera

WIDTH, HEIGHT, FOCAL, DEPTH = 68, 48, 60.0, 4.0


def camera(frame_index, center_x):
    return RegisteredCamera(frame_index, np.eye(3), np.array([-center_x, 0.0, 0.0]))


def texture(wx, wy):
    v = (128.0 + 55.0 * math.sin(wx * 15.0 + wy * 2.7) + 40.0 * math.cos(wy * 17.0 - wx * 3.1)
         + 25.0 * math.sin((wx + wy) * 11.0))
    return int(min(max(round_half_away(v), 0.0), 255.0))


def round_half_away(v):
    return math.floor(v + 0.5) if v >= 0 else -math.floor(-v + 0.5)


def plane_frame(width=WIDTH, height=HEIGHT, focal=FOCAL, center_x=0.0, depth=DEPTH):
    rgba = np.zeros((height, width, 4), dtype=np.uint8)
    for y in range(height):
        for x in range(width):
            wx = center_x + (x - width * 0.5) / focal * depth
            wy = (y - height * 0.5) / focal * depth
            v = texture(wx, wy)
            rgba[y, x] = (v, v, v, 255)
    return FrameInput(rgba)


def flat_frame(width=WIDTH, height=HEIGHT, value=120):
    return FrameInput(np.full((height, width, 4), value, dtype=np.uint8))


def plane_sparse_points(width=WIDTH, height=HEIGHT, focal=FOCAL, depth=DEPTH):
    pts = []
    for y in (10, 18, 26, 34):
        for x in (12, 24, 36, 48, 56):
            pts.append(((x - width * 0.5) / focal * depth, (y - height * 0.5) / focal * depth,
                        depth))
    return np.array(pts, dtype=np.float64)


def three_view_scene(offsets=(0.0, 0.18, -0.16)):
    """dense_legacy.rs:1262-1273 (0.18/-0.16) or dense.rs:1216-1222 (0.24/-0.22)."""
    frames = [plane_frame(center_x=c) for c in offsets]
    cams = [camera(i, c) for i, c in enumerate(offsets)]
    return frames, cams, plane_sparse_points()


SCENES = {
    "legacy_plane": (0.0, 0.18, -0.16),      # dense_legacy.rs:1262
    "multi_reference": (0.0, 0.24, -0.22),   # dense.rs:1211
    "completion": (0.0, 0.25, -0.22),        # surface_completion_tests.rs:56
    "two_view": (0.0, 0.24),                 # dense.rs:1270
}
