"""Host-side data types of the dense pass and their conversion to the C ABI.

The Python names follow the Rust API of video-to-3d-core:
``FrameInput`` (reconstruction/types.rs:17-21), ``RegisteredCamera``
(multi_view.rs:85-89), ``DenseAnalysis`` (dense_legacy.rs:62-68,
dense.rs:142-148) and ``MeshAnalysis`` (mesh_legacy.rs:40-43, mesh.rs:46-49).
"""
import ctypes as C
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

from . import abi

POINT_DTYPE = np.dtype([("x", "<f4"), ("y", "<f4"), ("z", "<f4"), ("confidence", "<f4"),
                        ("r", "u1"), ("g", "u1"), ("b", "u1"), ("pad", "u1")])
SITE_DTYPE = np.dtype([("x", "<u4"), ("y", "<u4")])
ATTR_DTYPE = np.dtype([("reciprocal_consistency", "<f4"), ("depth_margin", "<f4")])
TRIANGLE_DTYPE = np.dtype([("a", "<u8"), ("b", "<u8"), ("c", "<u8"), ("confidence", "<f4"),
                           ("pad", "<u4")])

_FORMAT_OF_DTYPE = {np.dtype(np.float32): abi.PIXEL_GRAY_F32,
                    np.dtype(np.float16): abi.PIXEL_GRAY_F16}


@dataclass
class FrameInput:
    """One frame: RGBA8 (h, w, 4) uint8, or a gray (h, w) float32/float16 plane, or a
    (h, w) uint16 array of bfloat16 bits with ``bf16=True``."""
    pixels: np.ndarray
    bf16: bool = False

    @property
    def width(self):
        return int(self.pixels.shape[1])

    @property
    def height(self):
        return int(self.pixels.shape[0])

    @property
    def format(self):
        if self.pixels.ndim == 3:
            return abi.PIXEL_RGBA8
        if self.bf16:
            return abi.PIXEL_GRAY_BF16
        return _FORMAT_OF_DTYPE[self.pixels.dtype]


@dataclass
class RegisteredCamera:
    """World-to-camera pose: x_cam = rotation @ x_world + translation."""
    frame_index: int
    rotation: np.ndarray = field(default_factory=lambda: np.eye(3))
    translation: np.ndarray = field(default_factory=lambda: np.zeros(3))

    def camera_center(self):
        return -(self.rotation.T @ self.translation)


@dataclass
class DenseAnalysis:
    stats: dict
    points: np.ndarray
    grid_sites: np.ndarray
    point_attributes: np.ndarray
    status: int = abi.OK


@dataclass
class MeshAnalysis:
    stats: dict
    triangles: np.ndarray
    reference_frames: List[int]
    reference_patches: List[dict]


class Inputs:
    """Keeps the ctypes arrays (and the numpy buffers they point at) alive."""

    def __init__(self, frames, cameras, sparse_points):
        self._keep = []
        n = len(frames)
        self.frames = (abi.Frame * max(n, 1))()
        for i, f in enumerate(frames):
            px = np.ascontiguousarray(f.pixels)
            self._keep.append(px)
            self.frames[i] = abi.Frame(f.width, f.height, f.format, 0, px.ctypes.data)
        self.n_frames = n
        m = len(cameras)
        self.cameras = (abi.Camera * max(m, 1))()
        for i, c in enumerate(cameras):
            R = np.asarray(c.rotation, dtype=np.float64).reshape(3, 3)
            t = np.asarray(c.translation, dtype=np.float64).reshape(3)
            self.cameras[i] = abi.Camera(int(c.frame_index), (C.c_double * 9)(*R.ravel()),
                                         (C.c_double * 3)(*t))
        self.n_cameras = m
        sp = np.ascontiguousarray(np.asarray(sparse_points, dtype=np.float64).reshape(-1, 3))
        self._keep.append(sp)
        self.sparse = sp.ctypes.data_as(C.POINTER(C.c_double))
        self.n_sparse = int(sp.shape[0])


def cancel_callback(control):
    """Wrap a Python callable (returns True when canceled) as a v3d_cancel_fn."""
    if control is None:
        return abi.CANCEL_FN(), None
    state = {"canceled": False}

    def poll(_user):
        if not state["canceled"] and control():
            state["canceled"] = True
        return 1 if state["canceled"] else 0

    fn = abi.CANCEL_FN(poll)
    return fn, fn


def _text(raw):
    return raw.decode("utf-8") if isinstance(raw, bytes) else raw


def _opt(has, value):
    return value if has else None


class ResultOwner:
    """Frees one C result when the last array viewing its memory is collected.

    The device library hands results back in page-locked memory shared by a
    whole batch; wrapping them without a copy keeps that memory alive exactly
    as long as a numpy view of it exists."""

    __slots__ = ("_free", "_ref")

    def __init__(self, free, struct):
        self._free = free
        self._ref = C.pointer(struct)  # keeps the struct (and its array) alive

    def __del__(self):
        free, self._free = self._free, None
        if free is not None:
            free(self._ref)


def _array(ptr, n, dtype, owner=None):
    if n == 0 or not ptr:
        return np.zeros(0, dtype=dtype)
    addr = C.cast(ptr, C.c_void_p).value
    buf = (C.c_char * (n * dtype.itemsize)).from_address(addr)
    if owner is None:
        return np.frombuffer(buf, dtype=dtype).copy()
    buf._owner = owner
    return np.frombuffer(buf, dtype=dtype)


def stats_dict(s):
    d = {
        "attempted": bool(s.attempted),
        "skip_reason": _text(s.skip_reason) if s.has_skip_reason else None,
        "skip_code": int(s.skip_code),
        "reference_frame": _opt(s.has_reference_frame, int(s.reference_frame)),
        "source_views": int(s.source_views),
        "grid_stride": int(s.grid_stride),
        "grid_border": int(s.grid_border),
        "median_fusion_observations": _opt(s.has_median_fusion_observations,
                                           float(s.median_fusion_observations)),
        "median_supporting_views": _opt(s.has_median_supporting_views,
                                        float(s.median_supporting_views)),
        "median_photometric_error": _opt(s.has_median_photometric_error,
                                         float(s.median_photometric_error)),
        "search_min_depth": _opt(s.has_search_min_depth, float(s.search_min_depth)),
        "search_max_depth": _opt(s.has_search_max_depth, float(s.search_max_depth)),
        "reference_view_limit": _opt(s.has_reference_view_limit, int(s.reference_view_limit)),
    }
    for name in abi._COUNTERS + ["reciprocal_checked_points", "reciprocal_rejected_points",
                                 "reciprocal_consistent_points", "fusion_input_observations",
                                 "fusion_rejected_observations", "fusion_rejected_points"]:
        d[name] = int(getattr(s, name))
    return d


def _attempt_dict(a):
    d = {"reference_frame": int(a.reference_frame), "attempted": bool(a.attempted),
         "accepted": bool(a.accepted),
         "skip_reason": _text(a.skip_reason) if a.has_skip_reason else None}
    for name, _ in abi.ReferenceAttempt._fields_:
        if name not in d and name not in ("has_skip_reason", "pad0"):
            d[name] = int(getattr(a, name))
    return d


def _patch_dict(p):
    return {
        "reference_frame": int(p.reference_frame),
        "source_frames": [int(p.source_frames[i]) for i in range(p.n_source_frames)],
        "primary_start": int(p.primary_start), "primary_points": int(p.primary_points),
        "completion_start": int(p.completion_start),
        "completed_points": int(p.completed_points),
        "sampled_pixels": int(p.sampled_pixels), "accepted_points": int(p.accepted_points),
        "reciprocal_consistent_points": int(p.reciprocal_consistent_points),
        "grid_stride": int(p.grid_stride), "grid_border": int(p.grid_border),
        "search_min_depth": _opt(p.has_search_min_depth, float(p.search_min_depth)),
        "search_max_depth": _opt(p.has_search_max_depth, float(p.search_max_depth)),
    }


def dense_from_result(r, status=abi.OK, owner=None):
    """DenseAnalysis of a C result; with `owner` (a ResultOwner of r) the point
    arrays are views of the result's memory, else copies."""
    stats = stats_dict(r.stats)
    stats["source_frames"] = [int(r.source_frames[i]) for i in range(r.n_source_frames)]
    stats["reference_frames"] = [int(r.reference_frames[i]) for i in range(r.n_reference_frames)]
    stats["reference_attempts"] = [_attempt_dict(r.attempts[i]) for i in range(r.n_attempts)]
    stats["reference_patches"] = [_patch_dict(r.patches[i]) for i in range(r.n_patches)]
    n = int(r.n_points)
    return DenseAnalysis(stats=stats, points=_array(r.points, n, POINT_DTYPE, owner),
                         grid_sites=_array(r.grid_sites, n, SITE_DTYPE, owner),
                         point_attributes=_array(r.point_attributes, n, ATTR_DTYPE, owner),
                         status=status)


def _mesh_stats_dict(s):
    d = {"attempted": bool(s.attempted),
         "skip_reason": _text(s.skip_reason) if s.has_skip_reason else None,
         "reference_frame": _opt(s.has_reference_frame, int(s.reference_frame))}
    for name in ("point_count", "grid_vertices", "rejected_grid_vertices", "candidate_cells",
                 "candidate_triangles", "accepted_triangles", "rejected_discontinuities",
                 "rejected_degenerate"):
        d[name] = int(getattr(s, name))
    return d


def mesh_from_result(r, owner=None):
    """MeshAnalysis of a C mesh result; `owner` as for dense_from_result."""
    return MeshAnalysis(
        stats=_mesh_stats_dict(r.stats),
        triangles=_array(r.triangles, int(r.n_triangles), TRIANGLE_DTYPE, owner),
        reference_frames=[int(r.reference_frames[i]) for i in range(r.n_reference_frames)],
        reference_patches=[_mesh_stats_dict(r.patches[i]) for i in range(r.n_patches)])


class MeshInputs:
    """ctypes view of dense points, grid sites and the DenseStats subset the mesh reads."""

    def __init__(self, points, grid_sites, stats):
        self.points = np.ascontiguousarray(points, dtype=POINT_DTYPE)
        self.sites = np.ascontiguousarray(grid_sites, dtype=SITE_DTYPE)
        patches = stats.get("reference_patches") or []
        self._patch_arr = (abi.ReferencePatch * max(len(patches), 1))()
        self._keep = []
        for i, p in enumerate(patches):
            src = np.asarray(p.get("source_frames", []), dtype=np.uint64)
            self._keep.append(src)
            q = self._patch_arr[i]
            q.reference_frame = p["reference_frame"]
            q.n_source_frames = len(src)
            q.source_frames = src.ctypes.data_as(C.POINTER(C.c_uint64))
            for k in ("primary_start", "primary_points", "completion_start", "completed_points",
                      "accepted_points", "grid_stride", "grid_border"):
                setattr(q, k, int(p.get(k, 0)))
        rf = stats.get("reference_frame")
        self.dense = abi.MeshDenseInput(
            int(bool(stats.get("attempted"))), int(rf is not None), int(rf or 0),
            int(stats.get("grid_stride", 0)), int(stats.get("grid_border", 0)), 0,
            len(patches), C.cast(self._patch_arr, C.POINTER(abi.ReferencePatch)))

    def args(self):
        return (self.points.ctypes.data_as(C.POINTER(abi.Point)), len(self.points),
                self.sites.ctypes.data_as(C.POINTER(abi.GridSite)), len(self.sites),
                C.byref(self.dense))


def site_records(buf, n):
    """numpy view of n v3d_site_record entries."""
    return np.frombuffer(bytes(buf)[: n * C.sizeof(abi.SiteRecord)],
                         dtype=np.dtype(abi.SITE_RECORD_DTYPE)).copy()
