"""Python mirror of video-to-3d-core's dense and mesh API over the CUDA library.

Function names and argument meaning follow crates/video-to-3d-core/src:
``estimate_depth_points_with_control`` (dense_legacy.rs:149-156),
``reconstruct_reference_patches`` (dense.rs:674-747, batched),
``estimate_depth_points_limited`` (dense.rs:250-330),
``has_distributed_landmarks`` (dense.rs:165-213), ``grid_stride``
(dense.rs:215-218) and ``reconstruct_dense_mesh_with_control``
(mesh.rs:74-220).  Every compute call runs on the GPU through
libv3d_dense.so; there is no CPU fallback, and a missing library or device
raises.
"""
import ctypes as C
import os

import numpy as np

from . import abi, profiles, types

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(HERE), "lib", "libv3d_dense.so")
_P = C.POINTER
_lib = None


class V3DError(RuntimeError):
    def __init__(self, status, message=""):
        self.status = status
        super().__init__("v3d status %d%s" % (status, (": " + message) if message else ""))


def library():
    """Load libv3d_dense.so (built by video-to-3d_b200/build.py)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise FileNotFoundError("%s is missing; run video-to-3d_b200/build.py" % LIB_PATH)
    L = C.CDLL(LIB_PATH)
    frames_args = [_P(abi.Frame), C.c_uint64, _P(abi.Camera), C.c_uint64, _P(C.c_double),
                   C.c_uint64, C.c_double]
    L.v3d_abi_version.restype = C.c_int32
    L.v3d_status_text.argtypes = [C.c_int32]
    L.v3d_status_text.restype = C.c_char_p
    L.v3d_skip_reason_text.argtypes = [C.c_int32]
    L.v3d_skip_reason_text.restype = C.c_char_p
    L.v3d_last_error.argtypes = [C.c_void_p]
    L.v3d_last_error.restype = C.c_char_p
    L.v3d_context_create.argtypes = [C.c_int32, _P(C.c_void_p)]
    L.v3d_context_create.restype = C.c_int32
    L.v3d_context_destroy.argtypes = [C.c_void_p]
    L.v3d_context_destroy.restype = None
    L.v3d_profile_reference.argtypes = [_P(abi.Profile)]
    L.v3d_profile_zncc.argtypes = [_P(abi.Profile), C.c_int32, C.c_int32, C.c_int32, C.c_int32]
    L.v3d_grid_stride.argtypes = [C.c_uint32, C.c_uint32, C.c_int32]
    L.v3d_grid_stride.restype = C.c_uint64
    L.v3d_estimate_depth_points_with_control.argtypes = [C.c_void_p] + frames_args + [
        C.c_int32, _P(abi.Profile), abi.CANCEL_FN, C.c_void_p, _P(abi.DenseResult)]
    L.v3d_estimate_depth_points_with_control.restype = C.c_int32
    L.v3d_reconstruct_reference_patches.argtypes = [C.c_void_p] + frames_args + [
        C.c_int32, _P(abi.Profile), _P(C.c_uint64), C.c_uint64, abi.CANCEL_FN, C.c_void_p,
        _P(abi.DenseResult), _P(C.c_int32)]
    L.v3d_reconstruct_reference_patches.restype = C.c_int32
    L.v3d_estimate_depth_points_limited.argtypes = [C.c_void_p] + frames_args + [
        C.c_uint64, C.c_int32, _P(abi.Profile), abi.CANCEL_FN, C.c_void_p, _P(abi.DenseResult),
        _P(C.c_int32)]
    L.v3d_estimate_depth_points_limited.restype = C.c_int32
    L.v3d_estimate_depth_points_with_budget_and_control.argtypes = [C.c_void_p] + frames_args + [
        C.c_uint64, C.c_uint64, C.c_uint32, _P(abi.Profile), abi.CANCEL_FN, C.c_void_p,
        _P(abi.DenseResult), _P(abi.DenseBudget)]
    L.v3d_estimate_depth_points_with_budget_and_control.restype = C.c_int32
    L.v3d_estimate_working_set.argtypes = [_P(abi.Frame), C.c_uint64, C.c_uint64, C.c_uint32,
                                           C.c_uint64, C.c_int32, _P(abi.WorkingSetEstimate)]
    L.v3d_estimate_working_set.restype = C.c_int32
    L.v3d_has_distributed_landmarks.argtypes = frames_args + [abi.CANCEL_FN, C.c_void_p]
    L.v3d_has_distributed_landmarks.restype = C.c_int32
    L.v3d_dense_result_free.argtypes = [_P(abi.DenseResult)]
    L.v3d_dense_result_free.restype = None
    L.v3d_reconstruct_dense_mesh_with_control.argtypes = [
        C.c_void_p, _P(abi.Point), C.c_uint64, _P(abi.GridSite), C.c_uint64,
        _P(abi.MeshDenseInput), _P(abi.Camera), C.c_uint64, C.c_uint32, C.c_uint32,
        C.c_double, abi.CANCEL_FN, C.c_void_p, _P(abi.MeshResult)]
    L.v3d_reconstruct_dense_mesh_with_control.restype = C.c_int32
    L.v3d_mesh_result_free.argtypes = [_P(abi.MeshResult)]
    L.v3d_mesh_result_free.restype = None
    L.v3d_debug_sweep.argtypes = [C.c_void_p] + frames_args + [
        C.c_int32, _P(abi.Profile), _P(abi.SiteRecord), C.c_uint64, _P(C.c_uint64)]
    L.v3d_debug_sweep.restype = C.c_int32
    L.v3d_reconstruct_reference_patches_meshed.argtypes = [C.c_void_p] + frames_args + [
        C.c_int32, _P(abi.Profile), _P(C.c_uint64), C.c_uint64, abi.CANCEL_FN, C.c_void_p,
        _P(abi.DenseResult), _P(abi.MeshResult), _P(C.c_int32)]
    L.v3d_reconstruct_reference_patches_meshed.restype = C.c_int32
    L.v3d_reconstruct_clips.argtypes = [C.c_void_p, _P(abi.Clip), C.c_uint64, C.c_int32,
                                        _P(abi.Profile), abi.CANCEL_FN, C.c_void_p,
                                        _P(abi.DenseResult), _P(abi.MeshResult), _P(C.c_int32)]
    L.v3d_reconstruct_clips.restype = C.c_int32
    L.v3d_server_create.argtypes = [_P(abi.ServerConfig), _P(C.c_void_p)]
    L.v3d_server_create.restype = C.c_int32
    L.v3d_server_destroy.argtypes = [C.c_void_p]
    L.v3d_server_destroy.restype = None
    L.v3d_server_add_clip.argtypes = [C.c_void_p, _P(abi.Frame), C.c_uint64, _P(abi.Camera),
                                      C.c_uint64, _P(C.c_double), C.c_uint64, C.c_double,
                                      _P(C.c_uint64)]
    L.v3d_server_add_clip.restype = C.c_int32
    L.v3d_server_submit.argtypes = [C.c_void_p, C.c_uint64, C.c_uint64, C.c_int32, C.c_int32,
                                    _P(C.c_uint64)]
    L.v3d_server_submit.restype = C.c_int32
    L.v3d_server_wait.argtypes = [C.c_void_p, C.c_uint64, C.c_int64, _P(abi.DenseResult),
                                  _P(abi.MeshResult), _P(C.c_int32), _P(abi.RequestTiming)]
    L.v3d_server_wait.restype = C.c_int32
    L.v3d_server_last_error.argtypes = [C.c_void_p, C.c_char_p, C.c_uint64]
    L.v3d_server_last_error.restype = C.c_uint64
    L.v3d_fuse_mutually_supported_vertices.argtypes = [
        C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint64, C.c_void_p, abi.CANCEL_FN,
        C.c_void_p, _P(abi.FusionStats), C.c_void_p, _P(C.c_uint64), C.c_void_p, _P(C.c_uint64)]
    L.v3d_fuse_mutually_supported_vertices.restype = C.c_int32
    L.v3d_merge_fused_patches_owned.argtypes = [
        C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p,
        C.c_uint64, C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint64, abi.CANCEL_FN, C.c_void_p,
        _P(_P(abi.MergeResult))]
    L.v3d_merge_fused_patches_owned.restype = C.c_int32
    L.v3d_merge_result_free.argtypes = [_P(abi.MergeResult)]
    L.v3d_merge_result_free.restype = None
    L.v3d_verify_depth_grids.argtypes = [
        C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint32,
        C.c_uint32, C.c_double, C.c_void_p, C.c_uint64, C.c_void_p, _P(abi.VerificationFunnel)]
    L.v3d_verify_depth_grids.restype = C.c_int32
    L.v3d_surface_topology_of.argtypes = [C.c_void_p, C.c_void_p, C.c_uint64, C.c_uint64,
                                          _P(abi.SurfaceTopology)]
    L.v3d_surface_topology_of.restype = C.c_int32
    L.v3d_plan_clips.argtypes = [C.c_void_p, C.c_void_p, C.c_uint64, _P(C.c_uint64),
                                 _P(C.c_uint64), _P(C.c_int32)]
    L.v3d_plan_clips.restype = C.c_int32
    L.v3d_verified_surface_bounds.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint64,
                                              _P(C.c_uint64), _P(C.c_uint64)]
    L.v3d_verified_surface_bounds.restype = None
    L.v3d_mesh_verified_depth_grids.argtypes = [
        C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint32,
        C.c_uint32, C.c_double, C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint64,
        C.c_void_p, _P(abi.VerifiedSurface)]
    L.v3d_mesh_verified_depth_grids.restype = C.c_int32
    L.v3d_dense_document_bound.argtypes = [C.c_uint64] * 5
    L.v3d_dense_document_bound.restype = C.c_uint64
    L.v3d_encode_dense_evidence.argtypes = [
        C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint64,
        C.c_char_p, C.c_uint64, C.c_char_p, C.c_uint64, C.c_void_p, C.c_uint64,
        _P(abi.DenseDocument)]
    L.v3d_encode_dense_evidence.restype = C.c_int32
    L.v3d_pack_dense_points.argtypes = [C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p]
    L.v3d_pack_dense_points.restype = None
    L.v3d_pack_mesh_triangles.argtypes = [C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint64,
                                          C.c_void_p, C.c_uint64, C.c_uint64] + [C.c_void_p] * 5 + [
                                          _P(C.c_char_p)]
    L.v3d_pack_mesh_triangles.restype = C.c_int32
    L.v3d_sha256.argtypes = [C.c_char_p, C.c_uint64, C.c_void_p]
    L.v3d_sha256.restype = None
    L.v3d_last_run_info.argtypes = [C.c_void_p, _P(abi.RunInfo)]
    L.v3d_last_run_info.restype = C.c_int32
    _lib = L
    return L


class Context:
    """A CUDA stream plus device buffers on one GPU (v3d_context)."""

    def __init__(self, device=0):
        self.lib = library()
        self.handle = C.c_void_p()
        st = self.lib.v3d_context_create(int(device), C.byref(self.handle))
        if st != abi.OK:
            raise V3DError(st, self.lib.v3d_status_text(st).decode())

    def close(self):
        if self.handle:
            self.lib.v3d_context_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st):
        if st < 0:
            raise V3DError(st, self.lib.v3d_last_error(self.handle).decode())
        return st

    # Results are wrapped without copying their arrays: the numpy views own the
    # C result and free it when they are collected.
    def _dense(self, out, st=abi.OK):
        return types.dense_from_result(
            out, st, types.ResultOwner(self.lib.v3d_dense_result_free, out))

    def _mesh(self, out):
        return types.mesh_from_result(out, types.ResultOwner(self.lib.v3d_mesh_result_free, out))

    def estimate_depth_points_with_control(self, frames, cameras, sparse_points, focal,
                                           fine_grid=False, control=None, profile=None):
        prof = profile if profile is not None else profiles.reference()
        inp = types.Inputs(frames, cameras, sparse_points)
        fn, _keep = types.cancel_callback(control)
        out = abi.DenseResult()
        st = self._check(self.lib.v3d_estimate_depth_points_with_control(
            self.handle, inp.frames, inp.n_frames, inp.cameras, inp.n_cameras, inp.sparse,
            inp.n_sparse, float(focal), int(fine_grid), C.byref(prof), fn, None, C.byref(out)))
        return self._dense(out, st)

    def reconstruct_reference_patches(self, frames, cameras, sparse_points, focal,
                                      camera_indices, profile=None, fine_grid=False,
                                      control=None):
        prof = profile if profile is not None else profiles.reference()
        inp = types.Inputs(frames, cameras, sparse_points)
        fn, _keep = types.cancel_callback(control)
        n = len(camera_indices)
        idx = (C.c_uint64 * max(n, 1))(*camera_indices)
        outs = (abi.DenseResult * max(n, 1))()
        present = (C.c_int32 * max(n, 1))()
        self._check(self.lib.v3d_reconstruct_reference_patches(
            self.handle, inp.frames, inp.n_frames, inp.cameras, inp.n_cameras, inp.sparse,
            inp.n_sparse, float(focal), int(fine_grid), C.byref(prof), idx, n, fn, None, outs,
            present))
        return [self._dense(outs[i]) if present[i] else None for i in range(n)]

    def reconstruct_reference_patches_meshed(self, frames, cameras, sparse_points, focal,
                                             camera_indices, profile=None, fine_grid=False,
                                             control=None):
        """Per-reference passes plus each patch's grid-mesh triangles, in one device batch.
        Returns a list of (DenseAnalysis, MeshAnalysis) or None per camera index."""
        prof = profile if profile is not None else profiles.reference()
        inp = types.Inputs(frames, cameras, sparse_points)
        fn, _keep = types.cancel_callback(control)
        n = len(camera_indices)
        idx = (C.c_uint64 * max(n, 1))(*camera_indices)
        outs = (abi.DenseResult * max(n, 1))()
        meshes = (abi.MeshResult * max(n, 1))()
        present = (C.c_int32 * max(n, 1))()
        self._check(self.lib.v3d_reconstruct_reference_patches_meshed(
            self.handle, inp.frames, inp.n_frames, inp.cameras, inp.n_cameras, inp.sparse,
            inp.n_sparse, float(focal), int(fine_grid), C.byref(prof), idx, n, fn, None, outs,
            meshes, present))
        res = []
        for i in range(n):
            if present[i]:
                res.append((self._dense(outs[i]), self._mesh(meshes[i])))
            else:
                self.lib.v3d_dense_result_free(C.byref(outs[i]))
                self.lib.v3d_mesh_result_free(C.byref(meshes[i]))
                res.append(None)
        return res

    def reconstruct_clips(self, clips, profile=None, fine_grid=False, meshed=False,
                          control=None):
        """The references of many clips of uneven size in one device batch.

        `clips` is a list of dicts with keys frames, cameras, sparse_points, focal,
        camera_indices and optionally depth_hypotheses / max_source_views (per-clip
        overrides of the profile's).  Returns one list per clip with, per camera
        index, a DenseAnalysis (a (DenseAnalysis, MeshAnalysis) pair when `meshed`)
        or None where the reference returns None."""
        prof = profile if profile is not None else profiles.reference()
        fn, _keep = types.cancel_callback(control)
        inputs, arr = [], (abi.Clip * max(len(clips), 1))()
        counts = []
        for c, clip in enumerate(clips):
            inp = types.Inputs(clip["frames"], clip["cameras"], clip["sparse_points"])
            idx = list(clip["camera_indices"])
            ids = (C.c_uint64 * max(len(idx), 1))(*idx)
            inputs.append((inp, ids))
            arr[c] = abi.Clip(inp.frames, inp.n_frames, inp.cameras, inp.n_cameras, inp.sparse,
                              inp.n_sparse, float(clip["focal"]), ids, len(idx),
                              int(clip.get("depth_hypotheses", 0)),
                              int(clip.get("max_source_views", 0)))
            counts.append(len(idx))
        n = sum(counts)
        outs = (abi.DenseResult * max(n, 1))()
        meshes = (abi.MeshResult * max(n, 1))() if meshed else None
        present = (C.c_int32 * max(n, 1))()
        self._check(self.lib.v3d_reconstruct_clips(
            self.handle, arr, len(clips), int(fine_grid), C.byref(prof), fn, None, outs, meshes,
            present))
        flat = []
        for i in range(n):
            if present[i]:
                flat.append((self._dense(outs[i]), self._mesh(meshes[i])) if meshed
                            else self._dense(outs[i]))
            else:
                self.lib.v3d_dense_result_free(C.byref(outs[i]))
                if meshed:
                    self.lib.v3d_mesh_result_free(C.byref(meshes[i]))
                flat.append(None)
        res, at = [], 0
        for k in counts:
            res.append(flat[at:at + k])
            at += k
        return res

    def estimate_depth_points_limited(self, frames, cameras, sparse_points, focal,
                                      reference_views, fine_grid, profile=None, control=None):
        prof = profile if profile is not None else profiles.reference()
        inp = types.Inputs(frames, cameras, sparse_points)
        fn, _keep = types.cancel_callback(control)
        out = abi.DenseResult()
        omitted = C.c_int32()
        st = self._check(self.lib.v3d_estimate_depth_points_limited(
            self.handle, inp.frames, inp.n_frames, inp.cameras, inp.n_cameras, inp.sparse,
            inp.n_sparse, float(focal), int(reference_views), int(fine_grid), C.byref(prof), fn,
            None, C.byref(out), C.byref(omitted)))
        return self._dense(out, st), bool(omitted.value)

    def estimate_depth_points_with_budget_and_control(self, frames, cameras, sparse_points, focal,
                                                      working_set_budget_bytes, max_features,
                                                      descriptor_radius, profile=None,
                                                      control=None):
        """dense.rs:355-420: the budget plan, then the limited pass.  Returns the
        analysis and the plan: {"working_set_estimate": {...}, "working_set_budget_bytes",
        "full_working_set_bytes", "fine_grid", "reference_views"}."""
        prof = profile if profile is not None else profiles.reference()
        inp = types.Inputs(frames, cameras, sparse_points)
        fn, _keep = types.cancel_callback(control)
        out = abi.DenseResult()
        plan = abi.DenseBudget()
        st = self._check(self.lib.v3d_estimate_depth_points_with_budget_and_control(
            self.handle, inp.frames, inp.n_frames, inp.cameras, inp.n_cameras, inp.sparse,
            inp.n_sparse, float(focal), int(working_set_budget_bytes), int(max_features),
            int(descriptor_radius), C.byref(prof), fn, None, C.byref(out), C.byref(plan)))
        return self._dense(out, st), budget_plan(plan)

    def last_run_info(self):
        """Device time, kernel launches and work units of the last dense call."""
        info = abi.RunInfo()
        self._check(self.lib.v3d_last_run_info(self.handle, C.byref(info)))
        return {name: (list(getattr(info, name)) if name == "merge_stage_ms" else getattr(info, name))
                for name, _ in abi.RunInfo._fields_}

    def debug_sweep(self, frames, cameras, sparse_points, focal, fine_grid=False, profile=None):
        """Per-site sweep records (status, plane, support, error, margin) in raster order."""
        prof = profile if profile is not None else profiles.reference()
        inp = types.Inputs(frames, cameras, sparse_points)
        n = C.c_uint64()
        st = self._check(self.lib.v3d_debug_sweep(
            self.handle, inp.frames, inp.n_frames, inp.cameras, inp.n_cameras, inp.sparse,
            inp.n_sparse, float(focal), int(fine_grid), C.byref(prof), None, 0, C.byref(n)))
        if st == abi.SKIPPED:
            return None
        buf = (abi.SiteRecord * max(n.value, 1))()
        self._check(self.lib.v3d_debug_sweep(
            self.handle, inp.frames, inp.n_frames, inp.cameras, inp.n_cameras, inp.sparse,
            inp.n_sparse, float(focal), int(fine_grid), C.byref(prof), buf, n.value, C.byref(n)))
        return types.site_records(buf, n.value)

    def reconstruct_dense_mesh_with_control(self, points, grid_sites, stats, cameras, width,
                                            height, focal, control=None):
        mi = types.MeshInputs(points, grid_sites, stats)
        cams = types.Inputs([], cameras, [])
        fn, _keep = types.cancel_callback(control)
        out = abi.MeshResult()
        self._check(self.lib.v3d_reconstruct_dense_mesh_with_control(
            self.handle, *mi.args(), cams.cameras, cams.n_cameras, int(width), int(height),
            float(focal), fn, None, C.byref(out)))
        return self._mesh(out)

    def plan_clips(self, clips):
        """reference_candidate_order (dense.rs:620-672) and has_distributed_landmarks
        (dense.rs:165-213) of many clips in one device pass.  `clips` is a list of
        dicts with frames, cameras, sparse_points and focal; returns one (order,
        distributed) pair per clip."""
        keep, arr = [], (abi.Clip * max(len(clips), 1))()
        total = 0
        for c, clip in enumerate(clips):
            inp = types.Inputs(clip["frames"], clip["cameras"], clip["sparse_points"])
            keep.append(inp)
            arr[c] = abi.Clip(inp.frames, inp.n_frames, inp.cameras, inp.n_cameras, inp.sparse,
                              inp.n_sparse, float(clip["focal"]), None, 0, 0, 0)
            total += len(clip["cameras"])
        orders = (C.c_uint64 * max(total, 1))()
        counts = (C.c_uint64 * max(len(clips), 1))()
        flags = (C.c_int32 * max(len(clips), 1))()
        self._check(self.lib.v3d_plan_clips(self.handle, arr, len(clips), orders, counts, flags))
        out, base = [], 0
        for c, clip in enumerate(clips):
            out.append(([int(orders[base + i]) for i in range(counts[c])], bool(flags[c])))
            base += len(clip["cameras"])
        return out

    def surface_topology(self, triangles, vertex_count):
        """surface_topology (colmap_surface.rs:125-157) on the device: a dict of
        islands, small_islands, small_island_triangles, largest_island_triangles
        and boundary_edges."""
        st, out = _topology(self.lib.v3d_surface_topology_of, (self.handle,), triangles,
                            vertex_count)
        self._check(st)
        return out

    def verify_depth_grids(self, views, reference_views, source_views, stride, reference_stride,
                           focal):
        """verify_patch and verified_union (colmap_surface.rs:175-314) for every
        reference on the device: (samples per reference, funnel dict)."""
        st, per_ref, funnel = _verify(self.lib.v3d_verify_depth_grids, (self.handle,), views,
                                      reference_views, source_views, stride, reference_stride,
                                      focal)
        self._check(st)
        return per_ref, funnel

    def encode_dense_evidence(self, points, grid_sites, point_attributes, prefix=b"",
                              suffix=b"", out=None):
        """DenseStageArtifact::to_json and content_hash
        (reconstruction_stages.rs:287-380) with the arrays formatted on the
        device: returns (document, info) where the document is
        prefix + the three arrays + suffix and info holds the array lengths,
        the count of non-finite floats (written as null) and content_hash
        ("sha256:" + 64 hex digits).  With `out` (a uint8 array of at least
        document_bound bytes, reused across calls) the document is a
        memoryview into it; otherwise new bytes."""
        st, doc, info = _encode(self.lib.v3d_encode_dense_evidence, (self.handle,), points,
                                grid_sites, point_attributes, prefix, suffix, out)
        self._check(st)
        return doc, info

    def mesh_verified_depth_grids(self, views, reference_views, source_views, stride,
                                  reference_stride, focal):
        """The geometric part of the COLMAP export (colmap_surface.rs:380-471)
        on the device: a VerifiedSurface.  A SKIPPED status (no triangle) is
        returned, not raised, with the diagnostics filled."""
        st, surf = _surface(self.lib.v3d_mesh_verified_depth_grids, (self.handle,), views,
                            reference_views, source_views, stride, reference_stride, focal)
        if st != abi.SKIPPED:
            self._check(st)
        return surf

    def merge_fused_patches_owned(self, points, triangles, membership, pairs, cameras,
                                  origins=None, control=None):
        """merge_fused_patches_owned_with_control (surface_merge.rs:312-353) on
        the device: a MergeOutcome, or MergeRejected with the reference's
        message."""
        st, out = _merge(self.lib.v3d_merge_fused_patches_owned, (self.handle,),
                         self.lib.v3d_merge_result_free,
                         lambda: self.lib.v3d_last_error(self.handle).decode(), points, triangles,
                         membership, pairs, cameras, origins, control)
        self._check(st)
        return out

    def fuse_mutually_supported_vertices(self, points, triangles, membership, control=None):
        """fuse_mutually_supported_vertices_with_control (surface_fusion.rs:369-549)
        on the device: moves `points` in place and returns a FusionOutcome."""
        st, out = _fuse(self.lib.v3d_fuse_mutually_supported_vertices, (self.handle,), points,
                        triangles, membership, control)
        self._check(st)
        return out


class FusionOutcome:
    """FusionOutcome (surface_fusion.rs:27-32): stats (a dict of FusionStats),
    pairs (n x 2 uint64, first < second) and moved_indices (ascending)."""

    def __init__(self, stats, pairs, moved_indices):
        self.stats = stats
        self.pairs = pairs
        self.moved_indices = moved_indices


def fusion_arguments(points, triangles, membership):
    """Checked contiguous arrays for v3d_fuse_mutually_supported_vertices:
    points (POINT_DTYPE, moved in place, so it must already be contiguous),
    triangles (TRIANGLE_DTYPE) and membership (int64, negative = no group)."""
    if not (isinstance(points, np.ndarray) and points.dtype == types.POINT_DTYPE
            and points.flags.c_contiguous and points.flags.writeable):
        raise TypeError("points must be a writable contiguous POINT_DTYPE array")
    tris = np.ascontiguousarray(triangles, dtype=types.TRIANGLE_DTYPE)
    mem = np.ascontiguousarray(membership, dtype=np.int64)
    if mem.shape != (len(points),):
        raise ValueError("membership needs one entry per point")
    return tris, mem


def fusion_outcome(stats, pairs, n_pairs, moved, n_moved):
    st = {name: int(getattr(stats, name)) for name, _ in abi.FusionStats._fields_}
    return FusionOutcome(st, pairs[:n_pairs].copy(), moved[:n_moved].copy())


def _fuse(lib_fn, head, points, triangles, membership, control):
    tris, mem = fusion_arguments(points, triangles, membership)
    n = len(points)
    fn, _keep = types.cancel_callback(control)
    stats = abi.FusionStats()
    pairs = np.empty((max(n // 2, 1), 2), dtype=np.uint64)
    moved = np.empty(max(n, 1), dtype=np.uint64)
    n_pairs, n_moved = C.c_uint64(), C.c_uint64()
    st = lib_fn(*head, points.ctypes.data, n, tris.ctypes.data, len(tris), mem.ctypes.data, fn,
                None, C.byref(stats), pairs.ctypes.data, C.byref(n_pairs), moved.ctypes.data,
                C.byref(n_moved))
    return st, fusion_outcome(stats, pairs, n_pairs.value, moved, n_moved.value)


DERIVED_DTYPE = np.dtype([("point_index", "<u8"), ("source_triangle", "<u8"),
                          ("source_corners", "<u8", (3,)), ("barycentric", "<f8", (3,))])
SOURCE_DTYPE = np.dtype([("triangle", "<u8"), ("corners", "<u8", (3,))])


class MergeOutcome:
    """OwnedMerge (surface_merge.rs:276-283): points (POINT_DTYPE, the input
    points then the derived ones), triangles (TRIANGLE_DTYPE), derived_vertices
    (DERIVED_DTYPE), and MergeStats as `stats` (a dict of the scalar fields)
    with uncalibrated_patch_pairs (n x 2), retained_by_group and
    triangle_sources (SOURCE_DTYPE)."""

    def __init__(self, r):
        def arr(ptr, n, dtype):
            if n == 0:
                return np.empty(0, dtype=dtype)
            buf = (C.c_char * (n * dtype.itemsize)).from_address(ptr)
            return np.frombuffer(buf, dtype=dtype, count=n).copy()
        self.stats = {f: getattr(r.stats, f) for f in abi.MERGE_STAT_FIELDS}
        self.points = arr(r.points, r.n_points, types.POINT_DTYPE)
        self.triangles = arr(r.triangles, r.n_triangles, types.TRIANGLE_DTYPE)
        self.derived_vertices = arr(r.derived_vertices, r.n_derived_vertices, DERIVED_DTYPE)
        self.uncalibrated_patch_pairs = arr(r.uncalibrated_patch_pairs,
                                            2 * r.n_uncalibrated_patch_pairs,
                                            np.dtype("<u8")).reshape(-1, 2)
        self.retained_by_group = arr(r.retained_by_group, r.n_retained_by_group, np.dtype("<u8"))
        self.triangle_sources = arr(r.triangle_sources, r.n_triangle_sources, SOURCE_DTYPE)


class MergeRejected(Exception):
    """The reference's Err(message) of merge_fused_patches_owned_with_control."""


def merge_arguments(points, triangles, membership, pairs, cameras, origins):
    """Contiguous arrays for v3d_merge_fused_patches_owned.  cameras: one entry
    per support group, None or an object with `rotation` (3x3) and
    `translation` (3); origins: None (an empty slice) or one origin per point
    (abi.ORIGIN_*, abi.ORIGIN_NONE for none)."""
    pts = np.ascontiguousarray(points, dtype=types.POINT_DTYPE)
    tris = np.ascontiguousarray(triangles, dtype=types.TRIANGLE_DTYPE)
    mem = np.ascontiguousarray(membership, dtype=np.int64)
    if len(mem) != len(pts):
        raise ValueError("membership needs one entry per point")
    prs = np.ascontiguousarray(np.asarray(pairs, dtype=np.uint64).reshape(-1, 2))
    cams = (abi.ReferenceCamera * max(len(cameras), 1))()
    for i, cam in enumerate(cameras):
        if cam is not None:
            R = np.asarray(cam.rotation, dtype=np.float64).reshape(9)
            t = np.asarray(cam.translation, dtype=np.float64).reshape(3)
            cams[i] = abi.ReferenceCamera(1, 0, (C.c_double * 9)(*R), (C.c_double * 3)(*t))
    org = np.ascontiguousarray(np.zeros(0) if origins is None else origins, dtype=np.int32)
    return pts, tris, mem, prs, cams, len(cameras), org


def _merge(lib_fn, head, free_fn, error_fn, points, triangles, membership, pairs, cameras,
           origins, control):
    pts, tris, mem, prs, cams, n_cams, org = merge_arguments(points, triangles, membership,
                                                             pairs, cameras, origins)
    fn, _keep = types.cancel_callback(control)
    out = C.POINTER(abi.MergeResult)()
    st = lib_fn(*head, pts.ctypes.data, len(pts), tris.ctypes.data, len(tris), mem.ctypes.data,
                prs.ctypes.data, len(prs), cams, n_cams, org.ctypes.data, len(org), fn, None,
                C.byref(out))
    if st == abi.REJECTED:
        raise MergeRejected(error_fn())
    if st != 0:
        return st, None
    try:
        return st, MergeOutcome(out.contents)
    finally:
        free_fn(out)


VERIFIED_DTYPE = np.dtype([("x", "<f4"), ("y", "<f4"), ("z", "<f4"), ("confidence", "<f4"),
                           ("r", "u1"), ("g", "u1"), ("b", "u1"), ("pad", "u1"),
                           ("site_x", "<u4"), ("site_y", "<u4"), ("source_mask", "<u4")])


def _depth_views(views, reference_views, source_views):
    """ctypes arrays of v3d_depth_view, references and 4 sources per reference
    (-1 for none), and the numpy arrays they point into."""
    keep = []
    arr = (abi.DepthView * max(len(views), 1))()
    for i, (rgba, depth, cam) in enumerate(views):
        rgba = np.ascontiguousarray(rgba, dtype=np.uint8)
        depth = np.ascontiguousarray(depth, dtype=np.float32)
        keep += [rgba, depth]
        R = np.asarray(cam.rotation, dtype=np.float64).reshape(9)
        t = np.asarray(cam.translation, dtype=np.float64).reshape(3)
        arr[i] = abi.DepthView(rgba.ctypes.data, depth.ctypes.data, rgba.shape[1], rgba.shape[0],
                               abi.Camera(int(cam.frame_index), (C.c_double * 9)(*R),
                                          (C.c_double * 3)(*t)))
    n_ref = len(reference_views)
    refs = np.ascontiguousarray(reference_views, dtype=np.uint32)
    src = np.full((max(n_ref, 1), 4), -1, dtype=np.int32)
    for r, s in enumerate(source_views):
        if len(s) > 4:
            raise ValueError("at most 4 source views per reference")
        src[r, :len(s)] = s
    return arr, keep, refs, src


DOMINANT_REJECTIONS = [None, "missing_reference_depth", "insufficient_parallax", "behind_source",
                       "outside_source", "missing_source_depth", "depth_disagreement",
                       "color_disagreement"]


class VerifiedSurface:
    """The geometric part of the COLMAP export: points (POINT_DTYPE), sites
    (SITE_DTYPE), triangles (TRIANGLE_DTYPE, indices into points), regions
    (dicts of reference_frame, first_point, point_count, source_frames) and
    diagnostics (verification, meshing, topology, dominant_rejection); status
    is OK, or SKIPPED when no triangle was exported."""

    def __init__(self, status, points, sites, triangles, regions, diagnostics):
        self.status = status
        self.points = points
        self.sites = sites
        self.triangles = triangles
        self.regions = regions
        self.diagnostics = diagnostics


def _surface(lib_fn, head, views, reference_views, source_views, stride, reference_stride, focal):
    arr, keep, refs, src = _depth_views(views, reference_views, source_views)
    n_ref = len(reference_views)
    h, w = (views[0][0].shape[0], views[0][0].shape[1]) if views else (0, 0)
    mp, mt = C.c_uint64(), C.c_uint64()
    library().v3d_verified_surface_bounds(w, h, int(reference_stride), n_ref, C.byref(mp), C.byref(mt))
    pts = np.empty(max(mp.value, 1), dtype=types.POINT_DTYPE)
    sites = np.empty(max(mp.value, 1), dtype=types.SITE_DTYPE)
    tris = np.empty(max(mt.value, 1), dtype=types.TRIANGLE_DTYPE)
    regs = (abi.VerifiedSurfaceRegion * max(n_ref, 1))()
    out = abi.VerifiedSurface()
    st = lib_fn(*head, arr, len(views), refs.ctypes.data, n_ref, src.ctypes.data, int(stride),
                int(reference_stride), float(focal), pts.ctypes.data, sites.ctypes.data, len(pts),
                tris.ctypes.data, len(tris), regs, C.byref(out))
    as_dict = lambda s: {name: int(getattr(s, name)) for name, _ in s._fields_}  # noqa: E731
    diag = {"verification": as_dict(out.verification), "meshing": as_dict(out.meshing),
            "topology": as_dict(out.topology),
            "dominant_rejection": DOMINANT_REJECTIONS[out.dominant_rejection]}
    if st != 0:
        return st, VerifiedSurface(st, pts[:0], sites[:0], tris[:0], [], diag)
    regions = [{"reference_frame": int(g.reference_frame), "first_point": int(g.first_point),
                "point_count": int(g.point_count),
                "source_frames": [int(g.source_frames[i]) for i in range(g.n_source_frames)]}
               for g in regs[:out.n_regions]]
    n, nt = out.n_points, out.n_triangles
    return st, VerifiedSurface(st, pts[:n], sites[:n], tris[:nt], regions, diag)


def _verify(lib_fn, head, views, reference_views, source_views, stride, reference_stride, focal):
    """Shared by the device entry point and the oracle: views is a list of
    (rgba uint8 [h, w, 4], depth float32 [rows, cols], camera); source_views one
    list of at most 4 view indices per reference.  Returns (samples per
    reference as VERIFIED_DTYPE arrays, funnel dict)."""
    arr, keep, refs, src = _depth_views(views, reference_views, source_views)
    n_ref = len(reference_views)
    h, w = (views[0][0].shape[0], views[0][0].shape[1]) if views else (0, 0)
    cap = max(n_ref * (-(-w // reference_stride)) * (-(-h // reference_stride)), 1)
    out = np.empty(cap, dtype=VERIFIED_DTYPE)
    offsets = np.zeros(n_ref + 1, dtype=np.uint64)
    funnel = abi.VerificationFunnel()
    st = lib_fn(*head, arr, len(views), refs.ctypes.data, n_ref, src.ctypes.data, int(stride),
                int(reference_stride), float(focal), out.ctypes.data, cap, offsets.ctypes.data,
                C.byref(funnel))
    # views into one buffer: no copy per reference
    per_ref = [out[int(offsets[r]):int(offsets[r + 1])] for r in range(n_ref)] if st >= 0 else []
    return st, per_ref, {name: int(getattr(funnel, name)) for name, _ in funnel._fields_}


def document_bound(n_points, n_grid_sites, n_point_attributes, prefix_bytes=0, suffix_bytes=0):
    """v3d_dense_document_bound: bytes that always hold the document."""
    return int(library().v3d_dense_document_bound(n_points, n_grid_sites, n_point_attributes,
                                                  prefix_bytes, suffix_bytes))


def _encode(lib_fn, head, points, grid_sites, point_attributes, prefix, suffix, out=None):
    """Shared by the device entry point and the oracle: points (POINT_DTYPE),
    grid_sites (SITE_DTYPE) and point_attributes (ATTR_DTYPE), any of them
    None for an empty array; prefix and suffix bytes; out an optional
    reusable uint8 buffer."""
    def arr(a, dt):
        return np.ascontiguousarray(np.zeros(0, dt) if a is None else a, dtype=dt)
    pts = arr(points, types.POINT_DTYPE)
    sites = arr(grid_sites, types.SITE_DTYPE)
    attrs = arr(point_attributes, types.ATTR_DTYPE)
    prefix, suffix = bytes(prefix), bytes(suffix)
    cap = document_bound(len(pts), len(sites), len(attrs), len(prefix), len(suffix))
    if out is None:
        buf = np.empty(max(cap, 1), dtype=np.uint8)
    else:
        buf = out
        if not (isinstance(buf, np.ndarray) and buf.dtype == np.uint8 and buf.flags.c_contiguous
                and buf.flags.writeable and buf.size >= cap):
            raise ValueError("out must be a writable contiguous uint8 array of %d bytes" % cap)
    res = abi.DenseDocument()
    st = lib_fn(*head, pts.ctypes.data, len(pts), sites.ctypes.data, len(sites), attrs.ctypes.data,
                len(attrs), prefix, len(prefix), suffix, len(suffix), buf.ctypes.data, buf.size,
                C.byref(res))
    info = {name: int(getattr(res, name)) for name, _ in res._fields_ if name != "sha256"}
    digest = bytes(res.sha256)
    info["content_hash"] = "sha256:" + digest.hex() if any(digest) else None
    if st != 0:
        return st, b"", info
    doc = buf[:res.document_bytes]
    return st, (doc.tobytes() if out is None else memoryview(doc)), info


def pack_dense_points(points):
    """pack_dense_points (crates/video-to-3d-wasm/src/lib.rs:227-240):
    (values_f32_le, rgb) byte strings.  Grid sites and point attributes need
    no packing: SITE_DTYPE and ATTR_DTYPE arrays are already those buffers."""
    pts = np.ascontiguousarray(points, dtype=types.POINT_DTYPE)
    values = np.empty(16 * len(pts), dtype=np.uint8)
    rgb = np.empty(3 * len(pts), dtype=np.uint8)
    library().v3d_pack_dense_points(pts.ctypes.data, len(pts), values.ctypes.data, rgb.ctypes.data)
    return values.tobytes(), rgb.tobytes()


TRIANGLE_SOURCE_DTYPE = np.dtype([("triangle", "<u8"), ("corners", "<u8", (3,))])
DERIVED_VERTEX_DTYPE = np.dtype([("point_index", "<u8"), ("source_triangle", "<u8"),
                                 ("source_corners", "<u8", (3,)), ("barycentric", "<f8", (3,))])


def pack_mesh_triangles(triangles, point_count, sources=None, derived=None):
    """pack_mesh_triangles (crates/video-to-3d-wasm/src/lib.rs:269-326): a dict
    of the five little-endian buffers; ValueError with the reference's message
    when an index does not fit the transport."""
    tris = np.ascontiguousarray(triangles, dtype=types.TRIANGLE_DTYPE)
    src = np.ascontiguousarray(np.zeros(0, TRIANGLE_SOURCE_DTYPE) if sources is None else sources,
                               dtype=TRIANGLE_SOURCE_DTYPE)
    der = np.ascontiguousarray(np.zeros(0, DERIVED_VERTEX_DTYPE) if derived is None else derived,
                               dtype=DERIVED_VERTEX_DTYPE)
    bufs = {"indices_u32_le": np.empty(12 * len(tris), np.uint8),
            "confidence_f32_le": np.empty(4 * len(tris), np.uint8),
            "sources_u32_le": np.empty(16 * len(src), np.uint8),
            "derived_u32_le": np.empty(20 * len(der), np.uint8),
            "derived_barycentric_f64_le": np.empty(24 * len(der), np.uint8)}
    err = C.c_char_p()
    st = library().v3d_pack_mesh_triangles(
        tris.ctypes.data, len(tris), src.ctypes.data, len(src), der.ctypes.data, len(der),
        int(point_count), *(b.ctypes.data for b in bufs.values()), C.byref(err))
    if st != 0:
        raise ValueError(err.value.decode() if err.value else "invalid arguments")
    return {k: v.tobytes() for k, v in bufs.items()}


def content_hash(data):
    """ContentHash::of_bytes (scene_project.rs:463-465) through the library's
    host SHA-256."""
    data = bytes(data)
    digest = (C.c_uint8 * 32)()
    library().v3d_sha256(data, len(data), digest)
    return "sha256:" + bytes(digest).hex()


def _topology(lib_fn, head, triangles, vertex_count):
    tris = np.ascontiguousarray(triangles, dtype=types.TRIANGLE_DTYPE)
    out = abi.SurfaceTopology()
    st = lib_fn(*head, tris.ctypes.data, len(tris), int(vertex_count), C.byref(out))
    return st, {name: int(getattr(out, name)) for name, _ in out._fields_}


def budget_plan(plan):
    est = plan.working_set_estimate
    return {"working_set_estimate": {n: int(getattr(est, n)) for n in abi.WORKING_SET_FIELDS},
            "working_set_budget_bytes": int(plan.working_set_budget_bytes),
            "full_working_set_bytes": int(plan.full_working_set_bytes),
            "fine_grid": bool(plan.fine_grid), "reference_views": int(plan.reference_views)}


def estimate_working_set(frames, max_features, descriptor_radius, reference_views, fine_grid):
    """dense.rs:423-605 on the host (no device needed)."""
    inp = types.Inputs(frames, [], [])
    out = abi.WorkingSetEstimate()
    st = library().v3d_estimate_working_set(inp.frames, inp.n_frames, int(max_features),
                                            int(descriptor_radius), int(reference_views),
                                            int(fine_grid), C.byref(out))
    if st != abi.OK:
        raise V3DError(st)
    return {n: int(getattr(out, n)) for n in abi.WORKING_SET_FIELDS}


def has_distributed_landmarks(frames, cameras, sparse_points, focal, control=None):
    inp = types.Inputs(frames, cameras, sparse_points)
    fn, _keep = types.cancel_callback(control)
    return bool(library().v3d_has_distributed_landmarks(
        inp.frames, inp.n_frames, inp.cameras, inp.n_cameras, inp.sparse, inp.n_sparse,
        float(focal), fn, None))


def grid_stride(width, height, fine_grid):
    return int(library().v3d_grid_stride(int(width), int(height), int(fine_grid)))


class Served:
    """Outcome of one served request: status, result (a DenseAnalysis, a
    (DenseAnalysis, MeshAnalysis) pair for a meshed server, or None where the
    reference returns None) and the request's timing."""

    def __init__(self, status, result, timing):
        self.status = status
        self.result = result
        self.timing = timing


class Server:
    """A device-resident request loop on one GPU (v3d_server).

    Clips are registered once (their frames stay in device memory); each request
    is one reference camera of a clip with optional per-request hypothesis and
    source-view counts.  `slots` batches run at once, each on its own stream."""

    def __init__(self, device=0, slots=2, memory_budget=0, max_batch_requests=0, meshed=False,
                 fine_grid=False, profile=None):
        self.lib = library()
        self.meshed = bool(meshed)
        cfg = abi.ServerConfig(int(device), int(slots), int(memory_budget), int(max_batch_requests),
                               int(self.meshed), int(bool(fine_grid)),
                               profile if profile is not None else profiles.reference())
        h = C.c_void_p()
        st = self.lib.v3d_server_create(C.byref(cfg), C.byref(h))
        if st < 0:
            raise V3DError(st, "v3d_server_create failed")
        self.handle = h

    def close(self):
        if self.handle:
            self.lib.v3d_server_destroy(self.handle)
            self.handle = None

    def __del__(self):
        self.close()

    def add_clip(self, frames, cameras, sparse_points, focal):
        inp = types.Inputs(frames, cameras, sparse_points)
        cid = C.c_uint64()
        st = self.lib.v3d_server_add_clip(self.handle, inp.frames, inp.n_frames, inp.cameras,
                                          inp.n_cameras, inp.sparse, inp.n_sparse, float(focal),
                                          C.byref(cid))
        if st < 0:
            raise V3DError(st, "v3d_server_add_clip failed")
        return cid.value

    def submit(self, clip_id, camera_index, depth_hypotheses=0, max_source_views=0):
        t = C.c_uint64()
        st = self.lib.v3d_server_submit(self.handle, int(clip_id), int(camera_index),
                                        int(depth_hypotheses), int(max_source_views), C.byref(t))
        if st < 0:
            raise V3DError(st, "v3d_server_submit failed")
        return t.value

    def wait(self, ticket, timeout_ms=-1):
        """The request's Served outcome, or None while it is not done within timeout_ms."""
        out = abi.DenseResult()
        mesh = abi.MeshResult()
        present = C.c_int32()
        timing = abi.RequestTiming()
        st = self.lib.v3d_server_wait(self.handle, int(ticket), int(timeout_ms), C.byref(out),
                                      C.byref(mesh) if self.meshed else None, C.byref(present),
                                      C.byref(timing))
        if st == abi.TIMEOUT:
            return None
        t = {name: getattr(timing, name) for name, _ in abi.RequestTiming._fields_}
        if st < 0:
            buf = C.create_string_buffer(1024)
            self.lib.v3d_server_last_error(self.handle, buf, len(buf))
            raise V3DError(st, "request failed: " + buf.value.decode(errors="replace"))
        if not present.value:
            self.lib.v3d_dense_result_free(C.byref(out))
            if self.meshed:
                self.lib.v3d_mesh_result_free(C.byref(mesh))
            return Served(st, None, t)
        dense = types.dense_from_result(
            out, st, types.ResultOwner(self.lib.v3d_dense_result_free, out))
        if self.meshed:
            m = types.mesh_from_result(mesh, types.ResultOwner(self.lib.v3d_mesh_result_free, mesh))
            return Served(st, (dense, m), t)
        return Served(st, dense, t)
