"""ctypes wrapper of the CPU oracle (oracle/_build/liboracle_v3d.so).

Test infrastructure only: the parity tests use it as the checker, bench.py
uses it as the timed CPU baseline.  Its functions take the same Python inputs
as ``v3d.dense`` and return the same result objects.
"""
import ctypes as C
import os

import numpy as np

from v3d import abi, types

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "oracle", "_build", "liboracle_v3d.so")

_P = C.POINTER

# ExplainRecord (oracle/oracle.hpp)
EXPLAIN_DTYPE = np.dtype([("x", "<u4"), ("y", "<u4"), ("stage", "<i4"), ("outcome", "<i4"),
                          ("plane", "<i4"), ("support", "<i4"), ("error", "<f8"),
                          ("margin", "<f8"), ("sweep_gap", "<f8"),
                          ("recip_gap", "<f8")])


class Oracle:
    def __init__(self, path=LIB):
        self.lib = C.CDLL(path)
        L = self.lib
        frames_args = [_P(abi.Frame), C.c_uint64, _P(abi.Camera), C.c_uint64,
                       _P(C.c_double), C.c_uint64, C.c_double]
        L.v3do_estimate_depth_points_with_control.argtypes = frames_args + [
            C.c_int32, _P(abi.Profile), abi.CANCEL_FN, C.c_void_p, _P(abi.DenseResult)]
        L.v3do_estimate_depth_points_with_control.restype = C.c_int32
        L.v3do_reconstruct_reference_patches.argtypes = frames_args + [
            C.c_int32, _P(abi.Profile), _P(C.c_uint64), C.c_uint64, C.c_int32,
            _P(abi.DenseResult), _P(C.c_int32)]
        L.v3do_reconstruct_reference_patches.restype = C.c_int32
        L.v3do_estimate_depth_points_limited.argtypes = frames_args + [
            C.c_uint64, C.c_int32, _P(abi.Profile), abi.CANCEL_FN, C.c_void_p,
            _P(abi.DenseResult), _P(C.c_int32)]
        L.v3do_estimate_depth_points_limited.restype = C.c_int32
        L.v3do_has_distributed_landmarks.argtypes = frames_args + [abi.CANCEL_FN, C.c_void_p]
        L.v3do_has_distributed_landmarks.restype = C.c_int32
        L.v3do_reconstruct_dense_mesh_with_control.argtypes = [
            _P(abi.Point), C.c_uint64, _P(abi.GridSite), C.c_uint64, _P(abi.MeshDenseInput),
            _P(abi.Camera), C.c_uint64, C.c_uint32, C.c_uint32, C.c_double, abi.CANCEL_FN,
            C.c_void_p, _P(abi.MeshResult)]
        L.v3do_reconstruct_dense_mesh_with_control.restype = C.c_int32
        L.v3do_dense_result_free.argtypes = [_P(abi.DenseResult)]
        L.v3do_mesh_result_free.argtypes = [_P(abi.MeshResult)]
        L.v3do_selftest.argtypes = [C.c_char_p, C.c_uint64, _P(C.c_int32)]
        L.v3do_selftest.restype = C.c_int32
        L.v3do_merge_fused_patches_owned.argtypes = [
            C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p, C.c_uint64,
            C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint64, abi.CANCEL_FN, C.c_void_p,
            _P(_P(abi.MergeResult))]
        L.v3do_merge_fused_patches_owned.restype = C.c_int32
        L.v3do_merge_result_free.argtypes = [_P(abi.MergeResult)]
        L.v3do_merge_result_free.restype = None
        L.v3do_merge_last_error.restype = C.c_char_p
        L.v3do_merge_selftest.argtypes = [C.c_char_p, C.c_uint64]
        L.v3do_merge_selftest.restype = C.c_int32
        L.v3do_merge_diagnostic.argtypes = [_P(abi.MergeResult), C.c_uint64, C.c_char_p,
                                            C.c_uint64]
        L.v3do_merge_diagnostic.restype = C.c_uint64
        L.v3do_patch_error.argtypes = [_P(abi.Profile), _P(abi.Camera), _P(abi.Camera),
                                       _P(abi.Frame), _P(abi.Frame), C.c_double, C.c_double,
                                       C.c_double, C.c_double, _P(C.c_double)]
        L.v3do_patch_error.restype = C.c_int32
        L.v3do_grid_stride.argtypes = [C.c_uint32, C.c_uint32, C.c_int32]
        L.v3do_grid_stride.restype = C.c_uint64
        L.v3do_max_threads.restype = C.c_int32
        L.v3do_debug_sweep.argtypes = frames_args + [C.c_int32, _P(abi.Profile),
                                                     _P(abi.SiteRecord), C.c_uint64,
                                                     _P(C.c_uint64)]
        L.v3do_debug_sweep.restype = C.c_int32
        L.v3do_fuse_mutually_supported_vertices.argtypes = [
            C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint64, C.c_void_p, abi.CANCEL_FN,
            C.c_void_p, _P(abi.FusionStats), C.c_void_p, _P(C.c_uint64), C.c_void_p,
            _P(C.c_uint64)]
        L.v3do_fuse_mutually_supported_vertices.restype = C.c_int32
        L.v3do_verify_depth_grids.argtypes = [
            C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint32, C.c_uint32,
            C.c_double, C.c_void_p, C.c_uint64, C.c_void_p, _P(abi.VerificationFunnel)]
        L.v3do_verify_depth_grids.restype = C.c_int32
        L.v3do_surface_topology_of.argtypes = [C.c_void_p, C.c_uint64, C.c_uint64,
                                               _P(abi.SurfaceTopology)]
        L.v3do_surface_topology_of.restype = C.c_int32
        L.v3do_reference_candidate_order.argtypes = frames_args + [_P(C.c_uint64), _P(C.c_uint64)]
        L.v3do_reference_candidate_order.restype = C.c_int32
        L.v3do_mesh_verified_depth_grids.argtypes = [
            C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint32, C.c_uint32,
            C.c_double, C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint64, C.c_void_p,
            _P(abi.VerifiedSurface)]
        L.v3do_mesh_verified_depth_grids.restype = C.c_int32
        L.v3do_shortest_f32.argtypes = [C.c_float, _P(C.c_uint32), _P(C.c_int32)]
        L.v3do_shortest_f32.restype = C.c_int32
        L.v3do_format_f32.argtypes = [C.c_float, C.c_char_p]
        L.v3do_format_f32.restype = C.c_uint64
        L.v3do_encode_dense_evidence.argtypes = [
            C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint64, C.c_char_p,
            C.c_uint64, C.c_char_p, C.c_uint64, C.c_void_p, C.c_uint64, _P(abi.DenseDocument)]
        L.v3do_encode_dense_evidence.restype = C.c_int32
        L.v3do_pack_dense_points.argtypes = [C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p]
        L.v3do_pack_mesh_triangles.argtypes = [C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint64,
                                               C.c_void_p, C.c_uint64, C.c_uint64] + [C.c_void_p] * 5
        L.v3do_pack_mesh_triangles.restype = C.c_int32

    def fuse_mutually_supported_vertices(self, points, triangles, membership, control=None):
        """surface_fusion.rs:369-549 on the CPU: moves `points` in place."""
        from v3d import dense
        st, out = dense._fuse(self.lib.v3do_fuse_mutually_supported_vertices, (), points,
                              triangles, membership, control)
        assert st == 0, st
        return out

    def verify_depth_grids(self, views, reference_views, source_views, stride, reference_stride,
                           focal):
        """colmap_surface.rs:175-314 on the CPU: (samples per reference, funnel)."""
        from v3d import dense
        st, per_ref, funnel = dense._verify(self.lib.v3do_verify_depth_grids, (), views,
                                            reference_views, source_views, stride,
                                            reference_stride, focal)
        assert st == 0, st
        return per_ref, funnel

    def surface_topology(self, triangles, vertex_count):
        """colmap_surface.rs:125-157 on the CPU."""
        from v3d import dense
        st, out = dense._topology(self.lib.v3do_surface_topology_of, (), triangles, vertex_count)
        assert st == 0, st
        return out

    def mesh_verified_depth_grids(self, views, reference_views, source_views, stride,
                                  reference_stride, focal):
        """colmap_surface.rs:380-471 on the CPU: a VerifiedSurface."""
        from v3d import dense
        st, surf = dense._surface(self.lib.v3do_mesh_verified_depth_grids, (), views,
                                  reference_views, source_views, stride, reference_stride, focal)
        assert st in (0, 1), st
        return surf

    def format_f32(self, value):
        """serde_json's text of one f32 (reconstruction_stages.rs:290-294)."""
        buf = C.create_string_buffer(32)
        n = self.lib.v3do_format_f32(float(value), buf)
        return buf.raw[:n].decode()

    def shortest_f32(self, value):
        """(digits, exponent) of the shortest round-trip decimal, None for 0
        and non-finite values."""
        d, k = C.c_uint32(), C.c_int32()
        if not self.lib.v3do_shortest_f32(float(value), C.byref(d), C.byref(k)):
            return None
        return d.value, k.value

    def encode_dense_evidence(self, points, grid_sites, point_attributes, prefix=b"",
                              suffix=b""):
        """The DenseEvidence arrays framed like v3d_encode_dense_evidence, on
        the CPU: (document bytes, info dict; its sha256 is left empty)."""
        from v3d import dense
        st, doc, info = dense._encode(self.lib.v3do_encode_dense_evidence, (), points, grid_sites,
                                      point_attributes, prefix, suffix)
        assert st == 0, st
        return doc, info

    def pack_dense_points(self, points):
        """pack_dense_points (wasm/src/lib.rs:227-240): (values_f32_le, rgb)."""
        import numpy as np
        pts = np.ascontiguousarray(points, dtype=types.POINT_DTYPE)
        values = np.empty(16 * len(pts), dtype=np.uint8)
        rgb = np.empty(3 * len(pts), dtype=np.uint8)
        self.lib.v3do_pack_dense_points(pts.ctypes.data, len(pts), values.ctypes.data,
                                        rgb.ctypes.data)
        return values.tobytes(), rgb.tobytes()

    def pack_mesh_triangles(self, triangles, point_count, sources, derived):
        """pack_mesh_triangles (wasm/src/lib.rs:269-326) on the CPU: (status,
        buffers dict); status 0, or 1 + the index of the failing message."""
        import numpy as np
        from v3d import dense
        tris = np.ascontiguousarray(triangles, dtype=types.TRIANGLE_DTYPE)
        src = np.ascontiguousarray(sources, dtype=dense.TRIANGLE_SOURCE_DTYPE)
        der = np.ascontiguousarray(derived, dtype=dense.DERIVED_VERTEX_DTYPE)
        bufs = [np.zeros(k * n, np.uint8) for k, n in
                ((12, len(tris)), (4, len(tris)), (16, len(src)), (20, len(der)), (24, len(der)))]
        st = self.lib.v3do_pack_mesh_triangles(
            tris.ctypes.data, len(tris), src.ctypes.data, len(src), der.ctypes.data, len(der),
            int(point_count), *(b.ctypes.data for b in bufs))
        names = ["indices_u32_le", "confidence_f32_le", "sources_u32_le", "derived_u32_le",
                 "derived_barycentric_f64_le"]
        return st, dict(zip(names, (b.tobytes() for b in bufs)))

    def reference_candidate_order(self, frames, cameras, sparse_points, focal):
        """dense.rs:620-672 on the CPU: camera indices in planning order."""
        inp = types.Inputs(frames, cameras, sparse_points)
        out = (C.c_uint64 * max(len(cameras), 1))()
        n = C.c_uint64()
        st = self.lib.v3do_reference_candidate_order(inp.frames, inp.n_frames, inp.cameras,
                                                     inp.n_cameras, inp.sparse, inp.n_sparse,
                                                     float(focal), out, C.byref(n))
        assert st == 0, st
        return [int(out[i]) for i in range(n.value)]

    def selftest(self):
        buf = C.create_string_buffer(1 << 16)
        checks = C.c_int32()
        failures = self.lib.v3do_selftest(buf, len(buf), C.byref(checks))
        return failures, checks.value, buf.value.decode()

    def merge_selftest(self):
        """The reference's surface-merge tests on the oracle: (checks, failure)."""
        buf = C.create_string_buffer(1 << 12)
        n = self.lib.v3do_merge_selftest(buf, len(buf))
        return n, buf.value.decode()

    def merge_fused_patches_owned(self, points, triangles, membership, pairs, cameras,
                                  origins=None, control=None):
        """surface_merge.rs:312-353 on the CPU: a MergeOutcome (MergeRejected on Err)."""
        from v3d import dense
        st, out = dense._merge(self.lib.v3do_merge_fused_patches_owned, (),
                               self.lib.v3do_merge_result_free,
                               lambda: self.lib.v3do_merge_last_error().decode(), points,
                               triangles, membership, pairs, cameras, origins, control)
        assert st == 0, st
        return out

    def max_threads(self):
        return self.lib.v3do_max_threads()

    def estimate_depth_points_with_control(self, frames, cameras, sparse_points, focal,
                                           fine_grid=False, control=None, profile=None):
        inp = types.Inputs(frames, cameras, sparse_points)
        fn, _keep = types.cancel_callback(control)
        out = abi.DenseResult()
        st = self.lib.v3do_estimate_depth_points_with_control(
            inp.frames, inp.n_frames, inp.cameras, inp.n_cameras, inp.sparse, inp.n_sparse,
            float(focal), int(fine_grid), C.byref(profile), fn, None, C.byref(out))
        if st < 0:
            raise ValueError("oracle rejected the inputs (status %d)" % st)
        try:
            return types.dense_from_result(out, st)
        finally:
            self.lib.v3do_dense_result_free(C.byref(out))

    def reconstruct_reference_patches(self, frames, cameras, sparse_points, focal,
                                      camera_indices, profile, fine_grid=False, threads=1):
        inp = types.Inputs(frames, cameras, sparse_points)
        n = len(camera_indices)
        idx = (C.c_uint64 * max(n, 1))(*camera_indices)
        outs = (abi.DenseResult * max(n, 1))()
        present = (C.c_int32 * max(n, 1))()
        st = self.lib.v3do_reconstruct_reference_patches(
            inp.frames, inp.n_frames, inp.cameras, inp.n_cameras, inp.sparse, inp.n_sparse,
            float(focal), int(fine_grid), C.byref(profile), idx, n, int(threads), outs, present)
        if st < 0:
            raise ValueError("oracle rejected the inputs (status %d)" % st)
        res = []
        for i in range(n):
            res.append(types.dense_from_result(outs[i]) if present[i] else None)
            self.lib.v3do_dense_result_free(C.byref(outs[i]))
        return res

    def explain_reference_patch(self, frames, cameras, sparse_points, focal, camera_index,
                                profile, fine_grid=False, rows=None):
        """The remapped pass of one reference (camera_index None: the legacy
        single call) and its decision records (ExplainRecord in
        oracle/oracle.hpp): primary sites in raster order, then the completion
        proposals of each pass.  None where the pass does not run.  rows=(a, b):
        only grid rows a..b-1, primaries only (no completion)."""
        L = self.lib
        if not getattr(self, "_explain_bound", False):
            L.v3do_explain_reference_patch.argtypes = [
                _P(abi.Frame), C.c_uint64, _P(abi.Camera), C.c_uint64, _P(C.c_double), C.c_uint64,
                C.c_double, C.c_int32, _P(abi.Profile), C.c_uint64, C.c_uint32, C.c_uint32,
                _P(abi.DenseResult), _P(C.c_void_p), _P(C.c_uint64)]
            L.v3do_explain_reference_patch.restype = C.c_int32
            L.v3do_free.argtypes = [C.c_void_p]
            self._explain_bound = True
        inp = types.Inputs(frames, cameras, sparse_points)
        out = abi.DenseResult()
        recs, n = C.c_void_p(), C.c_uint64()
        st = L.v3do_explain_reference_patch(
            inp.frames, inp.n_frames, inp.cameras, inp.n_cameras, inp.sparse, inp.n_sparse,
            float(focal), int(fine_grid), C.byref(profile),
            (1 << 64) - 1 if camera_index is None else int(camera_index),
            rows[0] if rows else 0, rows[1] if rows else 0, C.byref(out),
            C.byref(recs), C.byref(n))
        if st < 0:
            raise ValueError("oracle rejected the inputs (status %d)" % st)
        if st == abi.SKIPPED:
            return None, np.zeros(0, EXPLAIN_DTYPE)
        res = types.dense_from_result(out)
        L.v3do_dense_result_free(C.byref(out))
        rec = np.zeros(n.value, EXPLAIN_DTYPE)
        if n.value:
            C.memmove(rec.ctypes.data, recs, n.value * EXPLAIN_DTYPE.itemsize)
        L.v3do_free(recs)
        return res, rec

    def estimate_working_set(self, frames, max_features, descriptor_radius, reference_views,
                             fine_grid):
        L = self.lib
        L.v3do_estimate_working_set.argtypes = [_P(abi.Frame), C.c_uint64, C.c_uint64,
                                                C.c_uint32, C.c_uint64, C.c_int32,
                                                _P(C.c_uint64)]
        L.v3do_estimate_working_set.restype = C.c_int32
        inp = types.Inputs(frames, [], [])
        out = (C.c_uint64 * 12)()
        L.v3do_estimate_working_set(inp.frames, inp.n_frames, int(max_features),
                                    int(descriptor_radius), int(reference_views), int(fine_grid),
                                    out)
        return dict(zip(abi.WORKING_SET_FIELDS, [int(v) for v in out]))

    def estimate_depth_points_with_budget_and_control(self, frames, cameras, sparse_points, focal,
                                                      working_set_budget_bytes, max_features,
                                                      descriptor_radius, profile, control=None):
        L = self.lib
        L.v3do_estimate_depth_points_with_budget.argtypes = [
            _P(abi.Frame), C.c_uint64, _P(abi.Camera), C.c_uint64, _P(C.c_double), C.c_uint64,
            C.c_double, C.c_uint64, C.c_uint64, C.c_uint32, _P(abi.Profile), abi.CANCEL_FN,
            C.c_void_p, _P(abi.DenseResult), _P(C.c_uint64)]
        L.v3do_estimate_depth_points_with_budget.restype = C.c_int32
        inp = types.Inputs(frames, cameras, sparse_points)
        fn, _keep = types.cancel_callback(control)
        out = abi.DenseResult()
        plan = (C.c_uint64 * 16)()
        st = L.v3do_estimate_depth_points_with_budget(
            inp.frames, inp.n_frames, inp.cameras, inp.n_cameras, inp.sparse, inp.n_sparse,
            float(focal), int(working_set_budget_bytes), int(max_features),
            int(descriptor_radius), C.byref(profile), fn, None, C.byref(out), plan)
        if st < 0:
            raise ValueError("oracle rejected the inputs (status %d)" % st)
        res = types.dense_from_result(out, st)
        L.v3do_dense_result_free(C.byref(out))
        v = [int(x) for x in plan]
        return res, {"working_set_estimate": dict(zip(abi.WORKING_SET_FIELDS, v[:12])),
                     "working_set_budget_bytes": v[12], "full_working_set_bytes": v[13],
                     "fine_grid": bool(v[14]), "reference_views": v[15]}

    def estimate_depth_points_limited(self, frames, cameras, sparse_points, focal,
                                      reference_views, fine_grid, profile, control=None):
        inp = types.Inputs(frames, cameras, sparse_points)
        fn, _keep = types.cancel_callback(control)
        out = abi.DenseResult()
        omitted = C.c_int32()
        st = self.lib.v3do_estimate_depth_points_limited(
            inp.frames, inp.n_frames, inp.cameras, inp.n_cameras, inp.sparse, inp.n_sparse,
            float(focal), int(reference_views), int(fine_grid), C.byref(profile), fn, None,
            C.byref(out), C.byref(omitted))
        if st < 0:
            raise ValueError("oracle rejected the inputs (status %d)" % st)
        try:
            return types.dense_from_result(out, st), bool(omitted.value)
        finally:
            self.lib.v3do_dense_result_free(C.byref(out))

    def has_distributed_landmarks(self, frames, cameras, sparse_points, focal, control=None):
        inp = types.Inputs(frames, cameras, sparse_points)
        fn, _keep = types.cancel_callback(control)
        return bool(self.lib.v3do_has_distributed_landmarks(
            inp.frames, inp.n_frames, inp.cameras, inp.n_cameras, inp.sparse, inp.n_sparse,
            float(focal), fn, None))

    def reconstruct_dense_mesh_with_control(self, points, grid_sites, stats, cameras, width,
                                            height, focal, control=None):
        mi = types.MeshInputs(points, grid_sites, stats)
        cams = types.Inputs([], cameras, [])
        fn, _keep = types.cancel_callback(control)
        out = abi.MeshResult()
        self.lib.v3do_reconstruct_dense_mesh_with_control(
            *mi.args(), cams.cameras, cams.n_cameras, int(width), int(height), float(focal),
            fn, None, C.byref(out))
        try:
            return types.mesh_from_result(out)
        finally:
            self.lib.v3do_mesh_result_free(C.byref(out))

    def debug_sweep(self, frames, cameras, sparse_points, focal, fine_grid=False, profile=None):
        inp = types.Inputs(frames, cameras, sparse_points)
        n = C.c_uint64()
        cap = 1 << 22
        buf = (abi.SiteRecord * cap)()
        st = self.lib.v3do_debug_sweep(inp.frames, inp.n_frames, inp.cameras, inp.n_cameras,
                                       inp.sparse, inp.n_sparse, float(focal), int(fine_grid),
                                       C.byref(profile), buf, cap, C.byref(n))
        if st == abi.SKIPPED:
            return None
        if st < 0:
            raise ValueError("oracle rejected the inputs (status %d)" % st)
        return types.site_records(buf, n.value)

    def patch_error(self, profile, ref_cam, src_cam, ref_frame, src_frame, x, y, depth, focal):
        inp = types.Inputs([ref_frame, src_frame], [ref_cam, src_cam], [])
        cost = C.c_double()
        st = self.lib.v3do_patch_error(C.byref(profile), C.byref(inp.cameras[0]),
                                       C.byref(inp.cameras[1]), C.byref(inp.frames[0]),
                                       C.byref(inp.frames[1]), x, y, depth, focal,
                                       C.byref(cost))
        return cost.value if st == 0 else None
