"""The allocation-free mesh entry point against the allocating one.

v3d_mesh_patch_device_noalloc serves callers that cannot allocate GPU
memory — a host that hands the library pointers into its own pre-allocated
pool, or a serving loop that must never call cudaMalloc because it can
synchronise the whole device.  The test allocates the device buffers itself
(as such a caller's pool would), calls the entry point twice in a row through
the C ABI and checks that each call reproduces, triangle for triangle and
counter for counter, what the allocating v3d_reconstruct_dense_mesh_with_control
returns for the same patch.  It runs last so that a failure here leaves every
other test already run.
"""
import ctypes as C

import numpy as np
import pytest

from v3d import abi, profiles, synth

pytestmark = pytest.mark.gpu


class MeshCounts(C.Structure):
    _fields_ = [("grid_vertices", C.c_uint64), ("candidate_cells", C.c_uint64),
                ("candidate_triangles", C.c_uint64), ("accepted_triangles", C.c_uint64),
                ("rejected_discontinuities", C.c_uint64), ("rejected_degenerate", C.c_uint64)]


def _slots(w, h, border, stride):
    gw = -(-(w - 2 * border) // stride)
    gh = -(-(h - 2 * border) // stride)
    return 2 * (gw + 1) * (gh + 1) + max(gw - 2, 0) * gh + gw * max(gh - 2, 0)


def test_noalloc_mesh_matches_the_allocating_entry_point(oracle):
    import torch
    from v3d import dense

    lib = dense.library()
    fn = lib.v3d_mesh_patch_device_noalloc
    fn.argtypes = [C.c_void_p, C.c_void_p, C.c_uint64, C.POINTER(abi.Camera), C.c_uint32,
                   C.c_uint32, C.c_uint32, C.c_uint64, C.c_double, C.c_void_p, C.c_uint64,
                   C.c_void_p, C.c_void_p]
    fn.restype = C.c_int32

    clip = synth.make_clip(192, 112, 5, 15.0, 1.2, seed=31, noise_sigma=0.01,
                           landmark_cameras=[2], landmarks_per_camera=300)
    d = oracle.reconstruct_reference_patches(clip.frames("rgba8"), clip.cameras, clip.sparse,
                                             clip.focal, [2], profiles.reference())[0]
    assert len(d.points) > 50
    ref_cam = clip.cameras[d.stats["reference_frame"]]
    ctx = dense.Context(0)
    expected = ctx.reconstruct_dense_mesh_with_control(d.points, d.grid_sites, d.stats,
                                                       clip.cameras, clip.width, clip.height,
                                                       clip.focal)
    ctx.close()
    assert expected.stats["accepted_triangles"] > 0

    w, h = clip.width, clip.height
    border, stride = d.stats["grid_border"], d.stats["grid_stride"]
    cap = _slots(w, h, border, stride)
    dev = torch.device("cuda", 0)
    pts = torch.from_numpy(d.points.view(np.uint8).copy()).to(dev)
    sites = torch.from_numpy(d.grid_sites.view(np.uint8).copy()).to(dev)
    tris = torch.empty(cap * C.sizeof(abi.MeshTriangle), dtype=torch.uint8, device=dev)
    counts = torch.empty(C.sizeof(MeshCounts), dtype=torch.uint8, device=dev)
    cam = abi.Camera(0, (C.c_double * 9)(*np.asarray(ref_cam.rotation).ravel()),
                     (C.c_double * 3)(*np.asarray(ref_cam.translation)))
    stream = torch.cuda.current_stream(dev)

    for call in range(2):
        tris.fill_(0xAB)
        counts.fill_(0xCD)
        st = fn(pts.data_ptr(), sites.data_ptr(), len(d.points), C.byref(cam), w, h, border,
                stride, clip.focal, tris.data_ptr(), cap, counts.data_ptr(), stream.cuda_stream)
        assert st == abi.OK, (call, st)
        stream.synchronize()
        c = MeshCounts.from_buffer_copy(counts.cpu().numpy().tobytes())
        s = expected.stats
        assert c.grid_vertices == s["grid_vertices"], call
        assert c.candidate_cells == s["candidate_cells"], call
        assert c.candidate_triangles == s["candidate_triangles"], call
        assert c.accepted_triangles == s["accepted_triangles"], call
        assert c.rejected_discontinuities == s["rejected_discontinuities"], call
        assert c.rejected_degenerate == s["rejected_degenerate"], call
        n = c.accepted_triangles * C.sizeof(abi.MeshTriangle)
        assert tris[:n].cpu().numpy().tobytes() == expected.triangles.tobytes(), call

    # a lattice beyond the fixed working array is refused before any work is enqueued
    counts.fill_(0xCD)
    big = fn(pts.data_ptr(), sites.data_ptr(), len(d.points), C.byref(cam), 8192, 8192, 3, 1,
             clip.focal, tris.data_ptr(), 1 << 40, counts.data_ptr(), stream.cuda_stream)
    assert big == abi.ERR_INVALID_ARGUMENT
    stream.synchronize()
    assert bytes(counts.cpu().numpy()) == b"\xcd" * C.sizeof(MeshCounts)
