"""Depth-grid verification on the device against the CPU oracle, bit for bit:
every verified sample (position, colour, confidence, site, verifying sources)
and every funnel count, on the reference's own test plane and its rejected
variants, on seeded clips at three grid spacings, on a full-size clip, and on
the edge cases of no references and references without sources.  The mesh
topology figures of the same module against the oracle on the reference's
cases, grid meshes, triangle soups and long chains."""
import numpy as np
import pytest

from v3d import dense

from tests import depth_grid_scenes
from tests.oracle_ffi import Oracle


def _compare(views, refs, sources, stride, rstride, focal):
    g, gf = dense.Context(0).verify_depth_grids(views, refs, sources, stride, rstride, focal)
    o, of = Oracle().verify_depth_grids(views, refs, sources, stride, rstride, focal)
    assert gf == of
    assert len(g) == len(o)
    for a, b in zip(g, o):
        assert a.tobytes() == b.tobytes()
    return g, gf


@pytest.mark.gpu
def test_reference_plane_and_its_rejections():
    frame, other_color, first, second, depth, wrong = depth_grid_scenes.reference_plane()
    views = [(frame, depth, first), (frame, depth, second), (frame, wrong, second),
             (other_color, depth, second), (frame, depth, first)]
    per_ref, funnel = _compare(views, [0], [[1]], 4, 4, 20.0)
    assert len(per_ref[0]) == 20 and funnel["outside_source"] == 4
    per_ref, _ = _compare(views, [0], [[1]], 4, 8, 20.0)
    assert len(per_ref[0]) == 4
    per_ref, funnel = _compare(views, [0, 0, 0, 0], [[2], [3], [4], [1, 2, 3, 4]], 4, 4, 20.0)
    assert [len(p) for p in per_ref] == [0, 0, 0, 20]
    assert (per_ref[3]["source_mask"] == 1).all()


@pytest.mark.gpu
@pytest.mark.parametrize("seed,stride,rstride", [(1, 2, 2), (2, 2, 4), (3, 4, 8), (4, 3, 6)])
def test_seeded_clips(seed, stride, rstride):
    views, refs, sources, focal = depth_grid_scenes.clip_views(seed, stride=stride)
    per_ref, funnel = _compare(views, refs, sources, stride, rstride, focal)
    assert funnel["accepted"] > 0 and funnel["color_disagreement"] >= 0
    assert any(((p["source_mask"] & (p["source_mask"] - 1)) > 0).any() for p in per_ref)


@pytest.mark.gpu
def test_full_size_clip_and_edge_cases():
    views, refs, sources, focal = depth_grid_scenes.clip_views(5, width=640, height=360,
                                                               frames=12, stride=2)
    per_ref, funnel = _compare(views, refs, sources, 2, 4, focal)
    assert funnel["reference_samples"] > 100000
    per_ref, funnel = _compare(views, [], [], 2, 4, focal)
    assert per_ref == [] and all(v == 0 for v in funnel.values())
    per_ref, funnel = _compare(views, [0, 3], [[], [2]], 2, 2, focal)
    assert len(per_ref[0]) == 0 and len(per_ref[1]) > 0


def _tris(a, b, c):
    from v3d import types
    t = np.zeros(len(a), dtype=types.TRIANGLE_DTYPE)
    t["a"], t["b"], t["c"], t["confidence"] = a, b, c, 1.0
    return t


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["reference", "soup", "chain", "grids", "fusion_mesh"])
def test_surface_topology(case):
    rng = np.random.default_rng(11)
    if case == "reference":
        tris, n = _tris([0, 1, 4, 5], [1, 3, 5, 7], [2, 2, 6, 6]), 8
    elif case == "soup":  # many small islands, repeated and degenerate triangles
        n = 200000
        a = rng.integers(0, n, 150000)
        tris = _tris(a, np.minimum(a + rng.integers(0, 3, a.size), n - 1),
                     np.minimum(a + rng.integers(0, 40, a.size), n - 1))
    elif case == "chain":  # one island whose union order builds long parent chains
        n = 300001
        i = np.arange(0, n - 2)[::-1]
        tris = _tris(i, i + 1, i + 2)
    elif case == "grids":
        from tests import fusion_scenes
        pts, tris, _ = fusion_scenes.layered_grids(3, groups=6, nx=120, ny=90, defects=False)
        n = len(pts)
    else:
        from tests import fusion_scenes
        pts, tris, _ = fusion_scenes.layered_grids(4, groups=2, nx=30, ny=20)
        n = len(pts)
        tris = tris[(tris["a"] < n) & (tris["b"] < n) & (tris["c"] < n)]
    g = dense.Context(0).surface_topology(tris, n)
    o = Oracle().surface_topology(tris, n)
    assert g == o
    assert g["islands"] >= 1


@pytest.mark.gpu
def test_entry_points_reject_bad_arguments():
    import ctypes as C
    from v3d import abi, types
    ctx = dense.Context(0)
    lib = ctx.lib
    # a triangle index at the vertex count
    t = np.zeros(1, dtype=types.TRIANGLE_DTYPE)
    t[0] = (0, 1, 3, 1.0, 0)
    out = abi.SurfaceTopology()
    assert lib.v3d_surface_topology_of(ctx.handle, t.ctypes.data, 1, 3, C.byref(out)) == abi.ERR_INVALID_ARGUMENT
    # verified samples beyond the caller's capacity
    frame, _, first, second, depth, _ = depth_grid_scenes.reference_plane()
    views = (abi.DepthView * 2)()
    keep = [np.ascontiguousarray(frame), np.ascontiguousarray(depth)]
    for i, cam in enumerate([first, second]):
        views[i] = abi.DepthView(keep[0].ctypes.data, keep[1].ctypes.data, 24, 16,
                                 abi.Camera(i, (C.c_double * 9)(*np.asarray(cam.rotation).ravel()),
                                            (C.c_double * 3)(*np.asarray(cam.translation))))
    refs = np.zeros(1, dtype=np.uint32)
    src = np.array([1, -1, -1, -1], dtype=np.int32)
    samples = np.zeros(4, dtype=dense.VERIFIED_DTYPE)
    offsets = np.zeros(2, dtype=np.uint64)
    funnel = abi.VerificationFunnel()
    st = lib.v3d_verify_depth_grids(ctx.handle, views, 2, refs.ctypes.data, 1, src.ctypes.data, 4, 4,
                                    20.0, samples.ctypes.data, 4, offsets.ctypes.data, C.byref(funnel))
    assert st == abi.ERR_INVALID_ARGUMENT
    # a meshed spacing that is not a multiple of the grid spacing, a source past the views
    for rstride, s0 in [(6, 1), (4, 2)]:
        src[0] = s0
        st = lib.v3d_verify_depth_grids(ctx.handle, views, 2, refs.ctypes.data, 1, src.ctypes.data,
                                        4, rstride, 20.0, samples.ctypes.data, 4,
                                        offsets.ctypes.data, C.byref(funnel))
        assert st == abi.ERR_INVALID_ARGUMENT
    # the context stays usable after the refused calls
    per_ref, funnel = ctx.verify_depth_grids([(frame, depth, first), (frame, depth, second)], [0],
                                             [[1]], 4, 4, 20.0)
    assert len(per_ref[0]) == 20 and funnel["accepted"] == 20
    # membership of the wrong length
    pts = np.zeros(3, dtype=types.POINT_DTYPE)
    with pytest.raises(ValueError):
        ctx.fuse_mutually_supported_vertices(pts, t, np.zeros(2, dtype=np.int64))


def _compare_surface(views, refs, sources, stride, rstride, focal):
    g = dense.Context(0).mesh_verified_depth_grids(views, refs, sources, stride, rstride, focal)
    o = Oracle().mesh_verified_depth_grids(views, refs, sources, stride, rstride, focal)
    assert g.status == o.status
    assert g.diagnostics == o.diagnostics
    assert g.regions == o.regions
    assert g.points.tobytes() == o.points.tobytes()
    assert g.sites.tobytes() == o.sites.tobytes()
    assert g.triangles.tobytes() == o.triangles.tobytes()
    return g


@pytest.mark.gpu
@pytest.mark.parametrize("seed,stride,rstride", [(1, 2, 2), (2, 2, 4), (3, 4, 8), (4, 3, 6)])
def test_verified_surface_seeded_clips(seed, stride, rstride):
    views, refs, sources, focal = depth_grid_scenes.clip_views(seed, stride=stride)
    g = _compare_surface(views, refs, sources, stride, rstride, focal)
    assert g.status == 0 and len(g.triangles) > 100 and len(g.regions) > 1


@pytest.mark.gpu
def test_verified_surface_full_size_and_edge_cases():
    views, refs, sources, focal = depth_grid_scenes.clip_views(5, width=640, height=360,
                                                               frames=12, stride=2)
    g = _compare_surface(views, refs, sources, 2, 4, focal)
    assert g.diagnostics["meshing"]["exported_triangles"] > 50000
    # no references, a reference without sources, references in another order
    assert _compare_surface(views, [], [], 2, 4, focal).status == 1
    _compare_surface(views, [0, 3], [[], [2]], 2, 4, focal)
    _compare_surface(views, [5, 1, 7], [sources[5], sources[1], sources[7]], 2, 4, focal)
    # the reference plane: all-rejecting sources give no triangle
    frame, _, first, second, depth, wrong = depth_grid_scenes.reference_plane()
    assert _compare_surface([(frame, depth, first), (frame, wrong, second)], [0], [[1]], 4, 4,
                            20.0).status == 1
    _compare_surface([(frame, depth, first), (frame, depth, second)], [0, 1], [[1], [0]], 4, 4,
                     20.0)


@pytest.mark.gpu
def test_verified_surface_sparse_references():
    # references left with fewer than three samples, or none, between meshed ones
    views, refs, sources, focal = depth_grid_scenes.clip_views(6, stride=2, holes=0.995)
    dense_views, _, _, _ = depth_grid_scenes.clip_views(6, stride=2)
    mixed = [dense_views[i] if i % 3 else views[i] for i in range(len(views))]
    g = _compare_surface(mixed, refs, sources, 2, 4, focal)
    assert g.status == 0


@pytest.mark.gpu
def test_verified_surface_rejects_duplicate_frames():
    import ctypes as C
    from v3d import abi
    views, refs, sources, focal = depth_grid_scenes.clip_views(1, stride=2)
    dup = list(views)
    dup[1] = (views[1][0], views[1][1], views[0][2])
    ctx = dense.Context(0)
    st, _ = dense._surface(ctx.lib.v3d_mesh_verified_depth_grids, (ctx.handle,), dup, refs,
                           sources, 2, 4, focal)
    assert st == abi.ERR_INVALID_ARGUMENT
    assert _compare_surface(views, refs, sources, 2, 4, focal).status == 0


@pytest.mark.gpu
def test_verified_surface_refuses_short_capacities():
    import ctypes as C
    from v3d import abi, types
    views, refs, sources, focal = depth_grid_scenes.clip_views(2, stride=2)
    ctx = dense.Context(0)
    arr, keep, r, src = dense._depth_views(views, refs, sources)
    pts = np.zeros(10, dtype=types.POINT_DTYPE)
    sites = np.zeros(10, dtype=types.SITE_DTYPE)
    tris = np.zeros(10, dtype=types.TRIANGLE_DTYPE)
    regs = (abi.VerifiedSurfaceRegion * len(refs))()
    out = abi.VerifiedSurface()
    st = ctx.lib.v3d_mesh_verified_depth_grids(
        ctx.handle, arr, len(views), r.ctypes.data, len(refs), src.ctypes.data, 2, 4, float(focal),
        pts.ctypes.data, sites.ctypes.data, len(pts), tris.ctypes.data, len(tris), regs,
        C.byref(out))
    assert st == abi.ERR_INVALID_ARGUMENT
    full = _compare_surface(views, refs, sources, 2, 4, focal)
    # the refused call reports the sizes it needed
    assert (out.n_points, out.n_triangles) == (len(full.points), len(full.triangles))
