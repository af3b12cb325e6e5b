"""The headline profile at the full frame size (640x360, 7x7 ZNCC, 128 planes,
8 views, stride 2), checked through size-independent properties: the
reference's own statistic identities for every patch, ranges and lattice
positions of the outputs, mesh indices, and invariance of every result to the
batch it ran in (and so to the plane chunking the batch got)."""
import numpy as np
import pytest

from v3d import dense, profiles, synth

from tests.test_gpu_parity import check_reference_assertions


def _same(a, b):
    assert dict(a.stats) == dict(b.stats)
    assert a.points.tobytes() == b.points.tobytes()
    assert a.grid_sites.tobytes() == b.grid_sites.tobytes()
    assert a.point_attributes.tobytes() == b.point_attributes.tobytes()


@pytest.mark.gpu
def test_full_frame_properties_and_batch_invariance():
    clip = synth.full_clip(seed=9, n_frames=12)
    frames = clip.frames("f32")
    prof = profiles.zncc(3, 128, 8, 2)
    ctx = dense.Context(0)
    refs = list(range(12))
    whole = ctx.reconstruct_reference_patches_meshed(frames, clip.cameras, clip.sparse,
                                                     clip.focal, refs, profile=prof)
    again = ctx.reconstruct_reference_patches_meshed(frames, clip.cameras, clip.sparse,
                                                     clip.focal, refs, profile=prof)
    halves = (ctx.reconstruct_reference_patches_meshed(frames, clip.cameras, clip.sparse,
                                                       clip.focal, refs[:5], profile=prof) +
              ctx.reconstruct_reference_patches_meshed(frames, clip.cameras, clip.sparse,
                                                       clip.focal, refs[5:], profile=prof))
    total = 0
    for w, a, h in zip(whole, again, halves):
        assert w is not None
        d, m = w
        check_reference_assertions(d)
        _same(d, a[0])
        _same(d, h[0])
        assert m.triangles.tobytes() == a[1].triangles.tobytes() == h[1].triangles.tobytes()
        n = len(d.points)
        total += n
        assert n == d.stats["accepted_points"]
        # outputs in range and on the reference grid
        pts = d.points
        for c in "xyz":
            assert np.isfinite(pts[c]).all()
        assert ((pts["confidence"] >= 0.05) & (pts["confidence"] <= 1.0)).all()
        border, stride = d.stats["grid_border"], d.stats["grid_stride"]
        assert stride == 2 and border == 5
        xs, ys = d.grid_sites["x"].astype(np.int64), d.grid_sites["y"].astype(np.int64)
        assert ((xs - border) % stride == 0).all() and ((ys - border) % stride == 0).all()
        assert (xs < 640 - border).all() and (ys < 360 - border).all()
        assert len(set(zip(xs.tolist(), ys.tolist()))) == n  # one point per site
        att = d.point_attributes
        assert ((att["depth_margin"] >= 0) & (att["depth_margin"] <= 1)).all()
        # mesh indices refer to the patch's points, three distinct corners
        tri = m.triangles
        if len(tri):
            idx = np.stack([tri["a"], tri["b"], tri["c"]], -1)
            assert (idx < n).all()
            assert (idx[:, 0] != idx[:, 1]).all() and (idx[:, 1] != idx[:, 2]).all() and \
                   (idx[:, 0] != idx[:, 2]).all()
            assert m.stats["accepted_triangles"] == len(tri)
    assert total > 50000
