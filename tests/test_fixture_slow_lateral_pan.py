"""The reference's own committed fixture, case "slow-lateral-pan" (`--help/` in
the reference tree; tests/golden/slow_lateral_pan.npz, written by
tests/golden/make_slow_lateral_pan.py): 18 frames of a textured facade, 360x203,
seen by a camera panning sideways.

The dense pass runs with the fixture's true cameras and landmarks sampled
from its true surface, on the three references the reference's own run kept
(5, 17, 16; --help/rust-evidence.json `dense_reference_patches`).

* Golden values of the reference's own run that do not depend on its
  estimated cameras: the grid (stride 4, border 3), the number of sampled
  grid pixels after the contrast gate, and the source frames in order.
* The per-stage dense gate of the reference's benchmark (benchmarks/README.md,
  the `dense` row): per reference, the median relative depth error against
  the true depth through the same grid pixel, after the reference's scale
  bias is removed, at most 1 %; accurate coverage (points within 2 % / sampled
  grid pixels) at least 0.4; scale bias at most 10 %.  This pin is
  statistical.
* On the GPU: the same through the C ABI, bit-identical to the oracle.
"""
import os

import numpy as np
import pytest

from v3d import profiles
from v3d.types import FrameInput, RegisteredCamera

FIXTURE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                       "slow_lateral_pan.npz")
# --help/rust-evidence.json dense_reference_patches: reference -> (sampled pixels, sources)
RUST_RUN = {5: (3904, [4, 6, 3, 7]), 17: (3940, [16, 15, 14, 13]), 16: (3936, [15, 17, 14, 13])}


@pytest.fixture(scope="module")
def fixture():
    z = np.load(FIXTURE)
    frames = [FrameInput(np.concatenate([f, np.full(f.shape[:2] + (1,), 255, np.uint8)], -1))
              for f in z["frames"]]
    cams = [RegisteredCamera(i, z["R"][i], z["t"][i]) for i in range(len(frames))]
    depths = dict(zip((int(r) for r in z["reference_frames"]), z["depths"]))
    return frames, cams, z["sparse"], float(z["focal"]), depths


def dense_gate(result, ref, depths, cams):
    """benchmarks/README.md, `dense` row, as examples/reference_stages/mod.rs
    computes it: ratio = median(depth / truth), error = |depth / ratio - truth| / truth."""
    p = np.stack([result.points[c] for c in "xyz"], -1).astype(np.float64)
    z = (p @ cams[ref].rotation.T + cams[ref].translation)[:, 2]
    truth = depths[ref][result.grid_sites["y"], result.grid_sites["x"]].astype(np.float64)
    ratio = float(np.median(z / truth))
    err = np.abs(z / ratio - truth) / truth
    return {"median_error": float(np.median(err)),
            "accurate_coverage": float((err <= 0.02).sum()) / result.stats["sampled_pixels"],
            "scale_bias": abs(ratio - 1.0)}


def check_reference_run(results, fixture):
    frames, cams, sparse, focal, depths = fixture
    for ref, r in zip(RUST_RUN, results):
        s = r.stats
        assert (s["grid_stride"], s["grid_border"]) == (4, 3)
        assert s["sampled_pixels"] == RUST_RUN[ref][0], ref
        assert s["source_frames"] == RUST_RUN[ref][1], ref
        g = dense_gate(r, ref, depths, cams)
        assert g["median_error"] <= 0.01, (ref, g)
        assert g["accurate_coverage"] >= 0.4, (ref, g)
        assert g["scale_bias"] <= 0.10, (ref, g)


def test_oracle_on_the_reference_fixture(oracle, fixture):
    frames, cams, sparse, focal, _ = fixture
    res = oracle.reconstruct_reference_patches(frames, cams, sparse, focal, list(RUST_RUN),
                                               profiles.reference(), threads=3)
    check_reference_run(res, fixture)


@pytest.mark.gpu
def test_gpu_on_the_reference_fixture(oracle, fixture):
    from v3d import dense
    frames, cams, sparse, focal, _ = fixture
    ctx = dense.Context(0)
    g = ctx.reconstruct_reference_patches(frames, cams, sparse, focal, list(RUST_RUN),
                                          profile=profiles.reference())
    ctx.close()
    o = oracle.reconstruct_reference_patches(frames, cams, sparse, focal, list(RUST_RUN),
                                             profiles.reference(), threads=3)
    check_reference_run(g, fixture)
    for a, b in zip(g, o):
        assert dict(a.stats) == dict(b.stats)
        assert a.points.tobytes() == b.points.tobytes()
        assert a.grid_sites.tobytes() == b.grid_sites.tobytes()
        assert a.point_attributes.tobytes() == b.point_attributes.tobytes()
