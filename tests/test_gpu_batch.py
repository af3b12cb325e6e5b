"""Many clips of uneven size in one device batch (v3d_reconstruct_clips).

Per clip the batched results must equal the single-clip call with that clip's
inputs and profile overrides: bit for bit, since every reference is computed
from its own inputs whatever else shares the batch.
"""
import numpy as np
import pytest

from v3d import abi, dense, profiles, synth


def _small_specs():
    specs = synth.batched_clip_specs(n_clips=3, seed=11, min_frames=5, max_frames=8,
                                     min_edge=160, max_edge=256)
    for s, (planes, sources) in zip(specs, [(32, 2), (48, 3), (40, 4)]):
        s["planes"], s["sources"] = planes, sources
    return specs


def _same(a, b):
    assert a.status == b.status
    assert dict(a.stats) == dict(b.stats)
    assert a.points.tobytes() == b.points.tobytes()
    assert a.grid_sites.tobytes() == b.grid_sites.tobytes()
    assert a.point_attributes.tobytes() == b.point_attributes.tobytes()


def _with(prof, planes, sources):
    p = profiles.with_precision(prof, prof.precision)
    p.depth_hypotheses = planes
    p.max_source_views = sources
    return p


@pytest.mark.gpu
@pytest.mark.parametrize("storage", ["f32", "f16"])
def test_uneven_clips_batch_equals_each_clip_alone(storage):
    specs = _small_specs()
    clips = [synth.batched_clip(s) for s in specs]
    prof = profiles.zncc(2, 32, 4, 2)
    ctx = dense.Context(0)
    reqs = []
    for s, c in zip(specs, clips):
        reqs.append(dict(frames=c.frames(storage), cameras=c.cameras, sparse_points=c.sparse,
                         focal=c.focal, camera_indices=list(range(len(c.cameras)))[::2],
                         depth_hypotheses=s["planes"], max_source_views=s["sources"]))
    batched = ctx.reconstruct_clips(reqs, profile=prof, meshed=True)
    total = 0
    for r, s, got in zip(reqs, specs, batched):
        alone = ctx.reconstruct_reference_patches_meshed(
            r["frames"], r["cameras"], r["sparse_points"], r["focal"], r["camera_indices"],
            profile=_with(prof, s["planes"], s["sources"]))
        assert len(got) == len(alone)
        for g, a in zip(got, alone):
            assert (g is None) == (a is None)
            if g is None:
                continue
            _same(g[0], a[0])
            assert g[1].triangles.tobytes() == a[1].triangles.tobytes()
            assert dict(g[1].stats) == dict(a[1].stats)
            total += len(g[0].points)
            assert g[0].stats["depth_hypotheses"] == s["planes"]
    assert total > 0


@pytest.mark.gpu
def test_uneven_clips_exact_policy_matches_the_oracle(oracle):
    specs = _small_specs()
    clips = [synth.batched_clip(s) for s in specs]
    prof = profiles.reference()
    ctx = dense.Context(0)
    reqs = []
    for s, c in zip(specs, clips):
        reqs.append(dict(frames=c.frames("rgba8"), cameras=c.cameras, sparse_points=c.sparse,
                         focal=c.focal, camera_indices=[0, len(c.cameras) // 2],
                         depth_hypotheses=min(s["planes"], 32), max_source_views=min(s["sources"], 4)))
    batched = ctx.reconstruct_clips(reqs, profile=prof)
    for r, got in zip(reqs, batched):
        want = oracle.reconstruct_reference_patches(
            r["frames"], r["cameras"], r["sparse_points"], r["focal"], r["camera_indices"],
            _with(prof, r["depth_hypotheses"], r["max_source_views"]))
        for g, w in zip(got, want):
            assert (g is None) == (w is None)
            if g is not None:
                _same(g, w)


@pytest.mark.gpu
def test_sweep_chunk_tuning_never_changes_results():
    """The tiled sweep's tile shape (32x8 or 16x16) and plane chunking are tuned
    on live calls; whatever plan a call runs with, its results are the same bit
    for bit."""
    clip = synth.make_clip(232, 130, 5, 15.0, 1.2, 31, landmark_cameras=[2],
                           landmarks_per_camera=400)
    frames = clip.frames("f32")
    prof = profiles.zncc(2, 48, 4, 2)
    ctx = dense.Context(0)
    outs, plans = [], []
    for _ in range(8):
        outs.append(ctx.reconstruct_reference_patches(frames, clip.cameras, clip.sparse,
                                                      clip.focal, [2], profile=prof)[0])
        info = ctx.last_run_info()
        plans.append((info["sweep_tile_x"], info["sweep_chunks"]))
    assert len(outs[0].points) > 0
    for o in outs[1:]:
        _same(o, outs[0])
    assert {t for t, _ in plans} == {16, 32}     # both tiles were tried
    assert len({c for _, c in plans}) >= 2       # and several chunk counts
    assert plans[-1] == plans[-2] and plans[-1][1] > 1  # one plan was kept
