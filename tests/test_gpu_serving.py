"""The device-resident request loop (v3d_server).

Each request's result must be the same alone and in a mix of requests from
other clips, sizes, hypothesis counts and source-view limits: bit for bit,
since every reference is computed from its own inputs.  The loop's
bookkeeping (tickets, timing, batching, shutdown) is checked alongside.
"""
import numpy as np
import pytest

from v3d import abi, dense, profiles, synth


def _specs():
    specs = synth.batched_clip_specs(n_clips=3, seed=21, min_frames=5, max_frames=7,
                                     min_edge=160, max_edge=240)
    return specs


def _with(prof, planes, sources):
    p = profiles.with_precision(prof, prof.precision)
    if planes:
        p.depth_hypotheses = planes
    if sources:
        p.max_source_views = sources
    return p


def _same_dense(a, b):
    assert a.status == b.status
    assert dict(a.stats) == dict(b.stats)
    assert a.points.tobytes() == b.points.tobytes()
    assert a.grid_sites.tobytes() == b.grid_sites.tobytes()
    assert a.point_attributes.tobytes() == b.point_attributes.tobytes()


@pytest.mark.gpu
def test_served_requests_equal_each_request_alone():
    clips = [synth.batched_clip(s) for s in _specs()]
    frames = [c.frames("f32") for c in clips]
    prof = profiles.zncc(2, 32, 4, 2)
    server = dense.Server(slots=2, memory_budget=1 << 30, profile=prof, meshed=True)
    try:
        ids = [server.add_clip(f, c.cameras, c.sparse, c.focal) for f, c in zip(frames, clips)]
        rng = np.random.default_rng(5)
        reqs = []
        for ci, c in enumerate(clips):
            for cam in range(0, len(c.cameras), 2):
                reqs.append((ci, cam, int(rng.choice([0, 24, 40, 56])), int(rng.choice([0, 2, 3]))))
        rng.shuffle(reqs)
        tickets = [server.submit(ids[ci], cam, p, s) for ci, cam, p, s in reqs]
        served = [server.wait(t) for t in tickets]
        ctx = dense.Context(0)
        batched = 0
        for (ci, cam, p, s), out in zip(reqs, served):
            c = clips[ci]
            alone = ctx.reconstruct_reference_patches_meshed(
                frames[ci], c.cameras, c.sparse, c.focal, [cam], profile=_with(prof, p, s))[0]
            assert (out.result is None) == (alone is None)
            t = out.timing
            assert 0.0 <= t["queue_ms"] <= t["total_ms"] and 0.0 <= t["service_ms"] <= t["total_ms"]
            assert t["batch_requests"] >= 1
            batched = max(batched, t["batch_requests"])
            if alone is None:
                continue
            _same_dense(out.result[0], alone[0])
            assert out.result[1].triangles.tobytes() == alone[1].triangles.tobytes()
            assert dict(out.result[1].stats) == dict(alone[1].stats)
            if alone[0].stats["attempted"]:
                assert t["plane_view_units"] > 0
        assert batched > 1  # requests queued together ran as one device batch
        with pytest.raises(dense.V3DError):
            server.wait(tickets[0])  # a collected ticket is spent
    finally:
        server.close()


@pytest.mark.gpu
def test_server_shutdown_with_queued_requests():
    clip = synth.batched_clip(_specs()[0])
    server = dense.Server(slots=1, max_batch_requests=1, profile=profiles.zncc(2, 32, 4, 2))
    cid = server.add_clip(clip.frames("f32"), clip.cameras, clip.sparse, clip.focal)
    tickets = [server.submit(cid, i % len(clip.cameras)) for i in range(12)]
    first = server.wait(tickets[0])
    assert first.status in (abi.OK, abi.SKIPPED)
    # the remaining requests are either done or dropped; closing must not hang or leak
    server.close()
    with pytest.raises(Exception):
        server.submit(cid, 0)
