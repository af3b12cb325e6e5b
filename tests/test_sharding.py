"""Sharding a clip's references over ranks (v3d.sharding), on CPU.

The device batch of each rank is stood in for by the CPU oracle, so the test
checks the host side of the multi-GPU path: the round-robin split, the gather
of host results and the restored caller order, on two `gloo` ranks.
"""
import datetime
import multiprocessing as mp
import socket

import numpy as np
import pytest

from v3d import sharding

REFS = [4, 0, 3, 1, 2]  # caller order, deliberately not sorted


def test_round_robin_split_and_merge_are_inverse():
    idx = list(range(11))
    for world in (1, 2, 3, 4, 16):
        shares = [sharding.references_of_rank(idx, r, world) for r in range(world)]
        assert sorted(sum(shares, [])) == idx
        assert sharding.merge_rank_results(shares, len(idx)) == idx
    with pytest.raises(ValueError):
        sharding.references_of_rank(idx, 2, 2)
    with pytest.raises(ValueError):
        sharding.merge_rank_results([[0, 2], [1]], 5)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _same(a, b):
    if (a is None) != (b is None):
        return False
    if a is None:
        return True
    return (a.status == b.status and dict(a.stats) == dict(b.stats)
            and a.points.tobytes() == b.points.tobytes()
            and a.grid_sites.tobytes() == b.grid_sites.tobytes()
            and a.point_attributes.tobytes() == b.point_attributes.tobytes())


def _rank_main(rank, world, port, refs, queue):
    import torch.distributed as dist

    from tests import oracle_ffi
    from v3d import profiles, synth

    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        clip = synth.plain_small_clip(seed=7, width=200, height=120)
        frames = clip.frames("rgba8")
        orc = oracle_ffi.Oracle()
        prof = profiles.reference()
        shares = []

        def run(idx):
            shares.append(list(idx))
            return orc.reconstruct_reference_patches(frames, clip.cameras, clip.sparse,
                                                     clip.focal, idx, prof)

        got = sharding.reconstruct_reference_patches_sharded(run, refs)
        if rank == 0:
            want = orc.reconstruct_reference_patches(frames, clip.cameras, clip.sparse,
                                                     clip.focal, refs, prof)
            ok = len(got) == len(want) and all(_same(a, b) for a, b in zip(got, want))
            points = int(sum(len(r.points) for r in want if r is not None))
            queue.put(("rank0", ok, points, shares))
        else:
            queue.put(("rank%d" % rank, got is None, 0, shares))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,refs", [(2, REFS), (2, [3]), (3, REFS)])
def test_sharded_patches_match_one_unsharded_call(oracle, world, refs):
    ctx = mp.get_context("spawn")
    queue = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, refs, queue))
             for r in range(world)]
    for p in procs:
        p.start()
    try:
        out = {}
        for _ in range(world):
            name, ok, points, shares = queue.get(timeout=240)
            out[name] = (ok, points, shares)
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    ok, points, shares = out["rank0"]
    assert ok
    if len(refs) > 1:
        assert points > 0
    for r in range(world):
        mine = out["rank%d" % r][2]
        want = refs[r::world]
        assert mine == ([want] if want else [])
        assert out["rank%d" % r][0]
    assert np.isfinite(points)


@pytest.mark.gpu
def test_sharded_device_results_survive_the_gather(oracle):
    """One rank on the GPU: the zero-copy device results pickle through the
    gather and equal the unsharded device call."""
    import torch.distributed as dist

    from v3d import dense, profiles, synth

    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % _free_port(), rank=0,
                            world_size=1, timeout=datetime.timedelta(seconds=60))
    try:
        clip = synth.plain_small_clip(seed=7, width=200, height=120)
        frames = clip.frames("rgba8")
        ctx = dense.Context(0)
        prof = profiles.reference()

        def run(idx):
            return ctx.reconstruct_reference_patches(frames, clip.cameras, clip.sparse,
                                                     clip.focal, idx, profile=prof)

        got = sharding.reconstruct_reference_patches_sharded(run, REFS)
        want = run(REFS)
        assert all(_same(a, b) for a, b in zip(got, want))
        assert sum(len(r.points) for r in got if r is not None) > 0
    finally:
        dist.destroy_process_group()
