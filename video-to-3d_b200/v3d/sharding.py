"""References of one call spread over the ranks of a process group.

The dense pass reconstructs every reference from its own frames, cameras and
landmarks (dense.rs:246-249 runs the references of a clip independently), so a
clip shards by reference with no exchange step: rank r takes the caller's
references r, r + N, r + 2N, ..., runs them as one device batch on its own GPU,
and the per-reference results travel back to one rank in the caller's order,
the order in which dense.rs:842-870 concatenates patches.  Frames and cameras
are replicated (every rank is handed the whole clip); nothing on the data path
crosses GPUs, the gather carries host results only.
"""


def references_of_rank(camera_indices, rank, world):
    """Round-robin share of `camera_indices` for `rank` of `world` (order kept)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank %r outside a world of %r" % (rank, world))
    return list(camera_indices)[rank::world]


def merge_rank_results(per_rank, n):
    """Inverse of references_of_rank: per_rank[r][j] is reference r + j * world."""
    world = len(per_rank)
    out = [None] * n
    for r, results in enumerate(per_rank):
        expect = len(range(r, n, world))
        if len(results) != expect:
            raise ValueError("rank %d returned %d results for %d references"
                             % (r, len(results), expect))
        for j, res in enumerate(results):
            out[r + j * world] = res
    return out


def reconstruct_reference_patches_sharded(run, camera_indices, group=None, dst=0):
    """Runs `run(indices) -> [result per index]` on this rank's share and gathers
    every rank's results on `dst`, in the order of `camera_indices`.

    `run` is typically a bound Context.reconstruct_reference_patches (or the
    _meshed variant) with the clip's frames, cameras and profile filled in.
    Returns the full list on `dst` and None on the other ranks.  Every rank
    takes the same collective step, also when its share is empty."""
    import torch.distributed as dist

    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    mine = references_of_rank(camera_indices, rank, world)
    local = run(mine) if mine else []
    gathered = [None] * world if rank == dst else None
    dist.gather_object(local, gathered, dst=dst, group=group)
    if rank != dst:
        return None
    return merge_rank_results(gathered, len(camera_indices))
