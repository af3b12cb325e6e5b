"""The planner's landmark scans of many clips in one device pass
(v3d_plan_clips) against the CPU oracle's reference_candidate_order
(dense.rs:620-672) and has_distributed_landmarks (dense.rs:165-213), clip by
clip: uneven clips, cameras whose frame is missing, a clip with too few
landmarks, and no clips."""
import numpy as np
import pytest

from v3d import dense, synth
from v3d.types import RegisteredCamera

from tests.oracle_ffi import Oracle


def _clips():
    specs = synth.batched_clip_specs(5, seed=8, min_frames=6, max_frames=14, min_edge=160,
                                     max_edge=320)
    out = []
    for spec in specs:
        c = synth.batched_clip(spec)
        out.append({"frames": c.frames("f32"), "cameras": c.cameras, "sparse_points": c.sparse,
                     "focal": c.focal})
    # a camera whose frame index is past the frames, and a clip of 5 landmarks
    extra = dict(out[0])
    cams = list(extra["cameras"])
    cams.append(RegisteredCamera(len(extra["frames"]) + 3, cams[0].rotation, cams[0].translation))
    extra["cameras"] = cams
    out.append(extra)
    few = dict(out[1])
    few["sparse_points"] = np.asarray(few["sparse_points"])[:5]
    out.append(few)
    return out


@pytest.mark.gpu
def test_plan_clips_equals_the_oracle_clip_by_clip():
    clips = _clips()
    plans = dense.Context(0).plan_clips(clips)
    o = Oracle()
    assert len(plans) == len(clips)
    for clip, (order, distributed) in zip(clips, plans):
        assert order == o.reference_candidate_order(clip["frames"], clip["cameras"],
                                                    clip["sparse_points"], clip["focal"])
        assert distributed == o.has_distributed_landmarks(clip["frames"], clip["cameras"],
                                                          clip["sparse_points"], clip["focal"])
    assert any(len(order) > 0 for order, _ in plans)
    assert plans[-1][0] == []
    assert dense.Context(0).plan_clips([]) == []
