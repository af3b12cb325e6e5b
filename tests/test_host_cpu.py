"""Host-side logic of the library that runs without a GPU, against the oracle."""
import numpy as np

from tests import fixtures
from v3d import dense
from v3d.types import FrameInput, RegisteredCamera


def test_has_distributed_landmarks_matches_oracle(oracle):
    # dense.rs:1114-1136: 16 landmark pairs spread over 4x4 tiles vs a row of 32
    w = h = 240
    f = 200.0
    frames = [FrameInput(np.full((h, w, 4), 128, np.uint8))] * 2
    cams = [fixtures.camera(0, 0.0), fixtures.camera(1, 0.2)]

    def world(x, y):
        return ((x - 120.0) / f * 4.0, (y - 120.0) / f * 4.0, 4.0)

    distributed = []
    for y in (30.0, 90.0, 150.0, 210.0):
        for x in (30.0, 90.0, 150.0, 210.0):
            distributed += [world(x, y), world(x + 2.0, y)]
    concentrated = [world(90.0 + i, 90.0) for i in range(len(distributed))]
    for sparse, expected in ((distributed, True), (concentrated, False)):
        got = dense.has_distributed_landmarks(frames, cams, sparse, f)
        assert got == expected
        assert got == oracle.has_distributed_landmarks(frames, cams, sparse, f)


def test_landmark_scan_cancellation_polls_like_the_reference(oracle):
    # dense.rs:1089-1112: canceled on the third 256-landmark chunk
    frames = [FrameInput(np.zeros((240, 240, 4), np.uint8))]
    pts = np.tile([0.0, 0.0, 4.0], (4096, 1))
    for impl in (dense.has_distributed_landmarks, oracle.has_distributed_landmarks):
        polls = []

        def control():
            polls.append(1)
            return len(polls) == 3

        assert not impl(frames, [fixtures.camera(0, 0.0)], pts, 200.0, control=control)
        assert len(polls) == 3
