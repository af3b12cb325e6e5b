"""Writes tests/golden/slow_lateral_pan.npz from the reference's committed
fixture `--help/` (case "slow-lateral-pan", generated by
crates/video-to-3d-core/examples/reference_fixture.rs): the 18 sampled frames
(360x203 RGB), their true cameras (truth/truth.json: x_camera = R x_world + t,
R row-major), the true depth of the reference frames used by the tests
(truth/depth-NN.pfm, rows stored bottom to top), and sparse landmarks sampled
from the true surface at a fixed pixel lattice of every frame (the way the
reference's own dense tests build landmarks, dense_legacy.rs:1226-1238).

Run once in a checkout that has the reference at REFERENCE (default
/root/reference); the GPU box has no reference tree, so the tests read the
npz this writes.
"""
import json
import os
import sys

import numpy as np

REFERENCE = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
FIXTURE = os.path.join(REFERENCE, "--help")
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "slow_lateral_pan.npz")
REFERENCE_FRAMES = (5, 16, 17)  # the references the reference's own run kept (stage-report.json)


def read_ppm(path):
    with open(path, "rb") as f:
        data = f.read()
    parts, pos = [], 0
    while len(parts) < 4:  # magic, width, height, maxval
        while data[pos:pos + 1].isspace():
            pos += 1
        end = pos
        while not data[end:end + 1].isspace():
            end += 1
        parts.append(data[pos:end])
        pos = end
    assert parts[0] == b"P6" and parts[3] == b"255"
    w, h = int(parts[1]), int(parts[2])
    return np.frombuffer(data[pos + 1:pos + 1 + w * h * 3], np.uint8).reshape(h, w, 3)


def read_pfm(path):
    with open(path, "rb") as f:
        assert f.readline().strip() == b"Pf"
        w, h = map(int, f.readline().split())
        scale = float(f.readline())
        d = np.frombuffer(f.read(w * h * 4), "<f4" if scale < 0 else ">f4").reshape(h, w)
    return d[::-1].astype(np.float32)  # rows top to bottom


def main():
    truth = json.load(open(os.path.join(FIXTURE, "truth", "truth.json")))
    intr = truth["intrinsics"]
    w, h, focal = intr["width"], intr["height"], intr["fx"]
    frames, R, t, depths = [], [], [], {}
    sparse = []
    for fr in truth["frames"]:
        frames.append(read_ppm(os.path.join(FIXTURE, fr["image"])))
        Rm = np.array(fr["rotation_world_to_camera"], np.float64).reshape(3, 3)
        tv = np.array(fr["translation"], np.float64)
        R.append(Rm)
        t.append(tv)
        depth = read_pfm(os.path.join(FIXTURE, fr["depth"]))
        if fr["index"] in REFERENCE_FRAMES:
            depths[fr["index"]] = depth
        # landmarks: the true surface under a lattice of pixels, in world space
        for y in range(20, h - 20, 30):
            for x in range(20, w - 20, 40):
                z = float(depth[y, x])
                cam = np.array([(x - w * 0.5) / focal * z, (y - h * 0.5) / focal * z, z])
                sparse.append(Rm.T @ (cam - tv))
    np.savez_compressed(
        OUT, frames=np.stack(frames), R=np.stack(R), t=np.stack(t), focal=focal,
        sparse=np.array(sparse, np.float64), reference_frames=np.array(REFERENCE_FRAMES),
        depths=np.stack([depths[i] for i in REFERENCE_FRAMES]))
    print(OUT, os.path.getsize(OUT))


if __name__ == "__main__":
    main()
