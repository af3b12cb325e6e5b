"""Seeded external-depth inputs for the depth-grid verification tests: the
synthetic clip's true depth sampled on the grid, with multiplicative noise,
holes and missing surfaces, and RGBA frames whose channels some views tint so
that the colour gate has work; plus the reference's own test plane."""
import numpy as np

from v3d import synth
from v3d.types import RegisteredCamera


def reference_plane():
    """colmap_surface.rs:633-668: a 24x16 frame of grey 100, depth 5 everywhere,
    the second camera one unit to the side; also the other colour and the wrong
    depth the test swaps in."""
    frame = np.full((16, 24, 4), 100, dtype=np.uint8)
    other_color = np.full((16, 24, 4), 200, dtype=np.uint8)
    first = RegisteredCamera(0, np.eye(3), np.zeros(3))
    second = RegisteredCamera(1, np.eye(3), np.array([-1.0, 0.0, 0.0]))
    depth = np.full((4, 6), 5.0, dtype=np.float32)
    wrong = np.full((4, 6), 8.0, dtype=np.float32)
    return frame, other_color, first, second, depth, wrong


def clip_views(seed, width=192, height=112, frames=8, stride=2, noise=0.008, holes=0.05,
               tint_every=3):
    clip = synth.make_clip(width, height, frames, 20.0, 1.5, seed=seed, noise_sigma=0.01)
    rng = np.random.default_rng(seed + 100)
    views = []
    for k, (img, depth, cam) in enumerate(zip(clip.images, clip.depths, clip.cameras)):
        rgba = synth.to_rgba8(img).copy()
        if tint_every and k % tint_every == 1:
            rgba[..., 0] = np.clip(rgba[..., 0].astype(np.int32) + 70, 0, 255).astype(np.uint8)
            rgba[..., 2] = np.clip(rgba[..., 2].astype(np.int32) - 50, 0, 255).astype(np.uint8)
        g = depth[::stride, ::stride].astype(np.float64)
        g = g * (1.0 + rng.normal(0.0, noise, g.shape))
        g[~np.isfinite(g)] = 0.0
        g[rng.random(g.shape) < holes] = 0.0
        views.append((rgba, g.astype(np.float32), cam))
    refs = list(range(frames))
    sources = []
    for r in refs:
        near = sorted((abs(s - r), s) for s in refs if s != r)
        sources.append([s for _, s in near[: 1 + (r % 4)]])
    return views, refs, sources, clip.focal
