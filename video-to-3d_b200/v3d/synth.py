"""Seeded synthetic multi-view scenes for the dense plane sweep.

A scene is a set of textured planes (and boxes made of planes) ray-cast from
pinhole cameras that follow a horizontal arc.  Textures are 4-octave value
noise in [0, 1] whose lattice values come from a SplitMix64-style integer
finaliser (the published SplitMix64 mixing constants), so every image is a
pure function of the seed.  Pixel x, y samples the ray through image
coordinate (x, y) with the principal point at (w/2, h/2) and a shared focal
length, the camera model of dense_legacy.rs:996-1029.

Sparse landmarks are true-surface points under seeded visible pixels, the way
dense_legacy.rs:1226-1238 builds its test landmarks from the plane.
"""
from dataclasses import dataclass, field
from typing import List

import numpy as np

from .types import FrameInput, RegisteredCamera

_M1 = np.uint64(0x9E3779B97F4A7C15)
_M2 = np.uint64(0xC2B2AE3D27D4EB4F)
_M3 = np.uint64(0x165667B19E3779F9)
_F1 = np.uint64(0xBF58476D1CE4E5B9)
_F2 = np.uint64(0x94D049BB133111EB)


def _lattice(ix, iy, salt, seed):
    """Hash integer lattice coordinates to [0, 1)."""
    with np.errstate(over="ignore"):
        z = (np.uint64(seed) ^ (ix.astype(np.int64).view(np.uint64) * _M1)
             ^ (iy.astype(np.int64).view(np.uint64) * _M2) ^ (np.uint64(salt) * _M3))
        z = (z ^ (z >> np.uint64(30))) * _F1
        z = (z ^ (z >> np.uint64(27))) * _F2
        z = z ^ (z >> np.uint64(31))
    return (z >> np.uint64(11)).astype(np.float64) / float(1 << 53)


def _smooth(t):
    return t * t * (3.0 - 2.0 * t)


def value_noise(u, v, cell, salt, seed):
    gx = u / cell
    gy = v / cell
    ix = np.floor(gx)
    iy = np.floor(gy)
    fx = _smooth(gx - ix)
    fy = _smooth(gy - iy)
    ix = ix.astype(np.int64)
    iy = iy.astype(np.int64)
    top = _lattice(ix, iy, salt, seed) * (1 - fx) + _lattice(ix + 1, iy, salt, seed) * fx
    bot = _lattice(ix, iy + 1, salt, seed) * (1 - fx) + _lattice(ix + 1, iy + 1, salt, seed) * fx
    return top * (1 - fy) + bot * fy


def texture(u, v, plane_id, seed, base_cell=0.4, octaves=4, contrast=1.0):
    acc = np.zeros_like(u)
    norm = 0.0
    amp = 1.0
    cell = base_cell
    for o in range(octaves):
        acc += amp * value_noise(u, v, cell, plane_id * 16 + o, seed)
        norm += amp
        amp *= 0.5
        cell *= 0.5
    t = acc / norm
    # stretch the narrow distribution of summed noise to fill [0, 1]
    t = np.clip(0.5 + (t - 0.5) * 2.2 * contrast, 0.0, 1.0)
    return t


@dataclass
class Plane:
    point: np.ndarray
    normal: np.ndarray
    u_axis: np.ndarray
    v_axis: np.ndarray
    plane_id: int
    lo: np.ndarray = field(default_factory=lambda: np.full(3, -np.inf))
    hi: np.ndarray = field(default_factory=lambda: np.full(3, np.inf))
    contrast: float = 1.0


def _plane(point, normal, plane_id, lo=None, hi=None, contrast=1.0):
    n = np.asarray(normal, float)
    n = n / np.linalg.norm(n)
    a = np.array([0.0, 1.0, 0.0]) if abs(n[1]) < 0.9 else np.array([1.0, 0.0, 0.0])
    u = np.cross(a, n)
    u /= np.linalg.norm(u)
    v = np.cross(n, u)
    return Plane(np.asarray(point, float), n, u, v, plane_id,
                 np.full(3, -np.inf) if lo is None else np.asarray(lo, float),
                 np.full(3, np.inf) if hi is None else np.asarray(hi, float), contrast)


def _box(center, size, first_id, contrast=1.0):
    c = np.asarray(center, float)
    s = np.asarray(size, float) * 0.5
    lo, hi = c - s - 1e-9, c + s + 1e-9
    planes = []
    for axis in range(3):
        for sign in (-1.0, 1.0):
            n = np.zeros(3)
            n[axis] = sign
            p = c.copy()
            p[axis] += sign * s[axis]
            planes.append(_plane(p, n, first_id + len(planes), lo, hi, contrast))
    return planes


@dataclass
class Scene:
    planes: List[Plane]
    seed: int


def room_scene(seed, extra_planes=0, boxes=0, low_texture_fraction=0.0):
    """Floor plus two walls at depths 2-6 (the plain sweep scene), optionally
    with extra slanted planes, textured boxes and low-texture patches."""
    rng = np.random.default_rng(seed + 17)
    planes = [
        _plane([0.0, 0.0, 6.0], [0.0, 0.0, -1.0], 0),             # back wall
        _plane([-1.0, 0.0, 2.0], [0.95, 0.0, -0.31], 1),          # left wall, slanted
        _plane([0.0, 0.9, 0.0], [0.0, -1.0, 0.0], 2),             # floor (y down)
        _plane([0.7, 0.0, 2.0], [-0.9, 0.0, -0.44], 3,            # right wall, near
               lo=[-np.inf, -np.inf, 1.9]),
    ]
    for k in range(extra_planes):
        z = rng.uniform(2.5, 5.5)
        n = np.array([rng.uniform(-0.4, 0.4), rng.uniform(-0.3, 0.3), -1.0])
        x0, y0 = rng.uniform(-1.5, 1.5), rng.uniform(-0.8, 0.6)
        half = rng.uniform(0.3, 0.8)
        planes.append(_plane([x0, y0, z], n, 4 + k, lo=[x0 - half, y0 - half, -np.inf],
                             hi=[x0 + half, y0 + half, np.inf]))
    nid = 4 + extra_planes
    for b in range(boxes):
        c = [rng.uniform(-1.5, 1.5), rng.uniform(0.2, 0.6), rng.uniform(2.8, 5.0)]
        sz = [rng.uniform(0.3, 0.7), rng.uniform(0.3, 0.7), rng.uniform(0.3, 0.7)]
        planes += _box(c, sz, nid)
        nid += 6
    if low_texture_fraction > 0:
        for p in planes:
            if rng.uniform() < low_texture_fraction * 4:
                p.contrast = 0.08
    return Scene(planes, seed)


def look_rotation(forward, up=(0.0, -1.0, 0.0)):
    """World-to-camera rotation whose +z axis is `forward` and +y points down."""
    f = np.asarray(forward, float)
    f = f / np.linalg.norm(f)
    r = np.cross(np.asarray(up, float), f)
    r /= np.linalg.norm(r)
    d = np.cross(f, r)
    return np.stack([r, d, f])


def _yaw(deg):
    a = np.radians(deg)
    return np.array([[np.cos(a), 0, np.sin(a)], [0, 1, 0], [-np.sin(a), 0, np.cos(a)]])


def _pitch(deg):
    a = np.radians(deg)
    return np.array([[1, 0, 0], [0, np.cos(a), -np.sin(a)], [0, np.sin(a), np.cos(a)]])


def arc_cameras(n, arc_deg, pivot_distance, jitter_deg=0.0, seed=0):
    """`n` cameras on a horizontal arc of `arc_deg` degrees around a vertical
    axis through the pivot (0, 0, pivot_distance); each looks at the pivot,
    then turns by seeded yaw/pitch jitter of up to ±jitter_deg."""
    rng = np.random.default_rng(seed + 101)
    cams = []
    for i in range(n):
        phi = np.radians(-arc_deg / 2 + arc_deg * i / max(n - 1, 1))
        center = np.array([pivot_distance * np.sin(phi), 0.0,
                           pivot_distance - pivot_distance * np.cos(phi)])
        R = look_rotation(np.array([0.0, 0.0, pivot_distance]) - center)
        if jitter_deg:
            R = _pitch(rng.uniform(-jitter_deg, jitter_deg)) @ \
                _yaw(rng.uniform(-jitter_deg, jitter_deg)) @ R
        t = -R @ center
        cams.append(RegisteredCamera(i, R, t))
    return cams


def _rays(cam, w, h, f):
    xs = np.arange(w, dtype=np.float64)
    ys = np.arange(h, dtype=np.float64)
    X, Y = np.meshgrid(xs, ys)
    d_cam = np.stack([(X - w * 0.5) / f, (Y - h * 0.5) / f, np.ones_like(X)], -1)
    d_world = d_cam @ cam.rotation  # R^T d
    origin = cam.camera_center()
    return origin, d_world


def render(scene, cam, w, h, f, noise_sigma=0.0, rng=None):
    """Ray-cast one frame: (float32 gray image in [0,1], float64 depth map)."""
    origin, d = _rays(cam, w, h, f)
    best = np.full((h, w), np.inf)
    owner = np.full((h, w), -1, dtype=np.int32)
    with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
        for k, p in enumerate(scene.planes):
            denom = d @ p.normal
            s = ((p.point - origin) @ p.normal) / denom
            ok = (s > 1e-6) & np.isfinite(s) & (s < best)
            if not ok.any():
                continue
            hit = origin + s[ok][:, None] * d[ok]
            inside = np.all((hit >= p.lo) & (hit <= p.hi), axis=-1)
            idx = np.nonzero(ok)
            sel = (idx[0][inside], idx[1][inside])
            best[sel] = s[sel]
            owner[sel] = k
    # texture once per pixel, on the nearest plane
    value = np.full((h, w), 0.5)
    for k, p in enumerate(scene.planes):
        sel = owner == k
        if not sel.any():
            continue
        hit = origin + best[sel][:, None] * d[sel]
        rel = hit - p.point
        value[sel] = texture(rel @ p.u_axis, rel @ p.v_axis, p.plane_id, scene.seed,
                             contrast=p.contrast)
    if noise_sigma and rng is not None:
        value = value + rng.normal(0.0, noise_sigma, size=value.shape)
    img = np.clip(value, 0.0, 1.0).astype(np.float32)
    depth = best  # camera z equals s because the ray's camera-z component is 1
    return img, depth


def sample_landmarks(scene_depths, cams, w, h, f, per_camera, seed, border=8):
    """True-surface points under seeded pixels of the given cameras."""
    rng = np.random.default_rng(seed + 7)
    pts = []
    for cam, depth in zip(cams, scene_depths):
        xs = rng.integers(border, w - border, per_camera)
        ys = rng.integers(border, h - border, per_camera)
        z = depth[ys, xs]
        ok = np.isfinite(z)
        xs, ys, z = xs[ok], ys[ok], z[ok]
        pc = np.stack([(xs - w * 0.5) / f * z, (ys - h * 0.5) / f * z, z], -1)
        pts.append((pc - cam.translation) @ cam.rotation)
    return np.concatenate(pts, 0)


def to_rgba8(img):
    q = np.clip(np.round(img.astype(np.float64) * 255.0), 0, 255).astype(np.uint8)
    return np.ascontiguousarray(np.stack([q, q, q, np.full_like(q, 255)], -1))


def to_bf16_bits(img):
    b = np.ascontiguousarray(img.astype(np.float32)).view(np.uint32)
    # round to nearest even on the 16 dropped bits
    r = ((b >> 16) & 1) + 0x7FFF
    return ((b + r) >> 16).astype(np.uint16)


@dataclass
class Clip:
    width: int
    height: int
    focal: float
    cameras: List[RegisteredCamera]
    images: List[np.ndarray]          # float32 gray in [0, 1]
    depths: List[np.ndarray]
    sparse: np.ndarray

    def frames(self, storage="f32"):
        if storage == "f32":
            return [FrameInput(im) for im in self.images]
        if storage == "f16":
            return [FrameInput(im.astype(np.float16)) for im in self.images]
        if storage == "bf16":
            return [FrameInput(to_bf16_bits(im), bf16=True) for im in self.images]
        if storage == "rgba8":
            return [FrameInput(to_rgba8(im)) for im in self.images]
        raise ValueError(storage)


def make_clip(width, height, n_frames, arc_deg, pivot_distance, seed, noise_sigma=0.01,
              jitter_deg=0.0, landmark_cameras=None, landmarks_per_camera=400,
              extra_planes=0, boxes=0, low_texture_fraction=0.0, focal=None):
    scene = room_scene(seed, extra_planes, boxes, low_texture_fraction)
    f = float(focal if focal is not None else 1.2 * width)
    cams = arc_cameras(n_frames, arc_deg, pivot_distance, jitter_deg, seed)
    rng = np.random.default_rng(seed)
    images, depths = [], []
    for c in cams:
        im, d = render(scene, c, width, height, f, noise_sigma, rng)
        images.append(im)
        depths.append(d)
    if landmark_cameras is None:
        landmark_cameras = list(range(0, n_frames, max(1, n_frames // 12)))
    sparse = sample_landmarks([depths[i] for i in landmark_cameras],
                              [cams[i] for i in landmark_cameras], width, height, f,
                              landmarks_per_camera, seed)
    return Clip(width, height, f, cams, images, depths, sparse)


def plain_small_clip(seed=1, width=360, height=202):
    """1 reference + 4 source views, 15° arc, 0.08-unit baseline steps."""
    step = np.radians(15.0 / 4)
    pivot = 0.08 / (2 * np.sin(step / 2))
    return make_clip(width, height, 5, 15.0, pivot, seed, noise_sigma=0.01,
                     landmark_cameras=[2], landmarks_per_camera=600)


def full_clip(seed=2, width=640, height=360, n_frames=120, jitter_deg=2.0, arc_deg=40.0, **kw):
    """120 keyframes on a 40° arc around the scene centre, ±2° jitter."""
    return make_clip(width, height, n_frames, arc_deg, 4.0, seed, noise_sigma=0.01,
                     jitter_deg=jitter_deg, **kw)


def heavy_clip(seed=5, width=640, height=360, n_frames=120):
    """8 planes plus 4 boxes, 5 % low-texture regions, noise 0.02."""
    return make_clip(width, height, n_frames, 40.0, 4.0, seed, noise_sigma=0.02,
                     jitter_deg=2.0, extra_planes=4, boxes=4, low_texture_fraction=0.05)


def batched_clip_specs(n_clips=32, seed=3, min_frames=24, max_frames=120, min_edge=240,
                       max_edge=640):
    """Seeded parameters of the batched uneven clips: long edge uniform in
    [min_edge, max_edge] at 16:9, min_frames..max_frames frames, 2-12 source views
    per reference, 32-256 hypotheses, 0-2 extra planes and 0-1 boxes."""
    rng = np.random.default_rng(seed)
    specs = []
    for i in range(n_clips):
        w = int(rng.integers(min_edge, max_edge + 1))
        h = max(16, int(round(w * 9 / 16)))
        specs.append(dict(width=w, height=h, n_frames=int(rng.integers(min_frames, max_frames + 1)),
                          sources=int(rng.integers(2, 13)), planes=int(rng.integers(32, 257)),
                          extra_planes=int(rng.integers(0, 3)), boxes=int(rng.integers(0, 2)),
                          seed=seed * 1000 + i))
    return specs


def batched_clip(spec):
    """The clip of one batched_clip_specs entry (a 40-degree arc like the full clip)."""
    return make_clip(spec["width"], spec["height"], spec["n_frames"], 40.0, 4.0, spec["seed"],
                     noise_sigma=0.01, jitter_deg=2.0, extra_planes=spec["extra_planes"],
                     boxes=spec["boxes"], landmarks_per_camera=200)
