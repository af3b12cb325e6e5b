"""Inputs of the connected-surface merge (surface_merge.rs) for the tests.

* The reference's own fixtures (surface_merge_tests.rs:132-157, 370-410,
  948-1083, 1183-1298 and the derived acceptance tests), restated: each
  returns a dict of points (POINT_DTYPE), triangles (TRIANGLE_DTYPE),
  membership, pairs, cameras and origins.
* Seeded synthetic multi-reference patches: every camera of an arc sees the
  room scene; each patch is a grid mesh of ray-cast depth points of its own
  reference camera (one support group per patch), with a per-patch depth
  scale drift and per-point depth noise, so neighbouring patches overlap as
  the dense pass's reference patches do.  Fusion pairs come from the oracle's
  fusion (surface_fusion.rs) on the CPU.
"""
import numpy as np

from v3d import abi, synth, types


class Cam:
    def __init__(self, x=0.0, rotation=None, translation=None):
        self.rotation = np.eye(3) if rotation is None else np.asarray(rotation, np.float64)
        self.translation = (np.array([-x, 0.0, 0.0]) if translation is None
                            else np.asarray(translation, np.float64))


def _points(rows):
    p = np.zeros(len(rows), dtype=types.POINT_DTYPE)
    for i, (x, y, z) in enumerate(rows):
        p[i] = (np.float32(x), np.float32(y), np.float32(z), np.float32(1.0), 40, 80, 120, 0)
    return p


def _tris(rows, confidence=0.9):
    t = np.zeros(len(rows), dtype=types.TRIANGLE_DTYPE)
    for i, (a, b, c) in enumerate(rows):
        t[i]["a"], t[i]["b"], t[i]["c"] = a, b, c
        t[i]["confidence"] = np.float32(confidence)
    return t


def case(points, triangles, membership, pairs=(), cameras=(), origins=None):
    return {"points": _points(points) if not isinstance(points, np.ndarray) else points,
            "triangles": _tris(triangles) if not isinstance(triangles, np.ndarray) else triangles,
            "membership": np.asarray(membership, dtype=np.int64),
            "pairs": np.asarray(pairs, dtype=np.uint64).reshape(-1, 2),
            "cameras": list(cameras), "origins": origins}


class _Seam:
    def __init__(self):
        self.points, self.membership, self.triangles, self.origins = [], [], [], []
        self.pairs, self.cameras = [], []

    def grid(self, xs, ys, z, group):
        g = []
        for y in ys:
            row = []
            for x in xs:
                self.points.append((x, y, z))
                self.membership.append(group)
                self.origins.append(abi.ORIGIN_GEOMETRIC)
                row.append(len(self.points) - 1)
            g.append(row)
        for r in range(len(ys) - 1):
            for c in range(len(xs) - 1):
                p00, p10, p01, p11 = g[r][c], g[r][c + 1], g[r + 1][c], g[r + 1][c + 1]
                self.triangles += [(p00, p10, p01), (p10, p11, p01)]
        return g

    def case(self):
        return case(self.points, self.triangles, self.membership, self.pairs, self.cameras,
                    np.asarray(self.origins, dtype=np.int32))


OWNER_XS = [-1.84, -1.38, -0.92, -0.46, 0.0]
SEAM_ROWS = [-1.0, 0.0, 1.0]


def trimmed_seam():
    """surface_merge_tests.rs:1287-1298."""
    s = _Seam()
    owner = s.grid(OWNER_XS, SEAM_ROWS, 5.0, 0)
    lower = s.grid([-0.46, 0.04, 0.54, 1.04], SEAM_ROWS, 5.0, 1)
    s.pairs = [(owner[r][3], lower[r][0]) for r in range(3)]
    s.cameras = [Cam(0.0), Cam(0.4)]
    return s.case()


def three_patches():
    """surface_merge_tests.rs:1564-1590."""
    s = _Seam()
    owner = s.grid(OWNER_XS, SEAM_ROWS, 5.0, 0)
    lower = s.grid([-0.46, 0.04, 0.54, 1.04], SEAM_ROWS, 5.0, 1)
    s.grid([-2.3, -1.8, -1.3], SEAM_ROWS, 5.0, 2)
    s.pairs = [(owner[r][3], lower[r][0]) for r in range(3)]
    s.cameras = [Cam(0.0), Cam(0.4), Cam(-1.5)]
    return s.case()


def partial_overlap(sloped=False):
    """surface_merge_derived_acceptance_tests.rs:5-24."""
    s = _Seam()
    owner = s.grid(OWNER_XS, SEAM_ROWS, 5.0, 0)
    lower = s.grid([-0.46, -0.04, 0.46, 0.96], SEAM_ROWS, 5.0, 1)
    if sloped:
        pts = []
        for x, y, _ in s.points:
            x32, y32 = np.float32(x), np.float32(y)
            pts.append((x, y, np.float32(5.0) + np.float32(0.25) * x32 + np.float32(0.15) * y32))
        s.points = pts
    s.pairs = [(owner[r][3], lower[r][0]) for r in range(3)]
    s.cameras = [Cam(0.0), Cam(0.4)]
    return s.case()


def other_depth():
    """surface_merge_tests.rs:1511-1550."""
    s = _Seam()
    owner = s.grid(OWNER_XS, SEAM_ROWS, 5.0, 0)
    seam = s.grid([-0.46, 0.04], SEAM_ROWS, 5.0, 1)
    far = s.grid([0.04, 0.54, 1.04], SEAM_ROWS, 5.4, 1)
    s.origins[far[1][0]] = abi.ORIGIN_REVALIDATED
    s.pairs = [(owner[r][3], seam[r][0]) for r in range(3)] + [(owner[1][4], far[1][0])]
    s.cameras = [Cam(0.0), Cam(0.4)]
    return s.case()


def owned_overlap():
    """surface_merge_tests.rs:370-410."""
    pts = [(-1, -1, 5), (1, -1, 5), (1, 1, 5), (-1, 1, 5), (-4, -1, 5), (-3, -1, 5), (-3.5, 0, 5),
           (-0.5, -0.5, 5.05), (0.6, -0.4, 5.05), (0.1, 0.7, 5.05), (3, -0.5, 5), (3.5, 0.5, 5),
           (-0.5, -0.5, 5.05), (-0.6, 0.2, 5), (-0.2, 0.2, 5), (-0.4, 0.6, 5)]
    mem = [1 if (7 <= i < 12 or i >= 13) else 0 for i in range(len(pts))]
    tris = [(0, 1, 2), (0, 2, 3), (4, 5, 6), (0, 1, 12), (7, 8, 9), (8, 10, 11), (13, 14, 15)]
    return case(pts, tris, mem, [(12, 7)], [Cam(0.0), Cam(0.4)])


def adjacent_grids():
    """surface_merge_tests.rs:132-157, fused at x = 2, no cameras (the 3D test)."""
    pts, mem = [], []
    for start, z, patch in ((0.0, 0.0, 0), (1.0, 0.06, 1)):
        for y in range(2):
            for x in range(3):
                shared = patch == 1 and x == 1
                pts.append((start + x, y, 0.0 if shared else z))
                mem.append(patch)
    tris = []
    for off in (0, 6):
        for x in range(2):
            s = off + x
            tris += [(s, s + 1, s + 3), (s + 1, s + 4, s + 3)]
    return case(pts, tris, mem, [(2, 7), (5, 10)], [])


def crossing_strips(bound=512, cameras=True):
    """surface_merge_tests.rs:948-1008."""
    columns = 2 * bound + 4
    pts = []
    for row in range(3):
        for column in range(columns + 1):
            pts.append((np.float32(-1.0) + np.float32(2.0) * np.float32(column) / np.float32(columns),
                        row - 1.0, 5.0))
    comb = lambda r, c: r * (columns + 1) + c  # noqa: E731
    tris = []
    for row in range(2):
        for c in range(columns):
            tris += [(comb(row, c), comb(row, c + 1), comb(row + 1, c + 1)),
                     (comb(row, c), comb(row + 1, c + 1), comb(row + 1, c))]
    base = len(pts)
    xs = [-1.5, -1.0, 0.0, 1.0, 1.5]
    for y in (0.0, 0.05):
        for x in xs:
            pts.append((x, y, 5.0))
    for k in range(4):
        tris += [(base + k, base + k + 1, base + 5 + k + 1), (base + k, base + 5 + k + 1, base + 5 + k)]
    mem = [1 if i >= base else 0 for i in range(len(pts))]
    return case(pts, tris, mem, [(comb(1, 0), base + 1)], [Cam(0.0), Cam(0.0)] if cameras else [])


def sliver_fan(slivers):
    """surface_merge_tests.rs:1058-1083."""
    pts = [(0.0, -100.0, 0.0), (-2.0, 0.0, 0.0), (-2.0, -1.0, 0.0)]
    tris = [(0, 1, 2)]
    for s in range(slivers):
        x = np.float32(-2.0) + np.float32(4.0) * (np.float32(s) + np.float32(0.5)) / np.float32(slivers)
        i = len(pts)
        pts += [(x, 100.0, 0.0), (x + np.float32(0.01), 100.0, 0.0)]
        tris.append((0, i, i + 1))
    cand = len(pts)
    pts += [(-2.0, 0.0, 0.0), (2.0, 0.0, 0.0), (0.0, 2.0, 0.0)]
    tris.append((cand, cand + 1, cand + 2))
    mem = [1 if i >= cand else 0 for i in range(len(pts))]
    return case(pts, tris, mem, [(1, cand)], [])


def reference_cases():
    return {"trimmed_seam": trimmed_seam(), "three_patches": three_patches(),
            "partial_overlap": partial_overlap(False), "partial_overlap_sloped": partial_overlap(True),
            "other_depth": other_depth(), "owned_overlap": owned_overlap(),
            "adjacent_grids": adjacent_grids(), "crossing_strips": crossing_strips(),
            "crossing_strips_3d": crossing_strips(cameras=False), "sliver_fan_8": sliver_fan(8),
            "sliver_fan_160": sliver_fan(160)}


def synthetic_patches(n_patches=6, width=160, height=90, stride=2, arc_deg=12.0, seed=7,
                      scale_drift=0.01, noise=0.002):
    """Grid-mesh patches of ray-cast room-scene depth, one per arc camera.
    Returns (points, triangles, membership, cameras, groups) before fusion."""
    rng = np.random.default_rng(seed)
    scene = synth.room_scene(seed)
    cams = synth.arc_cameras(n_patches, arc_deg, 4.0, jitter_deg=1.0, seed=seed)
    f = 0.9 * width
    pts_all, tris_all, mem_all, cameras = [], [], [], []
    base = 0
    for k, cam in enumerate(cams):
        _, depth = synth.render(scene, cam, width, height, f)
        ys = np.arange(stride, height - stride, stride)
        xs = np.arange(stride, width - stride, stride)
        X, Y = np.meshgrid(xs, ys)
        d = depth[Y, X] * (1.0 + scale_drift * rng.uniform(-1, 1))
        d = d * (1.0 + noise * rng.standard_normal(d.shape))
        valid = np.isfinite(d) & (d > 0.1)
        pc = np.stack([(X - width * 0.5) / f * d, (Y - height * 0.5) / f * d, d], -1)
        R, t = np.asarray(cam.rotation), np.asarray(cam.translation)
        world = (pc - t) @ R  # R^T (p - t)
        idx = -np.ones(X.shape, dtype=np.int64)
        n = int(valid.sum())
        idx[valid] = base + np.arange(n)
        p = np.zeros(n, dtype=types.POINT_DTYPE)
        w = world[valid].astype(np.float32)
        p["x"], p["y"], p["z"] = w[:, 0], w[:, 1], w[:, 2]
        p["confidence"] = rng.uniform(0.5, 1.0, n).astype(np.float32)
        p["r"], p["g"], p["b"] = rng.integers(0, 256, (3, n), dtype=np.uint8)
        tl, tr, bl, br = idx[:-1, :-1], idx[:-1, 1:], idx[1:, :-1], idx[1:, 1:]
        dd = d
        cont = lambda a, b: np.abs(a - b) < 0.05 * np.minimum(a, b)  # noqa: E731
        ok1 = (tl >= 0) & (tr >= 0) & (bl >= 0) & cont(dd[:-1, :-1], dd[:-1, 1:]) & \
            cont(dd[:-1, :-1], dd[1:, :-1])
        ok2 = (tr >= 0) & (br >= 0) & (bl >= 0) & cont(dd[:-1, 1:], dd[1:, 1:]) & \
            cont(dd[1:, 1:], dd[1:, :-1])
        t1 = np.stack([tl[ok1], tr[ok1], bl[ok1]], -1)
        t2 = np.stack([tr[ok2], br[ok2], bl[ok2]], -1)
        tri = np.concatenate([t1, t2])
        tri = tri[np.lexsort((tri[:, 0],))] if len(tri) else tri
        tt = np.zeros(len(tri), dtype=types.TRIANGLE_DTYPE)
        tt["a"], tt["b"], tt["c"] = tri[:, 0], tri[:, 1], tri[:, 2]
        tt["confidence"] = rng.uniform(0.5, 1.0, len(tri)).astype(np.float32)
        pts_all.append(p)
        tris_all.append(tt)
        mem_all.append(np.full(n, k, dtype=np.int64))
        cameras.append(Cam(rotation=R, translation=t))
        base += n
    return (np.concatenate(pts_all), np.concatenate(tris_all), np.concatenate(mem_all), cameras,
            n_patches)


def synthetic_case(oracle, **kw):
    """synthetic_patches fused by the oracle's fusion: the merge's inputs."""
    pts, tris, mem, cams, _ = synthetic_patches(**kw)
    pts = np.ascontiguousarray(pts)
    out = oracle.fuse_mutually_supported_vertices(pts, tris, mem)
    origins = np.zeros(len(pts), dtype=np.int32)
    return case(pts, tris, mem, out.pairs, cams, origins)
