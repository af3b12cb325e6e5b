"""Seeded meshes for the surface-fusion parity tests: overlapping noisy grid
patches of one gently curved surface, one patch per camera-support group, plus
the defects the reference's fusion must survive (non-finite points, repeated,
degenerate, collinear and out-of-range triangles, points without a group)."""
import numpy as np

from v3d import types


def point_array(rows):
    a = np.zeros(len(rows), dtype=types.POINT_DTYPE)
    for i, (x, y, z, c) in enumerate(rows):
        a[i] = (x, y, z, c, 128, 128, 128, 0)
    return a


def triangle_array(rows, confidence=0.9):
    a = np.zeros(len(rows), dtype=types.TRIANGLE_DTYPE)
    for i, (p, q, r) in enumerate(rows):
        a[i] = (p, q, r, confidence, 0)
    return a


# The scenes of the reference's own fusion tests (surface_fusion.rs:917-1027):
# name -> (points, triangles, membership)
REFERENCE_SCENES = {
    "aligns_mutually_nearest_vertices": (
        [(0, 0, 0, 1), (1, 0, 0, 1), (0, 1, 0, 1), (0, 0, 0.06, 1), (1, 0, 0.06, 1),
         (0, 1, 0.06, 1)], [(0, 1, 2), (3, 4, 5)], [0, 0, 0, 1, 1, 1]),
    "rejects_when_normals_disagree": (
        [(0, 0, 0, 1), (1, 0, 0, 1), (0, 1, 0, 1), (0, 0, 0.05, 1), (1, 0, 0.05, 1),
         (0, 0.05, 1, 1)], [(0, 1, 2), (3, 4, 5)], [0, 0, 0, 1, 1, 1]),
    "rejects_a_weakening_seam_move": (
        [(0, 0, 0, 1), (1, 0, 0, 1), (0.9, 0.01, 0, 1), (0, 0.12, 0, 1), (1, 0.12, 0, 1),
         (0, 1.12, 0, 1)], [(0, 1, 2), (3, 4, 5)], [0, 0, 0, 1, 1, 1]),
    "never_fuses_within_a_group": (
        [(0, 0, 0, 1), (1, 0, 0, 1), (0, 1, 0, 1)], [(0, 1, 2)], [0, 0, 0]),
}


def reference_scene(name):
    pts, tris, mem = REFERENCE_SCENES[name]
    return point_array(pts), triangle_array(tris), np.array(mem, dtype=np.int64)


def layered_grids(seed, groups=3, nx=80, ny=60, spacing=0.05, jitter=0.004, separation=0.003,
                  half_shift=False, wall=False, defects=True):
    """`groups` grid patches of z = 2 + 0.05 sin(3x) cos(2y), each shifted in the
    plane (randomly, or by exactly half a spacing per group with half_shift, which
    makes equal distances and so the tie rule matter) and lifted by
    `separation` per group; `wall` adds a perpendicular patch whose normals
    disagree with the others."""
    rng = np.random.default_rng(seed)
    pts, tris, mem = [], [], []
    base = 0
    for g in range(groups + (1 if wall else 0)):
        is_wall = wall and g == groups
        if half_shift:
            ox, oy = g * spacing / 2, 0.0
        else:
            ox, oy = rng.uniform(0.0, spacing, 2)
        u = ox + spacing * np.arange(nx)
        v = oy + spacing * np.arange(ny)
        U, V = np.meshgrid(u, v)
        if is_wall:
            X = np.full_like(U, spacing * nx / 2) + rng.normal(0, jitter / 4, U.shape)
            Y = V
            Z = 1.9 + U * 0.05
        else:
            X, Y = U.copy(), V.copy()
            if not half_shift:
                X += rng.normal(0, jitter, X.shape)
                Y += rng.normal(0, jitter, Y.shape)
            Z = 2.0 + 0.05 * np.sin(3 * X) * np.cos(2 * Y) + g * separation
        n = X.size
        p = np.zeros(n, dtype=types.POINT_DTYPE)
        p["x"], p["y"], p["z"] = X.ravel(), Y.ravel(), Z.ravel()
        conf = rng.uniform(0.01, 1.0, n)
        conf[rng.random(n) < 0.05] = 1.0
        p["confidence"] = conf
        p["r"], p["g"], p["b"] = 10 * g, 128, 200
        pts.append(p)
        idx = base + np.arange(n).reshape(ny, nx)
        a, b = idx[:-1, :-1].ravel(), idx[:-1, 1:].ravel()
        c, d = idx[1:, :-1].ravel(), idx[1:, 1:].ravel()
        t = np.zeros(2 * a.size, dtype=types.TRIANGLE_DTYPE)
        t["a"] = np.concatenate([a, b])
        t["b"] = np.concatenate([b, d])
        t["c"] = np.concatenate([c, c])
        t["confidence"] = rng.uniform(0.0, 1.2, t.size)
        tris.append(t)
        mem.append(np.full(n, g, dtype=np.int64))
        base += n
    points = np.concatenate(pts)
    triangles = np.concatenate(tris)
    membership = np.concatenate(mem)
    if defects:
        n = len(points)
        bad = rng.choice(n, max(1, n // 400), replace=False)
        points["x"][bad[: len(bad) // 2]] = np.nan
        points["z"][bad[len(bad) // 2:]] = np.inf
        membership[rng.choice(n, max(1, n // 200), replace=False)] = -1
        extra = np.zeros(8, dtype=types.TRIANGLE_DTYPE)
        extra[0] = (0, 0, 1, 0.5, 0)                  # repeated vertex
        extra[1] = (1, 2, n + 5, 0.5, 0)              # out of range
        extra[2] = tuple(triangles[3])                 # repeated triangle
        extra[3] = tuple(triangles[3])
        extra[4] = (0, 1, 2, np.nan, 0)               # NaN confidence
        extra[5] = (5, 6, 7, 0.5, 0)                  # collinear (one grid row)
        extra[6] = (bad[0], 1, 2, 0.5, 0)             # non-finite vertex
        extra[7] = (3, 4, nx + 3, -1.0, 0)            # negative confidence
        triangles = np.concatenate([triangles, extra])
    return np.ascontiguousarray(points), np.ascontiguousarray(triangles), membership
