"""The dense artifact wire format on the CPU: the oracle's shortest f32
digits against numpy's shortest float32 repr and, on a small sample, against
an exact rational check; serde_json's f32 notation on known cases; the
library's host SHA-256 (both compression paths) against hashlib; the browser
transport's packed point buffers; and the oracle's document read back as
JSON."""
import hashlib
import json
import os
import subprocess
import sys
from fractions import Fraction

import numpy as np
import pytest

from v3d import dense, types

from tests.oracle_ffi import Oracle


def special_floats():
    """Every exponent with a few mantissas, both signs, the binade edges,
    subnormals, integers and short decimals."""
    bits = []
    for e in range(0, 255):
        for m in (0, 1, 2, 3, 0x400000, 0x7FFFFE, 0x7FFFFF, 0x2AAAAA, 0x555555, 0x123456):
            bits.append((e << 23) | m)
    v = np.array(bits, dtype=np.uint32).view(np.float32)
    extra = np.array([1.0, 0.1, 0.2, 0.3, 1e-7, 1.5e-7, 1e-6, 1.5e-5, 1e-5, 123456.7, 1e10, 1e12,
                      1e13, 9999999.0, 16777216.0, 3.4028235e38, 1.1754944e-38, 1e-45, 0.5, 2.5,
                      255.0, 0.999999, 7.038531e-26, 9.403955e-38, 1e23, 5e-324],
                     dtype=np.float32)
    v = np.concatenate([v, extra])
    v = v[np.isfinite(v) & (v != 0)]
    return np.concatenate([v, -v])


def random_floats(n, seed):
    rng = np.random.default_rng(seed)
    v = rng.integers(0, 2 ** 32, n, dtype=np.uint64).astype(np.uint32).view(np.float32)
    return v[np.isfinite(v) & (v != 0)]


def numpy_shortest(x):
    s = np.format_float_scientific(np.float32(x), unique=True, trim="-")
    mant, exp = s.split("e")
    digits = mant.lstrip("-").replace(".", "")
    d, k = int(digits), int(exp) - (len(digits) - 1)
    while d % 10 == 0:
        d //= 10
        k += 1
    return d, k


def test_shortest_digits_equal_numpy():
    o = Oracle()
    values = np.concatenate([special_floats(), random_floats(60000, 3)])
    bad = [(float(x), o.shortest_f32(x), numpy_shortest(x)) for x in values
           if o.shortest_f32(x) != numpy_shortest(x)]
    assert bad == []


def _exact(x):
    """Rounding interval of an f32 as exact rationals."""
    b = int(np.float32(x).view(np.uint32)) & 0x7FFFFFFF
    e, m = b >> 23, b & 0x7FFFFF
    m2, e2 = (m | (1 << 23), e - 150) if e else (m, -149)
    v = Fraction(m2) * Fraction(2) ** e2
    up = (Fraction(m2) + Fraction(1, 2)) * Fraction(2) ** e2
    gap = Fraction(1, 4) if (m == 0 and e > 1) else Fraction(1, 2)
    lo = (Fraction(m2) - gap) * Fraction(2) ** e2
    return v, lo, up, m2 % 2 == 0


def test_shortest_digits_exactly_on_a_sample():
    o = Oracle()
    rng = np.random.default_rng(5)
    values = np.concatenate([special_floats()[::9], random_floats(800, 6)])
    values = values[rng.permutation(len(values))][:1500]
    for x in values:
        d, k = o.shortest_f32(abs(float(x)))
        v, lo, up, inclusive = _exact(abs(x))

        def inside(q):
            return (lo <= q <= up) if inclusive else (lo < q < up)
        cand = Fraction(d) * Fraction(10) ** k
        assert inside(cand), x
        n = len(str(d))
        # no decimal with fewer digits lies inside the interval
        if n > 1:
            scale = Fraction(10) ** (k + 1)
            assert not any(inside(Fraction(q) * scale)
                           for q in (int(v / scale), int(v / scale) + 1)), x
        # no other decimal of the same length inside is closer
        unit = Fraction(10) ** k
        for q in (d - 1, d + 1):
            c = Fraction(q) * unit
            if q > 0 and inside(c):
                dist, best = abs(c - v), abs(cand - v)
                assert dist > best or (dist == best and d % 2 == 0), x


@pytest.mark.parametrize("value,text", [
    (1.0, "1.0"), (0.1, "0.1"), (-0.0, "-0.0"), (0.0, "0.0"), (1e-7, "1e-7"),
    (1.5e-7, "1.5e-7"), (1e-6, "0.000001"), (1.5e-5, "0.000015"), (123456.7, "123456.7"),
    (1e10, "10000000000.0"), (1e12, "1000000000000.0"), (1e13, "1e13"), (1.5e13, "1.5e13"),
    (3.4028235e38, "3.4028235e38"), (1.1754944e-38, "1.1754944e-38"), (1e-45, "1e-45"),
    (-2.5, "-2.5"), (16777216.0, "16777216.0"), (0.3, "0.3"), (float("nan"), "null"),
    (float("inf"), "null"), (float("-inf"), "null")])
def test_notation(value, text):
    assert Oracle().format_f32(np.float32(value)) == text


def test_formatted_floats_read_back():
    o = Oracle()
    for x in np.concatenate([special_floats()[::3], random_floats(20000, 9)]):
        assert np.float32(float(o.format_f32(x))) == x


@pytest.mark.parametrize("n", [0, 1, 55, 56, 63, 64, 65, 119, 120, 128, 1000, 1 << 20])
def test_sha256_equals_hashlib(n):
    data = np.random.default_rng(n).integers(0, 256, n, dtype=np.uint8).tobytes()
    assert dense.content_hash(data) == "sha256:" + hashlib.sha256(data).hexdigest()


def test_sha256_portable_path_equals_hashlib():
    code = ("import hashlib, numpy as np; from v3d import dense\n"
            "for n in (0, 3, 64, 100, 4096 + 17):\n"
            "    d = np.random.default_rng(n).integers(0, 256, n, dtype=np.uint8).tobytes()\n"
            "    assert dense.content_hash(d) == 'sha256:' + hashlib.sha256(d).hexdigest()\n")
    env = dict(os.environ, V3D_SHA256_PORTABLE="1", PYTHONPATH=os.pathsep.join(sys.path))
    r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def _evidence(n, seed, nonfinite=False):
    rng = np.random.default_rng(seed)
    pts = np.zeros(n, dtype=types.POINT_DTYPE)
    for f in ("x", "y", "z"):
        pts[f] = rng.normal(0, 3, n).astype(np.float32)
    pts["confidence"] = rng.random(n).astype(np.float32)
    for f in ("r", "g", "b"):
        pts[f] = rng.integers(0, 256, n)
    sites = np.zeros(n, dtype=types.SITE_DTYPE)
    sites["x"] = rng.integers(0, 1 << 32, n, dtype=np.uint64)
    sites["y"] = rng.integers(0, 5000, n)
    attrs = np.zeros(n, dtype=types.ATTR_DTYPE)
    attrs["reciprocal_consistency"] = rng.random(n).astype(np.float32)
    attrs["depth_margin"] = (rng.random(n) ** 6).astype(np.float32)
    if nonfinite and n > 3:
        pts["x"][1] = np.nan
        attrs["depth_margin"][2] = np.inf
    return pts, sites, attrs


def test_pack_dense_points():
    pts, _, _ = _evidence(1000, 1)
    values, rgb = dense.pack_dense_points(pts)
    assert (values, rgb) == Oracle().pack_dense_points(pts)
    f = np.stack([pts["x"], pts["y"], pts["z"], pts["confidence"]], axis=1).astype("<f4")
    assert values == f.tobytes()
    assert rgb == np.stack([pts["r"], pts["g"], pts["b"]], axis=1).astype(np.uint8).tobytes()


def test_oracle_document_reads_back():
    pts, sites, attrs = _evidence(500, 2, nonfinite=True)
    prefix, suffix = b'{"schema_version":1,"dense":{"stats":{},"points":', b',"warnings":[]}}'
    doc, info = Oracle().encode_dense_evidence(pts, sites, attrs, prefix, suffix)
    assert len(doc) == info["document_bytes"] <= dense.library().v3d_dense_document_bound(
        500, 500, 500, len(prefix), len(suffix))
    assert info["non_finite"] == 2
    parsed = json.loads(doc.replace(b"null", b"0"))["dense"]
    assert list(parsed) == ["stats", "points", "grid_sites", "point_attributes", "warnings"]
    assert list(parsed["points"][0]) == ["x", "y", "z", "confidence", "r", "g", "b"]
    ok = np.isfinite(pts["x"])
    assert (np.float32([p["x"] for p in parsed["points"]])[ok] == pts["x"][ok]).all()
    assert [s["x"] for s in parsed["grid_sites"]] == [int(v) for v in sites["x"]]
    assert (np.float32([a["reciprocal_consistency"] for a in parsed["point_attributes"]])
            == attrs["reciprocal_consistency"]).all()
    head = len(prefix)
    assert doc[head:head + info["points_bytes"]].startswith(b"[{")
    assert doc[head + info["points_bytes"]:].startswith(b',"grid_sites":[')
    empty, info = Oracle().encode_dense_evidence(None, None, None)
    assert empty == b'[],"grid_sites":[],"point_attributes":[]'
    assert (info["points_bytes"], info["grid_sites_bytes"], info["point_attributes_bytes"]) == (2, 2, 2)


def _mesh_records(n, seed, points=1000):
    rng = np.random.default_rng(seed)
    tris = np.zeros(n, dtype=types.TRIANGLE_DTYPE)
    for f in ("a", "b", "c"):
        tris[f] = rng.integers(0, points, n)
    tris["confidence"] = rng.random(n).astype(np.float32)
    src = np.zeros(n // 3, dtype=dense.TRIANGLE_SOURCE_DTYPE)
    src["triangle"] = np.sort(rng.integers(0, n, len(src)))
    src["corners"] = rng.integers(0, points, (len(src), 3))
    der = np.zeros(n // 5, dtype=dense.DERIVED_VERTEX_DTYPE)
    der["point_index"] = points + np.arange(len(der))
    der["source_triangle"] = rng.integers(0, n, len(der))
    der["source_corners"] = rng.integers(0, points, (len(der), 3))
    w = rng.random((len(der), 3))
    der["barycentric"] = w / w.sum(axis=1, keepdims=True)
    return tris, src, der


def test_pack_mesh_triangles():
    tris, src, der = _mesh_records(3000, 4)
    got = dense.pack_mesh_triangles(tris, 1000, src, der)
    st, want = Oracle().pack_mesh_triangles(tris, 1000, src, der)
    assert st == 0 and got == want
    idx = np.stack([tris["a"], tris["b"], tris["c"]], axis=1).astype("<u4").tobytes()
    assert got["indices_u32_le"] == idx
    assert got["confidence_f32_le"] == tris["confidence"].astype("<f4").tobytes()
    assert got["derived_barycentric_f64_le"] == der["barycentric"].astype("<f8").tobytes()
    assert dense.pack_mesh_triangles(tris[:0], 0) == {
        k: b"" for k in ("indices_u32_le", "confidence_f32_le", "sources_u32_le", "derived_u32_le",
                         "derived_barycentric_f64_le")}


@pytest.mark.parametrize("case,message", [
    ("missing", "mesh triangle references a missing dense point"),
    ("index", "dense point index exceeds browser transport range"),
    ("source", "triangle source exceeds browser transport range"),
    ("derived", "triangle source exceeds browser transport range")])
def test_pack_mesh_triangles_errors(case, message):
    tris, src, der = _mesh_records(30, 5)
    count = 1000
    if case == "missing":
        tris["b"][7] = 1000
    elif case == "index":
        count = 1 << 40
        tris["c"][3] = 1 << 33
    elif case == "source":
        src["corners"][2, 1] = 1 << 32
    else:
        der["source_triangle"][1] = 1 << 32
    with pytest.raises(ValueError, match=message):
        dense.pack_mesh_triangles(tris, count, src, der)
    st, _ = Oracle().pack_mesh_triangles(tris, count, src, der)
    assert st == {"source": 1, "derived": 1, "missing": 2, "index": 3}[case]


def test_reused_buffer_is_checked_before_any_call():
    pts, sites, attrs = _evidence(50, 3)
    fn = Oracle().lib.v3do_encode_dense_evidence
    bound = dense.document_bound(50, 50, 50)
    for bad in (np.zeros(bound - 1, np.uint8), np.zeros(bound, np.int8),
                np.zeros((2, bound), np.uint8)[:, ::2]):
        with pytest.raises(ValueError):
            dense._encode(fn, (), pts, sites, attrs, b"", b"", bad)
    buf = np.zeros(bound, np.uint8)
    st, view, info = dense._encode(fn, (), pts, sites, attrs, b"", b"", buf)
    assert st == 0 and isinstance(view, memoryview) and len(view) == info["document_bytes"]
    assert bytes(view) == Oracle().encode_dense_evidence(pts, sites, attrs)[0]
