"""The dense artifact's arrays formatted on the device against the CPU
oracle, byte for byte, and the document's SHA-256 against hashlib: a dense
result of the pipeline, every f32 exponent with edge mantissas, half a
million random f32 bit patterns (NaN, infinities, zeros and subnormals
included), empty and uneven arrays, and a buffer that is too small."""
import ctypes as C
import hashlib

import numpy as np
import pytest

from v3d import abi, dense, profiles, synth, types

from tests.oracle_ffi import Oracle
from tests.test_artifact_cpu import _evidence, special_floats

PREFIX = (b'{"schema_version":1,"request_hash":"sha256:' + b"0" * 64 +
          b'","cameras_hash":"sha256:' + b"1" * 64 + b'","dense":{"stats":{"attempted":true},'
          b'"points":')
SUFFIX = b',"warnings":["reference view 3 skipped"]}}'


def _compare(points, sites, attrs, prefix=PREFIX, suffix=SUFFIX):
    doc, info = dense.Context(0).encode_dense_evidence(points, sites, attrs, prefix, suffix)
    odoc, oinfo = Oracle().encode_dense_evidence(points, sites, attrs, prefix, suffix)
    assert doc == odoc
    assert info["content_hash"] == "sha256:" + hashlib.sha256(doc).hexdigest()
    assert {k: v for k, v in info.items() if k != "content_hash"} == \
        {k: v for k, v in oinfo.items() if k != "content_hash"}
    return doc, info


@pytest.mark.gpu
def test_pipeline_result():
    clip = synth.make_clip(320, 180, 6, 15.0, 1.5, seed=4, noise_sigma=0.01)
    res = dense.Context(0).estimate_depth_points_with_control(
        clip.frames("f32"), clip.cameras, clip.sparse, clip.focal,
        profile=profiles.zncc(2, 64, 4, 2))
    assert len(res.points) > 1000
    doc, info = _compare(res.points, res.grid_sites, res.point_attributes)
    assert info["non_finite"] == 0
    values, rgb = dense.pack_dense_points(res.points)
    assert (values, rgb) == Oracle().pack_dense_points(res.points)


def _float_attrs(values):
    if len(values) % 2:
        values = np.concatenate([values, values[:1]])
    a = np.zeros(len(values) // 2, dtype=types.ATTR_DTYPE)
    a["reciprocal_consistency"] = values[0::2]
    a["depth_margin"] = values[1::2]
    return a


@pytest.mark.gpu
def test_every_exponent_and_random_bit_patterns():
    special = special_floats()
    rng = np.random.default_rng(12)
    rand = rng.integers(0, 2 ** 32, 500000, dtype=np.uint64).astype(np.uint32).view(np.float32)
    odd = np.array([0.0, -0.0, np.nan, np.inf, -np.inf, 1e-45, -1e-45], dtype=np.float32)
    attrs = _float_attrs(np.concatenate([special, odd, rand]))
    doc, info = _compare(None, None, attrs, b"", b"")
    finite = np.isfinite(attrs["reciprocal_consistency"]) & np.isfinite(attrs["depth_margin"])
    assert info["non_finite"] == int((~np.isfinite(attrs["reciprocal_consistency"])).sum() +
                                     (~np.isfinite(attrs["depth_margin"])).sum())
    assert finite.sum() > 400000 // 2


@pytest.mark.gpu
@pytest.mark.parametrize("counts", [(0, 0, 0), (1, 1, 1), (7, 0, 3), (0, 40, 0), (33, 31, 64),
                                    (5000, 5000, 0)])
def test_empty_and_uneven_arrays(counts):
    n = max(counts)
    pts, sites, attrs = _evidence(max(n, 1), 7, nonfinite=n > 3)
    _compare(pts[:counts[0]], sites[:counts[1]], attrs[:counts[2]])
    _compare(pts[:counts[0]], sites[:counts[1]], attrs[:counts[2]], b"", b"")


@pytest.mark.gpu
def test_large_evidence_and_a_short_buffer():
    pts, sites, attrs = _evidence(300000, 8, nonfinite=True)
    doc, info = _compare(pts, sites, attrs)
    assert info["non_finite"] == 2 and len(doc) > 30_000_000
    ctx = dense.Context(0)
    out = abi.DenseDocument()
    buf = np.empty(1000, dtype=np.uint8)
    st = ctx.lib.v3d_encode_dense_evidence(
        ctx.handle, pts.ctypes.data, len(pts), sites.ctypes.data, len(sites), attrs.ctypes.data,
        len(attrs), PREFIX, len(PREFIX), SUFFIX, len(SUFFIX), buf.ctypes.data, len(buf), C.byref(out))
    assert st == abi.ERR_INVALID_ARGUMENT and out.document_bytes == len(doc)
    # the context stays usable; a reused buffer gives the same document
    again, _ = ctx.encode_dense_evidence(pts, sites, attrs, PREFIX, SUFFIX)
    assert again == doc
    buf = np.zeros(dense.document_bound(len(pts), len(sites), len(attrs), len(PREFIX),
                                        len(SUFFIX)), dtype=np.uint8)
    for _ in range(2):
        view, info2 = ctx.encode_dense_evidence(pts, sites, attrs, PREFIX, SUFFIX, out=buf)
        assert view == doc and info2 == info


@pytest.mark.gpu
def test_encode_refuses_inconsistent_arguments():
    pts, sites, attrs = _evidence(10, 9)
    ctx = dense.Context(0)
    out = abi.DenseDocument()
    buf = np.zeros(dense.document_bound(10, 10, 10, 8, 0), dtype=np.uint8)
    # a prefix length without a prefix, a count without its array
    assert ctx.lib.v3d_encode_dense_evidence(
        ctx.handle, pts.ctypes.data, 10, sites.ctypes.data, 10, attrs.ctypes.data, 10, None, 8,
        None, 0, buf.ctypes.data, len(buf), C.byref(out)) == abi.ERR_INVALID_ARGUMENT
    assert ctx.lib.v3d_encode_dense_evidence(
        ctx.handle, None, 10, sites.ctypes.data, 10, attrs.ctypes.data, 10, None, 0, None, 0,
        buf.ctypes.data, len(buf), C.byref(out)) == abi.ERR_INVALID_ARGUMENT
    doc, _ = ctx.encode_dense_evidence(pts, sites, attrs)
    assert doc == Oracle().encode_dense_evidence(pts, sites, attrs)[0]
