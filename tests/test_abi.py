"""The C-ABI library loads on a CPU-only machine and matches include/v3d_dense.h."""
import ctypes as C
import os
import re
import subprocess
import tempfile

import pytest

from v3d import abi, dense, profiles

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "v3d_dense.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(v3d_[a-z0-9_]+)\s*\(", text)) - {"v3d_cancel_fn"})


def test_library_exports_every_declared_function():
    lib = dense.library()
    names = declared_functions()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_struct_layouts_match_the_header():
    src = ['#include <stdio.h>', '#include <stddef.h>', '#include "%s"' % HEADER, "int main(void){"]
    for cname in abi.STRUCTS:
        src.append('printf("%s %%zu\\n", sizeof(%s));' % (cname, cname))
    src.append("return 0;}")
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "sizes.c")
        exe = os.path.join(d, "sizes")
        open(c, "w").write("\n".join(src))
        subprocess.run(["gcc", "-std=c99", c, "-o", exe], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    sizes = dict(line.split() for line in out.strip().splitlines())
    for cname, cls in abi.STRUCTS.items():
        assert int(sizes[cname]) == C.sizeof(cls), cname


def test_abi_version_and_texts():
    lib = dense.library()
    assert lib.v3d_abi_version() == abi.ABI_VERSION
    assert lib.v3d_skip_reason_text(9) == b"dense reconstruction canceled"
    assert b"two accepted registered cameras" in lib.v3d_skip_reason_text(2)
    assert lib.v3d_status_text(-4) == b"no CUDA device"


def test_profile_presets_match_python():
    lib = dense.library()
    p = abi.Profile()
    lib.v3d_profile_reference(C.byref(p))
    q = profiles.reference()
    for name, _ in abi.Profile._fields_:
        assert getattr(p, name) == getattr(q, name), name
    lib.v3d_profile_zncc(C.byref(p), 3, 128, 8, 2)
    q = profiles.zncc(3, 128, 8, 2)
    for name, _ in abi.Profile._fields_:
        assert getattr(p, name) == getattr(q, name), name


def test_grid_stride_matches_the_oracle(oracle):
    for w, h in [(68, 48), (240, 240), (360, 202), (640, 360), (1920, 1080), (16, 16)]:
        for fine in (0, 1):
            assert dense.grid_stride(w, h, fine) == oracle.lib.v3do_grid_stride(w, h, fine)


def test_context_without_device_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    with pytest.raises(dense.V3DError) as e:
        dense.Context(0)
    assert e.value.status == abi.ERR_NO_DEVICE


def test_record_dtypes_match_the_header():
    from v3d import types
    dtypes = {"v3d_point": types.POINT_DTYPE, "v3d_grid_site": types.SITE_DTYPE,
              "v3d_point_attributes": types.ATTR_DTYPE, "v3d_mesh_triangle": types.TRIANGLE_DTYPE,
              "v3d_verified_sample": dense.VERIFIED_DTYPE,
              "v3d_triangle_source": dense.TRIANGLE_SOURCE_DTYPE,
              "v3d_derived_vertex_source": dense.DERIVED_VERTEX_DTYPE}
    src = ['#include <stdio.h>', '#include "%s"' % HEADER, "int main(void){"]
    for cname in dtypes:
        src.append('printf("%s %%zu\\n", sizeof(%s));' % (cname, cname))
    src.append("return 0;}")
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "sizes.c")
        exe = os.path.join(d, "sizes")
        open(c, "w").write("\n".join(src))
        subprocess.run(["gcc", "-std=c99", c, "-o", exe], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    sizes = dict(line.split() for line in out.strip().splitlines())
    for cname, dt in dtypes.items():
        assert int(sizes[cname]) == dt.itemsize, cname
