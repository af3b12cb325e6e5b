"""B200 dense plane-sweep depth pass of video-to-3d (host-side Python API).

The compute path is the CUDA library video-to-3d_b200/lib/libv3d_dense.so,
reached through its C ABI (include/v3d_dense.h).  ``v3d.dense`` mirrors the
Rust API of crates/video-to-3d-core/src/dense*.rs and mesh*.rs.
"""
from . import abi, profiles, types  # noqa: F401
