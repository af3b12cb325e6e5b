"""Profiles of the dense pass (mirrors v3d_profile_reference / v3d_profile_zncc).

``reference()`` is the constant set of dense_legacy.rs:6-21.  ``zncc()`` is the
project-defined profile for windowed ZNCC on [0, 1] images; its thresholds
are in cost units of 1 - ZNCC (0 = identical windows, 1 = uncorrelated).
"""
from . import abi

# Project-defined ZNCC gate values (the reference has no ZNCC cost; these are
# the gates of this build's 1 - ZNCC profile, mirrored in v3d_profile_zncc).
ZNCC_MAX_COST = 0.5             # photometric gate: ZNCC >= 0.5
ZNCC_MIN_MARGIN = 0.002         # ambiguity gate: comparable second must be this much worse
ZNCC_MARGIN_SATURATION = 0.05   # depth_margin = margin / 0.05, clamped to [0, 1]
ZNCC_ERROR_SCALE = 0.2          # error confidence 1 / (1 + cost / 0.2)
ZNCC_MIN_CONTRAST = 14.0 / 255  # window max - min, the reference contrast gate on [0, 1] data
ZNCC_MIN_VARIANCE = 1.0e-5      # per-pixel variance floor of both windows


def reference(precision=abi.PRECISION_EXACT64):
    return abi.Profile(cost=abi.COST_ZSAD, patch_radius=1, depth_hypotheses=24,
                       max_source_views=4, grid_stride=0, precision=precision,
                       min_reference_contrast=14.0, max_photometric_error=18.0,
                       min_ambiguity_margin=1.0, depth_margin_saturation=6.0,
                       error_confidence_scale=8.0, min_window_variance=0.0)


def zncc(patch_radius, depth_hypotheses, max_source_views, grid_stride,
         precision=abi.PRECISION_FAST32):
    return abi.Profile(cost=abi.COST_ZNCC, patch_radius=patch_radius,
                       depth_hypotheses=depth_hypotheses, max_source_views=max_source_views,
                       grid_stride=grid_stride, precision=precision,
                       min_reference_contrast=ZNCC_MIN_CONTRAST,
                       max_photometric_error=ZNCC_MAX_COST,
                       min_ambiguity_margin=ZNCC_MIN_MARGIN,
                       depth_margin_saturation=ZNCC_MARGIN_SATURATION,
                       error_confidence_scale=ZNCC_ERROR_SCALE,
                       min_window_variance=ZNCC_MIN_VARIANCE)


def with_precision(profile, precision):
    p = abi.Profile()
    for name, _ in abi.Profile._fields_:
        setattr(p, name, getattr(profile, name))
    p.precision = precision
    return p
