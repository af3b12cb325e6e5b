"""ctypes mirror of include/v3d_dense.h (ABI version 1).

Every structure here has the same field order, types and padding as its C
declaration; ``tests/test_abi.py`` checks the sizes against the compiled
library.
"""
import ctypes as C

ABI_VERSION = 1
SKIP_REASON_BYTES = 320
MAX_PATCH_RADIUS = 4
MAX_SOURCE_VIEWS = 16
MAX_DEPTH_HYPOTHESES = 256

# v3d_status
OK = 0
SKIPPED = 1
ERR_INVALID_ARGUMENT = -1
ERR_CUDA = -2
ERR_OUT_OF_MEMORY = -3
ERR_NO_DEVICE = -4
ERR_INTERNAL = -5

# v3d_pixel_format
PIXEL_RGBA8 = 0
PIXEL_GRAY_F32 = 1
PIXEL_GRAY_F16 = 2
PIXEL_GRAY_BF16 = 3

# v3d_cost / v3d_precision
COST_ZSAD = 0
COST_ZNCC = 1
PRECISION_EXACT64 = 0
PRECISION_FAST32 = 1
PRECISION_FAST32_SUMS32 = 2


class Frame(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("format", C.c_int32),
                ("reserved", C.c_int32), ("data", C.c_void_p)]


class Camera(C.Structure):
    _fields_ = [("frame_index", C.c_uint64), ("rotation", C.c_double * 9),
                ("translation", C.c_double * 3)]


class Profile(C.Structure):
    _fields_ = [("cost", C.c_int32), ("patch_radius", C.c_int32),
                ("depth_hypotheses", C.c_int32), ("max_source_views", C.c_int32),
                ("grid_stride", C.c_int32), ("precision", C.c_int32),
                ("min_reference_contrast", C.c_double), ("max_photometric_error", C.c_double),
                ("min_ambiguity_margin", C.c_double), ("depth_margin_saturation", C.c_double),
                ("error_confidence_scale", C.c_double), ("min_window_variance", C.c_double)]


class Point(C.Structure):
    _fields_ = [("x", C.c_float), ("y", C.c_float), ("z", C.c_float), ("confidence", C.c_float),
                ("r", C.c_uint8), ("g", C.c_uint8), ("b", C.c_uint8), ("pad", C.c_uint8)]


class GridSite(C.Structure):
    _fields_ = [("x", C.c_uint32), ("y", C.c_uint32)]


class PointAttributes(C.Structure):
    _fields_ = [("reciprocal_consistency", C.c_float), ("depth_margin", C.c_float)]


_COUNTERS = [
    "sampled_pixels", "depth_hypotheses", "accepted_points", "surface_completion_proposals",
    "surface_completed_points", "surface_completion_rejected_texture",
    "surface_completion_rejected_cross_view", "surface_completion_rejected_reciprocal",
    "surface_completion_rejected_fusion", "surface_completion_rejected_footprint",
]


class DenseStats(C.Structure):
    _fields_ = ([("attempted", C.c_int32), ("skip_code", C.c_int32),
                 ("skip_reason", C.c_char * SKIP_REASON_BYTES), ("has_skip_reason", C.c_int32),
                 ("has_reference_frame", C.c_int32), ("reference_frame", C.c_uint64),
                 ("source_views", C.c_uint64)]
                + [(n, C.c_uint64) for n in _COUNTERS]
                + [("grid_stride", C.c_uint64), ("grid_border", C.c_uint32), ("pad0", C.c_uint32),
                   ("reciprocal_checked_points", C.c_uint64),
                   ("reciprocal_rejected_points", C.c_uint64),
                   ("reciprocal_consistent_points", C.c_uint64),
                   ("fusion_input_observations", C.c_uint64),
                   ("fusion_rejected_observations", C.c_uint64),
                   ("fusion_rejected_points", C.c_uint64),
                   ("has_median_fusion_observations", C.c_int32),
                   ("median_fusion_observations", C.c_float),
                   ("has_median_supporting_views", C.c_int32),
                   ("median_supporting_views", C.c_float),
                   ("has_median_photometric_error", C.c_int32),
                   ("median_photometric_error", C.c_float),
                   ("has_search_min_depth", C.c_int32), ("search_min_depth", C.c_float),
                   ("has_search_max_depth", C.c_int32), ("search_max_depth", C.c_float),
                   ("has_reference_view_limit", C.c_int32), ("pad1", C.c_int32),
                   ("reference_view_limit", C.c_uint64)])


class ReferenceAttempt(C.Structure):
    _fields_ = [("reference_frame", C.c_uint64), ("attempted", C.c_int32),
                ("accepted", C.c_int32), ("has_skip_reason", C.c_int32), ("pad0", C.c_int32),
                ("skip_reason", C.c_char * SKIP_REASON_BYTES),
                ("sampled_pixels", C.c_uint64), ("accepted_points", C.c_uint64),
                ("reciprocal_checked_points", C.c_uint64),
                ("reciprocal_rejected_points", C.c_uint64),
                ("reciprocal_consistent_points", C.c_uint64),
                ("surface_completion_proposals", C.c_uint64),
                ("surface_completed_points", C.c_uint64),
                ("surface_completion_rejected_texture", C.c_uint64),
                ("surface_completion_rejected_cross_view", C.c_uint64),
                ("surface_completion_rejected_reciprocal", C.c_uint64),
                ("surface_completion_rejected_fusion", C.c_uint64),
                ("surface_completion_rejected_footprint", C.c_uint64)]


class ReferencePatch(C.Structure):
    _fields_ = [("reference_frame", C.c_uint64), ("n_source_frames", C.c_uint64),
                ("source_frames", C.POINTER(C.c_uint64)), ("primary_start", C.c_uint64),
                ("primary_points", C.c_uint64), ("completion_start", C.c_uint64),
                ("completed_points", C.c_uint64), ("sampled_pixels", C.c_uint64),
                ("accepted_points", C.c_uint64), ("reciprocal_consistent_points", C.c_uint64),
                ("grid_stride", C.c_uint64), ("grid_border", C.c_uint32),
                ("has_search_min_depth", C.c_int32), ("search_min_depth", C.c_float),
                ("has_search_max_depth", C.c_int32), ("search_max_depth", C.c_float),
                ("pad0", C.c_int32)]


class DenseResult(C.Structure):
    _fields_ = [("stats", DenseStats), ("n_source_frames", C.c_uint64),
                ("source_frames", C.POINTER(C.c_uint64)), ("n_points", C.c_uint64),
                ("points", C.POINTER(Point)), ("grid_sites", C.POINTER(GridSite)),
                ("point_attributes", C.POINTER(PointAttributes)),
                ("n_reference_frames", C.c_uint64), ("reference_frames", C.POINTER(C.c_uint64)),
                ("n_attempts", C.c_uint64), ("attempts", C.POINTER(ReferenceAttempt)),
                ("n_patches", C.c_uint64), ("patches", C.POINTER(ReferencePatch)),
                ("internal", C.c_void_p)]


class MeshTriangle(C.Structure):
    _fields_ = [("a", C.c_uint64), ("b", C.c_uint64), ("c", C.c_uint64),
                ("confidence", C.c_float), ("pad", C.c_uint32)]


class MeshStats(C.Structure):
    _fields_ = [("attempted", C.c_int32), ("has_skip_reason", C.c_int32),
                ("skip_reason", C.c_char * SKIP_REASON_BYTES),
                ("has_reference_frame", C.c_int32), ("pad0", C.c_int32),
                ("reference_frame", C.c_uint64), ("point_count", C.c_uint64),
                ("grid_vertices", C.c_uint64), ("rejected_grid_vertices", C.c_uint64),
                ("candidate_cells", C.c_uint64), ("candidate_triangles", C.c_uint64),
                ("accepted_triangles", C.c_uint64), ("rejected_discontinuities", C.c_uint64),
                ("rejected_degenerate", C.c_uint64)]


class MeshResult(C.Structure):
    _fields_ = [("stats", MeshStats), ("n_triangles", C.c_uint64),
                ("triangles", C.POINTER(MeshTriangle)), ("n_reference_frames", C.c_uint64),
                ("reference_frames", C.POINTER(C.c_uint64)), ("n_patches", C.c_uint64),
                ("patches", C.POINTER(MeshStats)), ("internal", C.c_void_p)]


class MeshDenseInput(C.Structure):
    _fields_ = [("attempted", C.c_int32), ("has_reference_frame", C.c_int32),
                ("reference_frame", C.c_uint64), ("grid_stride", C.c_uint64),
                ("grid_border", C.c_uint32), ("pad0", C.c_uint32), ("n_patches", C.c_uint64),
                ("patches", C.POINTER(ReferencePatch))]


class SiteRecord(C.Structure):
    _fields_ = [("x", C.c_uint32), ("y", C.c_uint32), ("status", C.c_int32), ("plane", C.c_int32),
                ("support", C.c_int32), ("pad", C.c_int32), ("error", C.c_double),
                ("margin", C.c_double)]


SITE_RECORD_DTYPE = [("x", "<u4"), ("y", "<u4"), ("status", "<i4"), ("plane", "<i4"),
                     ("support", "<i4"), ("pad", "<i4"), ("error", "<f8"), ("margin", "<f8")]

class MeshCounts(C.Structure):
    _fields_ = [("grid_vertices", C.c_uint64), ("candidate_cells", C.c_uint64),
                ("candidate_triangles", C.c_uint64), ("accepted_triangles", C.c_uint64),
                ("rejected_discontinuities", C.c_uint64), ("rejected_degenerate", C.c_uint64)]


class RunInfo(C.Structure):
    _fields_ = [("device_ms", C.c_double), ("kernel_launches", C.c_uint64),
                ("grid_sites", C.c_uint64), ("plane_view_units", C.c_uint64),
                ("sweep_ms", C.c_double), ("reciprocal_ms", C.c_double),
                ("completion_ms", C.c_double), ("reciprocal_plane_evaluations", C.c_uint64),
                ("candidates", C.c_uint64), ("host_plan_ms", C.c_double),
                ("host_enqueue_ms", C.c_double), ("host_wait_ms", C.c_double),
                ("host_assemble_ms", C.c_double), ("mesh_ms", C.c_double),
                ("triangles", C.c_uint64), ("host_block_ms", C.c_double),
                ("host_readback_ms", C.c_double), ("result_bytes", C.c_uint64),
                ("sweep_chunks", C.c_uint64), ("recip_sweep_ms", C.c_double),
                ("recip_prepare_ms", C.c_double), ("sweep_tile_x", C.c_uint64),
                ("merge_stage_ms", C.c_double * 12)]


CANCEL_FN = C.CFUNCTYPE(C.c_int32, C.c_void_p)

class Clip(C.Structure):
    _fields_ = [("frames", C.POINTER(Frame)), ("n_frames", C.c_uint64),
                ("cameras", C.POINTER(Camera)), ("n_cameras", C.c_uint64),
                ("sparse_xyz", C.POINTER(C.c_double)), ("n_sparse", C.c_uint64),
                ("focal", C.c_double), ("camera_indices", C.POINTER(C.c_uint64)),
                ("n_references", C.c_uint64), ("depth_hypotheses", C.c_int32),
                ("max_source_views", C.c_int32)]


class ServerConfig(C.Structure):
    _fields_ = [("device", C.c_int32), ("slots", C.c_int32), ("memory_budget_bytes", C.c_uint64),
                ("max_batch_requests", C.c_uint32), ("meshed", C.c_int32),
                ("fine_grid", C.c_int32), ("profile", Profile)]


class RequestTiming(C.Structure):
    _fields_ = [("queue_ms", C.c_double), ("service_ms", C.c_double), ("total_ms", C.c_double),
                ("batch_requests", C.c_uint64), ("plane_view_units", C.c_uint64)]


TIMEOUT = -6
SHUTDOWN = -7

class FusionStats(C.Structure):
    _fields_ = [("eligible_vertices", C.c_uint64), ("candidate_pairs", C.c_uint64),
                ("rejected_normal_pairs", C.c_uint64), ("rejected_topology_pairs", C.c_uint64),
                ("fused_pairs", C.c_uint64)]


class FusionPair(C.Structure):
    _fields_ = [("first", C.c_uint64), ("second", C.c_uint64)]


class DepthView(C.Structure):
    _fields_ = [("rgba", C.c_void_p), ("depth", C.c_void_p), ("width", C.c_uint32),
                ("height", C.c_uint32), ("camera", Camera)]


class VerificationFunnel(C.Structure):
    _fields_ = [(name, C.c_uint64) for name in (
        "reference_samples", "missing_reference_depth", "insufficient_parallax", "behind_source",
        "outside_source", "missing_source_depth", "depth_disagreement", "color_disagreement",
        "accepted")]


class VerifiedSample(C.Structure):
    _fields_ = [("point", Point), ("site", GridSite), ("source_mask", C.c_uint32)]


class SurfaceTopology(C.Structure):
    _fields_ = [(name, C.c_uint64) for name in (
        "islands", "small_islands", "small_island_triangles", "largest_island_triangles",
        "boundary_edges")]


class MeshingFunnel(C.Structure):
    _fields_ = [(name, C.c_uint64) for name in (
        "depth_views", "meshed_reference_views", "candidate_cells", "rejected_discontinuities",
        "rejected_degenerate", "multiply_verified_samples", "exported_triangles")]


class VerifiedSurfaceRegion(C.Structure):
    _fields_ = [("reference_frame", C.c_uint64), ("first_point", C.c_uint64),
                ("point_count", C.c_uint64), ("source_frames", C.c_uint64 * 4),
                ("n_source_frames", C.c_uint32), ("reserved", C.c_uint32)]


class VerifiedSurface(C.Structure):
    _fields_ = [("verification", VerificationFunnel), ("meshing", MeshingFunnel),
                ("topology", SurfaceTopology), ("dominant_rejection", C.c_int32),
                ("reserved", C.c_int32), ("n_points", C.c_uint64), ("n_triangles", C.c_uint64),
                ("n_regions", C.c_uint64)]


class DenseDocument(C.Structure):
    _fields_ = [("document_bytes", C.c_uint64), ("points_bytes", C.c_uint64),
                ("grid_sites_bytes", C.c_uint64), ("point_attributes_bytes", C.c_uint64),
                ("non_finite", C.c_uint64), ("sha256", C.c_uint8 * 32)]


WORKING_SET_FIELDS = ("frame_bytes", "retry_frame_bytes", "remapped_frame_bytes",
                      "luminance_bytes", "sparse_pipeline_bytes", "dense_sample_bytes",
                      "topology_bytes", "mesh_builder_bytes", "surface_fusion_bytes",
                      "retained_candidate_bytes", "packed_output_bytes", "total_bytes")


class WorkingSetEstimate(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in WORKING_SET_FIELDS]


class DenseBudget(C.Structure):
    _fields_ = [("working_set_estimate", WorkingSetEstimate),
                ("working_set_budget_bytes", C.c_uint64), ("full_working_set_bytes", C.c_uint64),
                ("fine_grid", C.c_int32), ("pad0", C.c_int32), ("reference_views", C.c_uint64)]



class ReferenceCamera(C.Structure):
    _fields_ = [("present", C.c_int32), ("pad_", C.c_int32), ("rotation", C.c_double * 9),
                ("translation", C.c_double * 3)]


class DerivedVertexSource(C.Structure):
    _fields_ = [("point_index", C.c_uint64), ("source_triangle", C.c_uint64),
                ("source_corners", C.c_uint64 * 3), ("barycentric", C.c_double * 3)]


class TriangleSource(C.Structure):
    _fields_ = [("triangle", C.c_uint64), ("corners", C.c_uint64 * 3)]


MERGE_STAT_FIELDS = (
    "fused_pairs", "shared_vertices", "cross_reference_triangles",
    "removed_duplicate_triangles", "remaining_overlap_triangles", "provenance_separated_pairs",
    "trimmed_seam_triangles", "trimmed_seam_area_share", "stitched_seam_triangles",
    "patch_components", "meshed_patches", "max_postings_per_query", "posting_bound_hits",
    "clipping_budget_exhausted", "clipped_overlap_triangles", "clip_pieces", "derived_vertices",
    "unclipped_overlap_triangles", "conformed_triangles", "conformance_failures")


class MergeStats(C.Structure):
    _fields_ = [(f, C.c_double if f == "trimmed_seam_area_share" else C.c_uint64)
                for f in MERGE_STAT_FIELDS]


class MergeResult(C.Structure):
    _fields_ = [("stats", MergeStats),
                ("points", C.c_void_p), ("n_points", C.c_uint64),
                ("triangles", C.c_void_p), ("n_triangles", C.c_uint64),
                ("derived_vertices", C.c_void_p), ("n_derived_vertices", C.c_uint64),
                ("uncalibrated_patch_pairs", C.c_void_p), ("n_uncalibrated_patch_pairs", C.c_uint64),
                ("retained_by_group", C.c_void_p), ("n_retained_by_group", C.c_uint64),
                ("triangle_sources", C.c_void_p), ("n_triangle_sources", C.c_uint64)]


REJECTED = 2
ORIGIN_NONE, ORIGIN_GEOMETRIC, ORIGIN_REVALIDATED, ORIGIN_LEARNED, ORIGIN_GENERATIVE = -1, 0, 1, 2, 3

SKIP_WORKING_SET_BUDGET = 10

STRUCTS = {
    "v3d_reference_camera": ReferenceCamera, "v3d_derived_vertex_source": DerivedVertexSource,
    "v3d_triangle_source": TriangleSource, "v3d_merge_stats": MergeStats,
    "v3d_merge_result": MergeResult,
    "v3d_working_set_estimate": WorkingSetEstimate, "v3d_dense_budget": DenseBudget,
    "v3d_dense_document": DenseDocument,
    "v3d_meshing_funnel": MeshingFunnel, "v3d_verified_surface_region": VerifiedSurfaceRegion,
    "v3d_verified_surface": VerifiedSurface,
    "v3d_surface_topology": SurfaceTopology,
    "v3d_depth_view": DepthView, "v3d_verification_funnel": VerificationFunnel,
    "v3d_verified_sample": VerifiedSample,
    "v3d_fusion_stats": FusionStats, "v3d_fusion_pair": FusionPair,
    "v3d_frame": Frame, "v3d_camera": Camera, "v3d_profile": Profile, "v3d_point": Point,
    "v3d_grid_site": GridSite, "v3d_point_attributes": PointAttributes,
    "v3d_dense_stats": DenseStats, "v3d_reference_attempt": ReferenceAttempt,
    "v3d_reference_patch": ReferencePatch, "v3d_dense_result": DenseResult,
    "v3d_mesh_triangle": MeshTriangle, "v3d_mesh_stats": MeshStats,
    "v3d_mesh_result": MeshResult, "v3d_mesh_dense_input": MeshDenseInput,
    "v3d_site_record": SiteRecord, "v3d_run_info": RunInfo, "v3d_mesh_counts": MeshCounts,
    "v3d_clip": Clip, "v3d_server_config": ServerConfig, "v3d_request_timing": RequestTiming,
}
