/*
 * v3d_dense.h — C ABI of the B200 dense plane-sweep depth pass.
 *
 * This library replaces the per-reference dense pass of video-to-3d-core
 * (crates/video-to-3d-core/src/dense_legacy.rs) and the multi-reference
 * driver around it (crates/video-to-3d-core/src/dense.rs), plus the
 * reference-grid triangle gates of crates/video-to-3d-core/src/mesh_legacy.rs
 * and mesh.rs, with CUDA kernels written for sm_100a.  Every entry point takes
 * plain host pointers and sizes; results are returned in library-owned
 * host arrays that the caller releases with the matching *_free function.
 *
 * Reference interfaces replaced (file:line inside crates/video-to-3d-core/src):
 *   v3d_estimate_depth_points_with_control  dense_legacy.rs:149-470
 *   v3d_reconstruct_reference_patches       dense.rs:674-747 (one call per camera, batched)
 *   v3d_estimate_depth_points_limited       dense.rs:250-330
 *   v3d_estimate_depth_points_with_budget_and_control
 *                                           dense.rs:355-420
 *   v3d_estimate_working_set                dense.rs:423-605
 *   v3d_has_distributed_landmarks           dense.rs:165-213
 *   v3d_grid_stride                         dense.rs:215-218
 *   v3d_reconstruct_dense_mesh_samples      mesh_legacy.rs:150-358
 *   v3d_reconstruct_dense_mesh_with_control mesh.rs:74-220
 *   v3d_plan_clips                          dense.rs:165-213, 620-672 (many clips)
 *   v3d_fuse_mutually_supported_vertices    surface_fusion.rs:369-549
 *   v3d_merge_fused_patches_owned           surface_merge.rs:312-353 (with
 *                                           surface_merge_clip.rs, surface_merge_stitch.rs)
 *   v3d_verify_depth_grids                  colmap_surface.rs:175-314, 394-420
 *   v3d_mesh_verified_depth_grids           colmap_surface.rs:380-471
 *   v3d_surface_topology_of                 colmap_surface.rs:125-157
 *   v3d_encode_dense_evidence               reconstruction_stages.rs:287-380
 *   v3d_pack_dense_points, v3d_pack_mesh_triangles
 *                                           crates/video-to-3d-wasm/src/lib.rs:227-326
 *   v3d_sha256                              scene_project.rs:463-465
 *
 * Data contract (mirrors the Rust types bit for bit where a layout exists):
 *   FrameInput  (reconstruction/types.rs:17-21)  -> v3d_frame (RGBA8, tightly packed)
 *   RegisteredCamera (multi_view.rs:85-89)       -> v3d_camera (world->camera R,t;
 *                                                   R stored ROW-major here)
 *   Point3 (reconstruction/types.rs:69-77)       -> v3d_point (20 bytes)
 *   DenseGridSite (dense.rs:57-60)               -> v3d_grid_site
 *   EvidencePointAttributes
 *     (reconstruction_evidence.rs:108-115)       -> v3d_point_attributes
 *   MeshTriangle (mesh_legacy.rs:18-23)          -> v3d_mesh_triangle
 *
 * Errors: the reference never fails, it "skips" with an English reason
 * (dense_legacy.rs:157-236).  A skip is V3D_SKIPPED with stats.skip_code and
 * stats.skip_reason set to the exact reference string.  Negative statuses are
 * errors of this library (bad arguments, CUDA failures) and leave the result
 * zeroed.
 *
 * Threading: a v3d_context owns one CUDA stream and its device buffers; calls
 * on one context are serialised by an internal mutex.  Use one context per
 * host thread for concurrency.
 */
#ifndef V3D_DENSE_H
#define V3D_DENSE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define V3D_ABI_VERSION 1
#define V3D_SKIP_REASON_BYTES 320
#define V3D_MAX_PATCH_RADIUS 4       /* windows up to 9x9 */
#define V3D_MAX_SOURCE_VIEWS 16
#define V3D_MAX_DEPTH_HYPOTHESES 256

typedef enum v3d_status {
    V3D_OK = 0,
    V3D_SKIPPED = 1,                 /* the pass did not run; see stats.skip_code */
    V3D_ERR_INVALID_ARGUMENT = -1,
    V3D_ERR_CUDA = -2,
    V3D_ERR_OUT_OF_MEMORY = -3,
    V3D_ERR_NO_DEVICE = -4,
    V3D_ERR_INTERNAL = -5,
    V3D_ERR_TIMEOUT = -6,            /* v3d_server_wait: the request is not done yet */
    V3D_ERR_SHUTDOWN = -7,           /* the server stopped before running the request */
    V3D_REJECTED = 2                 /* the reference returns Err(message): v3d_last_error */
} v3d_status;

/* Skip reasons of dense_legacy.rs:157-236 and dense.rs, in the order the
 * reference tests them.  v3d_skip_reason_text() returns the exact string. */
typedef enum v3d_skip_code {
    V3D_SKIP_NONE = 0,
    V3D_SKIP_NO_FRAMES = 1,              /* dense_legacy.rs:158 */
    V3D_SKIP_FEWER_THAN_TWO_CAMERAS = 2, /* dense_legacy.rs:161 */
    V3D_SKIP_FEW_SPARSE_LANDMARKS = 3,   /* dense_legacy.rs:164-166 */
    V3D_SKIP_FRAMES_TOO_SMALL = 4,       /* dense_legacy.rs:172 */
    V3D_SKIP_NO_REFERENCE_CAMERA = 5,    /* dense_legacy.rs:188-190 */
    V3D_SKIP_NO_DEPTH_ENVELOPE = 6,      /* dense_legacy.rs:197-199 */
    V3D_SKIP_REFERENCE_FRAME_MISSING = 7,/* dense_legacy.rs:206 */
    V3D_SKIP_NO_SOURCE_VIEW = 8,         /* dense_legacy.rs:233-235 */
    V3D_SKIP_CANCELED = 9,               /* dense_legacy.rs:274 */
    V3D_SKIP_WORKING_SET_BUDGET = 10     /* dense.rs:385-402; the reason carries the sizes */
} v3d_skip_code;

typedef enum v3d_pixel_format {
    V3D_PIXEL_RGBA8 = 0,      /* width*height*4 bytes; luma = (77R+150G+29B)>>8 (dense_legacy.rs:1147-1157) */
    V3D_PIXEL_GRAY_F32 = 1,   /* width*height floats in [0,1] */
    V3D_PIXEL_GRAY_F16 = 2,   /* width*height IEEE binary16 */
    V3D_PIXEL_GRAY_BF16 = 3   /* width*height bfloat16 */
} v3d_pixel_format;

/* A frame holds fewer than 2^32 pixels (width * height). */
typedef struct v3d_frame {
    uint32_t width;
    uint32_t height;
    int32_t format;           /* v3d_pixel_format */
    int32_t reserved;
    const void* data;         /* host pointer, tightly packed rows */
} v3d_frame;

typedef struct v3d_camera {
    uint64_t frame_index;     /* index into the frames array */
    double rotation[9];       /* world->camera rotation, row-major R[row*3+col] */
    double translation[3];    /* world->camera translation t: x_cam = R x_world + t */
} v3d_camera;

typedef enum v3d_cost {
    V3D_COST_ZSAD = 0,        /* mean |(r-mean r)-(s-mean s)| (dense_legacy.rs:1032-1095) */
    V3D_COST_ZNCC = 1         /* 1 - zero-mean normalised cross-correlation */
} v3d_cost;

typedef enum v3d_precision {
    V3D_PRECISION_EXACT64 = 0,/* every tap in f64 with the reference's unproject/project formulas */
    V3D_PRECISION_FAST32 = 1, /* per-plane homographies composed in f64, taps in f32; the
                               * box-filtered depth sweep forms its window sums in f64, every
                               * other window cost sums in f32 */
    V3D_PRECISION_FAST32_SUMS32 = 2 /* FAST32 with the box-filtered sweep's window sums in
                                     * f32 too, on values shifted by the tile's centre texel */
} v3d_precision;

/* Hot-path constants.  v3d_profile_reference() fills dense_legacy.rs:6-21;
 * every other value is a project-defined profile (see the docs). */
typedef struct v3d_profile {
    int32_t cost;                     /* v3d_cost */
    int32_t patch_radius;             /* PATCH_RADIUS, window = 2r+1, 1..V3D_MAX_PATCH_RADIUS */
    int32_t depth_hypotheses;         /* DEPTH_HYPOTHESES, 2..V3D_MAX_DEPTH_HYPOTHESES */
    int32_t max_source_views;         /* MAX_SOURCE_VIEWS, 1..V3D_MAX_SOURCE_VIEWS */
    int32_t grid_stride;              /* 0: the reference grid_stride() rule; >0: fixed stride */
    int32_t precision;                /* v3d_precision */
    double min_reference_contrast;    /* MIN_REFERENCE_CONTRAST, image units */
    double max_photometric_error;     /* MAX_PHOTOMETRIC_ERROR, cost units */
    double min_ambiguity_margin;      /* MIN_AMBIGUITY_MARGIN, cost units */
    double depth_margin_saturation;   /* DEPTH_MARGIN_SATURATION, cost units */
    double error_confidence_scale;    /* 8.0 in 1/(1+error/8) (dense_legacy.rs:390) */
    double min_window_variance;       /* ZNCC: per-pixel variance floor of both windows */
} v3d_profile;

/* Output records, laid out like the Rust structs. */
typedef struct v3d_point {
    float x, y, z, confidence;
    uint8_t r, g, b, pad;
} v3d_point;

typedef struct v3d_grid_site {
    uint32_t x, y;
} v3d_grid_site;

typedef struct v3d_point_attributes {
    float reciprocal_consistency;
    float depth_margin;
} v3d_point_attributes;

/* DenseStats (dense_legacy.rs:23-53; dense.rs:99-139 adds the fields after
 * search_max_depth).  Option<T> fields carry a has_* flag. */
typedef struct v3d_dense_stats {
    int32_t attempted;
    int32_t skip_code;                        /* v3d_skip_code, or -1 for a reason with no code */
    char skip_reason[V3D_SKIP_REASON_BYTES];  /* "" when none */
    int32_t has_skip_reason;
    int32_t has_reference_frame;
    uint64_t reference_frame;
    uint64_t source_views;
    uint64_t sampled_pixels;
    uint64_t depth_hypotheses;
    uint64_t accepted_points;
    uint64_t surface_completion_proposals;
    uint64_t surface_completed_points;
    uint64_t surface_completion_rejected_texture;
    uint64_t surface_completion_rejected_cross_view;
    uint64_t surface_completion_rejected_reciprocal;
    uint64_t surface_completion_rejected_fusion;
    uint64_t surface_completion_rejected_footprint;
    uint64_t grid_stride;
    uint32_t grid_border;
    uint32_t pad0;
    uint64_t reciprocal_checked_points;
    uint64_t reciprocal_rejected_points;
    uint64_t reciprocal_consistent_points;
    uint64_t fusion_input_observations;
    uint64_t fusion_rejected_observations;
    uint64_t fusion_rejected_points;
    int32_t has_median_fusion_observations;
    float median_fusion_observations;
    int32_t has_median_supporting_views;
    float median_supporting_views;
    int32_t has_median_photometric_error;
    float median_photometric_error;
    int32_t has_search_min_depth;
    float search_min_depth;
    int32_t has_search_max_depth;
    float search_max_depth;
    /* dense.rs:136-138 (reference_view_limit is decided by the Rust budget plan) */
    int32_t has_reference_view_limit;
    int32_t pad1;
    uint64_t reference_view_limit;
} v3d_dense_stats;

/* DenseReferenceAttemptStats (dense.rs:63-80). */
typedef struct v3d_reference_attempt {
    uint64_t reference_frame;
    int32_t attempted;
    int32_t accepted;
    int32_t has_skip_reason;
    int32_t pad0;
    char skip_reason[V3D_SKIP_REASON_BYTES];
    uint64_t sampled_pixels;
    uint64_t accepted_points;
    uint64_t reciprocal_checked_points;
    uint64_t reciprocal_rejected_points;
    uint64_t reciprocal_consistent_points;
    uint64_t surface_completion_proposals;
    uint64_t surface_completed_points;
    uint64_t surface_completion_rejected_texture;
    uint64_t surface_completion_rejected_cross_view;
    uint64_t surface_completion_rejected_reciprocal;
    uint64_t surface_completion_rejected_fusion;
    uint64_t surface_completion_rejected_footprint;
} v3d_reference_attempt;

/* DenseReferencePatchStats (dense.rs:83-97). */
typedef struct v3d_reference_patch {
    uint64_t reference_frame;
    uint64_t n_source_frames;
    const uint64_t* source_frames;
    uint64_t primary_start;
    uint64_t primary_points;
    uint64_t completion_start;
    uint64_t completed_points;
    uint64_t sampled_pixels;
    uint64_t accepted_points;
    uint64_t reciprocal_consistent_points;
    uint64_t grid_stride;
    uint32_t grid_border;
    int32_t has_search_min_depth;
    float search_min_depth;
    int32_t has_search_max_depth;
    float search_max_depth;
    int32_t pad0;
} v3d_reference_patch;

/* DenseAnalysis (dense_legacy.rs:62-68; dense.rs:142-148).  All arrays are
 * owned by the library; release with v3d_dense_result_free(). */
typedef struct v3d_dense_result {
    v3d_dense_stats stats;
    uint64_t n_source_frames;
    uint64_t* source_frames;
    uint64_t n_points;
    v3d_point* points;
    v3d_grid_site* grid_sites;
    v3d_point_attributes* point_attributes;
    /* Multi-reference fields of dense.rs (empty for the per-reference pass). */
    uint64_t n_reference_frames;
    uint64_t* reference_frames;
    uint64_t n_attempts;
    v3d_reference_attempt* attempts;
    uint64_t n_patches;
    v3d_reference_patch* patches;
    void* internal;
} v3d_dense_result;

/* MeshTriangle (mesh_legacy.rs:18-23). */
typedef struct v3d_mesh_triangle {
    uint64_t a, b, c;
    float confidence;
    uint32_t pad;
} v3d_mesh_triangle;

/* MeshStats (mesh_legacy.rs:26-37) and MeshReferencePatchStats (mesh.rs:15-27). */
typedef struct v3d_mesh_stats {
    int32_t attempted;
    int32_t has_skip_reason;
    char skip_reason[V3D_SKIP_REASON_BYTES];
    int32_t has_reference_frame;
    int32_t pad0;
    uint64_t reference_frame;
    uint64_t point_count;             /* mesh.rs patch stats only */
    uint64_t grid_vertices;
    uint64_t rejected_grid_vertices;
    uint64_t candidate_cells;
    uint64_t candidate_triangles;
    uint64_t accepted_triangles;
    uint64_t rejected_discontinuities;
    uint64_t rejected_degenerate;
} v3d_mesh_stats;

typedef struct v3d_mesh_result {
    v3d_mesh_stats stats;
    uint64_t n_triangles;
    v3d_mesh_triangle* triangles;
    uint64_t n_reference_frames;
    uint64_t* reference_frames;
    uint64_t n_patches;
    v3d_mesh_stats* patches;
    void* internal;
} v3d_mesh_result;

/* The subset of DenseStats the mesh stage reads (mesh_legacy.rs:160-199;
 * mesh.rs:84-144). */
typedef struct v3d_mesh_dense_input {
    int32_t attempted;
    int32_t has_reference_frame;
    uint64_t reference_frame;
    uint64_t grid_stride;
    uint32_t grid_border;
    uint32_t pad0;
    uint64_t n_patches;                  /* 0: single legacy call (mesh.rs:84-99) */
    const v3d_reference_patch* patches;  /* reference patches of a multi-reference run */
} v3d_mesh_dense_input;

/* Cooperative cancellation (reconstruction/control.rs:35-57): polled where the
 * reference polls; nonzero means canceled, and cancellation is sticky. */
typedef int32_t (*v3d_cancel_fn)(void* user_data);

typedef struct v3d_context v3d_context;

/* ---- library / context ------------------------------------------------- */
int32_t v3d_abi_version(void);
const char* v3d_status_text(int32_t status);
const char* v3d_skip_reason_text(int32_t skip_code);
const char* v3d_last_error(const v3d_context* ctx);

/* Create a context on CUDA device `device`: one stream plus growable device
 * arenas sized on first use.  Returns V3D_ERR_NO_DEVICE without a GPU (there
 * is no CPU fallback). */
int32_t v3d_context_create(int32_t device, v3d_context** out);
void v3d_context_destroy(v3d_context* ctx);

/* Profile presets: the reference constants (dense_legacy.rs:6-21), and the
 * project-defined ZNCC profile for the given window radius, plane count,
 * source-view cap and fixed grid stride. */
void v3d_profile_reference(v3d_profile* out);
void v3d_profile_zncc(v3d_profile* out, int32_t patch_radius, int32_t depth_hypotheses,
                      int32_t max_source_views, int32_t grid_stride);

/* grid_stride (dense.rs:215-218). */
uint64_t v3d_grid_stride(uint32_t width, uint32_t height, int32_t fine_grid);

/* ---- dense pass ---------------------------------------------------------- */

/* legacy::estimate_depth_points_with_control (dense_legacy.rs:149-470):
 * one reference pass — reference and source selection, the depth sweep with
 * photometric and ambiguity gates, the reciprocal source-view check, fusion,
 * confidence and two surface-completion passes.  `sparse_xyz` holds
 * n_sparse world points as x,y,z doubles. */
int32_t v3d_estimate_depth_points_with_control(
    v3d_context* ctx,
    const v3d_frame* frames, uint64_t n_frames,
    const v3d_camera* cameras, uint64_t n_cameras,
    const double* sparse_xyz, uint64_t n_sparse,
    double focal, int32_t fine_grid,
    const v3d_profile* profile,
    v3d_cancel_fn cancel, void* cancel_user,
    v3d_dense_result* out);

/* reconstruct_reference_patch (dense.rs:674-747) for each camera index in
 * `camera_indices`, batched on the device.  out[i] receives the remapped
 * pass of camera_indices[i]; `present[i]` is set to 0 where the reference
 * returns None (fewer than 8 landmarks visible in that camera), else 1.
 * Frames are uploaded once per call and shared by every reference. */
int32_t v3d_reconstruct_reference_patches(
    v3d_context* ctx,
    const v3d_frame* frames, uint64_t n_frames,
    const v3d_camera* cameras, uint64_t n_cameras,
    const double* sparse_xyz, uint64_t n_sparse,
    double focal, int32_t fine_grid,
    const v3d_profile* profile,
    const uint64_t* camera_indices, uint64_t n_references,
    v3d_cancel_fn cancel, void* cancel_user,
    v3d_dense_result* out, int32_t* present);

/* v3d_reconstruct_reference_patches followed, on the device and in the same
 * batch, by the reference-grid triangle gates of every patch
 * (mesh_legacy.rs:150-358 over the patch's points with its reference camera,
 * as mesh.rs:100-207 runs them per patch).  mesh_out[i] holds patch i's
 * triangles (indices into out[i].points) and statistics; width and height are
 * the reference frame's. */
int32_t v3d_reconstruct_reference_patches_meshed(
    v3d_context* ctx,
    const v3d_frame* frames, uint64_t n_frames,
    const v3d_camera* cameras, uint64_t n_cameras,
    const double* sparse_xyz, uint64_t n_sparse,
    double focal, int32_t fine_grid,
    const v3d_profile* profile,
    const uint64_t* camera_indices, uint64_t n_references,
    v3d_cancel_fn cancel, void* cancel_user,
    v3d_dense_result* out, v3d_mesh_result* mesh_out, int32_t* present);

/* One clip of v3d_reconstruct_clips: its frames, cameras, landmarks and focal
 * length, the cameras to reconstruct as references, and its own hypothesis
 * count and source-view limit (0 takes the profile's). */
typedef struct v3d_clip {
    const v3d_frame* frames;
    uint64_t n_frames;
    const v3d_camera* cameras;
    uint64_t n_cameras;
    const double* sparse_xyz;
    uint64_t n_sparse;
    double focal;
    const uint64_t* camera_indices;
    uint64_t n_references;
    int32_t depth_hypotheses;
    int32_t max_source_views;
} v3d_clip;

/* The multi-reference planner's two landmark scans for many clips at once:
 * reference_candidate_order (dense.rs:620-672: cameras with at least 8
 * visible landmarks, the most-visible first, the rest farthest-from-it first)
 * and has_distributed_landmarks (dense.rs:165-213: a majority of cameras see
 * 2 or more landmarks in 8 of their 4x4 image tiles).  Every (camera,
 * landmark) projection of every clip runs in one device pass; the orders are
 * then sorted on the host exactly as the reference sorts them.  clips uses
 * frames (their sizes), cameras, sparse_xyz and focal of each v3d_clip.
 * orders needs the sum of the clips' n_cameras entries: clip k's order (camera
 * indices) starts at the sum of the earlier clips' n_cameras, and
 * order_counts[k] is its length; distributed[k] is 1 when the clip's
 * landmarks are distributed. */
int32_t v3d_plan_clips(v3d_context* ctx, const v3d_clip* clips, uint64_t n_clips,
                       uint64_t* orders, uint64_t* order_counts, int32_t* distributed);

/* reconstruct_reference_patch (dense.rs:674-747) for the references of many
 * clips of uneven size, as one device batch: every kernel runs once over the
 * references of all clips.  The reference has no multi-clip call; per clip
 * the results equal v3d_reconstruct_reference_patches(_meshed) with that
 * clip's inputs and profile.  out, present and (when not NULL) mesh_out hold
 * the references clip by clip, in each clip's camera_indices order.  All
 * frames of a call share one pixel format; the profile's cost, window,
 * stride, precision and gates apply to every clip. */
int32_t v3d_reconstruct_clips(
    v3d_context* ctx,
    const v3d_clip* clips, uint64_t n_clips,
    int32_t fine_grid, const v3d_profile* profile,
    v3d_cancel_fn cancel, void* cancel_user,
    v3d_dense_result* out, v3d_mesh_result* mesh_out, int32_t* present);

/* estimate_depth_points_limited (dense.rs:250-330): the multi-reference plan
 * (at most 6 attempts, `reference_views` accepted patches), the legacy
 * fallback, attempt merging and patch concatenation.  `omitted_references`
 * receives the second tuple element (a further candidate remained). */
int32_t v3d_estimate_depth_points_limited(
    v3d_context* ctx,
    const v3d_frame* frames, uint64_t n_frames,
    const v3d_camera* cameras, uint64_t n_cameras,
    const double* sparse_xyz, uint64_t n_sparse,
    double focal, uint64_t reference_views, int32_t fine_grid,
    const v3d_profile* profile,
    v3d_cancel_fn cancel, void* cancel_user,
    v3d_dense_result* out, int32_t* omitted_references);

/* ---- the working-set budget (dense.rs:354-605) ----------------------------
 * Pure host arithmetic: no context, no device. */

/* DenseWorkingSetEstimate (dense.rs:15-28). */
typedef struct v3d_working_set_estimate {
    uint64_t frame_bytes;
    uint64_t retry_frame_bytes;
    uint64_t remapped_frame_bytes;
    uint64_t luminance_bytes;
    uint64_t sparse_pipeline_bytes;
    uint64_t dense_sample_bytes;
    uint64_t topology_bytes;
    uint64_t mesh_builder_bytes;
    uint64_t surface_fusion_bytes;  /* peak of surface fusion and the connected-surface merge */
    uint64_t retained_candidate_bytes;
    uint64_t packed_output_bytes;
    uint64_t total_bytes;
} v3d_working_set_estimate;

/* The budget fields of DenseStats (dense.rs:133-136) and the plan that ran. */
typedef struct v3d_dense_budget {
    v3d_working_set_estimate working_set_estimate;
    uint64_t working_set_budget_bytes;
    uint64_t full_working_set_bytes;
    int32_t fine_grid;         /* the grid the plan ran on */
    int32_t pad0;
    uint64_t reference_views;  /* the plan's reference-view limit; 0 when the budget skipped */
} v3d_dense_budget;

/* estimate_working_set (dense.rs:423-605): the conservative bytes the Rust
 * process holds at the dense stage's peak with at most `reference_views`
 * reference patches, from the frames, the sparse-stage options (max_features,
 * descriptor_radius) and the grid.  Sizes are those of the x86-64 Rust
 * layouts of the containers the reference charges.  A frame counts its bytes
 * as handed in (the reference's RGBA frames: width x height x 4).
 * Saturating, like the reference. */
int32_t v3d_estimate_working_set(
    const v3d_frame* frames, uint64_t n_frames,
    uint64_t max_features, uint32_t descriptor_radius,
    uint64_t reference_views, int32_t fine_grid,
    v3d_working_set_estimate* out);

/* estimate_depth_points_with_budget_and_control (dense.rs:355-420): picks the
 * fine grid (when finer spacing exists, the landmarks are distributed and the
 * three-view fine plan fits), else the most reference views (3, 2, 1) whose
 * estimate fits `working_set_budget_bytes`, runs
 * v3d_estimate_depth_points_limited with that plan and reports the plan in
 * *budget.  When not even one view fits, returns V3D_SKIPPED with skip code
 * V3D_SKIP_WORKING_SET_BUDGET and the reference's message ("estimated dense
 * working set of N bytes exceeds the configured B byte budget even for one
 * reference view").  stats.reference_view_limit is set when the plan kept
 * fewer than 3 views and a further reference candidate remained.  The cancel
 * callback is sticky across the landmark test and the pass. */
int32_t v3d_estimate_depth_points_with_budget_and_control(
    v3d_context* ctx,
    const v3d_frame* frames, uint64_t n_frames,
    const v3d_camera* cameras, uint64_t n_cameras,
    const double* sparse_xyz, uint64_t n_sparse,
    double focal, uint64_t working_set_budget_bytes,
    uint64_t max_features, uint32_t descriptor_radius,
    const v3d_profile* profile,
    v3d_cancel_fn cancel, void* cancel_user,
    v3d_dense_result* out, v3d_dense_budget* budget);

/* has_distributed_landmarks (dense.rs:165-213), polling `cancel` once per
 * 256-landmark chunk like the reference. */
int32_t v3d_has_distributed_landmarks(
    const v3d_frame* frames, uint64_t n_frames,
    const v3d_camera* cameras, uint64_t n_cameras,
    const double* sparse_xyz, uint64_t n_sparse,
    double focal, v3d_cancel_fn cancel, void* cancel_user);

void v3d_dense_result_free(v3d_dense_result* result);

/* ---- diagnostics ----------------------------------------------------------- */

/* Device-side account of the last dense call on `ctx`: the CUDA-event time of
 * its kernels (uploads and read-back excluded) and how many kernels it
 * launched.  No counterpart in the reference. */
typedef struct v3d_run_info {
    double device_ms;
    uint64_t kernel_launches;
    uint64_t grid_sites;      /* all grid sites of the references that ran */
    uint64_t plane_view_units;/* sum over references of sites x planes x source views */
    double sweep_ms;          /* depth sweep kernel */
    double reciprocal_ms;     /* the primary reciprocal-check launch */
    double completion_ms;     /* both surface-completion passes, reciprocal included */
    uint64_t reciprocal_plane_evaluations; /* single-view hypotheses evaluated, all passes */
    uint64_t candidates;      /* primary + completion candidates checked */
    double host_plan_ms;      /* host planning of every reference */
    double host_enqueue_ms;   /* staging uploads, enqueueing every kernel, and (in the
                               * _meshed call) the mid-batch read of the per-reference
                               * point counts that size the mesh stage */
    double host_wait_ms;      /* waiting for the device, read-back included */
    double host_assemble_ms;  /* splitting the point pool per reference, medians */
    double mesh_ms;           /* device mesh stage of the _meshed call */
    uint64_t triangles;       /* accepted triangles of the _meshed call */
    double host_block_ms;     /* acquiring the pinned result block (within host_wait_ms) */
    double host_readback_ms;  /* result copies into that block (within host_wait_ms) */
    uint64_t result_bytes;    /* bytes of that block the results occupy */
    uint64_t sweep_chunks;    /* plane chunks of the box-filtered sweep (1: none) */
    double recip_sweep_ms;    /* the single-view reciprocal sweep kernel, all its launches
                               * (primary candidates and both completion passes) */
    double recip_prepare_ms;  /* the reciprocal prologue and its pair list, all launches */
    uint64_t sweep_tile_x;    /* tile width of the box-filtered sweep: 32 (32x8 sites) or 16
                               * (16x16); 0 when the sweep ran a warp per site */
    /* the last v3d_merge_fused_patches_owned call, wall milliseconds by stage:
     * [0] components, pairs, re-index, geometry and the device upload;
     * [1] the device lookups (job lists, launches, transfers);
     * [2] the per-candidate decisions and the 3D fallback;
     * [3] footprints (projection, grid, upload) and the kept-triangle grid;
     * [4] seam stitching; [5] overlap clips; [6] the edge-conforming split;
     * [7] assembly and topology; within them: [8] the depth-scale samples
     * (of [1]), [9] stitching's retained edges, [10] its seams, [11] its
     * greedy pass (of [4]) */
    double merge_stage_ms[12];
} v3d_run_info;

int32_t v3d_last_run_info(const v3d_context* ctx, v3d_run_info* out);

/* ---- geometric depth-grid verification (colmap_surface.rs:158-314) --------
 * The alternate dense provider's gate: every reference depth-grid sample is
 * checked against each of its source views (parallax, visibility, an
 * independent source depth within 2 %, colour within 105 summed RGB levels),
 * and the samples any source verified are merged into one reference grid. */

/* One view of external geometric depth (colmap_surface.rs:24-29, 158-173):
 * its RGBA8 frame, its depth grid of ceil(width / stride) x ceil(height /
 * stride) f32 samples in row-major order (0 = no depth) and its camera. */
typedef struct v3d_depth_view {
    const uint8_t* rgba;
    const float* depth;
    uint32_t width, height;
    v3d_camera camera;
} v3d_depth_view;

/* VerificationFunnel (colmap_surface.rs:56-66). */
typedef struct v3d_verification_funnel {
    uint64_t reference_samples;
    uint64_t missing_reference_depth;
    uint64_t insufficient_parallax;
    uint64_t behind_source;
    uint64_t outside_source;
    uint64_t missing_source_depth;
    uint64_t depth_disagreement;
    uint64_t color_disagreement;
    uint64_t accepted;
} v3d_verification_funnel;

/* VerifiedSample (colmap_surface.rs:277-283): the reference sample's point
 * (world position from the reference depth, the reference colour, the
 * strongest agreement of its verifying sources as confidence), its grid site,
 * and bit j set when the reference's j-th source view verified it. */
typedef struct v3d_verified_sample {
    v3d_point point;
    v3d_grid_site site;
    uint32_t source_mask;
} v3d_verified_sample;

/* verify_patch (colmap_surface.rs:175-275) of every reference against each of
 * its sources, then verified_union (colmap_surface.rs:289-314), for many
 * references in one device pass.  views [n_views] share one frame size;
 * reference_views [n_references] and source_views [n_references x 4] index
 * into views (sources in the grid's order, -1 = none; at most 4 per reference,
 * as the export accepts).  stride and reference_stride are the grid spacing
 * and the meshed spacing (a multiple of it).  samples get each reference's
 * verified samples in grid row-major order, reference after reference;
 * sample_offsets [n_references + 1] their ranges; capacity is the room in
 * samples (V3D_ERR_INVALID_ARGUMENT, and nothing written, when the samples
 * would not fit: n_references * ceil(width / reference_stride) *
 * ceil(height / reference_stride) always does).  funnel gets the counts summed
 * over every (reference, source) pair, as the export's diagnostics sum them. */
int32_t v3d_verify_depth_grids(
    v3d_context* ctx, const v3d_depth_view* views, uint64_t n_views,
    const uint32_t* reference_views, uint64_t n_references, const int32_t* source_views,
    uint32_t stride, uint32_t reference_stride, double focal,
    v3d_verified_sample* samples, uint64_t capacity, uint64_t* sample_offsets,
    v3d_verification_funnel* funnel);

/* SurfaceTopology (colmap_surface.rs:114-121): connected islands of a mesh
 * (vertices joined by triangle edges; islands counted over the triangles),
 * those with fewer than 32 triangles and their triangles, the largest
 * island's triangles, and the edges used by exactly one triangle. */
typedef struct v3d_surface_topology {
    uint64_t islands;
    uint64_t small_islands;
    uint64_t small_island_triangles;
    uint64_t largest_island_triangles;
    uint64_t boundary_edges;
} v3d_surface_topology;

/* surface_topology (colmap_surface.rs:125-157) on the device, for the export's
 * diagnostics.  Every index must be below vertex_count (the reference panics
 * otherwise; here V3D_ERR_INVALID_ARGUMENT); fewer than 2^32 vertices and
 * 2^30 triangles. */
int32_t v3d_surface_topology_of(v3d_context* ctx, const v3d_mesh_triangle* triangles,
                                uint64_t n_triangles, uint64_t vertex_count,
                                v3d_surface_topology* out);

/* MeshingFunnel (colmap_surface.rs:98-109). */
typedef struct v3d_meshing_funnel {
    uint64_t depth_views;
    uint64_t meshed_reference_views;
    uint64_t candidate_cells;
    uint64_t rejected_discontinuities;
    uint64_t rejected_degenerate;
    uint64_t multiply_verified_samples;
    uint64_t exported_triangles;
} v3d_meshing_funnel;

/* One exported SurfaceEvidenceRegion (colmap_surface.rs:448-455): the points
 * a meshed reference view added, [first_point, first_point + point_count),
 * and the source frames that verified them (frame_index of the source views,
 * ascending). */
typedef struct v3d_verified_surface_region {
    uint64_t reference_frame;
    uint64_t first_point;
    uint64_t point_count;
    uint64_t source_frames[4];
    uint32_t n_source_frames;
    uint32_t reserved;
} v3d_verified_surface_region;

/* SurfaceDiagnostics (colmap_surface.rs:44-53) and the export's counts. */
typedef struct v3d_verified_surface {
    v3d_verification_funnel verification;
    v3d_meshing_funnel meshing;
    v3d_surface_topology topology;
    int32_t dominant_rejection;  /* 1..7: the funnel field after reference_samples, in order; 0 none */
    int32_t reserved;
    uint64_t n_points, n_triangles, n_regions;
} v3d_verified_surface;

/* Capacities that always hold the outputs of v3d_mesh_verified_depth_grids. */
void v3d_verified_surface_bounds(uint32_t width, uint32_t height, uint32_t reference_stride,
                                 uint64_t n_references, uint64_t* max_points,
                                 uint64_t* max_triangles);

/* The geometric part of the COLMAP export (colmap_surface.rs:380-471, up to
 * the material bake and GLB encoding): for each reference in order, every
 * source is verified and the results united (as v3d_verify_depth_grids), the
 * union is meshed with the reference-grid gates at reference_stride (mesh.rs:
 * 74-220 over one patch, grid border 0, the reference view's camera), and the
 * vertices the triangles use are appended in the order the triangles first
 * use them; references that add no triangle are left out.  Then the
 * topology of the whole mesh and the dominant rejection.  All of it runs on
 * the device; the host reads counts between the three stages.  Views must
 * have distinct camera frame indices.  points and sites receive n_points
 * entries, triangles n_triangles (indices into points), regions n_regions
 * (at most n_references).  Returns V3D_SKIPPED with the reference's message
 * in v3d_last_error when no triangle is exported. */
int32_t v3d_mesh_verified_depth_grids(
    v3d_context* ctx, const v3d_depth_view* views, uint64_t n_views,
    const uint32_t* reference_views, uint64_t n_references, const int32_t* source_views,
    uint32_t stride, uint32_t reference_stride, double focal,
    v3d_point* points, v3d_grid_site* sites, uint64_t point_capacity,
    v3d_mesh_triangle* triangles, uint64_t triangle_capacity,
    v3d_verified_surface_region* regions, v3d_verified_surface* out);

/* ---- cross-reference surface fusion (surface_fusion.rs:356-852) ---------
 * The first step of surface consolidation after the grid mesh
 * (consolidate_surface_recording_with_control, surface_fusion.rs:128-231,
 * called from reconstruction_stages.rs:874): mesh vertices of different
 * camera-support groups that are mutually nearest within the local and global
 * edge-scale bounds, with aligned vertex normals, move to their
 * confidence-weighted mean unless the complete move set would weaken a
 * triangle incident to a moved vertex. */

/* FusionStats (surface_fusion.rs:17-24). */
typedef struct v3d_fusion_stats {
    uint64_t eligible_vertices;
    uint64_t candidate_pairs;
    uint64_t rejected_normal_pairs;
    uint64_t rejected_topology_pairs;
    uint64_t fused_pairs;
} v3d_fusion_stats;

/* One accepted pair (FusionOutcome::pairs, surface_fusion.rs:27-32):
 * first < second, both moved to one position. */
typedef struct v3d_fusion_pair {
    uint64_t first, second;
} v3d_fusion_pair;

/* fuse_mutually_supported_vertices_with_control (surface_fusion.rs:369-549),
 * replacing that function behind the same inputs and outputs.  points
 * [n_points] are moved in place; triangles [n_triangles] index into them;
 * membership [n_points] is each point's camera-support group as
 * evidence_support_membership (surface_fusion.rs:316-345) assigns it,
 * negative for none.  pairs needs room for n_points / 2 entries and moved for
 * n_points; *n_pairs and *n_moved get their counts (moved indices ascending:
 * FusionOutcome::moved_indices).  cancel (may be NULL) is polled between the
 * stages; a canceled call returns V3D_OK with zero stats, no pairs and the
 * points unchanged, the reference's FusionOutcome::default().  Device work
 * on the context's stream; the call returns when the results are on the host.
 * Takes fewer than 2^30 points and 2^30 triangles (V3D_ERR_INVALID_ARGUMENT). */
int32_t v3d_fuse_mutually_supported_vertices(
    v3d_context* ctx, v3d_point* points, uint64_t n_points,
    const v3d_mesh_triangle* triangles, uint64_t n_triangles, const int64_t* membership,
    v3d_cancel_fn cancel, void* cancel_user, v3d_fusion_stats* stats,
    v3d_fusion_pair* pairs, uint64_t* n_pairs, uint64_t* moved, uint64_t* n_moved);

/* ---- connected-surface merge (surface_merge.rs, surface_merge_clip.rs,
 * surface_merge_stitch.rs) ----------------------------------------------------
 * The second step of surface consolidation, after fusion
 * (surface_fusion.rs:206-214): fusion-accepted pairs become shared vertices,
 * lower-priority triangles owned by a linked higher-priority patch in that
 * patch's reference image are removed (a 3D coverage test where no image can
 * judge), trimmed seams are stitched over existing vertices, partially owned
 * overlap triangles are clipped against their owner with derived vertices,
 * and edges carrying a derived vertex are split. */

/* ReferenceCamera (surface_merge.rs:103-106), one per camera-support group. */
typedef struct v3d_reference_camera {
    int32_t present;          /* 0: None */
    int32_t pad_;
    double rotation[9];       /* row-major; x_cam = rotation * x + translation */
    double translation[3];
} v3d_reference_camera;

/* EvidenceOrigin (reconstruction_evidence.rs:74-79), per point. */
enum {
    V3D_ORIGIN_NONE = -1,
    V3D_ORIGIN_GEOMETRIC_MULTI_VIEW = 0,
    V3D_ORIGIN_REVALIDATED_COMPLETION = 1,
    V3D_ORIGIN_LEARNED_MULTI_VIEW = 2,
    V3D_ORIGIN_GENERATIVE_COMPLETION = 3
};

/* DerivedVertexSource (reconstruction_evidence.rs:144-153). */
typedef struct v3d_derived_vertex_source {
    uint64_t point_index;
    uint64_t source_triangle;
    uint64_t source_corners[3];
    double barycentric[3];
} v3d_derived_vertex_source;

/* TriangleSourceCorners (reconstruction_evidence.rs:125-130). */
typedef struct v3d_triangle_source {
    uint64_t triangle;
    uint64_t corners[3];
} v3d_triangle_source;

/* MergeStats (surface_merge.rs:131-202), its scalar fields; the vectors are
 * in v3d_merge_result. */
typedef struct v3d_merge_stats {
    uint64_t fused_pairs, shared_vertices, cross_reference_triangles,
        removed_duplicate_triangles, remaining_overlap_triangles, provenance_separated_pairs,
        trimmed_seam_triangles;
    double trimmed_seam_area_share;
    uint64_t stitched_seam_triangles, patch_components, meshed_patches, max_postings_per_query,
        posting_bound_hits, clipping_budget_exhausted, clipped_overlap_triangles, clip_pieces,
        derived_vertices, unclipped_overlap_triangles, conformed_triangles, conformance_failures;
} v3d_merge_stats;

/* OwnedMerge (surface_merge.rs:276-283), owned by the library. */
typedef struct v3d_merge_result {
    v3d_merge_stats stats;
    v3d_point* points;                       /* the input points, then the derived ones */
    uint64_t n_points;
    v3d_mesh_triangle* triangles;
    uint64_t n_triangles;
    v3d_derived_vertex_source* derived_vertices;
    uint64_t n_derived_vertices;
    v3d_fusion_pair* uncalibrated_patch_pairs; /* (owner group, candidate group) */
    uint64_t n_uncalibrated_patch_pairs;
    uint64_t* retained_by_group;
    uint64_t n_retained_by_group;
    v3d_triangle_source* triangle_sources;
    uint64_t n_triangle_sources;
} v3d_merge_result;

/* merge_fused_patches_owned_with_control (surface_merge.rs:312-353).
 * membership [n_points]: camera-support group per point, negative for none;
 * pairs: fusion's accepted pairs in its order; cameras [n_cameras]: the
 * reference camera of each group (indexed by group); origins [n_origins]:
 * each point's evidence origin (a shorter array leaves the rest absent, as a
 * shorter slice does).  V3D_OK with *out set, or V3D_REJECTED with the
 * reference's Err message in v3d_last_error ("reconstruction canceled"
 * when cancel fired, or the conformance rejection) and *out NULL. */
int32_t v3d_merge_fused_patches_owned(
    v3d_context* ctx, const v3d_point* points, uint64_t n_points,
    const v3d_mesh_triangle* triangles, uint64_t n_triangles, const int64_t* membership,
    const v3d_fusion_pair* pairs, uint64_t n_pairs, const v3d_reference_camera* cameras,
    uint64_t n_cameras, const int32_t* origins, uint64_t n_origins, v3d_cancel_fn cancel,
    void* cancel_user, v3d_merge_result** out);
void v3d_merge_result_free(v3d_merge_result* result);

/* ---- Serving (no counterpart in the reference, which runs one call at a time) ----
 *
 * A device-resident request loop.  Clips (frames, cameras, landmarks) are
 * registered once: their frames are copied to device memory and stay there.
 * A request asks for reconstruct_reference_patch (dense.rs:674-747) of one
 * camera of a registered clip, with its own hypothesis count and source-view
 * limit.  `slots` worker threads, each with its own CUDA stream and device
 * buffers, take the queued requests in arrival order, as many as the memory
 * budget of a slot admits, and run them as one device batch; while one slot's
 * batch is on the GPU, requests arriving meanwhile form the next batch on
 * another slot, so their work overlaps on the device.  Every request's result
 * is computed from its own inputs only, so it is the same alone and in any mix. */
typedef struct v3d_server v3d_server;

typedef struct v3d_server_config {
    int32_t device;
    int32_t slots;                 /* batches in flight at once, 1..8 */
    uint64_t memory_budget_bytes;  /* device buffers of all slots together (frames excluded); 0: 8 GiB */
    uint32_t max_batch_requests;   /* requests per batch at most; 0: as many as a slot's budget admits */
    int32_t meshed;                /* also run the reference-grid triangle gates of every patch */
    int32_t fine_grid;
    v3d_profile profile;           /* per-request overrides: hypotheses and source views */
} v3d_server_config;

/* Per-request timing, measured on the host from submission. */
typedef struct v3d_request_timing {
    double queue_ms;               /* submitted -> its batch started */
    double service_ms;             /* its batch started -> results ready */
    double total_ms;               /* submitted -> results ready */
    uint64_t batch_requests;       /* requests in its batch */
    uint64_t plane_view_units;     /* its grid sites x hypotheses x source views */
} v3d_request_timing;

int32_t v3d_server_create(const v3d_server_config* config, v3d_server** out);
/* Waits for the batches on the GPU; queued requests end with V3D_ERR_SHUTDOWN
 * and results not collected are freed. */
void v3d_server_destroy(v3d_server* server);
/* Copies the frames to device memory (one pixel format for all clips of a
 * server); cameras and landmarks are kept on the host for planning. */
int32_t v3d_server_add_clip(v3d_server* server, const v3d_frame* frames, uint64_t n_frames,
                            const v3d_camera* cameras, uint64_t n_cameras,
                            const double* sparse_xyz, uint64_t n_sparse, double focal,
                            uint64_t* clip_id);
/* Queues one reference camera of a registered clip; 0 keeps the server
 * profile's hypothesis count / source-view limit. */
int32_t v3d_server_submit(v3d_server* server, uint64_t clip_id, uint64_t camera_index,
                          int32_t depth_hypotheses, int32_t max_source_views, uint64_t* ticket);
/* Waits up to timeout_ms (negative: no limit) for a request.  On completion
 * returns its status, moves its result into *out (and *mesh_out for a meshed
 * server; may be NULL otherwise), sets *present as
 * v3d_reconstruct_reference_patches does and fills *timing (may be NULL);
 * the ticket is then spent.  V3D_ERR_TIMEOUT leaves the request pending. */
int32_t v3d_server_wait(v3d_server* server, uint64_t ticket, int64_t timeout_ms,
                        v3d_dense_result* out, v3d_mesh_result* mesh_out, int32_t* present,
                        v3d_request_timing* timing);
/* Copies the description of the most recent failed batch (empty when none
 * failed) into buf, NUL-terminated and cut to n bytes; returns its full
 * length.  A failed request's status says that it failed; this says why. */
uint64_t v3d_server_last_error(v3d_server* server, char* buf, uint64_t n);

/* Per-site outcome of the depth sweep (dense_legacy.rs:272-362) before the
 * reciprocal check: status 1 = below the contrast gate, 2 = no hypothesis had
 * a passing source view, 3 = photometric or ambiguity gate rejected,
 * 4 = accepted; plane is the chosen hypothesis index. */
typedef struct v3d_site_record {
    uint32_t x, y;
    int32_t status;
    int32_t plane;
    int32_t support;
    int32_t pad;
    double error;
    double margin;
} v3d_site_record;

/* Runs the planning and the depth sweep of
 * v3d_estimate_depth_points_with_control and returns the per-site records in
 * raster order (capacity >= rows * columns of the grid, *n_sites receives the
 * count; with out == NULL only the count is returned).  A diagnostic for parity measurements; it has no counterpart in the
 * reference, whose sweep keeps these values internal. */
int32_t v3d_debug_sweep(
    v3d_context* ctx,
    const v3d_frame* frames, uint64_t n_frames,
    const v3d_camera* cameras, uint64_t n_cameras,
    const double* sparse_xyz, uint64_t n_sparse,
    double focal, int32_t fine_grid,
    const v3d_profile* profile,
    v3d_site_record* out, uint64_t capacity, uint64_t* n_sites);

/* ---- reference-grid triangle gates -------------------------------------- */

/* mesh::reconstruct_dense_mesh_with_control (mesh.rs:74-220); with
 * dense->n_patches == 0 this is legacy::reconstruct_dense_mesh_samples
 * (mesh_legacy.rs:150-358) over all points. */
int32_t v3d_reconstruct_dense_mesh_with_control(
    v3d_context* ctx,
    const v3d_point* points, uint64_t n_points,
    const v3d_grid_site* grid_sites, uint64_t n_grid_sites,
    const v3d_mesh_dense_input* dense,
    const v3d_camera* cameras, uint64_t n_cameras,
    uint32_t width, uint32_t height, double focal,
    v3d_cancel_fn cancel, void* cancel_user,
    v3d_mesh_result* out);

void v3d_mesh_result_free(v3d_mesh_result* result);

/* ---- allocation-free variant ---------------------------------------------- */

/* Outcome counters of v3d_mesh_patch_device_noalloc, written to device memory. */
typedef struct v3d_mesh_counts {
    uint64_t grid_vertices;
    uint64_t candidate_cells;
    uint64_t candidate_triangles;
    uint64_t accepted_triangles;
    uint64_t rejected_discontinuities;
    uint64_t rejected_degenerate;
} v3d_mesh_counts;

#define V3D_NOALLOC_SCRATCH_BYTES (32u << 20)

/* Reference-grid triangle gates of one patch whose points already live in
 * device memory, for callers that may not allocate GPU memory: a host that
 * hands the library pointers into its own pre-allocated pool, a serving loop
 * that must not call cudaMalloc (which can synchronise the device), or a
 * plug-in running under an allocator it does not own.  No counterpart in the
 * reference; it computes what v3d_reconstruct_dense_mesh_with_control does for
 * a single patch (mesh_legacy.rs:200-358), triangle for triangle.
 *
 * Allocates nothing: no cudaMalloc, cudaFree or allocating library call.  All
 * working memory comes from one file-scope device array of
 * V3D_NOALLOC_SCRATCH_BYTES (32 MiB) that every GPU loading the library keeps
 * until exit; a patch whose lattice, points and candidate slots need more is
 * rejected with V3D_ERR_INVALID_ARGUMENT before anything is enqueued (about
 * 1280x720 at grid stride 2 fits).  The first call on a device looks up the
 * array's device address (cudaGetSymbolAddress) with that device current, so
 * make it before any stream capture; the address is kept for the life of the
 * process, so the device must not be reset (cudaDeviceReset) nor its primary
 * context replaced after that first call.  Every call shares the array and leaves
 * the last call's contents there; the call clears what must start at zero.
 * Calls that overlap on the GPU (other streams, other host threads) race on
 * the array: order them on one stream.
 *
 * Inputs: points_dev / sites_dev (device, n_points each), the reference camera
 * and geometry on the host.  Outputs (device): triangles_dev receives the
 * accepted triangles with indices into points_dev, *counts_dev the counters
 * (accepted_triangles = number written).  triangles_dev must hold
 * 2*(gw+1)*(gh+1) + (gw-2)*gh + gw*(gh-2) triangles, the number of candidate
 * slots, where gw and gh are the grid columns and rows
 * ceil((width - 2*border) / stride) and ceil((height - 2*border) / stride).
 * Work is enqueued on `stream` (a cudaStream_t, NULL for the legacy stream);
 * results are valid once the stream has reached them.  Fewer than 3 points
 * yield no triangles (the reference skips such a patch before the grid). */
int32_t v3d_mesh_patch_device_noalloc(
    const v3d_point* points_dev, const v3d_grid_site* sites_dev, uint64_t n_points,
    const v3d_camera* reference_camera,
    uint32_t width, uint32_t height, uint32_t grid_border, uint64_t grid_stride, double focal,
    v3d_mesh_triangle* triangles_dev, uint64_t triangle_capacity,
    v3d_mesh_counts* counts_dev, void* stream);

/* ---- the dense artifact wire format ---------------------------------------
 * DenseStageArtifact (reconstruction_stages.rs:153-161, 248-256) is stored as
 * serde_json's compact document of
 *   {"schema_version":..,"request_hash":..,"cameras_hash":..,"dense":{"stats":{..},
 *    "points":[..],"grid_sites":[..],"point_attributes":[..],"warnings":[..]}}
 * and identified by the SHA-256 of those bytes (stage_artifact_document!,
 * reconstruction_stages.rs:287-420).  The three arrays are nearly all of the
 * document; they are formatted here on the device.  Point3
 * (reconstruction/types.rs:68-77) is {"x":f,"y":f,"z":f,"confidence":f,"r":u,
 * "g":u,"b":u}, DenseGridSite (dense.rs:56-60) {"x":u,"y":u} and
 * EvidencePointAttributes (reconstruction_evidence.rs:107-115)
 * {"reciprocal_consistency":f,"depth_margin":f}.  Each f32 is written as the
 * shortest decimal that reads back to the same f32 (the closest such, ties to
 * an even last digit) in the notation serde_json uses for f32: plain decimals
 * for magnitudes from 1e-6 up to below 1e13 ("1.0", "0.000015",
 * "10000000000.0"), otherwise d.ddde±x without a '+' ("1e-7", "3.4028235e38");
 * a non-finite f32 is written as null, as serde_json does. */

typedef struct v3d_dense_document {
    uint64_t document_bytes;         /* prefix + arrays + suffix */
    uint64_t points_bytes;           /* the text of "[...]" for each array */
    uint64_t grid_sites_bytes;
    uint64_t point_attributes_bytes;
    uint64_t non_finite;             /* floats written as null (check_finite's rejections) */
    uint8_t sha256[32];              /* ContentHash::of_bytes of the document, raw digest */
} v3d_dense_document;

/* Upper bound of document_bytes for the given counts and host parts; a
 * document buffer of this size is always large enough. */
uint64_t v3d_dense_document_bound(uint64_t n_points, uint64_t n_grid_sites,
                                  uint64_t n_point_attributes, uint64_t prefix_bytes,
                                  uint64_t suffix_bytes);

/* DenseStageArtifact::to_json and content_hash (reconstruction_stages.rs:290-
 * 380) with the arrays formatted on the device:
 *   document = prefix ‖ points ‖ ,"grid_sites": ‖ sites ‖ ,"point_attributes": ‖ attributes ‖ suffix
 * where the caller serializes the prefix (everything up to and including
 * `"points":`) and the suffix (from `,"warnings":` to the end), which are
 * small.  Any array pointer may be NULL with count 0 ("[]").  The document is
 * written to `document` (capacity bytes; v3d_dense_document_bound is always
 * enough; when too small the call returns V3D_ERR_INVALID_ARGUMENT with
 * out->document_bytes set and nothing written) and hashed with SHA-256 while
 * it streams back.  out->non_finite counts the nulls; the reference's
 * to_json_with_cancel refuses such an artifact (NonFinite), to_json writes
 * null. */
int32_t v3d_encode_dense_evidence(
    v3d_context* ctx,
    const v3d_point* points, uint64_t n_points,
    const v3d_grid_site* grid_sites, uint64_t n_grid_sites,
    const v3d_point_attributes* point_attributes, uint64_t n_point_attributes,
    const char* prefix, uint64_t prefix_bytes, const char* suffix, uint64_t suffix_bytes,
    char* document, uint64_t capacity, v3d_dense_document* out);

/* The browser transport's packed point buffers (pack_dense_points,
 * crates/video-to-3d-wasm/src/lib.rs:227-240): values_f32_le gets x, y, z,
 * confidence of every point as little-endian f32 (16 bytes a point), rgb
 * three bytes a point.  PackedDenseGridSiteBuffer and
 * PackedDensePointAttributeBuffer (lib.rs:242-265) are byte for byte the
 * v3d_grid_site and v3d_point_attributes arrays on a little-endian host and
 * need no call.  Host only; no device or context. */
void v3d_pack_dense_points(const v3d_point* points, uint64_t n_points,
                           uint8_t* values_f32_le, uint8_t* rgb);

/* The browser transport's packed mesh buffers (pack_mesh_triangles,
 * crates/video-to-3d-wasm/src/lib.rs:269-326): indices_u32_le 12 bytes and
 * confidence_f32_le 4 bytes a triangle, sources_u32_le 16 bytes a source
 * record (triangle, a, b, c), derived_u32_le 20 bytes and
 * derived_barycentric_f64_le 24 bytes a derived record.  Checks in the
 * reference's order (sources, derived, then triangles); on failure returns
 * V3D_ERR_INVALID_ARGUMENT and, when error is not NULL, points it at the
 * reference's message ("failed to serialize reconstruction: ...").  Host
 * only; no device or context. */
int32_t v3d_pack_mesh_triangles(const v3d_mesh_triangle* triangles, uint64_t n_triangles,
                                const v3d_triangle_source* sources, uint64_t n_sources,
                                const v3d_derived_vertex_source* derived, uint64_t n_derived,
                                uint64_t point_count, uint8_t* indices_u32_le,
                                uint8_t* confidence_f32_le, uint8_t* sources_u32_le,
                                uint8_t* derived_u32_le, uint8_t* derived_barycentric_f64_le,
                                const char** error);

/* SHA-256 (FIPS 180-4) of bytes[n] into digest[32], on the host; the hash of
 * ContentHash::of_bytes (scene_project.rs:463-465). */
void v3d_sha256(const void* bytes, uint64_t n, uint8_t* digest);

#ifdef __cplusplus
}
#endif

#endif /* V3D_DENSE_H */
