// Device-only reference-grid triangle gates (mesh_legacy.rs:150-555) over any
// number of patches, with no host round trip between its kernels.
//
// The reference walks cell origins in BTreeSet order and bridges over the
// grid's bounding box; iterating every lattice origin and every bridge
// position of the full grid in x-major order visits the same candidates in
// the same relative order (an origin outside the occupied set has no corner
// and a bridge outside the bounding box lacks its end vertices), so the
// candidate layout is fixed by the grid size alone.  Triangles are emitted in
// two passes: gate statuses per slot, an order-preserving scan, then the
// accepted triangles are rebuilt and written at their output positions.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/v3d_dense.h"
#include "v3d_device.cuh"

namespace v3d {

struct MeshPatchDev {
    DevCamera cam;           // the patch's reference camera
    double focal;
    uint32_t width, height;  // reference image size
    uint32_t border, stride; // dense grid of the patch
    uint32_t gw, gh;         // lattice columns and rows
    uint64_t grid_off;       // first lattice cell of the patch in the shared grid arrays
    uint64_t slot_off;       // first candidate slot of the patch
    uint64_t n_points;       // points of the patch
};

// Per-patch outcome counters (integer atomics).
struct MeshCounters {
    unsigned long long vertices, candidate_cells, candidate_triangles, accepted,
        discontinuities, degenerate;
};

// Candidate slots of a gw x gh lattice: two per cell origin, one per bridge.
__host__ __device__ __forceinline__ uint64_t mesh_slots(uint32_t gw, uint32_t gh) {
    uint64_t cells = (uint64_t)(gw + 1) * (gh + 1);
    uint64_t hb = gw >= 3 ? (uint64_t)(gw - 2) * gh : 0;
    uint64_t vb = gh >= 3 ? (uint64_t)gw * (gh - 2) : 0;
    return 2 * cells + hb + vb;
}

// Device buffers of one mesh batch (caller-provided; see mesh_scratch_layout).
struct MeshScratch {
    MeshPatchDev* patches;           // [n_patches]
    MeshCounters* counters;          // [n_patches]
    unsigned long long* grid_keys;   // [total lattice cells]
    uint32_t* winners;               // [total lattice cells] point index of the kept vertex
    void* vtx;                       // [n_points] vertex records
    uint8_t* slot_status;            // [total slots]
    uint32_t* slot_idx;              // [total slots] compacted accepted slots
    uint32_t* count;                 // [1] accepted triangles
    void* compact_scratch;           // compaction block counts
};

// Bytes for a batch; fills `s` with offsets from `base` when base != nullptr.
size_t mesh_scratch_layout(void* base, uint32_t n_patches, uint64_t n_points,
                           uint64_t total_cells, uint64_t total_slots, MeshScratch* s);

// Enqueues the whole mesh pass on `stream`.  Points are points[i], sites[i]
// with patch patch_of[i] (0 when null) and patch-local index local_of[i]
// (i when null).  `tris` receives the accepted triangles of all patches in
// patch order, with patch-local indices; `tri_patch` (may be null) their patch.
cudaError_t mesh_batch_enqueue(const MeshScratch& s, uint32_t n_patches, uint64_t total_cells,
                               uint64_t total_slots, const v3d_point* points,
                               const v3d_grid_site* sites, const uint32_t* patch_of,
                               const uint32_t* local_of, uint64_t n_points,
                               v3d_mesh_triangle* tris, uint32_t* tri_patch,
                               cudaStream_t stream);

}  // namespace v3d
