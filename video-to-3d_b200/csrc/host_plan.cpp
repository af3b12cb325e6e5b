// Host planning of the dense pass: everything before the first grid site is
// touched.  Restates dense_legacy.rs:157-256 (reference and source selection,
// depth envelopes, grid), dense.rs:620-747 (reference order, the remapped
// per-reference call) and dense.rs:165-218 (landmark distribution, stride).
// It is O(cameras x landmarks) f64 arithmetic; the per-site work runs on the
// device.  Built with -ffp-contract=off so its f64 results (the hypothesis
// envelope above all) are the reference's to the bit.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <thread>

#include "host.hpp"

namespace v3d {

namespace {
constexpr size_t kMinVisibleSparsePoints = 8;  // dense_legacy.rs:8

// quantile (dense_legacy.rs:1168-1174) of the sorted values: the element of
// rank round((n - 1) q).  The depths are finite, so that order statistic is
// selected in place instead of sorting (any permutation of v is left behind).
double quantile_of(std::vector<double>& v, double q) {
    if (v.empty()) return std::nan("");
    double c = q < 0.0 ? 0.0 : (q > 1.0 ? 1.0 : q);
    const size_t k = static_cast<size_t>(std::round(static_cast<double>(v.size() - 1) * c));
    std::nth_element(v.begin(), v.begin() + k, v.end());
    return v[k];
}

std::vector<double> visible_depths(const HCamera& c, const std::vector<HVec3>& sparse, uint32_t w,
                                   uint32_t h, double focal) {
    std::vector<double> out;
    out.reserve(sparse.size());
    for (const HVec3& p : sparse) {
        HVec3 q;
        if (project_h(c, p, w, h, focal, q) && in_image_bounds_h(q.x, q.y, w, h)) out.push_back(q.z);
    }
    return out;
}

bool envelope(std::vector<double>& depths, double& mn, double& mx, double* median) {
    double lower = quantile_of(depths, 0.10), upper = quantile_of(depths, 0.90);
    if (!std::isfinite(lower) || !std::isfinite(upper) || lower <= 0.0 || upper <= 0.0) return false;
    mn = std::fmax(lower * 0.8, 1.0e-4);
    mx = std::fmax(upper * 1.25, mn * 1.2);
    if (median) *median = quantile_of(depths, 0.50);
    return true;
}

void skip(RefPlan& p, int code, const char* reason) {
    p.skipped = true;
    p.skip_code = code;
    p.skip_reason = reason;
}

size_t absdiff(size_t a, size_t b) { return a > b ? a - b : b - a; }
}  // namespace

uint32_t reference_grid_stride(uint32_t w, uint32_t h, bool fine) {
    uint32_t rows = fine ? 64 : 48;
    uint32_t s = std::min(w, h) / rows;
    return std::clamp<uint32_t>(s, 4, 12);
}

HVec3 camera_center(const HCamera& c) {
    // -R^T t, with the negated matrix applied in nalgebra's column order
    HVec3 r;
    r.x = ((-c.R[0]) * c.t[0] + (-c.R[3]) * c.t[1]) + (-c.R[6]) * c.t[2];
    r.y = ((-c.R[1]) * c.t[0] + (-c.R[4]) * c.t[1]) + (-c.R[7]) * c.t[2];
    r.z = ((-c.R[2]) * c.t[0] + (-c.R[5]) * c.t[1]) + (-c.R[8]) * c.t[2];
    return r;
}

HVec3 unproject_h(const HCamera& c, double x, double y, double depth, uint32_t w, uint32_t h,
                  double focal) {
    double cx = (x - w * 0.5) / focal * depth, cy = (y - h * 0.5) / focal * depth;
    double dx = cx - c.t[0], dy = cy - c.t[1], dz = depth - c.t[2];
    return {(c.R[0] * dx + c.R[3] * dy) + c.R[6] * dz, (c.R[1] * dx + c.R[4] * dy) + c.R[7] * dz,
            (c.R[2] * dx + c.R[5] * dy) + c.R[8] * dz};
}

bool project_h(const HCamera& c, HVec3 p, uint32_t w, uint32_t h, double focal, HVec3& out) {
    double x = ((c.R[0] * p.x + c.R[1] * p.y) + c.R[2] * p.z) + c.t[0];
    double y = ((c.R[3] * p.x + c.R[4] * p.y) + c.R[5] * p.z) + c.t[1];
    double z = ((c.R[6] * p.x + c.R[7] * p.y) + c.R[8] * p.z) + c.t[2];
    if (!(std::isfinite(x) && std::isfinite(y) && std::isfinite(z)) || z <= 1.0e-4) return false;
    out = {focal * x / z + w * 0.5, focal * y / z + h * 0.5, z};
    return true;
}

bool in_image_bounds_h(double x, double y, uint32_t w, uint32_t h) {
    return std::isfinite(x) && std::isfinite(y) && x >= 0.0 && y >= 0.0 &&
           x < static_cast<double>(w) && y < static_cast<double>(h);
}

RefPlan plan_legacy(const v3d_profile& prof, const v3d_frame* frames, size_t n_frames,
                    const std::vector<HCamera>& cams, const std::vector<HVec3>& sparse,
                    double focal, bool fine_grid, const std::vector<size_t>* slot_map,
                    bool first_camera_sees_all) {
    // `cams[i].frame_index` indexes the (possibly remapped) frame list whose
    // entry k lives in frames[slot_map ? (*slot_map)[k] : k].
    RefPlan p;
    const size_t n_view_frames = slot_map ? slot_map->size() : n_frames;
    auto frame_at = [&](size_t k) -> const v3d_frame& {
        return frames[slot_map ? (*slot_map)[k] : k];
    };
    if (n_view_frames == 0) {
        skip(p, V3D_SKIP_NO_FRAMES, "no sampled frames are available");
        return p;
    }
    if (cams.size() < 2) {
        skip(p, V3D_SKIP_FEWER_THAN_TWO_CAMERAS,
             "fewer than two accepted registered cameras are available");
        return p;
    }
    if (sparse.size() < kMinVisibleSparsePoints) {
        skip(p, V3D_SKIP_FEW_SPARSE_LANDMARKS, "fewer than 8 accepted sparse landmarks are available");
        return p;
    }
    const uint32_t width = frame_at(0).width, height = frame_at(0).height;
    if (width < 16 || height < 16) {
        skip(p, V3D_SKIP_FRAMES_TOO_SMALL, "sampled frames are too small for coarse depth estimation");
        return p;
    }
    // reference: most visible landmarks, ties to the smallest frame index (last maximum)
    const HCamera* reference = nullptr;
    std::vector<double> ref_depths;
    bool fast = false;
    if (first_camera_sees_all && cams[0].frame_index == 0) {
        // Every landmark lies inside cams[0]'s view at frame 0's size, so no
        // camera sees more and ties go to the smallest frame index: the scan
        // below would select cams[0].
        auto d = visible_depths(cams[0], sparse, width, height, focal);
        if (d.size() >= kMinVisibleSparsePoints && d.size() == sparse.size()) {
            reference = &cams[0];
            ref_depths = std::move(d);
            fast = true;
        }
    }
    for (size_t ci = 0; !fast && ci < cams.size(); ++ci) {
        const HCamera& c = cams[ci];
        auto d = visible_depths(c, sparse, width, height, focal);
        if (d.size() < kMinVisibleSparsePoints) continue;
        bool take = !reference || d.size() > ref_depths.size() ||
                    (d.size() == ref_depths.size() && c.frame_index <= reference->frame_index);
        if (take) {
            reference = &c;
            ref_depths = std::move(d);
        }
    }
    if (!reference) {
        skip(p, V3D_SKIP_NO_REFERENCE_CAMERA,
             "no registered camera sees at least 8 accepted sparse landmarks inside its image");
        return p;
    }
    double smin, smax, median;
    if (!envelope(ref_depths, smin, smax, &median)) {
        skip(p, V3D_SKIP_NO_DEPTH_ENVELOPE,
             "visible sparse landmarks do not provide a finite positive depth-search envelope");
        return p;
    }
    if (reference->frame_index >= n_view_frames) {
        skip(p, V3D_SKIP_REFERENCE_FRAME_MISSING, "the selected reference camera has no sampled frame");
        return p;
    }
    const v3d_frame& rf = frame_at(reference->frame_index);
    if (rf.width != width || rf.height != height) {
        // The reference indexes the reference luma with frame 0's size
        // (dense_legacy.rs:169-170, 277); other sizes are rejected as an error.
        skip(p, -2, "the selected reference frame differs in size from frame 0");
        return p;
    }
    struct Src {
        const HCamera* cam;
        double mn, mx;
    };
    // candidates sorted first (the filters are independent per camera), then
    // filtered lazily until max_source_views are accepted
    std::vector<const HCamera*> order;
    for (const HCamera& c : cams)
        if (c.frame_index != reference->frame_index && c.frame_index < n_view_frames)
            order.push_back(&c);
    const size_t rfi = reference->frame_index;
    std::stable_sort(order.begin(), order.end(), [&](const HCamera* a, const HCamera* b) {
        size_t da = absdiff(a->frame_index, rfi), db = absdiff(b->frame_index, rfi);
        if (da != db) return da < db;
        return a->frame_index < b->frame_index;
    });
    const HVec3 rc = camera_center(*reference);
    const int r = prof.patch_radius;
    std::vector<Src> srcs;
    for (const HCamera* c : order) {
        if (srcs.size() >= static_cast<size_t>(prof.max_source_views)) break;
        HVec3 cc = camera_center(*c);
        HVec3 d{cc.x - rc.x, cc.y - rc.y, cc.z - rc.z};
        double baseline = std::sqrt((d.x * d.x + d.y * d.y) + d.z * d.z);
        if (baseline < median * 0.005) continue;
        // projects_reference_center (dense_legacy.rs:975-994) with in_patch_bounds
        HVec3 world = unproject_h(*reference, width * 0.5, height * 0.5, median, width, height, focal);
        HVec3 q;
        if (!project_h(*c, world, width, height, focal, q)) continue;
        double margin = static_cast<double>(r + 1);
        if (!(q.x >= margin && q.y >= margin && q.x < static_cast<double>(width) - margin &&
              q.y < static_cast<double>(height) - margin))
            continue;
        const v3d_frame& sf = frame_at(c->frame_index);
        auto sd = visible_depths(*c, sparse, sf.width, sf.height, focal);
        if (sd.size() < kMinVisibleSparsePoints) continue;
        double mn, mx;
        if (!envelope(sd, mn, mx, nullptr)) continue;
        srcs.push_back({c, mn, mx});
    }
    if (srcs.empty()) {
        skip(p, V3D_SKIP_NO_SOURCE_VIEW,
             "no second registered camera has sufficient baseline, overlap, and at least 8 visible "
             "sparse landmarks for reciprocal depth consistency");
        return p;
    }
    p.have_reference = true;
    p.reference_frame = reference->frame_index;
    p.ref_slot = slot_map ? (*slot_map)[reference->frame_index] : reference->frame_index;
    p.ref_cam = *reference;
    for (const Src& s : srcs) {
        p.source_frames.push_back(s.cam->frame_index);
        p.src_slots.push_back(slot_map ? (*slot_map)[s.cam->frame_index] : s.cam->frame_index);
        p.src_cams.push_back(*s.cam);
        p.src_min.push_back(s.mn);
        p.src_max.push_back(s.mx);
    }
    p.search_min = smin;
    p.search_max = smax;
    p.width = width;
    p.height = height;
    p.stride = prof.grid_stride > 0 ? static_cast<uint32_t>(prof.grid_stride)
                                    : reference_grid_stride(width, height, fine_grid);
    p.border = static_cast<uint32_t>(r + 2);
    p.planes = prof.depth_hypotheses;
    p.focal = focal;
    p.nx = width > 2 * p.border ? (width - 2 * p.border + p.stride - 1) / p.stride : 0;
    p.ny = height > 2 * p.border ? (height - 2 * p.border + p.stride - 1) / p.stride : 0;
    return p;
}

RefPlan plan_reference_patch(const v3d_profile& prof, const Inputs& in, size_t ci, bool fine_grid,
                             bool& present) {
    // dense.rs:674-747
    present = false;
    RefPlan none;
    if (ci >= in.cameras.size()) return none;
    const HCamera& rc = in.cameras[ci];
    if (rc.frame_index >= in.n_frames) return none;
    const v3d_frame& rf = in.frames[rc.frame_index];
    std::vector<HVec3> visible;
    for (const HVec3& p : in.sparse) {
        HVec3 q;
        if (project_h(rc, p, rf.width, rf.height, in.focal, q) &&
            in_image_bounds_h(q.x, q.y, rf.width, rf.height))
            visible.push_back(p);
    }
    if (visible.size() < kMinVisibleSparsePoints) return none;
    std::vector<size_t> src;
    for (size_t i = 0; i < in.cameras.size(); ++i)
        if (i != ci && in.cameras[i].frame_index < in.n_frames) src.push_back(i);
    std::stable_sort(src.begin(), src.end(), [&](size_t a, size_t b) {
        size_t da = absdiff(in.cameras[a].frame_index, rc.frame_index);
        size_t db = absdiff(in.cameras[b].frame_index, rc.frame_index);
        if (da != db) return da < db;
        return in.cameras[a].frame_index < in.cameras[b].frame_index;
    });
    std::vector<size_t> order{ci};
    order.insert(order.end(), src.begin(), src.end());
    std::vector<HCamera> rcams;
    std::vector<size_t> slots;
    rcams.reserve(order.size());
    for (size_t k = 0; k < order.size(); ++k) {
        HCamera m = in.cameras[order[k]];
        slots.push_back(m.frame_index);
        m.frame_index = k;
        rcams.push_back(m);
    }
    present = true;
    RefPlan p = plan_legacy(prof, in.frames, in.n_frames, rcams, visible, in.focal, fine_grid, &slots,
                            true);
    // report frames in the caller's index space (dense.rs:734-745)
    p.have_reference = true;
    p.reference_frame = rc.frame_index;
    for (size_t& f : p.source_frames) f = in.cameras[order[f]].frame_index;
    return p;
}

std::vector<size_t> reference_candidate_order(const Inputs& in) {
    // dense.rs:620-672
    std::vector<int64_t> visible(in.cameras.size(), -1);
    for (size_t i = 0; i < in.cameras.size(); ++i) {
        const HCamera& c = in.cameras[i];
        if (c.frame_index >= in.n_frames) continue;
        const v3d_frame& f = in.frames[c.frame_index];
        int64_t n = 0;
        for (const HVec3& p : in.sparse) {
            HVec3 q;
            if (project_h(c, p, f.width, f.height, in.focal, q) &&
                in_image_bounds_h(q.x, q.y, f.width, f.height))
                ++n;
        }
        visible[i] = n;
    }
    return order_from_visible(in.cameras, visible);
}

std::vector<size_t> order_from_visible(const std::vector<HCamera>& cameras,
                                       const std::vector<int64_t>& visible) {
    // dense.rs:627-671, given each camera's visible landmark count
    std::vector<std::pair<size_t, size_t>> cands;
    for (size_t i = 0; i < cameras.size(); ++i)
        if (visible[i] >= static_cast<int64_t>(kMinVisibleSparsePoints))
            cands.push_back({i, static_cast<size_t>(visible[i])});
    std::stable_sort(cands.begin(), cands.end(), [&](const auto& a, const auto& b) {
        if (a.second != b.second) return a.second > b.second;
        return cameras[a.first].frame_index < cameras[b.first].frame_index;
    });
    if (cands.empty()) return {};
    HVec3 pc = camera_center(cameras[cands[0].first]);
    auto dist2 = [&](size_t i) {
        HVec3 c = camera_center(cameras[i]);
        double dx = c.x - pc.x, dy = c.y - pc.y, dz = c.z - pc.z;
        return (dx * dx + dy * dy) + dz * dz;
    };
    std::stable_sort(cands.begin() + 1, cands.end(), [&](const auto& a, const auto& b) {
        double da = dist2(a.first), db = dist2(b.first);
        if (da != db) return da > db;
        if (a.second != b.second) return a.second > b.second;
        return cameras[a.first].frame_index < cameras[b.first].frame_index;
    });
    std::vector<size_t> out;
    for (auto& c : cands) out.push_back(c.first);
    return out;
}

bool has_distributed_landmarks(const Inputs& in, CancelPoll& cancel) {
    // dense.rs:165-213
    size_t majority = in.cameras.size() / 2 + 1, covered = 0;
    for (const HCamera& c : in.cameras) {
        if (c.frame_index >= in.n_frames) continue;
        const v3d_frame& f = in.frames[c.frame_index];
        uint8_t tiles[4][4] = {};
        size_t supported = 0;
        bool stop = false;
        for (size_t start = 0; start < in.sparse.size() && !stop; start += 256) {
            if (cancel.poll()) return false;
            size_t end = std::min(in.sparse.size(), start + 256);
            for (size_t i = start; i < end; ++i) {
                HVec3 q;
                if (!project_h(c, in.sparse[i], f.width, f.height, in.focal, q)) continue;
                if (!(q.x >= 0.0 && q.x < static_cast<double>(f.width)) ||
                    !(q.y >= 0.0 && q.y < static_cast<double>(f.height)))
                    continue;
                size_t col = static_cast<size_t>(4.0 * q.x / static_cast<double>(f.width));
                size_t row = static_cast<size_t>(4.0 * q.y / static_cast<double>(f.height));
                uint8_t& t = tiles[row][col];
                if (t < 255) ++t;
                if (t == 2 && ++supported >= 8) {
                    if (++covered == majority) return true;
                    stop = true;
                    break;
                }
            }
        }
    }
    return false;
}

void parallel_for(size_t n, const std::function<void(size_t)>& fn) {
    size_t workers = std::min<size_t>(n, std::max(1u, std::thread::hardware_concurrency()));
    if (workers <= 1) {
        for (size_t i = 0; i < n; ++i) fn(i);
        return;
    }
    std::atomic<size_t> next{0};
    std::vector<std::thread> pool;
    pool.reserve(workers);
    for (size_t w = 0; w < workers; ++w)
        pool.emplace_back([&]() {
            for (size_t i = next++; i < n; i = next++) fn(i);
        });
    for (auto& t : pool) t.join();
}

void skip_result(PassResult& r, int code, const std::string& reason) {
    std::memset(&r.stats, 0, sizeof(r.stats));
    r.stats.skip_code = code;
    r.stats.has_skip_reason = 1;
    std::strncpy(r.stats.skip_reason, reason.c_str(), V3D_SKIP_REASON_BYTES - 1);
    r.points = {};
    r.sites = {};
    r.attrs = {};
    r.block.reset();
}

}  // namespace v3d
