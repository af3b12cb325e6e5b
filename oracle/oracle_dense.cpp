// TEST INFRASTRUCTURE — CPU oracle, per-reference dense pass.
// Restates crates/video-to-3d-core/src/dense_legacy.rs:1-1182 in f64.
// Compiled with -ffp-contract=off: the reference (Rust, no fast-math) never
// fuses a multiply-add, and neither may this restatement.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <stdexcept>

#include "oracle.hpp"

namespace v3do {

namespace {
constexpr size_t kMinVisibleSparsePoints = 8;          // dense_legacy.rs:8
constexpr double kMaxReciprocalRelativeDepthError = 0.08;  // :13
constexpr double kMaxFusionRelativePositionError = 0.08;   // :14
constexpr size_t kMinFusionObservations = 2;           // :15
constexpr size_t kSurfaceCompletionPasses = 2;         // :16
constexpr size_t kMinSurfaceNeighbors = 3;             // :17
constexpr double kMaxSurfaceNeighborSpread = 0.06;     // :18
constexpr double kSurfaceCompletionConfidenceScale = 0.85;  // :19
constexpr double kInf = std::numeric_limits<double>::infinity();

// Rust f64::clamp
double clampd(double v, double lo, double hi) {
    if (v < lo) v = lo;
    if (v > hi) v = hi;
    return v;
}

// Rust's sort_by(partial_cmp().unwrap_or(Equal)) on f64 is a stable sort in which NaN
// compares equal to everything; stable_sort with `a < b` matches it for the finite
// values this path produces.
void sort_f64(std::vector<double>& v) {
    std::stable_sort(v.begin(), v.end(), [](double a, double b) { return a < b; });
}

bool finite3(Vec3 v) { return std::isfinite(v.x) && std::isfinite(v.y) && std::isfinite(v.z); }

uint8_t quantize_u8(double v) {
    double q = std::round(v * 255.0);
    if (!(q >= 0.0)) q = 0.0;
    if (q > 255.0) q = 255.0;
    return static_cast<uint8_t>(q);
}

// sample_rgb (dense_legacy.rs:1159-1166); gray storage formats report the
// intensity quantised to 8 bits in all three channels.
void sample_rgb(const Frame& f, uint32_t x, uint32_t y, uint8_t& r, uint8_t& g, uint8_t& b) {
    size_t idx = static_cast<size_t>(y) * f.width + x;
    if (f.format == V3D_PIXEL_RGBA8) {
        r = f.bytes[idx * 4];
        g = f.bytes[idx * 4 + 1];
        b = f.bytes[idx * 4 + 2];
        return;
    }
    double v = 0;
    if (f.format == V3D_PIXEL_GRAY_F32) {
        float fv;
        std::memcpy(&fv, f.bytes.data() + idx * 4, 4);
        v = fv;
    } else {
        uint16_t h;
        std::memcpy(&h, f.bytes.data() + idx * 2, 2);
        v = f.format == V3D_PIXEL_GRAY_F16 ? half_to_double(h) : bf16_to_double(h);
    }
    r = g = b = quantize_u8(v);
}

double hypothesis_depth(int k, int count, double search_min, double search_max) {
    // dense_legacy.rs:286-293
    double t = count == 1 ? 0.0 : static_cast<double>(k) / static_cast<double>(count - 1);
    double inverse_depth = (1.0 / search_min) * (1.0 - t) + (1.0 / search_max) * t;
    return 1.0 / inverse_depth;
}

// in_patch_bounds (dense_legacy.rs:1142-1145)
bool in_patch_bounds(double x, double y, uint32_t w, uint32_t h, int radius) {
    double margin = static_cast<double>(radius + 1);
    return x >= margin && y >= margin && x < static_cast<double>(w) - margin &&
           y < static_cast<double>(h) - margin;
}

bool projects_reference_center(const Camera& ref, const Camera& src, double depth, uint32_t w,
                               uint32_t h, double focal, int radius) {
    Vec3 p = unproject(ref, w * 0.5, h * 0.5, depth, w, h, focal);
    auto q = project(src, p, w, h, focal);
    return q && in_patch_bounds(q->x, q->y, w, h, radius);
}

struct Candidate {
    double depth;
    Vec3 position;
    size_t support;
    double error;
    int plane;
};

LegacyAnalysis skipped(int code, std::string reason) {
    LegacyAnalysis a;
    a.stats.skip_reason = std::move(reason);
    a.stats.skip_code = code;
    return a;
}

double depth_margin_score(double margin, double saturation) {
    if (std::isfinite(margin)) return clampd(margin / saturation, 0.0, 1.0);
    return 1.0;
}
}  // namespace

Profile Profile::from_c(const v3d_profile& p) {
    Profile q;
    q.cost = p.cost;
    q.patch_radius = p.patch_radius;
    q.depth_hypotheses = p.depth_hypotheses;
    q.max_source_views = p.max_source_views;
    q.grid_stride = p.grid_stride;
    q.min_reference_contrast = p.min_reference_contrast;
    q.max_photometric_error = p.max_photometric_error;
    q.min_ambiguity_margin = p.min_ambiguity_margin;
    q.depth_margin_saturation = p.depth_margin_saturation;
    q.error_confidence_scale = p.error_confidence_scale;
    q.min_window_variance = p.min_window_variance;
    return q;
}

double half_to_double(uint16_t h) {
    int sign = (h >> 15) & 1;
    int exp = (h >> 10) & 0x1f;
    int man = h & 0x3ff;
    double v;
    if (exp == 0)
        v = std::ldexp(static_cast<double>(man), -24);
    else if (exp == 31)
        v = man ? std::numeric_limits<double>::quiet_NaN() : kInf;
    else
        v = std::ldexp(static_cast<double>(man | 0x400), exp - 25);
    return sign ? -v : v;
}

double bf16_to_double(uint16_t b) {
    uint32_t bits = static_cast<uint32_t>(b) << 16;
    float f;
    std::memcpy(&f, &bits, 4);
    return f;
}

double norm_squared(Vec3 v) { return (v.x * v.x + v.y * v.y) + v.z * v.z; }
double norm(Vec3 v) { return std::sqrt(norm_squared(v)); }
Vec3 cross(Vec3 a, Vec3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

Vec3 Camera::center() const {
    // -R^T t (multi_view.rs:92-94): the negated matrix times t, nalgebra order.
    Vec3 r;
    r.x = ((-R[0]) * t[0] + (-R[3]) * t[1]) + (-R[6]) * t[2];
    r.y = ((-R[1]) * t[0] + (-R[4]) * t[1]) + (-R[7]) * t[2];
    r.z = ((-R[2]) * t[0] + (-R[5]) * t[1]) + (-R[8]) * t[2];
    return r;
}

Plane to_luma(const Frame& f) {
    // dense_legacy.rs:1147-1157 for RGBA8; gray formats are decoded exactly.
    Plane p;
    p.width = f.width;
    p.height = f.height;
    size_t n = static_cast<size_t>(f.width) * f.height;
    p.v.resize(n);
    if (f.format == V3D_PIXEL_RGBA8) {
        size_t chunks = f.bytes.size() / 4;
        p.v.resize(chunks);
        for (size_t i = 0; i < chunks; ++i) {
            unsigned v = (77u * f.bytes[i * 4] + 150u * f.bytes[i * 4 + 1] +
                          29u * f.bytes[i * 4 + 2]) >> 8;
            p.v[i] = static_cast<double>(static_cast<uint8_t>(v));
        }
    } else if (f.format == V3D_PIXEL_GRAY_F32) {
        for (size_t i = 0; i < n; ++i) {
            float fv;
            std::memcpy(&fv, f.bytes.data() + i * 4, 4);
            p.v[i] = fv;
        }
    } else {
        for (size_t i = 0; i < n; ++i) {
            uint16_t h;
            std::memcpy(&h, f.bytes.data() + i * 2, 2);
            p.v[i] = f.format == V3D_PIXEL_GRAY_F16 ? half_to_double(h) : bf16_to_double(h);
        }
    }
    return p;
}

double quantile(const std::vector<double>& values, double q) {
    // dense_legacy.rs:1168-1174; f64::round is half-away-from-zero like std::round.
    if (values.empty()) return std::numeric_limits<double>::quiet_NaN();
    double idx = std::round(static_cast<double>(values.size() - 1) * clampd(q, 0.0, 1.0));
    return values[static_cast<size_t>(idx)];
}

std::optional<double> median_option(std::vector<double>& values) {
    if (values.empty()) return std::nullopt;
    sort_f64(values);
    return quantile(values, 0.5);
}

Vec3 unproject(const Camera& c, double x, double y, double depth, uint32_t w, uint32_t h,
               double focal) {
    // dense_legacy.rs:996-1011: R^T (camera_point - t), nalgebra gemv order.
    Vec3 cp{(x - w * 0.5) / focal * depth, (y - h * 0.5) / focal * depth, depth};
    Vec3 d{cp.x - c.t[0], cp.y - c.t[1], cp.z - c.t[2]};
    Vec3 r;
    r.x = (c.R[0] * d.x + c.R[3] * d.y) + c.R[6] * d.z;
    r.y = (c.R[1] * d.x + c.R[4] * d.y) + c.R[7] * d.z;
    r.z = (c.R[2] * d.x + c.R[5] * d.y) + c.R[8] * d.z;
    return r;
}

std::optional<Vec3> project(const Camera& c, Vec3 p, uint32_t w, uint32_t h, double focal) {
    // dense_legacy.rs:1013-1029: R p + t; reject non-finite or z <= 1e-4.
    Vec3 cp;
    cp.x = ((c.R[0] * p.x + c.R[1] * p.y) + c.R[2] * p.z) + c.t[0];
    cp.y = ((c.R[3] * p.x + c.R[4] * p.y) + c.R[5] * p.z) + c.t[1];
    cp.z = ((c.R[6] * p.x + c.R[7] * p.y) + c.R[8] * p.z) + c.t[2];
    if (!finite3(cp) || cp.z <= 1.0e-4) return std::nullopt;
    return Vec3{focal * cp.x / cp.z + w * 0.5, focal * cp.y / cp.z + h * 0.5, cp.z};
}

bool in_image_bounds(double x, double y, uint32_t w, uint32_t h) {
    return std::isfinite(x) && std::isfinite(y) && x >= 0.0 && y >= 0.0 &&
           x < static_cast<double>(w) && y < static_cast<double>(h);
}

bool in_bilinear_bounds(double x, double y, uint32_t w, uint32_t h) {
    double wm = w > 0 ? static_cast<double>(w - 1) : 0.0;
    double hm = h > 0 ? static_cast<double>(h - 1) : 0.0;
    return std::isfinite(x) && std::isfinite(y) && x >= 0.0 && y >= 0.0 && x < wm && y < hm;
}

std::optional<double> sample_bilinear(const Plane& img, double x, double y) {
    // dense_legacy.rs:1113-1127
    if (!in_bilinear_bounds(x, y, img.width, img.height)) return std::nullopt;
    uint32_t x0 = static_cast<uint32_t>(std::floor(x));
    uint32_t y0 = static_cast<uint32_t>(std::floor(y));
    uint32_t x1 = x0 + 1, y1 = y0 + 1;
    double tx = x - static_cast<double>(x0);
    double ty = y - static_cast<double>(y0);
    auto v = [&](uint32_t px, uint32_t py) {
        return img.v[static_cast<size_t>(py) * img.width + px];
    };
    double top = v(x0, y0) * (1.0 - tx) + v(x1, y0) * tx;
    double bottom = v(x0, y1) * (1.0 - tx) + v(x1, y1) * tx;
    return top * (1.0 - ty) + bottom * ty;
}

double patch_contrast(const Plane& img, double x, double y, int radius) {
    // dense_legacy.rs:1097-1111
    double mn = kInf, mx = -kInf;
    for (int dy = -radius; dy <= radius; ++dy)
        for (int dx = -radius; dx <= radius; ++dx) {
            auto v = sample_bilinear(img, x + dx, y + dy);
            if (!v) return 0.0;
            mn = std::fmin(mn, *v);
            mx = std::fmax(mx, *v);
        }
    return mx - mn;
}

std::optional<double> patch_error(const Profile& prof, const Camera& ref_cam,
                                  const Camera& src_cam, const Plane& ref_img,
                                  const Plane& src_img, double x, double y, double depth,
                                  double focal) {
    // dense_legacy.rs:1032-1095; the ZNCC branch is the project-defined cost.
    const int r = prof.patch_radius;
    double rv[81], sv[81];
    int n = 0;
    for (int dy = -r; dy <= r; ++dy)
        for (int dx = -r; dx <= r; ++dx) {
            double rx = x + dx, ry = y + dy;
            Vec3 world = unproject(ref_cam, rx, ry, depth, ref_img.width, ref_img.height, focal);
            auto s = project(src_cam, world, src_img.width, src_img.height, focal);
            if (!s) return std::nullopt;
            if (!in_bilinear_bounds(s->x, s->y, src_img.width, src_img.height))
                return std::nullopt;
            auto a = sample_bilinear(ref_img, rx, ry);
            if (!a) return std::nullopt;
            auto b = sample_bilinear(src_img, s->x, s->y);
            if (!b) return std::nullopt;
            rv[n] = *a;
            sv[n] = *b;
            ++n;
        }
    double sr = 0.0, ss = 0.0;
    for (int i = 0; i < n; ++i) sr += rv[i];
    for (int i = 0; i < n; ++i) ss += sv[i];
    double mr = sr / n, ms = ss / n;
    if (prof.cost == V3D_COST_ZSAD) {
        double acc = 0.0;
        for (int i = 0; i < n; ++i) acc += std::fabs((rv[i] - mr) - (sv[i] - ms));
        return acc / n;
    }
    double cov = 0.0, vr = 0.0, vs = 0.0;
    for (int i = 0; i < n; ++i) {
        double dr = rv[i] - mr, ds = sv[i] - ms;
        cov += dr * ds;
        vr += dr * dr;
        vs += ds * ds;
    }
    if (!(vr > 0.0) || !(vs > 0.0) || vr / n < prof.min_window_variance ||
        vs / n < prof.min_window_variance)
        return std::nullopt;
    return 1.0 - cov / std::sqrt(vr * vs);
}

std::vector<double> visible_depths(const Camera& c, const std::vector<Vec3>& sparse, uint32_t w,
                                   uint32_t h, double focal) {
    std::vector<double> out;
    for (const Vec3& p : sparse) {
        auto q = project(c, p, w, h, focal);
        if (q && in_image_bounds(q->x, q->y, w, h)) out.push_back(q->z);
    }
    return out;
}

std::optional<std::pair<double, double>> depth_search_bounds(const Camera& c,
                                                             const std::vector<Vec3>& sparse,
                                                             uint32_t w, uint32_t h,
                                                             double focal) {
    // dense_legacy.rs:755-775
    auto depths = visible_depths(c, sparse, w, h, focal);
    if (depths.size() < kMinVisibleSparsePoints) return std::nullopt;
    sort_f64(depths);
    double lower = quantile(depths, 0.10), upper = quantile(depths, 0.90);
    if (!std::isfinite(lower) || !std::isfinite(upper) || lower <= 0.0 || upper <= 0.0)
        return std::nullopt;
    double mn = std::fmax(lower * 0.8, 1.0e-4);
    double mx = std::fmax(upper * 1.25, mn * 1.2);
    return std::make_pair(mn, mx);
}

std::optional<double> surface_depth_prediction(std::vector<double>& depths) {
    // dense_legacy.rs:739-753
    if (depths.size() < kMinSurfaceNeighbors) return std::nullopt;
    sort_f64(depths);
    double mn = depths.front(), mx = depths.back();
    if (!std::isfinite(mn) || !std::isfinite(mx) || mn <= 0.0 || mx <= 0.0) return std::nullopt;
    if ((mx - mn) / mx > kMaxSurfaceNeighborSpread) return std::nullopt;
    return quantile(depths, 0.5);
}

bool reciprocal_depth_agrees(double expected, double estimated) {
    // dense_legacy.rs:951-957
    if (!std::isfinite(expected) || !std::isfinite(estimated) || expected <= 0.0 ||
        estimated <= 0.0)
        return false;
    double scale = std::fmax(std::fmax(expected, estimated), 1.0e-9);
    return std::fabs(expected - estimated) / scale <= kMaxReciprocalRelativeDepthError;
}

Fused fuse_depth_observations(Vec3 primary, const std::vector<Vec3>& reciprocal,
                              double reference_depth) {
    // dense_legacy.rs:859-884
    double radius = std::fmax(std::fabs(reference_depth) * kMaxFusionRelativePositionError, 1.0e-4);
    Vec3 sum = primary;
    size_t obs = 1, rejected = 0;
    for (const Vec3& p : reciprocal) {
        if (!finite3(p) || norm(sub(p, primary)) > radius) {
            ++rejected;
            continue;
        }
        sum = add(sum, p);
        ++obs;
    }
    double d = static_cast<double>(obs);
    return Fused{{sum.x / d, sum.y / d, sum.z / d}, obs, rejected};
}

std::optional<double> estimate_single_view_depth(const Profile& prof, const Camera& ref_cam,
                                                 const Camera& src_cam, const Plane& ref_img,
                                                 const Plane& src_img, double x, double y,
                                                 double search_min, double search_max,
                                                 double focal, double* gap) {
    // dense_legacy.rs:887-949: ref_cam/ref_img are the source view being checked.
    if (patch_contrast(ref_img, x, y, prof.patch_radius) < prof.min_reference_contrast)
        return std::nullopt;
    bool have = false;
    double best_depth = 0, best_error = 0;
    double second = kInf, nearest = kInf;  // decision gaps (ExplainRecord)
    for (int k = 0; k < prof.depth_hypotheses; ++k) {
        double depth = hypothesis_depth(k, prof.depth_hypotheses, search_min, search_max);
        auto e = patch_error(prof, ref_cam, src_cam, ref_img, src_img, x, y, depth, focal);
        if (!e) continue;
        nearest = std::fmin(nearest, std::fabs(*e - prof.max_photometric_error));
        if (!(*e <= prof.max_photometric_error)) continue;
        // sort by (error asc, depth asc), take the first
        if (!have || *e < best_error || (*e == best_error && depth < best_depth)) {
            if (have) second = std::fmin(second, best_error);
            have = true;
            best_error = *e;
            best_depth = depth;
        } else {
            second = std::fmin(second, *e);
        }
    }
    if (gap)
        *gap = have ? std::fmin(second - best_error,
                                std::fabs(best_error - prof.max_photometric_error))
                    : nearest;
    if (!have) return std::nullopt;
    return best_depth;
}

std::vector<Vec3> reciprocal_depth_observations(const Profile& prof, Vec3 position,
                                                const Camera& ref_cam, const Frame& ref_frame,
                                                const Plane& ref_luma,
                                                const std::vector<SourceView>& sources,
                                                double focal, double* gap) {
    // dense_legacy.rs:777-857
    std::vector<Vec3> out;
    double g = kInf;
    auto rp = project(ref_cam, position, ref_frame.width, ref_frame.height, focal);
    if (rp) {
        for (const SourceView& s : sources) {
            auto direct = patch_error(prof, ref_cam, *s.camera, ref_luma, s.luma, rp->x, rp->y,
                                      rp->z, focal);
            if (!direct) continue;
            g = std::fmin(g, std::fabs(*direct - prof.max_photometric_error));
            if (*direct > prof.max_photometric_error) continue;
            auto sp = project(*s.camera, position, s.frame->width, s.frame->height, focal);
            if (!sp) continue;
            double sg = kInf;
            auto rd = estimate_single_view_depth(prof, *s.camera, ref_cam, s.luma, ref_luma,
                                                 sp->x, sp->y, s.search_min_depth,
                                                 s.search_max_depth, focal, gap ? &sg : nullptr);
            g = std::fmin(g, sg);
            if (!rd) continue;
            if (!reciprocal_depth_agrees(sp->z, *rd)) continue;
            Vec3 pos =
                unproject(*s.camera, sp->x, sp->y, *rd, s.frame->width, s.frame->height, focal);
            if (finite3(pos)) out.push_back(pos);
        }
    }
    if (gap) *gap = g;
    return out;
}

CompletionStats complete_surface_samples(const Profile& prof, const Camera& ref_cam,
                                         const Frame& ref_frame, const Plane& ref_luma,
                                         const std::vector<SourceView>& sources,
                                         std::vector<Point3>& points,
                                         std::vector<GridSite>& grid_sites,
                                         std::vector<Attr>& attrs, std::vector<double>& errors,
                                         std::vector<double>& supports, uint32_t width,
                                         uint32_t height, uint32_t border, size_t stride,
                                         double focal, Control& control,
                                         std::vector<ExplainRecord>* explain) {
    // dense_legacy.rs:519-737
    CompletionStats stats;
    if (stride == 0 || sources.empty()) return stats;
    const double S = static_cast<double>(sources.size());
    const int64_t st = static_cast<int64_t>(stride);
    struct Addition {
        Point3 p;
        GridSite s;
        Attr a;
        double error, support;
    };
    // kind: -1 no proposal, 0 kept, 1 texture, 2 cross view, 3 reciprocal, 4 fusion,
    // 5 footprint (the order of the rejection counters)
    struct Outcome {
        int kind = -1;
        int support = 0;
        double sweep_gap = kInf, recip_gap = kInf;
        Addition add{};
    };
    std::vector<uint32_t> cols;
    for (uint32_t x = border; x < width - border; x += stride) cols.push_back(x);
    for (size_t pass = 0; pass < kSurfaceCompletionPasses; ++pass) {
        // occupied: BTreeMap<(x,y), index>; later entries overwrite earlier ones.
        // A dense lookup over the pixel raster is equivalent.
        std::vector<int64_t> occ(static_cast<size_t>(width) * height, -1);
        for (size_t i = 0; i < grid_sites.size(); ++i) {
            const GridSite& g = grid_sites[i];
            if (g.x < width && g.y < height) occ[static_cast<size_t>(g.y) * width + g.x] = i;
        }
        auto lookup = [&](int64_t x, int64_t y) -> int64_t {
            if (x < 0 || y < 0 || x >= width || y >= height) return -1;
            return occ[static_cast<size_t>(y) * width + x];
        };
        // The reference polls once per row before its sites (dense_legacy.rs:551)
        // and a cancel returns the counters of the rows before it; the rows are
        // polled here in order first, and only those rows run.
        std::vector<uint32_t> rows;
        bool canceled = false;
        for (uint32_t y = border; y < height - border; y += stride) {
            if (control.is_canceled()) {
                canceled = true;
                break;
            }
            rows.push_back(y);
        }
        const size_t nsites = rows.size() * cols.size();
        std::vector<Outcome> outs(nsites);
        // every proposal reads only the state before the pass
#pragma omp parallel for schedule(dynamic, 16)
        for (int64_t i = 0; i < static_cast<int64_t>(nsites); ++i) {
            const uint32_t y = rows[i / cols.size()], x = cols[i % cols.size()];
            Outcome& o = outs[i];
            if (lookup(x, y) >= 0) continue;
            std::vector<double> nd, nc, nm;
            for (int64_t oy = -1; oy <= 1; ++oy)
                for (int64_t ox = -1; ox <= 1; ++ox) {
                    if (ox == 0 && oy == 0) continue;
                    int64_t nx = static_cast<int64_t>(x) + ox * st;
                    int64_t ny = static_cast<int64_t>(y) + oy * st;
                    if (nx < 0 || ny < 0) continue;
                    int64_t pi = lookup(nx, ny);
                    if (pi < 0 || static_cast<size_t>(pi) >= points.size()) continue;
                    const Point3& pt = points[pi];
                    Vec3 pos{static_cast<double>(pt.x), static_cast<double>(pt.y),
                             static_cast<double>(pt.z)};
                    auto pr = project(ref_cam, pos, width, height, focal);
                    if (!pr) continue;
                    nd.push_back(pr->z);
                    nc.push_back(static_cast<double>(pt.confidence));
                    nm.push_back(static_cast<size_t>(pi) < attrs.size()
                                     ? static_cast<double>(attrs[pi].depth_margin)
                                     : 0.0);
                }
            auto predicted = surface_depth_prediction(nd);
            if (!predicted) continue;
            if (patch_contrast(ref_luma, x, y, prof.patch_radius) < prof.min_reference_contrast) {
                o.kind = 1;
                continue;
            }
            Vec3 ppos = unproject(ref_cam, x, y, *predicted, width, height, focal);
            std::vector<double> de;
            for (const SourceView& s : sources) {
                auto e = patch_error(prof, ref_cam, *s.camera, ref_luma, s.luma, x, y,
                                     *predicted, focal);
                if (!e) continue;
                o.sweep_gap = std::fmin(o.sweep_gap, std::fabs(*e - prof.max_photometric_error));
                if (*e <= prof.max_photometric_error) de.push_back(*e);
            }
            o.support = static_cast<int>(de.size());
            if (de.empty()) {
                o.kind = 2;
                continue;
            }
            sort_f64(de);
            double direct_error = quantile(de, 0.5);
            auto recip = reciprocal_depth_observations(prof, ppos, ref_cam, ref_frame, ref_luma,
                                                       sources, focal,
                                                       explain ? &o.recip_gap : nullptr);
            if (recip.empty()) {
                o.kind = 3;
                continue;
            }
            Fused fused = fuse_depth_observations(ppos, recip, *predicted);
            if (fused.observations < kMinFusionObservations) {
                o.kind = 4;
                continue;
            }
            auto fp = project(ref_cam, fused.position, width, height, focal);
            double limit = static_cast<double>(stride) * 0.5;
            if (!fp || std::fabs(fp->x - x) >= limit || std::fabs(fp->y - y) >= limit) {
                o.kind = 5;
                continue;
            }
            double csum = 0.0;
            for (double c : nc) csum += c;
            double neighbor_confidence = csum / static_cast<double>(nc.size());
            double support_confidence = static_cast<double>(de.size()) / S;
            double reciprocal_confidence =
                clampd(static_cast<double>(fused.observations - 1) / S, 0.0, 1.0);
            double error_confidence = 1.0 / (1.0 + direct_error / prof.error_confidence_scale);
            float confidence = static_cast<float>(
                clampd(neighbor_confidence * support_confidence * reciprocal_confidence *
                           error_confidence * kSurfaceCompletionConfidenceScale,
                       0.05, 0.9));
            double msum = 0.0;
            for (double m : nm) msum += m;
            double depth_margin = msum / static_cast<double>(nm.size());
            Addition& add_ = o.add;
            sample_rgb(ref_frame, x, y, add_.p.r, add_.p.g, add_.p.b);
            add_.p.x = static_cast<float>(fused.position.x);
            add_.p.y = static_cast<float>(fused.position.y);
            add_.p.z = static_cast<float>(fused.position.z);
            add_.p.confidence = confidence;
            add_.s = {x, y};
            add_.a.reciprocal_consistency = static_cast<float>(reciprocal_confidence);
            add_.a.depth_margin = static_cast<float>(clampd(depth_margin, 0.0, 1.0));
            add_.error = direct_error;
            add_.support = static_cast<double>(de.size());
            o.kind = 0;
        }
        // the counters and additions in raster order
        std::vector<Addition> additions;
        for (size_t i = 0; i < nsites; ++i) {
            const Outcome& o = outs[i];
            if (o.kind < 0) continue;
            stats.proposals++;
            switch (o.kind) {
                case 0: additions.push_back(o.add); break;
                case 1: stats.rejected_texture++; break;
                case 2: stats.rejected_cross_view++; break;
                case 3: stats.rejected_reciprocal++; break;
                case 4: stats.rejected_fusion++; break;
                default: stats.rejected_footprint++; break;
            }
            if (explain)
                explain->push_back({cols[i % cols.size()], rows[i / cols.size()],
                                    static_cast<int32_t>(pass + 1), o.kind, -1, o.support,
                                    o.kind == 0 ? o.add.error : 0.0, 0.0, o.sweep_gap,
                                    o.recip_gap});
        }
        if (canceled) return stats;
        if (additions.empty()) break;
        stats.accepted += additions.size();
        for (const Addition& a : additions) {
            points.push_back(a.p);
            grid_sites.push_back(a.s);
            attrs.push_back(a.a);
            errors.push_back(a.error);
            supports.push_back(a.support);
        }
    }
    return stats;
}

size_t grid_stride(uint32_t width, uint32_t height, bool fine_grid) {
    // dense.rs:215-218
    uint32_t rows = fine_grid ? 64 : 48;
    uint32_t s = std::min(width, height) / rows;
    return std::clamp<uint32_t>(s, 4, 12);
}

size_t profile_grid_stride(const Profile& prof, uint32_t width, uint32_t height, bool fine_grid) {
    return prof.grid_stride > 0 ? static_cast<size_t>(prof.grid_stride)
                                : grid_stride(width, height, fine_grid);
}

LegacyAnalysis estimate_depth_points_with_control(const Profile& prof,
                                                  const std::vector<Frame>& frames,
                                                  const std::vector<Camera>& cameras,
                                                  const std::vector<Vec3>& sparse, double focal,
                                                  bool fine_grid, Control& control) {
    std::vector<const Frame*> ptrs;
    for (const Frame& f : frames) ptrs.push_back(&f);
    return estimate_depth_points_ptr(prof, ptrs, cameras, sparse, focal, fine_grid, control,
                                     nullptr, nullptr);
}

LegacyAnalysis estimate_depth_points_ptr(const Profile& prof,
                                         const std::vector<const Frame*>& frames,
                                         const std::vector<Camera>& cameras,
                                         const std::vector<Vec3>& sparse, double focal,
                                         bool fine_grid, Control& control,
                                         std::vector<v3d_site_record>* sweep_records,
                                         const RowBand* band,
                                         std::vector<ExplainRecord>* explain) {
    // dense_legacy.rs:149-470
    if (frames.empty()) return skipped(V3D_SKIP_NO_FRAMES, "no sampled frames are available");
    if (cameras.size() < 2)
        return skipped(V3D_SKIP_FEWER_THAN_TWO_CAMERAS,
                       "fewer than two accepted registered cameras are available");
    if (sparse.size() < kMinVisibleSparsePoints)
        return skipped(V3D_SKIP_FEW_SPARSE_LANDMARKS,
                       "fewer than 8 accepted sparse landmarks are available");
    const uint32_t width = frames[0]->width, height = frames[0]->height;
    if (width < 16 || height < 16)
        return skipped(V3D_SKIP_FRAMES_TOO_SMALL,
                       "sampled frames are too small for coarse depth estimation");

    // max_by(len, then reversed frame_index): the last maximum wins.
    const Camera* reference = nullptr;
    std::vector<double> ref_depths;
    for (const Camera& c : cameras) {
        auto d = visible_depths(c, sparse, width, height, focal);
        if (d.size() < kMinVisibleSparsePoints) continue;
        bool greater_or_equal;
        if (!reference) {
            greater_or_equal = true;
        } else if (d.size() != ref_depths.size()) {
            greater_or_equal = d.size() > ref_depths.size();
        } else {
            // then_with(right.frame_index.cmp(left.frame_index)) with left = current max,
            // right = candidate: candidate >= max iff candidate.frame_index <= max.frame_index.
            greater_or_equal = c.frame_index <= reference->frame_index;
        }
        if (greater_or_equal) {
            reference = &c;
            ref_depths = std::move(d);
        }
    }
    if (!reference)
        return skipped(V3D_SKIP_NO_REFERENCE_CAMERA,
                       "no registered camera sees at least 8 accepted sparse landmarks inside its "
                       "image");
    sort_f64(ref_depths);
    double lower = quantile(ref_depths, 0.10), upper = quantile(ref_depths, 0.90);
    if (!std::isfinite(lower) || !std::isfinite(upper) || lower <= 0.0 || upper <= 0.0)
        return skipped(V3D_SKIP_NO_DEPTH_ENVELOPE,
                       "visible sparse landmarks do not provide a finite positive depth-search "
                       "envelope");
    const double search_min = std::fmax(lower * 0.8, 1.0e-4);
    const double search_max = std::fmax(upper * 1.25, search_min * 1.2);
    const double median_depth = quantile(ref_depths, 0.50);
    if (reference->frame_index >= frames.size())
        return skipped(V3D_SKIP_REFERENCE_FRAME_MISSING,
                       "the selected reference camera has no sampled frame");
    const Frame& ref_frame = *frames[reference->frame_index];
    // The reference indexes the reference luma with frames[0]'s size
    // (dense_legacy.rs:169-170, 277); a reference frame of another size is
    // outside its defined behaviour and is rejected here.
    if (ref_frame.width != width || ref_frame.height != height)
        throw std::invalid_argument("the selected reference frame differs in size from frame 0");

    struct Src {
        const Camera* cam;
        const Frame* frame;
        double mn, mx;
    };
    std::vector<Src> srcs;
    const Vec3 ref_center = reference->center();
    for (const Camera& c : cameras) {
        if (c.frame_index == reference->frame_index) continue;
        if (c.frame_index >= frames.size()) continue;
        const Frame& f = *frames[c.frame_index];
        double baseline = norm(sub(c.center(), ref_center));
        if (baseline < median_depth * 0.005 ||
            !projects_reference_center(*reference, c, median_depth, width, height, focal,
                                       prof.patch_radius))
            continue;
        auto b = depth_search_bounds(c, sparse, f.width, f.height, focal);
        if (!b) continue;
        srcs.push_back({&c, &f, b->first, b->second});
    }
    auto absdiff = [](size_t a, size_t b) { return a > b ? a - b : b - a; };
    const size_t rfi = reference->frame_index;
    std::stable_sort(srcs.begin(), srcs.end(), [&](const Src& a, const Src& b) {
        size_t da = absdiff(a.cam->frame_index, rfi), db = absdiff(b.cam->frame_index, rfi);
        if (da != db) return da < db;
        return a.cam->frame_index < b.cam->frame_index;
    });
    if (srcs.size() > static_cast<size_t>(prof.max_source_views))
        srcs.resize(prof.max_source_views);
    if (srcs.empty())
        return skipped(V3D_SKIP_NO_SOURCE_VIEW,
                       "no second registered camera has sufficient baseline, overlap, and at "
                       "least 8 visible sparse landmarks for reciprocal depth consistency");

    Plane ref_luma = to_luma(ref_frame);
    std::vector<SourceView> sources;
    for (const Src& s : srcs) sources.push_back({s.cam, s.frame, to_luma(*s.frame), s.mn, s.mx});
    std::vector<size_t> source_frames;
    for (const SourceView& s : sources) source_frames.push_back(s.camera->frame_index);

    const size_t stride = profile_grid_stride(prof, width, height, fine_grid);
    const uint32_t border = static_cast<uint32_t>(prof.patch_radius + 2);
    const double S = static_cast<double>(sources.size());
    LegacyAnalysis out;
    std::vector<double> errors, supports, fusion_counts;
    size_t sampled = 0, rchecked = 0, rrejected = 0, rconsistent = 0, finput = 0, frejobs = 0,
           frejpts = 0;
    auto record = [&](uint32_t x, uint32_t y, int status, const Candidate* c, double margin) {
        if (!sweep_records) return;
        v3d_site_record r{};
        r.x = x;
        r.y = y;
        r.status = status;
        r.plane = c ? c->plane : -1;
        r.support = c ? static_cast<int32_t>(c->support) : 0;
        r.error = c ? c->error : 0.0;
        r.margin = c ? margin : 0.0;
        sweep_records->push_back(r);
    };
    // The reference polls once per grid row before its sites (dense_legacy.rs:273)
    // and a cancel discards the pass; the rows are polled here in order first.
    std::vector<uint32_t> rows, cols;
    {
        uint32_t row = 0;
        for (uint32_t y = border; y < height - border; y += stride, ++row) {
            if (band && (row < band->begin || row >= band->end)) continue;
            if (control.is_canceled())
                return skipped(V3D_SKIP_CANCELED, "dense reconstruction canceled");
            rows.push_back(y);
        }
        for (uint32_t x = border; x < width - border; x += stride) cols.push_back(x);
    }
    const size_t nsites = rows.size() * cols.size();
    if (band)
        band->units += static_cast<uint64_t>(nsites) * prof.depth_hypotheses * sources.size();
    // Each site's sweep, reciprocal check and fusion depend only on the inputs,
    // so the sites run in parallel; the counters, records and points are then
    // reduced in raster order.
    struct SiteOutcome {
        int status = 1;  // 1 low contrast, 2 no candidate, 3 gate rejected, 4 accepted
        Candidate best{};
        double margin = 0.0;
        double sweep_gap = kInf, recip_gap = kInf;
        size_t n_recip = 0;
        Fused fused{};
    };
    std::vector<SiteOutcome> outs(nsites);
#pragma omp parallel
    {
        std::vector<Candidate> cands;
        std::vector<double> source_errors;
#pragma omp for schedule(dynamic, 8)
        for (int64_t i = 0; i < static_cast<int64_t>(nsites); ++i) {
            const uint32_t y = rows[i / cols.size()], x = cols[i % cols.size()];
            SiteOutcome& o = outs[i];
            if (patch_contrast(ref_luma, x, y, prof.patch_radius) < prof.min_reference_contrast)
                continue;
            cands.clear();
            double nearest = kInf;
            for (int k = 0; k < prof.depth_hypotheses; ++k) {
                double depth = hypothesis_depth(k, prof.depth_hypotheses, search_min, search_max);
                Vec3 position = unproject(*reference, x, y, depth, width, height, focal);
                source_errors.clear();
                for (const SourceView& s : sources) {
                    auto e = patch_error(prof, *reference, *s.camera, ref_luma, s.luma, x, y,
                                         depth, focal);
                    if (!e) continue;
                    nearest = std::fmin(nearest, std::fabs(*e - prof.max_photometric_error));
                    if (*e <= prof.max_photometric_error) source_errors.push_back(*e);
                }
                if (source_errors.empty()) continue;
                sort_f64(source_errors);
                cands.push_back({depth, position, source_errors.size(),
                                 quantile(source_errors, 0.5), k});
            }
            std::stable_sort(cands.begin(), cands.end(),
                             [](const Candidate& a, const Candidate& b) {
                                 if (a.support != b.support) return a.support > b.support;
                                 if (a.error != b.error) return a.error < b.error;
                                 return a.depth < b.depth;
                             });
            if (cands.empty()) {
                o.status = 2;
                o.sweep_gap = nearest;
                continue;
            }
            o.best = cands[0];
            double margin = kInf;
            for (size_t j = 1; j < cands.size(); ++j)
                if (cands[j].support == o.best.support) {
                    margin = cands[j].error - o.best.error;
                    break;
                }
            o.margin = margin;
            o.sweep_gap = std::fmin(std::fabs(o.best.error - prof.max_photometric_error),
                                    std::fabs(margin - prof.min_ambiguity_margin));
            if (o.best.error > prof.max_photometric_error || margin < prof.min_ambiguity_margin) {
                o.status = 3;
                continue;
            }
            o.status = 4;
            if (sweep_records) continue;
            auto recip = reciprocal_depth_observations(prof, o.best.position, *reference,
                                                       ref_frame, ref_luma, sources, focal,
                                                       explain ? &o.recip_gap : nullptr);
            o.n_recip = recip.size();
            if (!recip.empty()) o.fused = fuse_depth_observations(o.best.position, recip, o.best.depth);
        }
    }
    auto note = [&](uint32_t x, uint32_t y, int outcome, const SiteOutcome& o) {
        if (!explain) return;
        const bool c = o.status >= 3;
        explain->push_back({x, y, 0, outcome, c ? o.best.plane : -1,
                            c ? static_cast<int32_t>(o.best.support) : 0, c ? o.best.error : 0.0,
                            c ? o.margin : 0.0, o.sweep_gap, o.recip_gap});
    };
    for (size_t i = 0; i < nsites; ++i) {
        const uint32_t y = rows[i / cols.size()], x = cols[i % cols.size()];
        const SiteOutcome& o = outs[i];
        if (o.status == 1) {
            record(x, y, 1, nullptr, 0.0);
            continue;
        }
        ++sampled;
        if (o.status == 2) {
            record(x, y, 2, nullptr, 0.0);
            note(x, y, 2, o);
            continue;
        }
        const Candidate& best = o.best;
        const double margin = o.margin;
        if (o.status == 3) {
            record(x, y, 3, &best, margin);
            note(x, y, 3, o);
            continue;
        }
        record(x, y, 4, &best, margin);
        if (sweep_records) continue;
        ++rchecked;
        if (o.n_recip == 0) {
            ++rrejected;
            note(x, y, 5, o);
            continue;
        }
        ++rconsistent;
        finput += 1 + o.n_recip;
        const Fused& fused = o.fused;
        frejobs += fused.rejected_observations;
        if (fused.observations < kMinFusionObservations) {
            ++frejpts;
            note(x, y, 6, o);
            continue;
        }
        note(x, y, 7, o);
        fusion_counts.push_back(static_cast<double>(fused.observations));
        double support_confidence = static_cast<double>(best.support) / S;
        double reciprocal_confidence =
            clampd(static_cast<double>(fused.observations - 1) / S, 0.0, 1.0);
        double error_confidence = 1.0 / (1.0 + best.error / prof.error_confidence_scale);
        double depth_margin = depth_margin_score(margin, prof.depth_margin_saturation);
        double margin_confidence = std::fmax(depth_margin, 0.2);
        float confidence = static_cast<float>(clampd(
            support_confidence * reciprocal_confidence * error_confidence * margin_confidence,
            0.05, 1.0));
        Point3 p;
        sample_rgb(ref_frame, x, y, p.r, p.g, p.b);
        p.x = static_cast<float>(fused.position.x);
        p.y = static_cast<float>(fused.position.y);
        p.z = static_cast<float>(fused.position.z);
        p.confidence = confidence;
        out.points.push_back(p);
        out.grid_sites.push_back({x, y});
        out.point_attributes.push_back({static_cast<float>(reciprocal_confidence),
                                        static_cast<float>(depth_margin)});
        errors.push_back(best.error);
        supports.push_back(static_cast<double>(best.support));
    }

    if (sweep_records || band) return out;
    CompletionStats cs = complete_surface_samples(
        prof, *reference, ref_frame, ref_luma, sources, out.points, out.grid_sites,
        out.point_attributes, errors, supports, width, height, border, stride, focal, control,
        explain);

    LegacyStats& st = out.stats;
    st.attempted = true;
    st.reference_frame = reference->frame_index;
    st.source_views = sources.size();
    st.source_frames = source_frames;
    st.sampled_pixels = sampled;
    st.depth_hypotheses = static_cast<size_t>(prof.depth_hypotheses);
    st.accepted_points = out.points.size();
    st.surface_completion_proposals = cs.proposals;
    st.surface_completed_points = cs.accepted;
    st.surface_completion_rejected_texture = cs.rejected_texture;
    st.surface_completion_rejected_cross_view = cs.rejected_cross_view;
    st.surface_completion_rejected_reciprocal = cs.rejected_reciprocal;
    st.surface_completion_rejected_fusion = cs.rejected_fusion;
    st.surface_completion_rejected_footprint = cs.rejected_footprint;
    st.grid_stride = stride;
    st.grid_border = border;
    st.reciprocal_checked_points = rchecked;
    st.reciprocal_rejected_points = rrejected;
    st.reciprocal_consistent_points = rconsistent;
    st.fusion_input_observations = finput;
    st.fusion_rejected_observations = frejobs;
    st.fusion_rejected_points = frejpts;
    auto to_f32 = [](std::optional<double> v) -> std::optional<float> {
        if (!v) return std::nullopt;
        return static_cast<float>(*v);
    };
    st.median_fusion_observations = to_f32(median_option(fusion_counts));
    st.median_supporting_views = to_f32(median_option(supports));
    st.median_photometric_error = to_f32(median_option(errors));
    st.search_min_depth = static_cast<float>(search_min);
    st.search_max_depth = static_cast<float>(search_max);
    return out;
}

}  // namespace v3do
