// Device-resident request loop (v3d_server_*; the reference has no
// counterpart: it runs one dense call at a time on the caller's thread).
//
// Clips are registered once and their frames stay in device memory.  Requests
// (one reference camera of a clip, with its own hypothesis count and source
// limit) queue in arrival order.  `slots` worker threads, each with its own
// v3d_context (CUDA stream, device arena, pinned staging), take as many
// queued requests as a slot's share of the memory budget admits and run them
// as one device batch through clip_batch; while one slot's batch runs, the
// requests that arrive meanwhile form the next batch on another slot, so
// batches overlap on the device (continuous batching at batch granularity).
// Each request is planned and computed from its own inputs only, so its result
// does not depend on what else shares its batch.
#include <cuda_runtime.h>

#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <tuple>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include "host.hpp"
#include "pass_kernels.cuh"

using namespace v3d;
using clk = std::chrono::steady_clock;

namespace {

// Device bytes of one batch per grid site and per reference: the arena of a
// batch (site records, candidates, 16 reciprocal slots, fused and pooled
// points, output arrays, mesh lattice and slots) comes to about 1.2 KB per
// site with the mesh, plus up to 0.4 KB of plane-chunk rank states for
// batches of few tiles; these bounds round that up.
constexpr uint64_t kBytesPerSite = 2048;
constexpr uint64_t kBytesPerReference = 64u << 10;
constexpr uint64_t kDefaultBudget = 8ull << 30;
constexpr size_t kPinnedStaging = 16u << 20;

size_t bytes_per_pixel(int format) {
    return format == V3D_PIXEL_RGBA8 || format == V3D_PIXEL_GRAY_F32 ? 4 : 2;
}

double ms_between(clk::time_point a, clk::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
}

struct StoredClip {
    std::vector<v3d_frame> frames;         // sizes and format; pixels live in `resident`
    std::vector<ResidentFrame> resident;
    std::vector<void*> buffers;            // device allocations of the frames
    Inputs in;                             // cameras, landmarks, focal; frames -> `frames`
    uint64_t sites = 0;                    // grid sites of one reference
};

struct Request {
    uint64_t ticket = 0, clip = 0, camera = 0;
    int32_t planes = 0, sources = 0;
    clk::time_point submitted;
    uint64_t bytes = 0;
};

struct Finished {
    int32_t status = V3D_OK;
    v3d_dense_result out{};
    v3d_mesh_result mesh{};
    int32_t present = 0;
    v3d_request_timing timing{};
};

}  // namespace

struct v3d_server {
    v3d_server_config cfg{};
    uint64_t slot_budget = 0;
    cudaStream_t upload = nullptr;
    std::mutex store_mu;
    std::vector<std::unique_ptr<StoredClip>> clips;
    int format = -1;
    std::mutex mu;
    std::condition_variable work_cv, done_cv;
    std::deque<Request> pending;
    std::unordered_set<uint64_t> outstanding;
    std::unordered_map<uint64_t, Finished> finished;
    uint64_t next_ticket = 1;
    bool stop = false;
    std::string last_error;                // of the most recent failed batch
    std::vector<v3d_context*> ctxs;
    std::vector<std::thread> workers;
};

namespace {

// Runs one admitted batch on `ctx` and publishes every request's outcome.
void run_batch_of_requests(v3d_server* s, v3d_context* ctx, const std::vector<Request>& batch,
                           clk::time_point started) {
    // one job per (clip, hypotheses, sources): a job carries one profile
    std::map<std::tuple<uint64_t, int32_t, int32_t>, std::vector<size_t>> groups;
    for (size_t i = 0; i < batch.size(); ++i)
        groups[{batch[i].clip, batch[i].planes, batch[i].sources}].push_back(i);
    std::vector<ClipJob> jobs;
    std::vector<std::vector<uint64_t>> cams;
    std::vector<size_t> order;  // batch index of each reference, job by job
    jobs.reserve(groups.size());
    cams.reserve(groups.size());
    for (const auto& g : groups) {
        const StoredClip* c;
        {
            std::lock_guard<std::mutex> lock(s->store_mu);
            c = s->clips[std::get<0>(g.first)].get();
        }
        ClipJob J;
        J.in = c->in;
        J.prof = s->cfg.profile;
        if (std::get<1>(g.first) > 0) J.prof.depth_hypotheses = std::get<1>(g.first);
        if (std::get<2>(g.first) > 0) J.prof.max_source_views = std::get<2>(g.first);
        J.resident = c->resident.data();
        cams.emplace_back();
        for (size_t i : g.second) {
            cams.back().push_back(batch[i].camera);
            order.push_back(i);
        }
        jobs.push_back(std::move(J));
    }
    for (size_t j = 0; j < jobs.size(); ++j) {
        jobs[j].camera_indices = cams[j].data();
        jobs[j].n_refs = cams[j].size();
    }
    const size_t n = batch.size();
    std::vector<v3d_dense_result> outs(n);
    std::vector<v3d_mesh_result> meshes(s->cfg.meshed ? n : 0);
    std::vector<int32_t> present(n, 0);
    std::vector<uint64_t> units;
    const int32_t st = clip_batch(ctx, jobs, s->cfg.fine_grid, s->cfg.profile, nullptr, nullptr,
                                  outs.data(), s->cfg.meshed ? meshes.data() : nullptr,
                                  present.data(), &units);
    const clk::time_point done = clk::now();
    {
        std::lock_guard<std::mutex> lock(s->mu);
        if (st < 0)
            s->last_error = ctx->last_error.empty() ? std::string(v3d_status_text(st))
                                                    : ctx->last_error;
        for (size_t k = 0; k < n; ++k) {
            const Request& r = batch[order[k]];
            Finished f;
            f.out = outs[k];
            if (s->cfg.meshed) f.mesh = meshes[k];
            f.present = present[k];
            f.status = st < 0 ? st : (present[k] && !outs[k].stats.attempted ? V3D_SKIPPED : V3D_OK);
            f.timing.queue_ms = ms_between(r.submitted, started);
            f.timing.service_ms = ms_between(started, done);
            f.timing.total_ms = ms_between(r.submitted, done);
            f.timing.batch_requests = n;
            f.timing.plane_view_units = st < 0 || k >= units.size() ? 0 : units[k];
            s->finished[r.ticket] = f;
        }
    }
    s->done_cv.notify_all();
}

void worker_main(v3d_server* s, size_t slot) {
    cudaSetDevice(s->cfg.device);
    v3d_context* ctx = s->ctxs[slot];
    for (;;) {
        std::vector<Request> batch;
        {
            std::unique_lock<std::mutex> lock(s->mu);
            s->work_cv.wait(lock, [&] { return s->stop || !s->pending.empty(); });
            if (s->stop) return;
            // admission in arrival order against this slot's memory budget; a
            // request larger than the budget runs alone
            uint64_t bytes = 0;
            while (!s->pending.empty()) {
                const Request& r = s->pending.front();
                if (s->cfg.max_batch_requests && batch.size() >= s->cfg.max_batch_requests) break;
                if (!batch.empty() && bytes + r.bytes > s->slot_budget) break;
                bytes += r.bytes;
                batch.push_back(r);
                s->pending.pop_front();
            }
            if (!s->pending.empty()) s->work_cv.notify_one();  // another slot takes the rest
        }
        run_batch_of_requests(s, ctx, batch, clk::now());
    }
}

void free_finished(v3d_server* s, Finished& f) {
    v3d_dense_result_free(&f.out);
    if (s->cfg.meshed) v3d_mesh_result_free(&f.mesh);
}

}  // namespace

extern "C" {

int32_t v3d_server_create(const v3d_server_config* config, v3d_server** out) {
    if (!out || !config) return V3D_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    if (config->slots < 1 || config->slots > 8) return V3D_ERR_INVALID_ARGUMENT;
    const v3d_profile& p = config->profile;
    if (p.patch_radius < 1 || p.patch_radius > V3D_MAX_PATCH_RADIUS || p.depth_hypotheses < 2 ||
        p.depth_hypotheses > V3D_MAX_DEPTH_HYPOTHESES || p.max_source_views < 1 ||
        p.max_source_views > V3D_MAX_SOURCE_VIEWS)
        return V3D_ERR_INVALID_ARGUMENT;
    auto* s = new v3d_server;
    s->cfg = *config;
    const uint64_t budget = config->memory_budget_bytes ? config->memory_budget_bytes : kDefaultBudget;
    s->slot_budget = budget / static_cast<uint64_t>(config->slots);
    for (int i = 0; i < config->slots; ++i) {
        v3d_context* ctx = nullptr;
        int32_t st = v3d_context_create(config->device, &ctx);
        if (st != V3D_OK) {
            for (v3d_context* c : s->ctxs) v3d_context_destroy(c);
            delete s;
            return st;
        }
        // a slot's buffers are allocated up front: growing them later would
        // free device memory, which waits for the other slots' batches
        if (cudaMalloc(&ctx->arena, s->slot_budget) != cudaSuccess ||
            cudaMallocHost(&ctx->pinned, kPinnedStaging) != cudaSuccess) {
            cudaGetLastError();
            v3d_context_destroy(ctx);
            for (v3d_context* c : s->ctxs) v3d_context_destroy(c);
            delete s;
            return V3D_ERR_OUT_OF_MEMORY;
        }
        ctx->arena_bytes = s->slot_budget;
        ctx->pinned_bytes = kPinnedStaging;
        s->ctxs.push_back(ctx);
    }
    cudaSetDevice(config->device);
    if (cudaStreamCreateWithFlags(&s->upload, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        for (v3d_context* c : s->ctxs) v3d_context_destroy(c);
        delete s;
        return V3D_ERR_CUDA;
    }
    for (int i = 0; i < config->slots; ++i) s->workers.emplace_back(worker_main, s, static_cast<size_t>(i));
    *out = s;
    return V3D_OK;
}

void v3d_server_destroy(v3d_server* s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        s->stop = true;
    }
    s->work_cv.notify_all();
    for (std::thread& t : s->workers) t.join();  // a batch in flight finishes first
    {
        std::lock_guard<std::mutex> lock(s->mu);
        for (const Request& r : s->pending) {
            Finished f;
            f.status = V3D_ERR_SHUTDOWN;
            s->finished[r.ticket] = f;
        }
        s->pending.clear();
        for (auto& kv : s->finished) free_finished(s, kv.second);
        s->finished.clear();
        s->outstanding.clear();
    }
    s->done_cv.notify_all();
    cudaSetDevice(s->cfg.device);
    for (v3d_context* c : s->ctxs) v3d_context_destroy(c);
    for (auto& c : s->clips)
        for (void* b : c->buffers) cudaFree(b);
    if (s->upload) cudaStreamDestroy(s->upload);
    delete s;
}

int32_t v3d_server_add_clip(v3d_server* s, const v3d_frame* frames, uint64_t n_frames,
                            const v3d_camera* cameras, uint64_t n_cameras,
                            const double* sparse_xyz, uint64_t n_sparse, double focal,
                            uint64_t* clip_id) {
    if (!s || !clip_id || (n_frames && !frames) || (n_cameras && !cameras) ||
        (n_sparse && !sparse_xyz))
        return V3D_ERR_INVALID_ARGUMENT;
    for (uint64_t i = 0; i < n_frames; ++i) {
        const v3d_frame& f = frames[i];
        if (f.format < V3D_PIXEL_RGBA8 || f.format > V3D_PIXEL_GRAY_BF16 || !f.data ||
            f.width == 0 || f.height == 0 ||
            static_cast<uint64_t>(f.width) * f.height >= (uint64_t{1} << 32))  // 32-bit offsets
            return V3D_ERR_INVALID_ARGUMENT;
        if (f.format != frames[0].format) return V3D_ERR_INVALID_ARGUMENT;
    }
    {
        std::lock_guard<std::mutex> lock(s->store_mu);
        if (n_frames && s->format >= 0 && frames[0].format != s->format)
            return V3D_ERR_INVALID_ARGUMENT;  // one pixel format per server
    }
    cudaSetDevice(s->cfg.device);
    auto c = std::make_unique<StoredClip>();
    c->frames.assign(frames, frames + n_frames);
    c->resident.resize(n_frames);
    auto fail = [&](int32_t st) {
        cudaStreamSynchronize(s->upload);
        for (void* b : c->buffers) cudaFree(b);
        cudaGetLastError();
        return st;
    };
    for (uint64_t i = 0; i < n_frames; ++i) {
        const v3d_frame& f = frames[i];
        const size_t px = static_cast<size_t>(f.width) * f.height;
        void* raw = nullptr;
        if (cudaMalloc(&raw, px * bytes_per_pixel(f.format)) != cudaSuccess) return fail(V3D_ERR_OUT_OF_MEMORY);
        c->buffers.push_back(raw);
        if (cudaMemcpyAsync(raw, f.data, px * bytes_per_pixel(f.format), cudaMemcpyHostToDevice,
                            s->upload) != cudaSuccess)
            return fail(V3D_ERR_CUDA);
        const uint8_t* luma = static_cast<const uint8_t*>(raw);
        if (f.format == V3D_PIXEL_RGBA8) {
            void* l = nullptr;
            if (cudaMalloc(&l, px) != cudaSuccess) return fail(V3D_ERR_OUT_OF_MEMORY);
            c->buffers.push_back(l);
            if (launch_luma(static_cast<const uint8_t*>(raw), static_cast<uint8_t*>(l), px, s->upload) !=
                cudaSuccess)
                return fail(V3D_ERR_CUDA);
            luma = static_cast<const uint8_t*>(l);
        }
        c->resident[i] = ResidentFrame{raw, luma};
        c->frames[i].data = nullptr;  // the pixels are read from `resident`
    }
    // the caller's host buffers may be released once this returns
    if (cudaStreamSynchronize(s->upload) != cudaSuccess) return fail(V3D_ERR_CUDA);
    c->in = load_inputs(c->frames.data(), n_frames, cameras, n_cameras, sparse_xyz, n_sparse, focal);
    if (n_frames) {
        const v3d_profile& p = s->cfg.profile;
        const uint32_t w = frames[0].width, h = frames[0].height;
        const uint32_t stride = p.grid_stride > 0 ? static_cast<uint32_t>(p.grid_stride)
                                                  : reference_grid_stride(w, h, s->cfg.fine_grid != 0);
        const uint32_t border = static_cast<uint32_t>(p.patch_radius + 2);
        const uint64_t nx = w > 2 * border ? (w - 2 * border + stride - 1) / stride : 0;
        const uint64_t ny = h > 2 * border ? (h - 2 * border + stride - 1) / stride : 0;
        c->sites = nx * ny;
    }
    std::lock_guard<std::mutex> lock(s->store_mu);
    if (n_frames && s->format < 0) s->format = frames[0].format;
    *clip_id = s->clips.size();
    s->clips.push_back(std::move(c));
    return V3D_OK;
}

int32_t v3d_server_submit(v3d_server* s, uint64_t clip_id, uint64_t camera_index,
                          int32_t depth_hypotheses, int32_t max_source_views, uint64_t* ticket) {
    if (!s || !ticket) return V3D_ERR_INVALID_ARGUMENT;
    if (depth_hypotheses != 0 &&
        (depth_hypotheses < 2 || depth_hypotheses > V3D_MAX_DEPTH_HYPOTHESES))
        return V3D_ERR_INVALID_ARGUMENT;
    if (max_source_views != 0 && (max_source_views < 1 || max_source_views > V3D_MAX_SOURCE_VIEWS))
        return V3D_ERR_INVALID_ARGUMENT;
    Request r;
    {
        std::lock_guard<std::mutex> lock(s->store_mu);
        if (clip_id >= s->clips.size() || camera_index >= s->clips[clip_id]->in.cameras.size())
            return V3D_ERR_INVALID_ARGUMENT;
        r.bytes = s->clips[clip_id]->sites * kBytesPerSite + kBytesPerReference;
    }
    r.clip = clip_id;
    r.camera = camera_index;
    r.planes = depth_hypotheses;
    r.sources = max_source_views;
    r.submitted = clk::now();
    {
        std::lock_guard<std::mutex> lock(s->mu);
        if (s->stop) return V3D_ERR_SHUTDOWN;
        r.ticket = s->next_ticket++;
        s->outstanding.insert(r.ticket);
        s->pending.push_back(r);
        *ticket = r.ticket;
    }
    s->work_cv.notify_one();
    return V3D_OK;
}

int32_t v3d_server_wait(v3d_server* s, uint64_t ticket, int64_t timeout_ms, v3d_dense_result* out,
                        v3d_mesh_result* mesh_out, int32_t* present, v3d_request_timing* timing) {
    if (!s || !out || !present) return V3D_ERR_INVALID_ARGUMENT;
    std::memset(out, 0, sizeof(*out));
    if (mesh_out) std::memset(mesh_out, 0, sizeof(*mesh_out));
    *present = 0;
    Finished f;
    {
        std::unique_lock<std::mutex> lock(s->mu);
        if (!s->outstanding.count(ticket)) return V3D_ERR_INVALID_ARGUMENT;
        auto ready = [&] { return s->finished.count(ticket) > 0; };
        if (timeout_ms < 0)
            s->done_cv.wait(lock, ready);
        else if (!s->done_cv.wait_for(lock, std::chrono::milliseconds(timeout_ms), ready))
            return V3D_ERR_TIMEOUT;
        f = s->finished[ticket];
        s->finished.erase(ticket);
        s->outstanding.erase(ticket);
    }
    *out = f.out;
    if (s->cfg.meshed) {
        if (mesh_out)
            *mesh_out = f.mesh;
        else
            v3d_mesh_result_free(&f.mesh);
    }
    *present = f.present;
    if (timing) *timing = f.timing;
    return f.status;
}

uint64_t v3d_server_last_error(v3d_server* s, char* buf, uint64_t n) {
    if (!s) return 0;
    std::lock_guard<std::mutex> lock(s->mu);
    const std::string& e = s->last_error;
    if (buf && n) {
        const uint64_t k = std::min<uint64_t>(e.size(), n - 1);
        std::memcpy(buf, e.data(), k);
        buf[k] = '\0';
    }
    return e.size();
}

}  // extern "C"
