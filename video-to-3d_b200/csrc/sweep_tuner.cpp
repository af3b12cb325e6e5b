// Measured choice of the tiled sweep's tile shape and plane chunking.
//
// Neither changes a result (the chunks' rank states merge exactly, and every
// window sum is formed tap by tap in the same order whatever the tile), so
// both can be tuned on live calls.  Batches are keyed by their launch shape
// (window radius, stride, and the power-of-two buckets of their tile count,
// hypothesis count and source count).  A key's first calls each try one
// candidate: for each tile (32x8 first, then 16x16) the occupancy heuristic's
// chunk count, twice and four times it and half of it.  Every try records the
// sweep's device time per unit of work; once all candidates have run, the key
// keeps the fastest.
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "host.hpp"

namespace v3d {
namespace {

struct Entry {
    std::vector<SweepPlan> candidates;
    std::vector<double> ms_per_unit;  // < 0: not tried yet
    int chosen = 0;                   // 1 + the kept candidate; 0: still trying
    size_t next = 0;
};

int log2_bucket(uint64_t v) {
    int b = 0;
    while (v > 1) {
        v >>= 1;
        ++b;
    }
    return b;
}

struct Tuner {
    std::mutex mu;
    std::map<std::tuple<int, int, int, int, int, int>, Entry> entries;
};

Tuner& tuner() {
    static Tuner* t = new Tuner;
    return *t;
}

}  // namespace

SweepShapeKey sweep_shape_key(int device, int radius, int stride, uint64_t tiles, int planes,
                              int sources) {
    return SweepShapeKey{device, radius, stride, log2_bucket(tiles), log2_bucket((uint64_t)planes),
                         log2_bucket((uint64_t)sources)};
}

SweepPlan sweep_plan_pick(const SweepShapeKey& key, int heuristic32, int heuristic16,
                          int max_chunks) {
    Tuner& t = tuner();
    std::lock_guard<std::mutex> lock(t.mu);
    const auto k = std::make_tuple(key.device, key.radius, key.stride, key.tiles, key.planes,
                                   key.sources);
    auto it = t.entries.find(k);
    if (it == t.entries.end()) {
        Entry e;
        for (int tile : {32, 16}) {
            const int h = tile == 32 ? heuristic32 : heuristic16;
            for (int c : {h, h * 2, h * 4, h / 2}) {
                c = std::max(1, std::min(c, max_chunks));
                bool seen = false;
                for (const SweepPlan& d : e.candidates) seen = seen || (d.tile_x == tile && d.chunks == c);
                if (!seen) e.candidates.push_back(SweepPlan{tile, c});
            }
        }
        e.ms_per_unit.assign(e.candidates.size(), -1.0);
        it = t.entries.emplace(k, e).first;
    }
    Entry& e = it->second;
    if (e.chosen) return e.candidates[e.chosen - 1];
    return e.candidates[e.next % e.candidates.size()];
}

void sweep_plan_record(const SweepShapeKey& key, SweepPlan plan, double sweep_ms, uint64_t units) {
    if (!units || !(sweep_ms > 0.0)) return;
    Tuner& t = tuner();
    std::lock_guard<std::mutex> lock(t.mu);
    auto it = t.entries.find(std::make_tuple(key.device, key.radius, key.stride, key.tiles,
                                             key.planes, key.sources));
    if (it == t.entries.end() || it->second.chosen) return;
    Entry& e = it->second;
    for (size_t i = 0; i < e.candidates.size(); ++i) {
        if (e.candidates[i].tile_x != plan.tile_x || e.candidates[i].chunks != plan.chunks ||
            e.ms_per_unit[i] >= 0.0)
            continue;
        e.ms_per_unit[i] = sweep_ms / static_cast<double>(units);
        ++e.next;
        break;
    }
    // all tried: keep the fastest
    size_t best = 0;
    for (size_t i = 0; i < e.candidates.size(); ++i) {
        if (e.ms_per_unit[i] < 0.0) return;
        if (e.ms_per_unit[i] < e.ms_per_unit[best]) best = i;
    }
    e.chosen = static_cast<int>(best) + 1;
}

}  // namespace v3d
