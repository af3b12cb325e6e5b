// Pinned host blocks that result arrays live in.
//
// A batch's points, grid sites, attributes and triangles are copied from the
// device straight into one page-locked block, and every per-reference result
// of the batch points into it.  The block is reference counted (one count per
// PassResult copy, per C result and per mesh result); when the last holder
// lets go it returns to a process-wide cache instead of being unpinned.
// A fresh block is pinned together with a spare of its size, so a caller that
// keeps one call's results while it makes the next alternates between two
// blocks and never pins (or page-faults) again.
#include <cuda_runtime.h>

#include <map>
#include <mutex>

#include "host.hpp"

namespace v3d {
namespace {

// Blocks come in power-of-two sizes from 2 MiB, so results of varying size
// (one small request after another in a serving loop) share a few classes.
constexpr size_t kMinBlock = size_t{2} << 20;
// Bytes of free blocks kept pinned: unpinning waits for the device, so the
// cache lets go of blocks only beyond this.
constexpr size_t kCachedBytes = size_t{2} << 30;

size_t size_class(size_t bytes) {
    size_t c = kMinBlock;
    while (c < bytes) c <<= 1;
    return c;
}

struct BlockCache {
    std::mutex mu;
    std::multimap<size_t, void*> free;  // bytes -> block
    size_t free_bytes = 0;
};

// Never destroyed: holders may release blocks during static destruction.
BlockCache& cache() {
    static BlockCache* c = new BlockCache;
    return *c;
}

void recycle(void* p, size_t bytes) {
    BlockCache& c = cache();
    void* drop = nullptr;
    {
        std::lock_guard<std::mutex> lock(c.mu);
        c.free.emplace(bytes, p);
        c.free_bytes += bytes;
        if (c.free_bytes > kCachedBytes && c.free.size() > 1) {
            // unpin the largest other block: the cap is about bytes
            auto it = std::prev(c.free.end());
            if (it->second == p) --it;
            drop = it->second;
            c.free_bytes -= it->first;
            c.free.erase(it);
        }
    }
    if (drop) cudaFreeHost(drop);
}

// Deleter of a block: back to the cache; carries the block's capacity.
struct BlockRecycler {
    size_t bytes;
    void operator()(uint8_t* q) const { recycle(q, bytes); }
};

}  // namespace

HostBlock host_block(size_t bytes) {
    bytes = size_class(bytes);
    BlockCache& c = cache();
    void* p = nullptr;
    size_t have = 0;
    {
        std::lock_guard<std::mutex> lock(c.mu);
        // the smallest cached block that fits, at most two classes up
        auto it = c.free.lower_bound(bytes);
        if (it != c.free.end() && it->first <= 4 * bytes) {
            p = it->second;
            have = it->first;
            c.free_bytes -= it->first;
            c.free.erase(it);
        }
    }
    if (!p) {
        if (cudaHostAlloc(&p, bytes, cudaHostAllocPortable) != cudaSuccess) {
            cudaGetLastError();
            return HostBlock();
        }
        have = bytes;
        // Pin a spare of the same size as well: a caller that keeps one call's
        // results while it makes the next needs two blocks, and pinning (which
        // can stall the other CUDA calls of the process) then happens once.
        void* spare = nullptr;
        if (cudaHostAlloc(&spare, bytes, cudaHostAllocPortable) == cudaSuccess)
            recycle(spare, bytes);
        else
            cudaGetLastError();
    }
    return HostBlock(static_cast<uint8_t*>(p), BlockRecycler{have});
}

size_t host_block_bytes(const HostBlock& b) {
    const BlockRecycler* d = std::get_deleter<BlockRecycler>(b);
    return d ? d->bytes : 0;
}

}  // namespace v3d
