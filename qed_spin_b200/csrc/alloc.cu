// =============================================================================
// alloc.cu -- the device memory behind every DevBuf: a cache of released blocks.
//
// cudaFree synchronises the whole device, which would serialise solves that run concurrently from different host
// threads (the request server's workers). A released block instead goes to this per-device cache with an event
// recorded on the releasing thread's stream; a later allocation of about the same size reuses it once that event
// has completed, i.e. once every kernel the releasing thread had queued on the block has finished. Blocks are
// used and released on one thread's stream (or after a synchronisation) everywhere in this library. Idle blocks
// are capped (the oldest are freed past the cap) and freed when cudaMalloc runs out of memory.
// =============================================================================
#include <cuda_runtime.h>

#include <cstddef>
#include <list>
#include <mutex>

#include "qb_internal.cuh"

namespace qb {
namespace {

struct Block {
    void* p;
    std::size_t bytes;
    cudaEvent_t ev;
};

struct Cache {
    std::mutex mu;
    std::list<Block> idle;   // oldest first
    std::size_t idle_bytes = 0;
};

constexpr int kMaxDevices = 64;
constexpr std::size_t kIdleCap = std::size_t{16} << 30;

Cache& cache(int dev) {
    static Cache* caches = new Cache[kMaxDevices];   // never destroyed: blocks outlive static destructors at exit
    return caches[dev];
}

std::size_t rounded(std::size_t bytes) {
    const std::size_t g = bytes <= (std::size_t{1} << 20) ? 512 : (std::size_t{2} << 20);
    return (bytes + g - 1) / g * g;
}

int current_device() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) dev = 0;
    return dev;
}

// Frees idle blocks oldest first until at most `keep` idle bytes remain (the caller holds the lock).
void trim(Cache& c, std::size_t keep) {
    while (c.idle_bytes > keep && !c.idle.empty()) {
        Block b = c.idle.front();
        c.idle.pop_front();
        c.idle_bytes -= b.bytes;
        cudaEventSynchronize(b.ev);
        cudaEventDestroy(b.ev);
        cudaFree(b.p);
    }
}

}  // namespace

void* dev_alloc(std::size_t bytes) {
    const std::size_t want = rounded(bytes);
    Cache& c = cache(current_device());
    {
        std::lock_guard<std::mutex> lk(c.mu);
        for (auto it = c.idle.begin(); it != c.idle.end(); ++it) {
            if (it->bytes < want || it->bytes > want + want / 4) continue;
            if (cudaEventQuery(it->ev) != cudaSuccess) continue;   // still in use on its stream
            void* p = it->p;
            cudaEventDestroy(it->ev);
            c.idle_bytes -= it->bytes;
            c.idle.erase(it);
            return p;
        }
    }
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, want);
    if (e == cudaErrorMemoryAllocation) {
        (void)cudaGetLastError();
        {
            std::lock_guard<std::mutex> lk(c.mu);
            trim(c, 0);
        }
        e = cudaMalloc(&p, want);
    }
    cuda_check(e, "cudaMalloc");
    return p;
}

void dev_free(void* p, std::size_t bytes) {
    if (!p) return;
    Cache& c = cache(current_device());
    cudaEvent_t ev = nullptr;
    if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventRecord(ev, cudaStreamPerThread) != cudaSuccess) {
        (void)cudaGetLastError();
        if (ev) cudaEventDestroy(ev);
        cudaFree(p);   // no event: free it the synchronising way
        return;
    }
    std::lock_guard<std::mutex> lk(c.mu);
    c.idle.push_back(Block{p, rounded(bytes), ev});
    c.idle_bytes += rounded(bytes);
    trim(c, kIdleCap);
}

std::size_t idle_cached_bytes() {
    Cache& c = cache(current_device());
    std::lock_guard<std::mutex> lk(c.mu);
    return c.idle_bytes;
}

}  // namespace qb

extern "C" int qb_memory_trim(uint64_t keep_bytes, uint64_t* idle_bytes) {
    return qb::guarded([&] {
        qb::Cache& c = qb::cache(qb::current_device());
        std::lock_guard<std::mutex> lk(c.mu);
        qb::trim(c, static_cast<std::size_t>(keep_bytes));
        if (idle_bytes) *idle_bytes = c.idle_bytes;
    });
}
