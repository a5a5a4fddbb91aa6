// =============================================================================
// hostio.cu -- large host-to-device uploads from pageable memory at the link's speed.
//
// A start vector of the 6x6 sector is 4 GB of complex128 in ordinary (pageable) host memory. The driver copies
// pageable memory at about 10 GB/s on the B200 hosts here, pinned memory at about 55 GB/s. upload_host keeps a
// per-device set of pinned slots: worker threads copy the source chunk by chunk into the slots while the calling
// thread queues each chunk's DMA on the caller's stream, in order, and records the slot's event; a slot is
// refilled once its event has completed. The call returns when every chunk's copy has completed, as a pageable
// cudaMemcpy would, so the caller may reuse its buffer at once. Small copies, and sources that are not pageable host
// memory (pinned, managed or device memory), go straight to cudaMemcpyAsync.
// =============================================================================
#include <atomic>
#include <cstring>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "qb_internal.cuh"

namespace qb {
namespace {

constexpr std::size_t kChunk = std::size_t{16} << 20;
constexpr int kSlots = 16;     // 256 MB of pinned slots per device
constexpr int kWorkers = 8;    // kSlots is a multiple of kWorkers: chunk c and c - kSlots share a worker
constexpr std::size_t kStagedFrom = std::size_t{64} << 20;

struct Stager {
    std::mutex mu;                 // one staged upload at a time per device
    unsigned char* pinned = nullptr;
    cudaEvent_t ev[kSlots] = {};
    bool failed = false;           // pinned memory unavailable: plain copies
};

Stager& stager(int dev) {
    static Stager* s = new Stager[64];   // never destroyed: pinned slots live as long as the process
    return s[dev];
}

}  // namespace

void upload_host(void* dst, const void* src, std::size_t bytes, cudaStream_t st) {
    if (bytes == 0) return;
    cudaPointerAttributes attr{};
    const bool known = cudaPointerGetAttributes(&attr, src) == cudaSuccess;
    cudaGetLastError();   // an unregistered pointer may leave an error behind on older drivers
    // only ordinary (pageable) host memory is staged; pinned, managed or device sources are copied directly
    const bool pageable = !known || attr.type == cudaMemoryTypeUnregistered;
    int dev = 0;
    cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
    if (bytes < kStagedFrom || !pageable || dev < 0 || dev >= 64) {
        cuda_check(cudaMemcpyAsync(dst, src, bytes, pageable ? cudaMemcpyHostToDevice : cudaMemcpyDefault, st),
                   "upload");
        cuda_check(cudaStreamSynchronize(st), "upload");
        return;
    }
    Stager& S = stager(dev);
    std::lock_guard<std::mutex> lk(S.mu);
    if (!S.pinned && !S.failed) {
        if (cudaHostAlloc(reinterpret_cast<void**>(&S.pinned), kSlots * kChunk, cudaHostAllocPortable) != cudaSuccess) {
            cudaGetLastError();
            S.pinned = nullptr;
            S.failed = true;
        } else {
            for (auto& e : S.ev) cuda_check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event");
        }
    }
    if (S.failed) {
        cuda_check(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st), "upload");
        cuda_check(cudaStreamSynchronize(st), "upload");
        return;
    }
    const std::size_t n_chunks = (bytes + kChunk - 1) / kChunk;
    auto len_of = [&](std::size_t c) { return std::min(kChunk, bytes - c * kChunk); };
    std::unique_ptr<std::atomic<int>[]> ready(new std::atomic<int>[n_chunks]);
    for (std::size_t c = 0; c < n_chunks; ++c) ready[c].store(0, std::memory_order_relaxed);
    std::atomic<std::size_t> issued{0};   // chunks [0, issued) have their DMA queued and their slot's event recorded
    std::atomic<int> err{0};
    const auto* from = static_cast<const unsigned char*>(src);
    auto* to = static_cast<unsigned char*>(dst);
    std::vector<std::thread> workers;
    const int nw = static_cast<int>(std::min<std::size_t>(kWorkers, n_chunks));
    for (int w = 0; w < nw; ++w) {
        workers.emplace_back([&, w] {
            if (cudaSetDevice(dev) != cudaSuccess) err.store(1);
            for (std::size_t c = static_cast<std::size_t>(w); c < n_chunks; c += kWorkers) {
                const int slot = static_cast<int>(c % kSlots);
                if (c >= static_cast<std::size_t>(kSlots)) {
                    // the slot's previous chunk (c - kSlots, this worker's) must be queued, then copied out
                    while (issued.load(std::memory_order_acquire) <= c - kSlots && !err.load()) std::this_thread::yield();
                    if (err.load() || cudaEventSynchronize(S.ev[slot]) != cudaSuccess) {
                        err.store(1);
                        ready[c].store(1, std::memory_order_release);
                        continue;
                    }
                }
                std::memcpy(S.pinned + slot * kChunk, from + c * kChunk, len_of(c));
                ready[c].store(1, std::memory_order_release);
            }
        });
    }
    cudaError_t e = cudaSuccess;
    for (std::size_t c = 0; c < n_chunks; ++c) {
        while (!ready[c].load(std::memory_order_acquire)) std::this_thread::yield();
        if (e == cudaSuccess && !err.load()) {
            const int slot = static_cast<int>(c % kSlots);
            e = cudaMemcpyAsync(to + c * kChunk, S.pinned + slot * kChunk, len_of(c), cudaMemcpyHostToDevice, st);
            if (e == cudaSuccess) e = cudaEventRecord(S.ev[slot], st);
        }
        if (e != cudaSuccess) err.store(1);
        issued.store(c + 1, std::memory_order_release);
    }
    for (auto& t : workers) t.join();
    const cudaError_t s = cudaStreamSynchronize(st);
    cuda_check(e, "staged upload");
    cuda_check(s, "staged upload");
    if (err.load()) throw Error(QB_ECUDA, "staged upload: a pinned slot could not be reused");
}

}  // namespace qb
