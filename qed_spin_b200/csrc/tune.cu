// =============================================================================
// tune.cu -- the launch-shape tuner.
//
// A kernel family with several launch shapes that give the same result bit for bit (the row walk: one thread
// per state, a warp's states compacted, or for one vector a team of 4 to 32 lanes per state; the block walk:
// 4, 8, 16 or 32 lanes per state) asks tune_choose for a shape. The first call for a shape key (the kernel family, the sector's and
// program's size classes, the vector count and types, the device) times every candidate on the caller's stream
// with CUDA events -- each candidate runs once to warm up, then three times timed (once when a run takes more than
// 50 ms, and not at all when its warm-up is already half again slower than the pick) -- and keeps the fastest;
// later calls reuse it. Because the candidates agree bit for bit, a choice changes only the time.
//
// Modes (QB_TUNE, or qb_tune_mode): 1 measure on first use (default); 2 use only choices already known (from
// this process or a loaded cache file), else the family's default; 0 always the default. A stream that is
// capturing a graph is never timed. QB_TUNE_CACHE names a text file that is read on first use and to which
// every new choice is appended: "key<TAB>choice<TAB>ms of each candidate".
// No reference counterpart: the reference fixes its launch shapes (src/gpu/rep_matvec.cu).
// =============================================================================
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <map>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include "qb_internal.cuh"

namespace qb {
namespace {

struct Choice {
    int pick = 0;
    std::vector<float> ms;
};

struct Tuner {
    std::mutex mu;
    int mode = -1;   // resolved from QB_TUNE on first use
    bool loaded = false;
    std::string path;
    std::map<std::string, Choice> known;
    std::map<std::string, int> forced;   // kernel family -> candidate

    void init_locked() {
        if (mode < 0) {
            const char* e = std::getenv("QB_TUNE");
            mode = (e && *e) ? std::atoi(e) : 1;
            if (mode < 0 || mode > 2) mode = 1;
        }
        if (!loaded) {
            loaded = true;
            const char* p = std::getenv("QB_TUNE_CACHE");
            if (p && *p) {
                path = p;
                load_locked(path);
            }
        }
    }

    bool load_locked(const std::string& file) {
        std::FILE* f = std::fopen(file.c_str(), "r");
        if (!f) return false;
        char line[4096];
        while (std::fgets(line, sizeof line, f)) {
            char* tab = std::strchr(line, '\t');
            if (!tab) continue;
            *tab = '\0';
            Choice c;
            c.pick = std::atoi(tab + 1);
            known[line] = c;
        }
        std::fclose(f);
        return true;
    }
};

Tuner& tuner() {
    static Tuner* t = new Tuner;   // never destroyed: launches may run during static destruction
    return *t;
}

std::atomic<unsigned> g_generation{1};

// The device's architecture and SM count, resolved once per device.
const std::string& device_tag() {
    static std::mutex mu;
    static std::map<int, std::string> tags;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lk(mu);
    auto it = tags.find(dev);
    if (it != tags.end()) return it->second;
    int sms = 0, major = 0, minor = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
    cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, dev);
    return tags[dev] = "sm" + std::to_string(major) + std::to_string(minor) + "x" + std::to_string(sms);
}

}  // namespace

unsigned tune_generation() { return g_generation.load(std::memory_order_relaxed); }

int tune_choose(const char* family, const std::string& key, int n, int fallback, cudaStream_t st,
                const std::function<void(int)>& run) {
    Tuner& T = tuner();
    const std::string full = std::string(family) + "|" + key + "|" + device_tag();
    int mode;
    {
        std::lock_guard<std::mutex> lk(T.mu);
        T.init_locked();
        auto f = T.forced.find(family);
        if (f != T.forced.end()) return f->second < n ? f->second : fallback;
        auto it = T.known.find(full);
        if (it != T.known.end() && it->second.pick < n) return it->second.pick;
        mode = T.mode;
    }
    if (mode != 1 || n < 2) return fallback;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    cuda_check(cudaStreamIsCapturing(st, &cap), "capture status");
    if (cap != cudaStreamCaptureStatusNone) return fallback;
    cudaEvent_t e0, e1;
    cuda_check(cudaEventCreate(&e0), "event");
    cuda_check(cudaEventCreate(&e1), "event");
    Choice c;
    float best = 0.0f;
    try {
        for (int i = 0; i < n; ++i) {
            // warm-up: module load, first touch of the tables. A long candidate (above kLongMs) whose warm-up is
            // already half again slower than the pick is not timed further, and long candidates are timed once:
            // on a 252M-state sector one walk takes seconds, and three runs of every shape took two minutes.
            cuda_check(cudaEventRecord(e0, st), "event");
            run(i);
            cuda_check(cudaEventRecord(e1, st), "event");
            cuda_check(cudaEventSynchronize(e1), "tune");
            float wms = 0.0f;
            cuda_check(cudaEventElapsedTime(&wms, e0, e1), "event time");
            constexpr float kLongMs = 50.0f;
            if (i > 0 && wms > kLongMs && wms > 1.5f * best) {
                c.ms.push_back(wms);
                continue;
            }
            const int reps = wms > kLongMs ? 1 : 3;
            cuda_check(cudaEventRecord(e0, st), "event");
            for (int r = 0; r < reps; ++r) run(i);
            cuda_check(cudaEventRecord(e1, st), "event");
            cuda_check(cudaEventSynchronize(e1), "tune");
            float ms = 0.0f;
            cuda_check(cudaEventElapsedTime(&ms, e0, e1), "event time");
            ms /= static_cast<float>(reps);
            c.ms.push_back(ms);
            // a candidate must beat the current pick by 3% to replace it (lower indices are the defaults)
            if (i == 0 || ms < 0.97f * best) {
                best = ms;
                c.pick = i;
            }
        }
    } catch (...) {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        throw;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    std::lock_guard<std::mutex> lk(T.mu);
    T.known[full] = c;
    if (!T.path.empty()) {
        if (std::FILE* f = std::fopen(T.path.c_str(), "a")) {
            std::fprintf(f, "%s\t%d", full.c_str(), c.pick);
            for (float m : c.ms) std::fprintf(f, "\t%.6f", m);
            std::fprintf(f, "\n");
            std::fclose(f);
        }
    }
    return c.pick;
}

}  // namespace qb

extern "C" {

int qb_tune_mode(int mode, int* previous) {
    return qb::guarded([&] {
        using namespace qb;
        if (mode < -1 || mode > 2) throw Error(QB_EINVAL, "tune mode must be 0, 1 or 2 (-1: query)");
        Tuner& T = tuner();
        std::lock_guard<std::mutex> lk(T.mu);
        T.init_locked();
        if (previous) *previous = T.mode;
        if (mode >= 0) T.mode = mode;
        ++g_generation;
    });
}

int qb_tune_force(const char* family, int choice) {
    return qb::guarded([&] {
        using namespace qb;
        if (!family) throw Error(QB_EINVAL, "null kernel family");
        Tuner& T = tuner();
        std::lock_guard<std::mutex> lk(T.mu);
        if (choice < 0)
            T.forced.erase(family);
        else
            T.forced[family] = choice;
        ++g_generation;
    });
}

int qb_tune_clear(void) {
    return qb::guarded([&] {
        qb::Tuner& T = qb::tuner();
        std::lock_guard<std::mutex> lk(T.mu);
        T.known.clear();
        T.forced.clear();
        ++qb::g_generation;
    });
}

int qb_tune_save(const char* path) {
    return qb::guarded([&] {
        using namespace qb;
        if (!path) throw Error(QB_EINVAL, "null path");
        Tuner& T = tuner();
        std::lock_guard<std::mutex> lk(T.mu);
        std::FILE* f = std::fopen(path, "w");
        if (!f) throw Error(QB_EINVAL, std::string("cannot write ") + path);
        for (const auto& kv : T.known) {
            std::fprintf(f, "%s\t%d", kv.first.c_str(), kv.second.pick);
            for (float m : kv.second.ms) std::fprintf(f, "\t%.6f", m);
            std::fprintf(f, "\n");
        }
        std::fclose(f);
    });
}

int qb_tune_load(const char* path) {
    return qb::guarded([&] {
        using namespace qb;
        if (!path) throw Error(QB_EINVAL, "null path");
        Tuner& T = tuner();
        std::lock_guard<std::mutex> lk(T.mu);
        T.init_locked();
        if (!T.load_locked(path)) throw Error(QB_EINVAL, std::string("cannot read ") + path);
        ++g_generation;
    });
}

int qb_tune_entries(char* buf, uint64_t len, uint64_t* needed) {
    return qb::guarded([&] {
        using namespace qb;
        Tuner& T = tuner();
        std::ostringstream os;
        {
            std::lock_guard<std::mutex> lk(T.mu);
            for (const auto& kv : T.known) {
                os << kv.first << '\t' << kv.second.pick;
                for (float m : kv.second.ms) os << '\t' << m;
                os << '\n';
            }
        }
        const std::string s = os.str();
        if (needed) *needed = s.size() + 1;
        if (buf && len) {
            const std::size_t n = std::min<std::size_t>(s.size(), len - 1);
            std::memcpy(buf, s.data(), n);
            buf[n] = '\0';
        }
    });
}

}  // extern "C"
