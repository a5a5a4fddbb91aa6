// =============================================================================
// registry.cu -- sectors by content, and a file format for a sector's basis.
//
// qb_sector_acquire hands out one device sector per descriptor (the device, the group, the characters, the
// representative order and the lookup): repeated requests for the same block share it instead of enumerating
// it again, as the reference's content-keyed sector mirrors are shared (src/gpu/rep_matvec.cu:501-609, a weak
// registry plus a byte-bounded strong FIFO) and its orbit tables are kept in a registry
// (include/ed/basis/orbit_table.h). Released sectors stay cached, oldest evicted first past a byte capacity.
//
// qb_sector_save / qb_sector_load write and read a sector's descriptor, representatives and 1/norms
// (little-endian): "QBSECT01", u32 version, i32 n_sites, n_up, group_size, sublattice_mode, lookup, u32 has_flips,
// i32 perms[G N], u64 flips[G] (if any), f64 chars[2 G], u64 dim, u64 reps[dim], f64 inv_norms[dim], u64 FNV-1a of
// the representative and 1/norm bytes. Loading rebuilds the tables and the lookup from the descriptor.
// =============================================================================
#include <cstdio>
#include <cstring>
#include <list>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "qb_internal.cuh"

namespace qb {
namespace {

std::string key_of(const qb_sector_desc& d, int device) {
    std::string k;
    auto put = [&](const void* p, std::size_t n) { k.append(static_cast<const char*>(p), n); };
    const int head[6] = {device, d.n_sites, d.n_up, d.group_size, d.sublattice_mode, d.lookup};
    put(head, sizeof(head));
    put(d.perms, static_cast<std::size_t>(d.group_size) * d.n_sites * sizeof(int32_t));
    const char has = d.flips ? 1 : 0;
    put(&has, 1);
    if (d.flips) put(d.flips, static_cast<std::size_t>(d.group_size) * sizeof(uint64_t));
    put(d.chars, 2 * static_cast<std::size_t>(d.group_size) * sizeof(double));
    return k;
}

struct Entry {
    qb_sector* s = nullptr;
    int refs = 0;
    std::uint64_t bytes = 0;
};

struct Registry {
    std::mutex mu;
    std::map<std::string, Entry> by_key;
    std::map<const qb_sector*, std::string> key_of_ptr;
    std::list<std::string> idle;   // released entries, oldest first
    std::uint64_t idle_bytes = 0;
    std::uint64_t capacity = 4ULL << 30;

    // Evicts the oldest idle entries past the capacity; returns the sectors to delete outside the lock.
    std::vector<qb_sector*> trim() {
        std::vector<qb_sector*> out;
        while (idle_bytes > capacity && !idle.empty()) {
            const std::string k = idle.front();
            idle.pop_front();
            auto it = by_key.find(k);
            if (it == by_key.end()) continue;
            idle_bytes -= it->second.bytes;
            key_of_ptr.erase(it->second.s);
            out.push_back(it->second.s);
            by_key.erase(it);
        }
        return out;
    }
};

Registry& registry() {
    static Registry* r = new Registry;   // never destroyed: sectors outlive static destructors at exit
    return *r;
}

void drop(std::vector<qb_sector*>& v) {
    for (auto* s : v) {
        s->registered = false;
        delete s;
    }
}

std::uint64_t fnv1a(std::uint64_t h, const void* p, std::size_t n) {
    const unsigned char* b = static_cast<const unsigned char*>(p);
    for (std::size_t i = 0; i < n; ++i) {
        h ^= b[i];
        h *= 0x100000001b3ULL;
    }
    return h;
}

struct File {
    std::FILE* f = nullptr;
    ~File() {
        if (f) std::fclose(f);
    }
};

}  // namespace
}  // namespace qb

extern "C" {

int qb_sector_acquire(const qb_sector_desc* d, qb_sector** out) {
    return qb::guarded([&] {
        using namespace qb;
        if (!d || !out) throw Error(QB_EINVAL, "null argument");
        if (d->group_size < 1 || !d->perms || !d->chars || d->n_sites < 1 || d->n_sites > 64)
            throw Error(QB_EINVAL, "malformed sector description");
        int dev = 0;
        cuda_check(cudaGetDevice(&dev), "device");
        const std::string key = key_of(*d, dev);
        Registry& R = registry();
        {
            std::lock_guard<std::mutex> lk(R.mu);
            auto it = R.by_key.find(key);
            if (it != R.by_key.end()) {
                if (it->second.refs++ == 0) {
                    R.idle.remove(key);
                    R.idle_bytes -= it->second.bytes;
                }
                *out = it->second.s;
                return;
            }
        }
        qb_sector* s = nullptr;   // enumerated outside the lock: other blocks are acquired meanwhile
        const int rc = qb_sector_create(d, &s);
        if (rc != QB_OK) throw Error(rc, qb_last_error());
        std::lock_guard<std::mutex> lk(R.mu);
        auto it = R.by_key.find(key);
        if (it != R.by_key.end()) {   // another thread made it first: use that one
            if (it->second.refs++ == 0) {
                R.idle.remove(key);
                R.idle_bytes -= it->second.bytes;
            }
            delete s;
            *out = it->second.s;
            return;
        }
        s->registered = true;
        R.by_key[key] = Entry{s, 1, s->device_bytes()};
        R.key_of_ptr[s] = key;
        *out = s;
    });
}

int qb_sector_release(qb_sector* s) {
    return qb::guarded([&] {
        using namespace qb;
        if (!s) return;
        Registry& R = registry();
        std::vector<qb_sector*> gone;
        {
            std::lock_guard<std::mutex> lk(R.mu);
            auto p = R.key_of_ptr.find(s);
            if (p == R.key_of_ptr.end()) throw Error(QB_EINVAL, "the sector was not acquired");
            Entry& e = R.by_key[p->second];
            if (e.refs <= 0) throw Error(QB_EINVAL, "the sector was released more times than acquired");
            if (--e.refs == 0) {
                R.idle.push_back(p->second);
                R.idle_bytes += e.bytes;
                gone = R.trim();
            }
        }
        drop(gone);
    });
}

int qb_registry_capacity(uint64_t bytes) {
    return qb::guarded([&] {
        using namespace qb;
        Registry& R = registry();
        std::vector<qb_sector*> gone;
        {
            std::lock_guard<std::mutex> lk(R.mu);
            R.capacity = bytes;
            gone = R.trim();
        }
        drop(gone);
    });
}

int qb_registry_stats(uint64_t* sectors, uint64_t* idle_sectors, uint64_t* idle_bytes) {
    return qb::guarded([&] {
        qb::Registry& R = qb::registry();
        std::lock_guard<std::mutex> lk(R.mu);
        if (sectors) *sectors = R.by_key.size();
        if (idle_sectors) *idle_sectors = R.idle.size();
        if (idle_bytes) *idle_bytes = R.idle_bytes;
    });
}

int qb_sector_save(const qb_sector* s, const char* path) {
    return qb::guarded([&] {
        using namespace qb;
        if (!s || !path) throw Error(QB_EINVAL, "null argument");
        std::vector<std::uint64_t> reps(s->dim);
        std::vector<double> inv(s->dim);
        if (s->dim) {
            cuda_check(cudaMemcpy(reps.data(), s->reps.p, s->dim * 8, cudaMemcpyDeviceToHost), "download");
            cuda_check(cudaMemcpy(inv.data(), s->inv_norms.p, s->dim * 8, cudaMemcpyDeviceToHost), "download");
        }
        File f;
        f.f = std::fopen(path, "wb");
        if (!f.f) throw Error(QB_EINVAL, std::string("cannot write ") + path);
        auto w = [&](const void* p, std::size_t n) {
            if (n && std::fwrite(p, 1, n, f.f) != n) throw Error(QB_EINVAL, std::string("write failed: ") + path);
        };
        const std::uint32_t version = 1, has_flips = s->desc_flips.empty() ? 0 : 1;
        const std::int32_t head[5] = {s->N, s->n_up, s->G, s->desc_slc_mode, s->desc_lookup};
        w("QBSECT01", 8);
        w(&version, 4);
        w(head, sizeof(head));
        w(&has_flips, 4);
        w(s->desc_perms.data(), s->desc_perms.size() * 4);
        if (has_flips) w(s->desc_flips.data(), s->desc_flips.size() * 8);
        w(s->chars_host.data(), s->chars_host.size() * 8);
        const std::uint64_t dim = s->dim;
        w(&dim, 8);
        w(reps.data(), dim * 8);
        w(inv.data(), dim * 8);
        std::uint64_t h = fnv1a(0xcbf29ce484222325ULL, reps.data(), dim * 8);
        h = fnv1a(h, inv.data(), dim * 8);
        w(&h, 8);
    });
}

int qb_sector_load(const char* path, qb_sector** out) {
    return qb::guarded([&] {
        using namespace qb;
        if (!path || !out) throw Error(QB_EINVAL, "null argument");
        File f;
        f.f = std::fopen(path, "rb");
        if (!f.f) throw Error(QB_EINVAL, std::string("cannot read ") + path);
        auto r = [&](void* p, std::size_t n) {
            if (n && std::fread(p, 1, n, f.f) != n) throw Error(QB_EINVAL, std::string("truncated sector file ") + path);
        };
        char magic[8];
        r(magic, 8);
        if (std::memcmp(magic, "QBSECT01", 8) != 0) throw Error(QB_EINVAL, "not a sector file");
        std::uint32_t version = 0, has_flips = 0;
        std::int32_t head[5];
        r(&version, 4);
        if (version != 1) throw Error(QB_EUNSUPPORTED, "sector file version " + std::to_string(version));
        r(head, sizeof(head));
        r(&has_flips, 4);
        const int N = head[0], G = head[2];
        if (N < 1 || N > 64 || G < 1 || G > (1 << 20)) throw Error(QB_EINVAL, "malformed sector file");
        std::vector<std::int32_t> perms(static_cast<std::size_t>(G) * N);
        std::vector<std::uint64_t> flips(has_flips ? G : 0);
        std::vector<double> chars(2 * static_cast<std::size_t>(G));
        r(perms.data(), perms.size() * 4);
        if (has_flips) r(flips.data(), flips.size() * 8);
        r(chars.data(), chars.size() * 8);
        std::uint64_t dim = 0;
        r(&dim, 8);
        if (dim > (1ULL << 40)) throw Error(QB_EINVAL, "malformed sector file");
        std::vector<std::uint64_t> reps(dim);
        std::vector<double> inv(dim);
        r(reps.data(), dim * 8);
        r(inv.data(), dim * 8);
        std::uint64_t stored = 0;
        r(&stored, 8);
        std::uint64_t h = fnv1a(0xcbf29ce484222325ULL, reps.data(), dim * 8);
        h = fnv1a(h, inv.data(), dim * 8);
        if (h != stored) throw Error(QB_EINVAL, "sector file checksum mismatch");
        qb_sector_desc d{};
        d.n_sites = N;
        d.n_up = head[1];
        d.group_size = G;
        d.perms = perms.data();
        d.flips = has_flips ? flips.data() : nullptr;
        d.chars = chars.data();
        d.sublattice_mode = head[3];
        d.lookup = head[4];
        const int rc = qb_sector_create_from_reps(&d, reps.data(), inv.data(), dim, out);
        if (rc != QB_OK) throw Error(rc, qb_last_error());
    });
}

}  // extern "C"
