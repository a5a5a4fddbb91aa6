// =============================================================================
// sector.cu -- a symmetry sector on the device: the group tables, the sublattice key order, the
// device enumeration of the representatives, and the state -> index lookup.
//
// The enumeration replaces the reference's host orbit scan + filter
// (include/ed/basis/orbit_table.h:147-286, src/engine/group_sector.cpp:159-205): the C(N, n_up)
// states are cut into chunks of consecutive combinadic ranks; each thread unranks its chunk's
// first state and walks the rest in Gosper order (include/ed/basis/gosper.h:24), keeping a state
// when no element maps it below itself (in the key order with a sublattice code) and its projected
// norm |sum_{h in Stab} chi(h)|^2 / |Stab| exceeds 1e-12. A count pass, an exclusive scan and a
// write pass place the representatives in ascending order, bit-identical to the reference's table.
// =============================================================================
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <numeric>

#include "qb_canon.cuh"

namespace qb {

thread_local std::string g_last_error;
void set_last_error(const std::string& m) { g_last_error = m; }

thread_local std::size_t g_allowance = 0;
void set_thread_allowance(std::size_t bytes) { g_allowance = bytes; }
std::size_t available_bytes() {
    std::size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) free_b = 0;
    free_b += idle_cached_bytes();   // released blocks the cache would hand out again
    return g_allowance ? std::min(free_b, g_allowance) : free_b;
}

namespace {

// -------------------------------------------------------------------------------------------
// Host builders of the small tables.
// -------------------------------------------------------------------------------------------

// Byte-decomposition image table (compiled_group.h:108-140): lut[(g bpw + b) 256 + v].
std::vector<u64> build_lut(const int32_t* perms, int G, int N) {
    const int bpw = (N + 7) / 8;
    std::vector<u64> lut(static_cast<std::size_t>(G) * bpw * 256, 0ULL);
    for (int g = 0; g < G; ++g) {
        int inv[64];
        for (int i = 0; i < N; ++i) inv[perms[g * N + i]] = i;
        for (int b = 0; b < bpw; ++b)
            for (int v = 0; v < 256; ++v) {
                u64 out = 0;
                for (int t = 0; t < 8 && 8 * b + t < N; ++t)
                    if ((v >> t) & 1) out |= 1ULL << inv[8 * b + t];
                lut[(static_cast<std::size_t>(g) * bpw + b) * 256 + v] = out;
            }
    }
    return lut;
}

struct SlcHost {
    bool on = false;
    bool contig = false;
    int L = 0, m = 0;
    std::vector<u64> bmask;   // the sites of each block
    std::vector<u64> to_key;
    std::vector<u16> lead;
    std::vector<u32> cand_off;
    std::vector<u16> cand;
};

// ---- the sublattice key order ----------------------------------------------------------------
// The rule (the reference's, include/ed/basis/sublattice_code.h:23-34 and 164-191; the tables it fixes are
// what the representatives depend on, the code below is this file's own):
//   * a block system is a partition of the sites that every element of the group maps block onto block;
//   * for each site b = 1 .. N-1 in turn, the finest block system in which sites 0 and b share a block is a
//     candidate; the code takes the first candidate with the largest block size L whose blocks are all of
//     size L, with L <= 16 and 2 <= N / L <= 8 (none: no code);
//   * blocks are numbered by their smallest site, and the t-th smallest site of block j takes key bit
//     N - (j + 1) L + t, so block 0 leads the key;
//   * an element g brings one block j(g) of the state onto block 0 of the image. For a pattern x of block j
//     (bit t: the t-th site of the block), lead[j][x] is the least block-0 pattern (flips applied) among the
//     elements with j(g) = j, and cand[j][x] lists, ascending, the elements that reach it.
// The code applies only under the size rule of `mode`: 1 whenever a block system exists, -1 for N >= 24 and
// at least 16 distinct permutations, -2 the same with 64; 0 never; nor for G <= 1, N < 4, N > 64, G > 65535.

// The finest block system in which sites 0 and b share a block: as every element maps a block system onto
// itself, it is the set of connected components of the graph whose edges are the images of the pair (0, b)
// under the group. Returns the block of every site, blocks numbered by their smallest site.
std::vector<int> pair_closure(const std::vector<std::vector<int>>& perms, int N, int b) {
    std::vector<std::vector<int>> adj(N);
    for (const auto& p : perms) {
        adj[p[0]].push_back(p[b]);
        adj[p[b]].push_back(p[0]);
    }
    std::vector<int> label(N, -1);
    int next = 0;
    std::vector<int> stack;
    for (int s = 0; s < N; ++s) {   // ascending sites: labels come in order of the blocks' smallest sites
        if (label[s] >= 0) continue;
        label[s] = next;
        stack.assign(1, s);
        while (!stack.empty()) {
            const int u = stack.back();
            stack.pop_back();
            for (int v : adj[u])
                if (label[v] < 0) {
                    label[v] = next;
                    stack.push_back(v);
                }
        }
        ++next;
    }
    return label;
}

// The chosen block system (block of every site) and its block size L, or an empty vector.
std::vector<int> choose_blocks(const std::vector<std::vector<int>>& perms, int N, int& L) {
    L = 0;
    std::vector<int> chosen;
    for (int b = 1; b < N; ++b) {
        std::vector<int> block = pair_closure(perms, N, b);
        const int nblocks = *std::max_element(block.begin(), block.end()) + 1;
        if (N % nblocks != 0) continue;
        const int l = N / nblocks;
        if (l <= L || l > 16 || nblocks < 2 || nblocks > 8) continue;
        std::vector<int> size(nblocks, 0);
        for (int x : block) ++size[x];
        if (std::any_of(size.begin(), size.end(), [l](int z) { return z != l; })) continue;
        L = l;
        chosen = std::move(block);
    }
    return chosen;
}

// The key-order tables of the group (perms G x N, flips G or null) under `mode`.
SlcHost build_slc(const int32_t* perms, const u64* flips, int G, int N, int mode) {
    SlcHost c;
    if (mode == 0 || G <= 1 || N < 4 || N > 64 || G > 65535) return c;
    std::vector<std::vector<int>> distinct;
    for (int g = 0; g < G; ++g) {
        std::vector<int> p(perms + static_cast<std::size_t>(g) * N, perms + static_cast<std::size_t>(g + 1) * N);
        if (std::find(distinct.begin(), distinct.end(), p) == distinct.end()) distinct.push_back(std::move(p));
    }
    if (mode != 1) {
        const std::size_t least = mode == -1 ? 16 : 64;
        if (N < 24 || distinct.size() < least) return c;
    }
    int L = 0;
    const std::vector<int> block = choose_blocks(distinct, N, L);
    if (block.empty()) return c;
    const int m = N / L;
    // members[j]: block j's sites ascending; slot[s]: the position of site s in its block
    std::vector<std::vector<int>> members(m);
    std::vector<int> slot(N);
    for (int s = 0; s < N; ++s) {
        slot[s] = static_cast<int>(members[block[s]].size());
        members[block[s]].push_back(s);
    }
    c.on = true;
    c.L = L;
    c.m = m;
    c.bmask.assign(m, 0ULL);
    c.contig = true;
    for (int s = 0; s < N; ++s) {
        c.bmask[block[s]] |= 1ULL << s;
        if (block[s] != s / L || slot[s] != s % L) c.contig = false;
    }
    const int bpw = (N + 7) / 8;
    std::vector<int> key_bit(N);
    for (int s = 0; s < N; ++s) key_bit[s] = N - (block[s] + 1) * L + slot[s];
    c.to_key.assign(static_cast<std::size_t>(bpw) * 256, 0ULL);
    for (int s = 0; s < N; ++s)   // byte table b, value v: the key bits of the set sites of byte b
        for (int v = 0; v < 256; ++v)
            if ((v >> (s & 7)) & 1) c.to_key[static_cast<std::size_t>(s >> 3) * 256 + v] |= 1ULL << key_bit[s];
    // each element as two byte tables over a source-block pattern, its flip pattern and its source block
    struct Elem {
        int src;
        u32 flip;
        u32 lo[256], hi[256];
    };
    std::vector<Elem> el(G);
    for (int g = 0; g < G; ++g) {
        const int32_t* p = perms + static_cast<std::size_t>(g) * N;
        Elem& e = el[g];
        e.src = block[p[members[0][0]]];
        e.flip = 0;
        std::fill(e.lo, e.lo + 256, 0u);
        std::fill(e.hi, e.hi + 256, 0u);
        for (int t = 0; t < L; ++t) {
            const int from = slot[p[members[0][t]]];   // image bit t reads source-pattern bit `from`
            u32* tab = from < 8 ? e.lo : e.hi;
            for (int v = 0; v < 256; ++v)
                if ((v >> (from & 7)) & 1) tab[v] |= 1u << t;
            if (flips && ((flips[g] >> members[0][t]) & 1ULL)) e.flip |= 1u << t;
        }
    }
    const std::size_t P = std::size_t{1} << L;
    c.lead.assign(static_cast<std::size_t>(m) * P, 0);
    c.cand_off.assign(static_cast<std::size_t>(m) * P + 1, 0);
    c.cand.clear();
    std::vector<int> by_src;
    for (int j = 0; j < m; ++j) {
        by_src.clear();
        for (int g = 0; g < G; ++g)
            if (el[g].src == j) by_src.push_back(g);
        for (std::size_t x = 0; x < P; ++x) {
            const std::size_t at = static_cast<std::size_t>(j) * P + x;
            c.cand_off[at] = static_cast<u32>(c.cand.size());
            u32 best = 0xFFFFFFFFu;
            for (int g : by_src) {
                const Elem& e = el[g];
                const u32 img = (e.lo[x & 0xFF] | e.hi[(x >> 8) & 0xFF]) ^ e.flip;
                if (img < best) {
                    best = img;
                    c.cand.resize(c.cand_off[at]);
                }
                if (img == best) c.cand.push_back(static_cast<u16>(g));
            }
            c.lead[at] = static_cast<u16>(best);
        }
    }
    c.cand_off[static_cast<std::size_t>(m) * P] = static_cast<u32>(c.cand.size());
    return c;
}

// Pascal triangle C(n, k), n, k <= 64, row-major 65 x 65.
std::vector<u64> pascal() {
    std::vector<u64> c(65 * 65, 0ULL);
    for (int n = 0; n <= 64; ++n) {
        c[n * 65] = 1;
        for (int k = 1; k <= n; ++k) c[n * 65 + k] = c[(n - 1) * 65 + k - 1] + (k <= n - 1 ? c[(n - 1) * 65 + k] : 0);
    }
    return c;
}

// rank_lut[(b (N+1) + below) 256 + v]: the share of byte b (value v, `below` set bits under it) of
// the colex rank, sum over its set bits q (the i-th, 1-based) of C(8b + q, below + i).
std::vector<u64> build_rank_lut(int N) {
    const auto C = pascal();
    const int bpw = (N + 7) / 8;
    std::vector<u64> lut(static_cast<std::size_t>(bpw) * (N + 1) * 256, 0ULL);
    for (int b = 0; b < bpw; ++b)
        for (int below = 0; below <= N; ++below)
            for (int v = 0; v < 256; ++v) {
                u64 r = 0;
                int i = 0;
                for (int q = 0; q < 8 && 8 * b + q < N; ++q)
                    if ((v >> q) & 1) {
                        ++i;
                        const int n = 8 * b + q, k = below + i;
                        if (k <= 64 && n <= 64) r += C[n * 65 + k];
                    }
                lut[(static_cast<std::size_t>(b) * (N + 1) + below) * 256 + v] = r;
            }
    return lut;
}

// -------------------------------------------------------------------------------------------
// Device enumeration.
// -------------------------------------------------------------------------------------------
__device__ __forceinline__ u64 unrank_dev(u64 rank, int n, int k, const u64* C) {
    u64 s = 0;
    for (int i = k - 1; i >= 0; --i) {
        int p = i;
        while (p + 1 < n && __ldg(C + (p + 1) * 65 + (i + 1)) <= rank) ++p;
        s |= 1ULL << p;
        rank -= __ldg(C + p * 65 + (i + 1));
    }
    return s;
}

__device__ __forceinline__ u64 gosper_next(u64 v) {
    const u64 c = v & (~v + 1ULL);
    const u64 r = v + c;
    return (((r ^ v) >> 2) >> (__ffsll(static_cast<long long>(c)) - 1)) | r;
}

// visit_state + projected norm (orbit_table.h:93-99, 147-171; group_sector.cpp:183-186): 0 when s is
// not a kept representative, else 1/norm.
__device__ __forceinline__ double visit_inv_norm(const DSector& S, const Tables& T, u64 s) {
    double sre = 0.0, sim = 0.0;
    int cnt = 0;
    if (S.slc.on) {
        const u64 k = key_of<u64>(T.to_key, S.bpw, s);
        // the least leading block over the blocks vs the state's own (visit_state's early exit)
        u32 least = 0xFFFFFFFFu;
        for (int j = 0; j < S.slc.m; ++j) {
            const u32 v = static_cast<u32>(T.pack[(static_cast<u32>(j) << S.slc.L) + pattern_of<u64>(k, j, S.N, S.slc.L)] &
                                           0xFFFFu);
            least = v < least ? v : least;
        }
        if (least < pattern_of<u64>(k, 0, S.N, S.slc.L)) return 0.0;
        bool rep = true;
        for_each_candidate(S, T.pack, [&](int j) { return pattern_of<u64>(k, j, S.N, S.slc.L); }, [&](int g) {
            if (!rep) return;
            const u64 ik = key_of<u64>(T.to_key, S.bpw, apply_elem<u64>(S, T, s, g));
            if (ik < k) {
                rep = false;
            } else if (ik == k) {
                const double2 c = T.chars[g];
                sre = __dadd_rn(sre, c.x);
                sim = __dadd_rn(sim, c.y);
                ++cnt;
            }
        });
        if (!rep) return 0.0;
    } else {
        for (int g = 0; g < S.G; ++g) {
            const u64 img = apply_elem<u64>(S, T, s, g);
            if (img < s) return 0.0;
            if (img == s) {
                const double2 c = T.chars[g];
                sre = __dadd_rn(sre, c.x);
                sim = __dadd_rn(sim, c.y);
                ++cnt;
            }
        }
    }
    double nsq = 1.0;
    if (cnt != 1) {
        // |sum|^2 as std::norm takes it (|z| squared); exact for a real sum
        const double a = (sim == 0.0) ? fabs(sre) : hypot(sre, sim);
        nsq = __ddiv_rn(__dmul_rn(a, a), static_cast<double>(cnt));
    }
    return nsq <= 1e-12 ? 0.0 : __ddiv_rn(1.0, __dsqrt_rn(nsq));
}

__global__ void enum_kernel(DSector S, u64 total, u64 chunk, u64 n_chunks, const u64* C, u64* counts,
                            const u64* offsets, u64* out_reps, double* out_inv) {
    extern __shared__ __align__(16) unsigned char smem[];
    const Tables T = stage_tables(S, smem);
    __syncthreads();
    const u64 stride = static_cast<u64>(gridDim.x) * blockDim.x;
    for (u64 c = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x; c < n_chunks; c += stride) {
        const u64 begin = c * chunk;
        const u64 end = begin + chunk < total ? begin + chunk : total;
        u64 s = unrank_dev(begin, S.N, S.n_up, C);
        u64 cnt = 0;
        const u64 off = offsets ? offsets[c] : 0;
        for (u64 i = begin; i < end; ++i) {
            const double inv = visit_inv_norm(S, T, s);
            if (inv != 0.0) {
                if (offsets) {
                    out_reps[off + cnt] = s;
                    out_inv[off + cnt] = inv;
                }
                ++cnt;
            }
            if (i + 1 < end) s = gosper_next(s);
        }
        if (!offsets) counts[c] = cnt;
    }
}

__global__ void rank_table_kernel(DSector S, std::int32_t* table) {
    const u64 i = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= S.dim) return;
    table[rank_of(S, S.reps[i])] = static_cast<std::int32_t>(i);
}

__global__ void bucket_kernel(const u64* reps, u64 dim, u64 base, int shift, u64 nb, u32* off) {
    const u64 i = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= dim) return;
    const u64 b = (reps[i] - base) >> shift;
    const u64 from = i == 0 ? 0 : ((reps[i - 1] - base) >> shift) + 1;
    for (u64 c = from; c <= b; ++c) off[c] = static_cast<u32>(i);
    if (i == dim - 1)
        for (u64 c = b + 1; c <= nb; ++c) off[c] = static_cast<u32>(dim);
}

// The distinct 1/norm values (bit patterns) into a small open-addressing set; overflow flags a set
// too small (the lookup then reads inv_norms directly).
constexpr int kClassSet = 4096;
__global__ void class_set_kernel(const double* inv, u64 dim, u64* set, int* overflow) {
    const u64 i = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= dim) return;
    const u64 v = static_cast<u64>(__double_as_longlong(inv[i]));
    u32 h = static_cast<u32>((v * 0x9E3779B97F4A7C15ULL) >> 52) & (kClassSet - 1);
    for (int probe = 0; probe < kClassSet; ++probe) {
        const u64 old = atomicCAS(reinterpret_cast<unsigned long long*>(set + h), ~0ULL, v);
        if (old == ~0ULL || old == v) return;
        h = (h + 1) & (kClassSet - 1);
    }
    *overflow = 1;
}

// Insert every representative: its state, index and 1/norm class (binary search in the sorted classes).
__global__ void hash_insert_kernel(const u64* reps, const double* inv, u64 dim, ulonglong2* slots, int bits,
                                   const u64* classes, int n_class) {
    const u64 i = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= dim) return;
    const u64 s = reps[i];
    u64 cls = 0;
    if (n_class > 0) {
        const u64 v = static_cast<u64>(__double_as_longlong(inv[i]));
        int lo = 0, hi = n_class;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (classes[mid] < v)
                lo = mid + 1;
            else
                hi = mid;
        }
        cls = static_cast<u64>(lo);
    }
    const u64 mask = (1ULL << bits) - 1ULL;
    u64 h = hash_slot(s, bits);
    for (;;) {
        const u64 old = atomicCAS(reinterpret_cast<unsigned long long*>(&slots[h].x), ~0ULL, s);
        if (old == ~0ULL) {
            slots[h].y = i | (cls << 32);
            return;
        }
        h = (h + 1) & mask;
    }
}

// The compact table: every representative's 32-bit state and index | class << idx_bits in one 8-byte slot.
__global__ void hash_insert8_kernel(const u64* reps, const double* inv, u64 dim, u64* slots, int bits, int idx_bits,
                                    const u64* classes, int n_class) {
    const u64 i = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= dim) return;
    const u64 s = reps[i];
    u64 cls = 0;
    if (n_class > 0) {
        const u64 v = static_cast<u64>(__double_as_longlong(inv[i]));
        int lo = 0, hi = n_class;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (classes[mid] < v)
                lo = mid + 1;
            else
                hi = mid;
        }
        cls = static_cast<u64>(lo);
    }
    const u64 entry = (s & 0xFFFFFFFFULL) | ((i | (cls << idx_bits)) << 32);
    const u64 mask = (1ULL << bits) - 1ULL;
    u64 h = hash_slot(s, bits);
    for (u64 probe = 0; probe <= mask; ++probe) {
        if (atomicCAS(reinterpret_cast<unsigned long long*>(slots + h), ~0ULL, entry) == ~0ULL) return;
        h = (h + 1) & mask;
    }
}

__global__ void index_proj_kernel(DSector S, const u64* states, u64 n, long long* idx, double2* proj) {
    extern __shared__ __align__(16) unsigned char smem[];
    const Tables T = stage_tables(S, smem);
    __syncthreads();
    const u64 i = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double pr = 0.0, pi = 0.0;
    idx[i] = index_and_projection(S, T, states[i], pr, pi);
    proj[i] = make_double2(pr, pi);
}

int sm_count() {
    static int n = 0;
    static std::once_flag once;
    std::call_once(once, [] {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        if (n <= 0) n = 148;
    });
    return n;
}

// Arithmetic actions: chain rotations p[i] = i + t and reflections p[i] = t - i (mod N), or torus
// translations of rows of Lx sites, p[x + Lx y] = (x + a mod Lx) + Lx (y + b mod Ly). gkind 0 when some
// element is neither (the byte tables then act).
int classify_group(const int32_t* perms, int G, int N, int& Lx, std::vector<u64>& desc, std::vector<u64>& mask) {
    desc.assign(G, 0ULL);
    mask.assign(G, 0ULL);
    Lx = 0;
    bool chain = true;
    for (int g = 0; g < G && chain; ++g) {
        const int32_t* p = perms + g * N;
        const int t = p[0];
        bool rot = true, refl = true;
        for (int i = 0; i < N; ++i) {
            rot = rot && p[i] == (i + t) % N;
            refl = refl && p[i] == ((t - i) % N + N) % N;
        }
        if (rot)
            desc[g] = kElemRot | (static_cast<u64>(t) << 8);
        else if (refl)
            desc[g] = kElemRefl | (static_cast<u64>(((N - 1 - t) % N + N) % N) << 8);
        else
            chain = false;
    }
    if (chain) return 1;
    for (int lx = 2; lx < N; ++lx) {
        if (N % lx) continue;
        const int ly = N / lx;
        bool ok = true;
        for (int g = 0; g < G && ok; ++g) {
            const int32_t* p = perms + g * N;
            const int a = p[0] % lx, b = p[0] / lx;
            for (int y = 0; y < ly && ok; ++y)
                for (int x = 0; x < lx && ok; ++x) ok = p[x + lx * y] == (x + a) % lx + lx * ((y + b) % ly);
            if (!ok) break;
            u64 lo = 0;
            for (int y = 0; y < ly; ++y)
                for (int x = 0; x < lx - a; ++x) lo |= 1ULL << (x + lx * y);
            desc[g] = kElemTorus | (static_cast<u64>(lx * b) << 8) | (static_cast<u64>(a) << 16);
            mask[g] = lo;
        }
        if (ok) {
            Lx = lx;
            return 2;
        }
    }
    desc.assign(G, 0ULL);
    mask.assign(G, 0ULL);
    return 0;
}

void upload_group(qb_sector& s, const qb_sector_desc& d) {
    const int G = d.group_size, N = d.n_sites;
    s.lut.upload(build_lut(d.perms, G, N));
    std::vector<u64> fl(G, 0ULL);
    if (d.flips) std::copy(d.flips, d.flips + G, fl.begin());
    s.flips.upload(fl);
    std::vector<double2> ch(G);
    for (int g = 0; g < G; ++g) ch[g] = make_double2(d.chars[2 * g], d.chars[2 * g + 1]);
    s.chars.upload(ch);
    s.chars_host.assign(d.chars, d.chars + 2 * G);
    const SlcHost slc = build_slc(d.perms, reinterpret_cast<const u64*>(d.flips), G, N, d.sublattice_mode);
    s.slc_on = slc.on ? 1 : 0;
    if (slc.on) {
        s.slc_L = slc.L;
        s.slc_m = slc.m;
        s.slc_contig = slc.contig ? 1 : 0;
        for (int j = 0; j < slc.m; ++j) s.slc_bmask[j] = slc.bmask[j];
        s.to_key.upload(slc.to_key);
        std::vector<u64> pack(slc.lead.size());
        for (std::size_t i = 0; i < pack.size(); ++i) {
            const u64 cnt = slc.cand_off[i + 1] - slc.cand_off[i];
            if (cnt > 0xFFFF) throw Error(QB_EUNSUPPORTED, "sublattice code: more than 65535 candidates");
            const u64 pay = cnt == 1 ? slc.cand[slc.cand_off[i]] : slc.cand_off[i];
            pack[i] = static_cast<u64>(slc.lead[i]) | (cnt << 16) | (pay << 32);
        }
        s.lead_pack.upload(pack);
        s.cand.upload(slc.cand);
    }
    std::vector<u64> desc, mask;
    s.gkind = classify_group(d.perms, G, N, s.Lx, desc, mask);
    if (s.gkind) {
        s.edesc.upload(desc);
        s.emask.upload(mask);
    }
    s.rank_lut.upload(build_rank_lut(N));
}

void validate(const qb_sector_desc* d) {
    if (!d) throw Error(QB_EINVAL, "null sector description");
    if (d->n_sites < 1 || d->n_sites > 64) throw Error(QB_EINVAL, "n_sites must be in [1, 64]");
    if (d->n_up < 0 || d->n_up > d->n_sites) throw Error(QB_EINVAL, "n_up must be in [0, n_sites]");
    if (d->group_size < 1 || d->group_size > 65535) throw Error(QB_EINVAL, "group_size must be in [1, 65535]");
    if (!d->perms || !d->chars) throw Error(QB_EINVAL, "perms and chars are required");
    if (d->lookup < QB_LOOKUP_AUTO || d->lookup > QB_LOOKUP_HASH_WIDE) throw Error(QB_EINVAL, "unknown lookup kind");
    for (int g = 0; g < d->group_size; ++g) {
        std::vector<int> seen(d->n_sites, 0);
        for (int i = 0; i < d->n_sites; ++i) {
            const int p = d->perms[g * d->n_sites + i];
            if (p < 0 || p >= d->n_sites || seen[p]++) throw Error(QB_EINVAL, "element is not a permutation");
        }
        if (d->flips) {
            const u64 allm = d->n_sites == 64 ? ~0ULL : ((1ULL << d->n_sites) - 1ULL);
            const u64 f = d->flips[g];
            if (f & ~allm) throw Error(QB_EINVAL, "flip mask beyond n_sites");
            // an element must keep the popcount of every state of the sector
            if (f != 0 && !(f == allm && 2 * d->n_up == d->n_sites))
                throw Error(QB_EINVAL, "a flip element must be the global spin flip at half filling");
        }
    }
}

// The lookup structure: a rank table indexed by the combinadic rank, or state buckets over the
// ascending representatives (include/ed/basis/rep_sector.h:85-117, 275-307).
void build_lookup(qb_sector& s, int want) {
    if (s.dim == 0) {
        s.lookup = 0;
        return;
    }
    const auto C = pascal();
    const u64 ranks = C[s.N * 65 + s.n_up];
    const double table_bytes = 4.0 * static_cast<double>(ranks);
    // buckets: ~one per representative, at most 2^24
    std::vector<u64> ends(2);
    cuda_check(cudaMemcpy(&ends[0], s.reps.p, 8, cudaMemcpyDeviceToHost), "read reps");
    cuda_check(cudaMemcpy(&ends[1], s.reps.p + (s.dim - 1), 8, cudaMemcpyDeviceToHost), "read reps");
    int mode = want;
    const bool wide = mode == QB_LOOKUP_HASH_WIDE;
    if (mode == QB_LOOKUP_AUTO || mode == QB_LOOKUP_HASH_WIDE) mode = QB_LOOKUP_HASH;
    if (mode == QB_LOOKUP_HASH && (s.dim >= (1ULL << 32) || (s.N == 64 && s.n_up == 64))) mode = QB_LOOKUP_BUCKETS;
    (void)table_bytes;
    if (mode == QB_LOOKUP_HASH) {
        // the 1/norm classes
        DevBuf<u64> set(kClassSet);
        DevBuf<int> ovf(1);
        cuda_check(cudaMemset(set.p, 0xFF, kClassSet * 8), "class set clear");
        cuda_check(cudaMemset(ovf.p, 0, 4), "class set clear");
        const unsigned blocks = static_cast<unsigned>((s.dim + 255) / 256);
        class_set_kernel<<<blocks, 256>>>(s.inv_norms.p, s.dim, set.p, ovf.p);
        cuda_check(cudaGetLastError(), "class set");
        std::vector<u64> hs(kClassSet);
        int overflow = 0;
        cuda_check(cudaMemcpy(hs.data(), set.p, kClassSet * 8, cudaMemcpyDeviceToHost), "class set read");
        cuda_check(cudaMemcpy(&overflow, ovf.p, 4, cudaMemcpyDeviceToHost), "class set read");
        std::vector<u64> cls;
        for (u64 v : hs)
            if (v != ~0ULL) cls.push_back(v);
        std::sort(cls.begin(), cls.end());
        if (overflow || cls.size() > 2048) cls.clear();
        DevBuf<u64> dcls;
        dcls.upload(cls);
        if (!cls.empty()) {
            std::vector<double> vals(cls.size());
            std::memcpy(vals.data(), cls.data(), cls.size() * 8);
            s.inv_class.upload(vals);
        }
        s.n_class = static_cast<int>(cls.size());
        // compact 8-byte slots (load <= 2/3) when the state fits 32 bits and index + class fit 31 bits (so a full
        // slot is never all ones), else 16-byte slots (load <= 1/2)
        int idx_bits = 1, cls_bits = 0;
        while ((1ULL << idx_bits) < s.dim) ++idx_bits;
        while ((1 << cls_bits) < s.n_class) ++cls_bits;
        const bool compact = !wide && s.N <= 32 && !(s.N == 32 && s.n_up == 32) && idx_bits + cls_bits <= 31;
        int bits = 4;
        if (compact) {
            while ((1ULL << bits) < s.dim + s.dim / 2) ++bits;
            s.hash_bits = bits;
            s.idx_bits = idx_bits;
            s.slots8.alloc(1ULL << bits);
            cuda_check(cudaMemset(s.slots8.p, 0xFF, (1ULL << bits) * 8), "hash clear");
            hash_insert8_kernel<<<blocks, 256>>>(s.reps.p, s.inv_norms.p, s.dim, s.slots8.p, bits, idx_bits, dcls.p,
                                                 s.n_class);
            s.lookup = 4;
        } else {
            while ((1ULL << bits) < 2 * s.dim) ++bits;
            s.hash_bits = bits;
            s.slots.alloc(1ULL << bits);
            cuda_check(cudaMemset(s.slots.p, 0xFF, (1ULL << bits) * sizeof(ulonglong2)), "hash clear");
            hash_insert_kernel<<<blocks, 256>>>(s.reps.p, s.inv_norms.p, s.dim, s.slots.p, bits, dcls.p, s.n_class);
            s.lookup = 3;
        }
        cuda_check(cudaGetLastError(), "hash insert");
    } else if (mode == QB_LOOKUP_RANK) {
        if (s.dim >= (1ULL << 31)) throw Error(QB_EUNSUPPORTED, "rank table: more than 2^31 representatives");
        s.rank_table.alloc(static_cast<std::size_t>(ranks));
        cuda_check(cudaMemset(s.rank_table.p, 0xFF, ranks * 4), "rank table clear");
        s.lookup = 1;
        const DSector v = s.view();
        rank_table_kernel<<<static_cast<unsigned>((s.dim + 255) / 256), 256>>>(v, s.rank_table.p);
        cuda_check(cudaGetLastError(), "rank table");
    } else {
        const u64 base = ends[0], span = ends[1] - ends[0] + 1;
        int bits = 0;
        while ((1ULL << bits) < s.dim && bits < 24) ++bits;
        int key_bits = 0;
        while (key_bits < 63 && (1ULL << key_bits) < span) ++key_bits;
        const int shift = std::max(0, key_bits - bits);
        const u64 nb = ((span - 1) >> shift) + 1;
        s.bucket_off.alloc(static_cast<std::size_t>(nb + 1));
        s.bucket_base = base;
        s.bucket_shift = shift;
        s.bucket_count = nb;
        s.lookup = 2;
        bucket_kernel<<<static_cast<unsigned>((s.dim + 255) / 256), 256>>>(s.reps.p, s.dim, base, shift, nb,
                                                                              s.bucket_off.p);
        cuda_check(cudaGetLastError(), "buckets");
    }
    cuda_check(cudaStreamSynchronize(nullptr), "lookup build");
}

}  // namespace
}  // namespace qb

qb::DSector qb_sector::view() const {
    qb::DSector v;
    v.N = N;
    v.n_up = n_up;
    v.G = G;
    v.bpw = bpw;
    v.dim = dim;
    v.reps = reps.p;
    v.inv_norms = inv_norms.p;
    v.lut = lut.p;
    v.flips = flips.p;
    v.chars = chars.p;
    v.unit_chars = 1;
    for (std::size_t i = 0; i + 1 < chars_host.size(); i += 2)
        if (chars_host[i + 1] != 0.0 || (chars_host[i] != 1.0 && chars_host[i] != -1.0)) v.unit_chars = 0;
    v.slc.on = slc_on;
    v.slc.L = slc_L;
    v.slc.m = slc_m;
    v.slc.contig = slc_contig;
    for (int j = 0; j < 8; ++j) v.slc.bmask[j] = slc_bmask[j];
    v.slc.to_key = to_key.p;
    v.slc.pack = lead_pack.p;
    v.slc.cand = cand.p;
    v.gkind = gkind;
    v.Lx = Lx;
    v.edesc = edesc.p;
    v.emask = emask.p;
    v.lookup = lookup;
    v.rank_table = rank_table.p;
    v.rank_lut = rank_lut.p;
    v.bucket_off = bucket_off.p;
    v.bucket_base = bucket_base;
    v.bucket_count = bucket_count;
    v.bucket_shift = bucket_shift;
    v.slots = slots.p;
    v.slots8 = slots8.p;
    v.idx_bits = idx_bits;
    v.hash_bits = hash_bits;
    v.inv_class = inv_class.p;
    v.n_class = n_class;
    return v;
}

std::uint64_t qb_sector::device_bytes() const {
    return reps.bytes() + inv_norms.bytes() + lut.bytes() + flips.bytes() + chars.bytes() + to_key.bytes() +
           lead_pack.bytes() + cand.bytes() + edesc.bytes() + emask.bytes() + rank_table.bytes() + rank_lut.bytes() +
           bucket_off.bytes() + slots.bytes() + slots8.bytes() + inv_class.bytes();
}

extern "C" {

const char* qb_last_error(void) { return qb::g_last_error.c_str(); }

int qb_device_count(int* count) {
    return qb::guarded([&] {
        int n = 0;
        const cudaError_t e = cudaGetDeviceCount(&n);
        *count = e == cudaSuccess ? n : 0;
        if (e != cudaSuccess) (void)cudaGetLastError();
    });
}

int qb_key_order(const qb_sector_desc* d, int* L, int* m, uint64_t* n_cand, int32_t* key_bit, uint16_t* lead,
                 uint32_t* cand_off, uint16_t* cand) {
    return qb::guarded([&] {
        using namespace qb;
        if (!d || !L || !m || !n_cand || !d->perms || d->n_sites < 1 || d->n_sites > 64 || d->group_size < 1)
            throw Error(QB_EINVAL, "key order: bad descriptor");
        const SlcHost c = build_slc(d->perms, reinterpret_cast<const u64*>(d->flips), d->group_size, d->n_sites,
                                    d->sublattice_mode);
        *L = c.on ? c.L : 0;
        *m = c.on ? c.m : 0;
        *n_cand = c.on ? c.cand.size() : 0;
        if (!c.on) return;
        if (key_bit)
            for (int s = 0; s < d->n_sites; ++s) {   // the key bit of site s: the one bit of its byte table entry
                const u64 e = c.to_key[static_cast<std::size_t>(s >> 3) * 256 + (1u << (s & 7))];
                key_bit[s] = __builtin_ctzll(e);
            }
        if (lead) std::copy(c.lead.begin(), c.lead.end(), lead);
        if (cand_off) std::copy(c.cand_off.begin(), c.cand_off.end(), cand_off);
        if (cand) std::copy(c.cand.begin(), c.cand.end(), cand);
    });
}

}  // extern "C"

namespace qb {
void keep_desc(qb_sector& s, const qb_sector_desc& d) {
    s.desc_perms.assign(d.perms, d.perms + static_cast<std::size_t>(d.group_size) * d.n_sites);
    if (d.flips) s.desc_flips.assign(d.flips, d.flips + d.group_size);
    s.chars_host.assign(d.chars, d.chars + 2 * static_cast<std::size_t>(d.group_size));
    s.desc_slc_mode = d.sublattice_mode;
    s.desc_lookup = d.lookup;
}
}  // namespace qb

extern "C" {

int qb_sector_create(const qb_sector_desc* d, qb_sector** out) {
    return qb::guarded([&] {
        using namespace qb;
        validate(d);
        auto s = std::make_unique<qb_sector>();
        s->N = d->n_sites;
        s->n_up = d->n_up;
        s->G = d->group_size;
        s->bpw = (d->n_sites + 7) / 8;
        keep_desc(*s, *d);
        upload_group(*s, *d);
        const auto Ch = pascal();
        const u64 total = Ch[s->N * 65 + s->n_up];
        DevBuf<u64> C;
        C.upload(Ch);
        // chunks of consecutive ranks: enough for every SM to stay busy, at least 64 states each
        const u64 want_chunks = static_cast<u64>(sm_count()) * 2048 * 8;
        u64 chunk = std::max<u64>(64, (total + want_chunks - 1) / want_chunks);
        const u64 n_chunks = (total + chunk - 1) / chunk;
        DevBuf<u64> counts(n_chunks), offsets(n_chunks + 1);
        DSector v = s->view();
        const std::size_t smem = tables_smem_bytes(v);
        if (smem > 48 * 1024)
            cuda_check(cudaFuncSetAttribute(enum_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)),
                       "smem attribute");
        const unsigned threads = 256;
        const unsigned blocks =
            static_cast<unsigned>(std::min<u64>((n_chunks + threads - 1) / threads, static_cast<u64>(sm_count()) * 16));
        enum_kernel<<<blocks, threads, smem>>>(v, total, chunk, n_chunks, C.p, counts.p, nullptr, nullptr, nullptr);
        cuda_check(cudaGetLastError(), "enumeration (count)");
        std::size_t tmp_bytes = 0;
        cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, counts.p, offsets.p, static_cast<int>(n_chunks) + 0);
        DevBuf<unsigned char> tmp(std::max<std::size_t>(tmp_bytes, 1));
        cub::DeviceScan::ExclusiveSum(tmp.p, tmp_bytes, counts.p, offsets.p, static_cast<int>(n_chunks));
        cuda_check(cudaGetLastError(), "enumeration (scan)");
        u64 last_off = 0, last_cnt = 0;
        cuda_check(cudaMemcpy(&last_off, offsets.p + (n_chunks - 1), 8, cudaMemcpyDeviceToHost), "scan read");
        cuda_check(cudaMemcpy(&last_cnt, counts.p + (n_chunks - 1), 8, cudaMemcpyDeviceToHost), "scan read");
        s->dim = last_off + last_cnt;
        s->reps.alloc(s->dim);
        s->inv_norms.alloc(s->dim);
        if (s->dim > 0) {
            enum_kernel<<<blocks, threads, smem>>>(v, total, chunk, n_chunks, C.p, counts.p, offsets.p, s->reps.p,
                                                   s->inv_norms.p);
            cuda_check(cudaGetLastError(), "enumeration (write)");
        }
        cuda_check(cudaStreamSynchronize(nullptr), "enumeration");
        build_lookup(*s, d->lookup);
        *out = s.release();
    });
}

int qb_sector_create_from_reps(const qb_sector_desc* d, const uint64_t* reps, const double* inv_norms, uint64_t dim,
                               qb_sector** out) {
    return qb::guarded([&] {
        using namespace qb;
        validate(d);
        for (uint64_t i = 1; i < dim; ++i)
            if (reps[i] <= reps[i - 1]) throw Error(QB_EINVAL, "representatives must ascend");
        auto s = std::make_unique<qb_sector>();
        s->N = d->n_sites;
        s->n_up = d->n_up;
        s->G = d->group_size;
        s->bpw = (d->n_sites + 7) / 8;
        keep_desc(*s, *d);
        upload_group(*s, *d);
        s->dim = dim;
        s->reps.upload(reinterpret_cast<const u64*>(reps), dim);
        s->inv_norms.upload(inv_norms, dim);
        build_lookup(*s, d->lookup);
        *out = s.release();
    });
}

int qb_sector_destroy(qb_sector* s) {
    return qb::guarded([&] {
        if (s && s->registered) throw qb::Error(QB_EINVAL, "a sector from qb_sector_acquire is released, not destroyed");
        delete s;
    });
}

uint64_t qb_sector_dim(const qb_sector* s) { return s ? s->dim : 0; }

int qb_sector_download(const qb_sector* s, uint64_t* reps, double* inv_norms) {
    return qb::guarded([&] {
        if (!s) throw qb::Error(QB_EINVAL, "null sector");
        if (reps && s->dim)
            qb::cuda_check(cudaMemcpy(reps, s->reps.p, s->dim * 8, cudaMemcpyDeviceToHost), "download reps");
        if (inv_norms && s->dim)
            qb::cuda_check(cudaMemcpy(inv_norms, s->inv_norms.p, s->dim * 8, cudaMemcpyDeviceToHost), "download");
    });
}

int qb_sector_info(const qb_sector* s, uint64_t* device_bytes, int* slc_L, int* slc_m, int* lookup_kind) {
    return qb::guarded([&] {
        if (!s) throw qb::Error(QB_EINVAL, "null sector");
        if (device_bytes) *device_bytes = s->device_bytes();
        if (slc_L) *slc_L = s->slc_on ? s->slc_L : 0;
        if (slc_m) *slc_m = s->slc_on ? s->slc_m : 0;
        if (lookup_kind) *lookup_kind = s->lookup;
    });
}

int qb_index_and_projection(const qb_sector* s, const uint64_t* states, uint64_t n, int64_t* index, double* proj) {
    return qb::guarded([&] {
        using namespace qb;
        if (!s) throw Error(QB_EINVAL, "null sector");
        if (n == 0) return;
        DevBuf<u64> d_states;
        d_states.upload(reinterpret_cast<const u64*>(states), n);
        DevBuf<long long> d_idx(n);
        DevBuf<double2> d_proj(n);
        const std::size_t smem = tables_smem_bytes(s->view());
        if (smem > 48 * 1024)
            cuda_check(cudaFuncSetAttribute(index_proj_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)),
                       "smem attribute");
        index_proj_kernel<<<static_cast<unsigned>((n + 127) / 128), 128, smem>>>(s->view(), d_states.p, n, d_idx.p,
                                                                                    d_proj.p);
        cuda_check(cudaGetLastError(), "index_and_projection");
        cuda_check(cudaMemcpy(index, d_idx.p, n * 8, cudaMemcpyDeviceToHost), "download");
        cuda_check(cudaMemcpy(proj, d_proj.p, n * 16, cudaMemcpyDeviceToHost), "download");
    });
}

}  // extern "C"
