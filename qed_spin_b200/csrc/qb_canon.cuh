// =============================================================================
// qb_canon.cuh -- canonicalisation of a state on the device: its representative, the character sum
// over the elements that reach it, and its index in the sector.
//
// Follows the reference's index_and_projection (include/ed/matvec/rep_symmetry_basis_policy.h:142-241)
// and the sublattice candidates (include/ed/basis/sublattice_code.h:74-131): one pass over the elements
// that can reach the representative (every element, or the few candidates the key order leaves) with a
// running minimum; the character sum restarts at a new minimum and grows on ties, in ascending element
// order, so the sum equals the reference's bit for bit.
// =============================================================================
#pragma once

#include "qb_internal.cuh"

namespace qb {

// The small per-sector tables a kernel stages in shared memory (pointers into smem, or into global
// memory when a table is too large to stage).
struct Tables {
    const u64* to_key;      // bpw x 256
    const u64* flips;       // G
    const double2* chars;   // G
    const u64* edesc;       // G (arithmetic action)
    const u64* emask;       // G (torus rows)
    const double* inv_class;  // the distinct 1/norm values (hash lookup)
    const u64* pack;          // the sublattice leading-block table when small enough to stage
};

// States travel as ST: 32-bit for N <= 32 (half the integer instructions of 64-bit shifts, masks and
// compares), 64-bit otherwise.
template <class ST> struct StateOps;
template <> struct StateOps<u64> {
    __device__ static u64 brev(u64 s) { return __brevll(s); }
    static constexpr int kBits = 64;
};
template <> struct StateOps<u32> {
    __device__ static u32 brev(u32 s) { return __brev(s); }
    static constexpr int kBits = 32;
};

template <class ST> __device__ __forceinline__ ST full_mask(int N) {
    return N == StateOps<ST>::kBits ? static_cast<ST>(~static_cast<ST>(0)) : static_cast<ST>((static_cast<ST>(1) << N) - 1);
}

// Image of s under element g (include/ed/basis/compiled_group.h:73-78): new bit i = old bit perm[i], then
// XOR the flip mask. Chains and tori act by rotations, a reversal, and row rotations; any other group
// through its byte tables.
template <class ST>
__device__ __forceinline__ ST apply_elem(const DSector& S, const Tables& T, ST s, int g) {
    if (S.gkind != 0) {
        const u64 d = T.edesc[g];
        const int kind = static_cast<int>(d & 0xFF);
        const int c = static_cast<int>((d >> 8) & 0xFF);
        const int N = S.N;
        const ST full = full_mask<ST>(N);
        if (kind == kElemRefl) s = StateOps<ST>::brev(s) >> (StateOps<ST>::kBits - N);
        if (c) s = ((s >> c) | (s << (N - c))) & full;
        if (kind == kElemTorus) {
            const int a = static_cast<int>((d >> 16) & 0xFF);
            if (a) {
                const ST lo = static_cast<ST>(T.emask[g]);
                s = ((s >> a) & lo) | ((s << (S.Lx - a)) & static_cast<ST>(~lo) & full);
            }
        }
        return s ^ static_cast<ST>(T.flips[g]);
    }
    const u64* l = S.lut + static_cast<std::size_t>(g) * S.bpw * 256;
    ST r = 0;
#pragma unroll 8
    for (int b = 0; b < S.bpw; ++b) r |= static_cast<ST>(__ldg(l + b * 256 + static_cast<int>((s >> (8 * b)) & 0xFFu)));
    return r ^ static_cast<ST>(T.flips[g]);
}

// A state's bits moved to their key positions.
template <class ST> __device__ __forceinline__ ST key_of(const u64* to_key, int bpw, ST s) {
    ST k = 0;
#pragma unroll 8
    for (int b = 0; b < bpw; ++b) k |= static_cast<ST>(to_key[(b << 8) + static_cast<int>((s >> (8 * b)) & 0xFFu)]);
    return k;
}

template <class ST> __device__ __forceinline__ u32 pattern_of(ST k, int j, int N, int L) {
    return static_cast<u32>(k >> (N - (j + 1) * L)) & ((1u << L) - 1u);
}

// The several-blocks case of for_each_candidate: merge the ascending candidate lists of every block that
// reaches the least leading block (each element maps exactly one block to the lead).
template <class Pat, class Fn>
__device__ __forceinline__ void merge_candidates(const DSector& S, const u64* pack, const Pat& pat, u32 best, Fn& fn) {
    const int L = S.slc.L, m = S.slc.m;
    u64 sel[8];
    u32 pos[8];
    int n = 0;
    for (int j = 0; j < m; ++j) {
        const u64 e = pack[(static_cast<u32>(j) << L) + pat(j)];
        if (static_cast<u32>(e & 0xFFFFu) == best) {
            sel[n] = e;
            pos[n] = 0;
            ++n;
        }
    }
    for (;;) {
        int pick = -1;
        u32 g = 0xFFFFFFFFu;
        for (int i = 0; i < n; ++i) {
            const u32 cnt = static_cast<u32>((sel[i] >> 16) & 0xFFFFu);
            if (pos[i] >= cnt) continue;
            const u32 pay = static_cast<u32>(sel[i] >> 32);
            const u32 c = cnt == 1 ? pay : static_cast<u32>(__ldg(S.slc.cand + pay + pos[i]));
            if (c < g) {
                g = c;
                pick = i;
            }
        }
        if (pick < 0) return;
        ++pos[pick];
        fn(static_cast<int>(g));
    }
}

// fn(g) in ascending order for the elements whose image has the least leading block
// (sublattice_code.h:102-131); returns that least leading block. One packed load per block; pat(j) is block j's
// pattern.
template <class Pat, class Fn>
__device__ __forceinline__ u32 for_each_candidate(const DSector& S, const u64* pack, const Pat& pat, Fn&& fn) {
    const int L = S.slc.L, m = S.slc.m;
    u32 best = 0xFFFFFFFFu;
    u64 first = 0;
    int n = 0;
    for (int j = 0; j < m; ++j) {
        const u64 e = pack[(static_cast<u32>(j) << L) + pat(j)];
        const u32 v = static_cast<u32>(e & 0xFFFFu);
        if (v < best) {
            best = v;
            first = e;
            n = 1;
        } else if (v == best) {
            ++n;
        }
    }
    if (n == 1) {
        const u32 cnt = static_cast<u32>((first >> 16) & 0xFFFFu);
        const u32 pay = static_cast<u32>(first >> 32);
        if (cnt == 1) {
            fn(static_cast<int>(pay));
        } else {
            for (u32 p = 0; p < cnt; ++p) fn(static_cast<int>(__ldg(S.slc.cand + pay + p)));
        }
        return best;
    }
    if (S.unit_chars) {
        // +1/-1 characters: the sum over the ties is exact in any order, so each tied block's list is walked in
        // turn (the representative is the least key whichever order finds it)
        for (int j = 0; j < m; ++j) {
            const u64 e = pack[(static_cast<u32>(j) << L) + pat(j)];
            if (static_cast<u32>(e & 0xFFFFu) != best) continue;
            const u32 cnt = static_cast<u32>((e >> 16) & 0xFFFFu);
            const u32 pay = static_cast<u32>(e >> 32);
            if (cnt == 1) {
                fn(static_cast<int>(pay));
            } else {
                for (u32 p = 0; p < cnt; ++p) fn(static_cast<int>(__ldg(S.slc.cand + pay + p)));
            }
        }
        return best;
    }
    merge_candidates(S, pack, pat, best, fn);
    return best;
}

template <class ST> __device__ __forceinline__ int top_bit(ST x);
template <> __device__ __forceinline__ int top_bit<u64>(u64 x) { return 63 - __clzll(static_cast<long long>(x)); }
template <> __device__ __forceinline__ int top_bit<u32>(u32 x) { return 31 - __clz(static_cast<int>(x)); }

// key(a) < key(b) for a != b, read from the states themselves: the first block in which they differ decides, and
// within it the highest differing site (sublattice_code.h:23-34: block 0 leads the key, a block's sites in
// ascending order take ascending key bits).
template <class ST> __device__ __forceinline__ bool key_below(const DSlc& c, ST a, ST b) {
    const ST d = a ^ b;
    for (int j = 0; j < c.m; ++j) {
        const ST dj = d & static_cast<ST>(c.bmask[j]);
        if (dj) return ((a >> top_bit<ST>(dj)) & static_cast<ST>(1)) == 0;
    }
    return false;
}

// Block j's pattern of a state: its sites' bits in ascending site order (the key's block-j field).
template <class ST> struct BlockPattern {
    ST t;
    int N, L, contig;
    __device__ BlockPattern(const DSector& S, const u64* to_key, ST x)
        : t(S.slc.contig ? x : key_of<ST>(to_key, S.bpw, x)), N(S.N), L(S.slc.L), contig(S.slc.contig) {}
    __device__ u32 operator()(int j) const {
        return contig ? static_cast<u32>(t >> (j * L)) & ((1u << L) - 1u) : pattern_of<ST>(t, j, N, L);
    }
};

// Representative of t and the conjugated character sum over the elements that reach it.
// With a key order the images are compared in place (key_below), so no image is mapped to its key.
template <class ST>
__device__ __forceinline__ ST canonicalize(const DSector& S, const Tables& T, ST t, double& acc_re, double& acc_im) {
    ST rb = static_cast<ST>(~static_cast<ST>(0));
    acc_re = 0.0;
    acc_im = 0.0;
    if (S.slc.on) {
        bool have = false;
        auto visit = [&](int g) {
            const ST img = apply_elem<ST>(S, T, t, g);
            if (!have || (img != rb && key_below<ST>(S.slc, img, rb))) {
                have = true;
                rb = img;
                const double2 c = T.chars[g];
                acc_re = __dadd_rn(0.0, c.x);
                acc_im = __dsub_rn(0.0, c.y);
            } else if (img == rb) {
                const double2 c = T.chars[g];
                acc_re = __dadd_rn(acc_re, c.x);
                acc_im = __dsub_rn(acc_im, c.y);
            }
        };
        for_each_candidate(S, T.pack, BlockPattern<ST>(S, T.to_key, t), visit);
    } else {
        auto visit = [&](int g) {
            const ST img = apply_elem<ST>(S, T, t, g);
            if (img < rb) {
                rb = img;
                const double2 c = T.chars[g];
                acc_re = __dadd_rn(0.0, c.x);
                acc_im = __dsub_rn(0.0, c.y);
            } else if (img == rb) {
                const double2 c = T.chars[g];
                acc_re = __dadd_rn(acc_re, c.x);
                acc_im = __dsub_rn(acc_im, c.y);
            }
        };
        for (int g = 0; g < S.G; ++g) visit(g);
    }
    return rb;
}

// The combinadic (colex) rank of a state with n_up set bits (include/ed/basis/combinadic.h:63-80),
// from byte tables: byte b with k set bits below it contributes rank_lut[b][k][byte].
__device__ __forceinline__ u64 rank_of(const DSector& S, u64 s) {
    u64 r = 0;
    int below = 0;
#pragma unroll 8
    for (int b = 0; b < S.bpw; ++b) {
        const int v = static_cast<int>((s >> (8 * b)) & 0xFFu);
        r += __ldg(S.rank_lut + (static_cast<std::size_t>(b) * (S.N + 1) + below) * 256 + v);
        below += __popc(v);
    }
    return r;
}

// The slot a state hashes to (a 64-bit finaliser, then the top hash_bits bits).
__device__ __forceinline__ u64 hash_slot(u64 s, int bits) {
    s ^= s >> 31;
    s *= 0x7fb5d329728ea185ULL;
    s ^= s >> 27;
    s *= 0x81dadef4bc2dd44dULL;
    s ^= s >> 33;
    return s >> (64 - bits);
}

// Hash lookup: index of rb (or -1) and its 1/norm class, by linear probing.
__device__ __forceinline__ long long hash_find(const DSector& S, u64 rb, int& cls) {
    const u64 mask = (1ULL << S.hash_bits) - 1ULL;
    u64 h = hash_slot(rb, S.hash_bits);
    for (;;) {
        const ulonglong2 e = __ldg(S.slots + h);
        if (e.x == rb) {
            cls = static_cast<int>(e.y >> 32);
            return static_cast<long long>(e.y & 0xFFFFFFFFULL);
        }
        if (e.x == ~0ULL) return -1;
        h = (h + 1) & mask;
    }
}

// The compact table (N <= 32): an 8-byte slot holds the 32-bit state and index | class << idx_bits.
__device__ __forceinline__ long long hash_find8(const DSector& S, u64 rb, int& cls) {
    const u64 mask = (1ULL << S.hash_bits) - 1ULL;
    u64 h = hash_slot(rb, S.hash_bits);
    const u32 key = static_cast<u32>(rb);
    for (;;) {
        const u64 e = __ldg(S.slots8 + h);
        if (e == ~0ULL) return -1;
        if (static_cast<u32>(e) == key) {
            const u32 pay = static_cast<u32>(e >> 32);
            cls = static_cast<int>(pay >> S.idx_bits);
            return static_cast<long long>(pay & ((1u << S.idx_bits) - 1u));
        }
        h = (h + 1) & mask;
    }
}

// Index of representative rb in the sector, or -1 (index_of_rep, rep_symmetry_basis_policy.h:169-202).
__device__ __forceinline__ long long index_of_rep(const DSector& S, u64 rb) {
    if (S.lookup == 4) {
        int cls;
        return hash_find8(S, rb, cls);
    }
    if (S.lookup == 3) {
        int cls;
        return hash_find(S, rb, cls);
    }
    if (S.lookup == 1) return static_cast<long long>(__ldg(S.rank_table + rank_of(S, rb)));
    std::uint64_t lo = 0, hi = S.dim;
    if (S.lookup == 2) {
        if (rb < S.bucket_base) return -1;
        const u64 b = (rb - S.bucket_base) >> S.bucket_shift;
        if (b >= S.bucket_count) return -1;
        lo = __ldg(S.bucket_off + b);
        hi = __ldg(S.bucket_off + b + 1);
    }
    while (lo < hi) {
        const std::uint64_t mid = lo + ((hi - lo) >> 1);
        if (__ldg(S.reps + mid) < rb)
            lo = mid + 1;
        else
            hi = mid;
    }
    return (lo < S.dim && __ldg(S.reps + lo) == rb) ? static_cast<long long>(lo) : -1LL;
}

// index_and_projection: index of t's orbit in S (or -1) and conj(beta_t) * inv_norm[index].
template <class ST = u64>
__device__ __forceinline__ long long index_and_projection(const DSector& S, const Tables& T, ST t, double& pre,
                                                          double& pim) {
    if (__popcll(static_cast<u64>(t)) != S.n_up) return -1;
    double are, aim;
    const u64 rb = static_cast<u64>(canonicalize<ST>(S, T, t, are, aim));
    long long j;
    double s;
    if (S.lookup >= 3) {
        int cls = 0;
        j = S.lookup == 4 ? hash_find8(S, rb, cls) : hash_find(S, rb, cls);
        if (j < 0) return -1;
        s = S.n_class ? T.inv_class[cls] : __ldg(S.inv_norms + j);
    } else {
        j = index_of_rep(S, rb);
        if (j < 0) return -1;
        s = __ldg(S.inv_norms + j);
    }
    pre = __dmul_rn(are, s);
    pim = __dmul_rn(aim, s);
    return j;
}

// Bytes of shared memory stage_tables takes for a sector (0 for the parts left in global memory).
constexpr std::size_t kPackSmemMax = 16 * 1024;

// Byte offsets of the staged tables; every array starts on a 16-byte boundary. Host sizing and device
// staging both read this one layout.
struct TablesLayout {
    std::size_t key = 0, pack = 0, chars = 0, flips = 0, desc = 0, mask = 0, cls = 0, total = 0;
    bool stage_key = false, stage_pack = false, stage_elems = false, stage_cls = false;
};

__host__ __device__ inline std::size_t align16(std::size_t x) { return (x + 15) & ~std::size_t(15); }

__host__ __device__ inline TablesLayout tables_layout(const DSector& S) {
    TablesLayout l;
    std::size_t p = 0;
    if (S.slc.on) {
        l.stage_key = true;
        l.key = p;
        p = align16(p + static_cast<std::size_t>(S.bpw) * 256 * 8);
        const std::size_t np = (static_cast<std::size_t>(S.slc.m) << S.slc.L) * 8;
        if (np <= kPackSmemMax) {
            l.stage_pack = true;
            l.pack = p;
            p = align16(p + np);
        }
    }
    if (S.G <= 1024) {
        l.stage_elems = true;
        l.chars = p;
        p = align16(p + static_cast<std::size_t>(S.G) * 16);
        l.flips = p;
        p = align16(p + static_cast<std::size_t>(S.G) * 8);
        l.desc = p;
        p = align16(p + static_cast<std::size_t>(S.G) * 8);
        l.mask = p;
        p = align16(p + static_cast<std::size_t>(S.G) * 8);
    }
    if (S.n_class > 0) {
        l.stage_cls = true;
        l.cls = p;
        p = align16(p + static_cast<std::size_t>(S.n_class) * 8);
    }
    l.total = p;
    return l;
}

__host__ __device__ inline std::size_t tables_smem_bytes(const DSector& S) { return tables_layout(S).total; }

// Stage a sector's small tables into shared memory at `smem` (16-byte aligned, tables_smem_bytes long).
// Every thread of the block takes part; the caller synchronises afterwards.
__device__ __forceinline__ Tables stage_tables(const DSector& S, unsigned char* smem) {
    Tables T{S.slc.to_key, S.flips, S.chars, S.edesc, S.emask, S.inv_class, S.slc.pack};
    const TablesLayout l = tables_layout(S);
    if (l.stage_key) {
        u64* key = reinterpret_cast<u64*>(smem + l.key);
        for (int i = threadIdx.x; i < S.bpw * 256; i += blockDim.x) key[i] = S.slc.to_key[i];
        T.to_key = key;
    }
    if (l.stage_pack) {
        u64* pk = reinterpret_cast<u64*>(smem + l.pack);
        const std::size_t np = static_cast<std::size_t>(S.slc.m) << S.slc.L;
        for (std::size_t i = threadIdx.x; i < np; i += blockDim.x) pk[i] = S.slc.pack[i];
        T.pack = pk;
    }
    if (l.stage_elems) {
        double2* ch = reinterpret_cast<double2*>(smem + l.chars);
        u64* fl = reinterpret_cast<u64*>(smem + l.flips);
        u64* de = reinterpret_cast<u64*>(smem + l.desc);
        u64* em = reinterpret_cast<u64*>(smem + l.mask);
        for (int i = threadIdx.x; i < S.G; i += blockDim.x) {
            ch[i] = S.chars[i];
            fl[i] = S.flips[i];
            de[i] = S.edesc ? S.edesc[i] : 0ULL;
            em[i] = S.emask ? S.emask[i] : 0ULL;
        }
        T.chars = ch;
        T.flips = fl;
        T.edesc = de;
        T.emask = em;
    }
    if (l.stage_cls) {
        double* ic = reinterpret_cast<double*>(smem + l.cls);
        for (int i = threadIdx.x; i < S.n_class; i += blockDim.x) ic[i] = S.inv_class[i];
        T.inv_class = ic;
    }
    return T;
}

}  // namespace qb
