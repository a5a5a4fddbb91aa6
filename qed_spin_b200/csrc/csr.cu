// =============================================================================
// csr.cu -- the device reduced-CSR lane: an operator's merged rows built once from the row walk, then
// streamed by a sparse matvec.
//
// The rows are the reference's merged CSR (build_cross_csr / merge_row, include/ed/matvec/sector_rows.h:
// 147-404; its device twin build_sector_csr_gpu, src/gpu/rep_matvec.cu:1101-1253): each row's entries
// from the walk in group order, stably sorted by column, equal columns summed in emission order, exact
// zeros dropped. The values go into a dictionary when there are at most 65536 distinct ones (u8 ids for
// at most 256), else they are stored whole.
//
// Build: a count pass (merged row lengths; every merged value into a device hash set keyed by its bits) -> CUB
// scan -> a fill pass (columns and ids; each id's value is checked bit for bit). Each pass recomputes the rows
// from the walk.
//
// The matvec sums each row sequentially in CSR order, one thread per row; with k vectors interleaved by
// row each lane owns a slice of the columns and sums them in the same order, so every vector of a block
// apply equals its single apply bit for bit.
// =============================================================================
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <unordered_map>
#include <utility>
#include <vector>

#include "qb_walk.cuh"

namespace qb {

namespace {

constexpr int kMaxRowEntries = 256;   // a row's connections held at once (the reference's warp limit)
constexpr int kDictBits = 17;         // dictionary hash set: 2^17 slots
constexpr u64 kEmpty = ~0ULL;

__device__ __forceinline__ u64 value_key(cplx v) {
    u64 a = static_cast<u64>(__double_as_longlong(v.re));
    u64 b = static_cast<u64>(__double_as_longlong(v.im));
    a ^= (b << 29) | (b >> 35);
    a ^= a >> 33;
    a *= 0xff51afd7ed558ccdULL;
    a ^= a >> 33;
    a *= 0xc4ceb9fe1a85ec53ULL;
    a ^= a >> 33;
    return a == kEmpty ? 0x5555555555555555ULL : a;
}

struct Dict {
    u64* keys;        // mask + 1 slots (a power of two, at most 2^kDictBits)
    u64 mask;
    double2* vals;
    u32* ids;         // slot -> dictionary id (fill pass)
    int* overflow;    // set past 65536 values, or when two values share a key
    u32* count;       // values inserted
};

// One merged value into the dictionary set (the values pass).
__device__ __forceinline__ void dict_insert(const Dict& D, cplx v) {
    if (*static_cast<volatile int*>(D.overflow)) return;   // whole values: the set is no longer needed
    const u64 mask = D.mask;
    const u64 key = value_key(v);
    u64 h = key & mask;
    for (u64 probe = 0; probe <= mask; ++probe) {
        // a plain read first: most values are already in the set, and a key once written never changes
        const u64 seen = __ldcg(reinterpret_cast<const unsigned long long*>(D.keys + h));
        if (seen == key) return;
        if (seen != kEmpty) {
            h = (h + 1) & mask;
            continue;
        }
        const u64 old = atomicCAS(reinterpret_cast<unsigned long long*>(D.keys + h), kEmpty, key);
        if (old == kEmpty) {
            D.vals[h] = make_double2(v.re, v.im);
            if (atomicAdd(D.count, 1u) >= 65536u) *D.overflow = 1;
            return;
        }
        if (old == key) return;
        h = (h + 1) & mask;
    }
    *D.overflow = 1;
}

// The dictionary id of a merged value (the fill pass; the set is at most half full when ids are used, so the
// probe ends at the key or an empty slot). A different value under the same key raises the overflow flag:
// the caller then stores every value whole.
__device__ __forceinline__ u32 dict_id(const Dict& D, cplx v) {
    const u64 mask = D.mask;
    const u64 key = value_key(v);
    u64 h = key & mask;
    while (D.keys[h] != key && D.keys[h] != kEmpty) h = (h + 1) & mask;
    const double2 dv = D.vals[h];
    if (D.keys[h] != key || __double_as_longlong(dv.x) != __double_as_longlong(v.re) ||
        __double_as_longlong(dv.y) != __double_as_longlong(v.im)) {
        *D.overflow = 1;
        return 0;
    }
    return D.ids[h];
}

// The occupied slots of the value set numbered in slot order: ids[slot], the values compacted into dict (at
// most kMaxDict), and the count. One CTA of 1024 threads walks the slots 1024 at a time.
constexpr int kMaxDict = 65536;
__global__ void __launch_bounds__(1024) dict_compact(const u64* keys, const double2* vals, u64 nslots, u32* ids,
                                                     double2* dict, int* count) {
    __shared__ u32 warp_n[32], warp_off[32];
    __shared__ u32 base, round_n;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (threadIdx.x == 0) base = 0;
    __syncthreads();
    for (u64 s0 = 0; s0 < nslots; s0 += 1024) {
        const u64 slot = s0 + threadIdx.x;
        const bool occ = slot < nslots && keys[slot] != kEmpty;
        const unsigned bal = __ballot_sync(0xffffffffu, occ);
        if (lane == 0) warp_n[w] = __popc(bal);
        __syncthreads();
        if (threadIdx.x == 0) {
            u32 acc = 0;
            for (int i = 0; i < 32; ++i) {
                warp_off[i] = acc;
                acc += warp_n[i];
            }
            round_n = acc;
        }
        __syncthreads();
        if (occ) {
            const u32 id = base + warp_off[w] + __popc(bal & ((1u << lane) - 1u));
            ids[slot] = id;
            if (id < static_cast<u32>(kMaxDict)) dict[id] = vals[slot];
        }
        __syncthreads();
        if (threadIdx.x == 0) base += round_n;
        __syncthreads();
    }
    if (threadIdx.x == 0) *count = static_cast<int>(base);
}

// The device's default memory pool keeps up to 256 MB of freed scratch between builds (the default releases
// everything at each synchronisation, which makes many small builds pay for fresh allocations).
void keep_pool_scratch() {
    static std::once_flag once[64];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return;
    std::call_once(once[dev], [dev] {
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, dev) != cudaSuccess) return;
        std::uint64_t keep = 256ULL << 20;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    });
}

// Stream-ordered scratch from the device's memory pool (freed in stream order).
template <class T> struct PoolBuf {
    T* p = nullptr;
    explicit PoolBuf(std::size_t count) {
        if (count) cuda_check(cudaMallocAsync(reinterpret_cast<void**>(&p), count * sizeof(T), nullptr), "cudaMallocAsync");
    }
    PoolBuf(const PoolBuf&) = delete;
    PoolBuf& operator=(const PoolBuf&) = delete;
    ~PoolBuf() {
        if (p) cudaFreeAsync(p, nullptr);
    }
};

// A warp per row (the reference's csr_count / csr_fill, src/gpu/rep_matvec.cu:933-989, likewise deal a row's
// groups to the lanes of a warp). Lane l tests groups l, l + 32, ...; the acting ones' entries land in the
// warp's buffer in group (emission) order under the key column << 8 | emission index. A rank sort of the keys
// orders the entries by column and, within a column, by emission; each column's run is then summed in that order
// and kept when not exactly zero (merge_row, include/ed/matvec/sector_rows.h:147-158). Eight warps a block share
// the staged tables.
// pass 0: merged row lengths, and the merged values into the dictionary set; pass 2: columns and ids.
constexpr int kBuildWarps = 8;
constexpr int kColSetBits = 8;   // the count pass's per-warp column set: 256 slots, for rows of up to 128 entries
constexpr int kColSet = 1 << kColSetBits;

template <class ST, bool kSame>
__global__ void __launch_bounds__(32 * kBuildWarps) csr_pass(DSector row, DSector col, DProgram P, bool prog_in_smem,
                                                             std::size_t stage_bytes, int pass,
                                                             unsigned long long* counts,
                                                             const unsigned long long* row_ptr, u32* col_out,
                                                             unsigned char* ids, int id_bytes, double2* full_vals,
                                                             Dict D, int* too_long, bool tag_rows, int cap) {
    extern __shared__ __align__(16) unsigned char smem[];
    const SmemProgram sp = stage(P, col, smem, prog_in_smem);
    const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // each warp's row buffer holds cap entries (a multiple of 32, at least the program's groups up to 256)
    u64* keys = reinterpret_cast<u64*>(smem + stage_bytes) + wid * cap;
    double2* vals = reinterpret_cast<double2*>(smem + stage_bytes + static_cast<std::size_t>(kBuildWarps) * cap * 8) +
                    wid * cap;
    // the count pass's column set: a warp's slots tagged row << 32 | column, so no row clears them
    u64* cset = reinterpret_cast<u64*>(smem + stage_bytes + static_cast<std::size_t>(kBuildWarps) * cap * 24) +
                wid * kColSet;
    if (pass == 0) {
        for (int i = lane; i < kColSet; i += 32) cset[i] = ~0ULL;
        __syncwarp();
    }
    const unsigned lt = (1u << lane) - 1u;
    const u64 nwarps = static_cast<u64>(gridDim.x) * kBuildWarps;
    for (u64 r = static_cast<u64>(blockIdx.x) * kBuildWarps + wid; r < row.dim; r += nwarps) {
        const ST s = static_cast<ST>(__ldg(row.reps + r));
        const double w = __ldg(row.inv_norms + r);
        // Up to 256 groups: the acting groups first (cheap tests, 32 groups a round), then the canonicalisations
        // of the acting ones only, 32 at a time in group order (lane a of a round takes the a-th acting group).
        // More groups: 32 groups a round, each lane canonicalising its own when it acts. Either way the entries
        // come in group order.
        constexpr int kWords = kMaxRowEntries / 32;
        u32 amask[kWords];
        const int n_words = static_cast<int>((sp.P.n_groups + 31) / 32);
        const bool compact = n_words <= kWords;
        int n_items = n_words * 32;
        if (compact) {
            n_items = 0;
            for (int wi = 0; wi < n_words; ++wi) {
                const u32 g = static_cast<u32>(wi) * 32 + lane;
                const bool act = g < sp.P.n_groups && acting_subgroup<ST>(sp.P, s, g) >= 0;
                amask[wi] = __ballot_sync(0xffffffffu, act);
                n_items += __popc(amask[wi]);
            }
        }
        int m = 0;
        for (int a0 = 0; a0 < n_items; a0 += 32) {
            const int a = a0 + lane;
            bool ok = false;
            long long j = 0;
            cplx c{0.0, 0.0};
            u32 g = static_cast<u32>(a);
            bool go = false;
            if (compact) {
                if (a < n_items) {
                    int rem = a, wi = 0;
                    while (rem >= __popc(amask[wi])) rem -= __popc(amask[wi++]);
                    g = static_cast<u32>(wi) * 32 + __fns(amask[wi], 0, rem + 1);
                    go = true;
                }
            } else {
                go = g < sp.P.n_groups;
            }
            if (go) {
                const int vi = acting_subgroup<ST>(sp.P, s, g);
                if (vi >= 0) {
                    const cplx h = subgroup_value<ST>(sp.P, s, vi);
                    const ST t = s ^ static_cast<ST>(sp.P.group_flip[g]);
                    ok = entry<kSame, ST>(col, sp.T, s, static_cast<long long>(r), w, t, h, j, c);
                }
            }
            const unsigned bal = __ballot_sync(0xffffffffu, ok);
            const int pos = m + __popc(bal & lt);
            if (ok && pos < cap) {
                keys[pos] = (static_cast<u64>(j) << 8) | static_cast<u64>(pos);
                vals[pos] = make_double2(c.re, c.im);
            }
            m += __popc(bal);
        }
        if (m > cap) {
            if (lane == 0) {
                *too_long = 1;
                if (pass == 0) counts[r] = 0;
            }
            continue;
        }
        __syncwarp();
        if (pass == 0 && tag_rows && 2 * m <= kColSet) {
            // Does any column repeat? Each entry's column goes into the warp's set; a column already tagged with this
            // row is a repeat. Without one (the rule: 99.9% of the 6x6 J1-J2 rows) every entry is its own merged
            // value, so the row keeps its nonzero entries and needs no sort.
            bool rep = false;
            for (int i = lane; i < m; i += 32) {
                const u64 tag = (r << 32) | (keys[i] >> 8);
                u32 h = (static_cast<u32>(keys[i] >> 8) * 0x9E3779B1u) >> (32 - kColSetBits);
                // a slot tagged with another row is free; a lost race re-reads the slot. The loop is bounded (the
                // row fills at most half the set, and each lost race is another lane's win); past the bound the
                // row takes the sorting path, which is right whatever the set says.
                int tries = 0;
                for (;; ++tries) {
                    if (tries > 4 * kColSet) {
                        rep = true;
                        break;
                    }
                    const u64 v = *reinterpret_cast<volatile u64*>(cset + h);
                    if (v == tag) {
                        rep = true;
                        break;
                    }
                    if ((v >> 32) != (r & 0xFFFFFFFFULL)) {
                        if (atomicCAS(reinterpret_cast<unsigned long long*>(cset + h), v, tag) == v) break;
                        continue;
                    }
                    h = (h + 1) & (kColSet - 1);
                }
            }
            if (!__any_sync(0xffffffffu, rep)) {
                int kept = 0;
                for (int i = lane; i < m; i += 32) {
                    const double2 v = vals[i];
                    if (v.x != 0.0 || v.y != 0.0) {
                        dict_insert(D, {v.x, v.y});
                        ++kept;
                    }
                }
                for (int o = 16; o > 0; o >>= 1) kept += __shfl_xor_sync(0xffffffffu, kept, o);
                if (lane == 0) counts[r] = static_cast<unsigned long long>(kept);
                __syncwarp();
                continue;
            }
        }
        // the keys (distinct: column << 8 | emission index) sorted by rank: lane l holds keys l, l + 32, ...; every
        // key of the row is read once by the whole warp (a broadcast) and counted against the held ones, then each
        // held key is written to its rank
        {
            constexpr int kHeld = kMaxRowEntries / 32;
            u64 mine[kHeld];
            int rank[kHeld];
#pragma unroll
            for (int i = 0; i < kHeld; ++i) {
                const int at = i * 32 + lane;
                mine[i] = at < m ? keys[at] : ~0ULL;
                rank[i] = 0;
            }
            const int held = (m + 31) >> 5;
            for (int q = 0; q < m; ++q) {
                const u64 kq = keys[q];
#pragma unroll
                for (int i = 0; i < kHeld; ++i)
                    if (i < held) rank[i] += kq < mine[i] ? 1 : 0;
            }
            __syncwarp();
#pragma unroll
            for (int i = 0; i < kHeld; ++i)
                if (i * 32 + lane < m) keys[rank[i]] = mine[i];
            __syncwarp();
        }
        // each column's run summed in emission order; exact zeros dropped; kept entries compacted in order
        int mo = 0;
        const u64 base = pass == 2 ? row_ptr[r] : 0;
        for (int p0 = 0; p0 < m; p0 += 32) {
            const int p = p0 + lane;
            bool keep = false;
            u32 cj = 0;
            cplx sum{0.0, 0.0};
            if (p < m && (p == 0 || (keys[p] >> 8) != (keys[p - 1] >> 8))) {
                cj = static_cast<u32>(keys[p] >> 8);
                const double2 v0 = vals[keys[p] & 0xFF];
                sum = {v0.x, v0.y};
                for (int q = p + 1; q < m && static_cast<u32>(keys[q] >> 8) == cj; ++q) {
                    const double2 v = vals[keys[q] & 0xFF];
                    sum = cadd(sum, {v.x, v.y});
                }
                keep = sum.re != 0.0 || sum.im != 0.0;
            }
            const unsigned bal = __ballot_sync(0xffffffffu, keep);
            if (keep) {
                const u64 o = static_cast<u64>(mo + __popc(bal & lt));
                if (pass == 0) {
                    dict_insert(D, sum);
                } else if (pass == 2) {
                    col_out[base + o] = cj;
                    if (id_bytes == 0)
                        full_vals[base + o] = make_double2(sum.re, sum.im);
                    else if (id_bytes == 1)
                        ids[base + o] = static_cast<unsigned char>(dict_id(D, sum));
                    else
                        reinterpret_cast<unsigned short*>(ids)[base + o] = static_cast<unsigned short>(dict_id(D, sum));
                }
            }
            mo += __popc(bal);
        }
        if (pass == 0 && lane == 0) counts[r] = static_cast<unsigned long long>(mo);
        __syncwarp();
    }
}

// ---- the sparse matvec ----
constexpr int kPerLd = 4;
template <bool kF32> struct Ld;
template <> struct Ld<false> {
    using T = double2;
    __device__ static cplx load(const T* p, std::size_t i) {
        const double2 v = __ldg(p + i);
        return {v.x, v.y};
    }
    __device__ static cplx load(const T (&r)[kPerLd], int q) { return {r[q].x, r[q].y}; }
    __device__ static void store(T* p, std::size_t i, cplx v) { p[i] = make_double2(v.re, v.im); }
};
template <> struct Ld<true> {
    using T = float2;
    __device__ static cplx load(const T* p, std::size_t i) {
        const float2 v = __ldg(p + i);
        return {static_cast<double>(v.x), static_cast<double>(v.y)};
    }
    __device__ static cplx load(const T (&r)[kPerLd], int q) {
        return {static_cast<double>(r[q].x), static_cast<double>(r[q].y)};
    }
    __device__ static void store(T* p, std::size_t i, cplx v) {
        p[i] = make_float2(__double2float_rn(v.re), __double2float_rn(v.im));
    }
};

__device__ __forceinline__ double2 csr_value(const unsigned char* ids, int id_bytes, const double2* vals,
                                             const double2* dict_smem, u64 e) {
    if (id_bytes == 1) return dict_smem[ids[e]];
    if (id_bytes == 2) return __ldg(vals + reinterpret_cast<const unsigned short*>(ids)[e]);
    return __ldg(vals + e);
}

// One vector: a thread per row. The row's entries are read in aligned windows of 4 (one 16-byte load of
// columns, one 4- or 8-byte load of value ids; the column and id arrays are padded to a multiple of 4
// entries, so a window never leaves them); the window's entries outside the row are skipped, the others'
// x loads issued together and their products added in entry order. The sum is the reference's
// (ReducedSymmetryCsr::spmv, include/ed/matvec/reduced_csr.h:89-102: acc = 0, then acc += value * x in entry
// order), so y equals the host CSR's bit for bit. The x loads are random: with x in L2 the kernel is bound
// by L1/L2 sector traffic, beyond it by the DRAM sectors they fetch (32 bytes per 8- or 16-byte element).
constexpr int kRowsPerBlock = 256;
constexpr int kBatch = kPerLd;
static_assert(kBatch == 4, "the 16-byte column windows hold 4 entries");

template <bool kInF32, bool kOutF32>
__global__ void __launch_bounds__(kRowsPerBlock) spmv1(u64 rows, const unsigned long long* __restrict__ row_ptr,
                                                       const u32* __restrict__ col,
                                                       const unsigned char* __restrict__ ids, int id_bytes,
                                                       const double2* __restrict__ vals, int n_dict,
                                                       const void* in_v, void* out_v) {
    __shared__ double2 dict[256];
    if (id_bytes == 1)
        for (int i = threadIdx.x; i < n_dict; i += blockDim.x) dict[i] = vals[i];
    __syncthreads();
    using Li = Ld<kInF32>;
    using Lo = Ld<kOutF32>;
    const auto* in = static_cast<const typename Li::T*>(in_v);
    auto* out = static_cast<typename Lo::T*>(out_v);
    const u64 r = static_cast<u64>(blockIdx.x) * kRowsPerBlock + threadIdx.x;
    if (r >= rows) return;
    cplx acc{0.0, 0.0};
    const u64 e0 = row_ptr[r], e1 = row_ptr[r + 1];
    for (u64 w = e0 & ~3ULL; w < e1; w += 4) {
        const uint4 c4 = __ldg(reinterpret_cast<const uint4*>(col + w));
        const u32 cj[4] = {c4.x, c4.y, c4.z, c4.w};
        unsigned vid[4] = {0, 0, 0, 0};
        if (id_bytes == 1) {
            const unsigned i4 = __ldg(reinterpret_cast<const unsigned*>(ids + w));
#pragma unroll
            for (int q = 0; q < 4; ++q) vid[q] = (i4 >> (8 * q)) & 0xFFu;
        } else if (id_bytes == 2) {
            const uint2 i2 = __ldg(reinterpret_cast<const uint2*>(ids + 2 * w));
            vid[0] = i2.x & 0xFFFFu;
            vid[1] = i2.x >> 16;
            vid[2] = i2.y & 0xFFFFu;
            vid[3] = i2.y >> 16;
        }
        bool on[4];
        typename Li::T xv[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            on[q] = w + q >= e0 && w + q < e1;
            if (on[q]) xv[q] = __ldg(in + cj[q]);
        }
#pragma unroll
        for (int q = 0; q < 4; ++q)
            if (on[q]) {
                const double2 v = id_bytes == 1 ? dict[vid[q]]
                                                : (id_bytes == 2 ? __ldg(vals + vid[q]) : __ldg(vals + w + q));
                acc = cadd(acc, cmul({v.x, v.y}, Li::load(xv, q)));
            }
    }
    Lo::store(out, r, acc);
}

// One vector in FP32 storage (complex64 in; complex64 out, or complex128 into the FP64 scratch of the FP32-storage
// recurrences; FP64 arithmetic): 4 lanes per row. Lane l of a row reads the
// row's 16-byte column windows l, l + 4, ... (a row's four lanes read 64 contiguous bytes of columns and 16 of ids
// per step, where a thread per row reads 16 scattered bytes), issues the window's x loads together and sums its
// products in window order; the four partial sums are added in the fixed order (p0 + p1) + (p2 + p3). A
// different summation order than spmv1's, so it serves FP32 storage only, where results are compared within a
// tolerance; FP64 storage keeps spmv1 and its bit-for-bit sums. u8 dictionary ids only.
// It pays on long rows: 6x6 J1-J2 (75 entries a row) 87.4 -> 74.6 ms, 6x5 (62) 1.08 -> 0.96 ms; on short rows a
// thread per row stays ahead (chain-32, 17.5 entries a row: 0.27 against 0.35 ms).
constexpr int kTeamLanes = 4;
template <bool kOutF32>
__global__ void __launch_bounds__(256) spmv1_team32(u64 rows, const unsigned long long* __restrict__ row_ptr,
                                                    const u32* __restrict__ col, const unsigned char* __restrict__ ids,
                                                    const double2* __restrict__ vals, int n_dict,
                                                    const float2* __restrict__ in, typename Ld<kOutF32>::T* __restrict__ out) {
    __shared__ double2 dict[256];
    for (int i = threadIdx.x; i < n_dict; i += blockDim.x) dict[i] = vals[i];
    __syncthreads();
    const u64 t = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x;
    const u64 r = t / kTeamLanes;
    const int l = static_cast<int>(t % kTeamLanes);
    double ar = 0.0, ai = 0.0;
    if (r < rows) {
        const u64 e0 = row_ptr[r], e1 = row_ptr[r + 1];
        for (u64 w = (e0 & ~3ULL) + 4 * static_cast<u64>(l); w < e1; w += 4 * kTeamLanes) {
            const uint4 c4 = __ldg(reinterpret_cast<const uint4*>(col + w));
            const unsigned i4 = __ldg(reinterpret_cast<const unsigned*>(ids + w));
            const u32 cj[4] = {c4.x, c4.y, c4.z, c4.w};
            float2 xv[4];
            bool on[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                on[q] = w + q >= e0 && w + q < e1;
                if (on[q]) xv[q] = __ldg(in + cj[q]);
            }
#pragma unroll
            for (int q = 0; q < 4; ++q)
                if (on[q]) {
                    const double2 v = dict[(i4 >> (8 * q)) & 0xFFu];
                    const double xr = xv[q].x, xi = xv[q].y;
                    ar += v.x * xr - v.y * xi;
                    ai += v.x * xi + v.y * xr;
                }
        }
    }
    // (p0 + p1) + (p2 + p3) within each row's four lanes
    double br = __shfl_xor_sync(0xffffffffu, ar, 1), bi = __shfl_xor_sync(0xffffffffu, ai, 1);
    ar += br;
    ai += bi;
    br = __shfl_xor_sync(0xffffffffu, ar, 2);
    bi = __shfl_xor_sync(0xffffffffu, ai, 2);
    if (l == 0 && r < rows) Ld<kOutF32>::store(out, r, {ar + br, ai + bi});
}

// k vectors interleaved by row: 8 lanes per row, lane l owns columns l, l + 8, ...; each column summed in
// CSR order (the single apply's order).
template <bool kInF32, bool kOutF32, int kCpl>
__global__ void __launch_bounds__(256) spmvk(u64 rows, int k, const unsigned long long* __restrict__ row_ptr,
                                             const u32* __restrict__ col, const unsigned char* __restrict__ ids,
                                             int id_bytes, const double2* __restrict__ vals, int n_dict,
                                             const void* in_v, void* out_v) {
    __shared__ double2 dict[256];
    if (id_bytes == 1)
        for (int i = threadIdx.x; i < n_dict; i += blockDim.x) dict[i] = vals[i];
    __syncthreads();
    using Li = Ld<kInF32>;
    using Lo = Ld<kOutF32>;
    const auto* in = static_cast<const typename Li::T*>(in_v);
    auto* out = static_cast<typename Lo::T*>(out_v);
    const u64 t = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x;
    const u64 r = t >> 3;
    const int lane = static_cast<int>(t & 7);
    if (r >= rows) return;
    cplx acc[kCpl];
#pragma unroll
    for (int c = 0; c < kCpl; ++c) acc[c] = {0.0, 0.0};
    const u64 e1 = row_ptr[r + 1];
    for (u64 e = row_ptr[r]; e < e1; ++e) {
        const double2 v = csr_value(ids, id_bytes, vals, dict, e);
        const std::size_t base = static_cast<std::size_t>(__ldg(col + e)) * k;
#pragma unroll
        for (int c = 0; c < kCpl; ++c) {
            const int cc = lane + 8 * c;
            if (cc < k) acc[c] = cadd(acc[c], cmul({v.x, v.y}, Li::load(in, base + cc)));
        }
    }
#pragma unroll
    for (int c = 0; c < kCpl; ++c) {
        const int cc = lane + 8 * c;
        if (cc < k) Lo::store(out, static_cast<std::size_t>(r) * k + cc, acc[c]);
    }
}

// The FP32-storage single-vector kernel: four lanes per row when the rows hold at least kTeamMinRow entries on
// average, else one thread per row (spmv1). QB_SPMV_TEAM=0 or 1 forces one or the other. FP64 storage keeps spmv1:
// four lanes per row with spmv1's ordered sums (the products passed to the row's first lane by shuffles) was 7%
// slower on 6x6 (123 against 115 ms).
constexpr u64 kTeamMinRow = 32;
bool team32_for(const qb_csr* A) {
    static const int force = [] {
        const char* e = std::getenv("QB_SPMV_TEAM");
        return e && (e[0] == '0' || e[0] == '1') ? e[0] - '0' : -1;
    }();
    if (force >= 0) return force == 1;
    return A->rows > 0 && A->nnz >= kTeamMinRow * A->rows;
}

template <bool kInF32, bool kOutF32>
void spmv_launch(const qb_csr* A, const void* in, void* out, int k, cudaStream_t st) {
    const unsigned char* ids = A->ids.p;
    const double2* vals = A->vals.p;
    if (k == 1 && kInF32 && A->id_bytes == 1 && team32_for(A)) {
        const u64 threads = A->rows * kTeamLanes;
        spmv1_team32<kOutF32><<<static_cast<unsigned>((threads + 255) / 256), 256, 0, st>>>(
            A->rows, A->row_ptr.p, A->col_idx.p, ids, vals, A->n_dict, static_cast<const float2*>(in),
            static_cast<typename Ld<kOutF32>::T*>(out));
    } else if (k == 1) {
        spmv1<kInF32, kOutF32><<<static_cast<unsigned>((A->rows + kRowsPerBlock - 1) / kRowsPerBlock), kRowsPerBlock, 0, st>>>(
            A->rows, A->row_ptr.p, A->col_idx.p, ids, A->id_bytes, vals, A->n_dict, in, out);
    } else {
        const unsigned blocks = static_cast<unsigned>((A->rows * 8 + 255) / 256);
        const int cpl = (k + 7) / 8;
        if (cpl <= 1)
            spmvk<kInF32, kOutF32, 1><<<blocks, 256, 0, st>>>(A->rows, k, A->row_ptr.p, A->col_idx.p, ids, A->id_bytes, vals, A->n_dict, in, out);
        else if (cpl <= 2)
            spmvk<kInF32, kOutF32, 2><<<blocks, 256, 0, st>>>(A->rows, k, A->row_ptr.p, A->col_idx.p, ids, A->id_bytes, vals, A->n_dict, in, out);
        else if (cpl <= 4)
            spmvk<kInF32, kOutF32, 4><<<blocks, 256, 0, st>>>(A->rows, k, A->row_ptr.p, A->col_idx.p, ids, A->id_bytes, vals, A->n_dict, in, out);
        else if (cpl <= 5)
            spmvk<kInF32, kOutF32, 5><<<blocks, 256, 0, st>>>(A->rows, k, A->row_ptr.p, A->col_idx.p, ids, A->id_bytes, vals, A->n_dict, in, out);
        else if (cpl <= 8)
            spmvk<kInF32, kOutF32, 8><<<blocks, 256, 0, st>>>(A->rows, k, A->row_ptr.p, A->col_idx.p, ids, A->id_bytes, vals, A->n_dict, in, out);
        else
            throw Error(QB_EUNSUPPORTED, "CSR matvec: at most 64 vectors");
    }
    cuda_check(cudaGetLastError(), "CSR matvec launch");
}

template <class ST, bool kSame>
void run_pass(const qb_sector* row, const qb_sector* col, const qb_program* P, int pass, unsigned long long* counts,
              const unsigned long long* row_ptr, u32* col_out, unsigned char* ids, int id_bytes, double2* full,
              const Dict& D, int* too_long) {
    bool in_smem = false;
    const std::size_t stage_bytes = (smem_for(P, col, in_smem) + 15) & ~std::size_t(15);
    // a row holds at most one entry per group: buffers of the program's groups rounded up to 32 (256 at most), so
    // more warps fit an SM than with 256-entry buffers
    const u32 ng = P->view.n_groups;
    const int cap = ng <= static_cast<u32>(kMaxRowEntries) ? std::max(32, static_cast<int>((ng + 31) / 32 * 32))
                                                          : kMaxRowEntries;
    const std::size_t smem = stage_bytes + static_cast<std::size_t>(kBuildWarps) * cap * (8 + 16) +
                             static_cast<std::size_t>(kBuildWarps) * kColSet * 8;
    auto k = csr_pass<ST, kSame>;
    set_smem(k, smem);
    int sms = 148, dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const u64 want = (row->dim + kBuildWarps - 1) / kBuildWarps;
    const unsigned blocks = static_cast<unsigned>(std::max<u64>(1, std::min<u64>(want, static_cast<u64>(sms) * 16)));
    // row tags hold the low 32 bits of the row: rows past 2^32 take the sorting path
    const bool tag_rows = row->dim < (1ULL << 32);
    k<<<blocks, 32 * kBuildWarps, smem>>>(row->view(), col->view(), P->view, in_smem, stage_bytes, pass, counts,
                                          row_ptr, col_out, ids, id_bytes, full, D, too_long, tag_rows, cap);
    cuda_check(cudaGetLastError(), "CSR build pass");
}

template <class ST>
void build_passes(const qb_sector* row, const qb_sector* col, const qb_program* P, int pass, unsigned long long* counts,
                  const unsigned long long* row_ptr, u32* col_out, unsigned char* ids, int id_bytes, double2* full,
                  const Dict& D, int* too_long) {
    if (row == col)
        run_pass<ST, true>(row, col, P, pass, counts, row_ptr, col_out, ids, id_bytes, full, D, too_long);
    else
        run_pass<ST, false>(row, col, P, pass, counts, row_ptr, col_out, ids, id_bytes, full, D, too_long);
}

struct BitsHash {
    std::size_t operator()(const std::pair<u64, u64>& k) const noexcept {
        u64 a = k.first ^ (k.second * 0x9e3779b97f4a7c15ULL);
        a ^= a >> 31;
        return static_cast<std::size_t>(a * 0xbf58476d1ce4e5b9ULL);
    }
};

// The column and id arrays hold a multiple of 4 entries (at least 4): the matvec reads them in aligned
// windows of 4.
u64 padded(u64 nnz) { return ((nnz + 3) & ~3ULL) + (nnz == 0 ? 4 : 0); }

// The id width of a dictionary of n values over nnz entries: 1 (u8) up to 256 values, 2 (u16) up to 65536,
// 0 (whole values) beyond, or when the dictionary form is not the smaller one (build_cross_csr,
// include/ed/matvec/sector_rows.h:363-366).
int dict_id_bytes(std::size_t n, u64 nnz) {
    if (n > 65536) return 0;
    const int w = n <= 256 ? 1 : 2;
    if (n * 16 + nnz * static_cast<u64>(w) >= nnz * 16) return 0;
    return w;
}

// Refuses a CSR above the caller's byte budget (0: none) or the device's free memory.
void check_budget(u64 rows, u64 nnz, int id_bytes, std::size_t n_dict, uint64_t max_bytes) {
    const uint64_t need = (rows + 1) * 8 + nnz * (4 + (id_bytes ? id_bytes : 16)) + (id_bytes ? n_dict * 16 : 0);
    if (max_bytes && need > max_bytes)
        throw Error(QB_ENOMEM, "CSR: " + std::to_string(need) + " bytes exceed the budget of " +
                                   std::to_string(max_bytes));
    std::size_t free_b = 0, total_b = 0;
    cuda_check(cudaMemGetInfo(&free_b, &total_b), "cudaMemGetInfo");
    free_b += idle_cached_bytes();
    if (need > free_b) throw Error(QB_ENOMEM, "CSR: " + std::to_string(need) + " bytes, " + std::to_string(free_b) +
                                                  " free on the device");
}

}  // namespace

void csr_spmv(const qb_csr* A, const void* in, void* out, int k, int dtype_in, int dtype_out, cudaStream_t st) {
    if (A->rows == 0) return;
    if (dtype_in == QB_C64 && dtype_out == QB_C64)
        spmv_launch<true, true>(A, in, out, k, st);
    else if (dtype_in == QB_C64)
        spmv_launch<true, false>(A, in, out, k, st);
    else if (dtype_out == QB_C64)
        spmv_launch<false, true>(A, in, out, k, st);
    else
        spmv_launch<false, false>(A, in, out, k, st);
}

}  // namespace qb

extern "C" {

int qb_csr_build(const qb_sector* row, const qb_sector* col, const qb_program* prog, uint64_t max_bytes,
                 qb_csr** out) {
    return qb::guarded([&] {
        using namespace qb;
        if (!row || !col || !prog || !out) throw Error(QB_EINVAL, "null argument");
        if (row->N != col->N) throw Error(QB_EINVAL, "sectors of different sizes");
        if (col->dim >= (1ULL << 32)) throw Error(QB_EUNSUPPORTED, "CSR: column indices past 2^32");
        auto A = std::make_unique<qb_csr>();
        A->row = row;
        A->col = col;
        A->rows = row->dim;
        A->row_ptr.alloc(row->dim + 1);
        cuda_check(cudaMemset(A->row_ptr.p, 0, (row->dim + 1) * 8), "row_ptr clear");
        if (row->dim == 0) {
            *out = A.release();
            return;
        }
        const bool narrow = row->N <= 32 && col->N <= 32;
        keep_pool_scratch();
        // flags: [0] a row past 256 entries, [1] dictionary overflow, [2] values inserted, [3] dictionary size
        PoolBuf<int> flags(4);
        cuda_check(cudaMemsetAsync(flags.p, 0, 16, nullptr), "flags clear");
        int hflags[4] = {0, 0, 0, 0};
        // the value set, filled by the count pass: at most half full while it can still become a dictionary
        // (65536 values in 2^kDictBits slots), and no larger than twice the entries can fill (rows x groups)
        u64 nslots = 1024;
        const u64 most = row->dim * std::max<u64>(1, prog->view.n_groups);
        while (nslots < 2 * most && nslots < (1ULL << kDictBits)) nslots <<= 1;
        PoolBuf<u64> keys(nslots);
        PoolBuf<double2> dvals(nslots);
        PoolBuf<u32> dids(nslots);
        PoolBuf<double2> dict(kMaxDict);
        cuda_check(cudaMemsetAsync(keys.p, 0xFF, nslots * 8, nullptr), "dict clear");
        Dict D{keys.p, nslots - 1, dvals.p, dids.p, flags.p + 1, reinterpret_cast<u32*>(flags.p + 2)};
        {
            PoolBuf<unsigned long long> counts(row->dim);
            auto passes = [&](int pass, unsigned char* ids, int id_bytes, double2* full) {
                if (narrow)
                    build_passes<u32>(row, col, prog, pass, counts.p, A->row_ptr.p, A->col_idx.p, ids, id_bytes, full,
                                      D, flags.p);
                else
                    build_passes<u64>(row, col, prog, pass, counts.p, A->row_ptr.p, A->col_idx.p, ids, id_bytes, full,
                                      D, flags.p);
            };
            passes(0, nullptr, 0, nullptr);
            // row_ptr[1:] = inclusive scan of the counts
            std::size_t tmp = 0;
            cub::DeviceScan::InclusiveSum(nullptr, tmp, counts.p, A->row_ptr.p + 1, static_cast<int>(row->dim));
            PoolBuf<unsigned char> tmpb(std::max<std::size_t>(tmp, 1));
            cub::DeviceScan::InclusiveSum(tmpb.p, tmp, counts.p, A->row_ptr.p + 1, static_cast<int>(row->dim));
            cuda_check(cudaGetLastError(), "CSR scan");
        }
        cuda_check(cudaMemcpy(&A->nnz, A->row_ptr.p + row->dim, 8, cudaMemcpyDeviceToHost), "nnz read");
        cuda_check(cudaMemcpy(hflags, flags.p, 16, cudaMemcpyDeviceToHost), "flags read");
        if (hflags[0]) throw Error(QB_EUNSUPPORTED, "CSR: a row has more than 256 entries before merging");
        auto passes = [&](int pass, unsigned char* ids, int id_bytes, double2* full) {
            if (narrow)
                build_passes<u32>(row, col, prog, pass, nullptr, A->row_ptr.p, A->col_idx.p, ids, id_bytes, full, D,
                                  flags.p);
            else
                build_passes<u64>(row, col, prog, pass, nullptr, A->row_ptr.p, A->col_idx.p, ids, id_bytes, full, D,
                                  flags.p);
        };
        dict_compact<<<1, 1024>>>(keys.p, dvals.p, nslots, dids.p, dict.p, flags.p + 3);
        cuda_check(cudaGetLastError(), "dictionary");
        cuda_check(cudaMemcpy(hflags, flags.p, 16, cudaMemcpyDeviceToHost), "dictionary read");
        const std::size_t n_dict = static_cast<std::size_t>(hflags[3]);
        int id_bytes = hflags[1] ? 0 : dict_id_bytes(n_dict, A->nnz);
        check_budget(row->dim, A->nnz, id_bytes, n_dict, max_bytes);
        A->col_idx.alloc(padded(A->nnz));
        for (int attempt = 0; attempt < 2; ++attempt) {
            if (id_bytes) {
                A->ids.alloc(padded(A->nnz) * id_bytes);
                A->vals.alloc(n_dict);
                cuda_check(cudaMemcpy(A->vals.p, dict.p, n_dict * 16, cudaMemcpyDeviceToDevice), "dictionary copy");
                A->n_dict = static_cast<int>(n_dict);
            } else {
                A->ids.release();
                A->vals.alloc(A->nnz);
                A->n_dict = 0;
            }
            A->id_bytes = id_bytes;
            cuda_check(cudaMemsetAsync(flags.p + 1, 0, 4, nullptr), "flags clear");
            passes(2, A->ids.p, id_bytes, A->vals.p);
            cuda_check(cudaMemcpy(hflags, flags.p, 16, cudaMemcpyDeviceToHost), "fill read");
            if (!hflags[1] || id_bytes == 0) break;
            id_bytes = 0;   // a key collision: store every value whole
            A->ids.release();
            check_budget(row->dim, A->nnz, 0, 0, max_bytes);
        }
        *out = A.release();
    });
}

int qb_csr_upload(const qb_sector* row, const qb_sector* col, const uint64_t* row_ptr, const uint32_t* col_idx,
                  const double* val, uint64_t max_bytes, qb_csr** out) {
    return qb::guarded([&] {
        using namespace qb;
        if (!row || !col || !row_ptr || !out) throw Error(QB_EINVAL, "null argument");
        const u64 rows = row->dim;
        const u64 nnz = row_ptr[rows];
        if (row_ptr[0] != 0) throw Error(QB_EINVAL, "CSR: row_ptr[0] != 0");
        for (u64 r = 0; r < rows; ++r)
            if (row_ptr[r + 1] < row_ptr[r]) throw Error(QB_EINVAL, "CSR: row_ptr decreases");
        if (nnz && (!col_idx || !val)) throw Error(QB_EINVAL, "null argument");
        for (u64 e = 0; e < nnz; ++e)
            if (col_idx[e] >= col->dim) throw Error(QB_EINVAL, "CSR: a column past the column sector");
        // the dictionary in first-appearance order, keyed by the values' bits
        std::unordered_map<std::pair<u64, u64>, u32, BitsHash> index;
        std::vector<double2> dict;
        std::vector<u32> id(nnz);
        for (u64 e = 0; e < nnz && dict.size() <= 65536; ++e) {
            u64 re, im;
            std::memcpy(&re, val + 2 * e, 8);
            std::memcpy(&im, val + 2 * e + 1, 8);
            const auto [it, fresh] = index.try_emplace({re, im}, static_cast<u32>(dict.size()));
            if (fresh) dict.push_back(make_double2(val[2 * e], val[2 * e + 1]));
            id[e] = it->second;
        }
        const int id_bytes = dict_id_bytes(dict.size(), nnz);
        check_budget(rows, nnz, id_bytes, dict.size(), max_bytes);
        auto A = std::make_unique<qb_csr>();
        A->row = row;
        A->col = col;
        A->rows = rows;
        A->nnz = nnz;
        A->id_bytes = id_bytes;
        A->row_ptr.upload(reinterpret_cast<const unsigned long long*>(row_ptr), rows + 1);
        A->col_idx.alloc(padded(nnz));
        if (nnz) upload_host(A->col_idx.p, col_idx, nnz * 4, nullptr);
        if (id_bytes) {
            std::vector<unsigned char> ids(padded(nnz) * id_bytes, 0);
            for (u64 e = 0; e < nnz; ++e) {
                if (id_bytes == 1)
                    ids[e] = static_cast<unsigned char>(id[e]);
                else
                    reinterpret_cast<unsigned short*>(ids.data())[e] = static_cast<unsigned short>(id[e]);
            }
            A->ids.upload(ids);
            A->vals.upload(dict);
            A->n_dict = static_cast<int>(dict.size());
        } else {
            A->vals.upload(reinterpret_cast<const double2*>(val), nnz);
        }
        *out = A.release();
    });
}

int qb_csr_destroy(qb_csr* A) {
    return qb::guarded([&] { delete A; });
}

int qb_csr_info(const qb_csr* A, uint64_t* nnz, uint64_t* bytes, int* n_dict) {
    return qb::guarded([&] {
        if (!A) throw qb::Error(QB_EINVAL, "null CSR");
        if (nnz) *nnz = A->nnz;
        if (bytes) *bytes = A->bytes();
        if (n_dict) *n_dict = A->id_bytes ? A->n_dict : -1;
    });
}

int qb_csr_download(const qb_csr* A, uint64_t* row_ptr, uint32_t* col, double* val) {
    return qb::guarded([&] {
        using namespace qb;
        if (!A) throw Error(QB_EINVAL, "null CSR");
        if (row_ptr) cuda_check(cudaMemcpy(row_ptr, A->row_ptr.p, (A->rows + 1) * 8, cudaMemcpyDeviceToHost), "download");
        if (col && A->nnz) cuda_check(cudaMemcpy(col, A->col_idx.p, A->nnz * 4, cudaMemcpyDeviceToHost), "download");
        if (val && A->nnz) {
            if (A->id_bytes == 0) {
                cuda_check(cudaMemcpy(val, A->vals.p, A->nnz * 16, cudaMemcpyDeviceToHost), "download");
            } else {
                std::vector<unsigned char> ids(A->nnz * A->id_bytes);
                std::vector<double2> dict(A->n_dict);
                cuda_check(cudaMemcpy(ids.data(), A->ids.p, ids.size(), cudaMemcpyDeviceToHost), "download");
                cuda_check(cudaMemcpy(dict.data(), A->vals.p, dict.size() * 16, cudaMemcpyDeviceToHost), "download");
                for (uint64_t e = 0; e < A->nnz; ++e) {
                    const unsigned id = A->id_bytes == 1 ? ids[e] : reinterpret_cast<const unsigned short*>(ids.data())[e];
                    val[2 * e] = dict[id].x;
                    val[2 * e + 1] = dict[id].y;
                }
            }
        }
    });
}

int qb_csr_matvec(const qb_csr* A, const void* in, void* out, int k, int dtype, void* stream) {
    return qb::guarded([&] {
        if (!A) throw qb::Error(QB_EINVAL, "null CSR");
        if (dtype != QB_C128 && dtype != QB_C64) throw qb::Error(QB_EINVAL, "bad dtype");
        if (k < 1 || k > 64) throw qb::Error(QB_EINVAL, "k must be in [1, 64]");
        qb::csr_spmv(A, in, out, k, dtype, dtype, static_cast<cudaStream_t>(stream));
    });
}

int qb_program_attach_csr(qb_program* prog, const qb_csr* A) {
    return qb::guarded([&] {
        if (!prog) throw qb::Error(QB_EINVAL, "null program");
        prog->csr = A;
    });
}

}  // extern "C"
