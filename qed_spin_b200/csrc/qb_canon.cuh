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

// Image of s under element g: OR of bpw byte-table words, XOR the element's flip mask
// (include/ed/basis/compiled_group.h:73-78).
__device__ __forceinline__ u64 apply_elem(const DSector& S, u64 s, int g) {
    const u64* l = S.lut + static_cast<std::size_t>(g) * S.bpw * 256;
    u64 r = 0;
#pragma unroll 8
    for (int b = 0; b < S.bpw; ++b) r |= __ldg(l + b * 256 + static_cast<int>((s >> (8 * b)) & 0xFFu));
    return r ^ __ldg(S.flips + g);
}

// A state's bits moved to their key positions (to_key staged in shared memory).
__device__ __forceinline__ u64 key_of(const u64* to_key, int bpw, u64 s) {
    u64 k = 0;
#pragma unroll 8
    for (int b = 0; b < bpw; ++b) k |= to_key[(b << 8) + static_cast<int>((s >> (8 * b)) & 0xFFu)];
    return k;
}

__device__ __forceinline__ u32 pattern_of(u64 k, int j, int N, int L) {
    return static_cast<u32>(k >> (N - (j + 1) * L)) & ((1u << L) - 1u);
}

// fn(g) in ascending order for the elements whose image has the least leading block
// (sublattice_code.h:102-131). `first_lead`: the state's own leading block vs the least one
// (visit_state's early rejection) is reported through least / own.
template <class Fn>
__device__ __forceinline__ void for_each_candidate(const DSector& S, u64 k, Fn&& fn) {
    const int L = S.slc.L, m = S.slc.m, N = S.N;
    u32 entry[8];
    u32 best = 0xFFFFFFFFu;
    for (int j = 0; j < m; ++j) {
        entry[j] = (static_cast<u32>(j) << L) + pattern_of(k, j, N, L);
        const u32 v = __ldg(S.slc.lead + entry[j]);
        best = v < best ? v : best;
    }
    u32 pos[8], end[8];
    int n = 0;
    for (int j = 0; j < m; ++j)
        if (__ldg(S.slc.lead + entry[j]) == best) {
            pos[n] = __ldg(S.slc.cand_off + entry[j]);
            end[n] = __ldg(S.slc.cand_off + entry[j] + 1);
            ++n;
        }
    if (n == 1) {
        for (u32 p = pos[0]; p < end[0]; ++p) fn(static_cast<int>(__ldg(S.slc.cand + p)));
        return;
    }
    for (;;) {
        int pick = -1;
        u32 g = 0xFFFFFFFFu;
        for (int i = 0; i < n; ++i)
            if (pos[i] < end[i]) {
                const u32 c = __ldg(S.slc.cand + pos[i]);
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

// Representative of t and the conjugated character sum over the elements that reach it.
__device__ __forceinline__ u64 canonicalize(const DSector& S, const u64* to_key, u64 t, double& acc_re,
                                            double& acc_im) {
    u64 rb = ~0ULL, best = ~0ULL;
    acc_re = 0.0;
    acc_im = 0.0;
    auto visit = [&](int g) {
        const u64 img = apply_elem(S, t, g);
        const u64 k = S.slc.on ? key_of(to_key, S.bpw, img) : img;
        if (k < best) {
            best = k;
            rb = img;
            const double2 c = __ldg(S.chars + g);
            acc_re = __dadd_rn(0.0, c.x);
            acc_im = __dsub_rn(0.0, c.y);
        } else if (k == best) {
            const double2 c = __ldg(S.chars + g);
            acc_re = __dadd_rn(acc_re, c.x);
            acc_im = __dsub_rn(acc_im, c.y);
        }
    };
    if (S.slc.on) {
        for_each_candidate(S, key_of(to_key, S.bpw, t), visit);
    } else {
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

// Index of representative rb in the sector, or -1 (index_of_rep, rep_symmetry_basis_policy.h:169-202).
__device__ __forceinline__ long long index_of_rep(const DSector& S, u64 rb) {
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
__device__ __forceinline__ long long index_and_projection(const DSector& S, const u64* to_key, u64 t, double& pre,
                                                          double& pim) {
    if (__popcll(t) != S.n_up) return -1;
    double are, aim;
    const u64 rb = canonicalize(S, to_key, t, are, aim);
    const long long j = index_of_rep(S, rb);
    if (j < 0) return -1;
    const double s = __ldg(S.inv_norms + j);
    pre = __dmul_rn(are, s);
    pim = __dmul_rn(aim, s);
    return j;
}

}  // namespace qb
