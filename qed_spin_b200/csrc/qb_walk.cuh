// =============================================================================
// qb_walk.cuh -- the row walk shared by the matvec kernels and the CSR build: the program and sector
// tables staged in shared memory, a group's acting subgroup and value (include/ed/ops/row_walk.h:28-65),
// and one connection's matrix entry (include/ed/matvec/sector_rows.h:41-56).
// =============================================================================
#pragma once

#include <cstddef>

#include "qb_canon.cuh"

namespace qb {

// The column sector's tables and the row program staged in shared memory (the program stays in global
// memory when too large).
struct SmemProgram {
    DProgram P;
    Tables T;
};

__device__ __forceinline__ SmemProgram stage(const DProgram& P, const DSector& col, unsigned char* smem, bool in_smem) {
    SmemProgram out{P, stage_tables(col, smem)};
    unsigned char* p = smem + ((tables_smem_bytes(col) + 15) & ~std::size_t(15));
    auto take = [&](std::size_t bytes) {
        unsigned char* r = p;
        p += (bytes + 15) & ~std::size_t(15);
        return r;
    };
    if (in_smem) {
        u64* gf = reinterpret_cast<u64*>(take(P.n_groups * 8ull));
        int* gs = reinterpret_cast<int*>(take(P.n_groups * 4ull));
        u32* gv = reinterpret_cast<u32*>(take((P.n_groups + 1) * 4ull));
        u64* vv = reinterpret_cast<u64*>(take(P.n_vsub * 8ull));
        u32* vt = reinterpret_cast<u32*>(take((P.n_vsub + 1) * 4ull));
        u64* ts = reinterpret_cast<u64*>(take(P.n_terms * 8ull));
        double2* tc = reinterpret_cast<double2*>(take(P.n_terms * 16ull));
        for (u32 i = threadIdx.x; i < P.n_groups; i += blockDim.x) {
            gf[i] = P.group_flip[i];
            gs[i] = P.group_setbits[i];
        }
        for (u32 i = threadIdx.x; i <= P.n_groups; i += blockDim.x) gv[i] = P.group_vbegin[i];
        for (u32 i = threadIdx.x; i < P.n_vsub; i += blockDim.x) vv[i] = P.vsub_val[i];
        for (u32 i = threadIdx.x; i <= P.n_vsub; i += blockDim.x) vt[i] = P.vsub_tbegin[i];
        for (u32 i = threadIdx.x; i < P.n_terms; i += blockDim.x) {
            ts[i] = P.term_sign[i];
            tc[i] = P.term_coeff[i];
        }
        out.P.group_flip = gf;
        out.P.group_setbits = gs;
        out.P.group_vbegin = gv;
        out.P.vsub_val = vv;
        out.P.vsub_tbegin = vt;
        out.P.term_sign = ts;
        out.P.term_coeff = tc;
    }
    __syncthreads();
    return out;
}

template <class ST> __device__ __forceinline__ int popc(ST x);
template <> __device__ __forceinline__ int popc<u64>(u64 x) { return __popcll(x); }
template <> __device__ __forceinline__ int popc<u32>(u32 x) { return __popc(x); }

// The value subgroup of group g that s meets, or -1 (include/ed/ops/row_walk.h:32-43).
template <class ST> __device__ __forceinline__ int acting_subgroup(const DProgram& P, ST s, u32 g) {
    const ST F = static_cast<ST>(P.group_flip[g]);
    const ST v = s & F;
    const int sb = P.group_setbits[g];
    if (sb >= 0 && popc<ST>(v) != sb) return -1;
    u32 lo = P.group_vbegin[g], hi = P.group_vbegin[g + 1];
    const u32 end = hi;
    while (lo < hi) {
        const u32 mid = lo + ((hi - lo) >> 1);
        if (static_cast<ST>(P.vsub_val[mid]) < v)
            lo = mid + 1;
        else
            hi = mid;
    }
    return (lo == end || static_cast<ST>(P.vsub_val[lo]) != v) ? -1 : static_cast<int>(lo);
}

// h = <s ^ F|O^dagger|s>: the subgroup's terms summed in key order with their signs (row_walk.h:44-50).
template <class ST> __device__ __forceinline__ cplx subgroup_value(const DProgram& P, ST s, int vi) {
    cplx h{0.0, 0.0};
    for (u32 k = P.vsub_tbegin[vi]; k < P.vsub_tbegin[vi + 1]; ++k) {
        const double2 c = P.term_coeff[k];
        if (popc<ST>(s & static_cast<ST>(P.term_sign[k])) & 1)
            h = cadd(h, {-c.x, -c.y});
        else
            h = cadd(h, {c.x, c.y});
    }
    return h;
}

// connection (include/ed/ops/row_walk.h:28-52): whether group g acts on s; its target and h.
template <class ST> __device__ __forceinline__ bool connection(const DProgram& P, ST s, u32 g, ST& t, cplx& h) {
    const int vi = acting_subgroup<ST>(P, s, g);
    if (vi < 0) return false;
    h = subgroup_value<ST>(P, s, vi);
    t = s ^ static_cast<ST>(P.group_flip[g]);
    return true;
}

// The entry of one connection: column j and value c, or false when the target's orbit cancels.
template <bool kSame, class ST>
__device__ __forceinline__ bool entry(const DSector& col, const Tables& T, ST s, long long r, double w, ST t,
                                      cplx h, long long& j, cplx& c) {
    if (kSame && t == s) {
        j = r;
        c = cconj(h);
        return true;
    }
    double pre, pim;
    j = index_and_projection<ST>(col, T, t, pre, pim);
    if (j < 0) return false;
    c = rscale(w, cconj(cmul(h, {pre, pim})));
    return true;
}

template <bool kF32> struct Store;
template <> struct Store<false> {
    using T = double2;
    __device__ static cplx load(const T* p, std::size_t i) {
        const double2 v = __ldg(p + i);
        return {v.x, v.y};
    }
    __device__ static void store(T* p, std::size_t i, cplx v) { p[i] = make_double2(v.re, v.im); }
};
template <> struct Store<true> {
    using T = float2;
    __device__ static cplx load(const T* p, std::size_t i) {
        const float2 v = __ldg(p + i);
        return {static_cast<double>(v.x), static_cast<double>(v.y)};
    }
    __device__ static void store(T* p, std::size_t i, cplx v) { p[i] = make_float2(__double2float_rn(v.re), __double2float_rn(v.im)); }
};


inline std::size_t smem_for(const qb_program* P, const qb_sector* col, bool& in_smem) {
    const std::size_t tables = (tables_smem_bytes(col->view()) + 15) & ~std::size_t(15);
    in_smem = P->view.smem_bytes <= 40 * 1024;
    return tables + (in_smem ? P->view.smem_bytes : 0);
}

template <class K> void set_smem(K kernel, std::size_t bytes) {
    if (bytes > 48 * 1024)
        cuda_check(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes)),
                   "smem attribute");
}

}  // namespace qb
