// =============================================================================
// matvec.cu -- the on-the-fly symmetry-sector matvec on the device.
//
// Row r of O in the sector (include/ed/matvec/sector_rows.h:1-56): walk the row program from the
// representative s_r; every group that acts gives a target t and h = <t|O^dagger|s_r>; the entry is
// conj(h) at column r for the diagonal group, else inv_norm[r] conj(h proj(t)) at column j(t) with
// (j, proj) = index_and_projection(t). Each row sums its entries in group order with the host's
// complex arithmetic (no fused multiply-adds), so y equals the reference's sector_gather bit for bit
// in FP64 storage.
//
// Two kernels:
//   walk_rows   one thread per row, up to 8 separate vectors (the reference's multi-apply contract:
//               every output equals the single apply bit for bit). The row program and the key
//               table are staged in shared memory; a warp's lanes advance in step over their own
//               acting groups so the expensive canonicalisation runs with every lane busy.
//   walk_team   the block matvec of the sampled methods: k vectors interleaved by row. A team of
//               8 lanes owns a row: the lanes test 8 groups at once, canonicalise the acting targets
//               in parallel, then every lane accumulates its slice of the k columns from each target
//               in group order -- one canonicalisation per entry for all k vectors, and each x row
//               read as one contiguous segment.
// =============================================================================
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>

#include "qb_canon.cuh"

namespace qb {

namespace {

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

template <int NV> struct VecPtrs {
    const void* in[NV];
    void* out[NV];
};

// One thread per row. The row's groups are tested 32 at a time by every lane together (a converged
// pass that builds the bitmask of the groups acting on the lane's row); the lanes then walk their own
// acting groups in ascending order -- the diagonal first -- canonicalising one target each per step.
template <int NV, class ST, bool kInF32, bool kOutF32, bool kSame>
__global__ void __launch_bounds__(256, 4) walk_rows(DSector row, DSector col, DProgram P, bool prog_in_smem,
                                                    VecPtrs<NV> io) {
    extern __shared__ __align__(16) unsigned char smem[];
    using St = Store<kInF32>;
    using So = Store<kOutF32>;
    const SmemProgram sp = stage(P, col, smem, prog_in_smem);
    const std::uint64_t r = static_cast<std::uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const bool live = r < row.dim;
    const ST s = live ? static_cast<ST>(__ldg(row.reps + r)) : static_cast<ST>(0);
    const double w = live ? __ldg(row.inv_norms + r) : 0.0;
    cplx acc[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) acc[v] = {0.0, 0.0};
    const u32 ng = sp.P.n_groups;
    for (u32 g0 = 0; g0 < ng; g0 += 32) {
        const u32 gend = ng < g0 + 32 ? ng : g0 + 32;
        u32 mask = 0;
        if (live)
            for (u32 g = g0; g < gend; ++g)
                if (acting_subgroup<ST>(sp.P, s, g) >= 0) mask |= 1u << (g - g0);
        while (__any_sync(0xffffffffu, mask != 0)) {
            if (mask == 0) continue;
            const u32 g = g0 + static_cast<u32>(__ffs(mask) - 1);
            mask &= mask - 1;
            const int vi = acting_subgroup<ST>(sp.P, s, g);
            const cplx h = subgroup_value<ST>(sp.P, s, vi);
            const ST t = s ^ static_cast<ST>(sp.P.group_flip[g]);
            long long j;
            cplx c;
            if (!entry<kSame, ST>(col, sp.T, s, static_cast<long long>(r), w, t, h, j, c)) continue;
#pragma unroll
            for (int v = 0; v < NV; ++v)
                acc[v] = cadd(acc[v], cmul(c, St::load(static_cast<const typename St::T*>(io.in[v]), static_cast<std::size_t>(j))));
        }
    }
    if (!live) return;
#pragma unroll
    for (int v = 0; v < NV; ++v) So::store(static_cast<typename So::T*>(io.out[v]), r, acc[v]);
}

// Team kernel: kTeam lanes per row, kCpl columns per lane (k <= kTeam kCpl vectors).
template <int kCpl, bool kF32, bool kOutF32, bool kSame>
__global__ void __launch_bounds__(256) walk_team(DSector row, DSector col, DProgram P, bool prog_in_smem,
                                                 const void* in_v, void* out_v, int k) {
    constexpr int kTeam = 8;
    extern __shared__ __align__(16) unsigned char smem[];
    using St = Store<kF32>;
    using So = Store<kOutF32>;
    using T = typename St::T;
    const T* in = static_cast<const T*>(in_v);
    typename So::T* out = static_cast<typename So::T*>(out_v);
    const SmemProgram sp = stage(P, col, smem, prog_in_smem);
    const int lane = threadIdx.x & 31;
    const int team = lane / kTeam, tl = lane % kTeam;
    const unsigned team_mask = 0xFFu << (team * kTeam);
    const std::uint64_t warp = (static_cast<std::uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const std::uint64_t r = warp * (32 / kTeam) + team;
    const bool live = r < row.dim;
    const u64 s = live ? __ldg(row.reps + r) : 0;
    const double w = live ? __ldg(row.inv_norms + r) : 0.0;
    cplx acc[kCpl];
#pragma unroll
    for (int c = 0; c < kCpl; ++c) acc[c] = {0.0, 0.0};
    const int c0 = tl * kCpl;
    for (u32 g0 = 0; g0 < sp.P.n_groups; g0 += kTeam) {
        const u32 g = g0 + tl;
        u64 t = 0;
        cplx h{0.0, 0.0};
        long long j = -1;
        cplx cv{0.0, 0.0};
        bool act = live && g < sp.P.n_groups && connection<u64>(sp.P, s, g, t, h);
        if (act) act = entry<kSame, u64>(col, sp.T, s, static_cast<long long>(r), w, t, h, j, cv);
        unsigned acting = __ballot_sync(0xffffffffu, act) & team_mask;
        while (acting) {
            const int src = __ffs(acting) - 1;
            acting &= acting - 1;
            const long long jj = __shfl_sync(team_mask, j, src);
            const double cre = __shfl_sync(team_mask, cv.re, src);
            const double cim = __shfl_sync(team_mask, cv.im, src);
            const std::size_t base = static_cast<std::size_t>(jj) * k;
#pragma unroll
            for (int c = 0; c < kCpl; ++c)
                if (c0 + c < k) acc[c] = cadd(acc[c], cmul({cre, cim}, St::load(in, base + c0 + c)));
        }
    }
    if (!live) return;
#pragma unroll
    for (int c = 0; c < kCpl; ++c)
        if (c0 + c < k) So::store(out, static_cast<std::size_t>(r) * k + c0 + c, acc[c]);
}

std::size_t smem_for(const qb_program* P, const qb_sector* col, bool& in_smem) {
    const std::size_t tables = (tables_smem_bytes(col->view()) + 15) & ~std::size_t(15);
    in_smem = P->view.smem_bytes <= 40 * 1024;
    return tables + (in_smem ? P->view.smem_bytes : 0);
}

template <class K> void set_smem(K kernel, std::size_t bytes) {
    if (bytes > 48 * 1024)
        cuda_check(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes)),
                   "smem attribute");
}

template <int NV, class ST, bool kF32, bool kOutF32>
void launch_rows_st(const qb_sector* row, const qb_sector* col, const qb_program* P, const VecPtrs<NV>& io,
                    cudaStream_t st) {
    bool in_smem = false;
    const std::size_t smem = smem_for(P, col, in_smem);
    const unsigned blocks = static_cast<unsigned>((row->dim + 255) / 256);
    if (row == col) {
        auto k = walk_rows<NV, ST, kF32, kOutF32, true>;
        set_smem(k, smem);
        k<<<blocks, 256, smem, st>>>(row->view(), col->view(), P->view, in_smem, io);
    } else {
        auto k = walk_rows<NV, ST, kF32, kOutF32, false>;
        set_smem(k, smem);
        k<<<blocks, 256, smem, st>>>(row->view(), col->view(), P->view, in_smem, io);
    }
    cuda_check(cudaGetLastError(), "walk_rows launch");
}

template <int NV, bool kF32, bool kOutF32 = kF32>
void launch_rows_nv(const qb_sector* row, const qb_sector* col, const qb_program* P, const void* const* ins,
                    void* const* outs, cudaStream_t st) {
    VecPtrs<NV> io;
    for (int v = 0; v < NV; ++v) {
        io.in[v] = ins[v];
        io.out[v] = outs[v];
    }
    // 32-bit states when every state fits
    if (row->N <= 32 && col->N <= 32)
        launch_rows_st<NV, u32, kF32, kOutF32>(row, col, P, io, st);
    else
        launch_rows_st<NV, u64, kF32, kOutF32>(row, col, P, io, st);
}

template <int kCpl, bool kF32, bool kOutF32>
void launch_team_c(const qb_sector* row, const qb_sector* col, const qb_program* P, const void* in, void* out, int k,
                   cudaStream_t st) {
    bool in_smem = false;
    const std::size_t smem = smem_for(P, col, in_smem);
    const std::uint64_t warps = (row->dim + 3) / 4;
    const unsigned blocks = static_cast<unsigned>((warps * 32 + 255) / 256);
    if (row == col) {
        auto kk = walk_team<kCpl, kF32, kOutF32, true>;
        set_smem(kk, smem);
        kk<<<blocks, 256, smem, st>>>(row->view(), col->view(), P->view, in_smem, in, out, k);
    } else {
        auto kk = walk_team<kCpl, kF32, kOutF32, false>;
        set_smem(kk, smem);
        kk<<<blocks, 256, smem, st>>>(row->view(), col->view(), P->view, in_smem, in, out, k);
    }
    cuda_check(cudaGetLastError(), "walk_team launch");
}

template <bool kF32, bool kOutF32>
void launch_team(const qb_sector* row, const qb_sector* col, const qb_program* P, const void* in, void* out, int k,
                 cudaStream_t st) {
    const int cpl = (k + 7) / 8;
    if (cpl <= 1)
        launch_team_c<1, kF32, kOutF32>(row, col, P, in, out, k, st);
    else if (cpl <= 2)
        launch_team_c<2, kF32, kOutF32>(row, col, P, in, out, k, st);
    else if (cpl <= 4)
        launch_team_c<4, kF32, kOutF32>(row, col, P, in, out, k, st);
    else if (cpl <= 5)
        launch_team_c<5, kF32, kOutF32>(row, col, P, in, out, k, st);
    else if (cpl <= 8)
        launch_team_c<8, kF32, kOutF32>(row, col, P, in, out, k, st);
    else
        throw Error(QB_EUNSUPPORTED, "block matvec: at most 64 vectors");
}

void check_pair(const qb_sector* row, const qb_sector* col, const qb_program* P) {
    if (!row || !col || !P) throw Error(QB_EINVAL, "null sector or program");
    if (row->N != col->N) throw Error(QB_EINVAL, "sectors of different sizes");
}

}  // namespace

// Internal entry points shared with krylov.cu.
void launch_walk(const qb_sector* row, const qb_sector* col, const qb_program* P, const void* const* ins,
                 void* const* outs, int k, int dtype, cudaStream_t st) {
    check_pair(row, col, P);
    if (row->dim == 0 || k <= 0) return;
    int off = 0;
    while (off < k) {
        const int left = k - off;
        const int nv = left >= 8 ? 8 : left >= 4 ? 4 : left >= 2 ? 2 : 1;
        if (dtype == QB_C64) {
            if (nv == 8) launch_rows_nv<8, true>(row, col, P, ins + off, outs + off, st);
            if (nv == 4) launch_rows_nv<4, true>(row, col, P, ins + off, outs + off, st);
            if (nv == 2) launch_rows_nv<2, true>(row, col, P, ins + off, outs + off, st);
            if (nv == 1) launch_rows_nv<1, true>(row, col, P, ins + off, outs + off, st);
        } else {
            if (nv == 8) launch_rows_nv<8, false>(row, col, P, ins + off, outs + off, st);
            if (nv == 4) launch_rows_nv<4, false>(row, col, P, ins + off, outs + off, st);
            if (nv == 2) launch_rows_nv<2, false>(row, col, P, ins + off, outs + off, st);
            if (nv == 1) launch_rows_nv<1, false>(row, col, P, ins + off, outs + off, st);
        }
        off += nv;
    }
}

// One vector: x stored as dtype_in, y as dtype_out (the FP32-storage recurrence keeps its scratch in FP64).
void launch_walk_mixed(const qb_sector* row, const qb_sector* col, const qb_program* P, const void* in, void* out,
                       int dtype_in, int dtype_out, cudaStream_t st) {
    check_pair(row, col, P);
    if (row->dim == 0) return;
    const void* ins[1] = {in};
    void* outs[1] = {out};
    if (dtype_in == QB_C64 && dtype_out == QB_C128)
        launch_rows_nv<1, true, false>(row, col, P, ins, outs, st);
    else if (dtype_in == QB_C128 && dtype_out == QB_C64)
        launch_rows_nv<1, false, true>(row, col, P, ins, outs, st);
    else if (dtype_in == QB_C64)
        launch_rows_nv<1, true, true>(row, col, P, ins, outs, st);
    else
        launch_rows_nv<1, false, false>(row, col, P, ins, outs, st);
}

void launch_block(const qb_sector* row, const qb_sector* col, const qb_program* P, const void* in, void* out, int k,
                  int dtype, cudaStream_t st) {
    check_pair(row, col, P);
    if (row->dim == 0 || k <= 0) return;
    if (dtype == QB_C64)
        launch_team<true, true>(row, col, P, in, out, k, st);
    else
        launch_team<false, false>(row, col, P, in, out, k, st);
}

// k vectors interleaved by row, x stored as dtype_in, y as dtype_out.
void launch_block_mixed(const qb_sector* row, const qb_sector* col, const qb_program* P, const void* in, void* out,
                        int k, int dtype_in, int dtype_out, cudaStream_t st) {
    check_pair(row, col, P);
    if (row->dim == 0 || k <= 0) return;
    if (dtype_in == QB_C64 && dtype_out == QB_C128)
        launch_team<true, false>(row, col, P, in, out, k, st);
    else if (dtype_in == QB_C64)
        launch_team<true, true>(row, col, P, in, out, k, st);
    else if (dtype_out == QB_C64)
        launch_team<false, true>(row, col, P, in, out, k, st);
    else
        launch_team<false, false>(row, col, P, in, out, k, st);
}

}  // namespace qb

extern "C" {

int qb_program_create(const qb_program_desc* d, qb_program** out) {
    return qb::guarded([&] {
        using namespace qb;
        if (!d || !out) throw Error(QB_EINVAL, "null program description");
        if (!d->group_flip || !d->group_setbits || !d->group_vbegin || !d->vsub_val || !d->vsub_tbegin ||
            (d->n_terms && (!d->term_sign || !d->term_coeff)))
            throw Error(QB_EINVAL, "program arrays missing");
        if (d->group_vbegin[0] != 0 || d->group_vbegin[d->n_groups] != d->n_vsub || d->vsub_tbegin[0] != 0 ||
            d->vsub_tbegin[d->n_vsub] != d->n_terms)
            throw Error(QB_EINVAL, "program offsets inconsistent");
        for (uint32_t g = 0; g < d->n_groups; ++g) {
            if (d->group_vbegin[g + 1] <= d->group_vbegin[g]) throw Error(QB_EINVAL, "empty program group");
            if (g && d->group_flip[g] <= d->group_flip[g - 1]) throw Error(QB_EINVAL, "groups must ascend by flip");
            for (uint32_t v = d->group_vbegin[g] + 1; v < d->group_vbegin[g + 1]; ++v)
                if (d->vsub_val[v] <= d->vsub_val[v - 1]) throw Error(QB_EINVAL, "subgroups must ascend by value");
        }
        for (uint32_t v = 0; v < d->n_vsub; ++v)
            if (d->vsub_tbegin[v + 1] < d->vsub_tbegin[v]) throw Error(QB_EINVAL, "term offsets must ascend");
        auto p = std::make_unique<qb_program>();
        // one blob, each array 16-byte aligned
        std::vector<std::size_t> sizes = {d->n_groups * 8ull,        d->n_groups * 4ull, (d->n_groups + 1) * 4ull,
                                          d->n_vsub * 8ull,          (d->n_vsub + 1) * 4ull, d->n_terms * 8ull,
                                          d->n_terms * 16ull};
        std::vector<std::size_t> offs;
        std::size_t total = 0;
        for (auto s : sizes) {
            offs.push_back(total);
            total += (s + 15) & ~std::size_t(15);
        }
        std::vector<unsigned char> host(std::max<std::size_t>(total, 16), 0);
        std::memcpy(host.data() + offs[0], d->group_flip, sizes[0]);
        std::memcpy(host.data() + offs[1], d->group_setbits, sizes[1]);
        std::memcpy(host.data() + offs[2], d->group_vbegin, sizes[2]);
        std::memcpy(host.data() + offs[3], d->vsub_val, sizes[3]);
        std::memcpy(host.data() + offs[4], d->vsub_tbegin, sizes[4]);
        if (d->n_terms) {
            std::memcpy(host.data() + offs[5], d->term_sign, sizes[5]);
            std::memcpy(host.data() + offs[6], d->term_coeff, sizes[6]);
        }
        p->blob.upload(host);
        unsigned char* b = p->blob.p;
        DProgram& v = p->view;
        v.n_groups = d->n_groups;
        v.n_vsub = d->n_vsub;
        v.n_terms = d->n_terms;
        v.group_flip = reinterpret_cast<const u64*>(b + offs[0]);
        v.group_setbits = reinterpret_cast<const int*>(b + offs[1]);
        v.group_vbegin = reinterpret_cast<const u32*>(b + offs[2]);
        v.vsub_val = reinterpret_cast<const u64*>(b + offs[3]);
        v.vsub_tbegin = reinterpret_cast<const u32*>(b + offs[4]);
        v.term_sign = reinterpret_cast<const u64*>(b + offs[5]);
        v.term_coeff = reinterpret_cast<const double2*>(b + offs[6]);
        v.smem_bytes = total;
        for (uint32_t k = 0; k < d->n_terms; ++k) p->norm_bound += std::hypot(d->term_coeff[2 * k], d->term_coeff[2 * k + 1]);
        *out = p.release();
    });
}

int qb_program_destroy(qb_program* p) {
    return qb::guarded([&] { delete p; });
}

int qb_matvec(const qb_sector* row, const qb_sector* col, const qb_program* prog, const void* const* ins,
              void* const* outs, int k, int dtype, void* stream) {
    return qb::guarded([&] {
        if (dtype != QB_C128 && dtype != QB_C64) throw qb::Error(QB_EINVAL, "dtype must be QB_C128 or QB_C64");
        if (k < 0 || (k > 0 && (!ins || !outs))) throw qb::Error(QB_EINVAL, "vector pointers missing");
        qb::launch_walk(row, col, prog, ins, outs, k, dtype, static_cast<cudaStream_t>(stream));
    });
}

int qb_matvec_block(const qb_sector* row, const qb_sector* col, const qb_program* prog, const void* in, void* out,
                    int k, int dtype, void* stream) {
    return qb::guarded([&] {
        if (dtype != QB_C128 && dtype != QB_C64) throw qb::Error(QB_EINVAL, "dtype must be QB_C128 or QB_C64");
        if (k < 1 || k > 64) throw qb::Error(QB_EINVAL, "block width must be in [1, 64]");
        qb::launch_block(row, col, prog, in, out, k, dtype, static_cast<cudaStream_t>(stream));
    });
}

int qb_matvec_host(const qb_sector* row, const qb_sector* col, const qb_program* prog, const double* in_host,
                   double* out_host) {
    return qb::guarded([&] {
        using namespace qb;
        check_pair(row, col, prog);
        DevBuf<double2> x, y(row->dim);
        x.upload(reinterpret_cast<const double2*>(in_host), col->dim);
        const void* ins[1] = {x.p};
        void* outs[1] = {y.p};
        launch_walk(row, col, prog, ins, outs, 1, QB_C128, nullptr);
        cuda_check(cudaMemcpy(out_host, y.p, row->dim * 16, cudaMemcpyDeviceToHost), "download");
    });
}

}  // extern "C"
