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
// Three kernels, whose launch shapes the tuner (tune.cu) picks per size class; every shape gives the same y
// bit for bit:
//   walk_rows   one thread per row, up to 8 separate vectors (the reference's multi-apply contract:
//               every output equals the single apply bit for bit). The row program and the key
//               table are staged in shared memory; a warp's lanes advance in step over their own
//               acting groups.
//   walk_warp   the same with a warp's 32 rows compacted: the acting (row, group) pairs are laid out
//               row-major and canonicalised 32 at a time; each row adds its products in order.
//   walk_team   a team of 4, 8, 16 or 32 lanes owns a row: the lanes test that many groups at once,
//               canonicalise the acting targets in parallel, then every lane accumulates its slice of
//               the k columns from each target in group order -- the block matvec of the sampled methods
//               (k vectors interleaved by row), and for one vector on a small sector, where one thread
//               per row leaves most of the GPU idle.
// =============================================================================
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>

#include "qb_walk.cuh"

namespace qb {

namespace {

template <int NV> struct VecPtrs {
    const void* in[NV];
    void* out[NV];
};

// One or two vectors: six blocks per SM for 32-bit states (40 registers), five for 64-bit states (48 registers);
// the walk is bound by instruction issue and by the latency of its dependent loads, and the extra warps hide it.
// A sweep of 4, 5, 6 and 8 blocks per SM (CUDA events, one FP32 vector, copies of this kernel): chain-32 2.94 /
// 2.58 / 2.63 / 2.69 ms, 6x5 9.45 / 8.35 / 8.98 / 9.79 ms, 6x6 1,332 / 1,204 / 1,298 / 1,534 ms; in the library
// itself five blocks measured no faster than six on chain-32 (2.64 ms at six in four bench runs), so 32-bit states
// keep six. More vectors keep four.
// One thread per row. The row's groups are tested 32 at a time by every lane together (a converged
// pass that builds the bitmask of the groups acting on the lane's row); the lanes then walk their own
// acting groups in ascending order -- the diagonal first -- canonicalising one target each per step.
template <int NV, class ST, bool kInF32, bool kOutF32, bool kSame>
__global__ void __launch_bounds__(256, (NV <= 2 ? (sizeof(ST) == 4 ? 6 : 5) : 4)) walk_rows(DSector row, DSector col, DProgram P, bool prog_in_smem,
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
        u64 offs = 0;   // the acting subgroup of each group, as an offset from its first (programs with vsub4)
        if (live)
            for (u32 g = g0; g < gend; ++g) {
                const int vi = acting_subgroup<ST>(sp.P, s, g);
                if (vi >= 0) {
                    mask |= 1u << (g - g0);
                    offs |= static_cast<u64>(vi - static_cast<int>(sp.P.group_vbegin[g])) << (2 * (g - g0));
                }
            }
        while (__any_sync(0xffffffffu, mask != 0)) {
            if (mask == 0) continue;
            const u32 gi = static_cast<u32>(__ffs(mask) - 1);
            const u32 g = g0 + gi;
            mask &= mask - 1;
            const int vi = sp.P.vsub4 ? static_cast<int>(sp.P.group_vbegin[g] + ((offs >> (2 * gi)) & 3u))
                                      : acting_subgroup<ST>(sp.P, s, g);
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

// Warp-compacted walk (the same y as walk_rows, bit for bit): a warp owns 32 consecutive rows. For each window
// of 32 groups every lane builds its row's acting-group mask; a warp prefix sum lays the (row, group) pairs out
// row-major, and the warp canonicalises them 32 at a time, one pair per lane, so no lane idles while another row
// still has targets. Each pair's products c x_v[j] go to shared memory; the row's lane then adds its slots in
// order -- the row's entries in group order, with walk_rows's operations.
struct WarpSlots {
    u64 state[32];
    u64 offs[32];   // each row's acting-subgroup offsets in the window (programs with vsub4)
    double w[32];
    u32 mask[32], pre[32], incl[32];
    int ok[32];
};

template <int NV, class ST, bool kInF32, bool kOutF32, bool kSame>
__global__ void __launch_bounds__(256, 4) walk_warp(DSector row, DSector col, DProgram P, bool prog_in_smem,
                                                    std::size_t stage_bytes, VecPtrs<NV> io) {
    extern __shared__ __align__(16) unsigned char smem[];
    using St = Store<kInF32>;
    using So = Store<kOutF32>;
    const SmemProgram sp = stage(P, col, smem, prog_in_smem);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    WarpSlots& W = reinterpret_cast<WarpSlots*>(smem + stage_bytes)[wid];
    double2* prod = reinterpret_cast<double2*>(smem + stage_bytes + (blockDim.x >> 5) * sizeof(WarpSlots)) +
                    static_cast<std::size_t>(wid) * 32 * NV;
    const std::uint64_t r0 = (static_cast<std::uint64_t>(blockIdx.x) * blockDim.x) + (threadIdx.x & ~31u);
    const std::uint64_t r = r0 + lane;
    const bool live = r < row.dim;
    const ST s = live ? static_cast<ST>(__ldg(row.reps + r)) : static_cast<ST>(0);
    const double w = live ? __ldg(row.inv_norms + r) : 0.0;
    W.state[lane] = static_cast<u64>(s);
    W.w[lane] = w;
    cplx acc[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) acc[v] = {0.0, 0.0};
    const u32 ng = sp.P.n_groups;
    for (u32 g0 = 0; g0 < ng; g0 += 32) {
        const u32 gend = ng < g0 + 32 ? ng : g0 + 32;
        u32 mask = 0;
        u64 offs = 0;
        if (live)
            for (u32 g = g0; g < gend; ++g) {
                const int vi = acting_subgroup<ST>(sp.P, s, g);
                if (vi >= 0) {
                    mask |= 1u << (g - g0);
                    offs |= static_cast<u64>(vi - static_cast<int>(sp.P.group_vbegin[g])) << (2 * (g - g0));
                }
            }
        const u32 cnt = static_cast<u32>(__popc(mask));
        u32 incl = cnt;   // inclusive prefix over the lanes
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const u32 y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        const u32 pre = incl - cnt;
        const u32 total = __shfl_sync(0xffffffffu, incl, 31);
        W.mask[lane] = mask;
        W.offs[lane] = offs;
        W.pre[lane] = pre;
        W.incl[lane] = incl;
        __syncwarp();
        for (u32 b = 0; b < total; b += 32) {
            const u32 q = b + lane;
            int ok = 0;
            if (q < total) {
                // the owner: the number of rows whose pairs all come before q
                int o = 0;
#pragma unroll
                for (int step = 16; step > 0; step >>= 1)
                    if (W.incl[o + step - 1] <= q) o += step;
                const ST so = static_cast<ST>(W.state[o]);
                const u32 g = g0 + __fns(W.mask[o], 0, static_cast<int>(q - W.pre[o]) + 1);
                const int vi = sp.P.vsub4
                                   ? static_cast<int>(sp.P.group_vbegin[g] + ((W.offs[o] >> (2 * (g - g0))) & 3u))
                                   : acting_subgroup<ST>(sp.P, so, g);
                const cplx h = subgroup_value<ST>(sp.P, so, vi);
                const ST t = so ^ static_cast<ST>(sp.P.group_flip[g]);
                long long j;
                cplx c;
                if (entry<kSame, ST>(col, sp.T, so, static_cast<long long>(r0 + o), W.w[o], t, h, j, c)) {
                    ok = 1;
#pragma unroll
                    for (int v = 0; v < NV; ++v) {
                        const cplx p = cmul(c, St::load(static_cast<const typename St::T*>(io.in[v]),
                                                        static_cast<std::size_t>(j)));
                        prod[lane * NV + v] = make_double2(p.re, p.im);
                    }
                }
            }
            W.ok[lane] = ok;
            __syncwarp();
            const u32 lo = pre > b ? pre : b, hi = incl < b + 32 ? incl : b + 32;
            for (u32 p = lo; p < hi; ++p) {
                if (!W.ok[p - b]) continue;
#pragma unroll
                for (int v = 0; v < NV; ++v) {
                    const double2 d = prod[(p - b) * NV + v];
                    acc[v] = cadd(acc[v], {d.x, d.y});
                }
            }
            __syncwarp();
        }
    }
    if (!live) return;
#pragma unroll
    for (int v = 0; v < NV; ++v) So::store(static_cast<typename So::T*>(io.out[v]), r, acc[v]);
}

// Team kernel: kTeam lanes per row (4, 8, 16 or 32), kCpl columns per lane (k <= kTeam kCpl vectors). Every column
// adds its row's entries in group order whatever kTeam is, so the team size changes only the time.
template <int kTeam, int kCpl, bool kF32, bool kOutF32, bool kSame>
__global__ void __launch_bounds__(256) walk_team(DSector row, DSector col, DProgram P, bool prog_in_smem,
                                                 const void* in_v, void* out_v, int k) {
    extern __shared__ __align__(16) unsigned char smem[];
    using St = Store<kF32>;
    using So = Store<kOutF32>;
    using T = typename St::T;
    const T* in = static_cast<const T*>(in_v);
    typename So::T* out = static_cast<typename So::T*>(out_v);
    const SmemProgram sp = stage(P, col, smem, prog_in_smem);
    const int lane = threadIdx.x & 31;
    const int team = lane / kTeam, tl = lane % kTeam;
    const unsigned team_mask = kTeam == 32 ? 0xffffffffu : ((1u << kTeam) - 1u) << (team * kTeam);
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

template <int kTeam, int kCpl, bool kF32, bool kOutF32>
void launch_team_c(const qb_sector* row, const qb_sector* col, const qb_program* P, const void* in, void* out, int k,
                   cudaStream_t st) {
    bool in_smem = false;
    const std::size_t smem = smem_for(P, col, in_smem);
    constexpr int kRowsPerWarp = 32 / kTeam;
    const std::uint64_t warps = (row->dim + kRowsPerWarp - 1) / kRowsPerWarp;
    const unsigned blocks = static_cast<unsigned>((warps * 32 + 255) / 256);
    if (row == col) {
        auto kk = walk_team<kTeam, kCpl, kF32, kOutF32, true>;
        set_smem(kk, smem);
        kk<<<blocks, 256, smem, st>>>(row->view(), col->view(), P->view, in_smem, in, out, k);
    } else {
        auto kk = walk_team<kTeam, kCpl, kF32, kOutF32, false>;
        set_smem(kk, smem);
        kk<<<blocks, 256, smem, st>>>(row->view(), col->view(), P->view, in_smem, in, out, k);
    }
    cuda_check(cudaGetLastError(), "walk_team launch");
}

template <int kTeam, bool kF32, bool kOutF32>
void launch_team_t(const qb_sector* row, const qb_sector* col, const qb_program* P, const void* in, void* out, int k,
                   cudaStream_t st) {
    const int cpl = (k + kTeam - 1) / kTeam;
    if (cpl <= 1)
        launch_team_c<kTeam, 1, kF32, kOutF32>(row, col, P, in, out, k, st);
    else if (cpl <= 2)
        launch_team_c<kTeam, 2, kF32, kOutF32>(row, col, P, in, out, k, st);
    else if (cpl <= 4)
        launch_team_c<kTeam, 4, kF32, kOutF32>(row, col, P, in, out, k, st);
    else if (cpl <= 5)
        launch_team_c<kTeam, 5, kF32, kOutF32>(row, col, P, in, out, k, st);
    else if (cpl <= 8)
        launch_team_c<kTeam, 8, kF32, kOutF32>(row, col, P, in, out, k, st);
    else
        throw Error(QB_EUNSUPPORTED, "block matvec: at most 64 vectors");
}

// The calling thread's last shape choices by launch identity (the sectors, the program, a tag of the vectors),
// so that a step does not rebuild its size-class key. An entry made under another tuner generation is ignored;
// one left by a destroyed object whose address came back can only cost time, as every shape gives the same y.
struct ShapeMemo {
    struct Entry {
        const void *row = nullptr, *col = nullptr, *prog = nullptr;
        int tag = -1, shape = 0;
        unsigned gen = 0;
    };
    Entry e[8];
    int next = 0;
    int find(const void* r, const void* c, const void* p, int tag, unsigned gen) const {
        for (const auto& x : e)
            if (x.row == r && x.col == c && x.prog == p && x.tag == tag && x.gen == gen) return x.shape;
        return -1;
    }
    void put(const void* r, const void* c, const void* p, int tag, unsigned gen, int shape) {
        e[next] = Entry{r, c, p, tag, shape, gen};
        next = (next + 1) % 8;
    }
};
thread_local ShapeMemo t_memo;

// The size classes a launch shape is tuned for: the sector's group and lookup, the program's groups, the row
// count (by powers of two) and the vectors' number and types.
std::string walk_key(const qb_sector* row, const qb_sector* col, const qb_program* P, int nv, int st_bits, int in32,
                     int out32) {
    const DSector c = col->view();
    int lg = 0;
    while ((1ULL << lg) < row->dim) ++lg;
    return "N" + std::to_string(c.N) + ".G" + std::to_string(c.G) + ".gk" + std::to_string(c.gkind) + ".slc" +
           std::to_string(c.slc.on ? 1 : 0) + ".lk" + std::to_string(c.lookup) + ".ng" +
           std::to_string(P->view.n_groups) + ".d" + std::to_string(lg) + ".nv" + std::to_string(nv) + ".st" +
           std::to_string(st_bits) + "." + std::to_string(in32) + std::to_string(out32) +
           (row == col ? ".same" : ".cross");
}

template <int NV, class ST, bool kF32, bool kOutF32, bool kSame>
void launch_rows_shape(int shape, const qb_sector* row, const qb_sector* col, const qb_program* P,
                       const VecPtrs<NV>& io, cudaStream_t st) {
    bool in_smem = false;
    const std::size_t stage = (smem_for(P, col, in_smem) + 15) & ~std::size_t(15);
    const unsigned blocks = static_cast<unsigned>((row->dim + 255) / 256);
    if (shape == 0) {
        auto k = walk_rows<NV, ST, kF32, kOutF32, kSame>;
        set_smem(k, stage);
        k<<<blocks, 256, stage, st>>>(row->view(), col->view(), P->view, in_smem, io);
    } else {
        auto k = walk_warp<NV, ST, kF32, kOutF32, kSame>;
        const std::size_t smem = stage + 8 * (sizeof(WarpSlots) + 32 * NV * sizeof(double2));
        set_smem(k, smem);
        k<<<blocks, 256, smem, st>>>(row->view(), col->view(), P->view, in_smem, stage, io);
    }
    cuda_check(cudaGetLastError(), "walk launch");
}

// The row walk over NV vectors, as the tuner picks: one thread per state (walk_rows), a warp's states compacted
// (walk_warp), or -- one vector -- a team of 8, 16, 32 or 4 lanes per state (walk_team at k = 1). All give the
// same y bit for bit: each row adds c x_j in group order with the same operations.
template <int NV, class ST, bool kF32, bool kOutF32>
void launch_rows_st(const qb_sector* row, const qb_sector* col, const qb_program* P, const VecPtrs<NV>& io,
                    cudaStream_t st) {
    auto run = [&](int shape) {
        if (shape >= 2) {
            const void* in = io.in[0];
            void* out = io.out[0];
            if (shape == 2)
                launch_team_t<8, kF32, kOutF32>(row, col, P, in, out, 1, st);
            else if (shape == 3)
                launch_team_t<16, kF32, kOutF32>(row, col, P, in, out, 1, st);
            else if (shape == 4)
                launch_team_t<32, kF32, kOutF32>(row, col, P, in, out, 1, st);
            else
                launch_team_t<4, kF32, kOutF32>(row, col, P, in, out, 1, st);
        } else if (row == col) {
            launch_rows_shape<NV, ST, kF32, kOutF32, true>(shape, row, col, P, io, st);
        } else {
            launch_rows_shape<NV, ST, kF32, kOutF32, false>(shape, row, col, P, io, st);
        }
    };
    // teams of lanes per state fill the GPU on small sectors; from 2^20 rows one thread per row already does (on
    // chain-32 and 6x5, 4.7 M and 5.2 M rows, every team shape was 2-6x slower), so the tuner does not time them
    const int shapes = NV == 1 && row->dim < (1ULL << 20) ? 6 : 2;
    const int tag = (NV << 4) | (static_cast<int>(sizeof(ST)) << 1) | (kF32 ? 1 : 0) | (kOutF32 ? 256 : 0);
    const unsigned gen = tune_generation();
    int shape = t_memo.find(row, col, P, tag, gen);
    if (shape < 0) {
        shape = tune_choose("walk", walk_key(row, col, P, NV, sizeof(ST) * 8, kF32, kOutF32), shapes, 0, st, run);
        cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
        cudaStreamIsCapturing(st, &cap);
        if (cap == cudaStreamCaptureStatusNone) t_memo.put(row, col, P, tag, gen, shape);
    }
    run(shape);
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

// The block walk of k interleaved vectors with 8, 16, 32 or (k <= 32) 4 lanes per state, as the tuner picks (the
// same y bit for bit).
template <bool kF32, bool kOutF32>
void launch_team(const qb_sector* row, const qb_sector* col, const qb_program* P, const void* in, void* out, int k,
                 cudaStream_t st) {
    if (k > 64) throw Error(QB_EUNSUPPORTED, "block matvec: at most 64 vectors");
    auto run = [&](int shape) {
        if (shape == 0)
            launch_team_t<8, kF32, kOutF32>(row, col, P, in, out, k, st);
        else if (shape == 1)
            launch_team_t<16, kF32, kOutF32>(row, col, P, in, out, k, st);
        else if (shape == 2)
            launch_team_t<32, kF32, kOutF32>(row, col, P, in, out, k, st);
        else
            launch_team_t<4, kF32, kOutF32>(row, col, P, in, out, k, st);
    };
    const int shapes = k <= 32 ? 4 : 3;
    const int tag = 512 | (k << 10) | (kF32 ? 1 : 0) | (kOutF32 ? 2 : 0);
    const unsigned gen = tune_generation();
    int shape = t_memo.find(row, col, P, tag, gen);
    if (shape < 0) {
        shape = tune_choose("walk_team", walk_key(row, col, P, k, 64, kF32, kOutF32), shapes, 0, st, run);
        cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
        cudaStreamIsCapturing(st, &cap);
        if (cap == cudaStreamCaptureStatusNone) t_memo.put(row, col, P, tag, gen, shape);
    }
    run(shape);
}

void check_pair(const qb_sector* row, const qb_sector* col, const qb_program* P) {
    if (!row || !col || !P) throw Error(QB_EINVAL, "null sector or program");
    if (row->N != col->N) throw Error(QB_EINVAL, "sectors of different sizes");
}

}  // namespace

// Internal entry points shared with krylov.cu.
// The lane of (row, col, P): the attached reduced CSR when it serves this sector pair.
const qb_csr* csr_lane(const qb_sector* row, const qb_sector* col, const qb_program* P) {
    return (P->csr && P->csr->row == row && P->csr->col == col) ? P->csr : nullptr;
}

void launch_walk(const qb_sector* row, const qb_sector* col, const qb_program* P, const void* const* ins,
                 void* const* outs, int k, int dtype, cudaStream_t st) {
    check_pair(row, col, P);
    if (row->dim == 0 || k <= 0) return;
    if (const qb_csr* A = csr_lane(row, col, P)) {
        for (int v = 0; v < k; ++v) csr_spmv(A, ins[v], outs[v], 1, dtype, dtype, st);
        return;
    }
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
    if (const qb_csr* A = csr_lane(row, col, P)) {
        csr_spmv(A, in, out, 1, dtype_in, dtype_out, st);
        return;
    }
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
    if (const qb_csr* A = csr_lane(row, col, P)) {
        csr_spmv(A, in, out, k, dtype, dtype, st);
        return;
    }
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
    if (const qb_csr* A = csr_lane(row, col, P)) {
        csr_spmv(A, in, out, k, dtype_in, dtype_out, st);
        return;
    }
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
        v.vsub4 = 1;
        for (uint32_t g = 0; g < d->n_groups; ++g)
            if (d->group_vbegin[g + 1] - d->group_vbegin[g] > 4) v.vsub4 = 0;
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
