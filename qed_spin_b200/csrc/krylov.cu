// =============================================================================
// krylov.cu -- the Lanczos / FTLM / continued-fraction recurrences, device-resident.
//
// The recurrence of the reference's lanczos_kernel (include/ed/krylov/lanczos.h:266-576) with its
// vectors in HBM and every scalar in device memory: per step one matvec and three fused passes,
//   rec_alpha  w -= beta_j v_prev and the partial sums of <v_j, w>      -> alpha_j
//   rec_beta   w -= alpha_j v_j, the partial sums of ||w||^2 and of the
//              local reorthogonalisation overlap <v_j, w>               -> beta_{j+1}
//   rec_next   v_{j+1} = (w - o v_j) / beta_{j+1}   (o: the overlap when it passes sqrt(eps))
// Reductions are deterministic: a fixed grid, a fixed per-block tree, and the last block to finish
// summing the block partials in index order. alpha / beta / overlaps are FP64; the Lanczos vectors
// are stored in FP64 (QB_C128) or FP32 (QB_C64) while the matvec output w stays FP64.
//
// The host never waits on a scalar inside a step: it launches step j, then reads step j-1's alpha /
// beta (a 16-byte copy behind an event) and runs the convergence test while the device computes.
//
// Drivers:
//   qb_lanczos      the plain kernel (alpha, beta to the host).
//   qb_eigs_lowest  the k = 1 block lane (src/engine/block_solve.cpp:335-398, 528-598): start
//                   staged_seed(0x51ED0B70), Paige-gated ghost-aware lowest level, and for FP32 storage
//                   an FP64 restarted-Lanczos refinement of the lowest Ritz pair.
//   qb_ftlm         one block's FTLM (include/ed/thermal/ftlm.h:165-480): all samples as one block
//                   matvec, per-sample recurrences in lock step, Ritz weights and moments.
//   qb_cf           the T = 0 continued fraction (include/ed/dynamics/cf.h:39-160).
// =============================================================================
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstring>
#include <limits>
#include <math_constants.h>
#include <memory>
#include <mutex>
#include <numeric>
#include <random>
#include <string>
#include <thread>
#include <type_traits>
#include <vector>

#include "qb_internal.cuh"

#include "qb_krylov.cuh"
#include "qb_walk.cuh"

#ifndef QB_FMV_BLOCKS
#define QB_FMV_BLOCKS 5
#endif

namespace qb {
namespace {

// ---- FTLM: sample tables, the block recurrence of one sector's samples, the curves ----
// The sample vectors of a call (sample_engine + gaussian_vector, include/ed/thermal/sample_seed.h:37-89), in one of
// two modes:
//   QB_SEED_SHARED     sample s of every block is the first n_b draws of sample_engine(seed, s). One table of k
//                      streams, as long as the largest block, holds every block's samples as prefixes; a block
//                      normalises its prefix. One draw of the largest block serves the whole call.
//   QB_SEED_PER_BLOCK  the reference thermal driver's streams (src/engine/thermal.cpp:470-471): before each sampled
//                      block, in the order the blocks are given, the seed takes one step of the 64-bit LCG
//                      seed * 6364136223846793005 + 1442695040888963407, and block b's sample s is the first n_b draws
//                      of sample_engine(seed_b, s). Every block draws a table of its own.
// The tables are drawn on host threads with the reference's own generator and distribution.
std::vector<std::complex<double>> sample_table(std::uint64_t seed, int k, std::uint64_t len) {
    std::vector<std::complex<double>> G(static_cast<std::size_t>(k) * len);
    auto draw = [&](int s) {
        std::mt19937 gen = sample_engine(seed, static_cast<std::uint64_t>(s));
        std::normal_distribution<double> nd(0.0, 1.0);
        std::complex<double>* g = G.data() + static_cast<std::size_t>(s) * len;
        for (std::uint64_t i = 0; i < len; ++i) {
            const double im = nd(gen);   // the imaginary part is drawn first (see gaussian_fill)
            const double re = nd(gen);
            g[i] = std::complex<double>(re, im);
        }
    };
    const int nt = std::max(1, std::min<int>(k, static_cast<int>(std::thread::hardware_concurrency())));
    std::vector<std::thread> pool;
    std::atomic<int> next{0};
    for (int t = 0; t < nt; ++t)
        pool.emplace_back([&] {
            for (int s = next++; s < k; s = next++) draw(s);
        });
    for (auto& t : pool) t.join();
    return G;
}

// Block b's samples under QB_SEED_PER_BLOCK: k streams of dims[b] draws each at G[off[b] + s * dims[b] + i].
std::vector<std::complex<double>> sample_tables_per_block(std::uint64_t seed, int k, const std::vector<std::uint64_t>& dims,
                                                          std::vector<std::size_t>& off) {
    const std::size_t nb = dims.size();
    off.assign(nb, 0);
    std::vector<std::uint64_t> seeds(nb);
    std::size_t tot = 0;
    for (std::size_t b = 0; b < nb; ++b) {
        seed = seed * 6364136223846793005ULL + 1442695040888963407ULL;
        seeds[b] = seed;
        off[b] = tot;
        tot += static_cast<std::size_t>(k) * dims[b];
    }
    std::vector<std::complex<double>> G(tot);
    const std::size_t items = nb * static_cast<std::size_t>(k);
    auto draw = [&](std::size_t it) {
        const std::size_t b = it / k;
        const int s = static_cast<int>(it % k);
        std::mt19937 gen = sample_engine(seeds[b], static_cast<std::uint64_t>(s));
        std::normal_distribution<double> nd(0.0, 1.0);
        std::complex<double>* g = G.data() + off[b] + static_cast<std::size_t>(s) * dims[b];
        for (std::uint64_t i = 0; i < dims[b]; ++i) {
            const double im = nd(gen);   // the imaginary part is drawn first (see gaussian_fill)
            const double re = nd(gen);
            g[i] = std::complex<double>(re, im);
        }
    };
    const int nt = static_cast<int>(std::max<std::size_t>(
        1, std::min<std::size_t>(items, std::max(1u, std::thread::hardware_concurrency()))));
    std::vector<std::thread> pool;
    std::atomic<std::size_t> next{0};
    for (int t = 0; t < nt; ++t)
        pool.emplace_back([&] {
            for (std::size_t it = next++; it < items; it = next++) draw(it);
        });
    for (auto& t : pool) t.join();
    return G;
}

// One CTA per sample: 1 / ||G[s][0, n)|| by a fixed-order tree sum (the reference normalises with dznrm2).
__global__ void k_sample_norms(std::uint64_t n, const double2* G, std::uint64_t ld, double* inv) {
    __shared__ double sm[32];
    const double2* g = G + static_cast<std::size_t>(blockIdx.x) * ld;
    double v[1] = {0.0};
    for (std::uint64_t i = threadIdx.x; i < n; i += blockDim.x) v[0] += g[i].x * g[i].x + g[i].y * g[i].y;
    block_reduce<1>(v, sm);
    if (threadIdx.x == 0) inv[blockIdx.x] = v[0] > 0.0 ? 1.0 / sqrt(v[0]) : 0.0;
}

// w[i][s] = G[s][i] / ||G[s][0, n)||, the block's samples interleaved by row.
__global__ void k_sample_start(std::uint64_t n, int k, const double2* G, std::uint64_t ld, const double* inv,
                               double2* w) {
    const std::uint64_t total = n * k;
    for (std::uint64_t t = static_cast<std::uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; t < total;
         t += static_cast<std::uint64_t>(gridDim.x) * blockDim.x) {
        const int s = static_cast<int>(t % k);
        const std::uint64_t i = t / k;
        const double2 g = G[static_cast<std::size_t>(s) * ld + i];
        w[t] = make_double2(g.x * inv[s], g.y * inv[s]);
    }
}

// ---- the fused block recurrence on a block's reduced CSR (three passes a step) ----
// Working precision: float for FP32 storage, double for FP64; products and sums with fused multiply-adds (the
// FTLM curves are compared within a tolerance, not bit for bit).
template <class T> struct Work;
template <> struct Work<float2> {
    using R = float;
    __device__ static float2 ld(const float2* p, std::size_t i) { return __ldg(p + i); }
    __device__ static void st(float2* p, std::size_t i, float x, float y) { p[i] = make_float2(x, y); }
};
template <> struct Work<double2> {
    using R = double;
    __device__ static double2 ld(const double2* p, std::size_t i) { return __ldg(p + i); }
    __device__ static void st(double2* p, std::size_t i, double x, double y) { p[i] = make_double2(x, y); }
};

// Deterministic grid-wide sums of NQ per-column quantities, in two levels: every block writes its partials; the
// last block to finish in each group of 32 blocks sums the group's partials in block order; the last group to
// finish sums the group totals in group order into tot (shared memory) and returns true, in that one block only.
// Thread t < NQ k holds its block's partial of quantity t / k, column t % k in `mine`; every thread calls.
template <int NQ>
__device__ __forceinline__ bool grid_sum2(double mine, int k, const BScal& S, double (*tot)[kMaxCols]) {
    __shared__ bool last;
    const int t = threadIdx.x, nqk = NQ * k;
    const unsigned b = blockIdx.x, g = b >> 5, ng = (gridDim.x + 31) >> 5;
    const unsigned gsize = min(32u, gridDim.x - (g << 5));
    if (t < nqk) S.partials[static_cast<std::size_t>(t) * kMaxRedBlocks + b] = mine;
    __threadfence();
    __syncthreads();
    if (t == 0) last = atomicAdd(S.group_counter + g, 1u) == gsize - 1;
    __syncthreads();
    if (!last) return false;
    __threadfence();
    if (t < nqk) {
        const double* p = S.partials + static_cast<std::size_t>(t) * kMaxRedBlocks + (g << 5);
        double s = 0.0;
        for (unsigned i = 0; i < gsize; ++i) s += __ldcg(p + i);
        S.partials2[static_cast<std::size_t>(t) * kMaxGroups + g] = s;
    }
    if (t == 0) S.group_counter[g] = 0;
    __threadfence();
    __syncthreads();
    if (t == 0) last = atomicAdd(S.counter, 1u) == ng - 1;
    __syncthreads();
    if (!last) return false;
    __threadfence();
    if (t < nqk) {
        const double* p = S.partials2 + static_cast<std::size_t>(t) * kMaxGroups;
        double s = 0.0;
        for (unsigned i = 0; i < ng; ++i) s += __ldcg(p + i);
        tot[t / k][t % k] = s;
    }
    if (t == 0) *S.counter = 0;
    __syncthreads();
    return true;
}

// The row-tile shape of the streaming passes: a block of R k threads, thread t on column t % k and row t / k of
// each R-row tile, so a block reads whole rows contiguously and every thread keeps one column.
__host__ __device__ inline int tile_rows(int k) { return k >= 256 ? 1 : 256 / k; }

// Pass 1: w = A v_j - beta_j v_{j-1} on the CSR (8 lanes per row, lane l owns columns l, l + 8, ...), and
// alpha_j = Re <v_j, w> per column: block partials in shared memory summed in row order, the block sums in
// block order by the last block.
// Blocks per SM the pass is compiled for: FP32 storage fits 48 registers without spills at five (the batched
// FTLM's recurrences: 1.70 -> 1.62 s; six spill and take 1.75 s); FP64 holds three (80 registers, as unbounded).
template <class T> struct FmvBlocks {
    static constexpr int value = 3;
};
template <> struct FmvBlocks<float2> {
    static constexpr int value = QB_FMV_BLOCKS;
};

template <class T, int CPL>
__global__ void __launch_bounds__(256, FmvBlocks<T>::value) fmv_alpha(std::uint64_t rows, int k, int j,
                                                 const unsigned long long* __restrict__ row_ptr,
                                                 const std::uint32_t* __restrict__ col,
                                                 const unsigned char* __restrict__ ids, int id_bytes,
                                                 const double2* __restrict__ vals, int n_dict, const T* __restrict__ vc,
                                                 const T* __restrict__ vp, T* __restrict__ w, BScal S) {
    using Rt = typename Work<T>::R;
    __shared__ double2 dict[256];
    __shared__ double red[kMaxCols][33];
    if (id_bytes == 1)
        for (int i = threadIdx.x; i < n_dict; i += blockDim.x) dict[i] = vals[i];
    __syncthreads();
    const int lane = threadIdx.x & 7, rg = threadIdx.x >> 3;
    Rt b[CPL];
    double ap[CPL];
#pragma unroll
    for (int c = 0; c < CPL; ++c) {
        const int cc = lane + 8 * c;
        b[c] = (j > 0 && cc < k) ? static_cast<Rt>(S.beta[static_cast<std::size_t>(j) * k + cc]) : Rt(0);
        ap[c] = 0.0;
    }
    const std::uint64_t stride = static_cast<std::uint64_t>(gridDim.x) * 32;
    for (std::uint64_t r = static_cast<std::uint64_t>(blockIdx.x) * 32 + rg; r < rows; r += stride) {
        Rt ar[CPL], ai[CPL];
#pragma unroll
        for (int c = 0; c < CPL; ++c) ar[c] = ai[c] = Rt(0);
        const std::uint64_t e1 = row_ptr[r + 1];
        for (std::uint64_t e = row_ptr[r]; e < e1; ++e) {
            const double2 v2 = id_bytes == 1 ? dict[ids[e]]
                                             : (id_bytes == 2 ? __ldg(vals + reinterpret_cast<const unsigned short*>(ids)[e])
                                                              : __ldg(vals + e));
            const Rt vr = static_cast<Rt>(v2.x), vi = static_cast<Rt>(v2.y);
            const std::size_t base = static_cast<std::size_t>(__ldg(col + e)) * k;
#pragma unroll
            for (int c = 0; c < CPL; ++c) {
                const int cc = lane + 8 * c;
                if (cc < k) {
                    const T x = Work<T>::ld(vc, base + cc);
                    ar[c] = fma(vr, x.x, fma(-vi, x.y, ar[c]));
                    ai[c] = fma(vr, x.y, fma(vi, x.x, ai[c]));
                }
            }
        }
#pragma unroll
        for (int c = 0; c < CPL; ++c) {
            const int cc = lane + 8 * c;
            if (cc >= k) continue;
            const std::size_t i = static_cast<std::size_t>(r) * k + cc;
            Rt yr = ar[c], yi = ai[c];
            if (j > 0) {
                const T p = Work<T>::ld(vp, i);
                yr = fma(-b[c], p.x, yr);
                yi = fma(-b[c], p.y, yi);
            }
            Work<T>::st(w, i, yr, yi);
            const T z = Work<T>::ld(vc, i);
            ap[c] += static_cast<double>(z.x) * yr + static_cast<double>(z.y) * yi;
        }
    }
    // the block's partial per column: the 32 row groups in order
#pragma unroll
    for (int c = 0; c < CPL; ++c) {
        const int cc = lane + 8 * c;
        if (cc < k) red[cc][rg] = ap[c];
    }
    __syncthreads();
    __shared__ bool is_last;
    if (threadIdx.x < k) {
        double s = 0.0;
        for (int g = 0; g < 32; ++g) s += red[threadIdx.x][g];
        S.partials[static_cast<std::size_t>(threadIdx.x) * kMaxRedBlocks + blockIdx.x] = s;
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) is_last = atomicAdd(S.counter, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!is_last) return;
    __threadfence();
    const int wp = threadIdx.x >> 5, ln = threadIdx.x & 31;
    for (int c = wp; c < k; c += blockDim.x >> 5) {   // one warp per column, a fixed xor-butterfly
        const double* p = S.partials + static_cast<std::size_t>(c) * kMaxRedBlocks;
        double s = 0.0;
        for (unsigned g = ln; g < gridDim.x; g += 32) s += __ldcg(p + g);
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (ln == 0) S.alpha[static_cast<std::size_t>(j) * k + c] = s;
    }
    __syncthreads();
    if (threadIdx.x == 0) *S.counter = 0;
}

// Pass 2: the norms and the local-reorthogonalisation overlaps of w - alpha_j v_j (not stored) -> beta_{j+1}.
template <class T>
__global__ void __launch_bounds__(256) fbeta(std::uint64_t n, int k, int j, const T* __restrict__ w,
                                             const T* __restrict__ vc, BScal S) {
    __shared__ double sm[3][256];
    __shared__ double tot[3][kMaxCols];
    const int R = tile_rows(k);
    const int c = threadIdx.x % k, rr = threadIdx.x / k;
    const double a = S.alpha[static_cast<std::size_t>(j) * k + c];
    double q0 = 0.0, q1 = 0.0, q2 = 0.0;
    const std::uint64_t step = static_cast<std::uint64_t>(gridDim.x) * R;
    constexpr int U = 4;   // rows in flight per thread
    std::uint64_t r = static_cast<std::uint64_t>(blockIdx.x) * R + rr;
    auto add = [&](const T y0, const T z0) {
        const double zx = z0.x, zy = z0.y;
        const double yx = y0.x - a * zx, yy = y0.y - a * zy;
        q0 += yx * yx + yy * yy;
        q1 += zx * yx + zy * yy;
        q2 += zx * yy - zy * yx;
    };
    for (; r + (U - 1) * step < n; r += U * step) {
        T y[U], z[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const std::size_t i = (r + u * step) * k + c;
            y[u] = w[i];
            z[u] = vc[i];
        }
#pragma unroll
        for (int u = 0; u < U; ++u) add(y[u], z[u]);
    }
    for (; r < n; r += step) {
        const std::size_t i = r * k + c;
        add(w[i], vc[i]);
    }
    sm[0][threadIdx.x] = q0;
    sm[1][threadIdx.x] = q1;
    sm[2][threadIdx.x] = q2;
    __syncthreads();
    // the block's partial of (quantity q, column cc): its R row slots in order
    double mine = 0.0;
    if (threadIdx.x < 3 * k) {
        const int q = threadIdx.x / k, cc = threadIdx.x % k;
        for (int s = 0; s < R; ++s) mine += sm[q][s * k + cc];
    }
    if (grid_sum2<3>(mine, k, S, tot) && threadIdx.x < k) {
        const int cc = threadIdx.x;
        double nrm2 = tot[0][cc];
        const double ore = tot[1][cc], oim = tot[2][cc];
        const bool proj = j > 0 && sqrt(ore * ore + oim * oim) > kLocalThreshold;
        if (proj) nrm2 = fmax(nrm2 - (ore * ore + oim * oim), 0.0);
        S.ovl[cc] = proj ? -ore : 0.0;
        S.ovl[kMaxCols + cc] = proj ? -oim : 0.0;
        S.beta[static_cast<std::size_t>(j + 1) * k + cc] = sqrt(nrm2);
    }
}

// Pass 3: v_{j+1} = (w - alpha_j v_j + o v_j) / beta_{j+1}; a column past its breakdown goes to zero.
template <class T>
__global__ void __launch_bounds__(256) fnext(std::uint64_t n, int k, int j, double tol, const T* __restrict__ w,
                                             const T* __restrict__ vc, T* __restrict__ vn, BScal S) {
    const int R = tile_rows(k);
    const int c = threadIdx.x % k, rr = threadIdx.x / k;
    const double b = S.beta[static_cast<std::size_t>(j + 1) * k + c];
    const double inv = b >= tol && b > 0.0 ? 1.0 / b : 0.0;
    const double a = S.alpha[static_cast<std::size_t>(j) * k + c];
    const double ore = S.ovl[c], oim = S.ovl[kMaxCols + c];
    const std::uint64_t step = static_cast<std::uint64_t>(gridDim.x) * R;
    for (std::uint64_t r = static_cast<std::uint64_t>(blockIdx.x) * R + rr; r < n; r += step) {
        const std::size_t i = r * k + c;
        const T y0 = w[i], z0 = vc[i];
        const double zx = z0.x, zy = z0.y;
        double yx = y0.x - a * zx, yy = y0.y - a * zy;
        yx += ore * zx - oim * zy;
        yy += ore * zy + oim * zx;
        Work<T>::st(vn, i, static_cast<typename Work<T>::R>(yx * inv), static_cast<typename Work<T>::R>(yy * inv));
    }
}

// One wave of fmv_alpha blocks: as many as fit on the SMs at once (at least 2 kBlockRecGrid, at most
// kMaxRedBlocks), and none past the rows.
template <class T, int C> unsigned fmv_grid(std::uint64_t n) {
    static const unsigned wave = [] {
        int dev = 0, sms = 148, per_sm = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fmv_alpha<T, C>, 256, 0);
        return static_cast<unsigned>(std::min(kMaxRedBlocks, std::max(2 * kBlockRecGrid, per_sm * sms)));
    }();
    return static_cast<unsigned>(std::max<std::uint64_t>(1, std::min<std::uint64_t>((n + 31) / 32, wave)));
}

template <class T>
void fused_step(const qb_csr* A, std::uint64_t n, int k, int j, double tol, const T* vc, const T* vp, T* w, T* vn,
                BScal S, cudaStream_t st) {
    const int cpl = (k + 7) / 8;
#define QB_FMV(C) fmv_alpha<T, C><<<fmv_grid<T, C>(n), 256, 0, st>>>(n, k, j, A->row_ptr.p, A->col_idx.p, A->ids.p, \
                                                                   A->id_bytes, A->vals.p, A->n_dict, vc, vp, w, S)
    if (cpl <= 1) QB_FMV(1);
    else if (cpl <= 2) QB_FMV(2);
    else if (cpl <= 4) QB_FMV(4);
    else if (cpl <= 5) QB_FMV(5);
    else QB_FMV(8);
#undef QB_FMV
    const int R = tile_rows(k);
    const std::uint64_t tiles = (n + R - 1) / R;
    const unsigned rb = static_cast<unsigned>(std::min<std::uint64_t>(tiles, kMaxRedBlocks));
    fbeta<T><<<rb, R * k, 0, st>>>(n, k, j, w, vc, S);
    fnext<T><<<rb, R * k, 0, st>>>(n, k, j, tol, w, vc, vn, S);
    cuda_check(cudaGetLastError(), "fused ftlm step");
}

// The scratch of one stream's block recurrences, grown to the largest block it runs.
struct BlockBufs {
    DevBuf<double2> w;
    DevBuf<unsigned char> vb[2];
    DevBuf<double> ovl, part, part2, inv;
    DevBuf<unsigned> cnt;
    void ensure(std::uint64_t n, int k, std::size_t es) {
        const std::size_t nk = static_cast<std::size_t>(n) * k;
        if (w.n < nk) w.alloc(nk);
        for (auto& b : vb)
            if (b.n < nk * es) b.alloc(nk * es);
        if (ovl.n == 0) ovl.alloc(2 * kMaxCols);
        if (part.n == 0) part.alloc(static_cast<std::size_t>(3) * kMaxCols * kMaxRedBlocks);
        if (part2.n == 0) part2.alloc(static_cast<std::size_t>(3) * kMaxCols * kMaxGroups);
        if (inv.n == 0) inv.alloc(kMaxCols);
        if (cnt.n == 0) cnt.alloc(1 + kMaxGroups);
    }
};

// The lock-step recurrence of one block's k sample columns (ftlm_kernel's per-sample Lanczos with the
// local reorthogonalisation, include/ed/thermal/ftlm.h:277-480), from the unit start columns in B.w
// (FP64, interleaved by row), cap steps; writes alpha [cap][k] and beta [cap + 1][k] to the device arrays d_alpha,
// d_beta on st. The matvec runs on the block's reduced CSR when one is given, else on the row walk.
void block_recurrence(const qb_sector* sec, const qb_program* prog, const qb_csr* csr, int k, int cap, double tol,
                      int dtype, BlockBufs& B, cudaStream_t st, double* d_alpha, double* d_beta) {
    const std::uint64_t n = sec->dim;
    const std::size_t nk = static_cast<std::size_t>(n) * k;
    const std::size_t es = dtype == QB_C64 ? 8 : 16;
    cuda_check(cudaMemsetAsync(B.vb[0].p, 0, nk * es, st), "zero");
    if (dtype == QB_C64)
        k_cast_from<float2><<<red_blocks(nk), kThreads, 0, st>>>(nk, B.w.p, reinterpret_cast<float2*>(B.vb[1].p));
    else
        cuda_check(cudaMemcpyAsync(B.vb[1].p, B.w.p, nk * 16, cudaMemcpyDeviceToDevice, st), "copy");
    cuda_check(cudaMemsetAsync(d_beta, 0, static_cast<std::size_t>(cap + 1) * k * 8, st), "zero");
    cuda_check(cudaMemsetAsync(B.cnt.p, 0, (1 + kMaxGroups) * 4, st), "zero");
    BScal S{d_alpha, d_beta, B.ovl.p, B.part.p, B.cnt.p, B.part2.p, B.cnt.p + 1};
    int cur = 1;
    const int rb = static_cast<int>(std::max<std::uint64_t>(1, std::min<std::uint64_t>((n + 7) / 8, kBlockRecGrid)));
    const std::size_t bsm = static_cast<std::size_t>(3) * kMaxCols * 8 * sizeof(double);
    for (int j = 0; j < cap; ++j) {
        void* vc = B.vb[cur].p;
        void* vp = B.vb[cur ^ 1].p;
        if (csr) {   // the fused three passes, w in the storage type (it reuses the FP64 w buffer's memory)
            if (dtype == QB_C64)
                fused_step<float2>(csr, n, k, j, tol, (const float2*)vc, (const float2*)vp, (float2*)B.w.p,
                                   (float2*)vp, S, st);
            else
                fused_step<double2>(csr, n, k, j, tol, (const double2*)vc, (const double2*)vp, B.w.p, (double2*)vp,
                                    S, st);
            cur ^= 1;
            continue;
        }
        if (k == 1)
            launch_walk_mixed(sec, sec, prog, vc, B.w.p, dtype, QB_C128, st);   // one sample: the plain walk
        else
            launch_block_mixed(sec, sec, prog, vc, B.w.p, k, dtype, QB_C128, st);
        if (dtype == QB_C64) {
            if (k <= 32) {
                brec_alpha<float2, 1><<<rb, kThreads, bsm, st>>>(n, k, j, B.w.p, (float2*)vp, (float2*)vc, S);
                brec_beta<float2, 1><<<rb, kThreads, bsm, st>>>(n, k, j, 1, B.w.p, (float2*)vc, S);
            } else {
                brec_alpha<float2, 2><<<rb, kThreads, bsm, st>>>(n, k, j, B.w.p, (float2*)vp, (float2*)vc, S);
                brec_beta<float2, 2><<<rb, kThreads, bsm, st>>>(n, k, j, 1, B.w.p, (float2*)vc, S);
            }
            brec_next<float2><<<red_blocks(nk), kThreads, 0, st>>>(n, k, j, tol, B.w.p, (float2*)vc, (float2*)vp, S);
        } else {
            if (k <= 32) {
                brec_alpha<double2, 1><<<rb, kThreads, bsm, st>>>(n, k, j, B.w.p, (double2*)vp, (double2*)vc, S);
                brec_beta<double2, 1><<<rb, kThreads, bsm, st>>>(n, k, j, 1, B.w.p, (double2*)vc, S);
            } else {
                brec_alpha<double2, 2><<<rb, kThreads, bsm, st>>>(n, k, j, B.w.p, (double2*)vp, (double2*)vc, S);
                brec_beta<double2, 2><<<rb, kThreads, bsm, st>>>(n, k, j, 1, B.w.p, (double2*)vc, S);
            }
            brec_next<double2><<<red_blocks(nk), kThreads, 0, st>>>(n, k, j, tol, B.w.p, (double2*)vc, (double2*)vp, S);
        }
        cuda_check(cudaGetLastError(), "ftlm step");
        cur ^= 1;
    }
}

// ---- the small blocks, packed: one CTA runs a whole block ----
// A block's recurrence is launch-bound when the block is small: three launches a step do little work each. The
// packed kernel hands whole blocks to persistent CTAs instead (largest first, from an atomic counter): the CTA
// walks its block once into merged rows (each row's entries sorted by column, equal columns summed in emission
// order, exact zeros dropped: the rows of the block's reduced CSR, bit for bit), forms the start columns from the
// sample table, and runs every step of the block's recurrence with block-wide fixed-order reductions. It writes
// alpha and beta where the per-block path would; only the order of the inner-product sums differs from it.
struct PackItem {
    DSector sec;
    DProgram prog;
    unsigned long long a_off, b_off;
    unsigned long long g_off, g_ld;   // the block's sample table: sample s at G + g_off + s * g_ld
    double tol;
    int cap, in_smem;
};

// A CTA's scratch: each row's merged entries (at most max_entries) and the three working columns of the block.
struct PackSlot {
    std::size_t col_off, val_off, cnt_off, vec_off, vec_bytes, bytes;
};

__host__ __device__ inline PackSlot pack_slot(std::uint64_t n_max, int max_entries, int k, std::size_t es) {
    auto al = [](std::size_t x) { return (x + 255) & ~std::size_t(255); };
    PackSlot p;
    const std::size_t ne = static_cast<std::size_t>(n_max) * max_entries;
    p.col_off = 0;
    p.val_off = al(ne * 4);
    p.cnt_off = p.val_off + al(ne * 16);
    p.vec_off = p.cnt_off + al(static_cast<std::size_t>(n_max) * 4);
    p.vec_bytes = al(static_cast<std::size_t>(n_max) * k * es);
    p.bytes = p.vec_off + 3 * p.vec_bytes;
    return p;
}

// The column sums of a block-wide quantity: red[c][rg] holds row group rg's partial of column c; thread c < k
// sums the 32 row groups in order.
__device__ __forceinline__ double pack_col_sum(double (*red)[33], int c) {
    double s = 0.0;
    for (int g = 0; g < 32; ++g) s += red[c][g];
    return s;
}

template <class T, class ST, int CPL>
__global__ void __launch_bounds__(256) ftlm_pack(const PackItem* items, int n_items, unsigned* next_item, int k,
                                                 int max_entries, const double2* G_all, double* alpha,
                                                 double* beta, unsigned char* scratch, PackSlot slot) {
    using Rt = typename Work<T>::R;
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ double red[kMaxCols][33];
    __shared__ double sm[32];
    __shared__ double s_a[kMaxCols], s_b[kMaxCols], s_o[2][kMaxCols], s_inv[kMaxCols];
    __shared__ unsigned s_item;
    unsigned char* base = scratch + static_cast<std::size_t>(blockIdx.x) * slot.bytes;
    u32* ecol = reinterpret_cast<u32*>(base + slot.col_off);
    double2* eval = reinterpret_cast<double2*>(base + slot.val_off);
    int* ecnt = reinterpret_cast<int*>(base + slot.cnt_off);
    T* vbuf[3] = {reinterpret_cast<T*>(base + slot.vec_off), reinterpret_cast<T*>(base + slot.vec_off + slot.vec_bytes),
                  reinterpret_cast<T*>(base + slot.vec_off + 2 * slot.vec_bytes)};
    const int lane = threadIdx.x & 7, rg = threadIdx.x >> 3;
    for (;;) {
        __syncthreads();   // the previous block's last reads of the shared tables are done
        if (threadIdx.x == 0) s_item = atomicAdd(next_item, 1u);
        __syncthreads();
        const unsigned it = s_item;
        if (it >= static_cast<unsigned>(n_items)) return;
        const PackItem& I = items[it];
        const std::uint64_t n = I.sec.dim;
        const int cap = I.cap;
        const double2* G = G_all + I.g_off;
        const std::uint64_t ld = I.g_ld;
        // ---- the block's merged rows ----
        const SmemProgram sp = stage(I.prog, I.sec, smem, I.in_smem != 0);
        for (std::uint64_t r = threadIdx.x; r < n; r += blockDim.x) {
            const ST s = static_cast<ST>(__ldg(I.sec.reps + r));
            const double wr = __ldg(I.sec.inv_norms + r);
            u32* rc = ecol + r * max_entries;
            double2* rv = eval + r * max_entries;
            int m = 0;
            for (u32 g = 0; g < sp.P.n_groups; ++g) {
                const int vi = acting_subgroup<ST>(sp.P, s, g);
                if (vi < 0) continue;
                const cplx h = subgroup_value<ST>(sp.P, s, vi);
                const ST t = s ^ static_cast<ST>(sp.P.group_flip[g]);
                long long j;
                cplx c;
                if (!entry<true, ST>(I.sec, sp.T, s, static_cast<long long>(r), wr, t, h, j, c)) continue;
                // insertion by column; an equal column goes after the earlier emissions
                int p = m++;
                while (p > 0 && rc[p - 1] > static_cast<u32>(j)) {
                    rc[p] = rc[p - 1];
                    rv[p] = rv[p - 1];
                    --p;
                }
                rc[p] = static_cast<u32>(j);
                rv[p] = make_double2(c.re, c.im);
            }
            int mo = 0;
            for (int p = 0; p < m;) {
                const u32 cj = rc[p];
                cplx sum{rv[p].x, rv[p].y};
                int q = p + 1;
                for (; q < m && rc[q] == cj; ++q) sum = cadd(sum, {rv[q].x, rv[q].y});
                if (sum.re != 0.0 || sum.im != 0.0) {
                    rc[mo] = cj;
                    rv[mo] = make_double2(sum.re, sum.im);
                    ++mo;
                }
                p = q;
            }
            ecnt[r] = mo;
        }
        // ---- the start columns: sample s normalised over the block's prefix (the fixed tree of k_sample_norms) ----
        for (int s = 0; s < k; ++s) {
            const double2* g = G + static_cast<std::size_t>(s) * ld;
            double v[1] = {0.0};
            for (std::uint64_t i = threadIdx.x; i < n; i += blockDim.x) v[0] += g[i].x * g[i].x + g[i].y * g[i].y;
            block_reduce<1>(v, sm);
            if (threadIdx.x == 0) s_inv[s] = v[0] > 0.0 ? 1.0 / sqrt(v[0]) : 0.0;
            __syncthreads();
        }
        T* vp = vbuf[0];
        T* vc = vbuf[1];
        T* w = vbuf[2];
        for (std::uint64_t i = threadIdx.x; i < n * k; i += blockDim.x) {
            const int s = static_cast<int>(i % k);
            const double2 g = G[static_cast<std::size_t>(s) * ld + i / k];
            Work<T>::st(vc, i, static_cast<Rt>(g.x * s_inv[s]), static_cast<Rt>(g.y * s_inv[s]));
            Work<T>::st(vp, i, Rt(0), Rt(0));
        }
        double* al = alpha + I.a_off;
        double* be = beta + I.b_off;
        if (threadIdx.x < k) {
            s_b[threadIdx.x] = 0.0;
            be[threadIdx.x] = 0.0;   // beta_0
        }
        __syncthreads();
        for (int j = 0; j < cap; ++j) {
            // pass 1: w = A v_j - beta_j v_{j-1}, and alpha_j = Re <v_j, w>
            Rt b[CPL];
            double ap[CPL];
#pragma unroll
            for (int c = 0; c < CPL; ++c) {
                const int cc = lane + 8 * c;
                b[c] = (j > 0 && cc < k) ? static_cast<Rt>(s_b[cc]) : Rt(0);
                ap[c] = 0.0;
            }
            for (std::uint64_t r = rg; r < n; r += 32) {
                Rt ar[CPL], ai[CPL];
#pragma unroll
                for (int c = 0; c < CPL; ++c) ar[c] = ai[c] = Rt(0);
                const int m = ecnt[r];
                for (int e = 0; e < m; ++e) {
                    const double2 v2 = eval[r * max_entries + e];
                    const Rt vr = static_cast<Rt>(v2.x), vi = static_cast<Rt>(v2.y);
                    const std::size_t xb = static_cast<std::size_t>(ecol[r * max_entries + e]) * k;
#pragma unroll
                    for (int c = 0; c < CPL; ++c) {
                        const int cc = lane + 8 * c;
                        if (cc < k) {
                            const T x = vc[xb + cc];
                            ar[c] = fma(vr, x.x, fma(-vi, x.y, ar[c]));
                            ai[c] = fma(vr, x.y, fma(vi, x.x, ai[c]));
                        }
                    }
                }
#pragma unroll
                for (int c = 0; c < CPL; ++c) {
                    const int cc = lane + 8 * c;
                    if (cc >= k) continue;
                    const std::size_t i = static_cast<std::size_t>(r) * k + cc;
                    Rt yr = ar[c], yi = ai[c];
                    if (j > 0) {
                        const T p = vp[i];
                        yr = fma(-b[c], p.x, yr);
                        yi = fma(-b[c], p.y, yi);
                    }
                    Work<T>::st(w, i, yr, yi);
                    const T z = vc[i];
                    ap[c] += static_cast<double>(z.x) * yr + static_cast<double>(z.y) * yi;
                }
            }
#pragma unroll
            for (int c = 0; c < CPL; ++c) {
                const int cc = lane + 8 * c;
                if (cc < k) red[cc][rg] = ap[c];
            }
            __syncthreads();
            if (threadIdx.x < k) {
                const double a = pack_col_sum(red, threadIdx.x);
                s_a[threadIdx.x] = a;
                al[static_cast<std::size_t>(j) * k + threadIdx.x] = a;
            }
            __syncthreads();
            // pass 2: the norms and local overlaps of w - alpha_j v_j -> beta_{j+1}
            double q3[3][CPL];
#pragma unroll
            for (int c = 0; c < CPL; ++c) q3[0][c] = q3[1][c] = q3[2][c] = 0.0;
            for (std::uint64_t r = rg; r < n; r += 32) {
#pragma unroll
                for (int c = 0; c < CPL; ++c) {
                    const int cc = lane + 8 * c;
                    if (cc >= k) continue;
                    const std::size_t i = static_cast<std::size_t>(r) * k + cc;
                    const T y0 = w[i], z0 = vc[i];
                    const double zx = z0.x, zy = z0.y, a = s_a[cc];
                    const double yx = y0.x - a * zx, yy = y0.y - a * zy;
                    q3[0][c] += yx * yx + yy * yy;
                    q3[1][c] += zx * yx + zy * yy;
                    q3[2][c] += zx * yy - zy * yx;
                }
            }
            double tot[3] = {0.0, 0.0, 0.0};
            for (int q = 0; q < 3; ++q) {
#pragma unroll
                for (int c = 0; c < CPL; ++c) {
                    const int cc = lane + 8 * c;
                    if (cc < k) red[cc][rg] = q3[q][c];
                }
                __syncthreads();
                if (threadIdx.x < k) tot[q] = pack_col_sum(red, threadIdx.x);
                __syncthreads();
            }
            if (threadIdx.x < k) {
                const int c = threadIdx.x;
                double nrm2 = tot[0];
                const double ore = tot[1], oim = tot[2];
                const bool proj = j > 0 && sqrt(ore * ore + oim * oim) > kLocalThreshold;
                if (proj) nrm2 = fmax(nrm2 - (ore * ore + oim * oim), 0.0);
                s_o[0][c] = proj ? -ore : 0.0;
                s_o[1][c] = proj ? -oim : 0.0;
                s_b[c] = sqrt(nrm2);
                be[static_cast<std::size_t>(j + 1) * k + c] = s_b[c];
            }
            __syncthreads();
            // pass 3: v_{j+1} = (w - alpha_j v_j + o v_j) / beta_{j+1}, into v_{j-1}'s columns
            for (std::uint64_t i = threadIdx.x; i < n * k; i += blockDim.x) {
                const int c = static_cast<int>(i % k);
                const double bb = s_b[c];
                const double inv = bb >= I.tol && bb > 0.0 ? 1.0 / bb : 0.0;
                const double a = s_a[c], ore = s_o[0][c], oim = s_o[1][c];
                const T y0 = w[i], z0 = vc[i];
                const double zx = z0.x, zy = z0.y;
                double yx = y0.x - a * zx, yy = y0.y - a * zy;
                yx += ore * zx - oim * zy;
                yy += ore * zy + oim * zx;
                Work<T>::st(vp, i, static_cast<Rt>(yx * inv), static_cast<Rt>(yy * inv));
            }
            __syncthreads();
            T* t = vp;
            vp = vc;
            vc = t;
        }
    }
}

// The largest block the packed kernel takes whole (QB_FTLM_PACK_DIM, default 4096 states; 0 turns it off).
std::uint64_t pack_max_dim() {
    const char* e = std::getenv("QB_FTLM_PACK_DIM");
    if (!e || !*e) return 4096;
    return std::strtoull(e, nullptr, 10);
}

// Shared memory of a packed block's staged tables and program, and the most the packed kernel accepts.
constexpr std::size_t kPackSmemMax = 160 * 1024;
constexpr int kPackMaxEntries = 256;

// Launches ftlm_pack over the blocks `set` (largest first) on st; the scratch and item buffers are the caller's
// and must outlive the kernel.
template <class ST>
void launch_pack(const std::vector<int>& set, const qb_sector* const* secs, const qb_program* const* progs, int k,
                 int dtype, const std::vector<std::size_t>& a_off, const std::vector<std::size_t>& b_off,
                 const std::vector<int>& caps, const std::vector<double>& tol, const double2* G,
                 const std::vector<std::size_t>& g_off, const std::vector<std::uint64_t>& g_ld,
                 double* alpha, double* beta, DevBuf<PackItem>& d_items, DevBuf<unsigned>& counter,
                 DevBuf<unsigned char>& scratch, cudaStream_t st) {
    if (set.empty()) return;
    std::vector<PackItem> items(set.size());
    std::uint64_t n_max = 1;
    int max_entries = 1;
    std::size_t smem = 0;
    for (std::size_t i = 0; i < set.size(); ++i) {
        const int b = set[i];
        bool in_smem = false;
        smem = std::max(smem, smem_for(progs[b], secs[b], in_smem));
        items[i] = PackItem{secs[b]->view(), progs[b]->view, a_off[b], b_off[b], g_off[b], g_ld[b], tol[b], caps[b],
                            in_smem ? 1 : 0};
        n_max = std::max(n_max, secs[b]->dim);
        max_entries = std::max(max_entries, static_cast<int>(progs[b]->view.n_groups));
    }
    const std::size_t es = dtype == QB_C64 ? 8 : 16;
    const PackSlot slot = pack_slot(n_max, max_entries, k, es);
    const int cpl = (k + 7) / 8;
    auto go = [&](auto kernel) {
        set_smem(kernel, smem);
        int dev = 0, sms = 148, per_sm = 1;
        cuda_check(cudaGetDevice(&dev), "device");
        cuda_check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "SM count");
        cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, 256, smem), "occupancy");
        // at most two blocks per SM, and at most 2 GB of scratch in all (each block's results are its own,
        // whatever the grid)
        const std::size_t by_bytes = std::max<std::size_t>(1, (std::size_t(2) << 30) / slot.bytes);
        const int grid = static_cast<int>(std::min({set.size(), static_cast<std::size_t>(sms) *
                                                                    std::max(1, std::min(per_sm, 2)), by_bytes}));
        d_items.alloc(items.size());
        counter.alloc(1);
        scratch.alloc(slot.bytes * grid);
        cuda_check(cudaMemcpyAsync(d_items.p, items.data(), items.size() * sizeof(PackItem), cudaMemcpyHostToDevice,
                                   st), "pack items");
        cuda_check(cudaMemsetAsync(counter.p, 0, 4, st), "zero");
        kernel<<<grid, 256, smem, st>>>(d_items.p, static_cast<int>(items.size()), counter.p, k, max_entries, G,
                                        alpha, beta, scratch.p, slot);
        cuda_check(cudaGetLastError(), "ftlm_pack launch");
    };
#define QB_PACK(T, C) go(ftlm_pack<T, ST, C>)
#define QB_PACK_T(T)                  \
    if (cpl <= 1) QB_PACK(T, 1);      \
    else if (cpl <= 2) QB_PACK(T, 2); \
    else if (cpl <= 4) QB_PACK(T, 4); \
    else if (cpl <= 5) QB_PACK(T, 5); \
    else QB_PACK(T, 8);
    if (dtype == QB_C64) {
        QB_PACK_T(float2)
    } else {
        QB_PACK_T(double2)
    }
#undef QB_PACK_T
#undef QB_PACK
}

// ---- the curves on the device ----
// A block's place in the call's alpha [cap][k] / beta [cap + 1][k] arrays, its dimension and breakdown tolerance.
struct CurveBlock {
    unsigned long long a_off, b_off, dim;
    double tol;
    int cap;
};

// All eigenvalues and the first component of every unit eigenvector of the symmetric tridiagonal (d, e): implicit
// QL with Wilkinson shifts, the rotations applied to the first row of the eigenvector matrix only (the reference's
// tridiag_eig, include/ed/krylov/tridiag.h:42-80, returns the whole matrix; FTLM reads its first row). The arrays
// are one thread's strided columns, element i at p[i * ld]. Returns false when an eigenvalue takes over 100 sweeps.
__device__ bool ql_first_row(double* d, double* e, double* z, int m, std::size_t ld) {
#define QB_D(i) d[static_cast<std::size_t>(i) * ld]
#define QB_E(i) e[static_cast<std::size_t>(i) * ld]
#define QB_Z(i) z[static_cast<std::size_t>(i) * ld]
    const double eps = 2.220446049250313e-16;
    for (int l = 0; l < m; ++l) {
        for (int iter = 0;; ++iter) {
            int mm = l;
            for (; mm < m - 1; ++mm) {
                const double dd = fabs(QB_D(mm)) + fabs(QB_D(mm + 1));
                if (fabs(QB_E(mm)) <= eps * dd) break;
            }
            if (mm == l) break;
            if (iter > 100) return false;
            double g = (QB_D(l + 1) - QB_D(l)) / (2.0 * QB_E(l));
            double r = hypot(g, 1.0);
            g = QB_D(mm) - QB_D(l) + QB_E(l) / (g + (g >= 0 ? r : -r));
            double s = 1.0, c = 1.0, p = 0.0;
            int i = mm - 1;
            for (; i >= l; --i) {
                double f = s * QB_E(i);
                const double b = c * QB_E(i);
                r = hypot(f, g);
                QB_E(i + 1) = r;
                if (r == 0.0) {
                    QB_D(i + 1) -= p;
                    QB_E(mm) = 0.0;
                    break;
                }
                const double ir = 1.0 / r;
                s = f * ir;
                c = g * ir;
                g = QB_D(i + 1) - p;
                r = (QB_D(i) - g) * s + 2.0 * c * b;
                p = s * r;
                QB_D(i + 1) = g + p;
                g = c * r - b;
                f = QB_Z(i + 1);
                QB_Z(i + 1) = s * QB_Z(i) + c * f;
                QB_Z(i) = c * QB_Z(i) - s * f;
            }
            if (r == 0.0 && i >= l) continue;
            QB_D(l) -= p;
            QB_E(l) = g;
            QB_E(mm) = 0.0;
        }
    }
#undef QB_D
#undef QB_E
#undef QB_Z
    return true;
}

// One thread per (block, sample) item: the sample's run up to its breakdown, its Ritz values and first-component
// weights w_i = z_i^2, and its moments about its lowest weighted level e_min (sample_moments,
// include/ed/thermal/ftlm.h:165-192): Z_t = sum_i w_i e^{-beta_t x_i}, E1_t = sum_i x_i w_i e^{-beta_t x_i},
// E2_t = sum_i x_i^2 w_i e^{-beta_t x_i}, x_i = theta_i - e_min, summed in ascending theta (ties in QL order).
// mom[q * n_items + item]: q = 0 e_min, then Z, E1, E2 of temperature t at q = 1 + 3t, 2 + 3t, 3 + 3t. The
// tridiagonal and its order sit in shared memory when `in_smem` (cap_max 28-byte rows per thread, strided by the
// block's threads), else in `scratch` / `ord` (3 cap_max doubles and cap_max ints per item, strided by n_items).
__global__ void k_sample_moments(const CurveBlock* blocks, int n_items, int k, const double* alpha, const double* beta,
                                 const double* betas, int n_beta, int cap_max, bool in_smem, double* scratch, int* ord,
                                 double* mom, int* err) {
    extern __shared__ __align__(16) unsigned char csm[];
    const int item = blockIdx.x * blockDim.x + threadIdx.x;
    if (item >= n_items) return;
    const CurveBlock B = blocks[item / k];
    const int s = item % k;
    const std::size_t ld = in_smem ? blockDim.x : static_cast<std::size_t>(n_items);   // the tridiagonal's stride
    const std::size_t mld = static_cast<std::size_t>(n_items);                         // the output's stride
    double* base = in_smem ? reinterpret_cast<double*>(csm) + threadIdx.x : scratch + item;
    double* d = base;
    double* e = base + static_cast<std::size_t>(cap_max) * ld;
    double* z = base + 2 * static_cast<std::size_t>(cap_max) * ld;
    int* o = in_smem ? reinterpret_cast<int*>(reinterpret_cast<double*>(csm) + 3 * static_cast<std::size_t>(cap_max) *
                                                                                 blockDim.x) + threadIdx.x
                     : ord + item;
    const double* a = alpha + B.a_off;
    const double* b = beta + B.b_off;
    int m = 0;
    for (int j = 0; j < B.cap; ++j) {
        d[static_cast<std::size_t>(j) * ld] = a[static_cast<std::size_t>(j) * k + s];
        const double bj = b[static_cast<std::size_t>(j + 1) * k + s];
        e[static_cast<std::size_t>(j) * ld] = bj;
        z[static_cast<std::size_t>(j) * ld] = j == 0 ? 1.0 : 0.0;
        ++m;
        if (bj < B.tol) break;
    }
    e[static_cast<std::size_t>(m - 1) * ld] = 0.0;
    if (!ql_first_row(d, e, z, m, ld)) {
        atomicExch(err, 1);
        return;
    }
    // ascending order, stable: each value's rank among the values
    for (int i = 0; i < m; ++i) {
        const double vi = d[static_cast<std::size_t>(i) * ld];
        int r = 0;
        for (int q = 0; q < m; ++q) {
            const double vq = d[static_cast<std::size_t>(q) * ld];
            r += (vq < vi || (vq == vi && q < i)) ? 1 : 0;
        }
        o[static_cast<std::size_t>(r) * ld] = i;
    }
    double e_min = CUDART_INF, lo = CUDART_INF;
    for (int r = 0; r < m; ++r) {
        const int i = o[static_cast<std::size_t>(r) * ld];
        const double v = d[static_cast<std::size_t>(i) * ld], zz = z[static_cast<std::size_t>(i) * ld];
        lo = fmin(lo, v);
        if (zz * zz > 0.0) e_min = fmin(e_min, v);
    }
    if (!isfinite(e_min)) e_min = lo;
    mom[item] = e_min;
    for (int t = 0; t < n_beta; ++t) {
        const double bt = betas[t];
        double zs = 0.0, e1 = 0.0, e2 = 0.0;
        for (int r = 0; r < m; ++r) {
            const int i = o[static_cast<std::size_t>(r) * ld];
            const double x = d[static_cast<std::size_t>(i) * ld] - e_min;
            const double zz = z[static_cast<std::size_t>(i) * ld];
            const double bb = (zz * zz) * exp(-bt * x);
            zs += bb;
            e1 += x * bb;
            e2 += x * x * bb;
        }
        mom[(1 + 3 * static_cast<std::size_t>(t)) * mld + item] = zs;
        mom[(2 + 3 * static_cast<std::size_t>(t)) * mld + item] = e1;
        mom[(3 + 3 * static_cast<std::size_t>(t)) * mld + item] = e2;
    }
}

// One thread per (block, temperature): the block's samples combined in sample order about the least sample minimum
// e_ref (combine_samples, include/ed/thermal/ftlm.h:199-235), a log-sum-exp over the samples' shifted partition
// functions: lnZ = ln n + ln <Z> - beta e_ref, E = e_ref + <E1>/<Z>, V = <E2>/<Z> - (<E1>/<Z>)^2.
__global__ void k_block_combine(const CurveBlock* blocks, int n_blocks, int k, const double* mom, int n_items,
                                const double* betas, int n_beta, double* lnZ, double* E, double* V, double* e_min) {
    const int nt = n_beta > 0 ? n_beta : 1;   // no temperatures: e_min alone
    const long long idx = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (idx >= static_cast<long long>(n_blocks) * nt) return;
    const int b = static_cast<int>(idx / nt), t = static_cast<int>(idx % nt);
    const std::size_t ld = static_cast<std::size_t>(n_items);
    const int i0 = b * k;
    double e_ref = mom[i0];
    for (int s = 1; s < k; ++s) e_ref = fmin(e_ref, mom[i0 + s]);
    if (t == 0) e_min[b] = e_ref;
    if (n_beta == 0) return;
    const double bt = betas[t];
    double zz = 0.0, e1 = 0.0, e2 = 0.0;
    for (int s = 0; s < k; ++s) {
        const int it = i0 + s;
        const double dd = mom[it] - e_ref, r = exp(-bt * dd);
        const double Z = mom[(1 + 3 * static_cast<std::size_t>(t)) * ld + it];
        const double E1 = mom[(2 + 3 * static_cast<std::size_t>(t)) * ld + it];
        const double E2 = mom[(3 + 3 * static_cast<std::size_t>(t)) * ld + it];
        zz += Z * r;
        e1 += (E1 + dd * Z) * r;
        e2 += (E2 + 2.0 * dd * E1 + dd * dd * Z) * r;
    }
    zz /= k;
    e1 /= k;
    e2 /= k;
    const std::size_t o = static_cast<std::size_t>(b) * n_beta + t;
    if (zz > 1e-300) {
        const double m1 = e1 / zz, m2 = e2 / zz;
        lnZ[o] = log(static_cast<double>(blocks[b].dim)) + log(zz) - bt * e_ref;
        E[o] = e_ref + m1;
        V[o] = fmax(m2 - m1 * m1, 0.0);
    } else {
        lnZ[o] = -bt * e_ref;
        E[o] = e_ref;
        V[o] = 0.0;
    }
}

// FTLM over many blocks (qb_ftlm_blocks; one block: qb_ftlm).
void ftlm_blocks(const qb_sector* const* secs, const qb_program* const* progs, int n_blocks, int k, int depth,
                 std::uint64_t seed, int seed_mode, const double* betas, int n_beta, int dtype, bool use_csr, double* lnZ,
                 double* E, double* V, double* e_min, double* stats) {
    using clock = std::chrono::steady_clock;
    auto secs_since = [](clock::time_point t0) { return std::chrono::duration<double>(clock::now() - t0).count(); };
    auto t_phase = clock::now();
    double st_draw = 0.0, st_csr = 0.0, st_rec = 0.0, st_curves = 0.0;
    if (k < 1 || k > kMaxCols) throw Error(QB_EINVAL, "samples must be in [1, 64]");
    if (depth < 2) throw Error(QB_EINVAL, "depth must be >= 2");
    if (dtype != QB_C128 && dtype != QB_C64) throw Error(QB_EINVAL, "bad dtype");
    if (n_blocks < 1 || !secs || !progs) throw Error(QB_EINVAL, "no blocks");
    if (seed_mode != QB_SEED_SHARED && seed_mode != QB_SEED_PER_BLOCK) throw Error(QB_EINVAL, "bad seed mode");
    std::uint64_t len = 0;
    for (int b = 0; b < n_blocks; ++b) {
        if (!secs[b] || !progs[b]) throw Error(QB_EINVAL, "null block");
        if (secs[b]->dim == 0) throw Error(QB_EINVAL, "empty sector");
        len = std::max(len, secs[b]->dim);
    }
    const std::size_t es = dtype == QB_C64 ? 8 : 16;
    // the samples of every block: one table drawn once, or a table per block; block b's sample s at
    // dG + g_off[b] + s * g_ld[b]
    std::vector<std::size_t> g_off(n_blocks, 0);
    std::vector<std::uint64_t> g_ld(n_blocks, len);
    DevBuf<double2> dG;
    {
        std::vector<std::complex<double>> G;
        if (seed_mode == QB_SEED_SHARED) {
            G = sample_table(seed, k, len);
        } else {
            for (int b = 0; b < n_blocks; ++b) g_ld[b] = secs[b]->dim;
            G = sample_tables_per_block(seed, k, g_ld, g_off);
        }
        dG.alloc(G.size());
        cuda_check(cudaMemcpy(dG.p, G.data(), G.size() * 16, cudaMemcpyHostToDevice), "samples upload");
    }
    st_draw = secs_since(t_phase);
    // blocks, largest first, dealt round robin to a few streams so small blocks overlap
    std::vector<int> order(n_blocks);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return secs[a]->dim > secs[b]->dim; });
    const int ns = std::min(n_blocks, 4);
    std::vector<cudaStream_t> streams(ns);
    for (auto& st : streams) cuda_check(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "stream");
    struct StreamGuard {
        std::vector<cudaStream_t>& s;
        ~StreamGuard() {
            for (auto st : s)
                if (st) cudaStreamDestroy(st);
        }
    } guard{streams};
    std::vector<BlockBufs> bufs(ns);
    std::vector<int> caps(n_blocks);
    std::vector<std::size_t> a_off(n_blocks), b_off(n_blocks);
    std::size_t a_tot = 0, b_tot = 0;
    for (int b = 0; b < n_blocks; ++b) {
        caps[b] = static_cast<int>(std::min<std::uint64_t>(static_cast<std::uint64_t>(depth), secs[b]->dim));
        a_off[b] = a_tot;
        b_off[b] = b_tot;
        a_tot += static_cast<std::size_t>(caps[b]) * k;
        b_tot += static_cast<std::size_t>(caps[b] + 1) * k;
    }
    DevBuf<double> d_alpha(a_tot), d_beta(b_tot);
    std::vector<double> tol(n_blocks);
    for (int b = 0; b < n_blocks; ++b) tol[b] = 64.0 * std::numeric_limits<double>::epsilon() * norm_bound(progs[b]);
    // the small blocks, run whole by the packed kernel on a stream of their own while the others build their CSRs
    std::vector<char> packed(n_blocks, 0);
    std::vector<int> pack_set[2];   // 32-bit and 64-bit states
    if (use_csr) {
        const std::uint64_t pmax = pack_max_dim();
        for (int i = 0; i < n_blocks; ++i) {
            const int b = order[i];
            bool in_smem = false;
            if (secs[b]->dim > pmax || smem_for(progs[b], secs[b], in_smem) > kPackSmemMax ||
                progs[b]->view.n_groups > static_cast<u32>(kPackMaxEntries))
                continue;
            packed[b] = 1;
            pack_set[secs[b]->N <= 32 ? 0 : 1].push_back(b);
        }
    }
    cudaStream_t pst = nullptr;
    cuda_check(cudaStreamCreateWithFlags(&pst, cudaStreamNonBlocking), "stream");
    struct PackStream {
        cudaStream_t s;
        ~PackStream() {
            cudaStreamSynchronize(s);
            cudaStreamDestroy(s);
        }
    };
    DevBuf<PackItem> pack_items[2];
    DevBuf<unsigned> pack_counter[2];
    DevBuf<unsigned char> pack_scratch[2];
    PackStream pack_guard{pst};
    launch_pack<u32>(pack_set[0], secs, progs, k, dtype, a_off, b_off, caps, tol, dG.p, g_off, g_ld, d_alpha.p,
                     d_beta.p, pack_items[0], pack_counter[0], pack_scratch[0], pst);
    launch_pack<u64>(pack_set[1], secs, progs, k, dtype, a_off, b_off, caps, tol, dG.p, g_off, g_ld, d_alpha.p,
                     d_beta.p, pack_items[1], pack_counter[1], pack_scratch[1], pst);
    // every block's reduced CSR, built before the recurrences (a build synchronises the device); a block
    // whose CSR does not fit runs on the walk
    struct Csrs {
        std::vector<qb_csr*> h;
        ~Csrs() {
            for (auto* c : h)
                if (c) qb_csr_destroy(c);
        }
    } csrs{std::vector<qb_csr*>(n_blocks, nullptr)};
    t_phase = clock::now();
    if (use_csr) {
        // the builds synchronise with the host a few times each: a few host threads, each on its own stream, keep
        // the device busy across them
        int dev = 0;
        cuda_check(cudaGetDevice(&dev), "device");
        std::atomic<int> next_b{0};
        std::vector<std::thread> builders;
        const int nt = std::max(1, std::min(8, n_blocks));
        for (int t = 0; t < nt; ++t)
            builders.emplace_back([&] {
                cudaSetDevice(dev);
                for (int b = next_b++; b < n_blocks; b = next_b++)
                    if (!packed[b] && qb_csr_build(secs[b], secs[b], progs[b], 0, &csrs.h[b]) != QB_OK)
                        csrs.h[b] = nullptr;
                cudaStreamSynchronize(cudaStreamPerThread);
            });
        for (auto& t : builders) t.join();
    }
    st_csr = secs_since(t_phase);
    t_phase = clock::now();
    for (int i = 0, q = 0; i < n_blocks; ++i) {
        const int b = order[i];
        if (packed[b]) continue;
        const int si = q++ % ns;
        cudaStream_t st = streams[si];
        const qb_sector* sec = secs[b];
        const std::uint64_t n = sec->dim;
        // the buffers grow on the host's side of the stream: wait for the stream's previous block first
        BlockBufs& B = bufs[si];
        const bool grow = B.w.n < static_cast<std::size_t>(n) * k;
        if (grow) cuda_check(cudaStreamSynchronize(st), "stream");
        B.ensure(n, k, es);
        k_sample_norms<<<k, kThreads, 0, st>>>(n, dG.p + g_off[b], g_ld[b], B.inv.p);
        k_sample_start<<<red_blocks(static_cast<std::uint64_t>(n) * k), kThreads, 0, st>>>(n, k, dG.p + g_off[b], g_ld[b],
                                                                                            B.inv.p, B.w.p);
        block_recurrence(sec, progs[b], csrs.h[b], k, caps[b], tol[b], dtype, B, st, d_alpha.p + a_off[b],
                         d_beta.p + b_off[b]);
    }
    for (auto st : streams) cuda_check(cudaStreamSynchronize(st), "ftlm blocks");
    cuda_check(cudaStreamSynchronize(pst), "ftlm packed blocks");
    st_rec = secs_since(t_phase);
    t_phase = clock::now();
    // the curves on the device: one thread per (block, sample), then one per (block, temperature)
    const int n_items = n_blocks * k;
    int cap_max = 1;
    std::vector<CurveBlock> cb(n_blocks);
    for (int b = 0; b < n_blocks; ++b) {
        cb[b] = CurveBlock{a_off[b], b_off[b], secs[b]->dim, tol[b], caps[b]};
        cap_max = std::max(cap_max, caps[b]);
    }
    DevBuf<CurveBlock> d_cb(n_blocks);
    // a thread's tridiagonal in shared memory (32 threads a block) while it fits, else in global scratch
    const std::size_t row_bytes = static_cast<std::size_t>(cap_max) * (3 * 8 + 4);
    const bool in_smem = row_bytes * 32 <= 200 * 1024;
    const std::size_t n_scr = in_smem ? 1 : static_cast<std::size_t>(cap_max) * n_items;
    DevBuf<double> d_betas(std::max(1, n_beta)), scratch(3 * n_scr);
    DevBuf<double> mom((1 + 3 * static_cast<std::size_t>(n_beta)) * n_items);
    DevBuf<int> ord(n_scr), err(1);
    const std::size_t nbt = static_cast<std::size_t>(n_blocks) * n_beta;
    DevBuf<double> out(3 * nbt + n_blocks);
    cudaStream_t st0 = cudaStreamPerThread;
    cuda_check(cudaMemcpyAsync(d_cb.p, cb.data(), n_blocks * sizeof(CurveBlock), cudaMemcpyHostToDevice, st0), "upload");
    if (n_beta > 0)
        cuda_check(cudaMemcpyAsync(d_betas.p, betas, n_beta * 8, cudaMemcpyHostToDevice, st0), "upload");
    cuda_check(cudaMemsetAsync(err.p, 0, 4, st0), "zero");
    const int cthreads = in_smem ? 32 : 128;
    const std::size_t csmem = in_smem ? row_bytes * 32 : 0;
    if (csmem > 48 * 1024)
        cuda_check(cudaFuncSetAttribute(k_sample_moments, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        static_cast<int>(csmem)), "smem attribute");
    k_sample_moments<<<(n_items + cthreads - 1) / cthreads, cthreads, csmem, st0>>>(
        d_cb.p, n_items, k, d_alpha.p, d_beta.p, d_betas.p, n_beta, cap_max, in_smem, scratch.p, ord.p, mom.p, err.p);
    const std::size_t n_comb = static_cast<std::size_t>(n_blocks) * std::max(1, n_beta);
    k_block_combine<<<static_cast<unsigned>((n_comb + 127) / 128), 128, 0, st0>>>(
        d_cb.p, n_blocks, k, mom.p, n_items, d_betas.p, n_beta, out.p, out.p + nbt, out.p + 2 * nbt, out.p + 3 * nbt);
    cuda_check(cudaGetLastError(), "ftlm curves");
    std::vector<double> host(3 * nbt + n_blocks);
    int h_err = 0;
    cuda_check(cudaMemcpyAsync(host.data(), out.p, host.size() * 8, cudaMemcpyDeviceToHost, st0), "curves");
    cuda_check(cudaMemcpyAsync(&h_err, err.p, 4, cudaMemcpyDeviceToHost, st0), "curves");
    cuda_check(cudaStreamSynchronize(st0), "ftlm curves");
    if (h_err) throw Error(QB_ECUDA, "tridiagonal QL did not converge");
    std::copy(host.begin(), host.begin() + nbt, lnZ);
    std::copy(host.begin() + nbt, host.begin() + 2 * nbt, E);
    std::copy(host.begin() + 2 * nbt, host.begin() + 3 * nbt, V);
    std::copy(host.begin() + 3 * nbt, host.end(), e_min);
    st_curves = secs_since(t_phase);
    if (stats) {
        stats[0] = st_draw;
        stats[1] = st_csr;
        stats[2] = st_rec;
        stats[3] = st_curves;
    }
}

// ---- the allocation-free Lanczos (qb_lanczos_noalloc) ----
// Its scratch -- the alpha / beta history, the local-projection overlap, the block partials of the
// deterministic reductions and the last-block counter -- lives in this file-scope device array, held by
// every GPU that loads the library until the process exits. Calls share it: two calls that overlap on the
// GPU race on it.
constexpr int kNoAllocMaxIter = QB_NOALLOC_MAX_ITER;
constexpr std::size_t kNoAllocDoubles =
    static_cast<std::size_t>(kNoAllocMaxIter) + (kNoAllocMaxIter + 1) + 2 + 4 * kMaxRedBlocks + 2;
__device__ __align__(256) double g_noalloc_scratch[kNoAllocDoubles];

// The device address of g_noalloc_scratch on the current device, resolved once per device (host code
// cannot use the symbol's name as an address).
double* noalloc_scratch() {
    static std::mutex mu;
    static std::vector<double*> per_device;
    int dev = 0;
    cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
    std::lock_guard<std::mutex> lk(mu);
    if (per_device.size() <= static_cast<std::size_t>(dev)) per_device.resize(dev + 1, nullptr);
    if (!per_device[dev]) {
        void* ptr = nullptr;
        cuda_check(cudaGetSymbolAddress(&ptr, g_noalloc_scratch), "cudaGetSymbolAddress(scratch)");
        per_device[dev] = static_cast<double*>(ptr);
    }
    return per_device[dev];
}

}  // namespace
}  // namespace qb

extern "C" {

int qb_staged_start(uint64_t seed, uint64_t n, double* out) {
    return qb::guarded([&] {
        if (!out && n) throw qb::Error(QB_EINVAL, "null argument");
        qb::staged_seed_into(reinterpret_cast<std::complex<double>*>(out), static_cast<std::size_t>(n), seed);
    });
}

int qb_lanczos(const qb_sector* sec, const qb_program* prog, const double* v0_host, int max_iter, int reorth,
               double breakdown_tol, int dtype, double* alpha, double* beta, int* iters) {
    return qb::guarded([&] {
        using namespace qb;
        if (!sec || !prog || !v0_host || !alpha || !beta || !iters) throw Error(QB_EINVAL, "null argument");
        if (reorth != QB_REORTH_NONE && reorth != QB_REORTH_LOCAL && reorth != QB_REORTH_FULL)
            throw Error(QB_EINVAL, "qb_lanczos: unknown reorthogonalisation policy");
        if (dtype != QB_C128 && dtype != QB_C64) throw Error(QB_EINVAL, "bad dtype");
        *iters = 0;
        if (max_iter <= 0 || sec->dim == 0) return;
        Recurrence R(sec, prog, dtype, max_iter);
        R.start_from_host(reinterpret_cast<const std::complex<double>*>(v0_host));
        const ScanOut o = run_scan(R, max_iter, reorth, false, breakdown_tol, false);
        std::copy(o.alpha.begin(), o.alpha.end(), alpha);
        std::copy(o.beta.begin(), o.beta.end(), beta);
        *iters = static_cast<int>(o.alpha.size());
    });
}

int qb_eigs_lowest(const qb_sector* sec, const qb_program* prog, int max_iter, int dtype, int refine, double* e0,
                   int* iters, int* converged, int* matvecs) {
    return qb::guarded([&] {
        using namespace qb;
        if (!sec || !prog || !e0) throw Error(QB_EINVAL, "null argument");
        if (dtype != QB_C128 && dtype != QB_C64) throw Error(QB_EINVAL, "bad dtype");
        const std::uint64_t nb = sec->dim;
        *e0 = std::numeric_limits<double>::quiet_NaN();
        if (iters) *iters = 0;
        if (converged) *converged = 0;
        if (matvecs) *matvecs = 0;
        if (nb == 0) return;
        const int budget = max_iter > 0 ? max_iter : 400;
        const int mi = static_cast<int>(std::min<std::uint64_t>(nb, static_cast<std::uint64_t>(budget)));
        // a run that may span the whole block reorthogonalises fully (block_solve.cpp:544-548)
        const int reorth = static_cast<std::uint64_t>(mi) >= nb ? QB_REORTH_FULL : QB_REORTH_NONE;
        const auto v0 = staged_seed(nb, 0x51ED0B70ULL);
        const bool mixed = dtype == QB_C64 && refine;
        // FP32 storage keeps its Krylov basis when it fits comfortably (the Ritz vector for the
        // refinement); otherwise the scan runs twice (the second pass accumulates the Ritz vector).
        const std::size_t free_b = available_bytes();
        const bool keep = mixed && static_cast<double>(mi + 2) * nb * 8.0 < 0.5 * static_cast<double>(free_b);
        auto Rp = std::make_unique<Recurrence>(sec, prog, dtype, mi);
        Recurrence& R = *Rp;
        R.start_from_host(v0.data());
        ScanOut o = run_scan(R, mi, reorth, true, 1e-300, keep);
        int total_mv = o.matvecs;
        if (iters) *iters = static_cast<int>(o.alpha.size());
        if (!mixed || !o.converged) {
            *e0 = o.e0;
            if (converged) *converged = o.converged ? 1 : 0;
            if (matvecs) *matvecs = total_mv;
            return;
        }
        // ---- the Ritz vector of the lowest level ----
        const int m = leading_block(o.alpha, o.beta, static_cast<int>(o.alpha.size()));
        std::vector<double> e(std::max(1, m - 1));
        for (int i = 0; i + 1 < m; ++i) e[i] = o.beta[i + 1];
        double lo, hi;
        gershgorin(o.alpha.data(), e.data(), m, lo, hi);
        const double theta = kth_eigenvalue(o.alpha.data(), e.data(), m, 0, lo, hi);
        const std::vector<double> z = inverse_iteration(o.alpha.data(), e.data(), m, theta);
        DevBuf<double2> x(nb);
        cuda_check(cudaMemsetAsync(x.p, 0, nb * 16, R.st), "zero");
        if (keep) {
            for (int j = 0; j < m; ++j) R.accumulate(x.p, z[j], R.basis[j]);
            R.basis.clear();
        } else {
            // second pass from the same start: the same vectors, bit for bit
            Recurrence R2(sec, prog, dtype, m);
            R2.start_from_host(v0.data());
            for (int j = 0; j < m; ++j) {
                R2.accumulate(x.p, z[j], R2.vbuf[R2.cur].p);
                if (j + 1 < m) {
                    if (reorth == QB_REORTH_FULL) R2.keep_current();
                    R2.step(j, reorth);
                    ++total_mv;
                }
            }
            cuda_check(cudaStreamSynchronize(R2.st), "second pass");
        }
        cuda_check(cudaStreamSynchronize(R.st), "ritz vector");
        Rp.reset();
        // ---- FP64 refinement: restarted Lanczos from the Ritz vector ----
        const double scale = norm_bound(prog);
        const int cyc = static_cast<int>(std::min<std::uint64_t>(nb, 24));
        double best = theta;
        bool ok = false;
        for (int c = 0; c < 8 && !ok; ++c) {
            // the short FP64 cycle keeps its basis for the restart vector when it fits comfortably; otherwise
            // the cycle runs twice and the second pass accumulates the restart vector
            const bool keep_f = static_cast<double>(cyc + 4) * nb * 16.0 < 0.5 * static_cast<double>(available_bytes());
            std::vector<double> zz;
            int mm = 0;
            {
                Recurrence F(sec, prog, QB_C128, cyc);
                F.start_from_device(x.p);
                ScanOut f = run_scan(F, cyc, QB_REORTH_NONE, false, 1e-300, keep_f);
                total_mv += f.matvecs;
                mm = static_cast<int>(f.alpha.size());
                std::vector<double> ee(std::max(1, mm - 1));
                for (int i = 0; i + 1 < mm; ++i) ee[i] = f.beta[i + 1];
                double l2, h2;
                gershgorin(f.alpha.data(), ee.data(), mm, l2, h2);
                const double th = kth_eigenvalue(f.alpha.data(), ee.data(), mm, 0, l2, h2);
                zz = inverse_iteration(f.alpha.data(), ee.data(), mm, th);
                const double bound = std::abs(f.beta[mm]) * std::abs(zz[mm - 1]);
                best = th;
                if (bound <= 1e-7 * scale) {
                    ok = true;
                    break;
                }
                if (keep_f) {
                    cuda_check(cudaMemsetAsync(x.p, 0, nb * 16, F.st), "zero");
                    for (int j = 0; j < mm; ++j) F.accumulate(x.p, zz[j], F.basis[j]);
                    cuda_check(cudaStreamSynchronize(F.st), "refine");
                    continue;
                }
            }
            // second pass from the same start: the same vectors, bit for bit
            Recurrence F2(sec, prog, QB_C128, mm);
            F2.start_from_device(x.p);   // synchronises; x is free to be overwritten from here
            cuda_check(cudaMemsetAsync(x.p, 0, nb * 16, F2.st), "zero");
            for (int j = 0; j < mm; ++j) {
                F2.accumulate(x.p, zz[j], F2.vbuf[F2.cur].p);
                if (j + 1 < mm) {
                    F2.step(j, QB_REORTH_NONE);
                    ++total_mv;
                }
            }
            cuda_check(cudaStreamSynchronize(F2.st), "refine second pass");
        }
        *e0 = best;
        if (converged) *converged = ok ? 1 : 0;
        if (matvecs) *matvecs = total_mv;
    });
}

int qb_ftlm(const qb_sector* sec, const qb_program* prog, int samples, int depth, uint64_t seed, const double* betas,
            int n_beta, int dtype, double* lnZ, double* E, double* V, double* e_min) {
    return qb::guarded([&] {
        using namespace qb;
        if (!sec || !prog || !betas || !lnZ || !E || !V || !e_min) throw Error(QB_EINVAL, "null argument");
        const qb_sector* secs[1] = {sec};
        const qb_program* progs[1] = {prog};
        // the program's own lane: its attached CSR for this sector, else the walk
        ftlm_blocks(secs, progs, 1, samples, depth, seed, QB_SEED_SHARED, betas, n_beta, dtype, false, lnZ, E, V, e_min,
                    nullptr);
    });
}

int qb_ftlm_blocks(const qb_sector* const* secs, const qb_program* const* progs, int n_blocks, int samples, int depth,
                   uint64_t seed, int seed_mode, const double* betas, int n_beta, int dtype, int use_csr, double* lnZ,
                   double* E, double* V, double* e_min, double* stats) {
    return qb::guarded([&] {
        using namespace qb;
        if (!betas || !lnZ || !E || !V || !e_min) throw Error(QB_EINVAL, "null argument");
        ftlm_blocks(secs, progs, n_blocks, samples, depth, seed, seed_mode, betas, n_beta, dtype, use_csr != 0, lnZ, E, V,
                    e_min, stats);
    });
}

int qb_thermal_combine(int n_blocks, const double* weights, const double* lnZ, const double* E, const double* V,
                       const double* betas, int n_beta, double* lnZ_out, double* E_out, double* C_out, double* S_out,
                       double* F_out) {
    return qb::guarded([&] {
        using namespace qb;
        if (n_blocks < 1 || !lnZ || !E || !V || !betas || !lnZ_out || !E_out || !C_out || !S_out || !F_out)
            throw Error(QB_EINVAL, "null argument");
        std::vector<double> p(n_blocks);
        for (int i = 0; i < n_beta; ++i) {
            auto at = [&](const double* a, int b) { return a[static_cast<std::size_t>(b) * n_beta + i]; };
            double mx = -std::numeric_limits<double>::infinity();
            for (int b = 0; b < n_blocks; ++b)
                mx = std::max(mx, std::log(weights ? weights[b] : 1.0) + at(lnZ, b));
            double z = 0.0, e = 0.0;
            for (int b = 0; b < n_blocks; ++b) {
                p[b] = std::exp(std::log(weights ? weights[b] : 1.0) + at(lnZ, b) - mx);
                z += p[b];
                e += p[b] * at(E, b);
            }
            e /= z;
            // the law of total variance: each block's variance plus the spread of the block means
            double var = 0.0;
            for (int b = 0; b < n_blocks; ++b) {
                const double d = at(E, b) - e;
                var += p[b] * (at(V, b) + d * d);
            }
            var /= z;
            const double bt = betas[i];
            lnZ_out[i] = mx + std::log(z);
            E_out[i] = e;
            C_out[i] = bt * bt * var;
            S_out[i] = lnZ_out[i] + bt * e;
            F_out[i] = -lnZ_out[i] / bt;
        }
    });
}

int qb_cf(const qb_sector* sec, const qb_program* prog, const double* phi_host, int depth, const double* omega,
          int n_omega, double eta, double shift, double tolerance, double* S, double* shift_out) {
    return qb::guarded([&] {
        using namespace qb;
        if (!sec || !prog || !phi_host || !omega || !S || !shift_out) throw Error(QB_EINVAL, "null argument");
        for (int i = 0; i < n_omega; ++i) S[i] = 0.0;
        *shift_out = 0.0;
        const std::uint64_t n = sec->dim;
        if (n == 0 || depth <= 0) return;
        Recurrence R(sec, prog, QB_C128, depth);
        double nrm = 0.0;
        try {
            nrm = R.start_from_host(reinterpret_cast<const std::complex<double>*>(phi_host));
        } catch (const Error& e) {
            if (e.code == QB_EINVAL) return;   // a zero phi has no spectral weight
            throw;
        }
        if (nrm < 1e-14) return;
        ScanOut o = run_scan(R, depth, QB_REORTH_NONE, false, tolerance, false);
        if (o.alpha.empty()) return;
        const int m = static_cast<int>(o.alpha.size());
        *shift_out = cf_spectrum(o.alpha, o.beta, m, omega, n_omega, eta, shift, nrm * nrm, S);
    });
}


// The Lanczos kernel on caller-owned device buffers, allocating nothing (see include/qed_b200.h).
int qb_lanczos_noalloc(const qb_sector* sec, const qb_program* prog, const void* v0, void* work, int max_iter,
                       int reorth, double breakdown_tol, int dtype, double* alpha, double* beta, int* iters,
                       void* stream) {
    return qb::guarded([&] {
        using namespace qb;
        if (!sec || !prog || !v0 || !work || !alpha || !beta || !iters) throw Error(QB_EINVAL, "null argument");
        if (reorth != QB_REORTH_NONE && reorth != QB_REORTH_LOCAL)
            throw Error(QB_EUNSUPPORTED, "qb_lanczos_noalloc: reorth must be QB_REORTH_NONE or QB_REORTH_LOCAL");
        if (dtype != QB_C128 && dtype != QB_C64) throw Error(QB_EINVAL, "bad dtype");
        if (max_iter < 0 || max_iter > kNoAllocMaxIter)
            throw Error(QB_EINVAL, "qb_lanczos_noalloc: max_iter must be in [0, QB_NOALLOC_MAX_ITER = " +
                                       std::to_string(kNoAllocMaxIter) + "]");
        *iters = 0;
        const std::uint64_t n = sec->dim;
        if (max_iter == 0 || n == 0) return;
        const cudaStream_t st = static_cast<cudaStream_t>(stream);
        double* scratch = noalloc_scratch();
        Scal S{scratch, scratch + kNoAllocMaxIter, scratch + 2 * kNoAllocMaxIter + 1,
               scratch + 2 * kNoAllocMaxIter + 3, reinterpret_cast<unsigned*>(scratch + 2 * kNoAllocMaxIter + 3 + 4 * kMaxRedBlocks)};
        // the array keeps the last call's contents: clear the beta history and the counter
        cuda_check(cudaMemsetAsync(S.beta, 0, (kNoAllocMaxIter + 1) * sizeof(double), st), "scratch clear");
        cuda_check(cudaMemsetAsync(S.counter, 0, sizeof(unsigned), st), "scratch clear");
        const std::size_t es = dtype == QB_C64 ? 8 : 16;
        unsigned char* wk = static_cast<unsigned char*>(work);
        void* vb[2] = {wk, wk + n * es};
        double2* w = reinterpret_cast<double2*>(wk + 2 * n * es);
        cuda_check(cudaMemsetAsync(vb[0], 0, n * es, st), "work clear");
        const int nb = red_blocks(n);
        // v_0 = v0 / ||v0|| (v0 is FP64, untouched)
        k_norm<<<nb, kThreads, 0, st>>>(n, static_cast<const double2*>(v0), S);
        if (dtype == QB_C64)
            k_scale_into<float2><<<nb, kThreads, 0, st>>>(n, static_cast<const double2*>(v0), static_cast<float2*>(vb[1]), S.ovl);
        else
            k_scale_into<double2><<<nb, kThreads, 0, st>>>(n, static_cast<const double2*>(v0), static_cast<double2*>(vb[1]), S.ovl);
        cuda_check(cudaGetLastError(), "start");
        double nrm = 0.0;
        cuda_check(cudaMemcpyAsync(&nrm, S.ovl, 8, cudaMemcpyDeviceToHost, st), "norm read");
        cuda_check(cudaStreamSynchronize(st), "start");
        if (!(nrm > 0.0)) throw Error(QB_EINVAL, "qb_lanczos_noalloc: initial vector has non-positive norm");
        const int cap = static_cast<int>(std::min<std::uint64_t>(static_cast<std::uint64_t>(max_iter), n));
        const int local = reorth == QB_REORTH_LOCAL;
        int cur = 1;
        for (int j = 0; j < cap; ++j) {
            void* vc = vb[cur];
            void* vp = vb[cur ^ 1];
            launch_walk_mixed(sec, sec, prog, vc, w, dtype, QB_C128, st);
            if (dtype == QB_C64) {
                rec_alpha<float2><<<nb, kThreads, 0, st>>>(n, j, w, static_cast<float2*>(vp), static_cast<float2*>(vc), S);
                rec_beta<float2><<<nb, kThreads, 0, st>>>(n, j, local, w, static_cast<float2*>(vc), S);
                rec_next<float2><<<nb, kThreads, 0, st>>>(n, j, w, static_cast<float2*>(vc), static_cast<float2*>(vp), S);
            } else {
                rec_alpha<double2><<<nb, kThreads, 0, st>>>(n, j, w, static_cast<double2*>(vp), static_cast<double2*>(vc), S);
                rec_beta<double2><<<nb, kThreads, 0, st>>>(n, j, local, w, static_cast<double2*>(vc), S);
                rec_next<double2><<<nb, kThreads, 0, st>>>(n, j, w, static_cast<double2*>(vc), static_cast<double2*>(vp), S);
            }
            cuda_check(cudaGetLastError(), "recurrence");
            cur ^= 1;
        }
        // straight into the caller's arrays (no staging buffer)
        cuda_check(cudaMemcpyAsync(alpha, S.alpha, cap * 8, cudaMemcpyDeviceToHost, st), "alpha read");
        cuda_check(cudaMemcpyAsync(beta, S.beta, (cap + 1) * 8, cudaMemcpyDeviceToHost, st), "beta read");
        cuda_check(cudaStreamSynchronize(st), "lanczos");
        int m = 0;
        beta[0] = 0.0;
        for (int j = 0; j < cap; ++j) {
            ++m;
            if (beta[j + 1] < breakdown_tol) break;
        }
        *iters = m;
    });
}

}  // extern "C"
