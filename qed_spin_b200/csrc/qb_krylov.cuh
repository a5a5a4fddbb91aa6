// =============================================================================
// qb_krylov.cuh -- the device recurrence shared by the Krylov drivers (krylov.cu, lanes.cu): the fused
// recurrence passes and deterministic reductions, the block (multi-sample) recurrence, CGS2 against a kept
// basis, the host tridiagonal solvers, the reference's seeds, and the single-vector Recurrence / scan.
// Everything here has internal linkage: each translation unit that includes it gets its own copy.
// =============================================================================
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <complex>
#include <cstring>
#include <limits>
#include <memory>
#include <mutex>
#include <numeric>
#include <random>
#include <utility>
#include <vector>

#include <atomic>
#include <thread>

#include "qb_internal.cuh"

namespace qb {

void launch_walk(const qb_sector* row, const qb_sector* col, const qb_program* P, const void* const* ins,
                 void* const* outs, int k, int dtype, cudaStream_t st);
void launch_walk_mixed(const qb_sector* row, const qb_sector* col, const qb_program* P, const void* in, void* out,
                       int dtype_in, int dtype_out, cudaStream_t st);
void launch_block_mixed(const qb_sector* row, const qb_sector* col, const qb_program* P, const void* in, void* out,
                        int k, int dtype_in, int dtype_out, cudaStream_t st);

namespace {

constexpr int kThreads = 256;
constexpr int kMaxRedBlocks = 148 * 8;
constexpr double kLocalThreshold = 1.49011611938476562e-08;   // sqrt(eps), lanczos.h:189-193

int red_blocks(std::uint64_t n) {
    return static_cast<int>(std::max<std::uint64_t>(1, std::min<std::uint64_t>((n + kThreads - 1) / kThreads, kMaxRedBlocks)));
}

template <class T> struct V;
template <> struct V<double2> {
    __device__ static double2 ld(const double2* p, std::size_t i) { return p[i]; }
    __device__ static void st(double2* p, std::size_t i, double re, double im) { p[i] = make_double2(re, im); }
};
template <> struct V<float2> {
    __device__ static double2 ld(const float2* p, std::size_t i) {
        const float2 v = p[i];
        return make_double2(v.x, v.y);
    }
    __device__ static void st(float2* p, std::size_t i, double re, double im) {
        p[i] = make_float2(__double2float_rn(re), __double2float_rn(im));
    }
};

// Fixed-order block reduction of NQ doubles: warp butterflies, then warp 0 over the warps in order.
template <int NQ> __device__ __forceinline__ void block_reduce(double (&v)[NQ], double* sm) {
#pragma unroll
    for (int q = 0; q < NQ; ++q)
        for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_xor_sync(0xffffffffu, v[q], o);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    if (lane == 0)
#pragma unroll
        for (int q = 0; q < NQ; ++q) sm[q * 32 + warp] = v[q];
    __syncthreads();
    if (threadIdx.x == 0)
#pragma unroll
        for (int q = 0; q < NQ; ++q) {
            double s = 0.0;
            for (int w = 0; w < nw; ++w) s += sm[q * 32 + w];
            v[q] = s;
        }
}

// The last block to finish sums the block partials (index order) of NQ quantities into `total`.
template <int NQ>
__device__ __forceinline__ bool last_block_total(double (&v)[NQ], double* partials, unsigned* counter, double* sm,
                                                 double (&total)[NQ]) {
    __shared__ bool is_last;
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < NQ; ++q) partials[q * kMaxRedBlocks + blockIdx.x] = v[q];
        __threadfence();
        const unsigned t = atomicAdd(counter, 1u);
        is_last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!is_last) return false;
    __threadfence();
    double s[NQ];
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
        s[q] = 0.0;
        for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x)
            s[q] += reinterpret_cast<volatile double*>(partials)[q * kMaxRedBlocks + b];
    }
    __syncthreads();
    block_reduce<NQ>(s, sm);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < NQ; ++q) total[q] = s[q];
        *counter = 0;
    }
    return threadIdx.x == 0;
}

// Scalars the recurrence keeps on the device.
struct Scal {
    double* alpha;     // [max_iter]
    double* beta;      // [max_iter + 1]
    double* ovl;       // [2]: the overlap coefficient applied in rec_next (re, im)
    double* partials;  // [4 * kMaxRedBlocks]
    unsigned* counter;
};

// ||x||^2 of a host-staged FP64 vector, then v = x / ||x|| stored as T.
__global__ void k_norm(std::uint64_t n, const double2* x, Scal S) {
    __shared__ double sm[4 * 32];
    double v[1] = {0.0};
    for (std::uint64_t i = static_cast<std::uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<std::uint64_t>(gridDim.x) * blockDim.x) {
        const double2 a = x[i];
        v[0] += a.x * a.x + a.y * a.y;
    }
    block_reduce<1>(v, sm);
    double tot[1];
    if (last_block_total<1>(v, S.partials, S.counter, sm, tot)) S.ovl[0] = sqrt(tot[0]);
}

template <class T> __global__ void k_scale_into(std::uint64_t n, const double2* x, T* out, const double* nrm) {
    const double inv = 1.0 / *nrm;
    for (std::uint64_t i = static_cast<std::uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<std::uint64_t>(gridDim.x) * blockDim.x) {
        const double2 a = x[i];
        V<T>::st(out, i, a.x * inv, a.y * inv);
    }
}

// alpha_j = Re <v_j, w - beta_j v_{j-1}>, w updated in place (axpy_dot, cpu_backend.h:174-191).
template <class T>
__device__ __forceinline__ void rec_alpha_body(std::uint64_t n, int j, double2* w, const T* vp, const T* vc, Scal S) {
    __shared__ double sm[4 * 32];
    const double b = j > 0 ? S.beta[j] : 0.0;
    double v[1] = {0.0};
    for (std::uint64_t i = static_cast<std::uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<std::uint64_t>(gridDim.x) * blockDim.x) {
        double2 y = w[i];
        if (j > 0) {
            const double2 p = V<T>::ld(vp, i);
            y.x = y.x - b * p.x;
            y.y = y.y - b * p.y;
            w[i] = y;
        }
        const double2 z = V<T>::ld(vc, i);
        v[0] += z.x * y.x + z.y * y.y;
    }
    block_reduce<1>(v, sm);
    double tot[1];
    if (last_block_total<1>(v, S.partials, S.counter, sm, tot)) S.alpha[j] = tot[0];
}
template <class T>
__global__ void rec_alpha(std::uint64_t n, int j, double2* w, const T* vp, const T* vc, Scal S) {
    rec_alpha_body<T>(n, j, w, vp, vc, S);
}

// w -= alpha_j v_j; ||w||^2 and <v_j, w> -> beta_{j+1} and the deferred local projection.
template <class T>
__device__ __forceinline__ void rec_beta_body(std::uint64_t n, int j, int local, double2* w, const T* vc, Scal S) {
    __shared__ double sm[4 * 32];
    const double a = S.alpha[j];
    double v[3] = {0.0, 0.0, 0.0};
    for (std::uint64_t i = static_cast<std::uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<std::uint64_t>(gridDim.x) * blockDim.x) {
        double2 y = w[i];
        const double2 z = V<T>::ld(vc, i);
        y.x = y.x - a * z.x;
        y.y = y.y - a * z.y;
        w[i] = y;
        v[0] += y.x * y.x + y.y * y.y;
        v[1] += z.x * y.x + z.y * y.y;
        v[2] += z.x * y.y - z.y * y.x;
    }
    block_reduce<3>(v, sm);
    double tot[3];
    if (last_block_total<3>(v, S.partials, S.counter, sm, tot)) {
        double nrm2 = tot[0];
        const double ore = tot[1], oim = tot[2];
        const bool proj = local && j > 0 && sqrt(ore * ore + oim * oim) > kLocalThreshold;
        if (proj) nrm2 = fmax(nrm2 - (ore * ore + oim * oim), 0.0);
        S.ovl[0] = proj ? -ore : 0.0;
        S.ovl[1] = proj ? -oim : 0.0;
        S.beta[j + 1] = sqrt(nrm2);
    }
}
template <class T>
__global__ void rec_beta(std::uint64_t n, int j, int local, double2* w, const T* vc, Scal S) {
    rec_beta_body<T>(n, j, local, w, vc, S);
}

// v_{j+1} = (w + o v_j) / beta_{j+1}, written over v_{j-1}'s buffer.
template <class T>
__device__ __forceinline__ void rec_next_body(std::uint64_t n, int j, const double2* w, const T* vc, T* vn, Scal S) {
    const double b = S.beta[j + 1];
    const double inv = b > 0.0 ? 1.0 / b : 0.0;
    const double ore = S.ovl[0], oim = S.ovl[1];
    for (std::uint64_t i = static_cast<std::uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<std::uint64_t>(gridDim.x) * blockDim.x) {
        double2 y = w[i];
        if (ore != 0.0 || oim != 0.0) {
            const double2 z = V<T>::ld(vc, i);
            y.x += ore * z.x - oim * z.y;
            y.y += ore * z.y + oim * z.x;
        }
        V<T>::st(vn, i, y.x * inv, y.y * inv);
    }
}
template <class T> __global__ void rec_next(std::uint64_t n, int j, const double2* w, const T* vc, T* vn, Scal S) {
    rec_next_body<T>(n, j, w, vc, vn, S);
}

// The same three passes with the step index in device memory (*dj), so that a captured graph of steps replays
// unchanged: rec_next_dev advances *dj once every block has read it. k_keep_dev copies v_j into basis slot j.
template <class T>
__global__ void rec_alpha_dev(std::uint64_t n, const int* dj, double2* w, const T* vp, const T* vc, Scal S) {
    rec_alpha_body<T>(n, *dj, w, vp, vc, S);
}
template <class T>
__global__ void rec_beta_dev(std::uint64_t n, const int* dj, int local, double2* w, const T* vc, Scal S) {
    rec_beta_body<T>(n, *dj, local, w, vc, S);
}
template <class T> __global__ void rec_next_dev(std::uint64_t n, int* dj, const double2* w, const T* vc, T* vn, Scal S) {
    const int j = *dj;
    rec_next_body<T>(n, j, w, vc, vn, S);
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(S.counter, 1u) == gridDim.x - 1) {
            *dj = j + 1;
            *S.counter = 0;
        }
    }
}
__global__ void k_keep_dev(std::uint64_t bytes, const int* dj, const unsigned char* v, unsigned char* basis) {
    const std::uint64_t words = bytes / 8;   // a vector is n elements of 8 or 16 bytes
    const unsigned long long* src = reinterpret_cast<const unsigned long long*>(v);
    unsigned long long* dst = reinterpret_cast<unsigned long long*>(basis + static_cast<std::uint64_t>(*dj) * bytes);
    for (std::uint64_t i = static_cast<std::uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < words;
         i += static_cast<std::uint64_t>(gridDim.x) * blockDim.x)
        dst[i] = src[i];
}

// ---- full reorthogonalisation (CGS2 with the DGKS gate, lanczos.h:428-451) against the kept basis ----
constexpr double kDgksKappa = 0.7071067811865476;

// slot[0] = ||w|| (deterministic grid reduction).
__global__ void k_norm_to(std::uint64_t n, const double2* w, Scal S, double* slot, const int* flag) {
    if (flag && *flag == 0) return;
    __shared__ double sm[4 * 32];
    double v[1] = {0.0};
    for (std::uint64_t i = static_cast<std::uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<std::uint64_t>(gridDim.x) * blockDim.x) {
        const double2 a = w[i];
        v[0] += a.x * a.x + a.y * a.y;
    }
    block_reduce<1>(v, sm);
    double tot[1];
    if (last_block_total<1>(v, S.partials, S.counter, sm, tot)) *slot = sqrt(tot[0]);
}

// coeff[k] = -<V_k, w>: a grid of (chunk, basis vector) blocks writes partial sums, and k_dot_sum adds each
// vector's partials in chunk order (deterministic for a given chunk count).
template <class T>
__global__ void k_dot_part(std::uint64_t n, const T* const* basis, const double2* w, double2* part, int chunks,
                           const int* flag) {
    if (flag && *flag == 0) return;
    __shared__ double sm[4 * 32];
    const T* v = basis[blockIdx.y];
    const std::uint64_t per = (n + chunks - 1) / chunks;
    const std::uint64_t lo = static_cast<std::uint64_t>(blockIdx.x) * per;
    const std::uint64_t hi = lo + per < n ? lo + per : n;
    double acc[2] = {0.0, 0.0};
    for (std::uint64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
        const double2 b = V<T>::ld(v, i);
        const double2 y = w[i];
        acc[0] += b.x * y.x + b.y * y.y;
        acc[1] += b.x * y.y - b.y * y.x;
    }
    block_reduce<2>(acc, sm);
    if (threadIdx.x == 0) part[static_cast<std::size_t>(blockIdx.y) * chunks + blockIdx.x] = make_double2(acc[0], acc[1]);
}

// A warp per vector: lane l adds chunks l, l + 32, ... in order, then a fixed butterfly adds the lanes (the same
// order every call). Launch with kDotSumWarps warps a block: k_dot_sum<<<dot_sum_blocks(m), 32 * kDotSumWarps>>>.
constexpr int kDotSumWarps = 4;
inline int dot_sum_blocks(int m) { return (m + kDotSumWarps - 1) / kDotSumWarps; }
__global__ void k_dot_sum(int m, int chunks, const double2* part, double2* coeff, const int* flag) {
    if (flag && *flag == 0) return;
    const int k = blockIdx.x * kDotSumWarps + static_cast<int>(threadIdx.x >> 5);
    const int lane = static_cast<int>(threadIdx.x & 31);
    if (k >= m) return;   // whole warps leave together
    double sx = 0.0, sy = 0.0;
    for (int c = lane; c < chunks; c += 32) {
        const double2 p = part[static_cast<std::size_t>(k) * chunks + c];
        sx += p.x;
        sy += p.y;
    }
    for (int o = 16; o > 0; o >>= 1) {
        sx += __shfl_xor_sync(0xffffffffu, sx, o);
        sy += __shfl_xor_sync(0xffffffffu, sy, o);
    }
    if (lane == 0) coeff[k] = make_double2(-sx, -sy);
}

// The chunk count of a dot_many over m vectors of length n: about kMaxRedBlocks blocks in all.
int dot_chunks(std::uint64_t n, int m) {
    const std::uint64_t by_len = (n + 4095) / 4096;
    const int by_grid = std::max(1, kMaxRedBlocks / std::max(1, m));
    return static_cast<int>(std::max<std::uint64_t>(1, std::min<std::uint64_t>(by_len, by_grid)));
}

// coeff[0..m) = -<V_k, w>; part holds at least m * dot_chunks(n, m) entries.
template <class T>
void dot_many(std::uint64_t n, int m, const T* const* basis, const double2* w, double2* coeff, double2* part,
              const int* flag, cudaStream_t st) {
    const int chunks = dot_chunks(n, m);
    k_dot_part<T><<<dim3(chunks, m), kThreads, 0, st>>>(n, basis, w, part, chunks, flag);
    k_dot_sum<<<dot_sum_blocks(m), 32 * kDotSumWarps, 0, st>>>(m, chunks, part, coeff, flag);
}

// w += sum_k coeff[k] V_k, each element accumulated in k order.
template <class T>
__global__ void k_axpy_many(std::uint64_t n, int m, const T* const* basis, const double2* coeff, double2* w,
                            const int* flag) {
    if (flag && *flag == 0) return;
    for (std::uint64_t i = static_cast<std::uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<std::uint64_t>(gridDim.x) * blockDim.x) {
        double2 y = w[i];
        for (int k = 0; k < m; ++k) {
            const double2 c = coeff[k];
            const double2 b = V<T>::ld(basis[k], i);
            y.x += c.x * b.x - c.y * b.y;
            y.y += c.x * b.y + c.y * b.x;
        }
        w[i] = y;
    }
}

// The DGKS gate: a second pass only when the first removed more than 1 - kappa of the norm.
__global__ void k_dgks_gate(const double* before, const double* after, int* flag) {
    *flag = (*after < kDgksKappa * *before) ? 1 : 0;
}

// x += c v (a Ritz-vector accumulation, FP64 destination).
template <class T> __global__ void k_axpy_into(std::uint64_t n, double c, const T* v, double2* x) {
    for (std::uint64_t i = static_cast<std::uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<std::uint64_t>(gridDim.x) * blockDim.x) {
        const double2 a = V<T>::ld(v, i);
        double2 y = x[i];
        y.x += c * a.x;
        y.y += c * a.y;
        x[i] = y;
    }
}

template <class T> __global__ void k_cast_from(std::uint64_t n, const double2* x, T* v) {
    for (std::uint64_t i = static_cast<std::uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<std::uint64_t>(gridDim.x) * blockDim.x)
        V<T>::st(v, i, x[i].x, x[i].y);
}

template <class T> __global__ void k_copy_cast(std::uint64_t n, const T* v, double2* x) {
    for (std::uint64_t i = static_cast<std::uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<std::uint64_t>(gridDim.x) * blockDim.x)
        x[i] = V<T>::ld(v, i);
}

// ---- block (multi-sample) recurrence: k columns interleaved by row, lane c % 32 owns column c ----
constexpr int kMaxCols = 64;

struct BScal {
    double* alpha;     // [depth][k]
    double* beta;      // [depth + 1][k]
    double* ovl;       // [2][k]
    double* partials;  // [3][k][kMaxRedBlocks]
    unsigned* counter;
    double* partials2 = nullptr;          // [3][k][kMaxGroups]: the two-level sums' group totals
    unsigned* group_counter = nullptr;    // [kMaxGroups]
};
constexpr int kMaxGroups = (kMaxRedBlocks + 31) / 32;

template <int NQ, int CPL>
__device__ __forceinline__ bool block_cols_total(double (&v)[NQ][CPL], int k, BScal S, double* sm /*[NQ][kMaxCols][8]*/,
                                                 double (*total)[kMaxCols] /*[NQ][kMaxCols] in smem*/) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
#pragma unroll
    for (int q = 0; q < NQ; ++q)
#pragma unroll
        for (int c = 0; c < CPL; ++c) {
            const int col = lane + 32 * c;
            if (col < k) sm[(q * kMaxCols + col) * 8 + warp] = v[q][c];
        }
    __syncthreads();
    __shared__ bool is_last;
    if (threadIdx.x < k) {
        for (int q = 0; q < NQ; ++q) {
            double s = 0.0;
            for (int w2 = 0; w2 < nw; ++w2) s += sm[(q * kMaxCols + threadIdx.x) * 8 + w2];
            S.partials[(static_cast<std::size_t>(q) * kMaxCols + threadIdx.x) * kMaxRedBlocks + blockIdx.x] = s;
        }
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) is_last = atomicAdd(S.counter, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!is_last) return false;
    __threadfence();
    // the block sums, one warp per (quantity, column) pair: lanes stride over the blocks' partials (read from
    // L2, where the other blocks' fenced writes are), then a fixed xor-butterfly -- deterministic for a grid
    for (int pr = warp; pr < NQ * k; pr += nw) {
        const int q = pr / k, c = pr % k;
        const double* p = S.partials + (static_cast<std::size_t>(q) * kMaxCols + c) * kMaxRedBlocks;
        double s = 0.0;
        for (unsigned b = lane; b < gridDim.x; b += 32) s += __ldcg(p + b);
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) total[q][c] = s;
    }
    __syncthreads();
    if (threadIdx.x == 0) *S.counter = 0;
    return true;
}

// The grid of the block (multi-sample) recurrence passes: two blocks of 256 threads per SM of a B200 keep the
// memory system busy, and the last block's sums then run over few partials.
constexpr int kBlockRecGrid = 2 * 148;

template <class T, int CPL>
__global__ void brec_alpha(std::uint64_t n, int k, int j, double2* w, const T* vp, const T* vc, BScal S) {
    extern __shared__ double bsm[];
    __shared__ double tot[1][kMaxCols];
    const int lane = threadIdx.x & 31;
    double v[1][CPL];
    double b[CPL];
#pragma unroll
    for (int c = 0; c < CPL; ++c) {
        v[0][c] = 0.0;
        const int col = lane + 32 * c;
        b[c] = (j > 0 && col < k) ? S.beta[static_cast<std::size_t>(j) * k + col] : 0.0;
    }
    const std::uint64_t warps = static_cast<std::uint64_t>(gridDim.x) * (blockDim.x >> 5);
    for (std::uint64_t r = static_cast<std::uint64_t>(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5); r < n; r += warps) {
#pragma unroll
        for (int c = 0; c < CPL; ++c) {
            const int col = lane + 32 * c;
            if (col >= k) continue;
            const std::size_t i = r * k + col;
            double2 y = w[i];
            if (j > 0) {
                const double2 p = V<T>::ld(vp, i);
                y.x -= b[c] * p.x;
                y.y -= b[c] * p.y;
                w[i] = y;
            }
            const double2 z = V<T>::ld(vc, i);
            v[0][c] += z.x * y.x + z.y * y.y;
        }
    }
    if (block_cols_total<1, CPL>(v, k, S, bsm, tot) && threadIdx.x < k) S.alpha[static_cast<std::size_t>(j) * k + threadIdx.x] = tot[0][threadIdx.x];
}

template <class T, int CPL>
__global__ void brec_beta(std::uint64_t n, int k, int j, int local, double2* w, const T* vc, BScal S) {
    extern __shared__ double bsm[];
    __shared__ double tot[3][kMaxCols];
    const int lane = threadIdx.x & 31;
    double v[3][CPL];
    double a[CPL];
#pragma unroll
    for (int c = 0; c < CPL; ++c) {
        v[0][c] = v[1][c] = v[2][c] = 0.0;
        const int col = lane + 32 * c;
        a[c] = col < k ? S.alpha[static_cast<std::size_t>(j) * k + col] : 0.0;
    }
    const std::uint64_t warps = static_cast<std::uint64_t>(gridDim.x) * (blockDim.x >> 5);
    for (std::uint64_t r = static_cast<std::uint64_t>(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5); r < n; r += warps) {
#pragma unroll
        for (int c = 0; c < CPL; ++c) {
            const int col = lane + 32 * c;
            if (col >= k) continue;
            const std::size_t i = r * k + col;
            double2 y = w[i];
            const double2 z = V<T>::ld(vc, i);
            y.x -= a[c] * z.x;
            y.y -= a[c] * z.y;
            w[i] = y;
            v[0][c] += y.x * y.x + y.y * y.y;
            v[1][c] += z.x * y.x + z.y * y.y;
            v[2][c] += z.x * y.y - z.y * y.x;
        }
    }
    if (block_cols_total<3, CPL>(v, k, S, bsm, tot) && threadIdx.x < k) {
        const int c = threadIdx.x;
        double nrm2 = tot[0][c];
        const double ore = tot[1][c], oim = tot[2][c];
        const bool proj = local && j > 0 && sqrt(ore * ore + oim * oim) > kLocalThreshold;
        if (proj) nrm2 = fmax(nrm2 - (ore * ore + oim * oim), 0.0);
        S.ovl[c] = proj ? -ore : 0.0;
        S.ovl[kMaxCols + c] = proj ? -oim : 0.0;
        S.beta[static_cast<std::size_t>(j + 1) * k + c] = sqrt(nrm2);
    }
}

template <class T>
__global__ void brec_next(std::uint64_t n, int k, int j, double tol, const double2* w, const T* vc, T* vn, BScal S) {
    const std::uint64_t total = n * k;
    for (std::uint64_t i = static_cast<std::uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
         i += static_cast<std::uint64_t>(gridDim.x) * blockDim.x) {
        const int c = static_cast<int>(i % k);
        const double b = S.beta[static_cast<std::size_t>(j + 1) * k + c];
        // a column past its breakdown stops: its vector goes to zero and stays there
        const double inv = b >= tol && b > 0.0 ? 1.0 / b : 0.0;
        const double ore = S.ovl[c], oim = S.ovl[kMaxCols + c];
        double2 y = w[i];
        if (ore != 0.0 || oim != 0.0) {
            const double2 z = V<T>::ld(vc, i);
            y.x += ore * z.x - oim * z.y;
            y.y += ore * z.y + oim * z.x;
        }
        V<T>::st(vn, i, y.x * inv, y.y * inv);
    }
}

// -------------------------------------------------------------------------------------------
// Host: symmetric tridiagonal eigenproblems. Sturm-sequence bisection for selected eigenvalues,
// inverse iteration for their vectors, and implicit QL with the first row of the eigenvector
// matrix (FTLM weights).
// -------------------------------------------------------------------------------------------
// Number of eigenvalues of T (diag d, off-diag e[i] between i and i+1) below x.
int sturm_count(const double* d, const double* e, int m, double x) {
    int c = 0;
    double q = d[0] - x;
    if (q < 0) ++c;
    for (int i = 1; i < m; ++i) {
        const double qq = q != 0.0 ? q : std::numeric_limits<double>::min();
        q = d[i] - x - e[i - 1] * e[i - 1] / qq;
        if (q < 0) ++c;
    }
    return c;
}

// The k-th smallest eigenvalue (0-based) by bisection to full precision.
double kth_eigenvalue(const double* d, const double* e, int m, int k, double lo, double hi) {
    for (int it = 0; it < 200; ++it) {
        const double mid = 0.5 * (lo + hi);
        if (mid <= lo || mid >= hi) break;
        if (sturm_count(d, e, m, mid) > k)
            hi = mid;
        else
            lo = mid;
    }
    return 0.5 * (lo + hi);
}

void gershgorin(const double* d, const double* e, int m, double& lo, double& hi) {
    lo = std::numeric_limits<double>::infinity();
    hi = -lo;
    for (int i = 0; i < m; ++i) {
        const double r = (i > 0 ? std::abs(e[i - 1]) : 0.0) + (i + 1 < m ? std::abs(e[i]) : 0.0);
        lo = std::min(lo, d[i] - r);
        hi = std::max(hi, d[i] + r);
    }
    const double pad = 1e-14 * std::max({std::abs(lo), std::abs(hi), 1e-300}) + 1e-300;
    lo -= pad;
    hi += pad;
}

// Unit eigenvector of eigenvalue lam (inverse iteration with partial pivoting).
std::vector<double> inverse_iteration(const double* d, const double* e, int m, double lam) {
    std::vector<double> x(m, 1.0 / std::sqrt(static_cast<double>(m)));
    if (m == 1) return {1.0};
    double scale = 0.0;
    for (int i = 0; i < m; ++i) scale = std::max(scale, std::abs(d[i]) + (i + 1 < m ? std::abs(e[i]) : 0.0));
    const double mu = lam - std::max(scale, 1e-300) * 4e-15;
    for (int it = 0; it < 4; ++it) {
        // factor (T - mu) = P L U with rows i, i+1 possibly swapped; U has two superdiagonals
        std::vector<double> a(m), b(m, 0.0), c(m, 0.0), l(m, 0.0), rhs = x;
        std::vector<int> sw(m, 0);
        for (int i = 0; i < m; ++i) a[i] = d[i] - mu;
        for (int i = 0; i + 1 < m; ++i) b[i] = e[i];
        std::vector<double> sub(e, e + m - 1);
        for (int i = 0; i + 1 < m; ++i) {
            if (std::abs(a[i]) >= std::abs(sub[i])) {
                if (a[i] == 0.0) a[i] = 1e-300;
                l[i] = sub[i] / a[i];
                a[i + 1] -= l[i] * b[i];
                rhs[i + 1] -= l[i] * rhs[i];
            } else {
                sw[i] = 1;
                l[i] = a[i] / sub[i];
                // swap rows i and i+1
                const double ai1 = a[i + 1], bi1 = i + 2 < m ? b[i + 1] : 0.0;
                a[i] = sub[i];
                const double bi = b[i];
                b[i] = ai1;
                c[i] = bi1;
                a[i + 1] = bi - l[i] * ai1;
                if (i + 2 < m) b[i + 1] = -l[i] * bi1;
                std::swap(rhs[i], rhs[i + 1]);
                rhs[i + 1] -= l[i] * rhs[i];
            }
        }
        if (a[m - 1] == 0.0) a[m - 1] = 1e-300;
        std::vector<double> y(m);
        for (int i = m - 1; i >= 0; --i) {
            double s = rhs[i];
            if (i + 1 < m) s -= b[i] * y[i + 1];
            if (i + 2 < m) s -= c[i] * y[i + 2];
            y[i] = s / a[i];
        }
        double nrm = 0.0;
        for (double v : y) nrm += v * v;
        nrm = std::sqrt(nrm);
        for (int i = 0; i < m; ++i) x[i] = y[i] / nrm;
    }
    return x;
}

// All eigenvalues (ascending) and the first component of every unit eigenvector: implicit QL with
// Wilkinson shifts applied to the first row of the eigenvector matrix only.
void eig_first_row(std::vector<double> d, std::vector<double> e, std::vector<double>& vals, std::vector<double>& z0) {
    const int m = static_cast<int>(d.size());
    e.resize(m, 0.0);
    std::vector<double> z(m, 0.0);
    z[0] = 1.0;
    for (int l = 0; l < m; ++l) {
        for (int iter = 0;; ++iter) {
            int mm = l;
            for (; mm < m - 1; ++mm) {
                const double dd = std::abs(d[mm]) + std::abs(d[mm + 1]);
                if (std::abs(e[mm]) <= std::numeric_limits<double>::epsilon() * dd) break;
            }
            if (mm == l) break;
            if (iter > 100) throw Error(QB_ECUDA, "tridiagonal QL did not converge");
            double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
            double r = std::hypot(g, 1.0);
            g = d[mm] - d[l] + e[l] / (g + (g >= 0 ? r : -r));
            double s = 1.0, c = 1.0, p = 0.0;
            int i = mm - 1;
            for (; i >= l; --i) {
                double f = s * e[i];
                const double b = c * e[i];
                r = std::hypot(f, g);
                e[i + 1] = r;
                if (r == 0.0) {
                    d[i + 1] -= p;
                    e[mm] = 0.0;
                    break;
                }
                s = f / r;
                c = g / r;
                g = d[i + 1] - p;
                r = (d[i] - g) * s + 2.0 * c * b;
                p = s * r;
                d[i + 1] = g + p;
                g = c * r - b;
                f = z[i + 1];
                z[i + 1] = s * z[i] + c * f;
                z[i] = c * z[i] - s * f;
            }
            if (r == 0.0 && i >= l) continue;
            d[l] -= p;
            e[l] = g;
            e[mm] = 0.0;
        }
    }
    std::vector<int> order(m);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return d[a] < d[b]; });
    vals.resize(m);
    z0.resize(m);
    for (int j = 0; j < m; ++j) {
        vals[j] = d[order[j]];
        z0[j] = z[order[j]];
    }
}

// The lowest `count` eigenpairs' values and last components, and the top value.
struct Ends {
    std::vector<double> values, zlast;
    double top = 0.0;
};
Ends tridiag_ends(const std::vector<double>& alpha, const std::vector<double>& beta, int m, int count) {
    Ends out;
    std::vector<double> e(m > 1 ? m - 1 : 1, 0.0);
    for (int i = 0; i + 1 < m; ++i) e[i] = beta[i + 1];
    for (int i = 0; i < m; ++i)
        if (!std::isfinite(alpha[i]) || (i + 1 < m && !std::isfinite(e[i])))
            throw Error(QB_ECUDA, "tridiagonal eigensolve: non-finite entry");
    double lo, hi;
    gershgorin(alpha.data(), e.data(), m, lo, hi);
    count = std::max(1, std::min(count, m));
    for (int k = 0; k < count; ++k) {
        const double v = kth_eigenvalue(alpha.data(), e.data(), m, k, lo, hi);
        out.values.push_back(v);
        out.zlast.push_back(inverse_iteration(alpha.data(), e.data(), m, v)[m - 1]);
    }
    out.top = count == m ? out.values.back() : kth_eigenvalue(alpha.data(), e.data(), m, m - 1, lo, hi);
    return out;
}

// lowest_levels / leading_block / lowest_level (block_solve.cpp:335-385).
template <class Bound>
bool lowest_levels(int m, const double* w, Bound&& bound, double scale, std::vector<double>* out) {
    for (int j = 0; j < m;) {
        const double first = w[j];
        int i = j;
        bool converged = false;
        double value = first;
        for (; i < m && std::abs(w[i] - first) <= 1e-9 * scale; ++i)
            if (!converged && bound(i) <= 1e-7 * scale) {
                converged = true;
                value = w[i];
            }
        if (!converged) return false;
        if (out) out->push_back(value);
        return true;
    }
    return false;
}

int leading_block(const std::vector<double>& alpha, const std::vector<double>& beta, int m) {
    double scale = 0.0;
    for (int i = 0; i < m; ++i) {
        scale = std::max(scale, std::abs(alpha[i]));
        if (i + 1 < static_cast<int>(beta.size())) scale = std::max(scale, std::abs(beta[i + 1]));
    }
    for (int i = 1; i < m; ++i)
        if (std::abs(beta[i]) <= 1e-12 * scale) return i;
    return m;
}

bool lowest_level(const std::vector<double>& alpha, const std::vector<double>& beta, int m, std::vector<double>* out) {
    const double beta_m = static_cast<int>(beta.size()) > m ? std::abs(beta[m]) : 0.0;
    const Ends t = tridiag_ends(alpha, beta, m, 4);
    const int c = static_cast<int>(t.values.size());
    const double scale = std::max({std::abs(t.values.front()), std::abs(t.top), 1e-300});
    if (c < m && std::abs(t.values[c - 1] - t.values.front()) <= 1e-9 * scale) {
        // a cluster fills the four: every value and its vector
        std::vector<double> e(m - 1);
        for (int i = 0; i + 1 < m; ++i) e[i] = beta[i + 1];
        double lo, hi;
        gershgorin(alpha.data(), e.data(), m, lo, hi);
        std::vector<double> vals(m), zl(m);
        for (int k = 0; k < m; ++k) {
            vals[k] = kth_eigenvalue(alpha.data(), e.data(), m, k, lo, hi);
            zl[k] = inverse_iteration(alpha.data(), e.data(), m, vals[k])[m - 1];
        }
        return lowest_levels(m, vals.data(), [&](int j) { return beta_m * std::abs(zl[j]); }, scale, out);
    }
    return lowest_levels(c, t.values.data(), [&](int j) { return beta_m * std::abs(t.zlast[j]); }, scale, out);
}

// -------------------------------------------------------------------------------------------
// Seeds: the block lanes' staged Gaussian start (block_solve.cpp:268-277) and the FTLM sample
// vectors (sample_seed.h:37-89), drawn on the host exactly as the reference draws them.
// -------------------------------------------------------------------------------------------
// The reference draws each entry as Complex(nd(gen), nd(gen)); GCC evaluates those arguments right to
// left, so the imaginary part is the first draw. Written out here so no compiler reorders it.
template <class Gen> void gaussian_fill(std::vector<std::complex<double>>& v, Gen& gen) {
    std::normal_distribution<double> nd(0.0, 1.0);
    for (auto& c : v) {
        const double im = nd(gen);
        const double re = nd(gen);
        c = std::complex<double>(re, im);
    }
}

// The staged Gaussian start of dimension n from mt19937_64(seed): entry i = (re, im) with im drawn first, the
// stream of std::normal_distribution<double> over the generator (block_solve.cpp:263-277), bit for bit. Past 2^20
// entries the stream is produced in parallel. A normal pair comes from one accepted polar attempt: two raw 64-bit
// outputs u1, u2 give x = 2 c(u1) - 1, y = 2 c(u2) - 1 with c(u) = u / 2^64 (the largest double below 1 when that
// rounds to 1, as generate_canonical does), accepted when 0 < x^2 + y^2 <= 1; the first normal is y m, the second
// x m, m = sqrt(-2 log(r2) / r2); so entry i is (x_i m_i, y_i m_i) of the i-th accepted attempt. One thread runs
// the generator in order through a ring of chunk buffers and counts each chunk's accepted attempts (so it knows
// where the chunk's entries go); the other threads take the chunks in turn and form their entries in place.
inline double polar_canonical(std::uint64_t u) {
    const double r = static_cast<double>(u) / 18446744073709551616.0;
    return r >= 1.0 ? std::nextafter(1.0, 0.0) : r;
}

// MT19937-64 (M. Matsumoto and T. Nishimura, the 64-bit Mersenne Twister of 2000; the parameters std::mt19937_64
// is defined with), producing its outputs a state block (312 words) at a time: the same sequence as
// std::mt19937_64 seeded alike, faster than drawing word by word.
constexpr int kMtN = 312, kMtM = 156;

inline std::uint64_t mt_twist(std::uint64_t a, std::uint64_t b, std::uint64_t c) {
    const std::uint64_t x = (a & 0xFFFFFFFF80000000ULL) | (b & 0x7FFFFFFFULL);
    return c ^ (x >> 1) ^ ((0ULL - (x & 1ULL)) & 0xB5026F5AA96619E9ULL);
}

// One block: the state's kN words twisted in place, then the next kN outputs, tempered, into out. Written as plain
// loops so that the compiler vectorises them; mt_block_avx2 is the same code compiled for AVX2 (2.7x faster on the
// hosts here), chosen at run time.
#define QB_MT_BLOCK_BODY                                                                              \
    for (int i = 0; i < kMtN - kMtM; ++i) mt[i] = mt_twist(mt[i], mt[i + 1], mt[i + kMtM]);              \
    for (int i = kMtN - kMtM; i < kMtN - 1; ++i) mt[i] = mt_twist(mt[i], mt[i + 1], mt[i + kMtM - kMtN]); \
    mt[kMtN - 1] = mt_twist(mt[kMtN - 1], mt[0], mt[kMtM - 1]);                                       \
    for (int i = 0; i < kMtN; ++i) {                                                                  \
        std::uint64_t y = mt[i];                                                                      \
        y ^= (y >> 29) & 0x5555555555555555ULL;                                                       \
        y ^= (y << 17) & 0x71D67FFFEDA60000ULL;                                                       \
        y ^= (y << 37) & 0xFFF7EEE000000000ULL;                                                       \
        y ^= y >> 43;                                                                                 \
        out[i] = y;                                                                                   \
    }
inline void mt_block_plain(std::uint64_t* __restrict__ mt, std::uint64_t* __restrict__ out) { QB_MT_BLOCK_BODY }
__attribute__((target("avx2"))) inline void mt_block_avx2(std::uint64_t* __restrict__ mt,
                                                          std::uint64_t* __restrict__ out) {
    QB_MT_BLOCK_BODY
}
#undef QB_MT_BLOCK_BODY

inline bool host_has_avx2() {
    static const bool on = __builtin_cpu_supports("avx2");
    return on;
}

struct Mt64 {
    static constexpr int kN = kMtN;
    std::uint64_t mt[kN];
    explicit Mt64(std::uint64_t seed) {
        mt[0] = seed;
        for (int i = 1; i < kN; ++i) mt[i] = 6364136223846793005ULL * (mt[i - 1] ^ (mt[i - 1] >> 62)) + static_cast<std::uint64_t>(i);
    }
    // The next kN outputs, tempered, into out.
    void block(std::uint64_t* out) {
        if (host_has_avx2())
            mt_block_avx2(mt, out);
        else
            mt_block_plain(mt, out);
    }
};

// A polar attempt (u1, u2) with the exact generate_canonical arithmetic: x, y and r2, or -1 when rejected.
inline double polar_r2(std::uint64_t u1, std::uint64_t u2, double& x, double& y) {
    x = 2.0 * polar_canonical(u1) - 1.0;
    y = 2.0 * polar_canonical(u2) - 1.0;
    const double r2 = x * x + y * y;
    return (r2 > 1.0 || r2 == 0.0) ? -1.0 : r2;
}

// The top 52 bits of u as a double, exactly (the exponent trick: 2^52 + (u >> 12), less 2^52); u / 2^64 to within
// 2^-52, in integer and double operations the compiler vectorises.
inline double top52(std::uint64_t u) {
    const std::uint64_t b = 0x4330000000000000ULL | (u >> 12);
    double d;
    std::memcpy(&d, &b, 8);
    return d - 4503599627370496.0;
}
#define QB_POLAR_ESTIMATE_BODY                                                                        \
    for (std::size_t a = 0; a < count; ++a) {                                                         \
        const double xa = top52(r[2 * a]) * 0x1.0p-51 - 1.0;                                          \
        const double ya = top52(r[2 * a + 1]) * 0x1.0p-51 - 1.0;                                      \
        const double ra = xa * xa + ya * ya;                                                          \
        k += static_cast<std::size_t>(ra < 1.0);                                                      \
        near |= static_cast<int>(std::fabs(ra - 1.0) <= 1e-9) | static_cast<int>(ra <= 1e-9);         \
    }
inline void polar_estimate_plain(const std::uint64_t* __restrict__ r, std::size_t count, std::size_t& k, int& near) {
    QB_POLAR_ESTIMATE_BODY
}
__attribute__((target("avx2"))) inline void polar_estimate_avx2(const std::uint64_t* __restrict__ r, std::size_t count,
                                                                std::size_t& k, int& near) {
    QB_POLAR_ESTIMATE_BODY
}
#undef QB_POLAR_ESTIMATE_BODY

// The accepted polar attempts among `count` (raw output pairs at r): a cheap branch-free estimate of r2 (within
// 1e-15 of the exact one) decides every attempt unless one lies within 1e-9 of a boundary (r2 = 1 or r2 = 0), in
// which case the exact arithmetic recounts them all.
inline std::size_t polar_count(const std::uint64_t* r, std::size_t count) {
    std::size_t k = 0;
    int near = 0;
    if (host_has_avx2())
        polar_estimate_avx2(r, count, k, near);
    else
        polar_estimate_plain(r, count, k, near);
    if (!near) return k;
    k = 0;
    for (std::size_t a = 0; a < count; ++a) {
        double x, y;
        k += polar_r2(r[2 * a], r[2 * a + 1], x, y) >= 0.0 ? 1 : 0;
    }
    return k;
}

// A host vector of complex doubles left uninitialised (the draw writes every entry; its pages are touched by the
// threads that write them).
struct HostVec {
    std::unique_ptr<double[]> buf;
    std::size_t n = 0;
    explicit HostVec(std::size_t count) : buf(new double[2 * count]), n(count) {}
    std::complex<double>* data() { return reinterpret_cast<std::complex<double>*>(buf.get()); }
    const std::complex<double>* data() const { return reinterpret_cast<const std::complex<double>*>(buf.get()); }
    std::size_t size() const { return n; }
};

// The generator's ring of raw outputs, kept between draws: a fresh ring (77 MB with 16 host threads) cost its page
// faults on every draw. One ring per draw in flight; a draw takes an idle ring of its size or makes one.
struct SeedRings {
    std::mutex mu;
    std::vector<std::pair<std::size_t, std::unique_ptr<std::uint64_t[]>>> idle;
    std::pair<std::size_t, std::unique_ptr<std::uint64_t[]>> take(std::size_t n) {
        {
            std::lock_guard<std::mutex> lk(mu);
            for (auto it = idle.begin(); it != idle.end(); ++it)
                if (it->first == n) {
                    auto r = std::move(*it);
                    idle.erase(it);
                    return r;
                }
        }
        return {n, std::unique_ptr<std::uint64_t[]>(new std::uint64_t[n])};   // left uninitialised
    }
    void give(std::pair<std::size_t, std::unique_ptr<std::uint64_t[]>> r) {
        std::lock_guard<std::mutex> lk(mu);
        idle.push_back(std::move(r));
    }
};
inline SeedRings& seed_rings() {
    static SeedRings* r = new SeedRings;   // never destroyed: rings may outlive static destructors at exit
    return *r;
}

void staged_seed_into(std::complex<double>* v, std::size_t n, std::uint64_t seed) {
    if (n < (std::size_t{1} << 20)) {
        std::mt19937_64 gen(seed);
        std::normal_distribution<double> nd(0.0, 1.0);
        for (std::size_t i = 0; i < n; ++i) {
            const double im = nd(gen);
            const double re = nd(gen);
            v[i] = std::complex<double>(re, im);
        }
        return;
    }
    constexpr std::size_t kAtt = static_cast<std::size_t>(Mt64::kN) * 256;   // polar attempts per chunk
    const int nw = std::max(1, static_cast<int>(std::thread::hardware_concurrency()) - 1);
    const std::size_t ring = 4 * static_cast<std::size_t>(nw);
    auto ring_buf = seed_rings().take(ring * 2 * kAtt);
    std::uint64_t* const buf_p = ring_buf.second.get();
    struct Slot {
        std::atomic<std::size_t> chunk{~std::size_t{0}};   // the chunk it holds (ready), or none
        std::atomic<bool> busy{false};
        std::size_t off = 0;                              // where the chunk's first entry goes
    };
    std::vector<Slot> slots(ring);
    std::atomic<std::size_t> n_chunks{~std::size_t{0}}, next{0};
    std::vector<std::thread> pool;
    pool.emplace_back([&] {   // the generator, in order, counting each chunk's accepted attempts
        Mt64 gen(seed);
        std::size_t off = 0, c = 0;
        for (; off < n; ++c) {
            Slot& sl = slots[c % ring];
            while (sl.busy.load(std::memory_order_acquire)) std::this_thread::yield();
            sl.busy.store(true, std::memory_order_relaxed);
            std::uint64_t* r = buf_p + (c % ring) * 2 * kAtt;
            for (std::size_t b = 0; b < 2 * kAtt; b += Mt64::kN) gen.block(r + b);
            const std::size_t k = polar_count(r, kAtt);
            sl.off = off;
            off += k;
            sl.chunk.store(c, std::memory_order_release);
        }
        n_chunks.store(c, std::memory_order_release);
    });
    for (int t = 0; t < nw; ++t)
        pool.emplace_back([&] {
            for (std::size_t c = next++;; c = next++) {
                Slot& sl = slots[c % ring];
                for (;;) {   // wait for chunk c, or for the generator to stop short of it
                    if (sl.chunk.load(std::memory_order_acquire) == c) break;
                    const std::size_t nc = n_chunks.load(std::memory_order_acquire);
                    if (nc != ~std::size_t{0} && c >= nc) return;
                    std::this_thread::yield();
                }
                const std::uint64_t* r = buf_p + (c % ring) * 2 * kAtt;
                std::size_t i = sl.off;
                for (std::size_t a = 0; a < kAtt && i < n; ++a) {
                    double x, y;
                    const double r2 = polar_r2(r[2 * a], r[2 * a + 1], x, y);
                    if (r2 < 0.0) continue;
                    const double m = std::sqrt(-2 * std::log(r2) / r2);
                    v[i++] = std::complex<double>(x * m * 1.0 + 0.0, y * m * 1.0 + 0.0);
                }
                sl.chunk.store(~std::size_t{0}, std::memory_order_relaxed);
                sl.busy.store(false, std::memory_order_release);
            }
        });
    for (auto& t : pool) t.join();
    seed_rings().give(std::move(ring_buf));
}

HostVec staged_seed(std::size_t n, std::uint64_t seed) {
    HostVec hv(n);
    staged_seed_into(hv.data(), n, seed);
    return hv;
}

// A fresh random start on the device (no reference stream to follow): entry i = two unit normals by Box-Muller
// from a counter hash of (seed, i).
__device__ __forceinline__ std::uint64_t mix64(std::uint64_t z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}
__global__ void k_fresh_start(std::uint64_t n, std::uint64_t seed, double2* x) {
    for (std::uint64_t i = static_cast<std::uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<std::uint64_t>(gridDim.x) * blockDim.x) {
        const std::uint64_t a = mix64(seed + 0x9E3779B97F4A7C15ULL * (2 * i + 1));
        const std::uint64_t b = mix64(seed + 0x9E3779B97F4A7C15ULL * (2 * i + 2));
        const double u = (static_cast<double>(a >> 11) + 0.5) * 0x1.0p-53, w = static_cast<double>(b >> 11) * 0x1.0p-53;
        const double r = sqrt(-2.0 * log(u));
        double sn, cs;
        sincospi(2.0 * w, &sn, &cs);
        x[i] = make_double2(r * cs, r * sn);
    }
}

std::mt19937 sample_engine(std::uint64_t base_seed, std::uint64_t sample) {
    std::uint64_t z = base_seed + 0x9E3779B97F4A7C15ULL * (sample + 1);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    z = z ^ (z >> 31);
    return std::mt19937(static_cast<std::mt19937::result_type>(z));
}

// -------------------------------------------------------------------------------------------
// The single-vector recurrence on one sector.
// -------------------------------------------------------------------------------------------
struct Recurrence {
    const qb_sector* sec;
    const qb_program* prog;
    int dtype;
    std::uint64_t n;
    int max_iter;
    cudaStream_t st = nullptr;
    DevBuf<double2> w;                    // FP64 scratch (matvec output)
    DevBuf<unsigned char> vbuf[2];        // v_prev, v_curr (dtype)
    DevBuf<double> d_alpha, d_beta, d_ovl, d_partials;
    DevBuf<unsigned> d_counter;
    DevBuf<unsigned char> basis_block;          // kept Lanczos vectors, back to back (optional)
    std::vector<unsigned char*> basis;
    DevBuf<void*> d_basis;                      // their device pointers (full reorthogonalisation)
    DevBuf<double2> d_coeff, d_part;
    DevBuf<double> d_norms;                     // [0] before, [1] after
    DevBuf<int> d_flag;
    DevBuf<int> d_j;                            // the step index of the graph-ready steps
    cudaEvent_t ev = nullptr;
    int cur = 1;   // vbuf[cur] = v_j, vbuf[cur ^ 1] = v_{j-1}
    int host_j = 0;   // steps taken by advance()
    // captured batches of steps, by (steps, keep, reorth)
    struct Batch {
        int steps, keep, reorth;
        cudaGraphExec_t exec;
    };
    std::vector<Batch> graphs;

    std::size_t esize() const { return dtype == QB_C64 ? 8 : 16; }
    Scal scal() { return Scal{d_alpha.p, d_beta.p, d_ovl.p, d_partials.p, d_counter.p}; }

    Recurrence(const qb_sector* s, const qb_program* p, int dt, int mi) : sec(s), prog(p), dtype(dt), n(s->dim), max_iter(mi) {
        w.alloc(n);
        vbuf[0].alloc(n * esize());
        vbuf[1].alloc(n * esize());
        cuda_check(cudaMemset(vbuf[0].p, 0, n * esize()), "zero");
        d_alpha.alloc(std::max(1, max_iter));
        d_beta.alloc(max_iter + 1);
        cuda_check(cudaMemset(d_beta.p, 0, (max_iter + 1) * 8), "zero");
        d_ovl.alloc(2);
        d_partials.alloc(4 * kMaxRedBlocks);
        d_counter.alloc(1);
        cuda_check(cudaMemset(d_counter.p, 0, 4), "zero");
        d_j.alloc(1);
        cuda_check(cudaMemset(d_j.p, 0, 4), "zero");
        cuda_check(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), "event");
    }
    ~Recurrence() {
        if (ev) cudaEventDestroy(ev);
        if (!graphs.empty()) cudaStreamSynchronize(st);   // no batch of ours may still be running
        for (auto& g : graphs) cudaGraphExecDestroy(g.exec);
    }

    // v_0 = x / ||x|| from a device FP64 vector (x is overwritten scratch when x == w).
    double start_from_device(const double2* x) {
        const int nb = red_blocks(n);
        k_norm<<<nb, kThreads, 0, st>>>(n, x, scal());
        if (dtype == QB_C64)
            k_scale_into<float2><<<nb, kThreads, 0, st>>>(n, x, reinterpret_cast<float2*>(vbuf[cur].p), d_ovl.p);
        else
            k_scale_into<double2><<<nb, kThreads, 0, st>>>(n, x, reinterpret_cast<double2*>(vbuf[cur].p), d_ovl.p);
        cuda_check(cudaGetLastError(), "start");
        double nrm = 0.0;
        cuda_check(cudaMemcpyAsync(&nrm, d_ovl.p, 8, cudaMemcpyDeviceToHost, st), "norm read");
        cuda_check(cudaStreamSynchronize(st), "start");
        if (!(nrm > 0.0)) throw Error(QB_EINVAL, "lanczos: initial vector has non-positive norm");
        return nrm;
    }
    double start_from_host(const std::complex<double>* v0) {
        upload_host(w.p, v0, n * 16, st);
        return start_from_device(w.p);
    }

    void keep_current() {
        if (basis_block.n == 0) basis_block.alloc(static_cast<std::size_t>(max_iter + 1) * n * esize());
        if (basis.size() >= static_cast<std::size_t>(max_iter + 1)) throw Error(QB_EINVAL, "basis capacity exceeded");
        unsigned char* b = basis_block.p + basis.size() * n * esize();
        cuda_check(cudaMemcpyAsync(b, vbuf[cur].p, n * esize(), cudaMemcpyDeviceToDevice, st), "basis copy");
        basis.push_back(b);
    }

    // CGS2 of w against the kept basis V_0..V_j, then beta_{j+1} = ||w|| (lanczos.h:428-451, 481-484).
    void full_reorth(int j) {
        const int m = static_cast<int>(basis.size());
        if (m == 0) return;
        if (d_basis.n < static_cast<std::size_t>(max_iter + 1)) {
            d_basis.alloc(max_iter + 1);
            d_coeff.alloc(max_iter + 1);
            d_part.alloc(static_cast<std::size_t>(kMaxRedBlocks) + max_iter + 1);
            d_norms.alloc(2);
            d_flag.alloc(1);
        }
        std::vector<void*> ptrs(m);
        for (int k = 0; k < m; ++k) ptrs[k] = basis[k];
        cuda_check(cudaMemcpyAsync(d_basis.p, ptrs.data(), m * sizeof(void*), cudaMemcpyHostToDevice, st), "basis ptrs");
        cuda_check(cudaStreamSynchronize(st), "basis ptrs");
        const int nb = red_blocks(n);
        const int one = 1;
        cuda_check(cudaMemcpyAsync(d_flag.p, &one, 4, cudaMemcpyHostToDevice, st), "flag");
        for (int pass = 0; pass < 2; ++pass) {
            const int* flag = pass == 0 ? nullptr : d_flag.p;
            double* before = d_norms.p;
            k_norm_to<<<nb, kThreads, 0, st>>>(n, w.p, scal(), before, flag);
            if (dtype == QB_C64) {
                dot_many<float2>(n, m, reinterpret_cast<const float2* const*>(d_basis.p), w.p, d_coeff.p, d_part.p, flag, st);
                k_axpy_many<float2><<<nb, kThreads, 0, st>>>(n, m, reinterpret_cast<const float2* const*>(d_basis.p), d_coeff.p, w.p, flag);
            } else {
                dot_many<double2>(n, m, reinterpret_cast<const double2* const*>(d_basis.p), w.p, d_coeff.p, d_part.p, flag, st);
                k_axpy_many<double2><<<nb, kThreads, 0, st>>>(n, m, reinterpret_cast<const double2* const*>(d_basis.p), d_coeff.p, w.p, flag);
            }
            k_norm_to<<<nb, kThreads, 0, st>>>(n, w.p, scal(), d_norms.p + 1, flag);
            if (pass == 0) k_dgks_gate<<<1, 1, 0, st>>>(d_norms.p, d_norms.p + 1, d_flag.p);
        }
        k_norm_to<<<nb, kThreads, 0, st>>>(n, w.p, scal(), d_beta.p + j + 1, nullptr);
        cuda_check(cudaGetLastError(), "full reorthogonalisation");
        cuda_check(cudaStreamSynchronize(st), "full reorthogonalisation");
    }

    // Step j: w = H v_j, alpha_j, beta_{j+1}, v_{j+1}. Records the event after the scalars.
    // reorth: QB_REORTH_NONE, QB_REORTH_LOCAL, or QB_REORTH_FULL (against the kept basis)
    void step(int j, int reorth) {
        const int nb = red_blocks(n);
        void* vc = vbuf[cur].p;
        void* vp = vbuf[cur ^ 1].p;
        const int local = reorth == QB_REORTH_LOCAL;
        launch_walk_mixed(sec, sec, prog, vc, w.p, dtype, QB_C128, st);
        if (dtype == QB_C64) {
            rec_alpha<float2><<<nb, kThreads, 0, st>>>(n, j, w.p, static_cast<float2*>(vp), static_cast<float2*>(vc), scal());
            rec_beta<float2><<<nb, kThreads, 0, st>>>(n, j, local, w.p, static_cast<float2*>(vc), scal());
            if (reorth == QB_REORTH_FULL) full_reorth(j);
            rec_next<float2><<<nb, kThreads, 0, st>>>(n, j, w.p, static_cast<float2*>(vc), static_cast<float2*>(vp), scal());
        } else {
            rec_alpha<double2><<<nb, kThreads, 0, st>>>(n, j, w.p, static_cast<double2*>(vp), static_cast<double2*>(vc), scal());
            rec_beta<double2><<<nb, kThreads, 0, st>>>(n, j, local, w.p, static_cast<double2*>(vc), scal());
            if (reorth == QB_REORTH_FULL) full_reorth(j);
            rec_next<double2><<<nb, kThreads, 0, st>>>(n, j, w.p, static_cast<double2*>(vc), static_cast<double2*>(vp), scal());
        }
        cuda_check(cudaGetLastError(), "recurrence");
        cur ^= 1;
        cuda_check(cudaEventRecord(ev, st), "event");
    }

    // ---- graph-ready steps: the step index lives in d_j ----
    // One step j = host_j (reorth NONE or LOCAL): keep v_j in basis slot j when asked, then the walk and the three
    // passes reading j from d_j.
    void step_dev(bool keep, int reorth) {
        const int nb = red_blocks(n);
        void* vc = vbuf[cur].p;
        void* vp = vbuf[cur ^ 1].p;
        const int local = reorth == QB_REORTH_LOCAL;
        if (keep)
            k_keep_dev<<<nb, kThreads, 0, st>>>(n * esize(), d_j.p, static_cast<const unsigned char*>(vc),
                                                basis_block.p);
        launch_walk_mixed(sec, sec, prog, vc, w.p, dtype, QB_C128, st);
        if (dtype == QB_C64) {
            rec_alpha_dev<float2><<<nb, kThreads, 0, st>>>(n, d_j.p, w.p, static_cast<float2*>(vp), static_cast<float2*>(vc), scal());
            rec_beta_dev<float2><<<nb, kThreads, 0, st>>>(n, d_j.p, local, w.p, static_cast<float2*>(vc), scal());
            rec_next_dev<float2><<<nb, kThreads, 0, st>>>(n, d_j.p, w.p, static_cast<float2*>(vc), static_cast<float2*>(vp), scal());
        } else {
            rec_alpha_dev<double2><<<nb, kThreads, 0, st>>>(n, d_j.p, w.p, static_cast<double2*>(vp), static_cast<double2*>(vc), scal());
            rec_beta_dev<double2><<<nb, kThreads, 0, st>>>(n, d_j.p, local, w.p, static_cast<double2*>(vc), scal());
            rec_next_dev<double2><<<nb, kThreads, 0, st>>>(n, d_j.p, w.p, static_cast<double2*>(vc), static_cast<double2*>(vp), scal());
        }
        cuda_check(cudaGetLastError(), "recurrence");
        cur ^= 1;
    }

    // `count` more steps from host_j, in captured batches of `batch` steps (an even number, so the two working
    // vectors are back in place after each) while whole batches fit, the rest one launch sequence at a time.
    // keep: v_j goes to basis slot j (slot 0 must be kept before the first step). The same kernels in the same
    // order as step(), so the same scalars and vectors bit for bit.
    void advance(int count, bool keep, int reorth, int batch) {
        if (keep && basis_block.n == 0) basis_block.alloc(static_cast<std::size_t>(max_iter + 1) * n * esize());
        int done = 0;
        while (done < count) {
            if (batch >= 2 && batch % 2 == 0 && count - done >= batch) {
                launch_batch(batch, keep, reorth);
                done += batch;
            } else {
                step_dev(keep, reorth);
                ++done;
            }
        }
        if (keep)
            for (int j = host_j; j < host_j + count; ++j)
                if (j > 0) basis.push_back(basis_block.p + static_cast<std::size_t>(j) * n * esize());
        host_j += count;
    }

    void launch_batch(int steps, bool keep, int reorth) {
        cudaGraphExec_t exec = nullptr;
        for (const auto& g : graphs)
            if (g.steps == steps && g.keep == keep && g.reorth == reorth) exec = g.exec;
        if (!exec) {
            // one matvec into the scratch w first (the captured steps overwrite it), so that the walk's launch
            // shape is tuned before the capture records it
            launch_walk_mixed(sec, sec, prog, vbuf[cur].p, w.p, dtype, QB_C128, st);
            // captured on a private stream (nothing runs there), launched on st
            cudaStream_t cs = nullptr, saved = st;
            cuda_check(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking), "capture stream");
            cudaGraph_t graph = nullptr;
            const int cur0 = cur;
            st = cs;
            cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
            if (e == cudaSuccess) {
                try {
                    for (int i = 0; i < steps; ++i) step_dev(keep, reorth);
                } catch (...) {
                    cudaStreamEndCapture(cs, &graph);
                    if (graph) cudaGraphDestroy(graph);
                    st = saved;
                    cur = cur0;
                    cudaStreamDestroy(cs);
                    throw;
                }
                e = cudaStreamEndCapture(cs, &graph);
            }
            st = saved;
            cur = cur0;
            cudaStreamDestroy(cs);
            cuda_check(e, "step graph capture");
            e = cudaGraphInstantiate(&exec, graph, 0);
            cudaGraphDestroy(graph);
            cuda_check(e, "step graph instantiate");
            graphs.push_back(Batch{steps, keep ? 1 : 0, reorth, exec});
        }
        cuda_check(cudaGraphLaunch(exec, st), "step graph launch");
    }

    // alpha_j0 .. alpha_{j0+cnt-1} and beta_{j0+1} .. beta_{j0+cnt} in one read.
    void read_range(int j0, int cnt, double* a, double* b) {
        cuda_check(cudaMemcpyAsync(a, d_alpha.p + j0, cnt * 8, cudaMemcpyDeviceToHost, st), "alpha read");
        cuda_check(cudaMemcpyAsync(b, d_beta.p + j0 + 1, cnt * 8, cudaMemcpyDeviceToHost, st), "beta read");
        cuda_check(cudaStreamSynchronize(st), "scalars");
    }

    void read_scalars(int j, double& a, double& b) {
        double ab[2];
        cuda_check(cudaMemcpyAsync(&ab[0], d_alpha.p + j, 8, cudaMemcpyDeviceToHost, st), "alpha read");
        cuda_check(cudaMemcpyAsync(&ab[1], d_beta.p + j + 1, 8, cudaMemcpyDeviceToHost, st), "beta read");
        cuda_check(cudaStreamSynchronize(st), "scalars");
        a = ab[0];
        b = ab[1];
    }

    // x += c v, v a kept basis vector or the current one.
    void accumulate(double2* x, double c, const void* v) {
        const int nb = red_blocks(n);
        if (dtype == QB_C64)
            k_axpy_into<float2><<<nb, kThreads, 0, st>>>(n, c, static_cast<const float2*>(v), x);
        else
            k_axpy_into<double2><<<nb, kThreads, 0, st>>>(n, c, static_cast<const double2*>(v), x);
        cuda_check(cudaGetLastError(), "accumulate");
    }
};

// Run the scan from a prepared recurrence (start already loaded). Returns alpha / beta (host) of
// the steps done; `gate` true: the Paige-gated lowest-level exit after every step.
struct ScanOut {
    std::vector<double> alpha, beta;
    bool converged = false;
    double e0 = std::numeric_limits<double>::quiet_NaN();
    int matvecs = 0;
};

// Steps per captured graph for a sector of n states (0: launch step by step). Up to 2^20 states a step is a
// few short launches and the host's read of its scalars, so graphs of steps pay; a gated loop (one that tests
// convergence between steps) reads its scalars once per 8 steps and may run up to 7 steps past its stopping
// point, a cost that grows with the step time. QB_GRAPHS=0 turns graphs off. The k = 1 scan does not use
// them: it already tests step j while step j + 1 runs, and batches made it slower (3.57 against 3.15 ms on
// chain-20); the certified ground-state vector, whose test is heavier, gains 1.25x.
constexpr std::uint64_t kGraphMaxDim = 1ULL << 20;
inline int graph_batch(std::uint64_t n, bool gated) {
    const char* e = std::getenv("QB_GRAPHS");
    if ((e && *e == '0') || n > kGraphMaxDim) return 0;
    return gated ? 8 : 16;
}

ScanOut run_scan(Recurrence& R, int max_iter, int reorth, bool gate, double breakdown_tol, bool keep) {
    ScanOut o;
    o.beta.push_back(0.0);
    const int cap = static_cast<int>(std::min<std::uint64_t>(static_cast<std::uint64_t>(max_iter), R.n));
    if (reorth == QB_REORTH_FULL) keep = true;
    if (keep) R.keep_current();
    const int batch = (reorth == QB_REORTH_FULL || gate) ? 0 : graph_batch(R.n, false);
    if (batch > 0) {
        // graphs of `batch` steps; the scalars read once per batch (ungated: once)
        auto check = [&](int j) -> bool {
            const int m_all = j + 1;
            if (!gate) return false;
            const int m = leading_block(o.alpha, o.beta, m_all);
            if (m == m_all && m_all < 3) return false;
            return lowest_level(o.alpha, o.beta, m, nullptr);
        };
        std::vector<double> a, b;
        bool stop = false;
        int j = 0;
        while (j < cap && !stop) {
            const int cnt = gate ? std::min(batch, cap - j) : cap;
            R.advance(cnt, keep, reorth, batch);
            o.matvecs += cnt;
            a.resize(cnt);
            b.resize(cnt);
            R.read_range(j, cnt, a.data(), b.data());
            for (int i = 0; i < cnt && !stop; ++i) {
                o.alpha.push_back(a[i]);
                o.beta.push_back(b[i]);
                if (b[i] < breakdown_tol || check(j + i)) stop = true;
            }
            j += cnt;
        }
        if (keep && R.basis.size() > o.alpha.size()) R.basis.resize(o.alpha.size());
        if (gate && !o.alpha.empty()) {
            std::vector<double> vals;
            const int m = leading_block(o.alpha, o.beta, static_cast<int>(o.alpha.size()));
            o.converged = lowest_level(o.alpha, o.beta, m, &vals);
            if (!vals.empty()) o.e0 = vals.front();
        }
        return o;
    }
    // pipelined: step j runs while the host tests step j - 1's prefix
    int launched = 0;
    auto check = [&](int j) -> bool {   // after alpha_j, beta_{j+1} are known
        const int m_all = j + 1;
        if (!gate) return false;
        const int m = leading_block(o.alpha, o.beta, m_all);
        if (m == m_all && m_all < 3) return false;
        return lowest_level(o.alpha, o.beta, m, nullptr);
    };
    if (!gate) {
        // no test between steps: launch every step, read the scalars once, cut at the first breakdown
        for (int j = 0; j < cap; ++j) {
            if (keep && j > 0) R.keep_current();
            R.step(j, reorth);
            ++o.matvecs;
        }
        std::vector<double> a(cap), b(cap + 1);
        cuda_check(cudaMemcpyAsync(a.data(), R.d_alpha.p, cap * 8, cudaMemcpyDeviceToHost, R.st), "alpha read");
        cuda_check(cudaMemcpyAsync(b.data(), R.d_beta.p, (cap + 1) * 8, cudaMemcpyDeviceToHost, R.st), "beta read");
        cuda_check(cudaStreamSynchronize(R.st), "scan");
        for (int j = 0; j < cap; ++j) {
            o.alpha.push_back(a[j]);
            o.beta.push_back(b[j + 1]);
            if (b[j + 1] < breakdown_tol) break;
        }
        if (keep && R.basis.size() > o.alpha.size()) R.basis.resize(o.alpha.size());
        return o;
    }
    bool stop = false;
    for (int j = 0; j < cap && !stop; ++j) {
        if (launched == j) {
            R.step(j, reorth);
            ++launched;
            ++o.matvecs;
        }
        double a, b;
        R.read_scalars(j, a, b);
        o.alpha.push_back(a);
        o.beta.push_back(b);
        if (b < breakdown_tol) break;
        // launch step j + 1 before testing step j (the device stays busy while the host tests)
        if (j + 1 < cap) {
            if (keep) R.keep_current();
            R.step(j + 1, reorth);
            ++launched;
            ++o.matvecs;
        }
        if (check(j)) stop = true;
    }
    cuda_check(cudaStreamSynchronize(R.st), "scan");
    if (keep && static_cast<int>(R.basis.size()) > static_cast<int>(o.alpha.size())) R.basis.resize(o.alpha.size());
    if (gate && !o.alpha.empty()) {
        std::vector<double> vals;
        const int m = leading_block(o.alpha, o.beta, static_cast<int>(o.alpha.size()));
        o.converged = lowest_level(o.alpha, o.beta, m, &vals);
        if (!vals.empty()) o.e0 = vals.front();
    }
    return o;
}

double norm_bound(const qb_program* p) { return p->norm_bound > 0.0 ? p->norm_bound : 1.0; }

// The continued fraction of a Lanczos run from phi (include/ed/dynamics/cf.h:40-60, 142-147): the tridiagonal
// shifted by `shift` (NaN: its lowest eigenvalue), S(omega) = -Im G0 / pi with G built bottom-up,
// G0 = ||phi||^2 / (z - a_0 - G), z = omega + i eta. Returns the shift used.
double cf_spectrum(const std::vector<double>& alpha, const std::vector<double>& beta, int m, const double* omega,
                   int n_omega, double eta, double shift, double norm_sq, double* S) {
    std::vector<double> a(alpha.begin(), alpha.begin() + m);
    double sh = shift;
    if (std::isnan(sh)) {
        std::vector<double> e(std::max(1, m - 1));
        for (int i = 0; i + 1 < m; ++i) e[i] = beta[i + 1];
        double lo, hi;
        gershgorin(a.data(), e.data(), m, lo, hi);
        sh = kth_eigenvalue(a.data(), e.data(), m, 0, lo, hi);
    }
    for (auto& x : a) x -= sh;
    for (int iw = 0; iw < n_omega; ++iw) {
        const std::complex<double> z(omega[iw], eta);
        std::complex<double> G(0.0, 0.0);
        for (int nn = m - 1; nn >= 1; --nn) {
            const double b2 = beta[nn] * beta[nn];
            const std::complex<double> d = z - std::complex<double>(a[nn], 0.0) - G;
            G = std::abs(d) > 1e-300 ? std::complex<double>(b2, 0.0) / d : std::complex<double>(0.0, 0.0);
        }
        const std::complex<double> d = z - std::complex<double>(a[0], 0.0) - G;
        const std::complex<double> G0 =
            std::abs(d) > 1e-300 ? std::complex<double>(norm_sq, 0.0) / d : std::complex<double>(0.0, 0.0);
        S[iw] = -G0.imag() / 3.14159265358979323846;
    }
    return sh;
}

// max |S_m - S_{m/2}| / max S_m, the change of the fraction between half and full depth (cf.h:148-160).
double cf_change(const std::vector<double>& alpha, const std::vector<double>& beta, int m, const double* omega,
                 int n_omega, double eta, double shift, double norm_sq, const double* S) {
    if (m < 4) return 0.0;
    const int h = m / 2;
    std::vector<double> half(n_omega);
    cf_spectrum(alpha, beta, h, omega, n_omega, eta, shift, norm_sq, half.data());
    double smax = 0.0, dmax = 0.0;
    for (int i = 0; i < n_omega; ++i) {
        smax = std::max(smax, std::abs(S[i]));
        dmax = std::max(dmax, std::abs(S[i] - half[i]));
    }
    return smax > 0.0 ? dmax / smax : 0.0;
}

}  // namespace
}  // namespace qb
