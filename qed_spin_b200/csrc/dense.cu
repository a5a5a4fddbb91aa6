// =============================================================================
// dense.cu -- the dense tail on the device: the full spectra of many small blocks at once.
//
// The reference solves blocks up to dense_max_dim exactly (include/ed/sectors/thermal.h:35) through a pool of
// cusolverDnXsyevd streams (src/gpu/little_group.cu:185-188). Here every block is assembled on the device from
// the block matvec on identity columns (64 at a time) into one column-major buffer of all blocks, and one launch
// reduces them all, a CTA per block (largest first):
//   - Householder reflections to a Hermitian tridiagonal: for each column k, v = x - alpha e1 (alpha = -x0 /
//     |x0| ||x||) normalised, p = A22 v, w = p - (v^H p) v, A22 -= 2 (v w^H + w v^H) -- the O(n^2) products of
//     every step spread over the CTA's threads, v and w in shared memory;
//   - the moduli of the off-diagonal make a real symmetric tridiagonal with the same spectrum;
//   - every eigenvalue by Sturm-count bisection to full precision, the threads taking the indices in turn, so
//     the levels come out ascending.
// Blocks above kDenseDeviceMax states keep the host reduction (lanes.cu).
// =============================================================================
#include <algorithm>
#include <cmath>
#include <numeric>
#include <vector>

#include "qb_krylov.cuh"

namespace qb {

void launch_block_mixed(const qb_sector* row, const qb_sector* col, const qb_program* P, const void* in, void* out,
                        int k, int dtype_in, int dtype_out, cudaStream_t st);

namespace {

constexpr int kDenseDeviceMax = 1024;   // v and w in shared memory: 2 x 1024 x 16 bytes
constexpr int kDenseThreads = 256;

struct DenseBlock {
    unsigned long long a_off;   // the block's matrix at A + a_off (column-major, n x n)
    unsigned long long v_off;   // its levels at values + v_off
    int n;
};

// X[r][c] = (r == c0 + c) for kc identity columns interleaved by row.
__global__ void k_unit_cols(std::uint64_t n, int kc, std::uint64_t c0, double2* X) {
    const std::uint64_t total = n * kc;
    for (std::uint64_t t = static_cast<std::uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; t < total;
         t += static_cast<std::uint64_t>(gridDim.x) * blockDim.x)
        X[t] = make_double2(t / kc == c0 + t % kc ? 1.0 : 0.0, 0.0);
}

// A[:, c0 + c] = Y[:, c] for the kc columns of a block matvec (Y interleaved by row).
__global__ void k_put_cols(std::uint64_t n, int kc, std::uint64_t c0, const double2* Y, double2* A) {
    const std::uint64_t total = n * kc;
    for (std::uint64_t t = static_cast<std::uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; t < total;
         t += static_cast<std::uint64_t>(gridDim.x) * blockDim.x) {
        const std::uint64_t r = t / kc, c = t % kc;
        if (c0 + c < n) A[(c0 + c) * n + r] = Y[t];
    }
}

__device__ __forceinline__ double block_sum(double v, double* sm) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __syncthreads();
    if (lane == 0) sm[warp] = v;
    __syncthreads();
    double s = 0.0;
    for (int i = 0; i < static_cast<int>(blockDim.x >> 5); ++i) s += sm[i];   // the same order in every thread
    return s;
}

__device__ int sturm_below(const double* d, const double* e, int n, double x) {
    int c = 0;
    double q = d[0] - x;
    if (q < 0.0) ++c;
    for (int i = 1; i < n; ++i) {
        const double qq = q != 0.0 ? q : 2.2250738585072014e-308;
        q = d[i] - x - e[i - 1] * e[i - 1] / qq;
        if (q < 0.0) ++c;
    }
    return c;
}

__global__ void __launch_bounds__(kDenseThreads) k_dense_levels(const DenseBlock* blocks, double2* A_all,
                                                                double* values, double* tri) {
    __shared__ double2 v[kDenseDeviceMax], w[kDenseDeviceMax];
    __shared__ double sm[32];
    __shared__ double s_lo, s_hi;
    const DenseBlock B = blocks[blockIdx.x];
    const int n = B.n;
    double2* A = A_all + B.a_off;
    auto at = [&](int r, int c) -> double2& { return A[static_cast<std::size_t>(c) * n + r]; };
    for (int k = 0; k + 2 < n; ++k) {
        double part = 0.0;
        for (int i = k + 1 + threadIdx.x; i < n; i += blockDim.x) {
            const double2 x = at(i, k);
            part += x.x * x.x + x.y * x.y;
        }
        const double xn = sqrt(block_sum(part, sm));
        if (xn == 0.0) continue;
        const double2 x0 = at(k + 1, k);
        const double ax0 = sqrt(x0.x * x0.x + x0.y * x0.y);
        const double2 ph = ax0 > 0.0 ? make_double2(x0.x / ax0, x0.y / ax0) : make_double2(1.0, 0.0);
        const double2 alpha = make_double2(-ph.x * xn, -ph.y * xn);
        part = 0.0;
        for (int i = k + 1 + threadIdx.x; i < n; i += blockDim.x) {
            double2 y = at(i, k);
            if (i == k + 1) {
                y.x -= alpha.x;
                y.y -= alpha.y;
            }
            v[i] = y;
            part += y.x * y.x + y.y * y.y;
        }
        const double vn = sqrt(block_sum(part, sm));
        if (vn == 0.0) continue;
        for (int i = k + 1 + threadIdx.x; i < n; i += blockDim.x) {
            v[i].x /= vn;
            v[i].y /= vn;
        }
        __syncthreads();
        // p = A22 v (kept in w), K = Re v^H p
        part = 0.0;
        for (int i = k + 1 + threadIdx.x; i < n; i += blockDim.x) {
            double sr = 0.0, si = 0.0;
            for (int j = k + 1; j < n; ++j) {
                const double2 a = at(i, j), b = v[j];
                sr += a.x * b.x - a.y * b.y;
                si += a.x * b.y + a.y * b.x;
            }
            w[i] = make_double2(sr, si);
            part += v[i].x * sr + v[i].y * si;
        }
        const double K = block_sum(part, sm);
        for (int i = k + 1 + threadIdx.x; i < n; i += blockDim.x) {
            w[i].x -= K * v[i].x;
            w[i].y -= K * v[i].y;
        }
        __syncthreads();
        // A22 -= 2 (v w^H + w v^H), column by column across the threads
        const int m = n - k - 1;
        for (int t = threadIdx.x; t < m * m; t += blockDim.x) {
            const int i = k + 1 + t % m, j = k + 1 + t / m;
            const double2 vi = v[i], wi = w[i], vj = v[j], wj = w[j];
            double2& a = at(i, j);
            a.x -= 2.0 * ((vi.x * wj.x + vi.y * wj.y) + (wi.x * vj.x + wi.y * vj.y));
            a.y -= 2.0 * ((vi.y * wj.x - vi.x * wj.y) + (wi.y * vj.x - wi.x * vj.y));
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            at(k + 1, k) = alpha;
            at(k, k + 1) = make_double2(alpha.x, -alpha.y);
        }
        __syncthreads();
    }
    // the real tridiagonal: d = Re diag, e = |subdiagonal| (scratch of the block: 2n doubles)
    double* d = tri + 2 * B.v_off;
    double* e = d + n;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        d[i] = at(i, i).x;
        if (i + 1 < n) {
            const double2 s = at(i + 1, i);
            e[i] = sqrt(s.x * s.x + s.y * s.y);
        } else {
            e[i] = 0.0;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {   // Gershgorin bounds
        double lo = 1e300, hi = -1e300;
        for (int i = 0; i < n; ++i) {
            const double r = (i > 0 ? e[i - 1] : 0.0) + (i + 1 < n ? e[i] : 0.0);
            lo = fmin(lo, d[i] - r);
            hi = fmax(hi, d[i] + r);
        }
        const double pad = 1e-12 * fmax(fabs(lo), fabs(hi)) + 1e-300;
        s_lo = lo - pad;
        s_hi = hi + pad;
    }
    __syncthreads();
    for (int q = threadIdx.x; q < n; q += blockDim.x) {
        double lo = s_lo, hi = s_hi;
        for (int it = 0; it < 200; ++it) {
            const double mid = 0.5 * (lo + hi);
            if (mid <= lo || mid >= hi) break;
            if (sturm_below(d, e, n, mid) > q)
                hi = mid;
            else
                lo = mid;
        }
        values[B.v_off + q] = 0.5 * (lo + hi);
    }
}

}  // namespace

// The spectra of blocks of at most kDenseDeviceMax states, all on the device: block b's levels, ascending, at
// values[off[b] ...] (host). Returns false (nothing done) when a block is larger.
bool dense_levels_device(const qb_sector* const* secs, const qb_program* const* progs, int n_blocks,
                         const std::vector<std::size_t>& off, double* values) {
    std::uint64_t a_tot = 0, v_tot = 0;
    std::vector<DenseBlock> desc;
    for (int b = 0; b < n_blocks; ++b) {
        const std::uint64_t n = secs[b]->dim;
        if (n > static_cast<std::uint64_t>(kDenseDeviceMax)) return false;
        if (n == 0) continue;
        desc.push_back(DenseBlock{a_tot, off[b], static_cast<int>(n)});
        a_tot += n * n;
        v_tot = std::max<std::uint64_t>(v_tot, off[b] + n);
    }
    if (desc.empty()) return true;
    DevBuf<double2> A(a_tot);
    const int kc = 64;
    DevBuf<double2> X(static_cast<std::size_t>(kDenseDeviceMax) * kc), Y(static_cast<std::size_t>(kDenseDeviceMax) * kc);
    for (int b = 0, q = 0; b < n_blocks; ++b) {
        const std::uint64_t n = secs[b]->dim;
        if (n == 0) continue;
        double2* Ab = A.p + desc[q++].a_off;
        const int cols = static_cast<int>(std::min<std::uint64_t>(n, kc));
        for (std::uint64_t c0 = 0; c0 < n; c0 += cols) {
            k_unit_cols<<<red_blocks(n * cols), kThreads>>>(n, cols, c0, X.p);
            launch_block_mixed(secs[b], secs[b], progs[b], X.p, Y.p, cols, QB_C128, QB_C128, nullptr);
            k_put_cols<<<red_blocks(n * cols), kThreads>>>(n, cols, c0, Y.p, Ab);
        }
    }
    cuda_check(cudaGetLastError(), "dense assembly");
    std::vector<int> order(desc.size());
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int c) { return desc[a].n > desc[c].n; });
    std::vector<DenseBlock> sorted(desc.size());
    for (std::size_t i = 0; i < order.size(); ++i) sorted[i] = desc[order[i]];
    DevBuf<DenseBlock> dd;
    dd.upload(sorted.data(), sorted.size());
    DevBuf<double> dv(v_tot), tri(2 * v_tot);
    k_dense_levels<<<static_cast<unsigned>(sorted.size()), kDenseThreads>>>(dd.p, A.p, dv.p, tri.p);
    cuda_check(cudaGetLastError(), "dense levels");
    std::vector<double> hv(v_tot);
    cuda_check(cudaMemcpy(hv.data(), dv.p, v_tot * 8, cudaMemcpyDeviceToHost), "dense levels");
    for (const auto& d : desc) std::copy(hv.begin() + d.v_off, hv.begin() + d.v_off + d.n, values + d.v_off);
    return true;
}

}  // namespace qb
