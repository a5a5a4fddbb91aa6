// =============================================================================
// eigs_k.cu -- the k > 1 lane: the k lowest levels of a sector, and their vectors, on the device.
//
// Method: thick-restart Lanczos (K. Wu and H. Simon, SIAM J. Matrix Anal. Appl. 22 (2000) 602-616).
//   - A cycle extends a basis of m vectors by Lanczos steps, each fully reorthogonalised by two classical
//     Gram-Schmidt passes against the cycle's basis and the locked vectors. The step's scalars (alpha, beta)
//     are written to device memory by the kernels themselves; a breakdown (beta below 64 eps times the
//     scale) is marked on the device and the columns after it are zeroed. Nothing is read back inside a
//     cycle: its kernels are queued back to back and the host reads the cycle's scalars once at its end.
//   - At a restart the host solves the cycle's projected problem -- an arrowhead (the kept Ritz values and
//     their couplings to the residual direction) followed by the new tridiagonal -- and the device rotates
//     the basis onto the p lowest Ritz vectors; the last residual direction becomes column p.
//   - Once the `want` lowest Ritz pairs have residual bounds below the tolerance, they are formed and locked.
//   - Multiplicity: a Krylov space of one start holds one vector of each eigenspace. After the k lowest are
//     locked, a fresh random start orthogonalised against them searches once more below the k-th level; a
//     level found there joins the locked set (the highest then leaves it), until a search finds none.
//   - An invariant subspace (breakdown) gives exact pairs; a fresh deflated start then continues the search.
//
// FP32 storage (dtype QB_C64): the basis and the locked vectors are stored as complex64 (the arithmetic and
// all scalars stay FP64) and converged to 1e-6 of the scale, the level the storage rounding allows. With
// refine != 0 each returned pair is then refined in FP64, lowest first: a restarted Lanczos search for one
// level (cycles of 16 vectors), started from the pair's vector and deflated against the pairs refined before
// it, to the FP64 lock tolerance. A multiplet's members refine one after another inside their eigenspace.
//
// The contract is the reference's krylov_schur_lane (src/engine/block_solve.cpp:433-510): the k lowest
// levels of the block, ascending, each converged to a residual of kLockRel (1e-10) times the coefficient sum,
// multiplicities resolved, from the staged Gaussian start of seed 0x51ED0B70 (block_solve.cpp:263); the
// method and its code are this file's own.
// =============================================================================
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdlib>
#include <limits>
#include <memory>
#include <random>
#include <string>
#include <type_traits>
#include <vector>

#include "qb_krylov.cuh"

namespace qb {
namespace {

using cd = std::complex<double>;

constexpr std::uint64_t kStartSeed = 0x51ED0B70ULL;      // staged_seed of the k > 1 lane (block_solve.cpp:263)
constexpr std::uint64_t kFreshSeed = 0x7E57A27ULL;        // fresh starts of this lane (any seed serves)
constexpr double kLockTol = 1e-10;                       // kLockRel (include/ed/core/numerics.h:25)
constexpr double kLockTolF32 = 1e-6;                     // the FP32-storage phase, before the FP64 refinement
constexpr double kFloorRel = 64.0 * std::numeric_limits<double>::epsilon();   // kBreakdownRel (numerics.h:23)

// ---- kernels ----

// alpha[j] = -Re coef[j] (first pass) or alpha[j] -= Re coef[j] (second pass): the diagonal of the step.
__global__ void k_take_alpha(const double2* coef, int at, int j, int first, double* alpha) {
    if (first)
        alpha[j] = -coef[at].x;
    else
        alpha[j] -= coef[at].x;
}

// Partial inner products of w with up to 8 basis vectors per block: block (x, y) sums conj(V_b[i]) w[i] over chunk
// x of the rows for b in [8y, 8y + 8) and writes them to part[b * chunks + x] (k_dot_sum then adds the chunks in
// order and negates). w is read once per 8 vectors. flag (may be null): nothing is done when *flag == 0.
constexpr int kDotVecs = 8;
template <class T>
__global__ void k_dots8(std::uint64_t n, int m, const T* const* basis, const double2* w, double2* part, int chunks,
                        const int* flag) {
    if (flag && *flag == 0) return;
    __shared__ double sm[2 * kDotVecs * 32];
    const int b0 = blockIdx.y * kDotVecs;
    const int nv = min(kDotVecs, m - b0);
    const std::uint64_t per = (n + chunks - 1) / chunks;
    const std::uint64_t lo = static_cast<std::uint64_t>(blockIdx.x) * per;
    const std::uint64_t hi = lo + per < n ? lo + per : n;
    double acc[2 * kDotVecs];
#pragma unroll
    for (int q = 0; q < 2 * kDotVecs; ++q) acc[q] = 0.0;
    const T* vb[kDotVecs];
#pragma unroll
    for (int q = 0; q < kDotVecs; ++q) vb[q] = q < nv ? basis[b0 + q] : nullptr;
    for (std::uint64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
        const double2 y = w[i];
#pragma unroll
        for (int q = 0; q < kDotVecs; ++q)
            if (q < nv) {
                const double2 v = V<T>::ld(vb[q], i);
                acc[2 * q] += v.x * y.x + v.y * y.y;
                acc[2 * q + 1] += v.x * y.y - v.y * y.x;
            }
    }
    block_reduce<2 * kDotVecs>(acc, sm);
    if (threadIdx.x == 0)
        for (int q = 0; q < nv; ++q)
            part[static_cast<std::size_t>(b0 + q) * chunks + blockIdx.x] = make_double2(acc[2 * q], acc[2 * q + 1]);
}

// w -= alpha_j v_j + beta_j v_{j-1} (vp null: no beta term), the scalars read from device memory.
template <class T>
__global__ void k_recur(std::uint64_t n, double2* w, const T* vj, const T* vp, const double* alpha, const double* beta) {
    const double a = *alpha, b = vp ? *beta : 0.0;
    for (std::uint64_t i = static_cast<std::uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<std::uint64_t>(gridDim.x) * blockDim.x) {
        const double2 x = V<T>::ld(vj, i);
        double2 y = w[i];
        y.x -= a * x.x;
        y.y -= a * x.y;
        if (vp) {
            const double2 z = V<T>::ld(vp, i);
            y.x -= b * z.x;
            y.y -= b * z.y;
        }
        w[i] = y;
    }
}

// The DGKS gate of the reorthogonalisation pass just made: *flag = 1 (a second pass) when the projections it
// removed carry more than 1 - kappa^2 of the squared norm w had before it (||w||^2 before = *before^2; the
// projections on an orthonormal basis: sum |coef|^2), else 0. With `at` >= 0, alpha[j] -= Re coef[at].
__global__ void k_gate(const double2* coef, int nb, const double* before, int* flag, int at, int j, double* alpha) {
    double s = 0.0;
    for (int i = 0; i < nb; ++i) s += coef[i].x * coef[i].x + coef[i].y * coef[i].y;
    const double b2 = (*before) * (*before);
    *flag = s > (1.0 - 0.5) * b2 ? 1 : 0;   // kappa = 1/sqrt(2)
    if (at >= 0) alpha[j] -= coef[at].x;
}

// alpha[j] -= Re coef[at] when *flag != 0 (the gated second pass's correction).
__global__ void k_take_alpha_gated(const double2* coef, int at, int j, const int* flag, double* alpha) {
    if (*flag) alpha[j] -= coef[at].x;
}

// out = w / beta stored as T; a beta at or below floor marks a breakdown at step j (the smallest j wins) and
// zeroes the column, so the rest of the cycle runs on zeros.
template <class T>
__global__ void k_next_col(std::uint64_t n, const double2* w, T* out, const double* beta, double floor, int* brk,
                           int j) {
    const double b = *beta;
    const bool broken = !(b > floor);
    if (broken && blockIdx.x == 0 && threadIdx.x == 0) atomicMin(brk, j);
    const double s = broken ? 0.0 : 1.0 / b;
    for (std::uint64_t i = static_cast<std::uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<std::uint64_t>(gridDim.x) * blockDim.x) {
        const double2 a = w[i];
        V<T>::st(out, i, a.x * s, a.y * s);
    }
}

// out = x / *nrm stored as T (a start vector).
template <class T> __global__ void k_unit_into(std::uint64_t n, const double2* x, T* out, const double* nrm) {
    const double s = 1.0 / *nrm;
    for (std::uint64_t i = static_cast<std::uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<std::uint64_t>(gridDim.x) * blockDim.x) {
        const double2 a = x[i];
        V<T>::st(out, i, a.x * s, a.y * s);
    }
}

// out[:, c] = sum_r V[:, r] S[r, c] for c in [c0, c0 + kRotW) and c < cols: V columns of stride n stored as T,
// S real column-major mm x cols, out columns of stride n stored as T.
constexpr int kRotW = 8;
template <class T>
__global__ void k_rotate_real(std::uint64_t n, int mm, int cols, int c0, const T* Vb, const double* S, T* out) {
    extern __shared__ double Ss[];
    const int nc = min(kRotW, cols - c0);
    for (int t = threadIdx.x; t < mm * nc; t += blockDim.x) Ss[t] = S[static_cast<std::size_t>(c0) * mm + t];
    __syncthreads();
    for (std::uint64_t i = static_cast<std::uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<std::uint64_t>(gridDim.x) * blockDim.x) {
        double2 acc[kRotW];
#pragma unroll
        for (int c = 0; c < kRotW; ++c) acc[c] = make_double2(0.0, 0.0);
        for (int r = 0; r < mm; ++r) {
            const double2 v = V<T>::ld(Vb + static_cast<std::size_t>(r) * n, i);
#pragma unroll
            for (int c = 0; c < kRotW; ++c)
                if (c < nc) {
                    const double s = Ss[c * mm + r];
                    acc[c].x += s * v.x;
                    acc[c].y += s * v.y;
                }
        }
#pragma unroll
        for (int c = 0; c < kRotW; ++c)
            if (c < nc) V<T>::st(out + static_cast<std::size_t>(c0 + c) * n, i, acc[c].x, acc[c].y);
    }
}

// ---- small dense problems on the host ----

// Eigenpairs of a Hermitian m x m matrix (column-major): cyclic Jacobi, each rotation made real by a phase
// on its second index first; values ascending, vectors column-major.
void hermitian_eig(std::vector<cd> A, int m, std::vector<double>& vals, std::vector<cd>& vecs) {
    auto at = [&](int r, int c) -> cd& { return A[static_cast<std::size_t>(c) * m + r]; };
    std::vector<cd> Q(static_cast<std::size_t>(m) * m, cd(0.0, 0.0));
    for (int i = 0; i < m; ++i) Q[static_cast<std::size_t>(i) * m + i] = 1.0;
    double fro = 0.0;
    for (const cd& z : A) fro += std::norm(z);
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0.0;
        for (int c = 0; c < m; ++c)
            for (int r = 0; r < c; ++r) off += std::norm(at(r, c));
        if (off == 0.0 || off <= 1e-30 * fro) break;
        for (int p = 0; p + 1 < m; ++p)
            for (int q = p + 1; q < m; ++q) {
                const double mag = std::abs(at(p, q));
                if (mag == 0.0) continue;
                const cd ph = at(p, q) / mag;                 // a_pq = mag * ph
                const double app = at(p, p).real(), aqq = at(q, q).real();
                const double th = (aqq - app) / (2.0 * mag);
                const double t = (th >= 0.0 ? 1.0 : -1.0) / (std::abs(th) + std::sqrt(th * th + 1.0));
                const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
                const cd phc = std::conj(ph);
                for (int r = 0; r < m; ++r) {             // A <- A D R, D = diag(1, conj(ph)) on (p, q)
                    const cd x = at(r, p), y = at(r, q) * phc;
                    at(r, p) = c * x - s * y;
                    at(r, q) = s * x + c * y;
                }
                for (int r = 0; r < m; ++r) {             // A <- R^T D^H A
                    const cd x = at(p, r), y = at(q, r) * ph;
                    at(p, r) = c * x - s * y;
                    at(q, r) = s * x + c * y;
                }
                at(p, q) = at(q, p) = cd(0.0, 0.0);
                for (int r = 0; r < m; ++r) {             // Q <- Q D R
                    cd& qp = Q[static_cast<std::size_t>(p) * m + r];
                    cd& qq = Q[static_cast<std::size_t>(q) * m + r];
                    const cd x = qp, y = qq * phc;
                    qp = c * x - s * y;
                    qq = s * x + c * y;
                }
            }
    }
    std::vector<int> order(m);
    for (int i = 0; i < m; ++i) order[i] = i;
    std::sort(order.begin(), order.end(), [&](int a, int b) { return at(a, a).real() < at(b, b).real(); });
    vals.resize(m);
    vecs.assign(static_cast<std::size_t>(m) * m, cd(0.0, 0.0));
    for (int c = 0; c < m; ++c) {
        vals[c] = at(order[c], order[c]).real();
        std::copy(Q.begin() + static_cast<std::size_t>(order[c]) * m,
                  Q.begin() + static_cast<std::size_t>(order[c] + 1) * m, vecs.begin() + static_cast<std::size_t>(c) * m);
    }
}

// Eigenpairs of a real symmetric m x m matrix (column-major), ascending, through the Hermitian solver.
void symmetric_eig(const std::vector<double>& A, int m, std::vector<double>& vals, std::vector<double>& vecs) {
    std::vector<cd> Ac(A.begin(), A.end());
    std::vector<cd> vc;
    hermitian_eig(std::move(Ac), m, vals, vc);
    vecs.resize(vc.size());
    for (std::size_t i = 0; i < vc.size(); ++i) vecs[i] = vc[i].real();   // real to rounding for a real matrix
}

// ---- the lane ----

struct LevelsOut {
    std::vector<double> values;
    std::vector<DevBuf<double2>> vectors;   // FP64 copies, filled when asked
    bool converged = false;
    int matvecs = 0, cycles = 0, refine_rounds = 0;
};

template <class T> constexpr int dtype_of();
template <> constexpr int dtype_of<double2>() { return QB_C128; }
template <> constexpr int dtype_of<float2>() { return QB_C64; }

template <class T> class ThickRestart {
public:
    // cycle: the basis length of a cycle (0: 3k + 10, at least 16; QB_EIGS_CYCLE overrides), shortened to fit 85%
    // of the free memory. Short cycles keep the full reorthogonalisation cheap: over a sweep of 16 to 44 vectors on
    // the chain-32 sector (k = 2) and the chain-20 sector (k = 4) the shortest took the fewest matvecs and time.
    ThickRestart(const qb_sector* sec, const qb_program* prog, int k, std::uint64_t budget, std::size_t cycle = 0)
        : sec_(sec), prog_(prog), n_(sec->dim), k_(k), budget_(budget), scale_(norm_bound(prog)),
          floor_(kFloorRel * norm_bound(prog)), nb_(red_blocks(sec->dim)) {
        const std::size_t es = sizeof(T);
        if (cycle == 0) cycle = env_size("QB_EIGS_CYCLE");
        std::size_t m = cycle > 0 ? cycle
                                  : std::max<std::size_t>(3 * static_cast<std::size_t>(k) + 10, 16);
        keep_frac_ = env_size("QB_EIGS_KEEP");
        m = static_cast<std::size_t>(std::min<std::uint64_t>(m, n_));
        const double free_b = 0.85 * static_cast<double>(available_bytes());
        auto need = [&](std::size_t mm) {   // basis + kept Ritz vectors + locked + the FP64 work vector
            return (static_cast<double>(mm + 1 + keep_for(mm) + 2 * static_cast<std::size_t>(k)) * es + 16.0) *
                   static_cast<double>(n_);
        };
        while (m > static_cast<std::size_t>(k) + 4 && m > 2 && need(m) > free_b) --m;
        if (need(m) > free_b)
            throw Error(QB_ENOMEM, "eigs: " + std::to_string(m) + " Lanczos vectors of dimension " + std::to_string(n_) +
                                       " do not fit the free device memory");
        m_ = std::max<std::size_t>(1, m);
        p_ = keep_for(m_);
        Vb_.alloc((m_ + 1) * n_);
        U_.alloc(std::max<std::size_t>(p_, 1) * n_);
        w_.alloc(n_);
        const std::size_t cap = m_ + 1 + 2 * static_cast<std::size_t>(k) + 8;
        ptrs_.alloc(cap);
        coef_.alloc(cap);
        arrow_.alloc(cap);
        flag_.alloc(1);
        part_.alloc(static_cast<std::size_t>(kMaxRedBlocks) + cap * static_cast<std::size_t>(dot_chunks(n_, 1)));
        alpha_.alloc(m_ + 1);
        beta_.alloc(m_ + 2);
        slots_.alloc(8);
        brk_.alloc(1);
        red_part_.alloc(4 * kMaxRedBlocks);
        red_cnt_.alloc(1);
        cuda_check(cudaMemset(red_cnt_.p, 0, sizeof(unsigned)), "zero");
        S_.alloc(m_ * m_);
    }

    // The k lowest pairs: values ascending (fewer when the block is smaller); vectors kept as T.
    void run(LevelsOut& out) {
        start_from_host(staged_seed(n_, kStartSeed).data());
        std::mt19937_64 fresh(kFreshSeed);
        int null_starts = 0;
        bool stalled = false;
        // the main search and, after an invariant subspace, fresh deflated starts for what is left
        while (static_cast<int>(locked_vals_.size()) < k_) {
            const int got = search(k_ - static_cast<int>(locked_vals_.size()), std::numeric_limits<double>::infinity());
            if (exhausted_) break;
            if (got < 0) {   // the start vanished against the locked vectors: the block is exhausted
                if (++null_starts >= 2) break;
            } else if (got == 0 || budget_exhausted()) {
                stalled = static_cast<int>(locked_vals_.size()) < k_ && !exhausted_;
                break;
            }
            if (static_cast<int>(locked_vals_.size()) < k_) start_fresh(fresh);
        }
        // multiplicity: search below the k-th level from fresh deflated starts until nothing is found
        for (int round = 0; round < k_ && !locked_vals_.empty() && !exhausted_ && !budget_exhausted(); ++round) {
            const double top = *std::max_element(locked_vals_.begin(), locked_vals_.end());
            const double gap = std::max(10.0 * tol(), 1e-8 * std::abs(top));
            start_fresh(fresh);
            const std::size_t before = locked_vals_.size();
            const int got = search(1, top - gap);
            if (got <= 0 || locked_vals_.size() == before) break;
            if (locked_vals_.back() >= top - gap) {   // not below: the level was already there
                drop_locked(locked_vals_.size() - 1);
                break;
            }
            while (static_cast<int>(locked_vals_.size()) > k_) {
                const auto hi = std::max_element(locked_vals_.begin(), locked_vals_.end()) - locked_vals_.begin();
                drop_locked(static_cast<std::size_t>(hi));
            }
        }
        std::vector<std::size_t> order(locked_vals_.size());
        for (std::size_t i = 0; i < order.size(); ++i) order[i] = i;
        std::sort(order.begin(), order.end(), [&](std::size_t a, std::size_t b) { return locked_vals_[a] < locked_vals_[b]; });
        for (std::size_t i : order) {
            if (static_cast<int>(out.values.size()) >= k_) break;
            out.values.push_back(locked_vals_[i]);
            sorted_.push_back(locked_[i].p);
        }
        out.converged = !stalled && (static_cast<int>(out.values.size()) >= k_ || exhausted_);
        out.matvecs += matvecs_;
        out.cycles += cycles_;
    }

    // The returned vectors in ascending order of their levels (valid while this object lives).
    const std::vector<T*>& sorted_vectors() const { return sorted_; }

    // One level refined from an approximate eigenvector (device, FP64): a search for the lowest level of the
    // space deflated against the levels refined so far, started from x. Returns false when the budget ran out
    // first (the best pair so far is kept) or x vanishes against the refined levels.
    bool refine_from(const double2* x) {
        cuda_check(cudaMemcpy(w_.p, x, n_ * 16, cudaMemcpyDeviceToDevice), "refine start");
        have_start_ = true;
        const std::size_t before = locked_vals_.size();
        const int got = search(1, std::numeric_limits<double>::infinity(), true);
        return got == 1 && locked_vals_.size() == before + 1;
    }
    const std::vector<double>& locked_values() const { return locked_vals_; }
    const T* locked_vector(std::size_t i) const { return locked_[i].p; }
    int matvecs() const { return matvecs_; }

private:
    // kept Ritz vectors at a restart: about a third of the cycle (QB_EIGS_KEEP: that many instead)
    std::size_t keep_for(std::size_t m) const {
        if (m <= 2) return 1;
        if (keep_frac_ > 0) return std::min<std::size_t>(m - 1, std::max<std::size_t>(keep_frac_, static_cast<std::size_t>(k_)));
        return std::min<std::size_t>(m - 1, std::max<std::size_t>(m / 3, static_cast<std::size_t>(k_) + 4));
    }
    static std::size_t env_size(const char* name) {   // a tuning override from the environment (0: none)
        const char* e = std::getenv(name);
        return e ? static_cast<std::size_t>(std::strtoull(e, nullptr, 10)) : 0;
    }
    double tol() const { return (std::is_same<T, float2>::value ? kLockTolF32 : kLockTol) * scale_; }
    bool budget_exhausted() const { return static_cast<std::uint64_t>(matvecs_) >= budget_; }
    T* col(std::size_t j) { return Vb_.p + j * n_; }
    Scal red() { return Scal{nullptr, nullptr, nullptr, red_part_.p, red_cnt_.p}; }

    void start_from_host(const cd* v) {
        upload_host(w_.p, v, n_ * 16, nullptr);
        have_start_ = true;
    }
    void start_fresh(std::mt19937_64& gen) {   // drawn on the device from a seed the lane's generator gives
        k_fresh_start<<<nb_, kThreads>>>(n_, gen(), w_.p);
        cuda_check(cudaGetLastError(), "fresh start");
        have_start_ = true;
    }

    // Device pointer table: the locked vectors, then the cycle's columns 0..m.
    void write_ptrs() {
        std::vector<const void*> h;
        for (const auto& b : locked_) h.push_back(b.p);
        for (std::size_t j = 0; j <= m_; ++j) h.push_back(col(j));
        cuda_check(cudaMemcpy(ptrs_.p, h.data(), h.size() * sizeof(void*), cudaMemcpyHostToDevice), "pointers");
    }
    const T* const* basis() const { return reinterpret_cast<const T* const*>(ptrs_.p); }

    // coef_[0, nb) = -<table entry i, w> for the nb table entries from `from` (gated by flag when non-null).
    void dots(int from, int nb, const int* flag) {
        const int chunks = dot_chunks(n_, (nb + kDotVecs - 1) / kDotVecs);
        k_dots8<T><<<dim3(chunks, (nb + kDotVecs - 1) / kDotVecs), kThreads>>>(n_, nb, basis() + from, w_.p, part_.p,
                                                                               chunks, flag);
        k_dot_sum<<<dot_sum_blocks(nb), 32 * kDotSumWarps>>>(nb, chunks, part_.p, coef_.p, flag);
    }

    // One reorthogonalisation pass of w against the first nb table entries, then a second when the DGKS gate
    // asks (its decision on the device); with at >= 0 the pass's overlap with entry `at` corrects alpha[j].
    void reorth(int nb, int at, int j) {
        if (nb == 0) return;
        k_norm_to<<<nb_, kThreads>>>(n_, w_.p, red(), slots_.p + 1, nullptr);
        dots(0, nb, nullptr);
        k_axpy_many<T><<<nb_, kThreads>>>(n_, nb, basis(), coef_.p, w_.p, nullptr);
        k_gate<<<1, 1>>>(coef_.p, nb, slots_.p + 1, flag_.p, at, j, alpha_.p);
        dots(0, nb, flag_.p);
        k_axpy_many<T><<<nb_, kThreads>>>(n_, nb, basis(), coef_.p, w_.p, flag_.p);
        if (at >= 0) k_take_alpha_gated<<<1, 1>>>(coef_.p, at, j, flag_.p, alpha_.p);
    }

    // Step j of a cycle from w = A v_j: alpha_j = Re <v_j, w>; w -= alpha_j v_j and the recurrence's coupling to
    // the earlier basis (beta_j v_{j-1}, or the kept Ritz vectors' arrow after a restart); then the
    // reorthogonalisation against the whole basis and the locked vectors, which now removes only rounding-level
    // components (alpha_j takes its overlap too).
    void step_projections(int L, std::size_t j, std::size_t p) {
        const int jj = static_cast<int>(j);
        dots(L + jj, 1, nullptr);
        k_take_alpha<<<1, 1>>>(coef_.p, 0, jj, 1, alpha_.p);
        const T* vp = (j > p) ? col(j - 1) : nullptr;
        k_recur<T><<<nb_, kThreads>>>(n_, w_.p, col(j), vp, alpha_.p + j, beta_.p + j);
        if (j == p && p > 0)   // the arrow: w -= sum_i s_i u_i over the kept Ritz vectors (coefficients staged)
            k_axpy_many<T><<<nb_, kThreads>>>(n_, static_cast<int>(p), basis() + L, arrow_.p, w_.p, nullptr);
        reorth(L + jj + 1, L + jj, jj);
    }

    // One search from the start in w_: lock up to `want` of the lowest pairs. Returns the number locked, or -1
    // when the start is null against the locked vectors. give_up: a first cycle whose lowest Ritz value is at
    // or above it ends the search with nothing locked.
    int search(int want, double give_up, bool lock_best = false) {
        if (!have_start_) return -1;
        have_start_ = false;
        write_ptrs();
        const int L = static_cast<int>(locked_.size());
        reorth(L, -1, 0);
        k_norm_to<<<nb_, kThreads>>>(n_, w_.p, red(), slots_.p, nullptr);
        double nrm = 0.0;
        cuda_check(cudaMemcpy(&nrm, slots_.p, 8, cudaMemcpyDeviceToHost), "start norm");
        if (!(nrm > 1e-13 * std::max(1.0, std::sqrt(static_cast<double>(n_))))) return -1;
        k_unit_into<T><<<nb_, kThreads>>>(n_, w_.p, col(0), slots_.p);
        std::size_t p = 0;
        std::vector<double> theta, arrow;
        for (bool first = true;; first = false) {
            // extend the basis from column p to m, all scalars on the device
            const int big = std::numeric_limits<int>::max();
            cuda_check(cudaMemcpy(brk_.p, &big, sizeof(int), cudaMemcpyHostToDevice), "breakdown marker");
            std::size_t steps = m_ - p;
            if (budget_ > 0)
                steps = static_cast<std::size_t>(std::min<std::uint64_t>(steps, budget_ - std::min<std::uint64_t>(budget_, matvecs_)));
            if (steps == 0) return 0;
            const std::size_t mend = p + steps;
            if (p > 0) {   // the arrow couplings of the kept Ritz vectors, negated, as the axpy's coefficients
                std::vector<double2> ar(p);
                for (std::size_t i = 0; i < p; ++i) ar[i] = make_double2(-arrow[i], 0.0);
                cuda_check(cudaMemcpy(arrow_.p, ar.data(), p * 16, cudaMemcpyHostToDevice), "arrow");
            }
            for (std::size_t j = p; j < mend; ++j) {
                launch_walk_mixed(sec_, sec_, prog_, col(j), w_.p, dtype_of<T>(), QB_C128, nullptr);
                step_projections(L, j, p);
                k_norm_to<<<nb_, kThreads>>>(n_, w_.p, red(), beta_.p + j + 1, nullptr);
                k_next_col<T><<<nb_, kThreads>>>(n_, w_.p, col(j + 1), beta_.p + j + 1, floor_, brk_.p, static_cast<int>(j));
            }
            cuda_check(cudaGetLastError(), "lanczos cycle");
            matvecs_ += static_cast<int>(steps);
            ++cycles_;
            std::vector<double> a(mend), b(mend + 1);
            int brk = 0;
            cuda_check(cudaMemcpy(a.data(), alpha_.p, mend * 8, cudaMemcpyDeviceToHost), "alpha");
            cuda_check(cudaMemcpy(b.data(), beta_.p, (mend + 1) * 8, cudaMemcpyDeviceToHost), "beta");
            cuda_check(cudaMemcpy(&brk, brk_.p, sizeof(int), cudaMemcpyDeviceToHost), "breakdown");
            // the projected matrix: arrowhead (theta, arrow) then the tridiagonal of this cycle
            const std::size_t mm = brk < big ? static_cast<std::size_t>(brk) + 1 : mend;
            const double beta_last = brk < big ? 0.0 : b[mend];
            std::vector<double> Tm(mm * mm, 0.0);
            auto at = [&](std::size_t r, std::size_t c) -> double& { return Tm[c * mm + r]; };
            for (std::size_t i = 0; i < p; ++i) {
                at(i, i) = theta[i];
                at(i, p) = at(p, i) = arrow[i];
            }
            for (std::size_t j = p; j < mm; ++j) {
                at(j, j) = a[j];
                if (j + 1 < mm) at(j, j + 1) = at(j + 1, j) = b[j + 1];
            }
            std::vector<double> vals, vecs;
            symmetric_eig(Tm, static_cast<int>(mm), vals, vecs);
            if (first && vals[0] >= give_up) return 0;
            const std::size_t top = std::min<std::size_t>(static_cast<std::size_t>(want), mm);
            std::size_t conv = 0;
            while (conv < top && std::abs(beta_last * vecs[conv * mm + (mm - 1)]) < tol()) ++conv;
            const bool invariant = brk < big;
            if (invariant && mm == n_ - locked_.size()) exhausted_ = true;   // the whole (deflated) block is spanned
            if (conv == top || invariant || budget_exhausted()) {
                const std::size_t cnt = invariant ? top : (lock_best ? top : conv);
                lock(vecs, mm, cnt, vals);
                return static_cast<int>(invariant || conv == top ? top : conv);
            }
            // thick restart: the p lowest Ritz vectors, then the residual direction v_mm
            p = std::min(p_, mm - 1);
            rotate(vecs, mm, p, U_.p);
            cuda_check(cudaMemcpy(col(0), U_.p, p * n_ * sizeof(T), cudaMemcpyDeviceToDevice), "restart");
            cuda_check(cudaMemcpy(col(p), col(mm), n_ * sizeof(T), cudaMemcpyDeviceToDevice), "residual direction");
            theta.assign(vals.begin(), vals.begin() + static_cast<std::ptrdiff_t>(p));
            arrow.resize(p);
            for (std::size_t i = 0; i < p; ++i) arrow[i] = beta_last * vecs[i * mm + (mm - 1)];
        }
    }

    void rotate(const std::vector<double>& Y, std::size_t mm, std::size_t cols, T* out) {
        cuda_check(cudaMemcpy(S_.p, Y.data(), mm * cols * 8, cudaMemcpyHostToDevice), "rotation");
        for (std::size_t c0 = 0; c0 < cols; c0 += kRotW)
            k_rotate_real<T><<<nb_, kThreads, mm * kRotW * 8>>>(n_, static_cast<int>(mm), static_cast<int>(cols),
                                                                static_cast<int>(c0), Vb_.p, S_.p, out);
        cuda_check(cudaGetLastError(), "rotate");
    }

    void lock(const std::vector<double>& Y, std::size_t mm, std::size_t cnt, const std::vector<double>& vals) {
        if (cnt == 0) return;
        rotate(Y, mm, cnt, U_.p);
        for (std::size_t i = 0; i < cnt; ++i) {
            DevBuf<T> x(n_);
            cuda_check(cudaMemcpy(x.p, U_.p + i * n_, n_ * sizeof(T), cudaMemcpyDeviceToDevice), "lock");
            locked_.push_back(std::move(x));
            locked_vals_.push_back(vals[i]);
        }
    }
    void drop_locked(std::size_t i) {
        locked_.erase(locked_.begin() + static_cast<std::ptrdiff_t>(i));
        locked_vals_.erase(locked_vals_.begin() + static_cast<std::ptrdiff_t>(i));
    }

    const qb_sector* sec_;
    const qb_program* prog_;
    std::uint64_t n_;
    int k_;
    std::uint64_t budget_;
    double scale_, floor_;
    int nb_;
    std::size_t m_ = 0, p_ = 0, keep_frac_ = 0;
    DevBuf<T> Vb_, U_;
    DevBuf<double2> w_, coef_, part_, arrow_;
    DevBuf<int> flag_;
    DevBuf<void*> ptrs_;
    DevBuf<double> alpha_, beta_, slots_, red_part_, S_;
    DevBuf<unsigned> red_cnt_;
    DevBuf<int> brk_;
    std::vector<DevBuf<T>> locked_;
    std::vector<double> locked_vals_;
    std::vector<T*> sorted_;
    bool have_start_ = false, exhausted_ = false;
    int matvecs_ = 0, cycles_ = 0;
};

template <class T>
LevelsOut levels(const qb_sector* sec, const qb_program* prog, int k, std::uint64_t max_iter, bool refine,
                 bool want_vectors) {
    LevelsOut out;
    const std::uint64_t n = sec->dim;
    if (n == 0) {
        out.converged = true;
        return out;
    }
    const std::uint64_t budget = max_iter > 0 ? max_iter : std::max<std::uint64_t>(200ull * k, 2000);
    std::vector<DevBuf<double2>> X;
    {
        ThickRestart<T> tr(sec, prog, k, budget);
        tr.run(out);
        if (want_vectors || refine) {
            for (T* v : tr.sorted_vectors()) {
                DevBuf<double2> x(n);
                k_copy_cast<T><<<red_blocks(n), kThreads>>>(n, v, x.p);
                X.push_back(std::move(x));
            }
            cuda_check(cudaGetLastError(), "vectors");
        }
    }
    if (refine && !X.empty()) {
        // each pair, lowest first, refined in FP64 against the pairs refined before it
        const std::uint64_t left = budget > static_cast<std::uint64_t>(out.matvecs) ? budget - out.matvecs : 0;
        ThickRestart<double2> fine(sec, prog, static_cast<int>(X.size()), std::max<std::uint64_t>(left, 64), 16);
        bool all = true;
        for (const auto& x : X) all = fine.refine_from(x.p) && all;
        out.matvecs += fine.matvecs();
        out.refine_rounds = static_cast<int>(X.size());
        const auto& vals = fine.locked_values();
        std::vector<std::size_t> order(vals.size());
        for (std::size_t i = 0; i < order.size(); ++i) order[i] = i;
        std::sort(order.begin(), order.end(), [&](std::size_t a, std::size_t b) { return vals[a] < vals[b]; });
        out.values.clear();
        std::vector<DevBuf<double2>> R;
        for (std::size_t i : order) {
            out.values.push_back(vals[i]);
            if (want_vectors) {
                DevBuf<double2> y(n);
                cuda_check(cudaMemcpy(y.p, fine.locked_vector(i), n * 16, cudaMemcpyDeviceToDevice), "refined vector");
                R.push_back(std::move(y));
            }
        }
        X = std::move(R);
        if (!all || out.values.size() < static_cast<std::size_t>(std::min<std::uint64_t>(k, n))) out.converged = false;
    }
    if (want_vectors) out.vectors = std::move(X);
    return out;
}

}  // namespace
}  // namespace qb

extern "C" {

int qb_eigs_k(const qb_sector* sec, const qb_program* prog, int k, uint64_t max_iter, double* values, int* n_found,
              int* converged, int* matvecs, void* const* vecs_device) {
    return qb_eigs_levels(sec, prog, k, max_iter, QB_C128, 0, values, n_found, converged, matvecs, vecs_device);
}

int qb_eigs_levels(const qb_sector* sec, const qb_program* prog, int k, uint64_t max_iter, int dtype, int refine,
                   double* values, int* n_found, int* converged, int* matvecs, void* const* vecs_device) {
    return qb::guarded([&] {
        using namespace qb;
        if (!sec || !prog || !values || k < 1) throw Error(QB_EINVAL, "bad argument");
        if (dtype != QB_C128 && dtype != QB_C64) throw Error(QB_EINVAL, "dtype must be QB_C128 or QB_C64");
        const bool vecs = vecs_device != nullptr;
        LevelsOut r = dtype == QB_C64 ? levels<float2>(sec, prog, k, max_iter, refine != 0, vecs)
                                      : levels<double2>(sec, prog, k, max_iter, false, vecs);
        for (int i = 0; i < k; ++i) values[i] = i < static_cast<int>(r.values.size()) ? r.values[i] : std::nan("");
        if (n_found) *n_found = static_cast<int>(r.values.size());
        if (converged) *converged = r.converged ? 1 : 0;
        if (matvecs) *matvecs = r.matvecs;
        if (vecs)
            for (std::size_t i = 0; i < r.vectors.size(); ++i)
                if (vecs_device[i])
                    cuda_check(cudaMemcpy(vecs_device[i], r.vectors[i].p, sec->dim * 16, cudaMemcpyDeviceToDevice),
                               "vector copy");
    });
}

}  // extern "C"
