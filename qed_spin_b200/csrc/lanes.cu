// =============================================================================
// lanes.cu -- the eigenpair lanes above the k = 1 scan, device-resident:
//   qb_ground_state  the certified lowest eigenpair with its vector (gs_lanczos / gs_vector,
//                    src/engine/block_solve.cpp:697-845): a Paige-gated recurrence without
//                    reorthogonalisation from staged_seed(0x51ED900D), the Ritz vector from the basis kept
//                    on the way or from a replay of the recurrence, then H u: the Rayleigh quotient and
//                    the residual; restarted from u until ||H u - E u|| <= 1e-9 * scale.
//   qb_dynamics_t0   T = 0 dynamics of a cross-sector operator (src/engine/dynamics.cpp:442-566): the
//                    source's ground state, phi = O psi0 on the target sector, the continued fraction of
//                    H_target from phi with the source's E0 as the energy shift.
// Every vector stays on the device. (The k > 1 lane, qb_eigs_k / qb_eigs_levels, is in eigs_k.cu.)
// =============================================================================
#include <algorithm>
#include <cmath>
#include <complex>
#include <limits>
#include <memory>
#include <atomic>
#include <random>
#include <string>
#include <thread>
#include <vector>

#include "qb_krylov.cuh"

namespace qb {
namespace {

constexpr std::uint64_t kGsStartSeed = 0x51ED900DULL;    // block_solve.cpp:264
constexpr int kGsMaxIter = 600;                          // kLgGsMaxIter, src/engine/internal.h:118
constexpr int kGsRestarts = 4;                           // kLgGsRestarts, internal.h:119
constexpr double kGsResidRel = 1e-9;                     // include/ed/core/numerics.h:27
constexpr double kBreakdownRel = 64.0 * std::numeric_limits<double>::epsilon();   // numerics.h:23

// Scratch of the deterministic grid reductions of one driver.
struct Reducer {
    DevBuf<double> part, slots;
    DevBuf<unsigned> cnt;
    Reducer() {
        part.alloc(4 * kMaxRedBlocks);
        slots.alloc(8);
        cnt.alloc(1);
        cuda_check(cudaMemset(cnt.p, 0, 4), "zero");
    }
    Scal scal() { return Scal{nullptr, nullptr, nullptr, part.p, cnt.p}; }
};

// slot = Re <u, w>.
__global__ void k_dot_re(std::uint64_t n, const double2* u, const double2* w, Scal S, double* slot) {
    __shared__ double sm[4 * 32];
    double v[1] = {0.0};
    for (std::uint64_t i = static_cast<std::uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<std::uint64_t>(gridDim.x) * blockDim.x)
        v[0] += u[i].x * w[i].x + u[i].y * w[i].y;
    block_reduce<1>(v, sm);
    double tot[1];
    if (last_block_total<1>(v, S.partials, S.counter, sm, tot)) *slot = tot[0];
}

// slot = ||w - e u||, e = *ep.
__global__ void k_resid(std::uint64_t n, const double2* u, const double2* w, const double* ep, Scal S, double* slot) {
    __shared__ double sm[4 * 32];
    const double e = *ep;
    double v[1] = {0.0};
    for (std::uint64_t i = static_cast<std::uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<std::uint64_t>(gridDim.x) * blockDim.x) {
        const double rx = w[i].x - e * u[i].x, ry = w[i].y - e * u[i].y;
        v[0] += rx * rx + ry * ry;
    }
    block_reduce<1>(v, sm);
    double tot[1];
    if (last_block_total<1>(v, S.partials, S.counter, sm, tot)) *slot = sqrt(tot[0]);
}

// x /= *nrm.
__global__ void k_unit(std::uint64_t n, double2* x, const double* nrm) {
    const double s = 1.0 / *nrm;
    for (std::uint64_t i = static_cast<std::uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<std::uint64_t>(gridDim.x) * blockDim.x) {
        x[i].x *= s;
        x[i].y *= s;
    }
}

double read_slot(const double* slot) {
    double v = 0.0;
    cuda_check(cudaMemcpy(&v, slot, 8, cudaMemcpyDeviceToHost), "scalar read");
    return v;
}

// ---- the certified ground state ----
struct GsOut {
    double energy = std::numeric_limits<double>::quiet_NaN();
    double residual = std::numeric_limits<double>::infinity();
    bool certified = false;
    int matvecs = 0;
};

// u (device, n) <- the lowest eigenvector; the gs_lanczos attempts (block_solve.cpp:697-801).
GsOut gs_vector(const qb_sector* sec, const qb_program* prog, double2* u, int max_steps) {
    GsOut out;
    const std::uint64_t n = sec->dim;
    const double scale = norm_bound(prog);
    const double tol = kGsResidRel * scale;
    const int per_attempt = static_cast<int>(std::min<std::uint64_t>(n, kGsMaxIter));
    int left = max_steps > 0 ? max_steps : per_attempt * (kGsRestarts + 1);
    DevBuf<double2> seed(n), w(n);
    {
        const auto v0 = staged_seed(n, kGsStartSeed);
        upload_host(seed.p, v0.data(), n * 16, nullptr);
    }
    Reducer red;
    const int nb = red_blocks(n);
    for (int attempt = 0; attempt <= kGsRestarts && left > 0; ++attempt) {
        const int cap = std::min(per_attempt, left);
        const std::size_t free_b = available_bytes();
        const bool keep = static_cast<double>(cap + 6) * n * 16.0 < 0.5 * static_cast<double>(free_b);
        std::vector<double> alpha, beta{0.0};
        int m = 0;
        std::vector<double> z;
        {
            Recurrence R(sec, prog, QB_C128, cap);
            R.start_from_device(seed.p);
            if (keep) R.keep_current();
            double sc = 0.0;   // largest |alpha| or beta so far
            // one step's test: false once the run is done
            auto more = [&](double a, double b) {
                alpha.push_back(a);
                beta.push_back(b);
                ++m;
                sc = std::max(sc, std::abs(a));
                if (!(b > 1e-12 * sc)) return false;   // an invariant subspace: its tridiagonal is exact
                sc = std::max(sc, b);
                if (m >= 3) {
                    const Ends t = tridiag_ends(alpha, beta, m, 1);
                    const double ts = std::max({std::abs(t.values[0]), std::abs(t.top), 1e-300});
                    if (beta[m] * std::abs(t.zlast[0]) < 1e-9 * ts) return false;
                }
                return true;
            };
            int launched = 0;
            const int batch = graph_batch(n, true);
            if (batch > 0) {
                // graphs of `batch` steps; the tests run on each batch's scalars (up to batch - 1 steps past the end)
                std::vector<double> ab(batch), bb(batch);
                bool go = true;
                while (go && m < cap) {
                    const int cnt = std::min(batch, cap - m);
                    const int j0 = m;
                    R.advance(cnt, keep, QB_REORTH_NONE, batch);
                    launched += cnt;
                    R.read_range(j0, cnt, ab.data(), bb.data());
                    for (int i = 0; i < cnt && go; ++i) go = more(ab[i], bb[i]);
                }
                if (keep && static_cast<int>(R.basis.size()) > m) R.basis.resize(m);
            } else {
                while (m < cap) {
                    if (keep && m > 0) R.keep_current();
                    R.step(m, QB_REORTH_NONE);
                    ++launched;
                    double a, b;
                    R.read_scalars(m, a, b);
                    if (!more(a, b)) break;
                }
            }
            out.matvecs += launched;
            left -= launched;
            std::vector<double> e(std::max(1, m - 1));
            for (int i = 0; i + 1 < m; ++i) e[i] = beta[i + 1];
            double lo, hi;
            gershgorin(alpha.data(), e.data(), m, lo, hi);
            const double th = kth_eigenvalue(alpha.data(), e.data(), m, 0, lo, hi);
            z = inverse_iteration(alpha.data(), e.data(), m, th);
            cuda_check(cudaMemset(u, 0, n * 16), "zero");
            if (keep) {
                for (int j = 0; j < m; ++j) R.accumulate(u, z[j], R.basis[j]);
                cuda_check(cudaStreamSynchronize(R.st), "ritz vector");
            }
        }
        if (!keep) {   // a replay of the recurrence: the same vectors, bit for bit
            Recurrence R2(sec, prog, QB_C128, m);
            R2.start_from_device(seed.p);
            for (int j = 0; j < m; ++j) {
                R2.accumulate(u, z[j], R2.vbuf[R2.cur].p);
                if (j + 1 < m) {
                    R2.step(j, QB_REORTH_NONE);
                    ++out.matvecs;
                }
            }
            cuda_check(cudaStreamSynchronize(R2.st), "ritz replay");
        }
        // u normalised, then H u: the Rayleigh quotient and the residual
        k_norm_to<<<nb, kThreads>>>(n, u, red.scal(), red.slots.p, nullptr);
        if (!(read_slot(red.slots.p) > 0.0)) return out;
        k_unit<<<nb, kThreads>>>(n, u, red.slots.p);
        launch_walk_mixed(sec, sec, prog, u, w.p, QB_C128, QB_C128, nullptr);
        ++out.matvecs;
        k_dot_re<<<nb, kThreads>>>(n, u, w.p, red.scal(), red.slots.p + 1);
        k_resid<<<nb, kThreads>>>(n, u, w.p, red.slots.p + 1, red.scal(), red.slots.p + 2);
        cuda_check(cudaGetLastError(), "ground state");
        out.energy = read_slot(red.slots.p + 1);
        out.residual = read_slot(red.slots.p + 2);
        if (out.residual <= tol) {
            out.certified = true;
            break;
        }
        cuda_check(cudaMemcpy(seed.p, u, n * 16, cudaMemcpyDeviceToDevice), "restart");   // restarted refinement
    }
    return out;
}

// ---- the dense tail: the full spectrum of a small block ----
// X[r][c] = (r == c0 + c): kc identity columns, interleaved by row, for the block matvec.
__global__ void k_identity_cols(std::uint64_t n, int kc, std::uint64_t c0, double2* X) {
    const std::uint64_t total = n * kc;
    for (std::uint64_t t = static_cast<std::uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; t < total;
         t += static_cast<std::uint64_t>(gridDim.x) * blockDim.x) {
        const std::uint64_t r = t / kc, c = t % kc;
        X[t] = make_double2(r == c0 + c ? 1.0 : 0.0, 0.0);
    }
}

// The eigenvalues of a Hermitian matrix (column-major, n x n), ascending: Householder reflections to a
// Hermitian tridiagonal (A22 <- A22 - 2 (v w^H + w v^H), w = A22 v - (v^H A22 v) v), whose off-diagonal moduli
// make a real symmetric tridiagonal with the same spectrum, then implicit QL.
std::vector<double> hermitian_levels(std::vector<std::complex<double>> A, int n) {
    using cd = std::complex<double>;
    auto at = [&](int r, int c) -> cd& { return A[static_cast<std::size_t>(c) * n + r]; };
    std::vector<cd> v(n), p(n), w(n);
    for (int k = 0; k + 2 < n; ++k) {
        double xn = 0.0;
        for (int i = k + 1; i < n; ++i) xn += std::norm(at(i, k));
        xn = std::sqrt(xn);
        if (xn == 0.0) continue;
        const cd x0 = at(k + 1, k);
        const cd phase = std::abs(x0) > 0.0 ? x0 / std::abs(x0) : cd(1.0, 0.0);
        const cd alpha = -phase * xn;
        // v = x - alpha e1, normalised
        double vn = 0.0;
        for (int i = k + 1; i < n; ++i) {
            v[i] = at(i, k) - (i == k + 1 ? alpha : cd(0.0, 0.0));
            vn += std::norm(v[i]);
        }
        vn = std::sqrt(vn);
        if (vn == 0.0) continue;
        for (int i = k + 1; i < n; ++i) v[i] /= vn;
        // p = A22 v, K = v^H p (real), w = p - K v
        for (int i = k + 1; i < n; ++i) {
            cd s(0.0, 0.0);
            for (int j = k + 1; j < n; ++j) s += at(i, j) * v[j];
            p[i] = s;
        }
        cd K(0.0, 0.0);
        for (int i = k + 1; i < n; ++i) K += std::conj(v[i]) * p[i];
        for (int i = k + 1; i < n; ++i) w[i] = p[i] - K.real() * v[i];
        for (int j = k + 1; j < n; ++j)
            for (int i = k + 1; i < n; ++i) at(i, j) -= 2.0 * (v[i] * std::conj(w[j]) + w[i] * std::conj(v[j]));
        at(k + 1, k) = alpha;
        at(k, k + 1) = std::conj(alpha);
        for (int i = k + 2; i < n; ++i) at(i, k) = at(k, i) = cd(0.0, 0.0);
    }
    std::vector<double> d(n), e(std::max(1, n - 1), 0.0), vals, z0;
    for (int i = 0; i < n; ++i) d[i] = at(i, i).real();
    for (int i = 0; i + 1 < n; ++i) e[i] = std::abs(at(i + 1, i));
    eig_first_row(d, e, vals, z0);
    std::sort(vals.begin(), vals.end());
    return vals;
}

}  // namespace
}  // namespace qb

extern "C" {

}  // extern "C"

namespace qb {
bool dense_levels_device(const qb_sector* const* secs, const qb_program* const* progs, int n_blocks,
                         const std::vector<std::size_t>& off, double* values);
namespace {
// One block's full spectrum: assembled on the calling thread's stream, reduced on the host.
void dense_levels(const qb_sector* sec, const qb_program* prog, double* values) {
    const std::uint64_t n = sec->dim;
    if (n == 0) return;
    if (n > 8192) throw Error(QB_EINVAL, "dense levels: a block of more than 8192 states");
    const int kc = static_cast<int>(std::min<std::uint64_t>(n, 64));
    DevBuf<double2> X(n * kc), Y(n * kc);
    std::vector<std::complex<double>> A(static_cast<std::size_t>(n) * n), Yh(static_cast<std::size_t>(n) * kc);
    for (std::uint64_t c0 = 0; c0 < n; c0 += kc) {
        k_identity_cols<<<red_blocks(n * kc), kThreads>>>(n, kc, c0, X.p);
        launch_block_mixed(sec, sec, prog, X.p, Y.p, kc, QB_C128, QB_C128, nullptr);
        cuda_check(cudaMemcpy(Yh.data(), Y.p, n * kc * 16, cudaMemcpyDeviceToHost), "dense columns");
        for (int c = 0; c < kc && c0 + c < n; ++c)
            for (std::uint64_t r = 0; r < n; ++r) A[(c0 + c) * n + r] = Yh[r * kc + c];
    }
    const std::vector<double> lv = hermitian_levels(std::move(A), static_cast<int>(n));
    std::copy(lv.begin(), lv.end(), values);
}
}  // namespace
}  // namespace qb

extern "C" {

int qb_dense_levels(const qb_sector* sec, const qb_program* prog, double* values) {
    return qb::guarded([&] {
        if (!sec || !prog || !values) throw qb::Error(QB_EINVAL, "null argument");
        const qb_sector* secs[1] = {sec};
        const qb_program* progs[1] = {prog};
        if (!qb::dense_levels_device(secs, progs, 1, {0}, values)) qb::dense_levels(sec, prog, values);
    });
}

int qb_dense_levels_blocks(const qb_sector* const* secs, const qb_program* const* progs, int n_blocks,
                           double* values) {
    return qb::guarded([&] {
        using namespace qb;
        if (!secs || !progs || !values || n_blocks < 0) throw Error(QB_EINVAL, "null argument");
        std::vector<std::size_t> off(n_blocks + 1, 0);
        for (int b = 0; b < n_blocks; ++b) {
            if (!secs[b] || !progs[b]) throw Error(QB_EINVAL, "null block");
            off[b + 1] = off[b] + secs[b]->dim;
        }
        // blocks of at most 1024 states: all at once on the device (dense.cu)
        if (dense_levels_device(secs, progs, n_blocks, off, values)) return;
        // larger blocks: largest first over a pool of host threads, each assembling on its own stream and
        // reducing on the host
        std::vector<int> order(n_blocks);
        for (int b = 0; b < n_blocks; ++b) order[b] = b;
        std::sort(order.begin(), order.end(), [&](int a, int b) { return secs[a]->dim > secs[b]->dim; });
        int dev = 0;
        cuda_check(cudaGetDevice(&dev), "device");
        const int nt = std::max(1, std::min<int>(n_blocks, static_cast<int>(std::max(1u, std::thread::hardware_concurrency()))));
        std::atomic<int> next{0};
        std::vector<std::string> errs(nt);
        std::vector<std::thread> pool;
        for (int t = 0; t < nt; ++t)
            pool.emplace_back([&, t] {
                cudaSetDevice(dev);
                try {
                    for (int i = next++; i < n_blocks; i = next++)
                        dense_levels(secs[order[i]], progs[order[i]], values + off[order[i]]);
                } catch (const std::exception& e) {
                    errs[t] = e.what();
                }
            });
        for (auto& t : pool) t.join();
        for (const auto& e : errs)
            if (!e.empty()) throw Error(QB_EINVAL, e);
    });
}



int qb_ground_state(const qb_sector* sec, const qb_program* prog, int max_steps, double* e0, double* residual,
                    int* certified, void* vec_device, double* vec_host, int* matvecs) {
    return qb::guarded([&] {
        using namespace qb;
        if (!sec || !prog || !e0) throw Error(QB_EINVAL, "null argument");
        if (sec->dim == 0) throw Error(QB_EINVAL, "empty sector");
        DevBuf<double2> own;
        double2* u = static_cast<double2*>(vec_device);
        if (!u) {
            own.alloc(sec->dim);
            u = own.p;
        }
        const GsOut g = gs_vector(sec, prog, u, max_steps);
        *e0 = g.energy;
        if (residual) *residual = g.residual;
        if (certified) *certified = g.certified ? 1 : 0;
        if (matvecs) *matvecs = g.matvecs;
        if (vec_host) cuda_check(cudaMemcpy(vec_host, u, sec->dim * 16, cudaMemcpyDeviceToHost), "vector download");
    });
}

int qb_dynamics_t0(const qb_sector* src, const qb_program* h_src, const qb_sector* tgt, const qb_program* h_tgt,
                   const qb_program* op, int depth, const double* omega, int n_omega, double eta, double* S, double* e0,
                   double* conv_change, int* certified) {
    return qb::guarded([&] {
        using namespace qb;
        if (!src || !h_src || !tgt || !h_tgt || !op || !omega || !S || !e0) throw Error(QB_EINVAL, "null argument");
        if (src->N != tgt->N) throw Error(QB_EINVAL, "sectors of different sizes");
        for (int i = 0; i < n_omega; ++i) S[i] = 0.0;
        if (conv_change) *conv_change = 0.0;
        DevBuf<double2> psi(src->dim);
        const GsOut g = gs_vector(src, h_src, psi.p, 0);
        *e0 = g.energy;
        if (certified) *certified = g.certified ? 1 : 0;
        if (tgt->dim == 0) return;
        DevBuf<double2> phi(tgt->dim);
        launch_walk_mixed(tgt, src, op, psi.p, phi.p, QB_C128, QB_C128, nullptr);   // phi = O psi0
        cuda_check(cudaGetLastError(), "phi");
        const int kd = std::max(depth, 2);
        Recurrence R(tgt, h_tgt, QB_C128, kd);
        double nrm = 0.0;
        try {
            nrm = R.start_from_device(phi.p);
        } catch (const Error& e) {
            if (e.code == QB_EINVAL) return;   // phi = 0: no spectral weight
            throw;
        }
        const double tol = kBreakdownRel * norm_bound(h_tgt);
        ScanOut o = run_scan(R, kd, QB_REORTH_NONE, false, tol, false);
        if (o.alpha.empty()) return;
        const int m = static_cast<int>(o.alpha.size());
        cf_spectrum(o.alpha, o.beta, m, omega, n_omega, eta, g.energy, nrm * nrm, S);
        if (conv_change) *conv_change = cf_change(o.alpha, o.beta, m, omega, n_omega, eta, g.energy, nrm * nrm, S);
    });
}

int qb_dynamics_t0_manifold(int n_src, const qb_sector* const* srcs, const qb_program* const* h_srcs,
                            const qb_sector* const* tgts, const qb_program* const* h_tgts, const qb_program* const* ops,
                            int depth, const double* omega, int n_omega, double eta, double degeneracy_tol, double* S,
                            double* e0, int* manifold, int* certified) {
    return qb::guarded([&] {
        using namespace qb;
        if (n_src < 1 || !srcs || !h_srcs || !tgts || !h_tgts || !ops || !omega || !S || !e0 || degeneracy_tol < 0.0)
            throw Error(QB_EINVAL, "bad argument");
        for (int b = 0; b < n_src; ++b) {
            if (!srcs[b] || !h_srcs[b] || !tgts[b] || !h_tgts[b] || !ops[b]) throw Error(QB_EINVAL, "null block");
            if (srcs[b]->N != tgts[b]->N) throw Error(QB_EINVAL, "sectors of different sizes");
        }
        for (int i = 0; i < n_omega; ++i) S[i] = 0.0;
        // the lowest level of every source block (the k = 1 lane), and the window above the least of them
        std::vector<double> low(n_src, std::numeric_limits<double>::infinity());
        bool all_conv = true;
        for (int b = 0; b < n_src; ++b) {
            if (srcs[b]->dim == 0) continue;
            int it = 0, cv = 0, mv = 0;
            if (qb_eigs_lowest(srcs[b], h_srcs[b], 0, QB_C128, 0, &low[b], &it, &cv, &mv) != QB_OK)
                throw Error(QB_ECUDA, std::string("ground manifold: ") + qb_last_error());
            all_conv = all_conv && cv;
        }
        double emin = *std::min_element(low.begin(), low.end());
        if (!std::isfinite(emin)) throw Error(QB_EINVAL, "the source blocks hold no state");
        const double window = degeneracy_tol * norm_bound(h_srcs[0]);
        // every level within the window of each block at E0, with its vector: k levels, doubling k until one
        // lies above the window or the block is exhausted (a multiplet inside a block)
        struct State {
            int b;
            double e;
            DevBuf<double2> v;
        };
        std::vector<State> states;
        for (int b = 0; b < n_src; ++b) {
            if (!(low[b] <= emin + window)) continue;
            const std::uint64_t n = srcs[b]->dim;
            for (int pb = 2;; pb *= 2) {
                const int kk = static_cast<int>(std::min<std::uint64_t>(static_cast<std::uint64_t>(pb), n));
                std::vector<DevBuf<double2>> vec(kk);
                std::vector<void*> ptr(kk);
                for (int i = 0; i < kk; ++i) {
                    vec[i].alloc(n);
                    ptr[i] = vec[i].p;
                }
                std::vector<double> vals(kk);
                int nf = 0, cv = 0, mv = 0;
                if (qb_eigs_levels(srcs[b], h_srcs[b], kk, 0, QB_C128, 0, vals.data(), &nf, &cv, &mv, ptr.data()) != QB_OK)
                    throw Error(QB_ECUDA, std::string("ground manifold: ") + qb_last_error());
                const bool exhausted = nf < kk || static_cast<std::uint64_t>(kk) >= n;
                if (exhausted || vals[nf - 1] > emin + window) {
                    all_conv = all_conv && cv;
                    for (int i = 0; i < nf; ++i)
                        if (vals[i] <= emin + window) states.push_back(State{b, vals[i], std::move(vec[i])});
                    break;
                }
            }
        }
        if (states.empty()) throw Error(QB_ECUDA, "ground manifold: no level within the window");
        for (const auto& st : states) emin = std::min(emin, st.e);
        // one continued fraction per state from phi = O psi in its target block, shifted by E0, averaged
        std::vector<double> Sk(std::max(1, n_omega));
        for (const auto& st : states) {
            const qb_sector* tgt = tgts[st.b];
            if (tgt->dim == 0) continue;
            DevBuf<double2> phi(tgt->dim);
            launch_walk_mixed(tgt, srcs[st.b], ops[st.b], st.v.p, phi.p, QB_C128, QB_C128, nullptr);
            cuda_check(cudaGetLastError(), "phi");
            const int kd = std::max(depth, 2);
            Recurrence R(tgt, h_tgts[st.b], QB_C128, kd);
            double nrm = 0.0;
            try {
                nrm = R.start_from_device(phi.p);
            } catch (const Error& e) {
                if (e.code == QB_EINVAL) continue;   // O annihilates this state: no spectral weight
                throw;
            }
            const double tol = kBreakdownRel * norm_bound(h_tgts[st.b]);
            ScanOut o = run_scan(R, kd, QB_REORTH_NONE, false, tol, false);
            if (o.alpha.empty()) continue;
            cf_spectrum(o.alpha, o.beta, static_cast<int>(o.alpha.size()), omega, n_omega, eta, emin, nrm * nrm,
                        Sk.data());
            for (int i = 0; i < n_omega; ++i) S[i] += Sk[i];
        }
        for (int i = 0; i < n_omega; ++i) S[i] /= static_cast<double>(states.size());
        *e0 = emin;
        if (manifold) *manifold = static_cast<int>(states.size());
        if (certified) *certified = all_conv ? 1 : 0;
    });
}

}  // extern "C"
