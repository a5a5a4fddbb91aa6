// =============================================================================
// oracle/qed_oracle.cpp -- TEST INFRASTRUCTURE: the restated CPU oracle of the hot path.
//
// A serial restatement, written for checking, of the reference engine's CPU algorithm for:
//   * the compiled group action (byte LUT)         include/ed/basis/compiled_group.h:73-78, 108-140
//   * the sublattice key order and candidates      include/ed/basis/sublattice_code.h:64-131, 232-399
//   * the fused representative + stabiliser scan   include/ed/basis/orbit_table.h:147-286
//   * the 1-dim irrep sector (closed-form norms)    include/ed/basis/orbit_table.h:93-99,
//                                                  src/engine/group_sector.cpp:159-205
//   * index_and_projection (running minimum)       include/ed/matvec/rep_symmetry_basis_policy.h:142-241
//   * the row walk of a flip-grouped program       include/ed/ops/row_walk.h:28-65
//   * the sector gather / merged rows              include/ed/matvec/sector_rows.h:41-158
//   * the Lanczos kernel on host vectors           include/ed/krylov/lanczos.h:266-576,
//                                                  include/ed/matvec/cpu_backend.h:130-214
//   * the k = 1 scan lane                          src/engine/block_solve.cpp:335-398, 528-598
//   * FTLM sample moments and combine              include/ed/thermal/ftlm.h:165-235, 277-480
//   * the sample seeds                             include/ed/thermal/sample_seed.h:37-89
//   * the continued fraction                       include/ed/dynamics/cf.h:39-160
// The tridiagonal eigensolve (LAPACK dstevd/dstevx in the reference, include/ed/krylov/tridiag.h)
// is an implicit QL with Wilkinson shifts here, with inverse iteration for selected vectors.
//
// Only tests/, __graft_entry__.smoke() and bench.py's CPU baseline load this library.
// =============================================================================
#include "qed_oracle.h"

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <limits>
#include <memory>
#include <numeric>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

namespace {

using Complex = std::complex<double>;
thread_local std::string g_err;

// ---------------------------------------------------------------------------------------------
// Group action: byte LUT (compiled_group.h:108-140). lut[(g*bpw + b)*256 + v] is the image of byte
// b holding v; image = OR of the bpw words, XOR the element's flip mask.
// ---------------------------------------------------------------------------------------------
struct Group {
    int N = 0, G = 0, bpw = 0;
    std::vector<int> perms;           // G x N
    std::vector<std::uint64_t> flips;  // G
    std::vector<std::uint64_t> lut;    // G x bpw x 256

    void build() {
        bpw = (N + 7) / 8;
        lut.assign(static_cast<std::size_t>(G) * bpw * 256, 0ULL);
        for (int g = 0; g < G; ++g) {
            int inv[64];
            for (int i = 0; i < N; ++i) inv[perms[g * N + i]] = i;
            for (int b = 0; b < bpw; ++b)
                for (int v = 0; v < 256; ++v) {
                    std::uint64_t out = 0;
                    for (int t = 0; t < 8 && 8 * b + t < N; ++t)
                        if ((v >> t) & 1) out |= 1ULL << inv[8 * b + t];
                    lut[(static_cast<std::size_t>(g) * bpw + b) * 256 + v] = out;
                }
        }
    }
    std::uint64_t apply(std::uint64_t s, int g) const {
        const std::uint64_t* l = lut.data() + static_cast<std::size_t>(g) * bpw * 256;
        std::uint64_t r = 0;
        for (int b = 0; b < bpw; ++b) r |= l[b * 256 + static_cast<int>((s >> (8 * b)) & 0xFF)];
        return r ^ flips[g];
    }
};

// ---------------------------------------------------------------------------------------------
// Sublattice code (sublattice_code.h:232-399): the block system with the largest blocks (<= 16
// sites, 2..8 equal blocks) and its key order, leading-block table and candidate lists.
// ---------------------------------------------------------------------------------------------
struct Slc {
    bool on = false;
    int N = 0, bpw = 0, L = 0, m = 0;
    std::vector<int> key_bit;
    std::vector<std::uint64_t> to_key;
    std::vector<std::uint16_t> lead;
    std::vector<std::uint32_t> cand_off;
    std::vector<std::uint16_t> cand;

    std::uint64_t key(std::uint64_t s) const {
        std::uint64_t k = 0;
        for (int b = 0; b < bpw; ++b) k |= to_key[(b << 8) + static_cast<int>((s >> (8 * b)) & 0xFF)];
        return k;
    }
    std::uint32_t pattern(std::uint64_t k, int j) const {
        return static_cast<std::uint32_t>(k >> (N - (j + 1) * L)) & ((1u << L) - 1u);
    }
    std::uint32_t least_lead(std::uint64_t k) const {
        std::uint32_t best = 0xFFFFFFFFu;
        for (int j = 0; j < m; ++j) best = std::min<std::uint32_t>(best, lead[(static_cast<std::uint32_t>(j) << L) + pattern(k, j)]);
        return best;
    }
    // Elements reaching the least leading block, ascending (sublattice_code.h:102-131).
    template <class Fn> void for_each_candidate(std::uint64_t k, Fn&& fn) const {
        std::uint32_t entry[8], pos[8], end[8];
        std::uint32_t best = 0xFFFFFFFFu;
        for (int j = 0; j < m; ++j) {
            entry[j] = (static_cast<std::uint32_t>(j) << L) + pattern(k, j);
            best = std::min<std::uint32_t>(best, lead[entry[j]]);
        }
        int n = 0;
        for (int j = 0; j < m; ++j)
            if (lead[entry[j]] == best) {
                pos[n] = cand_off[entry[j]];
                end[n] = cand_off[entry[j] + 1];
                ++n;
            }
        for (;;) {
            int pick = -1;
            std::uint32_t g = 0xFFFFFFFFu;
            for (int i = 0; i < n; ++i)
                if (pos[i] < end[i] && cand[pos[i]] < g) {
                    g = cand[pos[i]];
                    pick = i;
                }
            if (pick < 0) return;
            ++pos[pick];
            fn(static_cast<int>(g));
        }
    }
};

// The finest partition invariant under the group that joins sites 0 and b, for every b; the one
// with the largest blocks wins (first found on ties) (sublattice_code.h:232-270).
std::vector<int> block_system(const std::vector<std::vector<int>>& sp, int N, int& L) {
    L = 0;
    std::vector<int> best, parent(N);
    auto find = [&](int x) {
        while (parent[x] != x) {
            parent[x] = parent[parent[x]];
            x = parent[x];
        }
        return x;
    };
    for (int b = 1; b < N; ++b) {
        std::iota(parent.begin(), parent.end(), 0);
        parent[b] = 0;
        std::vector<std::pair<int, int>> todo{{0, b}};
        while (!todo.empty()) {
            const auto [x, y] = todo.back();
            todo.pop_back();
            for (const auto& p : sp) {
                const int px = p[x], py = p[y];
                const int u = find(px), v = find(py);
                if (u == v) continue;
                parent[std::max(u, v)] = std::min(u, v);
                todo.emplace_back(px, py);
            }
        }
        std::vector<int> size(N, 0);
        for (int s = 0; s < N; ++s) ++size[find(s)];
        const int l = size[0];
        if (l > 16 || l <= L || N % l != 0 || N / l < 2 || N / l > 8) continue;
        bool equal = true;
        for (int s = 0; s < N && equal; ++s) equal = size[find(s)] == l;
        if (!equal) continue;
        std::vector<int> root_block(N, -1), block(N);
        int nb = 0;
        for (int s = 0; s < N; ++s) {
            int& rb = root_block[find(s)];
            if (rb < 0) rb = nb++;
            block[s] = rb;
        }
        L = l;
        best = std::move(block);
    }
    return best;
}

// SublatticeCode::of + build_ (sublattice_code.h:164-191, 300-399). min_perms 0: forced.
Slc make_slc(const Group& grp, int slc_mode) {
    Slc c;
    const int N = grp.N, G = grp.G;
    if (slc_mode == 0 || G <= 1 || N < 4 || N > 64 || G > 65535) return c;
    const std::size_t min_perms = slc_mode == 1 ? 0 : (slc_mode == -1 ? 16 : 64);
    std::vector<std::vector<int>> sp;
    for (int g = 0; g < G; ++g) {
        std::vector<int> p(grp.perms.begin() + g * N, grp.perms.begin() + (g + 1) * N);
        if (std::find(sp.begin(), sp.end(), p) == sp.end()) sp.push_back(std::move(p));
    }
    if (min_perms > 0 && (N < 24 || sp.size() < min_perms)) return c;
    int L = 0;
    const std::vector<int> block = block_system(sp, N, L);
    if (block.empty()) return c;
    c.on = true;
    c.N = N;
    c.L = L;
    c.m = N / L;
    c.bpw = (N + 7) / 8;
    c.key_bit.assign(N, 0);
    std::vector<std::vector<int>> sites(c.m);
    for (int s = 0; s < N; ++s) sites[block[s]].push_back(s);
    for (int j = 0; j < c.m; ++j)
        for (int t = 0; t < L; ++t) c.key_bit[sites[j][t]] = N - (j + 1) * L + t;
    c.to_key.assign(static_cast<std::size_t>(c.bpw) * 256, 0ULL);
    for (int b = 0; b < c.bpw; ++b)
        for (int v = 0; v < 256; ++v) {
            std::uint64_t out = 0;
            for (int t = 0; t < 8 && 8 * b + t < N; ++t)
                if ((v >> t) & 1) out |= 1ULL << c.key_bit[8 * b + t];
            c.to_key[b * 256 + v] = out;
        }
    const std::size_t P = std::size_t{1} << L;
    const std::uint32_t lmask = (1u << L) - 1u;
    std::vector<int> src_block(G), pos_in_block(N, -1);
    std::vector<std::vector<std::uint32_t>> e(G, std::vector<std::uint32_t>(L, 0u));
    std::vector<std::uint32_t> fl(G, 0u);
    for (int j = 0; j < c.m; ++j)
        for (int t = 0; t < L; ++t) pos_in_block[sites[j][t]] = t;
    for (int g = 0; g < G; ++g) {
        const int* p = grp.perms.data() + g * N;
        src_block[g] = block[p[sites[0][0]]];
        for (int t = 0; t < L; ++t) {
            const int i = sites[0][t];
            e[g][pos_in_block[p[i]]] = 1u << t;
            if ((grp.flips[g] >> i) & 1ULL) fl[g] |= 1u << t;
        }
    }
    const std::size_t M = static_cast<std::size_t>(c.m) * P;
    c.lead.assign(M, 0xFFFFu);
    std::vector<std::uint32_t> img(P), count(M, 0);
    auto images = [&](int g) {
        img[0] = 0;
        for (std::size_t x = 1; x < P; ++x) img[x] = img[x & (x - 1)] | e[g][__builtin_ctzll(x)];
        for (std::size_t x = 0; x < P; ++x) img[x] = (img[x] ^ fl[g]) & lmask;
    };
    for (int g = 0; g < G; ++g) {
        images(g);
        std::uint16_t* row = c.lead.data() + static_cast<std::size_t>(src_block[g]) * P;
        for (std::size_t x = 0; x < P; ++x)
            if (img[x] < row[x]) row[x] = static_cast<std::uint16_t>(img[x]);
    }
    for (int g = 0; g < G; ++g) {
        images(g);
        const std::size_t base = static_cast<std::size_t>(src_block[g]) * P;
        for (std::size_t x = 0; x < P; ++x) count[base + x] += c.lead[base + x] == img[x] ? 1u : 0u;
    }
    c.cand_off.assign(M + 1, 0);
    for (std::size_t i = 0; i < M; ++i) c.cand_off[i + 1] = c.cand_off[i] + count[i];
    c.cand.assign(c.cand_off[M], 0);
    std::vector<std::uint32_t> fill(c.cand_off.begin(), c.cand_off.end() - 1);
    for (int g = 0; g < G; ++g) {
        images(g);
        const std::size_t base = static_cast<std::size_t>(src_block[g]) * P;
        for (std::size_t x = 0; x < P; ++x)
            if (c.lead[base + x] == img[x]) c.cand[fill[base + x]++] = static_cast<std::uint16_t>(g);
    }
    return c;
}

// ---------------------------------------------------------------------------------------------
// Sector: the representatives ascending, their 1/norm, the characters (rep_sector.h:134-408).
// ---------------------------------------------------------------------------------------------
struct Sector {
    Group grp;
    Slc slc;
    int n_up = 0;
    std::vector<Complex> chars;
    std::vector<std::uint64_t> reps;
    std::vector<double> inv_norms;

    // fn(g, image, key) for the elements that can map `state` to its representative, ascending
    // (rep_symmetry_basis_policy.h:142-154).
    template <class Fn> void for_each_image(std::uint64_t state, Fn&& fn) const {
        if (slc.on) {
            slc.for_each_candidate(slc.key(state), [&](int g) {
                const std::uint64_t img = grp.apply(state, g);
                fn(g, img, slc.key(img));
            });
            return;
        }
        for (int g = 0; g < grp.G; ++g) {
            const std::uint64_t img = grp.apply(state, g);
            fn(g, img, img);
        }
    }
    std::int64_t index_of_rep(std::uint64_t rb) const {
        const auto it = std::lower_bound(reps.begin(), reps.end(), rb);
        if (it == reps.end() || *it != rb) return -1;
        return it - reps.begin();
    }
    // rep_symmetry_basis_policy.h:221-241: the running minimum; the character sum restarts at a new
    // minimum and grows on ties (conj: +re, -im).
    std::int64_t index_and_projection(std::uint64_t state, Complex& proj) const {
        if (__builtin_popcountll(state) != n_up) return -1;
        std::uint64_t rb = ~0ULL, best = ~0ULL;
        double re = 0.0, im = 0.0;
        for_each_image(state, [&](int g, std::uint64_t img, std::uint64_t k) {
            if (k < best) {
                best = k;
                rb = img;
                re = 0.0 + chars[g].real();
                im = 0.0 - chars[g].imag();
            } else if (k == best) {
                re += chars[g].real();
                im -= chars[g].imag();
            }
        });
        const std::int64_t k = index_of_rep(rb);
        if (k < 0) return -1;
        const double s = inv_norms[static_cast<std::size_t>(k)];
        proj = Complex(re * s, im * s);
        return k;
    }
};

// visit_state (orbit_table.h:147-171): false for a non-representative; else the stabiliser elements
// in the order the scan meets them.
bool visit_state(const Sector& S, std::uint64_t s, std::vector<int>& stab) {
    stab.clear();
    if (S.slc.on) {
        const std::uint64_t k = S.slc.key(s);
        if (S.slc.least_lead(k) < S.slc.pattern(k, 0)) return false;
        bool rep = true;
        S.slc.for_each_candidate(k, [&](int g) {
            if (!rep) return;
            const std::uint64_t ik = S.slc.key(S.grp.apply(s, g));
            if (ik < k)
                rep = false;
            else if (ik == k)
                stab.push_back(g);
        });
        return rep;
    }
    for (int g = 0; g < S.grp.G; ++g) {
        const std::uint64_t img = S.grp.apply(s, g);
        if (img < s) return false;
        if (img == s) stab.push_back(g);
    }
    return true;
}

// projected_norm_sq_stab (orbit_table.h:93-99) and filter_reps (group_sector.cpp:159-205).
double inv_norm_of(const std::vector<int>& stab, const std::vector<Complex>& chi) {
    double nsq = 1.0;
    if (stab.size() != 1) {
        Complex sum(0.0, 0.0);
        for (int g : stab) sum += chi[g];
        nsq = std::norm(sum) / static_cast<double>(stab.size());
    }
    return nsq <= 1e-12 ? 0.0 : 1.0 / std::sqrt(nsq);
}

// The fixed-Sz scan in ascending (Gosper) order (orbit_table.h:250-286, gosper.h:24).
void build_sector(Sector& S) {
    const int N = S.grp.N;
    S.reps.clear();
    S.inv_norms.clear();
    if (S.n_up < 0 || S.n_up > N) return;
    std::vector<int> stab;
    if (S.n_up == 0) {
        stab.resize(S.grp.G);
        std::iota(stab.begin(), stab.end(), 0);
        const double inv = inv_norm_of(stab, S.chars);
        if (inv != 0.0) {
            S.reps.push_back(0);
            S.inv_norms.push_back(inv);
        }
        return;
    }
    std::uint64_t total = 1;   // C(N, n_up)
    for (int i = 0; i < S.n_up; ++i) total = total * static_cast<std::uint64_t>(N - i) / static_cast<std::uint64_t>(i + 1);
    std::uint64_t s = (S.n_up == 64) ? ~0ULL : ((1ULL << S.n_up) - 1ULL);
    for (std::uint64_t i = 0; i < total; ++i) {
        if (visit_state(S, s, stab)) {
            const double inv = inv_norm_of(stab, S.chars);
            if (inv != 0.0) {
                S.reps.push_back(s);
                S.inv_norms.push_back(inv);
            }
        }
        if (i + 1 < total) {
            const std::uint64_t c = s & (~s + 1ULL);
            const std::uint64_t r = s + c;
            s = (((r ^ s) >> 2) / c) | r;
        }
    }
}

// ---------------------------------------------------------------------------------------------
// Program and row walk (program.h:66-94, row_walk.h:28-65).
// ---------------------------------------------------------------------------------------------
struct Program {
    std::vector<std::uint64_t> group_flip;
    std::vector<int> group_setbits;
    std::vector<std::uint32_t> group_vbegin;
    std::vector<std::uint64_t> vsub_val;
    std::vector<std::uint32_t> vsub_tbegin;
    std::vector<std::uint64_t> term_sign;
    std::vector<Complex> term_coeff;
    std::uint32_t n_groups() const { return static_cast<std::uint32_t>(group_flip.size()); }
    double norm_bound() const {
        double s = 0.0;
        for (const auto& c : term_coeff) s += std::abs(c);
        return s;
    }
};

bool connection(const Program& P, std::uint64_t s, std::uint32_t g, std::uint64_t& t, Complex& h) {
    const std::uint64_t F = P.group_flip[g];
    const std::uint64_t v = s & F;
    if (P.group_setbits[g] >= 0 && __builtin_popcountll(v) != P.group_setbits[g]) return false;
    std::uint32_t lo = P.group_vbegin[g], hi = P.group_vbegin[g + 1];
    while (lo < hi) {
        const std::uint32_t mid = lo + (hi - lo) / 2;
        if (P.vsub_val[mid] < v)
            lo = mid + 1;
        else
            hi = mid;
    }
    if (lo == P.group_vbegin[g + 1] || P.vsub_val[lo] != v) return false;
    h = Complex(0.0, 0.0);
    for (std::uint32_t k = P.vsub_tbegin[lo]; k < P.vsub_tbegin[lo + 1]; ++k) {
        if (__builtin_popcountll(s & P.term_sign[k]) & 1)
            h += -P.term_coeff[k];
        else
            h += P.term_coeff[k];
    }
    t = s ^ F;
    return true;
}

// for_each_cross_entry (sector_rows.h:41-56): emit(column, value) for row j, in group order.
template <class Emit>
void for_each_entry(const Program& P, const Sector& row, const Sector& col, bool same, std::uint64_t j, Emit&& emit) {
    const std::uint64_t s = row.reps[j];
    const double w = row.inv_norms[j];
    for (std::uint32_t g = 0; g < P.n_groups(); ++g) {
        std::uint64_t t;
        Complex h;
        if (!connection(P, s, g, t, h)) continue;
        if (same && t == s) {
            emit(j, std::conj(h));
            continue;
        }
        Complex proj;
        const std::int64_t c = col.index_and_projection(t, proj);
        if (c < 0) continue;
        emit(static_cast<std::uint64_t>(c), w * std::conj(h * proj));
    }
}

// ---------------------------------------------------------------------------------------------
// Host vector primitives in the CpuBackend's arithmetic (cpu_backend.h:130-214), serial.
// ---------------------------------------------------------------------------------------------
using Vec = std::vector<Complex>;

Complex vdot(const Vec& x, const Vec& y) {
    Complex s{};
    for (std::size_t i = 0; i < x.size(); ++i) {
        const Complex xc = std::conj(x[i]);
        s += Complex(xc.real() * y[i].real() - xc.imag() * y[i].imag(), xc.real() * y[i].imag() + xc.imag() * y[i].real());
    }
    return s;
}
double vnrm2(const Vec& x) {
    double s = 0.0;
    for (const auto& v : x) s += v.real() * v.real() + v.imag() * v.imag();
    return std::sqrt(s);
}
void vaxpy(Complex a, const Vec& x, Vec& y) {
    for (std::size_t i = 0; i < x.size(); ++i) y[i] += a * x[i];
}
void vscale(Complex a, Vec& x) {
    for (auto& v : x) v *= a;
}
// y += a x; return <z, y> (axpy_dot_local, cpu_backend.h:174-191).
Complex vaxpy_dot(Complex a, const Vec& x, Vec& y, const Vec& z) {
    Complex s{};
    const double ar = a.real(), ai = a.imag();
    for (std::size_t i = 0; i < x.size(); ++i) {
        const double yr = y[i].real() + ar * x[i].real() - ai * x[i].imag();
        const double yi = y[i].imag() + ar * x[i].imag() + ai * x[i].real();
        y[i] = Complex(yr, yi);
        s += Complex(z[i].real() * yr + z[i].imag() * yi, z[i].real() * yi - z[i].imag() * yr);
    }
    return s;
}
// y += a x; return ||y|| (axpy_nrm2sq_local, cpu_backend.h:192-207).
double vaxpy_nrm2(Complex a, const Vec& x, Vec& y) {
    double s = 0.0;
    const double ar = a.real(), ai = a.imag();
    for (std::size_t i = 0; i < x.size(); ++i) {
        const double yr = y[i].real() + ar * x[i].real() - ai * x[i].imag();
        const double yi = y[i].imag() + ar * x[i].imag() + ai * x[i].real();
        y[i] = Complex(yr, yi);
        s += yr * yr + yi * yi;
    }
    return std::sqrt(s);
}

// ---------------------------------------------------------------------------------------------
// Lanczos (lanczos.h:266-576): three-term recurrence; reorth None / FullCGS2 (DGKS kappa 1/sqrt 2) /
// LocalDGKS3 with K = 1 (threshold sqrt(eps)); breakdown on beta < tol; convergence callback.
// ---------------------------------------------------------------------------------------------
template <class Matvec, class Check>
void lanczos(Matvec&& H, const Vec& v0, std::size_t max_iter, int reorth, double breakdown_tol, Check&& check,
             std::vector<double>& alpha, std::vector<double>& beta) {
    const std::size_t n = v0.size();
    alpha.clear();
    beta.assign(1, 0.0);
    if (max_iter == 0) return;
    Vec v_prev(n), v_curr = v0, w(n);
    const double nrm = vnrm2(v_curr);
    if (!(nrm > 0.0)) throw std::invalid_argument("lanczos: initial vector has non-positive norm");
    vscale(Complex(1.0 / nrm), v_curr);
    std::vector<Vec> basis;
    const bool cgs2 = reorth == 1, local = reorth == 2;
    if (cgs2) basis.push_back(v_curr);
    const std::size_t cap = std::min(max_iter, n);
    for (std::size_t j = 0; j < cap; ++j) {
        H(v_curr, w);
        const Complex aj = j > 0 ? vaxpy_dot(Complex(-beta[j]), v_prev, w, v_curr) : vdot(v_curr, w);
        alpha.push_back(aj.real());
        const bool fuse = local && j > 0;
        Complex overlap{};
        if (fuse)
            overlap = vaxpy_dot(Complex(-alpha[j]), v_curr, w, v_curr);
        else
            vaxpy(Complex(-alpha[j]), v_curr, w);
        bool defer = false;
        Complex defer_coef{};
        if (cgs2) {
            for (int pass = 0; pass < 2; ++pass) {
                const double before = vnrm2(w);
                std::vector<Complex> c(basis.size());
                for (std::size_t k = 0; k < basis.size(); ++k) c[k] = -vdot(basis[k], w);
                for (std::size_t k = 0; k < basis.size(); ++k) vaxpy(c[k], basis[k], w);
                const double after = vnrm2(w);
                if (!(after < 0.7071067811865476 * before)) break;
            }
        } else if (local && j > 0) {
            if (std::abs(overlap) > 1.49011611938476562e-08) {
                defer = true;
                defer_coef = -overlap;
            }
        }
        const double bnext = defer ? vaxpy_nrm2(defer_coef, v_curr, w) : vnrm2(w);
        beta.push_back(bnext);
        if (bnext < breakdown_tol) break;
        vscale(Complex(1.0 / bnext), w);
        std::swap(v_prev, v_curr);
        std::swap(v_curr, w);
        if (check(alpha, beta)) break;
        if (j + 1 >= cap) break;
        if (cgs2) basis.push_back(v_curr);
    }
}

// ---------------------------------------------------------------------------------------------
// Symmetric tridiagonal eigensolve: implicit QL with Wilkinson shifts (the classical algorithm of
// Bowdler, Martin, Reinsch and Wilkinson), eigenvalues ascending, optional eigenvectors.
// d: diagonal (m), e: off-diagonal (m-1). z: column-major m x m (identity on entry) or empty.
// ---------------------------------------------------------------------------------------------
void tridiag_ql(std::vector<double>& d, std::vector<double> e, std::vector<double>* z) {
    const int m = static_cast<int>(d.size());
    if (m == 0) return;
    e.resize(m, 0.0);
    e[m - 1] = 0.0;
    for (int l = 0; l < m; ++l) {
        int iter = 0;
        for (;;) {
            int k = l;
            for (; k < m - 1; ++k) {
                const double dd = std::abs(d[k]) + std::abs(d[k + 1]);
                if (std::abs(e[k]) <= std::numeric_limits<double>::epsilon() * dd) break;
            }
            if (k == l) break;
            if (++iter > 60) throw std::runtime_error("tridiagonal QL did not converge");
            double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
            double r = std::hypot(g, 1.0);
            g = d[k] - d[l] + e[l] / (g + (g >= 0 ? r : -r));
            double s = 1.0, c = 1.0, p = 0.0;
            int i = k - 1;
            for (; i >= l; --i) {
                double f = s * e[i];
                const double b = c * e[i];
                r = std::hypot(f, g);
                e[i + 1] = r;
                if (r == 0.0) {
                    d[i + 1] -= p;
                    e[k] = 0.0;
                    break;
                }
                s = f / r;
                c = g / r;
                g = d[i + 1] - p;
                r = (d[i] - g) * s + 2.0 * c * b;
                p = s * r;
                d[i + 1] = g + p;
                g = c * r - b;
                if (z)
                    for (int q = 0; q < m; ++q) {
                        double* zc = z->data();
                        f = zc[(i + 1) * m + q];
                        zc[(i + 1) * m + q] = s * zc[i * m + q] + c * f;
                        zc[i * m + q] = c * zc[i * m + q] - s * f;
                    }
            }
            if (r == 0.0 && i >= l) continue;
            d[l] -= p;
            e[l] = g;
            e[k] = 0.0;
        }
    }
    // ascending, vectors along
    std::vector<int> order(m);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return d[a] < d[b]; });
    std::vector<double> d2(m);
    std::vector<double> z2(z ? static_cast<std::size_t>(m) * m : 0);
    for (int j = 0; j < m; ++j) {
        d2[j] = d[order[j]];
        if (z) std::copy(z->begin() + static_cast<std::ptrdiff_t>(order[j]) * m,
                         z->begin() + static_cast<std::ptrdiff_t>(order[j] + 1) * m, z2.begin() + static_cast<std::ptrdiff_t>(j) * m);
    }
    d = d2;
    if (z) *z = z2;
}

struct TriEig {
    std::vector<double> values, vectors;   // vectors column-major m x m
    std::size_t m = 0;
    double z(std::size_t row, std::size_t col) const { return vectors[col * m + row]; }
};

TriEig tridiag_eig(const std::vector<double>& alpha, const std::vector<double>& beta, std::size_t m, bool vectors) {
    TriEig t;
    t.m = m;
    if (m == 0) return t;
    for (std::size_t i = 0; i < m; ++i)
        if (!std::isfinite(alpha[i]) || (i + 1 < m && !std::isfinite(beta[i + 1])))
            throw std::runtime_error("tridiagonal eigensolve: non-finite entry");
    t.values.assign(alpha.begin(), alpha.begin() + static_cast<std::ptrdiff_t>(m));
    std::vector<double> e(m > 1 ? m - 1 : 0);
    for (std::size_t i = 0; i + 1 < m; ++i) e[i] = beta[i + 1];
    if (vectors) {
        t.vectors.assign(m * m, 0.0);
        for (std::size_t i = 0; i < m; ++i) t.vectors[i * m + i] = 1.0;
        tridiag_ql(t.values, e, &t.vectors);
        // sign convention: largest-magnitude component positive (the tests compare |z|)
    } else {
        tridiag_ql(t.values, e, nullptr);
    }
    return t;
}

// The unit eigenvector of eigenvalue lam by inverse iteration (tridiagonal LU with partial pivoting).
std::vector<double> tridiag_inverse_iteration(const std::vector<double>& a, const std::vector<double>& b,
                                              std::size_t m, double lam) {
    std::vector<double> x(m, 1.0);
    if (m == 1) return x;
    double scale = 0.0;
    for (std::size_t i = 0; i < m; ++i) scale = std::max(scale, std::abs(a[i]) + (i + 1 < m ? std::abs(b[i + 1]) : 0.0));
    const double shift = lam + std::max(scale, 1e-300) * 1e-13;
    for (int it = 0; it < 3; ++it) {
        // solve (T - shift) y = x with Gaussian elimination and partial pivoting on the band
        std::vector<double> dl(m), dd(m), du(m), du2(m, 0.0), rhs = x;
        for (std::size_t i = 0; i < m; ++i) {
            dd[i] = a[i] - shift;
            if (i + 1 < m) du[i] = b[i + 1], dl[i] = b[i + 1];
        }
        std::vector<int> swapped(m, 0);
        for (std::size_t i = 0; i + 1 < m; ++i) {
            if (std::abs(dd[i]) >= std::abs(dl[i])) {
                if (dd[i] == 0.0) dd[i] = 1e-300;
                const double f = dl[i] / dd[i];
                dd[i + 1] -= f * du[i];
                if (i + 2 < m) du2[i] = 0.0;
                rhs[i + 1] -= f * rhs[i];
                dl[i] = f;
            } else {
                const double f = dd[i] / dl[i];
                dd[i] = dl[i];
                const double tmp = dd[i + 1];
                dd[i + 1] = du[i] - f * tmp;
                if (i + 2 < m) {
                    du2[i] = du[i + 1];
                    du[i + 1] = -f * du2[i];
                }
                du[i] = tmp;
                std::swap(rhs[i], rhs[i + 1]);
                rhs[i + 1] -= f * rhs[i];
                dl[i] = f;
                swapped[i] = 1;
            }
        }
        if (dd[m - 1] == 0.0) dd[m - 1] = 1e-300;
        std::vector<double> y(m);
        y[m - 1] = rhs[m - 1] / dd[m - 1];
        if (m >= 2) y[m - 2] = (rhs[m - 2] - du[m - 2] * y[m - 1]) / dd[m - 2];
        for (std::size_t ii = m - 2; ii-- > 0;) y[ii] = (rhs[ii] - du[ii] * y[ii + 1] - du2[ii] * y[ii + 2]) / dd[ii];
        double nrm = 0.0;
        for (double v : y) nrm += v * v;
        nrm = std::sqrt(nrm);
        for (std::size_t i = 0; i < m; ++i) x[i] = y[i] / nrm;
    }
    return x;
}

// lowest_levels / leading_block / lowest_level (block_solve.cpp:335-385). The reference's
// tridiag_ends (LAPACK dstevx: the 4 lowest pairs and the top value) is restated as QL values
// plus inverse-iteration vectors.
template <class Bound>
bool lowest_levels(std::size_t m, const double* w, Bound&& bound, double scale, std::size_t k, std::vector<double>* out) {
    std::size_t found = 0;
    for (std::size_t j = 0; j < m && found < k;) {
        const double first = w[j];
        std::size_t i = j;
        bool converged = false;
        double value = first;
        for (; i < m && std::abs(w[i] - first) <= 1e-9 * scale; ++i)
            if (!converged && bound(i) <= 1e-7 * scale) {
                converged = true;
                value = w[i];
            }
        if (!converged) return false;
        if (out) out->push_back(value);
        ++found;
        j = i;
    }
    return found >= k;
}

std::size_t leading_block(const std::vector<double>& alpha, const std::vector<double>& beta, std::size_t m) {
    double scale = 0.0;
    for (std::size_t i = 0; i < m; ++i) {
        scale = std::max(scale, std::abs(alpha[i]));
        if (i + 1 < beta.size()) scale = std::max(scale, std::abs(beta[i + 1]));
    }
    for (std::size_t i = 1; i < m; ++i)
        if (std::abs(beta[i]) <= 1e-12 * scale) return i;
    return m;
}

bool lowest_level(const std::vector<double>& alpha, const std::vector<double>& beta, std::size_t m, std::vector<double>* out) {
    const double beta_m = beta.size() > m ? std::abs(beta[m]) : 0.0;
    const TriEig all = tridiag_eig(alpha, beta, m, false);
    const std::size_t c = std::min<std::size_t>(4, m);
    const double scale = std::max({std::abs(all.values.front()), std::abs(all.values.back()), 1e-300});
    if (c < m && std::abs(all.values[c - 1] - all.values.front()) <= 1e-9 * scale) {
        const TriEig f = tridiag_eig(alpha, beta, m, true);
        return lowest_levels(m, f.values.data(), [&](std::size_t j) { return beta_m * std::abs(f.z(m - 1, j)); }, scale, 1, out);
    }
    std::vector<double> zl(c);
    for (std::size_t j = 0; j < c; ++j) zl[j] = tridiag_inverse_iteration(alpha, beta, m, all.values[j])[m - 1];
    return lowest_levels(c, all.values.data(), [&](std::size_t j) { return beta_m * std::abs(zl[j]); }, scale, 1, out);
}

// ---------------------------------------------------------------------------------------------
// Seeds (sample_seed.h:37-89; block_solve.cpp:268-277).
// ---------------------------------------------------------------------------------------------
std::mt19937 sample_engine(std::uint64_t base_seed, std::uint64_t sample) {
    std::uint64_t z = base_seed + 0x9E3779B97F4A7C15ULL * (sample + 1);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    z = z ^ (z >> 31);
    return std::mt19937(static_cast<std::mt19937::result_type>(z));
}

// The reference draws Complex(nd(gen), nd(gen)) (sample_seed.h:84-85, lanczos.h:70-77); GCC evaluates
// those arguments right to left, so the imaginary part is the first draw (pinned by the seed tests).
template <class Gen> Vec gaussian_draw(std::size_t n, Gen& gen) {
    std::normal_distribution<double> nd(0.0, 1.0);
    Vec v(n);
    for (std::size_t i = 0; i < n; ++i) {
        const double im = nd(gen);
        const double re = nd(gen);
        v[i] = Complex(re, im);
    }
    return v;
}

Vec sample_vector(std::uint64_t base, std::uint64_t s, std::size_t n) {
    std::mt19937 gen = sample_engine(base, s);
    Vec v = gaussian_draw(n, gen);
    const double nrm = vnrm2(v);
    if (nrm > 0.0)
        for (auto& x : v) x *= Complex(1.0 / nrm, 0.0);
    return v;
}

Vec staged_seed(std::uint64_t seed, std::size_t n) {
    std::mt19937_64 gen(seed);
    return gaussian_draw(n, gen);
}

// ---------------------------------------------------------------------------------------------
// FTLM (ftlm.h:165-235): per-sample moments about the lowest weighted Ritz value, Jensen-correct
// combine about the common reference.
// ---------------------------------------------------------------------------------------------
struct Moments {
    double e_min = 0.0;
    std::vector<double> Z, E1, E2;
};

Moments sample_moments(const std::vector<double>& ritz, const std::vector<double>& w, const std::vector<double>& betas) {
    Moments m;
    m.e_min = std::numeric_limits<double>::infinity();
    for (std::size_t i = 0; i < ritz.size(); ++i)
        if (w[i] > 0.0) m.e_min = std::min(m.e_min, ritz[i]);
    if (!std::isfinite(m.e_min)) m.e_min = *std::min_element(ritz.begin(), ritz.end());
    for (double beta : betas) {
        double z = 0.0, e1 = 0.0, e2 = 0.0;
        for (std::size_t i = 0; i < ritz.size(); ++i) {
            const double x = ritz[i] - m.e_min;
            const double b = w[i] * std::exp(-beta * x);
            z += b;
            e1 += x * b;
            e2 += x * x * b;
        }
        m.Z.push_back(z);
        m.E1.push_back(e1);
        m.E2.push_back(e2);
    }
    return m;
}

void combine_samples(const std::vector<Moments>& S, std::uint64_t n, const std::vector<double>& betas, double* lnZ,
                     double* E, double* V) {
    double e_ref = S.front().e_min;
    for (const auto& s : S) e_ref = std::min(e_ref, s.e_min);
    const double ln_n = std::log(static_cast<double>(n));
    const double R = static_cast<double>(S.size());
    for (std::size_t t = 0; t < betas.size(); ++t) {
        const double beta = betas[t];
        double z = 0.0, e1 = 0.0, e2 = 0.0;
        for (const auto& s : S) {
            const double d = s.e_min - e_ref, r = std::exp(-beta * d);
            z += s.Z[t] * r;
            e1 += (s.E1[t] + d * s.Z[t]) * r;
            e2 += (s.E2[t] + 2.0 * d * s.E1[t] + d * d * s.Z[t]) * r;
        }
        z /= R;
        e1 /= R;
        e2 /= R;
        if (z > 1e-300) {
            const double m1 = e1 / z, m2 = e2 / z;
            lnZ[t] = ln_n + std::log(z) - beta * e_ref;
            E[t] = e_ref + m1;
            V[t] = std::max(m2 - m1 * m1, 0.0);
        } else {
            lnZ[t] = -beta * e_ref;
            E[t] = e_ref;
            V[t] = 0.0;
        }
    }
}

Moments moments_of_run(const std::vector<double>& alpha, const std::vector<double>& beta, const std::vector<double>& betas) {
    const TriEig t = tridiag_eig(alpha, beta, alpha.size(), true);
    std::vector<double> w(t.m);
    for (std::size_t j = 0; j < t.m; ++j) w[j] = t.vectors[j * t.m] * t.vectors[j * t.m];
    return sample_moments(t.values, w, betas);
}

// continued_fraction (cf.h:39-62).
void continued_fraction(const double* alpha, const double* beta, std::size_t M, const double* omega, int nw, double eta,
                        double norm_sq, double* S) {
    for (int iw = 0; iw < nw; ++iw) {
        S[iw] = 0.0;
        if (M == 0) continue;
        const Complex z(omega[iw], eta);
        Complex G(0.0, 0.0);
        for (std::size_t n = M - 1; n >= 1; --n) {
            const double b2 = beta[n] * beta[n];
            const Complex d = z - Complex(alpha[n], 0.0) - G;
            G = std::abs(d) > 1e-300 ? Complex(b2, 0.0) / d : Complex(0.0, 0.0);
        }
        const Complex d = z - Complex(alpha[0], 0.0) - G;
        const Complex G0 = std::abs(d) > 1e-300 ? Complex(norm_sq, 0.0) / d : Complex(0.0, 0.0);
        S[iw] = -G0.imag() / 3.14159265358979323846;
    }
}

template <class F> int guarded(F&& f) {
    try {
        f();
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

struct SectorWalk {
    const Program* P;
    const Sector* S;
    void operator()(const Vec& in, Vec& out) const {
        for (std::uint64_t r = 0; r < S->reps.size(); ++r) {
            Complex acc(0.0, 0.0);
            for_each_entry(*P, *S, *S, true, r, [&](std::uint64_t c, const Complex& v) { acc += v * in[c]; });
            out[r] = acc;
        }
    }
};

Vec to_vec(const double* p, std::size_t n) {
    Vec v(n);
    std::memcpy(static_cast<void*>(v.data()), p, n * sizeof(Complex));
    return v;
}

}  // namespace

extern "C" {

const char* qo_last_error(void) { return g_err.c_str(); }

void* qo_sector_new(int n_sites, int n_up, int G, const int32_t* perms, const uint64_t* flips, const double* chars,
                    int slc_mode) {
    try {
        if (n_sites < 1 || n_sites > 64 || G < 1) throw std::invalid_argument("qo_sector_new: bad sizes");
        auto* S = new Sector;
        S->grp.N = n_sites;
        S->grp.G = G;
        S->grp.perms.assign(perms, perms + static_cast<std::size_t>(G) * n_sites);
        S->grp.flips.assign(G, 0ULL);
        if (flips) S->grp.flips.assign(flips, flips + G);
        S->grp.build();
        S->slc = make_slc(S->grp, slc_mode);
        S->n_up = n_up;
        for (int g = 0; g < G; ++g) S->chars.emplace_back(chars[2 * g], chars[2 * g + 1]);
        build_sector(*S);
        return S;
    } catch (const std::exception& e) {
        g_err = e.what();
        return nullptr;
    }
}

void qo_sector_free(void* s) { delete static_cast<Sector*>(s); }
uint64_t qo_sector_dim(void* s) { return static_cast<Sector*>(s)->reps.size(); }

void qo_sector_get(void* s, uint64_t* reps, double* inv_norms) {
    const auto* S = static_cast<Sector*>(s);
    std::copy(S->reps.begin(), S->reps.end(), reps);
    std::copy(S->inv_norms.begin(), S->inv_norms.end(), inv_norms);
}

int qo_sector_slc(void* s, int* L, int* m, int32_t* key_bit) {
    const auto* S = static_cast<Sector*>(s);
    if (!S->slc.on) return 0;
    *L = S->slc.L;
    *m = S->slc.m;
    if (key_bit) std::copy(S->slc.key_bit.begin(), S->slc.key_bit.end(), key_bit);
    return 1;
}

int64_t qo_index_and_projection(void* s, uint64_t state, double* proj) {
    Complex p;
    const std::int64_t k = static_cast<Sector*>(s)->index_and_projection(state, p);
    proj[0] = p.real();
    proj[1] = p.imag();
    return k;
}

void* qo_prog_new(uint32_t n_groups, const uint64_t* group_flip, const int32_t* group_setbits,
                  const uint32_t* group_vbegin, uint32_t n_vsub, const uint64_t* vsub_val, const uint32_t* vsub_tbegin,
                  uint32_t n_terms, const uint64_t* term_sign, const double* term_coeff) {
    auto* P = new Program;
    P->group_flip.assign(group_flip, group_flip + n_groups);
    P->group_setbits.assign(group_setbits, group_setbits + n_groups);
    P->group_vbegin.assign(group_vbegin, group_vbegin + n_groups + 1);
    P->vsub_val.assign(vsub_val, vsub_val + n_vsub);
    P->vsub_tbegin.assign(vsub_tbegin, vsub_tbegin + n_vsub + 1);
    P->term_sign.assign(term_sign, term_sign + n_terms);
    for (uint32_t k = 0; k < n_terms; ++k) P->term_coeff.emplace_back(term_coeff[2 * k], term_coeff[2 * k + 1]);
    return P;
}

void qo_prog_free(void* p) { delete static_cast<Program*>(p); }

int qo_gather(void* row, void* col, void* prog, const double* in, double* out) {
    return guarded([&] {
        const auto* R = static_cast<Sector*>(row);
        const auto* Cs = static_cast<Sector*>(col);
        const auto* P = static_cast<Program*>(prog);
        const auto* x = reinterpret_cast<const Complex*>(in);
        auto* y = reinterpret_cast<Complex*>(out);
        for (std::uint64_t r = 0; r < R->reps.size(); ++r) {
            Complex acc(0.0, 0.0);
            for_each_entry(*P, *R, *Cs, R == Cs, r, [&](std::uint64_t c, const Complex& v) { acc += v * x[c]; });
            y[r] = acc;
        }
    });
}

int qo_csr(void* row, void* col_sector, void* prog, uint64_t* row_ptr, uint32_t* col, double* val) {
    return guarded([&] {
        const auto* R = static_cast<Sector*>(row);
        const auto* Cs = static_cast<Sector*>(col_sector);
        const auto* P = static_cast<Program*>(prog);
        std::vector<std::pair<std::uint64_t, Complex>> ents;
        row_ptr[0] = 0;
        for (std::uint64_t r = 0; r < R->reps.size(); ++r) {
            ents.clear();
            for_each_entry(*P, *R, *Cs, R == Cs, r, [&](std::uint64_t c, const Complex& v) { ents.emplace_back(c, v); });
            // merge_row (sector_rows.h:147-158)
            std::stable_sort(ents.begin(), ents.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
            std::uint64_t e = row_ptr[r];
            for (std::size_t i = 0; i < ents.size();) {
                Complex sum = ents[i].second;
                std::size_t k = i + 1;
                for (; k < ents.size() && ents[k].first == ents[i].first; ++k) sum += ents[k].second;
                if (sum != Complex(0.0, 0.0)) {
                    if (col) {
                        col[e] = static_cast<std::uint32_t>(ents[i].first);
                        val[2 * e] = sum.real();
                        val[2 * e + 1] = sum.imag();
                    }
                    ++e;
                }
                i = k;
            }
            row_ptr[r + 1] = e;
        }
    });
}

int qo_count_emitted(void* row, void* col, void* prog, uint64_t* emitted) {
    return guarded([&] {
        const auto* R = static_cast<Sector*>(row);
        const auto* Cs = static_cast<Sector*>(col);
        const auto* P = static_cast<Program*>(prog);
        std::uint64_t n = 0;
        for (std::uint64_t r = 0; r < R->reps.size(); ++r)
            for_each_entry(*P, *R, *Cs, R == Cs, r, [&](std::uint64_t, const Complex&) { ++n; });
        *emitted = n;
    });
}

int qo_lanczos(void* sec, void* prog, const double* v0, int max_iter, int reorth, double breakdown_tol, double* alpha,
               double* beta, int* iters) {
    return guarded([&] {
        const auto* S = static_cast<Sector*>(sec);
        const SectorWalk H{static_cast<Program*>(prog), S};
        std::vector<double> a, b;
        lanczos(H, to_vec(v0, S->reps.size()), static_cast<std::size_t>(max_iter), reorth, breakdown_tol,
                [](const std::vector<double>&, const std::vector<double>&) { return false; }, a, b);
        std::copy(a.begin(), a.end(), alpha);
        std::copy(b.begin(), b.end(), beta);
        *iters = static_cast<int>(a.size());
    });
}

int qo_scan_lowest(void* sec, void* prog, int max_iter, double* e0, int* iters, int* converged) {
    return guarded([&] {
        const auto* S = static_cast<Sector*>(sec);
        const std::uint64_t nb = S->reps.size();
        const SectorWalk H{static_cast<Program*>(prog), S};
        const std::size_t budget = max_iter > 0 ? static_cast<std::size_t>(max_iter) : 400;
        const std::size_t mi = std::min<std::size_t>(nb, budget);
        const int reorth = nb <= mi ? 1 : 0;
        std::vector<double> a, b;
        lanczos(H, staged_seed(0x51ED0B70ULL, nb), mi, reorth, 1e-300,
                [](const std::vector<double>& al, const std::vector<double>& be) {
                    const std::size_t m_all = al.size();
                    const std::size_t m = leading_block(al, be, m_all);
                    if (m == m_all && m_all < 3) return false;
                    return lowest_level(al, be, m, nullptr);
                },
                a, b);
        *iters = static_cast<int>(a.size());
        *converged = 0;
        *e0 = std::nan("");
        if (a.empty()) return;
        std::vector<double> vals;
        const std::size_t m = leading_block(a, b, a.size());
        *converged = lowest_level(a, b, m, &vals) ? 1 : 0;
        if (!vals.empty()) *e0 = vals.front();
    });
}

int qo_tridiag_eig(const double* alpha, const double* beta, int m, double* values, double* vectors) {
    return guarded([&] {
        std::vector<double> a(alpha, alpha + m), b(beta, beta + m + 1);
        const TriEig t = tridiag_eig(a, b, static_cast<std::size_t>(m), vectors != nullptr);
        std::copy(t.values.begin(), t.values.end(), values);
        if (vectors) std::copy(t.vectors.begin(), t.vectors.end(), vectors);
    });
}

void qo_sample_vector(uint64_t base_seed, uint64_t s, uint64_t n, double* out) {
    const Vec v = sample_vector(base_seed, s, static_cast<std::size_t>(n));
    std::memcpy(out, v.data(), n * sizeof(Complex));
}

void qo_staged_seed(uint64_t seed, uint64_t n, double* out) {
    const Vec v = staged_seed(seed, static_cast<std::size_t>(n));
    std::memcpy(out, v.data(), n * sizeof(Complex));
}

int qo_ftlm(void* sec, void* prog, int samples, int depth, uint64_t seed, const double* betas, int nb, double* lnZ,
            double* E, double* V, double* e_min) {
    return guarded([&] {
        const auto* S = static_cast<Sector*>(sec);
        const auto* P = static_cast<Program*>(prog);
        const SectorWalk H{P, S};
        const std::vector<double> bs(betas, betas + nb);
        const double tol = 64.0 * std::numeric_limits<double>::epsilon() * (P->norm_bound() > 0.0 ? P->norm_bound() : 1.0);
        std::vector<Moments> mom;
        double gs = std::numeric_limits<double>::infinity();
        for (int s = 0; s < samples; ++s) {
            std::vector<double> a, b;
            lanczos(H, sample_vector(seed, static_cast<std::uint64_t>(s), S->reps.size()), static_cast<std::size_t>(depth), 2,
                    tol, [](const std::vector<double>&, const std::vector<double>&) { return false; }, a, b);
            if (a.empty()) continue;
            mom.push_back(moments_of_run(a, b, bs));
            gs = std::min(gs, mom.back().e_min);
        }
        if (mom.empty()) throw std::runtime_error("qo_ftlm: every sample failed");
        combine_samples(mom, S->reps.size(), bs, lnZ, E, V);
        *e_min = gs;
    });
}

int qo_sample_moments(const double* alpha, const double* beta, int m, const double* betas, int nb, double* e_min,
                      double* Z, double* E1, double* E2) {
    return guarded([&] {
        std::vector<double> a(alpha, alpha + m), b(beta, beta + m + 1);
        const Moments mo = moments_of_run(a, b, std::vector<double>(betas, betas + nb));
        *e_min = mo.e_min;
        std::copy(mo.Z.begin(), mo.Z.end(), Z);
        std::copy(mo.E1.begin(), mo.E1.end(), E1);
        std::copy(mo.E2.begin(), mo.E2.end(), E2);
    });
}

void qo_continued_fraction(const double* alpha, const double* beta, int m, const double* omega, int nw, double eta,
                           double norm_sq, double* S) {
    continued_fraction(alpha, beta, static_cast<std::size_t>(m), omega, nw, eta, norm_sq, S);
}

int qo_cf(void* sec, void* prog, const double* phi, int depth, const double* omega, int nw, double eta, double shift,
          double tolerance, double* S_out, double* shift_out) {
    return guarded([&] {
        const auto* S = static_cast<Sector*>(sec);
        const SectorWalk H{static_cast<Program*>(prog), S};
        Vec p = to_vec(phi, S->reps.size());
        const double nrm = vnrm2(p);
        for (int i = 0; i < nw; ++i) S_out[i] = 0.0;
        *shift_out = 0.0;
        if (nrm < 1e-14) return;
        vscale(Complex(1.0 / nrm, 0.0), p);
        std::vector<double> a, b;
        lanczos(H, p, static_cast<std::size_t>(depth), 0, tolerance,
                [](const std::vector<double>&, const std::vector<double>&) { return false; }, a, b);
        if (a.empty()) return;
        double sh = shift;
        if (std::isnan(sh)) sh = tridiag_eig(a, b, a.size(), false).values.front();
        for (auto& x : a) x -= sh;
        *shift_out = sh;
        continued_fraction(a.data(), b.data(), a.size(), omega, nw, eta, nrm * nrm, S_out);
    });
}

}  // extern "C"
