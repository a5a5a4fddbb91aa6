// =============================================================================
// oracle/ref_glue.cpp -- TEST INFRASTRUCTURE, not product code.
//
// A C-ABI around the reference engine's own CPU implementation of the hot path, compiled from
// the reference's headers and src/ops/{algebra,program}.cpp where they lie (oracle/Makefile),
// into oracle/_ref/libqed_ref.so. The tests and bench.py's reference arm load it to check the
// restated oracle (oracle/qed_oracle.cpp) and the CUDA path against the reference itself.
//
// Everything that runs here is the reference's code (MaskedOperator, compile_operator /
// compile_program, CompiledGroup + SublatticeCode + build_orbit_table_fixed_sz_streaming,
// RepSectorData lookups, sector_gather, build_sector_csr + ReducedSymmetryCsr::spmv,
// lanczos_kernel<CpuBackend>, tridiag_ends/tridiag_eig, krylov_schur_kernel, ftlm_kernel,
// cf_spectral_from_vector) except the few driver lines that live in Eigen-bound source files
// the reference cannot compile without Eigen; those are restated below, each citing its origin:
//   filter_reps            src/engine/group_sector.cpp:159-205
//   lowest_scan_lane       src/engine/block_solve.cpp:335-398, 528-598
//   krylov_schur_lane      src/engine/block_solve.cpp:433-510
//   staged_seed            src/engine/block_solve.cpp:263-277
// =============================================================================
#include <ed/basis/combinadic.h>
#include <ed/basis/compiled_group.h>
#include <ed/basis/orbit_table.h>
#include <ed/basis/rep_sector.h>
#include <ed/basis/sublattice_code.h>
#include <ed/core/numerics.h>
#include <ed/dynamics/cf.h>
#include <ed/krylov/krylov_schur.h>
#include <ed/krylov/lanczos.h>
#include <ed/krylov/subspace_policy.h>
#include <ed/krylov/tridiag.h>
#include <ed/matvec/cpu_backend.h>
#include <ed/matvec/rep_symmetry_basis_policy.h>
#include <ed/matvec/sector_rows.h>
#include <ed/ops/algebra.h>
#include <ed/ops/program.h>
#include <ed/thermal/ftlm.h>
#include <ed/thermal/sample_seed.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <memory>
#include <optional>
#include <random>
#include <string>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

using Complex = std::complex<double>;

namespace {

thread_local std::string g_err;

struct RefSector {
    ed::symmetry::RepSectorData rd;
    std::shared_ptr<const ed::symmetry::SharedRankLookup> srl;
    std::uint64_t scanned = 0;
};

// Restated from src/engine/group_sector.cpp:159-205 (filter_reps): per representative of the orbit
// table, inv_norm = 1/sqrt(|sum_{h in Stab} chi(h)|^2 / |Stab|) (projected_norm_sq_stab,
// include/ed/basis/orbit_table.h:93-99), reps whose squared norm is <= 1e-12 dropped, order kept.
void filter_reps(const ed::symmetry::OrbitTable& tab, const std::vector<Complex>& chi,
                 ed::symmetry::RepSectorData& rd, std::vector<std::int32_t>* local) {
    rd.slc = tab.slc;
    const std::size_t n = tab.reps.size();
    rd.reps.clear();
    rd.inv_norms.clear();
    if (local) local->assign(n, -1);
    for (std::size_t i = 0; i < n; ++i) {
        const double nsq = ed::symmetry::projected_norm_sq_stab(tab.stabilizer_of(i), chi);
        const double inv = nsq <= 1e-12 ? 0.0 : 1.0 / std::sqrt(nsq);
        if (inv == 0.0) continue;
        if (local) (*local)[i] = static_cast<std::int32_t>(rd.reps.size());
        rd.reps.push_back(tab.reps[i]);
        rd.inv_norms.push_back(inv);
    }
}

// Restated from src/engine/block_solve.cpp:263-277 (staged_seed, host part): a unit-variance
// complex Gaussian start drawn from mt19937_64(seed), (re, im) per entry (gaussian_entry,
// include/ed/krylov/lanczos.h:70-77).
std::vector<Complex> staged_seed_host(std::size_t n, std::uint64_t seed) {
    std::vector<Complex> host(n);
    std::mt19937_64 gen(seed);
    std::normal_distribution<double> nd(0.0, 1.0);
    for (auto& c : host) c = ed::krylov::gaussian_entry<Complex>(nd, gen);
    return host;
}

// Restated from src/engine/block_solve.cpp:335-348 (lowest_levels).
template <class Bound>
bool lowest_levels(std::size_t m, const double* w, Bound&& bound, double scale, std::size_t k,
                   std::vector<double>* out) {
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

// Restated from src/engine/block_solve.cpp:357-368 (leading_block).
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

// Restated from src/engine/block_solve.cpp:373-385 (lowest_level).
bool lowest_level(const std::vector<double>& alpha, const std::vector<double>& beta, std::size_t m,
                  std::vector<double>* out) {
    const double beta_m = beta.size() > m ? std::abs(beta[m]) : 0.0;
    const ed::krylov::TridiagEnds t = ed::krylov::tridiag_ends(alpha, beta, m, 4);
    const std::size_t c = t.values.size();
    const double scale = std::max({std::abs(t.values.front()), std::abs(t.top), 1e-300});
    if (c < m && std::abs(t.values[c - 1] - t.values.front()) <= 1e-9 * scale) {
        const ed::krylov::TridiagEig f = ed::krylov::tridiag_eig(alpha, beta, m, true);
        return lowest_levels(
            m, f.values.data(), [&](std::size_t j) { return beta_m * std::abs(f.z(m - 1, j)); }, scale, 1, out);
    }
    return lowest_levels(
        c, t.values.data(), [&](std::size_t j) { return beta_m * std::abs(t.z(m - 1, j)); }, scale, 1, out);
}

struct Walk {
    const RefSector* row;
    const RefSector* col;
    const ed::ops::MaskedProgram* prog;
    bool same;
    ed::matvec::basis::RepSymmetryBasisPolicy rp, cp;
    void operator()(const Complex* in, Complex* out, std::size_t) const {
        ed::matvec::cross_gather(prog->view(), rp, cp, same, row->rd.dim(), in, out);
    }
};

double program_norm_bound(const ed::ops::MaskedProgram& P) {
    double s = 0.0;
    for (const auto& c : P.term_coeff) s += std::abs(c);
    return s;
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

}  // namespace

extern "C" {

const char* qref_last_error() { return g_err.c_str(); }

void qref_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

int qref_max_threads() {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

// ---------------- operators and programs ----------------
void* qref_op_new(int n_sites) {
    try {
        return new ed::ops::MaskedOperator(n_sites);
    } catch (const std::exception& e) {
        g_err = e.what();
        return nullptr;
    }
}
void qref_op_free(void* h) { delete static_cast<ed::ops::MaskedOperator*>(h); }

// O += coeff * prod_k ops[k](sites[k]) (MaskedOperator::product, include/ed/ops/algebra.h:25-28).
int qref_op_add_product(void* h, const char* ops, const int* sites, int nfac, double re, double im) {
    return guarded([&] {
        auto* O = static_cast<ed::ops::MaskedOperator*>(h);
        std::vector<int> s(sites, sites + nfac);
        O->add(ed::ops::MaskedOperator::product(O->n_sites(), std::string(ops, static_cast<std::size_t>(nfac)), s,
                                                Complex(re, im)));
    });
}

// The row program of O on one sector: compile_operator(O^dagger) (include/ed/ops/operator.h:132-137).
void* qref_prog_rows(void* h) {
    try {
        const auto* O = static_cast<ed::ops::MaskedOperator*>(h);
        return new ed::ops::MaskedProgram(ed::ops::compile_operator(O->dagger()));
    } catch (const std::exception& e) {
        g_err = e.what();
        return nullptr;
    }
}

// Rows in sector `row` of O from sector `col`: the program of (O_lambda)^dagger compiled with the
// row sector as the ket and the column sector as the bra (include/ed/matvec/sector_rows.h:16-19).
void* qref_prog_cross(void* h, void* row, void* col) {
    try {
        const auto* O = static_cast<ed::ops::MaskedOperator*>(h);
        const auto* R = static_cast<RefSector*>(row);
        const auto* C = static_cast<RefSector*>(col);
        return new ed::ops::MaskedProgram(ed::ops::compile_program({O->dagger()}, R->rd, C->rd));
    } catch (const std::exception& e) {
        g_err = e.what();
        return nullptr;
    }
}

void qref_prog_free(void* p) { delete static_cast<ed::ops::MaskedProgram*>(p); }

void qref_prog_sizes(void* p, std::uint32_t* n_groups, std::uint32_t* n_vsub, std::uint32_t* n_terms) {
    const auto* P = static_cast<ed::ops::MaskedProgram*>(p);
    *n_groups = static_cast<std::uint32_t>(P->group_flip.size());
    *n_vsub = static_cast<std::uint32_t>(P->vsub_val.size());
    *n_terms = static_cast<std::uint32_t>(P->term_sign.size());
}

void qref_prog_arrays(void* p, std::uint64_t* group_flip, std::int32_t* group_setbits, std::uint32_t* group_vbegin,
                      std::uint64_t* vsub_val, std::uint32_t* vsub_tbegin, std::uint64_t* term_sign,
                      double* term_coeff) {
    const auto* P = static_cast<ed::ops::MaskedProgram*>(p);
    std::copy(P->group_flip.begin(), P->group_flip.end(), group_flip);
    std::copy(P->group_setbits.begin(), P->group_setbits.end(), group_setbits);
    std::copy(P->group_vbegin.begin(), P->group_vbegin.end(), group_vbegin);
    std::copy(P->vsub_val.begin(), P->vsub_val.end(), vsub_val);
    std::copy(P->vsub_tbegin.begin(), P->vsub_tbegin.end(), vsub_tbegin);
    std::copy(P->term_sign.begin(), P->term_sign.end(), term_sign);
    for (std::size_t k = 0; k < P->term_coeff.size(); ++k) {
        term_coeff[2 * k] = P->term_coeff[k].real();
        term_coeff[2 * k + 1] = P->term_coeff[k].imag();
    }
}

// ---------------- sectors ----------------
// slc_mode: 0 off, 1 forced, -1 the size rule under the relaxed hint (device verbs, eigs), -2 the
// strict one (include/ed/basis/sublattice_code.h:23-34). lookup: 0 the engine's default (a shared
// rank table within ED_SYM_REP_RANKTABLE_BUDGET_GIB, else buckets), 1 force the rank table,
// 2 force buckets, 3 plain binary search.
void* qref_sector_new(int n_sites, int n_up, int G, const int* perms, const std::uint64_t* flips, const double* chars,
                      int slc_mode, int lookup) {
    try {
        std::vector<std::vector<int>> P(static_cast<std::size_t>(G));
        for (int g = 0; g < G; ++g) P[g].assign(perms + g * n_sites, perms + (g + 1) * n_sites);
        std::vector<std::uint64_t> F(static_cast<std::size_t>(G), 0ULL);
        if (flips) F.assign(flips, flips + G);
        // CompiledGroup::from_elements asks SublatticeCode::of, which reads ED_SYM_SUBLATTICE and the
        // relaxed-rule hint: set both for this build.
        if (slc_mode == 0)
            setenv("ED_SYM_SUBLATTICE", "0", 1);
        else if (slc_mode == 1)
            setenv("ED_SYM_SUBLATTICE", "1", 1);
        else
            unsetenv("ED_SYM_SUBLATTICE");
        const ed::symmetry::SublatticeRuleScope scope(slc_mode != -2);
        ed::symmetry::CompiledGroup cg = ed::symmetry::CompiledGroup::from_elements(P, F, n_sites);
        unsetenv("ED_SYM_SUBLATTICE");
        auto* S = new RefSector;
        ed::symmetry::OrbitTable tab =
            ed::symmetry::build_orbit_table_fixed_sz_streaming(static_cast<std::uint64_t>(n_sites), n_up, cg);
        S->scanned = tab.subspace_dim;
        auto& rd = S->rd;
        rd.n_sites = n_sites;
        rd.n_up = n_up;
        rd.group_size = G;
        rd.characters.resize(static_cast<std::size_t>(G));
        for (int g = 0; g < G; ++g) rd.characters[g] = Complex(chars[2 * g], chars[2 * g + 1]);
        for (const auto& p : P) rd.perms_flat.insert(rd.perms_flat.end(), p.begin(), p.end());
        bool any_flip = false;
        for (auto f : F) any_flip = any_flip || f != 0;
        if (any_flip) rd.flip_masks = F;
        const ed::core::combinadic::BinomialTable b(n_sites);
        const bool rank_ok = lookup == 1 || (lookup == 0 && ed::symmetry::rep_rank_table_enabled(b.at(n_sites, n_up)));
        if (rank_ok && lookup != 2 && lookup != 3) {
            S->srl = ed::symmetry::make_shared_rank_lookup(tab.reps, n_sites, n_up);
            rd.shared_rank = S->srl;
            filter_reps(tab, rd.characters, rd, &rd.local_of_shared);
        } else {
            filter_reps(tab, rd.characters, rd, nullptr);
        }
        rd.build_perm_lut();
        if (lookup != 3) rd.build_buckets();
        return S;
    } catch (const std::exception& e) {
        g_err = e.what();
        return nullptr;
    }
}

void qref_sector_free(void* s) { delete static_cast<RefSector*>(s); }
std::uint64_t qref_sector_dim(void* s) { return static_cast<RefSector*>(s)->rd.dim(); }
std::uint64_t qref_sector_scanned(void* s) { return static_cast<RefSector*>(s)->scanned; }

void qref_sector_get(void* s, std::uint64_t* reps, double* inv_norms) {
    const auto& rd = static_cast<RefSector*>(s)->rd;
    std::copy(rd.reps.begin(), rd.reps.end(), reps);
    std::copy(rd.inv_norms.begin(), rd.inv_norms.end(), inv_norms);
}

// The sublattice code the representatives were found with: 1 and its block size / blocks / mean
// candidates, or 0 (the plain order).
int qref_sector_slc(void* s, int* L, int* m, double* mean_cand) {
    const auto& rd = static_cast<RefSector*>(s)->rd;
    if (!rd.slc) return 0;
    *L = rd.slc->block_size();
    *m = rd.slc->blocks();
    *mean_cand = rd.slc->mean_candidates();
    return 1;
}

// The code's key position of every site (n_sites ints); 0 when there is no code.
int qref_sector_slc_keybits(void* s, int* key_bit) {
    const auto& rd = static_cast<RefSector*>(s)->rd;
    if (!rd.slc) return 0;
    std::copy(rd.slc->key_bit().begin(), rd.slc->key_bit().end(), key_bit);
    return 1;
}

// index_and_projection of a state (include/ed/matvec/rep_symmetry_basis_policy.h:221-241).
std::int64_t qref_index_and_projection(void* s, std::uint64_t state, double* proj) {
    const auto pol = static_cast<RefSector*>(s)->rd.make_policy();
    Complex p;
    const std::int64_t k = pol.index_and_projection(state, p);
    proj[0] = p.real();
    proj[1] = p.imag();
    return k;
}

// The reference's sublattice code of a group (SublatticeCode::of, include/ed/basis/sublattice_code.h:164-191)
// under a mode: 1 forced, 0 off, -1 the size rule with the relaxed hint (16 permutations), -2 the strict one
// (64). Outputs as qb_key_order: *L = *m = 0 when there is no code; arrays filled when non-null.
int qref_key_order(int n_sites, int G, const int* perms, const std::uint64_t* flips, int mode, int* L, int* m,
                   std::uint64_t* n_cand, int* key_bit, std::uint16_t* lead, std::uint32_t* cand_off,
                   std::uint16_t* cand) {
    return guarded([&] {
        std::optional<bool> om;
        if (mode == 1) om = true;
        if (mode == 0) om = false;
        const ed::symmetry::SublatticeRuleScope scope(mode != -2);
        const auto c = ed::symmetry::SublatticeCode::of(perms, flips, G, n_sites, om);
        *L = *m = 0;
        *n_cand = 0;
        if (!c) return;
        const auto v = c->view();
        *L = v.L;
        *m = v.m;
        const std::size_t P = static_cast<std::size_t>(v.m) << v.L;
        *n_cand = v.cand_off[P];
        if (key_bit) std::copy(c->key_bit().begin(), c->key_bit().end(), key_bit);
        if (lead) std::copy(v.lead, v.lead + P, lead);
        if (cand_off) std::copy(v.cand_off, v.cand_off + P + 1, cand_off);
        if (cand) std::copy(v.cand, v.cand + v.cand_off[P], cand);
    });
}

// ---------------- matvecs ----------------
// out = O in on one sector by the row walk (sector_gather, include/ed/matvec/sector_rows.h:137-140).
int qref_gather(void* sec, void* prog, const double* in, double* out) {
    return guarded([&] {
        const auto* S = static_cast<RefSector*>(sec);
        const auto* P = static_cast<ed::ops::MaskedProgram*>(prog);
        const auto pol = S->rd.make_policy();
        ed::matvec::sector_gather(P->view(), pol, S->rd.dim(), reinterpret_cast<const Complex*>(in),
                                  reinterpret_cast<Complex*>(out));
    });
}

// out[i] = row rows[i] of O in on one sector, for n listed rows: the body of sector_gather
// (for_each_sector_entry, sector_rows.h:58-63, summed as cross_gather does at sector_rows.h:128-132),
// OpenMP over the listed rows. The sampled form of the host walk lane for sectors whose full apply
// is too long to time or check whole.
int qref_gather_rows(void* sec, void* prog, const double* in, const std::uint64_t* rows, std::uint64_t n,
                     double* out) {
    return guarded([&] {
        const auto* S = static_cast<RefSector*>(sec);
        const auto* P = static_cast<ed::ops::MaskedProgram*>(prog);
        const auto pol = S->rd.make_policy();
        const auto view = P->view();
        const Complex* x = reinterpret_cast<const Complex*>(in);
        Complex* y = reinterpret_cast<Complex*>(out);
#pragma omp parallel for schedule(static)
        for (long long i = 0; i < static_cast<long long>(n); ++i) {
            Complex acc(0.0, 0.0);
            ed::matvec::for_each_sector_entry(view, pol, rows[i],
                                              [&](std::uint64_t c, const Complex& v) { acc += v * x[c]; });
            y[i] = acc;
        }
    });
}

// out = O in from sector `col` to sector `row` (cross_gather, sector_rows.h:110-135).
int qref_cross_gather(void* row, void* col, void* prog, const double* in, double* out) {
    return guarded([&] {
        const auto* R = static_cast<RefSector*>(row);
        const auto* C = static_cast<RefSector*>(col);
        const auto* P = static_cast<ed::ops::MaskedProgram*>(prog);
        const auto rp = R->rd.make_policy();
        const auto cp = C->rd.make_policy();
        ed::matvec::cross_gather(P->view(), rp, cp, R == C, R->rd.dim(), reinterpret_cast<const Complex*>(in),
                                 reinterpret_cast<Complex*>(out));
    });
}

struct RefCsr {
    ed::matvec::ReducedSymmetryCsr<Complex> csr;
};

// The merged reduced CSR of O on one sector (build_sector_csr, sector_rows.h:223-404).
void* qref_csr_build(void* sec, void* prog) {
    try {
        const auto* S = static_cast<RefSector*>(sec);
        const auto* P = static_cast<ed::ops::MaskedProgram*>(prog);
        const auto pol = S->rd.make_policy();
        auto* c = new RefCsr;
        c->csr = ed::matvec::build_sector_csr(P->view(), pol, S->rd.dim());
        return c;
    } catch (const std::exception& e) {
        g_err = e.what();
        return nullptr;
    }
}
void qref_csr_free(void* c) { delete static_cast<RefCsr*>(c); }
std::uint64_t qref_csr_nnz(void* c) {
    const auto& m = static_cast<RefCsr*>(c)->csr;
    return m.row_ptr.empty() ? 0 : m.row_ptr.back();
}
// row_ptr (dim+1), col (nnz), val (2 nnz doubles; entries decoded from the dictionary).
void qref_csr_get(void* c, std::uint64_t* row_ptr, std::uint32_t* col, double* val) {
    const auto& m = static_cast<RefCsr*>(c)->csr;
    std::copy(m.row_ptr.begin(), m.row_ptr.end(), row_ptr);
    const std::uint64_t nnz = m.row_ptr.empty() ? 0 : m.row_ptr.back();
    for (std::uint64_t e = 0; e < nnz; ++e) {
        col[e] = m.col_idx[e];
        Complex v;
        if (!m.val.empty())
            v = m.val[e];
        else if (!m.id8.empty())
            v = m.dict[m.id8[e]];
        else
            v = m.dict[m.id16[e]];
        if (val) {
            val[2 * e] = v.real();
            val[2 * e + 1] = v.imag();
        }
    }
}
std::uint64_t qref_csr_bytes(void* c) { return static_cast<RefCsr*>(c)->csr.bytes(); }
int qref_csr_spmv(void* c, const double* in, double* out) {
    return guarded([&] {
        static_cast<RefCsr*>(c)->csr.spmv(reinterpret_cast<const Complex*>(in), reinterpret_cast<Complex*>(out));
    });
}

// out = Re(A) in on real vectors (RealCsrView::spmv, include/ed/matvec/reduced_csr.h:111-135): the host lane
// of a real symmetry sector of a real H (RepSectorMatVec::is_real, src/engine/internal.h:264-283, chosen by
// with_backend, include/ed/core/select_backend.h:186). Returns 1 when the CSR is not real (nothing applied).
int qref_csr_spmv_real(void* c, const double* in, double* out) {
    const auto& m = static_cast<RefCsr*>(c)->csr;
    const auto view = ed::matvec::RealCsrView::of(m, ed::numerics::kRealBlockRel);
    if (!view) return 1;
    view->spmv(in, out);
    return 0;
}

namespace {
// Rows [r0, r0 + n) of a one-dimensional-irrep sector (or the listed rows, when `list` is set) as a row policy of
// their own (row j is the sector's row r0 + j, or list[j]; columns stay the whole sector's). Lets
// build_cross_csr build the merged rows of a block of rows.
struct RowBlock {
    const ed::matvec::basis::RepSymmetryBasisPolicy* p;
    std::uint64_t r0, n;
    const std::uint64_t* list = nullptr;
    int irrep_dim = 1;
    std::uint64_t row(std::uint64_t j) const noexcept { return list ? list[j] : r0 + j; }
    std::uint64_t dim() const noexcept { return n; }
    std::uint64_t state_of(std::uint64_t j) const noexcept { return p->state_of(row(j)); }
    double inv_norm_of(std::uint64_t j) const noexcept { return p->inv_norm_of(row(j)); }
    std::uint64_t first_state_of(std::uint64_t j) const noexcept { return j; }
    int rank_of(std::uint64_t) const noexcept { return 1; }
    const Complex* C_of(std::uint64_t) const noexcept { return nullptr; }   // (the d > 1 branch, never taken)
};
}  // namespace

// The merged CSR of the listed rows of O on one sector (the rows in the order listed; columns over the whole
// sector), as qref_csr_build_rows does for a contiguous block.
void* qref_csr_build_rowlist(void* sec, void* prog, const std::uint64_t* rows, std::uint64_t n) {
    try {
        const auto* S = static_cast<RefSector*>(sec);
        const auto* P = static_cast<ed::ops::MaskedProgram*>(prog);
        if (S->rd.irrep_dim != 1) throw std::invalid_argument("qref_csr_build_rowlist: d > 1");
        for (std::uint64_t j = 0; j < n; ++j)
            if (rows[j] >= S->rd.dim()) throw std::invalid_argument("qref_csr_build_rowlist: row out of range");
        const auto pol = S->rd.make_policy();
        RowBlock rb{&pol, 0, n, rows};
        auto* c = new RefCsr;
        c->csr = ed::matvec::build_cross_csr(P->view(), rb, pol, false, n);
        return c;
    } catch (const std::exception& e) {
        g_err = e.what();
        return nullptr;
    }
}

// The merged CSR of rows [r0, r0 + n) of O on one sector (build_cross_csr, sector_rows.h:223-404, over the
// block's rows, columns the whole sector): the reference's host CSR lane on a contiguous sample of rows, for
// sectors whose whole CSR is too large to build for a bounded timing. The diagonal goes through the lookup
// (the cross form), which gives the same entries up to the rounding of inv_norm * projection.
void* qref_csr_build_rows(void* sec, void* prog, std::uint64_t r0, std::uint64_t n) {
    try {
        const auto* S = static_cast<RefSector*>(sec);
        const auto* P = static_cast<ed::ops::MaskedProgram*>(prog);
        if (S->rd.irrep_dim != 1 || r0 + n > S->rd.dim()) throw std::invalid_argument("qref_csr_build_rows: bad rows");
        const auto pol = S->rd.make_policy();
        const RowBlock rows{&pol, r0, n, nullptr};
        auto* c = new RefCsr;
        c->csr = ed::matvec::build_cross_csr(P->view(), rows, pol, false, n);
        return c;
    } catch (const std::exception& e) {
        g_err = e.what();
        return nullptr;
    }
}

// ---------------- seeds ----------------
// The FTLM sample vector of sample s (sample_engine + gaussian_vector, include/ed/thermal/sample_seed.h:37-89).
void qref_sample_vector(std::uint64_t base_seed, std::uint64_t s, std::uint64_t n, double* out) {
    std::mt19937 gen = ed::thermal::sample_engine(base_seed, s);
    const auto v = ed::thermal::gaussian_vector(static_cast<std::size_t>(n), gen);
    std::memcpy(out, v.data(), n * sizeof(Complex));
}
// The unnormalised Gaussian start of the block lanes (staged_seed, block_solve.cpp:268-277).
void qref_staged_seed(std::uint64_t seed, std::uint64_t n, double* out) {
    const auto v = staged_seed_host(static_cast<std::size_t>(n), seed);
    std::memcpy(out, v.data(), n * sizeof(Complex));
}

// ---------------- Krylov ----------------
// lanczos_kernel<CpuBackend> on O's sector walk (include/ed/krylov/lanczos.h:266-576).
// reorth: 0 None, 1 FullCGS2, 2 LocalDGKS3 (ring 1). alpha: max_iter, beta: max_iter + 1.
int qref_lanczos(void* sec, void* prog, const double* v0, int max_iter, int reorth, double breakdown_tol,
                 double* alpha, double* beta, int* iters) {
    return guarded([&] {
        auto* S = static_cast<RefSector*>(sec);
        const auto* P = static_cast<ed::ops::MaskedProgram*>(prog);
        Walk W{S, S, P, true, S->rd.make_policy(), S->rd.make_policy()};
        ed::krylov::LanczosKernelOptions o;
        o.max_iter = static_cast<std::size_t>(max_iter);
        o.breakdown_tol = breakdown_tol;
        o.reorth = reorth == 0   ? ed::krylov::ReorthPolicy::None
                   : reorth == 1 ? ed::krylov::ReorthPolicy::FullCGS2
                                 : ed::krylov::ReorthPolicy::LocalDGKS3;
        o.keep_basis = reorth == 1;
        ed::matvec::CpuBackend be;
        auto R = ed::krylov::lanczos_kernel(be, W, S->rd.dim(), reinterpret_cast<const Complex*>(v0), o);
        std::copy(R.alpha.begin(), R.alpha.end(), alpha);
        std::copy(R.beta.begin(), R.beta.end(), beta);
        *iters = static_cast<int>(R.iters_done);
    });
}

// The k = 1 block lane (lowest_scan_lane, block_solve.cpp:528-598): Lanczos from staged_seed(0x51ED0B70),
// no reorthogonalisation (FullCGS2 when the budget spans the block), Paige-gated after every step.
int qref_scan_lowest(void* sec, void* prog, int max_iter, double* e0, int* iters, int* converged) {
    return guarded([&] {
        auto* S = static_cast<RefSector*>(sec);
        const auto* P = static_cast<ed::ops::MaskedProgram*>(prog);
        const std::uint64_t nb = S->rd.dim();
        Walk W{S, S, P, true, S->rd.make_policy(), S->rd.make_policy()};
        ed::krylov::LanczosKernelOptions kopts;
        const std::uint64_t budget = max_iter > 0 ? static_cast<std::uint64_t>(max_iter) : 400u;
        kopts.max_iter = static_cast<std::size_t>(std::min<std::uint64_t>(nb, budget));
        kopts.reorth = static_cast<std::size_t>(nb) <= kopts.max_iter ? ed::krylov::ReorthPolicy::FullCGS2
                                                                      : ed::krylov::ReorthPolicy::None;
        kopts.keep_basis = kopts.reorth == ed::krylov::ReorthPolicy::FullCGS2;
        kopts.convergence_check = [](const std::vector<double>& a, const std::vector<double>& b) -> bool {
            const std::size_t m_all = a.size();
            const std::size_t m = leading_block(a, b, m_all);
            if (m == m_all && m_all < 3) return false;
            return lowest_level(a, b, m, nullptr);
        };
        kopts.convergence_check_interval = 1;
        const auto v0 = staged_seed_host(nb, 0x51ED0B70ULL);
        ed::matvec::CpuBackend be;
        auto k = ed::krylov::lanczos_kernel(be, W, nb, v0.data(), kopts);
        *iters = static_cast<int>(k.iters_done);
        std::vector<double> vals;
        *converged = 0;
        *e0 = std::nan("");
        if (k.alpha.empty()) return;
        const std::size_t m = leading_block(k.alpha, k.beta, k.alpha.size());
        *converged = lowest_level(k.alpha, k.beta, m, &vals) ? 1 : 0;
        if (!vals.empty()) *e0 = vals.front();
    });
}

// The k > 1 block lane (krylov_schur_lane, block_solve.cpp:433-510) without a memory cap: thick-restart
// Krylov-Schur from staged_seed(0x51ED0B70), lock tolerance kLockRel * s_H.
int qref_ks_lowest_lane(void* sec, void* prog, int k, int use_csr, double* evals, int* n_found, int* converged,
                        int* applies) {
    return guarded([&] {
        auto* S = static_cast<RefSector*>(sec);
        const auto* P = static_cast<ed::ops::MaskedProgram*>(prog);
        const std::size_t nb = S->rd.dim();
        const std::size_t kk = static_cast<std::size_t>(k);
        Walk W{S, S, P, true, S->rd.make_policy(), S->rd.make_policy()};
        // the host default lane applies through the merged reduced CSR (build_sector_csr); the walk otherwise
        std::optional<ed::matvec::ReducedSymmetryCsr<Complex>> csr;
        if (use_csr) csr = ed::matvec::build_sector_csr(P->view(), S->rd.make_policy(), S->rd.dim());
        std::uint64_t count = 0;
        auto H = [&](const Complex* in, Complex* out, std::size_t n) {
            ++count;
            if (csr)
                csr->spmv(in, out);
            else
                W(in, out, n);
        };
        const std::uint64_t budget = std::max<std::uint64_t>(200u * kk, 2000u);
        const std::size_t per_cycle = std::min<std::size_t>(ed::krylov::krylov_subspace_dim(kk, 2 * kk + 60, nb, 0),
                                                            static_cast<std::size_t>(std::max<std::uint64_t>(budget, kk + 1)));
        const std::size_t p_keep = kk + std::max<std::size_t>(kk / 2, 8);
        const std::size_t fresh = std::max<std::size_t>(std::min(per_cycle, 2 * p_keep + 20), p_keep + 1) - p_keep;
        const std::size_t restarts = static_cast<std::size_t>(std::max<std::uint64_t>(1u, budget / fresh));
        const double scale = ed::numerics::scale_or_one(program_norm_bound(*P));
        ed::krylov::KrylovSchurOptions o;
        o.num_eigs = kk;
        o.max_iter = per_cycle;
        o.max_restarts = restarts;
        o.tolerance = ed::numerics::kLockRel * scale;
        o.breakdown_tol = ed::numerics::kBreakdownRel * scale;
        o.max_subspace_vectors = per_cycle;
        o.compute_vectors = false;
        const auto v0 = staged_seed_host(nb, 0x51ED0B70ULL);
        ed::matvec::CpuBackend be;
        auto r = ed::krylov::krylov_schur_kernel(be, H, nb, v0.data(), o);
        std::vector<double> ev = r.eigenvalues;
        std::sort(ev.begin(), ev.end());
        const std::size_t n = std::min(ev.size(), kk);
        std::copy(ev.begin(), ev.begin() + static_cast<std::ptrdiff_t>(n), evals);
        *n_found = static_cast<int>(n);
        *converged = (r.converged || r.exhausted) ? 1 : 0;
        *applies = static_cast<int>(count);
    });
}

int qref_ks_lowest(void* sec, void* prog, int k, double* evals, int* n_found, int* converged, int* applies) {
    return qref_ks_lowest_lane(sec, prog, k, 0, evals, n_found, converged, applies);
}

// FTLM on one block (ftlm_kernel<CpuBackend>, include/ed/thermal/ftlm.h:277-480) with the options the
// thermal verb passes for a sampled block (src/engine/thermal.cpp:299-312): breakdown 64 eps s_H.
int qref_ftlm(void* sec, void* prog, int samples, int depth, std::uint64_t seed, const double* betas, int nb,
              double* lnZ, double* E, double* V, double* gs) {
    return guarded([&] {
        auto* S = static_cast<RefSector*>(sec);
        const auto* P = static_cast<ed::ops::MaskedProgram*>(prog);
        Walk W{S, S, P, true, S->rd.make_policy(), S->rd.make_policy()};
        ed::thermal::FtlmOptions o;
        o.num_samples = static_cast<std::size_t>(samples);
        o.krylov_dim = static_cast<std::size_t>(depth);
        o.breakdown_tol = ed::numerics::kBreakdownRel * ed::numerics::scale_or_one(program_norm_bound(*P));
        o.betas.assign(betas, betas + nb);
        o.random_seed = seed;
        ed::matvec::CpuBackend be;
        auto r = ed::thermal::ftlm_kernel(be, W, S->rd.dim(), o);
        std::copy(r.curves.lnZ.begin(), r.curves.lnZ.end(), lnZ);
        std::copy(r.curves.E.begin(), r.curves.E.end(), E);
        std::copy(r.curves.V.begin(), r.curves.V.end(), V);
        *gs = r.ground_state_estimate;
    });
}

// The sampled thermal blocks of one call on the host, scheduled as the reference's thermal driver schedules
// them (src/engine/thermal.cpp:397-541): each block applies H through its merged reduced CSR (build_sector_csr,
// the host default lane), every block draws its samples from the call's base seed; blocks below 2^16 states
// (kHostPoolMaxDim, include/ed/core/device.h:67) run afterwards concurrently, one thread each (dynamic
// schedule), the larger ones one at a time on the full thread team. Per-block curves [b * nb + t].
int qref_ftlm_blocks(void* const* secs, void* prog, int n_blocks, int samples, int depth, std::uint64_t seed,
                     const double* betas, int nb, double* lnZ, double* E, double* V, double* gs) {
    return guarded([&] {
        const auto* P = static_cast<ed::ops::MaskedProgram*>(prog);
        const double tol = ed::numerics::kBreakdownRel * ed::numerics::scale_or_one(program_norm_bound(*P));
        auto run = [&](int b) {
            auto* S = static_cast<RefSector*>(secs[b]);
            const auto pol = S->rd.make_policy();
            const auto csr = ed::matvec::build_sector_csr(P->view(), pol, S->rd.dim());
            auto apply = [&csr](const Complex* in, Complex* out, std::size_t) { csr.spmv(in, out); };
            ed::thermal::FtlmOptions o;
            o.num_samples = static_cast<std::size_t>(samples);
            o.krylov_dim = static_cast<std::size_t>(depth);
            o.breakdown_tol = tol;
            o.betas.assign(betas, betas + nb);
            o.random_seed = seed;
            ed::matvec::CpuBackend be;
            auto r = ed::thermal::ftlm_kernel(be, apply, S->rd.dim(), o);
            std::copy(r.curves.lnZ.begin(), r.curves.lnZ.end(), lnZ + static_cast<std::size_t>(b) * nb);
            std::copy(r.curves.E.begin(), r.curves.E.end(), E + static_cast<std::size_t>(b) * nb);
            std::copy(r.curves.V.begin(), r.curves.V.end(), V + static_cast<std::size_t>(b) * nb);
            gs[b] = r.ground_state_estimate;
        };
        constexpr std::uint64_t kPoolMaxDim = std::uint64_t{1} << 16;
        std::vector<int> small;
        for (int b = 0; b < n_blocks; ++b) {
            if (static_cast<RefSector*>(secs[b])->rd.dim() >= kPoolMaxDim)
                run(b);
            else
                small.push_back(b);
        }
        std::string failure;
        {
            const ed::parallel::ThreadBudgetScope serial_inside(omp_get_max_threads(), 1);
#pragma omp parallel for schedule(dynamic, 1)
            for (long long q = 0; q < static_cast<long long>(small.size()); ++q) {
                try {
                    const ed::parallel::ThreadBudgetScope one(1, 1);
                    run(small[static_cast<std::size_t>(q)]);
                } catch (const std::exception& e) {
#pragma omp critical(qref_thermal_failure)
                    if (failure.empty()) failure = e.what();
                }
            }
        }
        if (!failure.empty()) throw std::runtime_error(failure);
    });
}

// The T = 0 continued fraction from a host vector phi (cf_spectral_from_vector, include/ed/dynamics/cf.h:104-160).
// shift: NaN lets the kernel use the tridiagonal's lowest value.
int qref_cf(void* sec, void* prog, const double* phi, int depth, const double* omega, int nw, double eta,
            double shift, double tolerance, double* S_out, double* shift_out, double* conv_change) {
    return guarded([&] {
        auto* S = static_cast<RefSector*>(sec);
        const auto* P = static_cast<ed::ops::MaskedProgram*>(prog);
        Walk W{S, S, P, true, S->rd.make_policy(), S->rd.make_policy()};
        ed::observables::CfSpectralOptions o;
        o.krylov_dim = static_cast<std::size_t>(depth);
        o.broadening = eta;
        if (!std::isnan(shift)) o.energy_shift = shift;
        o.tolerance = tolerance;
        std::vector<double> w(omega, omega + nw);
        ed::matvec::CpuBackend be;
        auto r = ed::observables::cf_spectral_from_vector(be, W, S->rd.dim(), reinterpret_cast<const Complex*>(phi),
                                                          w, o);
        std::copy(r.spectral_function.begin(), r.spectral_function.end(), S_out);
        *shift_out = r.energy_shift;
        *conv_change = r.convergence_change;
    });
}

// Tridiagonal eigenvalues + eigenvectors (tridiag_eig, include/ed/krylov/tridiag.h:42-65).
int qref_tridiag_eig(const double* alpha, const double* beta, int m, double* values, double* vectors) {
    return guarded([&] {
        std::vector<double> a(alpha, alpha + m), b(beta, beta + m + 1);
        const auto t = ed::krylov::tridiag_eig(a, b, static_cast<std::size_t>(m), vectors != nullptr);
        std::copy(t.values.begin(), t.values.end(), values);
        if (vectors) std::copy(t.vectors.begin(), t.vectors.end(), vectors);
    });
}

}  // extern "C"
