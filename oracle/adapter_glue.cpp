// =============================================================================
// oracle/adapter_glue.cpp -- TEST INFRASTRUCTURE, not product code.
//
// Drives the reference engine's own Lanczos kernel (lanczos_kernel<CpuBackend>, include/ed/krylov/lanczos.h:
// 266-576) through the reference-side binding of this library, include/qed_b200_linear_operator.hpp: the
// ed::LinearOperator a maintainer of the reference binds in place of its device lane. Compiled by
// oracle/Makefile from the reference's headers and src/ops/{algebra,program}.cpp where they lie, linked against
// the CUDA library (qed_spin_b200/libqed_b200.so), into oracle/_ref/libqed_adapter.so. The tests load it to show
// that the binding runs the reference's own kernels unchanged and gives the reference's numbers.
// =============================================================================
#include "qed_b200_linear_operator.hpp"

#include <ed/basis/compiled_group.h>
#include <ed/krylov/lanczos.h>
#include <ed/matvec/cpu_backend.h>
#include <ed/ops/algebra.h>
#include <ed/ops/program.h>

#include <cuda_runtime.h>

#include <complex>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

using Complex = std::complex<double>;

namespace {

thread_local std::string g_err;

// A RepSectorData from representatives and 1/norms computed elsewhere, with the group's key order
// (CompiledGroup::from_elements under the forced sublattice rule when slc != 0).
ed::symmetry::RepSectorData sector_data(int n_sites, int n_up, int G, const int* perms, const std::uint64_t* flips,
                                        const double* chars, const std::uint64_t* reps, const double* inv_norms,
                                        std::uint64_t dim, int slc) {
    ed::symmetry::RepSectorData rd;
    rd.n_sites = n_sites;
    rd.n_up = n_up;
    rd.group_size = G;
    rd.characters.resize(static_cast<std::size_t>(G));
    for (int g = 0; g < G; ++g) rd.characters[g] = Complex(chars[2 * g], chars[2 * g + 1]);
    rd.perms_flat.assign(perms, perms + static_cast<std::size_t>(G) * n_sites);
    if (flips) rd.flip_masks.assign(flips, flips + G);
    rd.reps.assign(reps, reps + dim);
    rd.inv_norms.assign(inv_norms, inv_norms + dim);
    if (slc) rd.slc = ed::symmetry::SublatticeCode::of(perms, flips, G, n_sites, true);
    return rd;
}

// The row program of sum_p coeff_p prod ops_p(sites_p): compile_operator(O^dagger) (operator.h:132-137).
ed::ops::MaskedProgram program(int n_sites, int n_prod, const char* ops, const int* nfac, const int* sites,
                               const double* coeffs) {
    ed::ops::MaskedOperator O(n_sites);
    int off = 0;
    for (int p = 0; p < n_prod; ++p) {
        std::vector<int> s(sites + off, sites + off + nfac[p]);
        O.add(ed::ops::MaskedOperator::product(n_sites, std::string(ops + off, static_cast<std::size_t>(nfac[p])), s,
                                               Complex(coeffs[2 * p], coeffs[2 * p + 1])));
        off += nfac[p];
    }
    return ed::ops::compile_operator(O.dagger());
}

}  // namespace

extern "C" {

const char* qad_last_error() { return g_err.c_str(); }

// Through qb_ed::B200SectorMatVec on one sector: y_apply = H x by apply() (host buffers), y_bind = H x by
// bind_cuda() (device buffers), its norm_bound(), and the reference's lanczos_kernel<CpuBackend> over apply() from
// v0 for max_iter steps without reorthogonalisation (alpha: max_iter, beta: max_iter + 1). With a second sector
// (col_reps != NULL), cross_norm_bound: the norm_bound() of the two-sector operator on the same program.
int qad_run(int n_sites, int n_up, int G, const int* perms, const std::uint64_t* flips, const double* chars,
            const std::uint64_t* reps, const double* inv_norms, std::uint64_t dim, int slc, int n_prod, const char* ops,
            const int* nfac, const int* sites, const double* coeffs, const double* x, double* y_apply, double* y_bind,
            const double* v0, int max_iter, double* alpha, double* beta, int* iters, double* norm_bound,
            double* cross_norm_bound) {
    try {
        const auto rd = sector_data(n_sites, n_up, G, perms, flips, chars, reps, inv_norms, dim, slc);
        const auto P = program(n_sites, n_prod, ops, nfac, sites, coeffs);
        const qb_ed::B200SectorMatVec op(rd, P);
        *norm_bound = op.norm_bound();
        if (cross_norm_bound) *cross_norm_bound = qb_ed::B200SectorMatVec(rd, rd, P).norm_bound();
        op.apply(reinterpret_cast<const Complex*>(x), reinterpret_cast<Complex*>(y_apply), dim);
        {
            Complex *dx = nullptr, *dy = nullptr;
            if (cudaMalloc(&dx, dim * sizeof(Complex)) != cudaSuccess || cudaMalloc(&dy, dim * sizeof(Complex)) != cudaSuccess)
                throw std::runtime_error("cudaMalloc");
            cudaMemcpy(dx, x, dim * sizeof(Complex), cudaMemcpyHostToDevice);
            const auto f = op.bind_cuda();
            f(dx, dy, dim);
            bool threw = false;   // a wrong length is refused, on both device applies
            try {
                f(dx, dy, dim + 1);
            } catch (const std::invalid_argument&) {
                threw = true;
            }
            try {
                const Complex* ins[1] = {dx};
                Complex* outs[1] = {dy};
                op.bind_cuda_multi()(ins, outs, dim + 1, 1);
                threw = false;
            } catch (const std::invalid_argument&) {
            }
            cudaMemcpy(y_bind, dy, dim * sizeof(Complex), cudaMemcpyDeviceToHost);
            cudaFree(dx);
            cudaFree(dy);
            if (!threw) throw std::runtime_error("a wrong length was not refused");
        }
        ed::krylov::LanczosKernelOptions o;
        o.max_iter = static_cast<std::size_t>(max_iter);
        o.reorth = ed::krylov::ReorthPolicy::None;
        o.keep_basis = false;
        ed::matvec::CpuBackend be;
        auto R = ed::krylov::lanczos_kernel(
            be, [&op](const Complex* in, Complex* out, std::size_t n) { op.apply(in, out, n); }, dim,
            reinterpret_cast<const Complex*>(v0), o);
        std::copy(R.alpha.begin(), R.alpha.end(), alpha);
        std::copy(R.beta.begin(), R.beta.end(), beta);
        *iters = static_cast<int>(R.iters_done);
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

}  // extern "C"
