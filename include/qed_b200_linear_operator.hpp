// =============================================================================
// include/qed_b200_linear_operator.hpp -- the reference-side binding of the B200 sector matvec.
//
// A header-only ed::LinearOperator (the reference's operator interface,
// include/ed/matvec/linear_operator.h:32-77) over the C-ABI of qed_b200.h. A maintainer of the
// reference engine includes this header where RepSectorMatVec binds its device lane
// (src/engine/internal.h:244-263) and returns B200SectorMatVec::bind_cuda() / bind_cuda_multi()
// instead of make_sector_matvec_gpu_rep(...): the lanczos_kernel<CudaBackend>, ftlm_kernel and
// cf_spectral_from_vector callers run unchanged on it.
//
// It needs the reference's headers (ed/matvec/linear_operator.h, ed/core/errors.h, ed/basis/rep_sector.h,
// ed/ops/program.h) and links libqed_b200.so. Status codes map onto the reference's exceptions:
// QB_EINVAL -> std::invalid_argument, QB_ENOMEM -> ed::ResourceLimit, QB_ENODEV -> ed::DeviceUnavailable,
// QB_EUNSUPPORTED -> ed::DeviceUnsupported, anything else -> std::runtime_error.
// =============================================================================
#pragma once

#include <ed/basis/rep_sector.h>
#include <ed/core/errors.h>
#include <ed/matvec/linear_operator.h>
#include <ed/ops/program.h>

#include <complex>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "qed_b200.h"

namespace qb_ed {

inline void check(int rc) {
    if (rc == QB_OK) return;
    const std::string msg = std::string("qed_b200: ") + qb_last_error();
    switch (rc) {
    case QB_EINVAL: throw std::invalid_argument(msg);
    case QB_ENOMEM: throw ed::ResourceLimit(msg);
    case QB_ENODEV: throw ed::DeviceUnavailable(msg);
    case QB_EUNSUPPORTED: throw ed::DeviceUnsupported(msg);
    default: throw std::runtime_error(msg);
    }
}

// A device sector from a RepSectorData (its representatives and 1/norms uploaded as they are).
inline std::shared_ptr<qb_sector> upload_sector(const ed::symmetry::RepSectorData& rd) {
    if (rd.irrep_dim != 1) throw ed::DeviceUnsupported("qed_b200: irreps of dimension > 1 are not on the device lane");
    std::vector<double> chars(2 * rd.characters.size());
    for (std::size_t g = 0; g < rd.characters.size(); ++g) {
        chars[2 * g] = rd.characters[g].real();
        chars[2 * g + 1] = rd.characters[g].imag();
    }
    qb_sector_desc d{};
    d.n_sites = rd.n_sites;
    d.n_up = rd.n_up;
    d.group_size = rd.group_size;
    d.perms = rd.perms_flat.data();
    d.flips = rd.flip_masks.empty() ? nullptr : rd.flip_masks.data();
    d.chars = chars.data();
    // the representatives were found with rd.slc's key order; the device lookup is by state, so the
    // order only matters for a sector the device enumerates itself
    d.sublattice_mode = rd.slc ? 1 : 0;
    d.lookup = QB_LOOKUP_AUTO;
    qb_sector* s = nullptr;
    check(qb_sector_create_from_reps(&d, rd.reps.data(), rd.inv_norms.data(), rd.reps.size(), &s));
    return std::shared_ptr<qb_sector>(s, [](qb_sector* p) { qb_sector_destroy(p); });
}

// A device program from a MaskedProgram (include/ed/ops/program.h:66-94).
inline std::shared_ptr<qb_program> upload_program(const ed::ops::MaskedProgram& P) {
    std::vector<double> coeff(2 * P.term_coeff.size());
    for (std::size_t k = 0; k < P.term_coeff.size(); ++k) {
        coeff[2 * k] = P.term_coeff[k].real();
        coeff[2 * k + 1] = P.term_coeff[k].imag();
    }
    qb_program_desc d{};
    d.n_groups = static_cast<uint32_t>(P.group_flip.size());
    d.group_flip = P.group_flip.data();
    d.group_setbits = P.group_setbits.data();
    d.group_vbegin = P.group_vbegin.data();
    d.n_vsub = static_cast<uint32_t>(P.vsub_val.size());
    d.vsub_val = P.vsub_val.data();
    d.vsub_tbegin = P.vsub_tbegin.data();
    d.n_terms = static_cast<uint32_t>(P.term_sign.size());
    d.term_sign = P.term_sign.data();
    d.term_coeff = coeff.data();
    qb_program* p = nullptr;
    check(qb_program_create(&d, &p));
    return std::shared_ptr<qb_program>(p, [](qb_program* q) { qb_program_destroy(q); });
}

// The drop-in: one sector (or a pair, rows in `row`, columns in `col`) and its row program.
class B200SectorMatVec final : public ed::LinearOperator {
public:
    using Complex = std::complex<double>;
    // norm_bound(): the sum of |coefficient| over the program's terms, the bound the reference's sector
    // operators report and its Krylov drivers scale their breakdown, cluster and degeneracy tolerances by.
    B200SectorMatVec(const ed::symmetry::RepSectorData& rd, const ed::ops::MaskedProgram& rows)
        : row_(upload_sector(rd)), col_(row_), prog_(upload_program(rows)), dim_(rd.reps.size()),
          norm_bound_(coeff_sum(rows)) {}
    B200SectorMatVec(const ed::symmetry::RepSectorData& row, const ed::symmetry::RepSectorData& col,
                     const ed::ops::MaskedProgram& rows)
        : row_(upload_sector(row)), col_(upload_sector(col)), prog_(upload_program(rows)), dim_(row.reps.size()),
          norm_bound_(coeff_sum(rows)) {}

    void apply(const Complex* in, Complex* out, std::size_t n) const override {
        if (n != dim_) throw std::invalid_argument("B200SectorMatVec: length != sector dim");
        check(qb_matvec_host(row_.get(), col_.get(), prog_.get(), reinterpret_cast<const double*>(in),
                             reinterpret_cast<double*>(out)));
    }
    [[nodiscard]] std::size_t dim() const override { return dim_; }
    [[nodiscard]] double norm_bound() const override { return norm_bound_; }
    [[nodiscard]] std::string description() const override { return "B200SectorMatVec"; }
    [[nodiscard]] bool has_device_kernel() const override { return true; }

    // Device pointers of complex128, on the calling thread's default stream (it synchronises with the
    // legacy default stream the reference's device lane orders its work on).
    [[nodiscard]] MatvecFn bind_cuda() const override {
        auto row = row_, col = col_;
        auto prog = prog_;
        const std::size_t dim = dim_;
        return [row, col, prog, dim](const Complex* in, Complex* out, std::size_t n) {
            if (n != dim) throw std::invalid_argument("B200SectorMatVec: length != sector dim");
            const void* ins[1] = {in};
            void* outs[1] = {out};
            check(qb_matvec(row.get(), col.get(), prog.get(), ins, outs, 1, QB_C128, nullptr));
        };
    }
    // Every output equals the single apply bit for bit (the multi-apply contract, rep_matvec.h:51-55).
    [[nodiscard]] MultiMatvecFn bind_cuda_multi() const override {
        auto row = row_, col = col_;
        auto prog = prog_;
        const std::size_t dim = dim_;
        return [row, col, prog, dim](const Complex* const* ins, Complex* const* outs, std::size_t n, std::size_t k) {
            if (n != dim) throw std::invalid_argument("B200SectorMatVec: length != sector dim");
            check(qb_matvec(row.get(), col.get(), prog.get(), reinterpret_cast<const void* const*>(ins),
                            reinterpret_cast<void* const*>(outs), static_cast<int>(k), QB_C128, nullptr));
        };
    }

private:
    static double coeff_sum(const ed::ops::MaskedProgram& P) {
        double s = 0.0;
        for (const auto& c : P.term_coeff) s += std::abs(c);
        return s;
    }
    std::shared_ptr<qb_sector> row_, col_;
    std::shared_ptr<qb_program> prog_;
    std::size_t dim_ = 0;
    double norm_bound_ = 0.0;
};

}  // namespace qb_ed
