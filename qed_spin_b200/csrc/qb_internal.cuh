// =============================================================================
// qb_internal.cuh -- device-side types shared by the sector, matvec and Krylov translation units.
//
// Layout in HBM of one sector (qb_sector):
//   reps       u64[dim]    the representatives, ascending (the basis index IS the array index)
//   inv_norms  f64[dim]    1/norm per representative
//   lut        u64[G][bpw][256]   the byte-decomposition image table of every group element (used when
//                                 the group has no arithmetic action: chains and tori rotate bits instead)
//   flips      u64[G], chars f64x2[G], edesc / emask u64[G]  per-element action parameters
//   to_key     u64[bpw][256]      sublattice key order (when engaged)
//   pack       u64[m][2^L]        least leading block | candidate count | candidate or list offset
//   cand       u16[...]           the candidate lists of the entries with more than one
//   lookup     hash slots u64x2[2^b]: (state, index | 1/norm class << 32), open addressing, load <= 1/2;
//              or rank_table i32[C(N, n_up)] indexed by the combinadic rank (rank_lut
//              u64[bpw][N+1][256]); or bucket_off u32[n_buckets + 1] over the ascending states.
// The small tables (program, to_key) are staged in shared memory by each kernel.
// =============================================================================
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <functional>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/qed_b200.h"

namespace qb {

using u64 = unsigned long long;
using u32 = std::uint32_t;
using u16 = std::uint16_t;

// ---------------------------------------------------------------------------------------------
// Errors: every C entry point catches qb::Error and returns its code.
// ---------------------------------------------------------------------------------------------
struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

void set_last_error(const std::string& m);

// The device bytes the calling thread's solves may plan their optional buffers with (a kept Krylov basis):
// the free device memory, or less when the thread has an allowance (a request server's worker sets one to
// the footprint it admitted the request with; 0: none).
std::size_t available_bytes();
void set_thread_allowance(std::size_t bytes);

// The launch shape of a kernel family for a size-class key (tune.cu): a forced or known choice, or -- when
// measuring and st is not capturing -- the fastest of n candidates, each run by run(c) on st; else fallback.
// The candidates must give the same result bit for bit.
int tune_choose(const char* family, const std::string& key, int n, int fallback, cudaStream_t st,
                const std::function<void(int)>& run);
// Changes whenever the tuner's modes, forces or known choices change (memos of choices compare it).
unsigned tune_generation();

inline void cuda_check(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return;
    const int code = (e == cudaErrorMemoryAllocation) ? QB_ENOMEM : (e == cudaErrorNoDevice ? QB_ENODEV : QB_ECUDA);
    (void)cudaGetLastError();
    throw Error(code, std::string(what) + ": " + cudaGetErrorString(e));
}

template <class F> int guarded(F&& f) {
    try {
        f();
        return QB_OK;
    } catch (const Error& e) {
        set_last_error(e.what());
        return e.code;
    } catch (const std::bad_alloc&) {
        set_last_error("host allocation failed");
        return QB_ENOMEM;
    } catch (const std::exception& e) {
        set_last_error(e.what());
        return QB_EINVAL;
    }
}

// Device memory from the library's cache of released blocks (alloc.cu): dev_free records an event on the
// calling thread's stream and the block is reused once it completes, so releasing never synchronises the device.
void* dev_alloc(std::size_t bytes);
void dev_free(void* p, std::size_t bytes);
// A host-to-device copy that has completed on return; large pageable sources go through pinned slots (hostio.cu).
void upload_host(void* dst, const void* src, std::size_t bytes, cudaStream_t st);
std::size_t idle_cached_bytes();

// A device allocation owned by a host object (released on the thread whose stream last used it, or after a
// synchronisation).
template <class T> struct DevBuf {
    T* p = nullptr;
    std::size_t n = 0;
    DevBuf() = default;
    explicit DevBuf(std::size_t count) { alloc(count); }
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    DevBuf(DevBuf&& o) noexcept : p(o.p), n(o.n) { o.p = nullptr, o.n = 0; }
    DevBuf& operator=(DevBuf&& o) noexcept {
        if (this != &o) {
            release();
            p = o.p, n = o.n;
            o.p = nullptr, o.n = 0;
        }
        return *this;
    }
    ~DevBuf() { release(); }
    void alloc(std::size_t count) {
        release();
        if (count == 0) return;
        p = static_cast<T*>(dev_alloc(count * sizeof(T)));
        n = count;
    }
    void release() {
        if (p) dev_free(p, n * sizeof(T));
        p = nullptr;
        n = 0;
    }
    void upload(const T* h, std::size_t count) {
        alloc(count);
        if (count) upload_host(p, h, count * sizeof(T), nullptr);
    }
    void upload(const std::vector<T>& v) { upload(v.data(), v.size()); }
    std::size_t bytes() const { return n * sizeof(T); }
};

// ---------------------------------------------------------------------------------------------
// Device views (trivially copyable; passed by value to kernels).
// ---------------------------------------------------------------------------------------------
struct DSlc {
    int on = 0, L = 0, m = 0;
    const u64* to_key = nullptr;    // bpw x 256
    // per (block j, pattern): least leading block (bits 0-15) | candidate count (16-31) | payload (32-63):
    // the candidate itself when there is one, else the offset of the block's list in `cand`
    const u64* pack = nullptr;      // m << L
    const u16* cand = nullptr;
    // the sites of block j as a state mask; within a block, a higher site holds a higher key bit, so two states
    // compare in the key order by the highest differing site of the first block in which they differ
    u64 bmask[8] = {};
    // block j is sites [jL, (j+1)L) in order: its pattern is state bits jL .. jL+L-1, no key needed
    int contig = 0;
};

// Group element kinds with an arithmetic action (0: the byte-LUT action).
enum : int { kElemLut = 0, kElemRot = 1, kElemRefl = 2, kElemTorus = 3 };

struct DSector {
    int N = 0, n_up = 0, G = 0, bpw = 0;
    std::uint64_t dim = 0;
    const u64* reps = nullptr;
    const double* inv_norms = nullptr;
    const u64* lut = nullptr;       // G x bpw x 256
    const u64* flips = nullptr;     // G
    const double2* chars = nullptr; // G
    // every character exactly +1 or -1 (imaginary part zero): a character sum is then an exact integer whatever
    // the order of its terms, so tied candidate lists need no ordered merge
    int unit_chars = 0;
    // arithmetic group action (gkind != 0): per element kind | rotation << 8 | row shift << 16, and the
    // torus row mask; gkind 1 chains (rotations, reflections), 2 torus translations with row length Lx
    int gkind = 0, Lx = 0;
    const u64* edesc = nullptr;     // G
    const u64* emask = nullptr;     // G
    DSlc slc;
    // lookup: kind 1 rank table, 2 state buckets, 3 hash slots
    int lookup = 0;
    const ulonglong2* slots = nullptr;   // [state, index | class << 32], 2^hash_bits slots; empty: state ~0
    const u64* slots8 = nullptr;         // state (low 32 bits) | (index | class << idx_bits) << 32; empty: ~0
    int idx_bits = 0;
    int hash_bits = 0;
    const double* inv_class = nullptr;   // the distinct 1/norm values, indexed by class (hash lookup)
    int n_class = 0;
    const std::int32_t* rank_table = nullptr;
    const u64* rank_lut = nullptr;  // bpw x (N + 1) x 256: byte b's share of the combinadic rank
    const u32* bucket_off = nullptr;
    u64 bucket_base = 0, bucket_count = 0;
    int bucket_shift = 0;
};

struct DProgram {
    u32 n_groups = 0, n_vsub = 0, n_terms = 0;
    const u64* group_flip = nullptr;
    const int* group_setbits = nullptr;
    const u32* group_vbegin = nullptr;
    const u64* vsub_val = nullptr;
    const u32* vsub_tbegin = nullptr;
    const u64* term_sign = nullptr;
    const double2* term_coeff = nullptr;
    std::size_t smem_bytes = 0;   // bytes to stage the whole program in shared memory
    int vsub4 = 0;                // every group has at most 4 value subgroups (a 2-bit offset names one)
};

}  // namespace qb

// The host objects behind the opaque handles.
struct qb_sector {
    int N = 0, n_up = 0, G = 0, bpw = 0;
    std::uint64_t dim = 0;
    qb::DevBuf<qb::u64> reps;
    qb::DevBuf<double> inv_norms;
    qb::DevBuf<qb::u64> lut, flips;
    qb::DevBuf<double2> chars;
    qb::DevBuf<qb::u64> to_key, lead_pack, edesc, emask;
    qb::DevBuf<qb::u16> cand;
    int gkind = 0, Lx = 0;
    qb::DevBuf<std::int32_t> rank_table;
    qb::DevBuf<qb::u64> rank_lut;
    qb::DevBuf<qb::u32> bucket_off;
    qb::DevBuf<ulonglong2> slots;
    qb::DevBuf<qb::u64> slots8;
    int idx_bits = 0;
    qb::DevBuf<double> inv_class;
    int hash_bits = 0, n_class = 0;
    int slc_on = 0, slc_L = 0, slc_m = 0, slc_contig = 0;
    qb::u64 slc_bmask[8] = {};
    int lookup = 0;
    qb::u64 bucket_base = 0, bucket_count = 0;
    int bucket_shift = 0;
    std::vector<double> chars_host;   // 2G
    // the descriptor the sector was made from (saved with it, and the key of the registry)
    std::vector<std::int32_t> desc_perms;
    std::vector<std::uint64_t> desc_flips;
    int desc_slc_mode = 0, desc_lookup = 0;
    bool registered = false;          // owned by the registry (qb_sector_acquire / qb_sector_release)
    qb::DSector view() const;
    std::uint64_t device_bytes() const;
};

struct qb_csr;

struct qb_program {
    qb::DevBuf<unsigned char> blob;   // every array back to back (8-byte aligned), staged as one copy
    qb::DProgram view;
    double norm_bound = 0.0;          // sum of |coeff|
    const qb_csr* csr = nullptr;      // the attached reduced CSR (qb_program_attach_csr), or none
};

// The merged reduced CSR of an operator between two sectors (csr.cu).
struct qb_csr {
    const qb_sector* row = nullptr;
    const qb_sector* col = nullptr;
    std::uint64_t rows = 0, nnz = 0;
    int id_bytes = 0;                 // 1: u8 dictionary ids, 2: u16 ids, 0: full values
    int n_dict = 0;
    qb::DevBuf<unsigned long long> row_ptr;
    qb::DevBuf<std::uint32_t> col_idx;
    qb::DevBuf<unsigned char> ids;    // nnz x id_bytes
    qb::DevBuf<double2> vals;         // the dictionary (n_dict) or every value (nnz)
    std::uint64_t bytes() const {
        return row_ptr.bytes() + col_idx.bytes() + ids.bytes() + vals.bytes();
    }
};

namespace qb {
// y = A x on k vectors (k == 1: one vector; else interleaved by row), x as dtype_in, y as dtype_out.
void csr_spmv(const qb_csr* A, const void* in, void* out, int k, int dtype_in, int dtype_out, cudaStream_t st);
}  // namespace qb

namespace qb {

// ---------------------------------------------------------------------------------------------
// Exact complex arithmetic: the operations std::complex<double> performs on the host, without
// fused multiply-adds, so device results equal the reference's host arithmetic bit for bit.
// ---------------------------------------------------------------------------------------------
struct cplx {
    double re, im;
};
__device__ __forceinline__ cplx cmul(cplx a, cplx b) {
    return {__dsub_rn(__dmul_rn(a.re, b.re), __dmul_rn(a.im, b.im)),
            __dadd_rn(__dmul_rn(a.re, b.im), __dmul_rn(a.im, b.re))};
}
__device__ __forceinline__ cplx cadd(cplx a, cplx b) { return {__dadd_rn(a.re, b.re), __dadd_rn(a.im, b.im)}; }
__device__ __forceinline__ cplx cconj(cplx a) { return {a.re, -a.im}; }
__device__ __forceinline__ cplx rscale(double w, cplx a) { return {__dmul_rn(w, a.re), __dmul_rn(w, a.im)}; }

}  // namespace qb
