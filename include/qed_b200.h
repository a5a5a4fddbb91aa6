/* =============================================================================
 * include/qed_b200.h -- the C-ABI of the B200 symmetry-sector matvec and its Krylov recurrences.
 *
 * The drop-in boundary for the reference engine's device lane: plain C types, opaque handles,
 * integer status codes, an explicit CUDA stream. NULL means the calling thread's default stream: the
 * library is built with per-thread default streams, and that stream synchronises with the legacy
 * default stream the reference's device lane orders its work on, so the lane's ordering holds; solves
 * driven from different host threads overlap on the device. Nothing here throws across the ABI.
 *
 * Conventions.
 *   - A basis state is a uint64 bit string, a SET bit an UP spin (include/ed/ops/term.h:27-34 in the
 *     reference). A group element maps s to permute_bits(s, perm) ^ flip, new bit i = old bit perm[i]
 *     (include/ed/basis/compiled_group.h:8-14).
 *   - Complex vectors are interleaved (re, im): double pairs (QB_C128, the reference's
 *     std::complex<double>) or float pairs (QB_C64, the FP32-storage form).
 *   - Multi-vector ("block") vectors are interleaved by row: element (row r, vector v) at r*k + v.
 *
 * Every function returns QB_OK or an error code; qb_last_error() describes the last failure of
 * the calling thread.
 * ============================================================================= */
#ifndef QED_B200_H
#define QED_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    QB_OK = 0,
    QB_EINVAL = 1,       /* malformed arguments (maps onto std::invalid_argument) */
    QB_ENOMEM = 2,       /* device allocation failed (maps onto ed::ResourceLimit) */
    QB_ECUDA = 3,        /* a CUDA runtime error (maps onto std::runtime_error) */
    QB_EUNSUPPORTED = 4, /* a form this build does not implement (maps onto ed::DeviceUnsupported) */
    QB_ETIMEOUT = 5,     /* a bounded device wait ran out */
    QB_ENODEV = 6        /* no CUDA device (maps onto ed::DeviceUnavailable) */
};

enum { QB_C128 = 0, QB_C64 = 1 };

enum { QB_REORTH_NONE = 0, QB_REORTH_FULL = 1, QB_REORTH_LOCAL = 2 };

/* The state -> index structure: AUTO picks HASH; RANK a table over the combinadic ranks; BUCKETS offsets
 * into the ascending representatives; HASH an open-addressing table whose slots hold the state, its index
 * and its 1/norm class (one probe answers index and norm): 8-byte slots at load <= 2/3 when the state fits 32
 * bits and index + class fit 31 (qb_sector_info reports kind 4), else 16-byte slots at load <= 1/2 (kind 3);
 * HASH_WIDE forces the 16-byte slots. */
enum { QB_LOOKUP_AUTO = 0, QB_LOOKUP_RANK = 1, QB_LOOKUP_BUCKETS = 2, QB_LOOKUP_HASH = 3, QB_LOOKUP_HASH_WIDE = 4 };

typedef struct qb_sector qb_sector;
typedef struct qb_program qb_program;

/* A sector: the fixed-S^z states of n_sites spins with n_up up spins, reduced by a group of
 * group_size elements in the one-dimensional irrep with characters chars (interleaved complex).
 * sublattice_mode picks the representative order (include/ed/basis/sublattice_code.h:23-34):
 * 0 the plain order, 1 the sublattice key order whenever a block system exists, -1 the size rule
 * of device verbs (N >= 24 and >= 16 distinct permutations), -2 the strict rule (>= 64).
 * All pointers are host memory. */
typedef struct {
    int n_sites;
    int n_up;
    int group_size;
    const int32_t* perms;  /* group_size x n_sites */
    const uint64_t* flips; /* group_size XOR masks, or NULL */
    const double* chars;   /* 2 x group_size */
    int sublattice_mode;
    int lookup;             /* QB_LOOKUP_* : state -> index structure */
} qb_sector_desc;

/* A row program in the reference's MaskedProgram layout (include/ed/ops/program.h:66-94):
 * groups by ascending flip mask, value subgroups ascending, terms in key order. Host memory. */
typedef struct {
    uint32_t n_groups;
    const uint64_t* group_flip;    /* n_groups */
    const int32_t* group_setbits;  /* n_groups; -1: the subgroups differ in popcount */
    const uint32_t* group_vbegin;  /* n_groups + 1 */
    uint32_t n_vsub;
    const uint64_t* vsub_val;      /* n_vsub */
    const uint32_t* vsub_tbegin;   /* n_vsub + 1 */
    uint32_t n_terms;
    const uint64_t* term_sign;     /* n_terms */
    const double* term_coeff;      /* 2 x n_terms */
} qb_program_desc;

const char* qb_last_error(void);
int qb_device_count(int* count);

/* ---- sectors -------------------------------------------------------------------------------
 * qb_sector_create enumerates the sector on the device: the representatives ascending, their
 * 1/norm, and the state -> index lookup. Replaces the reference's host orbit scan and sector
 * filter (include/ed/basis/orbit_table.h:250-286 build_orbit_table_fixed_sz_streaming,
 * src/engine/group_sector.cpp:159-205 filter_reps, src/engine/context.cpp:189-207 build_k_sector)
 * and its device mirror upload (src/gpu/rep_matvec.cu:253-383 build_sector_mirror). */
int qb_sector_create(const qb_sector_desc* desc, qb_sector** out);
/* The same from host representatives computed elsewhere (reps ascending, inv_norms): the upload
 * the reference's make_sector_matvec_gpu_rep performs from a RepSectorData
 * (include/ed/gpu/rep_matvec.h:43-60). */
int qb_sector_create_from_reps(const qb_sector_desc* desc, const uint64_t* reps, const double* inv_norms,
                               uint64_t dim, qb_sector** out);
int qb_sector_destroy(qb_sector* s);
uint64_t qb_sector_dim(const qb_sector* s);
/* Copies the representatives and 1/norms to host memory (either pointer may be NULL). */
int qb_sector_download(const qb_sector* s, uint64_t* reps, double* inv_norms);
/* Bytes of device memory the sector holds; sublattice block size L and block count m (0: none). */
int qb_sector_info(const qb_sector* s, uint64_t* device_bytes, int* slc_L, int* slc_m, int* lookup_kind);
/* The orbit index and projection phase of a state (index_and_projection,
 * include/ed/matvec/rep_symmetry_basis_policy.h:221-241), for n states at once (host arrays). */
int qb_index_and_projection(const qb_sector* s, const uint64_t* states, uint64_t n, int64_t* index, double* proj);

/* The sublattice key order a sector of this descriptor canonicalises in (host work only; no device needed):
 * the rule of include/ed/basis/sublattice_code.h:23-34 and 164-191 under desc->sublattice_mode -- a block
 * system of the group's site permutations with L sites in each of m blocks, block j holding key bits
 * [N - (j + 1) L, N - j L) -- and its tables: lead[j * 2^L + x], the least leading block an element reaches from
 * pattern x of block j, and cand[cand_off[j * 2^L + x] ...], the elements that reach it, ascending. *L = *m = 0:
 * no code (the plain order). Sizes: key_bit n_sites, lead m 2^L, cand_off m 2^L + 1, cand *n_cand; any output
 * array may be NULL (call once with NULLs for the sizes). */
int qb_key_order(const qb_sector_desc* desc, int* L, int* m, uint64_t* n_cand, int32_t* key_bit, uint16_t* lead,
                 uint32_t* cand_off, uint16_t* cand);

/* ---- sectors by content ----------------------------------------------------------------------
 * qb_sector_acquire returns the one device sector of a descriptor (the device, group, characters,
 * representative order and lookup), enumerating it on first use: repeated requests share it, as the
 * reference shares its content-keyed sector mirrors (src/gpu/rep_matvec.cu:501-609). Release it with
 * qb_sector_release (not qb_sector_destroy); released sectors stay cached up to a byte capacity (default
 * 4 GiB, oldest evicted first; qb_registry_capacity changes it, 0 empties the cache). */
int qb_sector_acquire(const qb_sector_desc* desc, qb_sector** out);
int qb_sector_release(qb_sector* s);
int qb_registry_capacity(uint64_t bytes);
int qb_registry_stats(uint64_t* sectors, uint64_t* idle_sectors, uint64_t* idle_bytes);
/* The library's cache of released device blocks on the current device (a released block is kept, up to 16 GiB,
 * for a later allocation of about its size, because cudaFree synchronises the device): free the oldest idle
 * blocks until at most keep_bytes remain, and report what remains in *idle_bytes (may be NULL). After a large
 * solve, trimming to 0 returns its buffers to the device, as torch.cuda.empty_cache does for torch's cache, so
 * later small solves do not pay the frees one by one. The reference has no such cache (it frees per call). */
int qb_memory_trim(uint64_t keep_bytes, uint64_t* idle_bytes);
/* A sector's descriptor, representatives and 1/norms in a file (a checksummed little-endian format), and a
 * sector made from such a file (the tables and lookup rebuilt, no enumeration): the cached sector-table
 * format of repeated runs (the reference keeps its orbit tables in a registry, include/ed/basis/orbit_table.h). */
int qb_sector_save(const qb_sector* s, const char* path);
int qb_sector_load(const char* path, qb_sector** out);

/* ---- programs ------------------------------------------------------------------------------ */
int qb_program_create(const qb_program_desc* desc, qb_program** out);
int qb_program_destroy(qb_program* p);

/* ---- the matvec ----------------------------------------------------------------------------
 * outs[i] = O ins[i] for i < k: rows in sector `row`, columns in sector `col` (row == col: one
 * sector, the diagonal without a lookup). Device pointers of the given dtype. Every output equals
 * the single apply bit for bit. Replaces make_sector_matvec_gpu_rep / _multi and
 * make_cross_matvec_gpu_rep (include/ed/gpu/rep_matvec.h:43-70, src/gpu/rep_matvec.cu:410-490) and
 * serves LinearOperator::bind_cuda / bind_cuda_multi (include/ed/matvec/linear_operator.h:45-69). */
int qb_matvec(const qb_sector* row, const qb_sector* col, const qb_program* prog, const void* const* ins,
              void* const* outs, int k, int dtype, void* stream);
/* out = O in on k vectors interleaved by row (element r*k + v): the block matvec of the sampled
 * methods, one canonicalisation per emitted entry for all k vectors. */
int qb_matvec_block(const qb_sector* row, const qb_sector* col, const qb_program* prog, const void* in, void* out,
                    int k, int dtype, void* stream);
/* The host-pointer twin (make_sector_matvec_gpu_rep_hostptr, include/ed/gpu/rep_matvec.h:61-66):
 * host complex128 in / out, staged through the device. */
int qb_matvec_host(const qb_sector* row, const qb_sector* col, const qb_program* prog, const double* in_host,
                   double* out_host);

/* ---- the reduced-CSR lane ------------------------------------------------------------------
 * The merged rows of an operator between two sectors, built once and streamed: columns ascending,
 * equal columns summed in emission order, exact zeros dropped (build_sector_csr / build_cross_csr,
 * include/ed/matvec/sector_rows.h:147-404). Values are stored as u8 or u16 ids into a dictionary of the
 * distinct values when that is the smaller form (ReducedSymmetryCsr, include/ed/matvec/reduced_csr.h:36-75),
 * else whole. */
typedef struct qb_csr qb_csr;
/* Built on the device from the row walk (build_sector_csr_gpu, include/ed/gpu/rep_matvec.h:78-85).
 * QB_ENOMEM when it would take more than max_bytes (0: no budget) or the device's free memory (the
 * reference returns null there); QB_EUNSUPPORTED when a row has more than 256 entries before merging or
 * the column sector has 2^32 states or more. */
int qb_csr_build(const qb_sector* row, const qb_sector* col, const qb_program* prog, uint64_t max_bytes,
                 qb_csr** out);
/* A CSR built on the host (row_ptr: row->dim + 1 entries; col_idx, val: row_ptr[dim] entries, val
 * interleaved complex128), uploaded as is (upload_csr_gpu, include/ed/gpu/rep_matvec.h:87-91). */
int qb_csr_upload(const qb_sector* row, const qb_sector* col, const uint64_t* row_ptr, const uint32_t* col_idx,
                  const double* val, uint64_t max_bytes, qb_csr** out);
int qb_csr_destroy(qb_csr* csr);
/* nnz, device bytes, and the dictionary size (-1: values stored whole) (device_csr_info,
 * include/ed/gpu/rep_matvec.h:98). Any output may be NULL. */
int qb_csr_info(const qb_csr* csr, uint64_t* nnz, uint64_t* bytes, int* n_dict);
/* The entries copied to host arrays (download_csr, include/ed/gpu/rep_matvec.h:100-101): row_ptr
 * (rows + 1), col (nnz), val (2 * nnz doubles). Any output may be NULL. */
int qb_csr_download(const qb_csr* csr, uint64_t* row_ptr, uint32_t* col, double* val);
/* out = A in on k vectors (k == 1: one vector; k <= 64: interleaved by row) of dtype, device pointers
 * (csr_matvec_gpu / csr_matvec_gpu_multi, include/ed/gpu/rep_matvec.h:93-96). Each row is summed in
 * entry order from zero, as ReducedSymmetryCsr::spmv does (include/ed/matvec/reduced_csr.h:89-102): in
 * FP64 storage y equals the host CSR's bit for bit, and every vector of a k-vector apply equals its
 * single apply. */
int qb_csr_matvec(const qb_csr* csr, const void* in, void* out, int k, int dtype, void* stream);
/* Routes every apply of prog on the CSR's sector pair (qb_matvec, qb_matvec_block, qb_matvec_host and
 * the Krylov drivers) through the CSR; NULL detaches. The CSR must outlive the attachment. This is the
 * lane choice of RepSectorMatVec (device_csr_, src/engine/internal.h:399-434). */
int qb_program_attach_csr(qb_program* prog, const qb_csr* csr);

/* ---- Krylov recurrences --------------------------------------------------------------------
 * The Lanczos kernel (include/ed/krylov/lanczos.h:266-576) on one sector, device-resident: alpha,
 * beta and every inner product in FP64, vectors stored as dtype. v0 is a host complex128 vector
 * (it is normalised on the device). alpha has room for max_iter values, beta for max_iter + 1
 * (beta[0] = 0). reorth: QB_REORTH_NONE or QB_REORTH_LOCAL (ring of 1, threshold sqrt(eps)). */
int qb_lanczos(const qb_sector* sec, const qb_program* prog, const double* v0_host, int max_iter, int reorth,
               double breakdown_tol, int dtype, double* alpha, double* beta, int* iters);

/* The lanes' staged Gaussian start of dimension n from mt19937_64(seed) (staged_seed, src/engine/block_solve.cpp:
 * 263-277; entry = (re, im) with the imaginary part drawn first): host work, out = 2n doubles. The reference's
 * stream bit for bit; drawn on the host's cores in parallel past 2^20 entries (the generator's raw outputs in
 * order on one thread, the normal transform of the accepted polar attempts on the others). */
int qb_staged_start(uint64_t seed, uint64_t n, double* out);

/* The k = 1 block lane (lowest_scan_lane, src/engine/block_solve.cpp:528-598): a Lanczos scan from
 * the staged Gaussian start of seed 0x51ED0B70 with the Paige-gated, ghost-aware lowest-level test
 * after every step; budget max_iter (0: 400). dtype QB_C64 runs the recurrence on FP32-stored
 * vectors; refine != 0 then polishes the level with FP64 restarted Lanczos from its Ritz vector to
 * |dE|/|E| <= 1e-12. e0: the lowest level (NaN if none converged). */
int qb_eigs_lowest(const qb_sector* sec, const qb_program* prog, int max_iter, int dtype, int refine, double* e0,
                   int* iters, int* converged, int* matvecs);

/* The certified lowest eigenpair of a sector with its vector (gs_vector / gs_lanczos,
 * src/engine/block_solve.cpp:697-845): a Paige-gated recurrence without reorthogonalisation from
 * staged_seed(0x51ED900D), the Ritz vector from the kept basis or a replay, restarted from it until
 * ||H u - E u|| <= 1e-9 * (sum |coeff|), at most 5 attempts of 600 steps (max_steps > 0 caps all of them).
 * vec_device (n complex128, device) and vec_host (2n doubles) may each be NULL. */
int qb_ground_state(const qb_sector* sec, const qb_program* prog, int max_steps, double* e0, double* residual,
                    int* certified, void* vec_device, double* vec_host, int* matvecs);

/* The k > 1 lane: the k lowest levels of a sector (the contract of krylov_schur_lane,
 * src/engine/block_solve.cpp:433-510: the k lowest levels ascending, each converged to a residual of
 * 1e-10 * (sum |coeff|), multiplicities resolved, from the staged Gaussian start of seed 0x51ED0B70) by
 * thick-restart Lanczos with full reorthogonalisation, its scalars kept on the device and read once per
 * restart cycle; a fresh start deflated against the found levels then searches below the k-th for
 * further members of a multiplet. values: the k lowest, ascending (NaN past n_found). max_iter: matvec
 * budget (0: max(200k, 2000)). vecs_device: NULL, or k device pointers (each n complex128, or NULL) for
 * the eigenvectors. qb_eigs_k is qb_eigs_levels with dtype QB_C128. */
int qb_eigs_k(const qb_sector* sec, const qb_program* prog, int k, uint64_t max_iter, double* values, int* n_found,
              int* converged, int* matvecs, void* const* vecs_device);
/* The same with the Lanczos vectors stored as dtype: QB_C64 stores them as complex64 (FP64 arithmetic and
 * scalars) and converges to 1e-6 * scale; refine != 0 then refines the returned pairs in FP64 (Rayleigh-Ritz
 * on the pairs and their residuals, repeated) to the 1e-10 * scale residual. */
int qb_eigs_levels(const qb_sector* sec, const qb_program* prog, int k, uint64_t max_iter, int dtype, int refine,
                   double* values, int* n_found, int* converged, int* matvecs, void* const* vecs_device);

/* T = 0 dynamics of an operator O from sector src to sector tgt (src/engine/dynamics.cpp:442-566): the
 * certified ground state psi0 of h_src, phi = O psi0 (op: the cross row program, rows in tgt, columns in
 * src), and the continued fraction of h_tgt from phi (cf_spectral_from_vector, include/ed/dynamics/cf.h:104-160)
 * at depth max(depth, 2), shifted by E0, tolerance 64 eps * scale. S: n_omega values; conv_change: the
 * half-depth change of the fraction. */
int qb_dynamics_t0(const qb_sector* src, const qb_program* h_src, const qb_sector* tgt, const qb_program* h_tgt,
                   const qb_program* op, int depth, const double* omega, int n_omega, double eta, double* S, double* e0,
                   double* conv_change, int* certified);

/* T = 0 dynamics averaged over the ground manifold (src/engine/dynamics.cpp:147-195, 395-566; the ground manifold
 * is every level within degeneracy_tol * (sum |coeff| of h_srcs[0]) of E0, include/ed/sectors/dynamics.h:17-21):
 * the lowest level of every source block (the k = 1 lane); in each block at E0, every level within the window
 * with its vector (the k > 1 lane, k doubled until a level lies above the window); then for each such state a,
 * the continued fraction of h_tgts[b] from phi = ops[b] |a> in the target block tgts[b] of its source block b
 * (ops[b]: rows in tgts[b], columns in srcs[b]), shifted by E0; S = the average over the manifold's states.
 * manifold: the number of states averaged; certified: every solve converged. */
int qb_dynamics_t0_manifold(int n_src, const qb_sector* const* srcs, const qb_program* const* h_srcs,
                            const qb_sector* const* tgts, const qb_program* const* h_tgts, const qb_program* const* ops,
                            int depth, const double* omega, int n_omega, double eta, double degeneracy_tol, double* S,
                            double* e0, int* manifold, int* certified);

/* The full spectrum of a small block (at most 8192 states), ascending, with multiplicity: the dense tail of
 * the thermal and eigs drivers (blocks up to dense_max_dim are solved exactly, include/ed/sectors/thermal.h:35;
 * the reference's device pool of dense eigensolves, src/gpu/little_group.cu:185-188). The block is assembled on
 * the device from the block matvec on identity columns. Blocks of at most 1024 states are reduced on the device
 * (Householder reflections to a real tridiagonal, a CTA per block, then every eigenvalue by Sturm bisection);
 * larger ones on the host (the same reflections, then implicit QL). */
int qb_dense_levels(const qb_sector* sec, const qb_program* prog, double* values);
/* The same for many blocks at once: block b's levels at values[sum of the earlier blocks' dims ...]. When every
 * block has at most 1024 states, all are assembled into one device buffer and reduced by one launch (a CTA per
 * block, largest first); else largest first over host threads, each assembling on its own stream. */
int qb_dense_levels_blocks(const qb_sector* const* secs, const qb_program* const* progs, int n_blocks,
                           double* values);

/* FTLM on one block (ftlm_kernel, include/ed/thermal/ftlm.h:277-480; sample vectors of
 * include/ed/thermal/sample_seed.h:37-89): all samples advance together as one block matvec.
 * Outputs per beta: lnZ, E, V; and the lowest weighted Ritz value. */
int qb_ftlm(const qb_sector* sec, const qb_program* prog, int samples, int depth, uint64_t seed, const double* betas,
            int n_beta, int dtype, double* lnZ, double* E, double* V, double* e_min);

/* FTLM over many blocks, the sampled per-block path of the thermal driver (src/engine/thermal.cpp:155-340
 * over the blocks of one call). seed_mode picks the sample vectors:
 *   QB_SEED_PER_BLOCK  the driver's own streams: before each block, in the order given, the seed takes one step
 *                      of the 64-bit LCG seed * 6364136223846793005 + 1442695040888963407 (thermal.cpp:470-471),
 *                      and sample s of block b is the first dim_b draws of sample_engine(seed_b, s)
 *                      (sample_seed.h:37-89): the reference's vectors draw for draw, given the blocks in its
 *                      order;
 *   QB_SEED_SHARED     every block uses the call's seed (sample s of block b: the first dim_b draws of
 *                      sample_engine(seed, s)), so one table of streams, drawn once, serves every block.
 * Blocks run largest first on a few streams; each block's samples advance together as one block matvec, on the
 * block's reduced CSR (built inside the call) when use_csr != 0 and it fits, else on the row walk. Outputs per
 * block b and beta t at [b * n_beta + t]: lnZ, E, V; e_min[b]. stats (NULL or 4 doubles): seconds spent drawing
 * the samples, building the CSRs, running the recurrences, and forming the curves (the per-block build / apply
 * times the thermal driver reports). */
enum { QB_SEED_SHARED = 0, QB_SEED_PER_BLOCK = 1 };
int qb_ftlm_blocks(const qb_sector* const* secs, const qb_program* const* progs, int n_blocks, int samples, int depth,
                   uint64_t seed, int seed_mode, const double* betas, int n_beta, int dtype, int use_csr, double* lnZ,
                   double* E, double* V, double* e_min, double* stats);

/* The blocks' curves combined in log space (src/engine/thermal.cpp:599-641): lnZ = logsumexp_b(ln w_b +
 * lnZ_b), E = sum_b p_b E_b, C = beta^2 sum_b p_b (V_b + (E_b - E)^2) (the law of total variance), S = lnZ +
 * beta E, F = -lnZ / beta. weights: per-block multiplicities (NULL: all 1). Inputs [b * n_beta + t]. */
int qb_thermal_combine(int n_blocks, const double* weights, const double* lnZ, const double* E, const double* V,
                       const double* betas, int n_beta, double* lnZ_out, double* E_out, double* C_out, double* S_out,
                       double* F_out);

/* The T = 0 continued fraction from a host complex128 vector phi on one sector
 * (cf_spectral_from_vector, include/ed/dynamics/cf.h:104-160): Lanczos without reorthogonalisation to
 * `depth`, breakdown at `tolerance`, S(w) = -Im G(w + i eta)/pi with G weighted by ||phi||^2; shift: the
 * energy w is measured from (NaN: the tridiagonal's lowest value). */
int qb_cf(const qb_sector* sec, const qb_program* prog, const double* phi_host, int depth, const double* omega,
          int n_omega, double eta, double shift, double tolerance, double* S, double* shift_out);

/* ---- the Lanczos kernel without allocation ---------------------------------------------------
 * No counterpart in the reference: an addition for callers that cannot let a library call cudaMalloc
 * -- a framework whose caching allocator already holds the device, or a service that fixed its memory
 * plan at start-up; there a mid-run cudaMalloc can fail on a full pool, and it synchronises the device.
 * Same recurrence as qb_lanczos, on buffers the caller owns:
 *   v0    device complex128, sector dim (the start, not necessarily normalised; left untouched)
 *   work  device scratch the caller owns: dim x (2 x element size of dtype + 16) bytes
 *   alpha / beta  host outputs as for qb_lanczos (max_iter and max_iter + 1 values)
 * Its own scratch (the alpha / beta history, reduction partials, a counter) is a file-scope device array
 * of about 54 KB that every GPU which loads the library holds until exit; max_iter above
 * QB_NOALLOC_MAX_ITER is refused (QB_EINVAL). The first call on a device resolves that array's device
 * address (cudaGetSymbolAddress), so make it before any stream capture. Calls share the array and clear
 * what must start at zero; calls that overlap on the GPU (two streams, two threads) race on it.
 * reorth: QB_REORTH_NONE or QB_REORTH_LOCAL. */
#define QB_NOALLOC_MAX_ITER 1024
int qb_lanczos_noalloc(const qb_sector* sec, const qb_program* prog, const void* v0, void* work, int max_iter,
                       int reorth, double breakdown_tol, int dtype, double* alpha, double* beta, int* iters,
                       void* stream);

/* ---- launch-shape tuning ----------------------------------------------------------------------
 * Kernel families with several launch shapes that give the same result bit for bit:
 *   "walk"       the row walk (qb_matvec and the Krylov lanes on the walk): 0 one thread per state,
 *                1 a warp's states compacted (every lane canonicalises a target while any row has one);
 *                for one vector also 2, 3, 4, 5 = a team of 8, 16, 32, 4 lanes per state;
 *   "walk_team"  the block walk of k interleaved vectors (qb_matvec_block, FTLM on the walk): 0, 1, 2, 3 =
 *                8, 16, 32, 4 lanes per state (4 only when k <= 32).
 * The first launch for a size class (the sector's group and lookup, the program's groups, the row count by
 * powers of two, the vectors' number and types, the device) times every shape on the caller's stream (one
 * warm-up and three timed runs each; this synchronises that stream once) and keeps the fastest. A stream
 * that is capturing a graph is never timed. No reference counterpart: the reference fixes its launch shapes
 * (src/gpu/rep_matvec.cu).
 * mode: 1 measure on first use (the default; QB_TUNE overrides it at start), 2 only choices already known
 * (this process, or a loaded file), else shape 0; 0 always shape 0; -1 only reads *previous.
 * QB_TUNE_CACHE=path: choices are read from path at first use and each new one is appended to it. */
int qb_tune_mode(int mode, int* previous);
/* Forces candidate `choice` for every launch of a family (choice < 0 removes the force). */
int qb_tune_force(const char* family, int choice);
/* Forgets every known choice and every force. */
int qb_tune_clear(void);
/* Writes the known choices ("key<TAB>choice<TAB>ms per candidate" lines) to path; reads such a file. */
int qb_tune_save(const char* path);
int qb_tune_load(const char* path);
/* The known choices as that text, NUL-terminated, in buf (len bytes); *needed: the bytes it takes. */
int qb_tune_entries(char* buf, uint64_t len, uint64_t* needed);

/* ---- the request server ---------------------------------------------------------------------
 * Eigs, thermal and T = 0 dynamics solves of sectors of different sizes served on one GPU with continuous
 * batching: requests queue in arrival order; a worker admits the head when one of max_active slots is
 * free and the request's estimated HBM footprint (sectors, reduced CSRs, Krylov vectors) fits what is
 * left of hbm_budget (0: 80% of the free memory); a request larger than the budget runs alone. Admitted
 * requests run concurrently, each on its worker's own stream. No reference counterpart: the reference
 * serves one call at a time through its verbs (python/qed/_verbs). A thermal request is one block of the
 * thermal driver's sampled path (the unit its driver dispatches per block, src/engine/thermal.cpp:470-490):
 * FTLM of the block from sample_engine(seed, s), s < samples, at depth `krylov`, per inverse temperature. */
typedef struct qb_server qb_server;
enum { QB_REQ_EIGS = 0, QB_REQ_DYNAMICS = 1, QB_REQ_THERMAL = 2 };
#define QB_SERVER_MAX_LEVELS 16
typedef struct {
    int kind;                 /* QB_REQ_EIGS, QB_REQ_DYNAMICS or QB_REQ_THERMAL */
    qb_sector_desc sector;    /* eigs, thermal: the sector; dynamics: the source sector */
    qb_program_desc h;        /* the Hamiltonian's row program (compile_operator(H^dagger)) */
    int k;                    /* eigs: levels wanted, 1..16 (k = 1: the scan lane; k > 1: the k > 1 lane) */
    qb_sector_desc target;    /* dynamics: the target sector */
    qb_program_desc op;       /* dynamics: the operator's cross row program (rows in target, columns in source) */
    int krylov;               /* dynamics: continued-fraction depth; thermal: Lanczos depth */
    const double* omega;      /* dynamics: n_omega frequencies */
    int n_omega;
    double eta;
    int samples;              /* thermal: sample vectors, 1..64 */
    uint64_t seed;            /* thermal: the block's base seed */
    const double* betas;      /* thermal: n_beta inverse temperatures */
    int n_beta;
} qb_request;
typedef struct {
    int status;               /* QB_OK, or the error of the solve (qb_last_error then describes it) */
    int n_values;
    double values[QB_SERVER_MAX_LEVELS];   /* eigs: the levels ascending; dynamics: E0; thermal: the lowest Ritz value */
    int converged;            /* eigs: converged; dynamics: the ground state certified; thermal: 1 */
    int matvecs;
    double e0, conv_change;   /* dynamics */
    double t_submit, t_admit, t_done;      /* seconds on the server's clock (qb_server_clock) */
    uint64_t footprint;       /* the bytes the request was admitted with */
} qb_result;
/* The request's descriptors are copied: the caller's arrays may be freed when submit returns. */
int qb_server_create(int max_active, uint64_t hbm_budget, qb_server** out);
int qb_server_submit(qb_server* s, const qb_request* r, uint64_t* ticket);
/* Waits up to timeout_ms (< 0: no limit) for a ticket; QB_ETIMEOUT when it is not done. A returned result
 * releases the ticket. S: NULL, or the request's curves: a dynamics request's spectrum (n_omega doubles); a
 * thermal request's lnZ, E and V per beta (3 x n_beta doubles, in that order). */
int qb_server_wait(qb_server* s, uint64_t ticket, int timeout_ms, qb_result* out, double* S);
int qb_server_clock(qb_server* s, double* seconds);
/* Finishes the admitted requests and drops the queued ones; call it once no thread waits on a ticket. */
int qb_server_destroy(qb_server* s);

#ifdef __cplusplus
}
#endif
#endif
