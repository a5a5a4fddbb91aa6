/* =============================================================================
 * oracle/qed_oracle.h -- TEST INFRASTRUCTURE: the C-ABI of the restated CPU oracle.
 *
 * A plain, serial restatement of the reference engine's CPU algorithm for the symmetry-sector
 * matvec and the Lanczos / FTLM / continued-fraction recurrences (every function in
 * qed_oracle.cpp cites the reference file:line it follows). It is the checker of the CUDA path:
 * only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load it.
 *
 * Complex vectors are interleaved (re, im) doubles. Return codes: 0 ok, -1 error (qo_last_error).
 * ============================================================================= */
#ifndef QED_ORACLE_H
#define QED_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

const char* qo_last_error(void);

/* A sector: the fixed-Sz states of n_sites with n_up set bits, reduced by a group of G elements
 * (perms: G x n_sites, new bit i = old bit perms[g*n+i]; flips: G XOR masks or NULL) in the 1-dim
 * irrep with characters chars (G interleaved complex). slc_mode: 0 plain order, 1 sublattice code
 * whenever a block system exists, -1 the size rule of device verbs (N >= 24, >= 16 distinct
 * permutations), -2 the strict rule (>= 64). */
void* qo_sector_new(int n_sites, int n_up, int G, const int32_t* perms, const uint64_t* flips, const double* chars,
                    int slc_mode);
void qo_sector_free(void* s);
uint64_t qo_sector_dim(void* s);
void qo_sector_get(void* s, uint64_t* reps, double* inv_norms);
/* 1 with the code's block size, block count and each site's key position, or 0 (plain order). */
int qo_sector_slc(void* s, int* L, int* m, int32_t* key_bit);
int64_t qo_index_and_projection(void* s, uint64_t state, double* proj);

/* A row program in the reference's MaskedProgram layout (term_coeff interleaved complex). */
void* qo_prog_new(uint32_t n_groups, const uint64_t* group_flip, const int32_t* group_setbits,
                  const uint32_t* group_vbegin, uint32_t n_vsub, const uint64_t* vsub_val, const uint32_t* vsub_tbegin,
                  uint32_t n_terms, const uint64_t* term_sign, const double* term_coeff);
void qo_prog_free(void* p);

/* out = O in, rows in sector row, columns in sector col (row == col: one sector). */
int qo_gather(void* row, void* col, void* prog, const double* in, double* out);
/* The merged row entries (columns ascending, equal columns summed in emission order, zeros dropped):
 * row_ptr (dim+1) and, when col != NULL, the columns and values. Two calls: sizes, then fill. */
int qo_csr(void* row, void* col_sector, void* prog, uint64_t* row_ptr, uint32_t* col, double* val);
/* The emitted entries (before merging) of every row: sum over rows, and the diagonal count. */
int qo_count_emitted(void* row, void* col, void* prog, uint64_t* emitted);

/* Lanczos (reorth 0 none, 1 full CGS2 with DGKS gate, 2 local K=1); alpha max_iter, beta max_iter+1. */
int qo_lanczos(void* sec, void* prog, const double* v0, int max_iter, int reorth, double breakdown_tol,
               double* alpha, double* beta, int* iters);
/* The k = 1 block lane: E0 of the sector from the staged start of seed 0x51ED0B70. */
int qo_scan_lowest(void* sec, void* prog, int max_iter, double* e0, int* iters, int* converged);
/* Tridiagonal eigenvalues (ascending) and, if vectors != NULL, eigenvectors column-major m x m. */
int qo_tridiag_eig(const double* alpha, const double* beta, int m, double* values, double* vectors);
/* The Gaussian sample vector s of base seed (unit norm) / the block lanes' unnormalised start. */
void qo_sample_vector(uint64_t base_seed, uint64_t s, uint64_t n, double* out);
void qo_staged_seed(uint64_t seed, uint64_t n, double* out);
/* FTLM of one block: lnZ, E, V per beta and the lowest weighted Ritz value. */
int qo_ftlm(void* sec, void* prog, int samples, int depth, uint64_t seed, const double* betas, int nb, double* lnZ,
            double* E, double* V, double* e_min);
/* Per-sample FTLM moments (e_min, Z, E1, E2 per beta) of one sample from its alpha/beta. */
int qo_sample_moments(const double* alpha, const double* beta, int m, const double* betas, int nb, double* e_min,
                      double* Z, double* E1, double* E2);
/* The continued fraction S(w) of a tridiagonal (alpha - shift), weight norm_sq. */
void qo_continued_fraction(const double* alpha, const double* beta, int m, const double* omega, int nw, double eta,
                           double norm_sq, double* S);
/* T = 0 spectral function from phi on one sector (Lanczos without reorth, depth, CF). */
int qo_cf(void* sec, void* prog, const double* phi, int depth, const double* omega, int nw, double eta, double shift,
          double tolerance, double* S, double* shift_out);

#ifdef __cplusplus
}
#endif
#endif
