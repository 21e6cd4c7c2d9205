/*
 * sqd_b200.h — C ABI of the B200 (sm_100a) implementation of the sample-based quantum
 * diagonalization (SQD) hot path of rqutils: Pauli-sum preprocessing, subspace build, the
 * matrix-free Pauli-sum matvec over a sorted subspace of computational-basis bitstrings, and the
 * single-vector LOCG/LOBPCG ground-state solver that drives it.
 *
 * Conventions
 *  - Every array argument is a DEVICE pointer unless its name ends in `_host`.  The library never
 *    frees memory it did not allocate.  Opaque handles own the tables they build (allocated
 *    stream-ordered on the stream passed at creation) and are released with *_destroy.
 *  - `stream` is a cudaStream_t passed as void* (NULL = legacy default stream).  All work is
 *    stream-ordered; functions that return host scalars synchronize that stream.
 *  - Return value: SQD_OK (0) or a negative status; sqd_last_error() gives the message of the
 *    last failure on the calling thread.  No C++ exception crosses the ABI.
 *  - A state is a uint64 whose bit q is qubit q (num_qubits <= 63).  A Pauli term is a pair of
 *    uint64 masks (x, z): X on qubits with x=1,z=0, Y on x=1,z=1, Z on x=0,z=1.
 *  - Vector dtypes: SQD_F64, SQD_C128 (interleaved re/im doubles), SQD_F32, SQD_C64.
 *
 * The rqutils functions each entry point replaces are cited as path:line within rqutils.
 */
#ifndef SQD_B200_H
#define SQD_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum sqd_status {
  SQD_OK = 0,
  SQD_ERR_INVALID = -1,    /* bad argument (maps to ValueError) */
  SQD_ERR_CUDA = -2,       /* CUDA runtime error */
  SQD_ERR_UNSUPPORTED = -3,
  SQD_ERR_DEVICE = -4,     /* a kernel reported an error through its device status word */
  SQD_ERR_MEMORY = -5
};

enum sqd_dtype { SQD_F64 = 0, SQD_C128 = 1, SQD_F32 = 2, SQD_C64 = 3 };

/* Flags for sqd_paulis_create. */
#define SQD_PAULIS_FORCE_REAL 1u

/* Lookup methods for the b XOR x search.  SQD_LOOKUP_PRODUCT (operators only): when the
 * subspace is the product of strings on the high and the low half of the qubits, each half is
 * looked up in its own sorted string list, once per string instead of once per row, and the
 * rows' pairs are assembled from those lists (same pairs, same order); SQD_ERR_UNSUPPORTED for
 * other subspaces.  SQD_LOOKUP_AUTO: SQD_LOOKUP_PRODUCT where it applies, else SQD_LOOKUP_HASH. */
enum sqd_lookup {
  SQD_LOOKUP_HASH = 0,
  SQD_LOOKUP_BSEARCH = 1,
  SQD_LOOKUP_AUTO = 2,
  SQD_LOOKUP_PRODUCT = 3
};

typedef struct sqd_paulis_s* sqd_paulis_t;
typedef struct sqd_space_s* sqd_space_t;
typedef struct sqd_op_s* sqd_op_t;
typedef struct sqd_batch_s* sqd_batch_t;

/* ---------------------------------------------------------------- library ------------------ */
const char* sqd_version(void);
const char* sqd_last_error(void);
/* The library allocates its tables and solver work vectors from its own stream-ordered memory
 * pool per device, which keeps freed memory for reuse (no counterpart in rqutils, where XLA
 * owns device memory).  This releases all but keep_bytes of the current device's pool back to
 * the driver (synchronizes the device). */
int sqd_trim_memory(uint64_t keep_bytes);
/* Usage of that pool on the current device (no counterpart in rqutils): bytes reserved from the
 * driver, bytes in live allocations, and the high-water mark of the latter, which reset_high
 * != 0 first resets to the current usage.  Any output pointer may be NULL. */
int sqd_memory_stats(uint64_t* reserved_host, uint64_t* used_host, uint64_t* used_high_host,
                     int reset_high);

/* ---------------------------------------------------------------- Pauli sums --------------- */
/* PauliSumXZ.from_paulisum (paulis/symplectic.py:50-124), on the device: drops zero
 * coefficients, merges duplicate (x, z) terms, groups by X mask (groups ascending in x, terms
 * ascending in z within a group — the reference's np.unique order), multiplies in the phase
 * (-i)^{popcount(x & z)}, and optionally keeps only real parts (force_real).  coef_im may be
 * NULL.  *imag_dropped_host (may be NULL) is set to 1 when force_real discarded a nonzero
 * imaginary part (the reference warns, symplectic.py:93-94). */
int sqd_paulis_create(const uint64_t* x, const uint64_t* z, const double* coef_re,
                      const double* coef_im, int64_t num_raw_terms, int num_qubits,
                      uint32_t flags, void* stream, sqd_paulis_t* out, int* imag_dropped_host);
/* The grouped table as the reference stores it (PauliSumXZ fields x, z, c; symplectic.py:41-48)
 * in CSR form: J groups, M merged terms, K_max = largest group. */
int sqd_paulis_info(sqd_paulis_t p, int64_t* num_groups, int64_t* num_terms, int64_t* max_k,
                    int* is_complex, int* num_qubits);
/* group_x[J], group_start[J+1] (int64), term_z[M], term_c[2M] (interleaved re/im), and
 * raw_to_term[num_raw] (int32, -1 for dropped zero coefficients). */
int sqd_paulis_export(sqd_paulis_t p, uint64_t* group_x, int64_t* group_start, uint64_t* term_z,
                      double* term_c, int32_t* raw_to_term, void* stream);
/* New coefficients for the same num_raw_terms terms (same order as at creation), keeping the
 * grouping: merged sums, phases and the per-group stop at the first zero coefficient are
 * recomputed as in sqd_paulis_create.  Terms dropped at creation (zero coefficient) must stay
 * zero, and a real sum must stay real; otherwise SQD_ERR_INVALID.  Operators built on p need
 * sqd_op_refresh afterwards.  No rqutils counterpart (rqutils rebuilds the PauliSumXZ); used by
 * the coefficient-gradient path. */
int sqd_paulis_set_coeffs(sqd_paulis_t p, const double* coef_re, const double* coef_im,
                          void* stream, int* imag_dropped_host);
void sqd_paulis_destroy(sqd_paulis_t p);

/* ---------------------------------------------------------------- subspace ----------------- */
/* np.packbits(np.pad(states,...)) of sqd.py:255 in the uint64 representation: bits[n_rows,
 * num_qubits] (uint8 0/1, last column = qubit 0, row-major) -> uint64 values. */
int sqd_pack_states(const uint8_t* bits, int64_t n_rows, int num_qubits, uint64_t* out,
                    void* stream);
/* uniquify_states (sqd.py:445-482): sorts and de-duplicates n_in states, keeps states_size >=
 * n_unique vector slots (the tail are fill-in slots), and builds the lookup structures. */
int sqd_space_create(const uint64_t* states, int64_t n_in, int num_qubits, int64_t states_size,
                     void* stream, sqd_space_t* out);
int sqd_space_info(sqd_space_t s, int64_t* n_unique, int64_t* states_size, int* num_sectors,
                   uint64_t* sector_masks_host /* [2] */);
/* Sorted unique states (n_unique values). */
int sqd_space_states(sqd_space_t s, uint64_t* out, void* stream);
/* get_xsource (sqd.py:485-548), sorted input: out[states_size] = index j with S[j] == S[i]^x,
 * else -1; fill-in slots get exactly the values the reference's sort-based algorithm gives.
 * lookup: SQD_LOOKUP_HASH or SQD_LOOKUP_BSEARCH (SQD_LOOKUP_AUTO means the hash table). */
int sqd_xsource(sqd_space_t s, uint64_t x, int lookup, int32_t* out, void* stream);
/* Sorted index of arbitrary keys: out[i] = j with S[j] == keys[i], else -1 (also for keys with
 * bits above num_qubits).  Replaces the index bookkeeping of get_xsource(sorted_input=False)
 * (sqd.py:515-516, 542-545: positions of unsorted input rows in the sorted list) and of
 * uniquify_states(return_indices=True) (sqd.py:478-481).  lookup as in sqd_xsource. */
int sqd_space_lookup(sqd_space_t s, const uint64_t* keys, int64_t n, int lookup, int32_t* out,
                     void* stream);
void sqd_space_destroy(sqd_space_t s);

/* ---------------------------------------------------------------- operator ----------------- */
/* The operator H projected on the subspace, with a connectivity cache chosen by
 * cache_strategy (SQDOptions.cache_strategy, sqd.py:187-189, run_sqd sqd.py:343-404):
 *   x_cache = 1: sources cached (sparse: only (row, group) pairs whose source exists);
 *   x_cache = 0: sources searched inside every matvec;
 *   z_cache = 2: matrix elements (composed diagonals) cached per stored pair;
 *   z_cache = 0 or 1: diagonals recomputed from popcounts inside every matvec.
 * lookup = enum sqd_lookup. */
int sqd_op_create(sqd_paulis_t p, sqd_space_t s, int x_cache, int z_cache, int lookup,
                  void* stream, sqd_op_t* out);
/* nnz = stored (row, group) pairs (0 when x_cache = 0); value_complex = 1 if H has complex
 * matrix elements. */
int sqd_op_info(sqd_op_t op, int64_t* nnz, int64_t* states_size, int* value_complex);
/* Tuning knob of the cached matvec (no rqutils counterpart; rqutils leaves the schedule to
 * XLA): lanes of a warp that share one output row, 1/2/4/8/16/32, kept separately for FP64
 * (precision 0: SQD_F64/SQD_C128) and FP32 (precision 1: SQD_F32/SQD_C64) vectors.  Chosen
 * from the mean row length at creation; the autotuner overrides it. */
int sqd_op_set_lanes(sqd_op_t op, int precision, int lanes_per_row);
int sqd_op_get_lanes(sqd_op_t op, int precision, int* lanes_per_row);
/* Second knob of the cached matvec: 0 = consecutive warps of the grid take consecutive rows;
 * > 0 = each thread block owns chunk_rows consecutive rows at a time (L1 reuse of the source
 * amplitudes that neighbouring rows share). */
int sqd_op_set_chunk(sqd_op_t op, int precision, int64_t chunk_rows);
/* Third knob of the cached matvec (no rqutils counterpart): the element layout it streams.
 * SQD_LAYOUT_CSR: one (source, element) list per row.  SQD_LAYOUT_PRODUCT: for a subspace
 * that is the product of strings on the high and the low half of the qubits (every high string
 * with every low string, no fill-in slots), the pairs that change one half only are stored as
 * dense slabs whose sources are implied by their position (coalesced loads, no index per
 * pair); the pairs that change both halves gather from their source slabs staged in shared
 * memory when all of a slab's sources fit there, else from their CSR lists.
 * SQD_LAYOUT_PRODUCT_CSR: the same slabs, with the two-half pairs always on the CSR lists.
 * Lanes and chunk knobs apply to the two-half pairs.  Setting a product layout builds the
 * slabs on first use (SQD_ERR_UNSUPPORTED when the subspace is not such a product); results
 * equal the CSR layout's up to the order of each row's sum. */
enum sqd_layout { SQD_LAYOUT_CSR = 0, SQD_LAYOUT_PRODUCT = 1, SQD_LAYOUT_PRODUCT_CSR = 2 };
int sqd_op_set_layout(sqd_op_t op, int precision, int layout, void* stream);
int sqd_op_get_layout(sqd_op_t op, int precision, int* layout);
/* Product structure: n_high x n_low rows (0, 0 when the subspace is not a product) and, once
 * the slabs are built, the stored pairs in high-half slabs, low-half slabs and CSR tails (-1
 * before). */
int sqd_op_product_info(sqd_op_t op, void* stream, int64_t* n_high, int64_t* n_low,
                        int64_t* pairs_high, int64_t* pairs_low, int64_t* pairs_mixed);
/* Hv on the subspace (apply_h_x_cached and friends, sqd.py:643-743 via
 * make_x_cached_matvec sqd.py:746-751).  v and out have states_size elements of dtype. */
int sqd_matvec(sqd_op_t op, const void* v, void* out, int dtype, void* stream);
/* Composed diagonal of group j (get_diagonal, sqd.py:603-628) for every slot (fill-in slots use
 * the all-ones state, as the reference's 255 rows do).  dtype SQD_F64 or SQD_C128. */
int sqd_diagonal(sqd_op_t op, int64_t group, void* out, int dtype, void* stream);
/* vinit of run_sqd (sqd.py:406-426): argmin of the real group-0 diagonal over real rows when
 * group 0 has x = 0, else 0. */
int sqd_vinit(sqd_op_t op, int64_t* index_host, void* stream);
/* Same result as sqd_vinit, allocating nothing.  No counterpart in rqutils.  For callers that
 * cannot allocate device memory when they pick the start vector (for example a process whose
 * device memory is fully reserved by its own caching allocator or arena): the partial minima
 * live in a fixed file-scope __device__ array (256 KiB, held by every GPU that loads the
 * library until exit) instead of a per-call cudaMallocAsync.  Limit: 67,108,864 real rows,
 * larger subspaces return SQD_ERR_INVALID.  The array is shared by all calls, so calls whose
 * GPU work overlaps race.  Set-up: the first call on a device looks up the array's device
 * address (cudaGetSymbolAddress, once per device) and keeps it; make that first call before
 * any stream capture begins, and do not use the function on a device after cudaDeviceReset
 * (the kept address then belongs to the destroyed context).  Every call synchronizes `stream`
 * and writes the index to the host. */
int sqd_vinit_noalloc(sqd_op_t op, int64_t* index_host, void* stream);
/* Projected matrix <i|H|j> in CSR (hproj, sqd.py:269-314, with its padding bug fixed):
 * indptr[states_size+1] (int64), indices[nnz] (int32), data[nnz] complex128 (interleaved). */
int sqd_op_csr(sqd_op_t op, int64_t* indptr, int32_t* indices, double* data, void* stream);
/* Hellmann-Feynman per-term reduction g_t = Re <u| P_t |v> for every merged term t (P_t the
 * t-th Pauli string with unit coefficient, projected), FP64; u, v of dtype (SQD_F64/C128). */
int sqd_grad_terms(sqd_op_t op, const void* u, const void* v, int dtype, double* out_terms,
                   void* stream);
/* Recomputes the cached matrix elements (cache z = 2) after sqd_paulis_set_coeffs; the
 * connectivity is unchanged. */
int sqd_op_refresh(sqd_op_t op, void* stream);
/* Turns an operator with cached sources and on-the-fly diagonals (cache_strategy (1, 0) or
 * (1, 1)) into one with cached elements ((1, 2)): computes the element of every stored pair
 * (8 bytes, 16 if complex), same values the on-the-fly matvec composes.  No rqutils counterpart
 * (there the strategy is fixed when run_sqd builds its matvec); rqutils_b200.sqd uses it when
 * the elements fit in device memory. */
int sqd_op_cache_values(sqd_op_t op, void* stream);
/* Frees the per-pair group indices of an operator with cached matrix elements (cache (1, 2)),
 * 4 bytes per stored pair; the matvec, LOCG and batching keep working, while sqd_grad_terms,
 * sqd_op_csr and sqd_op_refresh then return SQD_ERR_INVALID.  No rqutils counterpart. */
int sqd_op_release_groups(sqd_op_t op);
void sqd_op_destroy(sqd_op_t op);

/* ---------------------------------------------------------------- LOCG --------------------- */
/* y = A x for a caller-defined operator; must be stream-ordered on `stream`. */
typedef int (*sqd_matvec_fn)(void* ctx, const void* x, void* y, void* stream);

/* Matvec callback that applies an sqd_op_t passed as ctx (dtype fixed at solver creation). */
int sqd_op_matvec_cb(void* ctx, const void* x, void* y, void* stream);

enum sqd_locg_mode {
  SQD_LOCG_FP64 = 0,      /* faithful FP64 restatement of ground_locg */
  SQD_LOCG_MIXED = 1      /* FP32 inner sweeps + FP64 residual / Rayleigh-Ritz refinement */
};

/* ground_locg (ground_locg.py:128-162 -> _ground_locg_callable :188-423).
 *  n, dtype: vector space (SQD_F64 or SQD_C128 for the result).
 *  fn/ctx: the operator; for SQD_LOCG_MIXED ctx must be an sqd_op_t and fn sqd_op_matvec_cb.
 *  xinit: start vector (device, dtype) or NULL for the one-hot vector at xinit_index.
 *  orth/n_orth: device vectors to orthogonalize against (ground_locg `orth`), n_orth <= 8;
 *  in SQD_LOCG_MIXED the FP32 sweeps project every search direction against FP32 copies
 *  and the FP64 refinement runs the reference iteration with the vectors themselves.
 *  tol < 0 selects the dtype epsilon (:224-225).
 *  use_graph: capture each iteration in a CUDA graph (only with fn == sqd_op_matvec_cb).
 *  Outputs: eigval_host, eigvec (device, n elements of dtype), niter_host, and
 *  residual_host = final |r| (may be NULL).
 *  With an sqd_op_t and no orth vectors, the solver's work vectors and captured iteration
 *  graphs stay with the operator for its next solve (no rqutils counterpart: XLA caches its
 *  compiled loop per shape): 8 vectors of dtype, plus 8 FP32 ones after a mixed solve, held
 *  until sqd_op_destroy; they are rebuilt when lanes, chunk, layout or coefficients change. */
int sqd_locg(int64_t n, int dtype, sqd_matvec_fn fn, void* ctx, const void* xinit,
             int64_t xinit_index, const void* const* orth, int n_orth, double tol, int maxiter,
             int mode, int use_graph, void* stream, double* eigval_host, void* eigvec,
             int* niter_host, double* residual_host);

/* eigenpair_2x2 / eigenpair_3x3 (ground_locg.py:467-514): the lowest eigenpair of each of
 * `count` Hermitian dim x dim matrices (dim 2: closed form; dim 3: Cardano's method after Kopp
 * 2008, eigenvector from a cross product), with the device routines the solver's Rayleigh-Ritz
 * steps use.  mats: complex128 row-major [count, dim, dim]; vals: [count] doubles; vecs:
 * complex128 [count, dim].  Stream-ordered; no synchronization. */
int sqd_eigenpair_small(const void* mats, int64_t count, int dim, double* vals, void* vecs,
                        void* stream);

/* Per-iteration record of the NEXT sqd_locg call on the calling thread: the values behind the
 * reference's log_level <= DEBUG prints (ground_locg.py:330-331, 377-378).  After that call
 * returns, rows_host holds *count_host rows (at most max_rows) of 6 doubles: phase (0 = FP64
 * iteration, 1 = FP32 sweep of the mixed solver, which come first), iteration number, theta,
 * |r|, reltol = (|Ax| - theta) * 10 n (FP32 sweeps: their stopping threshold
 * 2e-7 |theta|), converged (0/1).  Recording costs one store per iteration.  rows_host = NULL
 * or max_rows = 0 cancels a pending request. */
int sqd_locg_record(double* rows_host, int64_t max_rows, int64_t* count_host);

/* ---------------------------------------------------------------- batched instances -------- */
/* Many independent SQD problems solved together (no rqutils counterpart: rqutils solves one
 * subspace per call).  The operators' stored pairs (cache_strategy (1, 2) required) are copied
 * into one block-diagonal operator; the operators may be destroyed afterwards. */
int sqd_batch_create(const sqd_op_t* ops, int n_ops, void* stream, sqd_batch_t* out);
int sqd_batch_info(sqd_batch_t b, int64_t* total_rows, int64_t* total_pairs);
int sqd_batch_set_lanes(sqd_batch_t b, int precision, int lanes_per_row);
/* Mixed-precision LOCG (as SQD_LOCG_MIXED of sqd_locg) for every instance at once: FP32 sweeps
 * then FP64 iterations until each instance meets the reference's residual test with `tol`
 * (< 0: dtype epsilon).  Start vectors: xinit (device, concatenated, dtype) or, if NULL,
 * one-hot vectors at xinit_index_host[i] (local row of instance i).  Outputs per instance:
 * eigvals_host[n], niters_host[n], residuals_host[n] (may be NULL); eigvecs concatenated. */
int sqd_batch_locg(sqd_batch_t b, int dtype, const void* xinit, const int64_t* xinit_index_host,
                   double tol, int maxiter, int use_graph, void* stream, double* eigvals_host,
                   void* eigvecs, int* niters_host, double* residuals_host);
void sqd_batch_destroy(sqd_batch_t b);

#ifdef __cplusplus
}
#endif

#endif /* SQD_B200_H */
