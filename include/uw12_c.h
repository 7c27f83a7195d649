/*
 * uw12_c.h -- C-ABI of the B200-native UW12 energy + Fock library.
 *
 * Plain pointers and sizes only.  Every entry point returns a status code
 * (UW12C_OK on success); the message of the last failure on the calling host
 * thread is available through uw12c_last_error().  Status codes map onto the
 * exception classes libuw12 throws: UW12C_ERR_RUNTIME <-> std::runtime_error
 * (user-input errors), UW12C_ERR_LOGIC <-> std::logic_error (shape errors).
 *
 * Layouts are libuw12's (column-major throughout):
 *   X3     packed three-index integrals (rho sigma|A): n_ao(n_ao+1)/2 x n_df,
 *          row i(i+1)/2 + j holds the pair (i, j <= i);
 *   X2     two-index metric (A|B): n_df x n_df;
 *   X3_ri  three-index RI integrals (mu rho|A): (n_ri * n_ao) x n_df, row
 *          nu + n_ri * mu;
 *   S      overlap of the combined AO+RI space, AO functions first;
 *   C      orbitals n_ao x (n_orb * n_spin), alpha columns then beta;
 *   occ    occupations packed alpha || beta;
 *   fock   n_ao x (n_ao * n_spin), spin blocks side by side.
 * All compute runs on the current CUDA device; there is no CPU fallback.
 */
#ifndef UW12_C_H
#define UW12_C_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define UW12C_OK 0
#define UW12C_ERR_RUNTIME 1
#define UW12C_ERR_LOGIC 2
#define UW12C_ERR_CUDA 3
#define UW12C_ERR_ALLOC 4
#define UW12C_ERR_INVALID 5

#define UW12C_MEM_HOST 0
#define UW12C_MEM_DEVICE 1

typedef struct uw12c_integrals uw12c_integrals;
typedef struct uw12c_abs uw12c_abs;

/* Status of the last call on this host thread; copies its message into buf
 * (truncated, NUL-terminated) when buf != NULL. */
int uw12c_last_error(char* buf, size_t len);

/* Library version string (static storage). */
const char* uw12c_version(void);

/* Replaces uw12::setup_base_integrals(X3, X2, X3_ri, n_ao, n_df, n_ri, copy)
 * (libuw12.hpp:42-50, libuw12.cpp:22-36) and, with X3_ri == NULL, the no-RI
 * overload (libuw12.hpp:64-70, libuw12.cpp:38-49).  The tensors are copied to
 * the device (mem_kind says where the caller's pointers live) and the metric
 * is diagonalised there: P2 = Q pinv(Lambda), df_vals = Lambda
 * (src/integrals/base_integrals.cpp:155-166). */
int uw12c_integrals_create(const double* X3, const double* X2, const double* X3_ri, size_t n_ao,
                           size_t n_df, size_t n_ri, int mem_kind, uw12c_integrals** out);
/* Replaces the BaseIntegrals(J3, df_vals) constructor
 * (src/integrals/base_integrals.hpp:104, base_integrals.cpp:308-326):
 * three-index integrals already in the metric eigenbasis (J3 = J3_0 P2,
 * n_ao(n_ao+1)/2 x n_df) and their eigenvalues; no RI. */
int uw12c_integrals_create_eigenbasis(const double* J3, const double* df_vals, size_t n_ao,
                                      size_t n_df, int mem_kind, uw12c_integrals** out);
/* A producer of three-index integrals: writes aux functions [first, first +
 * count) as the columns of out (leading dimension ld >= the tensor's rows:
 * n_ao(n_ao+1)/2 packed AO rows, or n_ri*n_ao RI rows) and returns 0, or
 * non-zero on failure.  For device producers out is device memory and the
 * work goes on the CUDA stream `stream` (a cudaStream_t); for host producers
 * out is host memory. */
typedef int (*uw12c_block_fn)(void* user, size_t first, size_t count, double* out, size_t ld,
                              void* stream);
/* Replaces the BaseIntegrals(two_index_fn, three_index_fn, three_index_ri_fn,
 * df_sizes, n_ao, n_df, n_ri, store_ao_integrals, store_ri_integrals)
 * constructors (src/integrals/base_integrals.hpp:52-72,
 * base_integrals.cpp:40-186).  X2 is the metric (n_df x n_df); the
 * three-index tensors come from the producers, each called with its own user
 * pointer (three_index_ri may be NULL: no RI).  A stored tensor is produced once, during this call, and kept on the
 * device; an unstored one (integral-direct mode) is produced again, in aux
 * blocks, at every use, so inputs larger than device memory can be evaluated;
 * the user data must then outlive the handle, and the producers may be called from
 * several host threads (batched evaluations).  x2_mem_kind says where X2
 * lives, block_mem_kind where the producers' out buffers are (device memory:
 * device producers; host memory: staged through pinned memory). */
int uw12c_integrals_create_callback(const double* X2, int x2_mem_kind,
                                    uw12c_block_fn three_index, void* user,
                                    uw12c_block_fn three_index_ri, void* user_ri, size_t n_ao,
                                    size_t n_df, size_t n_ri, int store_ao, int store_ri,
                                    int block_mem_kind, uw12c_integrals** out);
int uw12c_integrals_destroy(uw12c_integrals* h);
/* BaseIntegrals::get_number_ao/df/ri (src/integrals/base_integrals.hpp:196-202). */
int uw12c_integrals_dims(const uw12c_integrals* h, size_t* n_ao, size_t* n_df, size_t* n_ri);
/* BaseIntegrals::get_df_vals (src/integrals/base_integrals.hpp:169): n_df values, host. */
int uw12c_integrals_df_vals(const uw12c_integrals* h, double* out);

/* Replaces uw12::setup_abs_projectors(S, n_ao, n_ri) (libuw12.hpp:80,
 * libuw12.cpp:51-56 -> src/three_electron/ri_utils.hpp:45-74). */
int uw12c_abs_create(const double* S, size_t n_ao, size_t n_ri, int mem_kind, uw12c_abs** out);
int uw12c_abs_destroy(uw12c_abs* h);
/* The four ABSProjectors blocks (ri_utils.hpp:20-29) copied to host buffers
 * (any may be NULL): ri_ri R x R, ri_ao R x N, ao_ri N x R, ao_ao N x N. */
int uw12c_abs_blocks(const uw12c_abs* h, double* ri_ri, double* ri_ao, double* ao_ri,
                     double* ao_ao);

/* Replaces uw12::form_fock (src/uw12.hpp:129-142, src/uw12.cpp:22-119) with
 * per-spin orbital blocks: C_alpha (n_ao x n_orb[0]) and, for n_spin == 2,
 * C_beta, each with leading dimension ldc[s]; occ[s] holds n_occ[s]
 * occupations.  energy receives the total, terms (may be NULL) the two-,
 * three- and four-electron energies, fock (may be NULL) the Fock matrix. */
int uw12c_form_fock(const uw12c_integrals* W, const uw12c_integrals* V,
                    const uw12c_integrals* WV, const uw12c_abs* abs, size_t n_ao, size_t n_spin,
                    const double* const* C, const size_t* ldc, const size_t* n_orb,
                    const double* const* occ, const size_t* n_occ, const size_t* n_active,
                    int indirect_term, int calculate_fock, double scale_opp_spin,
                    double scale_same_spin, size_t print_level, double* energy, double* terms,
                    double* fock, int fock_mem_kind);

/* One molecule of a batched evaluation: the arguments of uw12c_form_fock. */
typedef struct uw12c_molecule {
  const uw12c_integrals* W;
  const uw12c_integrals* V;
  const uw12c_integrals* WV;
  const uw12c_abs* abs;
  size_t n_ao, n_spin;
  const double* const* C;
  const size_t* ldc;
  const size_t* n_orb;
  const double* const* occ;
  const size_t* n_occ;
  const size_t* n_active;
  double* energy; /* host scalar */
  double* terms;  /* host [3] or NULL */
  double* fock;   /* n_ao x (n_ao n_spin) or NULL */
  int fock_mem_kind;
} uw12c_molecule;

/* Evaluates n molecules of any sizes (no counterpart in libuw12, which takes
 * one system per call): uw12c_form_fock for each, with n_streams host worker
 * threads (0 = 8; the calling thread is one of them), each with its own
 * CUDA stream and an equal share of the memory budget, taking molecules
 * largest first, so that the evaluations of small molecules overlap on the
 * GPU.  The calling thread's split-precision settings apply to every
 * molecule.  statuses (n entries, may be NULL) receives each molecule's
 * status; the call returns the first failure. */
int uw12c_fock_batched(const uw12c_molecule* mols, size_t n, int indirect_term,
                       int calculate_fock, double scale_opp_spin, double scale_same_spin,
                       size_t n_streams, int* statuses);

/* Reverse mode of uw12c_form_fock (no counterpart in libuw12): the energy,
 * terms and Fock (dE/dD) of uw12c_form_fock with the same arguments plus the
 * gradient of that energy with respect to the stored integrals.
 * indirect_term = 0 differentiates the direct terms only (scale_same_spin
 * entering the direct same-spin pairs); indirect_term = 1 with
 * scale_same_spin != 0 adds the same-spin (exchange) energies of the two-,
 * three- and four-electron terms, i.e. the energy of uw12c_fock /
 * uw12_energy (libuw12.cpp:138 runs them when |scale_same_spin| > 4 eps).
 *   dE_dX3[3]    W, V, WV: packed n_ao(n_ao+1)/2 x n_df, entry (mn|P) of the
 *                packed storage (both triangle halves of sq(X3[:,P]) summed);
 *   dE_dX3_ri[2] W, V: (n_ri n_ao) x n_df, the X3_ri layout;
 *   dE_dX2[3]    W, V, WV: n_df x n_df symmetric (-J2^-1 G J2^-1; exact while
 *                no metric eigenvalue is below the 1e-10 pseudo-inverse cut).
 * Any array, or any of its entries, may be NULL (that gradient is skipped);
 * grad_mem_kind says where the gradient buffers live.  The intermediates of the
 * forward pass are recomputed, not kept between calls. */
int uw12c_fock_backward(const uw12c_integrals* W, const uw12c_integrals* V,
                        const uw12c_integrals* WV, const uw12c_abs* abs, size_t n_ao,
                        size_t n_spin, const double* const* C, const size_t* ldc,
                        const size_t* n_orb, const double* const* occ, const size_t* n_occ,
                        const size_t* n_active, int indirect_term, double scale_opp_spin,
                        double scale_same_spin,
                        double* energy, double* terms, double* fock, int fock_mem_kind,
                        double* const* dE_dX3, double* const* dE_dX3_ri, double* const* dE_dX2,
                        int grad_mem_kind);

/* A consumer of a three-index gradient in blocks (no counterpart in libuw12):
 * receives aux functions [first, first + count) as the columns of `block`
 * (leading dimension ld = the tensor's rows) and returns 0, or non-zero on
 * failure.  Device blocks may be read by work the sink enqueues on the CUDA
 * stream `stream` (a cudaStream_t) before it returns; later work on that
 * stream may overwrite them.  Host blocks are valid until the sink returns. */
typedef int (*uw12c_block_sink)(void* user, size_t first, size_t count, const double* block,
                                size_t ld, void* stream);
/* uw12c_fock_backward with the three-index gradients handed to sinks in aux
 * blocks instead of written to whole buffers (no counterpart in libuw12): a
 * gradient as large as an unstored (integral-direct) tensor is never held
 * whole on the device.  sink3[3] (W, V, WV; packed rows) and sink3_ri[2] (W,
 * V; RI rows), each with its user pointer, any entry NULL to skip that
 * gradient; block_mem_kind UW12C_MEM_DEVICE passes device blocks,
 * UW12C_MEM_HOST host blocks (staged through pinned memory, at most 256 MiB
 * per call).  Every aux function of a requested gradient is delivered once,
 * in increasing order.  The metric gradients go to dE_dX2 as in
 * uw12c_fock_backward. */
int uw12c_fock_backward_blocks(const uw12c_integrals* W, const uw12c_integrals* V,
                               const uw12c_integrals* WV, const uw12c_abs* abs, size_t n_ao,
                               size_t n_spin, const double* const* C, const size_t* ldc,
                               const size_t* n_orb, const double* const* occ,
                               const size_t* n_occ, const size_t* n_active,
                               int indirect_term, double scale_opp_spin,
                               double scale_same_spin, double* energy, double* terms,
                               double* fock, int fock_mem_kind,
                               const uw12c_block_sink* sink3, void* const* user3,
                               const uw12c_block_sink* sink3_ri, void* const* user3_ri,
                               int block_mem_kind, double* const* dE_dX2, int grad_mem_kind);
/* A device sink for uw12c_fock_backward_blocks that adds the sum of squares
 * of every block it receives to the double at `user` (device memory, on the
 * library's stream): the squared Frobenius norm of a streamed gradient. */
int uw12c_sink_norm2(void* user, size_t first, size_t count, const double* block, size_t ld,
                     void* stream);

/* Replaces uw12::uw12_fock(double* fock, ...) (libuw12.hpp:157-169,
 * libuw12.cpp:184-214) in its raw-pointer form: C is the setup_orbitals
 * buffer (n_ao x n_orb*n_spin), occ the setup_occupations buffer
 * (n_occ_alpha [+ n_occ_beta] values; n_occ_beta ignored for n_spin == 1),
 * n_active has n_spin entries.  The same-spin term runs when
 * |scale_same_spin| > 4 DBL_EPSILON (libuw12.cpp:138). */
int uw12c_fock(double* fock, const uw12c_integrals* W, const uw12c_integrals* V,
               const uw12c_integrals* WV, const uw12c_abs* abs, const double* C, size_t n_ao,
               size_t n_orb, size_t n_spin, const double* occ, size_t n_occ_alpha,
               size_t n_occ_beta, const size_t* n_active, double scale_opp_spin,
               double scale_same_spin, size_t print_level, double* energy);

/* Replaces uw12::uw12_energy (libuw12.hpp:129-140, libuw12.cpp:156-182). */
int uw12c_energy(const uw12c_integrals* W, const uw12c_integrals* V, const uw12c_integrals* WV,
                 const uw12c_abs* abs, const double* C, size_t n_ao, size_t n_orb, size_t n_spin,
                 const double* occ, size_t n_occ_alpha, size_t n_occ_beta,
                 const size_t* n_active, double scale_opp_spin, double scale_same_spin,
                 size_t print_level, double* energy);

/* Execution control (no counterpart in libuw12, whose calls are synchronous
 * CPU code): the CUDA stream (a cudaStream_t, NULL = legacy default) used by
 * this host thread, the byte budget for chunked intermediates (0 = 45% of free
 * device memory), and counters of this library's kernel launches and of the
 * FP64 GEMM kernel's time and FLOPs (events recorded around each launch while
 * profiling is on). */
int uw12c_set_stream(void* stream);
int uw12c_set_memory_budget(size_t bytes);
/* Splits the following evaluations of this host thread into n_shards parts
 * and computes part `shard` only (no counterpart in libuw12; one GPU per
 * shard).  Aux functions are dealt out in contiguous, balanced ranges: the
 * fitted densities, the MO transforms of the three-index tensors (W, V, WV)
 * and the 2-el Fock run over this shard's aux range, and their partial sums
 * are completed by the all-reduce hook (uw12c_set_allreduce) before use; the
 * t~ dX Fock term runs over this shard's range of W's aux functions.  The
 * occupied orbitals are dealt out likewise: X_AB and t (their M x M partials
 * all-reduced), the direct Fock and the same-spin three-electron energy and
 * Fock.  The remaining small terms (the energies built from the reduced
 * intermediates, the same-spin 2-el and 4-el terms) come from shard 0.
 * Energies and Fock matrices of the n_shards parts sum to the full result
 * (the caller's final all-reduce).  uw12c_set_shard(0, 1) restores full
 * evaluations; the adjoint evaluates unsharded. */
int uw12c_set_shard(size_t shard, size_t n_shards);
/* The all-reduce of sharded evaluations on this host thread: fn(data, count,
 * stream, user) must replace the `count` doubles at device pointer `data` by
 * their sum over the shards, ordered after the work already queued on
 * `stream` (a cudaStream_t) and before any work queued on it afterwards, and
 * return 0 (non-zero fails the evaluation).  Every shard calls it at the same
 * points with the same counts.  fn = NULL removes it; a sharded evaluation
 * without one fails with UW12C_ERR_INVALID.  (torch.distributed.all_reduce over
 * NCCL on the given stream is one such function: libuw12_b200.distributed.) */
typedef int (*uw12c_allreduce_fn)(double* data, size_t count, void* stream, void* user);
int uw12c_set_allreduce(uw12c_allreduce_fn fn, void* user);
/* The library keeps device memory freed by one call reserved for the next
 * (its own stream-ordered pool); this returns the unused part to the system. */
int uw12c_trim_memory(void);
unsigned long long uw12c_launch_count(void);
int uw12c_profile_enable(int on);
int uw12c_profile_read(unsigned long long* gemm_launches, double* gemm_ms, double* gemm_flops);
/* Device time per phase of the evaluation accumulated while profiling is on,
 * as "phase=milliseconds;..." (truncated to len); reading resets it. */
int uw12c_profile_phases(char* buf, size_t len);

/* The FP64 tensor-core GEMM engine on device pointers (no counterpart in
 * libuw12, which calls BLAS dgemm through Armadillo):
 *   C[bo] = alpha * sum_{r1<nbr1, r2<nbr2} op(A) op(B) + beta * C[bo],
 * A m x k with element (i, kk) at A[i + lda*kk] (a_kcontig = 0) or
 * A[kk + lda*i]; B k x n with (kk, j) at B[kk + ldb*j] (b_ncontig = 0) or
 * B[j + ldb*kk]; C column-major.  Output batch (bo1 < nbo1, bo2 < nbo2)
 * offsets A/B/C by so = {sAo1, sAo2, sBo1, sBo2, sCo1, sCo2}; reduction batch
 * (r1, r2) offsets A/B by sr = {sAr1, sAr2, sBr1, sBr2}.  split = 0 chooses
 * split-K automatically. */
int uw12c_dgemm(long long m, long long n, long long k, double alpha, const double* A,
                long long lda, int a_kcontig, const double* B, long long ldb, int b_ncontig,
                double beta, double* C, long long ldc, long long nbo1, long long nbo2,
                const long long* so, long long nbr1, long long nbr2, const long long* sr,
                int split);

/* uw12c_dgemm for callers that cannot allocate device memory (no counterpart
 * in libuw12).  Host programs that reserve the whole device heap for their own
 * memory pool at start-up, and code paths where a cudaMalloc/cudaFree would
 * fail or synchronise the device (cudaFree waits for all streams), cannot let
 * the library allocate; this entry point allocates nothing.  The caller still
 * passes A, B and C.  Split-K partial tiles go to one fixed device array of
 * UW12C_NOALLOC_SCRATCH_DOUBLES doubles (16 MiB) that every device which
 * loads the library keeps until the process exits.  An explicit split > 1
 * whose partials (split * nbo1 * nbo2 * m * n doubles) do not fit is rejected
 * with UW12C_ERR_INVALID; split = 0 chooses a split that fits (1 needs no
 * scratch).  All calls share the array, so calls that overlap on the GPU
 * race; the partial tiles are fully overwritten by each call, so nothing has
 * to start at zero.  The first call on a device looks up the array's device
 * address (once per device); make that first call before any stream capture.
 * With lazy module loading (the CUDA default since 12.2) that first call also
 * loads the library's device code and the array, which takes device memory:
 * make it before the host program reserves the heap for its pool.  This entry
 * point always computes in FP64 (the DMMA kernel): the split-precision mode of
 * uw12c_set_precision does not apply to it. */
#define UW12C_NOALLOC_SCRATCH_DOUBLES (1LL << 21)
int uw12c_dgemm_noalloc(long long m, long long n, long long k, double alpha, const double* A,
                        long long lda, int a_kcontig, const double* B, long long ldb,
                        int b_ncontig, double beta, double* C, long long ldc, long long nbo1,
                        long long nbo2, const long long* so, long long nbr1, long long nbr2,
                        const long long* sr, int split);

/* Split precision (no counterpart in libuw12, which computes in FP64 only).
 * uw12c_set_precision(L) makes the following evaluations of this host thread
 * run every GEMM of at least 2e9 FLOPs as a split-precision GEMM with L
 * moduli (1..16; 0 = FP64 DMMA GEMMs, the default): each FP64 row of A and
 * column of B is scaled by a power of two and rounded to an integer of beta
 * bits, its residues modulo L coprime moduli <= 256 are multiplied exactly as
 * int8 matrices on the tensor cores (int32 accumulation), and the Chinese
 * remainder theorem rebuilds the FP64 product.  The error of one GEMM is at
 * most 2^-beta (max|a_i.| sum_k |b_kj| + max|b_.j| sum_k |a_ik|) per element;
 * uw12c_split_bits gives beta for L moduli and a contraction of k_total terms
 * (48 bits for L = 14, k_total = 1500).  The metric and overlap
 * eigensolves, energy reductions and Fock symmetrisation stay FP64. */
int uw12c_set_precision(int n_moduli);
/* GEMMs below min_flops stay FP64 in split-precision mode (default 2e9), and
 * so do those whose estimated operand preparation, int8 products and
 * reconstruction would not beat the FP64 product (thin or short ones); 0
 * routes every GEMM through the split path. */
int uw12c_set_split_threshold(double min_flops);
int uw12c_split_bits(int n_moduli, long long k_total, int* bits);
/* uw12c_dgemm computed by the split-precision GEMM with n_moduli moduli. */
int uw12c_dgemm_split(long long m, long long n, long long k, double alpha, const double* A,
                      long long lda, int a_kcontig, const double* B, long long ldb, int b_ncontig,
                      double beta, double* C, long long ldc, long long nbo1, long long nbo2,
                      const long long* so, long long nbr1, long long nbr2, const long long* sr,
                      int n_moduli);
/* Timing of a kernel class while profiling is on: 0 FP64 DMMA GEMM (work =
 * FLOPs), 1 whole split-precision GEMMs (FP64-equivalent FLOPs), 2 their int8
 * tensor-core kernel (int8 operations), 3 their operand preparation and 4
 * their CRT reconstruction (bytes read + written), 5 the three-index producer
 * calls of integral-direct handles (bytes produced; device time on the
 * library's stream, host producers' staging included). */
int uw12c_profile_read_kind(int kind, unsigned long long* launches, double* ms, double* work);

/* Split-K autotuner of the FP64 GEMM engine (no counterpart in libuw12, which
 * leaves its BLAS to choose its own blocking).  The engine splits the
 * contraction of a GEMM whose output has too few tiles to fill the GPU; by
 * default a wave-occupancy rule picks the split.  mode 1 (tune): the first
 * GEMM with beta = 0 and an automatic split of each shape class (output CTA
 * count, power-of-two bucket of the k tiles over all reduction batches; output
 * CTA counts of at least 8 waves never split) is launched once with each
 * candidate split (1 .. 64, at least 4 k tiles per part, split-K partials
 * within 256 MiB or the rule's own), each timed on the
 * library's stream, which synchronises it; the fastest is recorded and the
 * GEMM's result is that of a launch with it.  mode 2 (use): the table's split
 * for every class it has, the rule otherwise, no timing.  mode 0: the rule
 * (default).  When path names an existing file (written by
 * uw12c_autotune_save: a comment line, then "output_ctas k_tile_bucket split
 * ms" per class) its classes are merged into the table first; a malformed file
 * is UW12C_ERR_INVALID.  The table and the mode are process-wide and apply to
 * every thread and device; tune on one device of the kind that will use the
 * table, with one evaluation at a time (timings overlapped by other work are
 * not representative).  Splits change the summation order only: results agree
 * to rounding with the rule's.  uw12c_dgemm_noalloc and the int8 products of
 * split precision do not use the table (GEMMs that split precision leaves in
 * FP64 do). */
int uw12c_autotune(int mode, const char* path);
int uw12c_autotune_save(const char* path);
int uw12c_autotune_clear(void);
int uw12c_autotune_size(long long* n_classes);
/* The table's split for a GEMM of this shape (0: its class is not in the table). */
int uw12c_autotune_lookup(long long m, long long n, long long k, long long nbo, long long nbr,
                          int* split);

/* Deterministic synthetic three-index tensors written on the device (no
 * counterpart in libuw12; benchmark input generation).  Element e of the
 * stream (seed, tag) is the Box-Muller normal of two SplitMix64 draws, times
 * exp(-|p - q| / decay) for the element's index pair (p, q).
 * kind 0: packed AO tensor n_ao(n_ao+1)/2 x n_df; kind 1: RI tensor
 * (n_ri*n_ao) x n_df. */
int uw12c_synth_three_index(double* out_device, int kind, size_t n_ao, size_t n_ri, size_t n_df,
                            unsigned long long seed, unsigned long long tag, double decay);
/* The same tensors as a device producer for uw12c_integrals_create_callback
 * (user = a uw12c_synth_spec*): columns [first, first + count) of the tensor
 * uw12c_synth_three_index writes, generated on the device. */
typedef struct uw12c_synth_spec {
  int kind;
  size_t n_ao, n_ri;
  unsigned long long seed, tag;
  double decay;
} uw12c_synth_spec;
int uw12c_synth_block(void* spec, size_t first, size_t count, double* out, size_t ld,
                      void* stream);

#ifdef __cplusplus
}
#endif

#endif /* UW12_C_H */
