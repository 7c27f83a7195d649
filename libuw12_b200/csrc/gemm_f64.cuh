// FP64 tensor-core GEMM engine for sm_100a.
//
// Blackwell's tcgen05 has no FP64 kind, so FP64 contractions run on the
// double-precision MMA path (mma.sync.aligned.m16n8k4 .f64).  One kernel
// covers every contraction of the UW12 schedule:
//
//   C[bo] = alpha * sum_{r1,r2} op(A)[bo,r] * op(B)[bo,r] + beta * C[bo]
//
// with arbitrary m, n, k, leading dimensions and element offsets, 2-D output
// batches (bo1, bo2) and 2-D reduction batches (r1, r2): the latter is how the
// reference's orbital-pair loops (parallel_sum_2d over (j,k) of N x N
// products) become a single launch.  Split-K partitions the flattened
// (reduction batch, k-tile) space across CTAs when the output has too few
// tiles to fill 148 SMs; partial tiles go to a workspace reduced in a fixed
// order (deterministic).
#pragma once

#include "common.cuh"
#include <string>

namespace uw12b {

struct GemmDesc {
  long long m = 0, n = 0, k = 0;
  // A is m x k: element (i, kk) at A[i + lda*kk] (a_kcontig=false) or A[kk + lda*i].
  const double* A = nullptr;
  long long lda = 0;
  bool a_kcontig = false;
  // B is k x n: element (kk, j) at B[kk + ldb*j] (b_ncontig=false) or B[j + ldb*kk].
  const double* B = nullptr;
  long long ldb = 0;
  bool b_ncontig = false;
  // C is m x n column-major.
  double* C = nullptr;
  long long ldc = 0;
  double alpha = 1.0, beta = 0.0;
  // output batches
  long long nbo1 = 1, nbo2 = 1;
  long long sAo1 = 0, sAo2 = 0, sBo1 = 0, sBo2 = 0, sCo1 = 0, sCo2 = 0;
  // reduction batches (summed into the same C)
  long long nbr1 = 1, nbr2 = 1;
  long long sAr1 = 0, sAr2 = 0, sBr1 = 0, sBr2 = 0;
  int split = 0;  // 0: automatic
};

// Launches on current_stream().  Zero-sized problems are no-ops (k == 0 or
// no reduction batches scales C by beta).  While split precision is selected
// on this host thread (set_split_moduli), GEMMs of at least kOzakiMinFlops
// run as split-precision int8 tensor-core GEMMs (ozaki.cuh); gemm_dmma always
// runs the FP64 DMMA kernel.
void gemm(const GemmDesc& d);
void gemm_dmma(const GemmDesc& d);

// Same contraction without any device allocation: split-K partial tiles go
// to a fixed per-device array of kNoAllocScratchDoubles doubles (16 MiB).  An
// explicit split > 1 whose partials (split * batches * m * n doubles) exceed it
// is rejected; an automatic split is reduced until they fit.  The array is
// shared by all calls: calls that overlap on the GPU race.  The first call on
// a device looks up the array's device address (once per device).
constexpr long long kNoAllocScratchDoubles = 1LL << 21;
void gemm_noalloc(const GemmDesc& d);

// Split-K autotuner of gemm_dmma (off by default).  Mode 0: the wave
// heuristic; 1: tune -- the first automatic-split GEMM with beta = 0 of a shape
// class (output CTAs, power-of-two bucket of the k tiles) not yet in the table
// is timed with every candidate split and the fastest recorded; 2: use the
// table only.  In modes 1 and 2 automatic splits come from the table when it
// has the class.  autotune_set also merges a table saved by autotune_save
// (text, one "output_ctas k_tile_bucket split ms" line per class) when `path`
// names an existing file; a malformed file throws.  The table is process-wide.
void autotune_set(int mode, const char* path);
void autotune_save(const char* path);
void autotune_clear();
long long autotune_size();
// the table's split for a GEMM of this shape (0: the class is not in it)
int autotune_lookup(long long m, long long n, long long k, long long nbo, long long nbr);

// Convenience wrappers in BLAS terms (column-major, 'N'/'T').
inline GemmDesc gemm_nn(long long m, long long n, long long k, double alpha, const double* A,
                        long long lda, const double* B, long long ldb, double beta, double* C,
                        long long ldc) {
  GemmDesc d;
  d.m = m; d.n = n; d.k = k; d.alpha = alpha; d.beta = beta;
  d.A = A; d.lda = lda; d.B = B; d.ldb = ldb; d.C = C; d.ldc = ldc;
  return d;
}

// Per-kernel-class timing (CUDA events around every launch) for roofline
// reporting.  Disabled by default.
struct KernelStats {
  unsigned long long launches = 0;
  double ms = 0.0;
  double flops = 0.0;  // algorithmic 2*m*n*k per launch
};
void profile_enable(bool on);
bool profile_enabled();
KernelStats profile_read_gemm();  // synchronises the recorded events
void profile_reset();
// Kernel classes: the FP64 DMMA GEMM; whole split-precision GEMMs (work =
// FP64-equivalent 2mnk FLOPs); their int8 tcgen05 product kernel (work = int8
// operations 2 m n K per modulus); their operand preparation and CRT
// reconstruction kernels (work = algorithmic bytes read + written); the
// three-index producers of integral-direct handles (work = bytes produced).
enum {
  kProfDgemm = 0,
  kProfSplitGemm,
  kProfI8Mma,
  kProfSplitPrep,
  kProfSplitCrt,
  kProfProducer,
  kProfKinds
};
KernelStats profile_read_kind(int kind);
// Adds one timed launch (the events are destroyed once read).
void profile_record(int kind, cudaEvent_t a, cudaEvent_t b, double work, std::string shape);

}  // namespace uw12b
