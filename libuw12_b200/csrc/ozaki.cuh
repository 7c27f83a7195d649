// Split-precision FP64 GEMM on the int8 tensor cores (tcgen05.mma kind::i8).
//
// Emulates C = alpha * sum_r op(A_r) op(B_r) + beta * C (the GemmDesc
// contract of gemm_f64.cuh) with the modular-integer scheme of Ozaki,
// Uchino and Imamura ("Ozaki scheme II", 2024):
//   1. every row i of A and column j of B is scaled by a power of two and
//      rounded to an integer of at most beta bits (A' = rint(A 2^sa_i),
//      B' = rint(B 2^sb_j)), beta chosen so that |A'B'| < M/4;
//   2. for each of L pairwise-coprime moduli p_l <= 256 (M = prod p_l) the
//      residues A' mod p_l and B' mod p_l are int8 matrices and their
//      product is exact in int32 (K split into chunks of <= 65536);
//   3. the Chinese remainder theorem rebuilds the integer A'B' exactly from
//      the L residue products (FP64 arithmetic on <= 41-bit chunks), whose
//      error-free sum gives A'B' to within one unit in the last place (exactly
//      when it is a double), and C = 2^-(sa_i + sb_j) A'B' (products of
//      small-integer matrices come out exact).
// The only error is the rounding of A and B to beta bits relative to the
// largest element of their row / column: |dC_ij| <= 2^-beta (max|a_i.| sum_k
// |b_kj| + max|b_.j| sum_k |a_ik|) (beta = 48 for L = 14, K = 1500).
#pragma once

#include "gemm_f64.cuh"

namespace uw12b {

constexpr int kOzakiMaxModuli = 16;
// The modulus count of FP64-level accuracy (about 48 bits kept per operand
// element at K = 1500); its residue and CRT kernels are compiled with the
// moduli loop fully unrolled and unguarded.
constexpr int kOzakiDefaultModuli = 14;

// Number of moduli of the split-precision GEMMs of this host thread
// (0 = plain FP64 DMMA GEMMs).  gemm() routes GEMMs of at least
// kOzakiMinFlops FLOPs here while it is non-zero.
void set_split_moduli(int n_moduli);
int split_moduli();
constexpr double kOzakiMinFlops = 2e9;
// Smallest GEMM (FLOPs) routed to the split-precision path on this host
// thread (default kOzakiMinFlops; GEMMs above it also have to pass
// ozaki_profitable).  0 routes every GEMM, whatever its shape.
void set_split_min_flops(double flops);
double split_min_flops();

// The split-precision GEMM with n_moduli moduli (1..16).
void gemm_ozaki(const GemmDesc& d, int n_moduli);
// Shapes the split-precision kernels take (K <= 8.4M, m, n <= 2^30).
bool ozaki_supported(const GemmDesc& d);
// Whether the split path with n_moduli moduli is expected to beat the FP64
// path (a cost model of operand preparation, int8 products and CRT against
// the FP64 GEMM).
bool ozaki_profitable(const GemmDesc& d, int n_moduli);

// beta (bits kept per operand element) for n_moduli moduli and a contraction
// of k_total terms.
int ozaki_bits(int n_moduli, long long k_total);

// Device flag set by a split-precision GEMM kernel whose pipeline wait timed
// out; read_and_clear returns it (0 = none) and resets it (synchronises the
// current stream).
int ozaki_error_read_and_clear();
// Error-flag slot of the calling host thread (0 .. kOzakiErrorSlots-1);
// returns the previous slot.  Threads that evaluate concurrently use
// different slots so that each reads and clears only its own kernels' flag.
constexpr int kOzakiErrorSlots = 64;
int set_error_slot(int slot);

}  // namespace uw12b
