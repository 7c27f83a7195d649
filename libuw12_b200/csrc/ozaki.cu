// Split-precision FP64 GEMM: int8 residue products on the tcgen05 tensor
// cores, recombined by the Chinese remainder theorem (see ozaki.cuh).
//
// Kernels per GEMM (slab):
//   k_row_exponent per row of A / column of B: the binary exponent of its
//                 largest element; rows are scaled by 2^(beta - exponent) so
//                 that every element is below 2^beta in magnitude;
//   k_residues    FP64 -> rint(x 2^shift) -> L int8 residue planes, K-major
//                 (row r of plane (l, p) is K_pad contiguous bytes);
//   k_i8_mma      persistent, one CTA per SM; work item = one 128 x 256
//                 output tile of one modulus and one K chunk: TMA (128-byte
//                 swizzled boxes, 4-stage ring) -> shared memory ->
//                 tcgen05.mma.kind::i8 with the int32 accumulator in TMEM (two
//                 256-column buffers) -> tcgen05.ld -> residue mod p -> uint8
//                 rows in HBM.  Warp roles: 0 TMA producer, 1 TMEM owner + MMA
//                 issuer, 2..5 epilogue (TMEM lane quarter = warp % 4);
//   k_crt         per output element: sum the K-chunk residues mod p, CRT on
//                 <= 41-bit chunks in FP64 (exact integer arithmetic), join the
//                 chunks error-free (TwoSum), scale by 2^-(sa+sb), apply
//                 alpha / beta, store FP64.
// The MMA's M side (TMEM lanes) runs over the output column j (B's n index)
// and its N side over the output row i (A's m index), so that one thread of
// the epilogue owns 256 consecutive i of one column j and the residue planes
// and C are both i-contiguous.
#include <cuda.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <mutex>
#include <string>

#include "ozaki.cuh"

namespace uw12b {

namespace {

// Pairwise-coprime moduli <= 256 (residues fit int8: [-128, 127]).
constexpr uint32_t kModuli[kOzakiMaxModuli] = {256, 255, 253, 251, 247, 241, 239, 233,
                                               229, 227, 223, 217, 211, 199, 197, 193};
// CRT weights are split into nch chunks of cw <= 41 bits: r_l * chunk < 2^49
// and the sum over <= 16 moduli < 2^53, so every chunk sum is exact in FP64.
constexpr int kMaxChunkBits = 41;
constexpr int kMaxChunks = 4;  // 4 x 41 bits >= log2(M) for 16 moduli (~125.3)
constexpr long long kMaxKChunk = 65536;  // |acc| <= 65536 * 128^2 = 2^30 per split

struct Consts {
  int L = 0, nch = 0, cw = 0, beta = 0;
  uint32_t p[kOzakiMaxModuli];
  uint32_t barrett[kOzakiMaxModuli];  // floor(2^32 / p)
  uint32_t off[kOzakiMaxModuli];      // multiple of p, >= 2^30
  double pd[kOzakiMaxModuli], inv_p[kOzakiMaxModuli];
  double w[kOzakiMaxModuli][kMaxChunks];  // chunks of (M/p_l) * ((M/p_l)^-1 mod p_l) mod M
  double mc[kMaxChunks];                  // chunks of M
  double inv_m;
  double log2_m;
};

using u128 = unsigned __int128;

long long inv_mod(long long a, long long p) {
  long long t = 0, nt = 1, r = p, nr = a % p;
  while (nr) {
    const long long q = r / nr;
    std::swap(t, nt); nt -= q * t;
    std::swap(r, nr); nr -= q * r;
  }
  if (r != 1) throw Error(kErrInvalid, "split-precision moduli are not coprime");
  return t < 0 ? t + p : t;
}

Consts make_consts(int L) {
  Consts c;
  c.L = L;
  u128 M = 1;
  c.log2_m = 0.0;
  for (int l = 0; l < L; ++l) {
    const uint32_t p = kModuli[l];
    M *= p;
    c.log2_m += std::log2(double(p));
    c.p[l] = p;
    c.barrett[l] = static_cast<uint32_t>((1ULL << 32) / p);
    c.off[l] = static_cast<uint32_t>(((1ULL << 30) + p - 1) / p * p);
    c.pd[l] = double(p);
    c.inv_p[l] = 1.0 / double(p);
  }
  int bits = 0;
  for (u128 t = M; t; t >>= 1) ++bits;
  c.nch = (bits + kMaxChunkBits - 1) / kMaxChunkBits;
  c.cw = (bits + c.nch - 1) / c.nch;
  const int kChunkBits = c.cw;
  const u128 mask = (u128(1) << kChunkBits) - 1;
  for (int l = 0; l < L; ++l) {
    const u128 Ml = M / kModuli[l];
    const long long y = inv_mod(static_cast<long long>(Ml % kModuli[l]), kModuli[l]);
    const u128 w = Ml * u128(y);  // < M: Ml * y < Ml * p_l
    for (int ch = 0; ch < kMaxChunks; ++ch)
      c.w[l][ch] = ch < c.nch ? double(static_cast<uint64_t>((w >> (kChunkBits * ch)) & mask))
                              : 0.0;
  }
  for (int ch = 0; ch < kMaxChunks; ++ch)
    c.mc[ch] = ch < c.nch ? double(static_cast<uint64_t>((M >> (kChunkBits * ch)) & mask)) : 0.0;
  c.inv_m = 1.0 / static_cast<double>(M);
  return c;
}

const Consts& consts_for(int L) {
  static std::once_flag once[kOzakiMaxModuli + 1];
  static Consts table[kOzakiMaxModuli + 1];
  std::call_once(once[L], [&] { table[L] = make_consts(L); });
  return table[L];
}

thread_local int g_split_moduli = 0;
thread_local double g_split_min_flops = kOzakiMinFlops;

// device error flags (a pipeline wait timed out): kOzakiErrorSlots ints per
// device; a host thread uses the slot set by set_error_slot (0 by default), so
// that concurrent evaluations on different threads (uw12c_fock_batched's
// workers) read and clear only their own flag
constexpr int kMaxDevices = 64;
std::mutex g_err_mu;
int* g_err_ptr[kMaxDevices] = {};
thread_local int t_err_slot = 0;

int* err_flag() {
  int dev = 0;
  UW12_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices)
    throw Error(kErrInvalid, "split-precision GEMM: device index beyond 63");
  std::lock_guard<std::mutex> lk(g_err_mu);
  if (!g_err_ptr[dev]) {
    UW12_CUDA(cudaMalloc(reinterpret_cast<void**>(&g_err_ptr[dev]),
                         kOzakiErrorSlots * sizeof(int)));
    UW12_CUDA(cudaMemset(g_err_ptr[dev], 0, kOzakiErrorSlots * sizeof(int)));
  }
  return g_err_ptr[dev] + t_err_slot;
}

// ---------------------------------------------------------------------------
// operand preparation
// ---------------------------------------------------------------------------
// Operand rows: element (row, kt) of plane (p1, p2), kt = kk + k * (r1 + nbr1 r2),
// lives at base + p1*po1 + p2*po2 + row*rs + kk*ks + r1*sr1 + r2*sr2.
struct OperandView {
  const double* base;
  long long rows, k, k_total;
  long long rs, ks, sr1, sr2, nbr1;
  long long po1, po2;
  int np1, np2;
};

// Offsets (kk*ks + r1*sr1 + r2*sr2) of the 128 k of the tile starting at k0
// (-1 beyond k_total), one division per k.
__device__ __forceinline__ void tile_k_offsets(const OperandView& v, long long k0,
                                               long long* koff) {
  if (threadIdx.x < 128) {
    const long long kt = k0 + threadIdx.x;
    long long off = -1;
    if (kt < v.k_total) {
      const long long r = kt / v.k, kk = kt - r * v.k;
      off = kk * v.ks + (r % v.nbr1) * v.sr1 + (r / v.nbr1) * v.sr2;
    }
    koff[threadIdx.x] = off;
  }
}

// Shared-memory tile of 32 rows x 128 k, unpadded, element (r, c) at
// r * 128 + (c ^ ((c >> 4) & 7) ^ (r & 15)).  The swizzle stays inside each
// 16-element group and is a bijection per row; every warp access of the
// kernels below touches all 16 8-byte bank pairs exactly twice (two
// wavefronts for 256 bytes, the minimum): the column fill of 32 rows at one k,
// the row fill of 32 consecutive k, and the compute reads (16 lanes per row,
// lane t at k = 8 t + q for one q).
__device__ __forceinline__ int tile_at(int r, int c) {
  return r * 128 + (c ^ ((c >> 4) & 7) ^ (r & 15));
}

// Loads the 32 x 128 tile (rows row0.., k k0..) of one plane, zeros outside,
// reading along whichever of rows / k is contiguous in memory: 16 asynchronous
// 8-byte copies per thread, all in flight at once (a copy of 0 source bytes
// writes a zero), then waits for them.
template <bool KCONTIG>
__device__ __forceinline__ void load_tile(const OperandView& v, int plane, long long row0,
                                          const long long* koff, double* tile) {
  const double* pb = v.base + (plane % v.np1) * v.po1 + (plane / v.np1) * v.po2;
#pragma unroll
  for (int it = 0; it < 16; ++it) {
    const int e = threadIdx.x + 256 * it;
    const int r = KCONTIG ? (e >> 7) : (e & 31);
    const int c = KCONTIG ? (e & 127) : (e >> 5);
    const long long row = row0 + r;
    const long long ko = koff[c];
    const bool in = row < v.rows && ko >= 0;
    const double* src = in ? pb + row * v.rs + ko : pb;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(
                     static_cast<unsigned>(__cvta_generic_to_shared(&tile[tile_at(r, c)]))),
                 "l"(src), "r"(in ? 8 : 0)
                 : "memory");
  }
  asm volatile("cp.async.commit_group;\n" ::: "memory");
  asm volatile("cp.async.wait_all;\n" ::: "memory");
}

// Per row: exponent e of its largest element (2^(e-1) <= max|x| < 2^e),
// stored as e + 2048 through atomicMax (0 = all zeros).  One block covers 32
// rows x kExpTileK k of one plane (grid: row tiles, k tiles, planes) and reads
// straight into registers, 64 independent loads per thread: KCONTIG (rows
// contiguous along k) lets each warp sweep 4 rows along k, otherwise each warp
// takes every 8th k of all 32 rows (consecutive rows per warp load).
constexpr int kExpTileK = 512;

template <bool KCONTIG>
__global__ void __launch_bounds__(256) k_row_exponent(OperandView v,
                                                      unsigned* __restrict__ eplus) {
  __shared__ long long koff[kExpTileK];
  __shared__ double part[8][33];
  const int plane = blockIdx.z;
  const long long row0 = static_cast<long long>(blockIdx.x) * 32;
  const long long k0 = static_cast<long long>(blockIdx.y) * kExpTileK;
  for (int c = threadIdx.x; c < kExpTileK; c += 256) {
    const long long kt = k0 + c;
    long long off = -1;
    if (kt < v.k_total) {
      const long long r = kt / v.k, kk = kt - r * v.k;
      off = kk * v.ks + (r % v.nbr1) * v.sr1 + (r / v.nbr1) * v.sr2;
    }
    koff[c] = off;
  }
  __syncthreads();
  const double* pb = v.base + (plane % v.np1) * v.po1 + (plane / v.np1) * v.po2;
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  if (KCONTIG) {
#pragma unroll
    for (int rr = 0; rr < 4; ++rr) {
      const long long row = row0 + warp * 4 + rr;
      double mx = 0.0;
      if (row < v.rows) {
        const double* rp = pb + row * v.rs;
#pragma unroll
        for (int t = 0; t < kExpTileK / 32; ++t) {
          const long long ko = koff[lane + 32 * t];
          if (ko >= 0) mx = fmax(mx, fabs(rp[ko]));
        }
      }
      for (int o = 16; o; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
      if (lane == 0 && row < v.rows && mx > 0.0) {
        int e = 0;
        frexp(mx, &e);
        atomicMax(&eplus[plane * v.rows + row], static_cast<unsigned>(e + 2048));
      }
    }
  } else {
    const long long row = row0 + lane;
    double mx = 0.0;
    if (row < v.rows) {
      const double* rp = pb + row * v.rs;
#pragma unroll 16
      for (int t = 0; t < kExpTileK / 8; ++t) {
        const long long ko = koff[warp + 8 * t];
        if (ko >= 0) mx = fmax(mx, fabs(rp[ko]));
      }
    }
    part[warp][lane] = mx;
    __syncthreads();
    if (warp == 0) {
      for (int w = 1; w < 8; ++w) mx = fmax(mx, part[w][lane]);
      if (row < v.rows && mx > 0.0) {
        int e = 0;
        frexp(mx, &e);
        atomicMax(&eplus[plane * v.rows + row], static_cast<unsigned>(e + 2048));
      }
    }
  }
}

// shift = beta - e (0 for an all-zero row).
__global__ void k_exponent_to_shift(const unsigned* __restrict__ eplus, long long n, int beta,
                                    int* __restrict__ shift) {
  const long long t = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t < n) shift[t] = eplus[t] ? beta - (static_cast<int>(eplus[t]) - 2048) : 0;
}

// x 2^e for exponents outside the normal range, out of line: kept off the
// per-element paths (inlined, its branches would run predicated on every
// element).
__device__ __noinline__ double ldexp_slow(double x, int e) { return ldexp(x, e); }

// 2^e as a double for -1022 <= e <= 1023 (exponent bits only).
__device__ __forceinline__ double pow2(int e) {
  return __longlong_as_double(static_cast<long long>(e + 1023) << 52);
}

struct ResidueMods {
  int L;
  int pi[kOzakiMaxModuli];
  double inv_p[kOzakiMaxModuli];
};

// FP64 integer tricks that keep the conversion unit out of the inner loops:
// (x + 1.5 2^52) - 1.5 2^52 rounds |x| < 2^51 to the nearest integer, and
// the low word of r + 1.5 2^52 is the integer r as a two's-complement int32.
constexpr double kRound = 6755399441055744.0;  // 1.5 * 2^52
__device__ __forceinline__ double round_int(double x) {
  return __dadd_rn(__dadd_rn(x, kRound), -kRound);
}
__device__ __forceinline__ int int_of(double r) { return __double2loint(__dadd_rn(r, kRound)); }

// Residues of the integer v (|v| <= 2^50) modulo p as int8 bytes.  With
// q = rint(v / p) the remainder r = v - q p lies in [-(p-1)/2, (p-1)/2] for odd
// p <= 255 and in [-128, 128] for p = 256; its low byte is r as int8 (128 as
// -128, congruent mod 256).  fma(v, 1/p, 1.5 2^52) rounds v / p exactly (for
// odd p, v / p is at least 1/(2p) >= 2^-9 away from a half-integer while the
// product's error is below |v / p| 2^-53 < 2^-10.6; p = 256 is exact) and its
// low word is q as an int32; with vl = v mod 2^32, r mod 2^32 = vl - q p.  One
// DFMA and one integer multiply-add per residue.
__device__ __forceinline__ uint32_t residue_low(int vl, double v, double inv_p, int p) {
  const int q = __double2loint(fma(v, inv_p, kRound));
  return static_cast<uint32_t>(vl - q * p);  // low byte = residue
}

// Tile of 32 rows x 128 k of one plane -> L residue rows per row: row r of
// modulus l of a plane is out row ((plane * tiles + r / T) * L + l) * T + r % T
// (T = 2^tile_log2, the MMA tile height of this operand; tiles = rows_pad / T),
// each k_pad bytes; zeros in padding.  The L residue rows of a tile are
// T * k_pad bytes apart.  Thread (row pair rr, rr + 16; lane t of 16) converts
// the 8 consecutive k 8t .. 8t+7 of each of its rows and stores 8 residue bytes
// per modulus (16 lanes: 128 contiguous bytes per row and modulus).  The
// moduli loop is unrolled to kOzakiMaxModuli, so that p and 1/p are
// immediate constant-bank operands.  Grid: (row tiles, k tiles, planes).
template <bool KCONTIG, int LM>
__global__ void __launch_bounds__(256) k_residues(OperandView v, const int* __restrict__ shift,
                                                  ResidueMods mods, int tile_log2,
                                                  long long tiles, long long k_pad,
                                                  uint8_t* __restrict__ out) {
  __shared__ __align__(16) double tile[32 * 128];
  __shared__ long long koff[128];
  const int plane = blockIdx.z;
  const long long row0 = static_cast<long long>(blockIdx.x) * 32;
  const long long k0 = static_cast<long long>(blockIdx.y) * 128;
  tile_k_offsets(v, k0, koff);
  __syncthreads();
  load_tile<KCONTIG>(v, plane, row0, koff, tile);
  __syncthreads();
  const int t = threadIdx.x & 15;
  const long long tmask = (1LL << tile_log2) - 1;
  const long long lstep = k_pad << tile_log2;  // next modulus of the same row
#pragma unroll 1
  for (int it = 0; it < 2; ++it) {
    const int r = (threadIdx.x >> 4) + 16 * it;
    const long long row = row0 + r;
    const int sh = row < v.rows ? shift[plane * v.rows + row] : 0;
    double x[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) x[q] = tile[tile_at(r, 8 * t + q)];
    if (sh > -1000 && sh < 1000) {  // 2^sh is a normal double: scale by one multiply
      const double sc = pow2(sh);
#pragma unroll
      for (int q = 0; q < 8; ++q) x[q] = round_int(x[q] * sc);
    } else {
      for (int q = 0; q < 8; ++q) x[q] = round_int(ldexp_slow(x[q], sh));
    }
    int vl[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) vl[q] = int_of(x[q]);
    // row of modulus 0 in the residue layout
    const long long base_row =
        (((plane * tiles + (row >> tile_log2)) * mods.L) << tile_log2) + (row & tmask);
    uint8_t* dst = out + base_row * k_pad + k0 + 8 * t;
#pragma unroll
    for (int l = 0; l < (LM ? LM : kOzakiMaxModuli); ++l) {
      if (LM || l < mods.L) {
        const double ip = mods.inv_p[l];
        const int p = mods.pi[l];
        const uint32_t b01 =
            __byte_perm(residue_low(vl[0], x[0], ip, p), residue_low(vl[1], x[1], ip, p), 0x0040);
        const uint32_t b23 =
            __byte_perm(residue_low(vl[2], x[2], ip, p), residue_low(vl[3], x[3], ip, p), 0x0040);
        const uint32_t b45 =
            __byte_perm(residue_low(vl[4], x[4], ip, p), residue_low(vl[5], x[5], ip, p), 0x0040);
        const uint32_t b67 =
            __byte_perm(residue_low(vl[6], x[6], ip, p), residue_low(vl[7], x[7], ip, p), 0x0040);
        *reinterpret_cast<uint2*>(dst + l * lstep) =
            make_uint2(__byte_perm(b01, b23, 0x5410), __byte_perm(b45, b67, 0x5410));
      }
    }
  }
}

// ---------------------------------------------------------------------------
// tcgen05 int8 product kernel
// ---------------------------------------------------------------------------
// Work-item tile: kJHalves x 128 output columns j by 256 output rows i.  One
// half: the two 256-column TMEM accumulators are double-buffered across items;
// two halves: both accumulators belong to one item (two MMAs per K step share
// the i operand), so each K step moves 64 KiB for twice the products.
#ifndef UW12_I8_JHALVES
#define UW12_I8_JHALVES 1
#endif
constexpr int kJHalves = UW12_I8_JHALVES;
static_assert(kJHalves == 1 || kJHalves == 2, "one or two j halves per work item");
constexpr int kTileJ = 128;  // MMA M (TMEM lanes): output columns j
constexpr int kItemJ = kTileJ * kJHalves;  // output columns j per work item
constexpr int kTileI = 256;  // MMA N (TMEM columns): output rows i
constexpr int kTileK = 128;  // bytes of K per pipeline stage (one 128-byte swizzle row)
constexpr int kBytesJ = kItemJ * kTileK;  // 16 or 32 KiB
constexpr int kBytesI = kTileI * kTileK;  // 32 KiB
constexpr int kMmaK = 32;                 // K of one kind::i8 MMA
constexpr int kAccBufs = 2 / kJHalves;    // accumulator sets (2 x 256 TMEM columns in all)
constexpr int kEpiWarps = 4 * kJHalves;   // one per TMEM lane quarter and j half
constexpr int kThreads = 64 + 32 * kEpiWarps;
constexpr unsigned long long kWaitLimitNs = 4000000000ULL;  // 4 s

struct MmaArgs {
  int tiles_j, tiles_i, L, splits, nbatch, nbo1;
  long long n_items;
  int a_var1, a_var2, b_var1, b_var2;  // operand planes vary with bo1 / bo2
  int planes_a, planes_b;
  long long m_pad, n_pad;
  int kb_per_split, kb_total;
  uint32_t p[kOzakiMaxModuli], barrett[kOzakiMaxModuli], off[kOzakiMaxModuli];
  uint8_t* R;
  int* err;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_test(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait for the phase of the given parity to complete.  Gives up
// (returns false, sets the CTA's abort flag and the device error flag) after
// kWaitLimitNs, or when another role of the CTA has aborted.
__device__ bool mbar_wait(uint32_t bar, uint32_t parity, volatile int* abort_flag, int* err,
                          int code) {
  if (mbar_test(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  for (unsigned it = 1;; ++it) {
    if (mbar_test(bar, parity)) return true;
    if ((it & 255u) == 0) {
      if (*abort_flag) return false;
      if (global_ns() - t0 > kWaitLimitNs) {
        *abort_flag = 1;
        atomicExch(err, code);
        return false;
      }
    }
  }
}
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y,
                                            uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes "
      "[%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
      : "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// Shared-memory matrix descriptor: K-major, 128-byte swizzle, 8-row core
// groups 1024 bytes apart (stride byte offset), version 1.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t addr) {
  return static_cast<uint64_t>((addr >> 4) & 0x3fffu) | (1ull << 16) |
         (static_cast<uint64_t>(1024 >> 4) << 32) | (1ull << 46) | (2ull << 61);
}
// Instruction descriptor of kind::i8: s32 accumulator, signed int8 A and B,
// both K-major, N = kTileI, M = kTileJ.
constexpr uint32_t kIdesc = (2u << 4) | (1u << 7) | (1u << 10) |
                            (static_cast<uint32_t>(kTileI >> 3) << 17) |
                            (static_cast<uint32_t>(kTileJ >> 4) << 24);

__device__ __forceinline__ void mma_i8(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                       uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(
          tmem_d),
      "l"(adesc), "l"(bdesc), "r"(kIdesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
      : "memory");
}
__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   bar)
               : "memory");
}

#define UW12_TMEM_LD32(taddr, v)                                                               \
  asm volatile(                                                                                \
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "  \
      "%11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, "  \
      "%28, %29, %30, %31}, [%32];"                                                            \
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),    \
        "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]),             \
        "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]),          \
        "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]),          \
        "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]),          \
        "=r"(v[31])                                                                            \
      : "r"(taddr))

// Product residues: byte (split, batch b, column j, modulus l, row i) at
// (((split * nbatch + b) * n_pad + j) * L + l) * m_pad + i, so that the L
// residues of one column lie within L * m_pad bytes of each other.
__device__ __forceinline__ long long residue_offset(const MmaArgs& a, int split, int b,
                                                    long long j, int l) {
  return (((static_cast<long long>(split) * a.nbatch + b) * a.n_pad + j) * a.L + l) * a.m_pad;
}

__device__ __forceinline__ uint32_t mod_u32(uint32_t u, uint32_t p, uint32_t barrett) {
  uint32_t r = u - __umulhi(u, barrett) * p;
  return r >= p ? r - p : r;
}

// One work item = one 128 x 256 output tile of one modulus, one K chunk and
// one batch; items are numbered tile fastest, then modulus, K chunk, batch.
struct WorkItem {
  int tj, ti, l, split, b, kb0, nkb, yj, yi;
};

__device__ __forceinline__ WorkItem decode_item(const MmaArgs& a, long long w) {
  WorkItem it;
  const long long tiles = static_cast<long long>(a.tiles_j) * a.tiles_i;
  const long long tile = w % tiles;
  long long rest = w / tiles;
  it.tj = static_cast<int>(tile % a.tiles_j);
  it.ti = static_cast<int>(tile / a.tiles_j);
  it.l = static_cast<int>(rest % a.L);
  rest /= a.L;
  it.split = static_cast<int>(rest % a.splits);
  it.b = static_cast<int>(rest / a.splits);
  const int b1 = it.b % a.nbo1, b2 = it.b / a.nbo1;
  const int pa = (a.a_var1 ? b1 : 0) + (a.a_var1 ? a.nbo1 : 1) * (a.a_var2 ? b2 : 0);
  const int pb = (a.b_var1 ? b1 : 0) + (a.b_var1 ? a.nbo1 : 1) * (a.b_var2 ? b2 : 0);
  it.kb0 = it.split * a.kb_per_split;
  it.nkb = min(a.kb_per_split, a.kb_total - it.kb0);
  // residue rows: ((plane * tiles + tile) * L + l) * tile_rows + row in tile
  it.yj = static_cast<int>(
      ((static_cast<long long>(pb) * (a.n_pad / kItemJ) + it.tj) * a.L + it.l) * kItemJ);
  it.yi = static_cast<int>(
      ((static_cast<long long>(pa) * (a.m_pad / kTileI) + it.ti) * a.L + it.l) * kTileI);
  return it;
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

// Persistent: one CTA per SM walks the work items blockIdx.x, + gridDim.x, ...
// through a STAGES-deep TMA ring; with one j half per item the two TMEM
// accumulators (2 x 256 columns) let the epilogue of one item overlap the MMAs
// of the next, with two halves they hold the item's two halves.
template <int STAGES>
__global__ void __launch_bounds__(kThreads, 1)
    k_i8_mma(const __grid_constant__ CUtensorMap tm_j, const __grid_constant__ CUtensorMap tm_i,
             const MmaArgs a) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* base = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) &
                                             ~static_cast<uintptr_t>(1023));
  uint8_t* sj = base;                            // STAGES x kBytesJ
  uint8_t* si = base + STAGES * kBytesJ;         // STAGES x 32 KiB
  uint64_t* bars = reinterpret_cast<uint64_t*>(si + STAGES * kBytesI);
  uint64_t* full = bars;
  uint64_t* empty = bars + STAGES;
  uint64_t* acc_full = bars + 2 * STAGES;       // [2]
  uint64_t* acc_empty = bars + 2 * STAGES + 2;  // [2]
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * STAGES + 4);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(smem_u32(&full[s]), 1);
      mbar_init(smem_u32(&empty[s]), 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(smem_u32(&acc_full[b]), 1);
      mbar_init(smem_u32(&acc_empty[b]), kEpiWarps);  // one arrival per epilogue warp
    }
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tmem_slot)),
                 "r"(static_cast<uint32_t>(2 * kTileI))
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0 && lane == 0) {
    // ---- TMA producer
    long long pos = 0;  // ring position, continued across items
    bool ok = true;
    for (long long w = blockIdx.x; ok && w < a.n_items; w += gridDim.x) {
      const WorkItem it = decode_item(a, w);
      for (int kb = 0; kb < it.nkb; ++kb) {
        const int s = static_cast<int>(pos % STAGES);
        const uint32_t ph = static_cast<uint32_t>(pos / STAGES) & 1;
        if (!mbar_wait(smem_u32(&empty[s]), ph ^ 1, abort_flag, a.err, 1)) {
          ok = false;
          break;
        }
        const uint32_t fb = smem_u32(&full[s]);
        mbar_expect_tx(fb, kBytesJ + kBytesI);
        const int x = (it.kb0 + kb) * kTileK;
        tma_load_2d(smem_u32(sj + s * kBytesJ), &tm_j, x, it.yj, fb);
        tma_load_2d(smem_u32(si + s * kBytesI), &tm_i, x, it.yi, fb);
        ++pos;
      }
    }
    if (!ok) {
      // let the copies already issued land before the CTA exits
      for (long long q = pos > STAGES ? pos - STAGES : 0; q < pos; ++q)
        (void)mbar_wait(smem_u32(&full[q % STAGES]), static_cast<uint32_t>(q / STAGES) & 1,
                        abort_flag, a.err, 1);
    }
  } else if (warp == 1 && lane == 0) {
    // ---- MMA issuer
    long long pos = 0;
    int t = 0, last_buf = -1;
    uint32_t last_use = 0;
    for (long long w = blockIdx.x; w < a.n_items; w += gridDim.x, ++t) {
      const WorkItem it = decode_item(a, w);
      const int buf = t % kAccBufs;
      const uint32_t use = static_cast<uint32_t>(t / kAccBufs);
      if (!mbar_wait(smem_u32(&acc_empty[buf]), (use & 1) ^ 1, abort_flag, a.err, 2)) break;
      tc_fence_after();
      const uint32_t d = tmem + static_cast<uint32_t>(buf * kJHalves * kTileI);
      bool ok = true;
      for (int kb = 0; kb < it.nkb; ++kb) {
        const int s = static_cast<int>(pos % STAGES);
        const uint32_t ph = static_cast<uint32_t>(pos / STAGES) & 1;
        if (!mbar_wait(smem_u32(&full[s]), ph, abort_flag, a.err, 2)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint64_t di = sw128_desc(smem_u32(si + s * kBytesI));
#pragma unroll
        for (int h = 0; h < kJHalves; ++h) {
          // j half h: rows 128 h .. of the stage, accumulator columns 256 h ..
          const uint64_t dj = sw128_desc(smem_u32(sj + s * kBytesJ + h * kTileJ * kTileK));
#pragma unroll
          for (int kk = 0; kk < kTileK / kMmaK; ++kk) {
            // advance along K inside the swizzle row: +32 bytes = +2 in the
            // 16-byte address field
            mma_i8(d + static_cast<uint32_t>(h * kTileI), dj + 2 * kk, di + 2 * kk,
                   (kb | kk) != 0);
          }
        }
        mma_commit(smem_u32(&empty[s]));
        ++pos;
      }
      mma_commit(smem_u32(&acc_full[buf]));  // also on failure, so the epilogue wakes
      last_buf = buf;
      last_use = use;
      if (!ok) break;
    }
    if (last_buf >= 0)  // every MMA of this CTA has completed before TMEM is released
      (void)mbar_wait(smem_u32(&acc_full[last_buf]), last_use & 1, abort_flag, a.err, 4);
  } else if (warp >= 2) {
    // ---- epilogue: TMEM -> residues mod p -> uint8 rows
    const int q = warp & 3;          // TMEM lane quarter this warp may access
    const int h = (warp - 2) / 4;    // j half
    int t = 0;
    for (long long w = blockIdx.x; w < a.n_items; w += gridDim.x, ++t) {
      const WorkItem it = decode_item(a, w);
      const int buf = t % kAccBufs;
      const uint32_t use = static_cast<uint32_t>(t / kAccBufs);
      // warp-uniform, so that the .sync.aligned TMEM loads below are convergent
      const bool ok =
          __all_sync(0xffffffffu, mbar_wait(smem_u32(&acc_full[buf]), use & 1, abort_flag, a.err, 3));
      tc_fence_after();
      if (!ok) break;
      const uint32_t p = a.p[it.l], bm = a.barrett[it.l], off = a.off[it.l];
      const long long j = static_cast<long long>(it.tj) * kItemJ + h * kTileJ + q * 32 + lane;
      uint8_t* rowp = a.R + residue_offset(a, it.split, it.b, j, it.l) +
                      static_cast<long long>(it.ti) * kTileI;
      const uint32_t tq = tmem + static_cast<uint32_t>((buf * kJHalves + h) * kTileI) +
                          (static_cast<uint32_t>(q * 32) << 16);
#pragma unroll 1
      for (int c = 0; c < kTileI / 32; ++c) {
        uint32_t v[32];
        UW12_TMEM_LD32(tq + c * 32, v);
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        uint32_t wd[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) {
          uint32_t word = 0;
#pragma unroll
          for (int u = 0; u < 4; ++u) word |= mod_u32(v[4 * e + u] + off, p, bm) << (8 * u);
          wd[e] = word;
        }
        uint4* dst = reinterpret_cast<uint4*>(rowp + c * 32);
        dst[0] = make_uint4(wd[0], wd[1], wd[2], wd[3]);
        dst[1] = make_uint4(wd[4], wd[5], wd[6], wd[7]);
      }
      // this warp's TMEM reads are done: release the accumulator
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(smem_u32(&acc_empty[buf]));
    }
  }

  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    __syncwarp();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(static_cast<uint32_t>(2 * kTileI))
                 : "memory");
  }
}

// ---------------------------------------------------------------------------
// CRT reconstruction
// ---------------------------------------------------------------------------
struct CrtArgs {
  const uint8_t* R;
  long long m, n, m_pad, n_pad;
  int splits, L, nch, nbatch, nbo1;
  const int* shift_a;
  const int* shift_b;
  int a_var1, a_var2, b_var1, b_var2;
  long long rows_a, rows_b;  // rows per shift plane (m, n)
  double* C;
  long long ldc, sCo1, sCo2;
  double alpha, beta;
  uint32_t p[kOzakiMaxModuli], barrett[kOzakiMaxModuli];
  double w[kOzakiMaxModuli][kMaxChunks];
  double mc[kMaxChunks];
  double inv_m;
  int cw;          // CRT chunk width in bits
  int c_aligned;   // C, ldc and the batch strides allow 16-byte accesses
};

// One thread = E (kCrtElems) consecutive rows i of a column j of one batch;
// grid (row blocks of 256 E, columns strided by gridDim.y, batches).  The L
// residue words of a column (and the E elements of C when beta != 0) are
// loaded before any is used (one load per modulus and K chunk in flight per
// thread), the K-chunk sums of the E bytes are kept as pairs of 16-bit lanes,
// the CRT runs on NCH chunks of cw bits, and C is read and written 16 bytes at
// a time when aligned.
// x 2^e: one multiply by an exactly representable power of two when 2^e is a
// normal double, ldexp otherwise.
__device__ __forceinline__ double scale_pow2(double x, int e) {
  if (e >= -1022 && e <= 1023) return x * pow2(e);
  return ldexp_slow(x, e);
}

// s + e = a + b exactly (Knuth's TwoSum, six FP64 operations).
__device__ __forceinline__ double two_sum(double a, double b, double& e) {
  const double s = __dadd_rn(a, b);
  const double bb = __dsub_rn(s, a);
  e = __dadd_rn(__dsub_rn(a, __dsub_rn(s, bb)), __dsub_rn(b, bb));
  return s;
}

// sum_c d[c] 2^(cw c) for integer-valued doubles |d[c]| < 2^53: every term
// d[c] 2^(cw c) is exact, the running sum is carried error-free (TwoSum) and
// the integer errors are added at the end, so the result equals the exact sum
// whenever that is a double and is within one unit in the last place
// otherwise.
template <int NCH>
__device__ __forceinline__ double join_chunks(const double (&d)[NCH], double chunk) {
  double pw = 1.0;
  double terms[NCH];
#pragma unroll
  for (int c = 0; c < NCH; ++c) {
    terms[c] = d[c] * pw;  // exact: a power-of-two scaling
    pw *= chunk;
  }
  double sum = terms[NCH - 1], err = 0.0;
#pragma unroll
  for (int c = NCH - 2; c >= 0; --c) {
    double e;
    sum = two_sum(sum, terms[c], e);
    err += e;
  }
  return sum + err;
}

// Byte b (0..3) of w as a double: the byte placed in the low word under the
// exponent of 2^52, minus 2^52.
__device__ __forceinline__ double byte_to_double(uint32_t w, int b) {
  return __dsub_rn(__hiloint2double(0x43300000, static_cast<int>(__byte_perm(w, 0, 0x4440 + b))),
                   4503599627370496.0);
}

// Residue (< 2^16) to double without the conversion unit.
__device__ __forceinline__ double small_to_double(uint32_t r) {
  return __dsub_rn(__hiloint2double(0x43300000, static_cast<int>(r)), 4503599627370496.0);
}

// Rows i per CRT thread: 4 (one 32-bit residue word per modulus) or 2 (one
// 16-bit word; fewer registers, more resident warps).
#ifndef UW12_CRT_ELEMS
#define UW12_CRT_ELEMS 4
#endif
constexpr int kCrtElems = UW12_CRT_ELEMS;
static_assert(kCrtElems == 2 || kCrtElems == 4, "2 or 4 rows per CRT thread");
constexpr int kCrtMinBlocks = kCrtElems == 4 ? 3 : 4;

template <int E>
__device__ __forceinline__ uint32_t load_residues(const uint8_t* p) {
  if (E == 4) return __ldg(reinterpret_cast<const uint32_t*>(p));
  return __ldg(reinterpret_cast<const unsigned short*>(p));
}

// REDUCE: several K chunks, whose residue sums are reduced mod p; with one K
// chunk the stored residues (already in [0, p)) enter the CRT sum directly.
template <int NCH, bool REDUCE>
__global__ void __launch_bounds__(256, REDUCE ? 2 : kCrtMinBlocks) k_crt(const CrtArgs a) {
  constexpr int E = kCrtElems;
  const long long i0 = (static_cast<long long>(blockIdx.x) * 256 + threadIdx.x) * E;
  if (i0 >= a.m) return;
  const int b = blockIdx.z;
  const int b1 = b % a.nbo1, b2 = b / a.nbo1;
  const int pa = (a.a_var1 ? b1 : 0) + (a.a_var1 ? a.nbo1 : 1) * (a.a_var2 ? b2 : 0);
  const int pb = (a.b_var1 ? b1 : 0) + (a.b_var1 ? a.nbo1 : 1) * (a.b_var2 ? b2 : 0);
  // residue layout of k_i8_mma: (((split * nbatch + b) * n_pad + j) * L + l) * m_pad + i
  const long long lstride = a.m_pad;                                             // next modulus
  const long long sstride = static_cast<long long>(a.nbatch) * a.n_pad * a.L * a.m_pad;  // K chunk
  int sa[E];
#pragma unroll
  for (int e = 0; e < E; ++e)
    sa[e] = i0 + e < a.m ? a.shift_a[pa * a.rows_a + i0 + e] : 0;
  const double chunk = __longlong_as_double(static_cast<long long>(a.cw + 1023) << 52);  // 2^cw

  const bool vec = i0 + E - 1 < a.m && a.c_aligned;
  for (long long j = blockIdx.y; j < a.n; j += gridDim.y) {
    const uint8_t* base = a.R + (static_cast<long long>(b) * a.n_pad + j) * a.L * a.m_pad + i0;
    double* Cb = a.C + b1 * a.sCo1 + b2 * a.sCo2 + j * a.ldc;
    // one residue word (E rows) per modulus and K chunk, and the E elements of
    // C when they are accumulated into: all loads issued first
    uint32_t w0[kOzakiMaxModuli];
#pragma unroll
    for (int l = 0; l < kOzakiMaxModuli; ++l)
      if (l < a.L) w0[l] = load_residues<E>(base + l * lstride);
    double cold[E];
#pragma unroll
    for (int e = 0; e < E; ++e) cold[e] = 0.0;
    if (a.beta != 0.0) {
      if (vec) {
#pragma unroll
        for (int e = 0; e < E; e += 2) {
          const double2 c2 = *reinterpret_cast<const double2*>(Cb + i0 + e);
          cold[e] = c2.x;
          cold[e + 1] = c2.y;
        }
      } else {
#pragma unroll
        for (int e = 0; e < E; ++e)
          if (i0 + e < a.m) cold[e] = Cb[i0 + e];
      }
    }
    double S[E][NCH];
#pragma unroll
    for (int e = 0; e < E; ++e)
#pragma unroll
      for (int c = 0; c < NCH; ++c) S[e][c] = 0.0;
    if (!REDUCE) {
      // one K chunk: the stored residues (in [0, p)) enter the CRT sum directly
#pragma unroll
      for (int l = 0; l < kOzakiMaxModuli; ++l) {
        if (l < a.L) {
#pragma unroll
          for (int e = 0; e < E; ++e) {
            const double r = byte_to_double(w0[l], e);
#pragma unroll
            for (int c = 0; c < NCH; ++c) S[e][c] = fma(r, a.w[l][c], S[e][c]);
          }
        }
      }
    } else {
      // K chunks: byte sums in 16-bit lanes (bytes 0, 2 and 1, 3), reduced mod p
      uint32_t s02[kOzakiMaxModuli], s13[kOzakiMaxModuli];
#pragma unroll
      for (int l = 0; l < kOzakiMaxModuli; ++l) {
        if (l < a.L) {
          s02[l] = w0[l] & 0x00ff00ffu;
          s13[l] = (w0[l] >> 8) & 0x00ff00ffu;
        }
      }
      for (int sp = 1; sp < a.splits; ++sp) {
#pragma unroll
        for (int l = 0; l < kOzakiMaxModuli; ++l) {
          if (l < a.L) {
            const uint32_t w = load_residues<E>(base + sp * sstride + l * lstride);
            s02[l] += w & 0x00ff00ffu;
            s13[l] += (w >> 8) & 0x00ff00ffu;
          }
        }
      }
#pragma unroll
      for (int l = 0; l < kOzakiMaxModuli; ++l) {
        if (l < a.L) {
          const uint32_t p = a.p[l], bm = a.barrett[l];
          const uint32_t u[4] = {s02[l] & 0xffffu, s13[l] & 0xffffu, s02[l] >> 16, s13[l] >> 16};
#pragma unroll
          for (int e = 0; e < E; ++e) {
            const double r = small_to_double(mod_u32(u[e], p, bm));
#pragma unroll
            for (int c = 0; c < NCH; ++c) S[e][c] = fma(r, a.w[l][c], S[e][c]);
          }
        }
      }
    }
    const int sb = a.shift_b[pb * a.rows_b + j];
    double out[E];
#pragma unroll
    for (int e = 0; e < E; ++e) {
      double approx = 0.0;
#pragma unroll
      for (int c = NCH - 1; c >= 0; --c) approx = fma(approx, chunk, S[e][c]);
      const double q = round_int(approx * a.inv_m);  // |q| < 2^13
      double dig[NCH];
#pragma unroll
      for (int c = 0; c < NCH; ++c) dig[c] = fma(-q, a.mc[c], S[e][c]);  // exact
      out[e] = a.alpha * scale_pow2(join_chunks<NCH>(dig, chunk), -(sa[e] + sb));
      if (a.beta != 0.0) out[e] = fma(a.beta, cold[e], out[e]);
    }
    if (vec) {
#pragma unroll
      for (int e = 0; e < E; e += 2)
        *reinterpret_cast<double2*>(Cb + i0 + e) = make_double2(out[e], out[e + 1]);
    } else {
#pragma unroll
      for (int e = 0; e < E; ++e)
        if (i0 + e < a.m) Cb[i0 + e] = out[e];
    }
  }
}

// One K chunk, pipelined: a block owns 1024 rows i of a batch and walks its
// columns j = blockIdx.y, + gridDim.y, ...; the L residue rows of the next
// kCrtStages - 1 columns are copied into shared memory (16-byte cp.async.cg,
// L x 1024 bytes per column) while the current one is reconstructed, so the
// copies of a block stay in flight during its FP64 work.  Thread = 4 rows, as
// in k_crt; the same arithmetic.
constexpr int kCrtStages = 3;
constexpr int kCrtRows = 1024;  // rows i per block

template <int NCH, int LM>
__global__ void __launch_bounds__(256, 3) k_crt_pipe(const CrtArgs a) {
  extern __shared__ __align__(16) uint8_t crt_smem[];  // kCrtStages x L x kCrtRows bytes
  const int L = a.L;
  const long long iblk = static_cast<long long>(blockIdx.x) * kCrtRows;
  const long long i0 = iblk + threadIdx.x * 4;
  const int b = blockIdx.z;
  const int b1 = b % a.nbo1, b2 = b / a.nbo1;
  const int pa = (a.a_var1 ? b1 : 0) + (a.a_var1 ? a.nbo1 : 1) * (a.a_var2 ? b2 : 0);
  const int pb = (a.b_var1 ? b1 : 0) + (a.b_var1 ? a.nbo1 : 1) * (a.b_var2 ? b2 : 0);
  // bytes of this block's rows inside one residue row (a multiple of 256)
  const long long row_bytes = min(static_cast<long long>(kCrtRows), a.m_pad - iblk);
  const long long nj = (a.n - blockIdx.y + gridDim.y - 1) / gridDim.y;
  const bool active = i0 < a.m;
  int sa[4];
#pragma unroll
  for (int e = 0; e < 4; ++e)
    sa[e] = i0 + e < a.m ? a.shift_a[pa * a.rows_a + i0 + e] : 0;
  const double chunk = __longlong_as_double(static_cast<long long>(a.cw + 1023) << 52);  // 2^cw
  const bool vec = i0 + 3 < a.m && a.c_aligned;

  auto issue = [&](long long q, int slot) {
    const long long j = blockIdx.y + q * gridDim.y;
    const uint8_t* src0 = a.R + (static_cast<long long>(b) * a.n_pad + j) * L * a.m_pad + iblk;
    uint8_t* dst0 = crt_smem + slot * L * kCrtRows;
    for (int c = threadIdx.x; c < L * (kCrtRows / 16); c += 256) {
      const int l = c / (kCrtRows / 16);
      const int off = (c % (kCrtRows / 16)) * 16;
      const bool in = off < row_bytes;
      const uint8_t* src = in ? src0 + l * a.m_pad + off : src0;
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(
                       static_cast<unsigned>(__cvta_generic_to_shared(dst0 + l * kCrtRows + off))),
                   "l"(src), "r"(in ? 16 : 0)
                   : "memory");
    }
  };

#pragma unroll
  for (int q = 0; q < kCrtStages - 1; ++q) {
    if (q < nj) issue(q, q);
    asm volatile("cp.async.commit_group;\n" ::: "memory");
  }
  for (long long q = 0; q < nj; ++q) {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(kCrtStages - 2) : "memory");
    __syncthreads();  // column q landed; the slot refilled below is no longer read
    {
      const long long qn = q + kCrtStages - 1;
      if (qn < nj) issue(qn, static_cast<int>(qn % kCrtStages));
      asm volatile("cp.async.commit_group;\n" ::: "memory");
    }
    if (!active) continue;
    const long long j = blockIdx.y + q * gridDim.y;
    const uint8_t* rs = crt_smem + static_cast<int>(q % kCrtStages) * L * kCrtRows + threadIdx.x * 4;
    double* Cb = a.C + b1 * a.sCo1 + b2 * a.sCo2 + j * a.ldc;
    double cold[4] = {0.0, 0.0, 0.0, 0.0};
    if (a.beta != 0.0) {
      if (vec) {
        const double2 c01 = *reinterpret_cast<const double2*>(Cb + i0);
        const double2 c23 = *reinterpret_cast<const double2*>(Cb + i0 + 2);
        cold[0] = c01.x; cold[1] = c01.y; cold[2] = c23.x; cold[3] = c23.y;
      } else {
#pragma unroll
        for (int e = 0; e < 4; ++e)
          if (i0 + e < a.m) cold[e] = Cb[i0 + e];
      }
    }
    double S[4][NCH];
#pragma unroll
    for (int e = 0; e < 4; ++e)
#pragma unroll
      for (int c = 0; c < NCH; ++c) S[e][c] = 0.0;
#pragma unroll
    for (int l = 0; l < (LM ? LM : kOzakiMaxModuli); ++l) {
      if (LM || l < L) {
        const uint32_t w = *reinterpret_cast<const uint32_t*>(rs + l * kCrtRows);
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const double r = byte_to_double(w, e);
#pragma unroll
          for (int c = 0; c < NCH; ++c) S[e][c] = fma(r, a.w[l][c], S[e][c]);
        }
      }
    }
    const int sb = a.shift_b[pb * a.rows_b + j];
    double out[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      double approx = 0.0;
#pragma unroll
      for (int c = NCH - 1; c >= 0; --c) approx = fma(approx, chunk, S[e][c]);
      const double qq = round_int(approx * a.inv_m);  // |q| < 2^13
      double dig[NCH];
#pragma unroll
      for (int c = 0; c < NCH; ++c) dig[c] = fma(-qq, a.mc[c], S[e][c]);  // exact
      out[e] = a.alpha * scale_pow2(join_chunks<NCH>(dig, chunk), -(sa[e] + sb));
      if (a.beta != 0.0) out[e] = fma(a.beta, cold[e], out[e]);
    }
    if (vec) {
      *reinterpret_cast<double2*>(Cb + i0) = make_double2(out[0], out[1]);
      *reinterpret_cast<double2*>(Cb + i0 + 2) = make_double2(out[2], out[3]);
    } else {
#pragma unroll
      for (int e = 0; e < 4; ++e)
        if (i0 + e < a.m) Cb[i0 + e] = out[e];
    }
  }
  asm volatile("cp.async.wait_all;\n" ::: "memory");
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                 const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                 const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                 CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encode_fn() {
  static std::once_flag once;
  static EncodeTiled fn = nullptr;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiled>(p);
  });
  if (!fn) throw Error(kErrCuda, "cuTensorMapEncodeTiled is not available");
  return fn;
}

// 2-D uint8 map over rows x k_pad bytes, box = box_rows x 128 bytes, 128-byte swizzle.
CUtensorMap make_map(const uint8_t* base, long long rows, long long k_pad, int box_rows) {
  CUtensorMap m;
  const cuuint64_t dims[2] = {static_cast<cuuint64_t>(k_pad), static_cast<cuuint64_t>(rows)};
  const cuuint64_t strides[1] = {static_cast<cuuint64_t>(k_pad)};
  const cuuint32_t box[2] = {static_cast<cuuint32_t>(kTileK), static_cast<cuuint32_t>(box_rows)};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = encode_fn()(&m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<uint8_t*>(base),
                                 dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                 CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                                 CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS)
    throw Error(kErrCuda, "cuTensorMapEncodeTiled failed (" + std::to_string(int(r)) + ")");
  return m;
}

constexpr int kStages = 4 / kJHalves + (kJHalves - 1);  // 4 x 48 or 3 x 64 KiB of stages
constexpr size_t kMmaSmem =
    size_t(kStages) * (kBytesJ + kBytesI) + 1024 /*alignment*/ + 256 /*barriers*/;

long long round_up(long long x, long long m) { return (x + m - 1) / m * m; }

int num_sms() {
  static int n[kMaxDevices] = {};
  static std::mutex mu;
  int dev = 0;
  UW12_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) throw Error(kErrInvalid, "device index out of range");
  std::lock_guard<std::mutex> lk(mu);
  if (!n[dev]) UW12_CUDA(cudaDeviceGetAttribute(&n[dev], cudaDevAttrMultiProcessorCount, dev));
  return n[dev];
}

struct Timer {
  int kind;
  double work;
  std::string shape;
  cudaEvent_t a = nullptr, b = nullptr;
  cudaStream_t s;
  Timer(int kind_, double work_, std::string shape_, cudaStream_t s_)
      : kind(kind_), work(work_), shape(std::move(shape_)), s(s_) {
    if (!profile_enabled()) return;
    UW12_CUDA(cudaEventCreate(&a));
    UW12_CUDA(cudaEventCreate(&b));
    UW12_CUDA(cudaEventRecord(a, s));
  }
  void stop() {
    if (!a) return;
    UW12_CUDA(cudaEventRecord(b, s));
    profile_record(kind, a, b, work, shape);
    a = b = nullptr;
  }
};

// Runs one GEMM whose temporaries fit.  d.nbo2 == 1 or both batch dims are
// handled through the plane maps.
void run_core(const GemmDesc& d, const Consts& cs, int beta, cudaStream_t s) {
  const int L = cs.L;
  const long long nbo1 = d.nbo1, nbo2 = d.nbo2, nbatch = nbo1 * nbo2;
  const long long k_total = d.k * d.nbr1 * d.nbr2;
  const long long k_pad = round_up(k_total, kTileK);
  const long long m_pad = round_up(d.m, kTileI), n_pad = round_up(d.n, kItemJ);
  const int a_var1 = d.sAo1 != 0 && nbo1 > 1, a_var2 = d.sAo2 != 0 && nbo2 > 1;
  const int b_var1 = d.sBo1 != 0 && nbo1 > 1, b_var2 = d.sBo2 != 0 && nbo2 > 1;
  const int pa1 = a_var1 ? int(nbo1) : 1, pa2 = a_var2 ? int(nbo2) : 1;
  const int pb1 = b_var1 ? int(nbo1) : 1, pb2 = b_var2 ? int(nbo2) : 1;
  const long long planes_a = pa1 * pa2, planes_b = pb1 * pb2;

  // K chunks: <= kMaxKChunk bytes each; more chunks when the tile grid alone
  // would leave SMs idle.
  const long long kb_total = k_pad / kTileK;
  const long long tiles_j = n_pad / kItemJ, tiles_i = m_pad / kTileI;
  const long long ctas = tiles_j * tiles_i * L * nbatch;
  long long splits = (k_pad + kMaxKChunk - 1) / kMaxKChunk;
  const long long want = (2 * num_sms() + ctas - 1) / ctas;
  splits = std::max(splits, std::min(want, std::max<long long>(1, kb_total / 8)));
  splits = std::min(splits, std::max<long long>(1, 65535 / nbatch));
  long long kb_per = (kb_total + splits - 1) / splits;
  kb_per = std::min<long long>(kb_per, kMaxKChunk / kTileK);
  splits = (kb_total + kb_per - 1) / kb_per;
  if (splits * nbatch > 65535) throw Error(kErrInvalid, "split-precision GEMM: too many batches");

  DevBuf resA((L * planes_a * m_pad * k_pad + 7) / 8, s);
  DevBuf resB((L * planes_b * n_pad * k_pad + 7) / 8, s);
  DevBuf shA((planes_a * d.m + 1) / 2, s), shB((planes_b * d.n + 1) / 2, s);
  DevBuf exA((planes_a * d.m + 1) / 2, s), exB((planes_b * d.n + 1) / 2, s);
  unsigned* ea = reinterpret_cast<unsigned*>(exA.get());
  unsigned* eb = reinterpret_cast<unsigned*>(exB.get());
  DevBuf R((splits * L * nbatch * n_pad * m_pad + 7) / 8, s);
  uint8_t* ra = reinterpret_cast<uint8_t*>(resA.get());
  uint8_t* rb = reinterpret_cast<uint8_t*>(resB.get());
  int* sa = reinterpret_cast<int*>(shA.get());
  int* sb = reinterpret_cast<int*>(shB.get());

  // ---- operand views: A rows = i (m), B rows = j (n)
  OperandView va{d.A, d.m, d.k, k_total,
                 d.a_kcontig ? d.lda : 1, d.a_kcontig ? 1 : d.lda, d.sAr1, d.sAr2, d.nbr1,
                 d.sAo1, d.sAo2, pa1, pa2};
  OperandView vb{d.B, d.n, d.k, k_total,
                 d.b_ncontig ? 1 : d.ldb, d.b_ncontig ? d.ldb : 1, d.sBr1, d.sBr2, d.nbr1,
                 d.sBo1, d.sBo2, pb1, pb2};
  ResidueMods mods;
  mods.L = L;
  for (int l = 0; l < L; ++l) {
    mods.pi[l] = static_cast<int>(cs.p[l]);
    mods.inv_p[l] = cs.inv_p[l];
  }
  {
    const double bytes = 8.0 * double(planes_a * d.m + planes_b * d.n) * double(k_total) * 2.0 +
                         double(L) * double(planes_a * m_pad + planes_b * n_pad) * double(k_pad);
    Timer tm(kProfSplitPrep, bytes, "prep", s);
    auto prep = [&](const OperandView& v, long long planes, long long rows_pad, int tile_rows,
                    int* sh, unsigned* ep, uint8_t* out) {
      UW12_CUDA(cudaMemsetAsync(ep, 0, planes * v.rows * sizeof(unsigned), s));
      dim3 ge(static_cast<unsigned>(rows_pad / 32),
              static_cast<unsigned>((k_pad + kExpTileK - 1) / kExpTileK),
              static_cast<unsigned>(planes));
      if (v.ks == 1)
        k_row_exponent<true><<<ge, 256, 0, s>>>(v, ep);
      else
        k_row_exponent<false><<<ge, 256, 0, s>>>(v, ep);
      dim3 g(static_cast<unsigned>(rows_pad / 32), static_cast<unsigned>(k_pad / 128),
             static_cast<unsigned>(planes));
      UW12_LAUNCHED();
      const long long nsh = planes * v.rows;
      k_exponent_to_shift<<<static_cast<unsigned>((nsh + 255) / 256), 256, 0, s>>>(ep, nsh, beta,
                                                                                  sh);
      UW12_LAUNCHED();
      const int tlog = tile_rows == 256 ? 8 : 7;
      const long long tiles = rows_pad / tile_rows;
      // the default modulus count runs a fully unrolled, unguarded moduli loop
      if (v.ks == 1 && L == kOzakiDefaultModuli)
        k_residues<true, kOzakiDefaultModuli><<<g, 256, 0, s>>>(v, sh, mods, tlog, tiles, k_pad, out);
      else if (v.ks == 1)
        k_residues<true, 0><<<g, 256, 0, s>>>(v, sh, mods, tlog, tiles, k_pad, out);
      else if (L == kOzakiDefaultModuli)
        k_residues<false, kOzakiDefaultModuli><<<g, 256, 0, s>>>(v, sh, mods, tlog, tiles, k_pad, out);
      else
        k_residues<false, 0><<<g, 256, 0, s>>>(v, sh, mods, tlog, tiles, k_pad, out);
      UW12_LAUNCHED();
    };
    prep(va, planes_a, m_pad, kTileI, sa, ea, ra);
    prep(vb, planes_b, n_pad, kItemJ, sb, eb, rb);
    tm.stop();
  }

  // ---- int8 products
  {
    static std::mutex attr_mu;
    static bool attr_set[64] = {};
    {
      int dev = 0;
      UW12_CUDA(cudaGetDevice(&dev));
      std::lock_guard<std::mutex> lk(attr_mu);
      if (!attr_set[dev]) {
        UW12_CUDA(cudaFuncSetAttribute(k_i8_mma<kStages>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(kMmaSmem)));
        attr_set[dev] = true;
      }
    }
    const CUtensorMap tmj = make_map(rb, L * planes_b * n_pad, k_pad, kItemJ);
    const CUtensorMap tmi = make_map(ra, L * planes_a * m_pad, k_pad, kTileI);
    MmaArgs ma{};
    ma.tiles_j = static_cast<int>(tiles_j);
    ma.tiles_i = static_cast<int>(tiles_i);
    ma.n_items = tiles_j * tiles_i * L * splits * nbatch;
    ma.L = L;
    ma.splits = static_cast<int>(splits);
    ma.nbatch = static_cast<int>(nbatch);
    ma.nbo1 = static_cast<int>(nbo1);
    ma.a_var1 = a_var1; ma.a_var2 = a_var2; ma.b_var1 = b_var1; ma.b_var2 = b_var2;
    ma.planes_a = static_cast<int>(planes_a);
    ma.planes_b = static_cast<int>(planes_b);
    ma.m_pad = m_pad;
    ma.n_pad = n_pad;
    ma.kb_per_split = static_cast<int>(kb_per);
    ma.kb_total = static_cast<int>(kb_total);
    for (int l = 0; l < L; ++l) {
      ma.p[l] = cs.p[l];
      ma.barrett[l] = cs.barrett[l];
      ma.off[l] = cs.off[l];
    }
    ma.R = reinterpret_cast<uint8_t*>(R.get());
    ma.err = err_flag();
    const double ops = 2.0 * double(d.m) * double(d.n) * double(k_total) * double(L) * nbatch;
    char shape[160];
    std::snprintf(shape, sizeof(shape), "i8 %lld %lld %lld %lld L%d s%lld", d.m, d.n, k_total,
                  nbatch, L, splits);
    Timer tm(kProfI8Mma, ops, shape, s);
    const unsigned grid = static_cast<unsigned>(std::min<long long>(ma.n_items, num_sms()));
    k_i8_mma<kStages><<<grid, kThreads, kMmaSmem, s>>>(tmj, tmi, ma);
    UW12_LAUNCHED();
    tm.stop();
  }

  // ---- CRT reconstruction
  {
    CrtArgs ca{};
    ca.R = reinterpret_cast<const uint8_t*>(R.get());
    ca.m = d.m; ca.n = d.n; ca.m_pad = m_pad; ca.n_pad = n_pad;
    ca.splits = static_cast<int>(splits);
    ca.L = L;
    ca.nch = cs.nch;
    ca.nbatch = static_cast<int>(nbatch);
    ca.nbo1 = static_cast<int>(nbo1);
    ca.shift_a = sa; ca.shift_b = sb;
    ca.a_var1 = a_var1; ca.a_var2 = a_var2; ca.b_var1 = b_var1; ca.b_var2 = b_var2;
    ca.rows_a = d.m; ca.rows_b = d.n;
    ca.C = d.C; ca.ldc = d.ldc; ca.sCo1 = d.sCo1; ca.sCo2 = d.sCo2;
    ca.alpha = d.alpha; ca.beta = d.beta;
    for (int l = 0; l < L; ++l) {
      ca.p[l] = cs.p[l];
      ca.barrett[l] = cs.barrett[l];
      for (int c = 0; c < kMaxChunks; ++c) ca.w[l][c] = cs.w[l][c];
    }
    for (int c = 0; c < kMaxChunks; ++c) ca.mc[c] = cs.mc[c];
    ca.inv_m = cs.inv_m;
    ca.cw = cs.cw;
    ca.c_aligned = (reinterpret_cast<std::uintptr_t>(d.C) % 16 == 0) && d.ldc % 2 == 0 &&
                   d.sCo1 % 2 == 0 && d.sCo2 % 2 == 0;
    const double bytes = double(splits * L) * double(d.m * d.n * nbatch) +
                         8.0 * double(d.m * d.n * nbatch) * (d.beta != 0.0 ? 2.0 : 1.0);
    Timer tm(kProfSplitCrt, bytes, "crt", s);
    const dim3 g(static_cast<unsigned>((d.m + 256 * kCrtElems - 1) / (256 * kCrtElems)),
                 static_cast<unsigned>(std::min<long long>(d.n, 65535)),
                 static_cast<unsigned>(nbatch));
    const bool reduce = splits > 1;
    if (!reduce) {
      // pipelined: about eight waves of 3 blocks per SM (a short tail), each
      // block walking its share of the columns
      const long long gx = (d.m + kCrtRows - 1) / kCrtRows;
      const long long per_col = gx * nbatch;
      const long long gy = std::min<long long>(
          std::min<long long>(d.n, 65535),
          std::max<long long>(1, (24LL * num_sms() + per_col - 1) / per_col));
      const dim3 gp(static_cast<unsigned>(gx), static_cast<unsigned>(gy), g.z);
      const size_t smem = size_t(kCrtStages) * L * kCrtRows;
      if (L == kOzakiDefaultModuli && cs.nch == 3) {
        k_crt_pipe<3, kOzakiDefaultModuli><<<gp, 256, smem, s>>>(ca);
      } else {
        switch (cs.nch) {
          case 1: k_crt_pipe<1, 0><<<gp, 256, smem, s>>>(ca); break;
          case 2: k_crt_pipe<2, 0><<<gp, 256, smem, s>>>(ca); break;
          case 3: k_crt_pipe<3, 0><<<gp, 256, smem, s>>>(ca); break;
          default: k_crt_pipe<4, 0><<<gp, 256, smem, s>>>(ca); break;
        }
      }
      UW12_LAUNCHED();
      tm.stop();
      return;
    }
    switch (cs.nch * 2 + (reduce ? 1 : 0)) {
      case 2: k_crt<1, false><<<g, 256, 0, s>>>(ca); break;
      case 3: k_crt<1, true><<<g, 256, 0, s>>>(ca); break;
      case 4: k_crt<2, false><<<g, 256, 0, s>>>(ca); break;
      case 5: k_crt<2, true><<<g, 256, 0, s>>>(ca); break;
      case 6: k_crt<3, false><<<g, 256, 0, s>>>(ca); break;
      case 7: k_crt<3, true><<<g, 256, 0, s>>>(ca); break;
      case 8: k_crt<4, false><<<g, 256, 0, s>>>(ca); break;
      default: k_crt<4, true><<<g, 256, 0, s>>>(ca); break;
    }
    UW12_LAUNCHED();
    tm.stop();
  }
}

long long slab_bytes(long long L, long long m, long long n, long long k_total, long long nbatch,
                     long long planes_a, long long planes_b) {
  const long long k_pad = round_up(k_total, kTileK);
  const long long m_pad = round_up(m, kTileI), n_pad = round_up(n, kItemJ);
  const long long splits = std::max<long long>(1, (k_pad + kMaxKChunk - 1) / kMaxKChunk);
  return L * (planes_a * m_pad + planes_b * n_pad) * k_pad +
         std::max<long long>(splits, 4) * L * nbatch * m_pad * n_pad;
}

constexpr long long kSlabBudget = 8LL << 30;  // temporaries of one slab

// Splits the GEMM into slabs (batches, then rows i / columns j) whose
// temporaries stay within kSlabBudget, and runs each.
void run_slabs(const GemmDesc& d, const Consts& cs, int beta, cudaStream_t s) {
  const long long L = cs.L;
  const long long k_total = d.k * d.nbr1 * d.nbr2;
  auto planes = [](long long var1n, long long var2n) { return var1n * var2n; };
  // 1. batches: one bo2 at a time, then ranges of bo1
  if (d.nbo2 > 1 &&
      slab_bytes(L, d.m, d.n, k_total, d.nbo1 * d.nbo2,
                 planes(d.sAo1 ? d.nbo1 : 1, d.sAo2 ? d.nbo2 : 1),
                 planes(d.sBo1 ? d.nbo1 : 1, d.sBo2 ? d.nbo2 : 1)) > kSlabBudget) {
    for (long long b2 = 0; b2 < d.nbo2; ++b2) {
      GemmDesc e = d;
      e.nbo2 = 1;
      e.A += b2 * d.sAo2; e.B += b2 * d.sBo2; e.C += b2 * d.sCo2;
      e.sAo2 = e.sBo2 = e.sCo2 = 0;
      run_slabs(e, cs, beta, s);
    }
    return;
  }
  if (d.nbo1 > 1) {
    long long nb = d.nbo1;
    while (nb > 1 && slab_bytes(L, d.m, d.n, k_total, nb * d.nbo2, d.sAo1 ? nb : 1,
                                d.sBo1 ? nb : 1) > kSlabBudget)
      nb = (nb + 1) / 2;
    if (nb < d.nbo1) {
      for (long long b0 = 0; b0 < d.nbo1; b0 += nb) {
        GemmDesc e = d;
        e.nbo1 = std::min(nb, d.nbo1 - b0);
        e.A += b0 * d.sAo1; e.B += b0 * d.sBo1; e.C += b0 * d.sCo1;
        run_slabs(e, cs, beta, s);
      }
      return;
    }
  }
  const long long nbatch = d.nbo1 * d.nbo2;
  const long long pa = (d.sAo1 && d.nbo1 > 1 ? d.nbo1 : 1) * (d.sAo2 && d.nbo2 > 1 ? d.nbo2 : 1);
  const long long pb = (d.sBo1 && d.nbo1 > 1 ? d.nbo1 : 1) * (d.sBo2 && d.nbo2 > 1 ? d.nbo2 : 1);
  // 2. long contractions into a small output: when the operands' residues
  // exceed half the budget but the output's fit in the other half, K is cut
  // into consecutive ranges (reduction batches, else k) whose products are
  // reconstructed one after another and accumulated in C (beta = 1 after the
  // first); row / column slabs would prepare each operand once per slab of
  // the other.  A large output is cut into row / column slabs instead (each
  // K range would reconstruct all of it).
  const long long m_pad = round_up(d.m, kTileI), n_pad = round_up(d.n, kItemJ);
  const long long op_bytes = L * (pa * m_pad + pb * n_pad) * round_up(k_total, kTileK);
  const long long out_bytes = 4 * L * nbatch * m_pad * n_pad;
  if (op_bytes > kSlabBudget / 2 && out_bytes <= kSlabBudget / 2 && k_total > kTileK) {
    const long long pieces = (2 * op_bytes + kSlabBudget - 1) / kSlabBudget;
    const long long nred = d.nbr1 * d.nbr2;
    if (nred > 1) {
      // ranges of reduction batches (r1 fastest); one r2 at a time when nbr2 > 1
      if (d.nbr2 > 1) {
        for (long long r2 = 0; r2 < d.nbr2; ++r2) {
          GemmDesc e = d;
          e.nbr2 = 1;
          e.A += r2 * d.sAr2; e.B += r2 * d.sBr2;
          e.sAr2 = e.sBr2 = 0;
          if (r2 > 0) e.beta = 1.0;
          run_slabs(e, cs, beta, s);
        }
        return;
      }
      const long long per = std::max<long long>(1, (d.nbr1 + pieces - 1) / pieces);
      for (long long r0 = 0; r0 < d.nbr1; r0 += per) {
        GemmDesc e = d;
        e.nbr1 = std::min(per, d.nbr1 - r0);
        e.A += r0 * d.sAr1; e.B += r0 * d.sBr1;
        if (r0 > 0) e.beta = 1.0;
        run_slabs(e, cs, beta, s);
      }
      return;
    }
    const long long kc = round_up((d.k + pieces - 1) / pieces, kTileK);
    if (kc < d.k) {
      for (long long k0 = 0; k0 < d.k; k0 += kc) {
        GemmDesc e = d;
        e.k = std::min(kc, d.k - k0);
        e.A += k0 * (d.a_kcontig ? 1 : d.lda);
        e.B += k0 * (d.b_ncontig ? d.ldb : 1);
        if (k0 > 0) e.beta = 1.0;
        run_slabs(e, cs, beta, s);
      }
      return;
    }
  }
  // 3. rows i / columns j
  long long ms = m_pad, ns = n_pad;
  while (slab_bytes(L, ms, ns, k_total, nbatch, pa, pb) > kSlabBudget) {
    if (ms >= ns && ms > kTileI)
      ms = round_up(ms / 2, kTileI);
    else if (ns > kItemJ)
      ns = round_up(ns / 2, kItemJ);
    else
      break;
  }
  for (long long i0 = 0; i0 < d.m; i0 += ms)
    for (long long j0 = 0; j0 < d.n; j0 += ns) {
      GemmDesc e = d;
      e.m = std::min(ms, d.m - i0);
      e.n = std::min(ns, d.n - j0);
      e.A += i0 * (d.a_kcontig ? d.lda : 1);
      e.B += j0 * (d.b_ncontig ? 1 : d.ldb);
      e.C += i0 + j0 * d.ldc;
      run_core(e, cs, beta, s);
    }
}

}  // namespace

void set_split_moduli(int n_moduli) {
  if (n_moduli < 0 || n_moduli > kOzakiMaxModuli)
    throw Error(kErrInvalid, "number of split-precision moduli must be 0..16");
  g_split_moduli = n_moduli;
}

int split_moduli() { return g_split_moduli; }

void set_split_min_flops(double flops) {
  if (!(flops >= 0.0)) throw Error(kErrInvalid, "split-precision threshold must be >= 0");
  g_split_min_flops = flops;
}

double split_min_flops() { return g_split_min_flops; }

int ozaki_bits(int n_moduli, long long k_total) {
  const Consts& cs = consts_for(n_moduli);
  const double kb = std::ceil(std::log2(double(std::max<long long>(k_total, 1))));
  const int beta = static_cast<int>(std::floor((cs.log2_m - 2.0 - kb) / 2.0));
  return std::min(beta, 50);  // |A'| <= 2^50: the FP64 rounding tricks stay exact
}

#ifndef UW12_COST_FP64_TFS
#define UW12_COST_FP64_TFS 26.0
#endif
#ifndef UW12_COST_PREP_TBS
#define UW12_COST_PREP_TBS 3.2
#endif
#ifndef UW12_COST_CRT_TBS
#define UW12_COST_CRT_TBS 2.0
#endif
#ifndef UW12_COST_I8_POPS
#define UW12_COST_I8_POPS 2.2
#endif

bool ozaki_profitable(const GemmDesc& d, int n_moduli) {
  // Estimated times on a B200 (fitted to measured kernels): operand
  // preparation streams each operand element twice in FP64 and writes L
  // residue bytes (UW12_COST_PREP_TBS TB/s); the CRT reads L residue bytes
  // (and C when beta != 0) and writes C (UW12_COST_CRT_TBS); the int8
  // products run at UW12_COST_I8_POPS; the FP64 DMMA GEMM at
  // UW12_COST_FP64_TFS TFLOP/s.  Split when it is clearly faster.
  const double L = double(n_moduli);
  const double k_total = double(d.k) * double(d.nbr1) * double(d.nbr2);
  const double nbatch = double(d.nbo1) * double(d.nbo2);
  const double pa = double(d.sAo1 && d.nbo1 > 1 ? d.nbo1 : 1) *
                    double(d.sAo2 && d.nbo2 > 1 ? d.nbo2 : 1);
  const double pb = double(d.sBo1 && d.nbo1 > 1 ? d.nbo1 : 1) *
                    double(d.sBo2 && d.nbo2 > 1 ? d.nbo2 : 1);
  const double m = double(d.m), n = double(d.n);
  const double flops = 2.0 * m * n * k_total * nbatch;
  const double t_fp64 = flops / (UW12_COST_FP64_TFS * 1e12);
  const double t_prep = (pa * m + pb * n) * k_total * (16.0 + L) / (UW12_COST_PREP_TBS * 1e12);
  const double t_crt = nbatch * m * n * (L + 8.0 + (d.beta != 0.0 ? 8.0 : 0.0)) /
                       (UW12_COST_CRT_TBS * 1e12);
  const double t_i8 = flops * L / (UW12_COST_I8_POPS * 1e15);
  return t_prep + t_crt + t_i8 + 30e-6 < 0.9 * t_fp64;
}

bool ozaki_supported(const GemmDesc& d) {
  const long long k_total = d.k * d.nbr1 * d.nbr2;
  return d.m <= (1LL << 30) && d.n <= (1LL << 30) && k_total <= 65535LL * kTileK &&
         d.nbo1 * d.nbo2 <= 65535;
}

void gemm_ozaki(const GemmDesc& d, int n_moduli) {
  if (n_moduli < 1 || n_moduli > kOzakiMaxModuli)
    throw Error(kErrInvalid, "number of split-precision moduli must be 1..16");
  if (d.m <= 0 || d.n <= 0 || d.nbo1 <= 0 || d.nbo2 <= 0) return;
  if (d.k <= 0 || d.nbr1 <= 0 || d.nbr2 <= 0) {
    gemm_dmma(d);  // C = beta C
    return;
  }
  if (!ozaki_supported(d)) throw Error(kErrInvalid, "split-precision GEMM: shape too large");
  const long long k_total = d.k * d.nbr1 * d.nbr2;
  const int beta = ozaki_bits(n_moduli, k_total);
  if (beta < 4)
    throw Error(kErrInvalid, "split-precision GEMM: too few moduli for a contraction of " +
                                 std::to_string(k_total) + " terms");
  cudaStream_t s = current_stream();
  const Consts& cs = consts_for(n_moduli);
  char shape[160];
  std::snprintf(shape, sizeof(shape), "split %lld %lld %lld %lld %lld L%d", d.m, d.n, d.k,
                d.nbo1 * d.nbo2, d.nbr1 * d.nbr2, n_moduli);
  Timer tm(kProfSplitGemm,
           2.0 * double(d.m) * double(d.n) * double(k_total) * double(d.nbo1 * d.nbo2), shape,
           s);
  run_slabs(d, cs, beta, s);
  tm.stop();
}

int set_error_slot(int slot) {
  const int prev = t_err_slot;
  t_err_slot = ((slot % kOzakiErrorSlots) + kOzakiErrorSlots) % kOzakiErrorSlots;
  return prev;
}

int ozaki_error_read_and_clear() {
  int* f = err_flag();
  cudaStream_t s = current_stream();
  int h = 0;
  UW12_CUDA(cudaMemcpyAsync(&h, f, sizeof(int), cudaMemcpyDeviceToHost, s));
  UW12_CUDA(cudaStreamSynchronize(s));
  if (h) UW12_CUDA(cudaMemsetAsync(f, 0, sizeof(int), s));
  return h;
}

}  // namespace uw12b
