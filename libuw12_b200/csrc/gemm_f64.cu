// FP64 DMMA GEMM for sm_100a: 128x128x16 CTA tiles, 8 warps of 64x32,
// 4-stage cp.async pipeline (16-byte copies when the operand allows it),
// grouped CTA raster for L2 reuse, m16n8k4 f64 tensor-core MMAs.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "gemm_f64.cuh"
#include "ozaki.cuh"

namespace uw12b {

namespace {

// k tile 16 with 4 stages measured 1.5% faster than 32 with 3 (and than 16
// with 5, 32 with 2) on a full evaluation with N = 500 AO, M = 1500 DF and
// R = 2000 RI functions; both are compile-time settings.
#ifndef UW12_DMMA_BK
#define UW12_DMMA_BK 16
#endif
#ifndef UW12_DMMA_STAGES
#define UW12_DMMA_STAGES 4
#endif
constexpr int BM = 128;
constexpr int BN = 128;
constexpr int BK = UW12_DMMA_BK;          // 16 or 32 (k extent of a pipeline stage)
constexpr int STAGES = UW12_DMMA_STAGES;  // stages in flight; shared memory <= 227 KiB
static_assert(BK == 16 || BK == 32, "k tile of 16 or 32");
constexpr int THREADS = 256;
constexpr int LDW = BM + 4;  // [k][m] / [k][n] tile rows (doubles); 132 % 16 == 4
constexpr int LDK = BK + 4;  // [m][k] / [n][k] tile rows (doubles); 20 (or 36) % 16 == 4, even
constexpr int STAGE_ELEMS = (BM * LDK > BK * LDW) ? BM * LDK : BK * LDW;  // 2560
constexpr size_t SMEM_BYTES = size_t(STAGES) * 2 * STAGE_ELEMS * sizeof(double);  // 160 KiB
static_assert(SMEM_BYTES <= 227 * 1024, "pipeline stages exceed shared memory");
constexpr int GROUP_N = 8;   // CTAs that run together share A panels across 8 n-tiles
constexpr long long kSMs = 148;

struct KParams {
  const double* A;
  const double* B;
  double* C;
  double* work;  // split > 1: partial tiles [split][nbo][m*n]
  long long lda, ldb, ldc;
  long long m, n, k;
  double alpha, beta;
  long long nbo1, nbo;
  long long sAo1, sAo2, sBo1, sBo2, sCo1, sCo2;
  long long nbr1;
  long long sAr1, sAr2, sBr1, sBr2;
  long long tiles_m, tiles_n, tiles_mn;
  long long ktiles_pb, ktiles_total;
  int split;
};

__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

// 8- or 16-byte asynchronous global -> shared copy; bytes beyond src_bytes
// are zero-filled (src_bytes = 0 reads nothing).
template <int BYTES>
__device__ __forceinline__ void cp_async(double* dst, const double* src, int src_bytes) {
  if (BYTES == 16)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_u32(dst)),
                 "l"(src), "r"(src_bytes));
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(smem_u32(dst)),
                 "l"(src), "r"(src_bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

__device__ __forceinline__ void dmma(double (&c)[4], double a0, double a1, double b0) {
  asm volatile(
      "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, "
      "{%0,%1,%2,%3};\n"
      : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
      : "d"(a0), "d"(a1), "d"(b0));
}

__device__ __forceinline__ void dmma16(double (&c)[4], const double (&a)[8], const double (&b)[4]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, "
      "{%4,%5,%6,%7,%8,%9,%10,%11}, {%12,%13,%14,%15}, {%0,%1,%2,%3};\n"
      : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
      : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(a[4]), "d"(a[5]), "d"(a[6]), "d"(a[7]),
        "d"(b[0]), "d"(b[1]), "d"(b[2]), "d"(b[3]));
}

// Loader of one operand tile (BK deep, 128 wide) into shared memory.
//   KC  : the operand is contiguous along k in global memory ([w][k] tile,
//         row LDK) -- otherwise along the 128-wide dimension ([k][w], row LDW);
//   VEC : copies of two consecutive doubles (16 bytes) along the contiguous
//         dimension; requires even leading dimension / offsets.
// Thread mapping: the contiguous index is the fastest-varying across threads.
template <bool KC, bool VEC>
struct TileLoader {
  static constexpr int W = VEC ? 2 : 1;                       // doubles per copy
  static constexpr int CONTIG = KC ? BK : 128;                // contiguous extent
  static constexpr int TPC = CONTIG / W;                      // threads along it
  static constexpr int OTHER_STEP = THREADS / TPC;            // other-dim stride
  static constexpr int OTHER = KC ? 128 : BK;                 // other extent
  static constexpr int COPIES = OTHER / OTHER_STEP;           // copies per thread

  int c0;   // contiguous index of this thread's first element
  int o0;   // other index of this thread's first copy

  __device__ __forceinline__ explicit TileLoader(int tid)
      : c0((tid % TPC) * W), o0(tid / TPC) {}

  // Element (w, kk) of the 128-wide x BK tile lives at global offset
  // w + ld*kk (not KC) or kk + ld*w (KC).
  __device__ __forceinline__ long long base(long long w0, long long ld) const {
    return KC ? (c0 + ld * (w0 + o0)) : (w0 + c0 + ld * o0);
  }
  __device__ __forceinline__ long long step(long long ld) const { return OTHER_STEP * ld; }
  __device__ __forceinline__ long long kstep(long long ld) const { return KC ? BK : BK * ld; }

  // Copies this thread's share of a tile.  wlim = extent left along the
  // 128-wide dimension from the tile start, klim = extent left along k.
  __device__ __forceinline__ void load(double* s, const double* g, const double* dummy,
                                       long long wlim, long long klim, long long ld) const {
#pragma unroll
    for (int r = 0; r < COPIES; ++r) {
      const int o = o0 + r * OTHER_STEP;
      const long long lim_c = KC ? klim : wlim;  // limit along the contiguous dim
      const long long lim_o = KC ? wlim : klim;  // limit along the other dim
      int bytes = 0;
      if (o < lim_o) {
        const long long left = lim_c - c0;
        bytes = left >= W ? 8 * W : (left > 0 ? 8 * static_cast<int>(left) : 0);
      }
      double* dst = KC ? s + o * LDK + c0 : s + o * LDW + c0;
      const double* src = bytes ? g + r * OTHER_STEP * ld : dummy;
      cp_async<8 * W>(dst, src, bytes);
    }
  }
};

template <bool AK, bool BNC, bool VA, bool VB>
__global__ void __launch_bounds__(THREADS, 1) dgemm_dmma(const KParams p) {
  extern __shared__ __align__(16) double smem[];
  double* As = smem;
  double* Bs = smem + STAGES * STAGE_ELEMS;

  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  const int g = lane >> 2;  // groupID
  const int t = lane & 3;   // thread in group
  const int wm = (warp & 1) * 64;
  const int wn = (warp >> 1) * 32;

  // Block -> (tile, output batch, split).  Tiles are visited in groups of
  // GROUP_N n-tiles, m-tile outermost inside a group, so the ~148 CTAs that
  // run at once touch a few A panels and GROUP_N B panels.
  long long bid = blockIdx.x;
  const long long tile = bid % p.tiles_mn;
  bid /= p.tiles_mn;
  const long long bo = bid % p.nbo;
  const int sp = static_cast<int>(bid / p.nbo);
  const long long per_group = p.tiles_m * GROUP_N;
  const long long grp = tile / per_group;
  const long long gn0 = grp * GROUP_N;
  const long long gsize = (p.tiles_n - gn0) < GROUP_N ? (p.tiles_n - gn0) : GROUP_N;
  const long long local = tile - grp * per_group;
  const long long tn = gn0 + local % gsize;
  const long long tm = local / gsize;
  const long long m0 = tm * BM;
  const long long n0 = tn * BN;
  const long long bo1 = bo % p.nbo1;
  const long long bo2 = bo / p.nbo1;
  const double* Ab = p.A + bo1 * p.sAo1 + bo2 * p.sAo2;
  const double* Bb = p.B + bo1 * p.sBo1 + bo2 * p.sBo2;

  const long long kt_begin = p.ktiles_total * sp / p.split;
  const long long kt_end = p.ktiles_total * (sp + 1) / p.split;

  const TileLoader<AK, VA> la(tid);
  const TileLoader<!BNC, VB> lb(tid);
  const long long a_base = la.base(m0, p.lda);
  const long long b_base = lb.base(n0, p.ldb);
  const long long a_kstep = la.kstep(p.lda);
  const long long b_kstep = lb.kstep(p.ldb);
  const long long a_wlim = p.m - m0;
  const long long b_wlim = p.n - n0;

  // Incremental (reduction batch, k offset) iterator of the next stage to
  // load: no integer division inside the main loop.
  long long it_kin, it_br1;
  const double* itA;
  const double* itB;
  {
    const long long br = kt_begin / p.ktiles_pb;
    const long long kt_in = kt_begin - br * p.ktiles_pb;
    it_kin = kt_in * BK;
    it_br1 = br % p.nbr1;
    const long long br2 = br / p.nbr1;
    itA = Ab + it_br1 * p.sAr1 + br2 * p.sAr2 + kt_in * a_kstep;
    itB = Bb + it_br1 * p.sBr1 + br2 * p.sBr2 + kt_in * b_kstep;
  }
  const long long k_pad = p.ktiles_pb * BK;

  auto load_stage = [&](int slot) {
    const long long klim = p.k - it_kin;
    la.load(As + slot * STAGE_ELEMS, itA + a_base, p.A, a_wlim, klim, p.lda);
    lb.load(Bs + slot * STAGE_ELEMS, itB + b_base, p.B, b_wlim, klim, p.ldb);
    it_kin += BK;
    itA += a_kstep;
    itB += b_kstep;
    if (it_kin >= k_pad) {
      it_kin = 0;
      itA += p.sAr1 - p.ktiles_pb * a_kstep;
      itB += p.sBr1 - p.ktiles_pb * b_kstep;
      if (++it_br1 == p.nbr1) {
        it_br1 = 0;
        itA += p.sAr2 - p.nbr1 * p.sAr1;
        itB += p.sBr2 - p.nbr1 * p.sBr1;
      }
    }
  };

  double acc[4][4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b)
#pragma unroll
      for (int c = 0; c < 4; ++c) acc[a][b][c] = 0.0;

#pragma unroll
  for (int s = 0; s < STAGES - 1; ++s) {
    if (kt_begin + s < kt_end) load_stage(s);
    cp_async_commit();
  }

  int slot = 0;
  int load_slot = STAGES - 1;
  for (long long kt = kt_begin; kt < kt_end; ++kt) {
    cp_async_wait<STAGES - 2>();
    __syncthreads();
    if (kt + STAGES - 1 < kt_end) load_stage(load_slot);
    cp_async_commit();
    load_slot = (load_slot + 1 == STAGES) ? 0 : load_slot + 1;

    const double* as = As + slot * STAGE_ELEMS;
    const double* bs = Bs + slot * STAGE_ELEMS;
#if UW12_DMMA_K16
    // m16n8k16: A fragment element q sits at row g + 8 (q & 1), k = t + 4 (q >> 1);
    // B fragment element q at k = t + 4 q, column g.
#pragma unroll
    for (int kh = 0; kh < BK / 16; ++kh) {
      double bf[4][4];
#pragma unroll
      for (int ni = 0; ni < 4; ++ni) {
        const int col = wn + ni * 8 + g;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int kk = kh * 16 + t + 4 * q;
          bf[ni][q] = BNC ? bs[kk * LDW + col] : bs[col * LDK + kk];
        }
      }
#pragma unroll
      for (int mi = 0; mi < 4; ++mi) {
        double af[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const int row = wm + mi * 16 + g + 8 * (q & 1);
          const int kk = kh * 16 + t + 4 * (q >> 1);
          af[q] = AK ? as[row * LDK + kk] : as[kk * LDW + row];
        }
#pragma unroll
        for (int ni = 0; ni < 4; ++ni) dmma16(acc[mi][ni], af, bf[ni]);
      }
    }
#else
#pragma unroll
    for (int kq = 0; kq < BK / 4; ++kq) {
      const int kk = kq * 4 + t;
      double af[4][2], bf[4];
#pragma unroll
      for (int mi = 0; mi < 4; ++mi) {
        const int row = wm + mi * 16 + g;
        af[mi][0] = AK ? as[row * LDK + kk] : as[kk * LDW + row];
        af[mi][1] = AK ? as[(row + 8) * LDK + kk] : as[kk * LDW + row + 8];
      }
#pragma unroll
      for (int ni = 0; ni < 4; ++ni) {
        const int col = wn + ni * 8 + g;
        bf[ni] = BNC ? bs[kk * LDW + col] : bs[col * LDK + kk];
      }
#pragma unroll
      for (int mi = 0; mi < 4; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni) dmma(acc[mi][ni], af[mi][0], af[mi][1], bf[ni]);
    }
#endif
    slot = (slot + 1 == STAGES) ? 0 : slot + 1;
  }
  cp_async_wait<0>();

  // Epilogue: C = alpha acc + beta C, or the raw partial tile for split-K.
  double* Cb = p.split == 1 ? p.C + bo1 * p.sCo1 + bo2 * p.sCo2
                            : p.work + (static_cast<long long>(sp) * p.nbo + bo) * (p.m * p.n);
  const long long ldc = p.split == 1 ? p.ldc : p.m;
#pragma unroll
  for (int mi = 0; mi < 4; ++mi)
#pragma unroll
    for (int ni = 0; ni < 4; ++ni)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const long long r = m0 + wm + mi * 16 + g + 8 * h;
        if (r >= p.m) continue;
#pragma unroll
        for (int q = 0; q < 2; ++q) {
          const long long c = n0 + wn + ni * 8 + 2 * t + q;
          if (c >= p.n) continue;
          double* dst = Cb + r + ldc * c;
          if (p.split == 1) {
            const double v = p.alpha * acc[mi][ni][2 * h + q];
            *dst = (p.beta == 0.0) ? v : v + p.beta * (*dst);
          } else {
            *dst = acc[mi][ni][2 * h + q];
          }
        }
      }
}

// C = alpha * sum_s work[s] + beta * C (fixed summation order).
__global__ void splitk_reduce(const double* __restrict__ work, int split, long long m, long long n,
                              long long nbo, long long nbo1, double alpha, double beta, double* C,
                              long long ldc, long long sCo1, long long sCo2) {
  const long long total = m * n * nbo;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const long long mn = m * n;
    const long long bo = idx / mn;
    const long long e = idx - bo * mn;
    const long long r = e % m, c = e / m;
    double s = 0.0;
    for (int q = 0; q < split; ++q) s += work[(q * nbo + bo) * mn + e];
    double* dst = C + (bo % nbo1) * sCo1 + (bo / nbo1) * sCo2 + r + ldc * c;
    const double v = alpha * s;
    *dst = (beta == 0.0) ? v : v + beta * (*dst);
  }
}

// C = beta * C for an empty contraction.
__global__ void scale_only(long long m, long long n, long long nbo, long long nbo1, double beta,
                           double* C, long long ldc, long long sCo1, long long sCo2) {
  const long long total = m * n * nbo;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const long long mn = m * n;
    const long long bo = idx / mn;
    const long long e = idx - bo * mn;
    double* dst = C + (bo % nbo1) * sCo1 + (bo / nbo1) * sCo2 + (e % m) + ldc * (e / m);
    *dst = (beta == 0.0) ? 0.0 : beta * (*dst);
  }
}

// Split-K factor: the CTAs of one launch run in waves of 148 (one per SM), so
// a launch with few output tiles, or with a last wave that is mostly empty,
// splits the contraction to fill the waves.  A split keeps >= 512 of k per
// CTA so the partial-tile round trip stays small against the MMA work.
int choose_split(long long ctas, long long ktiles_total) {
  auto eff = [&](long long c) {
    const long long waves = (c + kSMs - 1) / kSMs;
    return double(c) / double(waves * kSMs);
  };
  if (ctas >= 8 * kSMs) return 1;
  int best = 1;
  double best_eff = eff(ctas);
  for (int s = 2; s <= 64; ++s) {
    if (ktiles_total / s < 512 / BK) break;
    const double e = eff(ctas * s);
    if (e > best_eff + 0.05) {
      best = s;
      best_eff = e;
    }
  }
  return best;
}

// A 16-byte copy needs the operand base, leading dimension and every batch
// stride to be even (in doubles); tile origins are multiples of 32.
bool vec_ok(const double* base, long long ld, long long s1, long long s2, long long s3,
            long long s4) {
  return (reinterpret_cast<std::uintptr_t>(base) % 16 == 0) && (ld % 2 == 0) && (s1 % 2 == 0) &&
         (s2 % 2 == 0) && (s3 % 2 == 0) && (s4 % 2 == 0);
}

template <bool AK, bool BNC, bool VA, bool VB>
void launch_kernel(const KParams& p, long long grid, cudaStream_t s) {
  static bool attr_set[64] = {};
  static std::mutex mu;
  int dev = 0;
  UW12_CUDA(cudaGetDevice(&dev));
  {
    std::lock_guard<std::mutex> lk(mu);
    if (dev < 64 && !attr_set[dev]) {
      UW12_CUDA(cudaFuncSetAttribute(dgemm_dmma<AK, BNC, VA, VB>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     static_cast<int>(SMEM_BYTES)));
      attr_set[dev] = true;
    }
  }
  dgemm_dmma<AK, BNC, VA, VB><<<static_cast<unsigned>(grid), THREADS, SMEM_BYTES, s>>>(p);
  UW12_LAUNCHED();
}

template <bool AK, bool BNC>
void launch_layout(const KParams& p, bool va, bool vb, long long grid, cudaStream_t s) {
  if (va && vb) launch_kernel<AK, BNC, true, true>(p, grid, s);
  else if (va) launch_kernel<AK, BNC, true, false>(p, grid, s);
  else if (vb) launch_kernel<AK, BNC, false, true>(p, grid, s);
  else launch_kernel<AK, BNC, false, false>(p, grid, s);
}

// Fills the kernel parameters and chooses the split-K factor.  Returns false
// for an empty output; *empty_k is set when the contraction is empty
// (C = beta C).
bool prepare(const GemmDesc& d, KParams& p, bool* empty_k) {
  const long long nbo = d.nbo1 * d.nbo2;
  const long long nbr = d.nbr1 * d.nbr2;
  *empty_k = false;
  if (d.m <= 0 || d.n <= 0 || nbo <= 0) return false;
  if (d.k <= 0 || nbr <= 0) {
    *empty_k = true;
    return true;
  }
  if (!d.A || !d.B || !d.C) throw Error(kErrInvalid, "gemm: null operand");
  p = KParams{};
  p.A = d.A; p.B = d.B; p.C = d.C;
  p.lda = d.lda; p.ldb = d.ldb; p.ldc = d.ldc;
  p.m = d.m; p.n = d.n; p.k = d.k;
  p.alpha = d.alpha; p.beta = d.beta;
  p.nbo1 = d.nbo1; p.nbo = nbo;
  p.sAo1 = d.sAo1; p.sAo2 = d.sAo2; p.sBo1 = d.sBo1; p.sBo2 = d.sBo2;
  p.sCo1 = d.sCo1; p.sCo2 = d.sCo2;
  p.nbr1 = d.nbr1;
  p.sAr1 = d.sAr1; p.sAr2 = d.sAr2; p.sBr1 = d.sBr1; p.sBr2 = d.sBr2;
  p.tiles_m = (d.m + BM - 1) / BM;
  p.tiles_n = (d.n + BN - 1) / BN;
  p.tiles_mn = p.tiles_m * p.tiles_n;
  p.ktiles_pb = (d.k + BK - 1) / BK;
  p.ktiles_total = p.ktiles_pb * nbr;
  int split = d.split;
  if (split <= 0) split = choose_split(p.tiles_mn * nbo, p.ktiles_total);
  p.split = static_cast<int>(std::max<long long>(1, std::min<long long>(split, p.ktiles_total)));
  return true;
}

void launch_scale_only(const GemmDesc& d, cudaStream_t s) {
  if (d.beta == 1.0) return;
  const long long nbo = d.nbo1 * d.nbo2;
  const long long total = d.m * d.n * nbo;
  const int blocks = static_cast<int>(std::min<long long>((total + 255) / 256, kSMs * 16));
  scale_only<<<blocks, 256, 0, s>>>(d.m, d.n, nbo, d.nbo1, d.beta, d.C, d.ldc, d.sCo1, d.sCo2);
  UW12_LAUNCHED();
}

// Launches the GEMM (and the split-K reduction when p.split > 1, with
// partial tiles in p.work).
void launch(const GemmDesc& d, const KParams& p, cudaStream_t s) {
  const long long grid = p.tiles_mn * p.nbo * p.split;
  const bool va = vec_ok(d.A, d.lda, d.sAo1, d.sAo2, d.sAr1, d.sAr2);
  const bool vb = vec_ok(d.B, d.ldb, d.sBo1, d.sBo2, d.sBr1, d.sBr2);
  if (!d.a_kcontig && !d.b_ncontig) launch_layout<false, false>(p, va, vb, grid, s);
  else if (!d.a_kcontig && d.b_ncontig) launch_layout<false, true>(p, va, vb, grid, s);
  else if (d.a_kcontig && !d.b_ncontig) launch_layout<true, false>(p, va, vb, grid, s);
  else launch_layout<true, true>(p, va, vb, grid, s);
  if (p.split > 1) {
    const long long total = d.m * d.n * p.nbo;
    const int blocks = static_cast<int>(std::min<long long>((total + 255) / 256, kSMs * 16));
    splitk_reduce<<<blocks, 256, 0, s>>>(p.work, p.split, d.m, d.n, p.nbo, d.nbo1, d.alpha,
                                         d.beta, d.C, d.ldc, d.sCo1, d.sCo2);
    UW12_LAUNCHED();
  }
}

// ---- profiling -------------------------------------------------------------
struct ProfRec {
  cudaEvent_t a, b;
  double flops;
  std::string shape;  // "m n k nbo nbr split layout vec" for the per-launch log
  int kind;
};
std::mutex g_prof_mu;
bool g_prof_on = false;
std::vector<ProfRec> g_prof_recs;
KernelStats g_prof_acc[kProfKinds];

void prof_collect_locked() {
  for (auto& r : g_prof_recs) {
    UW12_CUDA(cudaEventSynchronize(r.b));
    float ms = 0.f;
    UW12_CUDA(cudaEventElapsedTime(&ms, r.a, r.b));
    KernelStats& acc = g_prof_acc[r.kind];
    acc.launches += 1;
    acc.ms += ms;
    acc.flops += r.flops;
    if (const char* path = std::getenv("UW12_PROFILE_LOG")) {
      if (FILE* f = std::fopen(path, "a")) {
        std::fprintf(f, "%.4f %s\n", ms, r.shape.c_str());
        std::fclose(f);
      }
    }
    cudaEventDestroy(r.a);
    cudaEventDestroy(r.b);
  }
  g_prof_recs.clear();
}

}  // namespace

void profile_enable(bool on) {
  std::lock_guard<std::mutex> lk(g_prof_mu);
  g_prof_on = on;
}

bool profile_enabled() {
  std::lock_guard<std::mutex> lk(g_prof_mu);
  return g_prof_on;
}

void profile_reset() {
  std::lock_guard<std::mutex> lk(g_prof_mu);
  prof_collect_locked();
  for (auto& a : g_prof_acc) a = KernelStats{};
}

KernelStats profile_read_gemm() { return profile_read_kind(kProfDgemm); }

KernelStats profile_read_kind(int kind) {
  std::lock_guard<std::mutex> lk(g_prof_mu);
  prof_collect_locked();
  return g_prof_acc[kind];
}

void profile_record(int kind, cudaEvent_t a, cudaEvent_t b, double work, std::string shape) {
  std::lock_guard<std::mutex> lk(g_prof_mu);
  g_prof_recs.push_back({a, b, work, std::move(shape), kind});
}

// ---- split-K autotuner ------------------------------------------------------
//
// choose_split's wave heuristic picks the split-K factor of a launch from its
// output CTA count alone.  The autotuner replaces it by measurement: a shape
// class is (output CTAs = tiles x output batches, power-of-two bucket of the
// k tiles over all reduction batches); in tuning mode the first automatic-split
// GEMM of a class not yet in the table is launched once with every candidate
// split (1, 2, 3, 4, 6, 8, 12, 16, 24, 32, 48, 64 while each CTA keeps >= 4 k
// tiles and the partial tiles stay within 256 MiB or the rule's), each timed with CUDA events on the current stream, and the fastest
// is recorded and launched last, so C holds its result.  Only GEMMs with
// beta = 0 are tuned (their repeated launches overwrite C); the others, and
// every GEMM in "use" mode, take the table's split for their class when it has
// one and the heuristic otherwise.  Output CTA counts of at least 8 waves never
// split and are not tuned.
namespace {
struct TuneKey {
  long long ctas;
  int kbucket;
  bool operator<(const TuneKey& o) const {
    return ctas != o.ctas ? ctas < o.ctas : kbucket < o.kbucket;
  }
};
struct TuneEntry {
  int split;
  double ms;
};
std::mutex g_tune_mu;
int g_tune_mode = 0;  // 0 off, 1 tune, 2 use
std::map<TuneKey, TuneEntry> g_tune;

int kbucket_of(long long ktiles_total) {
  int b = 0;
  while ((1LL << (b + 1)) <= ktiles_total) ++b;
  return b;
}

TuneKey tune_key(long long m, long long n, long long k, long long nbo, long long nbr) {
  const long long tiles = ((m + BM - 1) / BM) * ((n + BN - 1) / BN);
  return TuneKey{tiles * nbo, kbucket_of(((k + BK - 1) / BK) * nbr)};
}

// the table's split for p's class, or 0
int tuned_split(const KParams& p) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  if (g_tune_mode == 0) return 0;
  auto it = g_tune.find(TuneKey{p.tiles_mn * p.nbo, kbucket_of(p.ktiles_total)});
  return it == g_tune.end() ? 0 : it->second.split;
}

bool tuning_wanted(const GemmDesc& d, const KParams& p) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  if (g_tune_mode != 1 || d.split > 0 || d.beta != 0.0) return false;
  if (p.tiles_mn * p.nbo >= 8 * kSMs) return false;
  return g_tune.find(TuneKey{p.tiles_mn * p.nbo, kbucket_of(p.ktiles_total)}) == g_tune.end();
}

// Times every candidate split of d (beta = 0) on stream s, records the fastest
// for the class and leaves C with the result of a launch with it.
void tune_and_launch(const GemmDesc& d, KParams p, cudaStream_t s) {
  const int heuristic = choose_split(p.tiles_mn * p.nbo, p.ktiles_total);
  // a candidate's partial tiles stay within 2^25 doubles (256 MiB) or the
  // rule's own, so tuning needs no more memory than the evaluation around it
  const double per_split = double(p.nbo) * double(d.m) * double(d.n);
  const double cap = std::max(double(1LL << 25), per_split * heuristic);
  std::vector<int> cands;
  for (int c : {1, 2, 3, 4, 6, 8, 12, 16, 24, 32, 48, 64})
    if (c == 1 || (p.ktiles_total / c >= 4 && per_split * c <= cap)) cands.push_back(c);
  if (std::find(cands.begin(), cands.end(), heuristic) == cands.end()) cands.push_back(heuristic);
  struct Events {  // destroyed on every exit, a failed launch included
    cudaEvent_t a = nullptr, b = nullptr;
    ~Events() {
      if (a) cudaEventDestroy(a);
      if (b) cudaEventDestroy(b);
    }
  } ev;
  UW12_CUDA(cudaEventCreate(&ev.a));
  UW12_CUDA(cudaEventCreate(&ev.b));
  cudaEvent_t e0 = ev.a, e1 = ev.b;
  int best = heuristic;
  double best_ms = 1e300;
  for (int c : cands) {
    p.split = c;
    DevBuf work;
    if (c > 1) {
      work.alloc(static_cast<size_t>(c) * p.nbo * d.m * d.n, s);
      p.work = work.get();
    }
    launch(d, p, s);  // warm-up (caches, first-launch set-up)
    UW12_CUDA(cudaEventRecord(e0, s));
    launch(d, p, s);
    launch(d, p, s);
    UW12_CUDA(cudaEventRecord(e1, s));
    UW12_CUDA(cudaEventSynchronize(e1));
    float ms = 0.f;
    UW12_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    if (ms / 2.0 < best_ms) {
      best_ms = ms / 2.0;
      best = c;
    }
  }
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune[TuneKey{p.tiles_mn * p.nbo, kbucket_of(p.ktiles_total)}] = TuneEntry{best, best_ms};
  }
  p.split = best;
  DevBuf work;
  if (best > 1) {
    work.alloc(static_cast<size_t>(best) * p.nbo * d.m * d.n, s);
    p.work = work.get();
  }
  launch(d, p, s);
}
}  // namespace

void autotune_set(int mode, const char* path) {
  if (mode < 0 || mode > 2) throw Error(kErrInvalid, "autotune: mode must be 0, 1 or 2");
  std::map<TuneKey, TuneEntry> loaded;
  if (path && *path) {
    if (FILE* f = std::fopen(path, "r")) {
      char line[256];
      int lineno = 0;
      while (std::fgets(line, sizeof(line), f)) {
        ++lineno;
        if (line[0] == '#' || line[0] == '\n') continue;
        long long ctas = 0;
        int kb = 0, split = 0;
        double ms = 0.0;
        if (std::sscanf(line, "%lld %d %d %lf", &ctas, &kb, &split, &ms) != 4 || ctas <= 0 ||
            kb < 0 || kb > 62 || split < 1 || split > 64) {
          std::fclose(f);
          throw Error(kErrInvalid, std::string("autotune: malformed line ") +
                                       std::to_string(lineno) + " in " + path);
        }
        loaded[TuneKey{ctas, kb}] = TuneEntry{split, ms};
      }
      std::fclose(f);
    }
  }
  std::lock_guard<std::mutex> lk(g_tune_mu);
  for (const auto& kv : loaded) g_tune[kv.first] = kv.second;
  g_tune_mode = mode;
}

void autotune_save(const char* path) {
  if (!path || !*path) throw Error(kErrInvalid, "autotune: no path");
  std::lock_guard<std::mutex> lk(g_tune_mu);
  FILE* f = std::fopen(path, "w");
  if (!f) throw Error(kErrInvalid, std::string("autotune: cannot write ") + path);
  std::fprintf(f, "# output_ctas k_tile_bucket split ms\n");
  for (const auto& kv : g_tune)
    std::fprintf(f, "%lld %d %d %.6f\n", kv.first.ctas, kv.first.kbucket, kv.second.split,
                 kv.second.ms);
  std::fclose(f);
}

void autotune_clear() {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune.clear();
}

long long autotune_size() {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  return static_cast<long long>(g_tune.size());
}

int autotune_lookup(long long m, long long n, long long k, long long nbo, long long nbr) {
  if (m <= 0 || n <= 0 || k <= 0 || nbo <= 0 || nbr <= 0) return 0;
  std::lock_guard<std::mutex> lk(g_tune_mu);
  auto it = g_tune.find(tune_key(m, n, k, nbo, nbr));
  return it == g_tune.end() ? 0 : it->second.split;
}

void gemm(const GemmDesc& d) {
  const int L = split_moduli();
  if (L > 0) {
    const double flops = 2.0 * double(d.m) * double(d.n) * double(d.k) * double(d.nbo1) *
                         double(d.nbo2) * double(d.nbr1) * double(d.nbr2);
    const double min_flops = split_min_flops();
    if (flops >= min_flops && (min_flops == 0.0 || ozaki_profitable(d, L)) && ozaki_supported(d)) {
      gemm_ozaki(d, L);
      return;
    }
  }
  gemm_dmma(d);
}

void gemm_dmma(const GemmDesc& d) {
  KParams p;
  bool empty_k = false;
  if (!prepare(d, p, &empty_k)) return;
  cudaStream_t s = current_stream();
  if (empty_k) {
    launch_scale_only(d, s);
    return;
  }
  const bool prof = profile_enabled();
  if (d.split <= 0) {
    if (!prof && tuning_wanted(d, p)) {
      tune_and_launch(d, p, s);
      return;
    }
    if (const int t = tuned_split(p))
      p.split = static_cast<int>(std::min<long long>(t, p.ktiles_total));
  }
  DevBuf work;
  if (p.split > 1) {
    work.alloc(static_cast<size_t>(p.split) * p.nbo * d.m * d.n, s);
    p.work = work.get();
  }
  cudaEvent_t ev_a = nullptr, ev_b = nullptr;
  if (prof) {
    UW12_CUDA(cudaEventCreate(&ev_a));
    UW12_CUDA(cudaEventCreate(&ev_b));
    UW12_CUDA(cudaEventRecord(ev_a, s));
  }
  launch(d, p, s);
  if (prof) {
    UW12_CUDA(cudaEventRecord(ev_b, s));
    std::lock_guard<std::mutex> lk(g_prof_mu);
    char shape[256];
    std::snprintf(shape, sizeof(shape), "%lld %lld %lld %lld %lld %d %d%d %d%d", d.m, d.n, d.k,
                  p.nbo, d.nbr1 * d.nbr2, p.split, int(d.a_kcontig), int(d.b_ncontig),
                  int(vec_ok(d.A, d.lda, d.sAo1, d.sAo2, d.sAr1, d.sAr2)),
                  int(vec_ok(d.B, d.ldb, d.sBo1, d.sBo2, d.sBr1, d.sBr2)));
    g_prof_recs.push_back({ev_a, ev_b, 2.0 * double(d.m) * double(d.n) * double(d.k) *
                                           double(p.nbo) * double(d.nbr1 * d.nbr2),
                           shape, kProfDgemm});
  }
}

// ---- allocation-free variant -------------------------------------------------
//
// Split-K partial tiles normally live in a stream-ordered allocation.  For
// callers that must not allocate, they go into this fixed device array
// instead: every device that loads the library keeps it (16 MiB) until the
// process exits.  Host code cannot use the symbol itself as a pointer (it is a
// host-side shadow), so the device address is looked up once per device.
namespace {
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocScratchDoubles];

std::mutex g_scratch_mu;
double* g_scratch_ptr[64] = {};

double* noalloc_scratch_for_current_device() {
  int dev = 0;
  UW12_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) throw Error(kErrInvalid, "gemm_noalloc: device index out of range");
  std::lock_guard<std::mutex> lk(g_scratch_mu);
  if (!g_scratch_ptr[dev]) {
    void* ptr = nullptr;
    UW12_CUDA(cudaGetSymbolAddress(&ptr, g_noalloc_scratch));
    g_scratch_ptr[dev] = static_cast<double*>(ptr);
  }
  return g_scratch_ptr[dev];
}
}  // namespace

void gemm_noalloc(const GemmDesc& d) {
  KParams p;
  bool empty_k = false;
  if (!prepare(d, p, &empty_k)) return;
  cudaStream_t s = current_stream();
  if (empty_k) {
    launch_scale_only(d, s);
    return;
  }
  const double per_split = double(p.nbo) * double(d.m) * double(d.n);
  if (d.split > 1 && per_split * p.split > double(kNoAllocScratchDoubles))
    throw Error(kErrInvalid,
                "gemm_noalloc: split * batches * m * n = " +
                    std::to_string(static_cast<long long>(per_split * p.split)) +
                    " doubles exceeds the fixed scratch of " +
                    std::to_string(kNoAllocScratchDoubles) + " doubles (16 MiB)");
  if (p.split > 1 && per_split * p.split > double(kNoAllocScratchDoubles)) {
    // automatic split: shrink it until the partial tiles fit (split 1 needs none)
    p.split = static_cast<int>(std::max(1.0, std::floor(kNoAllocScratchDoubles / per_split)));
  }
  if (p.split > 1) p.work = noalloc_scratch_for_current_device();
  launch(d, p, s);
}

}  // namespace uw12b
