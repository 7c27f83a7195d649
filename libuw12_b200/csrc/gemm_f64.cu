// FP64 DMMA GEMM for sm_100a: 128x128x16 CTA tiles, 8 warps of 64x32,
// 4-stage cp.async pipeline, m16n8k4 f64 tensor-core MMAs.
#include <algorithm>
#include <cmath>
#include <mutex>
#include <string>

#include "gemm_f64.cuh"

namespace uw12b {

namespace {

constexpr int BM = 128;
constexpr int BN = 128;
constexpr int BK = 16;
constexpr int STAGES = 4;
constexpr int THREADS = 256;
constexpr int LDW = 132;  // row length of [k][m] / [k][n] tiles (doubles); 132 % 16 == 4
constexpr int LDK = 20;   // row length of [m][k] / [n][k] tiles (doubles); 20 % 16 == 4
constexpr int A_STAGE = (BM * LDK > BK * LDW) ? BM * LDK : BK * LDW;  // 2560
constexpr int B_STAGE = A_STAGE;
constexpr size_t SMEM_BYTES = size_t(STAGES) * (A_STAGE + B_STAGE) * sizeof(double);

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
  long long tiles_m, tiles_mn;
  long long ktiles_pb, ktiles_total;
  int split;
};

__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void cp_async8(double* dst, const double* src, bool valid) {
  const int bytes = valid ? 8 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(smem_u32(dst)), "l"(src),
               "r"(bytes));
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

template <bool AK, bool BNC>
__global__ void __launch_bounds__(THREADS, 1) dgemm_dmma(const KParams p) {
  extern __shared__ __align__(16) double smem[];
  double* As = smem;
  double* Bs = smem + STAGES * A_STAGE;

  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  const int g = lane >> 2;  // groupID
  const int t = lane & 3;   // thread in group
  const int wm = (warp & 1) * 64;
  const int wn = (warp >> 1) * 32;

  long long bid = blockIdx.x;
  const long long tile = bid % p.tiles_mn;
  bid /= p.tiles_mn;
  const long long bo = bid % p.nbo;
  const int sp = static_cast<int>(bid / p.nbo);
  const long long tm = tile % p.tiles_m;
  const long long tn = tile / p.tiles_m;
  const long long m0 = tm * BM;
  const long long n0 = tn * BN;
  const long long bo1 = bo % p.nbo1;
  const long long bo2 = bo / p.nbo1;
  const double* Ab = p.A + bo1 * p.sAo1 + bo2 * p.sAo2;
  const double* Bb = p.B + bo1 * p.sBo1 + bo2 * p.sBo2;

  const long long kt_begin = p.ktiles_total * sp / p.split;
  const long long kt_end = p.ktiles_total * (sp + 1) / p.split;

  // Per-thread fixed coordinates of the tile loads (8 elements per operand).
  // A: [k][m] tile (m-contiguous global) or [m][k] tile (k-contiguous global).
  const int a_i0 = AK ? (tid >> 4) : (tid & 127);
  const int a_k0 = AK ? (tid & 15) : (tid >> 7);
  const int b_j0 = BNC ? (tid & 127) : (tid >> 4);
  const int b_k0 = BNC ? (tid >> 7) : (tid & 15);
  // Offsets of element r = 0 within a (batch, k-tile) block, and the step per r.
  const long long a_base = AK ? (a_k0 + p.lda * (m0 + a_i0)) : (m0 + a_i0 + p.lda * a_k0);
  const long long a_step = AK ? 16 * p.lda : 2 * p.lda;
  const long long a_kstep = AK ? BK : BK * p.lda;  // advance of one k-tile
  const long long b_base = BNC ? (n0 + b_j0 + p.ldb * b_k0) : (b_k0 + p.ldb * (n0 + b_j0));
  const long long b_step = BNC ? 2 * p.ldb : 16 * p.ldb;
  const long long b_kstep = BNC ? BK * p.ldb : BK;
  // Rows / columns this thread loads that lie inside the matrix (bit r).
  unsigned a_rows_ok = 0, b_cols_ok = 0;
#pragma unroll
  for (int r = 0; r < 8; ++r) {
    const long long gi = m0 + (AK ? a_i0 + 16 * r : a_i0);
    const long long gj = n0 + (BNC ? b_j0 : b_j0 + 16 * r);
    a_rows_ok |= (gi < p.m ? 1u : 0u) << r;
    b_cols_ok |= (gj < p.n ? 1u : 0u) << r;
  }

  // Incremental (reduction batch, k offset) iterator of the next stage to load:
  // no integer division inside the main loop.
  long long it_kin, it_br1;
  const double* itA;
  const double* itB;
  {
    const long long br = kt_begin / p.ktiles_pb;
    it_kin = (kt_begin - br * p.ktiles_pb) * BK;
    it_br1 = br % p.nbr1;
    const long long br2 = br / p.nbr1;
    itA = Ab + it_br1 * p.sAr1 + br2 * p.sAr2 + (it_kin / BK) * a_kstep;
    itB = Bb + it_br1 * p.sBr1 + br2 * p.sBr2 + (it_kin / BK) * b_kstep;
  }
  const long long k_pad = p.ktiles_pb * BK;

  auto load_stage = [&](int slot) {
    double* as = As + slot * A_STAGE;
    double* bs = Bs + slot * B_STAGE;
    const double* pa = itA + a_base;
#pragma unroll
    for (int r = 0; r < 8; ++r) {
      const int i = AK ? a_i0 + 16 * r : a_i0;
      const int kk = AK ? a_k0 : a_k0 + 2 * r;
      const bool v = ((a_rows_ok >> r) & 1u) && (it_kin + kk < p.k);
      double* dst = AK ? as + i * LDK + kk : as + kk * LDW + i;
      cp_async8(dst, v ? pa + r * a_step : p.A, v);
    }
    const double* pb = itB + b_base;
#pragma unroll
    for (int r = 0; r < 8; ++r) {
      const int j = BNC ? b_j0 : b_j0 + 16 * r;
      const int kk = BNC ? b_k0 + 2 * r : b_k0;
      const bool v = ((b_cols_ok >> r) & 1u) && (it_kin + kk < p.k);
      double* dst = BNC ? bs + kk * LDW + j : bs + j * LDK + kk;
      cp_async8(dst, v ? pb + r * b_step : p.B, v);
    }
    // advance to the next k-tile / reduction batch
    it_kin += BK;
    itA += a_kstep;
    itB += b_kstep;
    if (it_kin >= k_pad) {
      const long long back = p.ktiles_pb;
      it_kin = 0;
      itA += p.sAr1 - back * a_kstep;
      itB += p.sBr1 - back * b_kstep;
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

  for (long long kt = kt_begin; kt < kt_end; ++kt) {
    cp_async_wait<STAGES - 2>();
    __syncthreads();
    {
      const long long nxt = kt + STAGES - 1;
      if (nxt < kt_end) load_stage(static_cast<int>((nxt - kt_begin) % STAGES));
      cp_async_commit();
    }
    const int slot = static_cast<int>((kt - kt_begin) % STAGES);
    const double* as = As + slot * A_STAGE;
    const double* bs = Bs + slot * B_STAGE;
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
  }
  cp_async_wait<0>();

  // Epilogue.
  if (p.split == 1) {
    double* Cb = p.C + bo1 * p.sCo1 + bo2 * p.sCo2;
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
            double* dst = Cb + r + p.ldc * c;
            const double v = p.alpha * acc[mi][ni][2 * h + q];
            *dst = (p.beta == 0.0) ? v : v + p.beta * (*dst);
          }
        }
  } else {
    double* Wb = p.work + (static_cast<long long>(sp) * p.nbo + bo) * (p.m * p.n);
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
            Wb[r + p.m * c] = acc[mi][ni][2 * h + q];
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
// splits the contraction to fill the waves.  A split must keep >= 512 of k
// per CTA so the partial-tile round trip stays small against the MMA work.
int choose_split(long long ctas, long long ktiles_total) {
  constexpr long long kSMs = 148;
  auto eff = [&](long long c) {
    const long long waves = (c + kSMs - 1) / kSMs;
    return double(c) / double(waves * kSMs);
  };
  if (ctas >= 8 * kSMs) return 1;
  int best = 1;
  double best_eff = eff(ctas);
  for (int s = 2; s <= 64; ++s) {
    if (ktiles_total / s < 32) break;
    const double e = eff(ctas * s);
    if (e > best_eff + 0.05) {
      best = s;
      best_eff = e;
    }
  }
  return best;
}

template <bool AK, bool BNC>
void launch_variant(const KParams& p, long long grid, cudaStream_t s) {
  static bool attr_set[64] = {};
  int dev = 0;
  UW12_CUDA(cudaGetDevice(&dev));
  static std::mutex mu;
  {
    std::lock_guard<std::mutex> lk(mu);
    if (dev < 64 && !attr_set[dev]) {
      UW12_CUDA(cudaFuncSetAttribute(dgemm_dmma<AK, BNC>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     static_cast<int>(SMEM_BYTES)));
      attr_set[dev] = true;
    }
  }
  dgemm_dmma<AK, BNC><<<static_cast<unsigned>(grid), THREADS, SMEM_BYTES, s>>>(p);
  UW12_LAUNCHED();
}

// ---- profiling -------------------------------------------------------------
struct ProfRec {
  cudaEvent_t a, b;
  double flops;
};
std::mutex g_prof_mu;
bool g_prof_on = false;
std::vector<ProfRec> g_prof_recs;
KernelStats g_prof_acc;

void prof_collect_locked() {
  for (auto& r : g_prof_recs) {
    UW12_CUDA(cudaEventSynchronize(r.b));
    float ms = 0.f;
    UW12_CUDA(cudaEventElapsedTime(&ms, r.a, r.b));
    g_prof_acc.launches += 1;
    g_prof_acc.ms += ms;
    g_prof_acc.flops += r.flops;
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
  g_prof_acc = KernelStats{};
}

KernelStats profile_read_gemm() {
  std::lock_guard<std::mutex> lk(g_prof_mu);
  prof_collect_locked();
  return g_prof_acc;
}

void gemm(const GemmDesc& d) {
  const long long nbo = d.nbo1 * d.nbo2;
  const long long nbr = d.nbr1 * d.nbr2;
  if (d.m <= 0 || d.n <= 0 || nbo <= 0) return;
  cudaStream_t s = current_stream();
  if (d.k <= 0 || nbr <= 0) {
    if (d.beta == 1.0) return;
    const long long total = d.m * d.n * nbo;
    const int blocks = static_cast<int>(std::min<long long>((total + 255) / 256, 148LL * 16));
    scale_only<<<blocks, 256, 0, s>>>(d.m, d.n, nbo, d.nbo1, d.beta, d.C, d.ldc, d.sCo1, d.sCo2);
    UW12_LAUNCHED();
    return;
  }
  if (!d.A || !d.B || !d.C) throw Error(kErrInvalid, "gemm: null operand");

  KParams p{};
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
  const long long tiles_n = (d.n + BN - 1) / BN;
  p.tiles_mn = p.tiles_m * tiles_n;
  p.ktiles_pb = (d.k + BK - 1) / BK;
  p.ktiles_total = p.ktiles_pb * nbr;

  const long long ctas = p.tiles_mn * nbo;
  int split = d.split;
  if (split <= 0) split = choose_split(ctas, p.ktiles_total);
  split = static_cast<int>(std::max<long long>(1, std::min<long long>(split, p.ktiles_total)));
  p.split = split;

  DevBuf work;
  if (split > 1) {
    work.alloc(static_cast<size_t>(split) * nbo * d.m * d.n, s);
    p.work = work.get();
  }

  cudaEvent_t ev_a = nullptr, ev_b = nullptr;
  bool prof = false;
  {
    std::lock_guard<std::mutex> lk(g_prof_mu);
    prof = g_prof_on;
  }
  if (prof) {
    UW12_CUDA(cudaEventCreate(&ev_a));
    UW12_CUDA(cudaEventCreate(&ev_b));
    UW12_CUDA(cudaEventRecord(ev_a, s));
  }

  const long long grid = ctas * split;
  if (!d.a_kcontig && !d.b_ncontig) launch_variant<false, false>(p, grid, s);
  else if (!d.a_kcontig && d.b_ncontig) launch_variant<false, true>(p, grid, s);
  else if (d.a_kcontig && !d.b_ncontig) launch_variant<true, false>(p, grid, s);
  else launch_variant<true, true>(p, grid, s);

  if (split > 1) {
    const long long total = d.m * d.n * nbo;
    const int blocks = static_cast<int>(std::min<long long>((total + 255) / 256, 148LL * 16));
    splitk_reduce<<<blocks, 256, 0, s>>>(p.work, split, d.m, d.n, nbo, d.nbo1, d.alpha, d.beta,
                                         d.C, d.ldc, d.sCo1, d.sCo2);
    UW12_LAUNCHED();
  }
  if (prof) {
    UW12_CUDA(cudaEventRecord(ev_b, s));
    std::lock_guard<std::mutex> lk(g_prof_mu);
    g_prof_recs.push_back({ev_a, ev_b, 2.0 * double(d.m) * double(d.n) * double(d.k) *
                                           double(nbo) * double(nbr)});
  }
}

// ---- allocation-free variant -------------------------------------------------
namespace {

// Kernel parameters and split-K factor of an allocation-free call (the same
// choice gemm() makes).  Returns false for an empty output; *empty_k is set
// when the contraction is empty (C = beta C).
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
  const long long tiles_n = (d.n + BN - 1) / BN;
  p.tiles_mn = p.tiles_m * tiles_n;
  p.ktiles_pb = (d.k + BK - 1) / BK;
  p.ktiles_total = p.ktiles_pb * nbr;
  const long long ctas = p.tiles_mn * nbo;
  int split = d.split;
  if (split <= 0) {
    constexpr long long kSMs = 148;
    split = 1;
    if (ctas < kSMs) {
      long long want = (kSMs + ctas - 1) / ctas;
      long long cap = std::max<long long>(1, p.ktiles_total / 8);  // >= 128 k per split
      split = static_cast<int>(std::min<long long>(std::min(want, cap), 64));
    }
  }
  p.split = static_cast<int>(std::max<long long>(1, std::min<long long>(split, p.ktiles_total)));
  return true;
}

void launch_scale_only(const GemmDesc& d, cudaStream_t s) {
  if (d.beta == 1.0) return;
  const long long nbo = d.nbo1 * d.nbo2;
  const long long total = d.m * d.n * nbo;
  const int blocks = static_cast<int>(std::min<long long>((total + 255) / 256, 148LL * 16));
  scale_only<<<blocks, 256, 0, s>>>(d.m, d.n, nbo, d.nbo1, d.beta, d.C, d.ldc, d.sCo1, d.sCo2);
  UW12_LAUNCHED();
}

// Launches the GEMM (and the split-K reduction when p.split > 1, with
// partial tiles in p.work).
void launch(const GemmDesc& d, const KParams& p, cudaStream_t s) {
  const long long grid = p.tiles_mn * p.nbo * p.split;
  if (!d.a_kcontig && !d.b_ncontig) launch_variant<false, false>(p, grid, s);
  else if (!d.a_kcontig && d.b_ncontig) launch_variant<false, true>(p, grid, s);
  else if (d.a_kcontig && !d.b_ncontig) launch_variant<true, false>(p, grid, s);
  else launch_variant<true, true>(p, grid, s);
  if (p.split > 1) {
    const long long total = d.m * d.n * p.nbo;
    const int blocks = static_cast<int>(std::min<long long>((total + 255) / 256, 148LL * 16));
    splitk_reduce<<<blocks, 256, 0, s>>>(p.work, p.split, d.m, d.n, p.nbo, d.nbo1, d.alpha,
                                         d.beta, d.C, d.ldc, d.sCo1, d.sCo2);
    UW12_LAUNCHED();
  }
}

}  // namespace

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
