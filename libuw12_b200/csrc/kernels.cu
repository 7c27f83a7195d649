#include <algorithm>

#include "kernels.cuh"

namespace uw12b {

namespace {

constexpr int kT = 256;

inline int grid_for(long long total, int per_sm = 16) {
  const long long want = (total + kT - 1) / kT;
  return static_cast<int>(std::max<long long>(1, std::min<long long>(want, 148LL * per_sm)));
}

__device__ __forceinline__ long long tri(long long i) { return i * (i + 1) / 2; }

__global__ void k_unpack_sym(const double* __restrict__ P, long long ldp, long long n,
                             long long ncols, double* out, long long ldo, long long so,
                             double alpha, double beta) {
  const long long nn = n * n;
  const long long total = nn * ncols;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const long long c = idx / nn;
    const long long e = idx - c * nn;
    const long long i = e % n, j = e / n;
    const long long pi = (i >= j) ? tri(i) + j : tri(j) + i;
    const double v = alpha * P[pi + ldp * c];
    double* dst = out + i + ldo * j + so * c;
    *dst = (beta == 0.0) ? v : v + beta * (*dst);
  }
}

__global__ void k_pack_density(const double* __restrict__ C, long long ldc, long long n,
                               long long nc, double scale, double* d) {
  const long long total = tri(n);
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    // invert idx = i(i+1)/2 + j
    long long i = static_cast<long long>((sqrt(8.0 * double(idx) + 1.0) - 1.0) * 0.5);
    while (tri(i) > idx) --i;
    while (tri(i + 1) <= idx) ++i;
    const long long j = idx - tri(i);
    double s = 0.0;
    for (long long k = 0; k < nc; ++k) s += C[i + ldc * k] * C[j + ldc * k];
    d[idx] = scale * (i != j ? 2.0 : 1.0) * s;
  }
}

__global__ void k_scale_rc(const double* __restrict__ X, long long ldx, long long rows,
                           long long cols, const double* __restrict__ r,
                           const double* __restrict__ c, double alpha, double* Y, long long ldy) {
  const long long total = rows * cols;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const long long i = idx % rows, j = idx / rows;
    double v = alpha * X[i + ldx * j];
    if (r) v *= r[i];
    if (c) v *= c[j];
    Y[i + ldy * j] = v;
  }
}

__global__ void k_copy3d(const double* __restrict__ src, long long s1, long long s2, double* dst,
                         long long d1, long long d2, long long n0, long long n1, long long n2,
                         double alpha, double beta) {
  const long long total = n0 * n1 * n2;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const long long i = idx % n0;
    const long long rest = idx / n0;
    const long long j = rest % n1, l = rest / n1;
    double* d = dst + i + d1 * j + d2 * l;
    const double v = alpha * src[i + s1 * j + s2 * l];
    *d = beta != 0.0 ? v + beta * *d : v;
  }
}

// Block partial sums -> partials[blockIdx.x]; fixed tree order.
__device__ __forceinline__ double block_sum(double v) {
  __shared__ double sh[kT / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) sh[w] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0) {
    for (int q = 0; q < kT / 32; ++q) s += sh[q];
  }
  __syncthreads();
  return s;
}

__global__ void k_wdot(const double* __restrict__ x, long long ldx, const double* __restrict__ y,
                       long long ldy, long long rows, long long cols, const double* __restrict__ rw,
                       const double* __restrict__ cw, double* partials) {
  const long long total = rows * cols;
  double s = 0.0;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const long long i = idx % rows, j = idx / rows;
    double v = x[i + ldx * j] * y[i + ldy * j];
    if (rw) v *= rw[i];
    if (cw) v *= cw[j];
    s += v;
  }
  s = block_sum(s);
  if (threadIdx.x == 0) partials[blockIdx.x] = s;
}

__global__ void k_finish(const double* partials, int n, double coef, double* acc, int slot) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double s = 0.0;
    for (int q = 0; q < n; ++q) s += partials[q];
    acc[slot] += coef * s;
  }
}

__global__ void k_permdot_4el(const double* __restrict__ X, const double* __restrict__ Y,
                              long long a, long long o, double* partials) {
  const long long ao = a * o;
  const long long total = ao * ao;  // (i, l, j, k)
  double s = 0.0;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const long long row = idx % ao, col = idx / ao;  // row = i + a*l, col = j + a*k
    const long long i = row % a, l = row / a, j = col % a, k = col / a;
    s += X[row + ao * col] * Y[(i + a * k) + ao * (j + a * l)];
  }
  s = block_sum(s);
  if (threadIdx.x == 0) partials[blockIdx.x] = s;
}

// One warp per (i, j, k) triple, summing the contiguous p index.
__global__ void k_permdot_3el(const double* __restrict__ Yw, const double* __restrict__ Zv,
                              long long rp, long long a, long long kc, double* partials) {
  const long long triples = a * a * kc;
  const int lane = threadIdx.x & 31;
  const long long warp_global = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  const long long ra = rp * a;
  double s = 0.0;
  for (long long tix = warp_global; tix < triples; tix += nwarps) {
    const long long i = tix % a;
    const long long rest = tix / a;
    const long long j = rest % a, k = rest / a;
    const double* y = Yw + rp * i + ra * (j + a * k);
    const double* z = Zv + rp * j + ra * (i + a * k);
    for (long long p = lane; p < rp; p += 32) s += y[p] * z[p];
  }
  s = block_sum(s);
  if (threadIdx.x == 0) partials[blockIdx.x] = s;
}

__global__ void k_symmetrise(const double* __restrict__ G, long long ldg, long long n, double* F,
                             long long ldf) {
  const long long total = n * n;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const long long i = idx % n, j = idx / n;
    F[i + ldf * j] = 0.5 * (G[i + ldg * j] + G[j + ldg * i]);
  }
}

__global__ void k_symmetry_stats(const double* __restrict__ A, long long lda, long long n,
                                 double* partials) {
  const long long total = n * n;
  double dmax = 0.0, amax = 0.0;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const long long i = idx % n, j = idx / n;
    const double v = A[i + lda * j];
    dmax = fmax(dmax, fabs(v - A[j + lda * i]));
    amax = fmax(amax, fabs(v));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    dmax = fmax(dmax, __shfl_down_sync(0xffffffffu, dmax, o));
    amax = fmax(amax, __shfl_down_sync(0xffffffffu, amax, o));
  }
  __shared__ double sd[kT / 32], sa[kT / 32];
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) { sd[w] = dmax; sa[w] = amax; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double d = 0.0, a = 0.0;
    for (int q = 0; q < kT / 32; ++q) { d = fmax(d, sd[q]); a = fmax(a, sa[q]); }
    partials[2 * blockIdx.x] = d;
    partials[2 * blockIdx.x + 1] = a;
  }
}

__global__ void k_max_pairs(const double* partials, int n, double* out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double d = 0.0, a = 0.0;
    for (int q = 0; q < n; ++q) { d = fmax(d, partials[2 * q]); a = fmax(a, partials[2 * q + 1]); }
    out[0] = d;
    out[1] = a;
  }
}

struct CombineArgs {
  const double* T[2];
  const double* X[2];
  double cT[2];
  double cX[2];
};

__global__ void k_combine_y(double* Y, long long m, CombineArgs a, int nq,
                            const double* __restrict__ r, const double* __restrict__ c) {
  const long long total = m * m;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const long long i = idx % m, j = idx / m;
    double t = 0.0, x = 0.0;
    for (int q = 0; q < nq; ++q) {
      if (a.cT[q] != 0.0) t += a.cT[q] * a.T[q][idx];
      if (a.cX[q] != 0.0) x += a.cX[q] * a.X[q][idx];
    }
    Y[idx] = t - r[i] * c[j] * x;
  }
}

struct VecArgs {
  double coef[4];
};

__global__ void k_combine_vecs(const double* __restrict__ U, long long m, int ns, VecArgs a,
                               const double* __restrict__ w, double* V) {
  const long long total = m * ns;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const long long i = idx % m;
    const int s = static_cast<int>(idx / m);
    double v = 0.0;
    for (int q = 0; q < ns; ++q) v += a.coef[s * ns + q] * U[i + m * q];
    V[idx] = w[i] * v;
  }
}

struct LincombArgs {
  const double* M[kMaxLincomb];
  double coef[kMaxLincomb];
  int scaled[kMaxLincomb];
};

__global__ void k_lincomb(double* Y, long long m, long long n, int nt, LincombArgs a,
                          const double* __restrict__ r, const double* __restrict__ c) {
  const long long total = m * n;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const long long i = idx % m, j = idx / m;
    const double rc = (r ? r[i] : 1.0) * (c ? c[j] : 1.0);
    double plain = 0.0, sc = 0.0;
    for (int q = 0; q < nt; ++q) {
      if (a.coef[q] == 0.0) continue;
      if (a.scaled[q])
        sc += a.coef[q] * a.M[q][idx];
      else
        plain += a.coef[q] * a.M[q][idx];
    }
    Y[idx] = plain + rc * sc;
  }
}

// out[i(i+1)/2 + j, a] = G[i, j, a] + G[j, i, a] (j < i), G[i, i, a] (j = i):
// the gradient of a function of sq(x) with respect to the packed x.
__global__ void k_pack_sym_sum(const double* __restrict__ G, long long n, long long na,
                               double* out, long long ldo, double beta) {
  const long long np = n * (n + 1) / 2;
  const long long total = np * na;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const long long p = idx % np, a = idx / np;
    // row i of the packed index: i(i+1)/2 <= p < (i+1)(i+2)/2
    long long i = static_cast<long long>((sqrt(8.0 * double(p) + 1.0) - 1.0) * 0.5);
    while (i * (i + 1) / 2 > p) --i;
    while ((i + 1) * (i + 2) / 2 <= p) ++i;
    const long long j = p - i * (i + 1) / 2;
    const double* g = G + n * n * a;
    const double v = (i == j) ? g[i + n * i] : g[i + n * j] + g[j + n * i];
    double* o = out + p + ldo * a;
    *o = beta != 0.0 ? beta * *o + v : v;
  }
}

// out[p + rp*i + rp*a*(j + a*kk)] = alpha * Z[p + rp*j + rp*a*(i + a*kk)]:
// the two active-orbital indices of the same-spin three-electron products
// exchanged (the permutation under which YW and ZV are contracted).
__global__ void k_perm_3el(const double* __restrict__ Z, double* __restrict__ out,
                           long long rp, long long a, long long kc, double alpha) {
  const long long total = rp * a * a * kc;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const long long p = idx % rp;
    long long t = idx / rp;
    const long long i = t % a;
    t /= a;
    const long long j = t % a;
    const long long kk = t / a;
    out[idx] = alpha * Z[p + rp * (j + a * (i + a * kk))];
  }
}

// out[i + a*l + ao*(j + a*k)] = alpha * V[i + a*k + ao*(j + a*l)], ao = a*o:
// the occupied indices of rows and columns of (ik|jl) exchanged.
__global__ void k_perm_4el(const double* __restrict__ V, double* __restrict__ out,
                           long long a, long long o, double alpha) {
  const long long ao = a * o, total = ao * ao;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const long long i = idx % a;
    long long t = idx / a;
    const long long l = t % o;
    t /= o;
    const long long j = t % a;
    const long long k = t / a;
    out[idx] = alpha * V[i + a * k + ao * (j + a * l)];
  }
}

__global__ void k_scale_pinv_cols(double* Q, long long n, const double* __restrict__ lam,
                                  double tol) {
  const long long total = n * n;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const long long j = idx / n;
    const double l = lam[j];
    Q[idx] = (fabs(l) > tol) ? Q[idx] / l : 0.0;
  }
}

__global__ void k_set_identity(double* A, long long n) {
  const long long total = n * n;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x)
    A[idx] = (idx % n == idx / n) ? 1.0 : 0.0;
}

__global__ void k_gather_scale_cols(const double* __restrict__ src, long long rows,
                                    const int* __restrict__ idxv, const double* __restrict__ s,
                                    long long nq, double* dst) {
  const long long total = rows * nq;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const long long i = idx % rows, q = idx / rows;
    dst[idx] = src[i + rows * idxv[q]] * s[q];
  }
}

void finish_reduction(const double* partials, int n, double coef, double* acc, int slot,
                      cudaStream_t s) {
  k_finish<<<1, 32, 0, s>>>(partials, n, coef, acc, slot);
  UW12_LAUNCHED();
}

}  // namespace

void unpack_sym(const double* P, long long ldp, long long n, long long ncols, double* out,
                long long ldo, long long so, double alpha, double beta) {
  const long long total = n * n * ncols;
  if (total <= 0) return;
  k_unpack_sym<<<grid_for(total), kT, 0, current_stream()>>>(P, ldp, n, ncols, out, ldo, so,
                                                              alpha, beta);
  UW12_LAUNCHED();
}

void pack_density(const double* C, long long ldc, long long n, long long nc, double scale,
                  double* d) {
  const long long total = n * (n + 1) / 2;
  if (total <= 0) return;
  k_pack_density<<<grid_for(total), kT, 0, current_stream()>>>(C, ldc, n, nc, scale, d);
  UW12_LAUNCHED();
}

void scale_rc(const double* X, long long ldx, long long rows, long long cols, const double* r,
              const double* c, double alpha, double* Y, long long ldy) {
  const long long total = rows * cols;
  if (total <= 0) return;
  k_scale_rc<<<grid_for(total), kT, 0, current_stream()>>>(X, ldx, rows, cols, r, c, alpha, Y,
                                                            ldy);
  UW12_LAUNCHED();
}

void copy3d(const double* src, long long s1, long long s2, double* dst, long long d1,
            long long d2, long long n0, long long n1, long long n2, double alpha, double beta) {
  const long long total = n0 * n1 * n2;
  if (total <= 0) return;
  k_copy3d<<<grid_for(total), kT, 0, current_stream()>>>(src, s1, s2, dst, d1, d2, n0, n1, n2,
                                                          alpha, beta);
  UW12_LAUNCHED();
}

void wdot(const double* x, long long ldx, const double* y, long long ldy, long long rows,
          long long cols, const double* rw, const double* cw, double coef, double* acc,
          int slot) {
  const long long total = rows * cols;
  if (total <= 0 || coef == 0.0) return;
  cudaStream_t s = current_stream();
  const int blocks = grid_for(total, 4);
  DevBuf part(blocks, s);
  k_wdot<<<blocks, kT, 0, s>>>(x, ldx, y, ldy, rows, cols, rw, cw, part.get());
  UW12_LAUNCHED();
  finish_reduction(part.get(), blocks, coef, acc, slot, s);
}

void permdot_4el(const double* X, const double* Y, long long a, long long o, double coef,
                 double* acc, int slot) {
  const long long total = a * o * a * o;
  if (total <= 0 || coef == 0.0) return;
  cudaStream_t s = current_stream();
  const int blocks = grid_for(total, 4);
  DevBuf part(blocks, s);
  k_permdot_4el<<<blocks, kT, 0, s>>>(X, Y, a, o, part.get());
  UW12_LAUNCHED();
  finish_reduction(part.get(), blocks, coef, acc, slot, s);
}

void permdot_3el(const double* Y, const double* Z, long long rp, long long a, long long kc,
                 double coef, double* acc, int slot) {
  const long long triples = a * a * kc;
  if (triples <= 0 || rp <= 0 || coef == 0.0) return;
  cudaStream_t s = current_stream();
  const int blocks = grid_for(triples * 32, 8);
  DevBuf part(blocks, s);
  k_permdot_3el<<<blocks, kT, 0, s>>>(Y, Z, rp, a, kc, part.get());
  UW12_LAUNCHED();
  finish_reduction(part.get(), blocks, coef, acc, slot, s);
}

void symmetrise(const double* G, long long ldg, long long n, double* F, long long ldf) {
  const long long total = n * n;
  if (total <= 0) return;
  k_symmetrise<<<grid_for(total), kT, 0, current_stream()>>>(G, ldg, n, F, ldf);
  UW12_LAUNCHED();
}

void symmetry_stats(const double* A, long long lda, long long n, double* out) {
  cudaStream_t s = current_stream();
  const long long total = n * n;
  const int blocks = grid_for(std::max<long long>(total, 1), 4);
  DevBuf part(2 * blocks, s);
  k_symmetry_stats<<<blocks, kT, 0, s>>>(A, lda, n, part.get());
  UW12_LAUNCHED();
  k_max_pairs<<<1, 32, 0, s>>>(part.get(), blocks, out);
  UW12_LAUNCHED();
}

void combine_y(double* Y, long long m, const double* const* T, const double* coefT,
               const double* const* X, const double* coefX, int nq, const double* r,
               const double* c) {
  const long long total = m * m;
  if (total <= 0) return;
  CombineArgs a{};
  for (int q = 0; q < nq; ++q) {
    a.T[q] = T[q]; a.X[q] = X[q]; a.cT[q] = coefT[q]; a.cX[q] = coefX[q];
  }
  k_combine_y<<<grid_for(total), kT, 0, current_stream()>>>(Y, m, a, nq, r, c);
  UW12_LAUNCHED();
}

void combine_vecs(const double* U, long long m, int ns, const double* coef, const double* w,
                  double* V) {
  if (m <= 0) return;
  VecArgs a{};
  for (int q = 0; q < ns * ns; ++q) a.coef[q] = coef[q];
  k_combine_vecs<<<grid_for(m * ns), kT, 0, current_stream()>>>(U, m, ns, a, w, V);
  UW12_LAUNCHED();
}

void lincomb(double* Y, long long m, long long n, int nt, const double* const* mats,
             const double* coefs, const int* scaled, const double* r, const double* c) {
  const long long total = m * n;
  if (total <= 0) return;
  if (nt > kMaxLincomb) throw Error(kErrInvalid, "lincomb: too many terms");
  LincombArgs a{};
  for (int q = 0; q < nt; ++q) {
    a.M[q] = mats[q];
    a.coef[q] = coefs[q];
    a.scaled[q] = scaled ? scaled[q] : 0;
  }
  k_lincomb<<<grid_for(total), kT, 0, current_stream()>>>(Y, m, n, nt, a, r, c);
  UW12_LAUNCHED();
}

void pack_sym_sum(const double* G, long long n, long long na, double* out, long long ldo,
                  double beta) {
  const long long total = n * (n + 1) / 2 * na;
  if (total <= 0) return;
  k_pack_sym_sum<<<grid_for(total), kT, 0, current_stream()>>>(G, n, na, out, ldo, beta);
  UW12_LAUNCHED();
}

void perm_3el(const double* Z, double* out, long long rp, long long a, long long kc,
              double alpha) {
  const long long total = rp * a * a * kc;
  if (total <= 0) return;
  k_perm_3el<<<grid_for(total), kT, 0, current_stream()>>>(Z, out, rp, a, kc, alpha);
  UW12_LAUNCHED();
}

void perm_4el(const double* V, double* out, long long a, long long o, double alpha) {
  const long long total = a * o * a * o;
  if (total <= 0) return;
  k_perm_4el<<<grid_for(total), kT, 0, current_stream()>>>(V, out, a, o, alpha);
  UW12_LAUNCHED();
}

void scale_pinv_cols(double* Q, long long n, const double* lambda, double tol) {
  if (n <= 0) return;
  k_scale_pinv_cols<<<grid_for(n * n), kT, 0, current_stream()>>>(Q, n, lambda, tol);
  UW12_LAUNCHED();
}

void set_identity(double* A, long long n) {
  if (n <= 0) return;
  k_set_identity<<<grid_for(n * n), kT, 0, current_stream()>>>(A, n);
  UW12_LAUNCHED();
}

void gather_scale_cols(const double* src, long long rows, const int* idx, const double* s,
                       long long nq, double* dst) {
  if (rows * nq <= 0) return;
  k_gather_scale_cols<<<grid_for(rows * nq), kT, 0, current_stream()>>>(src, rows, idx, s, nq,
                                                                        dst);
  UW12_LAUNCHED();
}

// out += sum of squares of the rows x cols block A (leading dimension lda):
// grid-stride partial sums, a warp-shuffle and shared-memory block reduction,
// one atomic add per block (summation order not fixed).
__global__ void k_sumsq_add(const double* __restrict__ A, long long lda, long long rows,
                            long long cols, double* out) {
  __shared__ double part[32];
  const long long total = rows * cols;
  double acc = 0.0;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const long long c = e / rows, r = e - c * rows;
    const double x = A[r + lda * c];
    acc = fma(x, x, acc);
  }
  for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) part[warp] = acc;
  __syncthreads();
  if (warp == 0) {
    acc = lane < (int)(blockDim.x >> 5) ? part[lane] : 0.0;
    for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) atomicAdd(out, acc);
  }
}

void sumsq_add(const double* A, long long lda, long long rows, long long cols, double* out,
               cudaStream_t s) {
  const long long total = rows * cols;
  if (total <= 0) return;
  k_sumsq_add<<<grid_for(total, 4), kT, 0, s>>>(A, lda, rows, cols, out);
  UW12_LAUNCHED();
}

}  // namespace uw12b
