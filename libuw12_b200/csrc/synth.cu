// Deterministic synthetic three-index tensors for benchmarks (see uw12_c.h,
// uw12c_synth_three_index).  Same counter-based formula as the Python test
// generator: key = mix(mix(seed) ^ tag); h_k = mix(key + 2e + k);
// g = sqrt(-2 ln u1) cos(2 pi u2); value = g * exp(-|p - q| / decay).
#include <algorithm>
#include <cmath>

#include "common.cuh"

namespace uw12b {

namespace {

__host__ __device__ __forceinline__ unsigned long long mix64(unsigned long long x) {
  unsigned long long z = x + 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

// Columns [first, first + count) of the tensor (rows x n_df), written with
// leading dimension ld; element e of the full tensor is e = r + rows * column.
// One thread per row (grid-stride), looping over the columns: the row's index
// pair and decay factor are computed once, and consecutive threads write
// consecutive rows of each column.
__global__ void k_synth(double* out, long long ld, int kind, long long n_ri, long long rows,
                        long long first, long long count, unsigned long long key,
                        double inv_decay) {
  const double two_pi = 6.283185307179586476925286766559;
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < rows;
       r += (long long)gridDim.x * blockDim.x) {
    long long p, q;
    if (kind == 0) {
      long long i = static_cast<long long>((sqrt(8.0 * double(r) + 1.0) - 1.0) * 0.5);
      while (i * (i + 1) / 2 > r) --i;
      while ((i + 1) * (i + 2) / 2 <= r) ++i;
      p = i;
      q = r - i * (i + 1) / 2;
    } else {
      p = r % n_ri;
      q = r / n_ri;
    }
    const long long d = p > q ? p - q : q - p;
    const double w = exp(-double(d) * inv_decay);
    for (long long col = 0; col < count; ++col) {
      const long long e = r + rows * (first + col);
      const unsigned long long base = key + 2ULL * static_cast<unsigned long long>(e);
      const unsigned long long h0 = mix64(base);
      const unsigned long long h1 = mix64(base + 1ULL);
      const double u1 = (static_cast<double>(h0 >> 11) + 1.0) * 0x1.0p-53;
      const double u2 = static_cast<double>(h1 >> 11) * 0x1.0p-53;
      const double g = sqrt(-2.0 * log(u1)) * cos(two_pi * u2);
      out[r + ld * col] = g * w;
    }
  }
}

}  // namespace

void synth_three_index_block(double* out, size_t ld, int kind, size_t n_ao, size_t n_ri,
                             size_t first, size_t count, unsigned long long seed,
                             unsigned long long tag, double decay, cudaStream_t stream) {
  if (kind != 0 && kind != 1) throw Error(kErrInvalid, "synth: kind must be 0 (AO) or 1 (RI)");
  if (!(decay > 0.0)) throw Error(kErrInvalid, "synth: decay must be positive");
  const long long rows = kind == 0 ? static_cast<long long>(n_ao * (n_ao + 1) / 2)
                                   : static_cast<long long>(n_ri * n_ao);
  if (ld < static_cast<size_t>(rows)) throw Error(kErrInvalid, "synth: ld smaller than the rows");
  if (rows <= 0 || count == 0) return;
  const unsigned long long key = mix64(mix64(seed) ^ tag);
  const long long blocks = std::min<long long>((rows + 255) / 256, 148LL * 32);
  k_synth<<<static_cast<unsigned>(blocks), 256, 0, stream>>>(
      out, static_cast<long long>(ld), kind, static_cast<long long>(n_ri), rows,
      static_cast<long long>(first), static_cast<long long>(count), key, 1.0 / decay);
  UW12_LAUNCHED();
}

void synth_three_index(double* out, int kind, size_t n_ao, size_t n_ri, size_t n_df,
                       unsigned long long seed, unsigned long long tag, double decay) {
  const size_t rows = kind == 0 ? n_ao * (n_ao + 1) / 2 : n_ri * n_ao;
  synth_three_index_block(out, rows, kind, n_ao, n_ri, 0, n_df, seed, tag, decay,
                          current_stream());
}

}  // namespace uw12b
