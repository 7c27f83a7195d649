// Streaming (HBM-bound) kernels of the UW12 schedule: packed-symmetric
// unpack/pack, diagonal scalings, strided copies, deterministic reductions
// and the permuted contractions of the same-spin energies.  All launch on
// current_stream().
#pragma once

#include "common.cuh"

namespace uw12b {

// out[i + ldo*j + so*c] = beta*out + alpha*S_c(i,j), S_c = square(P[:, c]) with
// P column-major (ldp), packed lower triangle row by row (idx = i(i+1)/2 + j).
void unpack_sym(const double* P, long long ldp, long long n, long long ncols, double* out,
                long long ldo, long long so, double alpha = 1.0, double beta = 0.0);

// d[idx(i,j)] = scale * (i != j ? 2 : 1) * sum_k C[i + ldc*k] C[j + ldc*k]
// (lower(scale * C C^T, 2) of libuw12's utils.hpp).
void pack_density(const double* C, long long ldc, long long n, long long nc, double scale,
                  double* d);

// Y[i + ldy*j] = alpha * r[i] * X[i + ldx*j] * c[j]   (r or c may be null = 1).
void scale_rc(const double* X, long long ldx, long long rows, long long cols, const double* r,
              const double* c, double alpha, double* Y, long long ldy);

// 3-D strided copy / scale: dst[i + d1*j + d2*l] = alpha * src[i + s1*j + s2*l]
// (+ beta * dst when beta != 0).
void copy3d(const double* src, long long s1, long long s2, double* dst, long long d1,
            long long d2, long long n0, long long n1, long long n2, double alpha = 1.0,
            double beta = 0.0);

// acc[slot] += coef * sum_{i<rows, j<cols} x[i + ldx*j] * y[i + ldy*j] * rw[i] * cw[j]
// (rw / cw may be null).  Two-pass, fixed-order reduction.
void wdot(const double* x, long long ldx, const double* y, long long ldy, long long rows,
          long long cols, const double* rw, const double* cw, double coef, double* acc, int slot);

// acc[slot] += coef * sum_{i,l<a; j,k<o} X[i + a*l + lda*(j + a*k)] * Y[i + a*k + lda*(j + a*l)]
// with lda = a*o: the same-spin four-electron energy over (ik|jl) blocks.
void permdot_4el(const double* X, const double* Y, long long a, long long o, double coef,
                 double* acc, int slot);

// acc[slot] += coef * sum_{p<rp; i,j<a; k in [k0,k1)} Y[p + rp*i + rp*a*(j + a*(k-k0))]
//                                                   * Z[p + rp*j + rp*a*(i + a*(k-k0))]
// the same-spin three-electron energy.
void permdot_3el(const double* Y, const double* Z, long long rp, long long a, long long kc,
                 double coef, double* acc, int slot);

// F[i + ld*j] = 0.5 * (G[i + ldg*j] + G[j + ldg*i]) written into column-block
// sigma of the output; F may alias nothing in G.
void symmetrise(const double* G, long long ldg, long long n, double* F, long long ldf);

// max |A - A^T| and max |A| into out[0], out[1] (device), n x n column-major.
void symmetry_stats(const double* A, long long lda, long long n, double* out);
// *out += sum of squares of the rows x cols block A (leading dimension lda), on s.
void sumsq_add(const double* A, long long lda, long long rows, long long cols, double* out,
               cudaStream_t s);

// Y = sum_q coefT[q]*T[q] - r[i]*c[j]*sum_q coefX[q]*X[q], M x M, q < nq <= 2.
void combine_y(double* Y, long long m, const double* const* T, const double* coefT,
               const double* const* X, const double* coefX, int nq, const double* r,
               const double* c);

// V[:, s] = w .* sum_q coef[s*ns + q] * U[:, q], columns of length m (ns <= 2).
void combine_vecs(const double* U, long long m, int ns, const double* coef, const double* w,
                  double* V);

// P2 = Q * diag(pinv(lambda)) with |lambda| <= tol -> 0; in place on Q (n x n).
void scale_pinv_cols(double* Q, long long n, const double* lambda, double tol);
// Y (m x n, contiguous) = sum_q coef_q M_q, the terms with scaled_q != 0
// multiplied elementwise by r_i c_j (r, c may be null); at most kMaxLincomb terms.
constexpr int kMaxLincomb = 8;
void lincomb(double* Y, long long m, long long n, int nt, const double* const* mats,
             const double* coefs, const int* scaled, const double* r, const double* c);
// Gradient with respect to packed symmetric storage: out[:, a] (ldo >= n(n+1)/2)
// = beta * out[:, a] + the packed sum of the n x n matrix G[:, :, a]
// (consecutive, n*n apart), G_ij + G_ji off the diagonal, G_ii on it.
void pack_sym_sum(const double* G, long long n, long long na, double* out, long long ldo,
                  double beta = 0.0);

// out[p + rp*i + rp*a*(j + a*k)] = alpha * Z[p + rp*j + rp*a*(i + a*k)] for
// p < rp, i, j < a, k < kc: the active-orbital pair of a same-spin
// three-electron product (YW or ZV, rp*a x a*kc) exchanged; out and Z distinct.
void perm_3el(const double* Z, double* out, long long rp, long long a, long long kc,
              double alpha);

// out[i + a*l + ao*(j + a*k)] = alpha * V[i + a*k + ao*(j + a*l)], ao = a*o:
// the occupied indices of an (ik|jl) matrix (ao x ao) exchanged between rows
// and columns; out and V distinct.
void perm_4el(const double* V, double* out, long long a, long long o, double alpha);

// A = I (n x n, column-major).
void set_identity(double* A, long long n);

// Gather columns: dst[:, q] = src[:, idx[q]] * s[q] (idx, s on device).
void gather_scale_cols(const double* src, long long rows, const int* idx, const double* s,
                       long long nq, double* dst);

}  // namespace uw12b
