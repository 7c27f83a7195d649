// UW12 energy + Fock engine: device-resident integral handles and the
// pair-loop-free FP64 schedule of libuw12's form_fock (src/uw12.cpp:22-119).
#pragma once

#include <functional>
#include <string>
#include <vector>

#include "common.cuh"

namespace uw12b {

// Persistent device array (cudaMalloc / cudaFree, independent of streams).
class DeviceArray {
 public:
  DeviceArray() = default;
  explicit DeviceArray(size_t n) { alloc(n); }
  DeviceArray(const DeviceArray&) = delete;
  DeviceArray& operator=(const DeviceArray&) = delete;
  ~DeviceArray() { if (p_) cudaFree(p_); }
  void alloc(size_t n) {
    if (p_) cudaFree(p_);
    p_ = nullptr;
    n_ = n;
    if (n_) UW12_CUDA(cudaMalloc(reinterpret_cast<void**>(&p_), n_ * sizeof(double)));
  }
  double* get() const { return p_; }
  size_t size() const { return n_; }

 private:
  double* p_ = nullptr;
  size_t n_ = 0;
};

// BaseIntegrals built from stored tensors (base_integrals.cpp:282-303):
// J3_0 (Np x M, packed (mn|A)), J3_ri_0 ((R N) x M, row nu + R mu) and the
// metric eigendecomposition P2 = Q pinv(Lambda), df_vals = Lambda
// (base_integrals.cpp:155-166).
//
// Integral-direct mode (the store_ao / store_ri = false constructors,
// base_integrals.hpp:52-72): a tensor that is not stored has a producer that
// writes aux functions [first, first + count) as columns of `out` (device
// memory, leading dimension ld) on `stream`; every use asks it for the aux
// functions it needs.
using AuxProducer =
    std::function<void(size_t first, size_t count, double* out, size_t ld, cudaStream_t stream)>;

struct IntegralsHandle {
  int device = 0;
  size_t n_ao = 0, n_df = 0, n_ri = 0;
  DeviceArray J3_0, J3_ri_0, P2, lam;
  std::vector<double> lam_host;
  AuxProducer ao_fn, ri_fn;  // set when J3_0 / J3_ri_0 are not stored
};

// ABS+ projectors (ri_utils.hpp:45-74) stored as one (N+R) x (N+R) matrix
// S^-1 = V_k Lambda_k^-1 V_k^T over the kept eigenpairs, AO block first.
struct AbsHandle {
  int device = 0;
  size_t n_ao = 0, n_ri = 0, n_kept = 0;
  DeviceArray Sinv;
};

IntegralsHandle* integrals_create(const double* X3, const double* X2, const double* X3_ri,
                                  size_t n_ao, size_t n_df, size_t n_ri, bool device_mem);
// BaseIntegrals(J3, df_vals) (base_integrals.cpp:308-326): three-index
// integrals already in the metric eigenbasis; P2 = I, Lambda = df_vals, no RI.
IntegralsHandle* integrals_create_eigenbasis(const double* J3, const double* df_vals, size_t n_ao,
                                             size_t n_df, bool device_mem);
AbsHandle* abs_create(const double* S, size_t n_ao, size_t n_ri, bool device_mem);
// BaseIntegrals(two_index_fn, three_index_fn, three_index_ri_fn, ..., store_ao,
// store_ri) (base_integrals.hpp:52-72, base_integrals.cpp:40-186): the metric X2
// (n_df x n_df) is given, the three-index tensors come from producers; a stored
// tensor is produced once, here, an unstored one at every use.  ri_fn may be
// empty (no RI).
IntegralsHandle* integrals_create_producer(const double* X2, bool x2_device, AuxProducer ao_fn,
                                           AuxProducer ri_fn, size_t n_ao, size_t n_df,
                                           size_t n_ri, bool store_ao, bool store_ri);

struct FockRequest {
  const IntegralsHandle* W = nullptr;
  const IntegralsHandle* V = nullptr;
  const IntegralsHandle* WV = nullptr;
  const AbsHandle* abs = nullptr;
  int n_spin = 0;
  size_t n_ao = 0;
  std::vector<const double*> C;     // per spin: n_ao x n_orb[s], column-major (host)
  std::vector<size_t> ldc;          // leading dimension of each C block
  std::vector<size_t> n_orb;
  std::vector<const double*> occ;   // per spin: n_occ[s] values (host)
  std::vector<size_t> n_occ;
  std::vector<size_t> n_active;
  bool indirect = false;
  bool calc_fock = true;
  double s_os = 1.0, s_ss = 0.0;
  size_t print_level = 0;
  double* energy = nullptr;         // host scalar
  double* fock = nullptr;           // n_ao x (n_ao * n_spin); may be null
  bool fock_device = false;         // fock points to device memory
  double* terms = nullptr;          // host: {E2, E3, E4} or null
  size_t mem_budget = 0;            // bytes for chunked intermediates (0 = auto)
  size_t shard = 0, n_shards = 1;   // partial evaluation: this shard's share only
  // Sum over the shards of a device buffer (in place, ordered on `stream`),
  // called at the same points, with the same counts, on every shard; needed
  // when n_shards > 1.  Returns 0 on success.
  int (*allreduce)(double* data, size_t count, void* stream, void* user) = nullptr;
  void* allreduce_user = nullptr;
};

void form_fock(const FockRequest& rq);

// Reverse mode of form_fock: the gradient of its energy (the direct terms, and
// with rq.indirect the same-spin terms too) with respect to the stored
// integrals.  Any
// pointer may be null (that gradient is skipped); device or host memory per
// device_mem.  Layouts are those of the inputs: dJ3 packed
// n_ao(n_ao+1)/2 x n_df (both triangle halves of (mn|P) summed into the packed
// entry), dJ3_ri (n_ri n_ao) x n_df, dJ2 n_df x n_df symmetric.  The metric
// gradient is -J2^-1 G J2^-1 (no eigenvector derivatives), exact when no metric
// eigenvalue falls below the pseudo-inverse cut-off (1e-10).  The energy and
// Fock of rq are computed first.
// A consumer of a three-index gradient in aux blocks: columns [first, first +
// count) as a device block (leading dimension ld) on `stream`; the block may be
// overwritten by later work on that stream once the call returns.
using GradSink =
    std::function<void(size_t first, size_t count, const double* block, size_t ld, cudaStream_t)>;

struct AdjointOutputs {
  double* dJ3[3] = {nullptr, nullptr, nullptr};  // W, V, WV
  double* dJ3_ri[2] = {nullptr, nullptr};        // W, V
  double* dJ2[3] = {nullptr, nullptr, nullptr};  // W, V, WV
  bool device_mem = false;
  // instead of dJ3 / dJ3_ri (which must then be null): the gradient in aux
  // blocks, never held whole on the device
  GradSink sink3[3], sink3_ri[2];
};
void form_fock_adjoint(const FockRequest& rq, const AdjointOutputs& out);

// Device time per schedule phase accumulated while GEMM profiling is on
// ("name=ms;..."); reading resets the accumulators.
std::string phase_profile_read();

}  // namespace uw12b
