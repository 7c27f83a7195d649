// UW12 energy + Fock schedule on the device.
//
// Every contraction of libuw12's two-, three- and four-electron terms is
// restated as a handful of large FP64 GEMMs (gemm_f64.cu); the reference's
// per-aux-function parallel_for loops and per-orbital-pair parallel_sum_2d
// loops become batched / reduction-batched GEMMs.  Notation: N = n_ao,
// M = n_df, R = n_ri, R' = N + R, per spin o occupied, a active, c = o - a core.
//
//  T1  B1[mu + N k, A]  = sum_nu sq(J3_0[:,A])[mu,nu] Co[nu,k], then * P2
//      (transformations.hpp:33-54, integrals.cpp:213-248)
//  T2  Bri[nu + R i, A] = sum_mu J3ri_A[nu,mu] Ca[mu,i], then * P2
//      (transformations.hpp:130-158, integrals.cpp:250-287)
//  T3  B2[i + a k, A]   = sum_mu Ca[mu,i] B1[mu + N k, A]  (transformations.hpp:79-106)
//  Wst rows p + R' j: p < N -> B1 orbital c+j, p >= N -> Bri orbital j (the
//      AO-then-RI stacking of the ABS+ space), SV = (I_a (x) S^-1) Wst.
//  X_AB = Wst_W^T SV_V replaces the four calculate_xab_component loops
//      (direct_utils.cpp:31-133); t = B2_W^T B2_V, t~ = Lw t Lv
//      (four_electron_utils.cpp:33-79).
//  Fock pieces are accumulated unsymmetrised per spin and symmetrised once;
//  libuw12 symmetrises the three- and four-electron terms and its
//  two-electron pieces are symmetric by construction (utils.hpp:215-224).
#include <cusolverDn.h>

#include <algorithm>
#include <cstdint>
#include <exception>
#include <vector>
#include <thread>
#include <cstring>
#include <cmath>
#include <cstdio>
#include <map>
#include <mutex>
#include <string>

#include "engine.cuh"
#include "gemm_f64.cuh"
#include "kernels.cuh"

namespace uw12b {

namespace {

void solver_check(cusolverStatus_t st, const char* what) {
  if (st != CUSOLVER_STATUS_SUCCESS)
    throw Error(kErrCuda, std::string(what) + ": cusolver status " + std::to_string(int(st)));
}

// Pinned chunks for host-to-device copies out of pageable memory: filled by
// several host threads at once while the previous chunk's DMA runs (a
// pageable cudaMemcpyAsync stages through the driver at ~10 GB/s).  One set
// per process, used under a mutex; an event per chunk guards its reuse.
struct Staging {
  static constexpr size_t kChunkBytes = size_t(64) << 20;
  static constexpr int kChunks = 4;
  std::mutex mu;
  char* buf[kChunks] = {};
  cudaEvent_t done[kChunks] = {};
  int device[kChunks] = {};
};

Staging& staging() {
  static Staging* st = new Staging();  // lives to process exit (pinned memory freed by it)
  return *st;
}

// memcpy of `bytes` split over up to `threads` host threads.
void parallel_memcpy(char* dst, const char* src, size_t bytes, unsigned threads) {
  const size_t per = (bytes + threads - 1) / threads;
  std::vector<std::thread> pool;
  for (unsigned t = 1; t < threads && t * per < bytes; ++t)
    pool.emplace_back([=] { std::memcpy(dst + t * per, src + t * per, std::min(per, bytes - t * per)); });
  std::memcpy(dst, src, std::min(per, bytes));
  for (auto& th : pool) th.join();
}

void upload_pageable(double* dst, const double* src, size_t n, cudaStream_t s) {
  Staging& st = staging();
  std::lock_guard<std::mutex> lk(st.mu);
  int dev = 0;
  UW12_CUDA(cudaGetDevice(&dev));
  for (int c = 0; c < Staging::kChunks; ++c) {
    if (!st.buf[c]) {
      UW12_CUDA(cudaMallocHost(reinterpret_cast<void**>(&st.buf[c]), Staging::kChunkBytes));
    }
    if (!st.done[c] || st.device[c] != dev) {
      if (st.done[c]) {
        UW12_CUDA(cudaEventSynchronize(st.done[c]));
        cudaEventDestroy(st.done[c]);
      }
      UW12_CUDA(cudaEventCreateWithFlags(&st.done[c], cudaEventDisableTiming));
      st.device[c] = dev;
    }
  }
  const unsigned threads = std::max(1u, std::min(8u, std::thread::hardware_concurrency() / 2));
  const char* from = reinterpret_cast<const char*>(src);
  char* to = reinterpret_cast<char*>(dst);
  const size_t bytes = n * sizeof(double);
  int c = 0;
  for (size_t off = 0; off < bytes; off += Staging::kChunkBytes, c = (c + 1) % Staging::kChunks) {
    const size_t len = std::min(Staging::kChunkBytes, bytes - off);
    UW12_CUDA(cudaEventSynchronize(st.done[c]));  // this chunk's previous copy is done
    parallel_memcpy(st.buf[c], from + off, len, threads);
    UW12_CUDA(cudaMemcpyAsync(to + off, st.buf[c], len, cudaMemcpyHostToDevice, s));
    UW12_CUDA(cudaEventRecord(st.done[c], s));
  }
  // the caller's buffer has been read; the chunks' copies finish in stream order
}

// n doubles to the device: device-to-device, a direct copy from pinned host
// memory, or the staged pipeline for large pageable host buffers.
void upload(double* dst, const double* src, size_t n, bool device_mem, cudaStream_t s) {
  if (!n) return;
  if (!device_mem && n * sizeof(double) >= (size_t(32) << 20)) {
    cudaPointerAttributes at{};
    const bool known = cudaPointerGetAttributes(&at, src) == cudaSuccess;
    if (!known) cudaGetLastError();  // clear the query's error
    if (!known || at.type == cudaMemoryTypeUnregistered) {
      upload_pageable(dst, src, n, s);
      return;
    }
  }
  UW12_CUDA(cudaMemcpyAsync(dst, src, n * sizeof(double),
                            device_mem ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s));
}

// libuw12's linalg::is_symmetric(mat, 1e-10) (linalg.hpp:309-330), relative
// to max(1, max|A|).
void require_symmetric(const double* A, size_t n, const char* msg) {
  cudaStream_t s = current_stream();
  DevBuf st(2, s);
  symmetry_stats(A, n, n, st.get());
  double h[2];
  UW12_CUDA(cudaMemcpyAsync(h, st.get(), sizeof(h), cudaMemcpyDeviceToHost, s));
  UW12_CUDA(cudaStreamSynchronize(s));
  if (!(h[0] <= 1e-10 * std::max(1.0, h[1]))) throw_logic(msg);
}

// One cuSOLVER handle per host thread and device, created on first use.
cusolverDnHandle_t solver_handle() {
  struct Handles {
    std::map<int, cusolverDnHandle_t> h;
    ~Handles() {
      for (auto& kv : h) cusolverDnDestroy(kv.second);
    }
  };
  thread_local Handles handles;
  int dev = 0;
  UW12_CUDA(cudaGetDevice(&dev));
  auto it = handles.h.find(dev);
  if (it != handles.h.end()) return it->second;
  cusolverDnHandle_t h = nullptr;
  solver_check(cusolverDnCreate(&h), "cusolverDnCreate");
  handles.h[dev] = h;
  return h;
}

// Ascending eigenpairs of a symmetric n x n matrix, in place (A -> vectors).
void eigh(double* A, size_t n, double* w) {
  cudaStream_t s = current_stream();
  cusolverDnHandle_t h = solver_handle();
  solver_check(cusolverDnSetStream(h, s), "cusolverDnSetStream");
  int lwork = 0;
  solver_check(cusolverDnDsyevd_bufferSize(h, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER,
                                           static_cast<int>(n), A, static_cast<int>(n), w, &lwork),
               "cusolverDnDsyevd_bufferSize");
  DevBuf work(static_cast<size_t>(std::max(lwork, 1)), s);
  int* info = nullptr;
  UW12_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&info), sizeof(int), s));
  solver_check(cusolverDnDsyevd(h, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER,
                                static_cast<int>(n), A, static_cast<int>(n), w, work.get(), lwork,
                                info),
               "cusolverDnDsyevd");
  UW12_LAUNCHED();
  int hinfo = 0;
  UW12_CUDA(cudaMemcpyAsync(&hinfo, info, sizeof(int), cudaMemcpyDeviceToHost, s));
  UW12_CUDA(cudaFreeAsync(info, s));
  UW12_CUDA(cudaStreamSynchronize(s));
  if (hinfo != 0) throw_runtime("eigen-decomposition failed");
}

// Chunk budget in doubles: the caller's, or `fraction` (45% by default) of
// the device memory available now (free memory plus what the library's pool
// holds unused).  The evaluations re-read it at the start of each chunked
// phase, after the phase's persistent intermediates are allocated.
size_t auto_budget_doubles(size_t requested_bytes, double fraction = 0.45) {
  if (requested_bytes)  // an explicit budget may be small (many small chunks)
    return std::max<size_t>(requested_bytes, size_t(64) << 10) / sizeof(double);
  size_t free_b = 0, total_b = 0;
  UW12_CUDA(cudaMemGetInfo(&free_b, &total_b));
  unsigned long long reserved = 0, used = 0;  // 64-bit pool attributes
  UW12_CUDA(cudaMemPoolGetAttribute(library_pool(), cudaMemPoolAttrReservedMemCurrent, &reserved));
  UW12_CUDA(cudaMemPoolGetAttribute(library_pool(), cudaMemPoolAttrUsedMemCurrent, &used));
  const double avail = double(free_b) + (reserved > used ? double(reserved - used) : 0.0);
  // the automatic budget never drops below 64 MiB
  return std::max<size_t>(static_cast<size_t>(fraction * avail), size_t(64) << 20) /
         sizeof(double);
}

inline long long LL(size_t v) { return static_cast<long long>(v); }

// Metric eigendecomposition (base_integrals.cpp:155-166): P2 = Q pinv(Lambda),
// df_vals = Lambda, after libuw12's symmetry check.
// A non-blocking stream that starts after the work already on `parent`;
// join() makes `parent` wait for it and waits for it on the host.  The
// destructor (also on an error path) waits for it before destroying it, so
// nothing it reads or writes is released while in flight.
class SideStream {
 public:
  explicit SideStream(cudaStream_t parent) : parent_(parent) {
    UW12_CUDA(cudaStreamCreateWithFlags(&s_, cudaStreamNonBlocking));
    UW12_CUDA(cudaEventCreateWithFlags(&ev_, cudaEventDisableTiming));
    UW12_CUDA(cudaEventRecord(ev_, parent_));
    UW12_CUDA(cudaStreamWaitEvent(s_, ev_, 0));
  }
  SideStream(const SideStream&) = delete;
  SideStream& operator=(const SideStream&) = delete;
  ~SideStream() {
    cudaStreamSynchronize(s_);
    cudaEventDestroy(ev_);
    cudaStreamDestroy(s_);
  }
  cudaStream_t get() const { return s_; }
  void join() {
    UW12_CUDA(cudaEventRecord(ev_, s_));
    UW12_CUDA(cudaStreamWaitEvent(parent_, ev_, 0));
    UW12_CUDA(cudaStreamSynchronize(s_));
  }

 private:
  cudaStream_t parent_ = nullptr, s_ = nullptr;
  cudaEvent_t ev_ = nullptr;
};

void setup_metric(IntegralsHandle* h, const double* X2, bool device_mem) {
  cudaStream_t s = current_stream();
  const size_t n_df = h->n_df;
  h->P2.alloc(n_df * n_df);
  upload(h->P2.get(), X2, n_df * n_df, device_mem, s);
  require_symmetric(h->P2.get(), n_df, "matrix must be symmetric");
  h->lam.alloc(n_df);
  eigh(h->P2.get(), n_df, h->lam.get());
  scale_pinv_cols(h->P2.get(), LL(n_df), h->lam.get(), 1e-10);
  h->lam_host.resize(n_df);
  UW12_CUDA(cudaMemcpyAsync(h->lam_host.data(), h->lam.get(), n_df * sizeof(double),
                            cudaMemcpyDeviceToHost, s));
  UW12_CUDA(cudaStreamSynchronize(s));
}

// Columns [a0, a0 + na) of X's AO (ri = false: Np rows) or RI (ri = true:
// R N rows) three-index tensor, column-major with leading dimension = rows: a
// pointer into the stored tensor, or the producer's output in `scratch`
// (integral-direct mode).
const double* aux_block(const IntegralsHandle& X, bool ri, size_t a0, size_t na,
                        DevBuf& scratch) {
  const size_t rows = ri ? X.n_ri * X.n_ao : packed_size(X.n_ao);
  const DeviceArray& stored = ri ? X.J3_ri_0 : X.J3_0;
  if (stored.get()) return stored.get() + rows * a0;
  const AuxProducer& fn = ri ? X.ri_fn : X.ao_fn;
  if (!fn) throw_runtime(ri ? "J3_ri_0 not stored" : "J3_0 not stored");
  if (scratch.size() < rows * na) scratch.alloc(rows * na);
  cudaStream_t s = current_stream();
  if (profile_enabled()) {
    cudaEvent_t a, b;
    UW12_CUDA(cudaEventCreate(&a));
    UW12_CUDA(cudaEventCreate(&b));
    UW12_CUDA(cudaEventRecord(a, s));
    fn(a0, na, scratch.get(), rows, s);
    UW12_CUDA(cudaEventRecord(b, s));
    profile_record(kProfProducer, a, b, 8.0 * double(rows) * double(na),
                   std::string(ri ? "produce ri " : "produce ao ") + std::to_string(na));
  } else {
    fn(a0, na, scratch.get(), rows, s);
  }
  return scratch.get();
}

// Aux functions per block when looping over a tensor: all of them when it is
// stored (one block, the tensor itself), else as many as a quarter of the
// budget holds.
size_t aux_step(const IntegralsHandle& X, bool ri, size_t budget) {
  const DeviceArray& stored = ri ? X.J3_ri_0 : X.J3_0;
  if (stored.get()) return X.n_df;
  const size_t rows = ri ? X.n_ri * X.n_ao : packed_size(X.n_ao);
  return std::max<size_t>(1, std::min(X.n_df, budget / (4 * rows)));
}

}  // namespace

// --------------------------------------------------------------------------
// handles
// --------------------------------------------------------------------------
IntegralsHandle* integrals_create(const double* X3, const double* X2, const double* X3_ri,
                                  size_t n_ao, size_t n_df, size_t n_ri, bool device_mem) {
  if (n_ao == 0) throw_runtime("Number of ao orbitals is zero");
  if (n_df == 0) throw_runtime("Number of density-fitting basis functions is zero");
  if (!X3 || !X2) throw Error(kErrInvalid, "null integral pointer");
  if (X3_ri && n_ri == 0) throw_runtime("Three index ri integrals given but n_ri is zero");
  auto h = new IntegralsHandle();
  try {
    UW12_CUDA(cudaGetDevice(&h->device));
    cudaStream_t s = current_stream();
    h->n_ao = n_ao;
    h->n_df = n_df;
    h->n_ri = X3_ri ? n_ri : 0;
    const size_t np = packed_size(n_ao);
    h->J3_0.alloc(np * n_df);
    if (X3_ri) h->J3_ri_0.alloc(n_ri * n_ao * n_df);
    // The three-index copies run on a side stream (after the caller's work on
    // the current stream, which may have produced device inputs) while the
    // metric is diagonalised on the current stream; both are complete when
    // this returns.
    SideStream side(s);
    // host sources are read on a second host thread (a pageable source is
    // copied through pinned chunks by host threads), so the eigensolve runs
    // meanwhile
    std::exception_ptr upload_err;
    const int dev = h->device;
    std::thread up([&] {
      try {
        UW12_CUDA(cudaSetDevice(dev));
        upload(h->J3_0.get(), X3, np * n_df, device_mem, side.get());
        if (X3_ri) upload(h->J3_ri_0.get(), X3_ri, n_ri * n_ao * n_df, device_mem, side.get());
      } catch (...) {
        upload_err = std::current_exception();
      }
    });
    try {
      setup_metric(h, X2, device_mem);
    } catch (...) {
      up.join();
      throw;
    }
    up.join();
    if (upload_err) std::rethrow_exception(upload_err);
    side.join();
  } catch (...) {
    delete h;
    throw;
  }
  return h;
}

IntegralsHandle* integrals_create_producer(const double* X2, bool x2_device, AuxProducer ao_fn,
                                           AuxProducer ri_fn, size_t n_ao, size_t n_df,
                                           size_t n_ri, bool store_ao, bool store_ri) {
  if (n_ao == 0) throw_runtime("Number of ao orbitals is zero");
  if (n_df == 0) throw_runtime("Number of density-fitting basis functions is zero");
  if (!X2 || !ao_fn) throw Error(kErrInvalid, "null metric or three-index producer");
  if (ri_fn && n_ri == 0) throw_runtime("Three index ri integrals given but n_ri is zero");
  auto h = new IntegralsHandle();
  try {
    UW12_CUDA(cudaGetDevice(&h->device));
    cudaStream_t s = current_stream();
    h->n_ao = n_ao;
    h->n_df = n_df;
    h->n_ri = ri_fn ? n_ri : 0;
    setup_metric(h, X2, x2_device);
    const size_t np = packed_size(n_ao);
    if (store_ao) {
      h->J3_0.alloc(np * n_df);
      ao_fn(0, n_df, h->J3_0.get(), np, s);
    } else {
      h->ao_fn = std::move(ao_fn);
    }
    if (ri_fn) {
      if (store_ri) {
        h->J3_ri_0.alloc(n_ri * n_ao * n_df);
        ri_fn(0, n_df, h->J3_ri_0.get(), n_ri * n_ao, s);
      } else {
        h->ri_fn = std::move(ri_fn);
      }
    }
    UW12_CUDA(cudaStreamSynchronize(s));
  } catch (...) {
    delete h;
    throw;
  }
  return h;
}

IntegralsHandle* integrals_create_eigenbasis(const double* J3, const double* df_vals, size_t n_ao,
                                             size_t n_df, bool device_mem) {
  if (n_ao == 0) throw_runtime("Number of ao orbitals is zero");
  if (n_df == 0) throw_runtime("Number of density-fitting basis functions is zero");
  if (!J3 || !df_vals) throw Error(kErrInvalid, "null integral pointer");
  auto h = new IntegralsHandle();
  try {
    UW12_CUDA(cudaGetDevice(&h->device));
    cudaStream_t s = current_stream();
    h->n_ao = n_ao;
    h->n_df = n_df;
    const size_t np = packed_size(n_ao);
    h->J3_0.alloc(np * n_df);
    upload(h->J3_0.get(), J3, np * n_df, device_mem, s);
    h->P2.alloc(n_df * n_df);
    set_identity(h->P2.get(), LL(n_df));
    h->lam.alloc(n_df);
    upload(h->lam.get(), df_vals, n_df, device_mem, s);
    h->lam_host.resize(n_df);
    UW12_CUDA(cudaMemcpyAsync(h->lam_host.data(), h->lam.get(), n_df * sizeof(double),
                              cudaMemcpyDeviceToHost, s));
    UW12_CUDA(cudaStreamSynchronize(s));
  } catch (...) {
    delete h;
    throw;
  }
  return h;
}

AbsHandle* abs_create(const double* S, size_t n_ao, size_t n_ri, bool device_mem) {
  if (!S) throw Error(kErrInvalid, "null overlap pointer");
  const size_t n = n_ao + n_ri;
  if (n == 0) throw_runtime("Total number of basis functions is inconsistent");
  auto h = new AbsHandle();
  try {
    UW12_CUDA(cudaGetDevice(&h->device));
    cudaStream_t s = current_stream();
    h->n_ao = n_ao;
    h->n_ri = n_ri;
    DevBuf vecs(n * n, s);
    upload(vecs.get(), S, n * n, device_mem, s);
    require_symmetric(vecs.get(), n, "matrix must be symmetric");
    DevBuf vals(n, s);
    eigh(vecs.get(), n, vals.get());
    std::vector<double> lam(n);
    UW12_CUDA(cudaMemcpyAsync(lam.data(), vals.get(), n * sizeof(double), cudaMemcpyDeviceToHost,
                              s));
    UW12_CUDA(cudaStreamSynchronize(s));
    // eigen_decomposition(S, 1e-6, 1e-8) (linalg.hpp:1157-1197).
    double max_eig = 0.0;
    for (double v : lam) max_eig = std::max(max_eig, std::fabs(v));
    const double thr = std::max(max_eig * 1e-8, 1e-6);
    std::vector<int> keep;
    std::vector<double> inv;
    for (size_t i = 0; i < n; ++i)
      if (std::fabs(lam[i]) > thr) {
        if (!(lam[i] > 0.0)) throw_runtime("inv_sym_pd(): matrix is not positive definite");
        keep.push_back(static_cast<int>(i));
        inv.push_back(1.0 / lam[i]);
      }
    h->n_kept = keep.size();
    h->Sinv.alloc(n * n);
    const size_t r = keep.size();
    if (r == 0) {
      UW12_CUDA(cudaMemsetAsync(h->Sinv.get(), 0, n * n * sizeof(double), s));
    } else {
      int* d_idx = nullptr;
      UW12_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&d_idx), r * sizeof(int), s));
      DevBuf d_inv(r, s), d_one(r, s), vk(n * r, s), vks(n * r, s);
      UW12_CUDA(cudaMemcpyAsync(d_idx, keep.data(), r * sizeof(int), cudaMemcpyHostToDevice, s));
      UW12_CUDA(cudaMemcpyAsync(d_inv.get(), inv.data(), r * sizeof(double),
                                cudaMemcpyHostToDevice, s));
      std::vector<double> ones(r, 1.0);
      UW12_CUDA(cudaMemcpyAsync(d_one.get(), ones.data(), r * sizeof(double),
                                cudaMemcpyHostToDevice, s));
      gather_scale_cols(vecs.get(), LL(n), d_idx, d_one.get(), LL(r), vk.get());
      gather_scale_cols(vecs.get(), LL(n), d_idx, d_inv.get(), LL(r), vks.get());
      GemmDesc g = gemm_nn(LL(n), LL(n), LL(r), 1.0, vks.get(), LL(n), vk.get(), LL(n), 0.0,
                           h->Sinv.get(), LL(n));
      g.b_ncontig = true;  // B = Vk^T
      gemm(g);
      UW12_CUDA(cudaFreeAsync(d_idx, s));
    }
    UW12_CUDA(cudaStreamSynchronize(s));
  } catch (...) {
    delete h;
    throw;
  }
  return h;
}

// --------------------------------------------------------------------------
// schedule helpers
// --------------------------------------------------------------------------
namespace {

// Phase timing: events recorded at phase boundaries while profiling is on.
std::mutex g_phase_mu;
std::map<std::string, double> g_phase_ms;

class PhaseClock {
 public:
  PhaseClock() : on_(profile_enabled()) {}
  ~PhaseClock() {
    if (!on_) return;
    for (auto& m : marks_) cudaEventDestroy(m.second);
  }
  void mark(const char* name) {
    if (!on_) return;
    cudaEvent_t e;
    UW12_CUDA(cudaEventCreate(&e));
    UW12_CUDA(cudaEventRecord(e, current_stream()));
    marks_.emplace_back(name, e);
  }
  // Accumulates the time from each mark to the next into its phase.
  void finish() {
    if (!on_ || marks_.size() < 2) return;
    UW12_CUDA(cudaEventSynchronize(marks_.back().second));
    std::lock_guard<std::mutex> lk(g_phase_mu);
    for (size_t i = 0; i + 1 < marks_.size(); ++i) {
      float ms = 0.f;
      UW12_CUDA(cudaEventElapsedTime(&ms, marks_[i].second, marks_[i + 1].second));
      g_phase_ms[marks_[i].first] += ms;
    }
  }

 private:
  bool on_;
  std::vector<std::pair<std::string, cudaEvent_t>> marks_;
};

enum Slot { kE2d = 0, kE2i = 1, kE3d = 2, kE3i = 3, kE4d = 4, kE4i = 5, kSlots = 8 };

double spin_factor(int ns, int s, int sp, double s_os, double s_ss) {
  // four_electron_utils.cpp:9-30
  if (ns == 1) return 2.0 * (s_os + s_ss);
  return (s == sp) ? s_ss : s_os;
}

// XDr (M x ns) = J3_0^T dmat: the unscaled fitted densities of libuw12's
// get_X_D (integrals.cpp:347-378), over aux blocks; only the rows of aux
// functions [a_lo, a_hi) are formed (the others are zero).
void fitted_density_raw(const IntegralsHandle& X, const double* dmat, int ns, double* XDr,
                        size_t budget, size_t a_lo = 0, size_t a_hi = SIZE_MAX) {
  const size_t M = X.n_df, np = packed_size(X.n_ao);
  a_hi = std::min(a_hi, M);
  if (a_lo > 0 || a_hi < M)
    UW12_CUDA(cudaMemsetAsync(XDr, 0, M * ns * sizeof(double), current_stream()));
  DevBuf scratch;
  const size_t step = aux_step(X, false, budget);
  for (size_t b0 = a_lo; b0 < a_hi; b0 += step) {
    const size_t nb = std::min(step, a_hi - b0);
    GemmDesc g = gemm_nn(LL(nb), ns, LL(np), 1.0, aux_block(X, false, b0, nb, scratch), LL(np),
                         dmat, LL(np), 0.0, XDr + b0, LL(M));
    g.a_kcontig = true;
    gemm(g);
  }
}

// H2 (R*na x (a_hi - a_lo)) = [J3_ri_0[:,A] (R x N) Cm] for A in [a_lo, a_hi)
// (transform_second_index, transformations.hpp:130-158), over aux blocks.
void ri_transform(const IntegralsHandle& X, const double* Cm, size_t na, double* H2,
                  size_t budget, size_t a_lo = 0, size_t a_hi = SIZE_MAX) {
  const size_t N = X.n_ao, R = X.n_ri;
  a_hi = std::min(a_hi, X.n_df);
  DevBuf scratch;
  const size_t step = aux_step(X, true, budget);
  for (size_t b0 = a_lo; b0 < a_hi; b0 += step) {
    const size_t nb = std::min(step, a_hi - b0);
    GemmDesc g = gemm_nn(LL(R), LL(na), LL(N), 1.0, aux_block(X, true, b0, nb, scratch), LL(R),
                         Cm, LL(N), 0.0, H2 + R * na * (b0 - a_lo), LL(R));
    g.nbo1 = LL(nb);
    g.sAo1 = LL(R * N);
    g.sCo1 = LL(R * na);
    gemm(g);
  }
}

// H (N*nc x (a_hi - a_lo)) = [sq(J3_0[:,A]) Cm] for A in [a_lo, a_hi), chunked
// over A.
void transform_ao(const IntegralsHandle& X, const double* Cm, size_t nc, double* H,
                  size_t budget, size_t a_lo = 0, size_t a_hi = SIZE_MAX) {
  const size_t N = X.n_ao, M = X.n_df, np = packed_size(N);
  a_hi = std::min(a_hi, M);
  if (nc == 0 || a_hi <= a_lo) return;
  const size_t ac =
      std::max<size_t>(1, std::min(a_hi - a_lo, budget / (N * N + (X.J3_0.get() ? 0 : np))));
  DevBuf U(N * N * ac), scratch;
  for (size_t a0 = a_lo; a0 < a_hi; a0 += ac) {
    const size_t na = std::min(ac, a_hi - a0);
    unpack_sym(aux_block(X, false, a0, na, scratch), LL(np), LL(N), LL(na), U.get(), LL(N),
               LL(N * N));
    GemmDesc g = gemm_nn(LL(N), LL(nc), LL(N), 1.0, U.get(), LL(N), Cm, LL(N), 0.0,
                         H + N * nc * (a0 - a_lo), LL(N));
    g.nbo1 = LL(na);
    g.sAo1 = LL(N * N);
    g.sCo1 = LL(N * nc);
    gemm(g);
  }
}

// Chunk size c <= max_chunk (in units of `unit` GEMM columns) for a loop over
// `total` units: the chunked GEMMs have n = unit * c columns, so c is chosen
// to fill the 128-wide column tiles over the whole loop (fewest wasted
// columns, then the largest chunk).
size_t tile_chunk(size_t total, size_t unit, size_t max_chunk) {
  max_chunk = std::max<size_t>(1, std::min(max_chunk, total));
  auto tiles = [](size_t cols) { return (cols + 127) / 128; };
  size_t best = max_chunk;
  double best_fill = -1.0;
  for (size_t c = max_chunk; c >= std::max<size_t>(1, max_chunk / 2); --c) {
    const size_t full = total / c, rem = total % c;
    const size_t used = full * tiles(unit * c) + (rem ? tiles(unit * rem) : 0);
    const double fill = double(total * unit) / double(used * 128);
    if (fill > best_fill + 1e-9) {
      best_fill = fill;
      best = c;
    }
    if (c == 1) break;
  }
  return best;
}

struct SpinDims {
  size_t o = 0, a = 0, c = 0, ooff = 0, aoff = 0;
};

// Occupation-weighted occupied orbitals Co (utils.hpp:289-310) of both spins side
// by side (N x o_tot) and their active (last n_active) columns Ca (freeze_core,
// utils.hpp:235-253; N x a_tot), on the device.
void upload_orbitals(const FockRequest& rq, std::vector<SpinDims>& sd, size_t& o_tot,
                     size_t& a_tot, DevBuf& Co, DevBuf& Ca) {
  const int ns = rq.n_spin;
  const size_t N = rq.n_ao;
  cudaStream_t st = current_stream();
  sd.assign(ns, SpinDims{});
  o_tot = a_tot = 0;
  for (int s = 0; s < ns; ++s) {
    sd[s].o = rq.n_occ[s];
    sd[s].a = rq.n_active[s];
    sd[s].c = sd[s].o - sd[s].a;
    sd[s].ooff = o_tot;
    sd[s].aoff = a_tot;
    o_tot += sd[s].o;
    a_tot += sd[s].a;
  }
  Co.alloc(N * o_tot);
  Ca.alloc(N * a_tot);
  DevBuf wts(o_tot);
  std::vector<double> w(o_tot);
  const double per = (ns == 1) ? 2.0 : 1.0;
  for (int s = 0; s < ns; ++s)
    for (size_t k = 0; k < sd[s].o; ++k) w[sd[s].ooff + k] = std::sqrt(rq.occ[s][k] / per);
  if (o_tot)
    UW12_CUDA(cudaMemcpyAsync(wts.get(), w.data(), o_tot * sizeof(double), cudaMemcpyHostToDevice,
                              st));
  for (int s = 0; s < ns; ++s) {
    if (!sd[s].o) continue;
    UW12_CUDA(cudaMemcpy2DAsync(Co.get() + N * sd[s].ooff, N * sizeof(double), rq.C[s],
                                rq.ldc[s] * sizeof(double), N * sizeof(double), sd[s].o,
                                cudaMemcpyHostToDevice, st));
  }
  if (o_tot) scale_rc(Co.get(), LL(N), LL(N), LL(o_tot), nullptr, wts.get(), 1.0, Co.get(), LL(N));
  for (int s = 0; s < ns; ++s)
    if (sd[s].a)
      UW12_CUDA(cudaMemcpyAsync(Ca.get() + N * sd[s].aoff, Co.get() + N * (sd[s].ooff + sd[s].c),
                                N * sd[s].a * sizeof(double), cudaMemcpyDeviceToDevice, st));
}

}  // namespace

// --------------------------------------------------------------------------
// form_fock
// --------------------------------------------------------------------------
void form_fock(const FockRequest& rq) {
  const IntegralsHandle& W = *rq.W;
  const IntegralsHandle& V = *rq.V;
  const IntegralsHandle& WV = *rq.WV;
  const AbsHandle& AB = *rq.abs;
  const int ns = rq.n_spin;
  const size_t N = rq.n_ao;
  const size_t np = packed_size(N);
  const size_t MW = W.n_df, MV = V.n_df, MX = WV.n_df;
  const size_t R = W.n_ri, Rp = N + R;
  const double s_os = rq.s_os, s_ss = rq.s_ss;
  const bool calc = rq.calc_fock;
  const bool do_ind = rq.indirect && s_ss != 0.0;
  const double half = (ns == 1) ? 0.5 : 1.0;
  const double two = (ns == 1) ? 2.0 : 1.0;
  const double kap4 = 2.0 * half;
  cudaStream_t st = current_stream();
  size_t budget = auto_budget_doubles(rq.mem_budget);
  // Sharding: aux functions and occupied orbitals are dealt out in
  // contiguous, balanced ranges (part).  The fitted densities, the MO
  // transforms and the 2-el Fock run over this shard's aux range, and the
  // partial intermediates (fitted densities, B1, the stacked RI rows) are
  // summed over the shards by rq.allreduce before use; X_AB and t are summed
  // from orbital ranges the same way.  The t~ dX Fock term runs over a range
  // of W's aux functions, the direct Fock and the same-spin 3-el energy and
  // Fock over ranges of occupied k.  The energies built from the reduced
  // intermediates and the same-spin 2-el / 4-el terms come from shard 0.  The
  // caller sums the partial energies and Fock matrices over the shards.
  const size_t n_shards = std::max<size_t>(1, rq.n_shards);
  const size_t shard = rq.shard;
  const bool lead = shard == 0;
  const bool sharded = n_shards > 1;
  auto part = [&](size_t total) {
    return std::make_pair(total * shard / n_shards, total * (shard + 1) / n_shards);
  };
  if (sharded && !rq.allreduce)
    throw Error(kErrInvalid, "a sharded evaluation needs an all-reduce (uw12c_set_allreduce)");
  auto allreduce = [&](double* buf, size_t count) {
    if (!sharded || count == 0) return;
    if (rq.allreduce(buf, count, st, rq.allreduce_user) != 0)
      throw Error(kErrInvalid, "the all-reduce of a sharded evaluation failed");
  };

  std::vector<SpinDims> sd;
  size_t o_tot = 0, a_tot = 0;
  PhaseClock clock;
  clock.mark("orbitals");
  DevBuf Co, Ca;
  upload_orbitals(rq, sd, o_tot, a_tot, Co, Ca);
  auto Ca_s = [&](int s) { return Ca.get() + N * sd[s].aoff; };

  DevBuf acc(kSlots);
  acc.zero();
  std::vector<DevBuf> Fp(ns);
  for (int s = 0; s < ns; ++s) {
    Fp[s].alloc(N * N);
    Fp[s].zero();
  }

  // =====================================================================
  // two-electron term (two_electron.cpp:11-153), WV integrals, active orbitals
  // =====================================================================
  clock.mark("two_electron");
  {
    // fitted densities and the 2-el Fock over this shard's aux range of WV
    const auto [xlo, xhi] = part(MX);
    DevBuf dmat(np * ns), XDr(MX * ns), XD(MX * ns);
    for (int s = 0; s < ns; ++s) pack_density(Ca_s(s), LL(N), LL(N), LL(sd[s].a), two, dmat.get() + np * s);
    fitted_density_raw(WV, dmat.get(), ns, XDr.get(), budget, xlo, xhi);
    allreduce(XDr.get(), MX * ns);
    GemmDesc g = gemm_nn(LL(MX), ns, LL(MX), 0.5 * ns, WV.P2.get(), LL(MX), XDr.get(), LL(MX), 0.0,
                         XD.get(), LL(MX));
    g.a_kcontig = true;
    gemm(g);
    double coef[4] = {0, 0, 0, 0};
    for (int s = 0; s < ns; ++s)
      for (int sp = 0; sp < ns; ++sp) {
        const double f = spin_factor(ns, s, sp, s_os, s_ss);
        if (f == 0.0) continue;
        if (lead)
          wdot(XD.get() + MX * s, LL(MX), XD.get() + MX * sp, LL(MX), LL(MX), 1, WV.lam.get(),
               nullptr, 0.5 * f, acc.get(), kE2d);
        coef[s * ns + sp] = 0.5 * ns * f;
      }
    if (calc) {
      DevBuf vc(MX * ns), u(MX * ns), gv(np * ns);
      combine_vecs(XD.get(), LL(MX), ns, coef, WV.lam.get(), vc.get());
      gemm(gemm_nn(LL(MX), ns, LL(MX), 1.0, WV.P2.get(), LL(MX), vc.get(), LL(MX), 0.0, u.get(),
                   LL(MX)));
      {
        // gv = J3_0 u over this shard's aux blocks
        DevBuf scratch;
        const size_t step = aux_step(WV, false, budget);
        if (xhi == xlo) gv.zero();
        for (size_t b0 = xlo; b0 < xhi; b0 += step) {
          const size_t nb = std::min(step, xhi - b0);
          gemm(gemm_nn(LL(np), ns, LL(nb), 1.0, aux_block(WV, false, b0, nb, scratch), LL(np),
                       u.get() + b0, LL(MX), b0 > xlo ? 1.0 : 0.0, gv.get(), LL(np)));
        }
      }
      for (int s = 0; s < ns; ++s)
        unpack_sym(gv.get() + np * s, LL(np), LL(N), 1, Fp[s].get(), LL(N), 0, 1.0, 1.0);
    }
    if (do_ind && a_tot > 0) {
      // B1 of the active orbitals: the shard's aux range of sq(J3_0) Ca times
      // the matching rows of P2, summed over the shards
      DevBuf H(N * a_tot * (xhi - xlo));
      transform_ao(WV, Ca.get(), a_tot, H.get(), budget / 2, xlo, xhi);
      for (int s = 0; s < ns; ++s) {
        const size_t a = sd[s].a;
        if (!a) continue;
        DevBuf B1(N * a * MX), B2(a * a * MX);
        gemm(gemm_nn(LL(N * a), LL(MX), LL(xhi - xlo), 1.0, H.get() + N * sd[s].aoff,
                     LL(N * a_tot), WV.P2.get() + xlo, LL(MX), 0.0, B1.get(), LL(N * a)));
        allreduce(B1.get(), N * a * MX);
        if (!lead) continue;
        GemmDesc g3 = gemm_nn(LL(a), LL(a * MX), LL(N), 1.0, Ca_s(s), LL(N), B1.get(), LL(N), 0.0,
                              B2.get(), LL(a));
        g3.a_kcontig = true;
        gemm(g3);
        wdot(B2.get(), LL(a * a), B2.get(), LL(a * a), LL(a * a), LL(MX), nullptr, WV.lam.get(),
             -0.5 * two, acc.get(), kE2i);
        if (calc) {
          DevBuf B1l(N * a * MX);
          scale_rc(B1.get(), LL(N * a), LL(N * a), LL(MX), nullptr, WV.lam.get(), 1.0, B1l.get(),
                   LL(N * a));
          GemmDesc gf = gemm_nn(LL(N), LL(N), LL(a * MX), -s_ss, B1.get(), LL(N), B1l.get(),
                                LL(N), 1.0, Fp[s].get(), LL(N));
          gf.b_ncontig = true;
          gemm(gf);
        }
      }
    }
  }

  // =====================================================================
  // MO transforms for W and V (integrals.cpp:184-345)
  // =====================================================================
  clock.mark("transforms");
  struct PerX {
    std::vector<DevBuf> B1, B2, Wst, SV;
  };
  PerX XW, XV;
  const bool need_sv_w = calc && do_ind;
  // Without same-spin terms the stacked transforms serve only X_AB, t and the
  // direct Fock, which are sums over orbitals: when the whole intermediates
  // (B1, B2, Wst of W and V, S^-1 Wst_V) exceed the chunk budget they are
  // formed for a chunk of orbitals at a time instead (orbital_chunked).
  budget = auto_budget_doubles(rq.mem_budget);
  size_t whole = 0;
  for (int s = 0; s < ns; ++s)
    whole += 2 * (N * sd[s].o * MW + sd[s].a * sd[s].o * MW) + 3 * Rp * sd[s].a * MW;
  bool orbital_chunked = !do_ind && whole > budget;
  if (sharded && !do_ind) {
    // every shard takes the same branch (the budgets may differ)
    DevBuf flag(1);
    const double one = orbital_chunked ? 1.0 : 0.0;
    UW12_CUDA(cudaMemcpyAsync(flag.get(), &one, sizeof(double), cudaMemcpyHostToDevice, st));
    allreduce(flag.get(), 1);
    double any = 0.0;
    UW12_CUDA(cudaMemcpyAsync(&any, flag.get(), sizeof(double), cudaMemcpyDeviceToHost, st));
    UW12_CUDA(cudaStreamSynchronize(st));
    orbital_chunked = any > 0.0;
  }
  for (int which = 0; which < 2 && !orbital_chunked; ++which) {
    const IntegralsHandle& X = which == 0 ? W : V;
    PerX& P = which == 0 ? XW : XV;
    const size_t M = X.n_df;
    budget = auto_budget_doubles(rq.mem_budget);
    P.B1.resize(ns);
    P.B2.resize(ns);
    P.Wst.resize(ns);
    P.SV.resize(ns);
    // this shard's aux functions [xlo, xhi): B1 and the stacked RI rows are
    // partial products H[:, xlo:xhi] P2[xlo:xhi, :], summed over the shards
    const auto [xlo, xhi] = part(M);
    {
      DevBuf H(N * o_tot * (xhi - xlo));
      transform_ao(X, Co.get(), o_tot, H.get(), budget / 2, xlo, xhi);
      for (int s = 0; s < ns; ++s) {
        const size_t o = sd[s].o;
        if (!o) continue;
        P.B1[s].alloc(N * o * M);
        gemm(gemm_nn(LL(N * o), LL(M), LL(xhi - xlo), 1.0, H.get() + N * sd[s].ooff,
                     LL(N * o_tot), X.P2.get() + xlo, LL(M), 0.0, P.B1[s].get(), LL(N * o)));
        allreduce(P.B1[s].get(), N * o * M);
      }
    }
    DevBuf H2(R * a_tot * (xhi - xlo));
    if (a_tot) ri_transform(X, Ca.get(), a_tot, H2.get(), budget, xlo, xhi);
    for (int s = 0; s < ns; ++s) {
      const size_t o = sd[s].o, a = sd[s].a, c = sd[s].c;
      if (!a) continue;
      P.B2[s].alloc(a * o * M);
      GemmDesc g3 = gemm_nn(LL(a), LL(o * M), LL(N), 1.0, Ca_s(s), LL(N), P.B1[s].get(), LL(N),
                            0.0, P.B2[s].get(), LL(a));
      g3.a_kcontig = true;
      gemm(g3);
      P.Wst[s].alloc(Rp * a * M);
      if (sharded) P.Wst[s].zero();  // AO rows stay zero through the sum
      GemmDesc g2 = gemm_nn(LL(R), LL(M), LL(xhi - xlo), 1.0, H2.get() + R * sd[s].aoff,
                            LL(R * a_tot), X.P2.get() + xlo, LL(M), 0.0, P.Wst[s].get() + N,
                            LL(Rp * a));
      g2.nbo1 = LL(a);
      g2.sAo1 = LL(R);
      g2.sCo1 = LL(Rp);
      gemm(g2);
      allreduce(P.Wst[s].get(), Rp * a * M);
      copy3d(P.B1[s].get() + N * c, LL(N), LL(N * o), P.Wst[s].get(), LL(Rp), LL(Rp * a), LL(N),
             LL(a), LL(M));
      if (which == 1 || need_sv_w) {
        // S^-1 Wst (R' x a M): this shard's aux columns, gathered by the sum
        P.SV[s].alloc(Rp * a * M);
        if (sharded) P.SV[s].zero();
        gemm(gemm_nn(LL(Rp), LL(a * (xhi - xlo)), LL(Rp), 1.0, AB.Sinv.get(), LL(Rp),
                     P.Wst[s].get() + Rp * a * xlo, LL(Rp), 0.0, P.SV[s].get() + Rp * a * xlo,
                     LL(Rp)));
        allreduce(P.SV[s].get(), Rp * a * M);
      }
    }
  }

  // =====================================================================
  // X_AB, t, t~ and the direct energies (direct_utils.cpp:62-157,
  // four_electron.cpp:80-137)
  // =====================================================================
  clock.mark("xab_t_energies");
  std::vector<DevBuf> Xab(ns), tab(ns), ttl(ns);
  // B1 (N*nk x M) of occupied orbitals [k0, k0 + nk) of spin s for potential X:
  // sq(J3_0[:, A]) Co[:, k] P2.
  auto b1_chunk = [&](const IntegralsHandle& X, int s, size_t k0, size_t nk, DevBuf& out) {
    const size_t M = X.n_df;
    DevBuf H(N * nk * M);
    transform_ao(X, Co.get() + N * (sd[s].ooff + k0), nk, H.get(), budget / 2);
    out.alloc(N * nk * M);
    gemm(gemm_nn(LL(N * nk), LL(M), LL(M), 1.0, H.get(), LL(N * nk), X.P2.get(), LL(M), 0.0,
                 out.get(), LL(N * nk)));
  };
  // occupied orbitals per chunk of the t and direct-Fock passes, active
  // orbitals per chunk of the X_AB pass
  // (per occupied orbital: B1 of W and V, the transform's output, Z or the two
  // B2 rows of its a active orbitals)
  // (the larger of the two potentials' aux counts sizes every buffer)
  const size_t Mmax = std::max(MW, MV);
  auto per_k = [&](int s) { return (4 * N + 2 * sd[s].a) * Mmax; };
  const size_t per_j = (N + R + 3 * Rp) * Mmax;
  if (orbital_chunked) {
    for (int s = 0; s < ns; ++s) {
      const size_t o = sd[s].o, a = sd[s].a, c = sd[s].c;
      Xab[s].alloc(MW * MV);
      tab[s].alloc(MW * MV);
      ttl[s].alloc(MW * MV);
      Xab[s].zero();
      tab[s].zero();
      if (a == 0) {
        ttl[s].zero();
        continue;
      }
      // X_AB = sum over active-orbital chunks of Wst_W[j]^T S^-1 Wst_V[j]
      // (this shard's orbitals; summed over the shards below)
      const auto [jlo, jhi] = part(a);
      const size_t jc = std::max<size_t>(1, std::min(jhi - jlo, budget / 2 / per_j));
      for (size_t j0 = jlo; j0 < jhi; j0 += jc) {
        const size_t nj = std::min(jc, jhi - j0);
        DevBuf St[2];
        for (int which = 0; which < 2; ++which) {
          const IntegralsHandle& X = which == 0 ? W : V;
          const size_t M = X.n_df;
          St[which].alloc(Rp * nj * M);
          // AO rows of orbital j: sq(J3_0) Co[:, c + j] P2, into rows [0, N) of its block
          DevBuf H(N * nj * M);
          transform_ao(X, Co.get() + N * (sd[s].ooff + c + j0), nj, H.get(), budget / 2);
          GemmDesc ga = gemm_nn(LL(N), LL(M), LL(M), 1.0, H.get(), LL(N * nj), X.P2.get(), LL(M),
                                0.0, St[which].get(), LL(Rp * nj));
          ga.nbo1 = LL(nj);
          ga.sAo1 = LL(N);
          ga.sCo1 = LL(Rp);
          gemm(ga);
          // RI rows: J3ri_0[:, A] Ca[:, j] P2, into rows [N, R') of its block
          DevBuf H2(R * nj * M);
          ri_transform(X, Ca_s(s) + N * j0, nj, H2.get(), budget);
          GemmDesc gr = gemm_nn(LL(R), LL(M), LL(M), 1.0, H2.get(), LL(R * nj), X.P2.get(), LL(M),
                                0.0, St[which].get() + N, LL(Rp * nj));
          gr.nbo1 = LL(nj);
          gr.sAo1 = LL(R);
          gr.sCo1 = LL(Rp);
          gemm(gr);
        }
        DevBuf SVj(Rp * nj * MV);
        gemm(gemm_nn(LL(Rp), LL(nj * MV), LL(Rp), 1.0, AB.Sinv.get(), LL(Rp), St[1].get(),
                     LL(Rp), 0.0, SVj.get(), LL(Rp)));
        GemmDesc gx = gemm_nn(LL(MW), LL(MV), LL(Rp * nj), 1.0, St[0].get(), LL(Rp * nj),
                              SVj.get(), LL(Rp * nj), 1.0, Xab[s].get(), LL(MW));
        gx.a_kcontig = true;
        gemm(gx);
      }
      // t = sum over occupied-orbital chunks of B2_W[k]^T B2_V[k], B2 = Ca^T B1
      // (this shard's orbitals)
      const auto [klo, khi] = part(o);
      const size_t kc = std::max<size_t>(1, std::min(khi - klo, budget / 2 / per_k(s)));
      for (size_t k0 = klo; k0 < khi; k0 += kc) {
        const size_t nk = std::min(kc, khi - k0);
        DevBuf B1w, B1v, B2w(a * nk * MW), B2v(a * nk * MV);
        b1_chunk(W, s, k0, nk, B1w);
        b1_chunk(V, s, k0, nk, B1v);
        GemmDesc g3 = gemm_nn(LL(a), LL(nk * MW), LL(N), 1.0, Ca_s(s), LL(N), B1w.get(), LL(N),
                              0.0, B2w.get(), LL(a));
        g3.a_kcontig = true;
        gemm(g3);
        g3 = gemm_nn(LL(a), LL(nk * MV), LL(N), 1.0, Ca_s(s), LL(N), B1v.get(), LL(N), 0.0,
                     B2v.get(), LL(a));
        g3.a_kcontig = true;
        gemm(g3);
        GemmDesc gt = gemm_nn(LL(MW), LL(MV), LL(a * nk), 1.0, B2w.get(), LL(a * nk), B2v.get(),
                              LL(a * nk), 1.0, tab[s].get(), LL(MW));
        gt.a_kcontig = true;
        gemm(gt);
      }
      allreduce(Xab[s].get(), MW * MV);
      allreduce(tab[s].get(), MW * MV);
      scale_rc(tab[s].get(), LL(MW), LL(MW), LL(MV), W.lam.get(), V.lam.get(), 1.0,
               ttl[s].get(), LL(MW));
    }
  }
  for (int s = 0; s < ns && !orbital_chunked; ++s) {
    const size_t o = sd[s].o, a = sd[s].a;
    Xab[s].alloc(MW * MV);
    tab[s].alloc(MW * MV);
    ttl[s].alloc(MW * MV);
    if (a == 0) {
      Xab[s].zero();
      tab[s].zero();
      ttl[s].zero();
      continue;
    }
    // sums over this shard's orbitals (rows p + R' j of Wst / S^-1 Wst, rows
    // i + a k of B2), completed over the shards
    const auto [jlo, jhi] = part(a);
    const auto [klo, khi] = part(o);
    GemmDesc gx = gemm_nn(LL(MW), LL(MV), LL(Rp * (jhi - jlo)), 1.0, XW.Wst[s].get() + Rp * jlo,
                          LL(Rp * a), XV.SV[s].get() + Rp * jlo, LL(Rp * a), 0.0, Xab[s].get(),
                          LL(MW));
    gx.a_kcontig = true;
    gemm(gx);
    GemmDesc gt = gemm_nn(LL(MW), LL(MV), LL(a * (khi - klo)), 1.0, XW.B2[s].get() + a * klo,
                          LL(a * o), XV.B2[s].get() + a * klo, LL(a * o), 0.0, tab[s].get(),
                          LL(MW));
    gt.a_kcontig = true;
    gemm(gt);
    allreduce(Xab[s].get(), MW * MV);
    allreduce(tab[s].get(), MW * MV);
    scale_rc(tab[s].get(), LL(MW), LL(MW), LL(MV), W.lam.get(), V.lam.get(), 1.0, ttl[s].get(),
             LL(MW));
  }
  for (int s = 0; s < ns && lead; ++s)
    for (int sp = 0; sp < ns; ++sp) {
      const double f = spin_factor(ns, s, sp, s_os, s_ss);
      wdot(Xab[s].get(), LL(MW), ttl[sp].get(), LL(MW), LL(MW), LL(MV), nullptr, nullptr, -f,
           acc.get(), kE3d);
      if (f != 0.0)
        wdot(ttl[sp].get(), LL(MW), tab[s].get(), LL(MW), LL(MW), LL(MV), nullptr, nullptr,
             0.5 * f, acc.get(), kE4d);
    }
  if (!do_ind && !orbital_chunked)  // the stacked transforms serve only X_AB and the same-spin terms
    for (int s = 0; s < ns; ++s) {
      XW.Wst[s].release();
      XW.SV[s].release();
      XV.Wst[s].release();
      XV.SV[s].release();
    }

  // =====================================================================
  // direct Fock: 4-el (four_electron.cpp:11-77) + 3-el X dt~ (direct_utils.cpp:164-204)
  // combined as sum_k w_k (B1_W Y)_k (x) (B1_V)_k, and 3-el t~ dX
  // (direct_utils.cpp:256-347) added to fock[sigma'] (three_electron.cpp:78)
  // =====================================================================
  if (calc) {
    clock.mark("direct_fock");
    for (int s = 0; s < ns; ++s) {
      const size_t o = sd[s].o, a = sd[s].a, c = sd[s].c;
      const auto [klo, khi] = part(o);  // this shard's occupied orbitals
      if (khi == klo) continue;
      const double* Tq[2] = {ttl[0].get(), ns > 1 ? ttl[1].get() : nullptr};
      const double* Xq[2] = {Xab[0].get(), ns > 1 ? Xab[1].get() : nullptr};
      double cT[2] = {0, 0}, cX[2] = {0, 0};
      for (int sp = 0; sp < ns; ++sp) {
        const double f = spin_factor(ns, s, sp, s_os, s_ss);
        cT[sp] = (f != 0.0) ? f * (a == 0 ? kap4 : 0.5 * kap4) : 0.0;
        cX[sp] = half * f;
      }
      DevBuf Y(MW * MV);
      combine_y(Y.get(), LL(MW), Tq, cT, Xq, cX, ns, W.lam.get(), V.lam.get());
      // whole B1 (rows of orbitals [klo, khi)), or B1 of W and V recomputed
      // for a chunk of occupied orbitals
      const size_t kc = orbital_chunked
                            ? std::max<size_t>(1, std::min(khi - klo, budget / 2 / per_k(s)))
                            : khi - klo;
      for (size_t k0 = klo; k0 < khi; k0 += kc) {
        const size_t nk = std::min(kc, khi - k0);
        DevBuf B1w, B1v, Z(N * nk * MV);
        if (orbital_chunked) {
          b1_chunk(W, s, k0, nk, B1w);
          b1_chunk(V, s, k0, nk, B1v);
        }
        const double* bw = orbital_chunked ? B1w.get() : XW.B1[s].get() + N * k0;
        const double* bv = orbital_chunked ? B1v.get() : XV.B1[s].get() + N * k0;
        const size_t ldb1 = orbital_chunked ? N * nk : N * o;
        gemm(gemm_nn(LL(N * nk), LL(MV), LL(MW), 1.0, bw, LL(ldb1), Y.get(), LL(MW), 0.0,
                     Z.get(), LL(N * nk)));
        // active orbitals (k >= c) weighted 2
        const size_t a0 = std::max(c, k0), a1 = k0 + nk;
        if (a > 0 && a1 > a0)
          copy3d(Z.get() + N * (a0 - k0), LL(N * nk), 0, Z.get() + N * (a0 - k0), LL(N * nk), 0,
                 LL(N * (a1 - a0)), LL(MV), 1, 2.0);
        GemmDesc gf = gemm_nn(LL(N), LL(N), LL(nk * MV), 1.0, Z.get(), LL(N), bv, LL(N), 1.0,
                              Fp[s].get(), LL(N));
        gf.b_ncontig = true;
        if (ldb1 != N * nk) {
          // part of the whole B1: K = (k, A) as MV reduction batches of nk
          gf.k = LL(nk);
          gf.nbr1 = LL(MV);
          gf.sAr1 = LL(N * nk);
          gf.sBr1 = LL(ldb1);
        }
        gemm(gf);
      }
    }
    if (!do_ind && !orbital_chunked)  // B1 and B2 serve only the direct Fock and the same-spin terms
      for (int s = 0; s < ns; ++s) {
        XW.B1[s].release();
        XW.B2[s].release();
        XV.B1[s].release();
        XV.B2[s].release();
      }
    // t~ dX: F[sigma'] -= sum_ab T2[a,b] G_W[a]^T S^-1 G_V[b] with
    // T2 = P2_W Tc[sigma'] P2_V^T and G_X[a] = [sq(J3_0^X[:,a]); J3ri_0^X[:,a]]
    // (R' x N).  L[a] = S^-1 G_W[a] does not depend on sigma', so it is formed
    // once per aux chunk and contracted with H[a] = sum_b T2[a,b] G_V[b] of
    // every spin.
    clock.mark("tdx_fock");
    std::vector<int> tdx_spins;
    std::vector<DevBuf> T2s;
    for (int sp = 0; sp < ns; ++sp) {
      const double* Tq[2] = {ttl[0].get(), ns > 1 ? ttl[1].get() : nullptr};
      double cT[2] = {0, 0}, cX[2] = {0, 0};
      bool any = false;
      for (int s = 0; s < ns; ++s) {
        cT[s] = half * spin_factor(ns, s, sp, s_os, s_ss);
        any = any || (cT[s] != 0.0 && sd[s].a > 0);
      }
      if (!any) continue;
      DevBuf Tc(MW * MV), tmp(MW * MV), T2(MW * MV);
      combine_y(Tc.get(), LL(MW), Tq, cT, Tq, cX, ns, W.lam.get(), V.lam.get());
      gemm(gemm_nn(LL(MW), LL(MV), LL(MW), 1.0, W.P2.get(), LL(MW), Tc.get(), LL(MW), 0.0,
                   tmp.get(), LL(MW)));
      GemmDesc gt2 = gemm_nn(LL(MW), LL(MV), LL(MV), 1.0, tmp.get(), LL(MW), V.P2.get(), LL(MV),
                             0.0, T2.get(), LL(MW));
      gt2.b_ncontig = true;
      gemm(gt2);
      tdx_spins.push_back(sp);
      T2s.push_back(std::move(T2));
    }
    if (!tdx_spins.empty()) {
      // The chunk buffers are the only large allocations of this phase, so
      // it takes 70% of the available memory.  Unstored V blocks are
      // produced again for every chunk of W's aux functions: V's RI blocks
      // take up to a quarter of the budget (their aux functions are the
      // contraction length of the p GEMM, whose output is large), its AO
      // blocks up to a sixteenth, the chunk the rest; unstored W blocks add
      // to the chunk's share.
      budget = auto_budget_doubles(rq.mem_budget, 0.7);
      const size_t vstep = aux_step(V, false, budget / 4), vrstep = aux_step(V, true, budget);
      const size_t vscr = (V.J3_0.get() ? 0 : np * vstep) + (V.J3_ri_0.get() ? 0 : R * N * vrstep);
      const size_t per_a = 2 * N * N + Rp * N + R * N + (W.J3_0.get() ? 0 : np);
      const size_t avail = budget > vscr ? budget - vscr : 0;
      const auto [alo, ahi] = part(MW);
      const size_t ac = tile_chunk(ahi - alo, 1,
                                   std::max<size_t>(1, std::min(ahi - alo, avail / per_a)));
      // Per chunk of W's aux functions a: Ga = sq(J3_0^W[:, a]) (N x N per a;
      // afterwards the packed s columns of each spin), L = S^-1 G_W (R' x N
      // per a), Hao = sq(s_a) (N x N per a) and Hr = p_a (R x N per a, RI rows
      // nu + R mu).  When W's RI tensor is produced, its block and Hr share
      // one buffer: the block is consumed by L before p overwrites it.
      DevBuf Ga(N * N * ac), Lb(Rp * N * ac), Hao(N * N * ac);
      DevBuf scrW, scrWr, scrV, scrVr, HrBuf;
      double* sbuf = Ga.get();
      double* Hr = nullptr;
      if (W.J3_ri_0.get()) {
        HrBuf.alloc(R * N * ac);
        Hr = HrBuf.get();
      } else {
        scrWr.alloc(R * N * ac);
        Hr = scrWr.get();
      }
      for (size_t a0 = alo; a0 < ahi; a0 += ac) {
        const size_t na = std::min(ac, ahi - a0);
        // L[a] = S^-1[:, AO] sq(J3_0^W[:, a]) + S^-1[:, RI] J3ri_0^W[:, a], the RI
        // block read where it lies (R x N per a, leading dimension R)
        unpack_sym(aux_block(W, false, a0, na, scrW), LL(np), LL(N), LL(na), Ga.get(), LL(N),
                   LL(N * N));
        gemm(gemm_nn(LL(Rp), LL(N * na), LL(N), 1.0, AB.Sinv.get(), LL(Rp), Ga.get(), LL(N), 0.0,
                     Lb.get(), LL(Rp)));
        gemm(gemm_nn(LL(Rp), LL(N * na), LL(R), 1.0, AB.Sinv.get() + Rp * N, LL(Rp),
                     aux_block(W, true, a0, na, scrWr), LL(R), 1.0, Lb.get(), LL(Rp)));
        for (size_t q = 0; q < tdx_spins.size(); ++q) {
          const double* T2 = T2s[q].get();
          // s = J3_0^V T2^T and p = J3_ri_0^V T2^T, accumulated over V's aux
          // blocks; p for all AO indices mu at once (rows nu + R mu)
          for (size_t b0 = 0; b0 < MV; b0 += vstep) {
            const size_t nb = std::min(vstep, MV - b0);
            GemmDesc gs = gemm_nn(LL(np), LL(na), LL(nb), 1.0, aux_block(V, false, b0, nb, scrV),
                                  LL(np), T2 + a0 + MW * b0, LL(MW), b0 ? 1.0 : 0.0, sbuf,
                                  LL(np));
            gs.b_ncontig = true;
            gemm(gs);
          }
          unpack_sym(sbuf, LL(np), LL(N), LL(na), Hao.get(), LL(N), LL(N * N));
          for (size_t b0 = 0; b0 < MV; b0 += vrstep) {
            const size_t nb = std::min(vrstep, MV - b0);
            GemmDesc gp = gemm_nn(LL(R * N), LL(na), LL(nb), 1.0,
                                  aux_block(V, true, b0, nb, scrVr), LL(R * N),
                                  T2 + a0 + MW * b0, LL(MW), b0 ? 1.0 : 0.0, Hr, LL(R * N));
            gp.b_ncontig = true;
            gemm(gp);
          }
          // F[sigma'] -= sum_a L[a]^T [Hao[a]; Hr[a]], AO rows then RI rows of L
          double* F = Fp[tdx_spins[q]].get();
          GemmDesc fa = gemm_nn(LL(N), LL(N), LL(N), -1.0, Lb.get(), LL(Rp), Hao.get(), LL(N),
                                1.0, F, LL(N));
          fa.a_kcontig = true;
          fa.nbr1 = LL(na);
          fa.sAr1 = LL(Rp * N);
          fa.sBr1 = LL(N * N);
          gemm(fa);
          GemmDesc fr = gemm_nn(LL(N), LL(N), LL(R), -1.0, Lb.get() + N, LL(Rp), Hr, LL(R), 1.0,
                                F, LL(N));
          fr.a_kcontig = true;
          fr.nbr1 = LL(na);
          fr.sAr1 = LL(Rp * N);
          fr.sBr1 = LL(R * N);
          gemm(fr);
        }
      }
    }
  }

  // =====================================================================
  // same-spin (indirect) terms
  // =====================================================================
  if (do_ind) {
    for (int s = 0; s < ns; ++s) {
      const size_t o = sd[s].o, a = sd[s].a, c = sd[s].c;
      if (a == 0 || o == 0) continue;
      const size_t ao = a * o, No = N * o;
      DevBuf b2wl(ao * MW), b2vl(ao * MV);
      scale_rc(XW.B2[s].get(), LL(ao), LL(ao), LL(MW), nullptr, W.lam.get(), 1.0, b2wl.get(), LL(ao));
      scale_rc(XV.B2[s].get(), LL(ao), LL(ao), LL(MV), nullptr, V.lam.get(), 1.0, b2vl.get(), LL(ao));
      clock.mark("ss_4el_energy");
      // ---- 4-el indirect energy (four_electron.cpp:143-179)
      if (lead) {
        DevBuf W4(ao * ao), V4(ao * ao);
        GemmDesc g = gemm_nn(LL(ao), LL(ao), LL(MW), 1.0, b2wl.get(), LL(ao), XW.B2[s].get(),
                             LL(ao), 0.0, W4.get(), LL(ao));
        g.b_ncontig = true;
        gemm(g);
        g = gemm_nn(LL(ao), LL(ao), LL(MV), 1.0, b2vl.get(), LL(ao), XV.B2[s].get(), LL(ao), 0.0,
                    V4.get(), LL(ao));
        g.b_ncontig = true;
        gemm(g);
        permdot_4el(W4.get(), V4.get(), LL(a), LL(o), -0.5 * two, acc.get(), kE4i);
      }
      clock.mark("ss_3el_energy");
      // ---- 3-el indirect energy (indirect_utils.cpp:101-133), chunked over k
      {
        budget = auto_budget_doubles(rq.mem_budget);
        const size_t per_k = 2 * Rp * a * a;
        const auto [klo, khi] = part(o);
        const size_t kc = tile_chunk(khi - klo, a,
                                     std::max<size_t>(1, std::min(khi - klo, budget / per_k)));
        DevBuf YW(Rp * a * a * kc), ZV(Rp * a * a * kc);
        for (size_t k0 = klo; k0 < khi; k0 += kc) {
          const size_t nk = std::min(kc, khi - k0);
          GemmDesc g = gemm_nn(LL(Rp * a), LL(a * nk), LL(MW), 1.0, XW.Wst[s].get(), LL(Rp * a),
                               b2wl.get() + a * k0, LL(ao), 0.0, YW.get(), LL(Rp * a));
          g.b_ncontig = true;
          gemm(g);
          g = gemm_nn(LL(Rp * a), LL(a * nk), LL(MV), 1.0, XV.SV[s].get(), LL(Rp * a),
                      b2vl.get() + a * k0, LL(ao), 0.0, ZV.get(), LL(Rp * a));
          g.b_ncontig = true;
          gemm(g);
          permdot_3el(YW.get(), ZV.get(), LL(Rp), LL(a), LL(nk), two, acc.get(), kE3i);
        }
      }
      if (!calc) continue;
      DevBuf b1wl(No * MW), b1vl(No * MV);
      scale_rc(XW.B1[s].get(), LL(No), LL(No), LL(MW), nullptr, W.lam.get(), 1.0, b1wl.get(), LL(No));
      scale_rc(XV.B1[s].get(), LL(No), LL(No), LL(MV), nullptr, V.lam.get(), 1.0, b1vl.get(), LL(No));
      clock.mark("ss_4el_fock");
      // ---- 4-el indirect Fock (four_electron.cpp:181-249)
      if (lead) {
        DevBuf W43(No * ao), V43(No * ao);
        GemmDesc g = gemm_nn(LL(No), LL(ao), LL(MW), 1.0, b1wl.get(), LL(No), XW.B2[s].get(),
                             LL(ao), 0.0, W43.get(), LL(No));
        g.b_ncontig = true;
        gemm(g);
        g = gemm_nn(LL(No), LL(ao), LL(MV), 1.0, b1vl.get(), LL(No), XV.B2[s].get(), LL(ao), 0.0,
                    V43.get(), LL(No));
        g.b_ncontig = true;
        gemm(g);
        GemmDesc gi = gemm_nn(LL(N), LL(N), LL(a), s_ss * (c > 0 ? -1.0 : -2.0),
                              W43.get() + N * c, LL(No), V43.get() + N * c, LL(N), 1.0,
                              Fp[s].get(), LL(N));
        gi.b_ncontig = true;
        gi.nbr1 = LL(a);
        gi.nbr2 = LL(o);
        gi.sAr1 = LL(N);
        gi.sAr2 = LL(No * a);
        gi.sBr1 = LL(No);
        gi.sBr2 = LL(No * a);
        gemm(gi);
        if (c > 0) {
          GemmDesc gf = gemm_nn(LL(N), LL(N), LL(a), -s_ss, W43.get(), LL(No), V43.get(), LL(No),
                                1.0, Fp[s].get(), LL(N));
          gf.b_ncontig = true;
          gf.nbr1 = LL(o);
          gf.nbr2 = LL(o);
          gf.sAr1 = LL(N);
          gf.sAr2 = LL(No * a);
          gf.sBr1 = LL(No * a);
          gf.sBr2 = LL(N);
          gemm(gf);
        }
      }
      clock.mark("ss_3el_fock");
      // ---- 3-el indirect Fock (indirect_utils.cpp:139-345), chunked over k
      {
        DevBuf xhW(MW * ao), xhV(MV * ao);
        GemmDesc g = gemm_nn(LL(MW), LL(ao), LL(MW), 1.0, W.P2.get(), LL(MW), b2wl.get(), LL(ao),
                             0.0, xhW.get(), LL(MW));
        g.b_ncontig = true;
        gemm(g);
        g = gemm_nn(LL(MV), LL(ao), LL(MV), 1.0, V.P2.get(), LL(MV), b2vl.get(), LL(ao), 0.0,
                    xhV.get(), LL(MV));
        g.b_ncontig = true;
        gemm(g);
        budget = auto_budget_doubles(rq.mem_budget);
        // unstored W / V blocks (accumulated over, for every k chunk) take at
        // most an eighth of the budget each
        size_t xscr = 0;
        for (const IntegralsHandle* Xi : {&W, &V})
          xscr = std::max(xscr, (Xi->J3_0.get() ? 0 : np * aux_step(*Xi, false, budget / 2)) +
                                    (Xi->J3_ri_0.get() ? 0 : R * N * aux_step(*Xi, true, budget / 2)));
        // two R' a N buffers per k: Z_W (term 1, done first), then W_k of the
        // k-term in the same memory; Z_V (term 0) lives until the k-term
        const size_t per_k = 2 * Rp * a * N + a * (N * N + R * N + np);
        const auto [klo, khi] = part(o);
        const size_t kavail = budget > xscr ? budget - xscr : 0;
        const size_t kc = tile_chunk(khi - klo, a,
                                     std::max<size_t>(1, std::min(khi - klo, kavail / per_k)));
        DevBuf ZYV(Rp * a * N * kc), ZYW(Rp * a * N * kc), gpk(np * a * kc), Gao(N * N * a * kc),
            gri(R * N * a * kc), scrX, scrXr;
        double* const Wk = ZYW.get();  // after term 1 has used Z_W
        for (size_t k0 = klo; k0 < khi; k0 += kc) {
          const size_t nk = std::min(kc, khi - k0);
          for (int term : {1, 0}) {
            // term 0: fock_i(W, V) over (j, k); term 1: fock_i(V, W) over (i, k)
            const IntegralsHandle& Xi = term == 0 ? W : V;
            const double* xh = term == 0 ? xhW.get() : xhV.get();
            const size_t MXi = Xi.n_df;
            const double* SVy = term == 0 ? XV.SV[s].get() : XW.SV[s].get();
            const double* b1yl = term == 0 ? b1vl.get() : b1wl.get();
            const size_t MY = term == 0 ? MV : MW;
            double* ZY = term == 0 ? ZYV.get() : ZYW.get();
            GemmDesc gz = gemm_nn(LL(Rp * a), LL(N * nk), LL(MY), 1.0, SVy, LL(Rp * a),
                                  b1yl + N * k0, LL(No), 0.0, ZY, LL(Rp * a));
            gz.b_ncontig = true;
            gemm(gz);
            // gpk = J3_0 xh, gri = J3_ri_0 xh, accumulated over Xi's aux blocks
            const size_t st_ao = aux_step(Xi, false, budget / 2);
            const size_t st_ri = aux_step(Xi, true, budget / 2);
            for (size_t b0 = 0; b0 < MXi; b0 += st_ao) {
              const size_t nb = std::min(st_ao, MXi - b0);
              gemm(gemm_nn(LL(np), LL(a * nk), LL(nb), 1.0, aux_block(Xi, false, b0, nb, scrX),
                           LL(np), xh + MXi * a * k0 + b0, LL(MXi), b0 ? 1.0 : 0.0, gpk.get(),
                           LL(np)));
            }
            unpack_sym(gpk.get(), LL(np), LL(N), LL(a * nk), Gao.get(), LL(N), LL(N * N));
            for (size_t b0 = 0; b0 < MXi; b0 += st_ri) {
              const size_t nb = std::min(st_ri, MXi - b0);
              gemm(gemm_nn(LL(R * N), LL(a * nk), LL(nb), 1.0, aux_block(Xi, true, b0, nb, scrXr),
                           LL(R * N), xh + MXi * a * k0 + b0, LL(MXi), b0 ? 1.0 : 0.0, gri.get(),
                           LL(R * N)));
            }
            GemmDesc fa = gemm_nn(LL(N), LL(N), LL(N), s_ss, Gao.get(), LL(N), ZY, LL(Rp * a),
                                  1.0, Fp[s].get(), LL(N));
            fa.nbr1 = LL(a);
            fa.nbr2 = LL(nk);
            fa.sAr1 = LL(N * N);
            fa.sAr2 = LL(N * N * a);
            fa.sBr1 = LL(Rp);
            fa.sBr2 = LL(Rp * a * N);
            gemm(fa);
            GemmDesc fr = gemm_nn(LL(N), LL(N), LL(R), s_ss, gri.get(), LL(R), ZY + N, LL(Rp * a),
                                  1.0, Fp[s].get(), LL(N));
            fr.a_kcontig = true;
            fr.nbr1 = LL(a);
            fr.nbr2 = LL(nk);
            fr.sAr1 = LL(R * N);
            fr.sAr2 = LL(R * N * a);
            fr.sBr1 = LL(Rp);
            fr.sBr2 = LL(Rp * a * N);
            gemm(fr);
          }
          // k-term (fock_k) for active orbitals c+i inside this chunk
          const long long i0 = std::max<long long>(0, LL(k0) - LL(c));
          const long long i1 = LL(k0 + nk) - LL(c);
          if (i1 > i0) {
            const size_t ni = static_cast<size_t>(i1 - i0);
            GemmDesc gw = gemm_nn(LL(Rp * ni), LL(N * a), LL(MW), 1.0,
                                  XW.Wst[s].get() + Rp * i0, LL(Rp * a), b1wl.get() + N * c,
                                  LL(No), 0.0, Wk, LL(Rp * ni));
            gw.b_ncontig = true;
            gemm(gw);
            GemmDesc fk = gemm_nn(LL(N), LL(N), LL(Rp), s_ss, Wk, LL(Rp * ni),
                                  ZYV.get() + Rp * a * N * (c + i0 - k0), LL(Rp * a), 1.0,
                                  Fp[s].get(), LL(N));
            fk.a_kcontig = true;
            fk.nbr1 = LL(ni);
            fk.nbr2 = LL(a);
            fk.sAr1 = LL(Rp);
            fk.sAr2 = LL(Rp * ni * N);
            fk.sBr1 = LL(Rp * a * N);
            fk.sBr2 = LL(Rp);
            gemm(fk);
          }
        }
      }
    }
  }

  // =====================================================================
  // energies and the symmetrised Fock matrix
  // =====================================================================
  clock.mark("finish");
  double e[kSlots];
  UW12_CUDA(cudaMemcpyAsync(e, acc.get(), sizeof(e), cudaMemcpyDeviceToHost, st));
  if (rq.fock && calc) {
    double* dst = rq.fock;
    DevBuf out;
    if (!rq.fock_device) {
      out.alloc(N * N * ns);
      dst = out.get();
    }
    for (int s = 0; s < ns; ++s) symmetrise(Fp[s].get(), LL(N), LL(N), dst + N * N * s, LL(N));
    if (!rq.fock_device)
      UW12_CUDA(cudaMemcpyAsync(rq.fock, dst, N * N * ns * sizeof(double), cudaMemcpyDeviceToHost,
                                st));
    UW12_CUDA(cudaStreamSynchronize(st));
  } else {
    if (rq.fock) {
      if (rq.fock_device)
        UW12_CUDA(cudaMemsetAsync(rq.fock, 0, N * N * ns * sizeof(double), st));
      else
        std::fill(rq.fock, rq.fock + N * N * ns, 0.0);
    }
    UW12_CUDA(cudaStreamSynchronize(st));
  }
  clock.mark("end");
  clock.finish();
  const double e2 = e[kE2d] + (do_ind ? s_ss * e[kE2i] : 0.0);
  const double e3 = e[kE3d] + (do_ind ? s_ss * e[kE3i] : 0.0);
  const double e4 = e[kE4d] + (do_ind ? s_ss * e[kE4i] : 0.0);
  const double total = e2 + e3 + e4;
  if (rq.energy) *rq.energy = total;
  if (rq.terms) {
    rq.terms[0] = e2;
    rq.terms[1] = e3;
    rq.terms[2] = e4;
  }
  if (rq.print_level > 0) {
    // print.hpp:13-42 formatting
    auto line = [](char ch) { for (int i = 0; i < 48; ++i) std::putchar(ch); std::putchar('\n'); };
    auto res = [](const char* s, double v) {
      std::string str(s);
      std::printf(" %s:%*s%12.6f\n", s, int(32 - str.size()), "", v);
    };
    if (rq.print_level > 2) {
      std::printf("\n");
      line('=');
      std::printf(" UW12 Calculation\n");
      line('=');
    }
    if (rq.print_level > 1) {
      res("Two electron energy", e2);
      res("Three electron energy", e3);
      res("Four electron energy", e4);
    }
    if (rq.print_level > 2) line('=');
    res("Total UW12 energy", total);
    std::fflush(stdout);
  }
}

// --------------------------------------------------------------------------
// reverse mode (direct terms, and the same-spin terms with indirect_term)
// --------------------------------------------------------------------------
// Energy of the direct terms, with f = f(s, s') the spin factor
// (four_electron_utils.cpp:9-30) and everything in the metric eigenbasis:
//   E = sum_{s,s'} f [ 1/2 X_D[s] . (L_WV X_D[s'])        (two_electron.cpp:37-81)
//                    + 1/2 < t~[s'], t[s] >               (four_electron.cpp:80-137)
//                    - < X[s], t~[s'] > ]                 (direct_utils.cpp:136-157)
// t = B2_W^T B2_V, t~ = L_W t L_V, X = Wst_W^T (I (x) S^-1) Wst_V.  Reverse sweep:
//   tbar[s] = sum_s' f (1/2 t~[s'] + L_W (1/2 t[s'] - X[s']) L_V),
//   Xbar[s] = -sum_s' f t~[s'];
//   B2bar_W = B2_V tbar^T, B2bar_V = B2_W tbar; Wstbar_W = SV_V Xbar^T,
//   Wstbar_V = SW_W Xbar (SW = (I (x) S^-1) Wst);
//   B1bar = Ca B2bar (+ the AO rows of Wstbar), Bribar = the RI rows of Wstbar;
//   B1bar_0 = B1bar P2^T, Bribar_0 = Bribar P2^T;
//   dE/dJ3_0[:, A] = packed-symmetric sum of B1bar_0[:, A] Co^T (N x N per A),
//   dE/dJ3_ri_0[:, A] = Bribar_0[:, A] Ca^T (R x N per A);
//   dE/dJ3_0^WV = 1/2 n_spin lower(D, 2) (P2 Xbar_D)^T, Xbar_D[s] = sum_s' f L X_D[s'].
// In the original aux basis E depends on each metric only through K = J2^-1
// (e.g. <t~[s'], t[s]> = tr(T0[s']^T K_W T0[s] K_V)), so dE/dJ2 = -K (dE/dK) K,
// which in the eigenbasis (Q = P2 L) reads
//   dE/dJ2_W  = -sym(Q_W [sum_s 1/2 T_s L_V t[s]^T - X[s] L_V T_s^T] Q_W^T),
//   dE/dJ2_V  = -sym(Q_V [sum_s 1/2 t[s]^T L_W T_s - T_s^T L_W X[s]] Q_V^T),
//   dE/dJ2_WV = -1/2 sum_{s,s'} f (Q X_D[s]) (Q X_D[s'])^T,
// with T_s = sum_s' f t[s'].  With indirect_term the same-spin energies
// (s_ss times E2-, E3-, E4-) add their own B2-bar, Wst-bar and metric terms
// (comment at the same-spin section below).
void form_fock_adjoint(const FockRequest& rq_in, const AdjointOutputs& out) {
  FockRequest rq = rq_in;
  if (rq.n_shards > 1) throw Error(kErrInvalid, "the adjoint evaluates unsharded");
  form_fock(rq);
  PhaseClock clock;
  clock.mark("adj_recompute");

  const IntegralsHandle& W = *rq.W;
  const IntegralsHandle& V = *rq.V;
  const IntegralsHandle& WV = *rq.WV;
  const AbsHandle& AB = *rq.abs;
  const int ns = rq.n_spin;
  const size_t N = rq.n_ao, np = packed_size(N);
  const size_t MW = W.n_df, MV = V.n_df, MX = WV.n_df;
  const size_t R = W.n_ri, Rp = N + R;
  const double two = (ns == 1) ? 2.0 : 1.0;
  cudaStream_t st = current_stream();
  size_t budget = auto_budget_doubles(rq.mem_budget);
  double F[2][2] = {{0, 0}, {0, 0}};
  for (int s = 0; s < ns; ++s)
    for (int sp = 0; sp < ns; ++sp) F[s][sp] = spin_factor(ns, s, sp, rq.s_os, rq.s_ss);

  std::vector<SpinDims> sd;
  size_t o_tot = 0, a_tot = 0;
  DevBuf Co, Ca;
  upload_orbitals(rq, sd, o_tot, a_tot, Co, Ca);
  auto Ca_s = [&](int s) { return Ca.get() + N * sd[s].aoff; };

  // output targets: the caller's device buffers, or device staging for host outputs
  std::vector<std::pair<DevBuf, double*>> staged;
  auto target = [&](double* user, size_t n) -> double* {
    if (!user) return nullptr;
    if (out.device_mem) return user;
    staged.emplace_back(DevBuf(n), user);
    return staged.back().first.get();
  };
  double* gJ3[3] = {target(out.dJ3[0], np * MW), target(out.dJ3[1], np * MV),
                    target(out.dJ3[2], np * MX)};
  double* gJ3ri[2] = {target(out.dJ3_ri[0], R * N * MW), target(out.dJ3_ri[1], R * N * MV)};
  double* gJ2[3] = {target(out.dJ2[0], MW * MW), target(out.dJ2[1], MV * MV),
                    target(out.dJ2[2], MX * MX)};

  // Without same-spin terms every recomputed intermediate enters the gradients
  // through sums over orbitals: X_AB and t over active / occupied orbitals,
  // B2-bar of occupied orbital k from the other potential's B2 of k alone, and
  // Wst-bar of active orbital j from the other potential's S^-1 Wst of j alone.
  // When the whole intermediates (B2, Wst and S^-1 Wst of W and V per spin,
  // and the transforms they come from) would not fit -- an explicit budget,
  // or 90 % of the free device memory -- they are formed for a chunk of
  // orbitals at a time instead (orbital_chunked), and only the gradient
  // factors B1-bar (N o x M) and, when the RI gradient is wanted, Bri-bar
  // (R a x M) are held whole.
  const bool same_spin = rq.indirect && rq.s_ss != 0.0;
  const size_t Mmax = std::max(MW, MV);
  size_t whole = (N * o_tot + R * a_tot) * Mmax;
  for (int s = 0; s < ns; ++s)
    whole += 2 * (sd[s].a * sd[s].o + 2 * Rp * sd[s].a) * Mmax;
  const bool orbital_chunked = !same_spin && whole > auto_budget_doubles(rq.mem_budget, 0.9);
  // B1 (N*nk x M) of occupied orbitals [k0, k0 + nk) of spin s for potential X:
  // sq(J3_0[:, A]) Co[:, k] P2
  auto b1_chunk = [&](const IntegralsHandle& X, int s, size_t k0, size_t nk, DevBuf& dst) {
    const size_t M = X.n_df;
    DevBuf H(N * nk * M);
    transform_ao(X, Co.get() + N * (sd[s].ooff + k0), nk, H.get(), budget / 2);
    dst.alloc(N * nk * M);
    gemm(gemm_nn(LL(N * nk), LL(M), LL(M), 1.0, H.get(), LL(N * nk), X.P2.get(), LL(M), 0.0,
                 dst.get(), LL(N * nk)));
  };
  // Wst (R' nj x M) of active orbitals [j0, j0 + nj) of spin s for potential
  // X: per orbital the AO rows sq(J3_0) Co[:, c + j] P2, then the RI rows
  // J3ri_0 Ca[:, j] P2
  auto wst_chunk = [&](const IntegralsHandle& X, int s, size_t j0, size_t nj, double* St) {
    const size_t M = X.n_df;
    {
      DevBuf H(N * nj * M);
      transform_ao(X, Co.get() + N * (sd[s].ooff + sd[s].c + j0), nj, H.get(), budget / 2);
      GemmDesc ga = gemm_nn(LL(N), LL(M), LL(M), 1.0, H.get(), LL(N * nj), X.P2.get(), LL(M),
                            0.0, St, LL(Rp * nj));
      ga.nbo1 = LL(nj);
      ga.sAo1 = LL(N);
      ga.sCo1 = LL(Rp);
      gemm(ga);
    }
    DevBuf H2(R * nj * M);
    ri_transform(X, Ca_s(s) + N * j0, nj, H2.get(), budget);
    GemmDesc gr = gemm_nn(LL(R), LL(M), LL(M), 1.0, H2.get(), LL(R * nj), X.P2.get(), LL(M), 0.0,
                          St + N, LL(Rp * nj));
    gr.nbo1 = LL(nj);
    gr.sAo1 = LL(R);
    gr.sCo1 = LL(Rp);
    gemm(gr);
  };
  // occupied orbitals per chunk (B1 and its transform, B2 of the chunk and its
  // adjoint) and active orbitals per chunk (the transforms, Wst of the chunk,
  // S^-1 Wst and Wst-bar), as in form_fock's chunked X_AB and t passes
  auto per_k = [&](int s) { return (4 * N + 2 * sd[s].a) * Mmax; };
  const size_t per_j = (N + R + 3 * Rp) * Mmax;

  // ---- forward intermediates (as in form_fock): B2, Wst, (I (x) S^-1) Wst per X, spin
  struct PerX {
    std::vector<DevBuf> B2, Wst, SW;
  };
  PerX XW, XV;
  for (int which = 0; which < 2 && !orbital_chunked; ++which) {
    const IntegralsHandle& X = which == 0 ? W : V;
    PerX& P = which == 0 ? XW : XV;
    const size_t M = X.n_df;
    P.B2.resize(ns);
    P.Wst.resize(ns);
    P.SW.resize(ns);
    budget = auto_budget_doubles(rq.mem_budget);
    DevBuf H(N * o_tot * M);
    transform_ao(X, Co.get(), o_tot, H.get(), budget / 2);
    DevBuf H2(R * a_tot * M);
    if (a_tot) ri_transform(X, Ca.get(), a_tot, H2.get(), budget);
    for (int s = 0; s < ns; ++s) {
      const size_t o = sd[s].o, a = sd[s].a, c = sd[s].c;
      if (!a) continue;
      DevBuf B1(N * o * M);
      gemm(gemm_nn(LL(N * o), LL(M), LL(M), 1.0, H.get() + N * sd[s].ooff, LL(N * o_tot),
                   X.P2.get(), LL(M), 0.0, B1.get(), LL(N * o)));
      P.B2[s].alloc(a * o * M);
      GemmDesc g3 = gemm_nn(LL(a), LL(o * M), LL(N), 1.0, Ca_s(s), LL(N), B1.get(), LL(N), 0.0,
                            P.B2[s].get(), LL(a));
      g3.a_kcontig = true;
      gemm(g3);
      P.Wst[s].alloc(Rp * a * M);
      copy3d(B1.get() + N * c, LL(N), LL(N * o), P.Wst[s].get(), LL(Rp), LL(Rp * a), LL(N),
             LL(a), LL(M));
      GemmDesc g2 = gemm_nn(LL(R), LL(M), LL(M), 1.0, H2.get() + R * sd[s].aoff, LL(R * a_tot),
                            X.P2.get(), LL(M), 0.0, P.Wst[s].get() + N, LL(Rp * a));
      g2.nbo1 = LL(a);
      g2.sAo1 = LL(R);
      g2.sCo1 = LL(Rp);
      gemm(g2);
      P.SW[s].alloc(Rp * a * M);
      gemm(gemm_nn(LL(Rp), LL(a * M), LL(Rp), 1.0, AB.Sinv.get(), LL(Rp), P.Wst[s].get(),
                   LL(Rp), 0.0, P.SW[s].get(), LL(Rp)));
    }
  }
  // X, t, t~ per spin (zero for a spin without active orbitals)
  std::vector<DevBuf> Xab(ns), tab(ns), ttl(ns);
  for (int s = 0; s < ns; ++s) {
    const size_t o = sd[s].o, a = sd[s].a;
    Xab[s].alloc(MW * MV);
    tab[s].alloc(MW * MV);
    ttl[s].alloc(MW * MV);
    if (a == 0) {
      Xab[s].zero();
      tab[s].zero();
      ttl[s].zero();
      continue;
    }
    if (orbital_chunked) {
      // X_AB = sum over active-orbital chunks of Wst_W[j]^T S^-1 Wst_V[j];
      // t = sum over occupied-orbital chunks of B2_W[k]^T B2_V[k]
      Xab[s].zero();
      tab[s].zero();
      const size_t jc = std::max<size_t>(1, std::min(a, budget / 2 / per_j));
      for (size_t j0 = 0; j0 < a; j0 += jc) {
        const size_t nj = std::min(jc, a - j0);
        DevBuf Sw(Rp * nj * MW), SVj(Rp * nj * MV);
        {
          DevBuf Sv(Rp * nj * MV);
          wst_chunk(V, s, j0, nj, Sv.get());
          gemm(gemm_nn(LL(Rp), LL(nj * MV), LL(Rp), 1.0, AB.Sinv.get(), LL(Rp), Sv.get(),
                       LL(Rp), 0.0, SVj.get(), LL(Rp)));
        }
        wst_chunk(W, s, j0, nj, Sw.get());
        GemmDesc gx = gemm_nn(LL(MW), LL(MV), LL(Rp * nj), 1.0, Sw.get(), LL(Rp * nj), SVj.get(),
                              LL(Rp * nj), 1.0, Xab[s].get(), LL(MW));
        gx.a_kcontig = true;
        gemm(gx);
      }
      const size_t kc = std::max<size_t>(1, std::min(o, budget / 2 / per_k(s)));
      for (size_t k0 = 0; k0 < o; k0 += kc) {
        const size_t nk = std::min(kc, o - k0);
        DevBuf B2w(a * nk * MW), B2v(a * nk * MV);
        for (int which = 0; which < 2; ++which) {
          const IntegralsHandle& X = which == 0 ? W : V;
          DevBuf B1;
          b1_chunk(X, s, k0, nk, B1);
          GemmDesc g3 = gemm_nn(LL(a), LL(nk * X.n_df), LL(N), 1.0, Ca_s(s), LL(N), B1.get(),
                                LL(N), 0.0, (which == 0 ? B2w : B2v).get(), LL(a));
          g3.a_kcontig = true;
          gemm(g3);
        }
        GemmDesc gt = gemm_nn(LL(MW), LL(MV), LL(a * nk), 1.0, B2w.get(), LL(a * nk), B2v.get(),
                              LL(a * nk), 1.0, tab[s].get(), LL(MW));
        gt.a_kcontig = true;
        gemm(gt);
      }
      scale_rc(tab[s].get(), LL(MW), LL(MW), LL(MV), W.lam.get(), V.lam.get(), 1.0,
               ttl[s].get(), LL(MW));
      continue;
    }
    GemmDesc gx = gemm_nn(LL(MW), LL(MV), LL(Rp * a), 1.0, XW.Wst[s].get(), LL(Rp * a),
                          XV.SW[s].get(), LL(Rp * a), 0.0, Xab[s].get(), LL(MW));
    gx.a_kcontig = true;
    gemm(gx);
    GemmDesc gt = gemm_nn(LL(MW), LL(MV), LL(a * o), 1.0, XW.B2[s].get(), LL(a * o),
                          XV.B2[s].get(), LL(a * o), 0.0, tab[s].get(), LL(MW));
    gt.a_kcontig = true;
    gemm(gt);
    scale_rc(tab[s].get(), LL(MW), LL(MW), LL(MV), W.lam.get(), V.lam.get(), 1.0, ttl[s].get(),
             LL(MW));
  }

  clock.mark("adj_t_x");
  // ---- adjoints of t and X
  std::vector<DevBuf> tbar(ns), Xbar(ns);
  for (int s = 0; s < ns; ++s) {
    const double* mats[6];
    double coefs[6];
    int scaled[6];
    int nt = 0;
    for (int sp = 0; sp < ns; ++sp) {
      mats[nt] = ttl[sp].get(); coefs[nt] = 0.5 * F[s][sp]; scaled[nt++] = 0;
      mats[nt] = tab[sp].get(); coefs[nt] = 0.5 * F[sp][s]; scaled[nt++] = 1;
      mats[nt] = Xab[sp].get(); coefs[nt] = -F[sp][s]; scaled[nt++] = 1;
    }
    tbar[s].alloc(MW * MV);
    lincomb(tbar[s].get(), LL(MW), LL(MV), nt, mats, coefs, scaled, W.lam.get(), V.lam.get());
    nt = 0;
    for (int sp = 0; sp < ns; ++sp) {
      mats[nt] = ttl[sp].get(); coefs[nt] = -F[s][sp]; scaled[nt++] = 0;
    }
    Xbar[s].alloc(MW * MV);
    lincomb(Xbar[s].get(), LL(MW), LL(MV), nt, mats, coefs, scaled, nullptr, nullptr);
  }

  // ---- same-spin terms (indirect_term with s_ss != 0), energy s_ss E_ss:
  //   E3- = esf <YW, P3(ZV)>, YW = Wst_W L_W B2_W^T, ZV = SW_V L_V B2_V^T
  //   E4- = -1/2 esf <W4, P4(V4)>, W4 = B2_W L_W B2_W^T, V4 = B2_V L_V B2_V^T
  //   E2- = -1/2 esf <B2_WV L_WV, B2_WV> (WV over the active orbitals, below)
  // (esf = 2 closed shell, 1 open; P3, P4 the index exchanges of perm_3el,
  // perm_4el). Their B2-bar and Wst-bar join the direct ones before the
  // transforms are reversed; each L between eigenbasis factors adds
  // (left factor)^T G (right factor) to the metric's A matrix:
  //   G_Y = s esf P3(ZV), G_Z = s esf P3(YW) (chunks of occupied k),
  //   Wst_W-bar = (sum_k G_Y B2_W,k) L_W, B2_W,k-bar = (G_Y^T Wst_W) L_W,
  //   SW_V-bar = (sum_k G_Z B2_V,k) L_V -> Wst_V-bar = (I (x) S^-1) SW_V-bar,
  //   B2_V,k-bar = (G_Z^T SW_V) L_V;  A_W += Wst_W^T T_Y, A_V += SW_V^T T_Z;
  //   G_W4 = -1/2 s esf P4(V4): B2_W-bar += 2 (G_W4 B2_W) L_W,
  //   A_W += B2_W^T G_W4 B2_W (and W <-> V with P4(W4)).
  clock.mark("adj_same_spin");
  std::vector<DevBuf> ssB2b[2], ssWsb[2];
  DevBuf ssA[2];
  if (same_spin) {
    const double gs = two * rq.s_ss;
    ssA[0].alloc(MW * MW);
    ssA[0].zero();
    ssA[1].alloc(MV * MV);
    ssA[1].zero();
    for (int which = 0; which < 2; ++which) {
      ssB2b[which].resize(ns);
      ssWsb[which].resize(ns);
    }
    for (int s = 0; s < ns; ++s) {
      const size_t o = sd[s].o, a = sd[s].a;
      if (a == 0 || o == 0) continue;
      const size_t ao = a * o, Ra = Rp * a;
      ssB2b[0][s].alloc(ao * MW);
      ssB2b[1][s].alloc(ao * MV);
      DevBuf b2wl(ao * MW), b2vl(ao * MV);
      scale_rc(XW.B2[s].get(), LL(ao), LL(ao), LL(MW), nullptr, W.lam.get(), 1.0, b2wl.get(),
               LL(ao));
      scale_rc(XV.B2[s].get(), LL(ao), LL(ao), LL(MV), nullptr, V.lam.get(), 1.0, b2vl.get(),
               LL(ao));
      // three-electron, chunks of occupied orbitals k
      {
        budget = auto_budget_doubles(rq.mem_budget);
        const size_t per_k = 3 * Ra * a + a * std::max(MW, MV);
        const size_t kc = tile_chunk(o, a, std::max<size_t>(1, std::min(o, budget / per_k)));
        DevBuf TY(Ra * MW), TZ(Ra * MV), Tmp(Ra * a * kc), GY(Ra * a * kc), GZ(Ra * a * kc),
            Bt(a * kc * std::max(MW, MV));
        for (size_t k0 = 0; k0 < o; k0 += kc) {
          const size_t nk = std::min(kc, o - k0);
          const double beta = k0 ? 1.0 : 0.0;
          GemmDesc g = gemm_nn(LL(Ra), LL(a * nk), LL(MV), 1.0, XV.SW[s].get(), LL(Ra),
                               b2vl.get() + a * k0, LL(ao), 0.0, Tmp.get(), LL(Ra));
          g.b_ncontig = true;
          gemm(g);
          perm_3el(Tmp.get(), GY.get(), LL(Rp), LL(a), LL(nk), gs);
          g = gemm_nn(LL(Ra), LL(a * nk), LL(MW), 1.0, XW.Wst[s].get(), LL(Ra),
                      b2wl.get() + a * k0, LL(ao), 0.0, Tmp.get(), LL(Ra));
          g.b_ncontig = true;
          gemm(g);
          perm_3el(Tmp.get(), GZ.get(), LL(Rp), LL(a), LL(nk), gs);
          gemm(gemm_nn(LL(Ra), LL(MW), LL(a * nk), 1.0, GY.get(), LL(Ra),
                       XW.B2[s].get() + a * k0, LL(ao), beta, TY.get(), LL(Ra)));
          gemm(gemm_nn(LL(Ra), LL(MV), LL(a * nk), 1.0, GZ.get(), LL(Ra),
                       XV.B2[s].get() + a * k0, LL(ao), beta, TZ.get(), LL(Ra)));
          g = gemm_nn(LL(a * nk), LL(MW), LL(Ra), 1.0, GY.get(), LL(Ra), XW.Wst[s].get(),
                      LL(Ra), 0.0, Bt.get(), LL(a * nk));
          g.a_kcontig = true;
          gemm(g);
          scale_rc(Bt.get(), LL(a * nk), LL(a * nk), LL(MW), nullptr, W.lam.get(), 1.0,
                   ssB2b[0][s].get() + a * k0, LL(ao));
          g = gemm_nn(LL(a * nk), LL(MV), LL(Ra), 1.0, GZ.get(), LL(Ra), XV.SW[s].get(), LL(Ra),
                      0.0, Bt.get(), LL(a * nk));
          g.a_kcontig = true;
          gemm(g);
          scale_rc(Bt.get(), LL(a * nk), LL(a * nk), LL(MV), nullptr, V.lam.get(), 1.0,
                   ssB2b[1][s].get() + a * k0, LL(ao));
        }
        Tmp = DevBuf();  // the chunk buffers are done: their memory goes to Wst-bar
        GY = DevBuf();
        GZ = DevBuf();
        Bt = DevBuf();
        GemmDesc g = gemm_nn(LL(MW), LL(MW), LL(Ra), 1.0, XW.Wst[s].get(), LL(Ra), TY.get(),
                             LL(Ra), 1.0, ssA[0].get(), LL(MW));
        g.a_kcontig = true;
        gemm(g);
        g = gemm_nn(LL(MV), LL(MV), LL(Ra), 1.0, XV.SW[s].get(), LL(Ra), TZ.get(), LL(Ra), 1.0,
                    ssA[1].get(), LL(MV));
        g.a_kcontig = true;
        gemm(g);
        // Wst_W-bar = T_Y L_W in place; Wst_V-bar = (I (x) S^-1) (T_Z L_V)
        scale_rc(TY.get(), LL(Ra), LL(Ra), LL(MW), nullptr, W.lam.get(), 1.0, TY.get(), LL(Ra));
        ssWsb[0][s] = std::move(TY);
        scale_rc(TZ.get(), LL(Ra), LL(Ra), LL(MV), nullptr, V.lam.get(), 1.0, TZ.get(), LL(Ra));
        ssWsb[1][s].alloc(Ra * MV);
        gemm(gemm_nn(LL(Rp), LL(a * MV), LL(Rp), 1.0, AB.Sinv.get(), LL(Rp), TZ.get(), LL(Rp),
                     0.0, ssWsb[1][s].get(), LL(Rp)));
        TZ = DevBuf();
      }
      // four-electron
      {
        DevBuf W4(ao * ao), V4(ao * ao), G4(ao * ao), T4(ao * std::max(MW, MV));
        GemmDesc g = gemm_nn(LL(ao), LL(ao), LL(MW), 1.0, b2wl.get(), LL(ao), XW.B2[s].get(),
                             LL(ao), 0.0, W4.get(), LL(ao));
        g.b_ncontig = true;
        gemm(g);
        g = gemm_nn(LL(ao), LL(ao), LL(MV), 1.0, b2vl.get(), LL(ao), XV.B2[s].get(), LL(ao), 0.0,
                    V4.get(), LL(ao));
        g.b_ncontig = true;
        gemm(g);
        for (int which = 0; which < 2; ++which) {
          const size_t M = which == 0 ? MW : MV;
          const DevBuf& B2 = which == 0 ? XW.B2[s] : XV.B2[s];
          const double* lam = which == 0 ? W.lam.get() : V.lam.get();
          perm_4el(which == 0 ? V4.get() : W4.get(), G4.get(), LL(a), LL(o), -0.5 * gs);
          gemm(gemm_nn(LL(ao), LL(M), LL(ao), 1.0, G4.get(), LL(ao), B2.get(), LL(ao), 0.0,
                       T4.get(), LL(ao)));
          GemmDesc ga = gemm_nn(LL(M), LL(M), LL(ao), 1.0, B2.get(), LL(ao), T4.get(), LL(ao),
                                1.0, ssA[which].get(), LL(M));
          ga.a_kcontig = true;
          gemm(ga);
          const double* mats[2] = {ssB2b[which][s].get(), T4.get()};
          const double coefs[2] = {1.0, 2.0};
          const int scaled[2] = {0, 1};
          lincomb(ssB2b[which][s].get(), LL(ao), LL(M), 2, mats, coefs, scaled, nullptr, lam);
        }
      }
    }
  }

  clock.mark("adj_three_index");
  // ---- dE/dJ3_0 and dE/dJ3_ri_0 of W and V, orbital-chunked: B2-bar of
  // occupied orbitals k (B2-bar_W = B2_V t-bar^T, B2-bar_V = B2_W t-bar) and
  // Wst-bar of active orbitals j (Wst-bar_W = S^-1 Wst_V X-bar^T,
  // Wst-bar_V = S^-1 Wst_W X-bar) from the other potential's intermediates of
  // those orbitals, formed afresh per chunk, into the whole B1-bar (and
  // Bri-bar); then B1-bar P2^T per block of aux functions
  for (int which = 0; which < 2 && orbital_chunked; ++which) {
    const IntegralsHandle& X = which == 0 ? W : V;
    const IntegralsHandle& Y = which == 0 ? V : W;  // the other potential
    const size_t M = X.n_df, MY = Y.n_df;
    double* g3 = gJ3[which];
    double* g3ri = gJ3ri[which];
    const GradSink& s3 = out.sink3[which];
    const GradSink& s3ri = out.sink3_ri[which];
    const bool want3 = g3 || s3, want_ri = g3ri || s3ri;
    if (!want3 && !want_ri) continue;
    DevBuf Bb1(N * o_tot * M), Bbri;
    Bb1.zero();  // the columns of spins without active orbitals stay zero
    if (want_ri && a_tot) Bbri.alloc(R * a_tot * M);
    budget = auto_budget_doubles(rq.mem_budget);
    for (int s = 0; s < ns; ++s) {
      const size_t o = sd[s].o, a = sd[s].a, c = sd[s].c;
      if (!a) continue;
      // B1-bar[:, k] = Ca B2-bar[:, k] over chunks of occupied k (written)
      const size_t kc = std::max<size_t>(1, std::min(o, budget / 2 / per_k(s)));
      for (size_t k0 = 0; k0 < o; k0 += kc) {
        const size_t nk = std::min(kc, o - k0);
        DevBuf B2y(a * nk * MY), B2b(a * nk * M);
        {
          DevBuf B1y;
          b1_chunk(Y, s, k0, nk, B1y);
          GemmDesc g3y = gemm_nn(LL(a), LL(nk * MY), LL(N), 1.0, Ca_s(s), LL(N), B1y.get(),
                                 LL(N), 0.0, B2y.get(), LL(a));
          g3y.a_kcontig = true;
          gemm(g3y);
        }
        GemmDesc gb = gemm_nn(LL(a * nk), LL(M), LL(MY), 1.0, B2y.get(), LL(a * nk),
                              tbar[s].get(), LL(MW), 0.0, B2b.get(), LL(a * nk));
        gb.b_ncontig = which == 0;  // t-bar is MW x MV
        gemm(gb);
        GemmDesc g1 = gemm_nn(LL(N), LL(nk), LL(a), 1.0, Ca_s(s), LL(N), B2b.get(), LL(a), 0.0,
                              Bb1.get() + N * (sd[s].ooff + k0), LL(N));
        g1.nbo1 = LL(M);
        g1.sBo1 = LL(a * nk);
        g1.sCo1 = LL(N * o_tot);
        gemm(g1);
      }
      // Wst-bar of active orbitals j: AO rows added to B1-bar[:, c + j], RI
      // rows into Bri-bar[:, j]
      const size_t jc = std::max<size_t>(1, std::min(a, budget / 2 / per_j));
      for (size_t j0 = 0; j0 < a; j0 += jc) {
        const size_t nj = std::min(jc, a - j0);
        DevBuf SYj(Rp * nj * MY);
        {
          DevBuf Sy(Rp * nj * MY);
          wst_chunk(Y, s, j0, nj, Sy.get());
          gemm(gemm_nn(LL(Rp), LL(nj * MY), LL(Rp), 1.0, AB.Sinv.get(), LL(Rp), Sy.get(),
                       LL(Rp), 0.0, SYj.get(), LL(Rp)));
        }
        DevBuf Wsb(Rp * nj * M);
        GemmDesc gw = gemm_nn(LL(Rp * nj), LL(M), LL(MY), 1.0, SYj.get(), LL(Rp * nj),
                              Xbar[s].get(), LL(MW), 0.0, Wsb.get(), LL(Rp * nj));
        gw.b_ncontig = which == 0;  // X-bar is MW x MV
        gemm(gw);
        copy3d(Wsb.get(), LL(Rp), LL(Rp * nj), Bb1.get() + N * (sd[s].ooff + c + j0), LL(N),
               LL(N * o_tot), LL(N), LL(nj), LL(M), 1.0, 1.0);
        if (Bbri.size())
          copy3d(Wsb.get() + N, LL(Rp), LL(Rp * nj), Bbri.get() + R * (sd[s].aoff + j0), LL(R),
                 LL(R * a_tot), LL(R), LL(nj), LL(M));
      }
    }
    if (want3) {
      // per block of aux functions: B1-bar_0 = B1-bar P2^T (the block's
      // columns), then per aux function the packed symmetric sum of B1-bar_0 Co^T
      const size_t ac = std::max<size_t>(1, std::min(M, budget / (2 * N * N + N * o_tot)));
      DevBuf Bb10(N * o_tot * ac), G(N * N * ac), Pk;
      if (!g3) Pk.alloc(np * ac);  // one streamed block
      for (size_t a0 = 0; a0 < M; a0 += ac) {
        const size_t na = std::min(ac, M - a0);
        GemmDesc gp = gemm_nn(LL(N * o_tot), LL(na), LL(M), 1.0, Bb1.get(), LL(N * o_tot),
                              X.P2.get() + a0, LL(M), 0.0, Bb10.get(), LL(N * o_tot));
        gp.b_ncontig = true;
        gemm(gp);
        GemmDesc g = gemm_nn(LL(N), LL(N), LL(o_tot), 1.0, Bb10.get(), LL(N), Co.get(), LL(N), 0.0,
                             G.get(), LL(N));
        g.b_ncontig = true;
        g.nbo1 = LL(na);
        g.sAo1 = LL(N * o_tot);
        g.sCo1 = LL(N * N);
        gemm(g);
        pack_sym_sum(G.get(), LL(N), LL(na), g3 ? g3 + np * a0 : Pk.get(), LL(np));
        if (!g3) s3(a0, na, Pk.get(), np, st);
      }
    }
    if (want_ri) {
      // as in the whole form: one batched GEMM into the whole gradient, or
      // aux blocks of at most a quarter of the budget when streamed
      const size_t rows = R * N;
      const size_t step = g3ri ? M : std::max<size_t>(1, std::min(M, budget / (4 * rows)));
      DevBuf Rk;
      if (!g3ri) Rk.alloc(rows * step);
      if (a_tot == 0) {
        if (g3ri) {
          UW12_CUDA(cudaMemsetAsync(g3ri, 0, R * N * M * sizeof(double), st));
        } else {
          Rk.zero();
          for (size_t b0 = 0; b0 < M; b0 += step) s3ri(b0, std::min(step, M - b0), Rk.get(), rows, st);
        }
      } else {
        DevBuf Bbri0(R * a_tot * M);
        GemmDesc gp = gemm_nn(LL(R * a_tot), LL(M), LL(M), 1.0, Bbri.get(), LL(R * a_tot),
                              X.P2.get(), LL(M), 0.0, Bbri0.get(), LL(R * a_tot));
        gp.b_ncontig = true;
        gemm(gp);
        Bbri = DevBuf();
        for (size_t b0 = 0; b0 < M; b0 += step) {
          const size_t nb = std::min(step, M - b0);
          GemmDesc g = gemm_nn(LL(R), LL(N), LL(a_tot), 1.0, Bbri0.get() + R * a_tot * b0, LL(R),
                               Ca.get(), LL(N), 0.0, g3ri ? g3ri + rows * b0 : Rk.get(), LL(R));
          g.b_ncontig = true;
          g.nbo1 = LL(nb);
          g.sAo1 = LL(R * a_tot);
          g.sCo1 = LL(R * N);
          gemm(g);
          if (!g3ri) s3ri(b0, nb, Rk.get(), rows, st);
        }
      }
    }
  }
  // ---- dE/dJ3_0 and dE/dJ3_ri_0 of W and V, whole intermediates
  for (int which = 0; which < 2 && !orbital_chunked; ++which) {
    const IntegralsHandle& X = which == 0 ? W : V;
    const size_t M = X.n_df;
    double* g3 = gJ3[which];
    double* g3ri = gJ3ri[which];
    const GradSink& s3 = out.sink3[which];
    const GradSink& s3ri = out.sink3_ri[which];
    if (!g3 && !g3ri && !s3 && !s3ri) continue;
    budget = auto_budget_doubles(rq.mem_budget);
    DevBuf Bb1(N * o_tot * M), Bbri(R * a_tot * M);
    Bb1.zero();
    for (int s = 0; s < ns; ++s) {
      const size_t o = sd[s].o, a = sd[s].a, c = sd[s].c;
      if (!a) continue;
      // B2bar (a*o x M)
      DevBuf B2b(a * o * M);
      if (which == 0) {
        GemmDesc g = gemm_nn(LL(a * o), LL(MW), LL(MV), 1.0, XV.B2[s].get(), LL(a * o),
                             tbar[s].get(), LL(MW), 0.0, B2b.get(), LL(a * o));
        g.b_ncontig = true;
        gemm(g);
      } else {
        gemm(gemm_nn(LL(a * o), LL(MV), LL(MW), 1.0, XW.B2[s].get(), LL(a * o), tbar[s].get(),
                     LL(MW), 0.0, B2b.get(), LL(a * o)));
      }
      if (same_spin && ssB2b[which][s].size()) {
        const double* mats[2] = {B2b.get(), ssB2b[which][s].get()};
        const double coefs[2] = {1.0, 1.0};
        lincomb(B2b.get(), LL(a * o), LL(M), 2, mats, coefs, nullptr, nullptr, nullptr);
      }
      // B1bar_A (N x o) = Ca_s B2bar_A, into the spin block of Bb1
      GemmDesc g1 = gemm_nn(LL(N), LL(o), LL(a), 1.0, Ca_s(s), LL(N), B2b.get(), LL(a), 0.0,
                            Bb1.get() + N * sd[s].ooff, LL(N));
      g1.nbo1 = LL(M);
      g1.sBo1 = LL(a * o);
      g1.sCo1 = LL(N * o_tot);
      gemm(g1);
      // Wstbar (R'a x M)
      DevBuf Wsb(Rp * a * M);
      if (which == 0) {
        GemmDesc g = gemm_nn(LL(Rp * a), LL(MW), LL(MV), 1.0, XV.SW[s].get(), LL(Rp * a),
                             Xbar[s].get(), LL(MW), 0.0, Wsb.get(), LL(Rp * a));
        g.b_ncontig = true;
        gemm(g);
      } else {
        gemm(gemm_nn(LL(Rp * a), LL(MV), LL(MW), 1.0, XW.SW[s].get(), LL(Rp * a), Xbar[s].get(),
                     LL(MW), 0.0, Wsb.get(), LL(Rp * a)));
      }
      if (same_spin && ssWsb[which][s].size()) {
        const double* mats[2] = {Wsb.get(), ssWsb[which][s].get()};
        const double coefs[2] = {1.0, 1.0};
        lincomb(Wsb.get(), LL(Rp * a), LL(M), 2, mats, coefs, nullptr, nullptr, nullptr);
      }
      // AO rows -> active orbitals of B1bar; RI rows -> Bribar
      copy3d(Wsb.get(), LL(Rp), LL(Rp * a), Bb1.get() + N * (sd[s].ooff + c), LL(N),
             LL(N * o_tot), LL(N), LL(a), LL(M), 1.0, 1.0);
      copy3d(Wsb.get() + N, LL(Rp), LL(Rp * a), Bbri.get() + R * sd[s].aoff, LL(R),
             LL(R * a_tot), LL(R), LL(a), LL(M));
    }
    if (g3 || s3) {
      // B1bar_0 = B1bar P2^T, then per aux function the packed symmetric sum of B1bar_0 Co^T
      DevBuf Bb10(N * o_tot * M);
      GemmDesc gp = gemm_nn(LL(N * o_tot), LL(M), LL(M), 1.0, Bb1.get(), LL(N * o_tot),
                            X.P2.get(), LL(M), 0.0, Bb10.get(), LL(N * o_tot));
      gp.b_ncontig = true;
      gemm(gp);
      const size_t ac = std::max<size_t>(1, std::min(M, budget / (2 * N * N)));
      DevBuf G(N * N * ac), Pk;
      if (!g3) Pk.alloc(np * ac);  // one streamed block
      for (size_t a0 = 0; a0 < M; a0 += ac) {
        const size_t na = std::min(ac, M - a0);
        GemmDesc g = gemm_nn(LL(N), LL(N), LL(o_tot), 1.0, Bb10.get() + N * o_tot * a0, LL(N),
                             Co.get(), LL(N), 0.0, G.get(), LL(N));
        g.b_ncontig = true;
        g.nbo1 = LL(na);
        g.sAo1 = LL(N * o_tot);
        g.sCo1 = LL(N * N);
        gemm(g);
        pack_sym_sum(G.get(), LL(N), LL(na), g3 ? g3 + np * a0 : Pk.get(), LL(np));
        if (!g3) s3(a0, na, Pk.get(), np, st);
      }
    }
    if (g3ri || s3ri) {
      // stored: one batched GEMM into the whole gradient; streamed: aux blocks
      // of at most a quarter of the budget
      const size_t rows = R * N;
      const size_t step = g3ri ? M : std::max<size_t>(1, std::min(M, budget / (4 * rows)));
      DevBuf Rk;
      if (!g3ri) Rk.alloc(rows * step);
      if (a_tot == 0) {
        if (g3ri) {
          UW12_CUDA(cudaMemsetAsync(g3ri, 0, R * N * M * sizeof(double), st));
        } else {
          Rk.zero();
          for (size_t b0 = 0; b0 < M; b0 += step) s3ri(b0, std::min(step, M - b0), Rk.get(), rows, st);
        }
      } else {
        DevBuf Bbri0(R * a_tot * M);
        GemmDesc gp = gemm_nn(LL(R * a_tot), LL(M), LL(M), 1.0, Bbri.get(), LL(R * a_tot),
                              X.P2.get(), LL(M), 0.0, Bbri0.get(), LL(R * a_tot));
        gp.b_ncontig = true;
        gemm(gp);
        for (size_t b0 = 0; b0 < M; b0 += step) {
          const size_t nb = std::min(step, M - b0);
          GemmDesc g = gemm_nn(LL(R), LL(N), LL(a_tot), 1.0, Bbri0.get() + R * a_tot * b0, LL(R),
                               Ca.get(), LL(N), 0.0, g3ri ? g3ri + rows * b0 : Rk.get(), LL(R));
          g.b_ncontig = true;
          g.nbo1 = LL(nb);
          g.sAo1 = LL(R * a_tot);
          g.sCo1 = LL(R * N);
          gemm(g);
          if (!g3ri) s3ri(b0, nb, Rk.get(), rows, st);
        }
      }
    }
  }

  clock.mark("adj_metric");
  // ---- metric gradients of W and V: -sym(Q A Q^T), Q = P2 L
  for (int which = 0; which < 2; ++which) {
    double* g2 = gJ2[which];
    if (!g2) continue;
    const IntegralsHandle& X = which == 0 ? W : V;
    const IntegralsHandle& Y = which == 0 ? V : W;  // the other potential
    const size_t M = X.n_df;
    DevBuf Amat(M * M), Ts(M * M), tmp(M * M);
    Amat.zero();
    for (int s = 0; s < ns; ++s) {
      const double* mats[2];
      double coefs[2];
      for (int sp = 0; sp < ns; ++sp) {
        mats[sp] = tab[sp].get();
        coefs[sp] = F[s][sp];
      }
      lincomb(Ts.get(), LL(MW), LL(MV), ns, mats, coefs, nullptr, nullptr, nullptr);
      if (which == 0) {
        // A_W += 1/2 T_s L_V t[s]^T - X[s] L_V T_s^T
        scale_rc(Ts.get(), LL(MW), LL(MW), LL(MV), nullptr, Y.lam.get(), 1.0, tmp.get(), LL(MW));
        GemmDesc g = gemm_nn(LL(MW), LL(MW), LL(MV), 0.5, tmp.get(), LL(MW), tab[s].get(), LL(MW),
                             1.0, Amat.get(), LL(MW));
        g.b_ncontig = true;
        gemm(g);
        scale_rc(Xab[s].get(), LL(MW), LL(MW), LL(MV), nullptr, Y.lam.get(), 1.0, tmp.get(),
                 LL(MW));
        g = gemm_nn(LL(MW), LL(MW), LL(MV), -1.0, tmp.get(), LL(MW), Ts.get(), LL(MW), 1.0,
                    Amat.get(), LL(MW));
        g.b_ncontig = true;
        gemm(g);
      } else {
        // A_V += 1/2 t[s]^T L_W T_s - T_s^T L_W X[s]
        scale_rc(Ts.get(), LL(MW), LL(MW), LL(MV), Y.lam.get(), nullptr, 1.0, tmp.get(), LL(MW));
        GemmDesc g = gemm_nn(LL(MV), LL(MV), LL(MW), 0.5, tab[s].get(), LL(MW), tmp.get(), LL(MW),
                             1.0, Amat.get(), LL(MV));
        g.a_kcontig = true;
        gemm(g);
        scale_rc(Xab[s].get(), LL(MW), LL(MW), LL(MV), Y.lam.get(), nullptr, 1.0, tmp.get(),
                 LL(MW));
        g = gemm_nn(LL(MV), LL(MV), LL(MW), -1.0, Ts.get(), LL(MW), tmp.get(), LL(MW), 1.0,
                    Amat.get(), LL(MV));
        g.a_kcontig = true;
        gemm(g);
      }
    }
    if (same_spin) {
      const double* mats[2] = {Amat.get(), ssA[which].get()};
      const double coefs[2] = {1.0, 1.0};
      lincomb(Amat.get(), LL(M), LL(M), 2, mats, coefs, nullptr, nullptr, nullptr);
    }
    DevBuf Q(M * M), QA(M * M);
    scale_rc(X.P2.get(), LL(M), LL(M), LL(M), nullptr, X.lam.get(), 1.0, Q.get(), LL(M));
    gemm(gemm_nn(LL(M), LL(M), LL(M), 1.0, Q.get(), LL(M), Amat.get(), LL(M), 0.0, QA.get(),
                 LL(M)));
    GemmDesc g = gemm_nn(LL(M), LL(M), LL(M), -1.0, QA.get(), LL(M), Q.get(), LL(M), 0.0,
                         tmp.get(), LL(M));
    g.b_ncontig = true;
    gemm(g);
    symmetrise(tmp.get(), LL(M), LL(M), g2, LL(M));
  }

  // ---- WV: dE/dJ3_0 and dE/dJ2 through the fitted density, and through the
  // same-spin exchange E2- = -1/2 esf <B2 L, B2> (B2 = Ca^T B1, B1 of the
  // active orbitals, two_electron.cpp:87-132): B2-bar = -s esf B2 L,
  // B1-bar = Ca B2-bar, then P2^T and the packed symmetric sum per aux
  // function with Ca; A_WV = -1/2 s esf B2^T B2
  clock.mark("adj_wv");
  const GradSink& s3x = out.sink3[2];
  std::vector<DevBuf> ssX10(ns);  // B1-bar_0 of WV per spin (N a x MX)
  DevBuf ssAX;
  if (same_spin && (gJ3[2] || s3x || gJ2[2])) {
    const double gs = two * rq.s_ss;
    ssAX.alloc(MX * MX);
    ssAX.zero();
    budget = auto_budget_doubles(rq.mem_budget);
    DevBuf H(N * a_tot * MX);
    transform_ao(WV, Ca.get(), a_tot, H.get(), budget / 2);
    for (int s = 0; s < ns; ++s) {
      const size_t a = sd[s].a;
      if (!a) continue;
      DevBuf B1(N * a * MX), B2(a * a * MX), B2b(a * a * MX), B1b(N * a * MX);
      gemm(gemm_nn(LL(N * a), LL(MX), LL(MX), 1.0, H.get() + N * sd[s].aoff, LL(N * a_tot),
                   WV.P2.get(), LL(MX), 0.0, B1.get(), LL(N * a)));
      GemmDesc g2 = gemm_nn(LL(a), LL(a * MX), LL(N), 1.0, Ca_s(s), LL(N), B1.get(), LL(N), 0.0,
                            B2.get(), LL(a));
      g2.a_kcontig = true;
      gemm(g2);
      GemmDesc ga = gemm_nn(LL(MX), LL(MX), LL(a * a), -0.5 * gs, B2.get(), LL(a * a), B2.get(),
                            LL(a * a), 1.0, ssAX.get(), LL(MX));
      ga.a_kcontig = true;
      gemm(ga);
      scale_rc(B2.get(), LL(a * a), LL(a * a), LL(MX), nullptr, WV.lam.get(), -gs, B2b.get(),
               LL(a * a));
      GemmDesc g1 = gemm_nn(LL(N), LL(a), LL(a), 1.0, Ca_s(s), LL(N), B2b.get(), LL(a), 0.0,
                            B1b.get(), LL(N));
      g1.nbo1 = LL(MX);
      g1.sBo1 = LL(a * a);
      g1.sCo1 = LL(N * a);
      gemm(g1);
      ssX10[s].alloc(N * a * MX);
      GemmDesc gp = gemm_nn(LL(N * a), LL(MX), LL(MX), 1.0, B1b.get(), LL(N * a), WV.P2.get(),
                            LL(MX), 0.0, ssX10[s].get(), LL(N * a));
      gp.b_ncontig = true;
      gemm(gp);
    }
  }
  // adds the same-spin part of dE/dJ3_0^WV for aux functions [b0, b0 + nb)
  // to dst (packed rows, leading dimension np)
  auto add_ss_wv = [&](size_t b0, size_t nb, double* dst) {
    if (!same_spin) return;
    const size_t ac = std::max<size_t>(1, std::min(nb, budget / (4 * N * N)));
    DevBuf G(N * N * ac);
    for (int s = 0; s < ns; ++s) {
      const size_t a = sd[s].a;
      if (!a) continue;
      for (size_t c0 = 0; c0 < nb; c0 += ac) {
        const size_t nc = std::min(ac, nb - c0);
        GemmDesc g = gemm_nn(LL(N), LL(N), LL(a), 1.0, ssX10[s].get() + N * a * (b0 + c0), LL(N),
                             Ca_s(s), LL(N), 0.0, G.get(), LL(N));
        g.b_ncontig = true;
        g.nbo1 = LL(nc);
        g.sAo1 = LL(N * a);
        g.sCo1 = LL(N * N);
        gemm(g);
        pack_sym_sum(G.get(), LL(N), LL(nc), dst + np * c0, LL(np), 1.0);
      }
    }
  };
  if (gJ3[2] || s3x || gJ2[2]) {
    DevBuf dmat(np * ns), XDr(MX * ns), XD(MX * ns), XDb(MX * ns), vb(MX * ns);
    for (int s = 0; s < ns; ++s)
      pack_density(Ca_s(s), LL(N), LL(N), LL(sd[s].a), two, dmat.get() + np * s);
    fitted_density_raw(WV, dmat.get(), ns, XDr.get(), budget);
    GemmDesc g = gemm_nn(LL(MX), ns, LL(MX), 0.5 * ns, WV.P2.get(), LL(MX), XDr.get(), LL(MX),
                         0.0, XD.get(), LL(MX));
    g.a_kcontig = true;
    gemm(g);
    double coef[4] = {0, 0, 0, 0};
    for (int s = 0; s < ns; ++s)
      for (int sp = 0; sp < ns; ++sp) coef[s * ns + sp] = F[s][sp];
    if (gJ3[2] || s3x) {
      // Xbar_D[s] = L sum_s' f X_D[s'];  dJ3 = 1/2 n_spin dmat (P2 Xbar_D)^T
      combine_vecs(XD.get(), LL(MX), ns, coef, WV.lam.get(), XDb.get());
      gemm(gemm_nn(LL(MX), ns, LL(MX), 1.0, WV.P2.get(), LL(MX), XDb.get(), LL(MX), 0.0, vb.get(),
                   LL(MX)));
      // whole, or in aux blocks of at most a quarter of the budget when streamed
      const size_t step = gJ3[2] ? MX : std::max<size_t>(1, std::min(MX, budget / (4 * np)));
      DevBuf Xk;
      if (!gJ3[2]) Xk.alloc(np * step);
      for (size_t b0 = 0; b0 < MX; b0 += step) {
        const size_t nb = std::min(step, MX - b0);
        double* dst = gJ3[2] ? gJ3[2] + np * b0 : Xk.get();
        GemmDesc gd = gemm_nn(LL(np), LL(nb), ns, 0.5 * ns, dmat.get(), LL(np), vb.get() + b0,
                              LL(MX), 0.0, dst, LL(np));
        gd.b_ncontig = true;
        gemm(gd);
        add_ss_wv(b0, nb, dst);
        if (!gJ3[2]) s3x(b0, nb, Xk.get(), np, st);
      }
    }
    if (gJ2[2]) {
      // U = Q X_D = P2 (L X_D); dJ2 = -1/2 U (U F)^T
      DevBuf LX(MX * ns), U(MX * ns), UF(MX * ns);
      scale_rc(XD.get(), LL(MX), LL(MX), ns, WV.lam.get(), nullptr, 1.0, LX.get(), LL(MX));
      gemm(gemm_nn(LL(MX), ns, LL(MX), 1.0, WV.P2.get(), LL(MX), LX.get(), LL(MX), 0.0, U.get(),
                   LL(MX)));
      for (int s = 0; s < ns; ++s) {
        const double* mats[2] = {U.get(), U.get() + MX};
        double coefs[2] = {F[s][0], ns > 1 ? F[s][1] : 0.0};
        lincomb(UF.get() + MX * s, LL(MX), 1, ns, mats, coefs, nullptr, nullptr, nullptr);
      }
      GemmDesc gd = gemm_nn(LL(MX), LL(MX), ns, -0.5, U.get(), LL(MX), UF.get(), LL(MX), 0.0,
                            gJ2[2], LL(MX));
      gd.b_ncontig = true;
      gemm(gd);
      if (same_spin) {
        // += -Q A_WV Q^T (A_WV symmetric), Q = P2 L
        DevBuf Q(MX * MX), QA(MX * MX);
        scale_rc(WV.P2.get(), LL(MX), LL(MX), LL(MX), nullptr, WV.lam.get(), 1.0, Q.get(),
                 LL(MX));
        gemm(gemm_nn(LL(MX), LL(MX), LL(MX), 1.0, Q.get(), LL(MX), ssAX.get(), LL(MX), 0.0,
                     QA.get(), LL(MX)));
        GemmDesc gq = gemm_nn(LL(MX), LL(MX), LL(MX), -1.0, QA.get(), LL(MX), Q.get(), LL(MX),
                              1.0, gJ2[2], LL(MX));
        gq.b_ncontig = true;
        gemm(gq);
      }
    }
  }

  clock.mark("adj_copy_out");
  for (auto& sg : staged)
    UW12_CUDA(cudaMemcpyAsync(sg.second, sg.first.get(), sg.first.size() * sizeof(double),
                              cudaMemcpyDeviceToHost, st));
  clock.mark("adj_end");
  UW12_CUDA(cudaStreamSynchronize(st));
  clock.finish();
}

std::string phase_profile_read() {
  std::lock_guard<std::mutex> lk(g_phase_mu);
  std::string out;
  for (const auto& kv : g_phase_ms) out += kv.first + "=" + std::to_string(kv.second) + ";";
  g_phase_ms.clear();
  return out;
}

}  // namespace uw12b
