// extern "C" boundary (include/uw12_c.h): argument checks that mirror
// libuw12's exceptions, status codes, per-thread error text and stream.
#include <atomic>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <exception>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>
#include <algorithm>

#include "../../include/uw12_c.h"
#include "engine.cuh"
#include "gemm_f64.cuh"
#include "kernels.cuh"
#include "ozaki.cuh"

namespace uw12b {

void synth_three_index_block(double* out, size_t ld, int kind, size_t n_ao, size_t n_ri,
                             size_t first, size_t count, unsigned long long seed,
                             unsigned long long tag, double decay, cudaStream_t stream);
void synth_three_index(double* out, int kind, size_t n_ao, size_t n_ri, size_t n_df,
                       unsigned long long seed, unsigned long long tag, double decay);

namespace {
std::atomic<unsigned long long> g_launches{0};
thread_local cudaStream_t g_stream = nullptr;
std::atomic<size_t> g_budget{0};
// Per-thread budget of the worker threads of a batched evaluation (0 = none).
thread_local size_t g_budget_override = 0;
thread_local size_t g_shard = 0, g_n_shards = 1;
thread_local uw12c_allreduce_fn g_allreduce = nullptr;
thread_local void* g_allreduce_user = nullptr;
thread_local int g_last_status = UW12C_OK;
thread_local std::string g_last_msg;
}  // namespace

void note_launch(const char* file, int line) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  const cudaError_t e = cudaPeekAtLastError();
  if (e != cudaSuccess) {
    cudaGetLastError();
    throw Error(kErrCuda, std::string("kernel launch failed: ") + cudaGetErrorString(e) + " (" +
                              file + ":" + std::to_string(line) + ")");
  }
}
unsigned long long launch_count() { return g_launches.load(); }
cudaStream_t current_stream() { return g_stream; }
void set_current_stream(cudaStream_t s) { g_stream = s; }

namespace {
std::mutex g_pool_mu;
cudaMemPool_t g_pools[64] = {};
}  // namespace

cudaMemPool_t library_pool() {
  int dev = 0;
  UW12_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) throw Error(kErrInvalid, "device index out of range");
  std::lock_guard<std::mutex> lk(g_pool_mu);
  if (!g_pools[dev]) {
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool = nullptr;
    UW12_CUDA(cudaMemPoolCreate(&pool, &props));
    unsigned long long thr = ~0ULL;
    UW12_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr));
    g_pools[dev] = pool;
  }
  return g_pools[dev];
}

void trim_pools() {
  std::lock_guard<std::mutex> lk(g_pool_mu);
  for (int d = 0; d < 64; ++d)
    if (g_pools[d]) UW12_CUDA(cudaMemPoolTrimTo(g_pools[d], 0));
}

}  // namespace uw12b

struct uw12c_integrals {
  std::unique_ptr<uw12b::IntegralsHandle> h;
};
struct uw12c_abs {
  std::unique_ptr<uw12b::AbsHandle> h;
};

namespace {

using uw12b::Error;

template <typename F>
int guarded(F&& f) {
  try {
    f();
    uw12b::g_last_status = UW12C_OK;
    uw12b::g_last_msg.clear();
    return UW12C_OK;
  } catch (const Error& e) {
    uw12b::g_last_status = e.code;
    uw12b::g_last_msg = e.what();
  } catch (const std::bad_alloc&) {
    uw12b::g_last_status = UW12C_ERR_ALLOC;
    uw12b::g_last_msg = "host allocation failed";
  } catch (const std::exception& e) {
    uw12b::g_last_status = UW12C_ERR_RUNTIME;
    uw12b::g_last_msg = e.what();
  } catch (...) {
    uw12b::g_last_status = UW12C_ERR_RUNTIME;
    uw12b::g_last_msg = "unknown error";
  }
  return uw12b::g_last_status;
}

void need(bool ok, const char* msg) {
  if (!ok) throw Error(UW12C_ERR_INVALID, msg);
}

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    UW12_CUDA(cudaGetDevice(&prev));
    if (prev != dev) UW12_CUDA(cudaSetDevice(dev));
  }
  ~DeviceGuard() {
    int cur = -1;
    if (cudaGetDevice(&cur) == cudaSuccess && cur != prev && prev >= 0) cudaSetDevice(prev);
  }
};

bool nearly_zero(double v) { return std::fabs(v) <= 4.0 * DBL_EPSILON; }  // utils.hpp:186-189

// A split-precision GEMM kernel whose pipeline wait timed out leaves a device
// flag; its results are not trusted.
void check_split_pipeline() {
  if (uw12b::split_moduli() > 0 && uw12b::ozaki_error_read_and_clear())
    throw uw12b::Error(uw12b::kErrCuda,
                       "split-precision GEMM: a tensor-core pipeline wait timed out");
}

void run_form_fock(const uw12c_integrals* W, const uw12c_integrals* V, const uw12c_integrals* WV,
                   const uw12c_abs* abs, size_t n_ao, size_t n_spin, const double* const* C,
                   const size_t* ldc, const size_t* n_orb, const double* const* occ,
                   const size_t* n_occ, const size_t* n_active, int indirect, int calc,
                   double s_os, double s_ss, size_t print_level, double* energy, double* terms,
                   double* fock, int fock_mem, const uw12b::AdjointOutputs* adjoint = nullptr) {
  need(W && V && WV && abs && W->h && V->h && WV->h && abs->h, "null handle");
  need(C && ldc && n_orb && occ && n_occ && n_active, "null orbital/occupation argument");
  need(fock_mem == UW12C_MEM_HOST || fock_mem == UW12C_MEM_DEVICE, "bad fock_mem_kind");
  // form_fock / spin_channels (uw12.cpp:40-50, utils.hpp:198-205)
  if (n_spin < 1 || n_spin > 2) uw12b::throw_logic("invalid number of spin channels");
  uw12b::FockRequest rq;
  rq.W = W->h.get();
  rq.V = V->h.get();
  rq.WV = WV->h.get();
  rq.abs = abs->h.get();
  rq.n_spin = static_cast<int>(n_spin);
  rq.n_ao = n_ao;
  for (size_t s = 0; s < n_spin; ++s) {
    // occupation_weighted_orbitals (utils.hpp:289-310), freeze_core (:235-253)
    for (size_t k = 0; k < n_occ[s]; ++k) {
      need(occ[s] != nullptr, "null occupation vector");
      if (!(occ[s][k] > 0.0)) uw12b::throw_runtime("occupations must be positive");
    }
    if (n_occ[s] > n_orb[s])
      uw12b::throw_logic("Cannot have submatix with more columns than parent matrix");
    if (n_active[s] > n_occ[s])
      uw12b::throw_logic("Cannot have submatix with more columns than parent matrix");
    if (n_occ[s]) need(C[s] != nullptr, "null orbital block");
    if (ldc[s] < n_ao) uw12b::throw_logic("orbital leading dimension smaller than n_ao");
    rq.C.push_back(C[s]);
    rq.ldc.push_back(ldc[s]);
    rq.n_orb.push_back(n_orb[s]);
    rq.occ.push_back(occ[s]);
    rq.n_occ.push_back(n_occ[s]);
    rq.n_active.push_back(n_active[s]);
  }
  const auto& w = *rq.W;
  const auto& v = *rq.V;
  const auto& wv = *rq.WV;
  // Integrals::number_ao_orbitals (integrals.cpp:394-402)
  if (w.n_ao != n_ao || v.n_ao != n_ao || wv.n_ao != n_ao)
    uw12b::throw_runtime("Inconsistent number of atomic orbitals");
  if (w.n_ri == 0 || v.n_ri == 0) uw12b::throw_runtime("J3_ri_0 not stored");
  // calculate_xab accumulates (M_W x M_V) components into an n_df(V)^2 matrix
  // (direct_utils.cpp:75-79, 107-111): libuw12 only supports equal df sizes.
  if (w.n_df != v.n_df) uw12b::throw_logic("addition: incompatible matrix dimensions");
  if (w.n_ri != v.n_ri || rq.abs->n_ri != w.n_ri || rq.abs->n_ao != n_ao)
    uw12b::throw_logic("ABS projectors and RI integrals are of incompatible sizes");
  if (w.device != v.device || w.device != wv.device || w.device != rq.abs->device)
    throw Error(UW12C_ERR_INVALID, "handles live on different devices");
  rq.indirect = indirect != 0;
  rq.calc_fock = calc != 0;
  rq.s_os = s_os;
  rq.s_ss = s_ss;
  rq.print_level = print_level;
  rq.energy = energy;
  rq.terms = terms;
  rq.fock = fock;
  rq.fock_device = fock_mem == UW12C_MEM_DEVICE;
  rq.mem_budget = uw12b::g_budget_override ? uw12b::g_budget_override : uw12b::g_budget.load();
  rq.shard = uw12b::g_shard;
  rq.n_shards = uw12b::g_n_shards;
  rq.allreduce = uw12b::g_allreduce;
  rq.allreduce_user = uw12b::g_allreduce_user;
  DeviceGuard dg(w.device);
  if (adjoint)
    uw12b::form_fock_adjoint(rq, *adjoint);
  else
    uw12b::form_fock(rq);
  check_split_pipeline();
}

void run_public(double* fock, const uw12c_integrals* W, const uw12c_integrals* V,
                const uw12c_integrals* WV, const uw12c_abs* abs, const double* C, size_t n_ao,
                size_t n_orb, size_t n_spin, const double* occ, size_t n_occ_alpha,
                size_t n_occ_beta, const size_t* n_active, double s_os, double s_ss,
                size_t print_level, double* energy, bool calc) {
  // setup_orbitals / setup_occupations (libuw12.cpp:58-112)
  if (n_spin != 1 && n_spin != 2) uw12b::throw_runtime("Number of spin channels must be 1 or 2");
  need(n_active != nullptr, "null n_active");
  const double* Cs[2] = {C, C ? C + n_ao * n_orb : nullptr};
  const size_t ldc[2] = {n_ao, n_ao};
  const size_t norb[2] = {n_orb, n_orb};
  const double* occs[2] = {occ, occ ? occ + n_occ_alpha : nullptr};
  const size_t nocc[2] = {n_occ_alpha, n_spin == 2 ? n_occ_beta : 0};
  const bool indirect = !nearly_zero(s_ss);  // libuw12.cpp:138
  run_form_fock(W, V, WV, abs, n_ao, n_spin, Cs, ldc, norb, occs, nocc, n_active,
                indirect ? 1 : 0, calc ? 1 : 0, s_os, s_ss, print_level, energy, nullptr,
                calc ? fock : nullptr, UW12C_MEM_HOST);
}

}  // namespace

extern "C" {

int uw12c_last_error(char* buf, size_t len) {
  if (buf && len) {
    std::strncpy(buf, uw12b::g_last_msg.c_str(), len - 1);
    buf[len - 1] = '\0';
  }
  return uw12b::g_last_status;
}

const char* uw12c_version(void) { return "uw12-b200 0.1 (sm_100a, fp64 dmma)"; }

int uw12c_integrals_create(const double* X3, const double* X2, const double* X3_ri, size_t n_ao,
                           size_t n_df, size_t n_ri, int mem_kind, uw12c_integrals** out) {
  return guarded([&] {
    need(out != nullptr, "null output handle");
    need(mem_kind == UW12C_MEM_HOST || mem_kind == UW12C_MEM_DEVICE, "bad mem_kind");
    *out = nullptr;
    auto h = std::make_unique<uw12c_integrals>();
    h->h.reset(uw12b::integrals_create(X3, X2, X3_ri, n_ao, n_df, n_ri,
                                       mem_kind == UW12C_MEM_DEVICE));
    *out = h.release();
  });
}

int uw12c_integrals_create_eigenbasis(const double* J3, const double* df_vals, size_t n_ao,
                                      size_t n_df, int mem_kind, uw12c_integrals** out) {
  return guarded([&] {
    need(out != nullptr, "null output handle");
    need(mem_kind == UW12C_MEM_HOST || mem_kind == UW12C_MEM_DEVICE, "bad mem_kind");
    *out = nullptr;
    auto h = std::make_unique<uw12c_integrals>();
    h->h.reset(uw12b::integrals_create_eigenbasis(J3, df_vals, n_ao, n_df,
                                                  mem_kind == UW12C_MEM_DEVICE));
    *out = h.release();
  });
}

int uw12c_integrals_destroy(uw12c_integrals* h) {
  return guarded([&] { delete h; });
}

int uw12c_integrals_dims(const uw12c_integrals* h, size_t* n_ao, size_t* n_df, size_t* n_ri) {
  return guarded([&] {
    need(h && h->h, "null handle");
    if (n_ao) *n_ao = h->h->n_ao;
    if (n_df) *n_df = h->h->n_df;
    if (n_ri) *n_ri = h->h->n_ri;
  });
}

int uw12c_integrals_df_vals(const uw12c_integrals* h, double* out) {
  return guarded([&] {
    need(h && h->h && out, "null argument");
    std::memcpy(out, h->h->lam_host.data(), h->h->lam_host.size() * sizeof(double));
  });
}

int uw12c_abs_create(const double* S, size_t n_ao, size_t n_ri, int mem_kind, uw12c_abs** out) {
  return guarded([&] {
    need(out != nullptr, "null output handle");
    need(mem_kind == UW12C_MEM_HOST || mem_kind == UW12C_MEM_DEVICE, "bad mem_kind");
    *out = nullptr;
    auto h = std::make_unique<uw12c_abs>();
    h->h.reset(uw12b::abs_create(S, n_ao, n_ri, mem_kind == UW12C_MEM_DEVICE));
    *out = h.release();
  });
}

int uw12c_abs_destroy(uw12c_abs* h) {
  return guarded([&] { delete h; });
}

int uw12c_abs_blocks(const uw12c_abs* h, double* ri_ri, double* ri_ao, double* ao_ri,
                     double* ao_ao) {
  return guarded([&] {
    need(h && h->h, "null handle");
    const size_t N = h->h->n_ao, R = h->h->n_ri, n = N + R;
    DeviceGuard dg(h->h->device);
    cudaStream_t s = uw12b::current_stream();
    auto block = [&](double* dst, size_t r0, size_t c0, size_t rows, size_t cols) {
      if (!dst || !rows || !cols) return;
      UW12_CUDA(cudaMemcpy2DAsync(dst, rows * sizeof(double), h->h->Sinv.get() + r0 + n * c0,
                                  n * sizeof(double), rows * sizeof(double), cols,
                                  cudaMemcpyDeviceToHost, s));
    };
    block(ri_ri, N, N, R, R);
    block(ri_ao, N, 0, R, N);
    block(ao_ri, 0, N, N, R);
    block(ao_ao, 0, 0, N, N);
    UW12_CUDA(cudaStreamSynchronize(s));
  });
}

int uw12c_form_fock(const uw12c_integrals* W, const uw12c_integrals* V,
                    const uw12c_integrals* WV, const uw12c_abs* abs, size_t n_ao, size_t n_spin,
                    const double* const* C, const size_t* ldc, const size_t* n_orb,
                    const double* const* occ, const size_t* n_occ, const size_t* n_active,
                    int indirect_term, int calculate_fock, double scale_opp_spin,
                    double scale_same_spin, size_t print_level, double* energy, double* terms,
                    double* fock, int fock_mem_kind) {
  return guarded([&] {
    run_form_fock(W, V, WV, abs, n_ao, n_spin, C, ldc, n_orb, occ, n_occ, n_active, indirect_term,
                  calculate_fock, scale_opp_spin, scale_same_spin, print_level, energy, terms,
                  fock, fock_mem_kind);
  });
}

int uw12c_fock(double* fock, const uw12c_integrals* W, const uw12c_integrals* V,
               const uw12c_integrals* WV, const uw12c_abs* abs, const double* C, size_t n_ao,
               size_t n_orb, size_t n_spin, const double* occ, size_t n_occ_alpha,
               size_t n_occ_beta, const size_t* n_active, double scale_opp_spin,
               double scale_same_spin, size_t print_level, double* energy) {
  return guarded([&] {
    need(fock != nullptr, "null fock buffer");
    run_public(fock, W, V, WV, abs, C, n_ao, n_orb, n_spin, occ, n_occ_alpha, n_occ_beta,
               n_active, scale_opp_spin, scale_same_spin, print_level, energy, true);
  });
}

int uw12c_energy(const uw12c_integrals* W, const uw12c_integrals* V, const uw12c_integrals* WV,
                 const uw12c_abs* abs, const double* C, size_t n_ao, size_t n_orb, size_t n_spin,
                 const double* occ, size_t n_occ_alpha, size_t n_occ_beta,
                 const size_t* n_active, double scale_opp_spin, double scale_same_spin,
                 size_t print_level, double* energy) {
  return guarded([&] {
    run_public(nullptr, W, V, WV, abs, C, n_ao, n_orb, n_spin, occ, n_occ_alpha, n_occ_beta,
               n_active, scale_opp_spin, scale_same_spin, print_level, energy, false);
  });
}

int uw12c_set_stream(void* stream) {
  return guarded([&] { uw12b::set_current_stream(static_cast<cudaStream_t>(stream)); });
}

int uw12c_set_shard(size_t shard, size_t n_shards) {
  return guarded([&] {
    need(n_shards >= 1 && shard < n_shards, "shard must be < n_shards, n_shards >= 1");
    uw12b::g_shard = shard;
    uw12b::g_n_shards = n_shards;
  });
}

int uw12c_set_allreduce(uw12c_allreduce_fn fn, void* user) {
  return guarded([&] {
    uw12b::g_allreduce = fn;
    uw12b::g_allreduce_user = fn ? user : nullptr;
  });
}

int uw12c_trim_memory(void) {
  return guarded([&] { uw12b::trim_pools(); });
}

int uw12c_set_memory_budget(size_t bytes) {
  return guarded([&] { uw12b::g_budget.store(bytes); });
}

unsigned long long uw12c_launch_count(void) { return uw12b::launch_count(); }

int uw12c_profile_enable(int on) {
  return guarded([&] {
    if (on) uw12b::profile_reset();
    uw12b::profile_enable(on != 0);
  });
}

int uw12c_profile_read(unsigned long long* gemm_launches, double* gemm_ms, double* gemm_flops) {
  return guarded([&] {
    const uw12b::KernelStats k = uw12b::profile_read_gemm();
    if (gemm_launches) *gemm_launches = k.launches;
    if (gemm_ms) *gemm_ms = k.ms;
    if (gemm_flops) *gemm_flops = k.flops;
  });
}

int uw12c_profile_phases(char* buf, size_t len) {
  return guarded([&] {
    need(buf != nullptr && len > 0, "null buffer");
    const std::string s = uw12b::phase_profile_read();
    std::strncpy(buf, s.c_str(), len - 1);
    buf[len - 1] = '\0';
  });
}

int uw12c_dgemm(long long m, long long n, long long k, double alpha, const double* A,
                long long lda, int a_kcontig, const double* B, long long ldb, int b_ncontig,
                double beta, double* C, long long ldc, long long nbo1, long long nbo2,
                const long long* so, long long nbr1, long long nbr2, const long long* sr,
                int split) {
  return guarded([&] {
    uw12b::GemmDesc d;
    d.m = m; d.n = n; d.k = k; d.alpha = alpha; d.beta = beta;
    d.A = A; d.lda = lda; d.a_kcontig = a_kcontig != 0;
    d.B = B; d.ldb = ldb; d.b_ncontig = b_ncontig != 0;
    d.C = C; d.ldc = ldc;
    d.nbo1 = nbo1; d.nbo2 = nbo2;
    if (so) { d.sAo1 = so[0]; d.sAo2 = so[1]; d.sBo1 = so[2]; d.sBo2 = so[3]; d.sCo1 = so[4]; d.sCo2 = so[5]; }
    d.nbr1 = nbr1; d.nbr2 = nbr2;
    if (sr) { d.sAr1 = sr[0]; d.sAr2 = sr[1]; d.sBr1 = sr[2]; d.sBr2 = sr[3]; }
    d.split = split;
    need(m >= 0 && n >= 0 && k >= 0 && nbo1 >= 0 && nbo2 >= 0 && nbr1 >= 0 && nbr2 >= 0,
         "negative size");
    uw12b::gemm(d);
  });
}

int uw12c_fock_backward(const uw12c_integrals* W, const uw12c_integrals* V,
                        const uw12c_integrals* WV, const uw12c_abs* abs, size_t n_ao,
                        size_t n_spin, const double* const* C, const size_t* ldc,
                        const size_t* n_orb, const double* const* occ, const size_t* n_occ,
                        const size_t* n_active, int indirect_term, double scale_opp_spin,
                        double scale_same_spin, double* energy, double* terms, double* fock,
                        int fock_mem_kind, double* const* dE_dX3, double* const* dE_dX3_ri,
                        double* const* dE_dX2, int grad_mem_kind) {
  return guarded([&] {
    need(grad_mem_kind == UW12C_MEM_HOST || grad_mem_kind == UW12C_MEM_DEVICE,
         "bad grad_mem_kind");
    need(uw12b::g_n_shards == 1, "the adjoint evaluates unsharded (uw12c_set_shard(0, 1))");
    uw12b::AdjointOutputs ad;
    for (int i = 0; i < 3; ++i) {
      ad.dJ3[i] = dE_dX3 ? dE_dX3[i] : nullptr;
      ad.dJ2[i] = dE_dX2 ? dE_dX2[i] : nullptr;
    }
    for (int i = 0; i < 2; ++i) ad.dJ3_ri[i] = dE_dX3_ri ? dE_dX3_ri[i] : nullptr;
    ad.device_mem = grad_mem_kind == UW12C_MEM_DEVICE;
    run_form_fock(W, V, WV, abs, n_ao, n_spin, C, ldc, n_orb, occ, n_occ, n_active,
                  indirect_term, fock != nullptr, scale_opp_spin, scale_same_spin, 0, energy,
                  terms, fock, fock_mem_kind, &ad);
  });
}

namespace {

// A user gradient sink as an engine sink: device blocks are passed on; host
// blocks are copied through a pinned stage (at most 256 MiB at a time, so one
// engine block may reach the user as several).
uw12b::GradSink wrap_sink(uw12c_block_sink fn, void* user, bool host, size_t rows) {
  if (!fn) return {};
  struct Stage {
    double* p = nullptr;
    size_t n = 0;
    ~Stage() {
      if (p) cudaFreeHost(p);
    }
  };
  auto stage = std::make_shared<Stage>();
  return [fn, user, host, rows, stage](size_t first, size_t count, const double* block,
                                       size_t ld, cudaStream_t s) {
    auto check = [](int rc) {
      if (rc != 0)
        throw uw12b::Error(UW12C_ERR_RUNTIME,
                           "gradient block sink returned " + std::to_string(rc));
    };
    if (!host) {
      check(fn(user, first, count, block, ld, static_cast<void*>(s)));
      return;
    }
    const size_t per = std::max<size_t>(1, std::min(count, (size_t(1) << 25) / rows));
    if (stage->n < rows * per) {
      if (stage->p) cudaFreeHost(stage->p);
      stage->p = nullptr;
      stage->n = 0;
      UW12_CUDA(cudaMallocHost(reinterpret_cast<void**>(&stage->p), rows * per * sizeof(double)));
      stage->n = rows * per;
    }
    for (size_t c0 = 0; c0 < count; c0 += per) {
      const size_t nc = std::min(per, count - c0);
      UW12_CUDA(cudaMemcpy2DAsync(stage->p, rows * sizeof(double), block + ld * c0,
                                  ld * sizeof(double), rows * sizeof(double), nc,
                                  cudaMemcpyDeviceToHost, s));
      UW12_CUDA(cudaStreamSynchronize(s));
      check(fn(user, first + c0, nc, stage->p, rows, static_cast<void*>(s)));
    }
  };
}

}  // namespace

int uw12c_fock_backward_blocks(const uw12c_integrals* W, const uw12c_integrals* V,
                               const uw12c_integrals* WV, const uw12c_abs* abs, size_t n_ao,
                               size_t n_spin, const double* const* C, const size_t* ldc,
                               const size_t* n_orb, const double* const* occ,
                               const size_t* n_occ, const size_t* n_active,
                               int indirect_term, double scale_opp_spin,
                               double scale_same_spin, double* energy, double* terms,
                               double* fock, int fock_mem_kind,
                               const uw12c_block_sink* sink3, void* const* user3,
                               const uw12c_block_sink* sink3_ri, void* const* user3_ri,
                               int block_mem_kind, double* const* dE_dX2, int grad_mem_kind) {
  return guarded([&] {
    need(grad_mem_kind == UW12C_MEM_HOST || grad_mem_kind == UW12C_MEM_DEVICE,
         "bad grad_mem_kind");
    need(block_mem_kind == UW12C_MEM_HOST || block_mem_kind == UW12C_MEM_DEVICE,
         "bad block_mem_kind");
    need(W && V && WV, "null integral handle");
    need(uw12b::g_n_shards == 1, "the adjoint evaluates unsharded (uw12c_set_shard(0, 1))");
    const bool host = block_mem_kind == UW12C_MEM_HOST;
    const uw12c_integrals* X[3] = {W, V, WV};
    uw12b::AdjointOutputs ad;
    for (int i = 0; i < 3; ++i) {
      ad.dJ2[i] = dE_dX2 ? dE_dX2[i] : nullptr;
      const size_t na = X[i]->h->n_ao;
      if (sink3 && sink3[i])
        ad.sink3[i] = wrap_sink(sink3[i], user3 ? user3[i] : nullptr, host, na * (na + 1) / 2);
    }
    for (int i = 0; i < 2; ++i)
      if (sink3_ri && sink3_ri[i])
        ad.sink3_ri[i] = wrap_sink(sink3_ri[i], user3_ri ? user3_ri[i] : nullptr, host,
                                   X[i]->h->n_ri * X[i]->h->n_ao);
    ad.device_mem = grad_mem_kind == UW12C_MEM_DEVICE;
    run_form_fock(W, V, WV, abs, n_ao, n_spin, C, ldc, n_orb, occ, n_occ, n_active,
                  indirect_term, fock != nullptr, scale_opp_spin, scale_same_spin, 0, energy,
                  terms, fock, fock_mem_kind, &ad);
  });
}

int uw12c_sink_norm2(void* user, size_t first, size_t count, const double* block, size_t ld,
                     void* stream) {
  (void)first;
  if (!user || !block) return 1;
  try {
    uw12b::sumsq_add(block, static_cast<long long>(ld), static_cast<long long>(ld),
                     static_cast<long long>(count), static_cast<double*>(user),
                     static_cast<cudaStream_t>(stream));
  } catch (...) {
    return 2;
  }
  return 0;
}

namespace {

// A user's uw12c_block_fn as an engine producer.  Host producers write into a
// pinned staging buffer (at most kStageDoubles doubles per call; the requested
// block is split into column groups) that is copied to the device; the buffer
// is reused under a mutex, so producers may be called from several host
// threads (batched evaluations) one at a time per tensor.
// A user producer.  Device producers are called directly.  Host producers
// write into pinned stages that are copied to the device on the caller's
// stream; two stages and a read-ahead thread overlap the user's function
// with the GPU: after block [first, first + count) is staged, the next
// range (the same count after it, or from 0 again at the end of the aux
// range, where loops restart) is produced in the background into the other
// stage, and a request for exactly that range takes it from there.  A stage
// is rewritten only after its last copy has completed (an event per stage);
// the caller's stream is not synchronised.
struct UserProducer {
  static constexpr size_t kStageDoubles = size_t(1) << 25;  // 256 MiB per stage
  uw12c_block_fn fn = nullptr;
  void* user = nullptr;
  bool host = false;
  size_t rows = 0, n_df = 0;
  std::mutex mu;  // one request at a time (handles may be shared by host threads)
  struct Stage {
    double* p = nullptr;
    size_t n = 0;
    cudaEvent_t copied = nullptr;  // last copy out of this stage
  } stage[2];
  // read-ahead job: range, stage, and its completion / failure
  std::thread ahead;
  bool ahead_on = false;
  size_t ahead_first = 0, ahead_count = 0;
  int ahead_stage = 0;
  int ahead_rc = 0;
  std::exception_ptr ahead_err;

  ~UserProducer() {
    if (ahead.joinable()) ahead.join();
    for (auto& st : stage) {
      if (st.copied) cudaEventDestroy(st.copied);
      if (st.p) cudaFreeHost(st.p);
    }
  }

  void check(int rc) const {
    if (rc != 0)
      throw uw12b::Error(UW12C_ERR_RUNTIME,
                         "three-index integral callback returned " + std::to_string(rc));
  }

  void ensure(Stage& st, size_t n) {
    if (!st.copied) UW12_CUDA(cudaEventCreateWithFlags(&st.copied, cudaEventDisableTiming));
    if (st.n >= n) return;
    UW12_CUDA(cudaEventSynchronize(st.copied));
    if (st.p) cudaFreeHost(st.p);
    st.p = nullptr;
    st.n = 0;
    UW12_CUDA(cudaMallocHost(reinterpret_cast<void**>(&st.p), n * sizeof(double)));
    st.n = n;
  }

  // Waits for the read-ahead job; true when it produced [first, first + count).
  bool take_ahead(size_t first, size_t count, int* which) {
    if (!ahead_on) return false;
    ahead.join();
    ahead_on = false;
    if (ahead_err) {
      auto e = ahead_err;
      ahead_err = nullptr;
      if (ahead_first == first && ahead_count == count) std::rethrow_exception(e);
      return false;
    }
    if (ahead_first != first || ahead_count != count) return false;
    check(ahead_rc);
    *which = ahead_stage;
    return true;
  }

  void operator()(size_t first, size_t count, double* out, size_t ld, cudaStream_t s) {
    if (!host) {
      check(fn(user, first, count, out, ld, static_cast<void*>(s)));
      return;
    }
    std::lock_guard<std::mutex> lk(mu);
    const size_t per = std::max<size_t>(1, std::min(count, kStageDoubles / rows));
    int which = 0;
    if (take_ahead(first, count, &which)) {  // (always joins a pending read-ahead)
      stage_out(which, count, out, ld, s);
    } else {
      // produced here, one stage-sized piece at a time
      for (size_t c0 = 0; c0 < count; c0 += per) {
        const size_t nc = std::min(per, count - c0);
        which = 1 - which;
        Stage& st = stage[which];
        ensure(st, rows * per);
        UW12_CUDA(cudaEventSynchronize(st.copied));  // its previous copy is done
        check(fn(user, first + c0, nc, st.p, rows, static_cast<void*>(s)));
        stage_out(which, nc, out + ld * c0, ld, s);
      }
      if (count > per) return;  // no read-ahead for blocks larger than a stage
    }
    // read ahead the next range into the other stage
    size_t nf = first + count, nc = count;
    if (nf >= n_df) nf = 0;
    nc = std::min(nc, n_df - nf);
    if (nc == 0) return;
    const int other = 1 - which;
    ensure(stage[other], rows * per);
    ahead_first = nf;
    ahead_count = nc;
    ahead_stage = other;
    ahead_rc = 0;
    ahead_err = nullptr;
    ahead_on = true;
    ahead = std::thread([this, nf, nc, other, s] {
      try {
        UW12_CUDA(cudaEventSynchronize(stage[other].copied));
        ahead_rc = fn(user, nf, nc, stage[other].p, rows, static_cast<void*>(s));
      } catch (...) {
        ahead_err = std::current_exception();
      }
    });
  }

  void stage_out(int which, size_t nc, double* out, size_t ld, cudaStream_t s) {
    Stage& st = stage[which];
    UW12_CUDA(cudaMemcpy2DAsync(out, ld * sizeof(double), st.p, rows * sizeof(double),
                                rows * sizeof(double), nc, cudaMemcpyHostToDevice, s));
    UW12_CUDA(cudaEventRecord(st.copied, s));
  }
};

uw12b::AuxProducer wrap_producer(uw12c_block_fn fn, void* user, bool host, size_t rows,
                                 size_t n_df) {
  if (!fn) return {};
  auto p = std::make_shared<UserProducer>();
  p->fn = fn;
  p->user = user;
  p->host = host;
  p->rows = rows;
  p->n_df = n_df;
  return [p](size_t f, size_t c, double* o, size_t l, cudaStream_t s) { (*p)(f, c, o, l, s); };
}

}  // namespace

int uw12c_integrals_create_callback(const double* X2, int x2_mem_kind,
                                    uw12c_block_fn three_index, void* user,
                                    uw12c_block_fn three_index_ri, void* user_ri, size_t n_ao,
                                    size_t n_df, size_t n_ri, int store_ao, int store_ri,
                                    int block_mem_kind, uw12c_integrals** out) {
  return guarded([&] {
    need(out != nullptr, "null output handle");
    need(x2_mem_kind == UW12C_MEM_HOST || x2_mem_kind == UW12C_MEM_DEVICE, "bad x2_mem_kind");
    need(block_mem_kind == UW12C_MEM_HOST || block_mem_kind == UW12C_MEM_DEVICE,
         "bad block_mem_kind");
    need(three_index != nullptr, "null three-index callback");
    *out = nullptr;
    const bool host = block_mem_kind == UW12C_MEM_HOST;
    auto ao = wrap_producer(three_index, user, host, n_ao * (n_ao + 1) / 2, n_df);
    auto ri = wrap_producer(three_index_ri, user_ri, host, n_ri * n_ao, n_df);
    auto h = std::make_unique<uw12c_integrals>();
    h->h.reset(uw12b::integrals_create_producer(X2, x2_mem_kind == UW12C_MEM_DEVICE,
                                                std::move(ao), std::move(ri), n_ao,
                                                n_df, n_ri, store_ao != 0, store_ri != 0));
    *out = h.release();
  });
}

int uw12c_synth_block(void* spec, size_t first, size_t count, double* out, size_t ld,
                      void* stream) {
  if (!spec) return 1;
  const auto* sp = static_cast<const uw12c_synth_spec*>(spec);
  try {
    uw12b::synth_three_index_block(out, ld, sp->kind, sp->n_ao, sp->n_ri, first, count, sp->seed,
                                   sp->tag, sp->decay, static_cast<cudaStream_t>(stream));
  } catch (...) {
    return 2;
  }
  return 0;
}

int uw12c_fock_batched(const uw12c_molecule* mols, size_t n, int indirect_term,
                       int calculate_fock, double scale_opp_spin, double scale_same_spin,
                       size_t n_streams, int* statuses) {
  return guarded([&] {
    need(mols != nullptr || n == 0, "null molecule array");
    if (n == 0) return;
    // at most kOzakiErrorSlots workers: each owns one split-precision error flag
    const size_t workers = std::min({n, n_streams ? n_streams : size_t(8),
                                     static_cast<size_t>(uw12b::kOzakiErrorSlots)});
    // largest molecules first, so that the tail of the batch is short
    std::vector<size_t> order(n);
    for (size_t i = 0; i < n; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(),
                     [&](size_t a, size_t b) { return mols[a].n_ao > mols[b].n_ao; });
    // the caller's per-thread settings apply to every worker; concurrent
    // evaluations share the memory budget (the explicit one, or 45% of the
    // free device memory now)
    const int moduli = uw12b::split_moduli();
    const double min_flops = uw12b::split_min_flops();
    size_t total_budget = uw12b::g_budget.load();
    if (!total_budget) {
      size_t free_b = 0, total_b = 0;
      UW12_CUDA(cudaMemGetInfo(&free_b, &total_b));
      total_budget = static_cast<size_t>(0.45 * double(free_b));
    }
    const size_t worker_budget = std::max<size_t>(total_budget / workers, size_t(64) << 20);
    std::atomic<size_t> next{0};
    std::vector<int> st(n, UW12C_OK);
    std::vector<std::string> msg(n);
    auto work = [&](int slot) {
      const int prev_slot = uw12b::set_error_slot(slot);
      cudaStream_t stream = nullptr;
      int dev = -1;
      uw12b::set_split_moduli(moduli);
      uw12b::set_split_min_flops(min_flops);
      uw12b::g_budget_override = worker_budget;
      for (size_t q; (q = next.fetch_add(1)) < n;) {
        const size_t i = order[q];
        const uw12c_molecule& m = mols[i];
        st[i] = guarded([&] {
          need(m.W && m.W->h, "null handle");
          if (m.W->h->device != dev) {
            if (stream) cudaStreamDestroy(stream);
            dev = m.W->h->device;
            UW12_CUDA(cudaSetDevice(dev));
            UW12_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
            uw12b::g_stream = stream;
          }
          run_form_fock(m.W, m.V, m.WV, m.abs, m.n_ao, m.n_spin, m.C, m.ldc, m.n_orb, m.occ,
                        m.n_occ, m.n_active, indirect_term, calculate_fock, scale_opp_spin,
                        scale_same_spin, 0, m.energy, m.terms, m.fock, m.fock_mem_kind);
        });
        if (st[i] != UW12C_OK) msg[i] = uw12b::g_last_msg;
      }
      if (stream) {
        cudaStreamSynchronize(stream);
        cudaStreamDestroy(stream);
      }
      uw12b::g_stream = nullptr;
      uw12b::g_budget_override = 0;
      uw12b::set_error_slot(prev_slot);
    };
    std::vector<std::thread> pool;
    for (size_t w = 1; w < workers; ++w) pool.emplace_back(work, static_cast<int>(w));
    {
      // the calling thread works too; its stream and device are restored afterwards
      const cudaStream_t saved = uw12b::g_stream;
      int saved_dev = 0;
      cudaGetDevice(&saved_dev);
      work(0);
      uw12b::g_stream = saved;
      cudaSetDevice(saved_dev);
    }
    for (auto& t : pool) t.join();
    if (statuses)
      for (size_t i = 0; i < n; ++i) statuses[i] = st[i];
    for (size_t i = 0; i < n; ++i)
      if (st[i] != UW12C_OK)
        throw Error(st[i], "molecule " + std::to_string(i) + ": " + msg[i]);
  });
}

int uw12c_set_precision(int n_moduli) {
  return guarded([&] { uw12b::set_split_moduli(n_moduli); });
}

int uw12c_dgemm_split(long long m, long long n, long long k, double alpha, const double* A,
                      long long lda, int a_kcontig, const double* B, long long ldb, int b_ncontig,
                      double beta, double* C, long long ldc, long long nbo1, long long nbo2,
                      const long long* so, long long nbr1, long long nbr2, const long long* sr,
                      int n_moduli) {
  return guarded([&] {
    uw12b::GemmDesc d;
    d.m = m; d.n = n; d.k = k; d.alpha = alpha; d.beta = beta;
    d.A = A; d.lda = lda; d.a_kcontig = a_kcontig != 0;
    d.B = B; d.ldb = ldb; d.b_ncontig = b_ncontig != 0;
    d.C = C; d.ldc = ldc;
    d.nbo1 = nbo1; d.nbo2 = nbo2;
    if (so) { d.sAo1 = so[0]; d.sAo2 = so[1]; d.sBo1 = so[2]; d.sBo2 = so[3]; d.sCo1 = so[4]; d.sCo2 = so[5]; }
    d.nbr1 = nbr1; d.nbr2 = nbr2;
    if (sr) { d.sAr1 = sr[0]; d.sAr2 = sr[1]; d.sBr1 = sr[2]; d.sBr2 = sr[3]; }
    need(m >= 0 && n >= 0 && k >= 0 && nbo1 >= 0 && nbo2 >= 0 && nbr1 >= 0 && nbr2 >= 0,
         "negative size");
    need(n_moduli >= 1 && n_moduli <= uw12b::kOzakiMaxModuli, "n_moduli must be 1..16");
    need(uw12b::ozaki_supported(d), "shape too large for the split-precision GEMM");
    uw12b::gemm_ozaki(d, n_moduli);
    if (uw12b::ozaki_error_read_and_clear())
      throw uw12b::Error(uw12b::kErrCuda,
                         "split-precision GEMM: a tensor-core pipeline wait timed out");
  });
}

int uw12c_set_split_threshold(double min_flops) {
  return guarded([&] { uw12b::set_split_min_flops(min_flops); });
}

int uw12c_split_bits(int n_moduli, long long k_total, int* bits) {
  return guarded([&] {
    need(n_moduli >= 1 && n_moduli <= uw12b::kOzakiMaxModuli && k_total >= 1 && bits,
         "n_moduli must be 1..16, k_total >= 1");
    *bits = uw12b::ozaki_bits(n_moduli, k_total);
  });
}

int uw12c_profile_read_kind(int kind, unsigned long long* launches, double* ms, double* work) {
  return guarded([&] {
    need(kind >= 0 && kind < uw12b::kProfKinds, "unknown kernel class");
    const uw12b::KernelStats k = uw12b::profile_read_kind(kind);
    if (launches) *launches = k.launches;
    if (ms) *ms = k.ms;
    if (work) *work = k.flops;
  });
}

int uw12c_autotune(int mode, const char* path) {
  return guarded([&] { uw12b::autotune_set(mode, path); });
}

int uw12c_autotune_save(const char* path) {
  return guarded([&] { uw12b::autotune_save(path); });
}

int uw12c_autotune_clear(void) {
  return guarded([&] { uw12b::autotune_clear(); });
}

int uw12c_autotune_size(long long* n_classes) {
  return guarded([&] {
    need(n_classes != nullptr, "null output");
    *n_classes = uw12b::autotune_size();
  });
}

int uw12c_autotune_lookup(long long m, long long n, long long k, long long nbo, long long nbr,
                          int* split) {
  return guarded([&] {
    need(split != nullptr, "null output");
    *split = uw12b::autotune_lookup(m, n, k, nbo, nbr);
  });
}

int uw12c_dgemm_noalloc(long long m, long long n, long long k, double alpha, const double* A,
                        long long lda, int a_kcontig, const double* B, long long ldb,
                        int b_ncontig, double beta, double* C, long long ldc, long long nbo1,
                        long long nbo2, const long long* so, long long nbr1, long long nbr2,
                        const long long* sr, int split) {
  static_assert(UW12C_NOALLOC_SCRATCH_DOUBLES == uw12b::kNoAllocScratchDoubles,
                "scratch size of the header and the library differ");
  return guarded([&] {
    uw12b::GemmDesc d;
    d.m = m; d.n = n; d.k = k; d.alpha = alpha; d.beta = beta;
    d.A = A; d.lda = lda; d.a_kcontig = a_kcontig != 0;
    d.B = B; d.ldb = ldb; d.b_ncontig = b_ncontig != 0;
    d.C = C; d.ldc = ldc;
    d.nbo1 = nbo1; d.nbo2 = nbo2;
    if (so) { d.sAo1 = so[0]; d.sAo2 = so[1]; d.sBo1 = so[2]; d.sBo2 = so[3]; d.sCo1 = so[4]; d.sCo2 = so[5]; }
    d.nbr1 = nbr1; d.nbr2 = nbr2;
    if (sr) { d.sAr1 = sr[0]; d.sAr2 = sr[1]; d.sBr1 = sr[2]; d.sBr2 = sr[3]; }
    d.split = split;
    need(m >= 0 && n >= 0 && k >= 0 && nbo1 >= 0 && nbo2 >= 0 && nbr1 >= 0 && nbr2 >= 0 &&
             split >= 0,
         "negative size");
    uw12b::gemm_noalloc(d);
  });
}

int uw12c_synth_three_index(double* out_device, int kind, size_t n_ao, size_t n_ri, size_t n_df,
                            unsigned long long seed, unsigned long long tag, double decay) {
  return guarded([&] {
    need(out_device != nullptr, "null output");
    uw12b::synth_three_index(out_device, kind, n_ao, n_ri, n_df, seed, tag, decay);
  });
}

}  // extern "C"
