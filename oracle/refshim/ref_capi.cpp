// C-ABI over the compiled libuw12 reference -- TEST INFRASTRUCTURE ONLY.
//
// Built by oracle/ref.mk together with libuw12's unmodified sources into
// oracle/_ref/libuw12_ref.so. Only the tests, the golden-fixture script and
// the CPU-baseline legs of bench.py load it, as the checker; the CUDA library
// never does.
//
// Every entry point calls libuw12's own functions:
//   * uw12ref_create        -> uw12::setup_base_integrals (libuw12.cpp:22-49),
//                              uw12::setup_abs_projectors (libuw12.cpp:51-56)
//   * uw12ref_evaluate      -> uw12::uw12_fock / uw12::uw12_energy
//                              (libuw12.cpp:156-214), or, when per-term energies
//                              are requested, the same sequence of term calls
//                              as uw12::form_fock (src/uw12.cpp:22-119)
//   * uw12ref_abs_blocks    -> three_el::ri::calculate_abs_projectors
//                              (src/three_electron/ri_utils.hpp:45-74)
//   * uw12ref_timing_*      (timing build only) the loop dispatcher's mode and
//                              the extrapolated time of skipped iterations
// Errors: status 1 = std::runtime_error, 2 = std::logic_error, 3 = other; the
// message is kept per thread for uw12ref_last_error.
#include <omp.h>

#include <chrono>
#include <cstddef>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "four_electron/four_electron.hpp"
#include "utils/parallel.hpp"
#include "integrals/base_integrals.hpp"
#include "integrals/integrals.hpp"
#include "libuw12.hpp"
#include "three_electron/ri_utils.hpp"
#include "three_electron/three_electron.hpp"
#include "two_electron/two_electron.hpp"
#include "utils/utils.hpp"
#include "uw12.hpp"

extern "C" void UW12REF_SYM(openblas_set_num_threads)(int);

namespace {
thread_local std::string g_error;

template <typename F>
int guarded(F&& f) {
  try {
    f();
    return 0;
  } catch (const std::runtime_error& e) {
    g_error = e.what();
    return 1;
  } catch (const std::logic_error& e) {
    g_error = e.what();
    return 2;
  } catch (const std::exception& e) {
    g_error = e.what();
    return 3;
  } catch (...) {
    g_error = "unknown exception";
    return 3;
  }
}

double seconds_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0)
      .count();
}
}  // namespace

struct uw12ref_problem {
  uw12::BaseIntegrals W, V, WV;
  uw12::ABSProjectors abs;
  size_t n_ao;
};

extern "C" {

int uw12ref_last_error(char* buf, size_t n) {
  if (buf && n) {
    std::strncpy(buf, g_error.c_str(), n - 1);
    buf[n - 1] = 0;
  }
  return (int)g_error.size();
}

// OpenMP threads for the reference's parallel loops and BLAS threads inside
// them (the reference calls BLAS inside its OpenMP loops, so 1 is the usual
// setting).
void uw12ref_set_threads(int omp_threads, int blas_threads) {
  if (omp_threads > 0) omp_set_num_threads(omp_threads);
  if (blas_threads > 0) UW12REF_SYM(openblas_set_num_threads)(blas_threads);
}

int uw12ref_max_threads(void) { return omp_get_max_threads(); }

// Builds W, V (with RI tensors), WV (no RI tensor) and the ABS projectors.
// The integrals are deep-copied by BaseIntegrals, so the caller's buffers may
// be released afterwards. setup_seconds (nullable) receives the wall time.
int uw12ref_create(const double* W3, const double* W2, const double* W3_ri,
                   const double* V3, const double* V2, const double* V3_ri,
                   const double* WV3, const double* WV2, const double* S,
                   size_t n_ao, size_t n_df, size_t n_ri,
                   uw12ref_problem** out, double* setup_seconds) {
  *out = nullptr;
  return guarded([&] {
    const auto t0 = std::chrono::steady_clock::now();
    auto W = uw12::setup_base_integrals(W3, W2, W3_ri, n_ao, n_df, n_ri);
    auto V = uw12::setup_base_integrals(V3, V2, V3_ri, n_ao, n_df, n_ri);
    auto WV = uw12::setup_base_integrals(WV3, WV2, n_ao, n_df);
    auto abs = uw12::setup_abs_projectors(S, n_ao, n_ri);
    // The metric eigendecompositions are lazy in libuw12; force them here so
    // that the timed evaluation excludes setup, as the GPU path does.
    W.get_P2();
    V.get_P2();
    WV.get_P2();
    *out = new uw12ref_problem{std::move(W), std::move(V), std::move(WV),
                               std::move(abs), n_ao};
    if (setup_seconds) *setup_seconds = seconds_since(t0);
  });
}

void uw12ref_destroy(uw12ref_problem* p) { delete p; }

// One energy (+ Fock) evaluation. C is n_ao x (n_orb * n_spin), alpha then
// beta; occ holds n_occ[0] (+ n_occ[1]) occupations; n_active holds
// n_active_len counts (one per spin channel for a valid call).
// fock (nullable => energy only) receives n_ao x (n_ao * n_spin).
// terms (nullable): when given, the evaluation runs uw12::form_fock's own
// sequence of term calls and writes the two-, three- and four-electron
// energies; otherwise it calls the public uw12_fock / uw12_energy.
int uw12ref_evaluate(uw12ref_problem* p, const double* C, size_t n_orb,
                     size_t n_spin, const double* occ, const size_t* n_occ,
                     const size_t* n_active, size_t n_active_len,
                     double s_os, double s_ss, double* fock, double* energy,
                     double* terms, double* seconds) {
  return guarded([&] {
    const auto t0 = std::chrono::steady_clock::now();
    const auto orbitals = uw12::setup_orbitals(C, p->n_ao, n_orb, n_spin);
    const auto occs =
        n_spin == 1 ? uw12::setup_occupations(occ, n_occ[0])
                    : uw12::setup_occupations(occ, n_occ[0], n_occ[1]);
    const std::vector<size_t> act(n_active, n_active + n_active_len);
    if (terms == nullptr) {
      if (fock) {
        *energy = uw12::uw12_fock(fock, p->W, p->V, p->WV, p->abs, orbitals,
                                  occs, act, s_os, s_ss);
      } else {
        *energy = uw12::uw12_energy(p->W, p->V, p->WV, p->abs, orbitals, occs,
                                    act, s_os, s_ss);
      }
    } else {
      // The calls of uw12::form_fock (src/uw12.cpp:22-119), kept apart so
      // that each term's energy can be returned.
      const bool indirect = !uw12::utils::nearly_zero(s_ss);
      const bool calc_fock = fock != nullptr;
      if (uw12::utils::spin_channels(occs) != n_spin ||
          uw12::utils::spin_channels(act) != n_spin)
        throw std::runtime_error("Different number of spin channels");
      const auto Co = uw12::utils::occupation_weighted_orbitals(orbitals, occs);
      const auto active_Co = uw12::utils::freeze_core(Co, act);
      const auto f2 = uw12::two_el::form_fock_two_el_df(
          p->WV, active_Co, indirect, calc_fock, s_os, s_ss);
      const auto W_ints = uw12::integrals::Integrals(p->W, Co, active_Co);
      const auto V_ints = uw12::integrals::Integrals(p->V, Co, active_Co);
      const auto f3 = uw12::three_el::form_fock_three_el_term_df_ri(
          W_ints, V_ints, p->abs, indirect, calc_fock, s_os, s_ss);
      const auto f4 = uw12::four_el::form_fock_four_el_df(
          W_ints, V_ints, indirect, calc_fock, s_os, s_ss);
      const auto total = f2 + f3 + f4;
      terms[0] = f2.energy;
      terms[1] = f3.energy;
      terms[2] = f4.energy;
      *energy = total.energy;
      if (fock) {
        const size_t n = p->n_ao;
        for (size_t s = 0; s < n_spin; ++s)
          std::memcpy(fock + s * n * n, uw12::linalg::mem_ptr(total.fock[s]),
                      n * n * sizeof(double));
      }
    }
    if (seconds) *seconds = seconds_since(t0);
  });
}

// The ABS+ projector blocks S^-1 over the kept eigenspace of the combined
// (n_ao + n_ri)^2 overlap: ri_ri (R x R), ri_ao (R x N), ao_ri (N x R),
// ao_ao (N x N), each column-major; n_kept (nullable) = kept eigenvectors.
int uw12ref_abs_blocks(const double* S, size_t n_ao, size_t n_ri,
                       double* ri_ri, double* ri_ao, double* ao_ri,
                       double* ao_ao, size_t* n_kept) {
  return guarded([&] {
    const auto abs = uw12::setup_abs_projectors(S, n_ao, n_ri);
    auto put = [](const uw12::linalg::Mat& m, double* dst) {
      if (dst)
        std::memcpy(dst, uw12::linalg::mem_ptr(m),
                    uw12::linalg::n_elem(m) * sizeof(double));
    };
    put(abs.s_inv_ri_ri, ri_ri);
    put(abs.s_inv_ri_ao, ri_ao);
    put(abs.s_inv_ao_ri, ao_ri);
    put(abs.s_inv_ao_ao, ao_ao);
    if (n_kept) {
      const auto Sm = uw12::linalg::mat(const_cast<double*>(S), n_ao + n_ri,
                                        n_ao + n_ri);
      const auto [vals, vecs] =
          uw12::linalg::eigen_decomposition(Sm, 1e-6, 1e-8);
      *n_kept = uw12::linalg::n_elem(vals);
    }
  });
}

#ifdef UW12REF_TIMING_BUILD
// Sampled loops (rounds > 0) or every iteration (0); resets the counters of
// the next evaluation (the per-loop estimates of the rotation are kept).
void uw12ref_timing_set(int rounds) {
  uw12ref_timing::sample_rounds = rounds;
  uw12ref_timing::extra_seconds = 0.0;
  uw12ref_timing::sampled_loops = 0;
  uw12ref_timing::full_loops = 0;
  uw12ref_timing::loop_index = 0;
  uw12ref_timing::loop_log.clear();
}

// The loop log of the last evaluation: up to max records of (iterations,
// sampled, seconds) into out (3 doubles each); returns the record count.
long uw12ref_timing_loops(double* out, long max) {
  const auto& lg = uw12ref_timing::loop_log;
  for (long i = 0; i < max && i < static_cast<long>(lg.size()); ++i) {
    out[3 * i] = static_cast<double>(lg[i].n);
    out[3 * i + 1] = lg[i].sampled;
    out[3 * i + 2] = lg[i].seconds;
  }
  return static_cast<long>(lg.size());
}

// Rotation over the sampled loops: of S consecutive evaluations, evaluation
// `phase` measures the loops q with q % S == phase (S = 0: all, and the cache
// of loop estimates is cleared).
void uw12ref_timing_rotation(int S, int phase) {
  uw12ref_timing::rotation = S;
  uw12ref_timing::phase = S > 0 ? phase % S : 0;
  if (S == 0) uw12ref_timing::cached.clear();
}

// Extrapolated seconds of the iterations skipped since the last set, and the
// numbers of sampled and fully run top-level loops.
void uw12ref_timing_read(double* extra_seconds, long* sampled_loops,
                         long* full_loops) {
  *extra_seconds = uw12ref_timing::extra_seconds;
  *sampled_loops = uw12ref_timing::sampled_loops;
  *full_loops = uw12ref_timing::full_loops;
}
#endif

}  // extern "C"
