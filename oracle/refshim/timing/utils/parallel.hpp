// Loop dispatcher of the TIMING build of the libuw12 reference -- TEST
// INFRASTRUCTURE ONLY (the CPU baseline of bench.py).
//
// oracle/ref.mk compiles libuw12's unmodified sources twice. The parity build
// (libuw12_ref.so) uses the reference's own src/utils/parallel.hpp. The timing
// build (libuw12_ref_timing.so) puts this directory first on the include path,
// so that src/integrals/{integral_functions,transformations}.hpp, the only
// files that include "utils/parallel.hpp", get this dispatcher instead. It has
// the interface of the reference's parallel.hpp:31-183 (parallel_for,
// parallel_sum, parallel_sum_2d, isolate) and two modes:
//
//   * full (sample_rounds == 0): every iteration runs, OpenMP-parallel at the
//     top level and serially inside an active parallel region, as in the
//     reference's OpenMP build;
//   * sampled (sample_rounds = r > 0): a top-level loop with more than r x T
//     iterations (T = OpenMP threads) runs r x T evenly spaced iterations,
//     r per thread, all threads at once, and adds the extrapolated time of the
//     rest to extra_seconds. The reference's OpenMP schedule gives each thread
//     a contiguous block of n / T or n / T + 1 iterations (two-index loops:
//     outer iterations of n2 inner ones each), so the whole loop takes
//     floor(n / T) rounds with every thread busy and, when T does not divide
//     n, one round with n mod T threads busy (two-index: floor(n1 / T) n2 and
//     n2 rounds).  The sample measures r full rounds under the same memory
//     contention, and the partial round by running n mod T iterations at once
//     (fewer busy threads contend less, so a partial round is faster than a
//     full one).  Loop results are then partial sums; only the time is used.
//   * rotation (rotation = S > 0, with sampling): the sampled loops of an
//     evaluation are numbered in the order they run; loop q is measured (as
//     above) only when q % S == phase and otherwise skipped, its estimate
//     taken from the last evaluation that measured it. S consecutive
//     evaluations (phase 0 .. S-1) measure every loop once, each at about
//     1/S of the sampled cost; the code outside the loops runs every time.
//
// The estimates are checked against full evaluations of the parity build by
// oracle/validate_sampler.py.
#ifndef UW12_PARALLEL_HPP
#define UW12_PARALLEL_HPP

#include <omp.h>

#include <functional>
#include <vector>

namespace uw12ref_timing {
inline int sample_rounds = 0;       // 0: every iteration runs
inline double extra_seconds = 0.0;  // extrapolated time of skipped iterations
inline long sampled_loops = 0;      // top-level loops that were sampled
inline long full_loops = 0;         // top-level loops that ran every iteration
inline int rotation = 0;            // 0: every sampled loop measured each time
inline int phase = 0;               // loops q with q % rotation == phase measured
inline long loop_index = 0;         // sampled loops seen in this evaluation
inline std::vector<double> cached;  // last estimate per loop index (< 0: none)
// every top-level loop of the evaluation in order: iterations, 1 if sampled,
// seconds (the estimate when sampled, the measured time otherwise)
struct LoopRecord {
  size_t n;
  int sampled;
  double seconds;
};
inline std::vector<LoopRecord> loop_log;

inline size_t ceil_div(size_t a, size_t b) { return (a + b - 1) / b; }

inline bool sampling_applies(size_t n, bool parallel) {
  return sample_rounds > 0 && parallel && !omp_in_parallel() &&
         n > static_cast<size_t>(sample_rounds) *
                 static_cast<size_t>(omp_get_max_threads());
}

// k evenly spaced indices of [0, n).
inline std::vector<size_t> spaced(size_t n, size_t k) {
  std::vector<size_t> idx(k);
  for (size_t t = 0; t < k; ++t)
    idx[t] = static_cast<size_t>((static_cast<double>(t) + 0.5) *
                                 static_cast<double>(n) /
                                 static_cast<double>(k));
  return idx;
}

// Runs body(slot, item) for every sampled item, r per thread, then the
// partial-round items at once, and books the extrapolated remainder: the full
// loop takes `rounds_full` rounds with every thread busy (the sample ran r)
// and `rounds_part` rounds with part.size() threads busy (the sample ran one).
// Under rotation a loop not due for measurement runs no iteration and books
// its cached estimate.
template <typename Body>
void run_sample(const std::vector<size_t>& items, size_t r, double rounds_full,
                const std::vector<size_t>& part, double rounds_part, Body&& body) {
  const long q_loop = loop_index++;
  if (cached.size() <= static_cast<size_t>(q_loop)) cached.resize(q_loop + 1, -1.0);
  if (rotation > 0 && q_loop % rotation != phase && cached[q_loop] >= 0.0) {
    extra_seconds += cached[q_loop];
    return;
  }
  const double t0 = omp_get_wtime();
#pragma omp parallel for schedule(static, 1)
  for (long q = 0; q < static_cast<long>(items.size()); ++q)
    body(static_cast<size_t>(q), items[static_cast<size_t>(q)]);
  const double t1 = omp_get_wtime();
  if (!part.empty()) {
#pragma omp parallel for schedule(static, 1)
    for (long q = 0; q < static_cast<long>(part.size()); ++q)
      body(static_cast<size_t>(q), part[static_cast<size_t>(q)]);
  }
  const double t2 = omp_get_wtime();
  const double estimate =
      (t1 - t0) * rounds_full / static_cast<double>(r) + (t2 - t1) * rounds_part;
  cached[q_loop] = estimate;
  extra_seconds += estimate - (t2 - t0);
  ++sampled_loops;
  loop_log.push_back({items.size(), 1, estimate});
}

// Times a top-level loop that runs every iteration (for the loop log).
template <typename F>
auto timed_full(size_t n, F&& f) {
  if (omp_in_parallel()) return f();
  const double t0 = omp_get_wtime();
  auto out = f();
  loop_log.push_back({n, 0, omp_get_wtime() - t0});
  return out;
}
}  // namespace uw12ref_timing

namespace uw12::parallel {

inline void parallel_for(size_t start, size_t stop,
                         const std::function<void(size_t)>& func,
                         bool parallel = true) {
  namespace ts = uw12ref_timing;
  const size_t n = stop > start ? stop - start : 0;
  if (ts::sampling_applies(n, parallel)) {
    const size_t T = static_cast<size_t>(omp_get_max_threads());
    const size_t r = static_cast<size_t>(ts::sample_rounds);
    ts::run_sample(ts::spaced(n, r * T), r, static_cast<double>(n / T),
                   ts::spaced(n, n % T), 1.0,
                   [&](size_t, size_t i) { func(start + i); });
    return;
  }
  if (!omp_in_parallel()) ++ts::full_loops;
  ts::timed_full(n, [&] {
    if (parallel) {
#pragma omp parallel for
      for (long i = static_cast<long>(start); i < static_cast<long>(stop); ++i)
        func(static_cast<size_t>(i));
    } else {
      for (size_t i = start; i < stop; ++i) func(i);
    }
    return 0;
  });
}

// Sum over every iteration with one partial result per thread, added up at
// the end (the reference's OpenMP reduction).
template <typename ReturnType, typename Fn>
ReturnType full_sum(size_t start, size_t stop, const ReturnType& identity,
                    const Fn& func, bool parallel) {
  if (!parallel) {
    ReturnType result(identity);
    for (size_t i = start; i < stop; ++i) result += func(i);
    return result;
  }
  std::vector<ReturnType> part;
#pragma omp parallel
  {
#pragma omp single
    part.assign(static_cast<size_t>(omp_get_num_threads()), identity);
    ReturnType& mine = part[static_cast<size_t>(omp_get_thread_num())];
#pragma omp for
    for (long i = static_cast<long>(start); i < static_cast<long>(stop); ++i)
      mine += func(static_cast<size_t>(i));
  }
  ReturnType result(identity);
  for (auto& p : part) result += p;
  return result;
}

template <typename ReturnType>
ReturnType parallel_sum(const size_t start, const size_t stop,
                        const ReturnType& identity,
                        const std::function<ReturnType(size_t)>& func,
                        const bool parallel = true) {
  namespace ts = uw12ref_timing;
  const size_t n = stop > start ? stop - start : 0;
  if (ts::sampling_applies(n, parallel)) {
    const size_t T = static_cast<size_t>(omp_get_max_threads());
    const size_t r = static_cast<size_t>(ts::sample_rounds);
    const auto items = ts::spaced(n, r * T);
    std::vector<ReturnType> part(items.size(), identity);
    ts::run_sample(items, r, static_cast<double>(n / T), ts::spaced(n, n % T), 1.0,
                   [&](size_t q, size_t i) { part[q] += func(start + i); });
    return part[0];
  }
  if (!omp_in_parallel()) ++ts::full_loops;
  return ts::timed_full(n, [&] { return full_sum(start, stop, identity, func, parallel); });
}

template <typename ReturnType>
ReturnType parallel_sum_2d(
    const size_t start1, const size_t stop1, const size_t start2,
    const size_t stop2, const ReturnType& identity,
    const std::function<ReturnType(size_t, size_t)>& func,
    const bool parallel = true) {
  namespace ts = uw12ref_timing;
  const size_t n1 = stop1 > start1 ? stop1 - start1 : 0;
  const size_t n2 = stop2 > start2 ? stop2 - start2 : 0;
  if (ts::sampling_applies(n1 * n2, parallel)) {
    const size_t T = static_cast<size_t>(omp_get_max_threads());
    const size_t r = static_cast<size_t>(ts::sample_rounds);
    const auto items = ts::spaced(n1 * n2, r * T);
    std::vector<ReturnType> part(items.size(), identity);
    // partial round: n1 mod T threads, one inner item each (outer iterations
    // evenly spaced)
    std::vector<size_t> rem;
    for (size_t i : ts::spaced(n1, n1 % T)) rem.push_back(i * n2 + n2 / 2);
    ts::run_sample(items, r, static_cast<double>((n1 / T) * n2), rem,
                   static_cast<double>(n2), [&](size_t q, size_t p) {
                     part[q] += func(start1 + p / n2, start2 + p % n2);
                   });
    return part[0];
  }
  if (!omp_in_parallel()) ++ts::full_loops;
  // outer iterations in parallel, the inner loop serial within each
  const auto outer = [&](size_t i) -> ReturnType {
    ReturnType result(identity);
    for (size_t j = start2; j < stop2; ++j) result += func(i, j);
    return result;
  };
  return ts::timed_full(n1 * n2,
                        [&] { return full_sum(start1, stop1, identity, outer, parallel); });
}

template <typename Func>
void isolate(Func&& func) {
  func();
}

}  // namespace uw12::parallel

#endif  // UW12_PARALLEL_HPP
