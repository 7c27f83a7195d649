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
//     iterations (T = OpenMP threads) runs a sample and adds the extrapolated
//     time of the rest to extra_seconds. The reference's OpenMP loops use the
//     static schedule: thread t runs one contiguous block of n / T or n / T + 1
//     iterations (the first n mod T threads the longer ones; two-index loops:
//     blocks of outer iterations, n2 inner ones each), and the loop ends with
//     its slowest thread. Thread t runs the first max(2, r) iterations of its
//     own block, in order, all threads at once (the same memory contention),
//     timing each: the first runs cold, the others warm, and the block is
//     estimated as the sampled times plus its remaining iterations at the
//     mean warm time; the loop as the slowest block. (Extrapolating one
//     round's wall time -- the slowest of T cold first iterations -- over all
//     rounds overestimated c1m by 18-22 %.) Loop results are then partial
//     sums; only the time is used.
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

#include <algorithm>
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


inline bool sampling_applies(size_t n, bool parallel) {
  return sample_rounds > 0 && parallel && !omp_in_parallel() &&
         n > static_cast<size_t>(sample_rounds) *
                 static_cast<size_t>(omp_get_max_threads());
}

// First iteration and size of thread t's block of the static schedule of n
// iterations over T threads.
inline void static_block(size_t n, size_t T, size_t t, size_t& first, size_t& size) {
  size_t q = n / T, extra = n % T;
  if (t < extra) {
    ++q;
    extra = 0;
  }
  first = q * t + extra;
  size = q;
}

// Sampled iterations: the first k = min(size, max(2, r)) iterations of every
// non-empty block, in order (block t run by thread t, as in the full loop).
struct Sample {
  std::vector<std::vector<size_t>> items;  // per block
  std::vector<size_t> block;               // block sizes
};

inline Sample block_sample(size_t n, size_t T, size_t r) {
  Sample smp;
  smp.items.assign(T, {});
  smp.block.assign(T, 0);
  const size_t want = r < 2 ? 2 : r;
  for (size_t t = 0; t < T; ++t) {
    size_t first = 0, size = 0;
    static_block(n, T, t, first, size);
    smp.block[t] = size;
    for (size_t u = 0; u < size && u < want; ++u) smp.items[t].push_back(first + u);
  }
  return smp;
}

// Thread t runs its block's sampled iterations one after another, all threads
// at once (the same memory contention as the full loop), timing each.  A
// block's first iteration runs cold (the thread's first touch of its
// temporaries), the later ones warm, so block t is estimated as its sampled
// iterations plus the rest of its units x size iterations at the mean warm
// time (`units`: inner iterations per block element, n2 for two-index loops,
// whose sample runs one inner iteration per outer one), and the loop as the
// slowest block.  Under rotation a loop not due for measurement runs no
// iteration and books its cached estimate.
template <typename Body>
void run_sample(const Sample& smp, double units, Body&& body) {
  const long q_loop = loop_index++;
  if (cached.size() <= static_cast<size_t>(q_loop)) cached.resize(q_loop + 1, -1.0);
  if (rotation > 0 && q_loop % rotation != phase && cached[q_loop] >= 0.0) {
    extra_seconds += cached[q_loop];
    return;
  }
  const long T = static_cast<long>(smp.block.size());
  std::vector<double> est(smp.block.size(), 0.0);
  const double t0 = omp_get_wtime();
#pragma omp parallel for schedule(static, 1)
  for (long t = 0; t < T; ++t) {
    const std::vector<size_t>& its = smp.items[static_cast<size_t>(t)];
    double first = 0.0, warm = 0.0;
    for (size_t u = 0; u < its.size(); ++u) {
      const double a = omp_get_wtime();
      body(static_cast<size_t>(t), its[u]);
      const double d = omp_get_wtime() - a;
      if (u == 0) first = d; else warm += d;
    }
    const double k = static_cast<double>(its.size());
    const double total = units * static_cast<double>(smp.block[static_cast<size_t>(t)]);
    if (k > 1.0)
      est[static_cast<size_t>(t)] = first + warm + (total - k) * warm / (k - 1.0);
    else if (k > 0.0)
      est[static_cast<size_t>(t)] = total * first;
  }
  const double wall = omp_get_wtime() - t0;
  double estimate = 0.0;
  for (double e : est) estimate = std::max(estimate, e);
  cached[q_loop] = estimate;
  extra_seconds += estimate - wall;
  ++sampled_loops;
  loop_log.push_back({smp.block.size(), 1, estimate});
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
    ts::run_sample(ts::block_sample(n, T, r), 1.0, [&](size_t, size_t i) { func(start + i); });
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
    const ts::Sample smp = ts::block_sample(n, T, r);
    std::vector<ReturnType> part(T, identity);
    ts::run_sample(smp, 1.0, [&](size_t q, size_t i) { part[q] += func(start + i); });
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
    // blocks of outer iterations; each sampled outer iteration runs one inner
    // iteration (the middle one), an n2-th of its cost
    ts::Sample smp = ts::block_sample(n1, T, r);
    for (auto& blk : smp.items)
      for (size_t& it : blk) it = it * n2 + n2 / 2;
    std::vector<ReturnType> part(T, identity);
    ts::run_sample(smp, static_cast<double>(n2), [&](size_t q, size_t p) {
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
