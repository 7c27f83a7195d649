// libuw12.hpp -- C++ drop-in for libuw12's public API on the B200 library.
//
// Same namespace, types and function signatures as libuw12's libuw12.hpp
// (setup_base_integrals, setup_abs_projectors, setup_orbitals,
// setup_occupations, uw12_energy, uw12_fock) plus form_fock (src/uw12.hpp)
// and the BaseIntegrals constructors of src/integrals/base_integrals.hpp,
// implemented header-only over the C-ABI in uw12_c.h.  Armadillo's arma::mat
// is replaced by uw12::linalg::Mat, a column-major matrix owning its storage.
// Failures throw std::runtime_error / std::logic_error as libuw12 does.
#ifndef UW12_B200_LIBUW12_HPP
#define UW12_B200_LIBUW12_HPP

#include <algorithm>
#include <array>
#include <cfloat>
#include <cmath>
#include <cstddef>
#include <cstring>
#include <exception>
#include <fstream>
#include <functional>
#include <memory>
#include <mutex>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "uw12_c.h"

namespace uw12 {

namespace linalg {

/// Column-major dense matrix (the role of arma::mat in libuw12).
class Mat {
 public:
  Mat() = default;
  Mat(size_t rows, size_t cols) : r_(rows), c_(cols), d_(rows * cols, 0.0) {}
  Mat(const double* data, size_t rows, size_t cols)
      : r_(rows), c_(cols), d_(data, data + rows * cols) {}
  size_t n_rows() const { return r_; }
  size_t n_cols() const { return c_; }
  size_t n_elem() const { return d_.size(); }
  double& operator()(size_t i, size_t j) { return d_[i + r_ * j]; }
  double operator()(size_t i, size_t j) const { return d_[i + r_ * j]; }
  double& operator[](size_t i) { return d_[i]; }
  double operator[](size_t i) const { return d_[i]; }
  double* memptr() { return d_.data(); }
  const double* memptr() const { return d_.data(); }

 private:
  size_t r_ = 0, c_ = 0;
  std::vector<double> d_;
};

/// Column vector (the role of arma::vec).
class Vec : public Mat {
 public:
  Vec() = default;
  explicit Vec(size_t n) : Mat(n, 1) {}
  Vec(size_t rows, size_t cols) : Mat(rows, cols) {}
  Vec(const double* data, size_t n) : Mat(data, n, 1) {}
  Vec(const double* data, size_t rows, size_t cols) : Mat(data, rows, cols) {}
};

inline size_t n_rows(const Mat& m) { return m.n_rows(); }
inline size_t n_cols(const Mat& m) { return m.n_cols(); }
inline size_t n_elem(const Mat& m) { return m.n_elem(); }
inline double elem(const Mat& m, size_t i, size_t j) { return m(i, j); }
inline const double* mem_ptr(const Mat& m) { return m.memptr(); }

/// Load a matrix from a comma-separated text file, one matrix row per line
/// (linalg::load_csv, src/utils/linalg.hpp:1070-1104).  Blank lines are
/// skipped; a missing file, an unparsable cell or rows of different lengths
/// throw std::runtime_error("cannot read data from file").
inline Mat load_csv(const std::string& filepath) {
  std::ifstream in(filepath);
  if (!in) throw std::runtime_error("cannot read data from file");
  std::vector<std::vector<double>> rows;
  std::string line;
  while (std::getline(in, line)) {
    if (!line.empty() && line.back() == '\r') line.pop_back();
    if (line.find_first_not_of(" \t") == std::string::npos) continue;
    std::vector<double> row;
    std::stringstream ls(line);
    std::string cell;
    while (std::getline(ls, cell, ',')) {
      try {
        size_t used = 0;
        row.push_back(std::stod(cell, &used));
        if (cell.find_first_not_of(" \t", used) != std::string::npos)
          throw std::runtime_error("cannot read data from file");
      } catch (const std::logic_error&) {
        throw std::runtime_error("cannot read data from file");
      }
    }
    if (!rows.empty() && row.size() != rows.front().size())
      throw std::runtime_error("cannot read data from file");
    rows.push_back(std::move(row));
  }
  const size_t r = rows.size(), c = r ? rows.front().size() : 0;
  Mat m(r, c);
  for (size_t i = 0; i < r; ++i)
    for (size_t j = 0; j < c; ++j) m(i, j) = rows[i][j];
  return m;
}

}  // namespace linalg

namespace detail {

inline std::string last_error() {
  char buf[1024];
  uw12c_last_error(buf, sizeof(buf));
  return std::string(buf);
}

inline void check(int status) {
  if (status == UW12C_OK) return;
  if (status == UW12C_ERR_LOGIC) throw std::logic_error(last_error());
  throw std::runtime_error(last_error());
}

}  // namespace detail

namespace integrals {

/// Returns the two-index integrals (A|w|B), n_df x n_df (integral_functions.hpp:17).
using TwoIndexFn = std::function<linalg::Mat()>;
/// Returns the three-index integrals of one df shell A: n_ao(n_ao+1)/2 x n_A
/// (AO) or n_ri*n_ao x n_A (RI) (integral_functions.hpp:20).
using ThreeIndexFn = std::function<linalg::Mat(size_t)>;

/// Device-resident density-fitting integrals (base_integrals.hpp:46-293).
class BaseIntegrals {
 public:
  BaseIntegrals() = default;

  /// Stored integrals with RI (base_integrals.hpp:94-96).
  BaseIntegrals(const linalg::Mat& J3_0, const linalg::Mat& J2, const linalg::Mat& J3_ri_0) {
    const size_t n_ao = n_ao_from_packed(J3_0.n_rows());
    create(J3_0.memptr(), J2.memptr(), J3_ri_0.memptr(), n_ao, J2.n_rows(),
           n_ao ? J3_ri_0.n_rows() / n_ao : 0, J3_0.n_cols(), J3_ri_0.n_cols());
  }

  /// Stored integrals without RI (base_integrals.hpp:99).
  BaseIntegrals(const linalg::Mat& J3_0, const linalg::Mat& J2) {
    create(J3_0.memptr(), J2.memptr(), nullptr, n_ao_from_packed(J3_0.n_rows()), J2.n_rows(), 0,
           J3_0.n_cols(), 0);
  }

  /// Integrals already in the metric eigenbasis, J3 = J3_0 P2, with their
  /// eigenvalues (base_integrals.hpp:104); cannot be used for RI.
  BaseIntegrals(const linalg::Mat& J3, const linalg::Vec& df_vals) {
    const size_t n_ao = n_ao_from_packed(J3.n_rows());
    if (J3.n_cols() != df_vals.n_elem())
      throw std::runtime_error("Number of density-fitting basis functions inconsistent");
    uw12c_integrals* h = nullptr;
    detail::check(uw12c_integrals_create_eigenbasis(J3.memptr(), df_vals.memptr(), n_ao,
                                                    df_vals.n_elem(), UW12C_MEM_HOST, &h));
    h_.reset(h, uw12c_integrals_destroy);
  }

  /// Integrals from callbacks, one df shell per three-index call
  /// (base_integrals.hpp:52-62).  A stored tensor is produced once and kept on
  /// the device; an unstored one is produced again, shell by shell, in the aux
  /// blocks each use needs (integral-direct mode), so the callbacks must stay
  /// callable for the object's lifetime and may run on several host threads.
  BaseIntegrals(const TwoIndexFn& two_index_fn, const ThreeIndexFn& three_index_fn,
                const ThreeIndexFn& three_index_ri_fn, const std::vector<size_t>& df_sizes,
                size_t n_ao, size_t n_df, size_t n_ri, bool store_ao_integrals = true,
                bool store_ri_integrals = true) {
    check_shells(df_sizes, n_ao, n_df);
    if (n_ri == 0)
      throw std::runtime_error(
          "Three index ri integrals requested but number of ri basis functions is zero");
    const linalg::Mat J2 = two_index_fn();
    auto ao = std::make_shared<ShellProducer>(three_index_fn, df_sizes, n_ao * (n_ao + 1) / 2);
    auto ri = std::make_shared<ShellProducer>(three_index_ri_fn, df_sizes, n_ao * n_ri);
    create_produced(J2, ao, ri, n_ao, n_df, n_ri, store_ao_integrals, store_ri_integrals);
  }

  /// Callback integrals without RI (base_integrals.hpp:65-72).
  BaseIntegrals(const TwoIndexFn& two_index_fn, const ThreeIndexFn& three_index_fn,
                const std::vector<size_t>& df_sizes, size_t n_ao, size_t n_df,
                bool store_ao_integrals = true) {
    check_shells(df_sizes, n_ao, n_df);
    const linalg::Mat J2 = two_index_fn();
    auto ao = std::make_shared<ShellProducer>(three_index_fn, df_sizes, n_ao * (n_ao + 1) / 2);
    create_produced(J2, ao, nullptr, n_ao, n_df, 0, store_ao_integrals, true);
  }

  /// Stored AO integrals with RI integrals from a callback (base_integrals.hpp:78-88);
  /// unless store_ri_integrals, the RI shells are produced at every use.
  BaseIntegrals(const linalg::Mat& J3_0, const linalg::Mat& J2,
                const ThreeIndexFn& three_index_ri, const std::vector<size_t>& df_sizes,
                bool use_ri, size_t n_ao, size_t n_df, size_t n_ri,
                bool store_ri_integrals = false) {
    if (!use_ri) {
      create(J3_0.memptr(), J2.memptr(), nullptr, n_ao_from_packed(J3_0.n_rows()), J2.n_rows(),
             0, J3_0.n_cols(), 0);
      return;
    }
    check_shells(df_sizes, n_ao, n_df);
    if (J3_0.n_rows() != n_ao * (n_ao + 1) / 2 || J3_0.n_cols() != n_df)
      throw std::runtime_error("Number of density-fitting basis functions inconsistent");
    // J3_0's columns, copied to the device during construction only
    auto ao = std::make_shared<ShellProducer>(nullptr, std::vector<size_t>{n_df}, J3_0.n_rows());
    ao->stored = J3_0.memptr();
    auto ri = std::make_shared<ShellProducer>(three_index_ri, df_sizes, n_ao * n_ri);
    create_produced(J2, ao, ri, n_ao, n_df, n_ri, true, store_ri_integrals);
  }

  /// From raw pointers in host or device memory (uw12c_integrals_create).
  static BaseIntegrals from_pointers(const double* X3, const double* X2, const double* X3_ri,
                                     size_t n_ao, size_t n_df, size_t n_ri, int mem_kind) {
    BaseIntegrals b;
    uw12c_integrals* h = nullptr;
    detail::check(uw12c_integrals_create(X3, X2, X3_ri, n_ao, n_df, n_ri, mem_kind, &h));
    b.h_.reset(h, uw12c_integrals_destroy);
    return b;
  }

  size_t get_number_ao() const { return dims(0); }
  size_t get_number_df() const { return dims(1); }
  size_t get_number_ri() const { return dims(2); }

  linalg::Vec get_df_vals() const {
    linalg::Vec v(get_number_df(), 1);
    detail::check(uw12c_integrals_df_vals(handle(), v.memptr()));
    return v;
  }

  const uw12c_integrals* handle() const {
    if (!h_) throw std::runtime_error("BaseIntegrals not initialised");
    return h_.get();
  }

 private:
  static size_t n_ao_from_packed(size_t n) {
    if (n == 0) throw std::runtime_error("Number of ao orbitals is zero");
    const auto n_ao = static_cast<size_t>(std::sqrt(8.0 * double(n) - 1.0) / 2.0);
    if (n_ao * (n_ao + 1) / 2 != n) throw std::logic_error("vector must be of length n(n+1)/2");
    return n_ao;
  }

  static void check_shells(const std::vector<size_t>& df_sizes, size_t n_ao, size_t n_df) {
    if (df_sizes.empty())
      throw std::runtime_error("no df_sizes provided, cannot calculate three index integrals");
    if (n_df == 0 || n_ao == 0)
      throw std::runtime_error(
          "Number of basis functions is zero, cannot calculate basis functions");
    if (df_sizes.size() > n_df)
      throw std::runtime_error("More shells than basis functions in df basis");
    size_t total = 0;
    for (size_t s : df_sizes) total += s;
    if (total != n_df)
      throw std::runtime_error("total df basis functions inconsistent with number in shells");
  }

  // A ThreeIndexFn as a uw12c_block_fn: columns [first, first + count) of
  // the tensor come from the shells that overlap them (coulomb_3idx,
  // integral_functions.hpp:33-55: shell A holds columns offset(A) ..
  // offset(A) + n_A).  The first exception a shell call throws is kept and
  // rethrown on the calling thread once the library reports the failure.
  struct ShellProducer {
    ShellProducer(ThreeIndexFn f, const std::vector<size_t>& df_sizes, size_t n_rows)
        : fn(std::move(f)), rows(n_rows) {
      offsets.push_back(0);
      for (size_t n : df_sizes) offsets.push_back(offsets.back() + n);
    }

    static int call(void* user, size_t first, size_t count, double* out, size_t ld,
                    void* /*stream*/) noexcept {
      auto* p = static_cast<ShellProducer*>(user);
      try {
        if (p->stored) {
          for (size_t c = 0; c < count; ++c)
            std::memcpy(out + c * ld, p->stored + (first + c) * p->rows, p->rows * sizeof(double));
          return 0;
        }
        const size_t end = first + count;
        size_t A = static_cast<size_t>(
            std::upper_bound(p->offsets.begin(), p->offsets.end(), first) - p->offsets.begin());
        for (A = A - 1; A + 1 < p->offsets.size() && p->offsets[A] < end; ++A) {
          const linalg::Mat shell = p->fn(A);
          if (shell.n_rows() != p->rows || shell.n_cols() != p->offsets[A + 1] - p->offsets[A])
            throw std::logic_error("three-index shell of unexpected size");
          const size_t c0 = std::max(first, p->offsets[A]);
          const size_t c1 = std::min(end, p->offsets[A + 1]);
          for (size_t c = c0; c < c1; ++c)
            std::memcpy(out + (c - first) * ld, shell.memptr() + (c - p->offsets[A]) * p->rows,
                        p->rows * sizeof(double));
        }
        return 0;
      } catch (...) {
        std::lock_guard<std::mutex> lock(p->mu);
        if (!p->error) p->error = std::current_exception();
        return 1;
      }
    }

    void rethrow() {
      std::lock_guard<std::mutex> lock(mu);
      if (error) std::rethrow_exception(error);
    }

    ThreeIndexFn fn;
    std::vector<size_t> offsets;
    size_t rows;
    const double* stored = nullptr;  // a tensor in memory instead of fn
    std::mutex mu;
    std::exception_ptr error;
  };

  void create_produced(const linalg::Mat& J2, const std::shared_ptr<ShellProducer>& ao,
                       const std::shared_ptr<ShellProducer>& ri, size_t n_ao, size_t n_df,
                       size_t n_ri, bool store_ao, bool store_ri) {
    if (J2.n_rows() != n_df || J2.n_cols() != n_df)
      throw std::runtime_error("Number of density-fitting basis functions inconsistent");
    uw12c_integrals* h = nullptr;
    const int status = uw12c_integrals_create_callback(
        J2.memptr(), UW12C_MEM_HOST, &ShellProducer::call, ao.get(),
        ri ? &ShellProducer::call : nullptr, ri.get(), n_ao, n_df, ri ? n_ri : 0, store_ao,
        store_ri, UW12C_MEM_HOST, &h);
    if (status != UW12C_OK) {
      ao->rethrow();
      if (ri) ri->rethrow();
      detail::check(status);
    }
    // the producers live as long as the handle that calls them
    h_.reset(h, [ao, ri](uw12c_integrals* p) { uw12c_integrals_destroy(p); });
  }

  void create(const double* X3, const double* X2, const double* X3_ri, size_t n_ao, size_t n_df,
              size_t n_ri, size_t cols3, size_t cols3_ri) {
    if (cols3 != n_df || (X3_ri && cols3_ri != n_df))
      throw std::runtime_error("Number of density-fitting basis functions inconsistent");
    uw12c_integrals* h = nullptr;
    detail::check(uw12c_integrals_create(X3, X2, X3_ri, n_ao, n_df, X3_ri ? n_ri : 0,
                                         UW12C_MEM_HOST, &h));
    h_.reset(h, uw12c_integrals_destroy);
  }

  size_t dims(int which) const {
    size_t d[3] = {0, 0, 0};
    detail::check(uw12c_integrals_dims(handle(), &d[0], &d[1], &d[2]));
    return d[which];
  }

  std::shared_ptr<uw12c_integrals> h_;
};

}  // namespace integrals

namespace three_el::ri {

/// ABS+ projectors (ri_utils.hpp:20-29), device resident.
class ABSProjectors {
 public:
  ABSProjectors() = default;
  ABSProjectors(const double* S, size_t n_ao, size_t n_ri, int mem_kind = UW12C_MEM_HOST)
      : n_ao_(n_ao), n_ri_(n_ri) {
    uw12c_abs* h = nullptr;
    detail::check(uw12c_abs_create(S, n_ao, n_ri, mem_kind, &h));
    h_.reset(h, uw12c_abs_destroy);
  }
  /// The four blocks s_inv_ri_ri, s_inv_ri_ao, s_inv_ao_ri, s_inv_ao_ao.
  std::vector<linalg::Mat> blocks() const {
    std::vector<linalg::Mat> b{linalg::Mat(n_ri_, n_ri_), linalg::Mat(n_ri_, n_ao_),
                               linalg::Mat(n_ao_, n_ri_), linalg::Mat(n_ao_, n_ao_)};
    detail::check(uw12c_abs_blocks(handle(), b[0].memptr(), b[1].memptr(), b[2].memptr(),
                                   b[3].memptr()));
    return b;
  }
  const uw12c_abs* handle() const {
    if (!h_) throw std::runtime_error("ABSProjectors not initialised");
    return h_.get();
  }

 private:
  size_t n_ao_ = 0, n_ri_ = 0;
  std::shared_ptr<uw12c_abs> h_;
};

/// calculate_abs_projectors (ri_utils.hpp:45-74) for a combined AO+RI overlap.
inline ABSProjectors calculate_abs_projectors(const linalg::Mat& S, size_t n_ao, size_t n_ri) {
  if (S.n_rows() != n_ao + n_ri || S.n_cols() != n_ao + n_ri)
    throw std::runtime_error("Total number of basis functions is inconsistent");
  return ABSProjectors(S.memptr(), n_ao, n_ri);
}

}  // namespace three_el::ri

namespace utils {
using Orbitals = std::vector<linalg::Mat>;
using Occupations = std::vector<linalg::Vec>;
using FockMatrix = std::vector<linalg::Mat>;
/// utils.hpp:142-146.
struct FockMatrixAndEnergy {
  FockMatrix fock;
  double energy = 0.0;
};
}  // namespace utils

using integrals::BaseIntegrals;
using three_el::ri::ABSProjectors;
using utils::Occupations;
using utils::Orbitals;

/// uw12::form_fock (src/uw12.hpp:129-142).
inline utils::FockMatrixAndEnergy form_fock(const BaseIntegrals& W, const BaseIntegrals& V,
                                            const BaseIntegrals& WV,
                                            const ABSProjectors& abs_projectors,
                                            const Orbitals& orbitals,
                                            const Occupations& occupations,
                                            const std::vector<size_t>& n_active,
                                            bool indirect_term, bool calculate_fock,
                                            double scale_opp_spin, double scale_same_spin,
                                            size_t print_level = 0) {
  const size_t n_spin = orbitals.size();
  if (n_spin < 1 || n_spin > 2) throw std::logic_error("invalid number of spin channels");
  if (occupations.size() < 1 || occupations.size() > 2)
    throw std::logic_error("invalid number of spin channels");
  if (occupations.size() != n_spin)
    throw std::runtime_error("Different number of spin channels for orbitals and occupations");
  if (n_active.size() < 1 || n_active.size() > 2)
    throw std::logic_error("invalid number of spin channels");
  if (n_active.size() != n_spin)
    throw std::runtime_error("Different number of spin channels in n_active and orbitals");
  const size_t n_ao = orbitals[0].n_rows();
  std::vector<const double*> C, occ;
  std::vector<size_t> ldc, n_orb, n_occ;
  for (size_t s = 0; s < n_spin; ++s) {
    if (orbitals[s].n_rows() != n_ao)
      throw std::runtime_error("Inconsistent number of atomic orbitals");
    C.push_back(orbitals[s].memptr());
    ldc.push_back(n_ao);
    n_orb.push_back(orbitals[s].n_cols());
    occ.push_back(occupations[s].memptr());
    n_occ.push_back(occupations[s].n_elem());
  }
  utils::FockMatrixAndEnergy out;
  linalg::Mat fock(n_ao, n_ao * n_spin);
  double terms[3];
  detail::check(uw12c_form_fock(W.handle(), V.handle(), WV.handle(), abs_projectors.handle(),
                                n_ao, n_spin, C.data(), ldc.data(), n_orb.data(), occ.data(),
                                n_occ.data(), n_active.data(), indirect_term ? 1 : 0,
                                calculate_fock ? 1 : 0, scale_opp_spin, scale_same_spin,
                                print_level, &out.energy, terms,
                                calculate_fock ? fock.memptr() : nullptr, UW12C_MEM_HOST));
  for (size_t s = 0; s < n_spin; ++s)
    out.fock.emplace_back(fock.memptr() + s * n_ao * n_ao, n_ao, n_ao);
  return out;
}

/// libuw12.hpp:42-50.
inline BaseIntegrals setup_base_integrals(const double* X3, const double* X2, const double* X3_ri,
                                          size_t n_ao, size_t n_df, size_t n_ri,
                                          bool /*copy_data*/ = false) {
  return BaseIntegrals::from_pointers(X3, X2, X3_ri, n_ao, n_df, n_ri, UW12C_MEM_HOST);
}

/// libuw12.hpp:64-70.
inline BaseIntegrals setup_base_integrals(const double* X3, const double* X2, size_t n_ao,
                                          size_t n_df, bool /*copy_data*/ = false) {
  return BaseIntegrals::from_pointers(X3, X2, nullptr, n_ao, n_df, 0, UW12C_MEM_HOST);
}

/// libuw12.hpp:80.
inline ABSProjectors setup_abs_projectors(const double* S, size_t n_ao, size_t n_ri) {
  return ABSProjectors(S, n_ao, n_ri);
}

/// libuw12.hpp:90-92 / libuw12.cpp:58-77: alpha columns then beta.
inline Orbitals setup_orbitals(const double* C, size_t n_ao, size_t n_orb, size_t n_spin) {
  if (n_spin != 1 && n_spin != 2)
    throw std::runtime_error("Number of spin channels must be 1 or 2");
  Orbitals out;
  for (size_t s = 0; s < n_spin; ++s) out.emplace_back(C + s * n_ao * n_orb, n_ao, n_orb);
  return out;
}

/// libuw12.hpp:101 (closed shell).
inline Occupations setup_occupations(const double* occ, size_t n_occ) {
  return {linalg::Vec(occ, n_occ, 1)};
}

/// libuw12.hpp:111-113 (open shell).
inline Occupations setup_occupations(const double* occ, size_t n_occ_alpha, size_t n_occ_beta) {
  return {linalg::Vec(occ, n_occ_alpha, 1), linalg::Vec(occ + n_occ_alpha, n_occ_beta, 1)};
}

/// libuw12.hpp:129-140.
inline double uw12_energy(const BaseIntegrals& W, const BaseIntegrals& V, const BaseIntegrals& WV,
                          const ABSProjectors& abs_projectors, const Orbitals& orbitals,
                          const Occupations& occ, const std::vector<size_t>& n_active,
                          double scale_opp_spin, double scale_same_spin,
                          size_t print_level = 0) {
  const bool indirect = !(std::fabs(scale_same_spin) <= 4 * DBL_EPSILON);
  return form_fock(W, V, WV, abs_projectors, orbitals, occ, n_active, indirect, false,
                   scale_opp_spin, scale_same_spin, print_level)
      .energy;
}

/// libuw12.hpp:157-169: fock receives n_ao x (n_ao * n_spin), spin blocks side by side.
inline double uw12_fock(double* fock, const BaseIntegrals& W, const BaseIntegrals& V,
                        const BaseIntegrals& WV, const ABSProjectors& abs_projectors,
                        const Orbitals& orbitals, const Occupations& occ,
                        const std::vector<size_t>& n_active, double scale_opp_spin,
                        double scale_same_spin, size_t print_level = 0) {
  const bool indirect = !(std::fabs(scale_same_spin) <= 4 * DBL_EPSILON);
  const auto res = form_fock(W, V, WV, abs_projectors, orbitals, occ, n_active, indirect, true,
                             scale_opp_spin, scale_same_spin, print_level);
  const size_t n_ao = orbitals[0].n_rows();
  for (size_t s = 0; s < res.fock.size(); ++s)
    for (size_t e = 0; e < n_ao * n_ao; ++e) fock[s * n_ao * n_ao + e] = res.fock[s][e];
  return res.energy;
}

/// Controls and entry points of the B200 library beyond libuw12's API (no
/// counterpart in libuw12).
namespace b200 {

/// Split-precision GEMMs (int8 tensor cores, n_moduli moduli) in the following
/// evaluations on this thread; 0 returns to FP64 (uw12c_set_precision).
inline void set_precision(int n_moduli) { detail::check(uw12c_set_precision(n_moduli)); }

/// Device-memory budget of the chunked loops in bytes; 0 restores the automatic
/// one (uw12c_set_memory_budget).
inline void set_memory_budget(size_t bytes) { detail::check(uw12c_set_memory_budget(bytes)); }

/// Gradients of the direct-term energy with respect to the integrals.
struct Gradients {
  std::vector<linalg::Mat> dX3;     ///< W, V, WV: packed n_ao(n_ao+1)/2 x n_df
  std::vector<linalg::Mat> dX3_ri;  ///< W, V: (n_ri n_ao) x n_df (empty when streamed)
  std::vector<linalg::Mat> dX2;     ///< W, V, WV: n_df x n_df
};

struct BackwardResult {
  utils::FockMatrixAndEnergy fock_energy;  ///< energy and Fock of form_fock without indirect term
  double terms[3] = {0, 0, 0};             ///< two-, three-, four-electron energies
  Gradients gradients;
};

/// A consumer of gradient blocks in host memory: aux functions [first, first +
/// count) as the columns of `block` (leading dimension ld), valid during the call.
using GradientSink =
    std::function<void(size_t first, size_t count, const double* block, size_t ld)>;

namespace detail_b200 {

struct SpinArgs {
  size_t n_ao = 0, n_spin = 0;
  std::vector<const double*> C, occ;
  std::vector<size_t> ldc, n_orb, n_occ;
};

inline SpinArgs spin_args(const Orbitals& orbitals, const Occupations& occupations,
                          const std::vector<size_t>& n_active) {
  SpinArgs a;
  a.n_spin = orbitals.size();
  if (a.n_spin < 1 || a.n_spin > 2 || occupations.size() != a.n_spin ||
      n_active.size() != a.n_spin)
    throw std::logic_error("invalid number of spin channels");
  a.n_ao = orbitals[0].n_rows();
  for (size_t s = 0; s < a.n_spin; ++s) {
    if (orbitals[s].n_rows() != a.n_ao)
      throw std::runtime_error("Inconsistent number of atomic orbitals");
    a.C.push_back(orbitals[s].memptr());
    a.ldc.push_back(a.n_ao);
    a.n_orb.push_back(orbitals[s].n_cols());
    a.occ.push_back(occupations[s].memptr());
    a.n_occ.push_back(occupations[s].n_elem());
  }
  return a;
}

// A GradientSink as a uw12c_block_sink; the first exception a sink throws is
// kept and rethrown once the library reports the failure.
struct SinkState {
  const GradientSink* fn = nullptr;
  std::exception_ptr error;
  static int call(void* user, size_t first, size_t count, const double* block, size_t ld,
                  void* /*stream*/) noexcept {
    auto* st = static_cast<SinkState*>(user);
    try {
      (*st->fn)(first, count, block, ld);
      return 0;
    } catch (...) {
      if (!st->error) st->error = std::current_exception();
      return 1;
    }
  }
};

}  // namespace detail_b200

/// Reverse mode of form_fock (uw12c_fock_backward): energy, terms and Fock
/// plus every gradient, in host memory; the direct terms only unless
/// indirect_term (then, with scale_same_spin != 0, the energy of uw12_energy).
inline BackwardResult fock_backward(const BaseIntegrals& W, const BaseIntegrals& V,
                                    const BaseIntegrals& WV, const ABSProjectors& abs_projectors,
                                    const Orbitals& orbitals, const Occupations& occupations,
                                    const std::vector<size_t>& n_active, double scale_opp_spin,
                                    double scale_same_spin, bool indirect_term = false) {
  const auto a = detail_b200::spin_args(orbitals, occupations, n_active);
  const BaseIntegrals* X[3] = {&W, &V, &WV};
  BackwardResult r;
  for (int i = 0; i < 3; ++i) {
    const size_t n = X[i]->get_number_ao(), m = X[i]->get_number_df();
    r.gradients.dX3.emplace_back(n * (n + 1) / 2, m);
    r.gradients.dX2.emplace_back(m, m);
    if (i < 2) r.gradients.dX3_ri.emplace_back(X[i]->get_number_ri() * n, m);
  }
  double* d3[3] = {r.gradients.dX3[0].memptr(), r.gradients.dX3[1].memptr(),
                   r.gradients.dX3[2].memptr()};
  double* d3ri[2] = {r.gradients.dX3_ri[0].memptr(), r.gradients.dX3_ri[1].memptr()};
  double* d2[3] = {r.gradients.dX2[0].memptr(), r.gradients.dX2[1].memptr(),
                   r.gradients.dX2[2].memptr()};
  linalg::Mat fock(a.n_ao, a.n_ao * a.n_spin);
  detail::check(uw12c_fock_backward(W.handle(), V.handle(), WV.handle(), abs_projectors.handle(),
                                    a.n_ao, a.n_spin, a.C.data(), a.ldc.data(), a.n_orb.data(),
                                    a.occ.data(), a.n_occ.data(), n_active.data(),
                                    indirect_term ? 1 : 0, scale_opp_spin, scale_same_spin,
                                    &r.fock_energy.energy, r.terms,
                                    fock.memptr(), UW12C_MEM_HOST, d3, d3ri, d2, UW12C_MEM_HOST));
  for (size_t s = 0; s < a.n_spin; ++s)
    r.fock_energy.fock.emplace_back(fock.memptr() + s * a.n_ao * a.n_ao, a.n_ao, a.n_ao);
  return r;
}

/// uw12c_fock_backward_blocks: the three-index gradients of W, V, WV and the RI
/// gradients of W, V (sinks[0..4]; an empty function skips that gradient)
/// delivered to the sinks in aux blocks, host memory; the metric gradients
/// are returned whole (gradients.dX3 and dX3_ri stay empty).
inline BackwardResult fock_backward_blocks(const BaseIntegrals& W, const BaseIntegrals& V,
                                           const BaseIntegrals& WV,
                                           const ABSProjectors& abs_projectors,
                                           const Orbitals& orbitals,
                                           const Occupations& occupations,
                                           const std::vector<size_t>& n_active,
                                           double scale_opp_spin, double scale_same_spin,
                                           const std::array<GradientSink, 5>& sinks,
                                           bool indirect_term = false) {
  const auto a = detail_b200::spin_args(orbitals, occupations, n_active);
  const BaseIntegrals* X[3] = {&W, &V, &WV};
  BackwardResult r;
  for (int i = 0; i < 3; ++i) {
    const size_t m = X[i]->get_number_df();
    r.gradients.dX2.emplace_back(m, m);
  }
  double* d2[3] = {r.gradients.dX2[0].memptr(), r.gradients.dX2[1].memptr(),
                   r.gradients.dX2[2].memptr()};
  detail_b200::SinkState st[5];
  uw12c_block_sink fn[5];
  void* users[5];
  for (int i = 0; i < 5; ++i) {
    st[i].fn = &sinks[i];
    fn[i] = sinks[i] ? &detail_b200::SinkState::call : nullptr;
    users[i] = &st[i];
  }
  linalg::Mat fock(a.n_ao, a.n_ao * a.n_spin);
  const int status = uw12c_fock_backward_blocks(
      W.handle(), V.handle(), WV.handle(), abs_projectors.handle(), a.n_ao, a.n_spin, a.C.data(),
      a.ldc.data(), a.n_orb.data(), a.occ.data(), a.n_occ.data(), n_active.data(),
      indirect_term ? 1 : 0, scale_opp_spin, scale_same_spin, &r.fock_energy.energy, r.terms,
      fock.memptr(),
      UW12C_MEM_HOST, fn, users, fn + 3, users + 3, UW12C_MEM_HOST, d2, UW12C_MEM_HOST);
  if (status != UW12C_OK) {
    for (auto& s : st)
      if (s.error) std::rethrow_exception(s.error);
    detail::check(status);
  }
  for (size_t s = 0; s < a.n_spin; ++s)
    r.fock_energy.fock.emplace_back(fock.memptr() + s * a.n_ao * a.n_ao, a.n_ao, a.n_ao);
  return r;
}

}  // namespace b200

}  // namespace uw12

#endif  // UW12_B200_LIBUW12_HPP
