// fixture_regression.cpp -- libuw12's regression run on a CSV fixture directory,
// through the C++ drop-in header (include/libuw12.hpp) and the B200 library.
//
// Usage:  fixture_regression <data_dir> <suffix> <n_spin> [tolerance]
//
// <data_dir> holds libuw12's test_data layout (tests/test_data.hpp:100-140,
// example/example.cpp): W2.csv, W3.csv, W3_ri.csv, V2.csv, V3.csv, V3_ri.csv,
// WV2.csv, WV3.csv, S.csv; orbitals.csv and occ.csv (n_spin = 1) or the
// _alpha / _beta pairs (n_spin = 2); n_active_<suffix>.csv; and, optionally,
// energy_<suffix>.csv and fock.csv (fock_alpha.csv / fock_beta.csv) with the
// expected results.  The run is the one of tests/test_water.cpp:11-67:
// form_fock with the indirect term and the Fock matrix, scale factors (1, 0.5).
// The energy must agree within tolerance * max(1, |E|) and every Fock element
// within 10 * tolerance * max(1, max|F|) (default tolerance 1e-8).
//
// Exit status: 0 results agree (or no expected results were given), 1 they
// differ, 2 bad arguments or unreadable data.
#include <libuw12.hpp>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

namespace {

using uw12::linalg::Mat;
using uw12::linalg::Vec;

bool exists(const std::string& path) { return std::ifstream(path).good(); }

uw12::BaseIntegrals load_integrals(const std::string& dir, const std::string& prefix, bool ri) {
  const Mat X3 = uw12::linalg::load_csv(dir + prefix + "3.csv");
  const Mat X2 = uw12::linalg::load_csv(dir + prefix + "2.csv");
  if (!ri) return uw12::BaseIntegrals(X3, X2);
  const Mat X3_ri = uw12::linalg::load_csv(dir + prefix + "3_ri.csv");
  return uw12::BaseIntegrals(X3, X2, X3_ri);
}

// libuw12's per-spin file naming (tests/test_data.hpp:22-43)
std::vector<Mat> load_spin(const std::string& dir, const std::string& name, size_t n_spin) {
  if (n_spin == 1) return {uw12::linalg::load_csv(dir + name + ".csv")};
  return {uw12::linalg::load_csv(dir + name + "_alpha.csv"),
          uw12::linalg::load_csv(dir + name + "_beta.csv")};
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 4) {
    std::fprintf(stderr, "usage: %s <data_dir> <suffix> <n_spin> [tolerance]\n", argv[0]);
    return 2;
  }
  std::string dir = argv[1];
  if (!dir.empty() && dir.back() != '/') dir += '/';
  const std::string suffix = argv[2];
  const size_t n_spin = std::strtoul(argv[3], nullptr, 10);
  const double tol = argc > 4 ? std::strtod(argv[4], nullptr) : 1e-8;
  if (n_spin != 1 && n_spin != 2) {
    std::fprintf(stderr, "n_spin must be 1 or 2\n");
    return 2;
  }
  try {
    const auto W = load_integrals(dir, "W", true);
    const auto V = load_integrals(dir, "V", true);
    const auto WV = load_integrals(dir, "WV", false);
    const size_t n_ao = W.get_number_ao(), n_ri = W.get_number_ri();
    const Mat S = uw12::linalg::load_csv(dir + "S.csv");
    const auto abs_projectors = uw12::three_el::ri::calculate_abs_projectors(S, n_ao, n_ri);

    const uw12::Orbitals orbitals = load_spin(dir, "orbitals", n_spin);
    uw12::Occupations occ;
    for (const auto& m : load_spin(dir, "occ", n_spin)) occ.emplace_back(m.memptr(), m.n_elem());
    const Mat na = uw12::linalg::load_csv(dir + "n_active_" + suffix + ".csv");
    std::vector<size_t> n_active;
    for (size_t j = 0; j < na.n_cols(); ++j)
      for (size_t i = 0; i < na.n_rows(); ++i) n_active.push_back(static_cast<size_t>(na(i, j)));

    std::printf("n_ao %zu  n_df %zu  n_ri %zu  n_spin %zu\n", n_ao, W.get_number_df(), n_ri,
                n_spin);
    const auto result = uw12::form_fock(W, V, WV, abs_projectors, orbitals, occ, n_active, true,
                                        true, 1.0, 0.5);
    std::printf("energy %.17e\n", result.energy);

    int status = 0;
    const std::string e_path = dir + "energy_" + suffix + ".csv";
    if (exists(e_path)) {
      const double expected = uw12::linalg::load_csv(e_path)(0, 0);
      const double diff = std::abs(result.energy - expected);
      const bool ok = diff <= tol * std::max(1.0, std::abs(expected));
      std::printf("expected energy %.17e  |dE| %.3e  %s\n", expected, diff, ok ? "ok" : "FAIL");
      if (!ok) status = 1;
    }
    const std::string f_path = dir + (n_spin == 1 ? "fock.csv" : "fock_alpha.csv");
    if (exists(f_path)) {
      const auto expected = load_spin(dir, "fock", n_spin);
      for (size_t s = 0; s < n_spin; ++s) {
        double diff = 0.0, scale = 1.0;
        for (size_t j = 0; j < n_ao; ++j)
          for (size_t i = 0; i < n_ao; ++i) {
            diff = std::max(diff, std::abs(result.fock[s](i, j) - expected[s](i, j)));
            scale = std::max(scale, std::abs(expected[s](i, j)));
          }
        const bool ok = diff <= 10.0 * tol * scale;
        std::printf("spin %zu  max|dF| %.3e  %s\n", s, diff, ok ? "ok" : "FAIL");
        if (!ok) status = 1;
      }
    }
    return status;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "error: %s\n", e.what());
    return 2;
  }
}
