// Drives the C++ drop-in header (include/libuw12.hpp) the way a libuw12 caller
// does (compare example/example.cpp of libuw12): raw-pointer setup calls,
// uw12_fock / uw12_energy, the callback BaseIntegrals constructor and the
// error behaviour.  Input and output are flat binary files written and read by
// tests/test_gpu_cpp_drop_in.py.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <iostream>
#include <stdexcept>
#include <vector>

#include "libuw12.hpp"

namespace {

std::vector<double> read_doubles(std::ifstream& f, size_t n) {
  std::vector<double> v(n);
  f.read(reinterpret_cast<char*>(v.data()), static_cast<std::streamsize>(n * sizeof(double)));
  if (!f) throw std::runtime_error("short input file");
  return v;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc != 3) {
    std::cerr << "usage: drop_in_check <input> <output>\n";
    return 2;
  }
  std::ifstream in(argv[1], std::ios::binary);
  int64_t hdr[9];
  in.read(reinterpret_cast<char*>(hdr), sizeof(hdr));
  const size_t n_ao = hdr[0], n_df = hdr[1], n_ri = hdr[2], n_spin = hdr[3], n_orb = hdr[4];
  const size_t n_occ_a = hdr[5], n_occ_b = hdr[6];
  const std::vector<size_t> n_active = n_spin == 1 ? std::vector<size_t>{size_t(hdr[7])}
                                                    : std::vector<size_t>{size_t(hdr[7]),
                                                                          size_t(hdr[8])};
  const size_t np = n_ao * (n_ao + 1) / 2;
  const auto W3 = read_doubles(in, np * n_df), W2 = read_doubles(in, n_df * n_df),
             W3r = read_doubles(in, n_ri * n_ao * n_df);
  const auto V3 = read_doubles(in, np * n_df), V2 = read_doubles(in, n_df * n_df),
             V3r = read_doubles(in, n_ri * n_ao * n_df);
  const auto WV3 = read_doubles(in, np * n_df), WV2 = read_doubles(in, n_df * n_df);
  const auto S = read_doubles(in, (n_ao + n_ri) * (n_ao + n_ri));
  const auto C = read_doubles(in, n_ao * n_orb * n_spin);
  const auto occ = read_doubles(in, n_occ_a + n_occ_b);
  const auto scales = read_doubles(in, 2);

  // libuw12's public API, raw pointers in (libuw12.hpp:42-169)
  const auto W = uw12::setup_base_integrals(W3.data(), W2.data(), W3r.data(), n_ao, n_df, n_ri);
  const auto V = uw12::setup_base_integrals(V3.data(), V2.data(), V3r.data(), n_ao, n_df, n_ri);
  const auto WV = uw12::setup_base_integrals(WV3.data(), WV2.data(), n_ao, n_df);
  const auto abs = uw12::setup_abs_projectors(S.data(), n_ao, n_ri);
  const auto orbitals = uw12::setup_orbitals(C.data(), n_ao, n_orb, n_spin);
  const auto occupations = n_spin == 1 ? uw12::setup_occupations(occ.data(), n_occ_a)
                                       : uw12::setup_occupations(occ.data(), n_occ_a, n_occ_b);
  std::vector<double> fock(n_ao * n_ao * n_spin);
  const double e_fock = uw12::uw12_fock(fock.data(), W, V, WV, abs, orbitals, occupations,
                                        n_active, scales[0], scales[1]);
  const double e_only = uw12::uw12_energy(W, V, WV, abs, orbitals, occupations, n_active,
                                          scales[0], scales[1]);

  // The callback constructor with df shells of sizes 1, 3, 5, 7, ...
  std::vector<size_t> shells, offsets;
  for (size_t off = 0, s = 1; off < n_df; s += 2) {
    const size_t w = std::min(s, n_df - off);
    shells.push_back(w);
    offsets.push_back(off);
    off += w;
  }
  const uw12::integrals::TwoIndexFn two = [&] { return uw12::linalg::Mat(W2.data(), n_df, n_df); };
  const uw12::integrals::ThreeIndexFn three = [&](size_t A) {
    return uw12::linalg::Mat(W3.data() + np * offsets[A], np, shells[A]);
  };
  const uw12::integrals::ThreeIndexFn three_ri = [&](size_t A) {
    return uw12::linalg::Mat(W3r.data() + n_ri * n_ao * offsets[A], n_ri * n_ao, shells[A]);
  };
  const uw12::BaseIntegrals W_cb(two, three, three_ri, shells, n_ao, n_df, n_ri);
  const double e_cb = uw12::uw12_energy(W_cb, V, WV, abs, orbitals, occupations, n_active,
                                        scales[0], scales[1]);

  // Integral-direct: nothing stored, the shells are produced at every use;
  // a 64 KiB budget splits every loop over aux functions into many blocks,
  // whose edges cut through shells
  const uw12::BaseIntegrals W_direct(two, three, three_ri, shells, n_ao, n_df, n_ri, false, false);
  const uw12::BaseIntegrals V_direct(uw12::linalg::Mat(V3.data(), np, n_df),
                                     uw12::linalg::Mat(V2.data(), n_df, n_df),
                                     [&](size_t A) {
                                       return uw12::linalg::Mat(V3r.data() + n_ri * n_ao * offsets[A],
                                                                n_ri * n_ao, shells[A]);
                                     },
                                     shells, true, n_ao, n_df, n_ri, false);
  uw12c_set_memory_budget(64 << 10);
  std::vector<double> fock_direct(n_ao * n_ao * n_spin);
  const double e_direct = uw12::uw12_fock(fock_direct.data(), W_direct, V_direct, WV, abs,
                                          orbitals, occupations, n_active, scales[0], scales[1]);
  uw12c_set_memory_budget(0);
  double fock_direct_diff = 0;
  for (size_t i = 0; i < fock.size(); ++i)
    fock_direct_diff = std::max(fock_direct_diff, std::abs(fock_direct[i] - fock[i]));

  // Error behaviour (libuw12.cpp:61-63, utils.hpp:235-253)
  double errors = 0;
  try {
    uw12::setup_orbitals(C.data(), n_ao, n_orb, 3);
  } catch (const std::runtime_error&) {
    errors += 1;
  }
  try {
    std::vector<size_t> too_many = n_active;
    too_many[0] = n_orb + 1;
    uw12::uw12_energy(W, V, WV, abs, orbitals, occupations, too_many, scales[0], scales[1]);
  } catch (const std::logic_error&) {
    errors += 1;
  }
  try {  // a shell of the wrong size, found while the stored tensor is produced
    const uw12::integrals::ThreeIndexFn bad = [&](size_t) { return uw12::linalg::Mat(np, 1); };
    const uw12::BaseIntegrals W_bad(two, bad, shells, n_ao, n_df);
  } catch (const std::logic_error&) {
    errors += 1;
  }
  try {  // the same shell, found at use in integral-direct mode
    const uw12::integrals::ThreeIndexFn bad = [&](size_t) { return uw12::linalg::Mat(np, 1); };
    const uw12::BaseIntegrals W_bad(two, bad, three_ri, shells, n_ao, n_df, n_ri, false, true);
    uw12::uw12_energy(W_bad, V, WV, abs, orbitals, occupations, n_active, scales[0], scales[1]);
  } catch (const std::runtime_error&) {
    errors += 1;
  }

  // B200 extensions: every gradient whole, then the three-index ones in blocks
  // (under a 64 KiB budget, so in many blocks), put together again
  const auto whole = uw12::b200::fock_backward(W, V, WV, abs, orbitals, occupations, n_active,
                                               scales[0], 0.0);
  std::vector<std::vector<double>> parts(5);
  std::array<uw12::b200::GradientSink, 5> sinks;
  for (int g = 0; g < 5; ++g)
    sinks[g] = [&parts, g](size_t first, size_t count, const double* block, size_t ld) {
      auto& v = parts[g];
      if (v.size() != first * ld) throw std::logic_error("blocks out of order");
      v.insert(v.end(), block, block + ld * count);
    };
  uw12c_set_memory_budget(64 << 10);
  const auto blocks = uw12::b200::fock_backward_blocks(W, V, WV, abs, orbitals, occupations,
                                                       n_active, scales[0], 0.0, sinks);
  uw12c_set_memory_budget(0);
  // relative differences (the blocked call's forward pass may run in orbital
  // chunks under the small budget, which changes rounding only)
  double grad_diff = std::abs(blocks.fock_energy.energy - whole.fock_energy.energy) /
                     std::max(1.0, std::abs(whole.fock_energy.energy));
  for (int g = 0; g < 5; ++g) {
    const auto& ref = g < 3 ? whole.gradients.dX3[g] : whole.gradients.dX3_ri[g - 3];
    double scale = 1e-300, diff = 0;
    if (parts[g].size() != ref.n_elem()) diff = 1.0;
    for (size_t e = 0; e < ref.n_elem() && e < parts[g].size(); ++e) {
      scale = std::max(scale, std::abs(ref[e]));
      diff = std::max(diff, std::abs(parts[g][e] - ref[e]));
    }
    grad_diff = std::max(grad_diff, diff / scale);
  }
  for (int g = 0; g < 3; ++g) {
    double scale = 1e-300, diff = 0;
    for (size_t e = 0; e < whole.gradients.dX2[g].n_elem(); ++e) {
      scale = std::max(scale, std::abs(whole.gradients.dX2[g][e]));
      diff = std::max(diff, std::abs(blocks.gradients.dX2[g][e] - whole.gradients.dX2[g][e]));
    }
    grad_diff = std::max(grad_diff, diff / scale);
  }
  try {  // a sink that throws: its exception reaches the caller
    std::array<uw12::b200::GradientSink, 5> bad;
    bad[4] = [](size_t, size_t, const double*, size_t) { throw std::logic_error("sink full"); };
    uw12::b200::fock_backward_blocks(W, V, WV, abs, orbitals, occupations, n_active, scales[0],
                                     0.0, bad);
  } catch (const std::logic_error&) {
    errors += 1;
  }

  std::ofstream out(argv[2], std::ios::binary);
  const double head[7] = {e_fock, e_only, e_cb, errors, e_direct, fock_direct_diff, grad_diff};
  out.write(reinterpret_cast<const char*>(head), sizeof(head));
  out.write(reinterpret_cast<const char*>(fock.data()),
            static_cast<std::streamsize>(fock.size() * sizeof(double)));
  std::printf("drop_in_check: E=%.15e (energy-only %.15e, callback integrals %.15e, "
              "integral-direct %.15e)\n", e_fock, e_only, e_cb, e_direct);
  return 0;
}
