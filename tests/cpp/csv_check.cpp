// Loads one CSV file with uw12::linalg::load_csv and prints its shape and every
// element in column-major order (checked against numpy by tests), or the
// error message with exit status 1.
#include <libuw12.hpp>

#include <cstdio>

int main(int argc, char** argv) {
  if (argc < 2) return 2;
  try {
    const auto m = uw12::linalg::load_csv(argv[1]);
    std::printf("%zu %zu\n", m.n_rows(), m.n_cols());
    for (size_t k = 0; k < m.n_elem(); ++k) std::printf("%.17e\n", m[k]);
    return 0;
  } catch (const std::exception& e) {
    std::printf("%s\n", e.what());
    return 1;
  }
}
