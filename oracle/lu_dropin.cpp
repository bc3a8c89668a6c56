// Test infrastructure: the reference's own il::LU
// (il/linear_algebra/dense/factorization/LU.h:79-120, compiled from the
// reference tree as it is) with its LAPACKE calls bound to the engine's
// libhfpx_lapacke.so instead of OpenBLAS -- the link-level drop-in of the
// engine's LU.  Built by `make -C oracle dropin` into oracle/_ref/.
//
//   lu_dropin in.bin out.bin
// in.bin: int64 n, int64 nrhs, then A (n x n) and B (n x nrhs), column-major
// doubles.  out.bin: int64 status (0, or the LU's singular "rank" + 1), then
// X (n x nrhs) from LU(A).solve(B).
#include <cstdint>
#include <cstdio>
#include <vector>

#include <il/linear_algebra/dense/factorization/LU.h>

int main(int argc, char** argv) {
  if (argc != 3) return 64;
  FILE* f = std::fopen(argv[1], "rb");
  if (!f) return 66;
  int64_t hdr[2] = {0, 0};
  if (std::fread(hdr, sizeof(int64_t), 2, f) != 2) return 65;
  const il::int_t n = hdr[0], nrhs = hdr[1];
  il::Array2D<double> A{n, n};
  il::Array2D<double> B{n, nrhs};
  std::vector<double> buf((size_t)(n * n + n * nrhs));
  if (std::fread(buf.data(), sizeof(double), buf.size(), f) != buf.size()) return 65;
  std::fclose(f);
  for (il::int_t j = 0; j < n; ++j)
    for (il::int_t i = 0; i < n; ++i) A(i, j) = buf[(size_t)(i + n * j)];
  for (il::int_t j = 0; j < nrhs; ++j)
    for (il::int_t i = 0; i < n; ++i) B(i, j) = buf[(size_t)(n * n + i + n * j)];
  il::Status status{};
  il::LU<il::Array2D<double>> lu(std::move(A), il::io, status);
  int64_t st = 0;
  std::vector<double> out((size_t)(n * nrhs), 0.0);
  if (!status.ok()) {
    st = 1 + status.toInteger("rank");
  } else {
    il::Array2D<double> X = lu.solve(B);
    for (il::int_t j = 0; j < nrhs; ++j)
      for (il::int_t i = 0; i < n; ++i) out[(size_t)(i + n * j)] = X(i, j);
  }
  FILE* g = std::fopen(argv[2], "wb");
  if (!g) return 73;
  std::fwrite(&st, sizeof(int64_t), 1, g);
  std::fwrite(out.data(), sizeof(double), out.size(), g);
  std::fclose(g);
  return 0;
}
