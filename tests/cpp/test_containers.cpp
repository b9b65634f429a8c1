// C++ use of the header-only containers (include/bclx_containers.hpp):
// reads A (the reference's binary CSR format) and B (int64 m, n; row-major
// floats) from <dir>, runs BCL::gemm's two forms through bclx, and writes
// C = A*A as <dir>/c.binary and C = A*B as <dir>/c.dense for the Python
// test to compare with the oracle.
#include <bclx_containers.hpp>

#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

static std::vector<float> read_dense(const std::string& path, size_t& m, size_t& n) {
  FILE* f = std::fopen(path.c_str(), "rb");
  if (!f) throw std::runtime_error("cannot open " + path);
  int64_t hdr[2];
  if (std::fread(hdr, sizeof(int64_t), 2, f) != 2) throw std::runtime_error("short read");
  m = (size_t)hdr[0], n = (size_t)hdr[1];
  std::vector<float> v(m * n);
  if (std::fread(v.data(), sizeof(float), v.size(), f) != v.size()) throw std::runtime_error("short read");
  std::fclose(f);
  return v;
}

static void write_dense(const std::string& path, const std::vector<float>& v, size_t m, size_t n) {
  FILE* f = std::fopen(path.c_str(), "wb");
  const int64_t hdr[2] = {(int64_t)m, (int64_t)n};
  std::fwrite(hdr, sizeof(int64_t), 2, f);
  std::fwrite(v.data(), sizeof(float), v.size(), f);
  std::fclose(f);
}

int main(int argc, char** argv) {
  if (argc != 5) {
    std::fprintf(stderr, "usage: %s <dir> <tile_m> <tile_k> <tile_n>\n", argv[0]);
    return 2;
  }
  const std::string dir = argv[1];
  const size_t tm = std::strtoull(argv[2], nullptr, 10), tk = std::strtoull(argv[3], nullptr, 10),
               tn = std::strtoull(argv[4], nullptr, 10);
  try {
    auto a = bclx::CSR<float>::read_binary(dir + "/a.binary");
    bclx::SPMatrix<float> A(a, {tm, tk}), B(a, {tk, tn});
    bclx::SPMatrix<float> C(a.m, a.n, {tm, tn});
    bclx::gemm(A, B, C);
    size_t sum = 0;
    for (size_t i = 0; i < C.grid_shape()[0]; i++)
      for (size_t j = 0; j < C.grid_shape()[1]; j++) sum += C.tile_nnz({i, j});
    if (sum != C.nnz()) throw std::runtime_error("tile nnz do not add up");
    C.get().write_binary(dir + "/c.binary");

    size_t bm = 0, bn = 0;
    auto b = read_dense(dir + "/b.dense", bm, bn);
    bclx::DMatrix<float> Bd(b, bm, bn, {tk, bn}), Cd(a.m, bn, {tm, bn});
    bclx::gemm(A, Bd, Cd);
    write_dense(dir + "/c.dense", Cd.get_matrix(), a.m, bn);
    std::printf("ok nnz=%zu\n", C.nnz());
  } catch (const std::exception& e) {
    std::fprintf(stderr, "error: %s\n", e.what());
    return 1;
  }
  return 0;
}
