// C++ use of the header-only containers (include/bclx_containers.hpp):
// reads A (the reference's binary CSR format) and B (int64 m, n; row-major
// floats) from <dir>, runs BCL::gemm's two forms through bclx, and writes
// C = A*A as <dir>/c.binary and C = A*B as <dir>/c.dense for the Python
// test to compare with the oracle; checks dot, the file constructor and the
// tile members, and writes A rebuilt tile by tile (assign_tile) as
// <dir>/e.binary.  `mmread` mode: the MatrixMarket reader alone (no GPU).
#include <bclx_containers.hpp>

#include <cstdio>
#include <cstdlib>
#include <cstring>
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

template <typename T>
static bool same(const bclx::CSR<T>& x, const bclx::CSR<T>& y) {
  return x.m == y.m && x.n == y.n && x.row_ptr == y.row_ptr && x.col_ind == y.col_ind &&
         std::memcmp(x.vals.data(), y.vals.data(), sizeof(T) * x.vals.size()) == 0 && x.vals.size() == y.vals.size();
}

int main(int argc, char** argv) {
  if (argc == 5 && std::string(argv[1]) == "mmread") {  // host only: the MatrixMarket reader
    try {
      if (std::string(argv[3]) == "f32")
        bclx::CSR<float>::read(argv[2]).write_binary(argv[4]);
      else
        bclx::CSR<int32_t>::read(argv[2]).write_binary(argv[4]);
    } catch (const std::exception& e) {
      std::fprintf(stderr, "error: %s\n", e.what());
      return 1;
    }
    return 0;
  }
  if (argc != 5) {
    std::fprintf(stderr, "usage: %s <dir> <tile_m> <tile_k> <tile_n> | mmread <in.mtx> <f32|i32> <out.binary>\n",
                 argv[0]);
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

    // the file constructor, dot, get_tile / arget_tile / assign_tile, tile_rank
    bclx::SPMatrix<float> Af(dir + "/a.binary", {tm, tk}), Bf(dir + "/a.binary", {tk, tn});
    bclx::SPMatrix<float> D = Af.dot(Bf);
    if (!same(D.get(), C.get())) throw std::runtime_error("dot differs from gemm");
    bclx::SPMatrix<float> E(a.m, a.n, {tm, tk});
    for (size_t i = 0; i < A.grid_shape()[0]; i++)
      for (size_t j = 0; j < A.grid_shape()[1]; j++) {
        if (A.tile_rank({i, j}) != 0) throw std::runtime_error("tile_rank");
        auto t = A.get_tile({i, j});
        if (!same(t, A.arget_tile({i, j}).get())) throw std::runtime_error("arget_tile differs from get_tile");
        if (t.m != A.tile_shape({i, j})[0] || t.nnz() != A.tile_nnz({i, j})) throw std::runtime_error("get_tile shape");
        E.assign_tile({i, j}, t);
      }
    E.get().write_binary(dir + "/e.binary");

    size_t bm = 0, bn = 0;
    auto b = read_dense(dir + "/b.dense", bm, bn);
    bclx::DMatrix<float> Bd(b, bm, bn, {tk, bn}), Cd(a.m, bn, {tm, bn});
    bclx::gemm(A, Bd, Cd);
    write_dense(dir + "/c.dense", Cd.get_matrix(), a.m, bn);
    bclx::DMatrix<float> Cd2(a.m, bn, {tm, bn});
    Cd2 = 2.5f;
    if (Cd2.get_tile({0, 0})[0] != 2.5f || Cd2.tile_rank({0, 0}) != 0) throw std::runtime_error("DMatrix fill");
    Cd2 = 0.0f;
    bclx::gemm(A, Bd, Cd2);
    const auto x = Cd.get_matrix(), y = Cd2.get_matrix();
    if (std::memcmp(x.data(), y.data(), sizeof(float) * x.size()) != 0) throw std::runtime_error("refilled DMatrix");
    std::printf("ok nnz=%zu\n", C.nnz());
  } catch (const std::exception& e) {
    std::fprintf(stderr, "error: %s\n", e.what());
    return 1;
  }
  return 0;
}
