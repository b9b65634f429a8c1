// Driver around the reference's own CPU implementation of the sparse tile
// multiply.  TEST INFRASTRUCTURE: it is compiled against the unmodified
// reference headers (bcl/containers/SPMatrix.hpp, DMatrix.hpp and
// bcl/containers/algorithms/spgemm.hpp) with the single-rank MPI/CBLAS stubs
// in ref_stubs/, and is used to
//   * pin the C restatement in oracle.c (bit-for-bit on the same inputs),
//   * generate the golden fixtures under tests/golden/,
//   * time the reference CPU path beside the GPU numbers.
//
// Inputs/outputs use the reference's binary CSR format
// (bcl/containers/sequential/CSRMatrix.hpp:489-530: size_t m, n, nnz; T vals;
// I col_ind; I row_ptr) and a plain dense format (int64 m, n; T data[m*n],
// row-major).
//
// usage:
//   bcl_ref spgemm <A.binary> <B.binary> <tm> <tk> <tn> <f32|i32> <out.binary|-> <warmup> <reps>
//   bcl_ref spmm   <A.binary> <B.dense>  <tm> <tk> <tn> <out.dense|-> <warmup> <reps>
//   bcl_ref dot    <A.binary> <B.binary> <f32|i32> <out.binary>
//   bcl_ref accumulate <f32|i32> <out.binary> <P1.binary> [P2.binary ...]
//   bcl_ref mmread <in.mtx> <f32|i32> <out.binary>      (CSRMatrix(fname): MatrixMarket reader)
//   bcl_ref tiles  <A.binary> <tm> <tn> <f32|i32> <out> (SPMatrix(fname, BlockCustom) slicing:
//                  every tile's CSR, row-major over the grid, one binary record after another)
//   bcl_ref rowwise <plain|cached|batched> <A.binary> <B.dense> <tm> <tk> <tn> <out.dense>
//                  (rowwise_gemm / cached_rowwise_gemm / batched_rowwise_gemm, C = 0 first)
//   bcl_ref dsum   <B.dense> <tm> <tn>                 (DMatrix::sum; prints the FP32 bits)
//   bcl_ref binop  <plus|minus|multiplies|divides|min|max|second> <A.binary> <B.dense> <f32|i32> <out.binary>
//                  (SPMatrix::binary_op_inplace on a 1x1 grid: the reference's loop bounds
//                  read grid_shape()[i] / [j], which stays in range only for one tile; the
//                  tile goes to out.binary and SPMatrix::get() of the matrix to out.binary.get)
// Prints one JSON line with the per-rep wall times of BCL::gemm.

#include <bcl/bcl.hpp>
#include <bcl/containers/SPMatrix.hpp>
#include <bcl/containers/DMatrix.hpp>
#include <bcl/containers/algorithms/experimental_gemm.hpp>

#include <chrono>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

// Every tile of SPMatrix(fname, BlockCustom({tm, tn})), appended to `out` as
// binary CSR records in row-major grid order.
template <typename T>
static int run_tiles(const std::string& fa, size_t tm, size_t tn, const std::string& out) {
  BCL::SPMatrix<T, int> a(fa, BCL::BlockCustom({tm, tn}, {1, 1}));
  FILE* f = fopen(out.c_str(), "wb");
  if (!f) return 1;
  for (size_t i = 0; i < a.grid_shape()[0]; i++)
    for (size_t j = 0; j < a.grid_shape()[1]; j++) {
      auto t = a.get_tile({i, j});
      const size_t hdr[3] = {t.shape()[0], t.shape()[1], t.nnz_};
      fwrite(hdr, sizeof(size_t), 3, f);
      fwrite(t.vals_.data(), sizeof(T), t.nnz_, f);
      fwrite(t.col_ind_.data(), sizeof(int), t.nnz_, f);
      fwrite(t.row_ptr_.data(), sizeof(int), t.shape()[0] + 1, f);
    }
  fclose(f);
  return 0;
}

static double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

static void print_times(const char* mode, const std::vector<double>& t, size_t nnz_out) {
  printf("{\"mode\": \"%s\", \"nnz_out\": %zu, \"times_s\": [", mode, nnz_out);
  for (size_t i = 0; i < t.size(); i++) printf("%s%.6f", i ? ", " : "", t[i]);
  printf("]}\n");
  fflush(stdout);
}

template <typename T>
static int run_spgemm(const std::string& fa, const std::string& fb, size_t tm, size_t tk, size_t tn,
                      const std::string& out, int warmup, int reps) {
  BCL::SPMatrix<T, int> a(fa, BCL::BlockCustom({tm, tk}, {1, 1}));
  BCL::SPMatrix<T, int> b(fb, BCL::BlockCustom({tk, tn}, {1, 1}));
  BCL::SPMatrix<T, int> c({a.shape()[0], b.shape()[1]}, BCL::BlockCustom({tm, tn}, {1, 1}));
  std::vector<double> times;
  for (int r = 0; r < warmup + reps; r++) {
    double t0 = now_s();
    BCL::gemm(a, b, c);
    double t1 = now_s();
    if (r >= warmup) times.push_back(t1 - t0);
  }
  if (out != "-") {
    auto cm = c.get();
    cm.write_Binary(out);
  }
  print_times("spgemm", times, c.nnz());
  return 0;
}

static int run_spmm(const std::string& fa, const std::string& fb, size_t tm, size_t tk, size_t tn,
                    const std::string& out, int warmup, int reps) {
  BCL::SPMatrix<float, int> a(fa, BCL::BlockCustom({tm, tk}, {1, 1}));
  FILE* f = fopen(fb.c_str(), "rb");
  if (!f) { fprintf(stderr, "cannot open %s\n", fb.c_str()); return 2; }
  int64_t bm, bn;
  if (fread(&bm, 8, 1, f) != 1 || fread(&bn, 8, 1, f) != 1) { fclose(f); return 2; }
  std::vector<float> bd((size_t)bm * bn);
  if (fread(bd.data(), sizeof(float), bd.size(), f) != bd.size()) { fclose(f); return 2; }
  fclose(f);
  if ((size_t)bm != a.shape()[1]) { fprintf(stderr, "shape mismatch\n"); return 2; }

  BCL::DMatrix<float> b({(size_t)bm, (size_t)bn}, BCL::BlockCustom({tk, tn}, {1, 1}));
  BCL::DMatrix<float> c({a.shape()[0], (size_t)bn}, BCL::BlockCustom({tm, tn}, {1, 1}));
  // Fill the padded row-major tiles of B (DMatrix.hpp:151-173: ld = tile_shape()[1]).
  for (size_t i = 0; i < b.grid_shape()[0]; i++)
    for (size_t j = 0; j < b.grid_shape()[1]; j++) {
      float* t = b.tile_ptr({i, j}).local();
      auto ts = b.tile_shape({i, j});
      for (size_t r = 0; r < ts[0]; r++)
        for (size_t q = 0; q < ts[1]; q++)
          t[r * b.tile_shape()[1] + q] = bd[(i * b.tile_shape()[0] + r) * bn + j * b.tile_shape()[1] + q];
    }
  std::vector<double> times;
  for (int r = 0; r < warmup + reps; r++) {
    c = 0.0f;
    double t0 = now_s();
    BCL::gemm(a, b, c);
    double t1 = now_s();
    if (r >= warmup) times.push_back(t1 - t0);
  }
  if (out != "-") {
    std::vector<float> cd(a.shape()[0] * (size_t)bn);
    for (size_t i = 0; i < c.grid_shape()[0]; i++)
      for (size_t j = 0; j < c.grid_shape()[1]; j++) {
        float* t = c.tile_ptr({i, j}).local();
        auto ts = c.tile_shape({i, j});
        for (size_t r = 0; r < ts[0]; r++)
          for (size_t q = 0; q < ts[1]; q++)
            cd[(i * c.tile_shape()[0] + r) * bn + j * c.tile_shape()[1] + q] = t[r * c.tile_shape()[1] + q];
      }
    FILE* g = fopen(out.c_str(), "wb");
    int64_t m = a.shape()[0];
    fwrite(&m, 8, 1, g);
    fwrite(&bn, 8, 1, g);
    fwrite(cd.data(), sizeof(float), cd.size(), g);
    fclose(g);
  }
  print_times("spmm", times, 0);
  return 0;
}

// Dense file (int64 m, n; T data[m*n] row-major) into a DMatrix with the
// given blocking (padded row-major tiles, DMatrix.hpp:151-173).
template <typename T>
static bool read_dense(const std::string& fb, std::vector<T>& bd, int64_t& bm, int64_t& bn) {
  FILE* f = fopen(fb.c_str(), "rb");
  if (!f) return false;
  bool ok = fread(&bm, 8, 1, f) == 1 && fread(&bn, 8, 1, f) == 1;
  if (ok) {
    bd.resize((size_t)bm * bn);
    ok = fread(bd.data(), sizeof(T), bd.size(), f) == bd.size();
  }
  fclose(f);
  return ok;
}

template <typename T>
static void fill_dmatrix(BCL::DMatrix<T>& d, const std::vector<T>& full, int64_t n) {
  for (size_t i = 0; i < d.grid_shape()[0]; i++)
    for (size_t j = 0; j < d.grid_shape()[1]; j++) {
      T* t = d.tile_ptr({i, j}).local();
      auto ts = d.tile_shape({i, j});
      for (size_t r = 0; r < ts[0]; r++)
        for (size_t q = 0; q < ts[1]; q++)
          t[r * d.tile_shape()[1] + q] = full[(i * d.tile_shape()[0] + r) * n + j * d.tile_shape()[1] + q];
    }
}

template <typename T>
static void write_dmatrix(BCL::DMatrix<T>& c, const std::string& out) {
  const int64_t m = c.shape()[0], n = c.shape()[1];
  std::vector<T> cd((size_t)m * n);
  for (size_t i = 0; i < c.grid_shape()[0]; i++)
    for (size_t j = 0; j < c.grid_shape()[1]; j++) {
      T* t = c.tile_ptr({i, j}).local();
      auto ts = c.tile_shape({i, j});
      for (size_t r = 0; r < ts[0]; r++)
        for (size_t q = 0; q < ts[1]; q++)
          cd[(i * c.tile_shape()[0] + r) * n + j * c.tile_shape()[1] + q] = t[r * c.tile_shape()[1] + q];
    }
  FILE* g = fopen(out.c_str(), "wb");
  fwrite(&m, 8, 1, g);
  fwrite(&n, 8, 1, g);
  fwrite(cd.data(), sizeof(T), cd.size(), g);
  fclose(g);
}

static int run_rowwise(const std::string& variant, const std::string& fa, const std::string& fb, size_t tm,
                       size_t tk, size_t tn, const std::string& out) {
  BCL::SPMatrix<float, int> a(fa, BCL::BlockCustom({tm, tk}, {1, 1}));
  std::vector<float> bd;
  int64_t bm, bn;
  if (!read_dense(fb, bd, bm, bn) || (size_t)bm != a.shape()[1]) return 2;
  BCL::DMatrix<float> b({(size_t)bm, (size_t)bn}, BCL::BlockCustom({tk, tn}, {1, 1}));
  BCL::DMatrix<float> c({a.shape()[0], (size_t)bn}, BCL::BlockCustom({tm, tn}, {1, 1}));
  fill_dmatrix(b, bd, bn);
  c = 0.0f;
  double t0 = now_s();
  if (variant == "plain") BCL::rowwise_gemm(a, b, c);
  else if (variant == "cached") BCL::cached_rowwise_gemm(a, b, c, size_t(1) << 20);
  else BCL::batched_rowwise_gemm(a, b, c);
  double t1 = now_s();
  write_dmatrix(c, out);
  print_times("rowwise", {t1 - t0}, 0);
  return 0;
}

static int run_dsum(const std::string& fb, size_t tm, size_t tn) {
  std::vector<float> bd;
  int64_t bm, bn;
  if (!read_dense(fb, bd, bm, bn)) return 2;
  BCL::DMatrix<float> d({(size_t)bm, (size_t)bn}, BCL::BlockCustom({tm, tn}, {1, 1}));
  fill_dmatrix(d, bd, bn);
  const float s = d.sum();
  uint32_t bits;
  memcpy(&bits, &s, 4);
  printf("{\"mode\": \"dsum\", \"sum\": %.9g, \"bits\": %u}\n", (double)s, bits);
  return 0;
}

template <typename T, typename Fn>
static int run_binop_fn(const std::string& fa, const std::vector<T>& bd, int64_t bn, Fn&& fn,
                        const std::string& out) {
  BCL::CSRMatrix<T, int> host(fa);
  BCL::SPMatrix<T, int> a(fa, BCL::BlockCustom({host.m_, host.n_}, {1, 1}));
  BCL::DMatrix<T> b({host.m_, host.n_}, BCL::BlockCustom({host.m_, host.n_}, {1, 1}));
  fill_dmatrix(b, bd, bn);
  a.binary_op_inplace(b, fn);
  // the tile itself, and the whole matrix through SPMatrix::get (which adds
  // every value to 0 in its SparseHashAccumulator: -0 comes back as +0)
  a.get_tile({0, 0}).write_Binary(out);
  a.get().write_Binary(out + ".get");
  return 0;
}

template <typename T>
static int run_binop(const std::string& op, const std::string& fa, const std::string& fb, const std::string& out) {
  std::vector<T> bd;
  int64_t bm, bn;
  if (!read_dense(fb, bd, bm, bn)) return 2;
  if (op == "plus") return run_binop_fn<T>(fa, bd, bn, std::plus<T>{}, out);
  if (op == "minus") return run_binop_fn<T>(fa, bd, bn, std::minus<T>{}, out);
  if (op == "multiplies") return run_binop_fn<T>(fa, bd, bn, std::multiplies<T>{}, out);
  if (op == "divides") return run_binop_fn<T>(fa, bd, bn, std::divides<T>{}, out);
  if (op == "min") return run_binop_fn<T>(fa, bd, bn, [](T x, T y) { return std::min(x, y); }, out);
  if (op == "max") return run_binop_fn<T>(fa, bd, bn, [](T x, T y) { return std::max(x, y); }, out);
  if (op == "second") return run_binop_fn<T>(fa, bd, bn, [](T, T y) { return y; }, out);
  return 2;
}

template <typename T>
static int run_dot(const std::string& fa, const std::string& fb, const std::string& out) {
  BCL::CSRMatrix<T, int> a(fa);
  BCL::CSRMatrix<T, int> b(fb);
  double t0 = now_s();
  auto c = a.dot(b);
  double t1 = now_s();
  c.write_Binary(out);
  print_times("dot", {t1 - t0}, c.nnz_);
  return 0;
}

// SparseHashAccumulator (SparseHashAccumulator.hpp:86-183): push the partial
// tiles in the given order, then get_matrix.
template <typename T>
static int run_accumulate(int nparts, char** files, const std::string& out) {
  BCL::SparseHashAccumulator<T, int> acc;
  size_t m = 0, n = 0;
  for (int p = 0; p < nparts; p++) {
    BCL::CSRMatrix<T, int> part(files[p]);
    m = part.m_;
    n = part.n_;
    acc.accumulate(std::move(part));
  }
  double t0 = now_s();
  auto c = acc.get_matrix(m, n);
  double t1 = now_s();
  c.write_Binary(out);
  print_times("accumulate", {t1 - t0}, c.nnz_);
  return 0;
}

int main(int argc, char** argv) {
  if (argc < 2) { fprintf(stderr, "usage: see source header\n"); return 2; }
  std::string mode = argv[1];
  if (mode == "mmread" && argc == 5) {  // no segment needed
    std::string dt = argv[3];
    if (dt == "f32") {
      BCL::CSRMatrix<float, int> a(argv[2]);
      a.write_Binary(argv[4]);
    } else {
      BCL::CSRMatrix<int, int> a(argv[2]);
      a.write_Binary(argv[4]);
    }
    return 0;
  }
  // Segment for tiles and the intermediate partial products (bcl_allocator);
  // the stub maps it lazily, so only touched pages are committed.
  const char* seg = getenv("BCLX_REF_SEGMENT_MB");
  BCL::init(seg ? strtoull(seg, nullptr, 10) : 32768);
  int rc = 2;
  if (mode == "spgemm" && argc == 11) {
    std::string dt = argv[7];
    size_t tm = strtoull(argv[4], nullptr, 10), tk = strtoull(argv[5], nullptr, 10), tn = strtoull(argv[6], nullptr, 10);
    if (dt == "f32") rc = run_spgemm<float>(argv[2], argv[3], tm, tk, tn, argv[8], atoi(argv[9]), atoi(argv[10]));
    else rc = run_spgemm<int>(argv[2], argv[3], tm, tk, tn, argv[8], atoi(argv[9]), atoi(argv[10]));
  } else if (mode == "spmm" && argc == 10) {
    rc = run_spmm(argv[2], argv[3], strtoull(argv[4], nullptr, 10), strtoull(argv[5], nullptr, 10),
                  strtoull(argv[6], nullptr, 10), argv[7], atoi(argv[8]), atoi(argv[9]));
  } else if (mode == "dot" && argc == 6) {
    std::string dt = argv[4];
    rc = dt == "f32" ? run_dot<float>(argv[2], argv[3], argv[5]) : run_dot<int>(argv[2], argv[3], argv[5]);
  } else if (mode == "tiles" && argc == 7) {
    std::string dt = argv[5];
    size_t tm = strtoull(argv[3], nullptr, 10), tn = strtoull(argv[4], nullptr, 10);
    rc = dt == "f32" ? run_tiles<float>(argv[2], tm, tn, argv[6]) : run_tiles<int>(argv[2], tm, tn, argv[6]);
  } else if (mode == "rowwise" && argc == 9) {
    rc = run_rowwise(argv[2], argv[3], argv[4], strtoull(argv[5], nullptr, 10), strtoull(argv[6], nullptr, 10),
                     strtoull(argv[7], nullptr, 10), argv[8]);
  } else if (mode == "dsum" && argc == 5) {
    rc = run_dsum(argv[2], strtoull(argv[3], nullptr, 10), strtoull(argv[4], nullptr, 10));
  } else if (mode == "binop" && argc == 7) {
    std::string dt = argv[5];
    rc = dt == "f32" ? run_binop<float>(argv[2], argv[3], argv[4], argv[6])
                     : run_binop<int>(argv[2], argv[3], argv[4], argv[6]);
  } else if (mode == "accumulate" && argc >= 5) {
    std::string dt = argv[2];
    rc = dt == "f32" ? run_accumulate<float>(argc - 4, argv + 4, argv[3])
                     : run_accumulate<int>(argc - 4, argv + 4, argv[3]);
  } else {
    fprintf(stderr, "bad arguments\n");
  }
  BCL::finalize();
  return rc;
}
