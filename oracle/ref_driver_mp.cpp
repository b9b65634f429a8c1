// The reference's own distributed BCL::gemm on several ranks.  TEST
// INFRASTRUCTURE: compiled against the unmodified reference headers with the
// multi-process MPI subset in ref_stubs_mp/ (the CBLAS stub from ref_stubs/),
// and started once per rank by oracle.py: run_ref_mp.  Every rank reads the
// inputs; the matrices are distributed over a pm x pn process grid
// (BlockCustom({tile}, {pm, pn}): tile (i, j) on rank (j % pn) + (i % pm) * pn,
// SPMatrix.hpp:230-237, DMatrix.hpp:75-90), so BCL::gemm
// (bcl/containers/algorithms/spgemm.hpp:153-242) fetches remote tiles,
// broadcasts tile pointers and meets at barriers as it does under MPI.
//
// usage (every rank the same arguments):
//   bcl_ref_mp spgemm <A.binary> <B.binary> <tm> <tk> <tn> <pm> <pn> <f32|i32> <out.binary|-> <warmup> <reps>
//   bcl_ref_mp spmm   <A.binary> <B.dense>  <tm> <tk> <tn> <pm> <pn> <out.dense|-> <warmup> <reps>
// Rank 0 gathers C (SPMatrix::get, or every DMatrix tile through get_tile),
// writes it in the formats of ref_driver.cpp, and prints one JSON line: the
// wall time of each repetition from a barrier before BCL::gemm to a barrier
// after it (the slowest rank's time).

#include <bcl/bcl.hpp>
#include <bcl/containers/SPMatrix.hpp>
#include <bcl/containers/DMatrix.hpp>

#include <chrono>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

static double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

static void print_times(const char* mode, const std::vector<double>& t, size_t nnz_out) {
  if (BCL::rank() != 0) return;
  printf("{\"mode\": \"%s\", \"ranks\": %zu, \"nnz_out\": %zu, \"times_s\": [", mode, (size_t)BCL::nprocs(), nnz_out);
  for (size_t i = 0; i < t.size(); i++) printf("%s%.6f", i ? ", " : "", t[i]);
  printf("]}\n");
  fflush(stdout);
}

template <typename T>
static int run_spgemm(const std::string& fa, const std::string& fb, size_t tm, size_t tk, size_t tn, size_t pm,
                      size_t pn, const std::string& out, int warmup, int reps) {
  BCL::SPMatrix<T, int> a(fa, BCL::BlockCustom({tm, tk}, {pm, pn}));
  BCL::SPMatrix<T, int> b(fb, BCL::BlockCustom({tk, tn}, {pm, pn}));
  BCL::SPMatrix<T, int> c({a.shape()[0], b.shape()[1]}, BCL::BlockCustom({tm, tn}, {pm, pn}));
  std::vector<double> times;
  for (int r = 0; r < warmup + reps; r++) {
    BCL::barrier();
    const double t0 = now_s();
    BCL::gemm(a, b, c);
    BCL::barrier();
    const double t1 = now_s();
    if (r >= warmup) times.push_back(t1 - t0);
  }
  if (out != "-" && BCL::rank() == 0) {
    auto cm = c.get();
    cm.write_Binary(out);
  }
  BCL::barrier();  // the tiles stay allocated until rank 0 has read them
  print_times("spgemm", times, c.nnz());
  return 0;
}

static bool read_dense(const std::string& fb, std::vector<float>& bd, int64_t& bm, int64_t& bn) {
  FILE* f = fopen(fb.c_str(), "rb");
  if (!f) return false;
  bool ok = fread(&bm, 8, 1, f) == 1 && fread(&bn, 8, 1, f) == 1;
  if (ok) {
    bd.resize((size_t)bm * bn);
    ok = fread(bd.data(), sizeof(float), bd.size(), f) == bd.size();
  }
  fclose(f);
  return ok;
}

// This rank's tiles of a DMatrix from the full row-major array (padded
// row-major tiles, DMatrix.hpp:151-173).
static void fill_local(BCL::DMatrix<float>& d, const std::vector<float>& full, int64_t n) {
  for (size_t i = 0; i < d.grid_shape()[0]; i++)
    for (size_t j = 0; j < d.grid_shape()[1]; j++) {
      auto p = d.tile_ptr({i, j});
      if (!p.is_local()) continue;
      float* t = p.local();
      auto ts = d.tile_shape({i, j});
      for (size_t r = 0; r < ts[0]; r++)
        for (size_t q = 0; q < ts[1]; q++)
          t[r * d.tile_shape()[1] + q] = full[(i * d.tile_shape()[0] + r) * n + j * d.tile_shape()[1] + q];
    }
}

static int run_spmm(const std::string& fa, const std::string& fb, size_t tm, size_t tk, size_t tn, size_t pm,
                    size_t pn, const std::string& out, int warmup, int reps) {
  BCL::SPMatrix<float, int> a(fa, BCL::BlockCustom({tm, tk}, {pm, pn}));
  std::vector<float> bd;
  int64_t bm, bn;
  if (!read_dense(fb, bd, bm, bn) || (size_t)bm != a.shape()[1]) {
    fprintf(stderr, "cannot read %s or shape mismatch\n", fb.c_str());
    return 2;
  }
  BCL::DMatrix<float> b({(size_t)bm, (size_t)bn}, BCL::BlockCustom({tk, tn}, {pm, pn}));
  BCL::DMatrix<float> c({a.shape()[0], (size_t)bn}, BCL::BlockCustom({tm, tn}, {pm, pn}));
  fill_local(b, bd, bn);
  std::vector<double> times;
  for (int r = 0; r < warmup + reps; r++) {
    c = 0.0f;
    BCL::barrier();
    const double t0 = now_s();
    BCL::gemm(a, b, c);
    BCL::barrier();
    const double t1 = now_s();
    if (r >= warmup) times.push_back(t1 - t0);
  }
  if (out != "-" && BCL::rank() == 0) {
    const int64_t m = (int64_t)a.shape()[0];
    std::vector<float> cd((size_t)m * bn);
    for (size_t i = 0; i < c.grid_shape()[0]; i++)
      for (size_t j = 0; j < c.grid_shape()[1]; j++) {
        const std::vector<float> t = c.get_tile({i, j});
        auto ts = c.tile_shape({i, j});
        for (size_t r = 0; r < ts[0]; r++)
          for (size_t q = 0; q < ts[1]; q++)
            cd[(i * c.tile_shape()[0] + r) * bn + j * c.tile_shape()[1] + q] = t[r * c.tile_shape()[1] + q];
      }
    FILE* g = fopen(out.c_str(), "wb");
    fwrite(&m, 8, 1, g);
    fwrite(&bn, 8, 1, g);
    fwrite(cd.data(), sizeof(float), cd.size(), g);
    fclose(g);
  }
  BCL::barrier();
  print_times("spmm", times, 0);
  return 0;
}

int main(int argc, char** argv) {
  if (argc < 2) {
    fprintf(stderr, "usage: see ref_driver_mp.cpp\n");
    return 2;
  }
  const std::string mode = argv[1];
  auto z = [&](int i) { return (size_t)strtoull(argv[i], nullptr, 10); };
  BCL::init(4096);
  int rc = 2;
  if (mode == "spgemm" && argc == 13) {
    const std::string vt = argv[9];
    rc = vt == "f32" ? run_spgemm<float>(argv[2], argv[3], z(4), z(5), z(6), z(7), z(8), argv[10], atoi(argv[11]),
                                         atoi(argv[12]))
                     : run_spgemm<int>(argv[2], argv[3], z(4), z(5), z(6), z(7), z(8), argv[10], atoi(argv[11]),
                                       atoi(argv[12]));
  } else if (mode == "spmm" && argc == 12) {
    rc = run_spmm(argv[2], argv[3], z(4), z(5), z(6), z(7), z(8), argv[9], atoi(argv[10]), atoi(argv[11]));
  } else {
    fprintf(stderr, "bad arguments for mode %s\n", mode.c_str());
  }
  BCL::finalize();
  return rc;
}
