// The reference's own containers through include/bclx_bcl.hpp.  TEST
// INFRASTRUCTURE: compiled against the unmodified reference headers (with the
// single-rank MPI/CBLAS stubs in ref_stubs/) and the bclx library.  On the
// same BCL::SPMatrix / BCL::DMatrix objects it runs the reference's
// BCL::gemm (bcl/containers/algorithms/spgemm.hpp:153-242) on the host and
// BCL::bclx::gemm on the GPU, and compares every output tile bit for bit.
//
// usage: bcl_glue_check <A.binary> <tm> <tk> <tn> <f32|i32> <N> [<pm> <pn>]
//   C = A*A on (tm x tk) / (tk x tn) tiles; then (f32 only) C2 += A*B for a
//   seeded dense B with N columns on (tk x N) tiles.  Prints one JSON line;
//   exit status 0 when everything is identical.  With pm x pn ranks (built
//   as bcl_glue_check_mp over ref_stubs_mp/, one process per rank) the
//   matrices are distributed over that process grid, both products run as
//   distributed products, and rank 0 compares every tile through get_tile.
#include <bcl/bcl.hpp>
#include <bcl/containers/DMatrix.hpp>
#include <bcl/containers/SPMatrix.hpp>

#include <bclx_bcl.hpp>

#include <cstdio>
#include <cstring>
#include <random>
#include <string>
#include <vector>

template <typename T>
static bool same_tiles(const BCL::SPMatrix<T, int>& x, const BCL::SPMatrix<T, int>& y, size_t& tiles, size_t& nnz) {
  bool ok = x.grid_shape()[0] == y.grid_shape()[0] && x.grid_shape()[1] == y.grid_shape()[1];
  for (size_t i = 0; ok && i < x.grid_shape()[0]; i++)
    for (size_t j = 0; ok && j < x.grid_shape()[1]; j++) {
      auto a = x.get_tile({i, j});
      auto b = y.get_tile({i, j});
      ok = a.m_ == b.m_ && a.n_ == b.n_ && a.nnz_ == b.nnz_ && a.row_ptr_ == b.row_ptr_ && a.col_ind_ == b.col_ind_ &&
           a.vals_.size() == b.vals_.size() &&
           std::memcmp(a.vals_.data(), b.vals_.data(), sizeof(T) * a.vals_.size()) == 0;
      tiles++;
      nnz += a.nnz_;
    }
  return ok;
}

template <typename T>
static int run(const std::string& fa, size_t tm, size_t tk, size_t tn, size_t N, size_t pm, size_t pn) {
  BCL::SPMatrix<T, int> a(fa, BCL::BlockCustom({tm, tk}, {pm, pn}));
  BCL::SPMatrix<T, int> b(fa, BCL::BlockCustom({tk, tn}, {pm, pn}));
  BCL::SPMatrix<T, int> c_ref({a.shape()[0], b.shape()[1]}, BCL::BlockCustom({tm, tn}, {pm, pn}));
  BCL::SPMatrix<T, int> c_gpu({a.shape()[0], b.shape()[1]}, BCL::BlockCustom({tm, tn}, {pm, pn}));
  BCL::gemm(a, b, c_ref);
  BCL::bclx::gemm(a, b, c_gpu);
  size_t tiles = 0, nnz = 0;
  const bool sp_ok = BCL::rank() != 0 || same_tiles(c_ref, c_gpu, tiles, nnz);
  bool dn_ok = true;
  size_t dn_elems = 0;
  if (std::is_same<T, float>::value && N > 0) {
    BCL::SPMatrix<float, int> af(fa, BCL::BlockCustom({tm, tk}, {pm, pn}));
    BCL::DMatrix<float> bd({af.shape()[1], N}, BCL::BlockCustom({tk, N}, {pm, pn}));
    BCL::DMatrix<float> cr({af.shape()[0], N}, BCL::BlockCustom({tm, N}, {pm, pn}));
    BCL::DMatrix<float> cg({af.shape()[0], N}, BCL::BlockCustom({tm, N}, {pm, pn}));
    // every rank draws the whole sequence and fills the tiles it holds
    std::mt19937 rng(7);
    std::uniform_real_distribution<float> u(-1.0f, 1.0f);
    for (size_t i = 0; i < bd.grid_shape()[0]; i++) {
      auto p = bd.tile_ptr({i, 0});
      for (size_t e = 0; e < bd.tile_size(); e++) {
        const float v = u(rng);
        if (p.is_local()) p.local()[e] = v;
      }
    }
    for (size_t i = 0; i < cr.grid_shape()[0]; i++) {  // the same nonzero start in both C's
      auto x = cr.tile_ptr({i, 0});
      auto y = cg.tile_ptr({i, 0});
      for (size_t e = 0; e < cr.tile_size(); e++) {
        const float v = u(rng);
        if (x.is_local()) x.local()[e] = v;
        if (y.is_local()) y.local()[e] = v;
      }
    }
    BCL::barrier();
    BCL::gemm(af, bd, cr);
    BCL::bclx::gemm(af, bd, cg);
    BCL::barrier();
    if (BCL::rank() == 0)
      for (size_t i = 0; i < cr.grid_shape()[0]; i++) {
        const size_t rows = cr.tile_shape({i, 0})[0];
        const std::vector<float> x = cr.get_tile({i, 0});
        const std::vector<float> y = cg.get_tile({i, 0});
        dn_ok = dn_ok && std::memcmp(x.data(), y.data(), sizeof(float) * rows * N) == 0;
        dn_elems += rows * N;
      }
    BCL::barrier();  // rank 0 has read every tile
  }
  BCL::barrier();
  if (BCL::rank() == 0)
    printf("{\"spgemm_identical\": %s, \"tiles\": %zu, \"nnz\": %zu, \"spmm_identical\": %s, "
           "\"spmm_elems\": %zu, \"ranks\": %zu}\n",
           sp_ok ? "true" : "false", tiles, nnz, dn_ok ? "true" : "false", dn_elems, (size_t)BCL::nprocs());
  return sp_ok && dn_ok ? 0 : 1;
}

int main(int argc, char** argv) {
  if (argc != 7 && argc != 9) {
    fprintf(stderr, "usage: bcl_glue_check <A.binary> <tm> <tk> <tn> <f32|i32> <N> [<pm> <pn>]\n");
    return 2;
  }
  BCL::init(4096);
  const size_t tm = strtoull(argv[2], nullptr, 10), tk = strtoull(argv[3], nullptr, 10),
               tn = strtoull(argv[4], nullptr, 10), N = strtoull(argv[6], nullptr, 10);
  const size_t pm = argc == 9 ? strtoull(argv[7], nullptr, 10) : 1, pn = argc == 9 ? strtoull(argv[8], nullptr, 10) : 1;
  int rc;
  try {
    rc = std::string(argv[5]) == "f32" ? run<float>(argv[1], tm, tk, tn, N, pm, pn)
                                       : run<int>(argv[1], tm, tk, tn, 0, pm, pn);
  } catch (const std::exception& e) {
    fprintf(stderr, "error: %s\n", e.what());
    rc = 3;
  }
  BCL::finalize();
  return rc;
}
