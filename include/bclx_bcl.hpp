// The drop-in for BCL programs: include this header after the reference's
// own container headers (bcl/containers/SPMatrix.hpp, DMatrix.hpp) and call
// BCL::bclx::gemm where the program called BCL::gemm.  The arguments are the
// reference's own containers, unchanged:
//
//   BCL::bclx::gemm(SPMatrix a, SPMatrix b, SPMatrix& c)
//       replaces BCL::gemm(SPMatrix, SPMatrix, SPMatrix&)
//       (bcl/containers/algorithms/spgemm.hpp:182-242);
//   BCL::bclx::gemm(SPMatrix a, DMatrix b, DMatrix& c)
//       replaces BCL::gemm(SPMatrix, DMatrix, DMatrix&) (spgemm.hpp:153-179).
//
// On one rank (every tile local, the reference's BlockCustom({tm, tn},
// {1, 1}) layout) the tiles are read through their GlobalPtr handles
// (SPMatrix::vals_ / col_ind_ / row_ptr_, DMatrix::tile_ptr), copied to the
// GPU, multiplied by the bclx kernels (include/bclx.h) and written back: the
// sparse result through SPMatrix::assign_tile and rebroadcast_tiles, as the
// reference's loop ends (spgemm.hpp:233-241); the dense result into each C
// tile in place.
//
// On several ranks (one GPU per rank) every rank takes the C tiles it owns
// (c.tile_rank({i, j}) == BCL::rank(), as the reference's loop does),
// fetches the A tiles of their tile rows and the B tiles of their tile
// columns through the containers' own get_tile (one-sided reads, remote or
// local), and computes all its C tiles in one sub-grid call
// (bclx_spgemm_symbolic_sub / bclx_spmm_grid_sub), each tile with the stage
// order of its global position; the sparse result is then assigned between
// two barriers and the tile pointers rebroadcast, as in spgemm.hpp:227-241.
//
// The values are those of the reference's CPU loop, bit for bit (same
// per-entry order of fused multiply-adds).  Errors are thrown as
// std::runtime_error.  Link with -lbclx -lcudart.
#pragma once

#include <bclx.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

namespace BCL {
namespace bclx {

namespace detail {

inline void check(int rc, const char* what) {
  if (rc != BCLX_OK) throw std::runtime_error(std::string(what) + ": " + bclx_last_error());
}
inline void check_cuda(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

// One bclx context per process on the legacy default stream: rank r uses
// GPU r mod (number of GPUs), so the ranks of one node spread over its GPUs
// (one rank: GPU 0).
inline bclx_context_t context() {
  struct Holder {
    bclx_context_t h = nullptr;
    ~Holder() {
      if (h) bclx_context_destroy(h);
    }
  };
  static Holder holder;
  if (!holder.h) {
    int ndev = 0;
    check_cuda(cudaGetDeviceCount(&ndev), "cudaGetDeviceCount");
    const int dev = ndev > 0 ? (int)(BCL::rank() % (uint64_t)ndev) : 0;
    check(bclx_context_create(dev, &holder.h), "bclx_context_create");
  }
  return holder.h;
}

// Device buffer freed on scope exit.
struct Buffer {
  void* p = nullptr;
  explicit Buffer(size_t bytes) { check_cuda(cudaMalloc(&p, std::max<size_t>(bytes, 16)), "cudaMalloc"); }
  ~Buffer() {
    if (p) cudaFree(p);
  }
  Buffer(const Buffer&) = delete;
  Buffer& operator=(const Buffer&) = delete;
  template <typename U>
  U* as() const {
    return reinterpret_cast<U*>(p);
  }
};

template <typename T>
constexpr int32_t dtype() {
  static_assert(std::is_same<T, float>::value || std::is_same<T, int32_t>::value,
                "bclx tiles hold float or int32_t values");
  return std::is_same<T, float>::value ? BCLX_F32 : BCLX_I32;
}

// Every tile of a reference SPMatrix on the device: packed col_ind / vals,
// per-tile row pointers (the tile's own rows), and the descriptor array
// the kernels read.
template <typename T, typename I>
struct DeviceTiles {
  static_assert(std::is_same<I, int32_t>::value, "bclx tiles use int32 indices (the reference's default)");
  size_t ntiles, nnz = 0, rp_total = 0;
  Buffer col, val, rp, desc;
  bclx_spgrid_t grid{};

  static size_t count_nnz(const SPMatrix<T, I>& a) {
    size_t s = 0;
    for (size_t t = 0; t < a.grid_shape()[0] * a.grid_shape()[1]; t++) s += a.nnzs_[t];
    return s;
  }
  static size_t count_rp(const SPMatrix<T, I>& a) {
    size_t s = 0;
    for (size_t i = 0; i < a.grid_shape()[0]; i++)
      for (size_t j = 0; j < a.grid_shape()[1]; j++) s += a.tile_shape({i, j})[0] + 1;
    return s;
  }

  explicit DeviceTiles(const SPMatrix<T, I>& a)
      : ntiles(a.grid_shape()[0] * a.grid_shape()[1]),
        nnz(count_nnz(a)),
        rp_total(count_rp(a)),
        col(sizeof(I) * count_nnz(a)),
        val(sizeof(T) * count_nnz(a)),
        rp(sizeof(I) * count_rp(a)),
        desc(sizeof(bclx_csr_t) * a.grid_shape()[0] * a.grid_shape()[1]) {
    std::vector<bclx_csr_t> d(ntiles);
    size_t off = 0, roff = 0;
    for (size_t i = 0; i < a.grid_shape()[0]; i++)
      for (size_t j = 0; j < a.grid_shape()[1]; j++) {
        const size_t t = i * a.grid_shape()[1] + j;
        if (!a.vals_[t].is_local()) throw std::runtime_error("BCL::bclx::gemm: every tile must be local (one rank)");
        const size_t rows = a.tile_shape({i, j})[0], nz = a.nnzs_[t];
        check_cuda(cudaMemcpy(rp.as<I>() + roff, a.row_ptr_[t].local(), sizeof(I) * (rows + 1),
                              cudaMemcpyHostToDevice), "cudaMemcpy");
        if (nz) {
          check_cuda(cudaMemcpy(col.as<I>() + off, a.col_ind_[t].local(), sizeof(I) * nz, cudaMemcpyHostToDevice),
                     "cudaMemcpy");
          check_cuda(cudaMemcpy(val.as<T>() + off, a.vals_[t].local(), sizeof(T) * nz, cudaMemcpyHostToDevice),
                     "cudaMemcpy");
        }
        d[t] = bclx_csr_t{(int64_t)rows, (int64_t)a.tile_shape({i, j})[1], (int64_t)nz, rp.as<I>() + roff,
                          col.as<I>() + off, val.as<T>() + off, dtype<T>(), 0};
        off += nz;
        roff += rows + 1;
      }
    check_cuda(cudaMemcpy(desc.p, d.data(), sizeof(bclx_csr_t) * ntiles, cudaMemcpyHostToDevice), "cudaMemcpy");
    grid.m = (int64_t)a.shape()[0];
    grid.n = (int64_t)a.shape()[1];
    grid.tile_m = (int64_t)a.tile_shape()[0];
    grid.tile_n = (int64_t)a.tile_shape()[1];
    grid.grid_m = (int64_t)a.grid_shape()[0];
    grid.grid_n = (int64_t)a.grid_shape()[1];
    grid.tiles = desc.as<bclx_csr_t>();
    grid.dtype = dtype<T>();
  }
};

// Tiles (rows[x], cols[y]) of a reference SPMatrix, fetched through its
// get_tile (local or remote) and packed on the device as a compact grid:
// grid tile (x, y) is matrix tile (rows[x], cols[y]).  rows and cols are
// increasing, so only the last tile of each can be a ragged edge tile.
template <typename T, typename I>
struct FetchedTiles {
  static_assert(std::is_same<I, int32_t>::value, "bclx tiles use int32 indices (the reference's default)");
  Buffer col, val, rp, desc;
  bclx_spgrid_t grid{};

  template <typename Tiles>
  static size_t total(const Tiles& t, bool rows) {
    size_t s = 0;
    for (const auto& x : t) s += rows ? x.shape()[0] + 1 : x.nnz_;
    return s;
  }

  template <typename Tiles>
  FetchedTiles(const SPMatrix<T, I>& a, const std::vector<size_t>& rows, const std::vector<size_t>& cols,
               const Tiles& t)
      : col(sizeof(I) * total(t, false)),
        val(sizeof(T) * total(t, false)),
        rp(sizeof(I) * total(t, true)),
        desc(sizeof(bclx_csr_t) * rows.size() * cols.size()) {
    std::vector<bclx_csr_t> d(t.size());
    size_t off = 0, roff = 0;
    for (size_t q = 0; q < t.size(); q++) {
      const size_t m = t[q].shape()[0], nz = t[q].nnz_;
      check_cuda(cudaMemcpy(rp.as<I>() + roff, t[q].row_ptr_.data(), sizeof(I) * (m + 1), cudaMemcpyHostToDevice),
                 "cudaMemcpy");
      if (nz) {
        check_cuda(cudaMemcpy(col.as<I>() + off, t[q].col_ind_.data(), sizeof(I) * nz, cudaMemcpyHostToDevice),
                   "cudaMemcpy");
        check_cuda(cudaMemcpy(val.as<T>() + off, t[q].vals_.data(), sizeof(T) * nz, cudaMemcpyHostToDevice),
                   "cudaMemcpy");
      }
      d[q] = bclx_csr_t{(int64_t)m, (int64_t)t[q].shape()[1], (int64_t)nz, rp.as<I>() + roff, col.as<I>() + off,
                        val.as<T>() + off, dtype<T>(), 0};
      off += nz;
      roff += m + 1;
    }
    check_cuda(cudaMemcpy(desc.p, d.data(), sizeof(bclx_csr_t) * d.size(), cudaMemcpyHostToDevice), "cudaMemcpy");
    grid.m = grid.n = 0;
    for (size_t x : rows) grid.m += (int64_t)a.tile_shape({x, cols.empty() ? 0 : cols[0]})[0];
    for (size_t y : cols) grid.n += (int64_t)a.tile_shape({rows.empty() ? 0 : rows[0], y})[1];
    grid.tile_m = (int64_t)a.tile_shape()[0];
    grid.tile_n = (int64_t)a.tile_shape()[1];
    grid.grid_m = (int64_t)rows.size();
    grid.grid_n = (int64_t)cols.size();
    grid.tiles = desc.as<bclx_csr_t>();
    grid.dtype = dtype<T>();
  }
};

template <typename T, typename I>
auto fetch_tiles(const SPMatrix<T, I>& a, const std::vector<size_t>& rows, const std::vector<size_t>& cols) {
  std::vector<decltype(a.get_tile({0, 0}))> t;
  t.reserve(rows.size() * cols.size());
  for (size_t x : rows)
    for (size_t y : cols) t.push_back(a.get_tile({x, y}));
  return t;
}

inline std::vector<size_t> all_of(size_t n) {
  std::vector<size_t> v(n);
  for (size_t i = 0; i < n; i++) v[i] = i;
  return v;
}

// The C tiles this rank owns, as groups (tile rows, tile columns) whose
// Cartesian products cover them: one group under the reference's
// block-cyclic layouts, one group per tile otherwise.
template <typename C>
std::vector<std::pair<std::vector<size_t>, std::vector<size_t>>> owned_groups(const C& c) {
  std::vector<size_t> rows, cols;
  size_t owned = 0;
  for (size_t i = 0; i < c.grid_shape()[0]; i++)
    for (size_t j = 0; j < c.grid_shape()[1]; j++)
      if (c.tile_rank({i, j}) == BCL::rank()) {
        owned++;
        if (std::find(rows.begin(), rows.end(), i) == rows.end()) rows.push_back(i);
        if (std::find(cols.begin(), cols.end(), j) == cols.end()) cols.push_back(j);
      }
  std::sort(rows.begin(), rows.end());
  std::sort(cols.begin(), cols.end());
  std::vector<std::pair<std::vector<size_t>, std::vector<size_t>>> g;
  if (owned == 0) return g;
  if (owned == rows.size() * cols.size()) {
    g.emplace_back(rows, cols);
  } else {
    for (size_t i : rows)
      for (size_t j : cols)
        if (c.tile_rank({i, j}) == BCL::rank()) g.emplace_back(std::vector<size_t>{i}, std::vector<size_t>{j});
  }
  return g;
}

inline std::vector<int64_t> as_i64(const std::vector<size_t>& v) { return std::vector<int64_t>(v.begin(), v.end()); }

// The distributed SP x SP product: each rank's C tiles through one sub-grid
// call per owned group, then the reference's assign / rebroadcast phase.
template <typename T, typename I>
void gemm_ranks(const SPMatrix<T, I>& a, const SPMatrix<T, I>& b, SPMatrix<T, I>& c) {
  bclx_context_t ctx = context();
  const std::vector<size_t> ks = all_of(a.grid_shape()[1]);
  std::vector<std::pair<std::array<size_t, 2>, CSRMatrix<T, I>>> done;
  for (const auto& grp : owned_groups(c)) {
    const std::vector<size_t>& rows = grp.first;
    const std::vector<size_t>& cols = grp.second;
    const auto at = fetch_tiles(a, rows, ks);
    const auto bt = fetch_tiles(b, ks, cols);
    FetchedTiles<T, I> fa(a, rows, ks, at), fb(b, ks, cols, bt);
    const size_t gm = rows.size(), gn = cols.size(), tm = c.tile_shape()[0];
    Buffer trp(sizeof(int32_t) * gm * gn * (tm + 1)), toff(sizeof(int64_t) * (gm * gn + 1));
    bclx_spgrid_out_t out{};
    out.m = fa.grid.m, out.n = fb.grid.n;
    out.tile_m = (int64_t)tm, out.tile_n = (int64_t)c.tile_shape()[1];
    out.grid_m = (int64_t)gm, out.grid_n = (int64_t)gn;
    out.tile_row_ptr = trp.as<int32_t>();
    out.tile_offset = toff.as<int64_t>();
    out.dtype = dtype<T>();
    const std::vector<int64_t> r64 = as_i64(rows), c64 = as_i64(cols);
    bclx_spgemm_plan_t plan = nullptr;
    int64_t nnz = 0;
    check(bclx_spgemm_symbolic_sub(ctx, &fa.grid, &fb.grid, &out, r64.data(), c64.data(), &plan, &nnz),
          "bclx_spgemm_symbolic_sub");
    Buffer col(sizeof(I) * (size_t)nnz), val(sizeof(T) * (size_t)nnz);
    out.col_ind = col.as<int32_t>();
    out.vals = val.p;
    const int rc = bclx_spgemm_numeric(ctx, plan, &fa.grid, &fb.grid, &out, 0, 0);
    bclx_spgemm_plan_destroy(plan);
    check(rc, "bclx_spgemm_numeric");
    check(bclx_context_synchronize(ctx), "bclx_context_synchronize");
    std::vector<int64_t> offs(gm * gn + 1);
    std::vector<int32_t> rps(gm * gn * (tm + 1));
    check_cuda(cudaMemcpy(offs.data(), toff.p, sizeof(int64_t) * offs.size(), cudaMemcpyDeviceToHost), "cudaMemcpy");
    check_cuda(cudaMemcpy(rps.data(), trp.p, sizeof(int32_t) * rps.size(), cudaMemcpyDeviceToHost), "cudaMemcpy");
    for (size_t x = 0; x < gm; x++)
      for (size_t y = 0; y < gn; y++) {
        const size_t t = x * gn + y, rn = c.tile_shape({rows[x], cols[y]})[0];
        const size_t nz = (size_t)(offs[t + 1] - offs[t]);
        std::vector<T> v(nz);
        std::vector<I> ci(nz), rp(rps.begin() + t * (tm + 1), rps.begin() + t * (tm + 1) + rn + 1);
        if (nz) {
          check_cuda(cudaMemcpy(v.data(), val.as<T>() + offs[t], sizeof(T) * nz, cudaMemcpyDeviceToHost),
                     "cudaMemcpy");
          check_cuda(cudaMemcpy(ci.data(), col.as<I>() + offs[t], sizeof(I) * nz, cudaMemcpyDeviceToHost),
                     "cudaMemcpy");
        }
        done.emplace_back(std::array<size_t, 2>{rows[x], cols[y]},
                          CSRMatrix<T, I>(rn, c.tile_shape({rows[x], cols[y]})[1], nz, std::move(v), std::move(rp),
                                          std::move(ci)));
      }
  }
  BCL::barrier();  // every rank has read its operands before any tile of c is replaced
  for (auto& d : done) c.assign_tile({d.first[0], d.first[1]}, d.second);
  BCL::barrier();
  c.rebroadcast_tiles();
}

inline bclx_dgrid_t dgrid_of(int64_t m, int64_t n, int64_t tm, int64_t tn, int64_t gm, int64_t gn, const Buffer& ptrs) {
  bclx_dgrid_t g{};
  g.m = m, g.n = n, g.tile_m = tm, g.tile_n = tn, g.grid_m = gm, g.grid_n = gn;
  g.tiles = ptrs.as<void*>();
  g.dtype = BCLX_F32;
  return g;
}

// The distributed SP x dense product: each rank's C tiles (its own, local)
// through one sub-grid call per owned group, with A's tiles fetched through
// SPMatrix::get_tile and B's through DMatrix::get_tile; no barrier, as in
// spgemm.hpp:153-179.
template <typename I>
void spmm_ranks(const SPMatrix<float, I>& a, const DMatrix<float>& b, DMatrix<float>& c) {
  bclx_context_t ctx = context();
  const std::vector<size_t> ks = all_of(a.grid_shape()[1]);
  for (const auto& grp : owned_groups(c)) {
    const std::vector<size_t>& rows = grp.first;
    const std::vector<size_t>& cols = grp.second;
    const auto at = fetch_tiles(a, rows, ks);
    FetchedTiles<float, I> fa(a, rows, ks, at);
    const size_t bts = b.tile_size(), cts = c.tile_size(), nb = ks.size() * cols.size(), nc = rows.size() * cols.size();
    Buffer bd(sizeof(float) * nb * bts), bp(sizeof(void*) * nb), cd(sizeof(float) * nc * cts), cp(sizeof(void*) * nc);
    std::vector<void*> bptr, cptr;
    for (size_t k : ks)
      for (size_t j : cols) {
        const std::vector<float> t = b.get_tile({k, j});
        float* dst = bd.as<float>() + bptr.size() * bts;
        check_cuda(cudaMemcpy(dst, t.data(), sizeof(float) * bts, cudaMemcpyHostToDevice), "cudaMemcpy");
        bptr.push_back(dst);
      }
    for (size_t i : rows)
      for (size_t j : cols) {
        auto gp = c.tile_ptr({i, j});
        if (!gp.is_local()) throw std::runtime_error("BCL::bclx::gemm: an owned C tile is not local");
        float* dst = cd.as<float>() + cptr.size() * cts;
        check_cuda(cudaMemcpy(dst, gp.local(), sizeof(float) * cts, cudaMemcpyHostToDevice), "cudaMemcpy");
        cptr.push_back(dst);
      }
    check_cuda(cudaMemcpy(bp.p, bptr.data(), sizeof(void*) * nb, cudaMemcpyHostToDevice), "cudaMemcpy");
    check_cuda(cudaMemcpy(cp.p, cptr.data(), sizeof(void*) * nc, cudaMemcpyHostToDevice), "cudaMemcpy");
    int64_t n = 0, m = 0;
    for (size_t j : cols) n += (int64_t)c.tile_shape({rows[0], j})[1];
    for (size_t i : rows) m += (int64_t)c.tile_shape({i, cols[0]})[0];
    const bclx_dgrid_t gb = dgrid_of((int64_t)b.shape()[0], n, (int64_t)b.tile_shape()[0], (int64_t)b.tile_shape()[1],
                                     (int64_t)ks.size(), (int64_t)cols.size(), bp);
    const bclx_dgrid_t gc = dgrid_of(m, n, (int64_t)c.tile_shape()[0], (int64_t)c.tile_shape()[1],
                                     (int64_t)rows.size(), (int64_t)cols.size(), cp);
    const std::vector<int64_t> r64 = as_i64(rows), c64 = as_i64(cols);
    check(bclx_spmm_grid_sub(ctx, &fa.grid, &gb, &gc, r64.data(), c64.data()), "bclx_spmm_grid_sub");
    check(bclx_context_synchronize(ctx), "bclx_context_synchronize");
    for (size_t q = 0; q < nc; q++) {
      auto gp = c.tile_ptr({rows[q / cols.size()], cols[q % cols.size()]});
      check_cuda(cudaMemcpy(gp.local(), cptr[q], sizeof(float) * cts, cudaMemcpyDeviceToHost), "cudaMemcpy");
    }
  }
}

}  // namespace detail

// BCL::gemm(SPMatrix a, SPMatrix b, SPMatrix& c) on the GPU.
template <typename T, typename I>
void gemm(const SPMatrix<T, I>& a, const SPMatrix<T, I>& b, SPMatrix<T, I>& c) {
  using namespace detail;
  if (a.shape()[1] != b.shape()[0] || a.shape()[0] != c.shape()[0] || b.shape()[1] != c.shape()[1] ||
      a.tile_shape()[1] != b.tile_shape()[0] || c.tile_shape()[0] != a.tile_shape()[0] ||
      c.tile_shape()[1] != b.tile_shape()[1])
    throw std::runtime_error("BCL::bclx::gemm: mismatched shapes or tile grids");
  if (BCL::nprocs() > 1) {
    gemm_ranks(a, b, c);
    return;
  }
  bclx_context_t ctx = context();
  DeviceTiles<T, I> da(a), db(b);
  const size_t gm = c.grid_shape()[0], gn = c.grid_shape()[1], tm = c.tile_shape()[0];
  Buffer trp(sizeof(int32_t) * gm * gn * (tm + 1)), toff(sizeof(int64_t) * (gm * gn + 1));
  bclx_spgrid_out_t out{};
  out.m = (int64_t)c.shape()[0], out.n = (int64_t)c.shape()[1];
  out.tile_m = (int64_t)tm, out.tile_n = (int64_t)c.tile_shape()[1];
  out.grid_m = (int64_t)gm, out.grid_n = (int64_t)gn;
  out.tile_row_ptr = trp.as<int32_t>();
  out.tile_offset = toff.as<int64_t>();
  out.dtype = dtype<T>();
  bclx_spgemm_plan_t plan = nullptr;
  int64_t nnz = 0;
  check(bclx_spgemm_symbolic(ctx, &da.grid, &db.grid, &out, &plan, &nnz), "bclx_spgemm_symbolic");
  Buffer col(sizeof(I) * (size_t)nnz), val(sizeof(T) * (size_t)nnz);
  out.col_ind = col.as<int32_t>();
  out.vals = val.p;
  const int rc = bclx_spgemm_numeric(ctx, plan, &da.grid, &db.grid, &out, 0, 0);
  bclx_spgemm_plan_destroy(plan);
  check(rc, "bclx_spgemm_numeric");
  check(bclx_context_synchronize(ctx), "bclx_context_synchronize");
  std::vector<int64_t> offs(gm * gn + 1);
  std::vector<int32_t> rps(gm * gn * (tm + 1));
  check_cuda(cudaMemcpy(offs.data(), toff.p, sizeof(int64_t) * offs.size(), cudaMemcpyDeviceToHost), "cudaMemcpy");
  check_cuda(cudaMemcpy(rps.data(), trp.p, sizeof(int32_t) * rps.size(), cudaMemcpyDeviceToHost), "cudaMemcpy");
  for (size_t i = 0; i < gm; i++)
    for (size_t j = 0; j < gn; j++) {
      const size_t t = i * gn + j, rows = c.tile_shape({i, j})[0];
      const size_t nz = (size_t)(offs[t + 1] - offs[t]);
      std::vector<T> v(nz);
      std::vector<I> ci(nz), rp(rps.begin() + t * (tm + 1), rps.begin() + t * (tm + 1) + rows + 1);
      if (nz) {
        check_cuda(cudaMemcpy(v.data(), val.as<T>() + offs[t], sizeof(T) * nz, cudaMemcpyDeviceToHost), "cudaMemcpy");
        check_cuda(cudaMemcpy(ci.data(), col.as<I>() + offs[t], sizeof(I) * nz, cudaMemcpyDeviceToHost),
                   "cudaMemcpy");
      }
      CSRMatrix<T, I> tile(rows, c.tile_shape({i, j})[1], nz, std::move(v), std::move(rp), std::move(ci));
      c.assign_tile({i, j}, tile);
    }
  c.rebroadcast_tiles();
}

// BCL::gemm(SPMatrix a, DMatrix b, DMatrix& c) on the GPU: c += a * b, FP32.
template <typename I>
void gemm(const SPMatrix<float, I>& a, const DMatrix<float>& b, DMatrix<float>& c) {
  using namespace detail;
  if (a.grid_shape()[0] != c.grid_shape()[0] || b.grid_shape()[1] != c.grid_shape()[1] ||
      a.grid_shape()[1] != b.grid_shape()[0])
    throw std::runtime_error("BCL::bclx::gemm: mismatched tile grids");
  if (BCL::nprocs() > 1) {
    spmm_ranks(a, b, c);
    return;
  }
  bclx_context_t ctx = context();
  DeviceTiles<float, I> da(a);
  auto upload = [](const DMatrix<float>& d, Buffer& data, Buffer& ptrs) {
    const size_t nt = d.grid_shape()[0] * d.grid_shape()[1], ts = d.tile_size();
    std::vector<void*> p(nt);
    for (size_t i = 0; i < d.grid_shape()[0]; i++)
      for (size_t j = 0; j < d.grid_shape()[1]; j++) {
        const size_t t = i * d.grid_shape()[1] + j;
        auto gp = d.tile_ptr({i, j});
        if (!gp.is_local()) throw std::runtime_error("BCL::bclx::gemm: every tile must be local (one rank)");
        check_cuda(cudaMemcpy(data.as<float>() + t * ts, gp.local(), sizeof(float) * ts, cudaMemcpyHostToDevice),
                   "cudaMemcpy");
        p[t] = data.as<float>() + t * ts;
      }
    check_cuda(cudaMemcpy(ptrs.p, p.data(), sizeof(void*) * nt, cudaMemcpyHostToDevice), "cudaMemcpy");
  };
  auto dgrid = [](const DMatrix<float>& d, const Buffer& ptrs) {
    bclx_dgrid_t g{};
    g.m = (int64_t)d.shape()[0], g.n = (int64_t)d.shape()[1];
    g.tile_m = (int64_t)d.tile_shape()[0], g.tile_n = (int64_t)d.tile_shape()[1];
    g.grid_m = (int64_t)d.grid_shape()[0], g.grid_n = (int64_t)d.grid_shape()[1];
    g.tiles = ptrs.as<void*>();
    g.dtype = BCLX_F32;
    return g;
  };
  const size_t nb = b.grid_shape()[0] * b.grid_shape()[1], nc = c.grid_shape()[0] * c.grid_shape()[1];
  Buffer bd(sizeof(float) * nb * b.tile_size()), bp(sizeof(void*) * nb);
  Buffer cd(sizeof(float) * nc * c.tile_size()), cp(sizeof(void*) * nc);
  upload(b, bd, bp);
  upload(c, cd, cp);
  const bclx_dgrid_t gb = dgrid(b, bp), gc = dgrid(c, cp);
  check(bclx_spmm_grid(ctx, &da.grid, &gb, &gc), "bclx_spmm_grid");
  check(bclx_context_synchronize(ctx), "bclx_context_synchronize");
  for (size_t i = 0; i < c.grid_shape()[0]; i++)
    for (size_t j = 0; j < c.grid_shape()[1]; j++) {
      const size_t t = i * c.grid_shape()[1] + j;
      check_cuda(cudaMemcpy(c.tile_ptr({i, j}).local(), cd.as<float>() + t * c.tile_size(),
                            sizeof(float) * c.tile_size(), cudaMemcpyDeviceToHost),
                 "cudaMemcpy");
    }
}

}  // namespace bclx
}  // namespace BCL
