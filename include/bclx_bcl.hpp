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
// tile in place.  The values are those of the reference's CPU loop, bit for
// bit (same per-entry order of fused multiply-adds).  Errors are thrown as
// std::runtime_error.  Link with -lbclx -lcudart.
#pragma once

#include <bclx.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <type_traits>
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

// One bclx context per process (device 0, legacy default stream).
inline bclx_context_t context() {
  struct Holder {
    bclx_context_t h = nullptr;
    ~Holder() {
      if (h) bclx_context_destroy(h);
    }
  };
  static Holder holder;
  if (!holder.h) check(bclx_context_create(0, &holder.h), "bclx_context_create");
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

}  // namespace detail

// BCL::gemm(SPMatrix a, SPMatrix b, SPMatrix& c) on the GPU.
template <typename T, typename I>
void gemm(const SPMatrix<T, I>& a, const SPMatrix<T, I>& b, SPMatrix<T, I>& c) {
  using namespace detail;
  if (a.shape()[1] != b.shape()[0] || a.shape()[0] != c.shape()[0] || b.shape()[1] != c.shape()[1] ||
      a.tile_shape()[1] != b.tile_shape()[0] || c.tile_shape()[0] != a.tile_shape()[0] ||
      c.tile_shape()[1] != b.tile_shape()[1])
    throw std::runtime_error("BCL::bclx::gemm: mismatched shapes or tile grids");
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
