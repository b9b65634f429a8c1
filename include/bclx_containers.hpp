// Header-only C++ containers over the bclx C ABI, with the names and
// argument meaning of BCL's matrix API for the sparse tile multiply:
//
//   bclx::SPMatrix<T>   BCL::SPMatrix<T, int>  (bcl/containers/SPMatrix.hpp:35-616)
//   bclx::DMatrix<T>    BCL::DMatrix<T>        (bcl/containers/DMatrix.hpp:27-587)
//   bclx::BlockCustom   BCL::BlockCustom       (bcl/containers/detail/Blocking.hpp:215-245)
//   bclx::gemm(a, b, c) BCL::gemm overloads    (bcl/containers/algorithms/spgemm.hpp:153-242)
//   bclx::CSR<T>        BCL::CSRMatrix<T, int> host matrix and its binary file
//                       format (bcl/containers/sequential/CSRMatrix.hpp:489-530)
//
// Every tile lives on one GPU (the one-rank case of the reference): an
// SPMatrix packs all its CSR tiles into four device arrays plus a device
// array of bclx_csr_t descriptors, a DMatrix keeps padded row-major tiles in
// one allocation.  Errors are thrown as std::runtime_error, as the reference
// does.  Link with -lbclx -lcudart.
#pragma once

#include <bclx.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cstdint>
#include <cstdio>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

namespace bclx {

inline void check(int rc, const char* what) {
  if (rc != BCLX_OK) throw std::runtime_error(std::string(what) + ": " + bclx_last_error());
}
inline void check_cuda(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

template <typename T>
struct dtype_of;
template <>
struct dtype_of<float> {
  static constexpr int32_t value = BCLX_F32;
};
template <>
struct dtype_of<int32_t> {
  static constexpr int32_t value = BCLX_I32;
};

// One context per process and device, on the legacy default stream.
inline bclx_context_t context(int device = 0) {
  struct Holder {
    bclx_context_t h = nullptr;
    ~Holder() {
      if (h) bclx_context_destroy(h);
    }
  };
  static Holder holders[64];
  Holder& x = holders[device & 63];
  if (!x.h) check(bclx_context_create(device, &x.h), "bclx_context_create");
  return x.h;
}

// Device buffer (cudaMalloc / cudaFree).
template <typename T>
class DeviceArray {
 public:
  DeviceArray() = default;
  explicit DeviceArray(size_t n) { resize(n); }
  DeviceArray(const DeviceArray&) = delete;
  DeviceArray& operator=(const DeviceArray&) = delete;
  DeviceArray(DeviceArray&& o) noexcept : p_(o.p_), n_(o.n_) { o.p_ = nullptr, o.n_ = 0; }
  DeviceArray& operator=(DeviceArray&& o) noexcept {
    std::swap(p_, o.p_);
    std::swap(n_, o.n_);
    return *this;
  }
  ~DeviceArray() {
    if (p_) cudaFree(p_);
  }
  void resize(size_t n) {
    if (p_) cudaFree(p_);
    p_ = nullptr;
    n_ = n;
    check_cuda(cudaMalloc(reinterpret_cast<void**>(&p_), sizeof(T) * (n > 0 ? n : 1)), "cudaMalloc");
  }
  void upload(const T* src, size_t n) {
    if (n) check_cuda(cudaMemcpy(p_, src, sizeof(T) * n, cudaMemcpyHostToDevice), "cudaMemcpy H2D");
  }
  void download(T* dst, size_t n) const {
    if (n) check_cuda(cudaMemcpy(dst, p_, sizeof(T) * n, cudaMemcpyDeviceToHost), "cudaMemcpy D2H");
  }
  T* data() const { return p_; }
  size_t size() const { return n_; }

 private:
  T* p_ = nullptr;
  size_t n_ = 0;
};

// BCL::BlockCustom({tile_m, tile_n}, {1, 1}): the tile shape (one rank).
struct BlockCustom {
  size_t tile_m, tile_n;
};

// Host CSR matrix (CSRMatrix<T, int>), with the reference's binary format:
// size_t m, n, nnz; T vals[nnz]; int col_ind[nnz]; int row_ptr[m+1].
template <typename T>
struct CSR {
  size_t m = 0, n = 0;
  std::vector<int32_t> row_ptr{0};
  std::vector<int32_t> col_ind;
  std::vector<T> vals;
  size_t nnz() const { return col_ind.size(); }

  static CSR read_binary(const std::string& path) {
    CSR a;
    std::unique_ptr<FILE, int (*)(FILE*)> f(std::fopen(path.c_str(), "rb"), std::fclose);
    if (!f) throw std::runtime_error("cannot open " + path);
    size_t hdr[3];
    if (std::fread(hdr, sizeof(size_t), 3, f.get()) != 3) throw std::runtime_error("short read: " + path);
    a.m = hdr[0], a.n = hdr[1];
    a.vals.resize(hdr[2]);
    a.col_ind.resize(hdr[2]);
    a.row_ptr.resize(a.m + 1);
    if (std::fread(a.vals.data(), sizeof(T), hdr[2], f.get()) != hdr[2] ||
        std::fread(a.col_ind.data(), sizeof(int32_t), hdr[2], f.get()) != hdr[2] ||
        std::fread(a.row_ptr.data(), sizeof(int32_t), a.m + 1, f.get()) != a.m + 1)
      throw std::runtime_error("short read: " + path);
    return a;
  }
  void write_binary(const std::string& path) const {
    std::unique_ptr<FILE, int (*)(FILE*)> f(std::fopen(path.c_str(), "wb"), std::fclose);
    if (!f) throw std::runtime_error("cannot open " + path);
    const size_t hdr[3] = {m, n, nnz()};
    std::fwrite(hdr, sizeof(size_t), 3, f.get());
    std::fwrite(vals.data(), sizeof(T), nnz(), f.get());
    std::fwrite(col_ind.data(), sizeof(int32_t), nnz(), f.get());
    std::fwrite(row_ptr.data(), sizeof(int32_t), m + 1, f.get());
  }
};

inline size_t ceil_div(size_t a, size_t b) { return (a + b - 1) / b; }

// Distributed sparse matrix with every tile on this GPU.
template <typename T>
class SPMatrix {
 public:
  // An empty m x n matrix with this blocking (the output of gemm).
  SPMatrix(size_t m, size_t n, BlockCustom blk, int device = 0)
      : m_(m), n_(n), tm_(blk.tile_m), tn_(blk.tile_n), gm_(ceil_div(m, blk.tile_m)), gn_(ceil_div(n, blk.tile_n)),
        device_(device) {
    std::vector<int64_t> off(ntiles() + 1, 0);
    std::vector<int32_t> trp(ntiles() * (tm_ + 1), 0);
    set_packed(trp, off, {}, {});
  }

  // Tile a host CSR matrix (SPMatrix(filename, blocking) reads and
  // assign_tile's every tile, SPMatrix.hpp:277-357).
  SPMatrix(const CSR<T>& a, BlockCustom blk, int device = 0)
      : m_(a.m), n_(a.n), tm_(blk.tile_m), tn_(blk.tile_n), gm_(ceil_div(a.m, blk.tile_m)),
        gn_(ceil_div(a.n, blk.tile_n)), device_(device) {
    std::vector<std::vector<int32_t>> tcol(ntiles());
    std::vector<std::vector<T>> tval(ntiles());
    std::vector<int32_t> trp(ntiles() * (tm_ + 1), 0);
    for (size_t r = 0; r < m_; r++) {
      const size_t ti = r / tm_, lr = r - ti * tm_;
      for (int32_t p = a.row_ptr[r]; p < a.row_ptr[r + 1]; p++) {
        const size_t c = (size_t)a.col_ind[p], tj = c / tn_;
        const size_t t = ti * gn_ + tj;
        tcol[t].push_back((int32_t)(c - tj * tn_));
        tval[t].push_back(a.vals[p]);
        trp[t * (tm_ + 1) + lr + 1]++;
      }
    }
    std::vector<int64_t> off(ntiles() + 1, 0);
    std::vector<int32_t> col;
    std::vector<T> val;
    for (size_t t = 0; t < ntiles(); t++) {
      int32_t* rp = trp.data() + t * (tm_ + 1);
      for (size_t r = 0; r < tm_; r++) rp[r + 1] += rp[r];
      off[t + 1] = off[t] + (int64_t)tcol[t].size();
      col.insert(col.end(), tcol[t].begin(), tcol[t].end());
      val.insert(val.end(), tval[t].begin(), tval[t].end());
    }
    set_packed(trp, off, col, val);
  }

  std::array<size_t, 2> shape() const { return {m_, n_}; }
  std::array<size_t, 2> grid_shape() const { return {gm_, gn_}; }
  // SPMatrix::tile_shape(index) (SPMatrix.hpp:401-405): edge tiles are smaller.
  std::array<size_t, 2> tile_shape(std::array<size_t, 2> idx) const {
    return {std::min(tm_, m_ - idx[0] * tm_), std::min(tn_, n_ - idx[1] * tn_)};
  }
  std::array<size_t, 2> tile_shape() const { return {tm_, tn_}; }
  size_t tile_nnz(std::array<size_t, 2> idx) const {
    const size_t t = idx[0] * gn_ + idx[1];
    return (size_t)(off_[t + 1] - off_[t]);
  }
  size_t nnz() const { return (size_t)off_.back(); }

  // The whole matrix on the host (SPMatrix::get_matrix-like gather).
  CSR<T> get() const {
    std::vector<int32_t> trp(ntiles() * (tm_ + 1));
    std::vector<int32_t> col(nnz());
    std::vector<T> val(nnz());
    tile_row_ptr_.download(trp.data(), trp.size());
    col_.download(col.data(), col.size());
    vals_.download(val.data(), val.size());
    CSR<T> a;
    a.m = m_, a.n = n_;
    a.row_ptr.assign(m_ + 1, 0);
    for (size_t r = 0; r < m_; r++) {
      const size_t ti = r / tm_, lr = r - ti * tm_;
      for (size_t tj = 0; tj < gn_; tj++) {
        const size_t t = ti * gn_ + tj;
        const int32_t* rp = trp.data() + t * (tm_ + 1);
        for (int32_t p = rp[lr]; p < rp[lr + 1]; p++) {
          a.col_ind.push_back(col[off_[t] + p] + (int32_t)(tj * tn_));
          a.vals.push_back(val[off_[t] + p]);
        }
      }
      a.row_ptr[r + 1] = (int32_t)a.col_ind.size();
    }
    return a;
  }

  bclx_spgrid_t grid() const {
    bclx_spgrid_t g{};
    g.m = (int64_t)m_, g.n = (int64_t)n_, g.tile_m = (int64_t)tm_, g.tile_n = (int64_t)tn_;
    g.grid_m = (int64_t)gm_, g.grid_n = (int64_t)gn_;
    g.tiles = desc_.data();
    g.dtype = dtype_of<T>::value;
    return g;
  }
  int device() const { return device_; }

 private:
  template <typename U>
  friend void gemm(const SPMatrix<U>&, const SPMatrix<U>&, SPMatrix<U>&);

  size_t ntiles() const { return gm_ * gn_; }

  // Device arrays from packed host arrays, and the tile descriptors.
  void set_packed(const std::vector<int32_t>& trp, const std::vector<int64_t>& off, const std::vector<int32_t>& col,
                  const std::vector<T>& val) {
    check_cuda(cudaSetDevice(device_), "cudaSetDevice");
    off_ = off;
    tile_row_ptr_.resize(trp.size());
    tile_row_ptr_.upload(trp.data(), trp.size());
    tile_offset_.resize(off.size());
    tile_offset_.upload(off.data(), off.size());
    col_.resize(col.size());
    col_.upload(col.data(), col.size());
    vals_.resize(val.size());
    vals_.upload(val.data(), val.size());
    make_descriptors();
  }

  void make_descriptors() {
    std::vector<bclx_csr_t> d(ntiles());
    for (size_t i = 0; i < gm_; i++)
      for (size_t j = 0; j < gn_; j++) {
        const size_t t = i * gn_ + j;
        const auto ts = tile_shape({i, j});
        d[t].m = (int64_t)ts[0], d[t].n = (int64_t)ts[1];
        d[t].nnz = off_[t + 1] - off_[t];
        d[t].row_ptr = tile_row_ptr_.data() + t * (tm_ + 1);
        d[t].col_ind = col_.data() + off_[t];
        d[t].vals = vals_.data() + off_[t];
        d[t].dtype = dtype_of<T>::value;
      }
    desc_.resize(d.size());
    desc_.upload(d.data(), d.size());
  }

  size_t m_, n_, tm_, tn_, gm_, gn_;
  int device_;
  std::vector<int64_t> off_;  // host copy of tile_offset
  DeviceArray<int32_t> tile_row_ptr_;
  DeviceArray<int64_t> tile_offset_;
  DeviceArray<int32_t> col_;
  DeviceArray<T> vals_;
  DeviceArray<bclx_csr_t> desc_;
};

// Distributed dense matrix with every tile on this GPU: grid_m*grid_n tiles
// of tile_m x tile_n, row-major, padded to full size at the edges.
template <typename T>
class DMatrix {
 public:
  DMatrix(size_t m, size_t n, BlockCustom blk, int device = 0)
      : m_(m), n_(n), tm_(blk.tile_m), tn_(blk.tile_n), gm_(ceil_div(m, blk.tile_m)), gn_(ceil_div(n, blk.tile_n)),
        device_(device) {
    check_cuda(cudaSetDevice(device_), "cudaSetDevice");
    tiles_.resize(gm_ * gn_ * tm_ * tn_);
    check_cuda(cudaMemset(tiles_.data(), 0, sizeof(T) * tiles_.size()), "cudaMemset");
    std::vector<void*> p(gm_ * gn_);
    for (size_t t = 0; t < p.size(); t++) p[t] = tiles_.data() + t * tm_ * tn_;
    ptrs_.resize(p.size());
    ptrs_.upload(p.data(), p.size());
  }
  // From a host row-major m x n array.
  DMatrix(const std::vector<T>& full, size_t m, size_t n, BlockCustom blk, int device = 0) : DMatrix(m, n, blk, device) {
    set_matrix(full);
  }
  void set_matrix(const std::vector<T>& full) {
    std::vector<T> h(tiles_.size(), T(0));
    for (size_t r = 0; r < m_; r++)
      for (size_t c = 0; c < n_; c++) {
        const size_t ti = r / tm_, tj = c / tn_;
        h[((ti * gn_ + tj) * tm_ + (r - ti * tm_)) * tn_ + (c - tj * tn_)] = full[r * n_ + c];
      }
    tiles_.upload(h.data(), h.size());
  }
  // DMatrix::get_matrix (DMatrix.hpp:531-560): the whole matrix, row-major.
  std::vector<T> get_matrix() const {
    std::vector<T> h(tiles_.size());
    tiles_.download(h.data(), h.size());
    std::vector<T> full(m_ * n_);
    for (size_t r = 0; r < m_; r++)
      for (size_t c = 0; c < n_; c++) {
        const size_t ti = r / tm_, tj = c / tn_;
        full[r * n_ + c] = h[((ti * gn_ + tj) * tm_ + (r - ti * tm_)) * tn_ + (c - tj * tn_)];
      }
    return full;
  }
  std::array<size_t, 2> shape() const { return {m_, n_}; }
  std::array<size_t, 2> grid_shape() const { return {gm_, gn_}; }
  std::array<size_t, 2> tile_shape() const { return {tm_, tn_}; }
  bclx_dgrid_t grid(int32_t dtype) const {
    bclx_dgrid_t g{};
    g.m = (int64_t)m_, g.n = (int64_t)n_, g.tile_m = (int64_t)tm_, g.tile_n = (int64_t)tn_;
    g.grid_m = (int64_t)gm_, g.grid_n = (int64_t)gn_;
    g.tiles = ptrs_.data();
    g.dtype = dtype;
    return g;
  }
  int device() const { return device_; }

 private:
  size_t m_, n_, tm_, tn_, gm_, gn_;
  int device_;
  DeviceArray<T> tiles_;
  DeviceArray<void*> ptrs_;
};

// BCL::gemm(SPMatrix a, SPMatrix b, SPMatrix& c) (spgemm.hpp:182-242):
// c = a * b over the tile grids, every C tile summing its stages in the
// reference's rotated order.  c must have a's tile height and b's tile width.
template <typename T>
void gemm(const SPMatrix<T>& a, const SPMatrix<T>& b, SPMatrix<T>& c) {
  if (a.n_ != b.m_ || a.m_ != c.m_ || b.n_ != c.n_ || a.tn_ != b.tm_ || c.tm_ != a.tm_ || c.tn_ != b.tn_)
    throw std::runtime_error("BCL::gemm: mismatched shapes or tile grids");
  bclx_context_t ctx = context(a.device());
  const bclx_spgrid_t ga = a.grid(), gb = b.grid();
  bclx_spgrid_out_t out{};
  out.m = (int64_t)c.m_, out.n = (int64_t)c.n_, out.tile_m = (int64_t)c.tm_, out.tile_n = (int64_t)c.tn_;
  out.grid_m = (int64_t)c.gm_, out.grid_n = (int64_t)c.gn_;
  out.dtype = dtype_of<T>::value;
  out.tile_row_ptr = c.tile_row_ptr_.data();
  out.tile_offset = c.tile_offset_.data();
  bclx_spgemm_plan_t plan = nullptr;
  int64_t nnz = 0;
  check(bclx_spgemm_symbolic(ctx, &ga, &gb, &out, &plan, &nnz), "bclx_spgemm_symbolic");
  c.col_.resize((size_t)nnz);
  c.vals_.resize((size_t)nnz);
  out.col_ind = c.col_.data();
  out.vals = c.vals_.data();
  const int rc = bclx_spgemm_numeric(ctx, plan, &ga, &gb, &out, 0, 0);
  bclx_spgemm_plan_destroy(plan);
  check(rc, "bclx_spgemm_numeric");
  check(bclx_context_synchronize(ctx), "bclx_context_synchronize");
  c.off_.assign(c.ntiles() + 1, 0);
  c.tile_offset_.download(c.off_.data(), c.off_.size());
  c.make_descriptors();
}

// BCL::gemm(SPMatrix a, DMatrix b, DMatrix& c) (spgemm.hpp:153-179):
// c += a * b in place over the tile grids (FP32 a; b and c FP32, or BF16
// storage through the C ABI's BCLX_BF16).
template <typename T>
void gemm(const SPMatrix<float>& a, const DMatrix<T>& b, DMatrix<T>& c) {
  static_assert(std::is_same<T, float>::value, "the container SpMM here is FP32; BF16 goes through bclx_spmm_grid");
  if (a.shape()[1] != b.shape()[0] || a.shape()[0] != c.shape()[0] || b.shape()[1] != c.shape()[1])
    throw std::runtime_error("BCL::gemm: mismatched shapes");
  bclx_context_t ctx = context(a.device());
  const bclx_spgrid_t ga = a.grid();
  const bclx_dgrid_t gb = b.grid(BCLX_F32), gc = c.grid(BCLX_F32);
  check(bclx_spmm_grid(ctx, &ga, &gb, &gc), "bclx_spmm_grid");
  check(bclx_context_synchronize(ctx), "bclx_context_synchronize");
}

}  // namespace bclx
