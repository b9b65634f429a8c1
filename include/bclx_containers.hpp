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
// Members kept from the reference: SPMatrix(fname | CSR, blocking), shape,
// grid_shape, tile_shape, tile_nnz, nnz, tile_rank, get_tile, arget_tile,
// assign_tile, dot, get; DMatrix shape, grid_shape, tile_shape, tile_size,
// tile_rank, tile_ptr, get_tile, operator=(value), get_matrix.
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
#include <fstream>
#include <future>
#include <memory>
#include <sstream>
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
  // Coordinate MatrixMarket (matrix_io.hpp:218-356, CSRMatrix.hpp:370-410):
  // `general` or `symmetric` (an off-diagonal entry is also stored
  // transposed), `pattern` values 1; an index repeated later in the file is
  // ignored (the first one stays); entries sorted by (row, column).  Other
  // formats, indices out of range and more entries than announced throw.
  static CSR read_matrix_market(const std::string& path) {
    std::ifstream f(path);
    if (!f.is_open()) throw std::runtime_error("mmread: cannot open " + path);
    std::string buf, word[5];
    std::getline(f, buf);
    {
      std::istringstream ss(buf);
      for (auto& w : word) ss >> w;
    }
    if (word[0] != "%%MatrixMarket" || word[1] != "matrix" || word[2] != "coordinate")
      throw std::runtime_error(path + " could not be parsed as a Matrix Market file.");
    const bool pattern = word[3] == "pattern";
    bool symmetric = false;
    if (word[4] == "symmetric")
      symmetric = true;
    else if (word[4] != "general")
      throw std::runtime_error(path + " has an unsupported matrix type");
    while (std::getline(f, buf) && !buf.empty() && buf[0] == '%') {
    }
    size_t m = 0, n = 0, announced = 0;
    {
      std::istringstream ss(buf);
      ss >> m >> n >> announced;
    }
    struct Entry {
      size_t i, j, order;
      T v;
    };
    std::vector<Entry> e;
    size_t lines = 0;
    while (std::getline(f, buf)) {
      std::istringstream ss(buf);
      long long i = 0, j = 0;
      T v = T(1);
      if (!(ss >> i >> j)) continue;  // blank line
      if (!pattern && !(ss >> v)) throw std::runtime_error("read_MatrixMarket: malformed entry line in " + path);
      i--, j--;
      if (i < 0 || j < 0 || (size_t)i >= m || (size_t)j >= n)
        throw std::runtime_error("read_MatrixMarket: file has nonzero out of bounds.");
      e.push_back({(size_t)i, (size_t)j, e.size(), v});
      if (symmetric && i != j) e.push_back({(size_t)j, (size_t)i, e.size(), v});
      if (++lines > announced)
        throw std::runtime_error(
            "read_MatrixMarket: error reading Matrix Market file, file has more nonzeros than reported.");
    }
    std::stable_sort(e.begin(), e.end(), [](const Entry& x, const Entry& y) {
      return x.i != y.i ? x.i < y.i : x.j < y.j;
    });
    CSR a;
    a.m = m, a.n = n;
    a.row_ptr.assign(m + 1, 0);
    for (size_t q = 0; q < e.size(); q++) {
      if (q > 0 && e[q].i == e[q - 1].i && e[q].j == e[q - 1].j) continue;  // the first insertion stays
      a.col_ind.push_back((int32_t)e[q].j);
      a.vals.push_back(e[q].v);
      a.row_ptr[e[q].i + 1]++;
    }
    for (size_t r = 0; r < m; r++) a.row_ptr[r + 1] += a.row_ptr[r];
    return a;
  }
  // By suffix, as matrix_io's detect_file_type: .mtx or .binary.
  static CSR read(const std::string& path) {
    auto ends = [&](const char* s) {
      const std::string x(s);
      return path.size() >= x.size() && path.compare(path.size() - x.size(), x.size(), x) == 0;
    };
    if (ends(".mtx")) return read_matrix_market(path);
    if (ends(".binary")) return read_binary(path);
    throw std::runtime_error("matrix_info: Could not detect file format for \"" + path + "\"");
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

  // Tile a host CSR matrix (columns ascending within rows): uploaded once
  // and cut into tiles on the device by bclx_csr_to_tiles (the slicing of
  // SPMatrix(fname, blocking), SPMatrix.hpp:194-271).
  SPMatrix(const CSR<T>& a, BlockCustom blk, int device = 0)
      : m_(a.m), n_(a.n), tm_(blk.tile_m), tn_(blk.tile_n), gm_(ceil_div(a.m, blk.tile_m)),
        gn_(ceil_div(a.n, blk.tile_n)), device_(device) {
    check_cuda(cudaSetDevice(device_), "cudaSetDevice");
    DeviceArray<int32_t> rp, ci;
    DeviceArray<T> v;
    rp.resize(a.row_ptr.size());
    rp.upload(a.row_ptr.data(), a.row_ptr.size());
    ci.resize(a.nnz());
    ci.upload(a.col_ind.data(), a.nnz());
    v.resize(a.nnz());
    v.upload(a.vals.data(), a.nnz());
    tile_row_ptr_.resize(ntiles() * (tm_ + 1));
    tile_offset_.resize(ntiles() + 1);
    col_.resize(a.nnz());
    vals_.resize(a.nnz());
    bclx_csr_t src{};
    src.m = (int64_t)a.m, src.n = (int64_t)a.n, src.nnz = (int64_t)a.nnz();
    src.row_ptr = rp.data(), src.col_ind = ci.data(), src.vals = v.data();
    src.dtype = dtype_of<T>::value;
    bclx_spgrid_out_t out = out_grid();
    check(bclx_csr_to_tiles(context(device_), &src, &out), "bclx_csr_to_tiles");
    off_.assign(ntiles() + 1, 0);
    tile_offset_.download(off_.data(), off_.size());
    make_descriptors();
  }

  // SPMatrix(fname, blocking) (SPMatrix.hpp:108-113): a .mtx or .binary file.
  SPMatrix(const std::string& fname, BlockCustom blk, int device = 0) : SPMatrix(CSR<T>::read(fname), blk, device) {}

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
  // Every tile is on this GPU: rank 0 of one (SPMatrix::tile_rank).
  size_t tile_rank(std::array<size_t, 2>) const { return 0; }

  // SPMatrix::get_tile (SPMatrix.hpp:476-494): one tile copied to the host,
  // tile-local columns.
  CSR<T> get_tile(std::array<size_t, 2> idx) const {
    const size_t t = idx[0] * gn_ + idx[1];
    const auto ts = tile_shape(idx);
    CSR<T> c;
    c.m = ts[0], c.n = ts[1];
    c.row_ptr.resize(ts[0] + 1);
    c.col_ind.resize(tile_nnz(idx));
    c.vals.resize(tile_nnz(idx));
    check_cuda(cudaMemcpy(c.row_ptr.data(), tile_row_ptr_.data() + t * (tm_ + 1), sizeof(int32_t) * (ts[0] + 1),
                          cudaMemcpyDeviceToHost),
               "cudaMemcpy");
    if (c.nnz()) {
      check_cuda(cudaMemcpy(c.col_ind.data(), col_.data() + off_[t], sizeof(int32_t) * c.nnz(), cudaMemcpyDeviceToHost),
                 "cudaMemcpy");
      check_cuda(cudaMemcpy(c.vals.data(), vals_.data() + off_[t], sizeof(T) * c.nnz(), cudaMemcpyDeviceToHost),
                 "cudaMemcpy");
    }
    return c;
  }
  // SPMatrix::arget_tile (SPMatrix.hpp:496-514): the same copy as a future.
  std::future<CSR<T>> arget_tile(std::array<size_t, 2> idx) const {
    return std::async(std::launch::deferred, [this, idx] { return get_tile(idx); });
  }

  // SPMatrix::assign_tile (SPMatrix.hpp:277-308): replace one tile (its
  // shape must be tile_shape(idx); tile-local, sorted columns).
  void assign_tile(std::array<size_t, 2> idx, const CSR<T>& tile) {
    const auto ts = tile_shape(idx);
    if (tile.m != ts[0] || tile.n != ts[1] || tile.row_ptr.size() != ts[0] + 1)
      throw std::runtime_error("BCL::SPMatrix::assign_tile: tile shape mismatch");
    const size_t t = idx[0] * gn_ + idx[1];
    std::vector<int32_t> trp(ntiles() * (tm_ + 1));
    std::vector<int32_t> col(nnz());
    std::vector<T> val(nnz());
    tile_row_ptr_.download(trp.data(), trp.size());
    col_.download(col.data(), col.size());
    vals_.download(val.data(), val.size());
    std::vector<int32_t> ncol(col.begin(), col.begin() + off_[t]);
    std::vector<T> nval(val.begin(), val.begin() + off_[t]);
    ncol.insert(ncol.end(), tile.col_ind.begin(), tile.col_ind.end());
    nval.insert(nval.end(), tile.vals.begin(), tile.vals.end());
    ncol.insert(ncol.end(), col.begin() + off_[t + 1], col.end());
    nval.insert(nval.end(), val.begin() + off_[t + 1], val.end());
    int32_t* rp = trp.data() + t * (tm_ + 1);
    for (size_t r = 0; r <= tm_; r++) rp[r] = r <= ts[0] ? tile.row_ptr[r] : (int32_t)tile.nnz();
    std::vector<int64_t> off(off_);
    const int64_t delta = (int64_t)tile.nnz() - (off_[t + 1] - off_[t]);
    for (size_t u = t + 1; u < off.size(); u++) off[u] += delta;
    set_packed(trp, off, ncol, nval);
  }

  // SPMatrix::dot (SPMatrix.hpp:550-553): this * other as a new matrix with
  // this matrix's tile height and other's tile width.
  SPMatrix dot(const SPMatrix& other) const {
    SPMatrix c(m_, other.n_, {tm_, other.tn_}, device_);
    gemm(*this, other, c);
    return c;
  }

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

  bclx_spgrid_out_t out_grid() {
    bclx_spgrid_out_t out{};
    out.m = (int64_t)m_, out.n = (int64_t)n_, out.tile_m = (int64_t)tm_, out.tile_n = (int64_t)tn_;
    out.grid_m = (int64_t)gm_, out.grid_n = (int64_t)gn_;
    out.dtype = dtype_of<T>::value;
    out.tile_row_ptr = tile_row_ptr_.data();
    out.tile_offset = tile_offset_.data();
    out.col_ind = col_.data();
    out.vals = vals_.data();
    return out;
  }

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
  // DMatrix::tile_shape(index): edge tiles hold fewer rows / columns (their
  // storage is still padded to tile_shape()).
  std::array<size_t, 2> tile_shape(std::array<size_t, 2> idx) const {
    return {std::min(tm_, m_ - idx[0] * tm_), std::min(tn_, n_ - idx[1] * tn_)};
  }
  size_t tile_size() const { return tm_ * tn_; }
  size_t tile_rank(std::array<size_t, 2>) const { return 0; }
  // DMatrix::tile_ptr (DMatrix.hpp:151-157): the tile's device storage.
  T* tile_ptr(std::array<size_t, 2> idx) const { return tiles_.data() + (idx[0] * gn_ + idx[1]) * tile_size(); }
  // DMatrix::get_tile (DMatrix.hpp:169-173): the padded tile, row-major.
  std::vector<T> get_tile(std::array<size_t, 2> idx) const {
    std::vector<T> h(tile_size());
    check_cuda(cudaMemcpy(h.data(), tile_ptr(idx), sizeof(T) * h.size(), cudaMemcpyDeviceToHost), "cudaMemcpy");
    return h;
  }
  // DMatrix::operator=(value) (DMatrix.hpp:226-242): every element of every
  // tile, padding included.
  DMatrix& operator=(T value) {
    if (value == T(0)) {
      check_cuda(cudaMemset(tiles_.data(), 0, sizeof(T) * tiles_.size()), "cudaMemset");
    } else {
      std::vector<T> h(tiles_.size(), value);
      tiles_.upload(h.data(), h.size());
    }
    return *this;
  }
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
