// MPX_matrix files in the reference's binary format: the .BLOCK environment
// checkpoints (BlocksStructure::save_* / load_*, DMRG_routines.cpp:65-186)
// and the .MPS_matrix / .MPX_matrix state files (MPS_matrix.cpp:140-165).
// Host code only; no device memory is touched.
//
// Layout (MPX_matrix::fprint_binary, MPX_matrix.cpp:219-233), native
// little-endian, as the reference writes it on x86-64 Linux:
//   size_t   number of indices
//   int64    number of row indices (SuiteSparse_long)
//   per index (MPXIndex::fprint_binary, MPXIndex.cpp:8-23):
//     bool inward, bool physical (one byte each), size_t size,
//     then, for a non-physical index of non-zero size, every element's
//     charges as nq int16 (State::fprint_binary, states.cpp:59-61)
//   the CSC matrix (SparseMatrix::fprint_binary, sparse_interface.cpp:727-764):
//     int64 nzmax, nz (= -1: compressed columns), rows, cols
//     int64 colptr[cols + 1]
//     if colptr[cols] == 0: one int64 0 and one complex 0 (a placeholder)
//     else: int64 rowind[nzmax], complex<double> values[nzmax]
// A physical index is stored without charges: the reader takes them from the
// model's basis (load_MPXIndex_binary, MPXIndex.cpp:98-121).  The reader
// follows load_SparseMatrix_binary (sparse_interface.cpp:767-835): it does
// not consume the placeholder of an empty matrix, and of nzmax stored entries
// it keeps the first colptr[cols].
#include <cstdint>
#include <cstdio>
#include <new>
#include <string>
#include <vector>

#include "internal.h"
#include "chainamps_b200.h"

namespace cmps {
namespace {

struct File {
  std::FILE* f = nullptr;
  ~File() {
    if (f) std::fclose(f);
  }
};

bool put(std::FILE* f, const void* p, size_t bytes) { return bytes == 0 || std::fwrite(p, 1, bytes, f) == bytes; }
bool get(std::FILE* f, void* p, size_t bytes) { return bytes == 0 || std::fread(p, 1, bytes, f) == bytes; }

// Bytes left between the read position and the end of the file: every count
// read from a file is checked against it before anything of that size is
// allocated, so a corrupt or truncated file is refused instead of exhausting
// host memory.
int64_t remaining(std::FILE* f) {
  const long pos = std::ftell(f);
  if (pos < 0 || std::fseek(f, 0, SEEK_END) != 0) return -1;
  const long end = std::ftell(f);
  if (end < 0 || std::fseek(f, pos, SEEK_SET) != 0) return -1;
  return (int64_t)end - (int64_t)pos;
}
// true if `count` items of `size` bytes fit in what is left of the file
bool fits(std::FILE* f, uint64_t count, uint64_t size) {
  const int64_t left = remaining(f);
  return left >= 0 && (size == 0 || count <= (uint64_t)left / size);
}

// Checked description of one stored MPX (sizes only).
struct Header {
  int64_t num_indices = 0, num_row_indices = 0;
  std::vector<uint8_t> inward, physical;
  std::vector<int64_t> sizes;
  int64_t total = 0;  // sum of sizes
  int64_t nzmax = 0, rows = 0, cols = 0, nnz = 0;
  // stored charges of the non-physical indices: run i starts at charges[charge_at[i]]
  // and belongs at element offset charge_pos[i]
  std::vector<int16_t> charges;
  std::vector<int64_t> charge_at, charge_pos;
};

// Reads the index section and the CSC header and column pointers; leaves the
// file positioned at the row indices.  charges (if non-null) receives the
// stored charges of non-physical indices at their element offsets.
int read_header(std::FILE* f, int32_t nq, Header& h, std::vector<int64_t>& colptr, int16_t* charges) {
  uint64_t n = 0;
  if (!get(f, &n, sizeof n) || !get(f, &h.num_row_indices, sizeof h.num_row_indices))
    return fail(CMPS_ERR_ARG, "MPX file: truncated header");
  if (n > 64 || h.num_row_indices < 0 || h.num_row_indices > (int64_t)n)
    return fail(CMPS_ERR_ARG, "MPX file: bad index count");
  h.num_indices = (int64_t)n;
  h.inward.resize(n);
  h.physical.resize(n);
  h.sizes.resize(n);
  std::vector<int16_t> buf;
  for (uint64_t i = 0; i < n; ++i) {
    uint8_t in = 0, ph = 0;
    uint64_t sz = 0;
    if (!get(f, &in, 1) || !get(f, &ph, 1) || !get(f, &sz, sizeof sz))
      return fail(CMPS_ERR_ARG, "MPX file: truncated index");
    if (in > 1 || ph > 1 || sz > (uint64_t)1 << 40) return fail(CMPS_ERR_ARG, "MPX file: bad index record");
    h.inward[i] = in;
    h.physical[i] = ph;
    h.sizes[i] = (int64_t)sz;
    if (!ph && sz > 0) {
      if (!fits(f, sz * (uint64_t)nq, sizeof(int16_t))) return fail(CMPS_ERR_ARG, "MPX file: truncated charges");
      buf.resize((size_t)sz * nq);
      if (!get(f, buf.data(), sizeof(int16_t) * buf.size())) return fail(CMPS_ERR_ARG, "MPX file: truncated charges");
      // kept here until the whole header has been checked
      h.charge_at.push_back((int64_t)h.charges.size());
      h.charge_pos.push_back(h.total);
      h.charges.insert(h.charges.end(), buf.begin(), buf.end());
    }
    h.total += (int64_t)sz;
  }
  int64_t params[4];
  if (!get(f, params, sizeof params)) return fail(CMPS_ERR_ARG, "MPX file: truncated matrix header");
  if (params[1] != -1) return fail(CMPS_ERR_ARG, "MPX file: matrix not in compressed-column form");
  h.nzmax = params[0];
  h.rows = params[2];
  h.cols = params[3];
  if (h.nzmax < 0 || h.rows < 0 || h.cols < 0 || h.cols > ((int64_t)1 << 40))
    return fail(CMPS_ERR_ARG, "MPX file: bad matrix shape");
  if (!fits(f, (uint64_t)h.cols + 1, sizeof(int64_t))) return fail(CMPS_ERR_ARG, "MPX file: truncated colptr");
  colptr.assign((size_t)h.cols + 1, 0);
  if (!get(f, colptr.data(), sizeof(int64_t) * colptr.size())) return fail(CMPS_ERR_ARG, "MPX file: truncated colptr");
  if (colptr[0] != 0) return fail(CMPS_ERR_ARG, "MPX file: colptr[0] != 0");
  for (int64_t c = 0; c < h.cols; ++c)
    if (colptr[c + 1] < colptr[c]) return fail(CMPS_ERR_ARG, "MPX file: colptr decreases");
  h.nnz = colptr[h.cols];
  if (h.nnz > h.nzmax) return fail(CMPS_ERR_ARG, "MPX file: more entries than nzmax");
  // the matrix shape is the product of the row / column index sizes
  if (h.num_indices > 0) {
    int64_t r = 1, c = 1;
    for (int64_t i = 0; i < h.num_indices; ++i) (i < h.num_row_indices ? r : c) *= h.sizes[i];
    if (r != h.rows || c != h.cols) return fail(CMPS_ERR_ARG, "MPX file: matrix shape differs from the index sizes");
  }
  // row indices and values of nzmax entries follow
  if (!fits(f, (uint64_t)h.nzmax, sizeof(int64_t) + 2 * sizeof(double)))
    return fail(CMPS_ERR_ARG, "MPX file: truncated entries");
  // the header is whole: only now does the caller's charges buffer get written
  if (charges)
    for (size_t i = 0; i < h.charge_at.size(); ++i) {
      const size_t from = (size_t)h.charge_at[i];
      const size_t to = i + 1 < h.charge_at.size() ? (size_t)h.charge_at[i + 1] : h.charges.size();
      for (size_t e = from; e < to; ++e) charges[(size_t)h.charge_pos[i] * nq + (e - from)] = h.charges[e];
    }
  return CMPS_OK;
}

int open_read(const char* path, File& f) {
  if (!path) return fail(CMPS_ERR_ARG, "null path");
  f.f = std::fopen(path, "rb");
  if (!f.f) return fail(CMPS_ERR_ARG, std::string("cannot open ") + path);
  return CMPS_OK;
}

}  // namespace
}  // namespace cmps

using namespace cmps;

extern "C" {

int cmps_mpx_store(const cmps_mpx_desc* m, int32_t nq, const char* path) {
  if (!m || !path) return fail(CMPS_ERR_ARG, "null argument");
  if (nq < 1 || nq > 16) return fail(CMPS_ERR_ARG, "nq must be 1..16");
  if (m->num_indices < 0 || m->num_indices > 64 || m->num_row_indices < 0 || m->num_row_indices > m->num_indices)
    return fail(CMPS_ERR_ARG, "bad index counts");
  if (m->num_indices > 0 && (!m->inward || !m->physical || !m->sizes)) return fail(CMPS_ERR_ARG, "null index arrays");
  if (m->rows < 0 || m->cols < 0 || !m->colptr) return fail(CMPS_ERR_ARG, "bad matrix shape");
  int64_t total = 0, r = 1, c = 1;
  for (int32_t i = 0; i < m->num_indices; ++i) {
    if (m->sizes[i] < 0) return fail(CMPS_ERR_ARG, "negative index size");
    (i < m->num_row_indices ? r : c) *= m->sizes[i];
    total += m->sizes[i];
  }
  if (m->num_indices > 0 && (r != m->rows || c != m->cols))
    return fail(CMPS_ERR_ARG, "matrix shape differs from the index sizes");
  if (total > 0 && !m->charges) return fail(CMPS_ERR_ARG, "null charges");
  if (m->colptr[0] != 0) return fail(CMPS_ERR_ARG, "colptr[0] != 0");
  for (int64_t j = 0; j < m->cols; ++j)
    if (m->colptr[j + 1] < m->colptr[j]) return fail(CMPS_ERR_ARG, "colptr decreases");
  const int64_t nnz = m->colptr[m->cols];
  if (nnz > 0 && (!m->rowind || !m->values)) return fail(CMPS_ERR_ARG, "null entries");
  for (int64_t p = 0; p < nnz; ++p)
    if (m->rowind[p] < 0 || m->rowind[p] >= m->rows) return fail(CMPS_ERR_ARG, "row index out of range");

  File f;
  f.f = std::fopen(path, "wb");
  if (!f.f) return fail(CMPS_ERR_ARG, std::string("cannot create ") + path);
  bool ok = true;
  const uint64_t n = (uint64_t)m->num_indices;
  const int64_t nrow = m->num_row_indices;
  ok = ok && put(f.f, &n, sizeof n) && put(f.f, &nrow, sizeof nrow);
  int64_t off = 0;
  for (int32_t i = 0; i < m->num_indices && ok; ++i) {
    const uint8_t in = m->inward[i] ? 1 : 0, ph = m->physical[i] ? 1 : 0;
    const uint64_t sz = (uint64_t)m->sizes[i];
    ok = put(f.f, &in, 1) && put(f.f, &ph, 1) && put(f.f, &sz, sizeof sz);
    if (ok && !ph && sz > 0) ok = put(f.f, m->charges + (size_t)off * nq, sizeof(int16_t) * (size_t)sz * nq);
    off += m->sizes[i];
  }
  // a finalised reference matrix holds nzmax = max(nnz, 1) (cs_spalloc)
  const int64_t params[4] = {nnz > 0 ? nnz : 1, -1, m->rows, m->cols};
  ok = ok && put(f.f, params, sizeof params) && put(f.f, m->colptr, sizeof(int64_t) * ((size_t)m->cols + 1));
  if (nnz == 0) {
    const int64_t zi = 0;
    const double zx[2] = {0.0, 0.0};
    ok = ok && put(f.f, &zi, sizeof zi) && put(f.f, zx, sizeof zx);
  } else {
    ok = ok && put(f.f, m->rowind, sizeof(int64_t) * (size_t)nnz) && put(f.f, m->values, 2 * sizeof(double) * (size_t)nnz);
  }
  if (!ok || std::fflush(f.f) != 0) return fail(CMPS_ERR_ARG, std::string("write failed: ") + path);
  return CMPS_OK;
}

int cmps_mpx_stat(const char* path, int32_t nq, int32_t* num_indices, int32_t* num_row_indices,
                  int64_t* total_elements, int64_t* rows, int64_t* cols, int64_t* nnz) {
  if (nq < 1 || nq > 16) return fail(CMPS_ERR_ARG, "nq must be 1..16");
  File f;
  CMPS_TRY(open_read(path, f));
  Header h;
  std::vector<int64_t> colptr;
  CMPS_TRY(read_header(f.f, nq, h, colptr, nullptr));
  if (num_indices) *num_indices = (int32_t)h.num_indices;
  if (num_row_indices) *num_row_indices = (int32_t)h.num_row_indices;
  if (total_elements) *total_elements = h.total;
  if (rows) *rows = h.rows;
  if (cols) *cols = h.cols;
  if (nnz) *nnz = h.nnz;
  return CMPS_OK;
}

int cmps_mpx_load(const char* path, int32_t nq, const int16_t* basis_charges, int64_t basis_size, uint8_t* inward,
                  uint8_t* physical, int64_t* sizes, int16_t* charges, int64_t* colptr, int64_t* rowind,
                  double* values) {
  if (nq < 1 || nq > 16) return fail(CMPS_ERR_ARG, "nq must be 1..16");
  File f;
  CMPS_TRY(open_read(path, f));
  Header h;
  std::vector<int64_t> cp;
  // the caller sized charges from cmps_mpx_stat; physical indices are filled below
  CMPS_TRY(read_header(f.f, nq, h, cp, charges));
  if (h.num_indices > 0 && (!inward || !physical || !sizes)) return fail(CMPS_ERR_ARG, "null index arrays");
  if (h.total > 0 && !charges) return fail(CMPS_ERR_ARG, "null charges");
  if (!colptr || (h.nnz > 0 && (!rowind || !values))) return fail(CMPS_ERR_ARG, "null matrix arrays");
  int64_t off = 0;
  for (int64_t i = 0; i < h.num_indices; ++i) {
    inward[i] = h.inward[i];
    physical[i] = h.physical[i];
    sizes[i] = h.sizes[i];
    if (h.physical[i]) {
      if (!basis_charges || basis_size != h.sizes[i])
        return fail(CMPS_ERR_ARG, "MPX file: a physical index needs the basis charges (size " +
                                      std::to_string(h.sizes[i]) + ")");
      for (int64_t e = 0; e < h.sizes[i] * nq; ++e) charges[off * nq + e] = basis_charges[e];
    }
    off += h.sizes[i];
  }
  for (size_t j = 0; j < cp.size(); ++j) colptr[j] = cp[j];
  if (h.nzmax > 0 && h.nnz > 0) {
    // nzmax is bounded by the file size (read_header), so these fit in memory
    // unless the host itself is out of it
    std::vector<int64_t> ri;
    std::vector<double> x;
    try {
      ri.resize((size_t)h.nzmax);
      x.resize(2 * (size_t)h.nzmax);
    } catch (const std::bad_alloc&) {
      return fail(CMPS_ERR_NOMEM, "MPX file: host allocation of " + std::to_string(h.nzmax) + " entries failed");
    }
    if (!get(f.f, ri.data(), sizeof(int64_t) * ri.size()) || !get(f.f, x.data(), sizeof(double) * x.size()))
      return fail(CMPS_ERR_ARG, "MPX file: truncated entries");
    for (int64_t p = 0; p < h.nnz; ++p) {
      if (ri[p] < 0 || ri[p] >= h.rows) return fail(CMPS_ERR_ARG, "MPX file: row index out of range");
      rowind[p] = ri[p];
      values[2 * p] = x[2 * p];
      values[2 * p + 1] = x[2 * p + 1];
    }
  }
  return CMPS_OK;
}

}  // extern "C"
