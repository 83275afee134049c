// exchange.cpp -- the reference's system exchange formats (host only).
//
// The lower triangle of a symmetric matrix (rows ascending, columns ascending
// within a row, diagonal last -- SymmetricSparseMatrix's storage order) is
// written and read in the five layouts BETA uses to dump systems for external
// solvers and cross-checks:
//   1 address, lower   SymmetricSparseMatrix::printMatrixAddressFormat       sparse.cpp:295-325
//   2 address, upper   SymmetricSparseMatrix::printMatrixAddressFormatUpper  sparse.cpp:263-293
//   3 compressed rows  SymmetricSparseMatrix::printCompressedRowFormat       sparse.cpp:327-355
//   4 CSR, ASCII       writeCSRMatrixInASCII / readCSRMatrixInASCII          SparseMatrixUtility.cpp:11-26, 60-78
//   5 CSR, binary      writeCSRMatrixInBinary / readCSRMatrixInBinary        SparseMatrixUtility.cpp:28-58
// Values are written as the reference writes them: width 24, 16 significant
// digits (DOUBLE_FORMAT, utility_defines.h:17), scientific notation in the
// CSR ASCII file (SET_SCIENTIFIC).  The CSR files carry the lower triangle's
// 0-based row pointers, columns and values as 32-bit ints and doubles.
#include "../../include/beta_gpu.h"

#include <algorithm>
#include <cstdint>
#include <fstream>
#include <iomanip>
#include <limits>
#include <sstream>
#include <string>
#include <tuple>
#include <vector>

namespace {

struct Lower {
  int n = 0;
  std::vector<long long> rp;
  std::vector<int> col;
  std::vector<double> val;
};

std::ostream& dbl(std::ostream& os, double v) { return os << std::setw(24) << std::setprecision(16) << v; }

int write_lower(const char* path, int format, int n, const long long* rp, const int* col, const double* val) {
  const long long nnz = rp[n];
  if (format == BETA_GPU_FMT_CSR_BINARY || format == BETA_GPU_FMT_CSR_ASCII) {
    if (nnz > std::numeric_limits<int>::max()) return BETA_GPU_ERR_TOO_LARGE;  // 32-bit ia/ja
  }
  if (format == BETA_GPU_FMT_CSR_BINARY) {
    std::ofstream os(path, std::ios::out | std::ios::binary);
    if (!os) return BETA_GPU_ERR_ARG;
    const int n32 = n, nnz32 = (int)nnz;
    std::vector<int> ia(n + 1);
    for (int i = 0; i <= n; ++i) ia[i] = (int)rp[i];
    os.write(reinterpret_cast<const char*>(&n32), sizeof(int));
    os.write(reinterpret_cast<const char*>(&nnz32), sizeof(int));
    os.write(reinterpret_cast<const char*>(ia.data()), sizeof(int) * (n + 1));
    os.write(reinterpret_cast<const char*>(col), sizeof(int) * nnz);
    os.write(reinterpret_cast<const char*>(val), sizeof(double) * nnz);
    return os ? BETA_GPU_OK : BETA_GPU_ERR_ARG;
  }
  std::ofstream os(path);
  if (!os) return BETA_GPU_ERR_ARG;
  switch (format) {
    case BETA_GPU_FMT_ADDRESS_LOWER:
      os << "1" << '\n' << n << " " << nnz << '\n';
      for (int i = 0; i < n; ++i) {
        for (long long k = rp[i]; k < rp[i + 1]; ++k) {
          os << '\t' << i << " " << col[k] << " ";
          dbl(os, val[k]);
        }
        os << '\n';
      }
      break;
    case BETA_GPU_FMT_ADDRESS_UPPER: {
      // entry (j, i) of the upper triangle for every stored (i, j): listed by
      // upper row j, columns ascending
      std::vector<long long> cnt(n + 1, 0);
      for (long long k = 0; k < nnz; ++k) cnt[col[k] + 1]++;
      for (int j = 0; j < n; ++j) cnt[j + 1] += cnt[j];
      std::vector<long long> fill(cnt.begin(), cnt.end() - 1), at(nnz);
      for (int i = 0; i < n; ++i)
        for (long long k = rp[i]; k < rp[i + 1]; ++k) at[fill[col[k]]++] = k;
      os << "2" << '\n' << n << " " << nnz << '\n';
      for (int j = 0; j < n; ++j) {
        for (long long t = cnt[j]; t < cnt[j + 1]; ++t) {
          const long long k = at[t];
          const int i = (int)(std::upper_bound(rp, rp + n + 1, k) - rp) - 1;
          os << '\t' << j << " " << i << " ";
          dbl(os, val[k]);
        }
        os << '\n';
      }
      break;
    }
    case BETA_GPU_FMT_COMPRESSED_ROW:
      os << "1-Lower triangular storage format" << '\n' << n << '\n';
      for (int i = 0; i < n; ++i) {
        os << (rp[i + 1] - rp[i]);
        for (long long k = rp[i]; k < rp[i + 1]; ++k) {
          os << " ";
          dbl(os, val[k]) << " " << col[k];
        }
        os << '\n';
      }
      break;
    case BETA_GPU_FMT_CSR_ASCII:
      os << std::resetiosflags(std::ios::floatfield) << std::setiosflags(std::ios::scientific);
      os << n << " " << nnz << '\n';
      for (int i = 0; i <= n; ++i) os << rp[i] << " ";
      os << '\n';
      for (long long k = 0; k < nnz; ++k) os << col[k] << " ";
      os << '\n';
      for (long long k = 0; k < nnz; ++k) dbl(os, val[k]) << '\n';
      os << '\n';
      break;
    default:
      return BETA_GPU_ERR_ARG;
  }
  return os ? BETA_GPU_OK : BETA_GPU_ERR_ARG;
}

// Triplets (row, col, value) of the lower triangle -> rows ascending, columns
// ascending, the order the writers use.
bool from_triplets(int n, std::vector<std::tuple<int, int, double>>& t, Lower& L) {
  std::stable_sort(t.begin(), t.end(), [](const auto& a, const auto& b) {
    return std::get<0>(a) != std::get<0>(b) ? std::get<0>(a) < std::get<0>(b) : std::get<1>(a) < std::get<1>(b);
  });
  L.n = n;
  L.rp.assign(n + 1, 0);
  L.col.resize(t.size());
  L.val.resize(t.size());
  for (size_t k = 0; k < t.size(); ++k) {
    const int i = std::get<0>(t[k]), j = std::get<1>(t[k]);
    if (i < 0 || i >= n || j < 0 || j > i) return false;
    L.rp[i + 1]++;
    L.col[k] = j;
    L.val[k] = std::get<2>(t[k]);
  }
  for (int i = 0; i < n; ++i) L.rp[i + 1] += L.rp[i];
  return true;
}

int read_lower(const char* path, int format, Lower& L) {
  if (format == BETA_GPU_FMT_CSR_BINARY) {
    std::ifstream is(path, std::ios::in | std::ios::binary);
    if (!is) return BETA_GPU_ERR_ARG;
    int n = 0, nnz = 0;
    is.read(reinterpret_cast<char*>(&n), sizeof(int));
    is.read(reinterpret_cast<char*>(&nnz), sizeof(int));
    if (!is || n < 0 || nnz < 0) return BETA_GPU_ERR_ARG;
    std::vector<int> ia(n + 1);
    L.n = n;
    L.col.resize(nnz);
    L.val.resize(nnz);
    is.read(reinterpret_cast<char*>(ia.data()), sizeof(int) * (n + 1));
    is.read(reinterpret_cast<char*>(L.col.data()), sizeof(int) * (size_t)nnz);
    is.read(reinterpret_cast<char*>(L.val.data()), sizeof(double) * (size_t)nnz);
    if (!is) return BETA_GPU_ERR_ARG;
    L.rp.assign(ia.begin(), ia.end());
    return BETA_GPU_OK;
  }
  std::ifstream is(path);
  if (!is) return BETA_GPU_ERR_ARG;
  std::vector<std::tuple<int, int, double>> t;
  int n = 0;
  if (format == BETA_GPU_FMT_ADDRESS_LOWER || format == BETA_GPU_FMT_ADDRESS_UPPER) {
    int kind = 0;
    long long nnz = 0;
    if (!(is >> kind >> n >> nnz) || kind != format || n < 0 || nnz < 0) return BETA_GPU_ERR_ARG;
    t.reserve(nnz);
    for (long long k = 0; k < nnz; ++k) {
      int i, j;
      double v;
      if (!(is >> i >> j >> v)) return BETA_GPU_ERR_ARG;
      if (format == BETA_GPU_FMT_ADDRESS_UPPER) std::swap(i, j);  // upper (j, i) is lower (i, j)
      t.emplace_back(i, j, v);
    }
    return from_triplets(n, t, L) ? BETA_GPU_OK : BETA_GPU_ERR_ARG;
  }
  if (format == BETA_GPU_FMT_COMPRESSED_ROW) {
    std::string header;
    if (!std::getline(is, header) || !(is >> n) || n < 0) return BETA_GPU_ERR_ARG;
    for (int i = 0; i < n; ++i) {
      long long cnt;
      if (!(is >> cnt) || cnt < 0) return BETA_GPU_ERR_ARG;
      for (long long k = 0; k < cnt; ++k) {
        double v;
        int j;
        if (!(is >> v >> j)) return BETA_GPU_ERR_ARG;
        t.emplace_back(i, j, v);
      }
    }
    return from_triplets(n, t, L) ? BETA_GPU_OK : BETA_GPU_ERR_ARG;
  }
  if (format == BETA_GPU_FMT_CSR_ASCII) {
    long long nnz = 0;
    if (!(is >> n >> nnz) || n < 0 || nnz < 0) return BETA_GPU_ERR_ARG;
    L.n = n;
    L.rp.resize(n + 1);
    L.col.resize(nnz);
    L.val.resize(nnz);
    for (int i = 0; i <= n; ++i)
      if (!(is >> L.rp[i])) return BETA_GPU_ERR_ARG;
    for (long long k = 0; k < nnz; ++k)
      if (!(is >> L.col[k])) return BETA_GPU_ERR_ARG;
    for (long long k = 0; k < nnz; ++k)
      if (!(is >> L.val[k])) return BETA_GPU_ERR_ARG;
    return BETA_GPU_OK;
  }
  return BETA_GPU_ERR_ARG;
}

}  // namespace

extern "C" {

BETA_GPU_API int beta_gpu_write_lower(const char* path, int format, int n, const long long* row_ptr, const int* col,
                                      const double* val) {
  if (!path || n < 0 || !row_ptr || (row_ptr[n] > 0 && (!col || !val))) return BETA_GPU_ERR_ARG;
  for (int i = 0; i < n; ++i)
    if (row_ptr[i + 1] < row_ptr[i]) return BETA_GPU_ERR_ARG;
  return write_lower(path, format, n, row_ptr, col, val);
}

BETA_GPU_API int beta_gpu_read_lower(const char* path, int format, int* n, long long* nnz, long long* row_ptr,
                                     int* col, double* val) {
  if (!path || !n || !nnz) return BETA_GPU_ERR_ARG;
  Lower L;
  const int rc = read_lower(path, format, L);
  if (rc != BETA_GPU_OK) return rc;
  *n = L.n;
  *nnz = (long long)L.col.size();
  if (row_ptr && col && val) {
    std::copy(L.rp.begin(), L.rp.end(), row_ptr);
    std::copy(L.col.begin(), L.col.end(), col);
    std::copy(L.val.begin(), L.val.end(), val);
  }
  return BETA_GPU_OK;
}

}  // extern "C"
