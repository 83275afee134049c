// pattern.hpp -- host-side integer structure of one finite-element system.
//
// Everything here is integer work done once per mesh (BETA does it once per
// analysis in BasicModel::allocateEquationsMatrix, BasicModel.cpp:1022-1033):
//   * node graph: for every node the sorted set of nodes sharing an element;
//   * element colouring: no two elements of one colour share a node, so the
//     device scatter needs no atomics and sums in a fixed order;
//   * element->slot map: for element e and local node pair (a,b) the position
//     of node conn[e][b] in node conn[e][a]'s graph row (16 bits; a block's
//     index is nrp[I] + position);
//   * two sliced-ELL layouts of the global matrix (32 rows per slice, entry
//     (row, k) stored at slice_base + k*32 + row%32 so a warp reads 128-byte
//     lines): node-block rows for the FP32 inner solver and scalar DOF rows
//     with restrained columns removed for the plain FP64 solver;
//   * the reference's lower-triangle pattern (Equations::specifyNonZeroLocation,
//     equation.cpp:1216-1267 + SymmetricSparseMatrix::allocate,
//     sparse.cpp:482-495), exported for the bit-exact structure check.
#pragma once
#include <cstdint>
#include <memory>
#include <new>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

namespace betagpu {

// Allocator whose resize() leaves new elements default-initialised (no zero
// fill) for the large outputs the build writes in full in parallel; a
// single-threaded zero fill before that would touch every page twice.
template <class T>
struct NoInitAlloc : std::allocator<T> {
  template <class U>
  struct rebind {
    using other = NoInitAlloc<U>;
  };
  NoInitAlloc() = default;
  template <class U>
  NoInitAlloc(const NoInitAlloc<U>&) noexcept {}
  template <class U>
  void construct(U* p) noexcept(std::is_nothrow_default_constructible<U>::value) {
    ::new (static_cast<void*>(p)) U;
  }
  template <class U, class... A>
  void construct(U* p, A&&... a) {
    ::new (static_cast<void*>(p)) U(std::forward<A>(a)...);
  }
};
template <class T>
using FillVec = std::vector<T, NoInitAlloc<T>>;

struct HostPattern {
  int nnode = 0, nelem = 0, nnpe = 0, ndpn = 0, ndof = 0;

  // node graph (CSR over nodes, columns ascending, self included)
  std::vector<int> nrp;       // nnode+1
  FillVec<int> ncol;          // nblk
  std::vector<int> ndiag;     // virtual position of node i's diagonal block in its row
  long long nblk = 0;
  // nodes that no element uses, ascending: their rows are the diagonal alone
  // in the reference's pattern (Equations gives an empty row its diagonal),
  // while the node graph keeps their (zero) diagonal block
  std::vector<int> unused;

  // element colouring
  int ncolor = 0;
  std::vector<int> color_ptr;     // ncolor+1
  std::vector<int> elem_by_color; // nelem

  // element -> position of node J in node I's row, nelem * nnpe * nnpe
  FillVec<uint16_t> slot;

  // node-block sliced ELL: slice s covers nodes [32s, 32s+32).  Values:
  // block (I, virtual position v) at chunk bsoff[I/32] + v, entry t at
  // (chunk*ND*ND + t)*32 + I%32.  Columns: with run == 1 one per block
  // (virtual position = graph position); with run == R > 1 one per run of R
  // consecutive node columns J0..J0+R-1 (chunks bsoff[s] + R*k .. + R*k+R-1
  // share the column bcol[(bsoff[s]/R + k)*32 + lane] = J0), so a row of a
  // lexicographically numbered hex mesh stores 9 column indices instead of
  // 27; block (I, graph position q) sits at virtual position
  // vpos[nrp[I] + q] = R*k + (J - J0), and the run's other slots are zero.
  int run_request = 1;        // input: the largest run the caller accepts (1 or 3)
  bool compact_request = true; // input: allow the compact form of column runs
  int run = 1;                // the run length built
  int nslice = 0;
  std::vector<int> bsoff;     // nslice+1, in (virtual) chunks of 32 blocks
  FillVec<int> bcol;          // nchunk/run*32, padding points at the row's own node
  FillVec<uint16_t> vpos;     // run > 1: nblk virtual positions (empty otherwise)
  long long nchunk = 0;       // virtual chunks (value storage = nchunk*32*ND*ND floats)
  // Column runs, compact form (when it makes the matrix at least 2 % smaller):
  // a slice whose 32 rows all have their runs at the same offsets from the
  // row (J0 - I equal across the lanes for every run: a slice inside one
  // x-row of a structured mesh) stores those w offsets once instead of 32 x w
  // columns.  cptr[s] >= 0: the slice's columns at ccol[cptr[s] + k*32 + lane];
  // cptr[s] < 0: its offsets at ccol[~cptr[s] + k], J0 = I + offset.  bcol
  // keeps the full columns (host only).
  bool compact = false;
  std::vector<int> cptr;      // nslice
  FillVec<int> ccol;

  // scalar sliced ELL over dofs (restrained rows: diagonal only; restrained
  // columns removed), slice s covers rows [32s, 32s+32)
  int nsslice = 0;
  std::vector<long long> ssoff;   // nsslice+1, in entries
  FillVec<int> scol;              // ssoff.back()
  std::vector<int> soff;          // per node-pair block: column offset of node J's
                                  // first free dof within rows of node I
  std::vector<int> srowlen;       // per dof
  std::vector<long long> sdiag;   // per dof: index of the diagonal entry
  long long nnz_full = 0;         // scalar nonzeros (without padding)

  // reference lower-triangle pattern
  long long nnz_lower = 0;

  // Scratch of the build.  A caller that rebuilds meshes of similar size
  // into the same HostPattern (a solver context) sets keep_scratch, so the
  // scratch and the outputs above keep their memory between builds and a
  // rebuild writes to resident pages instead of faulting fresh ones in;
  // otherwise the scratch is released when the build ends.
  bool keep_scratch = false;
  std::vector<int> s_icnt, s_inc, s_color, s_ufree, s_ccnt;
  std::vector<uint64_t> s_used;
  std::vector<std::vector<int>> s_mark;  // node-sized marker and position arrays per chunk (within a budget)
  std::vector<FillVec<int>> s_rows;      // per row chunk: its rows' sorted columns, from the row pass to the place
                                         // pass (kept with keep_scratch only within the marker budget)
};

// Builds everything above.  conn: nelem*nnpe; restrained: ndof (0/1).
// Returns an empty string on success, else an error message.
// with_scalar = false skips the scalar FP64 layout (mixed-precision-only
// users; build_scalar adds it later).  nnz_lower is always computed.
std::string build_pattern(int nnode, int nelem, int nnpe, int ndpn, const int* conn,
                          const int* first_dof, const unsigned char* restrained, HostPattern& P,
                          bool with_scalar = true);

// The scalar FP64 layout (soff, srowlen, nnz_full, ssoff, scol, sdiag) for a
// pattern built without it.  Returns an empty string on success.
std::string build_scalar(HostPattern& P, const unsigned char* restrained);

// Makes build_pattern on the calling thread single-threaded (for callers that
// already build many patterns in parallel).
void pattern_serial_on_this_thread(bool on);

// Lower-triangle pattern export in SymmetricSparseMatrix order.
void export_lower_pattern(const HostPattern& P, const unsigned char* restrained,
                          long long* row_ptr, int* col);

// Lower-triangle values export from the scalar FP64 sliced-ELL values.
void export_lower_values_scalar(const HostPattern& P, const unsigned char* restrained,
                                const double* sval, double* out);

// Lower-triangle values export from the node-block FP32 sliced-ELL values.
void export_lower_values_block(const HostPattern& P, const unsigned char* restrained,
                               const float* bval, double* out);

}  // namespace betagpu
