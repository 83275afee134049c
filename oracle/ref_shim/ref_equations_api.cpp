// C entry point over the reference's own Equations (equation.cpp, with
// addeqn.cpp), SymmetricSparseMatrix (sparse.cpp, largeMatrix.cpp) and
// Matrix (matrix.cpp), compiled unmodified into
// oracle/_ref/libbeta_ref_equations.so.  Test infrastructure: it runs the
// reference's assembly path -- restraints, setupStorage, the per-element
// sparsity pattern, allocate, addMatrix with its boundary-condition
// elimination, point loads, solve -- on element matrices and dof maps the
// caller supplies, so the oracle's pattern, scatter and right-hand side can
// be compared with the reference's.
#include <chrono>
#include <cstdio>
#include <cstring>
#include <fcntl.h>
#include <unistd.h>
#include <sstream>
#include <strings.h>
#include <vector>

#include "equation.hpp"
#include "sparse.hpp"

// Helpers equation.cpp calls from the reference's utility.cpp (not compiled
// here): the command reader is never driven by the entry point.
int getLineAndTokenize(std::istream* in, char* terminateString, char* tokenList[], int& numberOfTokens) {
  static char line[1024];
  for (;;) {
    numberOfTokens = 0;
    if (!in->getline(line, sizeof line)) return 1;
    char* save = nullptr;
    for (char* t = strtok_r(line, " \t\r", &save); t && numberOfTokens < 20; t = strtok_r(nullptr, " \t\r", &save))
      tokenList[numberOfTokens++] = t;
    if (numberOfTokens == 0 || std::strncmp(tokenList[0], "//", 2) == 0) continue;
    return strcasecmp(tokenList[0], terminateString) == 0 ? 1 : 0;
  }
}
void displayTime(const char*, std::ostream&) {}
std::ifstream* openFileForInput(char* filename) { return new std::ifstream(filename); }

namespace {
// The solvers report to cout/cerr and (ParCG) to C stdout; keep all of it
// out of the caller's output: the C++ streams go to a string, file
// descriptor 1 to /dev/null for the duration.
struct QuietStreams {
  std::stringstream sink;
  std::streambuf *out, *err;
  int saved_fd = -1;
  QuietStreams() : out(std::cout.rdbuf(sink.rdbuf())), err(std::cerr.rdbuf(sink.rdbuf())) {
    std::fflush(stdout);
    saved_fd = dup(1);
    const int devnull = open("/dev/null", O_WRONLY);
    if (saved_fd >= 0 && devnull >= 0) dup2(devnull, 1);
    if (devnull >= 0) close(devnull);
  }
  ~QuietStreams() {
    std::fflush(stdout);
    if (saved_fd >= 0) {
      dup2(saved_fd, 1);
      close(saved_fd);
    }
    std::cout.rdbuf(out);
    std::cerr.rdbuf(err);
  }
};
}  // namespace

extern "C" {
// The global internal force as the reference sums it for a residual
// (BasicModel::CalculateResidual): restraints set, setupStorage(Sparse, n),
// then Equations::assembleResultantVector per element with its force vector
// Fe (nelem x nde); out gets the resultant vector (restrained rows skipped).
int ref_equations_resultant(int n, int nelem, int nde, const int* maps, const double* Fe,
                            const unsigned char* restrained, double* out) {
  QuietStreams quiet;
  Equations eq;
  for (int i = 0; i < n; ++i)
    if (restrained[i]) eq.setRestraint(i, true);
  eq.setupStorage(Sparse, n);
  for (int e = 0; e < nelem; ++e)
    eq.assembleResultantVector(maps + (size_t)e * nde, nde, Fe + (size_t)e * nde);
  for (int i = 0; i < n; ++i) out[i] = eq.resultantVector[i];
  return 0;
}

// n unknowns; nelem elements of nde dofs each, maps (nelem x nde) their
// equation numbers and Ke (nelem x nde x nde, row-major, upper triangle read)
// their matrices, Fe (nelem x nde, may be null) their force vectors;
// restrained (n, 0/1) with prescribed values; point loads.
// Runs, in the reference's order: setRestraint for each restrained unknown,
// setupStorage(Sparse, n) -- or ParCG when parcg is nonzero, the
// reference's two-thread OpenMP solver --, setSolution of the prescribed values,
// specifyNonZeroLocation per element, allocate, zeroMatrix, addMatrix per
// element (with its force vector), addLoadToEqn per nonzero load, then (when
// x is non-null) solve with the reference's CG (tolerance eps, at most maxit
// iterations) from the initial guess x0 (null: the reference's default, its
// last solution, zero here) -- the sequence DiffusionModel's transient step
// runs with Mbar_e and Fbar_e and x0 = u_s.
// Outputs: the lower triangle as 0-based CSR (rp n+1, col/val up to cap
// entries, *nnz the count), the pseudo-load vector, the load vector, x, and
// (when non-null) seconds[3]: wall time of the structure (setup, pattern,
// allocate), of the element scatter (addMatrix, loads) and of the solve.
// zero_diag is the ReplaceZeroDiagonal option the storage gets (0: none;
// the reference's solve then exits on a zero diagonal).
// Returns 0; 1 when cap is too small; 2 when a load sits on a restrained
// unknown (the reference stops there with "Cannot add load to a restrained
// degree of freedom").
int ref_equations_assemble(int parcg, int n, int nelem, int nde, const int* maps, const double* Ke,
                           const double* Fe, const unsigned char* restrained, const double* prescribed,
                           const double* load, double eps, int maxit, const double* x0, long long* rp, int* col, double* val, long long cap,
                           long long* nnz, double* pseudo, double* loadvec, double* x, double* seconds,
                           double zero_diag) {
  for (int i = 0; i < n; ++i)
    if (restrained[i] && load[i] != 0.0) return 2;
  QuietStreams quiet;
  auto now = [] { return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count(); };
  double t0 = now(), t1 = 0.0, t2 = 0.0;
  Equations eq;
  eq.setMaxIterations(maxit);
  eq.setSOLUTION_EPSILON(eps);
  eq.setReplaceZeroDiagonal_Option(zero_diag);
  for (int i = 0; i < n; ++i)
    if (restrained[i]) eq.setRestraint(i, true);
  eq.setupStorage(parcg ? ParCG : Sparse, n);
  for (int i = 0; i < n; ++i)
    if (restrained[i]) eq.setSolution(prescribed[i], i);
  for (int e = 0; e < nelem; ++e) eq.specifyNonZeroLocation(maps + (size_t)e * nde, nde);
  eq.allocate();
  eq.zeroMatrix();
  t1 = now();
  Matrix K(nde, nde);
  for (int e = 0; e < nelem; ++e) {
    const double* ke = Ke + (size_t)e * nde * nde;
    for (int i = 0; i < nde; ++i)
      for (int j = 0; j < nde; ++j) K(i, j) = ke[i * nde + j];
    eq.addMatrix(K, maps + (size_t)e * nde, nde, Fe ? Fe + (size_t)e * nde : 0, 0);
  }
  for (int i = 0; i < n; ++i)
    if (load[i] != 0.0) eq.addLoadToEqn(load[i], i, false);
  t2 = now();
  SymmetricSparseMatrix& A = *static_cast<SymmetricSparseMatrix*>(eq.a);
  long long k = 0;
  rp[0] = 0;
  for (int i = 0; i < n; ++i) {
    const int m = A.row[i].getNum();
    if (k + m > cap) return 1;
    for (int t = 0; t < m; ++t, ++k) {
      col[k] = A.row[i][t];
      val[k] = A.mat[i][t];
    }
    rp[i + 1] = k;
  }
  *nnz = k;
  for (int i = 0; i < n; ++i) {
    pseudo[i] = eq.pseudoLoadVector[i];
    loadvec[i] = eq.loadVector[i];
  }
  if (x) {
    std::vector<double> guess;
    if (x0) guess.assign(x0, x0 + n);
    const double t3 = now();
    const double* u = eq.solve(x0 ? guess.data() : 0);
    if (seconds) seconds[2] = now() - t3;
    for (int i = 0; i < n; ++i) x[i] = u[i];
  }
  if (seconds) {
    seconds[0] = t1 - t0;
    seconds[1] = t2 - t1;
    if (!x) seconds[2] = 0.0;
  }
  return 0;
}

// ---- one persistent system, for timing the reference's own path ------------
// The bench's reference arm builds the full system once with these calls, in
// the reference's order (setRestraint, setupStorage, setSolution,
// specifyNonZeroLocation per element, allocate, zeroMatrix, addMatrix per
// element, addLoadToEqn), then times Equations::solve on it repeatedly.
struct RefEqSystem {
  Equations eq;
  int n = 0;
  int parcg = 0;
};

void* ref_eqsys_create(int parcg, int n, const unsigned char* restrained, const double* prescribed, int maxit) {
  QuietStreams quiet;
  auto* h = new RefEqSystem();
  h->n = n;
  h->parcg = parcg;
  h->eq.setMaxIterations(maxit);
  for (int i = 0; i < n; ++i)
    if (restrained[i]) h->eq.setRestraint(i, true);
  h->eq.setupStorage(parcg ? ParCG : Sparse, n);
  for (int i = 0; i < n; ++i)
    if (restrained[i]) h->eq.setSolution(prescribed[i], i);
  return h;
}

// specifyNonZeroLocation for nelem elements of nde dofs (maps nelem x nde)
int ref_eqsys_pattern(void* hp, int nelem, int nde, const int* maps) {
  auto* h = (RefEqSystem*)hp;
  QuietStreams quiet;
  for (int e = 0; e < nelem; ++e) h->eq.specifyNonZeroLocation(maps + (size_t)e * nde, nde);
  return 0;
}

int ref_eqsys_allocate(void* hp) {
  auto* h = (RefEqSystem*)hp;
  QuietStreams quiet;
  h->eq.allocate();
  h->eq.zeroMatrix();
  return 0;
}

// addMatrix of nelem element matrices Ke (nelem x nde x nde, row-major, upper
// triangle read) at their maps
int ref_eqsys_add(void* hp, int nelem, int nde, const int* maps, const double* Ke) {
  auto* h = (RefEqSystem*)hp;
  QuietStreams quiet;
  Matrix K(nde, nde);
  for (int e = 0; e < nelem; ++e) {
    const double* ke = Ke + (size_t)e * nde * nde;
    for (int i = 0; i < nde; ++i)
      for (int j = 0; j < nde; ++j) K(i, j) = ke[i * nde + j];
    h->eq.addMatrix(K, maps + (size_t)e * nde, nde, 0, 0);
  }
  return 0;
}

// addLoadToEqn per nonzero load; 2 when a load sits on a restrained unknown
int ref_eqsys_loads(void* hp, const double* load) {
  auto* h = (RefEqSystem*)hp;
  for (int i = 0; i < h->n; ++i)
    if (load[i] != 0.0 && h->eq.restraint[i]) return 2;
  QuietStreams quiet;
  for (int i = 0; i < h->n; ++i)
    if (load[i] != 0.0) h->eq.addLoadToEqn(load[i], i, false);
  return 0;
}

long long ref_eqsys_nnz(void* hp) {
  auto* h = (RefEqSystem*)hp;
  SymmetricSparseMatrix& A = *static_cast<SymmetricSparseMatrix*>(h->eq.a);
  long long k = 0;
  for (int i = 0; i < h->n; ++i) k += A.row[i].getNum();
  return k;
}

// The assembled lower triangle as 0-based CSR (rp n+1, col/val nnz) and the
// right-hand side Equations::solve forms from it (equation.cpp:1320-1322:
// load + pseudo-load on free rows, the prescribed value on restrained rows).
int ref_eqsys_export(void* hp, long long* rp, int* col, double* val, double* b) {
  auto* h = (RefEqSystem*)hp;
  SymmetricSparseMatrix& A = *static_cast<SymmetricSparseMatrix*>(h->eq.a);
  long long k = 0;
  rp[0] = 0;
  for (int i = 0; i < h->n; ++i) {
    const int m = A.row[i].getNum();
    for (int t = 0; t < m; ++t, ++k) {
      col[k] = A.row[i][t];
      val[k] = A.mat[i][t];
    }
    rp[i + 1] = k;
  }
  for (int i = 0; i < h->n; ++i)
    b[i] = h->eq.restraint[i] ? h->eq.solution[i] : h->eq.loadVector[i] + h->eq.pseudoLoadVector[i];
  return 0;
}

// Equations::solve from the initial guess x0 (null: the reference's last
// solution) with the storage's stop tolerance set to eps; x (may be null)
// gets the solution, *seconds the solve's wall time.  The reference exits the
// process when a solve reaches its iteration limit, so the caller picks eps
// from the oracle's trace of the same iterates.
int ref_eqsys_solve(void* hp, double eps, const double* x0, double* x, double* seconds) {
  auto* h = (RefEqSystem*)hp;
  static_cast<SymmetricSparseMatrix*>(h->eq.a)->setSOLUTION_EPSILON(eps);
  QuietStreams quiet;
  std::vector<double> guess;
  if (x0) guess.assign(x0, x0 + h->n);
  const auto t0 = std::chrono::steady_clock::now();
  const double* u = h->eq.solve(x0 ? guess.data() : 0);
  if (seconds) *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  if (x)
    for (int i = 0; i < h->n; ++i) x[i] = u[i];
  return 0;
}

void ref_eqsys_destroy(void* hp) {
  QuietStreams quiet;
  delete (RefEqSystem*)hp;
}
}
