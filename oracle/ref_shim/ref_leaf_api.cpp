// C entry points over the reference's own gauss.cpp, shape.cpp, sparse.cpp,
// largeMatrix.cpp, SparseMatrixUtility.cpp and element files (2D/3D
// diffusion, 2D/3D elasticity), compiled unmodified into
// oracle/_ref/libbeta_ref_leaf.so.
// Test infrastructure: used only to pin the oracle's restatement against the
// reference's code.
#include <fcntl.h>
#include <unistd.h>

#include <cstdio>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "gauss.hpp"
#include "hexQuadPoint.hpp"
#include "quadQuadPoint.hpp"
#include "sparse.hpp"
#include "HeatTransferElement2DTransient.hpp"
#include "HeatTransferElement3DTransient.hpp"
#include "ElasticityElement2D.hpp"

int verboseFlag = 0;  // a global the reference's element files declare extern

// SparseMatrixUtility.cpp (no header in the reference)
void writeCSRMatrixInASCII(char* filename, int*& ia, int*& ja, double*& a, int numberOfEquations, int ncoefs);
void writeCSRMatrixInBinary(char* filename, int*& ia, int*& ja, double*& a, int numberOfEquations, int ncoefs);
void readCSRMatrixInBinary(char* filename, int*& ia, int*& ja, double*& a, int& numberOfEquations, int& ncoefs);
void readCSRMatrixInASCII(char* filename, int*& ia, int*& ja, double*& a, int& n);

namespace {
// SymmetricSparseMatrix that counts its matrix-vector products (one for the
// initial residual, one per CG iteration).
class CountingSparse : public SymmetricSparseMatrix {
 public:
  explicit CountingSparse(int n) : SymmetricSparseMatrix(n) {}
  void vectorProduct(double* result, double* vector) override {
    ++products;
    SymmetricSparseMatrix::vectorProduct(result, vector);
  }
  int products = 0;
};
}  // namespace

void shapeHex8(double* S, double xi, double eta, double zeta);
void derivHex8(double* Sxi, double* Seta, double* Szeta, double xi, double eta, double zeta);
void shapeQuad4(double* S, double zeta, double eta);
void derivQuad4(double* Szeta, double* Seta, double zeta, double eta);
void shapeQuad8(double* S, double xi, double eta);
void derivQuad8(double* Szeta, double* Seta, double zeta, double eta);
void shapeTri6(double* S, double xi, double eta);
void derivTri6(double* Sxi, double* Seta, double xi, double eta);

namespace {
// Keeps what the reference code prints (C++ streams and C stdout) out of the
// caller's standard output while a timing entry point runs.
struct QuietStdout {
  std::stringstream sink;
  std::streambuf* out;
  int saved_fd = -1;
  QuietStdout() : out(std::cout.rdbuf(sink.rdbuf())) {
    std::fflush(stdout);
    saved_fd = dup(1);
    const int devnull = open("/dev/null", O_WRONLY);
    if (saved_fd >= 0 && devnull >= 0) dup2(devnull, 1);
    if (devnull >= 0) close(devnull);
  }
  ~QuietStdout() {
    std::fflush(stdout);
    if (saved_fd >= 0) {
      dup2(saved_fd, 1);
      close(saved_fd);
    }
    std::cout.rdbuf(out);
  }
};

// Shape functions and global gradients of a hex8 at one of the reference's
// Gauss points (shapeHex8 / derivHex8), with the Jacobian J (rows d/dxi,
// d/deta, d/dzeta of the coordinates X, 8 x 3), its determinant and inverse
// by cofactors -- IsoElement::jacobian (isoElement.cpp:250-389) restated,
// that file does not compile here.  Returns det J (<= 0: a bad element).
double hex8_point(const double* X, double xi, double eta, double zeta, InterpAndSolDerivatives& id) {
  double S[8], d0[8], d1[8], d2[8];
  shapeHex8(S, xi, eta, zeta);
  derivHex8(d0, d1, d2, xi, eta, zeta);
  double J[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  for (int a = 0; a < 8; ++a)
    for (int k = 0; k < 3; ++k) {
      J[0][k] += d0[a] * X[a * 3 + k];
      J[1][k] += d1[a] * X[a * 3 + k];
      J[2][k] += d2[a] * X[a * 3 + k];
    }
  const double c00 = J[1][1] * J[2][2] - J[1][2] * J[2][1], c01 = J[1][2] * J[2][0] - J[1][0] * J[2][2],
               c02 = J[1][0] * J[2][1] - J[1][1] * J[2][0];
  const double det = J[0][0] * c00 + J[0][1] * c01 + J[0][2] * c02;
  if (!(det > 0.0)) return det;
  const double inv[3][3] = {
      {c00 / det, (J[0][2] * J[2][1] - J[0][1] * J[2][2]) / det, (J[0][1] * J[1][2] - J[0][2] * J[1][1]) / det},
      {c01 / det, (J[0][0] * J[2][2] - J[0][2] * J[2][0]) / det, (J[0][2] * J[1][0] - J[0][0] * J[1][2]) / det},
      {c02 / det, (J[0][1] * J[2][0] - J[0][0] * J[2][1]) / det, (J[0][0] * J[1][1] - J[0][1] * J[1][0]) / det}};
  for (int a = 0; a < 8; ++a) {
    id.S[a] = S[a];
    id.p_S_x1[a] = inv[0][0] * d0[a] + inv[0][1] * d1[a] + inv[0][2] * d2[a];
    id.p_S_x2[a] = inv[1][0] * d0[a] + inv[1][1] * d1[a] + inv[1][2] * d2[a];
    id.p_S_x3[a] = inv[2][0] * d0[a] + inv[2][1] * d1[a] + inv[2][2] * d2[a];
  }
  return det;
}

// The same for a quad4 (shapeQuad4 / derivQuad4, 2 x 2 Jacobian).
double quad4_point(const double* X, double xi, double eta, InterpAndSolDerivatives& id) {
  double S[4], d0[4], d1[4];
  shapeQuad4(S, xi, eta);
  derivQuad4(d0, d1, xi, eta);
  double J[2][2] = {{0, 0}, {0, 0}};
  for (int a = 0; a < 4; ++a)
    for (int k = 0; k < 2; ++k) {
      J[0][k] += d0[a] * X[a * 2 + k];
      J[1][k] += d1[a] * X[a * 2 + k];
    }
  const double det = J[0][0] * J[1][1] - J[0][1] * J[1][0];
  if (!(det > 0.0)) return det;
  const double i00 = J[1][1] / det, i01 = -J[0][1] / det, i10 = -J[1][0] / det, i11 = J[0][0] / det;
  for (int a = 0; a < 4; ++a) {
    id.S[a] = S[a];
    id.p_S_x1[a] = i00 * d0[a] + i01 * d1[a];
    id.p_S_x2[a] = i10 * d0[a] + i11 * d1[a];
  }
  return det;
}

// One integration point of the reference's own elasticity element E
// (ElasticityElement3D or ElasticityElement2D): calculateBmatrix + addToKe
// into Ke (ndof x ndof row-major, upper triangle) and, when u is given,
// derivativesOfFields + calculateStrain, the material's stress C * strain and
// addToFe into Fe (ndof); strain (numStrains) is returned when non-null.
template <class E>
int elastic_point(int dim, int nnode, const double* C, const double* dx, const double* dy, const double* dz,
                  const double* u, double factor, double* Ke, double* Fe, double* strain) {
  E e;
  const int ndof = dim * nnode, ns = e.numStrains;
  if (ndof > (dim == 3 ? 96 : 36)) return 1;  // the reference's addToKe work arrays
  std::vector<double> brows((size_t)6 * ndof, 0.0);
  double* rows[6];
  for (int r = 0; r < 6; ++r) rows[r] = brows.data() + (size_t)r * ndof;
  Matrix K(ndof, ndof), c(ns, ns);
  for (int i = 0; i < ndof; ++i)
    for (int j = 0; j < ndof; ++j) K(i, j) = Ke[i * ndof + j];
  for (int i = 0; i < ns; ++i)
    for (int j = 0; j < ns; ++j) c(i, j) = C[i * ns + j];
  InterpAndSolDerivatives id(nnode, nnode);
  id.allocate();
  id.numberOfInterp = nnode;
  for (int a = 0; a < nnode; ++a) {
    id.p_S_x1[a] = dx[a];
    id.p_S_x2[a] = dy[a];
    id.p_S_x3[a] = dz ? dz[a] : 0.0;
    if (u) {
      id.nodalValues_u1[a] = u[a * dim];
      id.nodalValues_u2[a] = u[a * dim + 1];
      id.nodalValues_u3[a] = dim == 3 ? u[a * dim + 2] : 0.0;
    }
  }
  e.b = rows;
  e.Ke = &K;
  e.numDof = ndof;
  e.calculateBmatrix(&id, rows);
  double stress[6] = {0, 0, 0, 0, 0, 0}, eps[6] = {0, 0, 0, 0, 0, 0};
  e.addToKe(&c, &id, factor, stress);
  for (int i = 0; i < ndof; ++i)
    for (int j = 0; j < ndof; ++j) Ke[i * ndof + j] = K(i, j);
  if (u) {
    ElasticMaterial mat;
    mat.numStrains = ns;
    mat.cmat = c;
    e.derivativesOfFields(&id);
    e.calculateStrain(&id, eps);
    mat.calculateStress(stress, eps, nullptr, nullptr);
    e.addToFe(ndof, ns, rows, stress, factor, Fe);
    if (strain)
      for (int i = 0; i < ns; ++i) strain[i] = eps[i];
  }
  return 0;
}
// The ElementWorkspace arrays an elasticity element with nip points reads and
// writes: per point stresses, strains and their rotated copies; per element
// and total strain, stress, energy and local-stress integrals.
struct ElasticBag {
  ElementWorkspace w;
  std::vector<double> pts, sums;
  std::vector<double*> rows;
  explicit ElasticBag(int nip) : pts((size_t)4 * nip * 6, 0.0), sums(8 * 6, 0.0), rows((size_t)4 * nip) {
    for (int k = 0; k < 4 * nip; ++k) rows[k] = pts.data() + (size_t)k * 6;
    w.quadPointStresses = rows.data();
    w.quadPointStrains = rows.data() + nip;
    w.rotatedStresses = rows.data() + 2 * nip;
    w.rotatedStrains = rows.data() + 3 * nip;
    double* t = sums.data();
    w.strainVolume_element = t;
    w.stressVolume_element = t + 6;
    w.energyVolume_element = t + 12;
    w.localStressVolume_element = t + 18;
    w.strainVolume_total = t + 24;
    w.stressVolume_total = t + 30;
    w.energyVolume_total = t + 36;
    w.localStressVolume_total = t + 42;
  }
};

// One elasticity element E (ElasticityElement3D or ElasticityElement2D) set up
// as the reference's model would hand it over: nnode nodes at X (nnode x dim),
// local dof numbers 0..ndof-1, the constitutive matrix C, the integration
// order, its workspace, stiffness and force buffers.  run(e) then calls the
// reference's own member functions on it.
template <class E, class F>
int with_elastic(int dim, int nnode, const double* X, const double* C, int order, F run) {
  QuietStdout quiet;
  E e;
  const int ndof = dim * nnode, ns = e.numStrains;
  if (ndof > (dim == 3 ? 96 : 36)) return 1;
  const int nip = dim == 3 ? order * order * order : order * order;
  e.numNodesPerElement = nnode;
  e.numDof = ndof;
  e.setIntegrationOrder(order);
  std::vector<double> coords((size_t)nnode * 3, 0.0);
  for (int a = 0; a < nnode; ++a)
    for (int k = 0; k < dim; ++k) coords[a * 3 + k] = X[a * dim + k];
  std::vector<int> dofs(ndof);
  for (int i = 0; i < ndof; ++i) dofs[i] = i;
  e.coords = coords.data();
  e.edofs = dofs.data();
  std::vector<double> brows((size_t)6 * ndof, 0.0);
  double* rows[6];
  for (int r = 0; r < 6; ++r) rows[r] = brows.data() + (size_t)r * ndof;
  ElasticBag bag(nip);
  bag.w.b = rows;
  e.setPointers(&bag.w);
  Matrix K(ndof, ndof);
  std::vector<double> fe(ndof, 0.0), ife(ndof, 0.0);
  e.Ke = &K;
  e.Fe = fe.data();
  e.initialFe = ife.data();
  ElasticMaterial mat;
  mat.numStrains = ns;
  mat.cmat = Matrix(ns, ns);
  for (int i = 0; i < ns; ++i)
    for (int j = 0; j < ns; ++j) mat.cmat(i, j) = C[i * ns + j];
  e.material = &mat;
  e.isv.assign(nip, nullptr);
  return run(e, K, fe, bag);
}
}  // namespace

extern "C" {
// The reference's own element driver: ElasticityElement3D (dim 3, hex8) or
// ElasticityElement2D (dim 2, quad4) update(action, u) -> its
// loopOverIntegrationPoints and processActionCode ("K" stiffness, "F"
// internal force with the stresses it needs, "S" stresses), over the
// reference's Gauss rule.  u (element dofs, interleaved) may be null.  Ke
// (ndof x ndof, upper triangle), Fe (ndof) and sums (18: the element's
// strain, stress and energy integrals, 6 each, as loopOverIntegrationPoints
// adds them to the workspace totals).
// analysis: BasicElement::analysisType (LINEAR 0, GEOMETRIC_NONLINEAR 1).
int ref_elastic_update_analysis(int dim, int nnode, const double* X, const double* C, int order, const double* u,
                                const char* action, int analysis, double* Ke, double* Fe, double* sums) {
  auto run = [&](auto& e, Matrix& K, std::vector<double>& fe, ElasticBag& bag) {
    std::vector<double> uu;
    if (u) uu.assign(u, u + e.numDof);
    std::string act(action);
    e.analysisType = analysis;
    e.update(&act[0], u ? uu.data() : nullptr);
    const int n = e.numDof;
    for (int i = 0; i < n; ++i) {
      Fe[i] = fe[i];
      for (int j = 0; j < n; ++j) Ke[i * n + j] = K(i, j);
    }
    for (int k = 0; k < 18; ++k) sums[k] = bag.sums[24 + k];
    return 0;
  };
  if (dim == 3) return with_elastic<ElasticityElement3D>(3, nnode, X, C, order, run);
  if (dim == 2) return with_elastic<ElasticityElement2D>(2, nnode, X, C, order, run);
  return 1;
}

int ref_elastic_update(int dim, int nnode, const double* X, const double* C, int order, const double* u,
                       const char* action, double* Ke, double* Fe, double* sums) {
  return ref_elastic_update_analysis(dim, nnode, X, C, order, u, action, LINEAR, Ke, Fe, sums);
}

// The reference's own diffusion element driver: HeatTransferElement3Dtransient
// (dim 3, hex8) or HeatTransferElement2Dtransient (dim 2, quad4)
// update(action, u) -> loopOverIntegrationPoints and processActionCode ("K"
// conductivity, "M" capacity) over the reference's Gauss rule, with the
// diagonal conductivity k3 (k11, k22, k33) and capacity cap.  K and M: nnode x
// nnode, upper triangles.  u (nodal values) may be null.
int ref_heat_update(int dim, int nnode, const double* X, const double* k3, double cap, int order, const double* u,
                    const char* action, double* Kout, double* Mout) {
  QuietStdout quiet;
  auto run = [&](auto& e) {
    e.numNodesPerElement = nnode;
    e.numDof = nnode;
    e.setIntegrationOrder(order);
    std::vector<double> coords((size_t)nnode * 3, 0.0);
    for (int a = 0; a < nnode; ++a)
      for (int k = 0; k < dim; ++k) coords[a * 3 + k] = X[a * dim + k];
    std::vector<int> dofs(nnode);
    for (int i = 0; i < nnode; ++i) dofs[i] = i;
    e.coords = coords.data();
    e.edofs = dofs.data();
    TransientElementWorkspace bag;
    double flux_el[3] = {0, 0, 0}, grad_el[3] = {0, 0, 0}, flux_tot[3] = {0, 0, 0}, grad_tot[3] = {0, 0, 0};
    bag.fluxVolume_element = flux_el;
    bag.gradientVolume_element = grad_el;
    bag.fluxVolume_total = flux_tot;
    bag.gradientVolume_total = grad_tot;
    e.bag = &bag;
    Matrix K(nnode, nnode), Ko(nnode, nnode), M(nnode, nnode);
    std::vector<double> fe(nnode, 0.0), fo(nnode, 0.0);
    e.Ke = &K;
    e.Ke_orig = &Ko;
    e.Me = &M;
    e.Fe = fe.data();
    e.F_orig = fo.data();
    HeatTransferMaterial mat;
    mat.saturation = cap;
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) mat.cmat(i, j) = i == j ? k3[i] : 0.0;
    e.material = &mat;
    std::vector<double> uu;
    if (u) uu.assign(u, u + nnode);
    std::string act(action);
    e.update(&act[0], u ? uu.data() : nullptr);
    for (int i = 0; i < nnode; ++i)
      for (int j = 0; j < nnode; ++j) {
        Kout[i * nnode + j] = K(i, j);
        Mout[i * nnode + j] = M(i, j);
      }
    return 0;
  };
  if (dim == 3 && nnode == 8) {
    HeatTransferElement3Dtransient e;
    return run(e);
  }
  if (dim == 2 && nnode == 4) {
    HeatTransferElement2Dtransient e;
    return run(e);
  }
  return 1;
}

// ElasticityElement3D / ElasticityElement2D::getVolAvgValues, the reference's
// post-solve element outputs: out = [volume, stress integral (6), strain
// integral (6), SED (3)] for the element's displacement u (element dofs).
int ref_elastic_vol_avg(int dim, int nnode, const double* X, const double* C, int order, const double* u,
                        double* out) {
  auto run = [&](auto& e, Matrix&, std::vector<double>&, ElasticBag&) {
    std::vector<double> uu(u, u + e.numDof);
    double stress[6] = {0, 0, 0, 0, 0, 0}, strain[6] = {0, 0, 0, 0, 0, 0}, sed[3] = {0, 0, 0}, vol = 0.0;
    e.getVolAvgValues(uu.data(), stress, strain, sed, &vol);
    out[0] = vol;
    for (int k = 0; k < 6; ++k) {
      out[1 + k] = stress[k];
      out[7 + k] = strain[k];
    }
    for (int k = 0; k < 3; ++k) out[13 + k] = sed[k];
    return 0;
  };
  if (dim == 3) return with_elastic<ElasticityElement3D>(3, nnode, X, C, order, run);
  if (dim == 2) return with_elastic<ElasticityElement2D>(2, nnode, X, C, order, run);
  return 1;
}

int ref_gauss_1d(int k, double* x, double* w) {
  GAUSS g(k);
  for (int i = 0; i < k; ++i) { x[i] = g.getCoord(i); w[i] = g.getWeight(i); }
  return 0;
}
int ref_hex_points(int order, double* xi, double* eta, double* zeta, double* w) {
  double *a, *b, *c, *d;
  HexQuadPoints::getQuadraturePointsForHex(order, &a, &b, &c, &d);
  for (int i = 0; i < order * order * order; ++i) { xi[i] = a[i]; eta[i] = b[i]; zeta[i] = c[i]; w[i] = d[i]; }
  return 0;
}
int ref_quad_points(int order, double* xi, double* eta, double* w) {
  double *a, *b, *d;
  QuadQuadPoints::getQuadraturePointsForQuad(order, &a, &b, &d);
  for (int i = 0; i < order * order; ++i) { xi[i] = a[i]; eta[i] = b[i]; w[i] = d[i]; }
  return 0;
}
void ref_shape_hex8(double xi, double eta, double zeta, double* S, double* dxi, double* deta,
                    double* dzeta) {
  shapeHex8(S, xi, eta, zeta);
  derivHex8(dxi, deta, dzeta, xi, eta, zeta);
}
void ref_shape_quad4(double xi, double eta, double* S, double* dxi, double* deta) {
  shapeQuad4(S, xi, eta);
  derivQuad4(dxi, deta, xi, eta);
}
// surface elements of SurfaceLoad::applyTo (8-node quad, 6-node triangle)
void ref_shape_quad8(double xi, double eta, double* S, double* dxi, double* deta) {
  shapeQuad8(S, xi, eta);
  derivQuad8(dxi, deta, xi, eta);
}
void ref_shape_tri6(double xi, double eta, double* S, double* dxi, double* deta) {
  shapeTri6(S, xi, eta);
  derivTri6(dxi, deta, xi, eta);
}
// The reference's own Jacobi-PCG (SymmetricSparseMatrix::solve) on a lower
// triangle read by its own readMatrixAddressFormat from a file in the
// printMatrixAddressFormat layout ("1", "n nnz", then row-wise triples).
// x receives the solution (rhs copied in first: solve overwrites its
// argument); *iterations the CG iterations.  The reference exits the process
// when maxit is reached, so callers pass a generous maxit.
int ref_sparse_solve_file(const char* path, const double* rhs, double eps, int maxit, double* x, int* iterations) {
  std::ifstream is(path);
  int type = 0, n = 0;
  if (!(is >> type >> n) || type != 1 || n <= 0) return 1;
  CountingSparse A(n);
  A.readMatrixAddressFormat(&is);
  A.setSOLUTION_EPSILON(eps);
  A.setMAX_NUMBER_ITERATIONS(maxit);
  for (int i = 0; i < n; ++i) x[i] = rhs[i];
  A.products = 0;
  A.solve(x, 0);
  *iterations = A.products - 1;
  return 0;
}

// HeatTransferElement2Dtransient::addToKe (the reference's own) at one
// integration point: Ke (ndof x ndof, row-major, upper triangle accumulated)
// += the conductivity term for shape-function gradients dx, dy and the
// conductivity matrix [[k11, k12], [k12, k22]], times factor.
int ref_heat2d_add_to_ke(double k11, double k22, double k12, int ndof, const double* dx, const double* dy,
                         double factor, double* Ke) {
  HeatTransferElement2Dtransient e;
  Matrix K(ndof, ndof), c(2, 2);
  for (int i = 0; i < ndof; ++i)
    for (int j = 0; j < ndof; ++j) K(i, j) = Ke[i * ndof + j];
  c(0, 0) = k11;
  c(1, 1) = k22;
  c(0, 1) = c(1, 0) = k12;
  std::vector<double> gx(dx, dx + ndof), gy(dy, dy + ndof), S(ndof, 0.0);
  InterpAndSolDerivatives id;
  id.numberOfInterp = ndof;
  id.S = S.data();
  id.p_S_x1 = gx.data();
  id.p_S_x2 = gy.data();
  e.Ke = &K;
  e.numDof = ndof;
  e.addToKe(&c, &id, factor);
  for (int i = 0; i < ndof; ++i)
    for (int j = 0; j < ndof; ++j) Ke[i * ndof + j] = K(i, j);
  return 0;
}

// HeatTransferElement3Dtransient (the reference's own), one integration point
// of a hex8: addToKe with the 3x3 conductivity k9 (row-major) and addToMe with
// capacity cap, accumulated into K and M (8 x 8 row-major, upper triangles).
int ref_heat3d_add_to_km(const double* k9, double cap, const double* S, const double* dx, const double* dy,
                         const double* dz, double factor, double* K, double* M) {
  HeatTransferElement3Dtransient e;
  Matrix Km(8, 8), Mm(8, 8), c(3, 3);
  for (int i = 0; i < 8; ++i)
    for (int j = 0; j < 8; ++j) { Km(i, j) = K[i * 8 + j]; Mm(i, j) = M[i * 8 + j]; }
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) c(i, j) = k9[i * 3 + j];
  HeatTransferMaterial mat;
  mat.saturation = cap;
  std::vector<double> s(S, S + 8), gx(dx, dx + 8), gy(dy, dy + 8), gz(dz, dz + 8);
  InterpAndSolDerivatives id;
  id.numberOfInterp = 8;
  id.S = s.data();
  id.p_S_x1 = gx.data();
  id.p_S_x2 = gy.data();
  id.p_S_x3 = gz.data();
  e.material = &mat;
  e.Ke = &Km;
  e.Me = &Mm;
  e.numDof = 8;
  e.addToKe(&c, &id, factor);
  e.addToMe(nullptr, &id, factor);
  for (int i = 0; i < 8; ++i)
    for (int j = 0; j < 8; ++j) { K[i * 8 + j] = Km(i, j); M[i * 8 + j] = Mm(i, j); }
  return 0;
}

// ElasticityElement3D (dim 3, 6 strains) or ElasticityElement2D (dim 2,
// 3 strains), the reference's own, at one integration point: see
// elastic_point.  C is the numStrains x numStrains constitutive matrix
// (row-major); u (interleaved nodal displacements) may be null.
int ref_elastic_point(int dim, int nnode, const double* C, const double* dx, const double* dy, const double* dz,
                      const double* u, double factor, double* Ke, double* Fe, double* strain) {
  if (dim == 3) return elastic_point<ElasticityElement3D>(3, nnode, C, dx, dy, dz, u, factor, Ke, Fe, strain);
  if (dim == 2) return elastic_point<ElasticityElement2D>(2, nnode, C, dx, dy, nullptr, u, factor, Ke, Fe, strain);
  return 1;
}

// Hex8 elasticity stiffness of nel elements the way the reference forms it:
// its own HexQuadPoints rule of the given order and shapeHex8/derivHex8, the
// Jacobian J (rows d/dxi, d/deta, d/dzeta of the coordinates), its
// determinant and inverse by cofactors (IsoElement::jacobian,
// isoElement.cpp:250-389, restated: that file does not compile here), then
// ElasticityElement3D::calculateBmatrix + addToKe at every point.  xyz is
// nel x 8 x 3, C36 nel x 6 x 6 (row-major), Ke nel x 24 x 24 (upper
// triangles).  A serial loop, as the reference's SerialAssembler runs it.
int ref_elastic_hex8_ke(int nel, const double* xyz, const double* C36, int order, double* Ke) {
  QuietStdout quiet;  // the Gauss-rule code announces each order it computes
  double *gx, *gy, *gz, *gw;
  HexQuadPoints::getQuadraturePointsForHex(order, &gx, &gy, &gz, &gw);
  const int nip = order * order * order;
  ElasticityElement3D e;
  std::vector<double> brows(6 * 24, 0.0);
  double* rows[6];
  for (int r = 0; r < 6; ++r) rows[r] = brows.data() + r * 24;
  Matrix K(24, 24), c(6, 6);
  InterpAndSolDerivatives id(8, 8);
  id.allocate();
  id.numberOfInterp = 8;
  e.b = rows;
  e.Ke = &K;
  e.numDof = 24;
  double stress[6] = {0, 0, 0, 0, 0, 0};
  for (int el = 0; el < nel; ++el) {
    const double* X = xyz + (size_t)el * 24;
    for (int i = 0; i < 6; ++i)
      for (int j = 0; j < 6; ++j) c(i, j) = C36[(size_t)el * 36 + i * 6 + j];
    for (int i = 0; i < 24; ++i)
      for (int j = 0; j < 24; ++j) K(i, j) = 0.0;
    for (int ip = 0; ip < nip; ++ip) {
      const double det = hex8_point(X, gx[ip], gy[ip], gz[ip], id);
      if (!(det > 0.0)) return 2;
      e.calculateBmatrix(&id, rows);
      e.addToKe(&c, &id, det * gw[ip], stress);
    }
    double* out = Ke + (size_t)el * 576;
    for (int i = 0; i < 24; ++i)
      for (int j = 0; j < 24; ++j) out[i * 24 + j] = K(i, j);
  }
  return 0;
}

// Quad4 plane stiffness of nel elements the way the reference forms it: its
// QuadQuadPoints rule, shapeQuad4/derivQuad4, the 2 x 2 Jacobian restated,
// then ElasticityElement2D::calculateBmatrix + addToKe.  xy nel x 4 x 2, C9
// nel x 3 x 3, Ke nel x 8 x 8 (upper triangles).  A serial loop.
int ref_elastic_quad4_ke(int nel, const double* xy, const double* C9, int order, double* Ke) {
  QuietStdout quiet;
  double *gx, *gy, *gw;
  QuadQuadPoints::getQuadraturePointsForQuad(order, &gx, &gy, &gw);
  const int nip = order * order;
  ElasticityElement2D e;
  std::vector<double> brows(6 * 8, 0.0);
  double* rows[6];
  for (int r = 0; r < 6; ++r) rows[r] = brows.data() + r * 8;
  Matrix K(8, 8), c(3, 3);
  InterpAndSolDerivatives id(4, 4);
  id.allocate();
  id.numberOfInterp = 4;
  e.b = rows;
  e.Ke = &K;
  e.numDof = 8;
  double stress[6] = {0, 0, 0, 0, 0, 0};
  for (int el = 0; el < nel; ++el) {
    const double* X = xy + (size_t)el * 8;
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) c(i, j) = C9[(size_t)el * 9 + i * 3 + j];
    for (int i = 0; i < 8; ++i)
      for (int j = 0; j < 8; ++j) K(i, j) = 0.0;
    for (int ip = 0; ip < nip; ++ip) {
      const double det = quad4_point(X, gx[ip], gy[ip], id);
      if (!(det > 0.0)) return 2;
      e.calculateBmatrix(&id, rows);
      e.addToKe(&c, &id, det * gw[ip], stress);
    }
    double* out = Ke + (size_t)el * 64;
    for (int i = 0; i < 8; ++i)
      for (int j = 0; j < 8; ++j) out[i * 8 + j] = K(i, j);
  }
  return 0;
}

// Hex8 diffusion conductivity of nel elements (steady analyses): addToKe of
// HeatTransferElement3Dtransient with the diagonal conductivity k3 over the
// reference's Gauss rule.  K nel x 8 x 8 (upper triangles).  A serial loop.
int ref_heat_hex8_k(int nel, const double* xyz, const double* k3, int order, double* Kout) {
  QuietStdout quiet;
  double *gx, *gy, *gz, *gw;
  HexQuadPoints::getQuadraturePointsForHex(order, &gx, &gy, &gz, &gw);
  const int nip = order * order * order;
  HeatTransferElement3Dtransient e;
  Matrix K(8, 8), c(3, 3);
  InterpAndSolDerivatives id(8, 8);
  id.allocate();
  id.numberOfInterp = 8;
  e.Ke = &K;
  e.numDof = 8;
  for (int el = 0; el < nel; ++el) {
    const double* X = xyz + (size_t)el * 24;
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) c(i, j) = i == j ? k3[(size_t)el * 3 + i] : 0.0;
    for (int i = 0; i < 8; ++i)
      for (int j = 0; j < 8; ++j) K(i, j) = 0.0;
    for (int ip = 0; ip < nip; ++ip) {
      const double det = hex8_point(X, gx[ip], gy[ip], gz[ip], id);
      if (!(det > 0.0)) return 2;
      e.addToKe(&c, &id, det * gw[ip]);
    }
    double* out = Kout + (size_t)el * 64;
    for (int i = 0; i < 8; ++i)
      for (int j = 0; j < 8; ++j) out[i * 8 + j] = K(i, j);
  }
  return 0;
}

// The element side of DiffusionModel's step for nel hex8 diffusion elements,
// as the reference forms it: per element K (addToKe, diagonal conductivity
// k3) and M (addToMe, capacity cap) over its own HexQuadPoints rule and
// shapeHex8/derivHex8 with the Jacobian restated as in ref_elastic_hex8_ke,
// then formK_s (Mbar = (a1 K + M)/dt) and formF_s_new (F = -(a1+a2)/dt K u_s).
// xyz nel x 8 x 3, k3 nel x 3, cap nel, u_s nel x 8 (the element's nodal
// values); Mbar nel x 8 x 8 (upper triangles), F nel x 8.  A serial loop.
int ref_heat_hex8_step_terms(int nel, const double* xyz, const double* k3, const double* cap, int order,
                             const double* u_s, double a1, double a2, double dt, double* Mbar, double* F) {
  QuietStdout quiet;
  double *gx, *gy, *gz, *gw;
  HexQuadPoints::getQuadraturePointsForHex(order, &gx, &gy, &gz, &gw);
  const int nip = order * order * order;
  HeatTransferElement3Dtransient e;
  Matrix K(8, 8), M(8, 8), Kb(8, 8), c(3, 3);
  HeatTransferMaterial mat;
  InterpAndSolDerivatives id(8, 8);
  id.allocate();
  id.numberOfInterp = 8;
  std::vector<double> fe(8), us(8);
  int dofs[8] = {0, 1, 2, 3, 4, 5, 6, 7};
  e.material = &mat;
  e.Ke = &K;
  e.Me = &M;
  e.Ke_orig = &Kb;
  e.Fe = fe.data();
  e.dofList = dofs;
  e.numDof = 8;
  Array<double> ap(2);
  ap[0] = a1;
  ap[1] = a2;
  for (int el = 0; el < nel; ++el) {
    const double* X = xyz + (size_t)el * 24;
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) c(i, j) = i == j ? k3[(size_t)el * 3 + i] : 0.0;
    mat.saturation = cap[el];
    for (int i = 0; i < 8; ++i)
      for (int j = 0; j < 8; ++j) K(i, j) = M(i, j) = Kb(i, j) = 0.0;
    for (int ip = 0; ip < nip; ++ip) {
      const double det = hex8_point(X, gx[ip], gy[ip], gz[ip], id);
      if (!(det > 0.0)) return 2;
      e.addToKe(&c, &id, det * gw[ip]);
      e.addToMe(nullptr, &id, det * gw[ip]);
    }
    for (int i = 0; i < 8; ++i) {
      us[i] = u_s[(size_t)el * 8 + i];
      fe[i] = 0.0;
    }
    e.formK_s(ap, dt);
    e.formF_s_new(ap, us.data(), nullptr, nullptr, dt);
    for (int i = 0; i < 8; ++i) {
      F[(size_t)el * 8 + i] = fe[i];
      for (int j = 0; j < 8; ++j) Mbar[(size_t)el * 64 + i * 8 + j] = Kb(i, j);
    }
  }
  return 0;
}

// The element side of one backward-Euler step (DiffusionModel with a1, a2):
// formK_s gives Mbar = (a1 K + M)/dt, formF_s_new F = -(a1+a2)/dt K u_s, from
// the element's K and M (upper triangles, n x n row-major) and its nodal u_s.
// n = 8 for the hex8 element; n = 4 for the quad4 element, which inherits
// both from HeatTransferElement3Dtransient.
int ref_heat_step_terms(int n, const double* K, const double* M, const double* u_s, double a1, double a2, double dt,
                        double* Mbar, double* F) {
  if (n < 1 || n > 27) return 1;
  HeatTransferElement3Dtransient e;
  Matrix Km(n, n), Mm(n, n), Kb(n, n);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) { Km(i, j) = K[i * n + j]; Mm(i, j) = M[i * n + j]; }
  std::vector<double> fe(n, 0.0), us(u_s, u_s + n);
  std::vector<int> dofs(n);
  for (int i = 0; i < n; ++i) dofs[i] = i;
  e.Ke = &Km;
  e.Me = &Mm;
  e.Ke_orig = &Kb;
  e.Fe = fe.data();
  e.dofList = dofs.data();
  e.numDof = n;
  Array<double> ap(2);
  ap[0] = a1;
  ap[1] = a2;
  e.formK_s(ap, dt);
  e.formF_s_new(ap, us.data(), nullptr, nullptr, dt);
  for (int i = 0; i < n; ++i) {
    F[i] = fe[i];
    for (int j = 0; j < n; ++j) Mbar[i * n + j] = Kb(i, j);
  }
  return 0;
}
int ref_heat3d_step_terms(const double* K, const double* M, const double* u_s, double a1, double a2, double dt,
                          double* Mbar, double* F) {
  return ref_heat_step_terms(8, K, M, u_s, a1, a2, dt, Mbar, F);
}

// A lower triangle (0-based CSR, diagonal last in each row) written by the
// reference's own SymmetricSparseMatrix printers: format 1
// printMatrixAddressFormat, 2 printMatrixAddressFormatUpper, 3
// printCompressedRowFormat.
int ref_print_lower(const char* path, int format, int n, const long long* rp, const int* col, const double* val) {
  SymmetricSparseMatrix A(n);
  for (int i = 0; i < n; ++i)
    for (long long k = rp[i]; k < rp[i + 1]; ++k) A.specifyNonZeroLocation(i, col[k]);
  A.allocate();
  for (int i = 0; i < n; ++i)
    for (long long k = rp[i]; k < rp[i + 1]; ++k) A(i, col[k]) = val[k];
  std::ofstream os(path);
  char msg[1] = {0};
  if (format == 1) A.printMatrixAddressFormat(msg, &os);
  else if (format == 2) A.printMatrixAddressFormatUpper(msg, &os);
  else if (format == 3) A.printCompressedRowFormat(msg, &os);
  else return 1;
  return os.good() ? 0 : 1;
}

// The reference's CSR writers and readers (SparseMatrixUtility.cpp).
int ref_write_csr(const char* path, int binary, int n, int nnz, const int* ia_in, const int* ja_in,
                  const double* a_in) {
  int* ia = const_cast<int*>(ia_in);
  int* ja = const_cast<int*>(ja_in);
  double* a = const_cast<double*>(a_in);
  std::string p(path);
  if (binary) writeCSRMatrixInBinary(&p[0], ia, ja, a, n, nnz);
  else writeCSRMatrixInASCII(&p[0], ia, ja, a, n, nnz);
  return 0;
}
// Call with ia == NULL for *n and *nnz, then with arrays of n+1, nnz, nnz.
int ref_read_csr(const char* path, int binary, int* n, int* nnz, int* ia_out, int* ja_out, double* a_out) {
  int *ia = nullptr, *ja = nullptr, nn = 0, nz = 0;
  double* a = nullptr;
  std::string p(path);
  if (binary) {
    readCSRMatrixInBinary(&p[0], ia, ja, a, nn, nz);
  } else {
    readCSRMatrixInASCII(&p[0], ia, ja, a, nn);
    nz = ia ? ia[nn] - ia[0] : 0;
  }
  *n = nn;
  *nnz = nz;
  if (ia_out) {
    for (int i = 0; i <= nn; ++i) ia_out[i] = ia[i];
    for (int k = 0; k < nz; ++k) { ja_out[k] = ja[k]; a_out[k] = a[k]; }
  }
  delete[] ia;
  delete[] ja;
  delete[] a;
  return 0;
}
}
