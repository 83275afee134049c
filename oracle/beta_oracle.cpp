// beta_oracle.cpp -- TEST INFRASTRUCTURE ONLY (the checker, never the product).
//
// A CPU restatement, in FP64, of BETA's element-assembly and Jacobi-PCG path.
// Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load
// this library; the GPU product path never calls into it.
//
// Every routine names the reference function it restates (path within the
// kaushik-d/BetaNoOx tree).  The loop orders of the reference are kept where
// they decide floating-point summation order (addMatrix, the PCG sweeps), so
// the oracle reproduces the reference's arithmetic, not just its mathematics.
//
// Parity pins: Gauss points/weights and shape functions are checked against
// the reference's own gauss.cpp/shape.cpp compiled under oracle/_ref; the
// dense LU inverse is checked against the known answer printed by the
// reference's DEBUG_MATRIX_CLASS main (beta/math/matrix.cpp:694-696).

#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>
#include <thread>
#include <functional>

// Minimal static-schedule parallel loop on std::thread (no OpenMP runtime is
// loaded into the test process).  Partial sums are combined in thread order,
// so results are deterministic for a fixed thread count.
static int g_threads = 1;
static void par_for(int n, const std::function<void(int, int, int)>& body) {
  int t = g_threads < 1 ? 1 : g_threads;
  if (t == 1 || n < 4096) { body(0, n, 0); return; }
  std::vector<std::thread> th;
  for (int k = 0; k < t; ++k) {
    int lo = (int)((long long)n * k / t), hi = (int)((long long)n * (k + 1) / t);
    th.emplace_back(body, lo, hi, k);
  }
  for (auto& x : th) x.join();
}

extern "C" {

enum {
  OR_OK = 0,
  OR_ERR_ARG = 1,
  OR_ERR_NEG_DIAG = 6,   // BasicElement::checkForNegativeDiagonal / CheckAndFixZeroDiagonal
  OR_ERR_ZERO_DIAG = 7,  // LargeMatrix::CheckAndFixZeroDiagonal without replacement value
  OR_ERR_MAXIT = 4,      // sparse.cpp:225-229 "Solution not converged"
  OR_ERR_LOAD_ON_RESTRAINED = 12,  // equation.cpp:858-861
  OR_ERR_PATTERN = 13,   // sparse.cpp:91-97 "not on row"
};

// ---------------------------------------------------------------------------
// Gauss-Legendre points by Newton iteration on P_k.
// Restates GAUSS::GAUSS (beta/math/gaussQuadrature/gauss.cpp:14-60): same
// starting guess cos(pi*(i+0.75)/(k+0.5)), same three-term recurrence, same
// EPS = 3e-15 stop test, same weight formula 2/((1-z^2) P'^2), and the same
// placement x[i] = -z, x[k-1-i] = +z.
int oracle_gauss_1d(int k, double* x, double* w) {
  if (k < 1 || k > 32 || !x || !w) return OR_ERR_ARG;
  const double EPS = 3e-15;
  const int half = (k + 1) / 2;
  for (int i = 0; i < half; ++i) {
    double z = std::cos(M_PI * ((double)i + 1 - .25) / ((double)k + .5));
    double znew, dp, pk;
    for (;;) {
      double pkm1 = 0.0;
      pk = 1.0;
      for (int j = 0; j < k; ++j) {  // P_{j+1} = ((2j+1) z P_j - j P_{j-1}) / (j+1)
        double pkm2 = pkm1;
        pkm1 = pk;
        pk = ((2 * j + 1) * z * pkm1 - (j)*pkm2) / (j + 1);
      }
      dp = k * (z * pk - pkm1) / (z * z - 1);
      znew = z - pk / dp;
      bool done = std::fabs(znew - z) <= EPS;
      z = znew;
      if (done) break;
    }
    x[i] = 0.0 - 1.0 * z;
    x[k - i - 1] = 0.0 + 1.0 * z;
    w[i] = 2 * 1.0 / ((1 - z * z) * dp * dp);
    w[k - i - 1] = w[i];
  }
  return OR_OK;
}

// Tensor-product lists.  HexQuadPoints::getQuadraturePointsForHex
// (gauss.cpp:303-365): xi outermost, zeta innermost, w = (wxi*weta)*wzeta.
// QuadQuadPoints::getQuadraturePointsForQuad (gauss.cpp:825-877): xi outer.
int oracle_hex_points(int order, double* xi, double* eta, double* zeta, double* w) {
  double g[32], gw[32];
  int st = oracle_gauss_1d(order, g, gw);
  if (st) return st;
  int ip = 0;
  for (int i = 0; i < order; ++i)
    for (int j = 0; j < order; ++j)
      for (int k = 0; k < order; ++k, ++ip) {
        xi[ip] = g[i]; eta[ip] = g[j]; zeta[ip] = g[k];
        w[ip] = gw[i] * gw[j] * gw[k];
      }
  return OR_OK;
}

int oracle_quad_points(int order, double* xi, double* eta, double* w) {
  double g[32], gw[32];
  int st = oracle_gauss_1d(order, g, gw);
  if (st) return st;
  int ip = 0;
  for (int i = 0; i < order; ++i)
    for (int k = 0; k < order; ++k, ++ip) {
      xi[ip] = g[i]; eta[ip] = g[k]; w[ip] = gw[i] * gw[k];
    }
  return OR_OK;
}

// ---------------------------------------------------------------------------
// Trilinear / bilinear shape functions in BETA's local node order.
// hex8 (shape.cpp:210-260, BasicElement.cpp:518-525): nodes 0-3 on xi=-1 with
// (eta,zeta) = (-,-),(+,-),(+,+),(-,+); nodes 4-7 the same on xi=+1.
// quad4 (shape.cpp:147-168): counter-clockwise from (-,-).
static const int kHexSign[8][3] = {{-1, -1, -1}, {-1, 1, -1}, {-1, 1, 1}, {-1, -1, 1},
                                   {1, -1, -1},  {1, 1, -1},  {1, 1, 1},  {1, -1, 1}};
static const int kQuadSign[4][2] = {{-1, -1}, {1, -1}, {1, 1}, {-1, 1}};

void oracle_shape_hex8(double xi, double eta, double zeta, double* S, double* dxi,
                       double* deta, double* dzeta) {
  for (int a = 0; a < 8; ++a) {
    double fx = 1 + kHexSign[a][0] * xi, fy = 1 + kHexSign[a][1] * eta,
           fz = 1 + kHexSign[a][2] * zeta;
    if (S) S[a] = fx * fy * fz / 8;
    if (dxi) dxi[a] = kHexSign[a][0] * fy * fz / 8;
    if (deta) deta[a] = kHexSign[a][1] * fx * fz / 8;
    if (dzeta) dzeta[a] = kHexSign[a][2] * fx * fy / 8;
  }
}

void oracle_shape_quad4(double xi, double eta, double* S, double* dxi, double* deta) {
  for (int a = 0; a < 4; ++a) {
    double fx = 1 + kQuadSign[a][0] * xi, fy = 1 + kQuadSign[a][1] * eta;
    if (S) S[a] = .25 * fx * fy;
    if (dxi) dxi[a] = .25 * kQuadSign[a][0] * fy;
    if (deta) deta[a] = .25 * kQuadSign[a][1] * fx;
  }
}

// ---------------------------------------------------------------------------
// Dense inverse (Matrix::invert, beta/math/matrix.cpp:350-370, with its
// ludcmp :272-348 and lubksb :393-431).  The reference factors by Crout's
// method with implicit partial pivoting, the published algorithm of Press et
// al., Numerical Recipes in C, 2nd ed., sect. 2.3: each row is scaled by the
// reciprocal of its largest magnitude for the pivot search only, column j
// first finishes U(0..j-1, j) and then the candidates L(j.., j), the pivot is
// the last row of largest scaled magnitude, and the sub-diagonal column is
// multiplied by the reciprocal pivot (a zero pivot becomes 1e-20).  Each
// identity column is then solved by forward substitution (starting at its
// first nonzero) and back substitution.  The sums run in the same order as
// the reference's so that constitutive matrices come out bit-identical.
// A is row-major n x n, overwritten with its inverse.
int oracle_invert(int n, double* A) {
  if (n < 1 || n > 16 || !A) return OR_ERR_ARG;
  std::vector<double> a(A, A + n * n), scale(n), x(n);
  std::vector<int> piv(n);
  auto at = [&](int r, int c) -> double& { return a[r * n + c]; };
  for (int r = 0; r < n; ++r) {
    double big = 0.0;
    for (int c = 0; c < n; ++c) big = std::max(big, std::fabs(at(r, c)));
    if (big == 0.0) return OR_ERR_ZERO_DIAG;
    scale[r] = 1.0 / big;
  }
  for (int j = 0; j < n; ++j) {
    for (int r = 0; r < j; ++r) {
      double sum = at(r, j);
      for (int k = 0; k < r; ++k) sum -= at(r, k) * at(k, j);
      at(r, j) = sum;
    }
    double best = 0.0;
    int p = j;
    for (int r = j; r < n; ++r) {
      double sum = at(r, j);
      for (int k = 0; k < j; ++k) sum -= at(r, k) * at(k, j);
      at(r, j) = sum;
      const double score = scale[r] * std::fabs(sum);
      if (score >= best) { best = score; p = r; }
    }
    if (p != j) {
      for (int c = 0; c < n; ++c) std::swap(at(p, c), at(j, c));
      scale[p] = scale[j];
    }
    piv[j] = p;
    if (at(j, j) == 0.0) at(j, j) = 1e-20;
    if (j != n - 1) {
      const double rcp = 1.0 / at(j, j);
      for (int r = j + 1; r < n; ++r) at(r, j) *= rcp;
    }
  }
  std::vector<double> inv(n * n);
  for (int col = 0; col < n; ++col) {
    std::fill(x.begin(), x.end(), 0.0);
    x[col] = 1.0;
    int first = -1;
    for (int r = 0; r < n; ++r) {
      double sum = x[piv[r]];
      x[piv[r]] = x[r];
      if (first >= 0)
        for (int k = first; k < r; ++k) sum -= at(r, k) * x[k];
      else if (sum != 0.0)
        first = r;
      x[r] = sum;
    }
    for (int r = n - 1; r >= 0; --r) {
      double sum = x[r];
      for (int k = r + 1; k < n; ++k) sum -= at(r, k) * x[k];
      x[r] = sum / at(r, r);
    }
    for (int r = 0; r < n; ++r) inv[r * n + col] = x[r];
  }
  std::memcpy(A, inv.data(), sizeof(double) * n * n);
  return OR_OK;
}

// 3D elastic constitutive matrix from the nine engineering constants
// (E11,E22,E33,nu12,nu23,nu13,G12,G23,G13), Voigt order xx,yy,zz,xy,yz,xz:
// compliance S as ElasticMaterial::read "readModuli" fills it
// (beta/materials/3D/elastic.cpp:358-366), then C = S^-1 (:368-369).
int oracle_cmat_ortho3d(const double* m9, double* C36) {
  double S[36] = {0};
  S[0 * 6 + 0] = 1 / m9[0];
  S[0 * 6 + 1] = S[1 * 6 + 0] = -m9[3] / m9[0];
  S[0 * 6 + 2] = S[2 * 6 + 0] = -m9[5] / m9[0];
  S[1 * 6 + 1] = 1 / m9[1];
  S[2 * 6 + 1] = S[1 * 6 + 2] = -m9[4] / m9[1];
  S[2 * 6 + 2] = 1 / m9[2];
  S[3 * 6 + 3] = 1 / m9[6];
  S[4 * 6 + 4] = 1 / m9[7];
  S[5 * 6 + 5] = 1 / m9[8];
  int st = oracle_invert(6, S);
  if (st) return st;
  std::memcpy(C36, S, sizeof(S));
  return OR_OK;
}

// oracle_cmat_ortho3d for n materials (m9: n x 9, C36: n x 36); 0 or the first
// failing status.
int oracle_cmat_ortho3d_many(int n, const double* m9, double* C36) {
  for (int e = 0; e < n; ++e) {
    const int st = oracle_cmat_ortho3d(m9 + (size_t)e * 9, C36 + (size_t)e * 36);
    if (st) return st;
  }
  return 0;
}

// Plane-stress C from (E11,E22,nu12,G12) (beta/materials/2D/pStress.cpp:68-85).
void oracle_cmat_plane_stress(const double* m4, double* C9) {
  double s11 = 1 / m4[0], s12 = -m4[2] / m4[0], s22 = 1. / m4[1], s66 = 1. / m4[3];
  double den = s11 * s22 - s12 * s12;
  C9[0] = s22 / den; C9[1] = -s12 / den; C9[2] = 0.;
  C9[3] = -s12 / den; C9[4] = s11 / den; C9[5] = 0.;
  C9[6] = 0.; C9[7] = 0.; C9[8] = 1. / s66;
}

// ---------------------------------------------------------------------------
// Geometry at one integration point: IsoElement::interpolation + jacobian
// (beta/elements/isoElement.cpp:392-433, 250-372).  M[r][c] = sum_a dN_a/dxi_r
// * X_a[c]; global gradients g = M^-1 dN/dxi through the cofactor inverse.
static double jac3(const double* xyz, const double* d0, const double* d1, const double* d2,
                   double g[3][8]) {
  double M[3][3] = {{0}};
  const double* d[3] = {d0, d1, d2};
  for (int a = 0; a < 8; ++a)
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) M[r][c] += d[r][a] * xyz[3 * a + c];
  double c00 = M[1][1] * M[2][2] - M[1][2] * M[2][1];
  double c01 = M[1][2] * M[2][0] - M[1][0] * M[2][2];
  double c02 = M[1][0] * M[2][1] - M[1][1] * M[2][0];
  double det = M[0][0] * c00 + M[0][1] * c01 + M[0][2] * c02;
  double inv = 1. / det;
  double Mi[3][3];
  Mi[0][0] = c00 * inv;
  Mi[1][0] = c01 * inv;
  Mi[2][0] = c02 * inv;
  Mi[0][1] = (M[0][2] * M[2][1] - M[0][1] * M[2][2]) * inv;
  Mi[1][1] = (M[0][0] * M[2][2] - M[0][2] * M[2][0]) * inv;
  Mi[2][1] = (M[0][1] * M[2][0] - M[0][0] * M[2][1]) * inv;
  Mi[0][2] = (M[0][1] * M[1][2] - M[0][2] * M[1][1]) * inv;
  Mi[1][2] = (M[0][2] * M[1][0] - M[0][0] * M[1][2]) * inv;
  Mi[2][2] = (M[0][0] * M[1][1] - M[0][1] * M[1][0]) * inv;
  for (int a = 0; a < 8; ++a)
    for (int c = 0; c < 3; ++c)
      g[c][a] = Mi[c][0] * d0[a] + Mi[c][1] * d1[a] + Mi[c][2] * d2[a];
  return det;
}

static double jac2(const double* xy, const double* d0, const double* d1, double g[2][4]) {
  double J00 = 0, J01 = 0, J10 = 0, J11 = 0;
  for (int a = 0; a < 4; ++a) {
    J00 += d0[a] * xy[2 * a]; J01 += d0[a] * xy[2 * a + 1];
    J10 += d1[a] * xy[2 * a]; J11 += d1[a] * xy[2 * a + 1];
  }
  double det = J00 * J11 - J01 * J10, t = 1 / det;
  double i00 = J11 * t, i01 = -J01 * t, i10 = -J10 * t, i11 = J00 * t;
  for (int a = 0; a < 4; ++a) {
    g[0][a] = i00 * d0[a] + i01 * d1[a];
    g[1][a] = i10 * d0[a] + i11 * d1[a];
  }
  return det;
}

// Strain-displacement rows for one node, engineering shear.
// hex8 Voigt xx,yy,zz,xy,yz,xz (ElasticityElement3D::calculateBmatrix,
// ElasticityElement3D.cpp:57-81); quad4 xx,yy,xy (ElasticityElement2D.cpp:88-101).
static void bmat3(const double g[3][8], double B[6][24]) {
  std::memset(B, 0, sizeof(double) * 6 * 24);
  for (int a = 0; a < 8; ++a) {
    int c = 3 * a;
    B[0][c] = g[0][a];
    B[1][c + 1] = g[1][a];
    B[2][c + 2] = g[2][a];
    B[3][c] = g[1][a]; B[3][c + 1] = g[0][a];
    B[4][c + 1] = g[2][a]; B[4][c + 2] = g[1][a];
    B[5][c] = g[2][a]; B[5][c + 2] = g[0][a];
  }
}

// ---------------------------------------------------------------------------
// Element stiffness, hex8 linear elasticity: ElasticityElement3D::update("K")
// -> loopOverIntegrationPoints -> addToKe (ElasticityElement3D.cpp:983-1030,
// 560-611).  Only the upper triangle (j >= i) of the 24x24 row-major Ke is
// written, as in the reference; integration factor = detJ * w (unit
// thickness).  Returns OR_ERR_NEG_DIAG if a diagonal term is <= 0
// (BasicElement::checkForNegativeDiagonal, BasicElement.cpp:116-130).
int oracle_ke_hex8(const double* xyz24, const double* C36, int order, double* Ke) {
  double xi[64], eta[64], zeta[64], w[64];
  if (order < 1 || order > 4) return OR_ERR_ARG;
  oracle_hex_points(order, xi, eta, zeta, w);
  for (int i = 0; i < 24; ++i)
    for (int j = i; j < 24; ++j) Ke[i * 24 + j] = 0.;
  int nip = order * order * order;
  for (int ip = 0; ip < nip; ++ip) {
    double d0[8], d1[8], d2[8], g[3][8], B[6][24];
    oracle_shape_hex8(xi[ip], eta[ip], zeta[ip], nullptr, d0, d1, d2);
    double det = jac3(xyz24, d0, d1, d2, g);
    double f = det * w[ip];
    bmat3(g, B);
    double CB[6][24];
    for (int ii = 0; ii < 24; ++ii)
      for (int k = 0; k < 6; ++k) {
        double s = 0;
        for (int m = 0; m < 6; ++m) s += B[m][ii] * C36[m * 6 + k];
        CB[k][ii] = s;
      }
    for (int ii = 0; ii < 24; ++ii)
      for (int jj = ii; jj < 24; ++jj) {
        double s = 0;
        for (int k = 0; k < 6; ++k) s += CB[k][ii] * B[k][jj];
        Ke[ii * 24 + jj] += s * f;
      }
  }
  for (int i = 0; i < 24; ++i)
    if (Ke[i * 24 + i] <= 0) return OR_ERR_NEG_DIAG;
  return OR_OK;
}

// quad4 plane elasticity: ElasticityElement2D::addToKe (:22-58) on the shared
// Gauss loop; 8x8 upper triangle, dof order (ux,uy) per node.
int oracle_ke_quad4(const double* xy8, const double* C9, int order, double* Ke) {
  double xi[16], eta[16], w[16];
  if (order < 1 || order > 4) return OR_ERR_ARG;
  oracle_quad_points(order, xi, eta, w);
  for (int i = 0; i < 8; ++i)
    for (int j = i; j < 8; ++j) Ke[i * 8 + j] = 0.;
  for (int ip = 0; ip < order * order; ++ip) {
    double d0[4], d1[4], g[2][4];
    oracle_shape_quad4(xi[ip], eta[ip], nullptr, d0, d1);
    double f = jac2(xy8, d0, d1, g) * w[ip];
    double B[3][8] = {{0}};
    for (int a = 0; a < 4; ++a) {
      B[0][2 * a] = g[0][a];
      B[1][2 * a + 1] = g[1][a];
      B[2][2 * a] = g[1][a]; B[2][2 * a + 1] = g[0][a];
    }
    double CB[3][8];
    for (int ii = 0; ii < 8; ++ii)
      for (int k = 0; k < 3; ++k)
        CB[k][ii] = B[0][ii] * C9[0 * 3 + k] + B[1][ii] * C9[1 * 3 + k] + B[2][ii] * C9[2 * 3 + k];
    for (int ii = 0; ii < 8; ++ii)
      for (int jj = ii; jj < 8; ++jj)
        Ke[ii * 8 + jj] += (CB[0][ii] * B[0][jj] + CB[1][ii] * B[1][jj] + CB[2][ii] * B[2][jj]) * f;
  }
  for (int i = 0; i < 8; ++i)
    if (Ke[i * 8 + i] <= 0) return OR_ERR_NEG_DIAG;
  return OR_OK;
}

// hex8 diffusion: conductivity K = int grad N^T k grad N and capacity
// M = int c N N^T (HeatTransferElement3Dtransient::addToKe :153-197,
// addToMe :60-77, loop :665-698).  Upper triangles of 8x8 row-major K and M.
int oracle_km_hex8_heat(const double* xyz24, const double* k9, double c, int order, double* K,
                        double* M) {
  double xi[64], eta[64], zeta[64], w[64];
  if (order < 1 || order > 4) return OR_ERR_ARG;
  oracle_hex_points(order, xi, eta, zeta, w);
  for (int i = 0; i < 8; ++i)
    for (int j = 0; j < 8; ++j) K[i * 8 + j] = M[i * 8 + j] = 0.;
  int nip = order * order * order;
  for (int ip = 0; ip < nip; ++ip) {
    double S[8], d0[8], d1[8], d2[8], g[3][8];
    oracle_shape_hex8(xi[ip], eta[ip], zeta[ip], S, d0, d1, d2);
    double f = jac3(xyz24, d0, d1, d2, g) * w[ip];
    for (int i = 0; i < 8; ++i)
      for (int j = i; j < 8; ++j) {
        double kg0 = g[0][j] * k9[0] + g[1][j] * k9[1] + g[2][j] * k9[2];
        double kg1 = g[0][j] * k9[3] + g[1][j] * k9[4] + g[2][j] * k9[5];
        double kg2 = g[0][j] * k9[6] + g[1][j] * k9[7] + g[2][j] * k9[8];
        K[i * 8 + j] += (kg0 * g[0][i] + kg1 * g[1][i] + kg2 * g[2][i]) * f;
        M[i * 8 + j] += S[i] * S[j] * f * c;
      }
  }
  return OR_OK;
}

// quad4 diffusion: the 2D transient element's conductivity
// K = int grad N^T k grad N (HeatTransferElement2Dtransient::addToKe,
// HeatTransferElement2DTransient.cpp:67-108, k11/k12/k22 of the material's
// conductivity matrix; k12 = 0 for the unrotated orthotropic
// HeatTransferMaterial) and capacity M = int c N N^T, unit thickness.  Upper
// triangles of 4x4 row-major K and M.
int oracle_km_quad4_heat(const double* xy8, const double* k4, double c, int order, double* K, double* M) {
  double xi[16], eta[16], w[16];
  if (order < 1 || order > 4) return OR_ERR_ARG;
  oracle_quad_points(order, xi, eta, w);
  for (int i = 0; i < 16; ++i) K[i] = M[i] = 0.;
  for (int ip = 0; ip < order * order; ++ip) {
    double S[4], d0[4], d1[4], g[2][4];
    oracle_shape_quad4(xi[ip], eta[ip], S, d0, d1);
    double f = jac2(xy8, d0, d1, g) * w[ip];
    for (int i = 0; i < 4; ++i)
      for (int j = i; j < 4; ++j) {
        double kg0 = g[0][j] * k4[0] + g[1][j] * k4[1];
        double kg1 = g[0][j] * k4[2] + g[1][j] * k4[3];
        K[i * 4 + j] += (kg0 * g[0][i] + kg1 * g[1][i]) * f;
        M[i * 4 + j] += S[i] * S[j] * f * c;
      }
  }
  return OR_OK;
}

// Internal force of one hex8 element for nodal displacements ue[24]:
// strain = B ue (ElasticityElement3D::derivativesOfFields/calculateStrain
// :124-207), stress = C strain (ElasticMaterial::calculateStress,
// elastic.cpp:411-451, no hygrothermal strain), Fe += B^T stress * detJ*w
// (addToFe :41-55).
int oracle_fe_hex8(const double* xyz24, const double* C36, int order, const double* ue,
                   double* Fe) {
  double xi[64], eta[64], zeta[64], w[64];
  if (order < 1 || order > 4) return OR_ERR_ARG;
  oracle_hex_points(order, xi, eta, zeta, w);
  for (int i = 0; i < 24; ++i) Fe[i] = 0;
  int nip = order * order * order;
  for (int ip = 0; ip < nip; ++ip) {
    double d0[8], d1[8], d2[8], g[3][8], B[6][24];
    oracle_shape_hex8(xi[ip], eta[ip], zeta[ip], nullptr, d0, d1, d2);
    double f = jac3(xyz24, d0, d1, d2, g) * w[ip];
    bmat3(g, B);
    double eps[6], sig[6];
    for (int k = 0; k < 6; ++k) {
      double s = 0;
      for (int i = 0; i < 24; ++i) s += B[k][i] * ue[i];
      eps[k] = s;
    }
    for (int k = 0; k < 6; ++k) {
      double s = 0;
      for (int m = 0; m < 6; ++m) s += C36[k * 6 + m] * eps[m];
      sig[k] = s;
    }
    for (int i = 0; i < 24; ++i) {
      double s = 0.;
      for (int k = 0; k < 6; ++k) s += B[k][i] * sig[k];
      Fe[i] += s * f;
    }
  }
  return OR_OK;
}

// ---------------------------------------------------------------------------
// Geometric-nonlinear hex8: ElasticityElement3D with analysisType
// GEOMETRIC_NONLINEAR, the element of BasicModel::iterate.  At each
// integration point: the displacement gradient H_kj = sum_a dN_a/dx_j u_a,k
// (derivativesOfFields, ElasticityElement3D.cpp:162-207); B with the
// displacement-gradient terms added to the linear rows (calculateBmatrix
// :84-119); the Green-Lagrange strain in engineering shear (calculateStrain
// :124-160); stress = C strain (no hygrothermal strain); the tangent Ke +=
// (C B)^T B f with the initial-stress term K_sigma (addToKe :560-641, upper
// triangle) and Fe += B^T stress f (addToFe :41-55); f = detJ * w.  Either
// output may be null.  Same operation order as the reference's code.
int oracle_gnl_hex8(const double* xyz24, const double* C36, int order, const double* ue, double* Ke, double* Fe) {
  double xi[64], eta[64], zeta[64], w[64];
  if (order < 1 || order > 4) return OR_ERR_ARG;
  oracle_hex_points(order, xi, eta, zeta, w);
  if (Ke)
    for (int i = 0; i < 24; ++i)
      for (int j = i; j < 24; ++j) Ke[i * 24 + j] = 0.;
  if (Fe)
    for (int i = 0; i < 24; ++i) Fe[i] = 0.;
  const int nip = order * order * order;
  for (int ip = 0; ip < nip; ++ip) {
    double d0[8], d1[8], d2[8], g[3][8], B[6][24];
    oracle_shape_hex8(xi[ip], eta[ip], zeta[ip], nullptr, d0, d1, d2);
    const double f = jac3(xyz24, d0, d1, d2, g) * w[ip];
    // H[k][j] = du_k/dx_j
    double H[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    for (int a = 0; a < 8; ++a)
      for (int k = 0; k < 3; ++k)
        for (int j = 0; j < 3; ++j) H[k][j] += g[j][a] * ue[3 * a + k];
    bmat3(g, B);
    for (int a = 0; a < 8; ++a) {
      const double dg1 = g[0][a], dg2 = g[1][a], dg3 = g[2][a];
      for (int k = 0; k < 3; ++k) {
        const int c = 3 * a + k;
        B[0][c] += H[k][0] * dg1;
        B[1][c] += H[k][1] * dg2;
        B[2][c] += H[k][2] * dg3;
        B[3][c] += H[k][0] * dg2 + H[k][1] * dg1;
        B[4][c] += H[k][1] * dg3 + H[k][2] * dg2;
        B[5][c] += H[k][0] * dg3 + H[k][2] * dg1;
      }
    }
    double eps[6];
    eps[0] = H[0][0];
    eps[1] = H[1][1];
    eps[2] = H[2][2];
    eps[3] = H[0][1] + H[1][0];
    eps[4] = H[1][2] + H[2][1];
    eps[5] = H[0][2] + H[2][0];
    eps[0] += .5 * (H[0][0] * H[0][0] + H[1][0] * H[1][0] + H[2][0] * H[2][0]);
    eps[1] += .5 * (H[0][1] * H[0][1] + H[1][1] * H[1][1] + H[2][1] * H[2][1]);
    eps[2] += .5 * (H[0][2] * H[0][2] + H[1][2] * H[1][2] + H[2][2] * H[2][2]);
    eps[3] += H[0][0] * H[0][1] + H[1][0] * H[1][1] + H[2][0] * H[2][1];
    eps[4] += H[0][1] * H[0][2] + H[1][1] * H[1][2] + H[2][1] * H[2][2];
    eps[5] += H[0][0] * H[0][2] + H[1][0] * H[1][2] + H[2][0] * H[2][2];
    double sig[6];
    for (int k = 0; k < 6; ++k) {
      double s = 0;
      for (int m = 0; m < 6; ++m) s += C36[k * 6 + m] * eps[m];
      sig[k] = s;
    }
    if (Ke) {
      double CB[6][24];
      for (int ii = 0; ii < 24; ++ii)
        for (int k = 0; k < 6; ++k) {
          double s = 0;
          for (int m = 0; m < 6; ++m) s += B[m][ii] * C36[m * 6 + k];
          CB[k][ii] = s;
        }
      for (int ii = 0; ii < 24; ++ii)
        for (int jj = ii; jj < 24; ++jj) {
          double s = 0;
          for (int k = 0; k < 6; ++k) s += CB[k][ii] * B[k][jj];
          Ke[ii * 24 + jj] += s * f;
        }
      for (int a = 0; a < 8; ++a)
        for (int b = a; b < 8; ++b) {
          const double b11 = sig[0] * g[0][a] * g[0][b] + sig[1] * g[1][a] * g[1][b] + sig[2] * g[2][a] * g[2][b] +
                             sig[3] * (g[0][a] * g[1][b] + g[1][a] * g[0][b]) +
                             sig[4] * (g[1][a] * g[2][b] + g[2][a] * g[1][b]) +
                             sig[5] * (g[0][a] * g[2][b] + g[2][a] * g[0][b]);
          const double v = b11 * f;
          for (int k = 0; k < 3; ++k) Ke[(3 * a + k) * 24 + 3 * b + k] += v;
        }
    }
    if (Fe)
      for (int i = 0; i < 24; ++i) {
        double s = 0.;
        for (int k = 0; k < 6; ++k) s += B[k][i] * sig[k];
        Fe[i] += s * f;
      }
  }
  if (Ke)
    for (int i = 0; i < 24; ++i)
      if (Ke[i * 24 + i] <= 0) return OR_ERR_NEG_DIAG;
  return OR_OK;
}

// ---------------------------------------------------------------------------
// Equations + SymmetricSparseMatrix (default storage "SPARSE").
// Storage: per row a sorted column list of J <= I (SortedList<int>), values in
// the same order; the diagonal is the last entry of each row
// (beta/math/equation/sparse.cpp:15-24, 144, 479-495).
struct OracleSystem {
  int n = 0;
  std::vector<std::vector<int>> row;
  std::vector<std::vector<double>> mat;
  std::vector<unsigned char> rest;
  std::vector<double> solution, loadVector, pseudoLoad, lastSolution;
  bool allocated = false;
  double zeroDiagReplacement = 0.0;

  double* find(int I, int J) {
    auto& r = row[I];
    auto it = std::lower_bound(r.begin(), r.end(), J);
    if (it == r.end() || *it != J) return nullptr;
    return &mat[I][it - r.begin()];
  }
};

void* oracle_sys_create(int n) {
  if (n <= 0) return nullptr;
  auto* s = new OracleSystem();
  s->n = n;
  s->row.resize(n);
  s->rest.assign(n, 0);
  s->solution.assign(n, 0.0);
  s->loadVector.assign(n, 0.0);
  s->pseudoLoad.assign(n, 0.0);
  s->lastSolution.assign(n, 0.0);
  return s;
}

void oracle_sys_destroy(void* h) { delete (OracleSystem*)h; }

// The zero-diagonal replacement value (Equations::setReplaceZeroDiagonal_Option
// passed on to LargeMatrix; 0 = none, a zero diagonal is then an error).
void oracle_sys_set_zero_diag(void* h, double v) { ((OracleSystem*)h)->zeroDiagReplacement = v; }

// Restraints and prescribed values: Equations::setRestraint / setSolution
// (equation.cpp:306-341).  Loads: Equations::addLoadToEqn (:851-868) -- a
// nonzero load on a restrained dof is a fatal error in the reference.
int oracle_sys_set_bc(void* h, const unsigned char* restrained, const double* prescribed,
                      const double* load) {
  auto* s = (OracleSystem*)h;
  for (int i = 0; i < s->n; ++i) {
    s->rest[i] = restrained ? (restrained[i] != 0) : 0;
    if (s->rest[i]) s->solution[i] = prescribed ? prescribed[i] : 0.0;
  }
  for (int i = 0; i < s->n; ++i) s->loadVector[i] = 0.0;
  if (load)
    for (int i = 0; i < s->n; ++i) {
      if (s->rest[i]) {
        if (load[i] != 0.0) return OR_ERR_LOAD_ON_RESTRAINED;
      } else {
        s->loadVector[i] += load[i];
      }
    }
  return OR_OK;
}

// Equations::specifyNonZeroLocation (equation.cpp:1216-1267), without the
// additional-equation (MPC) branches: (I,J) for unrestrained I >= J of the
// same element, (I,I) for restrained I.
void oracle_sys_specify(void* h, const int* map, int size) {
  auto* s = (OracleSystem*)h;
  for (int i = 0; i < size; ++i) {
    int I = map[i];
    for (int j = 0; j < size; ++j) {
      int J = map[j];
      int add = -1;
      if (s->rest[J]) {
        if (I == J) add = I;
      } else if (s->rest[I]) {
      } else if (I >= J) {
        add = J;
      }
      if (add >= 0) {
        auto& r = s->row[I];
        auto it = std::lower_bound(r.begin(), r.end(), add);
        if (it == r.end() || *it != add) r.insert(it, add);
      }
    }
  }
}

// SymmetricSparseMatrix::allocate (sparse.cpp:482-495): empty rows get a
// diagonal; Equations::zeroMatrix (equation.cpp:387-396).
void oracle_sys_allocate(void* h) {
  auto* s = (OracleSystem*)h;
  s->mat.resize(s->n);
  for (int i = 0; i < s->n; ++i) {
    if (s->row[i].empty()) s->row[i].push_back(i);
    s->mat[i].assign(s->row[i].size(), 0.0);
  }
  std::fill(s->pseudoLoad.begin(), s->pseudoLoad.end(), 0.0);
  s->allocated = true;
}

void oracle_sys_zero(void* h) {
  auto* s = (OracleSystem*)h;
  for (auto& m : s->mat) std::fill(m.begin(), m.end(), 0.0);
  std::fill(s->pseudoLoad.begin(), s->pseudoLoad.end(), 0.0);
}

long long oracle_sys_nnz(void* h) {
  auto* s = (OracleSystem*)h;
  long long t = 0;
  for (auto& r : s->row) t += (long long)r.size();
  return t;
}

// Equations::addMatrix (equation.cpp:445-562) without MPC branches.
// `Ke` is size x size row-major with a valid upper triangle; force may be
// null.  Symmetric elimination: K(I,J) += Ke for unrestrained I >= J,
// F[I] -= Ke_IJ * u_J for unrestrained I and restrained J, K(I,I) = 1 for
// restrained I.
int oracle_sys_add_matrix(void* h, const double* Ke, const int* map, int size,
                          const double* force) {
  auto* s = (OracleSystem*)h;
  double* F = s->pseudoLoad.data();
  const unsigned char* rest = s->rest.data();
  for (int i = 0; i < size; ++i) {
    int I = map[i];
    if (force) {
      if (!rest[I]) F[I] += force[i];
    }
    for (int j = 0; j < size; ++j) {
      double kij = (i < j) ? Ke[i * size + j] : Ke[j * size + i];
      int J = map[j];
      if (rest[J]) {
        if (I == J) {
          double* p = s->find(I, I);
          if (!p) return OR_ERR_PATTERN;
          *p = 1;
        }
        if (!rest[I]) F[I] -= kij * s->solution[J];
      } else if (rest[I]) {
      } else if (I >= J) {
        double* p = s->find(I, J);
        if (!p) return OR_ERR_PATTERN;
        *p += kij;
      }
    }
  }
  return OR_OK;
}

// Lower-triangle export in the reference's row order (the layout written by
// SymmetricSparseMatrix::printMatrixAddressFormat, sparse.cpp:295-325).
void oracle_sys_export_lower(void* h, long long* rowptr, int* col, double* val) {
  auto* s = (OracleSystem*)h;
  long long p = 0;
  for (int i = 0; i < s->n; ++i) {
    if (rowptr) rowptr[i] = p;
    for (size_t k = 0; k < s->row[i].size(); ++k, ++p) {
      if (col) col[p] = s->row[i][k];
      if (val) val[p] = s->mat.empty() ? 0.0 : s->mat[i][k];
    }
  }
  if (rowptr) rowptr[s->n] = p;
}

void oracle_sys_pseudo_load(void* h, double* out) {
  auto* s = (OracleSystem*)h;
  std::memcpy(out, s->pseudoLoad.data(), sizeof(double) * s->n);
}

// y = A x from lower rows: row i contributes to y[i] and, off the diagonal,
// to y[col] (SymmetricSparseMatrix::vectorProduct, sparse.cpp:452-478).
static void lower_spmv(OracleSystem* s, double* y, const double* x) {
  const int L = s->n;
  for (int i = 0; i < L; ++i) y[i] = 0;
  for (int i = 0; i < L; ++i) {
    int nt = (int)s->row[i].size() - 1;
    if (nt < 0) continue;
    const std::vector<int>& cols = s->row[i];
    const double* m = s->mat[i].data();
    double xi = x[i], acc = 0;
    for (int j = 0; j < nt; ++j) {
      acc += m[j] * x[cols[j]];
      y[cols[j]] += m[j] * xi;
    }
    y[i] += m[nt] * x[cols[nt]] + acc;
    if (cols[nt] != i) y[cols[nt]] += m[nt] * xi;
  }
}

void oracle_sys_vector_product(void* h, const double* x, double* y) {
  lower_spmv((OracleSystem*)h, y, x);
}

struct OracleSolveStats {
  int status;
  int iterations;
  double last_norm;  // sqrt(r.r / x.x) at exit
};

// LargeMatrix::CheckAndFixZeroDiagonal (largeMatrix.cpp:43-79).
static int check_diag(OracleSystem* s) {
  bool zero = false;
  for (int i = 0; i < s->n; ++i) {
    double d = s->mat[i].back();
    if (s->row[i].back() != i) d = 0;
    if (d == 0) { zero = true; break; }
    if (d < 0) return OR_ERR_NEG_DIAG;
  }
  if (zero) {
    if (s->zeroDiagReplacement == 0) return OR_ERR_ZERO_DIAG;
    for (int i = 0; i < s->n; ++i)
      if (s->row[i].back() == i && s->mat[i].back() == 0) s->mat[i].back() = s->zeroDiagReplacement;
  }
  return OR_OK;
}

// Jacobi-PCG, SymmetricSparseMatrix::solve (sparse.cpp:114-242): b is
// overwritten with the solution; x0 may be null (zero guess).  Stop when
// sqrt(r.r / x.x) < eps (:202-223, x = current iterate, r = recursively
// updated residual).  The five vector sweeps keep the reference's order.
static int pcg_ref(OracleSystem* s, double* b, const double* x0, double eps, int maxit,
                   OracleSolveStats* st) {
  int ds = check_diag(s);
  if (ds) { if (st) st->status = ds; return ds; }
  const int L = s->n;
  std::vector<double> x(L), r(L), p(L), q(L), tmp(L), diag(L);
  for (int i = 0; i < L; ++i) diag[i] = s->mat[i].back();
  for (int i = 0; i < L; ++i) x[i] = x0 ? x0[i] : 0;
  lower_spmv(s, r.data(), x.data());
  for (int i = 0; i < L; ++i) r[i] = b[i] - r[i];
  for (int i = 0; i < L; ++i) p[i] = q[i] = r[i] / diag[i];
  for (int i = 0; i < L; ++i) b[i] = x0 ? x0[i] : 0;
  int it = 0;
  bool conv = false;
  double lastnorm = 0;
  while (!conv && it < maxit) {
    double pAp = 0, rq = 0, newrq = 0, rnorm = 0, xnorm = 0;
    lower_spmv(s, tmp.data(), p.data());
    for (int i = 0; i < L; ++i) { pAp += p[i] * tmp[i]; rq += r[i] * q[i]; }
    double a = rq / pAp;
    for (int i = 0; i < L; ++i) b[i] += a * p[i];
    for (int i = 0; i < L; ++i) r[i] -= a * tmp[i];
    for (int i = 0; i < L; ++i) q[i] = r[i] / diag[i];
    for (int i = 0; i < L; ++i) newrq += r[i] * q[i];
    double bk = newrq / rq;
    for (int i = 0; i < L; ++i) p[i] = q[i] + bk * p[i];
    for (int i = 0; i < L; ++i) rnorm += r[i] * r[i];
    for (int i = 0; i < L; ++i) xnorm += b[i] * b[i];
    ++it;
    lastnorm = std::sqrt(rnorm / xnorm);
    if (lastnorm < eps) conv = true;
  }
  if (st) { st->iterations = it; st->last_norm = lastnorm; st->status = conv ? OR_OK : OR_ERR_MAXIT; }
  return conv ? OR_OK : OR_ERR_MAXIT;
}

// Equations::solve (equation.cpp:1288-1405) for the default storage:
// solution = load + pseudoLoad on unrestrained dofs, prescribed values stay on
// restrained dofs; initial guess = init_guess (restrained dofs take their
// prescribed value, :1371-1377) or lastSolution (:1379).  `out` receives the
// solution (may alias nothing inside the system).
int oracle_sys_solve(void* h, const double* init_guess, double eps, int maxit, double* out,
                     OracleSolveStats* st) {
  auto* s = (OracleSystem*)h;
  const int L = s->n;
  for (int i = 0; i < L; ++i)
    if (!s->rest[i]) s->solution[i] = s->loadVector[i] + s->pseudoLoad[i];
  std::vector<double> guess(L);
  if (init_guess) {
    for (int i = 0; i < L; ++i) guess[i] = s->rest[i] ? s->solution[i] : init_guess[i];
  } else {
    guess = s->lastSolution;
  }
  std::vector<double> b = s->solution;
  int rc = pcg_ref(s, b.data(), guess.data(), eps, maxit, st);
  if (rc == OR_OK || rc == OR_ERR_MAXIT) {
    for (int i = 0; i < L; ++i) {
      // equation.cpp:1396-1399: lastSolution only follows entries that moved.
      if (std::fabs(guess[i] - b[i]) > 1e-9) s->lastSolution[i] = b[i];
    }
    if (out) std::memcpy(out, b.data(), sizeof(double) * L);
    // The reference solves in place in `solution` (equation.cpp:1377-1379).
    s->solution = b;
  }
  return rc;
}

// The right-hand side Equations::solve hands to the matrix (load + pseudo
// load, prescribed values on restrained rows), without solving.
void oracle_sys_rhs(void* h, double* out) {
  auto* s = (OracleSystem*)h;
  for (int i = 0; i < s->n; ++i)
    out[i] = s->rest[i] ? s->solution[i] : s->loadVector[i] + s->pseudoLoad[i];
}

// ---------------------------------------------------------------------------
// Mesh-level drivers: SerialAssembler::assembleK (SerialAssembler.cpp:35-59)
// with BasicElement::calculateDofList (BasicElement.cpp:49-68: dof of local
// node a, component j = first_dof[node] + j) and the pattern step
// BasicModel::allocateEquationsMatrix (BasicModel.cpp:1022-1033).
//
// kind: 1 = quad4 plane stress (4 params/elem: E11,E22,nu12,G12)
//       2 = hex8 elasticity (9 params/elem: readModuli order)
//       3 = hex8 heat K+M (4 params/elem: k11,k22,k33,c)
static void elem_dofs(int nnpe, int ndpn, const int* conn_e, const int* first_dof, int* map) {
  int k = 0;
  for (int a = 0; a < nnpe; ++a)
    for (int j = 0; j < ndpn; ++j) map[k++] = first_dof[conn_e[a]] + j;
}

void oracle_sys_specify_mesh(void* h, int nelem, int nnpe, int ndpn, const int* conn,
                             const int* first_dof) {
  int map[64];
  for (int e = 0; e < nelem; ++e) {
    elem_dofs(nnpe, ndpn, conn + (size_t)e * nnpe, first_dof, map);
    oracle_sys_specify(h, map, nnpe * ndpn);
  }
}

static void gather_xyz(int nnpe, int ndim, const int* conn_e, const double* xyz, double* out) {
  for (int a = 0; a < nnpe; ++a)
    for (int c = 0; c < ndim; ++c) out[ndim * a + c] = xyz[(size_t)conn_e[a] * ndim + c];
}

int oracle_element_matrix(int kind, const double* xe, const double* params, int order, double* Ke,
                          double* Me) {
  if (kind == 1) {
    double C9[9];
    oracle_cmat_plane_stress(params, C9);
    return oracle_ke_quad4(xe, C9, order, Ke);
  } else if (kind == 2) {
    double C36[36];
    int st = oracle_cmat_ortho3d(params, C36);
    if (st) return st;
    return oracle_ke_hex8(xe, C36, order, Ke);
  } else if (kind == 3) {
    double k9[9] = {params[0], 0, 0, 0, params[1], 0, 0, 0, params[2]};
    double Mtmp[64];
    return oracle_km_hex8_heat(xe, k9, params[3], order, Ke, Me ? Me : Mtmp);
  } else if (kind == 4) {
    double k4[4] = {params[0], 0, 0, params[1]};
    double Mtmp[16];
    return oracle_km_quad4_heat(xe, k4, params[3], order, Ke, Me ? Me : Mtmp);
  }
  return OR_ERR_ARG;
}

int oracle_sys_assemble_mesh(void* h, int kind, int nelem, int nnpe, int ndpn, int ndim,
                             const int* conn, const double* xyz, const int* first_dof,
                             const double* params, int nparams, int order) {
  double xe[24], Ke[24 * 24], Me[64];
  int map[64];
  oracle_sys_zero(h);
  for (int e = 0; e < nelem; ++e) {
    const int* ce = conn + (size_t)e * nnpe;
    gather_xyz(nnpe, ndim, ce, xyz, xe);
    int st = oracle_element_matrix(kind, xe, params + (size_t)e * nparams, order, Ke, Me);
    if (st) return st;
    elem_dofs(nnpe, ndpn, ce, first_dof, map);
    st = oracle_sys_add_matrix(h, Ke, map, nnpe * ndpn, nullptr);
    if (st) return st;
  }
  return OR_OK;
}

// oracle_sys_assemble_mesh with the element matrices of each block of
// elements computed on all threads first; they are then added in element
// order, so the assembled system is bit-identical to the serial one.
int oracle_sys_assemble_mesh_threaded(void* h, int kind, int nelem, int nnpe, int ndpn, int ndim,
                                      const int* conn, const double* xyz, const int* first_dof,
                                      const double* params, int nparams, int order, int threads) {
  g_threads = threads > 0 ? threads : (int)std::thread::hardware_concurrency();
  if (g_threads > 256) g_threads = 256;
  const int nd = nnpe * ndpn;
  const int block = std::max(1, std::min(nelem, 16384));
  std::vector<double> K((size_t)block * nd * nd);
  oracle_sys_zero(h);
  for (int e0 = 0; e0 < nelem; e0 += block) {
    const int e1 = std::min(nelem, e0 + block);
    std::vector<int> err(256, 0);
    par_for(e1 - e0, [&](int lo, int hi, int t) {
      double xe[24], Me[64];
      for (int k = lo; k < hi; ++k) {
        const int e = e0 + k;
        gather_xyz(nnpe, ndim, conn + (size_t)e * nnpe, xyz, xe);
        const int st = oracle_element_matrix(kind, xe, params + (size_t)e * nparams, order,
                                             K.data() + (size_t)k * nd * nd, Me);
        if (st && !err[t]) err[t] = st;
      }
    });
    for (int v : err)
      if (v) return v;
    int map[64];
    for (int e = e0; e < e1; ++e) {
      elem_dofs(nnpe, ndpn, conn + (size_t)e * nnpe, first_dof, map);
      const int st = oracle_sys_add_matrix(h, K.data() + (size_t)(e - e0) * nd * nd, map, nd, nullptr);
      if (st) return st;
    }
  }
  return OR_OK;
}

// The geometric-nonlinear tangent at total displacement u assembled through
// addMatrix (BasicModel::assembleK(currentSolution) with analysisType
// GEOMETRIC_NONLINEAR).
int oracle_sys_assemble_gnl(void* h, int nelem, const int* conn, const double* xyz, const int* first_dof,
                            const double* params, int order, const double* u) {
  double xe[24], ue[24], Ke[24 * 24], C36[36];
  int map[24];
  oracle_sys_zero(h);
  for (int e = 0; e < nelem; ++e) {
    const int* ce = conn + (size_t)e * 8;
    gather_xyz(8, 3, ce, xyz, xe);
    elem_dofs(8, 3, ce, first_dof, map);
    for (int i = 0; i < 24; ++i) ue[i] = u[map[i]];
    int st = oracle_cmat_ortho3d(params + (size_t)e * 9, C36);
    if (st) return st;
    st = oracle_gnl_hex8(xe, C36, order, ue, Ke, nullptr);
    if (st) return st;
    st = oracle_sys_add_matrix(h, Ke, map, 24, nullptr);
    if (st) return st;
  }
  return OR_OK;
}

// The geometric-nonlinear internal force sum_e Fe(u) over all rows (the
// restraint mapping left to the caller).
int oracle_fint_gnl(int nelem, const int* conn, const double* xyz, const int* first_dof, const double* params,
                    int order, const double* u, double* f, int n) {
  double xe[24], ue[24], Fe[24], C36[36];
  int map[24];
  for (int i = 0; i < n; ++i) f[i] = 0.0;
  for (int e = 0; e < nelem; ++e) {
    const int* ce = conn + (size_t)e * 8;
    gather_xyz(8, 3, ce, xyz, xe);
    elem_dofs(8, 3, ce, first_dof, map);
    for (int i = 0; i < 24; ++i) ue[i] = u[map[i]];
    int st = oracle_cmat_ortho3d(params + (size_t)e * 9, C36);
    if (st) return st;
    oracle_gnl_hex8(xe, C36, order, ue, nullptr, Fe);
    for (int i = 0; i < 24; ++i) f[map[i]] += Fe[i];
  }
  return OR_OK;
}

// BasicModel::iterate (BasicModel.cpp:1244-1381) for hex8 elasticity with
// analysisType GEOMETRIC_NONLINEAR, on a system whose restraints and loads are
// set: from the total displacement u (restrained entries hold their
// prescribed values), each Newton iteration
//   * sums the element forces Fe(u) into the resultant (getGlobalForces,
//     BasicModel.cpp:1063-1110; assembleResultantVector skips restrained
//     rows) and forms the residual R = load - resultant on free rows, 0 on
//     restrained ones (calculateResidualNorm, equation.cpp:1516-1529);
//   * stops once max |R| < max_residual (BasicModel.cpp:1292);
//   * assembles the tangent Ke(u) through addMatrix (assembleK(currentSolution));
//   * solves K d = R with the reference's PCG and stop rule from the initial
//     guess u itself, restrained entries their prescribed values
//     (incrementalSolutionUsingResidual, equation.cpp:1638-1703);
//   * adds d to the free entries of u (addIncrementalDisplacements :1707-1720).
// history[it] = max |R| of iteration it (up to max_newton + 1 entries);
// *iters = Newton solves done; *lin_iters = PCG iterations in all.
int oracle_newton_hex8(void* h, int nelem, const int* conn, const double* xyz, const int* first_dof,
                       const double* params, int order, double* u, double max_residual, int max_newton, double eps,
                       int maxit, double* history, int* iters, int* lin_iters) {
  auto* s = (OracleSystem*)h;
  const int L = s->n;
  std::vector<double> res(L), R(L), guess(L);
  double xe[24], ue[24], Ke[24 * 24], Fe[24], C36[36];
  int map[24];
  int total_lin = 0, it = 0;
  bool conv = false;
  for (;; ++it) {
    std::fill(res.begin(), res.end(), 0.0);
    for (int e = 0; e < nelem; ++e) {
      const int* ce = conn + (size_t)e * 8;
      gather_xyz(8, 3, ce, xyz, xe);
      elem_dofs(8, 3, ce, first_dof, map);
      for (int i = 0; i < 24; ++i) ue[i] = u[map[i]];
      int st = oracle_cmat_ortho3d(params + (size_t)e * 9, C36);
      if (st) return st;
      oracle_gnl_hex8(xe, C36, order, ue, nullptr, Fe);
      for (int i = 0; i < 24; ++i)
        if (!s->rest[map[i]]) res[map[i]] += Fe[i];
    }
    double mx = 0.0;
    for (int i = 0; i < L; ++i) {
      R[i] = s->rest[i] ? 0.0 : s->loadVector[i] - res[i];
      if (std::fabs(R[i]) > mx) mx = std::fabs(R[i]);
    }
    if (history) history[it] = mx;
    conv = mx < max_residual;
    if (conv || it >= max_newton) break;
    oracle_sys_zero(h);
    for (int e = 0; e < nelem; ++e) {
      const int* ce = conn + (size_t)e * 8;
      gather_xyz(8, 3, ce, xyz, xe);
      elem_dofs(8, 3, ce, first_dof, map);
      for (int i = 0; i < 24; ++i) ue[i] = u[map[i]];
      oracle_cmat_ortho3d(params + (size_t)e * 9, C36);
      int st = oracle_gnl_hex8(xe, C36, order, ue, Ke, nullptr);
      if (st) return st;
      st = oracle_sys_add_matrix(h, Ke, map, 24, nullptr);
      if (st) return st;
    }
    for (int i = 0; i < L; ++i) guess[i] = u[i];
    OracleSolveStats ls;
    std::memset(&ls, 0, sizeof(ls));
    int rc = pcg_ref(s, R.data(), guess.data(), eps, maxit, &ls);
    total_lin += ls.iterations;
    if (rc != OR_OK) {
      if (iters) *iters = it;
      if (lin_iters) *lin_iters = total_lin;
      return rc;
    }
    for (int i = 0; i < L; ++i)
      if (!s->rest[i]) u[i] += R[i];
  }
  if (iters) *iters = it;
  if (lin_iters) *lin_iters = total_lin;
  return conv ? OR_OK : OR_ERR_MAXIT;
}

// Global internal force f_int = sum_e Fe(u_e) (BasicModel::CalculateResidual,
// BasicModel.cpp:1035-1061; Equations::assembleResultantVector,
// equation.cpp:790-807, which skips restrained rows).  hex8 elasticity only.
int oracle_internal_force_hex8(int nelem, const int* conn, const double* xyz,
                               const int* first_dof, const double* params, int order,
                               const unsigned char* restrained, const double* u, double* fint) {
  double xe[24], ue[24], Fe[24], C36[36];
  int map[24];
  for (int e = 0; e < nelem; ++e) {
    const int* ce = conn + (size_t)e * 8;
    gather_xyz(8, 3, ce, xyz, xe);
    elem_dofs(8, 3, ce, first_dof, map);
    for (int i = 0; i < 24; ++i) ue[i] = u[map[i]];
    int st = oracle_cmat_ortho3d(params + (size_t)e * 9, C36);
    if (st) return st;
    oracle_fe_hex8(xe, C36, order, ue, Fe);
    for (int i = 0; i < 24; ++i)
      if (!restrained || !restrained[map[i]]) fint[map[i]] += Fe[i];
  }
  return OR_OK;
}

// Element volume integrals after a solve: ElasticityElement3D::getVolAvgValues
// (ElasticityElement3D.cpp:417-558) -- per integration point dV = detJ * w
// (unit thickness), strain = B u_e (engineering shear), stress = C strain,
// and the sums volume += dV, stress_int += stress dV, strain_int += strain dV,
// energy += 0.5 stress.strain dV.  The quad4 plane-stress element gets the
// same integrals with its 3 components (ElasticityElement2D).  ns = 6 (hex8)
// or 3 (quad4); out rows: [volume, stress_int[ns], strain_int[ns], energy].
int oracle_element_outputs(int kind, int nelem, const int* conn, const double* xyz, const int* first_dof,
                           const double* params, int order, const double* u, double* out) {
  const bool hex = kind == 2;
  if (!hex && kind != 1) return OR_ERR_ARG;
  if (order < 1 || order > 4) return OR_ERR_ARG;
  const int nnpe = hex ? 8 : 4, ndim = hex ? 3 : 2, ns = hex ? 6 : 3, nd = nnpe * ndim;
  double xi[64], eta[64], zeta[64], w[64];
  int nip;
  if (hex) {
    oracle_hex_points(order, xi, eta, zeta, w);
    nip = order * order * order;
  } else {
    oracle_quad_points(order, xi, eta, w);
    nip = order * order;
  }
  for (int e = 0; e < nelem; ++e) {
    const int* ce = conn + (size_t)e * nnpe;
    double xe[24], ue[24], C[36];
    int map[24];
    gather_xyz(nnpe, ndim, ce, xyz, xe);
    elem_dofs(nnpe, ndim, ce, first_dof, map);
    for (int i = 0; i < nd; ++i) ue[i] = u[map[i]];
    if (hex) {
      int st = oracle_cmat_ortho3d(params + (size_t)e * 9, C);
      if (st) return st;
    } else {
      oracle_cmat_plane_stress(params + (size_t)e * 4, C);
    }
    double* o = out + (size_t)e * (2 * ns + 2);
    for (int k = 0; k < 2 * ns + 2; ++k) o[k] = 0.0;
    for (int ip = 0; ip < nip; ++ip) {
      double eps[6] = {0}, sig[6] = {0}, dv;
      if (hex) {
        double d0[8], d1[8], d2[8], g[3][8], B[6][24];
        oracle_shape_hex8(xi[ip], eta[ip], zeta[ip], nullptr, d0, d1, d2);
        dv = jac3(xe, d0, d1, d2, g) * w[ip];
        bmat3(g, B);
        for (int k = 0; k < 6; ++k)
          for (int i = 0; i < 24; ++i) eps[k] += B[k][i] * ue[i];
      } else {
        double d0[4], d1[4], g[2][4];
        oracle_shape_quad4(xi[ip], eta[ip], nullptr, d0, d1);
        dv = jac2(xe, d0, d1, g) * w[ip];
        for (int a = 0; a < 4; ++a) {  // ElasticityElement2D::calculateBmatrix rows xx, yy, xy
          eps[0] += g[0][a] * ue[2 * a];
          eps[1] += g[1][a] * ue[2 * a + 1];
          eps[2] += g[1][a] * ue[2 * a] + g[0][a] * ue[2 * a + 1];
        }
      }
      for (int k = 0; k < ns; ++k)
        for (int m = 0; m < ns; ++m) sig[k] += C[k * ns + m] * eps[m];
      o[0] += dv;
      for (int k = 0; k < ns; ++k) {
        o[1 + k] += sig[k] * dv;
        o[1 + ns + k] += eps[k] * dv;
        o[1 + 2 * ns] += 0.5 * sig[k] * eps[k] * dv;
      }
    }
  }
  return OR_OK;
}

// One backward-Euler family step of DiffusionModel::DoTransientNonLinearAnalysis
// (DiffusionModel.cpp:743-818) with linear conductivity:
//   a1 = alpha*dt, a2 = (1-alpha)*dt                                  (:745-746)
//   per element "KM": Mbar_e = (a1*K_e + M_e)/dt (formK_s, :323-350),
//   F_e = -(a1+a2) K_e u_s / dt (formF_s_new, :372-405), addMatrix(Mbar, F)
//   delta = solve(initGuess = u_s)                                     (:786)
//   u_s <- u_s + delta                                                 (:800-818)
// Restraints/prescribed values must already be set (they prescribe delta).
int oracle_heat_step(void* h, int kind, int nelem, const int* conn, const double* xyz, const int* first_dof,
                     const double* params, int order, double dt, double alpha, double* u_s,
                     double eps, int maxit, OracleSolveStats* st) {
  auto* s = (OracleSystem*)h;
  if (kind != 3 && kind != 4) return OR_ERR_ARG;
  const int nn = kind == 3 ? 8 : 4, ndim = kind == 3 ? 3 : 2;  // hex8 / quad4 diffusion
  double a1 = alpha * dt, a2 = (1 - alpha) * dt;
  double xe[24], K[64], M[64], Mbar[64], Fe[8];
  int map[8];
  oracle_sys_zero(h);
  for (int e = 0; e < nelem; ++e) {
    const int* ce = conn + (size_t)e * nn;
    gather_xyz(nn, ndim, ce, xyz, xe);
    int rc = oracle_element_matrix(kind, xe, params + (size_t)e * 4, order, K, M);
    if (rc) return rc;
    elem_dofs(nn, 1, ce, first_dof, map);
    for (int i = 0; i < nn; ++i)
      for (int j = 0; j < nn; ++j) Mbar[i * nn + j] = (a1 * K[i * nn + j] + M[i * nn + j]) / dt;
    for (int i = 0; i < nn; ++i) {
      double acc = 0.0;
      for (int j = 0; j < nn; ++j) {
        double Ku = (j >= i ? K[i * nn + j] : K[j * nn + i]) * u_s[map[j]];
        acc += -(a1 + a2) * Ku;
      }
      Fe[i] = acc / dt;
    }
    rc = oracle_sys_add_matrix(h, Mbar, map, nn, Fe);
    if (rc) return rc;
  }
  std::vector<double> delta(s->n);
  int rc = oracle_sys_solve(h, u_s, eps, maxit, delta.data(), st);
  if (rc) return rc;
  for (int i = 0; i < s->n; ++i) u_s[i] += delta[i];
  return OR_OK;
}

// ---------------------------------------------------------------------------
// Multi-core CPU variant for timing (the "all host cores" baseline): the same
// arithmetic, restructured the way BETA's ESA assembler divides work
// (ESA_Assembler.cpp:9-68: element matrices computed by contiguous element
// ranges, then each thread adds only the rows it owns, equation.cpp:2029-2216)
// and a threaded CSR Jacobi-PCG with the reference stopping rule.  The
// threaded PCG keeps full (both-triangle) CSR rows so every row is
// independent.
struct OracleCsr {
  int n;
  std::vector<long long> rp;
  std::vector<int> ci;
  std::vector<double> v;
};

void* oracle_csr_from_sys(void* h) {
  auto* s = (OracleSystem*)h;
  auto* c = new OracleCsr();
  c->n = s->n;
  std::vector<long long> cnt(s->n + 1, 0);
  for (int i = 0; i < s->n; ++i)
    for (int j : s->row[i]) {
      cnt[i]++;
      if (j != i) cnt[j]++;
    }
  c->rp.assign(s->n + 1, 0);
  for (int i = 0; i < s->n; ++i) c->rp[i + 1] = c->rp[i] + cnt[i];
  c->ci.resize(c->rp[s->n]);
  c->v.resize(c->rp[s->n]);
  std::vector<long long> fill(c->rp.begin(), c->rp.end() - 1);
  for (int i = 0; i < s->n; ++i)
    for (size_t k = 0; k < s->row[i].size(); ++k) {
      int j = s->row[i][k];
      double m = s->mat[i][k];
      c->ci[fill[i]] = j; c->v[fill[i]++] = m;
      if (j != i) { c->ci[fill[j]] = i; c->v[fill[j]++] = m; }
    }
  return c;
}

void oracle_csr_destroy(void* c) { delete (OracleCsr*)c; }

// The full (both-triangle) CSR of a lower triangle given as 0-based CSR rows
// (rp n+1, col, val), as SymmetricSparseMatrix stores it (sparse.cpp:479-495).
void* oracle_csr_from_lower(int n, const long long* rp, const int* col, const double* val) {
  auto* c = new OracleCsr();
  c->n = n;
  std::vector<long long> cnt(n + 1, 0);
  for (int i = 0; i < n; ++i)
    for (long long k = rp[i]; k < rp[i + 1]; ++k) {
      cnt[i]++;
      if (col[k] != i) cnt[col[k]]++;
    }
  c->rp.assign(n + 1, 0);
  for (int i = 0; i < n; ++i) c->rp[i + 1] = c->rp[i] + cnt[i];
  c->ci.resize(c->rp[n]);
  c->v.resize(c->rp[n]);
  std::vector<long long> fill(c->rp.begin(), c->rp.end() - 1);
  for (int i = 0; i < n; ++i)
    for (long long k = rp[i]; k < rp[i + 1]; ++k) {
      const int j = col[k];
      c->ci[fill[i]] = j; c->v[fill[i]++] = val[k];
      if (j != i) { c->ci[fill[j]] = i; c->v[fill[j]++] = val[k]; }
    }
  return c;
}

// The threaded Jacobi-PCG with a choice of stop rule: rule 0 is the
// reference's sqrt(r.r / x.x) < eps (sparse.cpp:223), rule 1 is
// sqrt(r.r / b.b) < eps.  trace (may be null) receives the reference rule's
// quantity sqrt(r.r / x.x) after each of the first trace_len iterations.
int oracle_csr_pcg_threaded_rule(void* hc, const double* b, double* x, double eps, int maxit, int threads,
                                 int rule, double* trace, int trace_len, OracleSolveStats* st);

int oracle_csr_pcg_threaded(void* hc, const double* b, double* x, double eps, int maxit,
                            int threads, OracleSolveStats* st) {
  return oracle_csr_pcg_threaded_rule(hc, b, x, eps, maxit, threads, 0, nullptr, 0, st);
}

int oracle_csr_pcg_threaded_rule(void* hc, const double* b, double* x, double eps, int maxit, int threads,
                                 int rule, double* trace, int trace_len, OracleSolveStats* st) {
  auto* c = (OracleCsr*)hc;
  const int n = c->n;
  g_threads = threads > 0 ? threads : (int)std::thread::hardware_concurrency();
  if (g_threads > 256) g_threads = 256;
  std::vector<double> r(n), p(n), q(n), Ap(n), dinv(n);
  for (int i = 0; i < n; ++i) {
    double d = 0;
    for (long long k = c->rp[i]; k < c->rp[i + 1]; ++k)
      if (c->ci[k] == i) d = c->v[k];
    if (d <= 0) { if (st) st->status = OR_ERR_NEG_DIAG; return OR_ERR_NEG_DIAG; }
    dinv[i] = 1.0 / d;
  }
  std::vector<double> part(4 * 256, 0.0);
  auto sum_parts = [&](int k) { double s = 0; for (int t = 0; t < 256; ++t) s += part[4 * t + k]; return s; };
  std::fill(part.begin(), part.end(), 0.0);
  par_for(n, [&](int lo, int hi, int t) {
    double acc = 0;
    for (int i = lo; i < hi; ++i) {
      double s = 0;
      for (long long k = c->rp[i]; k < c->rp[i + 1]; ++k) s += c->v[k] * x[c->ci[k]];
      r[i] = b[i] - s;
      q[i] = r[i] * dinv[i];
      p[i] = q[i];
      acc += r[i] * q[i];
    }
    part[4 * t] = acc;
  });
  double rq = sum_parts(0);
  double bb = 0;
  for (int i = 0; i < n; ++i) bb += b[i] * b[i];
  int it = 0;
  bool conv = false;
  double lastnorm = 0;
  while (!conv && it < maxit) {
    std::fill(part.begin(), part.end(), 0.0);
    par_for(n, [&](int lo, int hi, int t) {
      double acc = 0;
      for (int i = lo; i < hi; ++i) {
        double s = 0;
        for (long long k = c->rp[i]; k < c->rp[i + 1]; ++k) s += c->v[k] * p[c->ci[k]];
        Ap[i] = s;
        acc += p[i] * s;
      }
      part[4 * t] = acc;
    });
    double a = rq / sum_parts(0);
    std::fill(part.begin(), part.end(), 0.0);
    par_for(n, [&](int lo, int hi, int t) {
      double s0 = 0, s1 = 0, s2 = 0;
      for (int i = lo; i < hi; ++i) {
        x[i] += a * p[i];
        r[i] -= a * Ap[i];
        q[i] = r[i] * dinv[i];
        s0 += r[i] * q[i];
        s1 += r[i] * r[i];
        s2 += x[i] * x[i];
      }
      part[4 * t] = s0; part[4 * t + 1] = s1; part[4 * t + 2] = s2;
    });
    double newrq = sum_parts(0), rn = sum_parts(1), xn = sum_parts(2);
    double bk = newrq / rq;
    rq = newrq;
    par_for(n, [&](int lo, int hi, int) {
      for (int i = lo; i < hi; ++i) p[i] = q[i] + bk * p[i];
    });
    if (trace && it < trace_len) trace[it] = std::sqrt(rn / xn);
    ++it;
    lastnorm = rule == 1 ? (bb > 0 ? std::sqrt(rn / bb) : std::sqrt(rn)) : std::sqrt(rn / xn);
    if (lastnorm < eps) conv = true;
  }
  if (st) { st->iterations = it; st->last_norm = lastnorm; st->status = conv ? OR_OK : OR_ERR_MAXIT; }
  return conv ? OR_OK : OR_ERR_MAXIT;
}

// Threaded element-matrix pass (the compute half of ESA_Assembler::assembleK,
// ESA_Assembler.cpp:22-35): element matrices for [e0, e1) into Kout
// (nelem x (ndof*ndof), upper triangles valid).
int oracle_element_matrices_threaded(int kind, int e0, int e1, int nnpe, int ndim,
                                     const int* conn, const double* xyz, const double* params,
                                     int nparams, int order, int ndof, double* Kout, int threads) {
  g_threads = threads > 0 ? threads : (int)std::thread::hardware_concurrency();
  if (g_threads > 256) g_threads = 256;
  std::vector<int> err(256, 0);
  par_for(e1 - e0, [&](int lo, int hi, int t) {
    for (int k = lo; k < hi; ++k) {
      int e = e0 + k;
      double xe[24];
      double Me[64];
      gather_xyz(nnpe, ndim, conn + (size_t)e * nnpe, xyz, xe);
      err[t] |= oracle_element_matrix(kind, xe, params + (size_t)e * nparams, order,
                                      Kout + (size_t)k * ndof * ndof, Me);
    }
  });
  for (int v : err)
    if (v) return OR_ERR_NEG_DIAG;
  return OR_OK;
}

}  // extern "C"
