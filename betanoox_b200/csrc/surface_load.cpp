// surface_load.cpp -- nodal loads of a surface flux (C ABI
// beta_gpu_surface_flux_load), the integration SurfaceLoad::applyTo does
// (beta/BCs/SurfaceLoad.cpp:16-255) without its shared-memory coupling: the
// caller passes the nodal flux values.  Host code: the work is O(surface
// elements) per call, far below one assembly.
#include "../../include/beta_gpu.h"

#include <cmath>
#include <cstring>
#include <vector>

namespace {

// 3-point Gauss-Legendre abscissa and the 7-point triangle rule's points.
constexpr double kG3 = 0.774596669241483;
constexpr double kT1 = 0.101286507323, kT2 = 0.797426985353, kT3 = 0.470142064105, kT4 = 0.059715871789;

struct Rule {
  int n;
  double xi[9], eta[9], w[9];
};

Rule quad_rule() {
  Rule r;
  r.n = 9;
  const double x[3] = {kG3, 0.0, -kG3}, w[3] = {5.0 / 9.0, 8.0 / 9.0, 5.0 / 9.0};
  for (int j = 0; j < 3; ++j)
    for (int i = 0; i < 3; ++i) {
      r.xi[3 * j + i] = x[i];
      r.eta[3 * j + i] = x[j];
      r.w[3 * j + i] = w[i] * w[j];
    }
  return r;
}

Rule tri_rule() {
  // weights sum to 1/2, the area of the reference triangle
  Rule r;
  r.n = 7;
  const double xi[7] = {1.0 / 3.0, kT1, kT1, kT2, kT3, kT3, kT4};
  const double eta[7] = {1.0 / 3.0, kT1, kT2, kT1, kT3, kT4, kT3};
  const double w[7] = {0.225, 0.125939180544, 0.125939180544, 0.125939180544,
                       0.132394152788, 0.132394152788, 0.132394152788};
  for (int k = 0; k < 7; ++k) {
    r.xi[k] = xi[k];
    r.eta[k] = eta[k];
    r.w[k] = 0.5 * w[k];
  }
  return r;
}

// Shape functions and their local derivatives.  Node orders: quad4
// counter-clockwise from (-1,-1); quad8 corner, mid-side, corner, ...
// counter-clockwise from (-1,-1); tri6 corner (0,0), mid-side, corner (1,0),
// mid-side, corner (0,1), mid-side.
void shape(int npe, double x, double e, double* N, double* dx, double* de) {
  if (npe == 4) {
    const double sx[4] = {-1, 1, 1, -1}, se[4] = {-1, -1, 1, 1};
    for (int i = 0; i < 4; ++i) {
      N[i] = 0.25 * (1 + sx[i] * x) * (1 + se[i] * e);
      dx[i] = 0.25 * sx[i] * (1 + se[i] * e);
      de[i] = 0.25 * se[i] * (1 + sx[i] * x);
    }
  } else if (npe == 8) {
    const double px[8] = {-1, 0, 1, 1, 1, 0, -1, -1}, pe[8] = {-1, -1, -1, 0, 1, 1, 1, 0};
    for (int i = 0; i < 8; ++i) {
      const double a = px[i], b = pe[i];
      if (a != 0 && b != 0) {
        N[i] = 0.25 * (1 + a * x) * (1 + b * e) * (a * x + b * e - 1);
        dx[i] = 0.25 * a * (1 + b * e) * (2 * a * x + b * e);
        de[i] = 0.25 * b * (1 + a * x) * (a * x + 2 * b * e);
      } else if (a == 0) {
        N[i] = 0.5 * (1 - x * x) * (1 + b * e);
        dx[i] = -x * (1 + b * e);
        de[i] = 0.5 * b * (1 - x * x);
      } else {
        N[i] = 0.5 * (1 + a * x) * (1 - e * e);
        dx[i] = 0.5 * a * (1 - e * e);
        de[i] = -e * (1 + a * x);
      }
    }
  } else {
    const double l = 1 - x - e;
    N[0] = l * (2 * l - 1);   dx[0] = 1 - 4 * l;       de[0] = 1 - 4 * l;
    N[1] = 4 * x * l;         dx[1] = 4 * (l - x);     de[1] = -4 * x;
    N[2] = x * (2 * x - 1);   dx[2] = 4 * x - 1;       de[2] = 0;
    N[3] = 4 * x * e;         dx[3] = 4 * e;           de[3] = 4 * x;
    N[4] = e * (2 * e - 1);   dx[4] = 0;               de[4] = 4 * e - 1;
    N[5] = 4 * e * l;         dx[5] = -4 * e;          de[5] = 4 * (l - e);
  }
}

}  // namespace

extern "C" int beta_gpu_surface_flux_load(int nsurf, int nodes_per_face, const int* face_conn, int nnode,
                                          const double* xyz, const double* nodal_flux, const int* first_dof,
                                          int ndof, double* load) {
  const int npe = nodes_per_face;
  if (nsurf < 0 || (npe != 4 && npe != 6 && npe != 8) || nnode <= 0 || ndof <= 0 ||
      (nsurf > 0 && (!face_conn || !xyz || !nodal_flux || !first_dof || !load)))
    return BETA_GPU_ERR_ARG;
  for (long long k = 0; k < (long long)nsurf * npe; ++k) {
    const int nd = face_conn[k];
    if (nd < 0 || nd >= nnode || first_dof[nd] < 0 || first_dof[nd] >= ndof) return BETA_GPU_ERR_ARG;
    if (!std::isfinite(nodal_flux[nd]) || !std::isfinite(xyz[3LL * nd]) || !std::isfinite(xyz[3LL * nd + 1]) ||
        !std::isfinite(xyz[3LL * nd + 2]))
      return BETA_GPU_ERR_NOT_FINITE;
  }
  const Rule R = npe == 6 ? tri_rule() : quad_rule();
  // shape values at the rule's points, shared by every face
  double N[9][8], DX[9][8], DE[9][8];
  for (int m = 0; m < R.n; ++m) shape(npe, R.xi[m], R.eta[m], N[m], DX[m], DE[m]);
  for (int f = 0; f < nsurf; ++f) {
    const int* c = face_conn + (long long)f * npe;
    double fe[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int m = 0; m < R.n; ++m) {
      double gx[3] = {0, 0, 0}, ge[3] = {0, 0, 0}, q = 0;
      for (int i = 0; i < npe; ++i) {
        const double* X = xyz + 3LL * c[i];
        for (int d = 0; d < 3; ++d) {
          gx[d] += DX[m][i] * X[d];
          ge[d] += DE[m][i] * X[d];
        }
        q += N[m][i] * nodal_flux[c[i]];
      }
      const double g1 = gx[1] * ge[2] - ge[1] * gx[2];
      const double g2 = gx[2] * ge[0] - ge[2] * gx[0];
      const double g3 = gx[0] * ge[1] - ge[0] * gx[1];
      const double s = R.w[m] * q * std::sqrt(g1 * g1 + g2 * g2 + g3 * g3);
      for (int i = 0; i < npe; ++i) fe[i] += s * N[m][i];
    }
    for (int i = 0; i < npe; ++i) load[first_dof[c[i]]] += fe[i];  // first dof of the node
  }
  return BETA_GPU_OK;
}
