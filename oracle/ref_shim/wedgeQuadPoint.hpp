// Shim declaration (definition in beta/math/gaussQuadrature/gauss.cpp).
#pragma once
class WedgeQuadPoints {
 public:
  static void getQuadraturePointsForWedge(int order, double** xi, double** eta, double** zeta, double** w);
  static void deleteAll();
  static double* xi[5];
  static double* eta[5];
  static double* zeta[5];
  static double* weight[5];
};
