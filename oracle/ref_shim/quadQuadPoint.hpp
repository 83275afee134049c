// Shim declaration (definition in beta/math/gaussQuadrature/gauss.cpp).
#pragma once
class QuadQuadPoints {
 public:
  static void getQuadraturePointsForQuad(int order, double** xi, double** eta, double** w);
  static void deleteAll();
  static double* xi[5];
  static double* eta[5];
  static double* weight[5];
};
