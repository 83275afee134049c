// Shim declaration (definition in beta/math/gaussQuadrature/gauss.cpp).
#pragma once
class LineQuadPoints {
 public:
  static void getQuadraturePointsForLine(int order, double** xi, double** w);
  static void deleteAll();
  static double* xi[5];
  static double* weight[5];
};
