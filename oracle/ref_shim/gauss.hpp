// Shim declaration of the reference's GAUSS class (definition in
// beta/math/gaussQuadrature/gauss.cpp); the header itself is not shipped.
#pragma once
#define MAX_Gauss_ORDER 20
class GAUSS {
 public:
  explicit GAUSS(int k);
  static void deleteAll();
  double getCoord(int i) const { return currentCoords[i]; }
  double getWeight(int i) const { return currentWeights[i]; }
  static double* coords[MAX_Gauss_ORDER];
  static double* weights[MAX_Gauss_ORDER];
  static bool calculated[MAX_Gauss_ORDER];
 private:
  int currentOrder;
  double* currentCoords;
  double* currentWeights;
};
