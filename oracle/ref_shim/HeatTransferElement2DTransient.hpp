// Shim: HeatTransferElement2Dtransient and the pieces of its base it touches,
// declared from how HeatTransferElement2DTransient.cpp uses them (the
// reference ships no headers): the interpolation record of one integration
// point, a dense matrix indexed as (*cMat)(i, j) and (*Ke)[i][j], and the
// element's counters.
#pragma once
#include <vector>

struct InterpAndSolDerivatives {
  int numberOfInterp = 0;
  double* S = nullptr;
  double *p_S_Lx1 = nullptr, *p_S_x1 = nullptr;
  double *p_S_Lx2 = nullptr, *p_S_x2 = nullptr;
  double* nodalValues_u1 = nullptr;
  double p_u1_x1 = 0.0, p_u1_x2 = 0.0;
};

class Matrix {
 public:
  Matrix(int rows, int cols) : cols_(cols), v_((size_t)rows * cols, 0.0) {}
  double& operator()(int i, int j) { return v_[(size_t)i * cols_ + j]; }
  double* operator[](int i) { return &v_[(size_t)i * cols_]; }

 private:
  int cols_;
  std::vector<double> v_;
};

class Material;
class HeatTransferMaterial;

class BasicElement {
 public:
  virtual ~BasicElement() {}
  void setIntegrationOrder(int order) { integrationOrder = order; }
  Material* material = nullptr;
  Matrix* Ke = nullptr;
  int numDof = 0;
  int numStrains = 0;
  int numberOfIntegrationDirections = 0;
  int integrationOrder = 2;
};

class HeatTransferElement2Dtransient : public BasicElement {
 public:
  HeatTransferElement2Dtransient(void);
  ~HeatTransferElement2Dtransient(void);
  void addToFe(int numDof, int numStrains, InterpAndSolDerivatives* id_ptr, double* flux, double integrationFactor,
               double* force);
  void gradientsOfFieldVariables(InterpAndSolDerivatives* id_ptr);
  void addToKe(Matrix* cMat, InterpAndSolDerivatives* id_ptr, double integrationFactor);
};
