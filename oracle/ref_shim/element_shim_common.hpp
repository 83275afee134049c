// Shim: the parts of the reference's element hierarchy that the element
// files compiled here (HeatTransferElement2DTransient.cpp,
// HeatTransferElement3DTransient.cpp, ElasticityElement3D.cpp,
// ElasticityElement2D.cpp) touch, declared from how those files use them
// because the reference ships no headers.  Only the routines a test calls do
// real work (the interpolation record, the dense matrix, the material's
// capacity and stiffness); every other base-class service is an inert stub
// so that the element files compile and link unmodified.
#pragma once
#include <algorithm>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <string>
#include <vector>

#include "hexQuadPoint.hpp"
#include "quadQuadPoint.hpp"
#include "utility/excepts.hpp"
#include "utility/utility_defines.h"

#ifndef BETA_OUT
#define BETA_OUT std::cout
#endif

#include "verbose_level.hpp"  // levels compared with verboseFlag

#ifndef GEOMETRIC_NONLINEAR
#define LINEAR 0
#define GEOMETRIC_NONLINEAR 1
#endif
#ifndef EXIT_BETA
#define EXIT_BETA(msg) do { std::cerr << (msg) << '\n'; std::abort(); } while (0)
#endif

template <class T>
class Array {
 public:
  explicit Array(int n = 0) : v_(n) {}
  T& operator[](int i) { return v_[i]; }
  int getNum() const { return (int)v_.size(); }

 private:
  std::vector<T> v_;
};

struct InterpAndSolDerivatives {
  InterpAndSolDerivatives() {}
  InterpAndSolDerivatives(int n, int) : numberOfInterp(n) {}
  void allocate() {
    store_.assign(16 * (size_t)(numberOfInterp > 0 ? numberOfInterp : 1), 0.0);
    double* p = store_.data();
    const int n = numberOfInterp > 0 ? numberOfInterp : 1;
    double** fields[] = {&S, &p_S_Lx1, &p_S_Lx2, &p_S_Lx3, &p_S_x1, &p_S_x2, &p_S_x3, &nodalValues_u1,
                         &nodalValues_u2, &nodalValues_u3, &xCoor, &yCoor, &zCoor};
    for (double** f : fields) { *f = p; p += n; }
  }
  int numberOfInterp = 0;
  double* S = nullptr;
  double *p_S_Lx1 = nullptr, *p_S_Lx2 = nullptr, *p_S_Lx3 = nullptr;
  double *p_S_x1 = nullptr, *p_S_x2 = nullptr, *p_S_x3 = nullptr;
  double *nodalValues_u1 = nullptr, *nodalValues_u2 = nullptr, *nodalValues_u3 = nullptr;
  double *xCoor = nullptr, *yCoor = nullptr, *zCoor = nullptr;
  double p_u1_x1 = 0.0, p_u1_x2 = 0.0, p_u1_x3 = 0.0;
  double p_u2_x1 = 0.0, p_u2_x2 = 0.0, p_u2_x3 = 0.0;
  double p_u3_x1 = 0.0, p_u3_x2 = 0.0, p_u3_x3 = 0.0;
  double detJ = 0.0;

 private:
  std::vector<double> store_;
};

class Matrix {
 public:
  Matrix(int rows = 1, int cols = 1) : cols_(cols), v_((size_t)rows * cols, 0.0) {}
  double& operator()(int i, int j) { return v_[(size_t)i * cols_ + j]; }
  double* operator[](int i) { return &v_[(size_t)i * cols_]; }
  void print(const char*, int, int, std::ostream*) const {}
  void printWithRowColumnNumbering(const char*, int, int, int*, int*, std::ostream*) const {}

 private:
  int cols_;
  std::vector<double> v_;
};

struct GaussPointList {
  int totalNumIPs = 0;
  double *xiList = nullptr, *etaList = nullptr, *zetaList = nullptr;
  double* weightList = nullptr;
};

struct IntegrationDataType {
  InterpAndSolDerivatives* id = nullptr;
  int ip = 0;
  double integrationFactor = 0.0;
  GaussPointList gaussPointList;
  double* elemDisp[3] = {nullptr, nullptr, nullptr};
  double* uGlobal = nullptr;
};

struct ElementWorkspace {
  double **rotatedFluxes = nullptr, **extrapolatedFluxes = nullptr, **quadPointFluxes = nullptr;
  double** quadPointStresses = nullptr;
  // elasticity: B rows, per-point strains/stresses and volume sums
  double** b = nullptr;
  double **quadPointStrains = nullptr, **rotatedStresses = nullptr, **rotatedStrains = nullptr;
  double **extrapolatedStresses = nullptr, **extrapolatedStrains = nullptr;
  double *strainVolume_total = nullptr, *stressVolume_total = nullptr;
  double *localStressVolume_total = nullptr, *energyVolume_total = nullptr;
  double *strainVolume_element = nullptr, *stressVolume_element = nullptr;
  double *energyVolume_element = nullptr, *localStressVolume_element = nullptr;
  double totalVolume = 0.0, temperatureVolume = 0.0, elementVolume = 0.0, temperatureVolume_element = 0.0;
  double *fluxVolume_total = nullptr, *gradientVolume_total = nullptr;
  double *fluxVolume_element = nullptr, *gradientVolume_element = nullptr;
  Matrix* Ke_original = nullptr;
  Array<Matrix>* MeList = nullptr;
  Matrix* Me = nullptr;
  double* F_original = nullptr;
};

class Rotation {
 public:
  void interpolate_rotation_by_angle(InterpAndSolDerivatives*, void*) {}
  // identity orientation: local and global axes coincide
  void rotate_Voigt_stress_from_global_to_local(double* g, double* l) const { std::copy(g, g + 6, l); }
  void rotate_Voigt_engineering_strain_from_global_to_local(double* g, double* l) const { std::copy(g, g + 6, l); }
};

class BasicISV {
 public:
  virtual ~BasicISV() {}
};

class Material {
 public:
  virtual ~Material() {}
  virtual void allocateISVs(std::vector<BasicISV*>&, const int&) const {}
};

// The capacity the 3D element's addToMe reads is the material's saturation
// value; the conductivity is the material's (global) cMat.
class HeatTransferMaterial : public Material {
 public:
  double getSaturationValue() const { return saturation; }
  void rotateMaterialToGlobal(Rotation*) {}
  void UpdateGlobalCmat(double) {}
  Matrix* getPointerToGlobalCmat() { return &cmat; }
  void calculateFlux(double*, InterpAndSolDerivatives*) {}
  double saturation = 1.0;
  Matrix cmat{3, 3};
};

class ElementGroup;

struct ElementNode {
  int nodeNum = 0;
  int numDof = 0;
};

class BasicElement {
 public:
  virtual ~BasicElement() {}
  void setIntegrationOrder(int order) { integrationOrder = order; }
  void setPointers(ElementWorkspace*) {}
  void allocateElementalDataMemory(int) {}
  int getMaterialNumber() const { return materialGroup; }
  int* getDofList() { return dofList; }
  int getNumDof() const { return numDof; }
  bool checkForAllocatedISVs() const { return !isv.empty(); }
  int getTotalNumberOfIPs() const { return 0; }
  void checkForNegativeDiagonal() {}
  int analysisType = LINEAR;
  bool activeElementFlag = true;
  int newElementNumber = 0;
  std::vector<BasicISV*> isv;
  Material* material = nullptr;
  Matrix* Ke = nullptr;
  double* Fe = nullptr;
  double* initialFe = nullptr;
  int* dofList = nullptr;
  int numDof = 0;
  int numStrains = 0;
  int numberOfIntegrationDirections = 0;
  int integrationOrder = 2;
  int elementNumber = 0;
  int materialGroup = 0;
  int numNodesPerElement = 0;
  bool requiresParallelESAConsideration = false;
  ElementNode* node = nullptr;
  ElementWorkspace* bag = nullptr;
};

// The reference's own Gauss rules and shape functions (gauss.cpp, shape.cpp,
// compiled into the same library).
void shapeHex8(double* S, double xi, double eta, double zeta);
void derivHex8(double* Sxi, double* Seta, double* Szeta, double xi, double eta, double zeta);
void shapeQuad4(double* S, double zeta, double eta);
void derivQuad4(double* Szeta, double* Seta, double zeta, double eta);

// IsoElement's services, written for this build because isoElement.cpp and
// BasicElement.cpp do not compile here: the reference's tensor Gauss rules
// and shape functions for hex8 / quad4 (numberOfIntegrationDirections 3 /
// 2), the Jacobian, its determinant and the global shape-function gradients
// at a point (the algebra of IsoElement::jacobian, isoElement.cpp:250-389),
// and the element's nodal coordinates and solution from tables a test
// attaches (coords: nnpe x 3; edofs: nnpe x dofs-per-node global numbers).
// Orientation is the identity.
class IsoElement : public BasicElement {
 public:
  void readSpecialCommand(std::istream&, ElementGroup*, int, char*) {}
  void getQuadraturePoints(GaussPointList& g) {
    if (numberOfIntegrationDirections == 3) {
      HexQuadPoints::getQuadraturePointsForHex(integrationOrder, &g.xiList, &g.etaList, &g.zetaList, &g.weightList);
      g.totalNumIPs = integrationOrder * integrationOrder * integrationOrder;
    } else {
      QuadQuadPoints::getQuadraturePointsForQuad(integrationOrder, &g.xiList, &g.etaList, &g.weightList);
      g.totalNumIPs = integrationOrder * integrationOrder;
    }
  }
  void interpolation(int ip, GaussPointList& g, InterpAndSolDerivatives* id) {
    id->numberOfInterp = numNodesPerElement;
    if (numberOfIntegrationDirections == 3) {
      shapeHex8(id->S, g.xiList[ip], g.etaList[ip], g.zetaList[ip]);
      derivHex8(id->p_S_Lx1, id->p_S_Lx2, id->p_S_Lx3, g.xiList[ip], g.etaList[ip], g.zetaList[ip]);
    } else {
      shapeQuad4(id->S, g.xiList[ip], g.etaList[ip]);
      derivQuad4(id->p_S_Lx1, id->p_S_Lx2, g.xiList[ip], g.etaList[ip]);
    }
  }
  void jacobian(InterpAndSolDerivatives* id) {
    const int n = id->numberOfInterp;
    const double *L1 = id->p_S_Lx1, *L2 = id->p_S_Lx2, *L3 = id->p_S_Lx3;
    const double *x = id->xCoor, *y = id->yCoor, *z = id->zCoor;
    if (numberOfIntegrationDirections == 3) {
      double J[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
      for (int a = 0; a < n; ++a) {
        const double L[3] = {L1[a], L2[a], L3[a]};
        for (int r = 0; r < 3; ++r) {
          J[r][0] += L[r] * x[a];
          J[r][1] += L[r] * y[a];
          J[r][2] += L[r] * z[a];
        }
      }
      const double c00 = J[1][1] * J[2][2] - J[1][2] * J[2][1], c01 = J[1][2] * J[2][0] - J[1][0] * J[2][2],
                   c02 = J[1][0] * J[2][1] - J[1][1] * J[2][0];
      const double det = J[0][0] * c00 + J[0][1] * c01 + J[0][2] * c02;
      id->detJ = det;
      const double inv[3][3] = {
          {c00 / det, (J[0][2] * J[2][1] - J[0][1] * J[2][2]) / det, (J[0][1] * J[1][2] - J[0][2] * J[1][1]) / det},
          {c01 / det, (J[0][0] * J[2][2] - J[0][2] * J[2][0]) / det, (J[0][2] * J[1][0] - J[0][0] * J[1][2]) / det},
          {c02 / det, (J[0][1] * J[2][0] - J[0][0] * J[2][1]) / det, (J[0][0] * J[1][1] - J[0][1] * J[1][0]) / det}};
      for (int a = 0; a < n; ++a) {
        id->p_S_x1[a] = inv[0][0] * L1[a] + inv[0][1] * L2[a] + inv[0][2] * L3[a];
        id->p_S_x2[a] = inv[1][0] * L1[a] + inv[1][1] * L2[a] + inv[1][2] * L3[a];
        id->p_S_x3[a] = inv[2][0] * L1[a] + inv[2][1] * L2[a] + inv[2][2] * L3[a];
      }
    } else {
      double J[2][2] = {{0, 0}, {0, 0}};
      for (int a = 0; a < n; ++a) {
        J[0][0] += L1[a] * x[a];
        J[0][1] += L1[a] * y[a];
        J[1][0] += L2[a] * x[a];
        J[1][1] += L2[a] * y[a];
      }
      const double det = J[0][0] * J[1][1] - J[0][1] * J[1][0];
      id->detJ = det;
      for (int a = 0; a < n; ++a) {
        id->p_S_x1[a] = (J[1][1] * L1[a] - J[0][1] * L2[a]) / det;
        id->p_S_x2[a] = (-J[1][0] * L1[a] + J[0][0] * L2[a]) / det;
      }
    }
  }
  double getIntegrationFactor() { return 1.0; }
  void calculateElementVolume(IntegrationDataType&) {}
  void extractNodalCoordinates(double* x, double* y, double* z) {
    for (int a = 0; a < numNodesPerElement; ++a) {
      x[a] = coords[a * 3];
      y[a] = coords[a * 3 + 1];
      z[a] = coords[a * 3 + 2];
    }
  }
  void extractSolution(double* u, double** d) {
    const int nd = numDof / numNodesPerElement;
    for (int a = 0; a < numNodesPerElement; ++a)
      for (int c = 0; c < nd; ++c) d[c][a] = u[edofs[a * nd + c]];
  }
  void AllocateRotations() {}
  void extrapolateQuadValuesToNodes(double**, int, double**) {}
  const double* coords = nullptr;
  const int* edofs = nullptr;
  Rotation own_rotation;
  Rotation* OrientationAtIP = &own_rotation;
  void* ElementNodeRotations = nullptr;
};
