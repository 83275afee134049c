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

class IsoElement : public BasicElement {
 public:
  void readSpecialCommand(std::istream&, ElementGroup*, int, char*) {}
  void interpolation(int, GaussPointList&, InterpAndSolDerivatives*) {}
  void jacobian(InterpAndSolDerivatives*) {}
  double getIntegrationFactor() { return 1.0; }
  void calculateElementVolume(IntegrationDataType&) {}
  void extractNodalCoordinates(double*, double*, double*) {}
  void extractSolution(double*, double**) {}
  void getQuadraturePoints(GaussPointList&) {}
  void AllocateRotations() {}
  void extrapolateQuadValuesToNodes(double**, int, double**) {}
  Rotation* OrientationAtIP = nullptr;
  void* ElementNodeRotations = nullptr;
};
