// Shim: ElasticityElement2D as ElasticityElement2D.cpp defines it (the
// reference ships no headers): the plane element specialises the 3D
// elasticity element's B matrix, strain and stiffness accumulation.
#pragma once
#include "ElasticityElement3D.hpp"

class ElasticityElement2D : public ElasticityElement3D {
 public:
  ElasticityElement2D(void);
  ~ElasticityElement2D(void);
  void addToKe(Matrix* cMat, InterpAndSolDerivatives* id_ptr, double integrationFactor, double* stress);
  void calculateBmatrix(InterpAndSolDerivatives* id_ptr, double** b);
  void calculateStrain(InterpAndSolDerivatives* id_ptr, double* strain);
  void derivativesOfFields(InterpAndSolDerivatives* id_ptr);
  void getVolAvgValues(double* uGlobal, double* volAvgStress, double* volAvgStrain, double* SED, double* volume);
};
