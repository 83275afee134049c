// Shim: HeatTransferElement2Dtransient as HeatTransferElement2DTransient.cpp
// defines it (the reference ships no headers): the 3D transient element with
// its 2D conductivity, gradients and flux force (it inherits addToMe,
// formK_s, formF_s_new and the driver).
#pragma once
#include "HeatTransferElement3DTransient.hpp"

class HeatTransferElement2Dtransient : public HeatTransferElement3Dtransient {
 public:
  HeatTransferElement2Dtransient(void);
  ~HeatTransferElement2Dtransient(void);
  void addToFe(int numDof, int numStrains, InterpAndSolDerivatives* id_ptr, double* flux, double integrationFactor,
               double* force);
  void gradientsOfFieldVariables(InterpAndSolDerivatives* id_ptr);
  void addToKe(Matrix* cMat, InterpAndSolDerivatives* id_ptr, double integrationFactor);
};
