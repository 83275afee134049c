// Shim: HeatTransferElement2Dtransient as HeatTransferElement2DTransient.cpp
// defines it (the reference ships no headers).
#pragma once
#include "element_shim_common.hpp"

class HeatTransferElement2Dtransient : public IsoElement {
 public:
  HeatTransferElement2Dtransient(void);
  ~HeatTransferElement2Dtransient(void);
  void addToFe(int numDof, int numStrains, InterpAndSolDerivatives* id_ptr, double* flux, double integrationFactor,
               double* force);
  void gradientsOfFieldVariables(InterpAndSolDerivatives* id_ptr);
  void addToKe(Matrix* cMat, InterpAndSolDerivatives* id_ptr, double integrationFactor);
};
