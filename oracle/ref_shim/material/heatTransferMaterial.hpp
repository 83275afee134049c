// Shim: HeatTransferMaterial as heatTransferMaterial.cpp defines it (the
// reference ships no headers): a conductivity tensor read from an input
// block, and the flux -k grad T at a point.
#pragma once
#include "elastic.hpp"
#include "elements/InterpAndSolDerivatives.hpp"

class HeatTransferMaterial : public Material {
 public:
  HeatTransferMaterial();
  HeatTransferMaterial(const HeatTransferMaterial& arg);
  virtual ~HeatTransferMaterial(void);
  void CommonHeatTransferMaterial(void);
  virtual void initialize();
  virtual bool read(std::istream* inStream);
  void calculateFlux(double* flux, InterpAndSolDerivatives* id_ptr);
  virtual void print(std::ostream& ostrm);
  void rotateMaterialToGlobal(const Rotation* OrientationAtPoint);

  Matrix *cMat = nullptr, *globalCmat = nullptr;
  int numberOfFluxes = 3;
  double angleZ = 0.0, currentRotationAngle = 0.0;
  int numberOfRotationAngles = 0;
  int rotationAxis[4] = {0, 0, 0, 0};
  double rotationAngle[4] = {0, 0, 0, 0};
};
