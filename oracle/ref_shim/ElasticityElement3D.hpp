// Shim: ElasticityElement3D (and the elastic material it calls) as
// ElasticityElement3D.cpp defines and uses them (the reference ships no
// headers): the member functions that file defines and the members it reads.
// The members ElasticityElement2D specialises are virtual, so that the 3D
// element's driver (update, loopOverIntegrationPoints) reaches the plane
// element's versions.
#pragma once
#include "element_shim_common.hpp"

class ElasticISV : public BasicISV {
 public:
  void setTemperature(double t) { temperature = t; }
  void setMoisture(double m) { moisture = m; }
  double temperature = 0.0, moisture = 0.0;
};

// The element reads the material's global constitutive matrix and asks it
// for the stress of a strain; with no hygrothermal strain that stress is
// C * strain (the Voigt product the reference's calculateStress forms).
class ElasticMaterial : public Material {
 public:
  void rotateMaterialToGlobal(const Rotation*) {}
  Matrix* getPointerToGlobalCmat() { return &cmat; }
  void calculateStress(double* stress, double* strain, BasicISV*, const Rotation*) {
    for (int i = 0; i < numStrains; ++i) {
      stress[i] = 0.0;
      for (int j = 0; j < numStrains; ++j) stress[i] += cmat(i, j) * strain[j];
    }
  }
  void calculateInitialStress(double* stress, BasicISV*, const Rotation*) {
    for (int i = 0; i < numStrains; ++i) stress[i] = 0.0;
  }
  int numStrains = 6;
  Matrix cmat{6, 6};
};

class ElasticityElement3D : public IsoElement {
 public:
  ElasticityElement3D(void);
  ~ElasticityElement3D(void);
  void addToFe(int numDof, int numStrains, double** b, double* stress, double integrationFactor, double* force);
  virtual void calculateBmatrix(InterpAndSolDerivatives* id_ptr, double** b);
  virtual void calculateStrain(InterpAndSolDerivatives* id_ptr, double* strain);
  virtual void derivativesOfFields(InterpAndSolDerivatives* id_ptr);
  void printNodalStressesInLCS(std::ostream& stressout);
  void printNodalStressesInGCS(std::ostream& stressout);
  void printNodalStrainsInLCS(std::ostream& strainout);
  void printNodalStrainsInGCS(std::ostream& strainout);
  void printQuadStrains(int totalNumIPs, std::ostream& SO);
  void printQuadStresses(int totalNumIPs, std::ostream& SO);
  void printNodalForcesByElement(std::ostream& forcesout);
  virtual void getVolAvgValues(double* uGlobal, double* volAvgStress, double* volAvgStrain, double* SED, double* volume);
  virtual void addToKe(Matrix* cMat, InterpAndSolDerivatives* id_ptr, double integrationFactor, double* stress);
  void initializeArrays();
  bool geometryCheck();
  void setPointers(ElementWorkspace* s);
  void initializeSummary();
  void addToSummary();
  void outputSummary();
  void readSpecialCommand(std::istream& inStream, ElementGroup* element, int numElements, char* command);
  void setTemperature(double temperature);
  void setMoisture(double moisture);
  void InitializeOutputSummary();
  void OutputSummary();
  void FinalizeSummary();
  void ConsolidateSummary(std::string outputtype, std::ofstream& ofile);
  void setConsolidate(bool flag);
  void processActionCode(char* action, IntegrationDataType& idt);
  void loopOverIntegrationPoints(char* action, IntegrationDataType& idt);
  void update(char* action, double* uGlobal);
  void calculateFe(IntegrationDataType& idt);
  void calculateInitialForce(IntegrationDataType& idt);
  void calculateKe(IntegrationDataType& idt);
  void calculateStress(IntegrationDataType& idt);

  double** b = nullptr;
  int reduceCMatFlag = 0;
  int ForceSingleNonZeroStressComponent = -1;
  static int effectiveModulusCase;
  static char weaveDescription[80];
  static std::ofstream* elematfile;
  static std::ofstream* manglesfile;
  static bool initialized;
  static bool consolidated;
};
