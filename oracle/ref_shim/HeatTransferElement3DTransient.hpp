// Shim: HeatTransferElement3Dtransient as HeatTransferElement3DTransient.cpp
// defines it (the reference ships no headers): its members and the element
// matrices and vectors it fills.  The members the 2D element specialises are
// virtual, so that this element's driver (update, loopOverIntegrationPoints)
// reaches the 2D versions.
#pragma once
#include "element_shim_common.hpp"

struct TransientElementWorkspace : public ElementWorkspace {
  double *F1 = nullptr, *F2 = nullptr, *M_deltaq = nullptr;
  bool StoreAllMe = false;
};

class HeatTransferElement3Dtransient : public IsoElement {
 public:
  HeatTransferElement3Dtransient(void);
  ~HeatTransferElement3Dtransient(void);
  virtual void addToFe(int numDof, int numStrains, InterpAndSolDerivatives* id_ptr, double* flux,
                       double integrationFactor, double* force);
  void addToMe(Matrix* cMat, InterpAndSolDerivatives* id_ptr, double integrationFactor);
  virtual void gradientsOfFieldVariables(InterpAndSolDerivatives* id_ptr);
  double pointValueOfFieldVariables(InterpAndSolDerivatives* id_ptr, double* nodeValue);
  void printNodalFluxesInLCS(std::ostream& outstream);
  void printNodalFluxesInGCS(std::ostream& outstream);
  virtual void addToKe(Matrix* cMat, InterpAndSolDerivatives* id_ptr, double integrationFactor);
  void readSpecialCommand(std::istream& inStream, ElementGroup* element, int numElements, char* command);
  void initializeArrays();
  void setPointers(ElementWorkspace* s);
  void initializeSummary();
  void addToSummary();
  void formK_s(Array<double>& AnalysisParameters, double timeStep);
  void formF_s(Array<double>& AnalysisParameters, double* u, double* ut, double timeStep);
  void formF_s_new(Array<double>& AnalysisParameters, double* u_s, double* delta_u, double* u_s1, double timeStep);
  void formEnhancedResultantVector(Array<double>& AnalysisParameters, double* u_s, double* delta_u, double* u_s1,
                                   double timeStep);
  void formResultantVector(Array<double>& AnalysisParameters, double* u_s, double* delta_u, double* u_s1,
                           double timeStep);
  void addA2TermToResultantVector(Array<double>& AnalysisParameters, double* u_s, double* delta_u, double* u_s1,
                                  double timeStep);
  void formFlowVector(Array<double>& AnalysisParameters, double* u_s, double* delta_u, double* u_s1, double timeStep);
  void addA2TermToFlowVector(Array<double>& AnalysisParameters, double* u_s, double* delta_u, double* u_s1,
                             double timeStep);
  void outputSummary();
  void calculateFe(IntegrationDataType& idt);
  void calculateMe(IntegrationDataType& idt);
  void calculateKe(IntegrationDataType& idt);
  void calculateFlux(IntegrationDataType& idt);
  void processActionCode(char* action, IntegrationDataType& idt);
  void loopOverIntegrationPoints(char* action, IntegrationDataType& idt);
  void update(char* action, double* uGlobal);
  void getVolAvgValues(double* uGlobal, double* volAvgFlux, double* volAvgGradient, double* SED, double* volume);
  void PrintActualConcentrations(double* uGlobal, std::ostream& SO);
  void PrintQuadFluxes(std::ostream& SO, int totalNumIPs);
  void allocateElementalDataMemory(int WorkspaceMaxNumberDof);

  double *F1 = nullptr, *F2 = nullptr, *M_deltaq = nullptr;
  Matrix* Me = nullptr;
  Matrix* Ke_orig = nullptr;
  double* F_orig = nullptr;
  double** quadPointFluxes = nullptr;
  bool MeAlreadyCalculated = false;
  static int effectivePropertyCase;
  static char configDescription[80];
};
