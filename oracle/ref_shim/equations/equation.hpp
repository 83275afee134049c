// Shim: Equations (the global system: restraints, multi-point constraints,
// the sparse matrix and its load vectors) and AdditionalEquation as
// equation.cpp and addeqn.cpp define and use them (the reference ships no
// headers).  The two ordered lists Equations keeps -- restrained unknowns
// and additional equations -- are a small pointer list written for this
// build with the cursor interface equation.cpp walks them by.
#pragma once
#include <cmath>
#include <iostream>
#include <string>
#include <vector>

#include "largeMatrix.hpp"
#include "linearEquation.hpp"
#include "math/matrix.hpp"
#include "utility/formWriter.hpp"
#include "utility/utility.h"

// An owning list of T* kept in insertion order (ascending for the restraint
// list, whose entries are inserted once each), walked with begin() /
// operator() / operator++(int) as equation.cpp does.
template <class T>
class PtrList {
 public:
  ~PtrList() { DestroyList(); }
  bool begin() {
    cur_ = 0;
    return !v_.empty();
  }
  T* operator()() { return v_[cur_]; }
  bool operator++(int) { return ++cur_ < v_.size(); }
  bool insert(T* p) {
    v_.push_back(p);
    return true;
  }
  T* find(const T& x) {
    for (T* p : v_)
      if (*p == x) return p;
    return 0;
  }
  void erase(const T& x) {
    for (size_t i = 0; i < v_.size(); ++i)
      if (*v_[i] == x) {
        delete v_[i];
        v_.erase(v_.begin() + i);
        return;
      }
  }
  void DestroyList() {
    for (T* p : v_) delete p;
    v_.clear();
  }
  int AreYouEmpty() const { return (int)v_.size(); }  // the number of entries

 private:
  std::vector<T*> v_;
  size_t cur_ = 0;
};

template <class T>
class Array {
 public:
  T& operator[](int i) { return v_[i]; }
  std::vector<T> v_;
};

struct IntList {
  void add(int v) { v_.push_back(v); }
  std::vector<int> v_;
};

struct threadWorkspace {
  int minEquationNumber = 0, maxEquationNumber = 0;
  IntList elementList, secondaryElementList;
};

class AdditionalEquation {
 public:
  enum Result { Good, Bad, Trivial };
  AdditionalEquation();
  ~AdditionalEquation();
  bool operator!=(const AdditionalEquation& ae) const;
  bool operator==(const AdditionalEquation& ae) const;
  void divideRHSby(const double& val);
  Result collectTerms(void);
  Result apply(AdditionalEquation& eqn);
  bool addAdditionalTerm(const int newMaster, const double newFactor);
  void replaceTerm(const int termNum, const int newMaster, const double& newFactor);
  void freeMasters(void);
  void removeTerm(int termNum);
  double resolve(const double* solution) const;
  double resolveResidual(const double* solution) const;
  void setSlave(int s) { slave = s; }
  void setConstant(double c) { constant = c; }

  int numTerms;
  std::vector<int> master;
  std::vector<double> factor;
  double constant;
  int slave;
};

std::ostream& operator<<(std::ostream& os, const AdditionalEquation& e);  // addeqn.cpp

enum StorageMethod {
  Sparse, Profile, Osparse, mklgbmat, LapackGB, PetSc, PetScUnsymm, MKLPardiso, MKLPardisoUnsymm, MKLCG, ParCG,
  Pardiso, WSMPSymm
};

class Equations {
 public:
  Equations();
  ~Equations();
  void setStorageMethod(std::istream* inStream);
  void setStorageMethod(char* method);
  bool readMPCNeutralFile(char* filename);
  bool addAdditionalEquation(AdditionalEquation* eqnToAdd);
  bool addAdditionalEquation_Kernel(AdditionalEquation* eqnToAdd);
  void restrainHangingDOF();
  void emptyRestraintList();
  void setRestraint(const int eqnNum, const bool val);
  void setSolution(const double& val, const int eqnNum);
  void updatePseudoLoadVectorUsingGK(const double& val, const int eqnNum, LargeMatrix* gK);
  void zeroMatrix(void);
  void zeroLoadVector(void);
  void zeroPseudoLoadVector(void);
  void zeroResultantVector(void);
  void zeroSolution(double val = 0.0);
  void addLinearEquations(LinearEquations& eqns, const int* map);
  void addMatrix(const Matrix& matrix, const int* map, const int size, const double* force = 0, int threadNum = 0);
  void addMatrix2(const Matrix& matrix, const int* map, const int size, const double* force);
  void addMatrixMKL(const Matrix& matrix, const int* map, const int size, const double* force);
  void subtractLinearEquations(LinearEquations& eqns, const int* map);
  void assembleResultantVector(const int* map, const int size, const double* force);
  void addToPseudoLoadVector(const int* map, const int size, const double* force);
  void addToLoadVector(const int* map, const int size, const double* force, int loadVecNum = 0);
  void addLoadToEqn(const double& load, const int eqnNum, bool ignoreIfRestrained = false);
  void setLoadForEqn(const double& load, const int eqnNum);
  void printResultantVector(FormWriter& fr);
  void printEquivalentLoadVector(FormWriter& fr);
  void printLoadVector(FormWriter& fr);
  void printMatrix(FormWriter& fr);
  void printSolution(FormWriter& fr);
  void printAdditionalEquations(FormWriter& fr);
  void printAdditionalEquations(std::ostream* os);
  void printRestraints(FormWriter& fr);
  void CreateMatrix(StorageMethod storageMethod, int n);
  void CreateAndInitializeArrays(int n);
  void InitializeArrays(int n);
  void cleanRestraints();
  void setupStorage(StorageMethod storageMethod, int n);
  void initializeStorage(int n);
  LargeMatrix* createCopyOfMatrix();
  void specifyNonZeroLocation(const int* map, const int size);
  void allocate(void);
  double* solve(double* initGuess = 0);
  double* solveMKL(double* initGuess);
  double* solveUsingResidual(double* initGuess);
  double calculateResidualNorm(void);
  void vectorProduct(double* result, double* vector);
  void releaseMemory();
  void deleteLargeMatrix();
  void setVerboseFlag(VerboseLevel level);
  void setMaxIterations(int max_iter);
  void setSOLUTION_EPSILON(double epsilon);
  void setReorderingScheme(std::string scheme);
  double* incrementalSolutionUsingResidual(double* initGuess);
  void addIncrementalDisplacements(double* deltaSolution);
  void applyAdditionalEquations();
  bool readCommands(std::ifstream* defaultStream);
  int processCommand(char** localTokenList, std::ifstream* currentStream, int numToken);
  void assignElementsToThreads(const int* map, const int size, Array<threadWorkspace>& tList, int elNum);
  void processDofForThreadAssignment(Array<threadWorkspace>& tList, int dof, int elNum);
  void addToLoadVector_Parallel(const int* map, const int size, const double* force, threadWorkspace* thread);
  void addMatrix_Parallel(const Matrix& matrix, const int* map, const int size, const double* force,
                          threadWorkspace* thread);
  void setReplaceZeroDiagonal_Option(double v) { zeroDiagonalReplacementValue = v; }
  void setUsePreviousFillInOrdering(bool v) { UsePreviousFillInOrdering = v; }
  void setUsePreviousFactorizedMatrix(bool v) { UsePreviousFactorizedMatrix = v; }

  LargeMatrix* a;
  double zeroDiagonalReplacementValue;
  int numberOfEquations;
  AdditionalEquation** additionalEquation;
  bool* restraint;
  double *solution, *lastSolution, *loadVector, *pseudoLoadVector, *resultantVector, *residualVector;
  bool allocated, solved;
  StorageMethod sm;
  VerboseLevel verbose;
  std::ostream* outStream;
  bool UsePreviousFillInOrdering, UsePreviousFactorizedMatrix;
  int num_threads_for_solver;
  int MaxIterations;
  double sol_epsilon;
  ReorderingScheme reorderingScheme;
  int numberOfOpenMPThreads;
  PtrList<int> restraintList;
  PtrList<AdditionalEquation> aeList;
};
