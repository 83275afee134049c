// Shim: the LargeMatrix base as largeMatrix.cpp, sparse.cpp and equation.cpp
// use it.  largeMatrix.cpp defines the constructors and the zero-diagonal
// check; the storage-specific operations are virtual, overridden by the
// sparse storage (sparse.cpp), and the solver options Equations passes on
// are plain setters.  Operations no compiled storage provides default to
// inert stubs.
#pragma once
#include <iostream>

#include "utility/excepts.hpp"
#include "verbose_level.hpp"

enum ReorderingScheme { METIS, MMD, PAR };

class LargeMatrix {
 public:
  explicit LargeMatrix(const int numEqns);
  LargeMatrix(const LargeMatrix& arg);
  virtual ~LargeMatrix(void);
  virtual double& operator()(const int ii, const int jj) = 0;
  void CheckAndFixZeroDiagonal();

  virtual void specifyNonZeroLocation(const int, const int) {}
  virtual bool checkNonZeroLocation(const int, const int) { return true; }
  virtual void allocate(void) {}
  virtual void zeroYourself(void) {}
  virtual void solve(double*, double* = 0) {}
  virtual void vectorProduct(double*, double*) {}
  virtual void setaij(const int i, const int j, double val) { (*this)(i, j) = val; }
  virtual void addtoaij(const int i, const int j, double val) { (*this)(i, j) += val; }
  virtual void printMatrix(char*) {}
  virtual void printMatrix(char*, std::ostream*) {}
  virtual void printMatrixAddressFormat(char*, std::ostream*) {}
  virtual void printCSRFormatASCII(char*, std::ostream&) {}
  virtual void printCSRFormatBinary(char*, std::ostream&) {}
  virtual LargeMatrix* clone() { return nullptr; }

  void setReplaceZeroDiagonal_Option(double v) { zeroDiagonalReplacementValue = v; }
  void setVerboseFlag(int v) { verbose = v; }
  void setUsePreviousFillInOrdering(bool v) { UsePreviousFillInOrdering = v; }
  void setUsePreviousFactorizedMatrix(bool v) { UsePreviousFactorizedMatrix = v; }
  void setReorderingScheme(ReorderingScheme) {}
  void setNum_threads_for_solver(int n) { num_threads_for_solver = n; }

  int numberOfEquations;
  double zeroDiagonalReplacementValue;
  int verbose;
  bool UsePreviousFillInOrdering, UsePreviousFactorizedMatrix, OrderingCompleted, FactorizeCompleted;
  int num_threads_for_solver;
};
