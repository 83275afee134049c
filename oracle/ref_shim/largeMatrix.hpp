// Shim: the LargeMatrix base as largeMatrix.cpp and sparse.cpp use it.
#pragma once
#include "utility/excepts.hpp"
enum { Off = 0, Basic = 1, Detailed = 2 };  // verbosity levels (verbose >= Basic prints)
class LargeMatrix {
 public:
  explicit LargeMatrix(const int numEqns);
  LargeMatrix(const LargeMatrix& arg);
  virtual ~LargeMatrix(void);
  virtual double& operator()(const int ii, const int jj) = 0;
  void CheckAndFixZeroDiagonal();
  int numberOfEquations;
  double zeroDiagonalReplacementValue;
  int verbose;
  bool UsePreviousFillInOrdering, UsePreviousFactorizedMatrix, OrderingCompleted, FactorizeCompleted;
  int num_threads_for_solver;
};
