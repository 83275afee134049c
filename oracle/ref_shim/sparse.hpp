// Shim: SymmetricSparseMatrix as sparse.cpp defines it -- per row a sorted
// column list (lower triangle, diagonal last) and the values.
#pragma once
#include <cstdio>
#include <iostream>
#include "largeMatrix.hpp"
#include "sorted_list.hpp"
class SparseMatrixInterface;
class SymmetricSparseMatrix : public LargeMatrix {
 public:
  explicit SymmetricSparseMatrix(const int numEqns);
  ~SymmetricSparseMatrix();
  void setMAX_NUMBER_ITERATIONS(int max_iter);
  void setSOLUTION_EPSILON(double sol_epsilon);
  void binaryWrite(FILE* outfile);
  void binaryRead(FILE* infile);
  double& operator()(const int ii, const int jj) override;
  void setaij(const int i, const int j, double val);
  double getaij(const int i, const int j);
  void solve(double* b, double* initialGuess = 0);
  void zeroYourself(void);
  void printMatrix(char* message);
  void printMatrixAddressFormatUpper(char* message, std::ostream* out);
  void printMatrixAddressFormat(char* message, std::ostream* out);
  void printCompressedRowFormat(char* message, std::ostream* out);
  void printCompressedRowFormatUpper(char* message, std::ostream* out);
  void CopyDataFromInterface(SparseMatrixInterface* smi);
  void readMatrixAddressFormat(std::istream* instream);
  virtual void vectorProduct(double* result, double* vector);  // virtual here so a test can count products
  void specifyNonZeroLocation(const int I, const int J);
  void allocate(void);
  void copyFrom(LargeMatrix* a);
  void add(LargeMatrix* a);

  SortedList<int>* row;
  double** mat;
  int MAX_NUMBER_ITERATIONS;
  double SOLUTION_EPSILON;
};
