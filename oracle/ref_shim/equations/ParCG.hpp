// Shim: ParCGMatrix as ParCG.cpp defines it (the reference ships no
// headers): the sparse storage of sparse.cpp with a two-thread OpenMP
// Jacobi-PCG and matrix-vector product, and the flattened column lists that
// solve builds for them.
#pragma once
#include "sparse.hpp"

class ParCGMatrix : public SymmetricSparseMatrix {
 public:
  explicit ParCGMatrix(const int numEqns);
  ~ParCGMatrix();
  void binaryWrite(FILE* outfile);
  void binaryRead(FILE* infile);
  double& operator()(const int ii, const int jj) override;
  void setaij(const int i, const int j, double val) override;
  double getaij(const int i, const int j);
  void solve(double* b, double* initialGuess = 0) override;
  void zeroYourself(void) override;
  void printMatrix(char* message) override;
  void printMatrixAddressFormatUpper(char* message, std::ostream* out);
  void printMatrixAddressFormat(char* message, std::ostream* out) override;
  void CopyDataFromInterface(SparseMatrixInterface* smi);
  void readMatrixAddressFormat(std::istream* instream);
  void vectorProduct(double* result, double* vector) override;
  void specifyNonZeroLocation(const int I, const int J) override;
  void allocate(void) override;

  int* rowcount = nullptr;
  int** colindex = nullptr;
};
