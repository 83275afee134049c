// Shim: the dense Matrix class as matrix.cpp defines it (the reference ships
// no headers): row-major storage in data, per-row skip flags for the solver,
// and every member function matrix.cpp defines.  Used only for the material
// library (oracle/_ref/libbeta_ref_material.so), which links matrix.cpp
// itself; the element library keeps its own small Matrix stand-in.
#pragma once
#include <cstring>  // matrix.cpp calls memcpy without including it
#include <iostream>

typedef double Coefficient;
enum { MATRIX_GENERAL = 0, MATRIX_SYMMETRIC = 1 };

class Matrix {
 public:
  Matrix(const Matrix& Arg);
  Matrix(Matrix& Arg, int nn, int mm);
  Matrix(int nn = 1, int mm = 1);
  ~Matrix(void);
  Matrix operator*(const Matrix& Arg) const;
  Matrix operator=(const Matrix& Other_Matrix);
  const double& operator=(const double& val);
  Matrix operator+(const Matrix& Arg) const;
  Matrix operator-(const Matrix& Arg) const;
  void operator+=(const Matrix& Arg);
  void operator-=(const Matrix& Arg);
  Matrix operator*(const double& Arg) const;
  Matrix multiplyWithMatrix(const Matrix& Arg, int MatrixProperty);
  void multiplyWithVector(const double* v, const int num, double*& F, int MatrixProperty);
  void convertSymmetricToGeneral();
  void resize(int nn, int mm);
  void allocate(int nn, int mm);
  void copy(const Matrix& Other_Matrix);
  void ludcmp(int* indx, double* d);
  Matrix invert(void);
  void SolverSkip(int i);
  void SolverDontSkip(int i);
  void Solve(double* vector);
  void lubksb(int* indx, double* b);
  void print(char* s) const;
  void print(char* s, std::ostream* out) const;
  void print(char* s, int m, int n) const;
  void print(char* s, int m, int n, std::ostream* out) const;
  void printWithRowColumnNumbering(char* s, int m, int n, int* rowNumber, int* columnNumber, std::ostream* out) const;
  void printInMaple(char* s, int mm, int nn, std::ostream* out) const;
  Matrix transpose(void);
  Matrix transposeSelf(void);
  Matrix transposeCopy(void);
  Matrix* transposeCopyNew(void);
  void PrintMatrix(const char*) const {}  // called by pStress.cpp; a no-op here

  Coefficient& operator()(int i, int j) { return data[i * numCols + j]; }
  const Coefficient& operator()(int i, int j) const { return data[i * numCols + j]; }
  Coefficient* operator[](int i) { return data + i * numCols; }
  const Coefficient* operator[](int i) const { return data + i * numCols; }

  int numRows = 0, numCols = 0;
  bool isSymmetric = true;
  Coefficient* data = nullptr;
  int* skip = nullptr;
};

std::ostream& operator<<(std::ostream& o, const Matrix& Arg);
