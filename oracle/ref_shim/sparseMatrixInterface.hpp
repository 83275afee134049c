// Shim: the fields of SparseMatrixInterface that
// SymmetricSparseMatrix::CopyDataFromInterface reads.
#pragma once
#include "sorted_list.hpp"
enum { LowerTriangular = 1, UpperTriangular = 2 };
class SparseMatrixInterface {
 public:
  int numEquations = 0;
  int type = LowerTriangular;
  SortedList<int>* row = nullptr;
  SortedList<int>* col = nullptr;
  double** mat = nullptr;
};
