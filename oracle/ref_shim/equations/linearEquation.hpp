// Shim: LinearEquations (a dense element system) as equation.cpp reads it.
#pragma once
#include "math/matrix.hpp"

typedef unsigned int unsignedInt;

class LinearEquations {
 public:
  explicit LinearEquations(const unsignedInt size);
  ~LinearEquations();
  Matrix K;
  double* F = nullptr;
  int numberOfEquations = 0;
};
