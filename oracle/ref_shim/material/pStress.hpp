// Shim: PlaneStress as pStress.cpp defines it (the reference ships no
// headers): an elastic material of three strains read from (E11, E22, nu12,
// G12, a11, a22).
#pragma once
#include "elastic.hpp"

typedef double REAL;

class PlaneStress : public ElasticMaterial {
 public:
  PlaneStress();
  ~PlaneStress(void);
  void initialize();
  void print(std::ostream& outStream);
  bool read(std::istream* inStream);
  double e11 = 0, e22 = 0, nu12 = 0, G12 = 0, a11 = 0, a22 = 0;
};
