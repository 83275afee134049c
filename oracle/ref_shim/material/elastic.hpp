// Shim: Material and ElasticMaterial as elastic.cpp defines and uses them
// (the reference ships no headers).  The orientation is the identity (no
// material angles), so the rotation calls copy.
#pragma once
#include <string>
#include <vector>

#include "materials/ElasticISV.hpp"
#include "math/matrix.hpp"

#ifndef BETA_OUT
#define BETA_OUT std::cout
#endif

class Rotation {
 public:
  Rotation() {}
  Rotation(int, double) {}
  void add_after_self(const Rotation&) {}
  void rotate_Voigt_engineering_strain_from_local_to_global(const double* l, double* g) const {
    for (int i = 0; i < 6; ++i) g[i] = l[i];
  }
  void rotate_Cmat_from_local_to_global(const Matrix& local, Matrix& global) const { global = local; }
  void rotate_3D_2nd_Order_Tensor_from_local_to_global(const Matrix& local, Matrix& global) const { global = local; }
};

enum { clear = 0, haveS = 1, haveC = 2 };

class Material {
 public:
  virtual ~Material() {}
  void setType(const char* t) { type = t; }
  const char* getGroupName() const { return name.c_str(); }
  int getGroupNum() const { return groupNum; }
  std::string name, type;
  int groupNum = 0;
  Rotation MaterialRotation;
};

class ElasticMaterial : public Material {
 public:
  ElasticMaterial();
  ElasticMaterial(const ElasticMaterial& arg);
  virtual ~ElasticMaterial(void);
  virtual void initialize();
  virtual void allocateISVs(std::vector<BasicISV*>& isv, const int& numISVs) const;
  virtual void deallocateISVs(std::vector<BasicISV*>& isv) const;
  void CommonElasticMaterial(void);
  virtual bool read(std::istream* inStream);
  virtual void calculateStress(double* stress, double* strain, BasicISV* isv, const Rotation* Orientation);
  virtual void calculateInitialStress(double* stress, BasicISV* isv, const Rotation* Orientation);
  virtual void print(std::ostream& ostrm);
  void rotateMaterialToGlobal(const Rotation* OrientationAtPoint);

  Matrix *cMat = nullptr, *S = nullptr, *globalCmat = nullptr, *rotatedCmat = nullptr, *localizedCmat = nullptr;
  int numberOfRotationAngles = 0;
  int rotationAxis[4] = {0, 0, 0, 0};
  double rotationAngle[4] = {0, 0, 0, 0};
  double angleZ = 0.0, currentRotationAngle = 0.0;
  int numStrains = 6;
  int FlagSingleAngle = 0;
  int materialState = clear;
  double alpha[6] = {0, 0, 0, 0, 0, 0}, beta[6] = {0, 0, 0, 0, 0, 0};
};
