// common.cuh -- shared device helpers for the BETA B200 path.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace betagpu {

constexpr int kWarp = 32;
constexpr int kMaxIP = 64;  // Gauss points per element (order <= 4 in 3D)

// Gauss table of one element type: per integration point the weight, the
// shape values N_a and the local derivatives dN_a/dxi_r (r-major, 8 nodes).
struct GaussTable {
  int nip;
  double w[kMaxIP];
  double N[kMaxIP][8];
  double dN[kMaxIP][3][8];
};

// Device-side status bits raised by kernels (OR-ed into one word).
enum : unsigned {
  kFlagNegDiag = 1u,   // element diagonal <= 0 (BasicElement::checkForNegativeDiagonal)
  kFlagNotFinite = 2u,
  kFlagSlot = 4u,      // slot outside the layout (defensive; never expected)
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Sum over the `width` lanes of a power-of-two lane group (xor butterfly).
template <int WIDTH, typename T>
__device__ __forceinline__ T group_sum(T v) {
#pragma unroll
  for (int o = 1; o < WIDTH; o <<= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Inverse of the 3x3 matrix M (row-major) by cofactors; returns det.
template <typename T>
__device__ __forceinline__ T inv3(const T* M, T* Mi) {
  T c00 = M[4] * M[8] - M[5] * M[7];
  T c01 = M[5] * M[6] - M[3] * M[8];
  T c02 = M[3] * M[7] - M[4] * M[6];
  T det = M[0] * c00 + M[1] * c01 + M[2] * c02;
  T id = T(1) / det;
  Mi[0] = c00 * id;
  Mi[3] = c01 * id;
  Mi[6] = c02 * id;
  Mi[1] = (M[2] * M[7] - M[1] * M[8]) * id;
  Mi[4] = (M[0] * M[8] - M[2] * M[6]) * id;
  Mi[7] = (M[1] * M[6] - M[0] * M[7]) * id;
  Mi[2] = (M[1] * M[5] - M[2] * M[4]) * id;
  Mi[5] = (M[2] * M[3] - M[0] * M[5]) * id;
  Mi[8] = (M[0] * M[4] - M[1] * M[3]) * id;
  return det;
}

// Orthotropic stiffness from (E11,E22,E33,nu12,nu23,nu13,G12,G23,G13): the
// normal 3x3 block is the inverse of the compliance block that
// ElasticMaterial::read builds (elastic.cpp:358-363); shear terms are G.
// Output: n[6] = (N00,N01,N02,N11,N12,N22), g[3] = (G12,G23,G13).
__device__ __forceinline__ void ortho_c(const double* m, double* n, double* g) {
  double S[9];
  S[0] = 1.0 / m[0];
  S[1] = S[3] = -m[3] / m[0];
  S[2] = S[6] = -m[5] / m[0];
  S[4] = 1.0 / m[1];
  S[5] = S[7] = -m[4] / m[1];
  S[8] = 1.0 / m[2];
  double Ci[9];
  inv3<double>(S, Ci);
  n[0] = Ci[0]; n[1] = Ci[1]; n[2] = Ci[2]; n[3] = Ci[4]; n[4] = Ci[5]; n[5] = Ci[8];
  g[0] = m[6]; g[1] = m[7]; g[2] = m[8];
}

// Plane-stress C from (E11,E22,nu12,G12) (pStress.cpp:68-85):
// c = (C00, C01, C11, C22).
__device__ __forceinline__ void pstress_c(const double* m, double* c) {
  double s11 = 1.0 / m[0], s12 = -m[2] / m[0], s22 = 1.0 / m[1];
  double den = s11 * s22 - s12 * s12;
  c[0] = s22 / den;
  c[1] = -s12 / den;
  c[2] = s11 / den;
  c[3] = m[3];
}

}  // namespace betagpu
