// mf_kernels.cuh -- FP64 matrix-free element operators.
//
//   y += K (c1*w1 + c2*w2) + cm * M w1
//
// evaluated element by element from the mesh, in FP64 (the outer residual of
// mixed-precision refinement and the internal force).  Per Gauss point:
// displacement gradient, strain (engineering shear), stress = C strain, and
// Fe += B^T stress * detJ * w -- ElasticityElement3D::derivativesOfFields /
// calculateStrain / calculateFe / addToFe (ElasticityElement3D.cpp:162-207,
// 124-134, 1053-1065, 41-55) with ElasticMaterial::calculateStress
// (elastic.cpp:411-451); for diffusion flux = k grad T and the capacity term
// (HeatTransferElement3DTransient.cpp:41-77).  One lane per element node, the
// element-level sums by xor butterflies; colours make the scatter exclusive.
#pragma once
#include "common.cuh"

namespace betagpu {

struct MfArgs {
  const double* xyz;
  const int* conn;
  const double* gparams;
  const int* egroup;
  int nparams;
  int nip;
  const GaussTable* gt;
  double c1, c2, cm;
};

// hex8 elasticity: 8 lanes per element, 4 elements per warp.
__device__ __forceinline__ void mf_hex8_elastic_warp(const MfArgs& A, const int* __restrict__ elems, int nel, int w,
    const double* w1, const double* w2, double* y, const double* s_dN, const double* s_w) {
  const int lane = threadIdx.x & 31, b = lane & 7;
  {
    const int idx = 4 * w + (lane >> 3);
    const bool valid = idx < nel;
    const int e = elems[valid ? idx : nel - 1];
    const int* ce = A.conn + (long long)e * 8;
    const int J = ce[b], n0 = ce[0];
    double xr[3], u[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      xr[c] = A.xyz[3LL * J + c] - A.xyz[3LL * n0 + c];
      u[c] = A.c1 * w1[3LL * J + c] + (w2 ? A.c2 * w2[3LL * J + c] : 0.0);
    }
    double nn[6], gg[3];
    ortho_c(A.gparams + (long long)(A.egroup ? A.egroup[e] : e) * A.nparams, nn, gg);
    double f0 = 0, f1 = 0, f2 = 0;
    for (int ip = 0; ip < A.nip; ++ip) {
      const double d0 = s_dN[ip * 24 + b], d1 = s_dN[ip * 24 + 8 + b], d2 = s_dN[ip * 24 + 16 + b];
      double M[9];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        M[c] = group_sum<8>(d0 * xr[c]);
        M[3 + c] = group_sum<8>(d1 * xr[c]);
        M[6 + c] = group_sum<8>(d2 * xr[c]);
      }
      double Mi[9];
      const double det = inv3<double>(M, Mi);
      const double g0 = Mi[0] * d0 + Mi[1] * d1 + Mi[2] * d2;
      const double g1 = Mi[3] * d0 + Mi[4] * d1 + Mi[5] * d2;
      const double g2 = Mi[6] * d0 + Mi[7] * d1 + Mi[8] * d2;
      double G[9];  // du_i/dx_c
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        G[3 * i] = group_sum<8>(u[i] * g0);
        G[3 * i + 1] = group_sum<8>(u[i] * g1);
        G[3 * i + 2] = group_sum<8>(u[i] * g2);
      }
      const double e0 = G[0], e1 = G[4], e2 = G[8];
      const double e3 = G[1] + G[3], e4 = G[5] + G[7], e5 = G[2] + G[6];
      const double s0 = nn[0] * e0 + nn[1] * e1 + nn[2] * e2;
      const double s1 = nn[1] * e0 + nn[3] * e1 + nn[4] * e2;
      const double s2 = nn[2] * e0 + nn[4] * e1 + nn[5] * e2;
      const double s3 = gg[0] * e3, s4 = gg[1] * e4, s5 = gg[2] * e5;
      const double fw = det * s_w[ip];
      f0 += fw * (g0 * s0 + g1 * s3 + g2 * s5);
      f1 += fw * (g1 * s1 + g0 * s3 + g2 * s4);
      f2 += fw * (g2 * s2 + g1 * s4 + g0 * s5);
    }
    if (valid) {
      y[3LL * J] += f0;
      y[3LL * J + 1] += f1;
      y[3LL * J + 2] += f2;
    }
  }
}

__global__ void __launch_bounds__(256) k_mf_hex8_elastic(MfArgs A, const int* __restrict__ elems, int nel,
    const double* __restrict__ w1, const double* __restrict__ w2, double* __restrict__ y) {
  __shared__ double s_dN[kMaxIP * 24];
  __shared__ double s_w[kMaxIP];
  for (int i = threadIdx.x; i < A.nip * 24; i += blockDim.x)
    s_dN[i] = A.gt->dN[i / 24][(i / 8) % 3][i % 8];
  for (int i = threadIdx.x; i < A.nip; i += blockDim.x) s_w[i] = A.gt->w[i];
  __syncthreads();
  const int wpb = blockDim.x >> 5;
  for (int w = blockIdx.x * wpb + (threadIdx.x >> 5); 4 * w < nel; w += gridDim.x * wpb)
    mf_hex8_elastic_warp(A, elems, nel, w, w1, w2, y, s_dN, s_w);
}

// Geometric-nonlinear internal force of hex8 elasticity at displacement u
// (ElasticityElement3D with analysisType GEOMETRIC_NONLINEAR, update("F")):
// per Gauss point F = I + grad u, the Green-Lagrange strain E (engineering
// shear, calculateStrain :124-160), S = C E, and Fe_b = B_b^T S = F (S dN_b)
// (the nonlinear B of calculateBmatrix :84-119 in addToFe :41-55); y += Fe.
// 8 lanes per element, 4 elements per warp, as mf_hex8_elastic_warp.
__device__ __forceinline__ void fint_hex8_gnl_warp(const MfArgs& A, const int* __restrict__ elems, int nel, int w,
                                                   const double* u, double* y, const double* s_dN, const double* s_w) {
  const int lane = threadIdx.x & 31, b = lane & 7;
  const int idx = 4 * w + (lane >> 3);
  const bool valid = idx < nel;
  const int e = elems[valid ? idx : nel - 1];
  const int* ce = A.conn + (long long)e * 8;
  const int J = ce[b], n0 = ce[0];
  double xr[3], ub[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    xr[c] = A.xyz[3LL * J + c] - A.xyz[3LL * n0 + c];
    ub[c] = u[3LL * J + c];
  }
  double nn[6], gg[3];
  ortho_c(A.gparams + (long long)(A.egroup ? A.egroup[e] : e) * A.nparams, nn, gg);
  double f0 = 0, f1 = 0, f2 = 0;
  for (int ip = 0; ip < A.nip; ++ip) {
    const double d0 = s_dN[ip * 24 + b], d1 = s_dN[ip * 24 + 8 + b], d2 = s_dN[ip * 24 + 16 + b];
    double M[9];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      M[c] = group_sum<8>(d0 * xr[c]);
      M[3 + c] = group_sum<8>(d1 * xr[c]);
      M[6 + c] = group_sum<8>(d2 * xr[c]);
    }
    double Mi[9];
    const double det = inv3<double>(M, Mi);
    const double g0 = Mi[0] * d0 + Mi[1] * d1 + Mi[2] * d2;
    const double g1 = Mi[3] * d0 + Mi[4] * d1 + Mi[5] * d2;
    const double g2 = Mi[6] * d0 + Mi[7] * d1 + Mi[8] * d2;
    double H[9];  // du_k/dx_j
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      H[3 * k] = group_sum<8>(ub[k] * g0);
      H[3 * k + 1] = group_sum<8>(ub[k] * g1);
      H[3 * k + 2] = group_sum<8>(ub[k] * g2);
    }
    const double E0 = H[0] + 0.5 * (H[0] * H[0] + H[3] * H[3] + H[6] * H[6]);
    const double E1 = H[4] + 0.5 * (H[1] * H[1] + H[4] * H[4] + H[7] * H[7]);
    const double E2 = H[8] + 0.5 * (H[2] * H[2] + H[5] * H[5] + H[8] * H[8]);
    const double E3 = H[1] + H[3] + H[0] * H[1] + H[3] * H[4] + H[6] * H[7];
    const double E4 = H[5] + H[7] + H[1] * H[2] + H[4] * H[5] + H[7] * H[8];
    const double E5 = H[2] + H[6] + H[0] * H[2] + H[3] * H[5] + H[6] * H[8];
    const double S0 = nn[0] * E0 + nn[1] * E1 + nn[2] * E2;
    const double S1 = nn[1] * E0 + nn[3] * E1 + nn[4] * E2;
    const double S2 = nn[2] * E0 + nn[4] * E1 + nn[5] * E2;
    const double S3 = gg[0] * E3, S4 = gg[1] * E4, S5 = gg[2] * E5;
    const double sg0 = S0 * g0 + S3 * g1 + S5 * g2;
    const double sg1 = S3 * g0 + S1 * g1 + S4 * g2;
    const double sg2 = S5 * g0 + S4 * g1 + S2 * g2;
    const double fw = det * s_w[ip];
    f0 += fw * ((1.0 + H[0]) * sg0 + H[1] * sg1 + H[2] * sg2);
    f1 += fw * (H[3] * sg0 + (1.0 + H[4]) * sg1 + H[5] * sg2);
    f2 += fw * (H[6] * sg0 + H[7] * sg1 + (1.0 + H[8]) * sg2);
  }
  if (valid) {
    y[3LL * J] += f0;
    y[3LL * J + 1] += f1;
    y[3LL * J + 2] += f2;
  }
}

__global__ void __launch_bounds__(256) k_fint_hex8_gnl(MfArgs A, const int* __restrict__ elems, int nel,
                                                       const double* __restrict__ u, double* __restrict__ y) {
  __shared__ double s_dN[kMaxIP * 24];
  __shared__ double s_w[kMaxIP];
  for (int i = threadIdx.x; i < A.nip * 24; i += blockDim.x)
    s_dN[i] = A.gt->dN[i / 24][(i / 8) % 3][i % 8];
  for (int i = threadIdx.x; i < A.nip; i += blockDim.x) s_w[i] = A.gt->w[i];
  __syncthreads();
  const int wpb = blockDim.x >> 5;
  for (int w = blockIdx.x * wpb + (threadIdx.x >> 5); 4 * w < nel; w += gridDim.x * wpb)
    fint_hex8_gnl_warp(A, elems, nel, w, u, y, s_dN, s_w);
}

// quad4 plane stress: 4 lanes per element, 8 elements per warp.
__device__ __forceinline__ void mf_quad4_pstress_warp(const MfArgs& A, const int* __restrict__ elems, int nel, int w,
    const double* w1, const double* w2, double* y, const double* s_dN, const double* s_w) {
  const int lane = threadIdx.x & 31, b = lane & 3;
  {
    const int idx = 8 * w + (lane >> 2);
    const bool valid = idx < nel;
    const int e = elems[valid ? idx : nel - 1];
    const int* ce = A.conn + (long long)e * 4;
    const int J = ce[b], n0 = ce[0];
    const double xr0 = A.xyz[2LL * J] - A.xyz[2LL * n0], xr1 = A.xyz[2LL * J + 1] - A.xyz[2LL * n0 + 1];
    const double u0 = A.c1 * w1[2LL * J] + (w2 ? A.c2 * w2[2LL * J] : 0.0);
    const double u1 = A.c1 * w1[2LL * J + 1] + (w2 ? A.c2 * w2[2LL * J + 1] : 0.0);
    double cc[4];
    pstress_c(A.gparams + (long long)(A.egroup ? A.egroup[e] : e) * A.nparams, cc);
    double f0 = 0, f1 = 0;
    for (int ip = 0; ip < A.nip; ++ip) {
      const double d0 = s_dN[ip * 8 + b], d1 = s_dN[ip * 8 + 4 + b];
      const double M00 = group_sum<4>(d0 * xr0), M01 = group_sum<4>(d0 * xr1);
      const double M10 = group_sum<4>(d1 * xr0), M11 = group_sum<4>(d1 * xr1);
      const double det = M00 * M11 - M01 * M10, id = 1.0 / det;
      const double g0 = (M11 * d0 - M01 * d1) * id, g1 = (-M10 * d0 + M00 * d1) * id;
      const double G00 = group_sum<4>(u0 * g0), G01 = group_sum<4>(u0 * g1);
      const double G10 = group_sum<4>(u1 * g0), G11 = group_sum<4>(u1 * g1);
      const double e0 = G00, e1 = G11, e2 = G01 + G10;
      const double s0 = cc[0] * e0 + cc[1] * e1, s1 = cc[1] * e0 + cc[2] * e1, s2 = cc[3] * e2;
      const double fw = det * s_w[ip];
      f0 += fw * (g0 * s0 + g1 * s2);
      f1 += fw * (g1 * s1 + g0 * s2);
    }
    if (valid) {
      y[2LL * J] += f0;
      y[2LL * J + 1] += f1;
    }
  }
}

__global__ void __launch_bounds__(256) k_mf_quad4_pstress(MfArgs A, const int* __restrict__ elems, int nel,
    const double* __restrict__ w1, const double* __restrict__ w2, double* __restrict__ y) {
  __shared__ double s_dN[kMaxIP * 8];
  __shared__ double s_w[kMaxIP];
  for (int i = threadIdx.x; i < A.nip * 8; i += blockDim.x) s_dN[i] = A.gt->dN[i / 8][(i / 4) % 2][i % 4];
  for (int i = threadIdx.x; i < A.nip; i += blockDim.x) s_w[i] = A.gt->w[i];
  __syncthreads();
  const int wpb = blockDim.x >> 5;
  for (int w = blockIdx.x * wpb + (threadIdx.x >> 5); 8 * w < nel; w += gridDim.x * wpb)
    mf_quad4_pstress_warp(A, elems, nel, w, w1, w2, y, s_dN, s_w);
}

// quad4 diffusion: y += K (c1 w1 + c2 w2) + cm M w1, 4 lanes per element
// (unit thickness, k12 = 0 as in the assembly).
__device__ __forceinline__ void mf_quad4_heat_warp(const MfArgs& A, const int* __restrict__ elems, int nel, int w,
    const double* w1, const double* w2, double* y, const double* s_dN, const double* s_N, const double* s_w) {
  const int lane = threadIdx.x & 31, b = lane & 3;
  const int idx = 8 * w + (lane >> 2);
  const bool valid = idx < nel;
  const int e = elems[valid ? idx : nel - 1];
  const int* ce = A.conn + (long long)e * 4;
  const int J = ce[b], n0 = ce[0];
  const double xr0 = A.xyz[2LL * J] - A.xyz[2LL * n0], xr1 = A.xyz[2LL * J + 1] - A.xyz[2LL * n0 + 1];
  const double vk = A.c1 * w1[J] + (w2 ? A.c2 * w2[J] : 0.0);
  const double vm = w1[J];
  const double* pm = A.gparams + (long long)(A.egroup ? A.egroup[e] : e) * A.nparams;
  double f = 0;
  for (int ip = 0; ip < A.nip; ++ip) {
    const double d0 = s_dN[ip * 8 + b], d1 = s_dN[ip * 8 + 4 + b];
    const double M00 = group_sum<4>(d0 * xr0), M01 = group_sum<4>(d0 * xr1);
    const double M10 = group_sum<4>(d1 * xr0), M11 = group_sum<4>(d1 * xr1);
    const double det = M00 * M11 - M01 * M10, id = 1.0 / det;
    const double g0 = (M11 * d0 - M01 * d1) * id, g1 = (-M10 * d0 + M00 * d1) * id;
    const double t0 = group_sum<4>(vk * g0), t1 = group_sum<4>(vk * g1);
    const double Sb = s_N[ip * 4 + b];
    const double tv = group_sum<4>(vm * Sb);
    const double fw = det * s_w[ip];
    f += fw * (g0 * pm[0] * t0 + g1 * pm[1] * t1 + A.cm * pm[3] * Sb * tv);
  }
  if (valid) y[J] += f;
}

__global__ void __launch_bounds__(256) k_mf_quad4_heat(MfArgs A, const int* __restrict__ elems, int nel,
    const double* __restrict__ w1, const double* __restrict__ w2, double* __restrict__ y) {
  __shared__ double s_dN[kMaxIP * 8];
  __shared__ double s_N[kMaxIP * 4];
  __shared__ double s_w[kMaxIP];
  for (int i = threadIdx.x; i < A.nip * 8; i += blockDim.x) s_dN[i] = A.gt->dN[i / 8][(i / 4) % 2][i % 4];
  for (int i = threadIdx.x; i < A.nip * 4; i += blockDim.x) s_N[i] = A.gt->N[i / 4][i % 4];
  for (int i = threadIdx.x; i < A.nip; i += blockDim.x) s_w[i] = A.gt->w[i];
  __syncthreads();
  const int wpb = blockDim.x >> 5;
  for (int w = blockIdx.x * wpb + (threadIdx.x >> 5); 8 * w < nel; w += gridDim.x * wpb)
    mf_quad4_heat_warp(A, elems, nel, w, w1, w2, y, s_dN, s_N, s_w);
}

// hex8 diffusion: y += K (c1 w1 + c2 w2) + cm M w1, 8 lanes per element.
__device__ __forceinline__ void mf_hex8_heat_warp(const MfArgs& A, const int* __restrict__ elems, int nel, int w,
    const double* w1, const double* w2, double* y, const double* s_dN, const double* s_N, const double* s_w) {
  const int lane = threadIdx.x & 31, b = lane & 7;
  {
    const int idx = 4 * w + (lane >> 3);
    const bool valid = idx < nel;
    const int e = elems[valid ? idx : nel - 1];
    const int* ce = A.conn + (long long)e * 8;
    const int J = ce[b], n0 = ce[0];
    double xr[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) xr[c] = A.xyz[3LL * J + c] - A.xyz[3LL * n0 + c];
    const double vk = A.c1 * w1[J] + (w2 ? A.c2 * w2[J] : 0.0);
    const double vm = w1[J];
    const double* pm = A.gparams + (long long)(A.egroup ? A.egroup[e] : e) * A.nparams;
    double f = 0;
    for (int ip = 0; ip < A.nip; ++ip) {
      const double d0 = s_dN[ip * 24 + b], d1 = s_dN[ip * 24 + 8 + b], d2 = s_dN[ip * 24 + 16 + b];
      double M[9];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        M[c] = group_sum<8>(d0 * xr[c]);
        M[3 + c] = group_sum<8>(d1 * xr[c]);
        M[6 + c] = group_sum<8>(d2 * xr[c]);
      }
      double Mi[9];
      const double det = inv3<double>(M, Mi);
      const double g0 = Mi[0] * d0 + Mi[1] * d1 + Mi[2] * d2;
      const double g1 = Mi[3] * d0 + Mi[4] * d1 + Mi[5] * d2;
      const double g2 = Mi[6] * d0 + Mi[7] * d1 + Mi[8] * d2;
      const double t0 = group_sum<8>(vk * g0), t1 = group_sum<8>(vk * g1), t2 = group_sum<8>(vk * g2);
      const double Sb = s_N[ip * 8 + b];
      const double tv = group_sum<8>(vm * Sb);
      const double fw = det * s_w[ip];
      f += fw * (g0 * pm[0] * t0 + g1 * pm[1] * t1 + g2 * pm[2] * t2 + A.cm * pm[3] * Sb * tv);
    }
    if (valid) y[J] += f;
  }
}

// hex8 diffusion, one thread per element: y += K (c1 w1 + c2 w2) + cm M w1
// for element elems[i].  A scalar field has 8 unknowns per element, so the
// whole element fits in one thread's registers; compared with 8 lanes per
// element this trades 13 group sums (39 FP64 shuffles) per Gauss point for
// plain FMAs.  The element gradients are recomputed in the second pass
// instead of held (fewer registers).
__device__ __forceinline__ void mf_hex8_heat_elem(const MfArgs& A, int e, const double* w1, const double* w2,
                                                  double* y, const double* s_dN, const double* s_N,
                                                  const double* s_w) {
  const int* ce = A.conn + (long long)e * 8;
  int nd[8];
  double x[8][3], vk[8], vm[8], f[8];
  const int n0 = ce[0];
#pragma unroll
  for (int a = 0; a < 8; ++a) {
    nd[a] = ce[a];
#pragma unroll
    for (int c = 0; c < 3; ++c) x[a][c] = A.xyz[3LL * nd[a] + c] - A.xyz[3LL * n0 + c];
    vm[a] = w1[nd[a]];
    vk[a] = A.c1 * vm[a] + (w2 ? A.c2 * w2[nd[a]] : 0.0);
    f[a] = 0.0;
  }
  const double* pm = A.gparams + (long long)(A.egroup ? A.egroup[e] : e) * A.nparams;
  const double k0 = pm[0], k1 = pm[1], k2 = pm[2], cap = A.cm * pm[3];
  for (int ip = 0; ip < A.nip; ++ip) {
    const double* d = s_dN + ip * 24;
    const double* N = s_N + ip * 8;
    double M[9];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        double t = 0.0;
#pragma unroll
        for (int a = 0; a < 8; ++a) t += d[r * 8 + a] * x[a][c];
        M[r * 3 + c] = t;
      }
    double Mi[9];
    const double det = inv3<double>(M, Mi);
    double t0 = 0.0, t1 = 0.0, t2 = 0.0, tv = 0.0;
#pragma unroll
    for (int a = 0; a < 8; ++a) {
      const double g0 = Mi[0] * d[a] + Mi[1] * d[8 + a] + Mi[2] * d[16 + a];
      const double g1 = Mi[3] * d[a] + Mi[4] * d[8 + a] + Mi[5] * d[16 + a];
      const double g2 = Mi[6] * d[a] + Mi[7] * d[8 + a] + Mi[8] * d[16 + a];
      t0 += vk[a] * g0;
      t1 += vk[a] * g1;
      t2 += vk[a] * g2;
      tv += vm[a] * N[a];
    }
    const double fw = det * s_w[ip];
    const double q0 = fw * k0 * t0, q1 = fw * k1 * t1, q2 = fw * k2 * t2, qm = fw * cap * tv;
#pragma unroll
    for (int a = 0; a < 8; ++a) {
      const double g0 = Mi[0] * d[a] + Mi[1] * d[8 + a] + Mi[2] * d[16 + a];
      const double g1 = Mi[3] * d[a] + Mi[4] * d[8 + a] + Mi[5] * d[16 + a];
      const double g2 = Mi[6] * d[a] + Mi[7] * d[8 + a] + Mi[8] * d[16 + a];
      f[a] += g0 * q0 + g1 * q1 + g2 * q2 + N[a] * qm;
    }
  }
#pragma unroll
  for (int a = 0; a < 8; ++a) y[nd[a]] += f[a];
}

__global__ void __launch_bounds__(256) k_mf_hex8_heat_t(MfArgs A, const int* __restrict__ elems, int nel,
    const double* __restrict__ w1, const double* __restrict__ w2, double* __restrict__ y) {
  __shared__ double s_dN[kMaxIP * 24];
  __shared__ double s_N[kMaxIP * 8];
  __shared__ double s_w[kMaxIP];
  for (int i = threadIdx.x; i < A.nip * 24; i += blockDim.x)
    s_dN[i] = A.gt->dN[i / 24][(i / 8) % 3][i % 8];
  for (int i = threadIdx.x; i < A.nip * 8; i += blockDim.x) s_N[i] = A.gt->N[i / 8][i % 8];
  for (int i = threadIdx.x; i < A.nip; i += blockDim.x) s_w[i] = A.gt->w[i];
  __syncthreads();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nel; i += gridDim.x * blockDim.x)
    mf_hex8_heat_elem(A, elems[i], w1, w2, y, s_dN, s_N, s_w);
}

// ---- cached FP64 element matrices of the hex8 diffusion operator ----------
// For a mesh whose conductivity and capacity do not change between applies
// (linear k, the transient steps and repeated solves), the element integrals
// K_e = int k grad N grad N^T and M_e = int c N N^T are computed once and the
// operator y = K (c1 w1 + c2 w2) + cm M w1 reads them instead of
// re-integrating: 72 FP64 values per element (the upper triangles, 36 + 36)
// against about 2,400 FP64 multiply-adds at 2x2x2 Gauss points.  Layout:
// element k of the colour-ordered list holds value t at
// (k/32)*72*32 + t*32 + k%32, so a warp of consecutive threads reads 256
// contiguous bytes per value.  Upper-triangle index of (a, b), a <= b:
// a*8 - a*(a-1)/2 + (b - a).
constexpr int kMfcHeat = 72;

__device__ __forceinline__ int tri8(int a, int b) { return a * 8 - (a * (a - 1)) / 2 + (b - a); }

// One thread per element; KM = 0 integrates K_e, KM = 1 M_e (two passes keep
// the accumulators and the Gauss-point gradients in registers).
template <int KM>
__global__ void __launch_bounds__(256) k_mfc_build_hex8_heat(MfArgs A, const int* __restrict__ elems, int nel,
                                                              double* __restrict__ cache) {
  __shared__ double s_dN[kMaxIP * 24];
  __shared__ double s_N[kMaxIP * 8];
  __shared__ double s_w[kMaxIP];
  for (int i = threadIdx.x; i < A.nip * 24; i += blockDim.x)
    s_dN[i] = A.gt->dN[i / 24][(i / 8) % 3][i % 8];
  for (int i = threadIdx.x; i < A.nip * 8; i += blockDim.x) s_N[i] = A.gt->N[i / 8][i % 8];
  for (int i = threadIdx.x; i < A.nip; i += blockDim.x) s_w[i] = A.gt->w[i];
  __syncthreads();
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nel; k += gridDim.x * blockDim.x) {
    const int e = elems[k];
    const int* ce = A.conn + (long long)e * 8;
    double x[8][3];
    const int n0 = ce[0];
#pragma unroll
    for (int a = 0; a < 8; ++a)
#pragma unroll
      for (int c = 0; c < 3; ++c) x[a][c] = A.xyz[3LL * ce[a] + c] - A.xyz[3LL * n0 + c];
    const double* pm = A.gparams + (long long)(A.egroup ? A.egroup[e] : e) * A.nparams;
    const double k0 = pm[0], k1 = pm[1], k2 = pm[2], cap = pm[3];
    double acc[36];
#pragma unroll
    for (int t = 0; t < 36; ++t) acc[t] = 0.0;
    for (int ip = 0; ip < A.nip; ++ip) {
      const double* d = s_dN + ip * 24;
      const double* N = s_N + ip * 8;
      double M[9];
#pragma unroll
      for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          double t = 0.0;
#pragma unroll
          for (int a = 0; a < 8; ++a) t += d[r * 8 + a] * x[a][c];
          M[r * 3 + c] = t;
        }
      double Mi[9];
      const double fw = inv3<double>(M, Mi) * s_w[ip];
      if constexpr (KM == 0) {
        double g[3][8];
#pragma unroll
        for (int a = 0; a < 8; ++a) {
          g[0][a] = Mi[0] * d[a] + Mi[1] * d[8 + a] + Mi[2] * d[16 + a];
          g[1][a] = Mi[3] * d[a] + Mi[4] * d[8 + a] + Mi[5] * d[16 + a];
          g[2][a] = Mi[6] * d[a] + Mi[7] * d[8 + a] + Mi[8] * d[16 + a];
        }
        const double w0 = fw * k0, w1 = fw * k1, w2 = fw * k2;
#pragma unroll
        for (int a = 0; a < 8; ++a)
#pragma unroll
          for (int b = a; b < 8; ++b)
            acc[tri8(a, b)] += w0 * g[0][a] * g[0][b] + w1 * g[1][a] * g[1][b] + w2 * g[2][a] * g[2][b];
      } else {
        const double wm = fw * cap;
#pragma unroll
        for (int a = 0; a < 8; ++a)
#pragma unroll
          for (int b = a; b < 8; ++b) acc[tri8(a, b)] += wm * N[a] * N[b];
      }
    }
    double* out = cache + (long long)(k >> 5) * kMfcHeat * 32 + KM * 36 * 32 + (k & 31);
#pragma unroll
    for (int t = 0; t < 36; ++t) out[t * 32] = acc[t];
  }
}

// y += K_e (c1 w1 + c2 w2) + cm M_e w1 over the elements [beg, beg+nel) of
// the colour-ordered list (one colour: no two elements share a node).
__global__ void __launch_bounds__(256) k_mfc_apply_hex8_heat(const int* __restrict__ conn,
    const int* __restrict__ elems, int beg, int nel, const double* __restrict__ cache, double c1, double c2,
    double cm, const double* __restrict__ w1, const double* __restrict__ w2, double* __restrict__ y) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nel; i += gridDim.x * blockDim.x) {
    const int k = beg + i;
    const int* ce = conn + (long long)elems[k] * 8;
    int nd[8];
    double vk[8], vm[8], f[8];
#pragma unroll
    for (int a = 0; a < 8; ++a) {
      nd[a] = ce[a];
      vm[a] = w1[nd[a]];
      vk[a] = c1 * vm[a] + (w2 ? c2 * w2[nd[a]] : 0.0);
      f[a] = 0.0;
    }
    const double* Kc = cache + (long long)(k >> 5) * kMfcHeat * 32 + (k & 31);
    const double* Mc = Kc + 36 * 32;
    // a term whose scale is zero is not read (the step scale needs M alone,
    // the FP64 right-hand side K alone): half the bytes
    if (c1 != 0.0 || c2 != 0.0) {
#pragma unroll
      for (int a = 0; a < 8; ++a)
#pragma unroll
        for (int b = a; b < 8; ++b) {
          const double kv = __ldcs(Kc + tri8(a, b) * 32);
          f[a] += kv * vk[b];
          if (b != a) f[b] += kv * vk[a];
        }
    }
    if (cm != 0.0) {
#pragma unroll
      for (int a = 0; a < 8; ++a)
#pragma unroll
        for (int b = a; b < 8; ++b) {
          const double mv = cm * __ldcs(Mc + tri8(a, b) * 32);
          f[a] += mv * vm[b];
          if (b != a) f[b] += mv * vm[a];
        }
    }
#pragma unroll
    for (int a = 0; a < 8; ++a) y[nd[a]] += f[a];
  }
}

}  // namespace betagpu
