// post_kernels.cuh -- element volume integrals after a solve.
//
// ElasticityElement3D::getVolAvgValues (ElasticityElement3D.cpp:417-558): at
// every integration point dV = detJ w (unit thickness), strain = B u_e
// (engineering shear; hex8 xx,yy,zz,xy,yz,xz, quad4 xx,yy,xy), stress =
// C strain, and per element volume = sum dV, stress_int = sum stress dV,
// strain_int = sum strain dV, energy = sum 0.5 stress.strain dV.  One thread
// per element, FP64; coordinates relative to the element's first node.
#pragma once
#include "common.cuh"

namespace betagpu {

// out row per element: [volume, stress_int[6], strain_int[6], energy]
__global__ void __launch_bounds__(128) k_outputs_hex8(int nelem, const double* __restrict__ xyz,
                                                     const int* __restrict__ conn,
                                                     const double* __restrict__ gparams,
                                                     const int* __restrict__ egroup, int nparams,
                                                     const GaussTable* __restrict__ gt, const double* __restrict__ u,
                                                     double* __restrict__ out) {
  __shared__ double s_dN[kMaxIP * 24], s_w[kMaxIP];
  const int nip = gt->nip;
  for (int i = threadIdx.x; i < nip * 24; i += blockDim.x) s_dN[i] = gt->dN[i / 24][(i / 8) % 3][i % 8];
  for (int i = threadIdx.x; i < nip; i += blockDim.x) s_w[i] = gt->w[i];
  __syncthreads();
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nelem) return;
  const int* ce = conn + (long long)e * 8;
  double x[8][3], ue[8][3];
  const int n0 = ce[0];
#pragma unroll
  for (int a = 0; a < 8; ++a) {
    const int J = ce[a];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      x[a][c] = xyz[3LL * J + c] - xyz[3LL * n0 + c];
      ue[a][c] = u[3LL * J + c];
    }
  }
  double nn[6], gg[3];
  ortho_c(gparams + (long long)(egroup ? egroup[e] : e) * nparams, nn, gg);
  double vol = 0, sig_i[6] = {0, 0, 0, 0, 0, 0}, eps_i[6] = {0, 0, 0, 0, 0, 0}, en = 0;
  for (int ip = 0; ip < nip; ++ip) {
    const double* d = s_dN + ip * 24;
    double M[9];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        double t = 0;
#pragma unroll
        for (int a = 0; a < 8; ++a) t += d[r * 8 + a] * x[a][c];
        M[r * 3 + c] = t;
      }
    double Mi[9];
    const double det = inv3<double>(M, Mi);
    double G[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};  // du_i / dx_c
#pragma unroll
    for (int a = 0; a < 8; ++a) {
      const double g0 = Mi[0] * d[a] + Mi[1] * d[8 + a] + Mi[2] * d[16 + a];
      const double g1 = Mi[3] * d[a] + Mi[4] * d[8 + a] + Mi[5] * d[16 + a];
      const double g2 = Mi[6] * d[a] + Mi[7] * d[8 + a] + Mi[8] * d[16 + a];
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        G[3 * i] += ue[a][i] * g0;
        G[3 * i + 1] += ue[a][i] * g1;
        G[3 * i + 2] += ue[a][i] * g2;
      }
    }
    const double eps[6] = {G[0], G[4], G[8], G[1] + G[3], G[5] + G[7], G[2] + G[6]};
    const double sig[6] = {nn[0] * eps[0] + nn[1] * eps[1] + nn[2] * eps[2],
                           nn[1] * eps[0] + nn[3] * eps[1] + nn[4] * eps[2],
                           nn[2] * eps[0] + nn[4] * eps[1] + nn[5] * eps[2],
                           gg[0] * eps[3], gg[1] * eps[4], gg[2] * eps[5]};
    const double dv = det * s_w[ip];
    vol += dv;
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      sig_i[k] += sig[k] * dv;
      eps_i[k] += eps[k] * dv;
      en += 0.5 * sig[k] * eps[k] * dv;
    }
  }
  double* o = out + (long long)e * 14;
  o[0] = vol;
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    o[1 + k] = sig_i[k];
    o[7 + k] = eps_i[k];
  }
  o[13] = en;
}

// out row per element: [area, stress_int[3], strain_int[3], energy]
__global__ void __launch_bounds__(128) k_outputs_quad4(int nelem, const double* __restrict__ xyz,
                                                      const int* __restrict__ conn,
                                                      const double* __restrict__ gparams,
                                                      const int* __restrict__ egroup, int nparams,
                                                      const GaussTable* __restrict__ gt, const double* __restrict__ u,
                                                      double* __restrict__ out) {
  __shared__ double s_dN[kMaxIP * 8], s_w[kMaxIP];
  const int nip = gt->nip;
  for (int i = threadIdx.x; i < nip * 8; i += blockDim.x) s_dN[i] = gt->dN[i / 8][(i / 4) % 2][i % 4];
  for (int i = threadIdx.x; i < nip; i += blockDim.x) s_w[i] = gt->w[i];
  __syncthreads();
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nelem) return;
  const int* ce = conn + (long long)e * 4;
  double x[4][2], ue[4][2];
  const int n0 = ce[0];
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    const int J = ce[a];
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      x[a][c] = xyz[2LL * J + c] - xyz[2LL * n0 + c];
      ue[a][c] = u[2LL * J + c];
    }
  }
  double pc[4];
  pstress_c(gparams + (long long)(egroup ? egroup[e] : e) * nparams, pc);
  double vol = 0, sig_i[3] = {0, 0, 0}, eps_i[3] = {0, 0, 0}, en = 0;
  for (int ip = 0; ip < nip; ++ip) {
    const double* d = s_dN + ip * 8;
    double J00 = 0, J01 = 0, J10 = 0, J11 = 0;
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      J00 += d[a] * x[a][0];
      J01 += d[a] * x[a][1];
      J10 += d[4 + a] * x[a][0];
      J11 += d[4 + a] * x[a][1];
    }
    const double det = J00 * J11 - J01 * J10, t = 1.0 / det;
    const double i00 = J11 * t, i01 = -J01 * t, i10 = -J10 * t, i11 = J00 * t;
    double e0 = 0, e1 = 0, e2 = 0;
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      const double g0 = i00 * d[a] + i01 * d[4 + a];
      const double g1 = i10 * d[a] + i11 * d[4 + a];
      e0 += g0 * ue[a][0];
      e1 += g1 * ue[a][1];
      e2 += g1 * ue[a][0] + g0 * ue[a][1];
    }
    const double eps[3] = {e0, e1, e2};
    const double sig[3] = {pc[0] * e0 + pc[1] * e1, pc[1] * e0 + pc[2] * e1, pc[3] * e2};
    const double dv = det * s_w[ip];
    vol += dv;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      sig_i[k] += sig[k] * dv;
      eps_i[k] += eps[k] * dv;
      en += 0.5 * sig[k] * eps[k] * dv;
    }
  }
  double* o = out + (long long)e * 8;
  o[0] = vol;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    o[1 + k] = sig_i[k];
    o[4 + k] = eps_i[k];
  }
  o[7] = en;
}

}  // namespace betagpu
