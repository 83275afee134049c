// elem_kernels.cuh -- element Gauss-point loops and the slot-mapped scatter.
//
// One warp owns a tile of elements (hex8: one element, quad4: two).  Lane
// (a,b) accumulates the ndpn x ndpn block K_ab of its local node pair(s) over
// the Gauss points; the Gauss tables (weights, N, dN/dxi) are staged in shared
// memory once per block.  The Jacobian M = sum_b dN_b/dxi (x) X_b is formed by
// a butterfly over the lanes of one element, using coordinates relative to
// the element's first node (no cancellation against absolute coordinates in
// FP32).  Elements of one colour share no node, so the scatter of K_ab into
// the global layouts is a plain read-modify-write: no atomics, a fixed
// summation order (colour by colour), bit-reproducible.
//
// Reference loops restated: ElasticityElement3D::loopOverIntegrationPoints
// + addToKe (ElasticityElement3D.cpp:983-1030, 560-611), ElasticityElement2D::
// addToKe (ElasticityElement2D.cpp:22-58), HeatTransferElement3Dtransient::
// addToKe/addToMe/formK_s (HeatTransferElement3DTransient.cpp:153-197, 60-77,
// 323-350), IsoElement::jacobian (isoElement.cpp:250-372), and the scatter of
// Equations::addMatrix (equation.cpp:445-562).
#pragma once
#include "common.cuh"

namespace betagpu {

struct ElemArgs {
  const double* xyz;          // nnode*ndim
  const int* conn;            // nelem*nnpe
  const double* gparams;      // ngroups*nparams
  const int* egroup;          // nelem or null
  int nparams;
  int nip;
  const GaussTable* gt;       // device
  const uint16_t* slot;       // nelem*nnpe*nnpe: position of node J in node I's graph row
  const int* nrp;             // node graph row pointers
  const unsigned char* rest;  // ndof
  const double* presc;        // ndof
  // FP32 node-block sliced ELL target; vpos: the block's virtual position
  // in its row for a layout of column runs (null: the graph position)
  const int* bsoff;
  const uint16_t* vpos;
  float* bval;
  // FP64 scalar sliced ELL target (+ pseudo load)
  const int* soff;
  const long long* ssoff;
  double* sval;
  double* pseudo;
  // heat: value = kscale*K + mscale*M
  double kscale, mscale;
  unsigned* flags;
};

// ---- shared-memory Gauss table staging --------------------------------
template <typename T, int NN, int NDIR>
__device__ __forceinline__ void stage_gauss(const GaussTable* gt, int nip, T* s_dN, T* s_N, T* s_w) {
  for (int i = threadIdx.x; i < nip * NDIR * NN; i += blockDim.x) {
    int ip = i / (NDIR * NN), r = (i / NN) % NDIR, a = i % NN;
    s_dN[i] = (T)gt->dN[ip][r][a];
  }
  for (int i = threadIdx.x; i < nip * NN; i += blockDim.x) s_N[i] = (T)gt->N[i / NN][i % NN];
  for (int i = threadIdx.x; i < nip; i += blockDim.x) s_w[i] = (T)gt->w[i];
  __syncthreads();
}

// ---- scatter of one ND x ND block K (row-major) for the node pair (I,J) --
// FP32 node-block layout: block (I, pos) lives in chunk bsoff[I/32] + v,
// v = pos (one column per block) or vpos[nrp[I] + pos] (column runs), entry
// (i,j) at chunk*32*ND*ND + (i*ND+j)*32 + I%32.  Restrained rows and
// columns stay zero; their diagonal is set to 1 afterwards (equation.cpp:500).
template <int ND>
__device__ __forceinline__ void scatter_block32(const ElemArgs& A, int I, int J, int pos,
                                                const float* K) {
  const int v = A.vpos ? (int)A.vpos[A.nrp[I] + pos] : pos;
  const long long chunk = (long long)A.bsoff[I >> 5] + v;
  float* base = A.bval + chunk * (32 * ND * ND) + (I & 31);
#pragma unroll
  for (int i = 0; i < ND; ++i) {
    if (A.rest[I * ND + i]) continue;
#pragma unroll
    for (int j = 0; j < ND; ++j) {
      if (A.rest[J * ND + j]) continue;
      base[(i * ND + j) * 32] += K[i * ND + j];
    }
  }
}

// FP64 scalar layout: row r = I*ND+i (free rows only), column offset of node
// J's first free dof = soff[blk]; restrained columns move to the pseudo load
// as F[I] -= K_IJ * u_J (equation.cpp:499-503).  Returns the row partials of
// the pseudo load in pl[ND].
template <int ND>
__device__ __forceinline__ void scatter_block64(const ElemArgs& A, int I, int J, int pos,
                                                const double* K, double* pl) {
  const int kb = A.soff[A.nrp[I] + pos];
#pragma unroll
  for (int i = 0; i < ND; ++i) {
    pl[i] = 0.0;
    const int r = I * ND + i;
    if (A.rest[r]) continue;
    const long long rowbase = A.ssoff[r >> 5] + (r & 31);
    int k = kb;
#pragma unroll
    for (int j = 0; j < ND; ++j) {
      const int c = J * ND + j;
      if (A.rest[c]) {
        pl[i] -= K[i * ND + j] * A.presc[c];
      } else {
        A.sval[rowbase + (long long)k * 32] += K[i * ND + j];
        ++k;
      }
    }
  }
}

// ---- hex8 linear elasticity, one warp per element ------------------------
// lane = 8*a0 + b handles pairs (a0,b) and (a0+4,b).
template <typename T>
__device__ __forceinline__ void asm_hex8_elastic_warp(const ElemArgs& A, const int* __restrict__ elems, int nel, int w,
    const T* s_dN, const T* s_N, const T* s_w) {
  const int lane = threadIdx.x & 31;
  const int b = lane & 7, a0 = lane >> 3, a1 = a0 + 4;
  {
    const int e = elems[w];
    const int* ce = A.conn + (long long)e * 8;
    const int J = ce[b];
    const int n0 = ce[0];
    T xr[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) xr[c] = (T)(A.xyz[3LL * J + c] - A.xyz[3LL * n0 + c]);
    double nn[6], gg[3];
    ortho_c(A.gparams + (long long)(A.egroup ? A.egroup[e] : e) * A.nparams, nn, gg);
    const T N00 = nn[0], N01 = nn[1], N02 = nn[2], N11 = nn[3], N12 = nn[4], N22 = nn[5];
    const T G4 = gg[0], G5 = gg[1], G6 = gg[2];
    T K0[9], K1[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) K0[k] = K1[k] = T(0);

    for (int ip = 0; ip < A.nip; ++ip) {
      const T* dn = s_dN + ip * 24;
      const T d0 = dn[b], d1 = dn[8 + b], d2 = dn[16 + b];
      T M[9];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        M[c] = group_sum<8>(d0 * xr[c]);
        M[3 + c] = group_sum<8>(d1 * xr[c]);
        M[6 + c] = group_sum<8>(d2 * xr[c]);
      }
      T Mi[9];
      const T det = inv3<T>(M, Mi);
      const T f = det * s_w[ip];
      const T g0 = Mi[0] * d0 + Mi[1] * d1 + Mi[2] * d2;
      const T g1 = Mi[3] * d0 + Mi[4] * d1 + Mi[5] * d2;
      const T g2 = Mi[6] * d0 + Mi[7] * d1 + Mi[8] * d2;
      T h[2][3];
      h[0][0] = __shfl_sync(0xffffffffu, g0, a0);
      h[0][1] = __shfl_sync(0xffffffffu, g1, a0);
      h[0][2] = __shfl_sync(0xffffffffu, g2, a0);
      h[1][0] = __shfl_sync(0xffffffffu, g0, a1);
      h[1][1] = __shfl_sync(0xffffffffu, g1, a1);
      h[1][2] = __shfl_sync(0xffffffffu, g2, a1);
      // K_ab = B_a^T C B_b for orthotropic C (Voigt xx,yy,zz,xy,yz,xz,
      // engineering shear), only the non-zero products of B.
#pragma unroll
      for (int p = 0; p < 2; ++p) {
        T* K = p ? K1 : K0;
        const T x0 = h[p][0] * f, x1 = h[p][1] * f, x2 = h[p][2] * f;
        K[0] += x0 * N00 * g0 + x1 * G4 * g1 + x2 * G6 * g2;
        K[1] += x0 * N01 * g1 + x1 * G4 * g0;
        K[2] += x0 * N02 * g2 + x2 * G6 * g0;
        K[3] += x1 * N01 * g0 + x0 * G4 * g1;
        K[4] += x1 * N11 * g1 + x0 * G4 * g0 + x2 * G5 * g2;
        K[5] += x1 * N12 * g2 + x2 * G5 * g1;
        K[6] += x2 * N02 * g0 + x0 * G6 * g2;
        K[7] += x2 * N12 * g1 + x1 * G5 * g2;
        K[8] += x2 * N22 * g2 + x1 * G5 * g1 + x0 * G6 * g0;
      }
    }
    // checkForNegativeDiagonal (BasicElement.cpp:116-130)
    if ((b == a0 && !(K0[0] > 0 && K0[4] > 0 && K0[8] > 0)) ||
        (b == a1 && !(K1[0] > 0 && K1[4] > 0 && K1[8] > 0)))
      atomicOr(A.flags, kFlagNegDiag);

    const int I0 = __shfl_sync(0xffffffffu, J, a0);
    const int I1 = __shfl_sync(0xffffffffu, J, a1);
    const uint16_t* sl = A.slot + (long long)e * 64;
    if constexpr (sizeof(T) == 4) {
      scatter_block32<3>(A, I0, J, sl[a0 * 8 + b], K0);
      scatter_block32<3>(A, I1, J, sl[a1 * 8 + b], K1);
    } else {
      double pl0[3], pl1[3];
      scatter_block64<3>(A, I0, J, sl[a0 * 8 + b], K0, pl0);
      scatter_block64<3>(A, I1, J, sl[a1 * 8 + b], K1, pl1);
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        pl0[i] = group_sum<8>(pl0[i]);
        pl1[i] = group_sum<8>(pl1[i]);
      }
      if (b == 0) {
#pragma unroll
        for (int i = 0; i < 3; ++i) {
          if (!A.rest[I0 * 3 + i]) A.pseudo[I0 * 3 + i] += pl0[i];
          if (!A.rest[I1 * 3 + i]) A.pseudo[I1 * 3 + i] += pl1[i];
        }
      }
    }
  }
}

template <typename T>
__global__ void __launch_bounds__(256) k_asm_hex8_elastic(ElemArgs A, const int* __restrict__ elems,
    int nel) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* s_dN = reinterpret_cast<T*>(smem_raw);
  T* s_N = s_dN + A.nip * 24;
  T* s_w = s_N + A.nip * 8;
  stage_gauss<T, 8, 3>(A.gt, A.nip, s_dN, s_N, s_w);
  const int wpb = blockDim.x >> 5;
  for (int w = blockIdx.x * wpb + (threadIdx.x >> 5); w < nel; w += gridDim.x * wpb)
    asm_hex8_elastic_warp<T>(A, elems, nel, w, s_dN, s_N, s_w);
}

// ---- hex8 geometric-nonlinear tangent (ElasticityElement3D with analysisType
// GEOMETRIC_NONLINEAR, ElasticityElement3D.cpp:84-119, 124-160, 560-641) ----
// At displacement u the strain-displacement rows of node a are those of the
// linear element applied to F^T, F = I + grad u (calculateBmatrix adds
// grad u * dN to every row), so the material block of a node pair is
// F K^L_ab F^T with K^L_ab the linear element's block above; the
// initial-stress term adds (dN_a . S dN_b) I, S = C E with E the
// Green-Lagrange strain (engineering shear) -- the stress the reference
// computes before addToKe when analysisType is GEOMETRIC_NONLINEAR.
template <typename T>
__device__ __forceinline__ void asm_hex8_gnl_warp(const ElemArgs& A, const int* __restrict__ elems, int nel, int w,
                                                  const double* __restrict__ u, const T* s_dN, const T* s_w) {
  const int lane = threadIdx.x & 31;
  const int b = lane & 7, a0 = lane >> 3, a1 = a0 + 4;
  const int e = elems[w];
  const int* ce = A.conn + (long long)e * 8;
  const int J = ce[b];
  const int n0 = ce[0];
  T xr[3], ub[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    xr[c] = (T)(A.xyz[3LL * J + c] - A.xyz[3LL * n0 + c]);
    ub[c] = (T)u[3LL * J + c];
  }
  double nn[6], gg[3];
  ortho_c(A.gparams + (long long)(A.egroup ? A.egroup[e] : e) * A.nparams, nn, gg);
  const T N00 = nn[0], N01 = nn[1], N02 = nn[2], N11 = nn[3], N12 = nn[4], N22 = nn[5];
  const T G4 = gg[0], G5 = gg[1], G6 = gg[2];
  T K0[9], K1[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) K0[k] = K1[k] = T(0);
  for (int ip = 0; ip < A.nip; ++ip) {
    const T* dn = s_dN + ip * 24;
    const T d0 = dn[b], d1 = dn[8 + b], d2 = dn[16 + b];
    T M[9];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      M[c] = group_sum<8>(d0 * xr[c]);
      M[3 + c] = group_sum<8>(d1 * xr[c]);
      M[6 + c] = group_sum<8>(d2 * xr[c]);
    }
    T Mi[9];
    const T det = inv3<T>(M, Mi);
    const T f = det * s_w[ip];
    const T g0 = Mi[0] * d0 + Mi[1] * d1 + Mi[2] * d2;
    const T g1 = Mi[3] * d0 + Mi[4] * d1 + Mi[5] * d2;
    const T g2 = Mi[6] * d0 + Mi[7] * d1 + Mi[8] * d2;
    // F[k][j] = delta_kj + du_k/dx_j
    T F[9];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      F[3 * k] = group_sum<8>(ub[k] * g0);
      F[3 * k + 1] = group_sum<8>(ub[k] * g1);
      F[3 * k + 2] = group_sum<8>(ub[k] * g2);
    }
    // Green-Lagrange strain (engineering shear) from H = F - I, then S = C E
    const T E0 = F[0] + T(0.5) * (F[0] * F[0] + F[3] * F[3] + F[6] * F[6]);
    const T E1 = F[4] + T(0.5) * (F[1] * F[1] + F[4] * F[4] + F[7] * F[7]);
    const T E2 = F[8] + T(0.5) * (F[2] * F[2] + F[5] * F[5] + F[8] * F[8]);
    const T E3 = F[1] + F[3] + F[0] * F[1] + F[3] * F[4] + F[6] * F[7];
    const T E4 = F[5] + F[7] + F[1] * F[2] + F[4] * F[5] + F[7] * F[8];
    const T E5 = F[2] + F[6] + F[0] * F[2] + F[3] * F[5] + F[6] * F[8];
    const T S0 = N00 * E0 + N01 * E1 + N02 * E2, S1 = N01 * E0 + N11 * E1 + N12 * E2;
    const T S2 = N02 * E0 + N12 * E1 + N22 * E2, S3 = G4 * E3, S4 = G5 * E4, S5 = G6 * E5;
    F[0] += T(1);
    F[4] += T(1);
    F[8] += T(1);
    // S dN_b (the initial-stress term of every pair with this lane's node)
    const T sg0 = S0 * g0 + S3 * g1 + S5 * g2;
    const T sg1 = S3 * g0 + S1 * g1 + S4 * g2;
    const T sg2 = S5 * g0 + S4 * g1 + S2 * g2;
    T h[2][3];
    h[0][0] = __shfl_sync(0xffffffffu, g0, a0);
    h[0][1] = __shfl_sync(0xffffffffu, g1, a0);
    h[0][2] = __shfl_sync(0xffffffffu, g2, a0);
    h[1][0] = __shfl_sync(0xffffffffu, g0, a1);
    h[1][1] = __shfl_sync(0xffffffffu, g1, a1);
    h[1][2] = __shfl_sync(0xffffffffu, g2, a1);
#pragma unroll
    for (int p = 0; p < 2; ++p) {
      T* K = p ? K1 : K0;
      const T x0 = h[p][0] * f, x1 = h[p][1] * f, x2 = h[p][2] * f;
      T L[9];  // the linear block K^L_ab (as in asm_hex8_elastic_warp)
      L[0] = x0 * N00 * g0 + x1 * G4 * g1 + x2 * G6 * g2;
      L[1] = x0 * N01 * g1 + x1 * G4 * g0;
      L[2] = x0 * N02 * g2 + x2 * G6 * g0;
      L[3] = x1 * N01 * g0 + x0 * G4 * g1;
      L[4] = x1 * N11 * g1 + x0 * G4 * g0 + x2 * G5 * g2;
      L[5] = x1 * N12 * g2 + x2 * G5 * g1;
      L[6] = x2 * N02 * g0 + x0 * G6 * g2;
      L[7] = x2 * N12 * g1 + x1 * G5 * g2;
      L[8] = x2 * N22 * g2 + x1 * G5 * g1 + x0 * G6 * g0;
      T FL[9];  // F L
#pragma unroll
      for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int m = 0; m < 3; ++m) FL[3 * k + m] = F[3 * k] * L[m] + F[3 * k + 1] * L[3 + m] + F[3 * k + 2] * L[6 + m];
      const T ks = x0 * sg0 + x1 * sg1 + x2 * sg2;
#pragma unroll
      for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int l = 0; l < 3; ++l)
          K[3 * k + l] += FL[3 * k] * F[3 * l] + FL[3 * k + 1] * F[3 * l + 1] + FL[3 * k + 2] * F[3 * l + 2] +
                          (k == l ? ks : T(0));
    }
  }
  if ((b == a0 && !(K0[0] > 0 && K0[4] > 0 && K0[8] > 0)) ||
      (b == a1 && !(K1[0] > 0 && K1[4] > 0 && K1[8] > 0)))
    atomicOr(A.flags, kFlagNegDiag);
  const int I0 = __shfl_sync(0xffffffffu, J, a0);
  const int I1 = __shfl_sync(0xffffffffu, J, a1);
  const uint16_t* sl = A.slot + (long long)e * 64;
  if constexpr (sizeof(T) == 4) {
    scatter_block32<3>(A, I0, J, sl[a0 * 8 + b], K0);
    scatter_block32<3>(A, I1, J, sl[a1 * 8 + b], K1);
  } else {
    double pl0[3], pl1[3];  // the pseudo-load of prescribed values: a Newton step does not use it
    scatter_block64<3>(A, I0, J, sl[a0 * 8 + b], K0, pl0);
    scatter_block64<3>(A, I1, J, sl[a1 * 8 + b], K1, pl1);
  }
}

template <typename T>
__global__ void __launch_bounds__(256) k_asm_hex8_gnl(ElemArgs A, const int* __restrict__ elems, int nel,
                                                      const double* __restrict__ u) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* s_dN = reinterpret_cast<T*>(smem_raw);
  T* s_N = s_dN + A.nip * 24;
  T* s_w = s_N + A.nip * 8;
  stage_gauss<T, 8, 3>(A.gt, A.nip, s_dN, s_N, s_w);
  const int wpb = blockDim.x >> 5;
  for (int w = blockIdx.x * wpb + (threadIdx.x >> 5); w < nel; w += gridDim.x * wpb)
    asm_hex8_gnl_warp<T>(A, elems, nel, w, u, s_dN, s_w);
}

// ---- quad4 plane stress, two elements per warp ---------------------------
// lane = 16*sub + 4*a + b handles pair (a,b) of element 2*warp+sub.
template <typename T>
__device__ __forceinline__ void asm_quad4_pstress_warp(const ElemArgs& A, const int* __restrict__ elems, int nel, int w,
    const T* s_dN, const T* s_N, const T* s_w) {
  const int lane = threadIdx.x & 31;
  const int sub = lane >> 4, q = lane & 15, a = q >> 2, b = q & 3;
  {
    const int idx = 2 * w + sub;
    const bool valid = idx < nel;
    const int e = elems[valid ? idx : nel - 1];
    const int* ce = A.conn + (long long)e * 4;
    const int J = ce[b];
    const int n0 = ce[0];
    const T xr0 = (T)(A.xyz[2LL * J] - A.xyz[2LL * n0]);
    const T xr1 = (T)(A.xyz[2LL * J + 1] - A.xyz[2LL * n0 + 1]);
    double cc[4];
    pstress_c(A.gparams + (long long)(A.egroup ? A.egroup[e] : e) * A.nparams, cc);
    const T C00 = cc[0], C01 = cc[1], C11 = cc[2], C22 = cc[3];
    T K[4] = {T(0), T(0), T(0), T(0)};
    const int src = (lane & 16) + a;  // lane holding node a of this element
    for (int ip = 0; ip < A.nip; ++ip) {
      const T d0 = s_dN[ip * 8 + b], d1 = s_dN[ip * 8 + 4 + b];
      const T M00 = group_sum<4>(d0 * xr0), M01 = group_sum<4>(d0 * xr1);
      const T M10 = group_sum<4>(d1 * xr0), M11 = group_sum<4>(d1 * xr1);
      const T det = M00 * M11 - M01 * M10;
      const T id = T(1) / det;
      const T g0 = (M11 * d0 - M01 * d1) * id;
      const T g1 = (-M10 * d0 + M00 * d1) * id;
      const T f = det * s_w[ip];
      const T h0 = __shfl_sync(0xffffffffu, g0, src) * f;
      const T h1 = __shfl_sync(0xffffffffu, g1, src) * f;
      K[0] += h0 * C00 * g0 + h1 * C22 * g1;
      K[1] += h0 * C01 * g1 + h1 * C22 * g0;
      K[2] += h1 * C01 * g0 + h0 * C22 * g1;
      K[3] += h1 * C11 * g1 + h0 * C22 * g0;
    }
    if (valid && a == b && !(K[0] > 0 && K[3] > 0)) atomicOr(A.flags, kFlagNegDiag);
    const int I = __shfl_sync(0xffffffffu, J, src);
    const int blk = A.slot[(long long)e * 16 + a * 4 + b];  // position in node I's row
    if constexpr (sizeof(T) == 4) {
      if (valid) scatter_block32<2>(A, I, J, blk, K);
    } else {
      double pl[2] = {0.0, 0.0};
      if (valid) scatter_block64<2>(A, I, J, blk, K, pl);
      pl[0] = group_sum<4>(pl[0]);
      pl[1] = group_sum<4>(pl[1]);
      if (valid && b == 0) {
        if (!A.rest[2 * I]) A.pseudo[2 * I] += pl[0];
        if (!A.rest[2 * I + 1]) A.pseudo[2 * I + 1] += pl[1];
      }
    }
  }
}

template <typename T>
__global__ void __launch_bounds__(256) k_asm_quad4_pstress(ElemArgs A, const int* __restrict__ elems,
    int nel) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* s_dN = reinterpret_cast<T*>(smem_raw);
  T* s_N = s_dN + A.nip * 8;
  T* s_w = s_N + A.nip * 4;
  stage_gauss<T, 4, 2>(A.gt, A.nip, s_dN, s_N, s_w);
  const int wpb = blockDim.x >> 5;
  for (int w = blockIdx.x * wpb + (threadIdx.x >> 5); 2 * w < nel; w += gridDim.x * wpb)
    asm_quad4_pstress_warp<T>(A, elems, nel, w, s_dN, s_N, s_w);
}

// ---- hex8 diffusion: kscale*K + mscale*M, one warp per element -------------
template <typename T>
__device__ __forceinline__ void asm_hex8_heat_warp(const ElemArgs& A, const int* __restrict__ elems, int nel, int w,
    const T* s_dN, const T* s_N, const T* s_w) {
  const int lane = threadIdx.x & 31;
  const int b = lane & 7, a0 = lane >> 3, a1 = a0 + 4;
  {
    const int e = elems[w];
    const int* ce = A.conn + (long long)e * 8;
    const int J = ce[b];
    const int n0 = ce[0];
    T xr[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) xr[c] = (T)(A.xyz[3LL * J + c] - A.xyz[3LL * n0 + c]);
    const double* pm = A.gparams + (long long)(A.egroup ? A.egroup[e] : e) * A.nparams;
    const T k11 = pm[0], k22 = pm[1], k33 = pm[2], cap = pm[3];
    T Kk[2] = {T(0), T(0)}, Km[2] = {T(0), T(0)};
    for (int ip = 0; ip < A.nip; ++ip) {
      const T* dn = s_dN + ip * 24;
      const T d0 = dn[b], d1 = dn[8 + b], d2 = dn[16 + b];
      T M[9];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        M[c] = group_sum<8>(d0 * xr[c]);
        M[3 + c] = group_sum<8>(d1 * xr[c]);
        M[6 + c] = group_sum<8>(d2 * xr[c]);
      }
      T Mi[9];
      const T det = inv3<T>(M, Mi);
      const T f = det * s_w[ip];
      const T g0 = Mi[0] * d0 + Mi[1] * d1 + Mi[2] * d2;
      const T g1 = Mi[3] * d0 + Mi[4] * d1 + Mi[5] * d2;
      const T g2 = Mi[6] * d0 + Mi[7] * d1 + Mi[8] * d2;
      const T Sb = s_N[ip * 8 + b];
#pragma unroll
      for (int p = 0; p < 2; ++p) {
        const int a = p ? a1 : a0;
        const T h0 = __shfl_sync(0xffffffffu, g0, a), h1 = __shfl_sync(0xffffffffu, g1, a),
                h2 = __shfl_sync(0xffffffffu, g2, a);
        const T Sa = s_N[ip * 8 + a];
        Kk[p] += (h0 * k11 * g0 + h1 * k22 * g1 + h2 * k33 * g2) * f;
        Km[p] += Sa * Sb * f * cap;
      }
    }
    T K0[1] = {T(A.kscale) * Kk[0] + T(A.mscale) * Km[0]};
    T K1[1] = {T(A.kscale) * Kk[1] + T(A.mscale) * Km[1]};
    const int I0 = __shfl_sync(0xffffffffu, J, a0);
    const int I1 = __shfl_sync(0xffffffffu, J, a1);
    const uint16_t* sl = A.slot + (long long)e * 64;
    if constexpr (sizeof(T) == 4) {
      scatter_block32<1>(A, I0, J, sl[a0 * 8 + b], K0);
      scatter_block32<1>(A, I1, J, sl[a1 * 8 + b], K1);
    } else {
      double pl0[1], pl1[1];
      scatter_block64<1>(A, I0, J, sl[a0 * 8 + b], K0, pl0);
      scatter_block64<1>(A, I1, J, sl[a1 * 8 + b], K1, pl1);
      pl0[0] = group_sum<8>(pl0[0]);
      pl1[0] = group_sum<8>(pl1[0]);
      if (b == 0) {
        if (!A.rest[I0]) A.pseudo[I0] += pl0[0];
        if (!A.rest[I1]) A.pseudo[I1] += pl1[0];
      }
    }
  }
}

template <typename T>
__global__ void __launch_bounds__(256) k_asm_hex8_heat(ElemArgs A, const int* __restrict__ elems,
    int nel) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* s_dN = reinterpret_cast<T*>(smem_raw);
  T* s_N = s_dN + A.nip * 24;
  T* s_w = s_N + A.nip * 8;
  stage_gauss<T, 8, 3>(A.gt, A.nip, s_dN, s_N, s_w);
  const int wpb = blockDim.x >> 5;
  for (int w = blockIdx.x * wpb + (threadIdx.x >> 5); w < nel; w += gridDim.x * wpb)
    asm_hex8_heat_warp<T>(A, elems, nel, w, s_dN, s_N, s_w);
}

// ---- quad4 diffusion: kscale*K + mscale*M, 16 lanes per element ----------
// HeatTransferElement2Dtransient (HeatTransferElement2DTransient.cpp:67-108):
// K = int grad N^T diag(k11, k22) grad N (k12 = 0 for the unrotated
// orthotropic material), M = int c N N^T, unit thickness.  Lane (a, b) of an
// element's 16 forms entry (a, b); two elements per warp.
template <typename T>
__device__ __forceinline__ void asm_quad4_heat_warp(const ElemArgs& A, const int* __restrict__ elems, int nel, int w,
    const T* s_dN, const T* s_N, const T* s_w) {
  const int lane = threadIdx.x & 31;
  const int sub = lane >> 4, q = lane & 15, a = q >> 2, b = q & 3;
  const int idx = 2 * w + sub;
  const bool valid = idx < nel;
  const int e = elems[valid ? idx : nel - 1];
  const int* ce = A.conn + (long long)e * 4;
  const int J = ce[b];
  const int n0 = ce[0];
  const T xr0 = (T)(A.xyz[2LL * J] - A.xyz[2LL * n0]);
  const T xr1 = (T)(A.xyz[2LL * J + 1] - A.xyz[2LL * n0 + 1]);
  const double* pm = A.gparams + (long long)(A.egroup ? A.egroup[e] : e) * A.nparams;
  const T k11 = pm[0], k22 = pm[1], cap = pm[3];
  const int src = (lane & 16) + a;  // a lane holding node a of this element (b == a there)
  T Kk = T(0), Km = T(0);
  for (int ip = 0; ip < A.nip; ++ip) {
    const T d0 = s_dN[ip * 8 + b], d1 = s_dN[ip * 8 + 4 + b];
    const T M00 = group_sum<4>(d0 * xr0), M01 = group_sum<4>(d0 * xr1);
    const T M10 = group_sum<4>(d1 * xr0), M11 = group_sum<4>(d1 * xr1);
    const T det = M00 * M11 - M01 * M10;
    const T id = T(1) / det;
    const T g0 = (M11 * d0 - M01 * d1) * id;
    const T g1 = (-M10 * d0 + M00 * d1) * id;
    const T f = det * s_w[ip];
    const T h0 = __shfl_sync(0xffffffffu, g0, src), h1 = __shfl_sync(0xffffffffu, g1, src);
    Kk += (h0 * k11 * g0 + h1 * k22 * g1) * f;
    Km += s_N[ip * 4 + a] * s_N[ip * 4 + b] * f * cap;
  }
  T K[1] = {T(A.kscale) * Kk + T(A.mscale) * Km};
  if (valid && a == b && !(K[0] > 0)) atomicOr(A.flags, kFlagNegDiag);
  const int I = __shfl_sync(0xffffffffu, J, src);
  const int blk = A.slot[(long long)e * 16 + a * 4 + b];  // position in node I's row
  if constexpr (sizeof(T) == 4) {
    if (valid) scatter_block32<1>(A, I, J, blk, K);
  } else {
    double pl[1] = {0.0};
    if (valid) scatter_block64<1>(A, I, J, blk, K, pl);
    pl[0] = group_sum<4>(pl[0]);
    if (valid && b == 0 && !A.rest[I]) A.pseudo[I] += pl[0];
  }
}

template <typename T>
__global__ void __launch_bounds__(256) k_asm_quad4_heat(ElemArgs A, const int* __restrict__ elems, int nel) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* s_dN = reinterpret_cast<T*>(smem_raw);
  T* s_N = s_dN + A.nip * 8;
  T* s_w = s_N + A.nip * 4;
  stage_gauss<T, 4, 2>(A.gt, A.nip, s_dN, s_N, s_w);
  const int wpb = blockDim.x >> 5;
  for (int w = blockIdx.x * wpb + (threadIdx.x >> 5); 2 * w < nel; w += gridDim.x * wpb)
    asm_quad4_heat_warp<T>(A, elems, nel, w, s_dN, s_N, s_w);
}

// Restrained diagonals = 1 (Equations::addMatrix, equation.cpp:500).
template <int ND>
__global__ void k_set_restrained_diag32(int nnode, const unsigned char* rest, const int* bsoff,
                                        const int* ndiag, float* bval) {
  for (int I = blockIdx.x * blockDim.x + threadIdx.x; I < nnode; I += gridDim.x * blockDim.x) {
    const long long chunk = (long long)bsoff[I >> 5] + ndiag[I];
    for (int i = 0; i < ND; ++i)
      if (rest[I * ND + i]) bval[chunk * (32 * ND * ND) + (i * ND + i) * 32 + (I & 31)] = 1.0f;
  }
}

__global__ void k_set_restrained_diag64(int ndof, const unsigned char* rest, const long long* sdiag,
                                        double* sval) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < ndof; r += gridDim.x * blockDim.x)
    if (rest[r]) sval[sdiag[r]] = 1.0;
}

}  // namespace betagpu
