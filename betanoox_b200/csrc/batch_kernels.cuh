// batch_kernels.cuh -- many independent systems in one persistent launch.
//
// Each thread-block cluster (1, 2, 4 or 8 CTAs, chosen at launch) takes whole
// systems off a device work list (largest first, one atomicAdd per system)
// and runs, for that system alone: FP32 assembly (colour by colour),
// block-Jacobi factors, the FP64 right-hand-side norm, and reliable-update
// mixed-precision PCG (FP32 node-block SpMV + FP64 matrix-free residual
// replacement).  The only barriers are the cluster's own hardware barrier
// (cluster.sync, which covers the CTA barrier); reductions go through
// distributed shared memory in fixed rank order, so every thread of the
// cluster sees bit-identical sums and takes the same branches.  Clusters never
// wait on each other.  An iteration budget per
// launch lets a serving loop preempt systems between launches: the full
// Krylov state stays in the system's own device memory.
//
// The per-warp element and matrix-free bodies are the ones the single-system
// kernels use (elem_kernels.cuh, mf_kernels.cuh).
#pragma once
#include <cooperative_groups.h>

#include "common.cuh"
#include "elem_kernels.cuh"
#include "mf_kernels.cuh"
#include "pcg_kernels.cuh"

namespace betagpu {

enum : int { kPhaseNew = 0, kPhaseIter = 1, kPhaseDone = 2 };
enum : int { kBConverged = 0, kBRunning = 1, kBMaxit = 4, kBBreakdown = 5, kBNegDiag = 6 };

struct BState {
  double rho, rr, maxrr, bn, rn;
  int iter, repl, phase, status;
};

// Device descriptor of one system (all pointers into the batch pool).
struct BSys {
  int kind, ndpn, nnode, nelem, ndof, nip, ncolor, nslice, nparams, ndim;
  const double* xyz;
  const int* conn;
  const double* gparams;
  const int* egroup;
  const unsigned char* rest;
  const double* presc;
  const double* load;
  const int* color_ptr;  // ncolor+1 offsets into elems
  const int* elems;
  const int* slot;
  const int* nrp;
  const int* ndiag;
  const int* bsoff;
  const int* bcol;
  float* bval;
  double* x64;
  double* r64;
  double* y64;
  float* y32;
  float* r32;
  float* p32;
  float* q32;
  float* minv;
  const GaussTable* gt;
  BState* st;
  long long nchunk;
};

struct BParams {
  double tol, delta;
  int maxit, max_repl, budget;  // budget: iterations per system per launch (0: no limit)
  int nactive;
};

namespace cg = cooperative_groups;

// Cluster-wide sum of NV doubles (NV <= 4); every thread of the cluster gets
// the same totals: per-CTA sums in fixed warp order, then the CTAs' sums read
// through distributed shared memory in rank order.
template <int NV>
__device__ __forceinline__ void cl_sum(double (&v)[NV], double* sh, double* shtot) {
  cg::cluster_group cl = cg::this_cluster();
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int k = 0; k < NV; ++k) {
    double t = warp_sum(v[k]);
    if (lane == 0) sh[k * 32 + wid] = t;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) {
      double t = 0.0;
      for (int i = 0; i < nw; ++i) t += sh[k * 32 + i];
      shtot[k] = t;
    }
  }
  cl.sync();
  const int C = (int)cl.num_blocks();
#pragma unroll
  for (int k = 0; k < NV; ++k) {
    double t = 0.0;
    for (int r = 0; r < C; ++r) t += cl.map_shared_rank(shtot, r)[k];
    v[k] = t;
  }
  cl.sync();
}

template <typename T>
__device__ __forceinline__ void b_stage(const GaussTable* gt, int nip, int nn, int ndir, T* s_dN, T* s_N, T* s_w) {
  for (int i = threadIdx.x; i < nip * ndir * nn; i += blockDim.x) {
    int ip = i / (ndir * nn), r = (i / nn) % ndir, a = i % nn;
    s_dN[i] = (T)gt->dN[ip][r][a];
  }
  for (int i = threadIdx.x; i < nip * nn; i += blockDim.x) s_N[i] = (T)gt->N[i / nn][i % nn];
  for (int i = threadIdx.x; i < nip; i += blockDim.x) s_w[i] = (T)gt->w[i];
}

// y = K x for one system (FP64, matrix-free), colour by colour.
__device__ void b_mf(const BSys& S, const MfArgs& M, const double* x, double* y, const double* s_dN,
                     const double* s_N, const double* s_w) {
  cg::cluster_group cl = cg::this_cluster();
  const int C = (int)cl.num_blocks(), rank = (int)cl.block_rank();
  const int gt = rank * blockDim.x + threadIdx.x, gn = C * blockDim.x;
  for (int i = gt; i < S.ndof; i += gn) y[i] = 0.0;
  cl.sync();
  const int nw = blockDim.x >> 5;
  const int wid = rank * nw + (threadIdx.x >> 5), gw = C * nw;
  for (int c = 0; c < S.ncolor; ++c) {
    const int beg = S.color_ptr[c], nel = S.color_ptr[c + 1] - beg;
    const int* el = S.elems + beg;
    if (S.kind == 2) {
      for (int w = wid; 4 * w < nel; w += gw) mf_hex8_elastic_warp(M, el, nel, w, x, nullptr, y, s_dN, s_w);
    } else if (S.kind == 3) {
      for (int w = wid; 4 * w < nel; w += gw) mf_hex8_heat_warp(M, el, nel, w, x, nullptr, y, s_dN, s_N, s_w);
    } else {
      for (int w = wid; 8 * w < nel; w += gw) mf_quad4_pstress_warp(M, el, nel, w, x, nullptr, y, s_dN, s_w);
    }
    cl.sync();
  }
}

template <int ND>
__device__ void b_solve(const BSys& S, const BParams& P, double* sh, double* shtot, const double* s_dN,
                        const double* s_N, const double* s_w, const float* s_dNf, const float* s_Nf,
                        const float* s_wf, unsigned* s_flag) {
  constexpr int SM = ND * (ND + 1) / 2;
  cg::cluster_group cl = cg::this_cluster();
  const int C = (int)cl.num_blocks(), rank = (int)cl.block_rank();
  // cluster-global thread and warp indices
  const int tid = rank * blockDim.x + threadIdx.x, nt = C * blockDim.x;
  const int lane = threadIdx.x & 31, wid = rank * (blockDim.x >> 5) + (threadIdx.x >> 5), nw = C * (blockDim.x >> 5);
  BState st = *S.st;
  MfArgs M;
  M.xyz = S.xyz; M.conn = S.conn; M.gparams = S.gparams; M.egroup = S.egroup; M.nparams = S.nparams;
  M.nip = S.nip; M.gt = S.gt; M.c1 = 1.0; M.c2 = 0.0; M.cm = 0.0;
  const int n = S.ndof, nn = S.nnode;
  BlockMat A{S.nnode, S.nslice, S.bsoff, S.bcol, S.bval};

  if (st.phase == kPhaseNew) {
    // ---- FP32 assembly: zero, colour by colour, unit restrained diagonals
    const long long nv = S.nchunk * 32LL * ND * ND;
    for (long long i = tid; i < nv; i += nt) S.bval[i] = 0.f;
    if (threadIdx.x == 0) *s_flag = 0u;
    cl.sync();
    ElemArgs E;
    E.xyz = S.xyz; E.conn = S.conn; E.gparams = S.gparams; E.egroup = S.egroup; E.nparams = S.nparams;
    E.nip = S.nip; E.gt = S.gt; E.slot = S.slot; E.nrp = S.nrp; E.rest = S.rest; E.presc = S.presc;
    E.bsoff = S.bsoff; E.bval = S.bval; E.soff = nullptr; E.ssoff = nullptr; E.sval = nullptr; E.pseudo = nullptr;
    E.kscale = 1.0; E.mscale = 0.0; E.flags = s_flag;
    for (int c = 0; c < S.ncolor; ++c) {
      const int beg = S.color_ptr[c], nel = S.color_ptr[c + 1] - beg;
      const int* el = S.elems + beg;
      if (S.kind == 2) {
        for (int w = wid; w < nel; w += nw) asm_hex8_elastic_warp<float>(E, el, nel, w, s_dNf, s_Nf, s_wf);
      } else if (S.kind == 3) {
        for (int w = wid; w < nel; w += nw) asm_hex8_heat_warp<float>(E, el, nel, w, s_dNf, s_Nf, s_wf);
      } else {
        for (int w = wid; 2 * w < nel; w += nw) asm_quad4_pstress_warp<float>(E, el, nel, w, s_dNf, s_Nf, s_wf);
      }
      cl.sync();
    }
    for (int I = tid; I < nn; I += nt) {
      const long long chunk = (long long)S.bsoff[I >> 5] + S.ndiag[I];
      for (int i = 0; i < ND; ++i)
        if (S.rest[I * ND + i]) S.bval[chunk * (32 * ND * ND) + (i * ND + i) * 32 + (I & 31)] = 1.0f;
    }
    double fneg[1] = {threadIdx.x == 0 && (*s_flag & kFlagNegDiag) ? 1.0 : 0.0};
    cl_sum<1>(fneg, sh, shtot);  // also the barrier after the diagonal fix-up
    if (fneg[0] > 0.0) {
      if (tid == 0) { st.phase = kPhaseDone; st.status = kBNegDiag; *S.st = st; }
      cl.sync();
      return;
    }
    // ---- block-Jacobi factors (FP64 inverse of the node diagonal block)
    for (int I = tid; I < nn; I += nt) {
      const long long chunk = (long long)S.bsoff[I >> 5] + S.ndiag[I];
      double D[9] = {0}, Di[9] = {0};
      for (int t = 0; t < ND * ND; ++t) D[t] = S.bval[chunk * 32 * ND * ND + t * 32 + (I & 31)];
      if (ND == 1) Di[0] = 1.0 / D[0];
      else if (ND == 2) {
        const double id = 1.0 / (D[0] * D[3] - D[1] * D[2]);
        Di[0] = D[3] * id; Di[1] = -D[1] * id; Di[2] = -D[2] * id; Di[3] = D[0] * id;
      } else {
        inv3<double>(D, Di);
      }
      int t = 0;
      for (int i = 0; i < ND; ++i)
        for (int j = i; j < ND; ++j) S.minv[(long long)SM * I + (t++)] = (float)(0.5 * (Di[i * ND + j] + Di[j * ND + i]));
    }
    // ---- x = prescribed on restrained dofs, 0 elsewhere; r = b = load - K x (free rows)
    for (int i = tid; i < n; i += nt) S.x64[i] = S.rest[i] ? S.presc[i] : 0.0;
    cl.sync();
    b_mf(S, M, S.x64, S.y64, s_dN, s_N, s_w);
    double acc[1] = {0.0};
    for (int i = tid; i < n; i += nt) {
      const double r = S.rest[i] ? 0.0 : (S.load ? S.load[i] : 0.0) - S.y64[i];
      S.r64[i] = r;
      const double bb = S.rest[i] ? S.presc[i] : r;
      acc[0] += bb * bb;
      S.r32[i] = (float)r;
      S.y32[i] = 0.f;
    }
    cl_sum<1>(acc, sh, shtot);
    st.bn = sqrt(acc[0]);
    double a2[2] = {0.0, 0.0};
    for (int I = tid; I < nn; I += nt) {
      float rv[ND], z[ND];
      NodeIO<ND>::ld(S.r32, I, rv);
      NodeIO<ND>::prec(S.minv, I, rv, z);
      PVec<ND>::st(S.p32, I, z);
#pragma unroll
      for (int i = 0; i < ND; ++i) { a2[0] += (double)rv[i] * z[i]; a2[1] += (double)rv[i] * rv[i]; }
    }
    cl_sum<2>(a2, sh, shtot);
    st.rho = a2[0];
    st.rr = st.maxrr = a2[1];
    st.iter = 0;
    st.repl = 0;
    st.phase = kPhaseIter;
    st.status = kBRunning;
    st.rn = sqrt(a2[1]);
    if (a2[1] == 0.0 || st.rn <= P.tol * st.bn) { st.phase = kPhaseDone; st.status = kBConverged; }
  }

  const double tolabs2 = (0.5 * P.tol * st.bn) * (0.5 * P.tol * st.bn);
  const double delta2 = P.delta * P.delta;
  int spent = 0;
  while (st.phase == kPhaseIter && (P.budget <= 0 || spent < P.budget)) {
    // q = A p, p.q
    double a1[1] = {0.0};
    for (int s = wid; s < S.nslice; s += nw) {
      float acc[ND];
      spmv_row_b<ND, true>(A, s, lane, S.p32, acc);
      const int I = s * 32 + lane;
      if (I < nn) {
        NodeIO<ND>::st(S.q32, I, acc);
        float pv[ND];
        PVec<ND>::ld(S.p32, I, pv);
        float t = 0.f;
#pragma unroll
        for (int i = 0; i < ND; ++i) t = fmaf(pv[i], acc[i], t);
        a1[0] += (double)t;
      }
    }
    cl_sum<1>(a1, sh, shtot);
    if (!(a1[0] > 0.0 && a1[0] < 1e308)) { st.phase = kPhaseDone; st.status = kBBreakdown; break; }
    const float alpha = (float)(st.rho / a1[0]);
    // y += alpha p, r -= alpha q, (r.z, r.r)
    double a2[2] = {0.0, 0.0};
    for (int I = tid; I < nn; I += nt) {
      float yv[ND], rv[ND], pv[ND], qv[ND], z[ND];
      NodeIO<ND>::ld(S.y32, I, yv);
      NodeIO<ND>::ld(S.r32, I, rv);
      PVec<ND>::ld(S.p32, I, pv);
      NodeIO<ND>::ld(S.q32, I, qv);
#pragma unroll
      for (int i = 0; i < ND; ++i) {
        yv[i] = fmaf(alpha, pv[i], yv[i]);
        rv[i] = fmaf(-alpha, qv[i], rv[i]);
      }
      NodeIO<ND>::st(S.y32, I, yv);
      NodeIO<ND>::st(S.r32, I, rv);
      NodeIO<ND>::prec(S.minv, I, rv, z);
#pragma unroll
      for (int i = 0; i < ND; ++i) { a2[0] += (double)rv[i] * z[i]; a2[1] += (double)rv[i] * rv[i]; }
    }
    cl_sum<2>(a2, sh, shtot);
    st.iter += 1;
    ++spent;
    if (!(a2[0] == a2[0])) { st.phase = kPhaseDone; st.status = kBBreakdown; break; }
    double beta;
    if (a2[1] > st.maxrr) st.maxrr = a2[1];
    if (a2[1] < tolabs2 || a2[1] < delta2 * st.maxrr || st.iter >= P.maxit) {
      // reliable update: fold y into x, replace r by the FP64 true residual
      for (int i = tid; i < n; i += nt) { S.x64[i] += (double)S.y32[i]; S.y32[i] = 0.f; }
      cl.sync();
      b_mf(S, M, S.x64, S.y64, s_dN, s_N, s_w);
      double a3[1] = {0.0};
      for (int i = tid; i < n; i += nt) {
        const double r = S.rest[i] ? 0.0 : (S.load ? S.load[i] : 0.0) - S.y64[i];
        S.r64[i] = r;
        S.r32[i] = (float)r;
        a3[0] += r * r;
      }
      cl_sum<1>(a3, sh, shtot);
      st.rn = sqrt(a3[0]);
      st.repl += 1;
      if (!(st.rn == st.rn)) { st.phase = kPhaseDone; st.status = kBBreakdown; break; }
      if (st.rn <= P.tol * st.bn) { st.phase = kPhaseDone; st.status = kBConverged; break; }
      if (st.iter >= P.maxit || st.repl > P.max_repl) { st.phase = kPhaseDone; st.status = kBMaxit; break; }
      double a4[2] = {0.0, 0.0};
      for (int I = tid; I < nn; I += nt) {
        float rv[ND], z[ND];
        NodeIO<ND>::ld(S.r32, I, rv);
        NodeIO<ND>::prec(S.minv, I, rv, z);
#pragma unroll
        for (int i = 0; i < ND; ++i) { a4[0] += (double)rv[i] * z[i]; a4[1] += (double)rv[i] * rv[i]; }
      }
      cl_sum<2>(a4, sh, shtot);
      beta = st.rho != 0.0 ? a4[0] / st.rho : 0.0;
      st.rho = a4[0];
      st.rr = st.maxrr = a4[1];
    } else {
      beta = a2[0] / st.rho;
      st.rho = a2[0];
      st.rr = a2[1];
    }
    // p = M r + beta p
    const float bt = (float)beta;
    for (int I = tid; I < nn; I += nt) {
      float rv[ND], pv[ND], z[ND];
      NodeIO<ND>::ld(S.r32, I, rv);
      PVec<ND>::ld(S.p32, I, pv);
      NodeIO<ND>::prec(S.minv, I, rv, z);
#pragma unroll
      for (int i = 0; i < ND; ++i) pv[i] = fmaf(bt, pv[i], z[i]);
      PVec<ND>::st(S.p32, I, pv);
    }
    cl.sync();
  }
  cl.sync();
  if (tid == 0) *S.st = st;
  cl.sync();
}

// The persistent batch kernel: clusters pull systems from active[] until
// empty.  Launched with a cluster dimension of 1, 2, 4 or 8 CTAs.
template <int THREADS>
__global__ void __launch_bounds__(THREADS, 1) k_batch_solve(const BSys* __restrict__ sys, const int* __restrict__ active,
                                                            int* counter, const BParams* __restrict__ prm) {
  __shared__ double sh[64];
  __shared__ double shtot[4];
  __shared__ double s_dN[kMaxIP * 24], s_N[kMaxIP * 8], s_w[kMaxIP];
  __shared__ float s_dNf[kMaxIP * 24], s_Nf[kMaxIP * 8], s_wf[kMaxIP];
  __shared__ int s_idx;
  __shared__ unsigned s_flag;
  cg::cluster_group cl = cg::this_cluster();
  const BParams P = *prm;
  for (;;) {
    if (cl.block_rank() == 0 && threadIdx.x == 0) s_idx = atomicAdd(counter, 1);
    cl.sync();
    const int k = *cl.map_shared_rank(&s_idx, 0);
    cl.sync();  // rank 0 may overwrite s_idx only after every CTA has read it
    if (k >= P.nactive) break;  // the same k in every CTA of the cluster
    const BSys S = sys[active[k]];
    const int nn = S.kind == 1 ? 4 : 8, ndir = S.kind == 1 ? 2 : 3;
    b_stage<double>(S.gt, S.nip, nn, ndir, s_dN, s_N, s_w);
    b_stage<float>(S.gt, S.nip, nn, ndir, s_dNf, s_Nf, s_wf);
    __syncthreads();
    if (S.ndpn == 3) b_solve<3>(S, P, sh, shtot, s_dN, s_N, s_w, s_dNf, s_Nf, s_wf, &s_flag);
    else if (S.ndpn == 2) b_solve<2>(S, P, sh, shtot, s_dN, s_N, s_w, s_dNf, s_Nf, s_wf, &s_flag);
    else b_solve<1>(S, P, sh, shtot, s_dN, s_N, s_w, s_dNf, s_Nf, s_wf, &s_flag);
  }
}

}  // namespace betagpu
