// pcg_kernels.cuh -- sliced-ELL SpMV and the fused Jacobi / block-Jacobi PCG.
//
// Restates SymmetricSparseMatrix::solve (sparse.cpp:114-242): the five vector
// sweeps per iteration become two fused kernels around the SpMV, and the
// scalars (alpha, beta, norms) are formed on the device in FP64 by the last
// block to finish (fixed-order reduction over per-block partials, so results
// are deterministic).  Every kernel returns at once when the solve is done, so
// the host can enqueue whole chunks of iterations and poll rarely.
//
// Two storage forms:
//   scalar  : FP64 values, one row per dof, restrained columns removed
//             (plain FP64 PCG, Jacobi)
//   block   : FP32 values, one row per node with ND x ND blocks, packed FP32
//             dof vectors (mixed-precision inner PCG, Jacobi or node
//             block-Jacobi, with reliable updates of the residual)
#pragma once
#include "common.cuh"

namespace betagpu {

enum : int { kStopRef = 0, kStopRB = 1, kStopRel = 2 };

struct PcgState {
  double rho;     // r.z
  double alpha, beta;
  double rr, xx, bb;
  double ref0;    // reference squared norm for kStopRB / kStopRel
  double tol2;    // squared tolerance
  double last;    // last stop quantity (not squared)
  double pq;
  double maxrr;   // reliable updates: largest r.r since the last replacement
  double delta2;  // reliable updates: replace when r.r < delta2 * maxrr
  double tolabs2; // reliable updates: also replace when r.r < tolabs2
  int iter, maxit, status, done;
  int rule;
  unsigned ticket;
};

constexpr int kStatusOk = 0, kStatusMaxit = 4, kStatusBreakdown = 5, kStatusReplace = 6;
enum : int { kRuleReliable = 3 };

// ---- block reduction with last-block finish --------------------------------
// Each block reduces NV values, writes them to partials[block*NV+k]; the last
// block to arrive sums all partials in a fixed order and returns true with
// the totals in out[] (valid in every thread of that block).
template <int NV>
__device__ __forceinline__ bool reduce_last(double (&v)[NV], double* partials, unsigned* ticket,
                                            double (&out)[NV]) {
  __shared__ double sh[NV][32];
  __shared__ bool s_last;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int k = 0; k < NV; ++k) {
    double t = warp_sum(v[k]);
    if (lane == 0) sh[k][wid] = t;
  }
  __syncthreads();
  if (wid == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) {
      double t = lane < nw ? sh[k][lane] : 0.0;
      t = warp_sum(t);
      if (lane == 0) partials[(long long)blockIdx.x * NV + k] = t;
    }
    if (lane == 0) {
      __threadfence();
      unsigned t = atomicAdd(ticket, 1u);
      s_last = (t == gridDim.x - 1);
    }
  }
  __syncthreads();
  if (!s_last) return false;
  __threadfence();
#pragma unroll
  for (int k = 0; k < NV; ++k) {
    double s = 0.0;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) s += __ldcg(partials + (long long)i * NV + k);
    v[k] = s;
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < NV; ++k) {
    double t = warp_sum(v[k]);
    if (lane == 0) sh[k][wid] = t;
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < NV; ++k) {
    double t = 0.0;
    for (int i = 0; i < nw; ++i) t += sh[k][i];
    out[k] = t;
  }
  if (threadIdx.x == 0) *ticket = 0u;
  return true;
}

__device__ __forceinline__ bool finite_pos(double x) { return x > 0.0 && x < 1e308; }

// Convergence bookkeeping after an update (last block, thread 0).
__device__ __forceinline__ void finish_update(PcgState* st, double rz, double rr, double xx) {
  st->iter += 1;
  st->rr = rr;
  st->xx = xx;
  double q;
  if (st->rule == kStopRef) q = xx > 0.0 ? rr / xx : 1e300;  // sparse.cpp:202-223
  else q = st->ref0 > 0.0 ? rr / st->ref0 : rr;
  st->last = sqrt(q);
  if (!(rz == rz) || !(rr == rr)) {
    st->status = kStatusBreakdown;
    st->done = 1;
    return;
  }
  if (st->rule == kRuleReliable) {
    // The FP32 recursive residual has dropped by delta (or below the target):
    // stop the chunk so the host can replace it with the FP64 true residual.
    // rho keeps r_old.z_old; beta is formed after the replacement.
    if (rr > st->maxrr) st->maxrr = rr;
    if (rr < st->tolabs2 || rr < st->delta2 * st->maxrr) {
      st->status = kStatusReplace;
      st->done = 1;
      return;
    }
  }
  st->beta = st->rho != 0.0 ? rz / st->rho : 0.0;
  st->rho = rz;
  if (st->rule != kRuleReliable && q < st->tol2) {
    st->status = kStatusOk;
    st->done = 1;
  } else if (st->iter >= st->maxit) {
    st->status = kStatusMaxit;
    st->done = 1;
  }
}

// ============================ scalar FP64 ================================
struct ScalarMat {
  int nrows, nslice;
  const long long* ssoff;  // nslice+1 (entries)
  const int* scol;
  const double* sval;
};

__device__ __forceinline__ double spmv_row_s(const ScalarMat& A, int s, int lane,
                                             const double* __restrict__ x) {
  const long long beg = A.ssoff[s] + lane;
  const int w = (int)((A.ssoff[s + 1] - A.ssoff[s]) >> 5);
  const int* cp = A.scol + beg;
  const double* vp = A.sval + beg;
  double acc0 = 0.0, acc1 = 0.0, acc2 = 0.0, acc3 = 0.0;
  int k = 0;
  for (; k + 3 < w; k += 4) {
    const long long o = (long long)k * 32;
    const int c0 = __ldcs(cp + o), c1 = __ldcs(cp + o + 32), c2 = __ldcs(cp + o + 64), c3 = __ldcs(cp + o + 96);
    const double v0 = __ldcs(vp + o), v1 = __ldcs(vp + o + 32), v2 = __ldcs(vp + o + 64), v3 = __ldcs(vp + o + 96);
    acc0 += v0 * __ldg(x + c0);
    acc1 += v1 * __ldg(x + c1);
    acc2 += v2 * __ldg(x + c2);
    acc3 += v3 * __ldg(x + c3);
  }
  for (; k < w; ++k) acc0 += __ldcs(vp + (long long)k * 32) * __ldg(x + __ldcs(cp + (long long)k * 32));
  return (acc0 + acc1) + (acc2 + acc3);
}

// y = A x (optionally y = b - A x), no reduction.
__global__ void __launch_bounds__(256) k_spmv_s(ScalarMat A, const double* __restrict__ x,
                                                double* __restrict__ y, const double* __restrict__ b) {
  const int lane = threadIdx.x & 31;
  for (int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; s < A.nslice; s += (gridDim.x * blockDim.x) >> 5) {
    const double v = spmv_row_s(A, s, lane, x);
    const int r = s * 32 + lane;
    if (r < A.nrows) y[r] = b ? b[r] - v : v;
  }
}

// q = A p, alpha = rho / (p.q).
__global__ void __launch_bounds__(256) k_spmv_dot_s(ScalarMat A, const double* __restrict__ p,
                                                    double* __restrict__ q, PcgState* st, double* partials) {
  if (st->done) return;
  const int lane = threadIdx.x & 31;
  double acc[1] = {0.0};
  for (int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; s < A.nslice; s += (gridDim.x * blockDim.x) >> 5) {
    const double v = spmv_row_s(A, s, lane, p);
    const int r = s * 32 + lane;
    if (r < A.nrows) {
      q[r] = v;
      acc[0] += p[r] * v;
    }
  }
  double out[1];
  if (reduce_last<1>(acc, partials, &st->ticket, out) && threadIdx.x == 0) {
    st->pq = out[0];
    if (!finite_pos(out[0])) {
      st->status = kStatusBreakdown;
      st->done = 1;
    } else {
      st->alpha = st->rho / out[0];
    }
  }
}

// x += alpha p; r -= alpha q; z = dinv r; (r.z, r.r, x.x)
__global__ void __launch_bounds__(256) k_update_s(int n, double* __restrict__ x, double* __restrict__ r,
                                                  const double* __restrict__ p, const double* __restrict__ q,
                                                  const double* __restrict__ dinv, PcgState* st,
                                                  double* partials) {
  if (st->done) return;
  const double a = st->alpha;
  double acc[3] = {0.0, 0.0, 0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double xi = x[i] + a * p[i];
    const double ri = r[i] - a * q[i];
    x[i] = xi;
    r[i] = ri;
    acc[0] += ri * (ri * dinv[i]);
    acc[1] += ri * ri;
    acc[2] += xi * xi;
  }
  double out[3];
  if (reduce_last<3>(acc, partials, &st->ticket, out) && threadIdx.x == 0) finish_update(st, out[0], out[1], out[2]);
}

// p = dinv r + beta p
__global__ void __launch_bounds__(256) k_pupd_s(int n, double* __restrict__ p, const double* __restrict__ r,
                                                const double* __restrict__ dinv, const PcgState* st) {
  if (st->done) return;
  const double bt = st->beta;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    p[i] = r[i] * dinv[i] + bt * p[i];
}

// Start: given r (= b - A x0), z = dinv r, p = z, rho = r.z, rr, xx(x0), bb.
__global__ void __launch_bounds__(256) k_start_s(int n, const double* __restrict__ x, const double* __restrict__ r,
                                                 const double* __restrict__ b, const double* __restrict__ dinv,
                                                 double* __restrict__ p, PcgState* st, double* partials) {
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double ri = r[i], zi = ri * dinv[i];
    p[i] = zi;
    acc[0] += ri * zi;
    acc[1] += ri * ri;
    acc[2] += x[i] * x[i];
    acc[3] += b[i] * b[i];
  }
  double out[4];
  if (reduce_last<4>(acc, partials, &st->ticket, out) && threadIdx.x == 0) {
    st->rho = out[0];
    st->rr = out[1];
    st->xx = out[2];
    st->bb = out[3];
    if (st->rule == kStopRB) st->ref0 = out[3];
    else if (st->rule == kStopRel) st->ref0 = out[1];
    st->iter = 0;
    st->status = kStatusOk;
    st->done = 0;
    if (!(out[0] == out[0])) { st->status = kStatusBreakdown; st->done = 1; }
    else if (out[1] == 0.0) { st->done = 1; st->last = 0.0; }
  }
}

// Jacobi inverse diagonal of the scalar layout; flags zero / negative.
__global__ void k_dinv_s(int n, const long long* sdiag, const double* sval, double* dinv, unsigned* flags) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double d = sval[sdiag[i]];
    if (!(d > 0.0)) atomicOr(flags, d == 0.0 ? 8u : 16u);
    dinv[i] = d != 0.0 ? 1.0 / d : 0.0;
  }
}

// =========================== node-block FP32 ===============================
// FP32 vectors are packed dof vectors (node I owns entries ND*I .. ND*I+ND-1,
// the node-major numbering), so no padding is read or written.  Block-Jacobi
// factors are the ND*(ND+1)/2 upper entries of the symmetric inverse of each
// node's diagonal block, packed per node.
template <int ND>
struct NodeIO {
  static constexpr int S = ND * (ND + 1) / 2;
  __device__ static __forceinline__ void ld(const float* v, long long I, float* o) {
    if constexpr (ND == 2) {
      const float2 t = reinterpret_cast<const float2*>(v)[I];
      o[0] = t.x; o[1] = t.y;
    } else {
#pragma unroll
      for (int i = 0; i < ND; ++i) o[i] = v[ND * I + i];
    }
  }
  __device__ static __forceinline__ void ldg(const float* __restrict__ v, long long I, float* o) {
    if constexpr (ND == 2) {
      const float2 t = __ldg(reinterpret_cast<const float2*>(v) + I);
      o[0] = t.x; o[1] = t.y;
    } else {
#pragma unroll
      for (int i = 0; i < ND; ++i) o[i] = __ldg(v + ND * I + i);
    }
  }
  __device__ static __forceinline__ void st(float* v, long long I, const float* a) {
    if constexpr (ND == 2) {
      reinterpret_cast<float2*>(v)[I] = make_float2(a[0], a[1]);
    } else {
#pragma unroll
      for (int i = 0; i < ND; ++i) v[ND * I + i] = a[i];
    }
  }
  // z = M r with M symmetric, packed upper rows: (00,01,02,11,12,22) for ND=3
  __device__ static __forceinline__ void prec(const float* m, long long I, const float* r, float* z) {
    float a[S];
#pragma unroll
    for (int t = 0; t < S; ++t) a[t] = m[S * I + t];
    if constexpr (ND == 1) {
      z[0] = a[0] * r[0];
    } else if constexpr (ND == 2) {
      z[0] = fmaf(a[0], r[0], a[1] * r[1]);
      z[1] = fmaf(a[1], r[0], a[2] * r[1]);
    } else {
      z[0] = fmaf(a[0], r[0], fmaf(a[1], r[1], a[2] * r[2]));
      z[1] = fmaf(a[1], r[0], fmaf(a[3], r[1], a[4] * r[2]));
      z[2] = fmaf(a[2], r[0], fmaf(a[4], r[1], a[5] * r[2]));
    }
  }
};

// The search direction p is the vector the SpMV gathers: for ND=3 it is
// padded to float4 per node so a gather is one 16-byte load.
template <int ND>
struct PVec {
  static constexpr int W = (ND == 3) ? 4 : ND;
  __device__ static __forceinline__ void ldg(const float* __restrict__ v, long long I, float* o) {
    if constexpr (ND == 3) {
      const float4 t = __ldg(reinterpret_cast<const float4*>(v) + I);
      o[0] = t.x; o[1] = t.y; o[2] = t.z;
    } else {
      NodeIO<ND>::ldg(v, I, o);
    }
  }
  __device__ static __forceinline__ void ld(const float* v, long long I, float* o) {
    if constexpr (ND == 3) {
      const float4 t = reinterpret_cast<const float4*>(v)[I];
      o[0] = t.x; o[1] = t.y; o[2] = t.z;
    } else {
      NodeIO<ND>::ld(v, I, o);
    }
  }
  __device__ static __forceinline__ void st(float* v, long long I, const float* a) {
    if constexpr (ND == 3) {
      reinterpret_cast<float4*>(v)[I] = make_float4(a[0], a[1], a[2], 0.f);
    } else {
      NodeIO<ND>::st(v, I, a);
    }
  }
};

struct BlockMat {
  int nnode, nslice;
  const int* bsoff;  // nslice+1 (chunks)
  const int* bcol;
  const float* bval;
  // compact column runs (nullptr: none): cptr[s] >= 0, the slice's columns at
  // bcol[cptr[s] + k*32 + lane]; cptr[s] < 0, its run offsets from the row at
  // bcol[~cptr[s] + k]
  const int* cptr = nullptr;
};

// NC: gather x through the read-only cache (only when x is not written
// during the kernel).
// U: column chunks whose loads are issued together (more bytes in flight per
// warp for kernels with few warps per SM).
// R: the layout's run length: each column index J0 serves R consecutive
// value chunks, for node columns J0 .. J0+R-1 (R = 1: one index per block).
// The blocks are visited in ascending column order for every R, and a run's
// empty slots hold zeros, so both layouts give the same sums.
template <int ND, bool PADDED, bool NC = true, int U = 2, int R = 1>
__device__ __forceinline__ void spmv_row_b(const BlockMat& A, int s, int lane, const float* x, float* acc) {
  constexpr int BB = ND * ND;
  const int c0 = A.bsoff[s], w = (A.bsoff[s + 1] - c0) / R;
  // run k's column: J0 = base + cp[k * stride] (a compact slice: the row plus
  // one offset that every lane reads; otherwise the lane's own column)
  const int* cp = A.bcol + (long long)(c0 / R) * 32 + lane;
  int stride = 32, base = 0;
  if constexpr (R > 1) {
    if (A.cptr) {
      const int p = A.cptr[s];
      if (p < 0) {
        cp = A.bcol + ~p;
        stride = 1;
        base = s * 32 + lane;
      } else {
        cp = A.bcol + p + lane;
      }
    }
  }
  const float* vp = A.bval + (long long)c0 * 32 * BB + lane;
#pragma unroll
  for (int i = 0; i < ND; ++i) acc[i] = 0.f;
#pragma unroll U
  for (int k = 0; k < w; ++k) {
    const int J0 = R > 1 ? base + __ldg(cp + k * stride) : __ldcs(cp + k * 32);
#pragma unroll
    for (int j = 0; j < R; ++j) {
      const int J = J0 + j;
      float xv[ND];
      if constexpr (PADDED) {
        if constexpr (NC) PVec<ND>::ldg(x, J, xv);
        else PVec<ND>::ld(x, J, xv);
      } else {
        if constexpr (NC) NodeIO<ND>::ldg(x, J, xv);
        else NodeIO<ND>::ld(x, J, xv);
      }
      float v[BB];
#pragma unroll
      for (int t = 0; t < BB; ++t) v[t] = __ldcs(vp + ((long long)(k * R + j) * BB + t) * 32);
#pragma unroll
      for (int i = 0; i < ND; ++i)
#pragma unroll
        for (int jj = 0; jj < ND; ++jj) acc[i] = fmaf(v[i * ND + jj], xv[jj], acc[i]);
    }
  }
}

// Loads in flight and resident blocks of the inner SpMV per layout, from
// measurements on the 100^3 cube (ND 3) and the 256x256x64 slab (ND 1):
// one column per block: four chunks per lane, 4 x 256 threads per SM;
// runs of 3 (ND 3): one run (27 values, 3 gathers) per lane, 4 blocks per SM;
// runs of 3 (ND 1): two runs per lane, 8 blocks per SM.
template <int ND, int R>
struct SpmvShape {
  static constexpr int U = R == 1 ? 4 : (ND == 3 ? 1 : 2);
  static constexpr int MINB = (R > 1 && ND == 1) ? 8 : 4;
};

template <int ND, int R = 1>
__global__ void __launch_bounds__(256) k_spmv_b(BlockMat A, const float* __restrict__ x, float* __restrict__ y) {
  const int lane = threadIdx.x & 31;
  for (int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; s < A.nslice; s += (gridDim.x * blockDim.x) >> 5) {
    float acc[ND];
    spmv_row_b<ND, false, true, 2, R>(A, s, lane, x, acc);
    const int I = s * 32 + lane;
    if (I < A.nnode) NodeIO<ND>::st(y, I, acc);
  }
}

// q = A p, alpha = rho / (p.q)
// One column per block: four chunks' loads in flight per lane (1024 threads
// per SM at up to 64 registers), 6 % faster than two at eight 256-thread
// blocks per SM on the 100^3 cube, bit-identical (the same sums in the same
// order).  Runs of 3 columns: 10 % (ND 3) and 30 % (ND 1) faster again.
template <int ND, int R = 1>
__global__ void __launch_bounds__(256, SpmvShape<ND, R>::MINB) k_spmv_dot_b(BlockMat A, const float* __restrict__ p,
                                                       float* __restrict__ q, PcgState* st, double* partials) {
  if (st->done) return;
  const int lane = threadIdx.x & 31;
  double acc_d[1] = {0.0};
  for (int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; s < A.nslice; s += (gridDim.x * blockDim.x) >> 5) {
    float acc[ND];
    spmv_row_b<ND, true, true, SpmvShape<ND, R>::U, R>(A, s, lane, p, acc);
    const int I = s * 32 + lane;
    if (I < A.nnode) {
      NodeIO<ND>::st(q, I, acc);
      float pv[ND];
      PVec<ND>::ld(p, I, pv);
      float t = 0.f;
#pragma unroll
      for (int i = 0; i < ND; ++i) t = fmaf(pv[i], acc[i], t);
      acc_d[0] += (double)t;
    }
  }
  double out[1];
  if (reduce_last<1>(acc_d, partials, &st->ticket, out) && threadIdx.x == 0) {
    st->pq = out[0];
    if (!finite_pos(out[0])) {
      st->status = kStatusBreakdown;
      st->done = 1;
    } else {
      st->alpha = st->rho / out[0];
    }
  }
}


// x += alpha p; r -= alpha q; z = M r; (r.z, r.r, x.x) in FP64
template <int ND>
__global__ void __launch_bounds__(256) k_update_b(int nnode, float* __restrict__ x, float* __restrict__ r,
                                                  const float* __restrict__ p, const float* __restrict__ q,
                                                  const float* __restrict__ minv, PcgState* st, double* partials) {
  if (st->done) return;
  const float a = (float)st->alpha;
  double acc[3] = {0.0, 0.0, 0.0};
  for (int I = blockIdx.x * blockDim.x + threadIdx.x; I < nnode; I += gridDim.x * blockDim.x) {
    float xv[ND], rv[ND], pv[ND], qv[ND], z[ND];
    NodeIO<ND>::ld(x, I, xv);
    NodeIO<ND>::ld(r, I, rv);
    PVec<ND>::ld(p, I, pv);
    NodeIO<ND>::ld(q, I, qv);
#pragma unroll
    for (int i = 0; i < ND; ++i) {
      xv[i] = fmaf(a, pv[i], xv[i]);
      rv[i] = fmaf(-a, qv[i], rv[i]);
    }
    NodeIO<ND>::st(x, I, xv);
    NodeIO<ND>::st(r, I, rv);
    NodeIO<ND>::prec(minv, I, rv, z);
    float rz = 0.f, r2 = 0.f, x2 = 0.f;
#pragma unroll
    for (int i = 0; i < ND; ++i) {
      rz = fmaf(rv[i], z[i], rz);
      r2 = fmaf(rv[i], rv[i], r2);
      x2 = fmaf(xv[i], xv[i], x2);
    }
    acc[0] += rz;
    acc[1] += r2;
    acc[2] += x2;
  }
  double out[3];
  if (reduce_last<3>(acc, partials, &st->ticket, out) && threadIdx.x == 0) finish_update(st, out[0], out[1], out[2]);
}

// ---- the same two vector passes, several consecutive nodes per thread -----
// NPT consecutive nodes' ND components are NPT*ND floats, the padded
// direction NPT*PVec::W and the packed block-Jacobi factors NPT*ND(ND+1)/2:
// a thread moves them with the widest aligned accesses those counts allow
// (16 or 8 bytes) instead of ND 4-byte ones per node.  Per node the arithmetic
// is the same; the FP64 partial sums add the nodes in another grouping.  The
// last nnode % NPT nodes go one per thread.  Used for one dof per node, four
// nodes (16-byte accesses; the one-node update reached 0.73 of HBM on the
// slab: transient step 30.4 -> 29.7 ms).  Two and three dofs per node keep
// the one-node kernels k_update_b and k_pupd_b: at three, this form with one
// node per thread took 32 us a cold update launch on the 100^3 cube against
// 27 (64-bit indexing, every load issued before the stores), two nodes
// measured the same cube step, four nodes at 80 registers slower.
template <int N>
__device__ __forceinline__ void ldn(const float* v, long long blk, float (&o)[N]) {
  if constexpr (N % 4 == 0) {
    const float4* q = reinterpret_cast<const float4*>(v) + blk * (N / 4);
#pragma unroll
    for (int k = 0; k < N / 4; ++k) {
      const float4 t = q[k];
      o[4 * k] = t.x; o[4 * k + 1] = t.y; o[4 * k + 2] = t.z; o[4 * k + 3] = t.w;
    }
  } else if constexpr (N % 2 == 0) {
    const float2* q = reinterpret_cast<const float2*>(v) + blk * (N / 2);
#pragma unroll
    for (int k = 0; k < N / 2; ++k) {
      const float2 t = q[k];
      o[2 * k] = t.x; o[2 * k + 1] = t.y;
    }
  } else {
#pragma unroll
    for (int k = 0; k < N; ++k) o[k] = v[blk * N + k];
  }
}
template <int N>
__device__ __forceinline__ void stn(float* v, long long blk, const float (&a)[N]) {
  if constexpr (N % 4 == 0) {
    float4* q = reinterpret_cast<float4*>(v) + blk * (N / 4);
#pragma unroll
    for (int k = 0; k < N / 4; ++k) q[k] = make_float4(a[4 * k], a[4 * k + 1], a[4 * k + 2], a[4 * k + 3]);
  } else if constexpr (N % 2 == 0) {
    float2* q = reinterpret_cast<float2*>(v) + blk * (N / 2);
#pragma unroll
    for (int k = 0; k < N / 2; ++k) q[k] = make_float2(a[2 * k], a[2 * k + 1]);
  } else {
#pragma unroll
    for (int k = 0; k < N; ++k) v[blk * N + k] = a[k];
  }
}

template <int ND>
__device__ __forceinline__ void prec_packed(const float* a, const float* r, float* z) {
  if constexpr (ND == 1) {
    z[0] = a[0] * r[0];
  } else if constexpr (ND == 2) {
    z[0] = fmaf(a[0], r[0], a[1] * r[1]);
    z[1] = fmaf(a[1], r[0], a[2] * r[1]);
  } else {
    z[0] = fmaf(a[0], r[0], fmaf(a[1], r[1], a[2] * r[2]));
    z[1] = fmaf(a[1], r[0], fmaf(a[3], r[1], a[4] * r[2]));
    z[2] = fmaf(a[2], r[0], fmaf(a[4], r[1], a[5] * r[2]));
  }
}

template <int ND>
struct PassNodes {
  static constexpr int N = ND == 1 ? 4 : 1;  // nodes per thread
};

// x += alpha p; r -= alpha q; z = M r; (r.z, r.r, x.x) in FP64
template <int ND>
__global__ void __launch_bounds__(256) k_update_bn(int nnode, float* __restrict__ x, float* __restrict__ r,
                                                   const float* __restrict__ p, const float* __restrict__ q,
                                                   const float* __restrict__ minv, PcgState* st,
                                                   double* partials) {
  if (st->done) return;
  constexpr int S = ND * (ND + 1) / 2, W = PVec<ND>::W, NP = PassNodes<ND>::N;
  const float a = (float)st->alpha;
  double acc[3] = {0.0, 0.0, 0.0};
  const long long nb = nnode / NP;
  const long long tid = blockIdx.x * (long long)blockDim.x + threadIdx.x, nt = (long long)gridDim.x * blockDim.x;
  for (long long ib = tid; ib < nb; ib += nt) {
    float xv[NP * ND], rv[NP * ND], qv[NP * ND], pv[NP * W], mv[NP * S];
    ldn<NP * ND>(x, ib, xv);
    ldn<NP * ND>(r, ib, rv);
    ldn<NP * W>(p, ib, pv);
    ldn<NP * ND>(q, ib, qv);
    ldn<NP * S>(minv, ib, mv);
#pragma unroll
    for (int j = 0; j < NP; ++j) {
#pragma unroll
      for (int i = 0; i < ND; ++i) {
        xv[ND * j + i] = fmaf(a, pv[W * j + i], xv[ND * j + i]);
        rv[ND * j + i] = fmaf(-a, qv[ND * j + i], rv[ND * j + i]);
      }
      float z[ND];
      prec_packed<ND>(mv + S * j, rv + ND * j, z);
      float rz = 0.f, r2 = 0.f, x2 = 0.f;
#pragma unroll
      for (int i = 0; i < ND; ++i) {
        rz = fmaf(rv[ND * j + i], z[i], rz);
        r2 = fmaf(rv[ND * j + i], rv[ND * j + i], r2);
        x2 = fmaf(xv[ND * j + i], xv[ND * j + i], x2);
      }
      acc[0] += rz;
      acc[1] += r2;
      acc[2] += x2;
    }
    stn<NP * ND>(x, ib, xv);
    stn<NP * ND>(r, ib, rv);
  }
  for (long long I = NP * nb + tid; I < nnode; I += nt) {  // the last nnode % NP nodes
    float xv[ND], rv[ND], pv[ND], qv[ND], z[ND];
    NodeIO<ND>::ld(x, I, xv);
    NodeIO<ND>::ld(r, I, rv);
    PVec<ND>::ld(p, I, pv);
    NodeIO<ND>::ld(q, I, qv);
#pragma unroll
    for (int i = 0; i < ND; ++i) {
      xv[i] = fmaf(a, pv[i], xv[i]);
      rv[i] = fmaf(-a, qv[i], rv[i]);
    }
    NodeIO<ND>::st(x, I, xv);
    NodeIO<ND>::st(r, I, rv);
    NodeIO<ND>::prec(minv, I, rv, z);
    float rz = 0.f, r2 = 0.f, x2 = 0.f;
#pragma unroll
    for (int i = 0; i < ND; ++i) {
      rz = fmaf(rv[i], z[i], rz);
      r2 = fmaf(rv[i], rv[i], r2);
      x2 = fmaf(xv[i], xv[i], x2);
    }
    acc[0] += rz;
    acc[1] += r2;
    acc[2] += x2;
  }
  double out[3];
  if (reduce_last<3>(acc, partials, &st->ticket, out) && threadIdx.x == 0) finish_update(st, out[0], out[1], out[2]);
}

// p = M r + beta p
template <int ND>
__global__ void __launch_bounds__(256) k_pupd_bn(int nnode, float* __restrict__ p, const float* __restrict__ r,
                                                 const float* __restrict__ minv, const PcgState* st) {
  if (st->done) return;
  constexpr int S = ND * (ND + 1) / 2, W = PVec<ND>::W, NP = PassNodes<ND>::N;
  const float bt = (float)st->beta;
  const long long nb = nnode / NP;
  const long long tid = blockIdx.x * (long long)blockDim.x + threadIdx.x, nt = (long long)gridDim.x * blockDim.x;
  for (long long ib = tid; ib < nb; ib += nt) {
    float rv[NP * ND], pv[NP * W], mv[NP * S];
    ldn<NP * ND>(r, ib, rv);
    ldn<NP * W>(p, ib, pv);
    ldn<NP * S>(minv, ib, mv);
#pragma unroll
    for (int j = 0; j < NP; ++j) {
      float z[ND];
      prec_packed<ND>(mv + S * j, rv + ND * j, z);
#pragma unroll
      for (int i = 0; i < ND; ++i) pv[W * j + i] = fmaf(bt, pv[W * j + i], z[i]);
      if constexpr (W > ND) pv[W * j + ND] = 0.f;  // the padding lane of a padded node
    }
    stn<NP * W>(p, ib, pv);
  }
  for (long long I = NP * nb + tid; I < nnode; I += nt) {
    float rv[ND], pv[ND], z[ND];
    NodeIO<ND>::ld(r, I, rv);
    PVec<ND>::ld(p, I, pv);
    NodeIO<ND>::prec(minv, I, rv, z);
#pragma unroll
    for (int i = 0; i < ND; ++i) pv[i] = fmaf(bt, pv[i], z[i]);
    PVec<ND>::st(p, I, pv);
  }
}

// p = M r + beta p
template <int ND>
__global__ void __launch_bounds__(256) k_pupd_b(int nnode, float* __restrict__ p, const float* __restrict__ r,
                                                const float* __restrict__ minv, const PcgState* st) {
  if (st->done) return;
  const float bt = (float)st->beta;
  for (int I = blockIdx.x * blockDim.x + threadIdx.x; I < nnode; I += gridDim.x * blockDim.x) {
    float rv[ND], pv[ND], z[ND];
    NodeIO<ND>::ld(r, I, rv);
    PVec<ND>::ld(p, I, pv);
    NodeIO<ND>::prec(minv, I, rv, z);
#pragma unroll
    for (int i = 0; i < ND; ++i) pv[i] = fmaf(bt, pv[i], z[i]);
    PVec<ND>::st(p, I, pv);
  }
}

// Inner start: x = 0, r given, p = z = M r, rho = r.z, ref0 = maxrr = r.r
template <int ND>
__global__ void __launch_bounds__(256) k_start_b(int nnode, float* __restrict__ x, const float* __restrict__ r,
                                                 float* __restrict__ p, const float* __restrict__ minv, PcgState* st,
                                                 double* partials) {
  double acc[2] = {0.0, 0.0};
  for (int I = blockIdx.x * blockDim.x + threadIdx.x; I < nnode; I += gridDim.x * blockDim.x) {
    float rv[ND], z[ND], zero[ND];
    NodeIO<ND>::ld(r, I, rv);
#pragma unroll
    for (int i = 0; i < ND; ++i) zero[i] = 0.f;
    NodeIO<ND>::prec(minv, I, rv, z);
    PVec<ND>::st(p, I, z);
    NodeIO<ND>::st(x, I, zero);
#pragma unroll
    for (int i = 0; i < ND; ++i) { acc[0] += (double)rv[i] * z[i]; acc[1] += (double)rv[i] * rv[i]; }
  }
  double out[2];
  if (reduce_last<2>(acc, partials, &st->ticket, out) && threadIdx.x == 0) {
    st->rho = out[0];
    st->rr = out[1];
    st->ref0 = out[1];
    st->maxrr = out[1];
    st->xx = 0.0;
    st->iter = 0;
    st->status = kStatusOk;
    st->done = 0;
    st->last = 1.0;
    if (!(out[0] == out[0])) { st->status = kStatusBreakdown; st->done = 1; }
    else if (out[1] == 0.0) { st->done = 1; st->last = 0.0; }
  }
}

// Reliable update, second half: r has been replaced by the true residual.
// rho_new = r.z, beta = rho_new / rho_old, rho = rho_new, maxrr = r.r, and
// the solve continues (done = 0).  The following k_pupd_b forms p.
template <int ND>
__global__ void __launch_bounds__(256) k_replace_b(int nnode, const float* __restrict__ r,
                                                   const float* __restrict__ minv, PcgState* st, double* partials) {
  double acc[2] = {0.0, 0.0};
  for (int I = blockIdx.x * blockDim.x + threadIdx.x; I < nnode; I += gridDim.x * blockDim.x) {
    float rv[ND], z[ND];
    NodeIO<ND>::ld(r, I, rv);
    NodeIO<ND>::prec(minv, I, rv, z);
#pragma unroll
    for (int i = 0; i < ND; ++i) { acc[0] += (double)rv[i] * z[i]; acc[1] += (double)rv[i] * rv[i]; }
  }
  double out[2];
  if (reduce_last<2>(acc, partials, &st->ticket, out) && threadIdx.x == 0) {
    st->beta = st->rho != 0.0 ? out[0] / st->rho : 0.0;
    st->rho = out[0];
    st->rr = out[1];
    st->maxrr = out[1];
    st->status = kStatusOk;
    st->done = (out[0] == out[0]) ? 0 : 1;
    if (st->done) st->status = kStatusBreakdown;
  }
}

// ---- LargeMatrix::CheckAndFixZeroDiagonal (largeMatrix.cpp:43-79) ----------
// first[0] gets the lowest unknown whose global diagonal is zero, first[1] the
// lowest whose diagonal is negative (the caller presets both to a sentinel):
// the reference scans in order and stops at the first zero, so a negative
// entry counts only below it.
__global__ void k_diag_scan_s(int n, const long long* __restrict__ sdiag, const double* __restrict__ sval,
                              int* first) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double d = sval[sdiag[i]];
    if (d == 0.0) atomicMin(first, i);
    else if (d < 0.0) atomicMin(first + 1, i);
  }
}

// every zero diagonal of the scalar matrix becomes value
__global__ void k_diag_fix_s(int n, const long long* __restrict__ sdiag, double* sval, double value) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    if (sval[sdiag[i]] == 0.0) sval[sdiag[i]] = value;
}

// the same scan over the diagonal entries of the node-block matrix (unknown
// ND*I + c is entry (c, c) of node I's diagonal block)
template <int ND>
__global__ void k_diag_scan_b(int nnode, const int* __restrict__ bsoff, const int* __restrict__ ndiag,
                              const float* __restrict__ bval, int* first) {
  constexpr int BB = ND * ND;
  for (int I = blockIdx.x * blockDim.x + threadIdx.x; I < nnode; I += gridDim.x * blockDim.x) {
    const long long base = ((long long)bsoff[I >> 5] + ndiag[I]) * 32 * BB + (I & 31);
    for (int c = 0; c < ND; ++c) {
      const float d = bval[base + (long long)(c * ND + c) * 32];
      if (d == 0.f) atomicMin(first, ND * I + c);
      else if (d < 0.f) atomicMin(first + 1, ND * I + c);
    }
  }
}

// every zero diagonal of the node-block matrix becomes value; zrep marks them
// (the FP64 matrix-free operator adds value * x there)
template <int ND>
__global__ void k_diag_fix_b(int nnode, const int* __restrict__ bsoff, const int* __restrict__ ndiag, float* bval,
                             float value, unsigned char* zrep) {
  constexpr int BB = ND * ND;
  for (int I = blockIdx.x * blockDim.x + threadIdx.x; I < nnode; I += gridDim.x * blockDim.x) {
    const long long base = ((long long)bsoff[I >> 5] + ndiag[I]) * 32 * BB + (I & 31);
    for (int c = 0; c < ND; ++c) {
      float* d = bval + base + (long long)(c * ND + c) * 32;
      if (*d == 0.f) {
        *d = value;
        zrep[ND * I + c] = 1;
      }
    }
  }
}

// y += value * w on the unknowns whose zero diagonal was replaced
__global__ void k_zdiag_apply(int n, const unsigned char* __restrict__ zrep, double value,
                              const double* __restrict__ w, double* y) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    if (zrep[i]) y[i] += value * w[i];
}

// Block-Jacobi factors: invert the node diagonal block in FP64 and store the
// packed upper triangle; jacobi_only keeps 1/diag.  Flags non-positive diagonals.
template <int ND>
__global__ void k_minv_b(int nnode, const int* bsoff, const int* ndiag, const float* bval, float* minv,
                         int jacobi_only, unsigned* flags) {
  constexpr int BB = ND * ND, S = ND * (ND + 1) / 2;
  for (int I = blockIdx.x * blockDim.x + threadIdx.x; I < nnode; I += gridDim.x * blockDim.x) {
    const long long chunk = (long long)bsoff[I >> 5] + ndiag[I];
    double D[9] = {0}, Di[9] = {0};
    for (int t = 0; t < BB; ++t) D[t] = bval[chunk * 32 * BB + t * 32 + (I & 31)];
    bool bad = false;
    for (int i = 0; i < ND; ++i) bad |= !(D[i * ND + i] > 0.0);
    if (bad) atomicOr(flags, 16u);
    if (jacobi_only || ND == 1) {
      for (int i = 0; i < ND; ++i) Di[i * ND + i] = D[i * ND + i] != 0.0 ? 1.0 / D[i * ND + i] : 0.0;
    } else if (ND == 2) {
      const double det = D[0] * D[3] - D[1] * D[2], id = 1.0 / det;
      Di[0] = D[3] * id; Di[1] = -D[1] * id; Di[2] = -D[2] * id; Di[3] = D[0] * id;
    } else {
      inv3<double>(D, Di);
    }
    int t = 0;
    for (int i = 0; i < ND; ++i)
      for (int j = i; j < ND; ++j) minv[(long long)S * I + (t++)] = (float)(0.5 * (Di[i * ND + j] + Di[j * ND + i]));
  }
}

// ======================== FP64 <-> FP32 glue ===========================
// r32 = (float)(r64 * scale)
__global__ void k_to32(long long n, const double* __restrict__ r64, double scale, float* __restrict__ r32) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    r32[i] = (float)(r64[i] * scale);
}

// x64 += scale * d32
__global__ void k_axpy_from32(long long n, double* __restrict__ x64, double scale, const float* __restrict__ d32) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    x64[i] += scale * (double)d32[i];
}

// ===================== caller-owned CSR (device pointers) =====================
// Full (both-triangle) CSR, 8 lanes per row, a warp covers 4 rows.
struct CsrMat {
  int n;
  const int* rp;
  const int* ci;
  const double* v;
};

__device__ __forceinline__ double csr_row8(const CsrMat& A, int row, int sub, const double* __restrict__ x) {
  double acc = 0.0;
  if (row < A.n)
    for (int k = A.rp[row] + sub; k < A.rp[row + 1]; k += 8) acc += A.v[k] * __ldg(x + A.ci[k]);
  return group_sum<8>(acc);
}

// y = A x, or y = b - A x when b is given
__global__ void __launch_bounds__(256) k_csr_spmv(CsrMat A, const double* __restrict__ x, double* __restrict__ y,
                                                  const double* __restrict__ b) {
  const int lane = threadIdx.x & 31, sub = lane & 7;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  for (int base = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 4; base < A.n; base += nwarps * 4) {
    const int row = base + (lane >> 3);
    const double v = csr_row8(A, row, sub, x);
    if (sub == 0 && row < A.n) y[row] = b ? b[row] - v : v;
  }
}

// q = A p, alpha = rho / (p.q)
__global__ void __launch_bounds__(256) k_csr_spmv_dot(CsrMat A, const double* __restrict__ p, double* __restrict__ q,
                                                      PcgState* st, double* partials) {
  if (st->done) return;
  const int lane = threadIdx.x & 31, sub = lane & 7;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  double acc[1] = {0.0};
  for (int base = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 4; base < A.n; base += nwarps * 4) {
    const int row = base + (lane >> 3);
    const double v = csr_row8(A, row, sub, p);
    if (sub == 0 && row < A.n) {
      q[row] = v;
      acc[0] += p[row] * v;
    }
  }
  double out[1];
  if (reduce_last<1>(acc, partials, &st->ticket, out) && threadIdx.x == 0) {
    st->pq = out[0];
    if (!finite_pos(out[0])) {
      st->status = kStatusBreakdown;
      st->done = 1;
    } else {
      st->alpha = st->rho / out[0];
    }
  }
}

// 1/diag of a CSR matrix (flags 8: zero diagonal, 16: negative)
__global__ void k_csr_dinv(CsrMat A, double* dinv, unsigned* flags) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < A.n; i += gridDim.x * blockDim.x) {
    double d = 0.0;
    for (int k = A.rp[i]; k < A.rp[i + 1]; ++k)
      if (A.ci[k] == i) d += A.v[k];
    if (!(d > 0.0)) atomicOr(flags, d == 0.0 ? 8u : 16u);
    dinv[i] = d != 0.0 ? 1.0 / d : 0.0;
  }
}

// ============================== FP64 vector ops ===============================
// r = rest ? 0 : load - y ; sums (r.r, x.x)
__global__ void __launch_bounds__(256) k_residual64(int n, const unsigned char* __restrict__ rest,
                                                    const double* __restrict__ load, const double* __restrict__ y,
                                                    const double* __restrict__ x, double* __restrict__ r,
                                                    double* sums, double* partials, unsigned* ticket) {
  double acc[2] = {0.0, 0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double ri = rest[i] ? 0.0 : (load ? load[i] : 0.0) - y[i];
    r[i] = ri;
    acc[0] += ri * ri;
    acc[1] += x[i] * x[i];
  }
  double out[2];
  if (reduce_last<2>(acc, partials, ticket, out) && threadIdx.x == 0) {
    sums[0] = out[0];
    sums[1] = out[1];
  }
}

// b = rest ? presc : load + pseudo ; x0 = rest ? presc : 0 (or keep)
__global__ void k_rhs64(int n, const unsigned char* rest, const double* presc, const double* load,
                        const double* pseudo, double* b) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    b[i] = rest[i] ? presc[i] : (load ? load[i] : 0.0) + (pseudo ? pseudo[i] : 0.0);
}

// The load that reproduces an eliminated right-hand side b: on free rows
// b + (K x_ext)_free with x_ext = b on restrained rows (y holds K x_ext), 0 on
// restrained rows (their value comes from the prescribed array).
__global__ void k_load_from_rhs(int n, const unsigned char* rest, const double* b, const double* y, double* load) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    load[i] = rest[i] ? 0.0 : b[i] + y[i];
}

// x_ext = rest ? presc : (x ? x : 0)
__global__ void k_ext64(int n, const unsigned char* rest, const double* presc, const double* x, double* out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    out[i] = rest[i] ? (presc ? presc[i] : 0.0) : (x ? x[i] : 0.0);
}

// b = rest ? presc : load - y (the eliminated right-hand side), sum b.b
__global__ void __launch_bounds__(256) k_rhs_elim64(int n, const unsigned char* __restrict__ rest,
                                                    const double* __restrict__ presc,
                                                    const double* __restrict__ load, const double* __restrict__ y,
                                                    double* __restrict__ b, double* sums, double* partials,
                                                    unsigned* ticket) {
  double acc[1] = {0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double bi = rest[i] ? (presc ? presc[i] : 0.0) : (load ? load[i] : 0.0) - y[i];
    b[i] = bi;
    acc[0] += bi * bi;
  }
  double out[1];
  if (reduce_last<1>(acc, partials, ticket, out) && threadIdx.x == 0) sums[0] = out[0];
}

// Newton residual r = rest ? 0 : load - y, and the largest |r| (bits of a
// non-negative double: integer order is IEEE order, so atomicMax is exact and
// order-free; a NaN ranks above every number).
__global__ void __launch_bounds__(256) k_newton_residual(int n, const unsigned char* __restrict__ rest,
                                                         const double* __restrict__ load,
                                                         const double* __restrict__ y, double* __restrict__ r,
                                                         unsigned long long* maxbits) {
  double m = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double ri = rest[i] ? 0.0 : (load ? load[i] : 0.0) - y[i];
    r[i] = ri;
    const double a = fabs(ri);
    if (a > m || a != a) m = a;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double t = __shfl_xor_sync(0xffffffffu, m, o);
    if (t > m || t != t) m = t;
  }
  if ((threadIdx.x & 31) == 0) atomicMax(maxbits, (unsigned long long)__double_as_longlong(m));
}

// u += d on free dofs
__global__ void k_add_free64(int n, const unsigned char* __restrict__ rest, double* __restrict__ u,
                             const double* __restrict__ d) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    if (!rest[i]) u[i] += d[i];
}

__global__ void k_add_free_from32(int n, const unsigned char* __restrict__ rest, double* __restrict__ u,
                                  const float* __restrict__ d) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    if (!rest[i]) u[i] += (double)d[i];
}

// y += a x
__global__ void k_axpy64(int n, double* __restrict__ y, double a, const double* __restrict__ x) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) y[i] += a * x[i];
}

// sum of squares of a - b (or of a)
__global__ void __launch_bounds__(256) k_norm2_diff(int n, const double* __restrict__ a, const double* __restrict__ b,
                                                    double* sums, double* partials, unsigned* ticket) {
  double acc[1] = {0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double d = b ? a[i] - b[i] : a[i];
    acc[0] += d * d;
  }
  double out[1];
  if (reduce_last<1>(acc, partials, ticket, out) && threadIdx.x == 0) sums[0] = out[0];
}

}  // namespace betagpu
