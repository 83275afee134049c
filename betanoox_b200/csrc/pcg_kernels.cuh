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
//   block   : FP32 values, one row per node with ND x ND blocks, vectors as
//             float / float2 / float4 per node (mixed-precision inner PCG,
//             Jacobi or node block-Jacobi)
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
  int iter, maxit, status, done;
  int rule;
  unsigned ticket;
};

constexpr int kStatusOk = 0, kStatusMaxit = 4, kStatusBreakdown = 5;

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
  st->beta = st->rho != 0.0 ? rz / st->rho : 0.0;
  st->rho = rz;
  if (q < st->tol2) {
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
  double acc0 = 0.0, acc1 = 0.0;
  int k = 0;
  for (; k + 1 < w; k += 2) {
    const int c0 = __ldcs(cp + (long long)k * 32), c1 = __ldcs(cp + (long long)(k + 1) * 32);
    const double v0 = __ldcs(vp + (long long)k * 32), v1 = __ldcs(vp + (long long)(k + 1) * 32);
    acc0 += v0 * __ldg(x + c0);
    acc1 += v1 * __ldg(x + c1);
  }
  if (k < w) acc0 += __ldcs(vp + (long long)k * 32) * __ldg(x + __ldcs(cp + (long long)k * 32));
  return acc0 + acc1;
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
template <int ND> struct NV;
template <> struct NV<1> { using T = float; };
template <> struct NV<2> { using T = float2; };
template <> struct NV<3> { using T = float4; };

template <int ND> __device__ __forceinline__ float comp(const typename NV<ND>::T& v, int i);
template <> __device__ __forceinline__ float comp<1>(const float& v, int) { return v; }
template <> __device__ __forceinline__ float comp<2>(const float2& v, int i) { return i ? v.y : v.x; }
template <> __device__ __forceinline__ float comp<3>(const float4& v, int i) { return i == 0 ? v.x : (i == 1 ? v.y : v.z); }

template <int ND> __device__ __forceinline__ typename NV<ND>::T mk(const float* a);
template <> __device__ __forceinline__ float mk<1>(const float* a) { return a[0]; }
template <> __device__ __forceinline__ float2 mk<2>(const float* a) { return make_float2(a[0], a[1]); }
template <> __device__ __forceinline__ float4 mk<3>(const float* a) { return make_float4(a[0], a[1], a[2], 0.f); }

struct BlockMat {
  int nnode, nslice;
  const int* bsoff;  // nslice+1 (chunks)
  const int* bcol;
  const float* bval;
};

template <int ND>
__device__ __forceinline__ void spmv_row_b(const BlockMat& A, int s, int lane,
                                           const typename NV<ND>::T* __restrict__ x, float* acc) {
  constexpr int BB = ND * ND;
  const int c0 = A.bsoff[s], w = A.bsoff[s + 1] - c0;
  const int* cp = A.bcol + (long long)c0 * 32 + lane;
  const float* vp = A.bval + (long long)c0 * 32 * BB + lane;
#pragma unroll
  for (int i = 0; i < ND; ++i) acc[i] = 0.f;
#pragma unroll 2
  for (int k = 0; k < w; ++k) {
    const int J = __ldcs(cp + k * 32);
    const typename NV<ND>::T xv = __ldg(x + J);
    float v[BB];
#pragma unroll
    for (int t = 0; t < BB; ++t) v[t] = __ldcs(vp + (long long)k * 32 * BB + t * 32);
#pragma unroll
    for (int i = 0; i < ND; ++i)
#pragma unroll
      for (int j = 0; j < ND; ++j) acc[i] = fmaf(v[i * ND + j], comp<ND>(xv, j), acc[i]);
  }
}

template <int ND>
__global__ void __launch_bounds__(256) k_spmv_b(BlockMat A, const typename NV<ND>::T* __restrict__ x,
                                                typename NV<ND>::T* __restrict__ y) {
  const int lane = threadIdx.x & 31;
  for (int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; s < A.nslice; s += (gridDim.x * blockDim.x) >> 5) {
    float acc[ND];
    spmv_row_b<ND>(A, s, lane, x, acc);
    const int I = s * 32 + lane;
    if (I < A.nnode) y[I] = mk<ND>(acc);
  }
}

template <int ND>
__global__ void __launch_bounds__(256) k_spmv_dot_b(BlockMat A, const typename NV<ND>::T* __restrict__ p,
                                                    typename NV<ND>::T* __restrict__ q, PcgState* st,
                                                    double* partials) {
  if (st->done) return;
  const int lane = threadIdx.x & 31;
  double acc_d[1] = {0.0};
  for (int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; s < A.nslice; s += (gridDim.x * blockDim.x) >> 5) {
    float acc[ND];
    spmv_row_b<ND>(A, s, lane, p, acc);
    const int I = s * 32 + lane;
    if (I < A.nnode) {
      q[I] = mk<ND>(acc);
      const typename NV<ND>::T pv = p[I];
      float t = 0.f;
#pragma unroll
      for (int i = 0; i < ND; ++i) t = fmaf(comp<ND>(pv, i), acc[i], t);
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

// Block-Jacobi apply z = Minv r with Minv stored as ND row vectors per node.
template <int ND>
__device__ __forceinline__ void prec_apply(const typename NV<ND>::T* __restrict__ minv, int nnode, int I,
                                           const float* r, float* z) {
#pragma unroll
  for (int i = 0; i < ND; ++i) {
    const typename NV<ND>::T m = minv[(long long)i * nnode + I];
    float t = 0.f;
#pragma unroll
    for (int j = 0; j < ND; ++j) t = fmaf(comp<ND>(m, j), r[j], t);
    z[i] = t;
  }
}

// x += alpha p; r -= alpha q; z = Minv r; (r.z, r.r, x.x) in FP64
template <int ND>
__global__ void __launch_bounds__(256) k_update_b(int nnode, typename NV<ND>::T* __restrict__ x,
                                                  typename NV<ND>::T* __restrict__ r,
                                                  const typename NV<ND>::T* __restrict__ p,
                                                  const typename NV<ND>::T* __restrict__ q,
                                                  const typename NV<ND>::T* __restrict__ minv, PcgState* st,
                                                  double* partials) {
  if (st->done) return;
  const float a = (float)st->alpha;
  double acc[3] = {0.0, 0.0, 0.0};
  for (int I = blockIdx.x * blockDim.x + threadIdx.x; I < nnode; I += gridDim.x * blockDim.x) {
    const typename NV<ND>::T xv = x[I], rv = r[I], pv = p[I], qv = q[I];
    float xn[ND], rn[ND], z[ND];
#pragma unroll
    for (int i = 0; i < ND; ++i) {
      xn[i] = fmaf(a, comp<ND>(pv, i), comp<ND>(xv, i));
      rn[i] = fmaf(-a, comp<ND>(qv, i), comp<ND>(rv, i));
    }
    x[I] = mk<ND>(xn);
    r[I] = mk<ND>(rn);
    prec_apply<ND>(minv, nnode, I, rn, z);
    float rz = 0.f, r2 = 0.f, x2 = 0.f;
#pragma unroll
    for (int i = 0; i < ND; ++i) {
      rz = fmaf(rn[i], z[i], rz);
      r2 = fmaf(rn[i], rn[i], r2);
      x2 = fmaf(xn[i], xn[i], x2);
    }
    acc[0] += rz;
    acc[1] += r2;
    acc[2] += x2;
  }
  double out[3];
  if (reduce_last<3>(acc, partials, &st->ticket, out) && threadIdx.x == 0) finish_update(st, out[0], out[1], out[2]);
}

// p = Minv r + beta p
template <int ND>
__global__ void __launch_bounds__(256) k_pupd_b(int nnode, typename NV<ND>::T* __restrict__ p,
                                                const typename NV<ND>::T* __restrict__ r,
                                                const typename NV<ND>::T* __restrict__ minv,
                                                const PcgState* st) {
  if (st->done) return;
  const float bt = (float)st->beta;
  for (int I = blockIdx.x * blockDim.x + threadIdx.x; I < nnode; I += gridDim.x * blockDim.x) {
    const typename NV<ND>::T rv = r[I], pv = p[I];
    float rr[ND], z[ND], pn[ND];
#pragma unroll
    for (int i = 0; i < ND; ++i) rr[i] = comp<ND>(rv, i);
    prec_apply<ND>(minv, nnode, I, rr, z);
#pragma unroll
    for (int i = 0; i < ND; ++i) pn[i] = fmaf(bt, comp<ND>(pv, i), z[i]);
    p[I] = mk<ND>(pn);
  }
}

// Inner start: x = 0, r given, p = z = Minv r, rho = r.z, ref0 = r.r
template <int ND>
__global__ void __launch_bounds__(256) k_start_b(int nnode, typename NV<ND>::T* __restrict__ x,
                                                 const typename NV<ND>::T* __restrict__ r,
                                                 typename NV<ND>::T* __restrict__ p,
                                                 const typename NV<ND>::T* __restrict__ minv, PcgState* st,
                                                 double* partials) {
  double acc[2] = {0.0, 0.0};
  for (int I = blockIdx.x * blockDim.x + threadIdx.x; I < nnode; I += gridDim.x * blockDim.x) {
    const typename NV<ND>::T rv = r[I];
    float rr[ND], z[ND], zero[ND];
#pragma unroll
    for (int i = 0; i < ND; ++i) { rr[i] = comp<ND>(rv, i); zero[i] = 0.f; }
    prec_apply<ND>(minv, nnode, I, rr, z);
    p[I] = mk<ND>(z);
    x[I] = mk<ND>(zero);
#pragma unroll
    for (int i = 0; i < ND; ++i) { acc[0] += (double)rr[i] * z[i]; acc[1] += (double)rr[i] * rr[i]; }
  }
  double out[2];
  if (reduce_last<2>(acc, partials, &st->ticket, out) && threadIdx.x == 0) {
    st->rho = out[0];
    st->rr = out[1];
    st->ref0 = out[1];
    st->xx = 0.0;
    st->iter = 0;
    st->status = kStatusOk;
    st->done = 0;
    st->last = 1.0;
    if (!(out[0] == out[0])) { st->status = kStatusBreakdown; st->done = 1; }
    else if (out[1] == 0.0) { st->done = 1; st->last = 0.0; }
  }
}

// Block-Jacobi factors: invert the node diagonal block (in FP64) and store its
// rows; jacobi_only keeps just 1/diag.  Flags non-positive diagonals.
template <int ND>
__global__ void k_minv_b(int nnode, const int* bsoff, const int* ndiag, const float* bval,
                         typename NV<ND>::T* minv, int jacobi_only, unsigned* flags) {
  constexpr int BB = ND * ND;
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
    for (int i = 0; i < ND; ++i) {
      float row[ND];
      for (int j = 0; j < ND; ++j) row[j] = (float)Di[i * ND + j];
      minv[(long long)i * nnode + I] = mk<ND>(row);
    }
  }
}

// ======================== FP64 <-> node-block glue ===========================
// r32 = (float)(r64 * scale) in node layout
template <int ND>
__global__ void k_to_node32(int nnode, const double* __restrict__ r64, double scale, typename NV<ND>::T* r32) {
  for (int I = blockIdx.x * blockDim.x + threadIdx.x; I < nnode; I += gridDim.x * blockDim.x) {
    float t[ND];
#pragma unroll
    for (int i = 0; i < ND; ++i) t[i] = (float)(r64[(long long)I * ND + i] * scale);
    r32[I] = mk<ND>(t);
  }
}

// x64 += scale * d32 (node layout)
template <int ND>
__global__ void k_axpy_from_node32(int nnode, double* __restrict__ x64, double scale,
                                   const typename NV<ND>::T* __restrict__ d32) {
  for (int I = blockIdx.x * blockDim.x + threadIdx.x; I < nnode; I += gridDim.x * blockDim.x) {
    const typename NV<ND>::T d = d32[I];
#pragma unroll
    for (int i = 0; i < ND; ++i) x64[(long long)I * ND + i] += scale * (double)comp<ND>(d, i);
  }
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
