// batch_kernels.cuh -- many independent systems in one persistent launch.
//
// One cooperative launch, one CTA per SM.  The host splits the CTAs into
// gangs for the big systems (a gang of g CTAs solves one system, g chosen in
// proportion to the system's share of the batch) and leaves the rest as
// single CTAs that pull the small systems off a device work list (largest
// first, one atomicAdd per system).  A gang's CTAs meet at a software barrier
// (one arrival counter per gang in global memory, release/acquire at GPU
// scope, a bounded wait); a single CTA only uses __syncthreads.  When its big
// system is done, a gang breaks up and its CTAs pull small systems too.
//
// For a system the group (gang or CTA) runs: FP32 assembly (colour by
// colour), block-Jacobi factors, the FP64 right-hand-side norm, and
// reliable-update mixed-precision PCG (FP32 node-block SpMV + FP64
// matrix-free residual replacement), for at most `budget` iterations per
// launch (the serving loop's preemption: the Krylov state stays in the
// system's own device memory).
//
// Every sum has one fixed order, whatever the group's size or the CTA's
// thread count: lanes of a 32-node slice are combined by a warp butterfly and
// written as that slice's partial; after the barrier every CTA adds the
// partials in slice order through 256 fixed strided accumulators and a fixed
// tree.  Element scatters are colour-exclusive, rows of the SpMV are summed in
// storage order, the rest is element-wise.  So a system's iterates are
// bit-identical whether it is solved alone, in any mix, by a gang of any size
// or by one CTA.
//
// Data that other CTAs write during the launch is never read through the
// read-only (non-coherent) cache path.
#pragma once
#include "common.cuh"
#include "elem_kernels.cuh"
#include "mf_kernels.cuh"
#include "pcg_kernels.cuh"

namespace betagpu {

enum : int { kPhaseNew = 0, kPhaseIter = 1, kPhaseDone = 2 };
enum : int { kBConverged = 0, kBRunning = 1, kBMaxit = 4, kBBreakdown = 5, kBNegDiag = 6, kBAborted = 10 };

struct BState {
  double rho, rr, maxrr, bn, rn;
  int iter, repl, phase, status;
  int mode;    // 0: FP32 inner PCG with FP64 reliable updates; 1: the same with FP64 vectors and arithmetic
  int cycle0;  // iteration at which the current FP32 replacement cycle began
  float bt;    // FP32 mode: beta of the direction update the next SpMV applies
  int pb;      // FP32 mode: which direction buffer holds the current p (0: p32, 1: p32b)
  long long busy_ns;  // device time spent on the system (its group's, summed over launches)
  long long setup_ns; // of which in the setup (assembly, factors, row sums, first residual)
  long long repl_ns;  // of which in reliable updates (FP64 matrix-free residual and restart)
  int sub;            // setup: the next step (kPhaseNew)
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
  const uint16_t* slot;  // position of node J in node I's graph row, per element node pair
  const int* nrp;
  const int* ndiag;
  const int* bsoff;
  const int* bcol;
  float* bval;
  double* x64;
  double* r64;
  double* y64;
  double* p64;  // FP64 mode: search direction
  double* q64;  // FP64 mode: K p, then M r
  double* w64;  // FP64 mode: correction since the last residual replacement
  float* y32;
  float* r32;
  float* p32;   // direction (double-buffered with p32b; padded to float4 for nd = 3)
  float* p32b;
  float* z32;   // z = M r of the last update (same padding)
  float* q32;
  float* minv;
  double* part;     // 2 buffers x 2 values x nslice slice partials
  unsigned* gflag;  // [0] assembly status bits; where a time slice ends: [1] iteration, [2] setup step
  const GaussTable* gt;
  BState* st;
  long long nchunk;
};

struct BParams {
  double tol, delta;
  int maxit, max_repl, budget;  // budget: iterations per system per launch (0: no limit)
  int nactive, nbig;            // active[0, nbig) are solved by gangs, the rest by single CTAs
  long long spin_ns;            // longest wait at a gang barrier before the launch gives up
  int switch_iters;             // FP32 cycle longer than this: continue in FP64 (0: never)
  long long slice_ns;           // time slice: systems stop after the iteration in which it ends (0: none)
  // With a time slice, the slice also ends once *preempt is non-zero (the
  // server sets it when it has admitted new work) and min_slice_ns have passed.
  int* preempt;
  long long min_slice_ns;
  // A system that finishes sets *preempt itself, so the launch ends soon and
  // its result can be collected (the server asks for this when no request
  // waits; with a backlog the slice runs out, and launches stay long).
  int end_on_done;
};

// The slice is over early: new work is waiting for the next launch.
__device__ __forceinline__ bool slice_preempted(const BParams& P, long long elapsed) {
  return P.preempt != nullptr && elapsed >= P.min_slice_ns && *(const volatile int*)P.preempt != 0;
}

// Per CTA: the gang it belongs to for this launch.
struct BPlan {
  int k;     // index into active[] of the gang's system, -1: no gang (single CTA from the start)
  int rank;  // rank of this CTA in the gang
  int size;  // CTAs in the gang
  int bar;   // index of the gang's arrival counter
};

struct GangShared {
  unsigned bar_no;
  int abort;
  int idx, skip;
  // time-slice bookkeeping of the system being solved (thread 0 only; kept
  // here rather than in registers, which the SpMV loop needs)
  long long t_in, t_mark;
  long long t_repl;  // start of the reliable update in progress (0: none)
  int stop_sent;
  double wred[2][8];
  double red[2];
};

__device__ __forceinline__ long long globaltimer_ns() {
  long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Slice partials of a CTA working alone stay in shared memory up to this
// many slices (32K nodes); bigger systems and gangs use the pool.
constexpr int kSharedSlices = 1024;

// The CTAs working on one system: a gang (ctr != nullptr) or this CTA alone.
struct Grp {
  int rank, size;
  unsigned* ctr;
  GangShared* gs;
  int* gabort;
  long long spin_ns;
  double* spart;  // shared partials (2 x kSharedSlices) for a CTA alone
  long long t0;   // %globaltimer when this CTA started
};

// Barrier of the group.  Returns false once the launch is aborting (a wait
// ran past spin_ns here or in another gang); the caller then stops.
__device__ __forceinline__ bool gsync(const Grp& g) {
  __syncthreads();
  if (g.ctr == nullptr) return true;
  if (threadIdx.x == 0) {
    const unsigned target = (++g.gs->bar_no) * (unsigned)g.size;
    // arrive: releases every write of this CTA ordered before the CTA barrier
    asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(g.ctr), "r"(1u) : "memory");
    unsigned polls = 0;
    long long t0 = 0;
    while (ld_acquire_u32(g.ctr) < target) {
      if ((++polls & 255u) == 0u) {
        if (t0 == 0) t0 = globaltimer_ns();
        if (*(volatile int*)g.gabort) { g.gs->abort = 1; break; }
        if (globaltimer_ns() - t0 > g.spin_ns) {
          g.gs->abort = 1;
          atomicExch(g.gabort, 1);
          break;
        }
      }
    }
    __threadfence();  // the other CTAs' writes are visible to every thread after the CTA barrier
  }
  __syncthreads();
  return g.gs->abort == 0;
}

// Stage 1 of a fixed-order sum: the warp that owns slice s adds its 32 lane
// values (butterfly) and lane 0 stores the slice partial.
template <int NV>
__device__ __forceinline__ void slice_partial(double* part, int nsl, int s, const double (&v)[NV]) {
#pragma unroll
  for (int k = 0; k < NV; ++k) {
    const double t = warp_sum(v[k]);
    if ((threadIdx.x & 31) == 0) part[(long long)k * nsl + s] = t;
  }
}

// Stage 2: barrier, then every CTA adds the nsl slice partials of each value
// in the same order (256 strided accumulators, warp butterflies, warps 0..7 in
// order); all threads of the group get bit-identical totals.
template <int NV>
__device__ __forceinline__ bool group_sum(const Grp& g, const double* part, int nsl, double (&out)[NV]) {
  if (!gsync(g)) return false;
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  if (t < 256) {
    double a[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) a[k] = 0.0;
    if (part == g.spart) {
      for (int i = t; i < nsl; i += 256) {
#pragma unroll
        for (int k = 0; k < NV; ++k) a[k] += part[k * nsl + i];
      }
    } else {
      // Loads of 8 strided partials are issued before they are added (in the
      // same order), so a long partial array costs a few L2 round trips, not
      // one per partial.
      int i = t;
      for (; i + 7 * 256 < nsl; i += 8 * 256) {
        double b[NV][8];
#pragma unroll
        for (int u = 0; u < 8; ++u)
#pragma unroll
          for (int k = 0; k < NV; ++k) b[k][u] = __ldcg(part + (long long)k * nsl + i + u * 256);
#pragma unroll
        for (int u = 0; u < 8; ++u)
#pragma unroll
          for (int k = 0; k < NV; ++k) a[k] += b[k][u];
      }
      for (; i < nsl; i += 256) {
#pragma unroll
        for (int k = 0; k < NV; ++k) a[k] += __ldcg(part + (long long)k * nsl + i);
      }
    }
#pragma unroll
    for (int k = 0; k < NV; ++k) {
      a[k] = warp_sum(a[k]);
      if (lane == 0) g.gs->wred[k][w] = a[k];
    }
  }
  __syncthreads();
  if (t == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) {
      double s = 0.0;
      for (int i = 0; i < 8; ++i) s += g.gs->wred[k][i];
      g.gs->red[k] = s;
    }
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < NV; ++k) out[k] = g.gs->red[k];
  return true;
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
__device__ bool b_mf(const BSys& S, const MfArgs& M, const double* x, double* y, const double* s_dN,
                     const double* s_N, const double* s_w, const Grp& g) {
  const int gt = g.rank * blockDim.x + threadIdx.x, gn = g.size * blockDim.x;
  for (int i = gt; i < S.ndof; i += gn) y[i] = 0.0;
  if (!gsync(g)) return false;
  const int nw = blockDim.x >> 5;
  const int wid = g.rank * nw + (threadIdx.x >> 5), gw = g.size * nw;
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
    if (!gsync(g)) return false;
  }
  return true;
}

// Residual b - K x on free dofs (0 on restrained ones) into r64 and r32, and
// its squared norm (fixed order); with bb also ||b||^2, b = the prescribed
// value on restrained dofs.  y64 holds K x.
template <int ND>
__device__ __forceinline__ bool b_residual(const BSys& S, const Grp& g, double* part, double (&out)[2], bool bb) {
  const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  const int wid = g.rank * nw + (threadIdx.x >> 5), gw = g.size * nw;
  for (int s = wid; s < S.nslice; s += gw) {
    double v[2] = {0.0, 0.0};
#pragma unroll
    for (int k = 0; k < ND; ++k) {
      const long long i = 32LL * ND * s + 32 * k + lane;
      if (i < S.ndof) {
        const double r = S.rest[i] ? 0.0 : (S.load ? S.load[i] : 0.0) - S.y64[i];
        S.r64[i] = r;
        S.r32[i] = (float)r;
        v[0] += r * r;
        if (bb) {
          const double b = S.rest[i] ? S.presc[i] : r;
          v[1] += b * b;
        }
      }
    }
    slice_partial<2>(part, S.nslice, s, v);
  }
  return group_sum<2>(g, part, S.nslice, out);
}

// (r.z, r.r) with z = M r, optionally storing p = z (start of a cycle).
template <int ND>
__device__ __forceinline__ bool b_rz(const BSys& S, const Grp& g, double* part, double (&out)[2], bool set_p) {
  const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  const int wid = g.rank * nw + (threadIdx.x >> 5), gw = g.size * nw;
  for (int s = wid; s < S.nslice; s += gw) {
    const int I = 32 * s + lane;
    double v[2] = {0.0, 0.0};
    if (I < S.nnode) {
      float rv[ND], z[ND];
      NodeIO<ND>::ld(S.r32, I, rv);
      NodeIO<ND>::prec(S.minv, I, rv, z);
      PVec<ND>::st(S.z32, I, z);
      if (set_p) PVec<ND>::st(S.p32, I, z);
#pragma unroll
      for (int i = 0; i < ND; ++i) { v[0] += (double)rv[i] * z[i]; v[1] += (double)rv[i] * rv[i]; }
    }
    slice_partial<2>(part, S.nslice, s, v);
  }
  return group_sum<2>(g, part, S.nslice, out);
}

// Row-sum form of the FP32 matrix.  The diagonal block of node I holds the
// block row sum S_I = sum_J A_IJ, taken from the FP64 operator, and the
// product is formed from differences:
//   (A p)_I = sum_{J != I} A_IJ (p_J - p_I) + S_I p_I.
// Rounding every stored entry to FP32 perturbs the low-frequency modes of a
// stiffness matrix by about eps32 * ||A|| unless the row sums are kept exact
// (they are zero away from the boundary: rigid translations cost no energy);
// with them kept the inner iteration count stays close to the FP64 one, and
// the differences of a smooth p carry no cancellation.  Padding entries hold
// zeros, so their column does not matter.

// ---- matrix chunks staged in shared memory --------------------------------
// A warp multiplies its slice chunk by chunk; chunk k's 32 column indices and
// 32*ND*ND values (contiguous in the sliced layout, 256-byte aligned pool
// regions) are copied into a per-warp ring of kDepth chunks with 16-byte
// cp.async.cg, kDepth-1 chunks ahead of the one being multiplied.  The copies
// in flight live in shared memory, not registers, so a warp keeps several
// chunks of HBM traffic in flight with few warps per SM (loads into registers,
// two chunks ahead, left the one-CTA-per-SM kernel at about half of HBM).
// The arithmetic and its order are unchanged by the staging.  cp.async.cg reads
// through L2, where the matrix written earlier in the launch (assembly, row
// sums) is visible after the group barrier.
constexpr int kStageFloats = 32 * (1 + 9);  // one chunk of the widest (3 dofs per node) layout

// Chunks staged per warp (measured on one B200: 512 threads, 6 against 4 stages,
// +3.5 % capacity on the serving mix; 1024 threads, 4 against 3 stages, 7 %
// slower on 64 RVEs, the shared memory of the deeper ring costing more than
// the copies in flight gain).
template <int T>
__host__ __device__ constexpr int stage_depth() { return T >= 1024 ? 3 : (T >= 512 ? 6 : 8); }

template <int T>
__host__ __device__ constexpr size_t stage_bytes() {
  return (size_t)(T / 32) * stage_depth<T>() * kStageFloats * sizeof(float);
}

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// Chunk (cols: 32 ints, vals: 32*ND*ND floats) into dst: cols first, then vals.
template <int ND>
__device__ __forceinline__ void stage_chunk(float* dst, const int* cols, const float* vals, int lane) {
  constexpr int kPieces = 8 + 8 * ND * ND;  // 16-byte pieces
  for (int q = lane; q < kPieces; q += 32) {
    const void* src = q < 8 ? (const void*)(cols + 4 * q) : (const void*)(vals + 4 * (q - 8));
    cp_async16(dst + 4 * q, src);
  }
}

// One 32-node slice of q = A p in FP32.  FUSED: the direction update is
// folded into the gather, p_new[J] = fmaf(bt, p_old[J], z[J]) for every
// column J -- the same arithmetic, and so the same bits, as updating p in a
// separate pass; pI receives p_new of the lane's own node.  Otherwise p was
// written before the pass and pI receives p[I].  RS: the matrix is in
// row-sum form (else the plain assembled one).  ring: this warp's
// kDepth * kStageFloats floats.
template <int ND, bool RS, bool FUSED, int D>
__device__ __forceinline__ void spmv_row_staged(const BlockMat& A, int s, int lane, const float* p, const float* z,
                                                float bt, float* acc, float* pI, float* ring) {
  constexpr int BB = ND * ND;
  const int I = 32 * s + lane;
  const int c0 = A.bsoff[s], w = A.bsoff[s + 1] - c0;
  const int* cb = A.bcol + (long long)c0 * 32;
  const float* vb = A.bval + (long long)c0 * 32 * BB;
#pragma unroll
  for (int i = 0; i < ND; ++i) { acc[i] = 0.f; pI[i] = 0.f; }
  if (I < A.nnode) {
    if constexpr (FUSED) {
      float po[ND], zv[ND];
      PVec<ND>::ld(p, I, po);
      PVec<ND>::ld(z, I, zv);
#pragma unroll
      for (int i = 0; i < ND; ++i) pI[i] = fmaf(bt, po[i], zv[i]);
    } else {
      PVec<ND>::ld(p, I, pI);
    }
  }
#pragma unroll
  for (int k = 0; k < D - 1; ++k) {
    if (k < w) stage_chunk<ND>(ring + k * kStageFloats, cb + k * 32, vb + (long long)k * 32 * BB, lane);
    cp_async_commit();  // empty groups keep the count uniform
  }
  for (int k = 0; k < w; ++k) {
    const int kn = k + D - 1;
    if (kn < w) stage_chunk<ND>(ring + (kn % D) * kStageFloats, cb + kn * 32, vb + (long long)kn * 32 * BB, lane);
    cp_async_commit();
    cp_async_wait<D - 1>();  // chunk k's copies of this lane have landed
    __syncwarp();            // ... and every lane's
    const float* st = ring + (k % D) * kStageFloats;
    const int J = reinterpret_cast<const int*>(st)[lane];
    float v[BB];
#pragma unroll
    for (int t = 0; t < BB; ++t) v[t] = st[32 + t * 32 + lane];
    float d[ND];
    if constexpr (FUSED) {
      float po[ND], zv[ND];
      PVec<ND>::ld(p, J, po);
      PVec<ND>::ld(z, J, zv);
#pragma unroll
      for (int j = 0; j < ND; ++j) {
        const float pj = fmaf(bt, po[j], zv[j]);
        if constexpr (RS) d[j] = J == I ? pI[j] : pj - pI[j];
        else d[j] = pj;
      }
    } else {
      float pj[ND];
      PVec<ND>::ld(p, J, pj);
#pragma unroll
      for (int j = 0; j < ND; ++j) d[j] = J == I ? pI[j] : pj[j] - pI[j];
    }
#pragma unroll
    for (int i = 0; i < ND; ++i)
#pragma unroll
      for (int j = 0; j < ND; ++j) acc[i] = fmaf(v[i * ND + j], d[j], acc[i]);
    __syncwarp();  // every lane has read this stage before it is refilled
  }
  cp_async_wait<0>();  // only empty groups can remain; none is left pending
}

// One 32-node slice of q = A p with FP64 vectors and arithmetic on the FP32
// row-sum matrix (p64 node-interleaved).
template <int ND>
__device__ __forceinline__ void spmv_row_rs64(const BlockMat& A, int s, int lane, const double* p, double* acc,
                                              double* pI) {
  constexpr int BB = ND * ND;
  const int I = 32 * s + lane;
  const int c0 = A.bsoff[s], w = A.bsoff[s + 1] - c0;
  const int* cp = A.bcol + (long long)c0 * 32 + lane;
  const float* vp = A.bval + (long long)c0 * 32 * BB + lane;
#pragma unroll
  for (int i = 0; i < ND; ++i) { acc[i] = 0.0; pI[i] = 0.0; }
  if (I < A.nnode)
#pragma unroll
    for (int i = 0; i < ND; ++i) pI[i] = p[(long long)I * ND + i];
#pragma unroll 1
  for (int k = 0; k < w; ++k) {
    const int J = __ldcs(cp + k * 32);
    double pj[ND];
    if constexpr (ND == 2) {
      const double2 t = reinterpret_cast<const double2*>(p)[J];
      pj[0] = t.x; pj[1] = t.y;
    } else {
#pragma unroll
      for (int j = 0; j < ND; ++j) pj[j] = p[(long long)J * ND + j];
    }
    float v[BB];
#pragma unroll
    for (int t = 0; t < BB; ++t) v[t] = __ldcs(vp + (long long)k * 32 * BB + t * 32);
    double d[ND];
#pragma unroll
    for (int j = 0; j < ND; ++j) d[j] = J == I ? pI[j] : pj[j] - pI[j];
#pragma unroll
    for (int i = 0; i < ND; ++i)
#pragma unroll
      for (int j = 0; j < ND; ++j) acc[i] = fma((double)v[i * ND + j], d[j], acc[i]);
  }
}

// z = M r for one node in FP64 arithmetic (packed symmetric FP32 factor).
template <int ND>
__device__ __forceinline__ void prec64(const float* m, long long I, const double* r, double* z) {
  constexpr int S = ND * (ND + 1) / 2;
  double a[S];
#pragma unroll
  for (int t = 0; t < S; ++t) a[t] = (double)m[S * I + t];
  if constexpr (ND == 1) {
    z[0] = a[0] * r[0];
  } else if constexpr (ND == 2) {
    z[0] = a[0] * r[0] + a[1] * r[1];
    z[1] = a[1] * r[0] + a[2] * r[1];
  } else {
    z[0] = a[0] * r[0] + a[1] * r[1] + a[2] * r[2];
    z[1] = a[1] * r[0] + a[3] * r[1] + a[4] * r[2];
    z[2] = a[2] * r[0] + a[4] * r[1] + a[5] * r[2];
  }
}

// FP64 mode: zdst = z = M r64 (p64 to start a Krylov cycle, q64 for a
// reliable update), returns (r.z, r.r).
template <int ND>
__device__ __forceinline__ bool b_rz64(const BSys& S, const Grp& g, double* part, double (&out)[2], double* zdst) {
  const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  const int wid = g.rank * nw + (threadIdx.x >> 5), gw = g.size * nw;
  for (int s = wid; s < S.nslice; s += gw) {
    const int I = 32 * s + lane;
    double v[2] = {0.0, 0.0};
    if (I < S.nnode) {
      double rv[ND], z[ND];
#pragma unroll
      for (int i = 0; i < ND; ++i) rv[i] = S.r64[(long long)I * ND + i];
      prec64<ND>(S.minv, I, rv, z);
#pragma unroll
      for (int i = 0; i < ND; ++i) {
        zdst[(long long)I * ND + i] = z[i];
        v[0] += rv[i] * z[i];
        v[1] += rv[i] * rv[i];
      }
    }
    slice_partial<2>(part, S.nslice, s, v);
  }
  return group_sum<2>(g, part, S.nslice, out);
}

template <int ND, int SD>
__device__ void b_solve(const BSys& S, const BParams& P, const Grp& g, const double* s_dN, const double* s_N,
                        const double* s_w, const float* s_dNf, const float* s_Nf, const float* s_wf, float* s_ring) {
  float* const ring = s_ring + (threadIdx.x >> 5) * SD * kStageFloats;
  constexpr int SM = ND * (ND + 1) / 2;
  const int tid = g.rank * blockDim.x + threadIdx.x, nt = g.size * blockDim.x;
  const int lane = threadIdx.x & 31, nwc = blockDim.x >> 5;
  const int wid = g.rank * nwc + (threadIdx.x >> 5), nw = g.size * nwc;
  const int nsl = S.nslice;
  double* const partA = S.part;
  double* const partB = S.part + 2LL * nsl;
  // Partial buffers alternate: a buffer is rewritten only after the next
  // sum's barrier, by which time every CTA has read it.  A CTA alone reads
  // its partials back before the sum's last __syncthreads, so one shared
  // buffer serves it.
  const bool in_smem = g.ctr == nullptr && nsl <= kSharedSlices;
  int pb = 0;
  auto part = [&]() {
    pb ^= 1;
    return in_smem ? g.spart : (pb ? partA : partB);
  };
  BState st = *S.st;
  MfArgs M;
  M.xyz = S.xyz; M.conn = S.conn; M.gparams = S.gparams; M.egroup = S.egroup; M.nparams = S.nparams;
  M.nip = S.nip; M.gt = S.gt; M.c1 = 1.0; M.c2 = 0.0; M.cm = 0.0;
  const int n = S.ndof, nn = S.nnode;
  BlockMat A{S.nnode, S.nslice, S.bsoff, S.bcol, S.bval};
  auto aborted = [&]() {
    if (tid == 0) { st.status = kBAborted; *S.st = st; }
  };
  // Time slice.  Thread 0 of rank 0 decides once, before the barrier of an
  // iteration's second sum, that the group stops after that iteration and
  // publishes the iteration number; every CTA reads it after that barrier, so
  // all CTAs of a gang stop after the same iteration.  A CTA that reads it one
  // iteration early sees a number it has not reached yet and goes on.  The
  // group stops as soon as one more iteration, as long as the last one, would
  // end past the slice, so a slow group does not hold the whole launch.
  volatile unsigned* const stop_at = S.gflag + 1;
  if (threadIdx.x == 0) {
    g.gs->t_in = g.gs->t_mark = globaltimer_ns();
    g.gs->stop_sent = 0;
  }
  if (tid == 0) *stop_at = 0xFFFFFFFFu;
  bool slice_end = false;
  auto mark_slice = [&]() {
    if (P.slice_ns > 0 && tid == 0 && !g.gs->stop_sent) {
      const long long now = globaltimer_ns();
      const long long t_step = now - g.gs->t_mark;
      g.gs->t_mark = now;
      if (now + t_step - g.t0 >= P.slice_ns || slice_preempted(P, now - g.t0)) {
        *stop_at = (unsigned)(st.iter + 1);
        g.gs->stop_sent = 1;
      }
    }
  };

  // The FP32 inner solve runs on the row-sum form for elasticity: on quad4
  // it costs nothing per iteration and saves iterations on long plates, on
  // hex8 it costs ~16 % per iteration and saves 8 % of the iterations of the
  // 512-RVE batch (2.03 s -> 1.84 s per step).  For diffusion (1 dof per
  // node) the differences cost ~27 % per iteration, so the plain assembled
  // matrix is kept until a switch to FP64 vectors, which converts it (FP64
  // arithmetic needs the row sums).
  constexpr bool kRowSum0 = ND != 1;
  // Row-sum form, column j: column j of every diagonal block becomes (K t_j)
  // on the free rows, t_j = 1 on the free dofs of component j (restrained
  // columns are eliminated), and the unit row on restrained rows.  t is
  // scratch for t_j; y64 receives K t_j.
  auto row_sum_column = [&](int j, double* t) -> bool {
    for (int i = tid; i < n; i += nt) t[i] = (i % ND == j && !S.rest[i]) ? 1.0 : 0.0;
    if (!gsync(g)) return false;
    if (!b_mf(S, M, t, S.y64, s_dN, s_N, s_w, g)) return false;
    for (int I = tid; I < nn; I += nt) {
      const long long chunk = (long long)S.bsoff[I >> 5] + S.ndiag[I];
      for (int c = 0; c < ND; ++c) {
        const long long d = (long long)I * ND + c;
        S.bval[chunk * (32 * ND * ND) + (c * ND + j) * 32 + (I & 31)] =
            S.rest[d] ? (c == j ? 1.f : 0.f) : (float)S.y64[d];
      }
    }
    return true;
  };
  if (st.phase == kPhaseNew) {
    // Setup in steps that each end at a group barrier: zero the matrix, one
    // step per element colour (FP32 assembly), unit restrained diagonals and
    // the block-Jacobi factors, one step per column of the row sums
    // (elasticity), and the start of the solve.  Under a time slice a group stops between steps,
    // decided as for iterations, so a long setup spreads over launches
    // instead of holding one.
    volatile unsigned* const stop_step = S.gflag + 2;
    if (tid == 0) *stop_step = 0xFFFFFFFFu;
    ElemArgs E;
    E.xyz = S.xyz; E.conn = S.conn; E.gparams = S.gparams; E.egroup = S.egroup; E.nparams = S.nparams;
    E.nip = S.nip; E.gt = S.gt; E.slot = S.slot; E.nrp = S.nrp; E.rest = S.rest; E.presc = S.presc;
    E.bsoff = S.bsoff; E.vpos = nullptr; E.bval = S.bval; E.soff = nullptr; E.ssoff = nullptr; E.sval = nullptr; E.pseudo = nullptr;
    E.kscale = 1.0; E.mscale = 0.0; E.flags = S.gflag;
    while (st.phase == kPhaseNew) {
      const int k = st.sub;
      if (k == 0) {
        const long long nv = S.nchunk * 32LL * ND * ND;
        for (long long i = tid; i < nv; i += nt) S.bval[i] = 0.f;
        if (tid == 0) *S.gflag = 0u;
      } else if (k <= S.ncolor) {
        const int c = k - 1;
        const int beg = S.color_ptr[c], nel = S.color_ptr[c + 1] - beg;
        const int* el = S.elems + beg;
        if (S.kind == 2) {
          for (int w = wid; w < nel; w += nw) asm_hex8_elastic_warp<float>(E, el, nel, w, s_dNf, s_Nf, s_wf);
        } else if (S.kind == 3) {
          for (int w = wid; w < nel; w += nw) asm_hex8_heat_warp<float>(E, el, nel, w, s_dNf, s_Nf, s_wf);
        } else {
          for (int w = wid; 2 * w < nel; w += nw) asm_quad4_pstress_warp<float>(E, el, nel, w, s_dNf, s_Nf, s_wf);
        }
      } else if (k == S.ncolor + 1) {
        for (int I = tid; I < nn; I += nt) {
          const long long chunk = (long long)S.bsoff[I >> 5] + S.ndiag[I];
          for (int i = 0; i < ND; ++i)
            if (S.rest[I * ND + i]) S.bval[chunk * (32 * ND * ND) + (i * ND + i) * 32 + (I & 31)] = 1.0f;
        }
        if (!gsync(g)) return aborted();
        if (ld_acquire_u32(S.gflag) & kFlagNegDiag) {
          if (tid == 0) {
            st.phase = kPhaseDone;
            st.status = kBNegDiag;
            st.busy_ns += globaltimer_ns() - g.gs->t_in;
            *S.st = st;
          }
          gsync(g);
          return;
        }
        // block-Jacobi factors (FP64 inverse of the node diagonal block)
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
            for (int j = i; j < ND; ++j)
              S.minv[(long long)SM * I + (t++)] = (float)(0.5 * (Di[i * ND + j] + Di[j * ND + i]));
        }
      } else if (k <= S.ncolor + 1 + ND) {
        if (!row_sum_column(k - S.ncolor - 2, S.x64)) return aborted();
      } else {
        // x = prescribed on restrained dofs, 0 elsewhere; r = b = load - K x (free rows)
        for (int i = tid; i < n; i += nt) {
          S.x64[i] = S.rest[i] ? S.presc[i] : 0.0;
          S.w64[i] = 0.0;
          S.y32[i] = 0.f;
        }
        if (!gsync(g)) return aborted();
        if (!b_mf(S, M, S.x64, S.y64, s_dN, s_N, s_w, g)) return aborted();
        double a0[2];
        if (!b_residual<ND>(S, g, part(), a0, true)) return aborted();
        st.bn = sqrt(a0[1]);
        double a2[2];
        if (!b_rz<ND>(S, g, part(), a2, true)) return aborted();
        st.rho = a2[0];
        st.rr = st.maxrr = a2[1];
        st.iter = 0;
        st.repl = 0;
        st.mode = 0;
        st.cycle0 = 0;
        st.bt = 0.f;  // p32 = z32 = M r: the first fused update gives p = z exactly
        st.pb = 0;
        st.phase = kPhaseIter;
        st.status = kBRunning;
        st.rn = sqrt(a2[1]);
        if (a2[1] == 0.0 || st.rn <= P.tol * st.bn) { st.phase = kPhaseDone; st.status = kBConverged; }
        break;
      }
      if (P.slice_ns > 0 && tid == 0 && !g.gs->stop_sent &&
          (globaltimer_ns() - g.t0 >= P.slice_ns || slice_preempted(P, globaltimer_ns() - g.t0))) {
        *stop_step = (unsigned)k;
        g.gs->stop_sent = 1;
      }
      if (!gsync(g)) return aborted();
      st.sub = (k == S.ncolor + 1 && !kRowSum0) ? S.ncolor + 2 + ND : k + 1;
      if ((unsigned)k >= *stop_step) {
        slice_end = true;
        break;
      }
    }
    if (tid == 0) st.setup_ns += globaltimer_ns() - g.gs->t_in;
  }

  const double tolabs2 = (0.5 * P.tol * st.bn) * (0.5 * P.tol * st.bn);
  const double delta2 = P.delta * P.delta;
  int spent = 0;
  if (threadIdx.x == 0) g.gs->t_repl = 0;
  while (st.phase == kPhaseIter && (P.budget <= 0 || spent < P.budget) && !slice_end) {
    if (tid == 0 && g.gs->t_repl) {
      st.repl_ns += globaltimer_ns() - g.gs->t_repl;
      g.gs->t_repl = 0;
    }
    if (st.mode == 1) {
      // ---- FP64 vectors and arithmetic on the FP32 row-sum matrix, with the
      // same reliable updates (restrained dofs stay fixed)
      double* pq = part();
      for (int s = wid; s < nsl; s += nw) {
        double acc[ND], pI[ND];
        spmv_row_rs64<ND>(A, s, lane, S.p64, acc, pI);
        const int I = 32 * s + lane;
        double v[1] = {0.0};
        if (I < nn) {
#pragma unroll
          for (int i = 0; i < ND; ++i) {
            const long long d = (long long)I * ND + i;
            S.q64[d] = acc[i];
            if (!S.rest[d]) v[0] += pI[i] * acc[i];
          }
        }
        slice_partial<1>(pq, nsl, s, v);
      }
      double a1[1];
      if (!group_sum<1>(g, pq, nsl, a1)) return aborted();
      if (!(a1[0] > 0.0 && a1[0] < 1e308)) { st.phase = kPhaseDone; st.status = kBBreakdown; break; }
      const double alpha = st.rho / a1[0];
      double* rz = part();
      for (int s = wid; s < nsl; s += nw) {
        const int I = 32 * s + lane;
        double v[2] = {0.0, 0.0};
        if (I < nn) {
          double rv[ND], z[ND];
#pragma unroll
          for (int i = 0; i < ND; ++i) {
            const long long d = (long long)I * ND + i;
            S.w64[d] += alpha * S.p64[d];
            rv[i] = S.rest[d] ? 0.0 : S.r64[d] - alpha * S.q64[d];
            S.r64[d] = rv[i];
          }
          prec64<ND>(S.minv, I, rv, z);
#pragma unroll
          for (int i = 0; i < ND; ++i) {
            S.q64[(long long)I * ND + i] = z[i];
            v[0] += rv[i] * z[i];
            v[1] += rv[i] * rv[i];
          }
        }
        slice_partial<2>(rz, nsl, s, v);
      }
      double a2[2];
      mark_slice();
      if (!group_sum<2>(g, rz, nsl, a2)) return aborted();
      st.iter += 1;
      ++spent;
      slice_end = (unsigned)st.iter >= *stop_at;
      if (!(a2[0] == a2[0])) { st.phase = kPhaseDone; st.status = kBBreakdown; break; }
      if (a2[1] > st.maxrr) st.maxrr = a2[1];
      double beta;
      if (a2[1] < tolabs2 || a2[1] < delta2 * st.maxrr || st.iter >= P.maxit) {
        if (tid == 0) g.gs->t_repl = globaltimer_ns();
        // reliable update: fold the correction into x (x changes only here,
        // so its rounding does not pile up over the iterations), r64 = the
        // FP64 matrix-free true residual
        for (int i = tid; i < n; i += nt) { S.x64[i] += S.w64[i]; S.w64[i] = 0.0; }
        if (!gsync(g)) return aborted();
        if (!b_mf(S, M, S.x64, S.y64, s_dN, s_N, s_w, g)) return aborted();
        double a3[2];
        if (!b_residual<ND>(S, g, part(), a3, false)) return aborted();
        st.rn = sqrt(a3[0]);
        st.repl += 1;
        if (!(st.rn == st.rn)) { st.phase = kPhaseDone; st.status = kBBreakdown; break; }
        if (st.rn <= P.tol * st.bn) { st.phase = kPhaseDone; st.status = kBConverged; break; }
        if (st.iter >= P.maxit || st.repl > P.max_repl) { st.phase = kPhaseDone; st.status = kBMaxit; break; }
        double a4[2];
        if (!b_rz64<ND>(S, g, part(), a4, S.q64)) return aborted();
        beta = st.rho != 0.0 ? a4[0] / st.rho : 0.0;
        st.rho = a4[0];
        st.rr = st.maxrr = a4[1];
      } else {
        beta = a2[0] / st.rho;
        st.rho = a2[0];
        st.rr = a2[1];
      }
      for (int I = tid; I < nn; I += nt) {
#pragma unroll
        for (int i = 0; i < ND; ++i) {
          const long long d = (long long)I * ND + i;
          S.p64[d] = S.q64[d] + beta * S.p64[d];
        }
      }
      if (!gsync(g)) return aborted();
      continue;
    }
    // p_new = z + bt p_old, q = A p_new, p_new.q (one warp per 32-node
    // slice).  With 1-2 dofs per node the update is formed inside the SpMV's
    // gather (the warp keeps p_new of its own rows), saving a pass and a group
    // barrier; with 3 dofs per node (27 columns per row) the doubled gather
    // costs more than that, so p_new is written in a pass of its own.  Both
    // give the same bits.
    constexpr bool kFused = ND < 3;
    float* pold = st.pb ? S.p32b : S.p32;
    float* pnew = st.pb ? S.p32 : S.p32b;
    const float bt0 = st.bt;
    if constexpr (!kFused) {
      for (int I = tid; I < nn; I += nt) {
        float po[ND], zv[ND], pv[ND];
        PVec<ND>::ld(pold, I, po);
        PVec<ND>::ld(S.z32, I, zv);
#pragma unroll
        for (int i = 0; i < ND; ++i) pv[i] = fmaf(bt0, po[i], zv[i]);
        PVec<ND>::st(pnew, I, pv);
      }
      if (!gsync(g)) return aborted();
    }
    double* pq = part();
    for (int s = wid; s < nsl; s += nw) {
      float acc[ND], pv[ND];
      if constexpr (kFused) {
        spmv_row_staged<ND, kRowSum0, true, SD>(A, s, lane, pold, S.z32, bt0, acc, pv, ring);
      } else {
        spmv_row_staged<ND, true, false, SD>(A, s, lane, pnew, nullptr, 0.f, acc, pv, ring);
      }
      const int I = s * 32 + lane;
      double v[1] = {0.0};
      if (I < nn) {
        NodeIO<ND>::st(S.q32, I, acc);
        if constexpr (kFused) PVec<ND>::st(pnew, I, pv);
        float t = 0.f;
#pragma unroll
        for (int i = 0; i < ND; ++i) t = fmaf(pv[i], acc[i], t);
        v[0] = (double)t;
      }
      slice_partial<1>(pq, nsl, s, v);
    }
    double a1[1];
    if (!group_sum<1>(g, pq, nsl, a1)) return aborted();
    st.pb ^= 1;  // p_new is the current direction from here on
    if (!(a1[0] > 0.0 && a1[0] < 1e308)) { st.phase = kPhaseDone; st.status = kBBreakdown; break; }
    const float alpha = (float)(st.rho / a1[0]);
    // y += alpha p, r -= alpha q, z = M r (kept for the next gather), (r.z, r.r)
    double* rz = part();
    for (int s = wid; s < nsl; s += nw) {
      const int I = 32 * s + lane;
      double v[2] = {0.0, 0.0};
      if (I < nn) {
        float yv[ND], rv[ND], pv[ND], qv[ND], z[ND];
        NodeIO<ND>::ld(S.y32, I, yv);
        NodeIO<ND>::ld(S.r32, I, rv);
        PVec<ND>::ld(pnew, I, pv);
        NodeIO<ND>::ld(S.q32, I, qv);
#pragma unroll
        for (int i = 0; i < ND; ++i) {
          yv[i] = fmaf(alpha, pv[i], yv[i]);
          rv[i] = fmaf(-alpha, qv[i], rv[i]);
        }
        NodeIO<ND>::st(S.y32, I, yv);
        NodeIO<ND>::st(S.r32, I, rv);
        NodeIO<ND>::prec(S.minv, I, rv, z);
        PVec<ND>::st(S.z32, I, z);
#pragma unroll
        for (int i = 0; i < ND; ++i) { v[0] += (double)rv[i] * z[i]; v[1] += (double)rv[i] * rv[i]; }
      }
      slice_partial<2>(rz, nsl, s, v);
    }
    double a2[2];
    mark_slice();
    if (!group_sum<2>(g, rz, nsl, a2)) return aborted();
    st.iter += 1;
    ++spent;
    slice_end = (unsigned)st.iter >= *stop_at;
    if (!(a2[0] == a2[0])) { st.phase = kPhaseDone; st.status = kBBreakdown; break; }
    double beta;
    if (a2[1] > st.maxrr) st.maxrr = a2[1];
    const bool long_cycle = P.switch_iters > 0 && st.iter - st.cycle0 >= P.switch_iters;
    if (a2[1] < tolabs2 || a2[1] < delta2 * st.maxrr || st.iter >= P.maxit || long_cycle) {
      if (tid == 0) g.gs->t_repl = globaltimer_ns();
      // reliable update: fold y into x, replace r by the FP64 true residual
      for (int i = tid; i < n; i += nt) { S.x64[i] += (double)S.y32[i]; S.y32[i] = 0.f; }
      if (!gsync(g)) return aborted();
      if (!b_mf(S, M, S.x64, S.y64, s_dN, s_N, s_w, g)) return aborted();
      double a3[2];
      if (!b_residual<ND>(S, g, part(), a3, false)) return aborted();
      st.rn = sqrt(a3[0]);
      st.repl += 1;
      if (!(st.rn == st.rn)) { st.phase = kPhaseDone; st.status = kBBreakdown; break; }
      if (st.rn <= P.tol * st.bn) { st.phase = kPhaseDone; st.status = kBConverged; break; }
      if (st.iter >= P.maxit || st.repl > P.max_repl) { st.phase = kPhaseDone; st.status = kBMaxit; break; }
      if (long_cycle) {
        // the FP32 recurrences have lost their rate: continue with FP64
        // vectors from x64, r64, on the row-sum form of the matrix (q64 is
        // free here and serves as scratch)
        if constexpr (!kRowSum0) {
          for (int j = 0; j < ND; ++j)
            if (!row_sum_column(j, S.q64)) return aborted();
          if (!gsync(g)) return aborted();
        }
        st.mode = 1;
        double a4[2];
        if (!b_rz64<ND>(S, g, part(), a4, S.p64)) return aborted();
        st.rho = a4[0];
        st.rr = st.maxrr = a4[1];
        continue;
      }
      st.cycle0 = st.iter;
      double a4[2];
      if (!b_rz<ND>(S, g, part(), a4, false)) return aborted();  // z32 = M r of the new r
      beta = st.rho != 0.0 ? a4[0] / st.rho : 0.0;
      st.rho = a4[0];
      st.rr = st.maxrr = a4[1];
    } else {
      beta = a2[0] / st.rho;
      st.rho = a2[0];
      st.rr = a2[1];
    }
    st.bt = (float)beta;  // applied by the next SpMV's gather
  }
  if (tid == 0) {
    if (g.gs->t_repl) st.repl_ns += globaltimer_ns() - g.gs->t_repl;
    st.busy_ns += globaltimer_ns() - g.gs->t_in;
    *S.st = st;
    if (P.end_on_done && st.phase == kPhaseDone && P.preempt) *(volatile int*)P.preempt = 1;
  }
  gsync(g);
}

// The persistent batch kernel (cooperative launch: all CTAs resident).  CTAs
// of a gang first solve their big system together; then every CTA pulls
// small systems active[nbig..nactive) off the work counter on its own.  With
// a time slice, every system stops after the iteration in which the slice
// ends, and no CTA takes a new system after it; the host puts the systems a
// launch did not reach first in the next one.
template <int THREADS>
__global__ void __launch_bounds__(THREADS, 1) k_batch_solve(const BSys* __restrict__ sys, const int* __restrict__ active,
                                                            const BPlan* __restrict__ plan, unsigned* bar, int* counter,
                                                            int* gabort, const BParams* __restrict__ prm) {
  __shared__ GangShared gs;
  __shared__ double s_part[2 * kSharedSlices];
  __shared__ double s_dN[kMaxIP * 24], s_N[kMaxIP * 8], s_w[kMaxIP];
  __shared__ float s_dNf[kMaxIP * 24], s_Nf[kMaxIP * 8], s_wf[kMaxIP];
  __shared__ long long s_t0;
  extern __shared__ __align__(16) float s_ring[];  // stage_bytes<THREADS>() of matrix staging
  const BParams P = *prm;
  const BPlan pl = plan[blockIdx.x];
  if (threadIdx.x == 0) {
    gs.bar_no = 0;
    gs.abort = 0;
    s_t0 = globaltimer_ns();
  }
  __syncthreads();
  const long long t0 = s_t0;
  auto solve = [&](const BSys& S, const Grp& g) {
    const int nn = S.kind == 1 ? 4 : 8, ndir = S.kind == 1 ? 2 : 3;
    b_stage<double>(S.gt, S.nip, nn, ndir, s_dN, s_N, s_w);
    b_stage<float>(S.gt, S.nip, nn, ndir, s_dNf, s_Nf, s_wf);
    __syncthreads();
    constexpr int D = stage_depth<THREADS>();
    if (S.ndpn == 3) b_solve<3, D>(S, P, g, s_dN, s_N, s_w, s_dNf, s_Nf, s_wf, s_ring);
    else if (S.ndpn == 2) b_solve<2, D>(S, P, g, s_dN, s_N, s_w, s_dNf, s_Nf, s_wf, s_ring);
    else b_solve<1, D>(S, P, g, s_dN, s_N, s_w, s_dNf, s_Nf, s_wf, s_ring);
  };
  if (pl.k >= 0 && pl.k < P.nbig) {
    const Grp gang{pl.rank, pl.size, bar + pl.bar, &gs, gabort, P.spin_ns, nullptr, t0};
    solve(sys[active[pl.k]], gang);
    if (gs.abort) return;
  }
  const Grp alone{0, 1, nullptr, &gs, gabort, P.spin_ns, s_part, t0};
  for (;;) {
    if (threadIdx.x == 0) {
      // past the time slice no CTA starts another system, and an assembly,
      // which is not cut short, starts only in the first half of it
      const long long el = globaltimer_ns() - t0;
      const bool over = P.slice_ns > 0 && (el >= P.slice_ns || slice_preempted(P, el));
      const int k = (*(volatile int*)gabort || over) ? P.nactive : P.nbig + atomicAdd(counter, 1);
      gs.skip = k < P.nactive && P.slice_ns > 0 && 2 * el > P.slice_ns && sys[active[k]].st->phase == kPhaseNew;
      gs.idx = k;
    }
    __syncthreads();
    const int k = gs.idx;
    const bool skip = gs.skip != 0;
    __syncthreads();  // gs.idx is rewritten only after every thread has read it
    if (k >= P.nactive) return;
    if (skip) continue;
    solve(sys[active[k]], alone);
  }
}

}  // namespace betagpu
