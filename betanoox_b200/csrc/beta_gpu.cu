// beta_gpu.cu -- C ABI of the B200 assembly + PCG path (see include/beta_gpu.h).
#include "../../include/beta_gpu.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstddef>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <tuple>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "common.cuh"
#include "elem_kernels.cuh"
#include "mf_kernels.cuh"
#include "pattern.hpp"
#include "pcg_kernels.cuh"
#include "batch_kernels.cuh"
#include "post_kernels.cuh"

using namespace betagpu;

namespace {

template <typename T>
struct DBuf {
  T* p = nullptr;
  size_t n = 0;
  DBuf() = default;
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
  ~DBuf() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  cudaError_t alloc(size_t count) {
    if (count == n && p) return cudaSuccess;
    release();
    if (count == 0) return cudaSuccess;
    cudaError_t e = cudaMalloc(&p, count * sizeof(T));
    if (e == cudaSuccess) n = count;
    else p = nullptr;
    return e;
  }
};

// Gauss-Legendre nodes and weights on [-1,1] by Newton iteration on the
// three-term Legendre recurrence (the published Golub/Numerical-Recipes
// construction BETA also uses in gauss.cpp:14-60).
void gauss_legendre(int k, double* x, double* w) {
  for (int i = 0; i < (k + 1) / 2; ++i) {
    double z = std::cos(M_PI * (i + 0.75) / (k + 0.5)), dp = 1.0;
    for (int it = 0; it < 100; ++it) {
      double p0 = 1.0, p1 = 0.0;
      for (int j = 0; j < k; ++j) {
        double p2 = p1;
        p1 = p0;
        p0 = ((2.0 * j + 1.0) * z * p1 - j * p2) / (j + 1.0);
      }
      dp = k * (z * p0 - p1) / (z * z - 1.0);
      double dz = p0 / dp;
      z -= dz;
      if (std::fabs(dz) <= 3e-15) break;
    }
    x[i] = -z;
    x[k - 1 - i] = z;
    w[i] = w[k - 1 - i] = 2.0 / ((1.0 - z * z) * dp * dp);
  }
}

// BETA local node order (BasicElement.cpp:464-467, 518-525).
const int kHex[8][3] = {{-1, -1, -1}, {-1, 1, -1}, {-1, 1, 1}, {-1, -1, 1},
                        {1, -1, -1},  {1, 1, -1},  {1, 1, 1},  {1, -1, 1}};
const int kQuad[4][2] = {{-1, -1}, {1, -1}, {1, 1}, {-1, 1}};

void make_gauss_table(int ndim, int order, GaussTable& gt) {
  std::memset(&gt, 0, sizeof(gt));
  double g[8], gw[8];
  gauss_legendre(order, g, gw);
  int ip = 0;
  if (ndim == 3) {
    for (int i = 0; i < order; ++i)
      for (int j = 0; j < order; ++j)
        for (int k = 0; k < order; ++k, ++ip) {
          double xi = g[i], et = g[j], ze = g[k];
          gt.w[ip] = gw[i] * gw[j] * gw[k];
          for (int a = 0; a < 8; ++a) {
            double fx = 1 + kHex[a][0] * xi, fy = 1 + kHex[a][1] * et, fz = 1 + kHex[a][2] * ze;
            gt.N[ip][a] = fx * fy * fz / 8;
            gt.dN[ip][0][a] = kHex[a][0] * fy * fz / 8;
            gt.dN[ip][1][a] = kHex[a][1] * fx * fz / 8;
            gt.dN[ip][2][a] = kHex[a][2] * fx * fy / 8;
          }
        }
  } else {
    for (int i = 0; i < order; ++i)
      for (int k = 0; k < order; ++k, ++ip) {
        double xi = g[i], et = g[k];
        gt.w[ip] = gw[i] * gw[k];
        for (int a = 0; a < 4; ++a) {
          double fx = 1 + kQuad[a][0] * xi, fy = 1 + kQuad[a][1] * et;
          gt.N[ip][a] = fx * fy / 4;
          gt.dN[ip][0][a] = kQuad[a][0] * fy / 4;
          gt.dN[ip][1][a] = kQuad[a][1] * fx / 4;
        }
      }
  }
  gt.nip = ip;
}

}  // namespace

struct beta_gpu_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t own_stream = nullptr;
  long long n_launch = 0, n_h2d = 0, n_d2h = 0;
  int nsm = 148;
  std::string err;

  // mesh
  int kind = 0, ndim = 0, nnode = 0, nelem = 0, nnpe = 0, ndpn = 0, ndof = 0, order = 0;
  std::vector<int> h_conn, h_first_dof;
  DBuf<double> xyz;
  DBuf<int> conn;
  GaussTable h_gt;
  DBuf<GaussTable> gt;
  // materials
  int ngroups = 0, nparams = 0;
  DBuf<double> gparams;
  // cached FP64 element matrices of the operator (hex8 diffusion): built at
  // the first operator use after the mesh, materials or element order change
  DBuf<double> mfc;
  bool mfc_on = true, mfc_valid = false;
  // per-iteration log rate of the last PCG loop's stop quantity (0: unknown),
  // for sizing the first chunk of the next loop
  double lnrate = 0.0;
  DBuf<int> egroup;
  bool have_egroup = false, have_mat = false;
  // boundary conditions
  std::vector<unsigned char> h_rest;
  DBuf<unsigned char> rest;
  DBuf<double> presc, load;
  bool have_bc = false;
  // structure
  bool have_pattern = false;
  bool have_scalar = false;  // scalar FP64 layout built and uploaded
  HostPattern P;
  DBuf<int> elems, nrp, bsoff, bcol, ndiag, soff, scol, cptr;
  DBuf<uint16_t> slot, vpos;
  DBuf<long long> ssoff, sdiag;
  // matrices
  DBuf<double> sval, pseudo;
  DBuf<float> bval;
  bool have64 = false, have32 = false;
  int what64 = 0, what32 = 0;
  double kscale64 = 1, mscale64 = 0, kscale32 = 1, mscale32 = 0;
  // solver workspace
  DBuf<PcgState> st;
  DBuf<double> partials, sums;
  DBuf<unsigned> flags, ticket;
  PcgState* h_st = nullptr;   // pinned
  double* h_sums = nullptr;   // pinned
  DBuf<double> b64, x64, r64, p64, q64, d64, y64, t64;
  DBuf<float> v32[5];         // node-layout float vectors: x(d), r, p, q, spare
  DBuf<float> minv;
  int minv_kind = -1;
  // ReplaceZeroDiagonal: 0 refuses a zero global diagonal; otherwise the value
  // that replaces it.  zrep marks the unknowns replaced in the FP32 matrix
  // (zrep_on: at least one), for the FP64 matrix-free operator.
  double zdiag = 0.0;
  DBuf<unsigned char> zrep;
  bool zrep_on = false;
  DBuf<int> dfirst;
  DBuf<unsigned long long> dmax;  // Newton: bits of the largest |residual|
  // solution / transient state
  DBuf<double> u, us;
  bool have_u = false, have_us = false;
  DBuf<double> dprev;        // transient: the last step's increment, the next step's initial guess
  bool have_dprev = false;
  DBuf<double> rhs_presc, rhs_load;  // beta_gpu_solve_rhs: the caller's right-hand side as prescribed/load
  bool rhs_staged = false;           // b64 already holds the caller's right-hand side (FP64 mode)
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  std::vector<cudaEvent_t> evs;
  int max_grid = 0;
  std::map<std::tuple<const void*, int, size_t>, int> occ;
};

namespace {

// BETA_GPU_TRACE=1 in the environment prints each traced step to stderr.
bool trace_on() {
  static int on = -1;
  if (on < 0) {
    const char* e = std::getenv("BETA_GPU_TRACE");
    on = (e && e[0] && e[0] != '0') ? 1 : 0;
  }
  return on == 1;
}
// milliseconds on the host's steady clock, for the traced steps
double trace_ms() {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
#define TRACE(msg)                                                                                      \
  do {                                                                                                  \
    if (trace_on()) std::fprintf(stderr, "[beta_gpu] %.3f %s:%d %s\n", trace_ms(), __func__, __LINE__, msg); \
  } while (0)

int fail(beta_gpu_ctx* c, int code, const std::string& msg) {
  if (c) c->err = msg;
  return code;
}

int cuda_fail(beta_gpu_ctx* c, cudaError_t e, const char* what) {
  std::string m = std::string(what) + ": " + cudaGetErrorString(e);
  cudaGetLastError();
  return fail(c, e == cudaErrorMemoryAllocation ? BETA_GPU_ERR_OOM : BETA_GPU_ERR_CUDA, m);
}

#define CK(call)                                       \
  do {                                                 \
    cudaError_t e_ = (call);                           \
    if (e_ != cudaSuccess) return cuda_fail(c, e_, #call); \
  } while (0)

#define CKL(what)                                          \
  do {                                                     \
    cudaError_t e_ = cudaGetLastError();                   \
    if (e_ != cudaSuccess) return cuda_fail(c, e_, what);  \
  } while (0)

// Resident blocks per SM of a kernel at (block, smem), cached per context.
int occupancy(beta_gpu_ctx* c, const void* k, int block, size_t smem) {
  auto key = std::make_tuple(k, block, smem);
  auto it = c->occ.find(key);
  if (it != c->occ.end()) return it->second;
  int nb = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k, block, smem) != cudaSuccess || nb < 1) {
    cudaGetLastError();
    nb = 1;
  }
  c->occ[key] = nb;
  return nb;
}

// Kernel launch on the context stream, counted.  Every kernel here is a
// grid-stride loop, so the grid is clamped to one full wave of resident
// blocks (SM count x occupancy): no partial second wave.
template <typename... KArgs, typename... Args>
void launch(beta_gpu_ctx* c, void (*k)(KArgs...), int grid, int block, size_t smem, Args... args) {
  const int wave = c->nsm * occupancy(c, (const void*)k, block, smem);
  if (grid > wave) grid = wave;
  k<<<grid, block, smem, c->stream>>>(args...);
  ++c->n_launch;
}

// Runs body(lo, hi) over [0, n) on the host's threads when n is large (the
// input checks of a million-element mesh are otherwise tens of ms on one core).
template <class F>
void host_parallel(size_t n, F&& body) {
  constexpr size_t kGrain = 1 << 20;
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  const size_t nt = std::min<size_t>(std::min<size_t>(hw, 32), (n + kGrain - 1) / kGrain);
  if (nt <= 1) {
    body(size_t(0), n);
    return;
  }
  std::vector<std::thread> th;
  const size_t step = (n + nt - 1) / nt;
  for (size_t t = 0; t < nt; ++t) {
    const size_t lo = t * step, hi = std::min(n, lo + step);
    if (lo < hi) th.emplace_back([&body, lo, hi] { body(lo, hi); });
  }
  for (auto& x : th) x.join();
}

// Uploads of at least kStageMin bytes from pageable host memory go through a
// pinned staging buffer: all host threads copy one half while the DMA of the
// other half runs, instead of the driver's single-threaded staging of a
// pageable copy.  Like a pageable copy, the source may be reused as soon as
// the call returns.  There is one buffer per device for the whole process,
// allocated at the first such upload and kept until the process ends (so a
// short-lived context pays no pinned allocation), shared by the contexts on
// that device under a mutex; each half has an event recorded on the stream
// of the copy that last read it, and a refill waits for that event.
constexpr size_t kStageHalf = size_t(32) << 20;
constexpr size_t kStageMin = size_t(4) << 20;
constexpr int kStageDevices = 64;

struct Stage {
  std::mutex mu;
  char* buf = nullptr;
  cudaEvent_t ev[2] = {nullptr, nullptr};
  bool failed = false;  // no pinned memory to be had: plain pageable copies
};
Stage g_stage[kStageDevices];

bool pageable(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return true;
  }
  return a.type == cudaMemoryTypeUnregistered;
}

// S.mu held; false: use a plain copy
bool stage_ready(Stage& S) {
  if (S.buf) return true;
  if (S.failed) return false;
  bool ok = cudaHostAlloc((void**)&S.buf, 2 * kStageHalf, cudaHostAllocDefault) == cudaSuccess;
  for (auto& ev : S.ev) ok = ok && cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) == cudaSuccess;
  if (!ok) {
    cudaGetLastError();
    for (auto& ev : S.ev)
      if (ev) cudaEventDestroy(ev);
    if (S.buf) cudaFreeHost(S.buf);
    S.buf = nullptr;
    S.ev[0] = S.ev[1] = nullptr;
    S.failed = true;
  }
  return ok;
}

cudaError_t h2d_staged(beta_gpu_ctx* c, char* dst, const char* src, size_t bytes) {
  if (c->device < 0 || c->device >= kStageDevices)
    return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, c->stream);
  Stage& S = g_stage[c->device];
  std::lock_guard<std::mutex> lock(S.mu);
  if (!stage_ready(S)) return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, c->stream);
  cudaError_t e;
  for (size_t off = 0, k = 0; off < bytes; off += kStageHalf, ++k) {
    const size_t n = std::min(kStageHalf, bytes - off);
    const int h = (int)(k & 1);
    char* st = S.buf + h * kStageHalf;
    if ((e = cudaEventSynchronize(S.ev[h])) != cudaSuccess) return e;  // its last copy has finished
    host_parallel(n, [&](size_t lo, size_t hi) { std::memcpy(st + lo, src + off + lo, hi - lo); });
    if ((e = cudaMemcpyAsync(dst + off, st, n, cudaMemcpyHostToDevice, c->stream)) != cudaSuccess) return e;
    if ((e = cudaEventRecord(S.ev[h], c->stream)) != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t h2d(beta_gpu_ctx* c, void* dst, const void* src, size_t bytes) {
  c->n_h2d += (long long)bytes;
  if (bytes >= kStageMin && pageable(src)) return h2d_staged(c, (char*)dst, (const char*)src, bytes);
  return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, c->stream);
}

cudaError_t d2h(beta_gpu_ctx* c, void* dst, const void* src, size_t bytes) {
  c->n_d2h += (long long)bytes;
  return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, c->stream);
}

int grid_for(beta_gpu_ctx* c, long long work_items, int per_block) {
  long long g = (work_items + per_block - 1) / per_block;
  if (g < 1) g = 1;
  if (g > c->max_grid) g = c->max_grid;
  return (int)g;
}

template <typename T>
int upload(beta_gpu_ctx* c, DBuf<T>& d, const T* h, size_t n) {
  if (trace_on()) std::fprintf(stderr, "[beta_gpu] upload %zu x %zu bytes, buf %p/%zu, stream %p\n", n, sizeof(T), (void*)d.p, d.n, (void*)c->stream);
  CK(d.alloc(n));
  TRACE("allocated");
  if (n) CK(h2d(c, d.p, h, n * sizeof(T)));
  TRACE("copy queued");
  return BETA_GPU_OK;
}

bool all_finite(const double* a, size_t n) {
  std::atomic<bool> ok{true};
  host_parallel(n, [&](size_t lo, size_t hi) {
    for (size_t i = lo; i < hi; ++i)
      if (!std::isfinite(a[i])) {
        ok = false;
        return;
      }
  });
  return ok;
}

void invalidate_matrices(beta_gpu_ctx* c) {
  c->have64 = c->have32 = false;
  c->minv_kind = -1;
  c->lnrate = 0.0;
}

// ---- element launches (colour by colour) ----------------------------------
ElemArgs elem_args(beta_gpu_ctx* c) {
  ElemArgs A;
  A.xyz = c->xyz.p;
  A.conn = c->conn.p;
  A.gparams = c->gparams.p;
  A.egroup = c->have_egroup ? c->egroup.p : nullptr;
  A.nparams = c->nparams;
  A.nip = c->h_gt.nip;
  A.gt = c->gt.p;
  A.slot = c->slot.p;
  A.nrp = c->nrp.p;
  A.rest = c->rest.p;
  A.presc = c->presc.p;
  A.bsoff = c->bsoff.p;
  A.vpos = c->P.run > 1 ? c->vpos.p : nullptr;
  A.bval = c->bval.p;
  A.soff = c->soff.p;
  A.ssoff = c->ssoff.p;
  A.sval = c->sval.p;
  A.pseudo = c->pseudo.p;
  A.kscale = 1.0;
  A.mscale = 0.0;
  A.flags = c->flags.p;
  return A;
}

// ugnl: the displacement of a geometric-nonlinear tangent (hex8 elasticity),
// null for the linear element.
template <typename T>
int launch_assembly(beta_gpu_ctx* c, const ElemArgs& A, const double* ugnl = nullptr) {
  const int nip = c->h_gt.nip;
  for (int col = 0; col < c->P.ncolor; ++col) {
    const int beg = c->P.color_ptr[col], nel = c->P.color_ptr[col + 1] - beg;
    if (nel == 0) continue;
    const int* el = c->elems.p + beg;
    if (ugnl) {
      size_t sm = (size_t)nip * 33 * sizeof(T);
      launch(c, k_asm_hex8_gnl<T>, grid_for(c, nel, 8), 256, sm, A, el, nel, ugnl);
    } else if (c->kind == BETA_GPU_HEX8_ELASTIC) {
      size_t sm = (size_t)nip * 33 * sizeof(T);
      launch(c, k_asm_hex8_elastic<T>, grid_for(c, nel, 8), 256, sm, A, el, nel);
    } else if (c->kind == BETA_GPU_HEX8_HEAT) {
      size_t sm = (size_t)nip * 33 * sizeof(T);
      launch(c, k_asm_hex8_heat<T>, grid_for(c, nel, 8), 256, sm, A, el, nel);
    } else if (c->kind == BETA_GPU_QUAD4_HEAT) {
      size_t sm = (size_t)nip * 13 * sizeof(T);
      launch(c, k_asm_quad4_heat<T>, grid_for(c, nel, 16), 256, sm, A, el, nel);
    } else {
      size_t sm = (size_t)nip * 13 * sizeof(T);
      launch(c, k_asm_quad4_pstress<T>, grid_for(c, nel, 16), 256, sm, A, el, nel);
    }
    CKL("element kernel launch");
  }
  return BETA_GPU_OK;
}

bool is_diffusion(int kind) { return kind == BETA_GPU_HEX8_HEAT || kind == BETA_GPU_QUAD4_HEAT; }

// y = K (c1 w1 + c2 w2) + cm M w1 (FP64, matrix-free), y zeroed first.
// Builds the cached element matrices of a hex8 diffusion mesh when they are
// enabled, not yet built and fit in a quarter of the free device memory
// (otherwise the operator keeps integrating on the fly).
int ensure_mfc(beta_gpu_ctx* c, const MfArgs& A) {
  if (c->mfc_valid || !c->mfc_on || c->kind != BETA_GPU_HEX8_HEAT) return BETA_GPU_OK;
  const size_t vals = (size_t)((c->nelem + 31) / 32) * 32 * kMfcHeat;
  if (c->mfc.n != vals) {
    c->mfc.release();
    size_t fr = 0, tot = 0;
    CK(cudaMemGetInfo(&fr, &tot));
    if (vals * sizeof(double) > fr / 4) return BETA_GPU_OK;
    CK(c->mfc.alloc(vals));
  }
  launch(c, k_mfc_build_hex8_heat<0>, grid_for(c, c->nelem, 256), 256, 0, A, (const int*)c->elems.p, c->nelem,
         c->mfc.p);
  launch(c, k_mfc_build_hex8_heat<1>, grid_for(c, c->nelem, 256), 256, 0, A, (const int*)c->elems.p, c->nelem,
         c->mfc.p);
  CKL("k_mfc_build_hex8_heat");
  c->mfc_valid = true;
  return BETA_GPU_OK;
}

int mf_apply(beta_gpu_ctx* c, double c1, const double* w1, double c2, const double* w2, double cm,
             double* y) {
  MfArgs A;
  A.xyz = c->xyz.p;
  A.conn = c->conn.p;
  A.gparams = c->gparams.p;
  A.egroup = c->have_egroup ? c->egroup.p : nullptr;
  A.nparams = c->nparams;
  A.nip = c->h_gt.nip;
  A.gt = c->gt.p;
  A.c1 = c1;
  A.c2 = c2;
  A.cm = cm;
  int rc;
  if ((rc = ensure_mfc(c, A)) != BETA_GPU_OK) return rc;
  CK(cudaMemsetAsync(y, 0, sizeof(double) * c->ndof, c->stream));
  if (c->mfc_valid) {
    for (int col = 0; col < c->P.ncolor; ++col) {
      const int beg = c->P.color_ptr[col], nel = c->P.color_ptr[col + 1] - beg;
      if (nel == 0) continue;
      launch(c, k_mfc_apply_hex8_heat, grid_for(c, nel, 256), 256, 0, (const int*)c->conn.p,
             (const int*)c->elems.p, beg, nel, (const double*)c->mfc.p, c1, c2, cm, w1, w2, y);
      CKL("k_mfc_apply_hex8_heat launch");
    }
    return BETA_GPU_OK;
  }
  for (int col = 0; col < c->P.ncolor; ++col) {
    const int beg = c->P.color_ptr[col], nel = c->P.color_ptr[col + 1] - beg;
    if (nel == 0) continue;
    const int* el = c->elems.p + beg;
    if (c->kind == BETA_GPU_HEX8_ELASTIC)
      launch(c, k_mf_hex8_elastic, grid_for(c, nel, 32), 256, 0, A, el, nel, w1, w2, y);
    else if (c->kind == BETA_GPU_HEX8_HEAT)
      launch(c, k_mf_hex8_heat_t, grid_for(c, nel, 256), 256, 0, A, el, nel, w1, w2, y);
    else if (c->kind == BETA_GPU_QUAD4_HEAT)
      launch(c, k_mf_quad4_heat, grid_for(c, nel, 64), 256, 0, A, el, nel, w1, w2, y);
    else
      launch(c, k_mf_quad4_pstress, grid_for(c, nel, 64), 256, 0, A, el, nel, w1, w2, y);
    CKL("matrix-free kernel launch");
  }
  return BETA_GPU_OK;
}

// y = geometric-nonlinear internal force at displacement u (FP64), y zeroed
// first; hex8 elasticity.
int fint_apply(beta_gpu_ctx* c, const double* u, double* y) {
  MfArgs A;
  A.xyz = c->xyz.p;
  A.conn = c->conn.p;
  A.gparams = c->gparams.p;
  A.egroup = c->have_egroup ? c->egroup.p : nullptr;
  A.nparams = c->nparams;
  A.nip = c->h_gt.nip;
  A.gt = c->gt.p;
  A.c1 = 1.0;
  A.c2 = 0.0;
  A.cm = 0.0;
  CK(cudaMemsetAsync(y, 0, sizeof(double) * c->ndof, c->stream));
  for (int col = 0; col < c->P.ncolor; ++col) {
    const int beg = c->P.color_ptr[col], nel = c->P.color_ptr[col + 1] - beg;
    if (nel == 0) continue;
    launch(c, k_fint_hex8_gnl, grid_for(c, nel, 32), 256, 0, A, (const int*)c->elems.p + beg, nel, u, y);
    CKL("k_fint_hex8_gnl launch");
  }
  return BETA_GPU_OK;
}

int read_flags(beta_gpu_ctx* c, unsigned* out) {
  CK(d2h(c, c->h_sums, c->flags.p, sizeof(unsigned)));
  CK(cudaStreamSynchronize(c->stream));
  std::memcpy(out, c->h_sums, sizeof(unsigned));
  return BETA_GPU_OK;
}

int read_state(beta_gpu_ctx* c, PcgState* out) {
  CK(d2h(c, c->h_st, c->st.p, sizeof(PcgState)));
  CK(cudaStreamSynchronize(c->stream));
  *out = *c->h_st;
  return BETA_GPU_OK;
}

int read_sums(beta_gpu_ctx* c, int n, double* out) {
  CK(d2h(c, c->h_sums, c->sums.p, sizeof(double) * n));
  CK(cudaStreamSynchronize(c->stream));
  for (int i = 0; i < n; ++i) out[i] = c->h_sums[i];
  return BETA_GPU_OK;
}

int init_state(beta_gpu_ctx* c, int rule, double tol, int maxit) {
  PcgState s;
  std::memset(&s, 0, sizeof(s));
  s.rule = rule;
  s.tol2 = tol * tol;
  s.maxit = maxit;
  *c->h_st = s;
  CK(h2d(c, c->st.p, c->h_st, sizeof(PcgState)));
  return BETA_GPU_OK;
}

int ensure_events(beta_gpu_ctx* c, int n) {
  while ((int)c->evs.size() < n) {
    cudaEvent_t e;
    CK(cudaEventCreate(&e));
    c->evs.push_back(e);
  }
  return BETA_GPU_OK;
}

struct ProfAcc {
  bool on = false;
  double ms = 0.0;
  long long launches = 0;
};

// Runs PCG iterations in chunks until the device state says done.  kind 0:
// scalar FP64; kind ND (1..3): node-block FP32.
// With profiling on, the SpMV launches at k = kProfEvery/2, 3 kProfEvery/2, ...
// of each chunk are bracketed by events (a sample: an event pair around every
// launch costs the iteration a few microseconds).
constexpr int kProfEvery = 16;
inline bool prof_sample(int k, int ce) {
  return ce < kProfEvery ? k == ce / 2 : k % kProfEvery == kProfEvery / 2;
}

// Host polling of the device-side PCG: a chunk of iterations is launched, the
// state read back, and so on until the state says done.  The iterations of a
// chunk that follow the one that ends the loop cost a few microseconds per
// launch for nothing (each kernel returns at once), and a chunk that ends
// short costs a host round trip; so a chunk is sized to end a little past
// the predicted end, from the rate at which the loop's stop quantity has
// been falling (log-linear between the first poll and the latest one; for
// the first chunk, the rate of the context's previous loop), within
// [kMinChunk, check_every].  rr0 > 0: r.r when the loop starts (known to the
// caller of a reliable-update loop from its FP64 residual), which makes the
// first poll's prediction a measured one too.
constexpr int kMinChunk = 4;

inline double stop_quantity(const PcgState& s) {
  return s.rule == kRuleReliable ? s.rr : s.last * s.last;
}
inline double stop_target(const PcgState& s) {
  return s.rule == kRuleReliable ? std::max(s.tolabs2, s.delta2 * s.maxrr) : s.tol2;
}

template <int ND>
int pcg_loop(beta_gpu_ctx* c, int check_every, ProfAcc* prof, PcgState* out, double rr0 = -1.0) {
  const int ce = std::max(1, check_every);
  int rc;
  if (prof && prof->on && (rc = ensure_events(c, 2 * ce)) != BETA_GPU_OK) return rc;
  int n = ce;
  const int it_start = c->h_st->iter;
  const bool rel = c->h_st->rule == kRuleReliable;
  // a reliable-update loop ends when r.r has fallen by delta2 from its start,
  // or below tolabs2
  if (rel && c->lnrate < 0.0 && c->h_st->delta2 > 0.0) {
    double fall = c->h_st->delta2;
    if (rr0 > 0.0 && c->h_st->tolabs2 > 0.0) fall = std::max(fall, c->h_st->tolabs2 / rr0);
    n = std::min(ce, std::max(kMinChunk, (int)(0.85 * std::log(fall) / c->lnrate)));
  }
  double g0 = rel && rr0 > 0.0 ? rr0 : -1.0;
  int it0 = it_start;
  for (;;) {
    for (int k = 0; k < n; ++k) {
      const bool sample = prof && prof->on && prof_sample(k, n);
      if (sample) CK(cudaEventRecord(c->evs[2 * k], c->stream));
      if constexpr (ND == 0) {
        ScalarMat A{c->ndof, c->P.nsslice, c->ssoff.p, c->scol.p, c->sval.p};
        launch(c, k_spmv_dot_s, grid_for(c, (long long)c->P.nsslice * 32, 256), 256, 0, 
            A, c->p64.p, c->q64.p, c->st.p, c->partials.p);
      } else {
        BlockMat A{c->nnode, c->P.nslice, c->bsoff.p, c->bcol.p, c->bval.p, c->P.compact ? c->cptr.p : nullptr};
        if (c->P.run == 3)
          launch(c, k_spmv_dot_b<ND, 3>, grid_for(c, (long long)c->P.nslice * 32, 256), 256, 0,
              A, (const float*)c->v32[2].p, c->v32[3].p, c->st.p, c->partials.p);
        else
          launch(c, k_spmv_dot_b<ND, 1>, grid_for(c, (long long)c->P.nslice * 32, 256), 256, 0,
              A, (const float*)c->v32[2].p, c->v32[3].p, c->st.p, c->partials.p);
      }
      if (sample) CK(cudaEventRecord(c->evs[2 * k + 1], c->stream));
      if constexpr (ND == 0) {
        launch(c, k_update_s, grid_for(c, c->ndof, 256), 256, 0, c->ndof, c->x64.p, c->r64.p, c->p64.p,
                                                                     c->q64.p, c->d64.p, c->st.p, c->partials.p);
        launch(c, k_pupd_s, grid_for(c, c->ndof, 256), 256, 0, c->ndof, c->p64.p, c->r64.p, c->d64.p, c->st.p);
      } else if constexpr (PassNodes<ND>::N == 1) {  // two and three dofs per node
        launch(c, k_update_b<ND>, grid_for(c, c->nnode, 256), 256, 0, c->nnode, c->v32[0].p, c->v32[1].p,
               (const float*)c->v32[2].p, (const float*)c->v32[3].p, (const float*)c->minv.p, c->st.p,
               c->partials.p);
        launch(c, k_pupd_b<ND>, grid_for(c, c->nnode, 256), 256, 0, c->nnode, c->v32[2].p,
               (const float*)c->v32[1].p, (const float*)c->minv.p, (const PcgState*)c->st.p);
      } else {
        // several nodes per thread with 16-byte accesses (one dof per node: four)
        const long long blocks = c->nnode / PassNodes<ND>::N + 1;
        launch(c, k_update_bn<ND>, grid_for(c, blocks, 256), 256, 0, c->nnode, c->v32[0].p, c->v32[1].p,
               (const float*)c->v32[2].p, (const float*)c->v32[3].p, (const float*)c->minv.p, c->st.p,
               c->partials.p);
        launch(c, k_pupd_bn<ND>, grid_for(c, blocks, 256), 256, 0, c->nnode, c->v32[2].p,
               (const float*)c->v32[1].p, (const float*)c->minv.p, (const PcgState*)c->st.p);
      }
    }
    CKL("pcg launch");
    int before = c->h_st->iter;
    PcgState s;
    if ((rc = read_state(c, &s)) != BETA_GPU_OK) return rc;
    if (prof && prof->on) {
      int real = std::min(n, std::max(0, s.iter - before) + (s.done && s.status == kStatusBreakdown ? 1 : 0));
      for (int k = 0; k < real; ++k) {
        if (!prof_sample(k, n)) continue;
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, c->evs[2 * k], c->evs[2 * k + 1]));
        prof->ms += ms;
        prof->launches += 1;
      }
    }
    const double g = stop_quantity(s);
    const bool measured = g0 > 0.0 && g > 0.0 && s.iter > it0;
    const double lr = measured ? std::log(g / g0) / (s.iter - it0) : c->lnrate;
    if (s.done) {
      double lr_end = measured ? lr : 0.0;
      // a loop that ended at its first poll: a reliable-update loop has cut
      // r.r from its largest value since the last replacement to s.rr in
      // the loop's own iterations
      if (!measured && s.rule == kRuleReliable && s.status == kStatusReplace && s.rr > 0.0 && s.maxrr > s.rr &&
          s.iter > it_start)
        lr_end = std::log(s.rr / s.maxrr) / (s.iter - it_start);
      if (lr_end < 0.0 && std::isfinite(lr_end)) c->lnrate = lr_end;
      *out = s;
      return BETA_GPU_OK;
    }
    if (g0 <= 0.0 && g > 0.0) {
      g0 = g;
      it0 = s.iter;
    }
    const double target = stop_target(s);
    n = ce;
    if (lr < 0.0 && std::isfinite(lr) && target > 0.0 && g > target) {
      const double left = std::log(target / g) / lr;
      if (left < ce) n = std::min(ce, std::max(kMinChunk, (int)std::ceil(left) + 2));
    } else if (target > 0.0 && g <= target) {
      n = kMinChunk;
    }
  }
}

int ensure_workspace(beta_gpu_ctx* c) {
  const size_t n = c->ndof;
  for (DBuf<double>* b : {&c->b64, &c->x64, &c->r64, &c->p64, &c->q64, &c->d64, &c->y64, &c->t64})
    CK(b->alloc(n));
  for (auto& v : c->v32) CK(v.alloc((size_t)c->nnode * (c->ndpn == 3 ? 4 : c->ndpn)));  // p (v32[2]) padded for ndpn 3
  CK(c->minv.alloc((size_t)c->nnode * (c->ndpn * (c->ndpn + 1) / 2)));
  CK(c->zrep.alloc(n));
  CK(c->u.alloc(n));
  return BETA_GPU_OK;
}

// LargeMatrix::CheckAndFixZeroDiagonal (largeMatrix.cpp:43-79) on the matrix a
// solve is about to use (ND 0: the FP64 scalar matrix; 1..3: the FP32
// node-block matrix).  The reference scans the diagonal in order: a negative
// entry met before any zero one is refused; a zero one is refused unless a
// replacement value is set, and then every zero diagonal becomes that value
// (the matrix keeps it until the next assembly, as the reference's does).
template <int ND>
int check_fix_diag(beta_gpu_ctx* c) {
  constexpr int kNone = 0x7f7f7f7f;  // the byte pattern of the preset below
  CK(c->dfirst.alloc(2));
  CK(cudaMemsetAsync(c->dfirst.p, 0x7f, 2 * sizeof(int), c->stream));
  if constexpr (ND == 0) {
    launch(c, k_diag_scan_s, grid_for(c, c->ndof, 256), 256, 0, c->ndof, (const long long*)c->sdiag.p,
           (const double*)c->sval.p, c->dfirst.p);
  } else {
    launch(c, k_diag_scan_b<ND>, grid_for(c, c->nnode, 256), 256, 0, c->nnode, (const int*)c->bsoff.p,
           (const int*)c->ndiag.p, (const float*)c->bval.p, c->dfirst.p);
  }
  CKL("diagonal scan");
  int first[2];
  CK(d2h(c, c->h_sums, c->dfirst.p, sizeof(first)));
  CK(cudaStreamSynchronize(c->stream));
  std::memcpy(first, c->h_sums, sizeof(first));
  if constexpr (ND > 0) {
    CK(cudaMemsetAsync(c->zrep.p, 0, c->ndof, c->stream));
    c->zrep_on = false;
  }
  if (first[1] < first[0])
    return fail(c, BETA_GPU_ERR_NEGDIAG, "The diagonal term(s) are less than zero - here is one of them : (" +
                                             std::to_string(first[1]) + "," + std::to_string(first[1]) + ")");
  if (first[0] == kNone) return BETA_GPU_OK;
  if (c->zdiag == 0.0)
    return fail(c, BETA_GPU_ERR_ZERODIAG,
                "The diagonal term(s) are zero - here is one of them : (" + std::to_string(first[0]) + "," +
                    std::to_string(first[0]) + "); set a replacement value with beta_gpu_set_zero_diagonal "
                    "(the ReplaceZeroDiagonal option)");
  if constexpr (ND == 0) {
    launch(c, k_diag_fix_s, grid_for(c, c->ndof, 256), 256, 0, c->ndof, (const long long*)c->sdiag.p, c->sval.p,
           c->zdiag);
  } else {
    launch(c, k_diag_fix_b<ND>, grid_for(c, c->nnode, 256), 256, 0, c->nnode, (const int*)c->bsoff.p,
           (const int*)c->ndiag.p, c->bval.p, (float)c->zdiag, c->zrep.p);
    c->zrep_on = true;
  }
  CKL("diagonal fix");
  return BETA_GPU_OK;
}

template <int ND>
int compute_minv(beta_gpu_ctx* c, int precond) {
  if (c->minv_kind == precond) return BETA_GPU_OK;
  int rc = check_fix_diag<ND>(c);
  if (rc != BETA_GPU_OK) return rc;
  CK(cudaMemsetAsync(c->flags.p, 0, sizeof(unsigned), c->stream));
  launch(c, k_minv_b<ND>, grid_for(c, c->nnode, 256), 256, 0, 
      c->nnode, c->bsoff.p, c->ndiag.p, c->bval.p, c->minv.p,
      precond == BETA_GPU_PRECOND_JACOBI ? 1 : 0, c->flags.p);
  CKL("k_minv_b");
  unsigned f = 0;
  rc = read_flags(c, &f);
  if (rc) return rc;
  if (f & 16u) return fail(c, BETA_GPU_ERR_NEGDIAG, "non-positive diagonal in the assembled matrix");
  c->minv_kind = precond;
  return BETA_GPU_OK;
}

// Mixed-precision solve of A64 x = b with reliable updates:
//   * inner: FP32 block-Jacobi PCG on the assembled node-block matrix,
//     accumulating its correction y32; alpha, beta and norms are FP64
//     reductions of FP32 products;
//   * whenever the FP32 recursive residual has fallen by `delta`
//     (opts.inner_tol) since the last replacement, or below the target,
//     x64 += y32 and the residual is replaced by the FP64 true residual
//       r = rest ? 0 : load - [K (c1 x + c2 w2) + cm M x]
//     (matrix-free, FP64); the search direction p is kept, so the Krylov
//     process continues instead of restarting.
// x64 holds the initial iterate (prescribed values on restrained dofs) on
// entry and the solution on exit.  bnorm is ||b||.
template <int ND>
// start_from_rhs: x64 is the boundary extension of the prescribed values and
// b64 the eliminated right-hand side, so the first residual is b64 itself
// (free rows) and no operator apply is needed for it.
int mpir_core(beta_gpu_ctx* c, const beta_gpu_solve_opts* o, double c1, double c2, const double* w2,
              double cm, const double* loadv, double bnorm, beta_gpu_solve_stats* stats, ProfAcc* prof,
              bool start_from_rhs) {
  int rc;
  if ((rc = compute_minv<ND>(c, o->precond)) != BETA_GPU_OK) return rc;
  const int n = c->ndof;
  const int maxit = o->maxit > 0 ? o->maxit : 10000;
  const int max_repl = o->max_outer > 0 ? o->max_outer : 40;
  const double delta = (o->inner_tol > 0 && o->inner_tol < 1) ? o->inner_tol : 0.1;
  const int ce = o->check_every > 0 ? o->check_every : std::max(8, std::min(64, c->ndof / 20000));
  const bool ref_rule = o->stop_rule == BETA_GPU_STOP_REF;
  int status = BETA_GPU_OK, repl = 0;
  double q = 1.0;
  float* y32 = c->v32[0].p;
  float* r32 = c->v32[1].p;
  // true residual of x64 -> r64, returns ||r|| and ||x||
  auto true_residual = [&](double* rn, double* xn) -> int {
    int e;
    if ((e = mf_apply(c, c1, c->x64.p, c2, w2, cm, c->y64.p)) != BETA_GPU_OK) return e;
    if (c->zrep_on)  // the replaced zero diagonals are entries of the system matrix
      launch(c, k_zdiag_apply, grid_for(c, n, 256), 256, 0, n, (const unsigned char*)c->zrep.p, c->zdiag,
             (const double*)c->x64.p, c->y64.p);
    launch(c, k_residual64, grid_for(c, n, 256), 256, 0, n, c->rest.p, loadv, c->y64.p, c->x64.p, c->r64.p,
           c->sums.p, c->partials.p, c->ticket.p);
    CKL("k_residual64");
    double s2[2];
    if ((e = read_sums(c, 2, s2)) != BETA_GPU_OK) return e;
    *rn = std::sqrt(s2[0]);
    *xn = std::sqrt(s2[1]);
    return BETA_GPU_OK;
  };
  auto stop_q = [&](double rn, double xn) {
    return ref_rule ? (xn > 0 ? rn / xn : (rn == 0 ? 0.0 : 1e300)) : (bnorm > 0 ? rn / bnorm : rn);
  };
  auto set_tolabs = [&](double xn) -> int {
    // replace early once the FP32 residual says the target is met
    const double ta = 0.5 * o->tol * (ref_rule ? xn : bnorm);
    c->h_st->tolabs2 = ta * ta;
    CK(h2d(c, (char*)c->st.p + offsetof(PcgState, tolabs2), &c->h_st->tolabs2, sizeof(double)));
    return BETA_GPU_OK;
  };
  double rn = 0.0, xn = 0.0;
  if (start_from_rhs) {
    CK(cudaMemsetAsync(c->y64.p, 0, sizeof(double) * n, c->stream));
    launch(c, k_residual64, grid_for(c, n, 256), 256, 0, n, c->rest.p, (const double*)c->b64.p,
           (const double*)c->y64.p, (const double*)c->x64.p, c->r64.p, c->sums.p, c->partials.p, c->ticket.p);
    CKL("k_residual64");
    double s2[2];
    if ((rc = read_sums(c, 2, s2)) != BETA_GPU_OK) return rc;
    rn = std::sqrt(s2[0]);
    xn = std::sqrt(s2[1]);
  } else if ((rc = true_residual(&rn, &xn)) != BETA_GPU_OK) {
    return rc;
  }
  q = stop_q(rn, xn);
  int iters = 0;
  if (!std::isfinite(q)) {
    status = BETA_GPU_BREAKDOWN;
  } else if (!(q < o->tol) && rn != 0.0) {
    launch(c, k_to32, grid_for(c, n, 256), 256, 0, (long long)n, (const double*)c->r64.p, 1.0, r32);
    if ((rc = init_state(c, kRuleReliable, o->tol, maxit)) != BETA_GPU_OK) return rc;
    c->h_st->delta2 = delta * delta;
    CK(h2d(c, (char*)c->st.p + offsetof(PcgState, delta2), &c->h_st->delta2, sizeof(double)));
    if ((rc = set_tolabs(xn)) != BETA_GPU_OK) return rc;
    launch(c, k_start_b<ND>, grid_for(c, c->nnode, 256), 256, 0, c->nnode, y32, (const float*)r32, c->v32[2].p,
           (const float*)c->minv.p, c->st.p, c->partials.p);
    CKL("k_start_b");
    for (;;) {
      PcgState s;
      if ((rc = pcg_loop<ND>(c, ce, prof, &s, rn * rn)) != BETA_GPU_OK) return rc;
      iters = s.iter;
      if (s.status == kStatusBreakdown) { status = BETA_GPU_BREAKDOWN; break; }
      // fold the FP32 correction into the FP64 iterate, then measure the truth
      launch(c, k_axpy_from32, grid_for(c, n, 256), 256, 0, (long long)n, c->x64.p, 1.0, (const float*)y32);
      CK(cudaMemsetAsync(y32, 0, sizeof(float) * n, c->stream));
      if ((rc = true_residual(&rn, &xn)) != BETA_GPU_OK) return rc;
      q = stop_q(rn, xn);
      if (!std::isfinite(q)) { status = BETA_GPU_BREAKDOWN; break; }
      if (q < o->tol || rn == 0.0) break;
      if (s.status == kStatusMaxit || iters >= maxit || repl >= max_repl) { status = BETA_GPU_MAXIT; break; }
      ++repl;
      // residual replacement, keep the search direction
      launch(c, k_to32, grid_for(c, n, 256), 256, 0, (long long)n, (const double*)c->r64.p, 1.0, r32);
      if (ref_rule && (rc = set_tolabs(xn)) != BETA_GPU_OK) return rc;
      launch(c, k_replace_b<ND>, grid_for(c, c->nnode, 256), 256, 0, c->nnode, (const float*)r32,
             (const float*)c->minv.p, c->st.p, c->partials.p);
      launch(c, k_pupd_b<ND>, grid_for(c, c->nnode, 256), 256, 0, c->nnode, c->v32[2].p, (const float*)r32,
             (const float*)c->minv.p, (const PcgState*)c->st.p);
      CKL("replacement");
    }
  }
  if (stats) {
    stats->status = status;
    stats->iterations = iters;
    stats->outer_iterations = repl;
    stats->final_norm = q;
  }
  return status;
}

// One inexact Newton step in FP32: the residual r64 (FP64) rounded to FP32,
// block-Jacobi PCG on the FP32 tangent from zero until the FP32 recursive
// residual has fallen by o->inner_tol (default 1e-3); the correction is left
// in v32[0].
template <int ND>
int newton_step32(beta_gpu_ctx* c, const beta_gpu_solve_opts* o, int* iterations) {
  int rc;
  if ((rc = compute_minv<ND>(c, o->precond)) != BETA_GPU_OK) return rc;
  const int n = c->ndof;
  const double delta = (o->inner_tol > 0 && o->inner_tol < 1) ? o->inner_tol : 1e-3;
  const int ce = o->check_every > 0 ? o->check_every : std::max(8, std::min(64, c->ndof / 20000));
  launch(c, k_to32, grid_for(c, n, 256), 256, 0, (long long)n, (const double*)c->r64.p, 1.0, c->v32[1].p);
  if ((rc = init_state(c, kRuleReliable, 1.0, o->maxit > 0 ? o->maxit : 10000)) != BETA_GPU_OK) return rc;
  c->h_st->delta2 = delta * delta;
  c->h_st->tolabs2 = 0.0;
  CK(h2d(c, (char*)c->st.p + offsetof(PcgState, delta2), &c->h_st->delta2, sizeof(double)));
  CK(h2d(c, (char*)c->st.p + offsetof(PcgState, tolabs2), &c->h_st->tolabs2, sizeof(double)));
  launch(c, k_start_b<ND>, grid_for(c, c->nnode, 256), 256, 0, c->nnode, c->v32[0].p, (const float*)c->v32[1].p,
         c->v32[2].p, (const float*)c->minv.p, c->st.p, c->partials.p);
  CKL("k_start_b");
  PcgState s;
  if ((rc = pcg_loop<ND>(c, ce, nullptr, &s)) != BETA_GPU_OK) return rc;
  *iterations = s.iter;
  if (s.status == kStatusBreakdown) return fail(c, BETA_GPU_BREAKDOWN, "PCG breakdown in a Newton step");
  return BETA_GPU_OK;
}

int mpir_dispatch(beta_gpu_ctx* c, bool start_from_rhs, const beta_gpu_solve_opts* o, double c1, double c2,
                  const double* w2,
                  double cm, const double* loadv, double bnorm, beta_gpu_solve_stats* stats, ProfAcc* prof) {
  switch (c->ndpn) {
    case 1: return mpir_core<1>(c, o, c1, c2, w2, cm, loadv, bnorm, stats, prof, start_from_rhs);
    case 2: return mpir_core<2>(c, o, c1, c2, w2, cm, loadv, bnorm, stats, prof, start_from_rhs);
    default: return mpir_core<3>(c, o, c1, c2, w2, cm, loadv, bnorm, stats, prof, start_from_rhs);
  }
}

// Plain FP64 Jacobi-PCG on the assembled scalar matrix: b64 must hold the
// right-hand side, x64 the initial guess.
int fp64_core(beta_gpu_ctx* c, const beta_gpu_solve_opts* o, beta_gpu_solve_stats* stats, ProfAcc* prof) {
  int rc;
  const int n = c->ndof;
  ScalarMat A{n, c->P.nsslice, c->ssoff.p, c->scol.p, c->sval.p};
  if ((rc = check_fix_diag<0>(c)) != BETA_GPU_OK) return rc;
  CK(cudaMemsetAsync(c->flags.p, 0, sizeof(unsigned), c->stream));
  launch(c, k_dinv_s, grid_for(c, n, 256), 256, 0, n, c->sdiag.p, c->sval.p, c->d64.p, c->flags.p);
  CKL("k_dinv_s");
  unsigned f = 0;
  if ((rc = read_flags(c, &f)) != BETA_GPU_OK) return rc;
  if (f & 8u) return fail(c, BETA_GPU_ERR_ZERODIAG, "zero diagonal (LargeMatrix::CheckAndFixZeroDiagonal)");
  if (f & 16u) return fail(c, BETA_GPU_ERR_NEGDIAG, "negative diagonal (LargeMatrix::CheckAndFixZeroDiagonal)");
  launch(c, k_spmv_s, grid_for(c, (long long)c->P.nsslice * 32, 256), 256, 0, A, c->x64.p, c->r64.p, c->b64.p);
  const int rule = o->stop_rule == BETA_GPU_STOP_REF ? kStopRef : kStopRB;
  if ((rc = init_state(c, rule, o->tol, o->maxit > 0 ? o->maxit : 10000)) != BETA_GPU_OK) return rc;
  launch(c, k_start_s, grid_for(c, n, 256), 256, 0, n, c->x64.p, c->r64.p, c->b64.p, c->d64.p, c->p64.p,
                                                        c->st.p, c->partials.p);
  CKL("k_start_s");
  const int ce = o->check_every > 0 ? o->check_every : std::max(8, std::min(64, n / 20000));
  PcgState s;
  if ((rc = pcg_loop<0>(c, ce, prof, &s)) != BETA_GPU_OK) return rc;
  // true residual ||b - A x|| / ||b||
  launch(c, k_spmv_s, grid_for(c, (long long)c->P.nsslice * 32, 256), 256, 0, A, c->x64.p, c->t64.p, c->b64.p);
  launch(c, k_norm2_diff, grid_for(c, n, 256), 256, 0, n, c->t64.p, nullptr, c->sums.p, c->partials.p,
                                                           c->ticket.p);
  CKL("true residual");
  double rr;
  if ((rc = read_sums(c, 1, &rr)) != BETA_GPU_OK) return rc;
  int status = s.status == kStatusOk ? BETA_GPU_OK : (s.status == kStatusMaxit ? BETA_GPU_MAXIT : BETA_GPU_BREAKDOWN);
  if (stats) {
    stats->status = status;
    stats->iterations = s.iter;
    stats->outer_iterations = 0;
    stats->final_norm = s.last;
    stats->true_rel_residual = s.bb > 0 ? std::sqrt(rr / s.bb) : std::sqrt(rr);
  }
  return status;
}

}  // namespace

#include "batch_host.cuh"

namespace {

// A system checked and structured on the host, ready to be copied into a pool
// (CPU work only; safe to run on any thread).
struct PreparedSys {
  int kind = 0, ndim = 0, nnode = 0, nelem = 0, nnpe = 0, ndpn = 0, order = 0, ngroups = 0, nparams = 0;
  std::vector<double> xyz, gp, presc, load;
  std::vector<int> conn, eg;
  std::vector<unsigned char> rest;
  HostPattern P;
  SysLayout L;
  size_t ndof() const { return (size_t)nnode * ndpn; }
};

int prepare_system(int kind, int ndim, int nnode, const double* xyz, int nelem, int nnpe, const int* conn,
                   const int* first_dof, int ndpn, int order, int ngroups, int nparams, const double* gp,
                   const int* eg, const unsigned char* restrained, const double* prescribed, const double* load,
                   PreparedSys& S, std::string& err) {
  int want_nnpe = 0, want_ndim = 0, want_ndpn = 0, want_np = 0;
  switch (kind) {
    case BETA_GPU_QUAD4_PSTRESS: want_nnpe = 4; want_ndim = 2; want_ndpn = 2; want_np = 4; break;
    case BETA_GPU_HEX8_ELASTIC: want_nnpe = 8; want_ndim = 3; want_ndpn = 3; want_np = 9; break;
    case BETA_GPU_HEX8_HEAT: want_nnpe = 8; want_ndim = 3; want_ndpn = 1; want_np = 4; break;
    case BETA_GPU_QUAD4_HEAT: err = "the 2D diffusion element is solved as a single system, not in batches";
      return BETA_GPU_ERR_UNSUPPORTED;
    default: err = "unknown element kind"; return BETA_GPU_ERR_UNSUPPORTED;
  }
  if (nnpe != want_nnpe || ndim != want_ndim || ndpn != want_ndpn || nparams != want_np) {
    err = "sizes do not match the element kind";
    return BETA_GPU_ERR_ARG;
  }
  if (nnode <= 0 || nelem <= 0 || !xyz || !conn || !first_dof || !gp || ngroups <= 0 || order < 1 || order > 4) {
    err = "bad mesh or material arguments";
    return BETA_GPU_ERR_ARG;
  }
  if (!eg && ngroups != nelem) { err = "without elem_group there must be one group per element"; return BETA_GPU_ERR_ARG; }
  const size_t ndof = (size_t)nnode * ndpn;
  if (!all_finite(xyz, (size_t)nnode * ndim) || !all_finite(gp, (size_t)ngroups * nparams) ||
      (prescribed && !all_finite(prescribed, ndof)) || (load && !all_finite(load, ndof))) {
    err = "non-finite input";
    return BETA_GPU_ERR_NOT_FINITE;
  }
  for (long long k = 0; k < (long long)nelem * nnpe; ++k)
    if (conn[k] < 0 || conn[k] >= nnode) { err = "connectivity out of range"; return BETA_GPU_ERR_ARG; }
  if (eg)
    for (int e = 0; e < nelem; ++e)
      if (eg[e] < 0 || eg[e] >= ngroups) { err = "elem_group out of range"; return BETA_GPU_ERR_ARG; }
  S.kind = kind; S.ndim = ndim; S.nnode = nnode; S.nelem = nelem; S.nnpe = nnpe; S.ndpn = ndpn; S.order = order;
  S.ngroups = ngroups; S.nparams = nparams;
  S.rest.assign(ndof, 0);
  if (restrained)
    for (size_t i = 0; i < ndof; ++i) S.rest[i] = restrained[i] ? 1 : 0;
  if (load)
    for (size_t i = 0; i < ndof; ++i)
      if (S.rest[i] && load[i] != 0.0) {
        err = "Cannot add load to a restrained degree of freedom.";
        return BETA_GPU_ERR_LOAD_ON_RESTRAINED;
      }
  std::string msg = build_pattern(nnode, nelem, nnpe, ndpn, conn, first_dof, S.rest.data(), S.P, false);
  if (!msg.empty()) { err = msg; return BETA_GPU_ERR_UNSUPPORTED; }
  S.xyz.assign(xyz, xyz + (size_t)nnode * ndim);
  S.conn.assign(conn, conn + (size_t)nelem * nnpe);
  S.gp.assign(gp, gp + (size_t)ngroups * nparams);
  if (eg) S.eg.assign(eg, eg + nelem);
  S.presc.assign(ndof, 0.0);
  S.load.assign(ndof, 0.0);
  if (prescribed) std::copy(prescribed, prescribed + ndof, S.presc.begin());
  if (load) std::copy(load, load + ndof, S.load.begin());
  S.L = layout_for(ndim, nnode, nelem, nnpe, ndpn, ngroups, nparams, eg != nullptr, S.P);
  return BETA_GPU_OK;
}

// Copies a prepared system into the pool: BETA_GPU_REJECTED when it does not fit.
int admit_system(beta_gpu_batch* b, const PreparedSys& Q, int* sys_id) {
  cudaSetDevice(b->device);
  const HostPattern& P = Q.P;
  const SysLayout& L = Q.L;
  const size_t ndof = Q.ndof();
  int id;
  if (!b->free_ids.empty()) id = b->free_ids.back();
  else if ((int)b->sys.size() < b->cap) id = (int)b->sys.size();
  else return bfail(b, BETA_GPU_REJECTED, "batch holds max_systems systems");
  const long long off = pool_alloc(b, L.total);
  if (off < 0) return bfail(b, BETA_GPU_REJECTED, "HBM budget exhausted: the system does not fit in the pool");
  if (!b->free_ids.empty()) b->free_ids.pop_back();
  else b->sys.emplace_back();
  unsigned char* base = b->pool + off;
  const GaussTable* gt = batch_gauss(b, Q.ndim, Q.order);
  int rc = gt ? BETA_GPU_OK : BETA_GPU_ERR_CUDA;
  // on the copy stream: a launch may be running on b->stream meanwhile (the
  // memory is free pool space that no running system uses); the next launch
  // waits for these copies (batch_prepare)
  auto up = [&](size_t o, const void* src, size_t bytes) {
    if (!rc) rc = batch_h2d(b, base + o, src, bytes, b->copy);
  };
  up(L.o_xyz, Q.xyz.data(), sizeof(double) * Q.xyz.size());
  up(L.o_conn, Q.conn.data(), sizeof(int) * Q.conn.size());
  up(L.o_gp, Q.gp.data(), sizeof(double) * Q.gp.size());
  if (!Q.eg.empty()) up(L.o_eg, Q.eg.data(), sizeof(int) * Q.eg.size());
  up(L.o_rest, Q.rest.data(), ndof);
  up(L.o_presc, Q.presc.data(), sizeof(double) * ndof);
  up(L.o_load, Q.load.data(), sizeof(double) * ndof);
  up(L.o_cptr, P.color_ptr.data(), sizeof(int) * P.color_ptr.size());
  up(L.o_elems, P.elem_by_color.data(), sizeof(int) * P.elem_by_color.size());
  up(L.o_slot, P.slot.data(), sizeof(uint16_t) * P.slot.size());
  up(L.o_nrp, P.nrp.data(), sizeof(int) * P.nrp.size());
  up(L.o_ndiag, P.ndiag.data(), sizeof(int) * P.ndiag.size());
  up(L.o_bsoff, P.bsoff.data(), sizeof(int) * P.bsoff.size());
  up(L.o_bcol, P.bcol.data(), sizeof(int) * P.bcol.size());
  beta_gpu_batch::Sys& S = b->sys[id];
  if (rc != BETA_GPU_OK) {
    cudaStreamSynchronize(b->copy);
    cudaGetLastError();
    pool_free(b, off, L.total);
    S.live = false;
    b->free_ids.push_back(id);
    return bfail(b, rc, "upload of the system failed");
  }
  S.live = true;
  S.last_iters = 0;
  S.kind = Q.kind; S.ndim = Q.ndim; S.nnode = Q.nnode; S.nelem = Q.nelem; S.nnpe = Q.nnpe; S.ndpn = Q.ndpn;
  S.ndof = (int)ndof; S.order = Q.order; S.off = (size_t)off; S.bytes = L.total;
  S.work = (long long)P.nchunk * 32 * Q.ndpn * Q.ndpn;
  S.nslice = P.nslice;
  BSys& D = S.desc;
  std::memset(&D, 0, sizeof(D));
  GaussTable hg;
  make_gauss_table(Q.ndim, Q.order, hg);
  D.kind = Q.kind; D.ndpn = Q.ndpn; D.nnode = Q.nnode; D.nelem = Q.nelem; D.ndof = (int)ndof; D.nip = hg.nip;
  D.ncolor = P.ncolor; D.nslice = P.nslice; D.nparams = Q.nparams; D.ndim = Q.ndim;
  D.xyz = (const double*)(base + L.o_xyz);
  D.conn = (const int*)(base + L.o_conn);
  D.gparams = (const double*)(base + L.o_gp);
  D.egroup = Q.eg.empty() ? nullptr : (const int*)(base + L.o_eg);
  D.rest = base + L.o_rest;
  D.presc = (const double*)(base + L.o_presc);
  D.load = (const double*)(base + L.o_load);
  D.color_ptr = (const int*)(base + L.o_cptr);
  D.elems = (const int*)(base + L.o_elems);
  D.slot = (const uint16_t*)(base + L.o_slot);
  D.nrp = (const int*)(base + L.o_nrp);
  D.ndiag = (const int*)(base + L.o_ndiag);
  D.bsoff = (const int*)(base + L.o_bsoff);
  D.bcol = (const int*)(base + L.o_bcol);
  D.bval = (float*)(base + L.o_bval);
  D.x64 = (double*)(base + L.o_x64);
  D.r64 = (double*)(base + L.o_r64);
  D.y64 = (double*)(base + L.o_y64);
  D.p64 = (double*)(base + L.o_p64);
  D.q64 = (double*)(base + L.o_q64);
  D.w64 = (double*)(base + L.o_w64);
  D.y32 = (float*)(base + L.o_y32);
  D.r32 = (float*)(base + L.o_r32);
  D.p32 = (float*)(base + L.o_p32);
  D.p32b = (float*)(base + L.o_p32b);
  D.z32 = (float*)(base + L.o_z32);
  D.q32 = (float*)(base + L.o_q32);
  D.minv = (float*)(base + L.o_minv);
  D.part = (double*)(base + L.o_part);
  D.gflag = (unsigned*)(base + L.o_gflag);
  D.gt = gt;
  D.st = b->d_states + id;
  D.nchunk = P.nchunk;
  BState s0;
  std::memset(&s0, 0, sizeof(s0));
  s0.phase = kPhaseNew;
  s0.status = kBRunning;
  S.st = s0;
  b->h_states[id] = s0;
  S.fresh = true;
  // from s0 itself (pageable: staged before the call returns), not from the
  // pinned h_states, which the next state read-back may overwrite first
  if ((rc = batch_h2d(b, b->d_states + id, &s0, sizeof(BState), b->copy))) return rc;
  BCK(cudaEventRecord(b->ev_copy, b->copy));
  b->copy_pending = true;
  *sys_id = id;
  return BETA_GPU_OK;
}

// A launch in two halves, so that a caller (the server) can do host work and
// copies on the copy stream while the launch runs: batch_start issues it
// (nothing to do: *launched = false), batch_finish waits for it and reads the
// states back.
int batch_start(beta_gpu_batch* b, const beta_gpu_solve_opts* o, int iters_per_launch, bool* launched) {
  int na = 0, rc;
  *launched = false;
  if ((rc = batch_prepare(b, o, iters_per_launch, &na))) return rc;
  if (na > 0) {
    BCK(cudaMemsetAsync(b->d_preempt, 0, sizeof(int), b->stream));
    BCK(cudaEventRecord(b->ev0, b->stream));
    if ((rc = batch_launch_graph(b))) return rc;
    BCK(cudaEventRecord(b->ev1, b->stream));
    *launched = true;
  }
  return BETA_GPU_OK;
}

// Ends the slice of the launch in flight early (the copy stream writes the
// flag while the launch runs; the kernel reads it at its slice checks).
int batch_preempt(beta_gpu_batch* b) {
  static const int one = 1;
  BCK(cudaMemcpyAsync(b->d_preempt, &one, sizeof(int), cudaMemcpyHostToDevice, b->copy));
  // the next launch zeroes the flag only after this write (batch_prepare waits)
  BCK(cudaEventRecord(b->ev_copy, b->copy));
  b->copy_pending = true;
  return BETA_GPU_OK;
}

int batch_finish(beta_gpu_batch* b) {
  const int rc = batch_pull_states(b);
  if (rc == BETA_GPU_TIMEOUT) {
    // the launch stopped mid-iteration: unfinished systems restart from scratch next time
    const std::string msg = b->err;
    for (size_t i = 0; i < b->sys.size(); ++i)
      if (b->sys[i].live && b->sys[i].st.phase != kPhaseDone) {
        std::memset(&b->sys[i].st, 0, sizeof(BState));
        b->sys[i].st.phase = kPhaseNew;
        b->sys[i].st.status = kBRunning;
      }
    for (size_t i = 0; i < b->sys.size(); ++i) b->h_states[i] = b->sys[i].st;
    if (!b->sys.empty() && batch_h2d(b, b->d_states, b->h_states, sizeof(BState) * b->sys.size()) == BETA_GPU_OK)
      cudaStreamSynchronize(b->stream);
    b->err = msg;
  }
  if (rc != BETA_GPU_OK) return rc;
  BCK(cudaEventElapsedTime(&b->last_ms, b->ev0, b->ev1));
  return BETA_GPU_OK;
}

}  // namespace

#include "server_host.cuh"

// ---- scratch of beta_gpu_csr_pcg_device_noalloc ----------------------------
// One fixed array per GPU that loads the library (held until process exit).
// Host code must never pass g_noalloc_scratch itself to a kernel: on the host
// the name is a stand-in, not a device address.  noalloc_scratch_address()
// looks up the real address of the current device's copy with
// cudaGetSymbolAddress on every call: the first call on a device loads the
// library's module there (the set-up), later lookups are cheap, and an address
// is never kept across a cudaDeviceReset that would have made it stale.
static __device__ __align__(256) unsigned char g_noalloc_scratch[BETA_GPU_NOALLOC_SCRATCH_BYTES];

namespace {
// Device address of the scratch array on the current device.
cudaError_t noalloc_scratch_address(unsigned char** out) {
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess) return e;
  *out = (unsigned char*)p;
  return cudaSuccess;
}
}  // namespace

// =============================== C ABI ======================================
extern "C" {

int beta_gpu_version(void) { return 10000; }

const char* beta_gpu_last_error(const beta_gpu_ctx* c) { return c ? c->err.c_str() : "null context"; }

int beta_gpu_create(beta_gpu_ctx** out, int device) {
  if (!out) return BETA_GPU_ERR_ARG;
  *out = nullptr;
  std::unique_ptr<beta_gpu_ctx> c(new beta_gpu_ctx());
  c->device = device;
  c->P.keep_scratch = true;  // a context rebuilds its structure into the same memory
  c->P.run_request = 3;      // column runs where they shrink the FP32 matrix
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) { cudaGetLastError(); return BETA_GPU_ERR_CUDA; }
  beta_gpu_ctx* cp = c.get();
  {
    beta_gpu_ctx* c = cp;  // for CK
    CK(cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking));
    c->stream = c->own_stream;
    CK(cudaDeviceGetAttribute(&c->nsm, cudaDevAttrMultiProcessorCount, device));
    c->max_grid = c->nsm * 8;
    CK(c->st.alloc(1));
    CK(c->partials.alloc((size_t)c->max_grid * 4 + 64));
    CK(c->sums.alloc(8));
    CK(c->flags.alloc(1));
    CK(c->ticket.alloc(1));
    CK(cudaMemset(c->ticket.p, 0, sizeof(unsigned)));
    CK(cudaMemset(c->flags.p, 0, sizeof(unsigned)));
    CK(cudaMallocHost(&c->h_st, sizeof(PcgState)));
    CK(cudaMallocHost(&c->h_sums, 8 * sizeof(double)));
    std::memset(c->h_st, 0, sizeof(PcgState));
    CK(cudaEventCreate(&c->ev0));
    CK(cudaEventCreate(&c->ev1));
  }
  *out = c.release();
  return BETA_GPU_OK;
}

int beta_gpu_destroy(beta_gpu_ctx* c) {
  if (!c) return BETA_GPU_OK;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  for (auto e : c->evs) cudaEventDestroy(e);
  if (c->ev0) cudaEventDestroy(c->ev0);
  if (c->ev1) cudaEventDestroy(c->ev1);
  if (c->h_st) cudaFreeHost(c->h_st);
  if (c->h_sums) cudaFreeHost(c->h_sums);
  cudaStream_t s = c->own_stream;
  delete c;  // DBuf destructors free device memory
  if (s) cudaStreamDestroy(s);
  return BETA_GPU_OK;
}

int beta_gpu_set_stream(beta_gpu_ctx* c, void* stream) {
  if (!c) return BETA_GPU_ERR_ARG;
  cudaSetDevice(c->device);
  CK(cudaStreamSynchronize(c->stream));
  c->stream = stream ? (cudaStream_t)stream : c->own_stream;
  return BETA_GPU_OK;
}

int beta_gpu_set_zero_diagonal(beta_gpu_ctx* c, double value) {
  if (!c) return BETA_GPU_ERR_ARG;
  if (!std::isfinite(value)) return fail(c, BETA_GPU_ERR_ARG, "the zero-diagonal replacement must be finite");
  c->zdiag = value;
  return BETA_GPU_OK;
}

int beta_gpu_set_block_runs(beta_gpu_ctx* c, int run) {
  if (!c) return BETA_GPU_ERR_ARG;
  if (run != 1 && run != 3) return fail(c, BETA_GPU_ERR_ARG, "the column run length must be 1 or 3");
  if (c->P.run_request != run && c->have_pattern) {
    c->have_pattern = false;  // the next build_pattern lays the columns out anew
    invalidate_matrices(c);
  }
  c->P.run_request = run;
  return BETA_GPU_OK;
}

int beta_gpu_set_operator_cache(beta_gpu_ctx* c, int on) {
  if (!c || (on != 0 && on != 1)) return BETA_GPU_ERR_ARG;
  c->mfc_on = on != 0;
  c->mfc_valid = false;
  if (!on) c->mfc.release();
  return BETA_GPU_OK;
}

int beta_gpu_block_layout(const beta_gpu_ctx* c, long long* out, int n) {
  if (!c || !out || n < 0 || n > 5) return BETA_GPU_ERR_ARG;
  if (!c->have_pattern) return BETA_GPU_ERR_STATE;
  const HostPattern& P = c->P;
  const long long bb = (long long)P.ndpn * P.ndpn;
  const long long cols = P.compact ? (long long)(P.ccol.size() + P.cptr.size()) : (long long)P.bcol.size();
  const long long v[5] = {P.run, P.nchunk, cols, P.nchunk * 32 * bb * 4 + cols * 4, P.compact ? 1 : 0};
  for (int i = 0; i < n; ++i) out[i] = v[i];
  return BETA_GPU_OK;
}

int beta_gpu_counters(const beta_gpu_ctx* c, long long* out, int n) {
  if (!c || !out || n < 0 || n > 3) return BETA_GPU_ERR_ARG;
  const long long v[3] = {c->n_launch, c->n_h2d, c->n_d2h};
  for (int i = 0; i < n; ++i) out[i] = v[i];
  return BETA_GPU_OK;
}

int beta_gpu_mesh_upload(beta_gpu_ctx* c, int kind, int ndim, int nnode, const double* xyz, int nelem,
                         int nnpe, const int* conn, const int* first_dof, int ndpn, int order) {
  if (!c) return BETA_GPU_ERR_ARG;
  TRACE("enter");
  cudaSetDevice(c->device);
  TRACE("device set");
  int want_nnpe = 0, want_ndim = 0, want_ndpn = 0;
  switch (kind) {
    case BETA_GPU_QUAD4_PSTRESS: want_nnpe = 4; want_ndim = 2; want_ndpn = 2; break;
    case BETA_GPU_HEX8_ELASTIC: want_nnpe = 8; want_ndim = 3; want_ndpn = 3; break;
    case BETA_GPU_HEX8_HEAT: want_nnpe = 8; want_ndim = 3; want_ndpn = 1; break;
    case BETA_GPU_QUAD4_HEAT: want_nnpe = 4; want_ndim = 2; want_ndpn = 1; break;
    default: return fail(c, BETA_GPU_ERR_UNSUPPORTED, "unknown element kind");
  }
  if (nnpe != want_nnpe || ndim != want_ndim || ndpn != want_ndpn)
    return fail(c, BETA_GPU_ERR_ARG, "nnpe/ndim/ndof_per_node do not match the element kind");
  if (nnode <= 0 || nelem <= 0 || !xyz || !conn || !first_dof)
    return fail(c, BETA_GPU_ERR_ARG, "empty mesh");
  if (order < 1 || order > 4) return fail(c, BETA_GPU_ERR_ARG, "integration order must be 1..4");
  if ((long long)nnode * ndpn > 2000000000LL) return fail(c, BETA_GPU_ERR_ARG, "too many dofs");
  if (!all_finite(xyz, (size_t)nnode * ndim)) return fail(c, BETA_GPU_ERR_NOT_FINITE, "non-finite coordinates");
  {
    std::atomic<bool> in_range{true};
    host_parallel((size_t)nelem * nnpe, [&](size_t lo, size_t hi) {
      for (size_t k = lo; k < hi; ++k)
        if (conn[k] < 0 || conn[k] >= nnode) {
          in_range = false;
          return;
        }
    });
    if (!in_range) return fail(c, BETA_GPU_ERR_ARG, "connectivity out of range");
  }
  c->kind = kind; c->ndim = ndim; c->nnode = nnode; c->nelem = nelem; c->nnpe = nnpe; c->ndpn = ndpn;
  c->ndof = nnode * ndpn; c->order = order;
  TRACE("validated");
  c->h_conn.resize((size_t)nelem * nnpe);
  host_parallel(c->h_conn.size(), [&](size_t lo, size_t hi) {
    std::memcpy(c->h_conn.data() + lo, conn + lo, (hi - lo) * sizeof(int));
  });
  c->h_first_dof.assign(first_dof, first_dof + nnode);
  int rc;
  if ((rc = upload(c, c->xyz, xyz, (size_t)nnode * ndim))) return rc;
  TRACE("xyz uploaded");
  if ((rc = upload(c, c->conn, conn, (size_t)nelem * nnpe))) return rc;
  TRACE("conn uploaded");
  make_gauss_table(ndim, order, c->h_gt);
  TRACE("gauss table built");
  if ((rc = upload(c, c->gt, &c->h_gt, 1))) return rc;
  TRACE("gauss table uploaded");
  CK(cudaStreamSynchronize(c->stream));
  TRACE("synchronized");
  c->have_pattern = false;
  c->have_bc = false;
  c->have_mat = false;
  c->have_u = c->have_us = false;
  c->mfc_valid = false;
  invalidate_matrices(c);
  return BETA_GPU_OK;
}

int beta_gpu_materials_upload(beta_gpu_ctx* c, int ngroups, int nparams, const double* gp, const int* eg) {
  if (!c) return BETA_GPU_ERR_ARG;
  if (!c->nelem) return fail(c, BETA_GPU_ERR_STATE, "upload the mesh first");
  cudaSetDevice(c->device);
  int want = c->kind == BETA_GPU_HEX8_ELASTIC ? 9 : 4;
  if (nparams != want) return fail(c, BETA_GPU_ERR_ARG, "wrong number of material parameters for the element kind");
  if (ngroups <= 0 || !gp) return fail(c, BETA_GPU_ERR_ARG, "no material groups");
  if (!eg && ngroups != c->nelem) return fail(c, BETA_GPU_ERR_ARG, "without elem_group there must be one group per element");
  if (!all_finite(gp, (size_t)ngroups * nparams)) return fail(c, BETA_GPU_ERR_NOT_FINITE, "non-finite material parameters");
  if (eg)
    for (int e = 0; e < c->nelem; ++e)
      if (eg[e] < 0 || eg[e] >= ngroups) return fail(c, BETA_GPU_ERR_ARG, "elem_group out of range");
  int rc;
  if ((rc = upload(c, c->gparams, gp, (size_t)ngroups * nparams))) return rc;
  c->have_egroup = eg != nullptr;
  if (eg && (rc = upload(c, c->egroup, eg, (size_t)c->nelem))) return rc;
  CK(cudaStreamSynchronize(c->stream));
  c->ngroups = ngroups;
  c->nparams = nparams;
  c->have_mat = true;
  c->mfc_valid = false;
  invalidate_matrices(c);
  return BETA_GPU_OK;
}

int beta_gpu_bc_upload(beta_gpu_ctx* c, const unsigned char* restrained, const double* prescribed,
                       const double* load) {
  if (!c) return BETA_GPU_ERR_ARG;
  if (!c->ndof) return fail(c, BETA_GPU_ERR_STATE, "upload the mesh first");
  cudaSetDevice(c->device);
  const size_t n = c->ndof;
  std::vector<unsigned char> r(n, 0);
  std::vector<double> pz, lz;  // zeros stand in for a missing array
  if (!prescribed) pz.assign(n, 0.0);
  if (!load) lz.assign(n, 0.0);
  const double* p = prescribed ? prescribed : pz.data();
  const double* l = load ? load : lz.data();
  // one pass: 0/1 restraints, finite values, no load on a restrained dof
  std::atomic<int> bad{0};  // 1 non-finite, 2 load on a restrained dof
  host_parallel(n, [&](size_t lo, size_t hi) {
    for (size_t i = lo; i < hi; ++i) {
      const unsigned char ri = restrained && restrained[i] ? 1 : 0;
      r[i] = ri;
      if (!std::isfinite(p[i]) || !std::isfinite(l[i])) {
        bad = 1;
        return;
      }
      if (ri && l[i] != 0.0) {
        int z = 0;
        bad.compare_exchange_strong(z, 2);
      }
    }
  });
  if (bad == 1) return fail(c, BETA_GPU_ERR_NOT_FINITE, "non-finite boundary data");
  if (bad == 2)
    return fail(c, BETA_GPU_ERR_LOAD_ON_RESTRAINED, "Cannot add load to a restrained degree of freedom.");
  if (c->have_pattern && r != c->h_rest) {
    c->have_pattern = false;
    invalidate_matrices(c);
  }
  c->h_rest = r;
  int rc;
  if ((rc = upload(c, c->rest, r.data(), n))) return rc;
  if ((rc = upload(c, c->presc, p, n))) return rc;
  if ((rc = upload(c, c->load, l, n))) return rc;
  CK(cudaStreamSynchronize(c->stream));
  c->have_bc = true;
  if (c->have64 || c->have32) invalidate_matrices(c);  // pseudo load depends on prescribed values
  return BETA_GPU_OK;
}

int beta_gpu_build_pattern(beta_gpu_ctx* c, long long* nnz_lower) {
  if (!c) return BETA_GPU_ERR_ARG;
  if (!c->ndof || !c->have_bc) return fail(c, BETA_GPU_ERR_STATE, "upload mesh and boundary conditions first");
  cudaSetDevice(c->device);
  // node-level structure only: the scalar FP64 layout is built the first
  // time an FP64 assembly needs it (ensure_scalar)
  TRACE("enter");
  std::string msg = build_pattern(c->nnode, c->nelem, c->nnpe, c->ndpn, c->h_conn.data(), c->h_first_dof.data(),
                                  c->h_rest.data(), c->P, false);
  if (!msg.empty()) return fail(c, BETA_GPU_ERR_UNSUPPORTED, msg);
  TRACE("host structure built");
  const HostPattern& P = c->P;
  int rc;
  if ((rc = upload(c, c->elems, P.elem_by_color.data(), P.elem_by_color.size()))) return rc;
  if ((rc = upload(c, c->slot, P.slot.data(), P.slot.size()))) return rc;
  if ((rc = upload(c, c->nrp, P.nrp.data(), P.nrp.size()))) return rc;
  if ((rc = upload(c, c->bsoff, P.bsoff.data(), P.bsoff.size()))) return rc;
  if (P.compact) {  // the SpMV reads the compact columns; the full ones stay on the host
    if ((rc = upload(c, c->bcol, P.ccol.data(), P.ccol.size()))) return rc;
    if ((rc = upload(c, c->cptr, P.cptr.data(), P.cptr.size()))) return rc;
  } else if ((rc = upload(c, c->bcol, P.bcol.data(), P.bcol.size()))) {
    return rc;
  }
  if ((rc = upload(c, c->ndiag, P.ndiag.data(), P.ndiag.size()))) return rc;
  if (P.run > 1 && (rc = upload(c, c->vpos, P.vpos.data(), P.vpos.size()))) return rc;
  TRACE("uploads queued");
  CK(cudaStreamSynchronize(c->stream));
  TRACE("uploads done");
  c->have_pattern = true;
  c->have_scalar = false;
  c->mfc_valid = false;  // the cache follows the colour order of the elements
  invalidate_matrices(c);
  if (nnz_lower) *nnz_lower = P.nnz_lower;
  return BETA_GPU_OK;
}

int beta_gpu_pattern_lower(beta_gpu_ctx* c, long long* row_ptr, int* col) {
  if (!c || !row_ptr || !col) return BETA_GPU_ERR_ARG;
  if (!c->have_pattern) return fail(c, BETA_GPU_ERR_STATE, "build the pattern first");
  export_lower_pattern(c->P, c->h_rest.data(), row_ptr, col);
  return BETA_GPU_OK;
}

int beta_gpu_pattern_lower_host(int nnode, int nelem, int nnpe, int ndpn, const int* conn, const int* first_dof,
                                const unsigned char* restrained, long long* nnz_lower, long long* row_ptr, int* col) {
  if (!conn || !first_dof || !restrained || !nnz_lower) return BETA_GPU_ERR_ARG;
  HostPattern P;
  std::vector<unsigned char> r((size_t)nnode * ndpn);
  for (size_t i = 0; i < r.size(); ++i) r[i] = restrained[i] ? 1 : 0;
  std::string msg = build_pattern(nnode, nelem, nnpe, ndpn, conn, first_dof, r.data(), P);
  if (!msg.empty()) return BETA_GPU_ERR_UNSUPPORTED;
  *nnz_lower = P.nnz_lower;
  if (row_ptr && col) export_lower_pattern(P, r.data(), row_ptr, col);
  return BETA_GPU_OK;
}

int beta_gpu_export_matrix(beta_gpu_ctx* c, int precision, int format, const char* path) {
  if (!c || !path) return BETA_GPU_ERR_ARG;
  if (!c->have_pattern) return fail(c, BETA_GPU_ERR_STATE, "build the pattern first");
  const size_t n = c->ndof;
  std::vector<long long> rp(n + 1);
  std::vector<int> col(c->P.nnz_lower);
  std::vector<double> val(c->P.nnz_lower);
  export_lower_pattern(c->P, c->h_rest.data(), rp.data(), col.data());
  int rc = beta_gpu_matrix_lower_values(c, precision, val.data(), nullptr);
  if (rc != BETA_GPU_OK) return rc;
  rc = beta_gpu_write_lower(path, format, (int)n, rp.data(), col.data(), val.data());
  if (rc != BETA_GPU_OK) return fail(c, rc, "writing the matrix failed");
  return BETA_GPU_OK;
}

int beta_gpu_assemble(beta_gpu_ctx* c, int what, int precision, double dt, double alpha) {
  if (!c) return BETA_GPU_ERR_ARG;
  if (!c->have_pattern || !c->have_mat) return fail(c, BETA_GPU_ERR_STATE, "pattern and materials required");
  cudaSetDevice(c->device);
  double ks = 1.0, ms = 0.0;
  const double* ugnl = nullptr;
  if (what == BETA_GPU_ASM_TANGENT) {
    if (c->kind != BETA_GPU_HEX8_ELASTIC)
      return fail(c, BETA_GPU_ERR_UNSUPPORTED, "the geometric-nonlinear tangent is for hex8 elasticity");
    if (!c->have_u) return fail(c, BETA_GPU_ERR_STATE, "the tangent needs a current solution");
    ugnl = c->u.p;
  } else if (what == BETA_GPU_ASM_MBAR) {
    if (!is_diffusion(c->kind)) return fail(c, BETA_GPU_ERR_UNSUPPORTED, "Mbar assembly is for diffusion elements");
    if (!(dt > 0)) return fail(c, BETA_GPU_ERR_ARG, "dt must be positive");
    ks = alpha * dt / dt;  // (a1 K + M)/dt with a1 = alpha*dt (formK_s, HeatTransferElement3DTransient.cpp:341)
    ms = 1.0 / dt;
  } else if (what != BETA_GPU_ASM_K) {
    return fail(c, BETA_GPU_ERR_ARG, "unknown assembly action");
  }
  ElemArgs A = elem_args(c);
  A.kscale = ks;
  A.mscale = ms;
  CK(cudaMemsetAsync(c->flags.p, 0, sizeof(unsigned), c->stream));
  int rc;
  if (precision == BETA_GPU_FP64) {
    if (!c->have_scalar) {
      std::string m2 = build_scalar(c->P, c->h_rest.data());
      if (!m2.empty()) return fail(c, BETA_GPU_ERR_UNSUPPORTED, m2);
      const HostPattern& P = c->P;
      if ((rc = upload(c, c->soff, P.soff.data(), P.soff.size()))) return rc;
      if ((rc = upload(c, c->ssoff, P.ssoff.data(), P.ssoff.size()))) return rc;
      if ((rc = upload(c, c->scol, P.scol.data(), P.scol.size()))) return rc;
      if ((rc = upload(c, c->sdiag, P.sdiag.data(), P.sdiag.size()))) return rc;
      CK(cudaStreamSynchronize(c->stream));
      c->have_scalar = true;
    }
    A.soff = c->soff.p;
    A.ssoff = c->ssoff.p;
    CK(c->sval.alloc(c->P.ssoff.back()));
    CK(c->pseudo.alloc(c->ndof));
    CK(cudaMemsetAsync(c->sval.p, 0, sizeof(double) * c->sval.n, c->stream));
    CK(cudaMemsetAsync(c->pseudo.p, 0, sizeof(double) * c->ndof, c->stream));
    A.sval = c->sval.p;
    A.pseudo = c->pseudo.p;
    if ((rc = launch_assembly<double>(c, A, ugnl))) return rc;
    launch(c, k_set_restrained_diag64, grid_for(c, c->ndof, 256), 256, 0, c->ndof, c->rest.p, c->sdiag.p,
                                                                              c->sval.p);
    CKL("k_set_restrained_diag64");
    c->have64 = true;
    c->what64 = what;
    c->kscale64 = ks;
    c->mscale64 = ms;
  } else if (precision == BETA_GPU_FP32) {
    const size_t nv = (size_t)c->P.nchunk * 32 * c->ndpn * c->ndpn;
    CK(c->bval.alloc(nv));
    CK(cudaMemsetAsync(c->bval.p, 0, sizeof(float) * nv, c->stream));
    A.bval = c->bval.p;
    if ((rc = launch_assembly<float>(c, A, ugnl))) return rc;
    const int g = grid_for(c, c->nnode, 256);
    if (c->ndpn == 3) launch(c, k_set_restrained_diag32<3>, g, 256, 0, c->nnode, c->rest.p, c->bsoff.p, c->ndiag.p, c->bval.p);
    else if (c->ndpn == 2) launch(c, k_set_restrained_diag32<2>, g, 256, 0, c->nnode, c->rest.p, c->bsoff.p, c->ndiag.p, c->bval.p);
    else launch(c, k_set_restrained_diag32<1>, g, 256, 0, c->nnode, c->rest.p, c->bsoff.p, c->ndiag.p, c->bval.p);
    CKL("k_set_restrained_diag32");
    c->have32 = true;
    c->what32 = what;
    c->kscale32 = ks;
    c->mscale32 = ms;
    c->minv_kind = -1;
  } else {
    return fail(c, BETA_GPU_ERR_ARG, "unknown precision");
  }
  unsigned f = 0;
  if ((rc = read_flags(c, &f))) return rc;
  if (f & kFlagNegDiag) {
    if (precision == BETA_GPU_FP64) c->have64 = false; else c->have32 = false;
    return fail(c, BETA_GPU_ERR_NEGDIAG, "BasicElement::bad diagonal in K (element diagonal <= 0)");
  }
  return BETA_GPU_OK;
}

int beta_gpu_matrix_lower_values(beta_gpu_ctx* c, int precision, double* vals, double* pseudo_load) {
  if (!c || !vals) return BETA_GPU_ERR_ARG;
  cudaSetDevice(c->device);
  if (precision == BETA_GPU_FP64) {
    if (!c->have64) return fail(c, BETA_GPU_ERR_STATE, "no FP64 matrix assembled");
    std::vector<double> h(c->sval.n);
    CK(d2h(c, h.data(), c->sval.p, sizeof(double) * h.size()));
    if (pseudo_load)
      CK(d2h(c, pseudo_load, c->pseudo.p, sizeof(double) * c->ndof));
    CK(cudaStreamSynchronize(c->stream));
    export_lower_values_scalar(c->P, c->h_rest.data(), h.data(), vals);
  } else {
    if (!c->have32) return fail(c, BETA_GPU_ERR_STATE, "no FP32 matrix assembled");
    std::vector<float> h(c->bval.n);
    CK(d2h(c, h.data(), c->bval.p, sizeof(float) * h.size()));
    CK(cudaStreamSynchronize(c->stream));
    export_lower_values_block(c->P, c->h_rest.data(), h.data(), vals);
    if (pseudo_load) std::memset(pseudo_load, 0, sizeof(double) * c->ndof);
  }
  return BETA_GPU_OK;
}

int beta_gpu_solve(beta_gpu_ctx* c, const beta_gpu_solve_opts* o, beta_gpu_solve_stats* stats) {
  if (!c || !o) return BETA_GPU_ERR_ARG;
  cudaSetDevice(c->device);
  if (stats) std::memset(stats, 0, sizeof(*stats));
  int rc;
  if ((rc = ensure_workspace(c))) return rc;
  const int n = c->ndof;
  const bool last = o->use_last_solution && c->have_u;
  ProfAcc prof;
  prof.on = o->reserved & 1;
  CK(cudaEventRecord(c->ev0, c->stream));
  int status;
  if (o->mode == BETA_GPU_MODE_FP64) {
    if (!c->have64) return fail(c, BETA_GPU_ERR_STATE, "assemble in FP64 before an FP64 solve");
    if (c->what64 != BETA_GPU_ASM_K) return fail(c, BETA_GPU_ERR_STATE, "static solve needs the K assembly");
    if (!c->rhs_staged)
      launch(c, k_rhs64, grid_for(c, n, 256), 256, 0, n, c->rest.p, c->presc.p, c->load.p, c->pseudo.p, c->b64.p);
    if (last) CK(cudaMemcpyAsync(c->x64.p, c->u.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, c->stream));
    else CK(cudaMemsetAsync(c->x64.p, 0, sizeof(double) * n, c->stream));
    CKL("k_rhs64");
    status = fp64_core(c, o, stats, &prof);
  } else if (o->mode == BETA_GPU_MODE_MPIR) {
    if (!c->have32) return fail(c, BETA_GPU_ERR_STATE, "assemble in FP32 before a mixed-precision solve");
    if (c->what32 != BETA_GPU_ASM_K) return fail(c, BETA_GPU_ERR_STATE, "static solve needs the K assembly");
    // ||b|| with b = rest ? presc : load - K ubar_ext
    launch(c, k_ext64, grid_for(c, n, 256), 256, 0, n, c->rest.p, c->presc.p, nullptr, c->t64.p);
    if ((rc = mf_apply(c, 1.0, c->t64.p, 0.0, nullptr, 0.0, c->y64.p))) return rc;
    launch(c, k_rhs_elim64, grid_for(c, n, 256), 256, 0, n, c->rest.p, c->presc.p, c->load.p, c->y64.p,
                                                            c->b64.p, c->sums.p, c->partials.p, c->ticket.p);
    CKL("k_rhs_elim64");
    double bb;
    if ((rc = read_sums(c, 1, &bb))) return rc;
    launch(c, k_ext64, grid_for(c, n, 256), 256, 0, n, c->rest.p, c->presc.p, last ? c->u.p : nullptr, c->x64.p);
    CKL("k_ext64");
    status = mpir_dispatch(c, !last, o, 1.0, 0.0, nullptr, 0.0, c->load.p, std::sqrt(bb), stats, &prof);
    if (stats && (status == BETA_GPU_OK || status == BETA_GPU_MAXIT)) {
      // true FP64 residual of the returned iterate
      if ((rc = mf_apply(c, 1.0, c->x64.p, 0.0, nullptr, 0.0, c->y64.p))) return rc;
      if (c->zrep_on)
        launch(c, k_zdiag_apply, grid_for(c, n, 256), 256, 0, n, (const unsigned char*)c->zrep.p, c->zdiag,
               (const double*)c->x64.p, c->y64.p);
      launch(c, k_residual64, grid_for(c, n, 256), 256, 0, n, c->rest.p, c->load.p, c->y64.p, c->x64.p,
                                                              c->r64.p, c->sums.p, c->partials.p, c->ticket.p);
      double s2[2];
      if ((rc = read_sums(c, 2, s2))) return rc;
      stats->true_rel_residual = bb > 0 ? std::sqrt(s2[0] / bb) : std::sqrt(s2[0]);
    }
  } else {
    return fail(c, BETA_GPU_ERR_ARG, "unknown solve mode");
  }
  CK(cudaEventRecord(c->ev1, c->stream));
  CK(cudaEventSynchronize(c->ev1));
  if (status == BETA_GPU_OK || status == BETA_GPU_MAXIT) {
    CK(cudaMemcpyAsync(c->u.p, c->x64.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, c->stream));
    c->have_u = true;
  }
  if (stats) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    stats->ms_solve = ms;
    stats->ms_spmv_avg = prof.launches ? prof.ms / prof.launches : 0.0;
  }
  if (status == BETA_GPU_MAXIT) c->err = "Solution not converged...";
  if (status == BETA_GPU_BREAKDOWN) c->err = "PCG breakdown (p.Ap <= 0 or non-finite)";
  return status;
}

int beta_gpu_solve_rhs(beta_gpu_ctx* c, const double* b, const double* x0, const beta_gpu_solve_opts* o,
                       beta_gpu_solve_stats* stats) {
  if (!c || !b || !o) return BETA_GPU_ERR_ARG;
  if (c->ndof <= 0 || !c->have_bc) return fail(c, BETA_GPU_ERR_STATE, "mesh and restraints required");
  cudaSetDevice(c->device);
  const int n = c->ndof;
  if (!all_finite(b, (size_t)n) || (x0 && !all_finite(x0, (size_t)n)))
    return fail(c, BETA_GPU_ERR_NOT_FINITE, "non-finite right-hand side or initial guess");
  int rc;
  if ((rc = ensure_workspace(c))) return rc;
  CK(c->rhs_presc.alloc(n));
  CK(c->rhs_load.alloc(n));
  CK(h2d(c, c->b64.p, b, sizeof(double) * n));
  if (x0) {
    CK(h2d(c, c->u.p, x0, sizeof(double) * n));
    c->have_u = true;
  }
  CK(cudaStreamSynchronize(c->stream));  // b and x0 read before any way out (pinned inputs copy asynchronously)
  beta_gpu_solve_opts o2 = *o;
  o2.use_last_solution = x0 ? 1 : 0;
  if (o->mode == BETA_GPU_MODE_FP64) {
    // the scalar FP64 matrix is already eliminated: b is its right-hand side as is
    c->rhs_staged = true;
    rc = beta_gpu_solve(c, &o2, stats);
    c->rhs_staged = false;
    return rc;
  }
  // prescribed := b on restrained rows, load := b + K x_ext on free rows, so
  // that the solver's right-hand side load - K x_ext equals b
  CK(cudaMemcpyAsync(c->rhs_presc.p, c->b64.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, c->stream));
  launch(c, k_ext64, grid_for(c, n, 256), 256, 0, n, c->rest.p, (const double*)c->b64.p, (const double*)nullptr,
         c->t64.p);
  if ((rc = mf_apply(c, 1.0, c->t64.p, 0.0, nullptr, 0.0, c->y64.p))) return rc;
  launch(c, k_load_from_rhs, grid_for(c, n, 256), 256, 0, n, c->rest.p, (const double*)c->b64.p,
         (const double*)c->y64.p, c->rhs_load.p);
  CKL("k_load_from_rhs");
  std::swap(c->presc.p, c->rhs_presc.p);
  std::swap(c->load.p, c->rhs_load.p);
  rc = beta_gpu_solve(c, &o2, stats);
  std::swap(c->presc.p, c->rhs_presc.p);
  std::swap(c->load.p, c->rhs_load.p);
  return rc;
}

int beta_gpu_download(beta_gpu_ctx* c, double* u) {
  if (!c || !u) return BETA_GPU_ERR_ARG;
  if (!c->have_u) return fail(c, BETA_GPU_ERR_STATE, "no solution");
  cudaSetDevice(c->device);
  CK(d2h(c, u, c->u.p, sizeof(double) * c->ndof));
  CK(cudaStreamSynchronize(c->stream));
  return BETA_GPU_OK;
}

int beta_gpu_matvec(beta_gpu_ctx* c, int precision, const double* x, double* y) {
  if (!c || !x || !y) return BETA_GPU_ERR_ARG;
  cudaSetDevice(c->device);
  int rc;
  if (precision == BETA_GPU_FP64 ? !c->have64 : !c->have32)  // checked before x is queued for copying
    return fail(c, BETA_GPU_ERR_STATE, precision == BETA_GPU_FP64 ? "no FP64 matrix" : "no FP32 matrix");
  if ((rc = ensure_workspace(c))) return rc;
  const int n = c->ndof;
  CK(h2d(c, c->t64.p, x, sizeof(double) * n));
  if (precision == BETA_GPU_FP64) {
    ScalarMat A{n, c->P.nsslice, c->ssoff.p, c->scol.p, c->sval.p};
    launch(c, k_spmv_s, grid_for(c, (long long)c->P.nsslice * 32, 256), 256, 0, A, c->t64.p, c->y64.p, nullptr);
  } else {
    BlockMat A{c->nnode, c->P.nslice, c->bsoff.p, c->bcol.p, c->bval.p, c->P.compact ? c->cptr.p : nullptr};
    const int g = grid_for(c, (long long)c->P.nslice * 32, 256), gn = grid_for(c, n, 256);
    launch(c, k_to32, gn, 256, 0, (long long)n, (const double*)c->t64.p, 1.0, c->v32[0].p);
    const float* xv = c->v32[0].p;
    float* yv = c->v32[1].p;
    if (c->P.run == 3) {
      if (c->ndpn == 3) launch(c, k_spmv_b<3, 3>, g, 256, 0, A, xv, yv);
      else if (c->ndpn == 2) launch(c, k_spmv_b<2, 3>, g, 256, 0, A, xv, yv);
      else launch(c, k_spmv_b<1, 3>, g, 256, 0, A, xv, yv);
    } else {
      if (c->ndpn == 3) launch(c, k_spmv_b<3>, g, 256, 0, A, xv, yv);
      else if (c->ndpn == 2) launch(c, k_spmv_b<2>, g, 256, 0, A, xv, yv);
      else launch(c, k_spmv_b<1>, g, 256, 0, A, xv, yv);
    }
    CK(cudaMemsetAsync(c->y64.p, 0, sizeof(double) * n, c->stream));
    launch(c, k_axpy_from32, gn, 256, 0, (long long)n, c->y64.p, 1.0, (const float*)c->v32[1].p);
  }
  CKL("matvec");
  CK(d2h(c, y, c->y64.p, sizeof(double) * n));
  CK(cudaStreamSynchronize(c->stream));
  return BETA_GPU_OK;
}

int beta_gpu_internal_force(beta_gpu_ctx* c, const double* u, double* f) {
  if (!c || !u || !f) return BETA_GPU_ERR_ARG;
  if (!c->have_pattern || !c->have_mat) return fail(c, BETA_GPU_ERR_STATE, "pattern and materials required");
  cudaSetDevice(c->device);
  int rc;
  if ((rc = ensure_workspace(c))) return rc;
  CK(h2d(c, c->t64.p, u, sizeof(double) * c->ndof));
  if ((rc = mf_apply(c, 1.0, c->t64.p, 0.0, nullptr, 0.0, c->y64.p))) return rc;
  CK(d2h(c, f, c->y64.p, sizeof(double) * c->ndof));
  CK(cudaStreamSynchronize(c->stream));
  return BETA_GPU_OK;
}

int beta_gpu_element_outputs(beta_gpu_ctx* c, const double* u, double* per_element, double* totals) {
  if (!c) return BETA_GPU_ERR_ARG;
  if (c->kind != BETA_GPU_HEX8_ELASTIC && c->kind != BETA_GPU_QUAD4_PSTRESS)
    return fail(c, BETA_GPU_ERR_UNSUPPORTED, "element outputs are defined for the elasticity elements");
  if (!c->have_mat || !c->ndof) return fail(c, BETA_GPU_ERR_STATE, "mesh and materials required");
  if (!u && !c->have_u) return fail(c, BETA_GPU_ERR_STATE, "no solution");
  cudaSetDevice(c->device);
  int rc;
  if ((rc = ensure_workspace(c))) return rc;
  const double* ud = c->u.p;
  if (u) {
    CK(h2d(c, c->t64.p, u, sizeof(double) * c->ndof));
    ud = c->t64.p;
  }
  const int ns = c->kind == BETA_GPU_HEX8_ELASTIC ? 6 : 3, w = 2 * ns + 2;
  DBuf<double> out;
  CK(out.alloc((size_t)c->nelem * w));
  const int grid = (c->nelem + 127) / 128;
  const int* eg = c->have_egroup ? c->egroup.p : nullptr;
  if (c->kind == BETA_GPU_HEX8_ELASTIC)
    k_outputs_hex8<<<grid, 128, 0, c->stream>>>(c->nelem, c->xyz.p, c->conn.p, c->gparams.p, eg, c->nparams,
                                                c->gt.p, ud, out.p);
  else
    k_outputs_quad4<<<grid, 128, 0, c->stream>>>(c->nelem, c->xyz.p, c->conn.p, c->gparams.p, eg, c->nparams,
                                                 c->gt.p, ud, out.p);
  c->n_launch += 1;
  CKL("element outputs");
  std::vector<double> h;
  double* dst = per_element;
  if (!dst) {
    h.resize((size_t)c->nelem * w);
    dst = h.data();
  }
  CK(d2h(c, dst, out.p, sizeof(double) * (size_t)c->nelem * w));
  CK(cudaStreamSynchronize(c->stream));
  if (totals) {  // element order: the same sum on every call
    for (int k = 0; k < w; ++k) totals[k] = 0.0;
    for (long long e = 0; e < c->nelem; ++e)
      for (int k = 0; k < w; ++k) totals[k] += dst[e * w + k];
  }
  return BETA_GPU_OK;
}

int beta_gpu_heat_set_state(beta_gpu_ctx* c, const double* u0) {
  if (!c || !u0) return BETA_GPU_ERR_ARG;
  if (!is_diffusion(c->kind)) return fail(c, BETA_GPU_ERR_UNSUPPORTED, "transient state is for diffusion");
  cudaSetDevice(c->device);
  if (!all_finite(u0, c->ndof)) return fail(c, BETA_GPU_ERR_NOT_FINITE, "non-finite initial field");
  int rc;
  if ((rc = upload(c, c->us, u0, c->ndof))) return rc;
  CK(cudaStreamSynchronize(c->stream));
  c->have_us = true;
  c->have_dprev = false;
  return BETA_GPU_OK;
}

int beta_gpu_heat_get_state(beta_gpu_ctx* c, double* u) {
  if (!c || !u) return BETA_GPU_ERR_ARG;
  if (!c->have_us) return fail(c, BETA_GPU_ERR_STATE, "no transient state");
  cudaSetDevice(c->device);
  CK(d2h(c, u, c->us.p, sizeof(double) * c->ndof));
  CK(cudaStreamSynchronize(c->stream));
  return BETA_GPU_OK;
}

int beta_gpu_heat_run(beta_gpu_ctx* c, double dt, double alpha, int nsteps, const beta_gpu_solve_opts* o,
                      beta_gpu_solve_stats* stats, int* total_iterations) {
  if (!c || !o || nsteps < 0) return BETA_GPU_ERR_ARG;
  if (!is_diffusion(c->kind) || !c->have_us) return fail(c, BETA_GPU_ERR_STATE, "diffusion mesh and state required");
  cudaSetDevice(c->device);
  int rc;
  const int prec = o->mode == BETA_GPU_MODE_MPIR ? BETA_GPU_FP32 : BETA_GPU_FP64;
  const double a1 = alpha * dt, a2 = (1.0 - alpha) * dt;
  const double ks = a1 / dt, ms = 1.0 / dt, kf = (a1 + a2) / dt;
  bool have = prec == BETA_GPU_FP64 ? (c->have64 && c->what64 == BETA_GPU_ASM_MBAR && c->kscale64 == ks && c->mscale64 == ms)
                                    : (c->have32 && c->what32 == BETA_GPU_ASM_MBAR && c->kscale32 == ks && c->mscale32 == ms);
  if (!have && (rc = beta_gpu_assemble(c, BETA_GPU_ASM_MBAR, prec, dt, alpha))) return rc;
  if ((rc = ensure_workspace(c))) return rc;
  CK(c->dprev.alloc(c->ndof));
  const int n = c->ndof;
  int total = 0;
  beta_gpu_solve_stats s;
  std::memset(&s, 0, sizeof(s));
  ProfAcc prof;
  prof.on = o->reserved & 1;
  for (int step = 0; step < nsteps; ++step) {
    if (prec == BETA_GPU_FP64) {
      // F = load - (a1+a2)/dt K u_s (formF_s_new) on free rows, + pseudo load;
      // the load holds the step's external heat input (point loads, surface
      // flux: beta_gpu_surface_flux_load), as Equations adds it per step
      if ((rc = mf_apply(c, -kf, c->us.p, 0.0, nullptr, 0.0, c->y64.p))) return rc;
      launch(c, k_axpy64, grid_for(c, n, 256), 256, 0, n, c->y64.p, 1.0, (const double*)c->load.p);
      launch(c, k_rhs64, grid_for(c, n, 256), 256, 0, n, c->rest.p, c->presc.p, c->y64.p, c->pseudo.p, c->b64.p);
      if (c->have_dprev)  // start from the last increment (a smooth field changes little per step)
        CK(cudaMemcpyAsync(c->x64.p, c->dprev.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, c->stream));
      else
        CK(cudaMemsetAsync(c->x64.p, 0, sizeof(double) * n, c->stream));
      CKL("k_rhs64");
      rc = fp64_core(c, o, &s, &prof);
    } else {
      // Scale of the step: ||(M/dt) u_s||, the right-hand side of the
      // backward-Euler system for the new state.  The increment solved below
      // has the same residual vector, but its own right-hand side shrinks as
      // the field smooths out, below what an FP64 residual of a smooth field
      // can resolve; the stop is taken relative to the larger of the two.
      if ((rc = mf_apply(c, 0.0, c->us.p, 0.0, nullptr, ms, c->y64.p))) return rc;
      launch(c, k_norm2_diff, grid_for(c, n, 256), 256, 0, n, (const double*)c->y64.p, (const double*)nullptr,
             c->sums.p, c->partials.p, c->ticket.p);
      CKL("k_norm2_diff");
      double ff;
      if ((rc = read_sums(c, 1, &ff))) return rc;
      // b = rest ? presc : load - (kf K u_s + Mbar ubar_ext) ; r = load - (K(ks x + kf u_s) + ms M x)
      launch(c, k_ext64, grid_for(c, n, 256), 256, 0, n, c->rest.p, c->presc.p, nullptr, c->t64.p);
      if ((rc = mf_apply(c, ks, c->t64.p, kf, c->us.p, ms, c->y64.p))) return rc;
      launch(c, k_rhs_elim64, grid_for(c, n, 256), 256, 0, n, c->rest.p, c->presc.p, (const double*)c->load.p, c->y64.p,
                                                              c->b64.p, c->sums.p, c->partials.p, c->ticket.p);
      CKL("k_rhs_elim64");
      double bb;
      if ((rc = read_sums(c, 1, &bb))) return rc;
      if (c->have_dprev)  // start from the last increment (a smooth field changes little per step)
        launch(c, k_ext64, grid_for(c, n, 256), 256, 0, n, c->rest.p, c->presc.p, (const double*)c->dprev.p,
               c->x64.p);
      else
        CK(cudaMemcpyAsync(c->x64.p, c->t64.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, c->stream));
      rc = mpir_dispatch(c, !c->have_dprev, o, ks, kf, c->us.p, ms, c->load.p, std::sqrt(std::max(bb, ff)), &s,
                         &prof);
    }
    if (rc != BETA_GPU_OK) {
      if (stats) *stats = s;
      return rc;
    }
    total += s.iterations;
    s.ms_spmv_avg = prof.launches ? prof.ms / prof.launches : 0.0;
    // u_s <- u_s + delta (DiffusionModel.cpp:800-818)
    launch(c, k_axpy64, grid_for(c, n, 256), 256, 0, n, c->us.p, 1.0, c->x64.p);
    CKL("k_axpy64");
    CK(cudaMemcpyAsync(c->dprev.p, c->x64.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, c->stream));
    c->have_dprev = true;
  }
  if (stats) *stats = s;
  if (total_iterations) *total_iterations = total;
  return BETA_GPU_OK;
}

int beta_gpu_set_solution(beta_gpu_ctx* c, const double* u) {
  if (!c || !u) return BETA_GPU_ERR_ARG;
  if (!c->have_pattern) return fail(c, BETA_GPU_ERR_STATE, "mesh and pattern required");
  if (!all_finite(u, c->ndof)) return fail(c, BETA_GPU_ERR_NOT_FINITE, "non-finite solution");
  cudaSetDevice(c->device);
  int rc;
  if ((rc = ensure_workspace(c))) return rc;
  CK(h2d(c, c->u.p, u, sizeof(double) * c->ndof));
  CK(cudaStreamSynchronize(c->stream));
  c->have_u = true;
  return BETA_GPU_OK;
}

int beta_gpu_internal_force_nonlinear(beta_gpu_ctx* c, const double* u, double* f) {
  if (!c || !u || !f) return BETA_GPU_ERR_ARG;
  if (!c->have_pattern || !c->have_mat) return fail(c, BETA_GPU_ERR_STATE, "pattern and materials required");
  if (c->kind != BETA_GPU_HEX8_ELASTIC)
    return fail(c, BETA_GPU_ERR_UNSUPPORTED, "the geometric-nonlinear internal force is for hex8 elasticity");
  cudaSetDevice(c->device);
  int rc;
  if ((rc = ensure_workspace(c))) return rc;
  CK(h2d(c, c->t64.p, u, sizeof(double) * c->ndof));
  if ((rc = fint_apply(c, c->t64.p, c->y64.p))) return rc;
  CK(d2h(c, f, c->y64.p, sizeof(double) * c->ndof));
  CK(cudaStreamSynchronize(c->stream));
  return BETA_GPU_OK;
}

// BasicModel::iterate (BasicModel.cpp:1244-1381) with the hex8 element in its
// geometric-nonlinear form.  Each iteration: the internal force f(u) in FP64
// (getGlobalForces), R = load - f on free dofs (0 on restrained ones), stop
// once max |R| < opts->max_residual; the tangent K_T(u) (assembleK at the
// current solution); K_T d = R; u += d on free dofs
// (incrementalSolutionUsingResidual + addIncrementalDisplacements,
// equation.cpp:1638-1720).  FP64 steps solve with the FP64 tangent and the
// reference's PCG from the current solution as initial guess, as the
// reference passes it; mixed steps assemble the tangent in FP32 and reduce
// the FP32 residual by opts->solve.inner_tol with block-Jacobi PCG -- the
// FP64 residual of the next iteration refines each step (an inexact Newton).
int beta_gpu_newton(beta_gpu_ctx* c, const beta_gpu_newton_opts* o, beta_gpu_newton_stats* stats,
                    double* history) {
  if (stats) std::memset(stats, 0, sizeof(*stats));
  if (!c || !o) return BETA_GPU_ERR_ARG;
  if (c->kind != BETA_GPU_HEX8_ELASTIC)
    return fail(c, BETA_GPU_ERR_UNSUPPORTED, "the geometric-nonlinear Newton loop is for hex8 elasticity");
  if (!c->have_pattern || !c->have_mat || !c->have_bc)
    return fail(c, BETA_GPU_ERR_STATE, "mesh, pattern, materials and boundary conditions required");
  cudaSetDevice(c->device);
  int rc;
  if ((rc = ensure_workspace(c))) return rc;
  CK(c->dmax.alloc(1));
  const int n = c->ndof;
  const int max_newton = o->max_newton > 0 ? o->max_newton : 400;
  const double tol = o->max_residual > 0 ? o->max_residual : 1e-10;
  const bool mixed = o->solve.mode == BETA_GPU_MODE_MPIR;
  if (!(o->use_last_solution && c->have_u)) {
    launch(c, k_ext64, grid_for(c, n, 256), 256, 0, n, c->rest.p, c->presc.p, (const double*)nullptr, c->u.p);
    CKL("k_ext64");
  }
  c->have_u = true;
  int status = BETA_GPU_OK, it = 0;
  long long lin = 0;
  double maxr = 0.0;
  for (;; ++it) {
    if ((rc = fint_apply(c, c->u.p, c->y64.p))) return rc;
    CK(cudaMemsetAsync(c->dmax.p, 0, sizeof(unsigned long long), c->stream));
    launch(c, k_newton_residual, grid_for(c, n, 256), 256, 0, n, c->rest.p, (const double*)c->load.p,
           (const double*)c->y64.p, c->r64.p, c->dmax.p);
    CKL("k_newton_residual");
    unsigned long long bits = 0;
    CK(d2h(c, c->h_sums, c->dmax.p, sizeof(bits)));
    CK(cudaStreamSynchronize(c->stream));
    std::memcpy(&bits, c->h_sums, sizeof(bits));
    std::memcpy(&maxr, &bits, sizeof(maxr));
    if (history) history[it] = maxr;
    if (!(maxr < 1e300)) { status = BETA_GPU_BREAKDOWN; break; }
    if (maxr < tol) break;
    if (it >= max_newton) { status = BETA_GPU_MAXIT; break; }
    if ((rc = beta_gpu_assemble(c, BETA_GPU_ASM_TANGENT, mixed ? BETA_GPU_FP32 : BETA_GPU_FP64, 0.0, 1.0)) !=
        BETA_GPU_OK) {
      status = rc;
      break;
    }
    if (!mixed) {
      CK(cudaMemcpyAsync(c->b64.p, c->r64.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, c->stream));
      CK(cudaMemcpyAsync(c->x64.p, c->u.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, c->stream));
      beta_gpu_solve_stats ls;
      std::memset(&ls, 0, sizeof(ls));
      rc = fp64_core(c, &o->solve, &ls, nullptr);
      lin += ls.iterations;
      if (rc != BETA_GPU_OK && rc != BETA_GPU_MAXIT) { status = rc; break; }
      launch(c, k_add_free64, grid_for(c, n, 256), 256, 0, n, c->rest.p, c->u.p, (const double*)c->x64.p);
    } else {
      int its = 0;
      rc = newton_step32<3>(c, &o->solve, &its);
      lin += its;
      if (rc != BETA_GPU_OK) { status = rc; break; }
      launch(c, k_add_free_from32, grid_for(c, n, 256), 256, 0, n, c->rest.p, c->u.p,
             (const float*)c->v32[0].p);
    }
    CKL("Newton update");
  }
  if (stats) {
    stats->status = status;
    stats->iterations = it;
    stats->linear_iterations = (int)std::min<long long>(lin, 2000000000LL);
    stats->max_residual = maxr;
  }
  if (status == BETA_GPU_MAXIT) c->err = "Newton iterations exhausted before max |residual| < max_residual";
  if (status == BETA_GPU_BREAKDOWN) c->err = "non-finite residual in the Newton loop";
  return status;
}

// Jacobi-PCG on caller-owned device CSR; scratch from cudaMalloc, freed on return.
int beta_gpu_csr_pcg_device(int n, const int* d_rp, const int* d_ci, const double* d_v, const double* d_b,
                            double* d_x, int stop_rule, double tol, int maxit, void* stream_ptr,
                            beta_gpu_solve_stats* stats) {
  if (stats) std::memset(stats, 0, sizeof(*stats));
  if (n <= 0 || !d_rp || !d_ci || !d_v || !d_b || !d_x || !(tol > 0)) {
    if (stats) stats->status = BETA_GPU_ERR_ARG;
    return BETA_GPU_ERR_ARG;
  }
  cudaStream_t s = (cudaStream_t)stream_ptr;
  int dev = 0, nsm = 148;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
    cudaGetLastError();
    return BETA_GPU_ERR_CUDA;
  }
  const int max_grid = nsm * 8;
  auto grid = [&](long long items) { long long g = (items + 255) / 256; return (int)std::max(1LL, std::min<long long>(g, max_grid)); };
  // scratch: r, p, q, dinv (n each), partials, state, counters
  const size_t need = sizeof(double) * ((size_t)4 * n + (size_t)max_grid * 4 + 8) + sizeof(PcgState) + 64;
  unsigned char* scratch = nullptr;
  if (cudaMalloc(&scratch, need) != cudaSuccess) { cudaGetLastError(); return BETA_GPU_ERR_OOM; }
  double* r = (double*)scratch;
  double* p = r + n;
  double* q = p + n;
  double* dinv = q + n;
  double* partials = dinv + n;
  double* sums = partials + (size_t)max_grid * 4;
  PcgState* st = (PcgState*)(sums + 8);
  unsigned* flags = (unsigned*)(st + 1);
  unsigned* ticket = flags + 1;
  int status = BETA_GPU_OK;
  PcgState h;
  std::memset(&h, 0, sizeof(h));
  h.rule = stop_rule == BETA_GPU_STOP_REF ? kStopRef : kStopRB;
  h.tol2 = tol * tol;
  h.maxit = maxit > 0 ? maxit : 10000;
  CsrMat A{n, d_rp, d_ci, d_v};
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, s);
  cudaMemsetAsync(flags, 0, 2 * sizeof(unsigned), s);
  cudaMemcpyAsync(st, &h, sizeof(h), cudaMemcpyHostToDevice, s);
  k_csr_dinv<<<grid(n), 256, 0, s>>>(A, dinv, flags);
  k_csr_spmv<<<grid((long long)n * 8), 256, 0, s>>>(A, d_x, r, d_b);
  k_start_s<<<grid(n), 256, 0, s>>>(n, d_x, r, d_b, dinv, p, st, partials);
  unsigned hf[2] = {0, 0};
  cudaMemcpyAsync(hf, flags, sizeof(hf), cudaMemcpyDeviceToHost, s);
  if (cudaStreamSynchronize(s) != cudaSuccess) status = BETA_GPU_ERR_CUDA;
  else if (hf[0] & 8u) status = BETA_GPU_ERR_ZERODIAG;
  else if (hf[0] & 16u) status = BETA_GPU_ERR_NEGDIAG;
  while (status == BETA_GPU_OK) {
    for (int k = 0; k < 16; ++k) {
      k_csr_spmv_dot<<<grid((long long)n * 8), 256, 0, s>>>(A, p, q, st, partials);
      k_update_s<<<grid(n), 256, 0, s>>>(n, d_x, r, p, q, dinv, st, partials);
      k_pupd_s<<<grid(n), 256, 0, s>>>(n, p, r, dinv, st);
    }
    cudaMemcpyAsync(&h, st, sizeof(h), cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) { status = BETA_GPU_ERR_CUDA; break; }
    if (h.done) {
      status = h.status == kStatusOk ? BETA_GPU_OK : (h.status == kStatusMaxit ? BETA_GPU_MAXIT : BETA_GPU_BREAKDOWN);
      break;
    }
  }
  if (status == BETA_GPU_OK || status == BETA_GPU_MAXIT) {
    k_csr_spmv<<<grid((long long)n * 8), 256, 0, s>>>(A, d_x, q, d_b);
    k_norm2_diff<<<grid(n), 256, 0, s>>>(n, q, nullptr, sums, partials, ticket);
    double rr = 0.0;
    cudaMemcpyAsync(&rr, sums, sizeof(double), cudaMemcpyDeviceToHost, s);
    cudaEventRecord(e1, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) status = BETA_GPU_ERR_CUDA;
    if (stats) {
      stats->iterations = h.iter;
      stats->final_norm = h.last;
      stats->true_rel_residual = h.bb > 0 ? std::sqrt(rr / h.bb) : std::sqrt(rr);
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      stats->ms_solve = ms;
    }
  }
  if (stats) stats->status = status;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(scratch);
  if (cudaGetLastError() != cudaSuccess && status == BETA_GPU_OK) status = BETA_GPU_ERR_CUDA;
  return status;
}

// Jacobi-PCG on caller-owned device CSR with scratch in g_noalloc_scratch:
// no cudaMalloc/cudaFree, no event creation.  See include/beta_gpu.h.
int beta_gpu_csr_pcg_device_noalloc(int n, const int* d_rp, const int* d_ci, const double* d_v, const double* d_b,
                                    double* d_x, int stop_rule, double tol, int maxit, void* stream_ptr,
                                    beta_gpu_solve_stats* stats) {
  if (stats) std::memset(stats, 0, sizeof(*stats));
  if (n > BETA_GPU_NOALLOC_MAX_ROWS) {
    if (stats) stats->status = BETA_GPU_ERR_TOO_LARGE;
    return BETA_GPU_ERR_TOO_LARGE;
  }
  if (n <= 0 || !d_rp || !d_ci || !d_v || !d_b || !d_x || !(tol > 0)) {
    if (stats) stats->status = BETA_GPU_ERR_ARG;
    return BETA_GPU_ERR_ARG;
  }
  cudaStream_t s = (cudaStream_t)stream_ptr;
  int dev = 0, nsm = 148;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
    cudaGetLastError();
    return BETA_GPU_ERR_CUDA;
  }
  unsigned char* scratch = nullptr;
  if (noalloc_scratch_address(&scratch) != cudaSuccess) {
    cudaGetLastError();
    return BETA_GPU_ERR_CUDA;
  }
  const int max_grid = std::min(nsm * 8, BETA_GPU_NOALLOC_MAX_BLOCKS);
  auto grid = [&](long long items) { long long g = (items + 255) / 256; return (int)std::max(1LL, std::min<long long>(g, max_grid)); };
  // layout inside the fixed array (sized for BETA_GPU_NOALLOC_MAX_ROWS rows)
  double* r = (double*)scratch;
  double* p = r + BETA_GPU_NOALLOC_MAX_ROWS;
  double* q = p + BETA_GPU_NOALLOC_MAX_ROWS;
  double* dinv = q + BETA_GPU_NOALLOC_MAX_ROWS;
  double* partials = dinv + BETA_GPU_NOALLOC_MAX_ROWS;
  double* sums = partials + (size_t)BETA_GPU_NOALLOC_MAX_BLOCKS * 4;
  PcgState* st = (PcgState*)(sums + 8);
  unsigned* flags = (unsigned*)(st + 1);
  unsigned* ticket = flags + 1;
  static_assert(sizeof(PcgState) + 2 * sizeof(unsigned) <= 256, "noalloc scratch tail");
  int status = BETA_GPU_OK;
  PcgState h;
  std::memset(&h, 0, sizeof(h));
  h.rule = stop_rule == BETA_GPU_STOP_REF ? kStopRef : kStopRB;
  h.tol2 = tol * tol;
  h.maxit = maxit > 0 ? maxit : 10000;
  CsrMat A{n, d_rp, d_ci, d_v};
  // The array keeps the previous call's contents: reset the counters and state.
  cudaMemsetAsync(flags, 0, 2 * sizeof(unsigned), s);
  cudaMemcpyAsync(st, &h, sizeof(h), cudaMemcpyHostToDevice, s);
  k_csr_dinv<<<grid(n), 256, 0, s>>>(A, dinv, flags);
  k_csr_spmv<<<grid((long long)n * 8), 256, 0, s>>>(A, d_x, r, d_b);
  k_start_s<<<grid(n), 256, 0, s>>>(n, d_x, r, d_b, dinv, p, st, partials);
  unsigned hf[2] = {0, 0};
  cudaMemcpyAsync(hf, flags, sizeof(hf), cudaMemcpyDeviceToHost, s);
  if (cudaStreamSynchronize(s) != cudaSuccess) status = BETA_GPU_ERR_CUDA;
  else if (hf[0] & 8u) status = BETA_GPU_ERR_ZERODIAG;
  else if (hf[0] & 16u) status = BETA_GPU_ERR_NEGDIAG;
  while (status == BETA_GPU_OK) {
    for (int k = 0; k < 16; ++k) {
      k_csr_spmv_dot<<<grid((long long)n * 8), 256, 0, s>>>(A, p, q, st, partials);
      k_update_s<<<grid(n), 256, 0, s>>>(n, d_x, r, p, q, dinv, st, partials);
      k_pupd_s<<<grid(n), 256, 0, s>>>(n, p, r, dinv, st);
    }
    cudaMemcpyAsync(&h, st, sizeof(h), cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) { status = BETA_GPU_ERR_CUDA; break; }
    if (h.done) {
      status = h.status == kStatusOk ? BETA_GPU_OK : (h.status == kStatusMaxit ? BETA_GPU_MAXIT : BETA_GPU_BREAKDOWN);
      break;
    }
  }
  if (status == BETA_GPU_OK || status == BETA_GPU_MAXIT) {
    k_csr_spmv<<<grid((long long)n * 8), 256, 0, s>>>(A, d_x, q, d_b);
    k_norm2_diff<<<grid(n), 256, 0, s>>>(n, q, nullptr, sums, partials, ticket);
    double rr = 0.0;
    cudaMemcpyAsync(&rr, sums, sizeof(double), cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) status = BETA_GPU_ERR_CUDA;
    if (stats) {
      stats->iterations = h.iter;
      stats->final_norm = h.last;
      stats->true_rel_residual = h.bb > 0 ? std::sqrt(rr / h.bb) : std::sqrt(rr);
    }
  }
  if (stats) stats->status = status;
  if (cudaGetLastError() != cudaSuccess && status == BETA_GPU_OK) status = BETA_GPU_ERR_CUDA;
  return status;
}


// ============================ batch C ABI ====================================
int beta_gpu_batch_create(beta_gpu_batch** out, int device, long long budget, int max_systems) {
  if (!out || budget <= 0 || max_systems <= 0 || max_systems > (1 << 20)) return BETA_GPU_ERR_ARG;
  *out = nullptr;
  std::unique_ptr<beta_gpu_batch> bp(new beta_gpu_batch());
  beta_gpu_batch* b = bp.get();
  b->device = device;
  if (cudaSetDevice(device) != cudaSuccess) { cudaGetLastError(); return BETA_GPU_ERR_CUDA; }
  BCK(cudaDeviceGetAttribute(&b->nsm, cudaDevAttrMultiProcessorCount, device));
  BCK(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
  BCK(cudaStreamCreateWithFlags(&b->copy, cudaStreamNonBlocking));
  BCK(cudaEventCreateWithFlags(&b->ev_copy, cudaEventDisableTiming));
  BCK(cudaEventCreate(&b->ev0));
  BCK(cudaEventCreate(&b->ev1));
  BCK(cudaMalloc(&b->pool, (size_t)budget));
  b->pool_bytes = (size_t)budget;
  b->free_list[0] = b->pool_bytes & ~size_t(255);
  b->cap = max_systems;
  BCK(cudaMalloc(&b->d_sys, sizeof(BSys) * max_systems));
  BCK(cudaMalloc(&b->d_states, sizeof(BState) * max_systems));
  BCK(cudaMalloc(&b->d_active, sizeof(int) * max_systems));
  BCK(cudaMalloc(&b->d_params, sizeof(BParams)));
  BCK(cudaMalloc(&b->d_plan, sizeof(BPlan) * beta_gpu_batch::kMaxCtas));
  BCK(cudaMalloc(&b->d_ctl, sizeof(int) * (2 + beta_gpu_batch::kMaxCtas)));
  BCK(cudaMalloc(&b->d_preempt, 256));
  BCK(cudaMemset(b->d_preempt, 0, 256));
  BCK(cudaMallocHost(&b->h_plan, sizeof(BPlan) * beta_gpu_batch::kMaxCtas));
  BCK(cudaMallocHost(&b->h_ctl, sizeof(int) * 2));
  BCK(cudaMallocHost(&b->h_sys, sizeof(BSys) * max_systems));
  BCK(cudaMallocHost(&b->h_states, sizeof(BState) * max_systems));
  BCK(cudaMallocHost(&b->h_active, sizeof(int) * max_systems));
  BCK(cudaMallocHost(&b->h_params, sizeof(BParams)));
  *out = bp.release();
  return BETA_GPU_OK;
}

int beta_gpu_batch_destroy(beta_gpu_batch* b) {
  if (!b) return BETA_GPU_OK;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  if (b->copy) cudaStreamSynchronize(b->copy);
  for (auto& g : b->graphs) cudaGraphExecDestroy(g.second);
  for (auto& t : b->gts) cudaFree(t.second);
  cudaFree(b->pool);
  cudaFree(b->d_sys);
  cudaFree(b->d_states);
  cudaFree(b->d_active);
  cudaFree(b->d_params);
  cudaFree(b->d_plan);
  cudaFree(b->d_ctl);
  cudaFree(b->d_preempt);
  cudaFreeHost(b->h_plan);
  cudaFreeHost(b->h_ctl);
  cudaFreeHost(b->h_sys);
  cudaFreeHost(b->h_states);
  cudaFreeHost(b->h_active);
  cudaFreeHost(b->h_params);
  if (b->ev0) cudaEventDestroy(b->ev0);
  if (b->ev1) cudaEventDestroy(b->ev1);
  if (b->ev_copy) cudaEventDestroy(b->ev_copy);
  if (b->copy) cudaStreamDestroy(b->copy);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
  return BETA_GPU_OK;
}

const char* beta_gpu_batch_last_error(const beta_gpu_batch* b) { return b ? b->err.c_str() : "null batch"; }

int beta_gpu_batch_add(beta_gpu_batch* b, int kind, int ndim, int nnode, const double* xyz, int nelem, int nnpe,
                       const int* conn, const int* first_dof, int ndpn, int order, int ngroups, int nparams,
                       const double* gp, const int* eg, const unsigned char* restrained, const double* prescribed,
                       const double* load, int* sys_id) {
  if (!b || !sys_id) return BETA_GPU_ERR_ARG;
  PreparedSys P;
  std::string err;
  int rc = prepare_system(kind, ndim, nnode, xyz, nelem, nnpe, conn, first_dof, ndpn, order, ngroups, nparams, gp,
                          eg, restrained, prescribed, load, P, err);
  if (rc != BETA_GPU_OK) return bfail(b, rc, err);
  return admit_system(b, P, sys_id);
}

int beta_gpu_batch_add_many(beta_gpu_batch* b, int count, const beta_gpu_system* sy, int host_threads,
                            int* ids) {
  if (!b || count < 0 || (count > 0 && (!sy || !ids))) return BETA_GPU_ERR_ARG;
  std::vector<PreparedSys> P(count);
  std::vector<int> rc(count, BETA_GPU_OK);
  std::vector<std::string> err(count);
  unsigned hw = std::thread::hardware_concurrency();
  int nt = host_threads > 0 ? host_threads : (int)(hw ? hw : 1);
  nt = std::max(1, std::min(nt, count));
  std::atomic<int> next(0);
  auto work = [&]() {
    pattern_serial_on_this_thread(nt > 1);
    for (int i; (i = next.fetch_add(1)) < count;) {
      const beta_gpu_system& q = sy[i];
      rc[i] = prepare_system(q.kind, q.ndim, q.nnode, q.xyz, q.nelem, q.nnpe, q.conn, q.first_dof, q.ndof_per_node,
                             q.integration_order, q.ngroups, q.nparams, q.group_params, q.elem_group, q.restrained,
                             q.prescribed, q.load, P[i], err[i]);
    }
    pattern_serial_on_this_thread(false);
  };
  if (nt == 1) {
    work();
  } else {
    std::vector<std::thread> th;
    for (int k = 0; k < nt; ++k) th.emplace_back(work);
    for (auto& t : th) t.join();
  }
  int first = BETA_GPU_OK;
  for (int i = 0; i < count; ++i) {
    int id = -1;
    if (rc[i] == BETA_GPU_OK) rc[i] = admit_system(b, P[i], &id);
    else bfail(b, rc[i], err[i]);
    P[i] = PreparedSys();  // release host copies as we go
    ids[i] = rc[i] == BETA_GPU_OK ? id : -rc[i];
    if (rc[i] != BETA_GPU_OK && first == BETA_GPU_OK) first = rc[i];
  }
  return first;
}

int beta_gpu_batch_run(beta_gpu_batch* b, const beta_gpu_solve_opts* o, int iters_per_launch, int* n_unfinished) {
  if (!b || !o) return BETA_GPU_ERR_ARG;
  cudaSetDevice(b->device);
  bool launched = false;
  int rc;
  if ((rc = batch_start(b, o, iters_per_launch, &launched))) return rc;
  if (launched && (rc = batch_finish(b))) return rc;
  int left = 0;
  for (auto& S : b->sys)
    if (S.live && S.st.phase != kPhaseDone) ++left;
  if (n_unfinished) *n_unfinished = left;
  return BETA_GPU_OK;
}

int beta_gpu_batch_result(beta_gpu_batch* b, int id, double* u, beta_gpu_solve_stats* st) {
  if (!b || id < 0 || id >= (int)b->sys.size() || !b->sys[id].live) return BETA_GPU_ERR_ARG;
  cudaSetDevice(b->device);
  const beta_gpu_batch::Sys& S = b->sys[id];
  int status;
  switch (S.st.status) {
    case kBConverged: status = S.st.phase == kPhaseDone ? BETA_GPU_OK : BETA_GPU_ERR_STATE; break;
    case kBMaxit: status = BETA_GPU_MAXIT; break;
    case kBBreakdown: status = BETA_GPU_BREAKDOWN; break;
    case kBNegDiag: status = BETA_GPU_ERR_NEGDIAG; break;
    default: status = BETA_GPU_ERR_STATE;  // still running
  }
  if (st) {
    std::memset(st, 0, sizeof(*st));
    st->status = status;
    st->iterations = S.st.iter;
    st->outer_iterations = S.st.repl;
    st->reserved = S.st.mode;  // 1: finished in FP64 (matrix-free) after the FP32 inner solve stalled
    st->final_norm = S.st.bn > 0 ? S.st.rn / S.st.bn : S.st.rn;
    st->true_rel_residual = st->final_norm;
    st->ms_solve = 1e-6 * (double)S.st.busy_ns;
  }
  if (u) {
    // on the copy stream: a finished system is in no launch, so its
    // solution can be read while another launch runs
    b->n_d2h += (long long)(sizeof(double) * S.ndof);
    BCK(cudaMemcpyAsync(u, S.desc.x64, sizeof(double) * S.ndof, cudaMemcpyDeviceToHost, b->copy));
    BCK(cudaStreamSynchronize(b->copy));
  }
  return status;
}

int beta_gpu_batch_remove(beta_gpu_batch* b, int id) {
  if (!b || id < 0 || id >= (int)b->sys.size() || !b->sys[id].live) return BETA_GPU_ERR_ARG;
  beta_gpu_batch::Sys& S = b->sys[id];
  b->rm_busy_ns += S.st.busy_ns;
  b->rm_setup_ns += S.st.setup_ns;
  b->rm_repl_ns += S.st.repl_ns;
  b->rm_iters += S.st.iter;
  pool_free(b, S.off, S.bytes);
  S.live = false;
  S.st.phase = kPhaseDone;
  b->free_ids.push_back(id);
  return BETA_GPU_OK;
}

int beta_gpu_batch_tune(beta_gpu_batch* b, int threads, int gang_boost) {
  if (!b || !(threads == 256 || threads == 512 || threads == 1024) || gang_boost < 0 || gang_boost > 64)
    return BETA_GPU_ERR_ARG;
  cudaSetDevice(b->device);
  const int ot = b->threads;
  b->threads = threads;
  if (batch_ctas(b) < 1) {
    b->threads = ot;
    return bfail(b, BETA_GPU_ERR_UNSUPPORTED, "no CTA of this launch shape fits on the GPU");
  }
  b->gang_boost = gang_boost;
  return BETA_GPU_OK;
}

int beta_gpu_batch_autotune(beta_gpu_batch* b, const beta_gpu_solve_opts* o, int budget, int* threads_out,
                            int* boost_out) {
  if (!b || !o || budget < 0) return BETA_GPU_ERR_ARG;
  cudaSetDevice(b->device);
  // (threads per CTA, gang boost)
  const int shapes[][2] = {{1024, 2}, {1024, 4}, {1024, 8}, {1024, 16}, {512, 1}, {512, 2}, {512, 4},
                           {512, 16}, {256, 4}};
  double best = 1e300;
  int bt = b->threads, bg = b->gang_boost, rc = BETA_GPU_OK;
  const long long slice = b->slice_ns;
  b->slice_ns = 0;  // each shape runs the same iterations
  cudaEvent_t e0, e1;
  BCK(cudaEventCreate(&e0));
  BCK(cudaEventCreate(&e1));
  for (auto& sh : shapes) {
    if (beta_gpu_batch_tune(b, sh[0], sh[1]) != BETA_GPU_OK) continue;
    if ((rc = batch_reset_states(b))) break;
    int na = 0;
    if ((rc = batch_prepare(b, o, budget, &na))) break;
    if (na == 0) break;
    cudaEventRecord(e0, b->stream);
    if ((rc = batch_launch_graph(b))) break;
    cudaEventRecord(e1, b->stream);
    if ((rc = batch_pull_states(b))) break;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    // the measure is time per unit of work: iterations x matrix size
    double work = 0.0;
    for (auto& S : b->sys)
      if (S.live) work += (double)S.st.iter * (double)S.work;
    const double per = work > 0 ? ms / work : 1e300;
    if (per < best) { best = per; bt = sh[0]; bg = sh[1]; }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  b->slice_ns = slice;
  if (rc != BETA_GPU_OK) return rc;
  b->threads = bt;
  b->gang_boost = bg;
  if ((rc = batch_reset_states(b))) return rc;
  BCK(cudaStreamSynchronize(b->stream));
  if (threads_out) *threads_out = bt;
  if (boost_out) *boost_out = bg;
  return BETA_GPU_OK;
}

int beta_gpu_batch_set_switch(beta_gpu_batch* b, int iters_per_cycle) {
  if (!b || iters_per_cycle < 0) return BETA_GPU_ERR_ARG;
  b->switch_iters = iters_per_cycle;
  return BETA_GPU_OK;
}

int beta_gpu_batch_set_slice(beta_gpu_batch* b, long long slice_us) {
  if (!b || slice_us < 0 || slice_us > 60000000LL) return BETA_GPU_ERR_ARG;
  b->slice_ns = slice_us * 1000LL;
  return BETA_GPU_OK;
}

int beta_gpu_batch_test_barrier(beta_gpu_batch* b, long long limit_ns, int phantom) {
  if (!b || limit_ns < 1000000LL || limit_ns > 10000000000LL) return BETA_GPU_ERR_ARG;
  b->spin_ns = limit_ns;
  b->phantom = phantom ? 1 : 0;
  return BETA_GPU_OK;
}

int beta_gpu_gang_plan(int nsys, const long long* matrix_values, const int* slices, int ctas, int threads_per_cta,
                       int gang_boost, int* gang_ctas) {
  if (nsys < 0 || (nsys > 0 && (!matrix_values || !slices || !gang_ctas)) || ctas < 1 || threads_per_cta < 32 ||
      gang_boost < 0)
    return -BETA_GPU_ERR_ARG;
  for (int i = 0; i < nsys; ++i)
    if (matrix_values[i] < 0 || slices[i] < 0 || (i > 0 && matrix_values[i] > matrix_values[i - 1]))
      return -BETA_GPU_ERR_ARG;
  return gang_plan(nsys, matrix_values, slices, ctas, threads_per_cta / 32, gang_boost, gang_ctas);
}

int beta_gpu_batch_reset(beta_gpu_batch* b) {
  if (!b) return BETA_GPU_ERR_ARG;
  cudaSetDevice(b->device);
  int rc = batch_reset_states(b);
  if (rc) return rc;
  BCK(cudaStreamSynchronize(b->stream));
  return BETA_GPU_OK;
}

int beta_gpu_batch_info(const beta_gpu_batch* b, long long* out, int n) {
  if (!b || !out || n < 0 || n > 15) return BETA_GPU_ERR_ARG;
  long long live = 0, busy = b->rm_busy_ns, setup = b->rm_setup_ns, repl = b->rm_repl_ns, its = b->rm_iters;
  for (auto& S : b->sys) {
    if (!S.live) continue;
    ++live;
    busy += S.st.busy_ns;
    setup += S.st.setup_ns;
    repl += S.st.repl_ns;
    its += S.st.iter;
  }
  const long long v[15] = {live, (long long)b->used, (long long)b->pool_bytes, b->n_launch, b->n_h2d, b->n_d2h,
                           (long long)((double)b->last_ms * 1e6), b->last_ngang, b->last_gang_ctas, b->threads,
                           b->gang_boost, busy, setup, repl, its};
  for (int i = 0; i < n; ++i) out[i] = v[i];
  return BETA_GPU_OK;
}

// ============================ server C ABI ===================================
int beta_gpu_server_create(beta_gpu_server** out, int device, long long budget, int max_systems,
                           const beta_gpu_solve_opts* o, int iters_per_launch, int threads, int gang_boost) {
  if (!out || !o || iters_per_launch <= 0) return BETA_GPU_ERR_ARG;
  *out = nullptr;
  beta_gpu_batch* b = nullptr;
  int rc = beta_gpu_batch_create(&b, device, budget, max_systems);
  if (rc != BETA_GPU_OK) return rc;
  if ((threads || gang_boost >= 0) && (rc = beta_gpu_batch_tune(b, threads ? threads : b->threads,
                                                                 gang_boost >= 0 ? gang_boost : b->gang_boost)) !=
                                           BETA_GPU_OK) {
    beta_gpu_batch_destroy(b);
    return rc;
  }
  std::unique_ptr<beta_gpu_server> S(new beta_gpu_server());
  S->batch = b;
  b->keep_singles = true;  // small requests start next to big ones
  S->opts = *o;
  S->iters_per_launch = iters_per_launch;
  S->pool_bytes = (long long)b->pool_bytes;
  try {
    S->worker = std::thread(server_loop, S.get());
  } catch (...) {
    beta_gpu_batch_destroy(b);
    return BETA_GPU_ERR_STATE;
  }
  *out = S.release();
  return BETA_GPU_OK;
}

int beta_gpu_server_set_slice(beta_gpu_server* S, long long slice_us) {
  if (!S || slice_us < 0 || slice_us > 60000000LL) return BETA_GPU_ERR_ARG;
  S->slice_us.store(slice_us);
  return BETA_GPU_OK;
}

int beta_gpu_server_destroy(beta_gpu_server* S) {
  if (!S) return BETA_GPU_OK;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->stop = true;
  }
  S->wake.notify_all();
  if (S->worker.joinable()) S->worker.join();
  beta_gpu_batch_destroy(S->batch);
  delete S;
  return BETA_GPU_OK;
}

const char* beta_gpu_server_last_error(const beta_gpu_server* S) { return S ? S->err.c_str() : "null server"; }

int beta_gpu_server_submit(beta_gpu_server* S, int kind, int ndim, int nnode, const double* xyz, int nelem,
                           int nnpe, const int* conn, const int* first_dof, int ndpn, int order, int ngroups,
                           int nparams, const double* gp, const int* eg, const unsigned char* restrained,
                           const double* prescribed, const double* load, long long* request_id) {
  if (!S || !request_id) return BETA_GPU_ERR_ARG;
  const auto t0 = beta_gpu_server::clock::now();
  std::unique_ptr<PreparedSys> P(new PreparedSys());
  std::string err;
  const int rc = prepare_system(kind, ndim, nnode, xyz, nelem, nnpe, conn, first_dof, ndpn, order, ngroups, nparams,
                                gp, eg, restrained, prescribed, load, *P, err);
  std::lock_guard<std::mutex> lk(S->mu);
  if (rc != BETA_GPU_OK) {
    S->err = err;
    return rc;
  }
  if (S->stop) return BETA_GPU_ERR_STATE;
  const long long id = S->next_id++;
  beta_gpu_server::Req& R = S->reqs[id];
  R.ndof = (int)P->ndof();
  R.prep = std::move(P);
  R.t_submit = t0;
  std::memset(&R.st, 0, sizeof(R.st));
  S->queue.push_back(id);
  ++S->n_submitted;
  *request_id = id;
  S->wake.notify_one();
  return BETA_GPU_OK;
}

int beta_gpu_server_poll(beta_gpu_server* S, long long id, int wait_ms, int* state, int* ndof, double* u,
                         beta_gpu_solve_stats* st, double* latency_ms, int release) {
  if (!S) return BETA_GPU_ERR_ARG;
  std::unique_lock<std::mutex> lk(S->mu);
  auto it = S->reqs.find(id);
  if (it == S->reqs.end()) return BETA_GPU_ERR_ARG;
  if (wait_ms > 0 && !req_final(it->second.state)) {
    const auto until = beta_gpu_server::clock::now() + std::chrono::milliseconds(wait_ms);
    S->done.wait_until(lk, until, [&] { return req_final(S->reqs.at(id).state); });
  }
  beta_gpu_server::Req& R = S->reqs.at(id);
  if (state) *state = R.state;
  if (ndof) *ndof = R.ndof;
  if (st) {
    *st = R.st;
    st->status = req_final(R.state) ? R.status : BETA_GPU_ERR_STATE;
  }
  if (latency_ms)
    *latency_ms = req_final(R.state) ? std::chrono::duration<double, std::milli>(R.t_done - R.t_submit).count() : -1.0;
  if (u && R.state == kReqDone) std::copy(R.u.begin(), R.u.end(), u);
  if (release && req_final(R.state)) S->reqs.erase(id);
  return BETA_GPU_OK;
}

int beta_gpu_server_cancel(beta_gpu_server* S, long long id) {
  if (!S) return BETA_GPU_ERR_ARG;
  std::lock_guard<std::mutex> lk(S->mu);
  auto it = S->reqs.find(id);
  if (it == S->reqs.end()) return BETA_GPU_ERR_ARG;
  if (!req_final(it->second.state)) it->second.cancel = true;
  S->wake.notify_one();
  return BETA_GPU_OK;
}

int beta_gpu_server_stats(beta_gpu_server* S, long long* out, int n) {
  if (!S || !out || n < 0 || n > 17) return BETA_GPU_ERR_ARG;
  std::lock_guard<std::mutex> lk(S->mu);
  const long long v[17] = {S->n_submitted, S->n_done,      S->n_rejected,          S->n_failed,
                           S->n_cancelled, (long long)S->queue.size(), S->n_running, S->n_launches,
                           S->pool_used,   S->pool_bytes, (long long)(S->busy_ms * 1000.0), S->h2d, S->d2h,
                           S->sys_busy_ns, S->sys_setup_ns, S->sys_repl_ns, S->sys_iters};
  for (int i = 0; i < n; ++i) out[i] = v[i];
  return BETA_GPU_OK;
}

}  // extern "C"
