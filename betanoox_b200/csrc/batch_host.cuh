// batch_host.cuh -- host side of the batched persistent solver (C ABI
// beta_gpu_batch_*): a device memory pool with first-fit allocation and an
// HBM budget, per-system structure building and upload, the descriptor table
// and work list, the gang plan of each launch, the cooperative launch
// (captured once into a CUDA graph and replayed), and a small autotuner over
// CTA size and gang sizing.
// Included by beta_gpu.cu (one translation unit).
#pragma once

struct beta_gpu_batch {
  int device = 0;
  int nsm = 148;
  cudaStream_t stream = nullptr;
  // uploads of admitted systems and downloads of results, which may overlap
  // a launch on `stream`; a launch waits for ev_copy when uploads are pending
  cudaStream_t copy = nullptr;
  cudaEvent_t ev_copy = nullptr;
  bool copy_pending = false;
  // set during a sliced launch to end its slice early (batch_preempt), after
  // at least min_slice_ns; zeroed before every launch
  int* d_preempt = nullptr;
  long long min_slice_ns = 2000000LL;
  int end_on_done = 0;  // the next launch ends its slice once a system finishes
  bool keep_singles = false;  // gang plans keep CTAs for single-CTA systems (server)
  std::string err;
  // pool
  unsigned char* pool = nullptr;
  size_t pool_bytes = 0, used = 0;
  std::map<size_t, size_t> free_list;  // offset -> size
  // systems
  struct Sys {
    bool live = false;
    int kind = 0, ndim = 0, nnode = 0, nelem = 0, nnpe = 0, ndpn = 0, ndof = 0, order = 0;
    size_t off = 0, bytes = 0;
    long long work = 0;  // stored FP32 matrix values
    int nslice = 0;
    long long served = 0;  // last launch in which the system made progress
    int last_iters = 0;    // inner iterations of its last completed solve (0: none yet)
    bool fresh = false;    // admitted after the launch in flight was issued: not in it
    BSys desc;
    BState st;
  };
  std::vector<Sys> sys;
  std::vector<int> free_ids;
  std::map<std::pair<int, int>, GaussTable*> gts;
  // device tables (fixed capacity so a captured graph stays valid)
  int cap = 0;
  BSys* d_sys = nullptr;
  BState* d_states = nullptr;
  int* d_active = nullptr;
  BParams* d_params = nullptr;
  BPlan* d_plan = nullptr;  // one entry per CTA slot (kMaxCtas)
  int* d_ctl = nullptr;     // [0] work counter, [1] abort flag, [2..2+kMaxCtas) gang arrival counters
  BSys* h_sys = nullptr;    // pinned staging
  BState* h_states = nullptr;
  int* h_active = nullptr;
  BParams* h_params = nullptr;
  BPlan* h_plan = nullptr;
  int* h_ctl = nullptr;
  // launch shape: threads per CTA; gang sizing: a system gets about
  // gang_boost x (its share of the batch's matrix values) of the CTAs, and a
  // gang when that is at least 2 (0: every system on one CTA)
  // (1024 threads: 32 warps per SM at 64 registers; faster than 512 at 128
  // registers on the RVE batches and the serving mix)
  int threads = 1024, gang_boost = 4;
  // a system whose FP32 inner solve needs more than this many iterations for
  // one residual-replacement cycle continues in FP64, matrix-free (0: never)
  int switch_iters = 500;
  // gang barrier wait limit, and the failure-path test hook (see
  // beta_gpu_batch_test_barrier): plan the first gang one CTA larger than it gets
  long long spin_ns = 2000000000LL;
  int phantom = 0;
  // time slice of a launch (0: a launch ends when every system has converged
  // or used its iteration budget)
  long long slice_ns = 0;
  int last_ngang = 0, last_gang_ctas = 0;
  std::map<int, cudaGraphExec_t> graphs;
  long long n_launch = 0, n_h2d = 0, n_d2h = 0;
  // group device time of removed systems: in all, in setup, in reliable
  // updates; and their inner iterations (live systems are added on query)
  long long rm_busy_ns = 0, rm_setup_ns = 0, rm_repl_ns = 0, rm_iters = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;  // bracket the last launch on `stream`
  float last_ms = 0.f;
  static constexpr int kMaxCtas = 4096;
};

namespace {

int bfail(beta_gpu_batch* b, int code, const std::string& m) {
  if (b) b->err = m;
  return code;
}

#define BCK(call)                                                                                  \
  do {                                                                                             \
    cudaError_t e_ = (call);                                                                       \
    if (e_ != cudaSuccess) {                                                                       \
      cudaGetLastError();                                                                          \
      return bfail(b, e_ == cudaErrorMemoryAllocation ? BETA_GPU_ERR_OOM : BETA_GPU_ERR_CUDA,      \
                   std::string(#call) + ": " + cudaGetErrorString(e_));                            \
    }                                                                                              \
  } while (0)

// first-fit allocation of `bytes` (256-aligned) from the pool
long long pool_alloc(beta_gpu_batch* b, size_t bytes) {
  bytes = (bytes + 255) & ~size_t(255);
  for (auto it = b->free_list.begin(); it != b->free_list.end(); ++it) {
    if (it->second >= bytes) {
      const size_t off = it->first, sz = it->second;
      b->free_list.erase(it);
      if (sz > bytes) b->free_list[off + bytes] = sz - bytes;
      b->used += bytes;
      return (long long)off;
    }
  }
  return -1;
}

void pool_free(beta_gpu_batch* b, size_t off, size_t bytes) {
  bytes = (bytes + 255) & ~size_t(255);
  b->used -= bytes;
  auto it = b->free_list.emplace(off, bytes).first;
  auto nx = std::next(it);
  if (nx != b->free_list.end() && it->first + it->second == nx->first) {
    it->second += nx->second;
    b->free_list.erase(nx);
  }
  if (it != b->free_list.begin()) {
    auto pv = std::prev(it);
    if (pv->first + pv->second == it->first) {
      pv->second += it->second;
      b->free_list.erase(it);
    }
  }
}

// Byte layout of one system's region in the pool.
struct SysLayout {
  size_t total = 0;
  size_t o_xyz, o_conn, o_gp, o_eg, o_rest, o_presc, o_load, o_cptr, o_elems, o_slot, o_nrp, o_ndiag, o_bsoff,
      o_bcol, o_bval, o_x64, o_r64, o_y64, o_p64, o_q64, o_w64, o_y32, o_r32, o_p32, o_p32b, o_z32, o_q32, o_minv, o_part, o_gflag;
  size_t add(size_t bytes) {
    const size_t o = total;
    total += (bytes + 255) & ~size_t(255);
    return o;
  }
};

SysLayout layout_for(int ndim, int nnode, int nelem, int nnpe, int ndpn, int ngroups, int nparams, bool eg,
                     const HostPattern& P) {
  SysLayout L;
  const size_t ndof = (size_t)nnode * ndpn;
  L.o_xyz = L.add(sizeof(double) * nnode * ndim);
  L.o_conn = L.add(sizeof(int) * (size_t)nelem * nnpe);
  L.o_gp = L.add(sizeof(double) * (size_t)ngroups * nparams);
  L.o_eg = L.add(eg ? sizeof(int) * nelem : 0);
  L.o_rest = L.add(ndof);
  L.o_presc = L.add(sizeof(double) * ndof);
  L.o_load = L.add(sizeof(double) * ndof);
  L.o_cptr = L.add(sizeof(int) * (P.ncolor + 1));
  L.o_elems = L.add(sizeof(int) * nelem);
  L.o_slot = L.add(sizeof(uint16_t) * P.slot.size());
  L.o_nrp = L.add(sizeof(int) * P.nrp.size());
  L.o_ndiag = L.add(sizeof(int) * P.ndiag.size());
  L.o_bsoff = L.add(sizeof(int) * P.bsoff.size());
  L.o_bcol = L.add(sizeof(int) * P.bcol.size());
  L.o_bval = L.add(sizeof(float) * (size_t)P.nchunk * 32 * ndpn * ndpn);
  L.o_x64 = L.add(sizeof(double) * ndof);
  L.o_r64 = L.add(sizeof(double) * ndof);
  L.o_y64 = L.add(sizeof(double) * ndof);
  L.o_p64 = L.add(sizeof(double) * ndof);
  L.o_q64 = L.add(sizeof(double) * ndof);
  L.o_w64 = L.add(sizeof(double) * ndof);
  L.o_y32 = L.add(sizeof(float) * ndof);
  L.o_r32 = L.add(sizeof(float) * ndof);
  L.o_p32 = L.add(sizeof(float) * (size_t)nnode * (ndpn == 3 ? 4 : ndpn));
  L.o_p32b = L.add(sizeof(float) * (size_t)nnode * (ndpn == 3 ? 4 : ndpn));
  L.o_z32 = L.add(sizeof(float) * (size_t)nnode * (ndpn == 3 ? 4 : ndpn));
  L.o_q32 = L.add(sizeof(float) * ndof);
  L.o_minv = L.add(sizeof(float) * (size_t)nnode * (ndpn * (ndpn + 1) / 2));
  L.o_part = L.add(sizeof(double) * 4 * (size_t)P.nslice);
  L.o_gflag = L.add(16);
  return L;
}

int batch_h2d(beta_gpu_batch* b, void* dst, const void* src, size_t bytes, cudaStream_t st = nullptr) {
  if (!bytes) return BETA_GPU_OK;
  b->n_h2d += (long long)bytes;
  BCK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st ? st : b->stream));
  return BETA_GPU_OK;
}

const GaussTable* batch_gauss(beta_gpu_batch* b, int ndim, int order) {
  auto key = std::make_pair(ndim, order);
  auto it = b->gts.find(key);
  if (it != b->gts.end()) return it->second;
  GaussTable h;
  make_gauss_table(ndim, order, h);
  GaussTable* d = nullptr;
  if (cudaMalloc(&d, sizeof(GaussTable)) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  if (cudaMemcpy(d, &h, sizeof(GaussTable), cudaMemcpyHostToDevice) != cudaSuccess) {
    cudaGetLastError();
    cudaFree(d);
    return nullptr;
  }
  b->gts[key] = d;
  return d;
}

template <int T>
cudaLaunchConfig_t batch_cfg(beta_gpu_batch* b, int grid, cudaLaunchAttribute* attr) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid, 1, 1);
  cfg.blockDim = dim3(T, 1, 1);
  cfg.dynamicSmemBytes = stage_bytes<T>();
  cfg.stream = b->stream;
  attr[0].id = cudaLaunchAttributeCooperative;  // every CTA resident: gang barriers can complete
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cfg;
}

// CTAs of the current shape that are resident at once (one full wave).
template <int T>
int batch_ctas_raw(beta_gpu_batch* b) {
  int per_sm = 0;
  // the matrix staging ring is dynamic shared memory beyond the default 48 KB
  if (cudaFuncSetAttribute(k_batch_solve<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)stage_bytes<T>()) !=
      cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch_solve<T>, T, stage_bytes<T>()) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return std::min(per_sm * b->nsm, beta_gpu_batch::kMaxCtas);
}

int batch_ctas(beta_gpu_batch* b) {
  switch (b->threads) {
    case 256: return batch_ctas_raw<256>(b);
    case 1024: return batch_ctas_raw<1024>(b);
    default: return batch_ctas_raw<512>(b);
  }
}

template <int T>
cudaError_t batch_launch_raw(beta_gpu_batch* b, int nctas) {
  cudaLaunchAttribute attr[1];
  cudaLaunchConfig_t cfg = batch_cfg<T>(b, nctas, attr);
  return cudaLaunchKernelEx(&cfg, k_batch_solve<T>, (const BSys*)b->d_sys, (const int*)b->d_active,
                            (const BPlan*)b->d_plan, (unsigned*)(b->d_ctl + 2), b->d_ctl, b->d_ctl + 1,
                            (const BParams*)b->d_params);
}

cudaError_t batch_launch(beta_gpu_batch* b, int nctas) {
  switch (b->threads) {
    case 256: return batch_launch_raw<256>(b, nctas);
    case 1024: return batch_launch_raw<1024>(b, nctas);
    default: return batch_launch_raw<512>(b, nctas);
  }
}

// One persistent launch over the active list: a graph of (zero the work
// counter, abort flag and gang counters; kernel) captured once per CTA size
// and replayed.  The kernel reads the plan, work list and parameters from
// fixed device buffers, so the graph stays valid while systems come and go.
int batch_launch_graph(beta_gpu_batch* b) {
  const int nctas = batch_ctas(b);
  if (nctas < 1) return bfail(b, BETA_GPU_ERR_UNSUPPORTED, "no CTA of this launch shape fits on the GPU");
  const size_t ctl_bytes = sizeof(int) * (2 + (size_t)nctas);
  auto it = b->graphs.find(b->threads);
  if (it == b->graphs.end()) {
    cudaGraph_t g = nullptr;
    BCK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    cudaError_t e1 = cudaMemsetAsync(b->d_ctl, 0, ctl_bytes, b->stream);
    cudaError_t e2 = batch_launch(b, nctas);
    cudaError_t e3 = cudaStreamEndCapture(b->stream, &g);
    cudaGraphExec_t ge = nullptr;
    cudaError_t e4 = cudaErrorUnknown;
    if (e1 == cudaSuccess && e2 == cudaSuccess && e3 == cudaSuccess) e4 = cudaGraphInstantiate(&ge, g, 0);
    if (g) cudaGraphDestroy(g);
    if (e4 != cudaSuccess) {
      // a cooperative launch that cannot be captured still runs directly
      cudaGetLastError();
      BCK(cudaMemsetAsync(b->d_ctl, 0, ctl_bytes, b->stream));
      BCK(batch_launch(b, nctas));
      b->n_launch += 1;
      return BETA_GPU_OK;
    }
    it = b->graphs.emplace(b->threads, ge).first;
  }
  BCK(cudaGraphLaunch(it->second, b->stream));
  b->n_launch += 1;
  return BETA_GPU_OK;
}

// Gang sizes for systems sorted by stored matrix values, largest first.  With
// N resident CTAs and W values in all, system i (w values, s 32-node slices)
// wants g = floor(boost * w * N / W) CTAs, capped so every warp of the gang
// keeps at least two slices; g >= 2 makes it a gang.  When the gangs want
// more than the CTAs they may have (N less those kept for single-CTA
// systems) they shrink in proportion (to at least 2 each) and the smallest
// are demoted to single-CTA systems until they fit.  CTAs outside
// the gangs start on the small systems at once; a gang joins them when its
// system is done.  Fills g[0..ngang) and returns ngang (the gangs solve
// systems 0..ngang-1).
int gang_plan(int na, const long long* work, const int* nslice, int nctas, int warps, int boost, int* g,
              bool keep_singles = false) {
  double W = 0.0;
  for (int i = 0; i < na; ++i) W += (double)work[i];
  auto want = [&](int i) {
    const int cap = std::max(1, nslice[i] / (2 * warps));
    return std::min(cap, (int)std::min<double>(nctas, std::floor(boost * (double)work[i] * nctas / W)));
  };
  std::vector<double> tail(na + 1, 0.0);  // work of systems i.. (the single-CTA ones past the gangs)
  for (int i = na - 1; i >= 0; --i) tail[i] = tail[i + 1] + (double)work[i];
  int ngang = 0;
  if (boost > 0 && W > 0)
    while (ngang < na && ngang < nctas / 2 && want(ngang) >= 2) ++ngang;  // sorted: later systems want less
  for (; ngang > 0; --ngang) {
    // keep_singles (the server): CTAs kept for the single-CTA systems when
    // there are any -- their share of the work, at least one, at most an
    // eighth of the CTAs -- so that a small request next to big ones starts
    // at once instead of after a gang's system is done.  A closed batch does
    // not keep them: CTAs kept beyond their share idle once the small
    // systems are done (they cannot join a running gang), 64 RVEs 252 ->
    // 269 ms.
    const int singles = na - ngang;
    int keep = 0;
    if (keep_singles && singles > 0) {
      const int share = (int)std::ceil(tail[ngang] / W * nctas);
      keep = std::min(std::min(singles, std::max(1, nctas / 8)), std::max(1, share));
    }
    const int room = nctas - keep;
    if (room < 2 * ngang) continue;
    long long want_sum = 0;
    for (int i = 0; i < ngang; ++i) want_sum += (g[i] = want(i));
    long long sum = want_sum;
    if (want_sum > room) {
      sum = 0;
      for (int i = 0; i < ngang; ++i) sum += (g[i] = std::max(2, (int)((long long)g[i] * room / want_sum)));
    }
    if (sum <= room) break;
  }
  return ngang;
}

// Expected remaining cost of a system, the weight of the gang plan: its stored
// matrix values x the inner iterations it still needs.  The iterations are
// those of its last completed solve when it has one (a repeat solve after a
// reset), else an estimate that grows like the number of nodes along one side
// of the mesh, nnode^(1/ndim) (CG iterations on these elliptic systems grow
// with the elements along a side), less the iterations already done (at least
// a tenth is kept).  Weighting by size alone gave every system about its
// share of the CTAs by size, so the largest, which also need the most
// iterations, held the launch long after the others had finished (64 RVEs:
// the launch took exactly as long as its slowest system).
long long plan_weight(const beta_gpu_batch::Sys& S) {
  double it = S.last_iters > 0 ? (double)S.last_iters
                                : std::pow((double)std::max(1, S.nnode), 1.0 / (double)std::max(1, S.ndim));
  it = std::max(0.1 * it, it - (double)S.st.iter);
  return std::max(1LL, (long long)((double)S.work * it));
}

// Gang plan of one launch over act[0..na) (sorted by plan weight, largest
// first) into h_plan.
int batch_plan(beta_gpu_batch* b, const int* act, int na, int nctas) {
  std::vector<long long> work(na);
  std::vector<int> nsl(na), g(std::max(1, na));
  for (int i = 0; i < na; ++i) {
    work[i] = plan_weight(b->sys[act[i]]);
    nsl[i] = b->sys[act[i]].nslice;
  }
  const int ngang =
      gang_plan(na, work.data(), nsl.data(), nctas, b->threads / 32, b->gang_boost, g.data(), b->keep_singles);
  int c = 0;
  for (int i = 0; i < ngang; ++i) {
    const int size = g[i] + (i == 0 && b->phantom ? 1 : 0);  // a member that never arrives
    for (int r = 0; r < g[i]; ++r, ++c) b->h_plan[c] = BPlan{i, r, size, i};
  }
  b->phantom = 0;
  b->last_gang_ctas = c;
  for (; c < nctas; ++c) b->h_plan[c] = BPlan{-1, 0, 1, 0};
  b->last_ngang = ngang;
  return ngang;
}

// Uploads descriptors of live systems, the active list (unfinished, largest
// first) and the parameters; returns the number of active systems.
int batch_prepare(beta_gpu_batch* b, const beta_gpu_solve_opts* o, int budget, int* nactive) {
  if (b->copy_pending) {  // systems admitted since the last launch: their uploads first
    BCK(cudaStreamWaitEvent(b->stream, b->ev_copy, 0));
    b->copy_pending = false;
  }
  for (auto& S : b->sys) S.fresh = false;
  int na = 0;
  std::vector<std::pair<long long, int>> order;
  for (int i = 0; i < (int)b->sys.size(); ++i)
    if (b->sys[i].live && b->sys[i].st.phase != kPhaseDone) order.push_back({-plan_weight(b->sys[i]), i});
  std::sort(order.begin(), order.end());
  for (auto& w : order) b->h_active[na++] = w.second;
  for (int i = 0; i < (int)b->sys.size(); ++i)
    if (b->sys[i].live) b->h_sys[i] = b->sys[i].desc;
  const int nctas = batch_ctas(b);
  if (nctas < 1) return bfail(b, BETA_GPU_ERR_UNSUPPORTED, "no CTA of this launch shape fits on the GPU");
  const int ngang = batch_plan(b, b->h_active, na, nctas);
  // single-CTA systems: the least recently served first, so that under a
  // time slice every system is reached within a few launches
  std::stable_sort(b->h_active + ngang, b->h_active + na,
                   [&](int x, int y) { return b->sys[x].served < b->sys[y].served; });
  BParams& P = *b->h_params;
  P.tol = o->tol > 0 ? o->tol : 1e-10;
  P.delta = (o->inner_tol > 0 && o->inner_tol < 1) ? o->inner_tol : 0.01;
  P.maxit = o->maxit > 0 ? o->maxit : 100000;
  P.max_repl = o->max_outer > 0 ? o->max_outer : 60;
  P.budget = budget;
  P.nactive = na;
  P.nbig = ngang;
  P.spin_ns = b->spin_ns;  // default 2 s at one barrier: far beyond any phase of a resident gang
  P.switch_iters = b->switch_iters;
  P.slice_ns = b->slice_ns;
  P.preempt = b->d_preempt;
  P.min_slice_ns = b->min_slice_ns;
  P.end_on_done = b->end_on_done;

  int rc;
  if (!b->sys.empty() && (rc = batch_h2d(b, b->d_sys, b->h_sys, sizeof(BSys) * b->sys.size()))) return rc;
  if ((rc = batch_h2d(b, b->d_active, b->h_active, sizeof(int) * std::max(1, na)))) return rc;
  if ((rc = batch_h2d(b, b->d_plan, b->h_plan, sizeof(BPlan) * nctas))) return rc;
  if ((rc = batch_h2d(b, b->d_params, b->h_params, sizeof(BParams)))) return rc;
  *nactive = na;
  return BETA_GPU_OK;
}

// Reads back every system's state and the launch's abort flag; a launch that
// gave up at a gang barrier returns BETA_GPU_TIMEOUT.
int batch_pull_states(beta_gpu_batch* b) {
  const size_t n = b->sys.size();
  b->n_d2h += (long long)(sizeof(BState) * n + 2 * sizeof(int));
  if (n) BCK(cudaMemcpyAsync(b->h_states, b->d_states, sizeof(BState) * n, cudaMemcpyDeviceToHost, b->stream));
  BCK(cudaMemcpyAsync(b->h_ctl, b->d_ctl, 2 * sizeof(int), cudaMemcpyDeviceToHost, b->stream));
  BCK(cudaStreamSynchronize(b->stream));
  for (size_t i = 0; i < n; ++i) {
    if (!b->sys[i].live || b->sys[i].fresh) continue;  // a fresh system keeps its initial state
    const BState& s = b->h_states[i];
    if (s.iter != b->sys[i].st.iter || s.phase != b->sys[i].st.phase) b->sys[i].served = b->n_launch;
    b->sys[i].st = s;
  }
  if (b->h_ctl[1]) return bfail(b, BETA_GPU_TIMEOUT, "a gang barrier waited past its limit; the launch stopped");
  return BETA_GPU_OK;
}

int batch_reset_states(beta_gpu_batch* b) {
  if (b->sys.empty()) return BETA_GPU_OK;
  for (size_t i = 0; i < b->sys.size(); ++i) {
    const BState& o = b->sys[i].st;
    if (b->sys[i].live && o.phase == kPhaseDone && o.status == kBConverged && o.iter > 0)
      b->sys[i].last_iters = o.iter;
    BState s;
    std::memset(&s, 0, sizeof(s));
    s.phase = b->sys[i].live ? kPhaseNew : kPhaseDone;
    s.status = kBRunning;
    b->sys[i].st = s;
    b->h_states[i] = s;
  }
  return batch_h2d(b, b->d_states, b->h_states, sizeof(BState) * b->sys.size());
}

}  // namespace
