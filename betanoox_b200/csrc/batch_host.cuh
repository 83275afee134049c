// batch_host.cuh -- host side of the batched persistent solver (C ABI
// beta_gpu_batch_*): a device memory pool with first-fit allocation and an
// HBM budget, per-system structure building and upload, the descriptor table
// and work list, the launch (captured once into a CUDA graph and replayed),
// and a small autotuner over CTA size and cluster size.
// Included by beta_gpu.cu (one translation unit).
#pragma once

struct beta_gpu_batch {
  int device = 0;
  int nsm = 148;
  cudaStream_t stream = nullptr;
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
    long long work = 0;
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
  int* d_counter = nullptr;
  BParams* d_params = nullptr;
  BSys* h_sys = nullptr;  // pinned staging
  BState* h_states = nullptr;
  int* h_active = nullptr;
  BParams* h_params = nullptr;
  // launch shape: threads per CTA and CTAs per cluster (one system per cluster)
  int threads = 512, cluster = 1;
  std::map<std::pair<int, int>, cudaGraphExec_t> graphs;
  long long n_launch = 0, n_h2d = 0, n_d2h = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;  // bracket the last launch on `stream`
  float last_ms = 0.f;
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
      o_bcol, o_bval, o_x64, o_r64, o_y64, o_y32, o_r32, o_p32, o_q32, o_minv;
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
  L.o_slot = L.add(sizeof(int) * P.slot.size());
  L.o_nrp = L.add(sizeof(int) * P.nrp.size());
  L.o_ndiag = L.add(sizeof(int) * P.ndiag.size());
  L.o_bsoff = L.add(sizeof(int) * P.bsoff.size());
  L.o_bcol = L.add(sizeof(int) * P.bcol.size());
  L.o_bval = L.add(sizeof(float) * (size_t)P.nchunk * 32 * ndpn * ndpn);
  L.o_x64 = L.add(sizeof(double) * ndof);
  L.o_r64 = L.add(sizeof(double) * ndof);
  L.o_y64 = L.add(sizeof(double) * ndof);
  L.o_y32 = L.add(sizeof(float) * ndof);
  L.o_r32 = L.add(sizeof(float) * ndof);
  L.o_p32 = L.add(sizeof(float) * (size_t)nnode * (ndpn == 3 ? 4 : ndpn));
  L.o_q32 = L.add(sizeof(float) * ndof);
  L.o_minv = L.add(sizeof(float) * (size_t)nnode * (ndpn * (ndpn + 1) / 2));
  return L;
}

int batch_h2d(beta_gpu_batch* b, void* dst, const void* src, size_t bytes) {
  if (!bytes) return BETA_GPU_OK;
  b->n_h2d += (long long)bytes;
  BCK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, b->stream));
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
  cfg.dynamicSmemBytes = 0;
  cfg.stream = b->stream;
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = b->cluster;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cfg;
}

// Clusters of the current shape that are resident at once (one full wave).
template <int T>
int batch_clusters_raw(beta_gpu_batch* b) {
  cudaLaunchAttribute attr[1];
  cudaLaunchConfig_t cfg = batch_cfg<T>(b, b->cluster, attr);
  int n = 0;
  if (cudaOccupancyMaxActiveClusters(&n, k_batch_solve<T>, &cfg) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

int batch_clusters(beta_gpu_batch* b) {
  switch (b->threads) {
    case 256: return batch_clusters_raw<256>(b);
    case 1024: return batch_clusters_raw<1024>(b);
    default: return batch_clusters_raw<512>(b);
  }
}

template <int T>
cudaError_t batch_launch_raw(beta_gpu_batch* b, int nclusters) {
  cudaLaunchAttribute attr[1];
  cudaLaunchConfig_t cfg = batch_cfg<T>(b, nclusters * b->cluster, attr);
  return cudaLaunchKernelEx(&cfg, k_batch_solve<T>, (const BSys*)b->d_sys, (const int*)b->d_active, b->d_counter,
                            (const BParams*)b->d_params);
}

cudaError_t batch_launch(beta_gpu_batch* b, int nclusters) {
  switch (b->threads) {
    case 256: return batch_launch_raw<256>(b, nclusters);
    case 1024: return batch_launch_raw<1024>(b, nclusters);
    default: return batch_launch_raw<512>(b, nclusters);
  }
}

// One persistent launch over the active list: a graph of (reset work
// counter, kernel) captured once per launch shape and replayed.  The kernel
// reads the work list and parameters from fixed device buffers, so the graph
// stays valid while systems come and go.
int batch_launch_graph(beta_gpu_batch* b) {
  const int ncl = batch_clusters(b);
  if (ncl < 1) return bfail(b, BETA_GPU_ERR_UNSUPPORTED, "no cluster of this launch shape fits on the GPU");
  auto key = std::make_pair(b->threads, b->cluster);
  auto it = b->graphs.find(key);
  if (it == b->graphs.end()) {
    cudaGraph_t g = nullptr;
    BCK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    cudaError_t e1 = cudaMemsetAsync(b->d_counter, 0, sizeof(int), b->stream);
    cudaError_t e2 = batch_launch(b, ncl);
    cudaError_t e3 = cudaStreamEndCapture(b->stream, &g);
    if (e1 != cudaSuccess || e2 != cudaSuccess || e3 != cudaSuccess) {
      cudaGetLastError();
      if (g) cudaGraphDestroy(g);
      return bfail(b, BETA_GPU_ERR_CUDA, "capturing the batch launch failed");
    }
    cudaGraphExec_t ge = nullptr;
    cudaError_t e4 = cudaGraphInstantiate(&ge, g, 0);
    cudaGraphDestroy(g);
    if (e4 != cudaSuccess) {
      cudaGetLastError();
      return bfail(b, BETA_GPU_ERR_CUDA, "instantiating the batch graph failed");
    }
    it = b->graphs.emplace(key, ge).first;
  }
  BCK(cudaGraphLaunch(it->second, b->stream));
  b->n_launch += 1;
  return BETA_GPU_OK;
}

// Uploads descriptors of live systems, the active list (unfinished, largest
// first) and the parameters; returns the number of active systems.
int batch_prepare(beta_gpu_batch* b, const beta_gpu_solve_opts* o, int budget, int* nactive) {
  int na = 0;
  std::vector<std::pair<long long, int>> order;
  for (int i = 0; i < (int)b->sys.size(); ++i)
    if (b->sys[i].live && b->sys[i].st.phase != kPhaseDone) order.push_back({-b->sys[i].work, i});
  std::sort(order.begin(), order.end());
  for (auto& w : order) b->h_active[na++] = w.second;
  for (int i = 0; i < (int)b->sys.size(); ++i)
    if (b->sys[i].live) b->h_sys[i] = b->sys[i].desc;
  BParams& P = *b->h_params;
  P.tol = o->tol > 0 ? o->tol : 1e-10;
  P.delta = (o->inner_tol > 0 && o->inner_tol < 1) ? o->inner_tol : 0.01;
  P.maxit = o->maxit > 0 ? o->maxit : 100000;
  P.max_repl = o->max_outer > 0 ? o->max_outer : 60;
  P.budget = budget;
  P.nactive = na;
  int rc;
  if (!b->sys.empty() && (rc = batch_h2d(b, b->d_sys, b->h_sys, sizeof(BSys) * b->sys.size()))) return rc;
  if ((rc = batch_h2d(b, b->d_active, b->h_active, sizeof(int) * std::max(1, na)))) return rc;
  if ((rc = batch_h2d(b, b->d_params, b->h_params, sizeof(BParams)))) return rc;
  *nactive = na;
  return BETA_GPU_OK;
}

int batch_pull_states(beta_gpu_batch* b) {
  const size_t n = b->sys.size();
  if (!n) return BETA_GPU_OK;
  b->n_d2h += (long long)(sizeof(BState) * n);
  BCK(cudaMemcpyAsync(b->h_states, b->d_states, sizeof(BState) * n, cudaMemcpyDeviceToHost, b->stream));
  BCK(cudaStreamSynchronize(b->stream));
  for (size_t i = 0; i < n; ++i)
    if (b->sys[i].live) b->sys[i].st = b->h_states[i];
  return BETA_GPU_OK;
}

int batch_reset_states(beta_gpu_batch* b) {
  if (b->sys.empty()) return BETA_GPU_OK;
  for (size_t i = 0; i < b->sys.size(); ++i) {
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
