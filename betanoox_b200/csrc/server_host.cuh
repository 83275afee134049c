// server_host.cuh -- continuous-batching solve server (C ABI beta_gpu_server_*).
//
// A request is one finite-element system.  submit() checks it and builds its
// structure on the caller's thread, then queues it.  One worker thread owns a
// batch (beta_gpu_batch) and loops:
//   1. admit queued requests in arrival order while the HBM pool has room
//      (a request that cannot fit even into an empty pool is rejected);
//   2. run one persistent launch in which every admitted system gets at most
//      iters_per_launch PCG iterations, and with a time slice (set_slice)
//      stops after the iteration in which the slice ends -- systems admitted
//      since the last launch are assembled inside it, so new work overlaps
//      running work;
//   3. retire finished systems: copy the solution to host memory, free their
//      pool memory, record the completion time.
// Requests join and leave between launches while the Krylov state of running
// ones stays on the device.  Only the worker touches the batch; the mutex
// guards the request table, the queue and the counters, and is never held
// across device work.  Included by beta_gpu.cu after prepare_system and
// admit_system.
#pragma once
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <thread>

enum : int {
  kReqQueued = BETA_GPU_REQ_QUEUED,
  kReqRunning = BETA_GPU_REQ_RUNNING,
  kReqDone = BETA_GPU_REQ_DONE,
  kReqRejected = BETA_GPU_REQ_REJECTED,
  kReqCancelled = BETA_GPU_REQ_CANCELLED,
  kReqFailed = BETA_GPU_REQ_FAILED,
};

struct beta_gpu_server {
  using clock = std::chrono::steady_clock;
  struct Req {
    int state = kReqQueued;
    int status = BETA_GPU_OK;  // solve status once DONE; admission error once REJECTED/FAILED
    bool cancel = false;
    int ndof = 0;
    std::unique_ptr<PreparedSys> prep;
    std::vector<double> u;
    beta_gpu_solve_stats st;
    clock::time_point t_submit, t_admit, t_done;
  };
  struct Running {
    long long id;
    int sys;
  };

  beta_gpu_batch* batch = nullptr;
  beta_gpu_solve_opts opts;
  int iters_per_launch = 0;
  std::thread worker;
  std::mutex mu;
  std::condition_variable wake;  // worker: new request, cancel or stop
  std::condition_variable done;  // pollers: some request reached a final state
  bool stop = false;
  std::string err;
  std::map<long long, Req> reqs;
  std::deque<long long> queue;
  long long next_id = 1;
  long long n_submitted = 0, n_done = 0, n_rejected = 0, n_failed = 0, n_cancelled = 0, n_launches = 0;
  long long n_running = 0;
  long long pool_used = 0, pool_bytes = 0;  // copied from the batch by the worker
  long long h2d = 0, d2h = 0;                // bytes copied host->device / device->host
  double busy_ms = 0.0;  // wall time the worker spent in launches
  std::atomic<long long> slice_us{0};  // time slice of a launch (0: iteration budget only)
};

namespace {

bool req_final(int s) { return s >= kReqDone; }

// Admits queued requests in arrival order; stops at the first that does not
// fit while others run (it waits for their memory), and rejects one that does
// not fit into an empty pool.
void server_admit(beta_gpu_server* S, std::vector<beta_gpu_server::Running>& run) {
  beta_gpu_batch* b = S->batch;
  for (;;) {
    long long id;
    std::unique_ptr<PreparedSys> prep;
    {
      std::lock_guard<std::mutex> lk(S->mu);
      if (S->queue.empty()) return;
      id = S->queue.front();
      auto& R = S->reqs.at(id);
      if (R.cancel) {
        R.state = kReqCancelled;
        R.prep.reset();
        R.t_done = beta_gpu_server::clock::now();
        ++S->n_cancelled;
        S->queue.pop_front();
        S->done.notify_all();
        continue;
      }
      prep = std::move(R.prep);
    }
    int sid = -1;
    const int rc = admit_system(b, *prep, &sid);
    std::lock_guard<std::mutex> lk(S->mu);
    auto& R = S->reqs.at(id);
    if (rc == BETA_GPU_OK) {
      R.state = kReqRunning;
      R.t_admit = beta_gpu_server::clock::now();
      run.push_back({id, sid});
      ++S->n_running;
      S->pool_used = (long long)b->used;
      S->queue.pop_front();
      continue;
    }
    if (rc == BETA_GPU_REJECTED && !run.empty()) {
      R.prep = std::move(prep);  // retry once running systems have left
      return;
    }
    R.state = rc == BETA_GPU_REJECTED ? kReqRejected : kReqFailed;
    R.status = rc;
    R.t_done = beta_gpu_server::clock::now();
    if (rc == BETA_GPU_REJECTED) ++S->n_rejected; else ++S->n_failed;
    S->queue.pop_front();
    S->done.notify_all();
  }
}

void server_loop(beta_gpu_server* S) {
  beta_gpu_batch* b = S->batch;
  cudaSetDevice(b->device);
  std::vector<beta_gpu_server::Running> run;  // admitted systems, worker-owned
  for (;;) {
    {
      std::unique_lock<std::mutex> lk(S->mu);
      if (run.empty() && S->queue.empty() && !S->stop)
        S->wake.wait_for(lk, std::chrono::milliseconds(50));
      if (S->stop) break;
    }
    server_admit(S, run);
    if (run.empty()) continue;

    const auto t0 = beta_gpu_server::clock::now();
    b->slice_ns = S->slice_us.load() * 1000LL;
    int left = 0;
    const int rc = beta_gpu_batch_run(b, &S->opts, S->iters_per_launch, &left);
    const auto t1 = beta_gpu_server::clock::now();

    // retirement: device work outside the lock, publication under it
    std::vector<char> cancel(run.size(), 0);
    {
      std::lock_guard<std::mutex> lk(S->mu);
      ++S->n_launches;
      S->h2d = b->n_h2d;
      S->d2h = b->n_d2h;
      S->busy_ms += std::chrono::duration<double, std::milli>(t1 - t0).count();
      for (size_t k = 0; k < run.size(); ++k) cancel[k] = S->reqs.at(run[k].id).cancel ? 1 : 0;
    }
    struct Out {
      long long id;
      int state, status;
      std::vector<double> u;
      beta_gpu_solve_stats st;
    };
    std::vector<Out> out;
    std::vector<beta_gpu_server::Running> still;
    std::string fail_msg;
    if (rc != BETA_GPU_OK) fail_msg = b->err;
    for (size_t k = 0; k < run.size(); ++k) {
      const int sid = run[k].sys;
      const beta_gpu_batch::Sys& Y = b->sys[sid];
      if (rc == BETA_GPU_OK && !cancel[k] && Y.st.phase != kPhaseDone) {
        still.push_back(run[k]);
        continue;
      }
      Out o;
      o.id = run[k].id;
      std::memset(&o.st, 0, sizeof(o.st));
      if (rc != BETA_GPU_OK) {
        o.state = kReqFailed;
        o.status = rc;
      } else if (cancel[k]) {
        o.state = kReqCancelled;
        o.status = BETA_GPU_OK;
      } else {
        o.u.resize(Y.ndof);
        o.status = beta_gpu_batch_result(b, sid, o.u.data(), &o.st);
        o.state = o.status == BETA_GPU_ERR_CUDA ? kReqFailed : kReqDone;
      }
      beta_gpu_batch_remove(b, sid);
      out.push_back(std::move(o));
    }
    run.swap(still);
    if (!out.empty()) {
      const auto now = beta_gpu_server::clock::now();
      std::lock_guard<std::mutex> lk(S->mu);
      if (!fail_msg.empty()) S->err = fail_msg;
      S->pool_used = (long long)b->used;
      S->h2d = b->n_h2d;
      S->d2h = b->n_d2h;
      for (auto& o : out) {
        auto& R = S->reqs.at(o.id);
        R.state = o.state;
        R.status = o.status;
        R.u = std::move(o.u);
        R.st = o.st;
        R.t_done = now;
        --S->n_running;
        if (o.state == kReqDone) ++S->n_done;
        else if (o.state == kReqCancelled) ++S->n_cancelled;
        else ++S->n_failed;
      }
      S->done.notify_all();
    }
  }
  for (auto& r : run) beta_gpu_batch_remove(b, r.sys);
  std::lock_guard<std::mutex> lk(S->mu);
  for (auto& r : run) {
    auto& R = S->reqs.at(r.id);
    R.state = kReqCancelled;
    R.t_done = beta_gpu_server::clock::now();
    --S->n_running;
    ++S->n_cancelled;
  }
  for (long long id : S->queue) {
    auto& R = S->reqs.at(id);
    R.state = kReqCancelled;
    R.prep.reset();
    ++S->n_cancelled;
  }
  S->queue.clear();
  S->done.notify_all();
}

}  // namespace
