// server_host.cuh -- continuous-batching solve server (C ABI beta_gpu_server_*).
//
// A request is one finite-element system.  submit() checks it and builds its
// structure on the caller's thread, then queues it.  One worker thread owns a
// batch (beta_gpu_batch) and loops:
//   1. issue one persistent launch in which every admitted system gets at
//      most iters_per_launch PCG iterations, and with a time slice
//      (set_slice) stops after the iteration in which the slice ends --
//      systems admitted since the last launch are assembled inside it, so new
//      work overlaps running work;
//   2. while it runs, retire the systems the previous launch finished (copy
//      the solution to host memory, free their pool memory, record the
//      completion time) and admit queued requests in arrival order while the
//      HBM pool has room (a request that cannot fit even into an empty pool
//      is rejected), both through the batch's copy stream;
//   3. wait for the launch and collect the systems it finished.
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
  double busy_ms = 0.0;  // device time of the launches (CUDA events)
  bool launch_done = false;  // set by a host callback on the batch stream after each launch
  // group device time of the retired systems (all, setup, reliable updates) and their iterations
  long long sys_busy_ns = 0, sys_setup_ns = 0, sys_repl_ns = 0, sys_iters = 0;
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

// A system that left the batch's work this cycle: how = 0 finished (or
// stopped) in a launch, 1 cancelled, 2 failed with the launch's error rc.
struct Leaving {
  long long id;
  int sys, how, rc;
};

// Retires leaving systems: the solution and statistics of finished ones are
// copied to host memory (the batch's copy stream, so a launch may be running),
// pool memory is freed, and the requests are published under the lock.
void server_retire(beta_gpu_server* S, std::vector<Leaving>& leave) {
  if (leave.empty()) return;
  beta_gpu_batch* b = S->batch;
  struct Out {
    long long id;
    int state, status;
    std::vector<double> u;
    beta_gpu_solve_stats st;
  };
  std::vector<Out> out;
  out.reserve(leave.size());
  for (const Leaving& l : leave) {
    Out o;
    o.id = l.id;
    std::memset(&o.st, 0, sizeof(o.st));
    if (l.how == 2) {
      o.state = kReqFailed;
      o.status = l.rc;
    } else if (l.how == 1) {
      o.state = kReqCancelled;
      o.status = BETA_GPU_OK;
    } else {
      o.u.resize(b->sys[l.sys].ndof);
      o.status = beta_gpu_batch_result(b, l.sys, o.u.data(), &o.st);
      o.state = o.status == BETA_GPU_ERR_CUDA ? kReqFailed : kReqDone;
    }
    beta_gpu_batch_remove(b, l.sys);
    out.push_back(std::move(o));
  }
  leave.clear();
  const auto now = beta_gpu_server::clock::now();
  std::lock_guard<std::mutex> lk(S->mu);
  S->pool_used = (long long)b->used;
  S->h2d = b->n_h2d;
  S->d2h = b->n_d2h;
  S->sys_busy_ns = b->rm_busy_ns;
  S->sys_setup_ns = b->rm_setup_ns;
  S->sys_repl_ns = b->rm_repl_ns;
  S->sys_iters = b->rm_iters;
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

void CUDART_CB server_launch_done(void* p) {
  beta_gpu_server* S = static_cast<beta_gpu_server*>(p);
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->launch_done = true;
  }
  S->wake.notify_all();
}

// The worker.  Each cycle issues one launch over the admitted systems and,
// while it runs, retires the systems the previous launch finished and admits
// queued requests (both on the batch's copy stream; the new systems join the
// next launch).  Requests that arrive while the launch runs are admitted at
// once, and when that leaves no request waiting the launch is told to end its
// time slice early (batch_preempt: after at least the batch's minimum
// slice), so new work waits for about one iteration, not for the rest of the
// slice.  Then it
// collects the systems the launch finished.  With nothing admitted the queue
// is admitted first, so an idle device starts on new work at once.
void server_loop(beta_gpu_server* S) {
  beta_gpu_batch* b = S->batch;
  cudaSetDevice(b->device);
  std::vector<beta_gpu_server::Running> run;  // admitted, unfinished; worker-owned
  std::vector<Leaving> leave;                 // to retire in the next cycle
  for (;;) {
    {
      std::unique_lock<std::mutex> lk(S->mu);
      if (run.empty() && leave.empty() && S->queue.empty() && !S->stop)
        S->wake.wait_for(lk, std::chrono::milliseconds(50));
      if (S->stop) break;
    }
    if (run.empty()) server_admit(S, run);
    bool launched = false;
    int rc = BETA_GPU_OK;
    if (!run.empty()) {
      b->slice_ns = S->slice_us.load() * 1000LL;
      {
        std::lock_guard<std::mutex> lk(S->mu);
        S->launch_done = false;
        // nothing waits: end the launch once a request finishes, so its
        // result goes out at once (with a backlog the slice runs out)
        b->end_on_done = S->queue.empty() ? 1 : 0;
      }
      rc = batch_start(b, &S->opts, S->iters_per_launch, &launched);
      if (launched && cudaLaunchHostFunc(b->stream, server_launch_done, S) != cudaSuccess) {
        cudaGetLastError();
        std::lock_guard<std::mutex> lk(S->mu);
        S->launch_done = true;  // no callback: wait in batch_finish alone
      }
    }
    // while the launch runs
    server_retire(S, leave);
    if (rc == BETA_GPU_OK) server_admit(S, run);
    if (launched && rc == BETA_GPU_OK) {
      bool preempted = false, blocked = false;
      for (;;) {
        {
          std::unique_lock<std::mutex> lk(S->mu);
          S->wake.wait(lk, [&] {
            return S->launch_done || S->stop || (!preempted && !blocked && !S->queue.empty());
          });
          if (S->launch_done || S->stop) break;
        }
        const size_t before = run.size();
        server_admit(S, run);
        bool drained;
        {
          std::lock_guard<std::mutex> lk(S->mu);
          drained = S->queue.empty();
        }
        if (!drained) {
          blocked = true;  // the queue head waits for pool memory: until the launch ends
        } else if (run.size() > before && S->slice_us.load() > 0 && batch_preempt(b) == BETA_GPU_OK) {
          // every waiting request is admitted: end the slice so that they start
          // (with a backlog the launch keeps its slice: preempting would only
          // add launches, the backlog waits for memory either way)
          preempted = true;
        }
      }
    }
    if (launched) rc = batch_finish(b);
    if (rc != BETA_GPU_OK) cudaStreamSynchronize(b->stream);  // nothing of a failed launch stays in flight

    std::vector<char> cancel(run.size(), 0);
    {
      std::lock_guard<std::mutex> lk(S->mu);
      if (launched) {
        ++S->n_launches;
        S->busy_ms += b->last_ms;
      }
      S->h2d = b->n_h2d;
      S->d2h = b->n_d2h;
      if (rc != BETA_GPU_OK) S->err = b->err;
      for (size_t k = 0; k < run.size(); ++k) cancel[k] = S->reqs.at(run[k].id).cancel ? 1 : 0;
    }
    std::vector<beta_gpu_server::Running> still;
    for (size_t k = 0; k < run.size(); ++k) {
      const beta_gpu_batch::Sys& Y = b->sys[run[k].sys];
      if (rc != BETA_GPU_OK) leave.push_back({run[k].id, run[k].sys, 2, rc});
      else if (cancel[k]) leave.push_back({run[k].id, run[k].sys, 1, BETA_GPU_OK});
      else if (!Y.fresh && Y.st.phase == kPhaseDone) leave.push_back({run[k].id, run[k].sys, 0, BETA_GPU_OK});
      else still.push_back(run[k]);
    }
    run.swap(still);
    if (run.empty()) server_retire(S, leave);  // no launch to overlap with: publish now
  }
  server_retire(S, leave);
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
