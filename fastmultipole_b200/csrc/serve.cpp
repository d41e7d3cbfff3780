// serve.cpp -- concurrent request serving on one device (fmm_serve_*).
//
// n_workers general workers and n_workers / 2 (at least one) express workers, each a
// thread owning a solver context (its own non-blocking stream, trees, lists and
// scratch) on the serving context's device, and one queue of requests in arrival
// order.  A general worker takes the oldest queued request; an express worker takes the
// oldest request of at most kExpressBodies source plus target bodies and runs it on a
// highest-priority stream, so that small requests neither wait for a worker behind
// large ones nor queue for SMs behind their kernels.  A worker takes its next request
// as soon as it finishes one.  Results are kept until polled.
//
// Device memory is one shared account of hbm_budget_bytes (0: unlimited).  Each worker
// holds the device buffers of its context (they stay allocated between requests, so
// repeated sizes do not reallocate).  Before a request runs, its worker reserves the
// growth the request needs (its footprint estimate above what the worker holds); when
// that does not fit, the worker releases its own buffers and waits until it fits: every
// worker that finishes a request, or sits idle, while someone waits hands its buffers
// back.  A request larger than the whole budget fails with FMM_ERR_MEMORY; one that
// fits waits for memory instead of failing.  After a request the worker's holding is
// set to what its buffers actually take, so estimate errors do not accumulate.
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/fmm_b200.h"

namespace fmmb {
void*& ctx_serve_slot(fmm_ctx* c);
int ctx_device(fmm_ctx* c);
size_t request_footprint(const fmm_request* r);
void ctx_release_buffers(fmm_ctx* c);
}  // namespace fmmb

namespace {

struct Done {
  int status;
  fmm_result result;
};

constexpr int64_t kExpressBodies = 65536;

struct Job {
  uint64_t id;
  fmm_request req;
  int64_t size;  // source + target bodies
};

struct Server {
  std::mutex mu;
  std::condition_variable cv_work, cv_done, cv_mem;
  std::deque<Job> queue;  // arrival order
  std::unordered_map<uint64_t, Done> done;
  uint64_t next_id = 1;
  bool stopping = false;
  std::vector<std::thread> workers;
  std::vector<fmm_ctx*> ctxs;
  std::vector<cudaStream_t> streams;
  // shared HBM account
  size_t budget = 0;              // 0: unlimited
  size_t held_total = 0;          // sum of held
  std::vector<size_t> held;       // device bytes each worker holds or has reserved
  int waiting = 0;                // workers waiting for memory
  uint64_t next_ticket = 0, admit_ticket = 0;  // waiters are admitted in arrival order
};

// releases worker w's buffers (called with the lock held; drops it around the frees)
void release_holding(Server* S, int w, std::unique_lock<std::mutex>& lk) {
  if (S->held[w] == 0) return;
  lk.unlock();
  fmmb::ctx_release_buffers(S->ctxs[w]);
  lk.lock();
  S->held_total -= S->held[w];
  S->held[w] = 0;
  S->cv_mem.notify_all();
}

void worker_loop(Server* S, int w, bool express) {
  fmm_ctx* c = S->ctxs[w];
  for (;;) {
    Job job;
    {
      std::unique_lock<std::mutex> lk(S->mu);
      size_t pick = 0;
      auto eligible = [&] {
        for (pick = 0; pick < S->queue.size(); ++pick)
          if (!express || S->queue[pick].size <= kExpressBodies) return true;
        return false;
      };
      for (;;) {
        // an idle worker hands its buffers back while another waits for memory
        S->cv_work.wait(lk, [&] { return S->stopping || eligible() || (S->waiting > 0 && S->held[w] > 0); });
        if (S->waiting > 0 && S->held[w] > 0 && !eligible()) {
          release_holding(S, w, lk);
          continue;
        }
        break;
      }
      if (!eligible()) return;  // stopping, and nothing left for this worker
      job = S->queue[pick];
      S->queue.erase(S->queue.begin() + (std::ptrdiff_t)pick);
      if (S->budget) {
        const size_t need_total = fmmb::request_footprint(&job.req);
        if (need_total > S->budget) {
          Done d;
          std::memset(&d.result, 0, sizeof(d.result));
          d.status = FMM_ERR_MEMORY;  // larger than the whole budget: it can never run
          S->done[job.id] = d;
          S->cv_done.notify_all();
          continue;
        }
        auto growth = [&] { return need_total > S->held[w] ? need_total - S->held[w] : 0; };
        if (S->waiting > 0 || S->held_total + growth() > S->budget) {
          // wait behind the earlier waiters (first come, first admitted)
          const uint64_t ticket = S->next_ticket++;
          ++S->waiting;
          release_holding(S, w, lk);
          S->cv_work.notify_all();  // idle workers release theirs
          S->cv_mem.wait(lk, [&] { return S->admit_ticket == ticket && S->held_total + growth() <= S->budget; });
          ++S->admit_ticket;
          --S->waiting;
          S->cv_mem.notify_all();
        }
        const size_t g = growth();
        S->held[w] += g;
        S->held_total += g;
      }
    }
    Done d;
    std::memset(&d.result, 0, sizeof(d.result));
    d.status = fmm_solve(c, &job.req.target, &job.req.source, &job.req.options, &d.result);
    {
      std::unique_lock<std::mutex> lk(S->mu);
      S->done[job.id] = d;
      if (S->budget) {
        const size_t actual = fmm_ctx_device_bytes(c);
        S->held_total = S->held_total - S->held[w] + actual;
        S->held[w] = actual;
        if (S->waiting > 0) release_holding(S, w, lk);
        S->cv_mem.notify_all();
      }
    }
    S->cv_done.notify_all();
  }
}

}  // namespace

extern "C" {

int fmm_serve_start(fmm_ctx* ctx, int n_workers, size_t hbm_budget_bytes) {
  if (!ctx || n_workers < 1 || n_workers > 64) return FMM_ERR_ARGUMENT;
  void*& slot = fmmb::ctx_serve_slot(ctx);
  if (slot) return FMM_OK;  // already serving
  Server* S = new Server();
  const int dev = fmmb::ctx_device(ctx);
  const int n_express = n_workers / 2 > 0 ? n_workers / 2 : 1, n_all = n_workers + n_express;
  int least = 0, greatest = 0;
  if (cudaSetDevice(dev) != cudaSuccess || cudaDeviceGetStreamPriorityRange(&least, &greatest) != cudaSuccess) {
    delete S;
    return FMM_ERR_CUDA;
  }
  for (int w = 0; w < n_all; ++w) {
    fmm_ctx* c = nullptr;
    int rc = fmm_ctx_create(&c, dev);
    cudaStream_t st = nullptr;
    if (rc == FMM_OK &&
        cudaStreamCreateWithPriority(&st, cudaStreamNonBlocking, w < n_workers ? least : greatest) != cudaSuccess)
      rc = FMM_ERR_CUDA;
    if (rc == FMM_OK) rc = fmm_ctx_set_stream(c, st);
    if (rc != FMM_OK) {
      if (c) fmm_ctx_destroy(c);
      if (st) cudaStreamDestroy(st);
      for (size_t i = 0; i < S->ctxs.size(); ++i) {
        fmm_ctx_destroy(S->ctxs[i]);
        cudaStreamDestroy(S->streams[i]);
      }
      delete S;
      return rc;
    }
    S->ctxs.push_back(c);
    S->streams.push_back(st);
  }
  S->budget = hbm_budget_bytes;
  S->held.assign((size_t)n_all, 0);
  for (int w = 0; w < n_all; ++w) S->workers.emplace_back(worker_loop, S, w, w >= n_workers);
  slot = S;
  return FMM_OK;
}

int fmm_serve_submit(fmm_ctx* ctx, const fmm_request* request, uint64_t* id) {
  if (!ctx || !request || !id) return FMM_ERR_ARGUMENT;
  Server* S = static_cast<Server*>(fmmb::ctx_serve_slot(ctx));
  if (!S) return FMM_ERR_STATE;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    if (S->stopping) return FMM_ERR_STATE;
    *id = S->next_id++;
    const int64_t nt = request->target.positions ? request->target.n_bodies : 0;
    S->queue.push_back(Job{*id, *request, request->source.n_bodies + nt});
  }
  S->cv_work.notify_all();  // general and express workers wait for different requests
  return FMM_OK;
}

int fmm_serve_poll(fmm_ctx* ctx, uint64_t id, fmm_result* result, int timeout_ms) {
  if (!ctx) return FMM_ERR_ARGUMENT;
  Server* S = static_cast<Server*>(fmmb::ctx_serve_slot(ctx));
  if (!S) return FMM_ERR_STATE;
  std::unique_lock<std::mutex> lk(S->mu);
  if (id == 0 || id >= S->next_id) return FMM_ERR_ARGUMENT;
  auto ready = [&] { return S->done.count(id) != 0; };
  if (timeout_ms < 0)
    S->cv_done.wait(lk, ready);
  else if (!S->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready))
    return FMM_PENDING;
  auto it = S->done.find(id);
  if (it == S->done.end()) return FMM_ERR_ARGUMENT;  // polled before
  const Done d = it->second;
  S->done.erase(it);
  if (result) *result = d.result;
  return d.status;
}

size_t fmm_request_footprint(const fmm_request* request) {
  return request ? fmmb::request_footprint(request) : 0;
}

int fmm_serve_stop(fmm_ctx* ctx) {
  if (!ctx) return FMM_ERR_ARGUMENT;
  void*& slot = fmmb::ctx_serve_slot(ctx);
  Server* S = static_cast<Server*>(slot);
  if (!S) return FMM_OK;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->stopping = true;
  }
  S->cv_work.notify_all();
  for (auto& t : S->workers) t.join();
  for (size_t i = 0; i < S->ctxs.size(); ++i) {
    fmm_ctx_destroy(S->ctxs[i]);
    cudaStreamDestroy(S->streams[i]);
  }
  delete S;
  slot = nullptr;
  return FMM_OK;
}

}  // extern "C"
