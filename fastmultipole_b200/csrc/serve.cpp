// serve.cpp -- concurrent request serving on one device (fmm_serve_*).
//
// n_workers threads, each owning a solver context (its own non-blocking stream,
// trees, lists and scratch) on the serving context's device; a FIFO queue of
// requests; a worker runs fmm_solve on the next request as soon as it finishes
// one, so small requests overlap on the GPU instead of queueing behind each other.
// Results are kept until polled.
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
}  // namespace fmmb

namespace {

struct Done {
  int status;
  fmm_result result;
};

struct Server {
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<std::pair<uint64_t, fmm_request>> queue;
  std::unordered_map<uint64_t, Done> done;
  uint64_t next_id = 1;
  bool stopping = false;
  std::vector<std::thread> workers;
  std::vector<fmm_ctx*> ctxs;
  std::vector<cudaStream_t> streams;
};

void worker_loop(Server* S, fmm_ctx* c) {
  for (;;) {
    std::pair<uint64_t, fmm_request> job;
    {
      std::unique_lock<std::mutex> lk(S->mu);
      S->cv_work.wait(lk, [&] { return S->stopping || !S->queue.empty(); });
      if (S->queue.empty()) return;  // stopping and drained
      job = S->queue.front();
      S->queue.pop_front();
    }
    Done d;
    std::memset(&d.result, 0, sizeof(d.result));
    d.status = fmm_solve(c, &job.second.target, &job.second.source, &job.second.options, &d.result);
    {
      std::lock_guard<std::mutex> lk(S->mu);
      S->done[job.first] = d;
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
  for (int w = 0; w < n_workers; ++w) {
    fmm_ctx* c = nullptr;
    int rc = fmm_ctx_create(&c, dev);
    cudaStream_t st = nullptr;
    if (rc == FMM_OK && cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) rc = FMM_ERR_CUDA;
    if (rc == FMM_OK) rc = fmm_ctx_set_stream(c, st);
    if (rc == FMM_OK && hbm_budget_bytes) rc = fmm_ctx_set_hbm_budget(c, hbm_budget_bytes / n_workers);
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
  for (int w = 0; w < n_workers; ++w) S->workers.emplace_back(worker_loop, S, S->ctxs[w]);
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
    S->queue.emplace_back(*id, *request);
  }
  S->cv_work.notify_one();
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
