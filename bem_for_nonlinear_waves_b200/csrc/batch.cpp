// Batch / asynchronous solving of many boundary-value problems (the batch variant of the C ABI,
// bem_gpu_batch_*).  A batch owns n_workers solver contexts, each with its own CUDA stream and
// host thread; submitted problems go to a FIFO queue and the first free worker takes the next
// one.  While one worker builds the host plan of its problem (tree, lists, near sparsity),
// another's problem runs on the GPU, and the device work of different workers overlaps on the
// GPU through their streams.  Only the public entry points of bem_b200.h are used.
#include <condition_variable>
#include <cstdint>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include "../../include/bem_b200.h"

struct bem_gpu_batch {
  struct Job {
    int64_t ticket;
    bem_bvp_desc desc;
    const double* known;
    double* phi;
    double* phin;
    bem_gpu_stats* stats;
  };
  std::vector<bem_gpu_ctx*> ctx;
  std::vector<std::thread> workers;
  std::mutex mu;
  std::condition_variable cv_job, cv_done;
  std::deque<Job> queue;
  std::unordered_set<int64_t> running;
  // ticket -> status of finished problems, and their error messages; an entry lives until
  // bem_gpu_batch_release(ticket) (or the batch's destruction), so a long-running batch holds
  // only the tickets its caller has not collected yet
  std::unordered_map<int64_t, int> done;
  std::unordered_map<int64_t, std::string> errors;
  int64_t next_ticket = 1;
  bool stop = false;

  void run(int w) {
    for (;;) {
      Job job;
      {
        std::unique_lock<std::mutex> lk(mu);
        cv_job.wait(lk, [&] { return stop || !queue.empty(); });
        if (queue.empty()) return;  // stop requested and nothing left
        job = queue.front();
        queue.pop_front();
        running.insert(job.ticket);
      }
      const int rc = bem_gpu_solve_bvp(ctx[w], &job.desc, job.known, nullptr, job.phi, job.phin, job.stats);
      {
        std::lock_guard<std::mutex> lk(mu);
        done[job.ticket] = rc;
        running.erase(job.ticket);
        if (rc != BEM_OK && rc != BEM_ERR_NOT_CONVERGED) errors[job.ticket] = bem_gpu_last_error(ctx[w]);
      }
      cv_done.notify_all();
    }
  }
};

extern "C" {

bem_gpu_batch* bem_gpu_batch_create(const bem_gpu_opts* opts, int32_t n_workers) {
  if (!opts || n_workers < 1 || n_workers > 64) return nullptr;
  auto* b = new bem_gpu_batch();
  for (int w = 0; w < n_workers; ++w) {
    bem_gpu_ctx* c = bem_gpu_create(opts);
    if (!c) {
      for (auto* x : b->ctx) bem_gpu_destroy(x);
      delete b;
      return nullptr;
    }
    b->ctx.push_back(c);
  }
  for (int w = 0; w < n_workers; ++w) b->workers.emplace_back([b, w] { b->run(w); });
  return b;
}

int bem_gpu_batch_submit(bem_gpu_batch* b, const bem_bvp_desc* desc, const double* known, double* out_phi, double* out_phin,
                         bem_gpu_stats* stats, int64_t* ticket) {
  if (!b || !desc || !known || !out_phi || !out_phin || !ticket) return BEM_ERR_INVALID_ARGUMENT;
  {
    std::lock_guard<std::mutex> lk(b->mu);
    if (b->stop) return BEM_ERR_NOT_READY;
    bem_gpu_batch::Job j{b->next_ticket++, *desc, known, out_phi, out_phin, stats};
    *ticket = j.ticket;
    b->queue.push_back(j);
  }
  b->cv_job.notify_one();
  return BEM_OK;
}

// The message of the last poll is kept per calling thread: pollers on different threads never
// see each other's messages.
static thread_local std::string t_batch_err;

int bem_gpu_batch_poll(bem_gpu_batch* b, int64_t ticket, int32_t wait) {
  if (!b || ticket < 1) return BEM_ERR_INVALID_ARGUMENT;
  std::unique_lock<std::mutex> lk(b->mu);
  if (ticket >= b->next_ticket) return BEM_ERR_INVALID_ARGUMENT;
  auto queued = [&] {
    for (const auto& j : b->queue)
      if (j.ticket == ticket) return true;
    return false;
  };
  auto it = b->done.find(ticket);
  if (it == b->done.end() && !wait) return BEM_ERR_NOT_READY;
  if (it == b->done.end()) {
    // a ticket that is neither finished nor queued nor running was released already
    if (!queued() && b->running.count(ticket) == 0) return BEM_ERR_INVALID_ARGUMENT;
    b->cv_done.wait(lk, [&] { return b->done.count(ticket) > 0; });
    it = b->done.find(ticket);
  }
  const int rc = it->second;
  auto e = b->errors.find(ticket);
  t_batch_err = (e == b->errors.end()) ? std::string() : e->second;
  return rc;
}

int bem_gpu_batch_release(bem_gpu_batch* b, int64_t ticket) {
  if (!b || ticket < 1) return BEM_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(b->mu);
  auto it = b->done.find(ticket);
  if (it == b->done.end()) return BEM_ERR_NOT_READY;  // unknown, released, or not finished yet
  b->done.erase(it);
  b->errors.erase(ticket);
  return BEM_OK;
}

const char* bem_gpu_batch_last_error(const bem_gpu_batch* b) { return b ? t_batch_err.c_str() : "null batch"; }

void bem_gpu_batch_destroy(bem_gpu_batch* b) {
  if (!b) return;
  {
    std::lock_guard<std::mutex> lk(b->mu);
    b->stop = true;
  }
  b->cv_job.notify_all();
  for (auto& t : b->workers) t.join();
  for (auto* c : b->ctx) bem_gpu_destroy(c);
  delete b;
}

}  // extern "C"
