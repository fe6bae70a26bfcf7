// Batch / asynchronous solving of many boundary-value problems (the batch variant of the C ABI,
// bem_gpu_batch_*).  A batch owns n_workers solver contexts, each with its own CUDA stream and
// host thread; submitted requests go to a FIFO queue and the first free worker takes the next
// one.  While one worker builds the host plan of its problem (tree, lists, near sparsity),
// another's problem runs on the GPU, and the device work of different workers overlaps on the
// GPU through their streams (continuous batching: a request that arrives while others run starts
// as soon as a worker and device memory are free).
//
// Admission by device memory: with a budget set, the queue's head request starts only when the
// device bytes the worker contexts hold (their buffers keep their size between requests), with
// this worker's replaced by the larger of its own and the request's estimate
// (bem_gpu_estimate_bytes), stay within the budget.  An idle worker whose buffers keep a
// request out gives them back (its context is recreated).  A request larger than the budget
// alone is refused with BEM_ERR_OUT_OF_MEMORY.
//
// A request is one BVP solve (set-up + GMRES), or a whole Runge-Kutta time-stepping chain of a
// BEM-MEL simulation: n_steps steps of 4 stages, each a set-up at the stage positions (the first
// in full, then bem_gpu_setup_refresh), a solve warm-started from the previous stage's solution
// and the MEL stage update on the device, whose new positions and free-surface phi feed the next
// stage (bem/main_time_domain.cpp:1071-2600).  Only the public entry points of bem_b200.h are used.
#include <algorithm>
#include <condition_variable>
#include <cstdint>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include <omp.h>

#include "../../include/bem_b200.h"

struct bem_gpu_batch {
  struct Job {
    int64_t ticket = 0;
    bem_bvp_desc desc{};
    const double* known = nullptr;
    double* phi = nullptr;
    double* phin = nullptr;
    bem_gpu_stats* stats = nullptr;
    int64_t est = 0;  // device-memory estimate
    // chain requests (n_steps > 0)
    int32_t n_steps = 0;
    double dt = 0.0, gravity = 9.81;
    const uint8_t* point_flags = nullptr;
    double* out_X = nullptr;
    double* out_phi_point = nullptr;
  };
  bem_gpu_opts opts{};
  std::vector<bem_gpu_ctx*> ctx;
  std::vector<bem_gpu_mel*> mel;
  std::vector<int64_t> held;      // device bytes each worker's context holds (after its last request)
  std::vector<int64_t> reserved;  // estimate of the request a worker runs (0 when idle)
  std::vector<std::thread> workers;
  std::mutex mu;
  std::condition_variable cv_job, cv_done;
  std::deque<Job> queue;
  std::unordered_set<int64_t> running;
  // ticket -> status of finished requests, and their error messages; an entry lives until
  // bem_gpu_batch_release(ticket) (or the batch's destruction), so a long-running batch holds
  // only the tickets its caller has not collected yet
  std::unordered_map<int64_t, int> done;
  std::unordered_map<int64_t, std::string> errors;
  int64_t next_ticket = 1;
  int64_t budget = 0;  // 0: no limit
  int64_t admitted = 0, waited_for_memory = 0, contexts_recycled = 0;
  bool stop = false;

  int64_t others(int w) const {
    int64_t s = 0;
    for (size_t v = 0; v < held.size(); ++v)
      if ((int)v != w) s += std::max(held[v], reserved[v]);
    return s;
  }
  // called under mu: whether worker w may start the queue's head now; *recycle: only after
  // giving back its own buffers
  bool admissible(int w, const Job& j, bool* recycle) const {
    *recycle = false;
    if (budget <= 0) return true;
    const int64_t rest = others(w);
    if (rest + std::max(held[w], j.est) <= budget) return true;
    if (held[w] > j.est && rest + j.est <= budget) {
      *recycle = true;
      return true;
    }
    return false;
  }

  int run_solve(int w, const Job& job) {
    return bem_gpu_solve_bvp(ctx[w], &job.desc, job.known, nullptr, job.phi, job.phin, job.stats);
  }

  int run_chain(int w, const Job& job, std::string* msg) {
    const bem_bvp_desc& d0 = job.desc;
    const int np = d0.n_points, ndof = d0.n_dof;
    if (!mel[w]) mel[w] = bem_gpu_mel_create(opts.device);
    if (!mel[w]) {
      *msg = "could not create the MEL stage context";
      return BEM_ERR_DEVICE;
    }
    std::vector<double> X(d0.X, d0.X + 3 * (size_t)np), Xn(3 * (size_t)np), phip(np);
    std::vector<double> known(job.known, job.known + ndof), phi(ndof), phin(ndof), ans(ndof);
    std::vector<double> rkX0(3 * (size_t)np), rkphi0(np), rkaccX(3 * (size_t)np), rkaccphi(np);
    bem_bvp_desc d = d0;
    bem_gpu_stats tot{}, st{};
    tot.converged = 1;
    bool first = true;
    for (int step = 0; step < job.n_steps; ++step)
      for (int k = 0; k < 4; ++k) {
        d.X = X.data();
        const int rs = first ? bem_gpu_setup(ctx[w], &d) : bem_gpu_setup_refresh(ctx[w], &d);
        if (rs < 0) {
          *msg = bem_gpu_last_error(ctx[w]);
          return rs;
        }
        int rc = bem_gpu_solve(ctx[w], known.data(), first ? nullptr : ans.data(), phi.data(), phin.data(), &st);
        if (rc != BEM_OK && rc != BEM_ERR_NOT_CONVERGED) {
          *msg = bem_gpu_last_error(ctx[w]);
          return rc;
        }
        first = false;
        tot.iterations += st.iterations;
        tot.converged = tot.converged && st.converged;
        tot.residual = std::max(tot.residual, st.residual);
        tot.time_setup_s += st.time_setup_s;
        tot.time_solve_s += st.time_solve_s;
        tot.time_device_s += st.time_device_s;
        tot.matvecs += st.matvecs;
        tot.matvecs_lo += st.matvecs_lo;
        tot.h2d_bytes += st.h2d_bytes;
        tot.d2h_bytes += st.d2h_bytes;
        tot.kernel_launches += st.kernel_launches;
        tot.time_plan_s += st.time_plan_s;
        tot.time_upload_s += st.time_upload_s;
        tot.time_setup_device_s += st.time_setup_device_s;
        tot.nnz_near = st.nnz_near;
        tot.m2l_pairs = st.m2l_pairs;
        tot.n_nodes = st.n_nodes;
        tot.n_leaves = st.n_leaves;
        for (int i = 0; i < ndof; ++i) ans[i] = d.dof_kind[i] == BEM_DOF_DIRICHLET ? phin[i] : phi[i];
        bem_mel_surface s{np, X.data(), d.n_faces, d.tri, d.face_dirichlet, job.point_flags, ndof, d.face_dof, phi.data(), phin.data()};
        rc = bem_gpu_mel_stage(mel[w], &s, k, job.dt, job.gravity, nullptr, nullptr, rkX0.data(), rkphi0.data(), rkaccX.data(),
                               rkaccphi.data(), Xn.data(), phip.data(), nullptr, nullptr);
        if (rc != BEM_OK) {
          *msg = bem_gpu_mel_last_error(mel[w]);
          return rc;
        }
        X.swap(Xn);
        for (int i = 0; i < ndof; ++i)
          if (d.dof_kind[i] == BEM_DOF_DIRICHLET) known[i] = phip[d.dof_point[i]];
      }
    std::copy(X.begin(), X.end(), job.out_X);
    std::copy(phip.begin(), phip.end(), job.out_phi_point);
    if (job.stats) *job.stats = tot;
    return tot.converged ? BEM_OK : BEM_ERR_NOT_CONVERGED;
  }

  void run(int w) {
    for (;;) {
      Job job;
      bool recycle = false;
      {
        std::unique_lock<std::mutex> lk(mu);
        bool counted = false;
        cv_job.wait(lk, [&] {
          if (stop && queue.empty()) return true;
          if (queue.empty()) return false;
          if (admissible(w, queue.front(), &recycle)) return true;
          if (!counted) {
            ++waited_for_memory;
            counted = true;
          }
          return false;
        });
        if (queue.empty()) return;  // stop requested and nothing left
        job = queue.front();
        queue.pop_front();
        running.insert(job.ticket);
        reserved[w] = job.est;
        if (recycle) held[w] = 0;
        ++admitted;
      }
      if (recycle) {  // give the context's device buffers back before this request allocates its own
        bem_gpu_destroy(ctx[w]);
        ctx[w] = bem_gpu_create(&opts);
      }
      std::string msg;
      int rc;
      if (!ctx[w]) {
        rc = BEM_ERR_OUT_OF_MEMORY;
        msg = "could not recreate the worker's solver context";
        ctx[w] = bem_gpu_create(&opts);
      } else {
        rc = job.n_steps > 0 ? run_chain(w, job, &msg) : run_solve(w, job);
        if (job.n_steps == 0 && rc != BEM_OK && rc != BEM_ERR_NOT_CONVERGED) msg = bem_gpu_last_error(ctx[w]);
      }
      const int64_t now_held = ctx[w] ? bem_gpu_device_bytes(ctx[w]) : 0;
      {
        std::lock_guard<std::mutex> lk(mu);
        done[job.ticket] = rc;
        running.erase(job.ticket);
        reserved[w] = 0;
        held[w] = now_held;
        if (recycle) ++contexts_recycled;
        if (rc != BEM_OK && rc != BEM_ERR_NOT_CONVERGED) errors[job.ticket] = msg;
      }
      cv_done.notify_all();
      cv_job.notify_all();  // memory freed: a waiting worker may now admit the head
    }
  }

  int submit(Job j, int64_t* ticket) {
    {
      std::lock_guard<std::mutex> lk(mu);
      if (stop) return BEM_ERR_NOT_READY;
      j.ticket = next_ticket++;
      *ticket = j.ticket;
      if (budget > 0 && j.est > budget) {  // can never be admitted
        done[j.ticket] = BEM_ERR_OUT_OF_MEMORY;
        errors[j.ticket] = "request needs an estimated " + std::to_string(j.est) + " device bytes, above the batch's budget of " +
                           std::to_string(budget);
        cv_done.notify_all();
        return BEM_OK;
      }
      queue.push_back(j);
    }
    cv_job.notify_all();
    return BEM_OK;
  }
};

extern "C" {

bem_gpu_batch* bem_gpu_batch_create(const bem_gpu_opts* opts, int32_t n_workers) {
  if (!opts || n_workers < 1 || n_workers > 64) return nullptr;
  auto* b = new bem_gpu_batch();
  b->opts = *opts;
  for (int w = 0; w < n_workers; ++w) {
    bem_gpu_ctx* c = bem_gpu_create(opts);
    if (!c) {
      for (auto* x : b->ctx) bem_gpu_destroy(x);
      delete b;
      return nullptr;
    }
    b->ctx.push_back(c);
  }
  b->mel.assign(n_workers, nullptr);
  b->held.assign(n_workers, 0);
  b->reserved.assign(n_workers, 0);
  // the host plan of each worker runs OpenMP regions: the workers share the host's cores
  const int threads = std::max(1, omp_get_num_procs() / std::max(1, n_workers));
  for (int w = 0; w < n_workers; ++w)
    b->workers.emplace_back([b, w, threads] {
      omp_set_num_threads(threads);
      b->run(w);
    });
  return b;
}

int bem_gpu_batch_set_budget(bem_gpu_batch* b, int64_t bytes) {
  if (!b || bytes < 0) return BEM_ERR_INVALID_ARGUMENT;
  {
    std::lock_guard<std::mutex> lk(b->mu);
    b->budget = bytes;
  }
  b->cv_job.notify_all();
  return BEM_OK;
}

int bem_gpu_batch_submit(bem_gpu_batch* b, const bem_bvp_desc* desc, const double* known, double* out_phi, double* out_phin,
                         bem_gpu_stats* stats, int64_t* ticket) {
  if (!b || !desc || !known || !out_phi || !out_phin || !ticket) return BEM_ERR_INVALID_ARGUMENT;
  bem_gpu_batch::Job j;
  j.desc = *desc;
  j.known = known;
  j.phi = out_phi;
  j.phin = out_phin;
  j.stats = stats;
  j.est = bem_gpu_estimate_bytes(&b->opts, desc);
  return b->submit(j, ticket);
}

int bem_gpu_batch_submit_chain(bem_gpu_batch* b, const bem_bvp_desc* desc, const uint8_t* point_flags, const double* known,
                               int32_t n_steps, double dt, double gravity, double* out_X, double* out_phi_point, bem_gpu_stats* stats,
                               int64_t* ticket) {
  if (!b || !desc || !point_flags || !known || n_steps < 1 || !(dt > 0.0) || !out_X || !out_phi_point || !ticket)
    return BEM_ERR_INVALID_ARGUMENT;
  bem_gpu_batch::Job j;
  j.desc = *desc;
  j.known = known;
  j.stats = stats;
  j.n_steps = n_steps;
  j.dt = dt;
  j.gravity = gravity;
  j.point_flags = point_flags;
  j.out_X = out_X;
  j.out_phi_point = out_phi_point;
  j.est = bem_gpu_estimate_bytes(&b->opts, desc);
  return b->submit(j, ticket);
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

int bem_gpu_batch_stats(bem_gpu_batch* b, int64_t* out) {
  if (!b || !out) return BEM_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(b->mu);
  int64_t held = 0;
  for (size_t w = 0; w < b->held.size(); ++w) held += std::max(b->held[w], b->reserved[w]);
  out[0] = b->admitted;
  out[1] = b->waited_for_memory;
  out[2] = b->contexts_recycled;
  out[3] = held;
  out[4] = b->budget;
  out[5] = (int64_t)b->queue.size();
  return BEM_OK;
}

const char* bem_gpu_batch_last_error(const bem_gpu_batch* b) { return b ? t_batch_err.c_str() : "null batch"; }

void bem_gpu_batch_destroy(bem_gpu_batch* b) {
  if (!b) return;
  {
    std::lock_guard<std::mutex> lk(b->mu);
    b->stop = true;
    b->budget = 0;  // finish every queued request
  }
  b->cv_job.notify_all();
  for (auto& t : b->workers) t.join();
  for (auto* c : b->ctx) bem_gpu_destroy(c);
  for (auto* m : b->mel) bem_gpu_mel_destroy(m);
  delete b;
}

}  // extern "C"
