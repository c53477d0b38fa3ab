// Request server (extension): a device-resident serving loop for eigenproblems
// of uneven size. Requests are admitted in arrival order as soon as a worker slot
// and enough of the device-memory budget are free (each request's blocks and
// workspaces, bounded by solve_memory_bytes); every admitted solve runs on its
// own stream with all of its state (subspace, Ritz values, locking) on the
// device, so the work of concurrently admitted requests overlaps on the GPU and
// requests that arrive while others run join as soon as memory frees up. Blocks that
// finished solves left in the library's caches are returned to the device when free
// memory falls short of a request's bound; a request that still runs out of memory
// while other solves run beside it goes back to the head of the queue once and runs
// when nothing else does.
//
// Grouped lanes (continuous batching on the device): a request that asks for it
// (group=1) and that the grouped Chebyshev engine accepts goes to the lane of its
// width and degree instead of a worker slot. A lane is one host thread driving one
// group: between two cycles it admits the lane's queued requests whose memory fits
// the same budget, and every cycle advances all admitted members together in
// grouped kernels (one CUDA graph while the membership is stable); members leave
// as they converge and their memory returns to the budget.
//
// The reference serves nothing: fasteig_problem::solve (src/fasteig_problem.cpp:
// 340-437) is one blocking solve per call. Each worker request here runs exactly
// that solve (the same code path as fe_solve), so its result does not depend on
// what else is in flight; a grouped member's arithmetic reads only its own rows of
// the group's blocks, so its result does not depend on the other members either.

#include "device.hpp"
#include "grouped.hpp"

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

namespace fe {
void solve_problem(const Csr& A, const Csr* B, const char* options, double* eigenvalues,
                   double* residual_norms, double* eigenvectors, double* stats);
size_t solve_memory_bytes(const Csr& A, const Csr* B, const char* options);
int64_t options_nev(const char* options);
}  // namespace fe

struct fe_server {
  using clock = std::chrono::steady_clock;
  struct Request {
    int64_t id = 0;
    const fe::Csr* A = nullptr;
    const fe::Csr* B = nullptr;
    std::string options;
    int64_t nev = 0;
    size_t bytes = 0;
    std::vector<double> eigenvalues, residuals, stats;
    int state = 0;  // 0 queued, 1 running, 2 done
    int retries = 0;  // allocation failures retried alone
    int rc = FE_OK;
    std::string error;
    clock::time_point t_submit, t_start, t_end;
    fe::GroupMember member;  // grouped lane requests
  };
  // One grouped lane per (width, degree): its queue and its driving thread.
  struct Lane {
    int64_t width = 0, degree = 0;
    std::deque<Request*> pending;
    std::thread thread;
  };

  int device = 0;
  clock::time_point t_created = clock::now();
  size_t budget = 0, in_use = 0;
  int64_t next_id = 1;
  int running = 0;
  bool stopping = false;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Request*> queue;
  std::map<int64_t, std::unique_ptr<Request>> requests;
  std::vector<std::thread> workers;
  std::vector<std::unique_ptr<Lane>> lanes;
  std::condition_variable cv_lane;
  bool stopping_lanes = false;
  // counters of the grouped lanes (fe_server_stats)
  int64_t grouped_served = 0, group_cycles = 0, group_replays = 0, group_repacks = 0;
  int64_t max_group_members = 0;

  // Head-of-line admission: the oldest request starts when it fits the budget,
  // or when nothing is running (a request larger than the budget still runs,
  // alone).
  bool can_admit() const {
    if (queue.empty()) return false;
    const Request* r = queue.front();
    return running == 0 || in_use + r->bytes <= budget;
  }

  void worker_loop() {
    cudaSetDevice(device);
    while (true) {
      Request* r = nullptr;
      {
        std::unique_lock<std::mutex> lock(mu);
        cv_work.wait(lock, [&] { return stopping || can_admit(); });
        if (stopping) return;
        r = queue.front();
        queue.pop_front();
        in_use += r->bytes;
        ++running;
        r->state = 1;
        r->t_start = clock::now();
      }
      // Memory that finished solves left in the library's caches is not in the
      // admission budget: give it back when the device has less free than this
      // request may take.
      {
        size_t free_b = 0, total_b = 0;
        if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess && free_b < r->bytes + (r->bytes >> 3))
          fe::release_cached_memory(device);
        else
          cudaGetLastError();
      }
      const int rc = fe::guarded("fe_server request", [&] {
        fe::solve_problem(*r->A, r->B, r->options.c_str(), r->eigenvalues.data(),
                          r->residuals.data(), nullptr, r->stats.data());
      });
      const std::string err = rc != FE_OK ? std::string(fe_last_error()) : std::string();
      const bool out_of_memory =
          rc == FE_ERR_ALLOC ||
          (rc == FE_ERR_CUDA && err.find("out of memory") != std::string::npos);
      if (out_of_memory && r->retries == 0) fe::release_cached_memory(device);
      {
        std::lock_guard<std::mutex> lock(mu);
        if (out_of_memory && r->retries == 0 && running > 1) {
          // Out of device memory while other solves ran beside it (the admission
          // estimate is a bound on this solve alone, not on allocator fragmentation):
          // back to the head of the queue, to run when nothing else does.
          r->retries = 1;
          in_use -= r->bytes;
          --running;
          r->bytes = std::max(r->bytes, budget);
          r->state = 0;
          queue.push_front(r);
          cv_work.notify_all();
          continue;
        }
        r->rc = rc;
        if (rc != FE_OK) r->error = err;
        r->t_end = clock::now();
        r->state = 2;
        in_use -= r->bytes;
        --running;
      }
      cv_done.notify_all();
      cv_work.notify_all();
      cv_lane.notify_all();
    }
  }

  void finish_request(Request* r, int rc, const std::string& error) {
    {
      std::lock_guard<std::mutex> lock(mu);
      r->rc = rc;
      if (rc != FE_OK) r->error = error;
      r->t_end = clock::now();
      r->state = 2;
      in_use -= r->bytes;
      --running;
    }
    cv_done.notify_all();
    cv_work.notify_all();
    cv_lane.notify_all();
  }

  void lane_loop(Lane* L) {
    cudaSetDevice(device);
    // the lane's groups: [0] FP64 filter, [1] FP32 filter (mixed members until their
    // FP32 floor, then they move to [0])
    std::unique_ptr<fe::ChebGroup> groups[2];
    size_t active = 0;
    std::vector<fe::GroupMember*> done;
    int64_t last_replays[2] = {0, 0}, last_repacks[2] = {0, 0};  // counters already added
    while (true) {
      std::vector<Request*> admit;
      {
        std::unique_lock<std::mutex> lock(mu);
        auto admissible = [&] {
          return !L->pending.empty() &&
                 (running == 0 || in_use + L->pending.front()->bytes <= budget);
        };
        if (active == 0)
          cv_lane.wait(lock, [&] { return (stopping_lanes && L->pending.empty()) || admissible(); });
        if (active == 0 && L->pending.empty() && stopping_lanes) return;
        while (admissible()) {
          Request* r = L->pending.front();
          L->pending.pop_front();
          in_use += r->bytes;
          ++running;
          r->state = 1;
          r->t_start = clock::now();
          admit.push_back(r);
        }
      }
      for (Request* r : admit) {
        size_t free_b = 0, total_b = 0;
        if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess && free_b < r->bytes + (r->bytes >> 3))
          fe::release_cached_memory(device);
        else
          cudaGetLastError();
        // per-member setup (option checks, Lanczos bounds) on its own stream
        const int rc = fe::guarded("fe_server grouped request", [&] {
          r->member.A = r->A;
          r->member.tag = r;
          fe::chebyshev_group_setup(*r->A, r->options.c_str(), r->member.g);
          const int gi = r->member.g.mixed ? 1 : 0;
          if (!groups[gi]) groups[gi].reset(new fe::ChebGroup(device, L->width, L->degree, gi == 1));
          groups[gi]->join(&r->member);
        });
        if (rc != FE_OK) {
          finish_request(r, rc, fe_last_error());
          continue;
        }
        ++active;
      }
      bool any = false;
      for (auto& g : groups) any = any || (g && !g->empty());
      if (!any) continue;
      done.clear();
      const int rc = fe::guarded("fe_server grouped cycle", [&] {
        int64_t members = 0;
        for (auto& g : groups) {
          if (!g || g->empty()) continue;
          members += static_cast<int64_t>(g->size());
          g->launch_cycle();
        }
        {
          std::lock_guard<std::mutex> lock(mu);
          max_group_members = std::max<int64_t>(max_group_members, members);
        }
        for (auto& g : groups)
          if (g) g->finish_cycle(done);
      });
      std::string cycle_error;
      if (rc != FE_OK) {
        cycle_error = fe_last_error();
        for (auto& g : groups)
          if (g) g->fail_all(rc, cycle_error, done);
      }
      {
        std::lock_guard<std::mutex> lock(mu);
        group_cycles += rc == FE_OK ? 1 : 0;
        for (int gi = 0; gi < 2; ++gi) {
          if (!groups[gi]) continue;
          group_replays += groups[gi]->graph_replays - last_replays[gi];
          group_repacks += groups[gi]->repacks - last_repacks[gi];
          last_replays[gi] = groups[gi]->graph_replays;
          last_repacks[gi] = groups[gi]->repacks;
        }
      }
      for (fe::GroupMember* m : done) {
        if (m->switched && m->rc == FE_OK && rc == FE_OK) {
          // at its FP32 floor: on to the FP64 group of the lane
          const int jrc = fe::guarded("fe_server grouped request", [&] {
            if (!groups[0]) groups[0].reset(new fe::ChebGroup(device, L->width, L->degree, false));
            groups[0]->join(m);
          });
          if (jrc == FE_OK) continue;
          m->rc = jrc;
          m->error = fe_last_error();
        } else if (m->switched) {
          // moved out of its FP32 group in a cycle that failed in the other group
          m->rc = rc != FE_OK ? rc : m->rc;
          m->error = cycle_error;
        }
        m->switched = false;
        m->carry.release();
        Request* r = static_cast<Request*>(m->tag);
        std::copy(m->eigenvalues.begin(), m->eigenvalues.end(), r->eigenvalues.begin());
        std::copy(m->residuals.begin(), m->residuals.end(), r->residuals.begin());
        r->stats[0] = static_cast<double>(m->iterations);
        r->stats[1] = m->converged ? 0.0 : 1.0;
        r->stats[2] = m->seconds;
        r->stats[3] = static_cast<double>(m->iterations * (L->degree + 1));
        r->stats[4] = static_cast<double>(m->fp32_iterations);
        r->stats[5] = static_cast<double>(m->iterations - m->fp32_iterations);
        r->stats[6] = m->g.lower;
        r->stats[7] = m->g.upper;
        {
          std::lock_guard<std::mutex> lock(mu);
          ++grouped_served;
        }
        --active;
        finish_request(r, m->rc, m->error);
      }
      if (rc != FE_OK) {
        for (int gi = 0; gi < 2; ++gi) {  // fresh groups (and streams) for the next members
          groups[gi].reset();
          last_replays[gi] = last_repacks[gi] = 0;
        }
      }
    }
  }
};

extern "C" int fe_server_create(int32_t device, int32_t slots, int64_t memory_budget_bytes,
                                fe_server_t* out) {
  return fe::guarded("fe_server_create", [&] {
    FE_REQUIRE(out, "null output handle");
    FE_REQUIRE(slots >= 1 && slots <= 64, "slots must be in [1, 64]");
    FE_CHECK_CUDA(cudaSetDevice(device));
    auto srv = std::make_unique<fe_server>();
    srv->device = device;
    if (memory_budget_bytes > 0) {
      srv->budget = static_cast<size_t>(memory_budget_bytes);
    } else {
      size_t free_b = 0, total_b = 0;
      FE_CHECK_CUDA(cudaMemGetInfo(&free_b, &total_b));
      srv->budget = free_b / 10 * 9;
    }
    for (int i = 0; i < slots; ++i) srv->workers.emplace_back([s = srv.get()] { s->worker_loop(); });
    *out = srv.release();
  });
}

extern "C" int fe_server_submit(fe_server_t srv, fe_csr_t A, fe_csr_t B, const char* options,
                                int64_t* request_id) {
  return fe::guarded("fe_server_submit", [&] {
    FE_REQUIRE(srv && A && request_id, "null argument");
    FE_REQUIRE(A->m.device == srv->device, "request operator lives on another device");
    auto r = std::make_unique<fe_server::Request>();
    r->A = &A->m;
    r->B = B ? &B->m : nullptr;
    r->options = options ? options : "";
    r->bytes = fe::solve_memory_bytes(A->m, r->B, r->options.c_str());
    // nev as the solve will parse it (unknown keys and bad values fail here, not
    // in a worker).
    r->nev = fe::options_nev(r->options.c_str());
    FE_REQUIRE(r->nev >= 1 && r->nev <= A->m.rows, "nev must be in [1, n]");
    int64_t width = 0, degree = 0;
    bool mixed = false;
    const bool grouped = fe::chebyshev_group_key(A->m, r->B, r->options.c_str(), true, &width,
                                                 &degree, &mixed);
    if (grouped) r->bytes = fe::group_member_bytes(A->m, width, mixed);
    r->eigenvalues.assign(r->nev, 0.0);
    r->residuals.assign(r->nev, 0.0);
    r->stats.assign(12, 0.0);
    r->t_submit = fe_server::clock::now();
    {
      std::lock_guard<std::mutex> lock(srv->mu);
      FE_REQUIRE(!srv->stopping, "server is shutting down");
      r->id = srv->next_id++;
      *request_id = r->id;
      if (grouped) {
        fe_server::Lane* lane = nullptr;
        for (auto& l : srv->lanes)
          if (l->width == width && l->degree == degree) lane = l.get();
        if (!lane) {
          srv->lanes.emplace_back(new fe_server::Lane);
          lane = srv->lanes.back().get();
          lane->width = width;
          lane->degree = degree;
          lane->thread = std::thread([s = srv, lane] { s->lane_loop(lane); });
        }
        lane->pending.push_back(r.get());
      } else {
        srv->queue.push_back(r.get());
      }
      srv->requests.emplace(r->id, std::move(r));
    }
    srv->cv_work.notify_one();
    srv->cv_lane.notify_all();
  });
}

extern "C" int fe_server_stats(fe_server_t srv, double* out, int32_t count) {
  return fe::guarded("fe_server_stats", [&] {
    FE_REQUIRE(srv && out && count >= 0, "null argument");
    std::lock_guard<std::mutex> lock(srv->mu);
    const double v[] = {static_cast<double>(srv->grouped_served),
                        static_cast<double>(srv->group_cycles),
                        static_cast<double>(srv->group_replays),
                        static_cast<double>(srv->group_repacks),
                        static_cast<double>(srv->lanes.size()),
                        static_cast<double>(srv->max_group_members)};
    for (int32_t i = 0; i < count; ++i) out[i] = i < 6 ? v[i] : 0.0;
  });
}

extern "C" int fe_server_wait(fe_server_t srv, int64_t request_id, double timeout_seconds,
                              double* eigenvalues, double* residual_norms, double* stats) {
  int solve_rc = FE_OK;
  std::string solve_error;
  const int rc = fe::guarded("fe_server_wait", [&] {
    FE_REQUIRE(srv, "null server");
    std::unique_ptr<fe_server::Request> r;
    {
      std::unique_lock<std::mutex> lock(srv->mu);
      auto it = srv->requests.find(request_id);
      FE_REQUIRE(it != srv->requests.end(), "unknown or already collected request id");
      fe_server::Request* req = it->second.get();
      auto done = [&] { return req->state == 2; };
      if (timeout_seconds < 0) {
        srv->cv_done.wait(lock, done);
      } else if (!srv->cv_done.wait_for(lock, std::chrono::duration<double>(timeout_seconds),
                                        done)) {
        throw fe::Error(FE_PENDING, "request still queued or running");
      }
      r = std::move(it->second);
      srv->requests.erase(it);
    }
    if (eigenvalues) std::copy(r->eigenvalues.begin(), r->eigenvalues.end(), eigenvalues);
    if (residual_norms) std::copy(r->residuals.begin(), r->residuals.end(), residual_norms);
    if (stats) {
      std::copy(r->stats.begin(), r->stats.end(), stats);
      auto sec = [](fe_server::clock::time_point a, fe_server::clock::time_point b) {
        return std::chrono::duration<double>(b - a).count();
      };
      stats[12] = sec(r->t_submit, r->t_start);  // queueing
      stats[13] = sec(r->t_start, r->t_end);     // on the device
      stats[14] = sec(r->t_submit, r->t_end);    // latency
      stats[15] = static_cast<double>(r->bytes);
      stats[16] = sec(srv->t_created, r->t_start);  // start, seconds since server creation
      stats[17] = sec(srv->t_created, r->t_end);    // end
    }
    solve_rc = r->rc;
    solve_error = r->error;
  });
  if (rc != FE_OK) return rc;
  if (solve_rc != FE_OK) fe::set_last_error(solve_error);
  return solve_rc;
}

extern "C" int fe_server_destroy(fe_server_t srv) {
  return fe::guarded("fe_server_destroy", [&] {
    if (!srv) return;
    {
      // Let admitted requests finish; queued ones are dropped (and reported so).
      std::unique_lock<std::mutex> lock(srv->mu);
      auto drop = [](fe_server::Request* r) {
        r->state = 2;
        r->rc = FE_ERR_INVALID;
        r->error = "fe_server: server destroyed before the request ran";
        r->t_start = r->t_end = fe_server::clock::now();
      };
      for (auto* r : srv->queue) drop(r);
      srv->queue.clear();
      for (auto& l : srv->lanes) {
        for (auto* r : l->pending) drop(r);
        l->pending.clear();
      }
      srv->cv_done.notify_all();
      srv->cv_done.wait(lock, [&] { return srv->running == 0; });
      srv->stopping = true;
      srv->stopping_lanes = true;
    }
    srv->cv_work.notify_all();
    srv->cv_lane.notify_all();
    for (auto& t : srv->workers) t.join();
    for (auto& l : srv->lanes) l->thread.join();
    delete srv;
  });
}
