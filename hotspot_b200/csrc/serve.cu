// serve.cu -- the serving loop: steady and transient requests over resident
// models, with continuous admission.
//
// Models are registered once and stay resident on the device (state,
// coefficients and solver workspaces).  hsb_server_run() releases every
// request at its arrival time (seconds after the run starts) and keeps
// `workers` requests in flight: as soon as one finishes, the next request
// that has arrived, whose model is idle, and that passes admission starts
// on the freed worker.  Each request runs on its own model's CUDA stream,
// so the work of the requests in flight overlaps on the device.
//
// Admission: a model's first request allocates its solver workspace, so it
// is admitted only while the device's free memory (cudaMemGetInfo) exceeds
// the model's declared workspace plus the reserve; later requests of that
// model allocate nothing.  Among admissible requests the one with the least
// estimated work (cells x passes) goes first, so short requests are not
// held behind long ones; ties go to the earlier arrival.
//
// Priority classes (hsb_server_set_priority): requests of high-priority
// models are dispatched before all others, run on high-priority streams (the
// device schedules their thread blocks ahead of pending ones of other
// streams), and have HIGH_SLOTS worker threads of their own, so they never
// wait for a worker.  In a run that holds high-priority requests, while any
// of them runs, the other requests pause at their next yield point: between
// transient chunks (a background transient then runs its intervals in
// chunks of about CHUNK_CELL_INTERVALS cell-intervals, so one launch holds
// the device for under a millisecond), between the refinement passes of
// steady solves and, on large models, between their PCG iterations.  A
// priority request starts once the background requests in flight have all
// reached a yield point (at most DRAIN_MS later), so it runs on a drained
// device instead of interleaving with their kernels.
//
// Each request's result depends only on its model and inputs: the kernels
// are deterministic and models share no mutable device state, so a result
// is the same alone and in any mix.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "dev_model.cuh"

// worker threads reserved for high-priority requests
#define HIGH_SLOTS 2
// cell-intervals per launch of a background transient while a priority class runs
#define CHUNK_CELL_INTERVALS (1LL << 20)
// longest wait of a priority request for background work to reach a yield point
#define DRAIN_MS 4.0
#define CHUNK_MAX_INTERVALS 64

struct hsb_server {
  int workers = 1;
  long long reserve = 0;
  struct Model {
    hsb_dev_model *m;
    hsb_solver_opts opts;
    long long workspace;
    bool warm = false;   // workspace allocated by an earlier request
    bool busy = false;
    int high = 0;        // priority class
    int cls = 0;         // the pool: index of the first model registered for this class
  };
  std::vector<Model> models;
};

using namespace hsb;

extern "C" {

int hsb_server_create(hsb_server **out, int workers, long long reserve_bytes) {
  if (!out || workers < 1) return set_error(HSB_E_ARG, "bad server arguments");
  hsb_server *s = new hsb_server();
  s->workers = workers;
  s->reserve = reserve_bytes;
  *out = s;
  return HSB_OK;
}

void hsb_server_destroy(hsb_server *s) { delete s; }

int hsb_server_add_model(hsb_server *s, hsb_dev_model *m, int form, double steady_tol, long long workspace_bytes) {
  if (!s || !m) return set_error(HSB_E_ARG, "null argument");
  hsb_server::Model e;
  e.m = m;
  e.opts.form = form;
  e.opts.steady_method = HSB_STEADY_AUTO;
  e.opts.steady_tol = steady_tol;
  e.opts.max_iters = 0;
  e.workspace = workspace_bytes;
  e.cls = (int)s->models.size();
  s->models.push_back(e);
  return (int)s->models.size() - 1;
}

int hsb_server_add_replica(hsb_server *s, int model, hsb_dev_model *m) {
  if (!s || !m || model < 0 || model >= (int)s->models.size()) return set_error(HSB_E_ARG, "unknown model");
  const hsb_server::Model &p = s->models[s->models[model].cls];
  if (m->nl != p.m->nl || m->nr != p.m->nr || m->nc != p.m->nc || m->nx != p.m->nx ||
      m->total_n_blocks != p.m->total_n_blocks)
    return set_error(HSB_E_ARG, "a replica must have its pool's grid and block vector");
  hsb_server::Model e;
  e.m = m;
  e.opts = p.opts;
  e.workspace = p.workspace;
  e.cls = p.cls;
  if (p.high) {
    const int rc = hsb_dev_set_priority(m, 1);
    if (rc) return rc;
    e.high = 1;
  }
  s->models.push_back(e);
  return (int)s->models.size() - 1;
}

int hsb_server_set_priority(hsb_server *s, int model, int high) {
  if (!s || model < 0 || model >= (int)s->models.size()) return set_error(HSB_E_ARG, "unknown model");
  const int cls = s->models[model].cls;
  for (auto &M : s->models)   // the whole pool
    if (M.cls == cls) {
      const int rc = hsb_dev_set_priority(M.m, high);
      if (rc) return rc;
      M.high = high ? 1 : 0;
    }
  return HSB_OK;
}

// the pause of background requests while high-priority ones run
struct Gate {
  std::mutex *mu;
  std::condition_variable *cv;
  const int *high_running;
  int *paused_low;               // background requests waiting here
};

static void gate_wait(void *ctx) {
  Gate *g = (Gate *)ctx;
  std::unique_lock<std::mutex> lk(*g->mu);
  if (*g->high_running == 0) return;
  ++*g->paused_low;
  g->cv->notify_all();           // a priority request may be waiting for the device to drain
  while (*g->high_running > 0) g->cv->wait_for(lk, std::chrono::milliseconds(10));
  --*g->paused_low;
}

// one request, synchronously, on the calling thread; gate: null, or the
// pause a background request takes between chunks and refinement passes
static int run_request(hsb_server::Model &M, hsb_request *r, Gate *gate) {
  hsb_dev_model *m = M.m;
  const size_t nb = (size_t)m->total_n_blocks + m->nx;
  hsb_stats st;
  memset(&st, 0, sizeof(st));
  if (cudaSetDevice(m->device) != cudaSuccess) return set_error(HSB_E_CUDA, "cudaSetDevice");
  if (r->kind == HSB_REQ_STEADY) {
    m->yield_fn = gate ? gate_wait : nullptr;
    m->yield_ctx = gate;
    const int rc = hsb_dev_steady(m, r->power, r->out, &M.opts, &st);
    m->yield_fn = nullptr;
    m->yield_ctx = nullptr;
    return rc;
  }
  if (r->kind != HSB_REQ_TRANSIENT || r->steps < 1) return set_error(HSB_E_ARG, "bad request kind or step count");
  if (!gate)   // all intervals in one call (one persistent launch in the fast form)
    return hsb_dev_transient_trace(m, r->power, r->steps, r->temp_in, r->dt, r->out, &M.opts, &st);
  long long K = CHUNK_CELL_INTERVALS / (m->ncell > 0 ? m->ncell : 1);
  if (K < 1) K = 1;
  if (K > CHUNK_MAX_INTERVALS) K = CHUNK_MAX_INTERVALS;
  for (int k0 = 0; k0 < r->steps; k0 += (int)K) {
    const int k = (int)std::min<long long>(K, r->steps - k0);
    const bool last = k0 + k >= r->steps;
    const int rc = hsb_dev_transient_trace(m, r->power + (size_t)k0 * nb, k, k0 == 0 ? r->temp_in : nullptr, r->dt,
                                           last ? r->out : nullptr, &M.opts, &st);
    if (rc) return rc;
    if (!last) gate_wait(gate);
  }
  return HSB_OK;
}

int hsb_server_run(hsb_server *s, hsb_request *reqs, int n) {
  if (!s || (!reqs && n > 0)) return set_error(HSB_E_ARG, "null argument");
  for (int k = 0; k < n; k++)
    if (reqs[k].model < 0 || reqs[k].model >= (int)s->models.size())
      return set_error(HSB_E_ARG, "request names an unknown model");
  std::mutex mu;
  std::condition_variable cv;
  std::vector<int> state(n, 0);   // 0 pending, 1 running, 2 done
  std::vector<int> served_by(n, -1);
  int done = 0, running = 0, running_high = 0, running_low = 0, paused_low = 0;
  bool any_high = false;   // a high-priority request is in this run
  for (int k = 0; k < n; k++) any_high = any_high || s->models[reqs[k].model].high;
  Gate gate{&mu, &cv, &running_high, &paused_low};
  std::string first_error;        // message of the first failed request
  using clk = std::chrono::steady_clock;
  const auto t0 = clk::now();
  auto now = [&]() { return std::chrono::duration<double>(clk::now() - t0).count(); };
  auto cost = [&](const hsb_request &r) {
    const double cells = (double)s->models[r.model].m->ncell;
    return cells * (r.kind == HSB_REQ_STEADY ? 40.0 : 8.0 * 4.0 * r.steps);
  };
  auto worker = [&](int wid) {
    std::unique_lock<std::mutex> lk(mu);
    for (;;) {
      if (done == n) return;
      const double t = now();
      int best = -1;
      double next_arrival = 1e300;
      size_t free_b = 0, total_b = 0;
      bool mem_known = false;
      for (int k = 0; k < n; k++) {
        if (state[k] != 0) continue;
        const hsb_request &r = reqs[k];
        if (r.arrival > t) {
          next_arrival = std::min(next_arrival, r.arrival);
          continue;
        }
        // the pool member to serve it: the named model, or any idle replica
        // of its pool (a transient that continues the state of the named
        // model -- no initial temperatures -- needs that model)
        const int cls = s->models[r.model].cls;
        const bool any = !(r.kind == HSB_REQ_TRANSIENT && !r.temp_in);
        int pick = -1;
        for (int q = any ? cls : r.model; q < (int)s->models.size(); q++) {
          hsb_server::Model &Q = s->models[q];
          if (Q.cls != cls || Q.busy) {
            if (!any) break;
            continue;
          }
          if (!Q.warm) {   // first use: admission by free device memory
            if (!mem_known) {
              cudaSetDevice(Q.m->device);
              cudaMemGetInfo(&free_b, &total_b);
              mem_known = true;
            }
            if ((long long)free_b < Q.workspace + s->reserve) {
              if (!any) break;
              continue;
            }
          }
          if (pick < 0 || (Q.warm && !s->models[pick].warm)) pick = q;   // warm members first
          if (!any || Q.warm) break;
        }
        if (pick < 0) continue;
        hsb_server::Model &M = s->models[pick];
        if (!M.high && running_low >= s->workers) continue;   // the other threads are kept for high priority
        if (!M.high && running_high > 0) continue;             // no new background work while a priority request runs
        served_by[k] = pick;
        // high-priority models first, then the least work, then the earliest arrival
        if (best < 0) {
          best = k;
          continue;
        }
        const int hb = s->models[reqs[best].model].high, hr = M.high;
        if (hr != hb) {
          if (hr > hb) best = k;
          continue;
        }
        if (cost(r) < cost(reqs[best]) || (cost(r) == cost(reqs[best]) && r.arrival < reqs[best].arrival))
          best = k;
      }
      if (best < 0 && running == 0 && next_arrival >= 1e300) {
        // nothing runs, nothing more arrives: what is left waits on memory
        // that no request will free -- fail those requests
        for (int k = 0; k < n; k++)
          if (state[k] == 0 && reqs[k].arrival <= t) {
            reqs[k].status = set_error(HSB_E_NOMEM, "request not admitted: not enough free device memory");
            reqs[k].start = reqs[k].finish = t;
            state[k] = 2;
            done++;
          }
        cv.notify_all();
        continue;
      }
      if (best < 0) {
        if (next_arrival < 1e300)
          cv.wait_until(lk, t0 + std::chrono::duration_cast<clk::duration>(std::chrono::duration<double>(next_arrival)));
        else
          cv.wait(lk);
        continue;
      }
      hsb_request &r = reqs[best];
      hsb_server::Model &M = s->models[served_by[best]];
      state[best] = 1;
      running++;
      const bool high = M.high != 0;
      (high ? running_high : running_low)++;
      M.busy = true;
      r.start = t;
      r.worker = wid;
      if (high) {
        // let the background work already on the device drain: every
        // running background request reaches its next yield point within
        // one chunk or iteration (bounded wait, DRAIN_MS at most)
        const auto until = clk::now() + std::chrono::microseconds((long long)(DRAIN_MS * 1000));
        while (paused_low < running_low && clk::now() < until) cv.wait_until(lk, until);
      }
      lk.unlock();
      const int rc = run_request(M, &r, (any_high && !high) ? &gate : nullptr);
      lk.lock();
      (high ? running_high : running_low)--;
      r.finish = now();
      r.status = rc;
      if (rc != HSB_OK && first_error.empty()) first_error = hsb_dev_last_error();
      if (rc == HSB_OK) M.warm = true;
      M.busy = false;
      state[best] = 2;
      running--;
      done++;
      cv.notify_all();
    }
  };
  std::vector<std::thread> pool;
  const int threads = s->workers + (any_high ? HIGH_SLOTS : 0);
  for (int w = 0; w < threads; w++) pool.emplace_back(worker, w);
  for (auto &th : pool) th.join();
  int failed = 0;
  for (int k = 0; k < n; k++)
    if (reqs[k].status != HSB_OK) failed++;
  if (failed)
    return set_error(HSB_E_CUDA, std::to_string(failed) + " request(s) failed (see their status); first: " +
                                     (first_error.empty() ? std::string("not admitted") : first_error));
  return HSB_OK;
}

}  // extern "C"
