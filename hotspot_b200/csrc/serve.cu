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
// Continuous batching (hsb_server_set_batching): the fast-form models whose
// layers the temporally blocked kernel takes are gathered into one batch
// (hsb_batch), and their transient requests are served by a batch engine
// instead of the workers.  The engine advances every admitted transient of
// one interval length together, a few intervals per launch (a tick, about
// TICK_CELL_INTERVALS cell-intervals): between ticks it admits the requests
// that have arrived onto idle pool members (loading their initial
// temperatures) and retires the finished ones (reading their block
// temperatures), so requests join and leave a running batch without waiting
// for each other.  Steady requests keep running on the workers meanwhile.
//
// Each request's result depends only on its model and inputs: the kernels
// are deterministic, models share no mutable device state and a chip's
// result does not depend on which CTAs advance it or on how its intervals
// are split over launches, so a result is the same alone and in any mix.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "dev_model.cuh"
#include "rk4_tb.cuh"

// worker threads reserved for high-priority requests
#define HIGH_SLOTS 2
// cell-intervals per launch of a background transient while a priority class runs
#define CHUNK_CELL_INTERVALS (1LL << 20)
// longest wait of a priority request for background work to reach a yield point
#define DRAIN_MS 2.0
#define CHUNK_MAX_INTERVALS 64
// cell-intervals per launch of the batch engine, and its interval cap
#define TICK_CELL_INTERVALS (1LL << 21)
#define TICK_MAX_INTERVALS 16

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
    int slot = -1;       // index in the batch, -1: not batched
  };
  std::vector<Model> models;
  // continuous batching of transients
  int batching = 0;
  hsb_batch *batch = nullptr;
  int batch_built = -1;        // models registered when the batch was built
  std::vector<long long> boff;  // the batch's block-vector offsets
  long long ticks = 0, tick_requests = 0, tick_intervals = 0;
  ~hsb_server() {
    if (batch) hsb_batch_destroy(batch);
  }
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

int hsb_server_set_batching(hsb_server *s, int on) {
  if (!s) return set_error(HSB_E_ARG, "null server");
  s->batching = on ? 1 : 0;
  if (!on && s->batch) {
    hsb_batch_destroy(s->batch);
    s->batch = nullptr;
    s->batch_built = -1;
    for (auto &M : s->models) M.slot = -1;
  }
  return HSB_OK;
}

int hsb_server_batch_stats(hsb_server *s, long long *ticks, long long *request_ticks, long long *request_intervals) {
  if (!s) return set_error(HSB_E_ARG, "null server");
  if (ticks) *ticks = s->ticks;
  if (request_ticks) *request_ticks = s->tick_requests;
  if (request_intervals) *request_intervals = s->tick_intervals;
  return HSB_OK;
}

// (re)build the batch over the registered fast-form models the temporally
// blocked kernel takes
static int build_batch(hsb_server *s) {
  if (s->batch && s->batch_built == (int)s->models.size()) return HSB_OK;
  if (s->batch) hsb_batch_destroy(s->batch);
  s->batch = nullptr;
  std::vector<hsb_dev_model *> ms;
  for (auto &M : s->models) {
    M.slot = -1;
    if ((M.opts.form == HSB_FORM_FAST || M.opts.form == HSB_FORM_FAST_BLOCKED) && tb_eligible(M.m)) {
      M.slot = (int)ms.size();
      ms.push_back(M.m);
    }
  }
  s->batch_built = (int)s->models.size();
  if (ms.empty()) return HSB_OK;
  int rc = hsb_batch_create(&s->batch, ms.data(), (int)ms.size());
  if (rc) {
    s->batch = nullptr;
    for (auto &M : s->models) M.slot = -1;
    return rc;
  }
  s->boff.assign(ms.size() + 1, 0);
  return hsb_batch_offsets(s->batch, s->boff.data());
}

// the initial block temperatures of a transient into the model's state
static int load_temps(hsb_dev_model *m, const double *block_temp) {
  const size_t nb = (size_t)m->total_n_blocks + m->nx;
  if (cudaSetDevice(m->device) != cudaSuccess) return set_error(HSB_E_CUDA, "cudaSetDevice");
  HSB_CUDA(cudaMemcpyAsync(m->blk_in + nb, block_temp, sizeof(double) * nb, cudaMemcpyHostToDevice, m->stream));
  int rc = b2g(m, m->blk_in + nb, m->y, HSB_V_TEMP);
  if (rc) return rc;
  return cuda_ok(cudaStreamSynchronize(m->stream), "initial temperatures");
}

// the block temperatures of the model's state
static int read_temps(hsb_dev_model *m, double *block_temp) {
  const size_t nb = (size_t)m->total_n_blocks + m->nx;
  if (cudaSetDevice(m->device) != cudaSuccess) return set_error(HSB_E_CUDA, "cudaSetDevice");
  int rc = g2b(m, m->y, m->blk_out);
  if (rc) return rc;
  HSB_CUDA(cudaMemcpyAsync(block_temp, m->blk_out, sizeof(double) * nb, cudaMemcpyDeviceToHost, m->stream));
  return cuda_ok(cudaStreamSynchronize(m->stream), "block temperatures");
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
  if (s->batching) {
    const int rc = build_batch(s);
    if (rc) return rc;
  }
  // transients the batch engine serves: a batched, normal-priority pool
  std::vector<char> isb(n, 0);
  int n_engine = 0;
  for (int k = 0; k < n; k++) {
    const hsb_server::Model &M = s->models[reqs[k].model];
    isb[k] = s->batch && reqs[k].kind == HSB_REQ_TRANSIENT && reqs[k].steps >= 1 && M.slot >= 0 && !M.high;
    n_engine += isb[k];
  }
  std::mutex mu;
  std::condition_variable cv;
  std::vector<int> state(n, 0);   // 0 pending, 1 running, 2 done
  std::vector<int> served_by(n, -1);
  int done = 0, running = 0, running_high = 0, running_low = 0, paused_low = 0;
  int engine_on = 0;              // the engine holds admitted requests
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
        if (state[k] != 0 || isb[k]) continue;
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
        // nothing runs, nothing more arrives: what is left for the workers
        // waits on memory that no request will free -- fail those requests
        bool failed_some = false;
        for (int k = 0; k < n; k++)
          if (state[k] == 0 && !isb[k] && reqs[k].arrival <= t) {
            reqs[k].status = set_error(HSB_E_NOMEM, "request not admitted: not enough free device memory");
            reqs[k].start = reqs[k].finish = t;
            state[k] = 2;
            done++;
            failed_some = true;
          }
        if (failed_some) {
          cv.notify_all();
          continue;
        }
        // nothing of the workers' is left: wait for the batch engine's requests
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
        while (paused_low < running_low + engine_on && clk::now() < until) cv.wait_until(lk, until);
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
  // the batch engine: admit, advance one tick, retire
  auto engine = [&]() {
    std::vector<int> act, fresh, grp, chips;
    std::vector<int> prog(n, 0);
    std::vector<double> rows;
    std::unique_lock<std::mutex> lk(mu);
    int eng_done = 0;
    for (;;) {
      if (eng_done == n_engine) return;
      const double t = now();
      double next_arrival = 1e300;
      for (int k = 0; k < n; k++) {
        if (!isb[k] || state[k] != 0) continue;
        const hsb_request &r = reqs[k];
        if (r.arrival > t) {
          next_arrival = std::min(next_arrival, r.arrival);
          continue;
        }
        // an idle batched member of the pool; a transient that continues
        // the named model's state waits for that model
        const int cls = s->models[r.model].cls;
        const bool any = r.temp_in != nullptr;
        int pick = -1;
        for (int q = any ? cls : r.model; q < (int)s->models.size(); q++) {
          const hsb_server::Model &Q = s->models[q];
          if (Q.cls == cls && !Q.busy && Q.slot >= 0) {
            pick = q;
            break;
          }
          if (!any) break;
        }
        if (pick < 0) continue;
        served_by[k] = pick;
        s->models[pick].busy = true;
        state[k] = 1;
        running++;
        reqs[k].start = t;
        reqs[k].worker = -1;
        act.push_back(k);
        fresh.push_back(k);
      }
      engine_on = act.empty() ? 0 : 1;
      if (act.empty()) {
        if (next_arrival < 1e300)
          cv.wait_until(lk, t0 + std::chrono::duration_cast<clk::duration>(std::chrono::duration<double>(next_arrival)));
        else
          cv.wait(lk);
        continue;
      }
      if (running_high > 0) {   // a priority request runs: pause between ticks
        ++paused_low;
        cv.notify_all();
        while (running_high > 0) cv.wait_for(lk, std::chrono::milliseconds(10));
        --paused_low;
        continue;
      }
      // one tick over the admitted requests of the first one's interval length
      const double dt = reqs[act[0]].dt;
      grp.clear();
      chips.clear();
      long long cells = 0;
      int rem = 1 << 30;
      for (int k : act)
        if (reqs[k].dt == dt) {
          grp.push_back(k);
          const hsb_server::Model &M = s->models[served_by[k]];
          chips.push_back(M.slot);
          cells += M.m->ncell;
          rem = std::min(rem, reqs[k].steps - prog[k]);
        }
      int K = (int)std::max(1LL, std::min<long long>(TICK_MAX_INTERVALS, TICK_CELL_INTERVALS / std::max(1LL, cells)));
      K = std::min(K, rem);
      std::vector<int> load(fresh);
      fresh.clear();
      lk.unlock();
      int rc = HSB_OK;
      std::vector<int> failed;
      for (int k : load)   // initial temperatures of the requests admitted at this tick
        if (reqs[k].temp_in) {
          const int r2 = load_temps(s->models[served_by[k]].m, reqs[k].temp_in);
          if (r2) {
            reqs[k].status = r2;
            failed.push_back(k);
          }
        }
      if (!failed.empty()) rc = HSB_E_CUDA;
      if (rc == HSB_OK) {   // K rows of the group's block vectors, packed in group order
        size_t nbt = 0;
        for (int c : chips) nbt += (size_t)(s->boff[c + 1] - s->boff[c]);
        rows.resize((size_t)K * nbt);
        size_t o = 0;
        for (size_t q = 0; q < grp.size(); q++) {
          const hsb_request &r = reqs[grp[q]];
          const size_t nb = (size_t)(s->boff[chips[q] + 1] - s->boff[chips[q]]);
          for (int i = 0; i < K; i++)
            memcpy(rows.data() + (size_t)i * nbt + o, r.power + (size_t)(prog[grp[q]] + i) * nb, sizeof(double) * nb);
          o += nb;
        }
        hsb_stats st;
        memset(&st, 0, sizeof(st));
        rc = hsb_batch_run_subset(s->batch, chips.data(), (int)chips.size(), rows.data(), K, dt, &st);
      }
      std::vector<int> fin;
      for (int k : grp) {
        const bool last = prog[k] + K >= reqs[k].steps;
        if (rc == HSB_OK && last) {
          const int r2 = read_temps(s->models[served_by[k]].m, reqs[k].out);
          reqs[k].status = r2;
          fin.push_back(k);
        } else if (rc != HSB_OK) {
          if (std::find(failed.begin(), failed.end(), k) == failed.end()) reqs[k].status = rc;
          fin.push_back(k);
        }
      }
      lk.lock();
      if (rc == HSB_OK) {
        s->ticks++;
        s->tick_requests += (long long)grp.size();
        s->tick_intervals += (long long)grp.size() * K;
      }
      for (int k : grp) prog[k] += K;
      if (rc != HSB_OK && first_error.empty()) first_error = hsb_dev_last_error();
      for (int k : fin) {
        hsb_request &r = reqs[k];
        r.finish = now();
        if (r.status != HSB_OK && first_error.empty()) first_error = hsb_dev_last_error();
        hsb_server::Model &M = s->models[served_by[k]];
        if (r.status == HSB_OK) M.warm = true;
        M.busy = false;
        state[k] = 2;
        running--;
        done++;
        eng_done++;
        act.erase(std::find(act.begin(), act.end(), k));
      }
      // a request that failed while loading its temperatures, outside the tick's group
      for (int k : failed)
        if (state[k] == 1) {
          reqs[k].finish = now();
          s->models[served_by[k]].busy = false;
          state[k] = 2;
          running--;
          done++;
          eng_done++;
          act.erase(std::find(act.begin(), act.end(), k));
        }
      engine_on = act.empty() ? 0 : 1;
      cv.notify_all();
    }
  };
  std::vector<std::thread> pool;
  const int threads = s->workers + (any_high ? HIGH_SLOTS : 0);
  for (int w = 0; w < threads; w++) pool.emplace_back(worker, w);
  if (n_engine) pool.emplace_back(engine);
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
