// rk4_batch.cu -- many grid models (chips) advanced together: the batched
// fast transient form.
//
// A batch is a set of independent models of uneven size: grid sides, layer
// counts and floorplans differ.  One persistent cooperative launch of the
// temporally blocked kernel (rk4_tb.cu) advances every chip by K sampling
// intervals; each chip keeps its own adaptive RK4 step sequence
// (RCutil.c:440-640 as compute_temp_grid drives it, temperature_grid.c:
// 3603-3704), and its arithmetic is exactly that of the single-model fast
// form with the same tile shape.  The block powers of all K intervals are
// copied in once and mapped to each chip's grid inside the kernel
// (xlate_vector_b2g, temperature_grid.c:1888-1929).  The copy, the launch and
// the read-back of the per-chip counters are replayed from a CUDA graph.
//
// Schedule: the co-resident CTAs are divided among the chips.  A chip whose
// work is worth more than a CTA's fair share gets a group of CTAs that meet
// at chip-local barriers (two per RK4 attempt); smaller chips are packed
// several to a CTA and run one after another.  Every CTA belongs to at most
// one group, which it serves first, so groups never wait on each other.
//
// Autotuner: the tile shape of each size class of chips (a tile policy) and
// how finely big chips are split over CTA groups are chosen on the real
// work: while tuning, each call runs one candidate and the fastest per
// cell-step is kept, and remembered for batches of the same shape in the
// process.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "fast_common.cuh"
#include "rk4_tb.cuh"

using namespace hsb;

namespace {

// tile policies: own-tile shape (rows x columns) by grid side
struct Policy {
  int big[2], mid[2], small[2];   // side >= 256, 64..128, < 64
};
const Policy kPolicies[] = {
    {{16, 64}, {16, 32}, {32, 32}},   // 0: wide tiles on big chips
    {{32, 32}, {32, 32}, {32, 32}},   // 1: square tiles
    {{16, 32}, {16, 32}, {16, 32}},   // 2: small tiles (more CTAs per chip)
};
constexpr int kNumPolicies = 3;

void policy_tile(int policy, int nr, int nc, int nl, size_t cap, int *oi, int *oj) {
  const Policy &P = kPolicies[policy];
  const int side = std::max(nr, nc);
  const int *t = side >= 256 ? P.big : side >= 64 ? P.mid : P.small;
  *oi = t[0];
  *oj = t[1];
  // smaller tiles when the layer count does not fit shared memory or the
  // threads' accumulator slots
  while ((2 * (size_t)tb_rcap(nl, *oi, *oj, false, cap) * nl * 4 + tb_static_smem() > cap ||
          *oi * *oj > TB_THREADS * tb_slots_rt(false, nl)) &&
         (*oi > 8 || *oj > 16)) {
    if (*oj >= *oi * 2) *oj /= 2;
    else *oi /= 2;
  }
}

}  // namespace

struct hsb_batch {
  int n = 0, device = 0;
  std::vector<hsb_dev_model *> models;
  std::vector<TChip> h_chips;
  TChip *d_chips = nullptr;
  int4 *d_work = nullptr;
  int *d_wptr = nullptr;
  long long *d_out = nullptr, *h_out = nullptr;
  unsigned *d_bar = nullptr;
  int grid = 0;
  size_t dyn = 0, cap = 0;
  int nsm = 0;
  int cta_cap = 0;      // at most this many CTAs per launch (0: every co-resident CTA)
  // work lists of launches over a subset of the chips (hsb_batch_run_subset)
  int4 *d_swork = nullptr;
  int *d_swptr = nullptr, *h_swptr = nullptr;
  int4 *h_swork = nullptr;
  int scap = 0;         // entries the subset list buffers hold
  cudaStream_t stream = nullptr;
  // schedule
  double split = 1.0;   // a chip gets about split * (its share of the work) CTAs
  int policy = 0;
  int version = 0;      // bumped when the schedule or the buffers change: graphs are re-captured
  // online autotuning: candidate k runs on call k; the fastest per cell-step wins
  struct Cand {
    int policy;
    double split;
    double ms_per_gcs;
  };
  std::vector<Cand> cands;
  int tune_next = -1;
  unsigned long long signature = 0;
  // block powers: K intervals x every chip's vector, chip after chip
  std::vector<long long> boff;
  long long nbtotal = 0;
  double *d_bpow = nullptr, *h_bpow = nullptr;
  int bpow_cap = 0;     // intervals the buffers hold
  // the replayed launch
  struct G {
    int K;
    double T;
    int version, has_power;
    cudaGraphExec_t exec;
  } graph[2] = {};
  int graph_next = 0;
  cudaEvent_t ev[4] = {};
};

static void batch_free(hsb_batch *b) {
  if (!b) return;
  void *d[] = {b->d_chips, b->d_work, b->d_wptr, b->d_out, b->d_bar, b->d_bpow, b->d_swork, b->d_swptr};
  for (void *p : d)
    if (p) cudaFree(p);
  if (b->h_out) cudaFreeHost(b->h_out);
  if (b->h_swork) cudaFreeHost(b->h_swork);
  if (b->h_swptr) cudaFreeHost(b->h_swptr);
  if (b->h_bpow) cudaFreeHost(b->h_bpow);
  for (auto &g : b->graph)
    if (g.exec) cudaGraphExecDestroy(g.exec);
  for (auto e : b->ev)
    if (e) cudaEventDestroy(e);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
}

// tiles of every chip under the current policy, the launch's shared memory,
// and the chips' descriptors on the device
static int batch_tiles(hsb_batch *b) {
  b->dyn = 0;
  for (int c = 0; c < b->n; c++) {
    hsb_dev_model *m = b->models[c];
    FastWork *w = (FastWork *)m->fast;
    TbRes *r = (TbRes *)w->tb;
    int oi, oj;
    policy_tile(b->policy, m->nr, m->nc, m->nl, b->cap, &oi, &oj);
    TChip &C = b->h_chips[c];
    double *y0 = C.y[0], *y1 = C.y[1];
    int rc;
    if ((rc = tb_fill_chip(m, r, y0, y1, w->pf, w->t1, oi, oj, false, b->cap, &C))) return rc;
    C.bar = b->d_bar + 2 * c;
    b->dyn = std::max(b->dyn, tb_dyn_smem(m->nl, oi, oj, false, b->cap));
  }
  if (b->dyn + tb_static_smem() > b->cap) return set_error(HSB_E_ARG, "batch tiles do not fit shared memory");
  HSB_CUDA(h2d_on(b->d_chips, b->h_chips.data(), sizeof(TChip) * b->n, b->stream));
  return raise_smem_limit(tb_kernel(), b->dyn);
}

// CTA work lists of the chips in `chips` over G CTAs: a chip worth more than
// a CTA's fair share gets a group of CTAs (chip-local barriers), the rest are
// packed onto single CTAs, longest first onto the least loaded
// work item: (chip, rank in its CTA group, group size, offset of the chip's
// block powers in a row of the launch's power rows); off[k] for chips[k]
static void batch_lists(const hsb_batch *b, const std::vector<int> &chips, const std::vector<long long> &off, int G,
                        std::vector<int4> &work, std::vector<int> &wptr) {
  const int n = (int)chips.size();
  // work of a chip: its tiles x the work of a tile x layers
  std::vector<double> wk(n);
  double W = 0;
  for (int k = 0; k < n; k++) {
    const TChip &C = b->h_chips[chips[k]];
    wk[k] = (double)C.ntiles * tb_tile_work(C.oi, C.oj) * C.nl;
    W += wk[k];
  }
  std::vector<int> order(n);
  for (int k = 0; k < n; k++) order[k] = k;
  std::sort(order.begin(), order.end(), [&](int a, int c) { return wk[a] > wk[c]; });
  const double share = W / G;
  std::vector<int> g(n, 1);
  double w_small = 0.0, sum_g = 0.0;
  for (int k = 0; k < n; k++) {
    // a chip worth more than one fair share gets enough CTAs that none of
    // them carries more than a share (rounded up), at most one per tile
    const double ratio = wk[k] / share * b->split;
    int q = ratio > 1.0 ? (int)ceil(ratio) : 1;
    if (q > b->h_chips[chips[k]].ntiles) q = b->h_chips[chips[k]].ntiles;
    if (q >= 2) {
      g[k] = q;
      sum_g += q;
    } else {
      g[k] = 1;
      w_small += wk[k];
    }
  }
  int g_small = (int)ceil(w_small / share);
  if (w_small > 0 && g_small < 1) g_small = 1;
  if (g_small > G - 1) g_small = G - 1;
  const double avail = G - g_small;
  if (sum_g > avail) {   // scale the groups down to the CTAs left
    const double f = avail / sum_g;
    for (int k = 0; k < n; k++)
      if (g[k] >= 2) {
        int q = (int)(g[k] * f);
        if (q < 2) {
          q = 1;
          w_small += wk[k];
        }
        g[k] = q;
      }
  }
  std::vector<std::vector<int4>> lists;
  std::vector<double> load;
  for (int k : order)
    if (g[k] >= 2)
      for (int r = 0; r < g[k]; r++) {
        lists.push_back({make_int4(chips[k], r, g[k], (int)off[k])});
        load.push_back(wk[k] / g[k]);
      }
  const int base = (int)lists.size();
  const int remaining = G - base > 0 ? G - base : 1;
  for (int k = 0; k < remaining; k++) {
    lists.push_back({});
    load.push_back(0.0);
  }
  for (int k : order) {
    if (g[k] >= 2) continue;
    int best = base;
    for (int q = base; q < (int)lists.size(); q++)
      if (load[q] < load[best]) best = q;
    lists[best].push_back(make_int4(chips[k], 0, 1, (int)off[k]));
    load[best] += wk[k];
  }
  work.clear();
  wptr.assign(1, 0);
  for (auto &l : lists) {
    if (l.empty()) continue;
    for (auto &a : l) work.push_back(a);
    wptr.push_back((int)work.size());
  }
}

// co-resident CTAs of a launch (at most the cap set by hsb_batch_set_ctas)
static int batch_ctas(hsb_batch *b, int *G) {
  int per_sm = 0;
  HSB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, tb_kernel(), TB_THREADS, b->dyn));
  if (per_sm < 1) return set_error(HSB_E_ARG, "batch kernel does not fit an SM");
  *G = per_sm * b->nsm;
  if (b->cta_cap > 0 && *G > b->cta_cap) *G = b->cta_cap;
  return HSB_OK;
}

// CTA work lists for the current schedule (every chip)
static int batch_schedule(hsb_batch *b) {
  int rc, G;
  if ((rc = batch_tiles(b))) return rc;
  if ((rc = batch_ctas(b, &G))) return rc;
  std::vector<int> all(b->n);
  std::vector<long long> off(b->n);
  for (int c = 0; c < b->n; c++) {
    all[c] = c;
    off[c] = b->boff[c];
  }
  std::vector<int4> work;
  std::vector<int> wptr;
  batch_lists(b, all, off, G, work, wptr);
  if (b->d_work) cudaFree(b->d_work);
  if (b->d_wptr) cudaFree(b->d_wptr);
  b->d_work = nullptr;
  b->d_wptr = nullptr;
  HSB_CUDA(cudaMalloc(&b->d_work, sizeof(int4) * (work.size() + 1)));
  HSB_CUDA(cudaMalloc(&b->d_wptr, sizeof(int) * wptr.size()));
  HSB_CUDA(h2d_on(b->d_work, work.data(), sizeof(int4) * work.size(), b->stream));
  HSB_CUDA(h2d_on(b->d_wptr, wptr.data(), sizeof(int) * wptr.size(), b->stream));
  b->grid = (int)wptr.size() - 1;
  b->version++;
  return HSB_OK;
}

// block-power buffers for K intervals
static int batch_bpow(hsb_batch *b, int K) {
  if (K <= b->bpow_cap) return HSB_OK;
  if (b->d_bpow) cudaFree(b->d_bpow);
  if (b->h_bpow) cudaFreeHost(b->h_bpow);
  b->d_bpow = nullptr;
  b->h_bpow = nullptr;
  b->bpow_cap = 0;
  HSB_CUDA(cudaMalloc(&b->d_bpow, sizeof(double) * b->nbtotal * K));
  HSB_CUDA(cudaMallocHost(&b->h_bpow, sizeof(double) * b->nbtotal * K));
  b->bpow_cap = K;
  b->version++;   // the graphs captured the old buffers
  return HSB_OK;
}

// the launch sequence (power copy, barrier reset, kernel, counters back) on
// the batch's stream; events 1 and 2 bracket the kernel
static int batch_enqueue(hsb_batch *b, int K, double T, bool power) {
  const unsigned rec = cudaEventRecordExternal;
  if (power)
    HSB_CUDA(cudaMemcpyAsync(b->d_bpow, b->h_bpow, sizeof(double) * b->nbtotal * K, cudaMemcpyHostToDevice,
                             b->stream));
  HSB_CUDA(cudaMemsetAsync(b->d_bar, 0, sizeof(unsigned) * 2 * b->n, b->stream));
  HSB_CUDA(cudaEventRecordWithFlags(b->ev[1], b->stream, rec));
  const TChip *chips = b->d_chips;
  const int4 *work = b->d_work;
  const int *wptr = b->d_wptr;
  long long *out = b->d_out;
  const double *bpow = b->d_bpow;
  long long nbtot = b->nbtotal;
  long long max_attempts = 10000000;
  int Kk = power ? K : 0;
  void *args[] = {&chips, &work, &wptr, &out, &T, &Kk, &bpow, &nbtot, &max_attempts};
  cudaLaunchConfig_t cfg;
  memset(&cfg, 0, sizeof(cfg));
  cfg.gridDim = dim3(b->grid);
  cfg.blockDim = dim3(TB_THREADS);
  cfg.dynamicSmemBytes = b->dyn;
  cfg.stream = b->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  HSB_CUDA(cudaLaunchKernelExC(&cfg, tb_kernel(), args));
  HSB_CUDA(cudaEventRecordWithFlags(b->ev[2], b->stream, rec));
  HSB_CUDA(cudaMemcpyAsync(b->h_out, b->d_out, sizeof(long long) * TB_OUT * b->n, cudaMemcpyDeviceToHost,
                           b->stream));
  return HSB_OK;
}

// the graph of (K, T, power) for the current schedule, captured on first use
static int batch_graph(hsb_batch *b, int K, double T, bool power, cudaGraphExec_t *exec) {
  for (auto &g : b->graph)
    if (g.exec && g.K == K && g.T == T && g.version == b->version && g.has_power == (int)power) {
      *exec = g.exec;
      return HSB_OK;
    }
  hsb_batch::G &g = b->graph[b->graph_next];
  b->graph_next ^= 1;
  if (g.exec) cudaGraphExecDestroy(g.exec);
  g.exec = nullptr;
  HSB_CUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
  const int rc = batch_enqueue(b, K, T, power);
  cudaGraph_t graph = nullptr;
  const cudaError_t ce = cudaStreamEndCapture(b->stream, &graph);
  if (rc || ce != cudaSuccess || !graph) {
    if (graph) cudaGraphDestroy(graph);
    return rc ? rc : cuda_check(ce, "batch graph capture");
  }
  const cudaError_t ie = cudaGraphInstantiate(&g.exec, graph, 0);
  cudaGraphDestroy(graph);
  if (ie != cudaSuccess) {
    g.exec = nullptr;
    return cuda_check(ie, "batch graph instantiation");
  }
  g.K = K;
  g.T = T;
  g.version = b->version;
  g.has_power = power;
  *exec = g.exec;
  return HSB_OK;
}

extern "C" {

int hsb_batch_create(hsb_batch **out, hsb_dev_model *const *models, int n) {
  if (!out || !models || n < 1) return set_error(HSB_E_ARG, "null argument");
  if (!models[0]) return set_error(HSB_E_ARG, "null model in batch");
  hsb_batch *b = new hsb_batch();
  b->n = n;
  b->models.assign(models, models + n);
  b->device = models[0]->device;
  int rc;
  auto fail = [&](int code) {
    batch_free(b);
    return code;
  };
  if (cudaSetDevice(b->device) != cudaSuccess) return fail(set_error(HSB_E_CUDA, "cudaSetDevice"));
  int capi = 0;
  cudaDeviceGetAttribute(&b->nsm, cudaDevAttrMultiProcessorCount, b->device);
  cudaDeviceGetAttribute(&capi, cudaDevAttrMaxSharedMemoryPerBlockOptin, b->device);
  b->cap = (size_t)capi;
  if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess)
    return fail(set_error(HSB_E_CUDA, "batch stream"));
  for (auto &e : b->ev)
    if (cudaEventCreate(&e) != cudaSuccess) return fail(set_error(HSB_E_CUDA, "batch events"));
  if (cudaMalloc(&b->d_bar, sizeof(unsigned) * 2 * n) != cudaSuccess ||
      cudaMalloc(&b->d_out, sizeof(long long) * TB_OUT * n) != cudaSuccess ||
      cudaMallocHost(&b->h_out, sizeof(long long) * TB_OUT * n) != cudaSuccess ||
      cudaMalloc(&b->d_chips, sizeof(TChip) * n) != cudaSuccess)
    return fail(set_error(HSB_E_NOMEM, "batch control arrays"));
  b->h_chips.resize(n);
  b->boff.resize(n + 1, 0);
  for (int c = 0; c < n; c++) {
    hsb_dev_model *m = models[c];
    if (!m) return fail(set_error(HSB_E_ARG, "null model in batch"));
    if (m->device != b->device) return fail(set_error(HSB_E_ARG, "batch models must share one device"));
    if (!tb_eligible(m))
      return fail(set_error(HSB_E_ARG, "batched transient takes models with per-layer conductances and 3..12 layers"));
    if (!m->b2g_ptr) return fail(set_error(HSB_E_ARG, "batch model without block-grid maps"));
    FastWork *w;
    if ((rc = fast_prepare(m, &w))) return fail(rc);
    TbRes *r = (TbRes *)w->tb;
    rc = tb_res_prepare(m, &r, w->pk);
    w->tb = r;
    if (rc) return fail(rc);
    b->h_chips[c].y[0] = m->y;
    b->h_chips[c].y[1] = w->ytemp;
    b->boff[c + 1] = b->boff[c] + m->total_n_blocks + m->nx;
  }
  b->nbtotal = b->boff[n];
  if (b->nbtotal >= (1LL << 31)) return fail(set_error(HSB_E_ARG, "batch block vectors exceed 2^31 entries"));
  memset(b->h_out, 0, sizeof(long long) * TB_OUT * n);
  if (h2d_on(b->d_out, b->h_out, sizeof(long long) * TB_OUT * n, b->stream) != cudaSuccess)
    return fail(set_error(HSB_E_CUDA, "batch outputs"));
  if ((rc = batch_schedule(b))) return fail(rc);
  if ((rc = batch_bpow(b, 1))) return fail(rc);
  *out = b;
  return HSB_OK;
}

void hsb_batch_destroy(hsb_batch *b) { batch_free(b); }

int hsb_batch_set_schedule(hsb_batch *b, int policy, double split) {
  if (!b || policy < 0 || policy >= kNumPolicies || !(split > 0)) return set_error(HSB_E_ARG, "bad batch schedule");
  b->policy = policy;
  b->split = split;
  return batch_schedule(b);
}

// schedules chosen by the autotuner, by batch shape (process-wide)
static std::mutex g_tune_mu;
static std::vector<std::pair<unsigned long long, hsb_batch::Cand>> g_tuned;

static unsigned long long batch_signature(const hsb_batch *b) {
  std::vector<unsigned long long> keys;
  for (auto *m : b->models)
    keys.push_back(((unsigned long long)m->nl << 40) | ((unsigned long long)m->nr << 20) | m->nc);
  std::sort(keys.begin(), keys.end());
  unsigned long long h = 1469598103934665603ull;
  for (auto k : keys) {
    h ^= k;
    h *= 1099511628211ull;
  }
  return h;
}

int hsb_batch_autotune(hsb_batch *b, int enable) {
  if (!b) return set_error(HSB_E_ARG, "null batch");
  if (!enable) {
    b->tune_next = -1;
    return HSB_OK;
  }
  b->signature = batch_signature(b);
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    for (auto &e : g_tuned)
      if (e.first == b->signature) {   // tuned before: reuse
        b->policy = e.second.policy;
        b->split = e.second.split;
        b->tune_next = -1;
        return batch_schedule(b);
      }
  }
  b->cands.clear();
  const double split[3] = {1.0, 1.5, 2.0};
  for (int p = 0; p < kNumPolicies; p++)
    for (double sp : split) b->cands.push_back({p, sp, 0.0});
  b->tune_next = 0;
  return HSB_OK;
}

int hsb_batch_info(hsb_batch *b, int *grid, long long *cells, int *policy, double *split) {
  if (!b) return set_error(HSB_E_ARG, "null batch");
  long long n = 0;
  for (auto *m : b->models) n += m->ncell;
  if (grid) *grid = b->grid;
  if (cells) *cells = n;
  if (policy) *policy = b->policy;
  if (split) *split = b->split;
  return HSB_OK;
}

int hsb_batch_transient_trace(hsb_batch *b, const double *block_powers, int K, double time_elapsed,
                              hsb_stats *st) {
  if (!b || K < 1) return set_error(HSB_E_ARG, "null batch or no intervals");
  hsb_stats local;
  if (!st) st = &local;
  cudaSetDevice(b->device);
  int rc;
  const int tuning = b->tune_next;
  if (tuning >= 0) {
    b->policy = b->cands[tuning].policy;
    b->split = b->cands[tuning].split;
    if ((rc = batch_schedule(b))) return rc;
  }
  const bool power = block_powers != nullptr;
  if (!power) K = 1;
  if ((rc = batch_bpow(b, K))) return rc;
  if (power) memcpy(b->h_bpow, block_powers, sizeof(double) * b->nbtotal * K);
  // which buffer holds each model's state (single-model calls may have swapped them)
  {
    bool changed = false;
    for (int c = 0; c < b->n; c++) {
      hsb_dev_model *m = b->models[c];
      const long long cur = m->y == b->h_chips[c].y[0] ? 0 : 1;
      if (m->y != b->h_chips[c].y[cur] || ((FastWork *)m->fast)->ytemp != b->h_chips[c].y[cur ^ 1])
        return set_error(HSB_E_ARG, "a batch model's state buffers were reallocated");
      if (b->h_out[(size_t)c * TB_OUT + 6] != cur) changed = true;
      b->h_out[(size_t)c * TB_OUT + 6] = cur;
    }
    if (changed)
      HSB_CUDA(cudaMemcpyAsync(b->d_out, b->h_out, sizeof(long long) * TB_OUT * b->n, cudaMemcpyHostToDevice,
                               b->stream));
  }
  cudaGraphExec_t exec = nullptr;
  if ((rc = batch_graph(b, K, time_elapsed, power, &exec))) return rc;
  HSB_CUDA(cudaEventRecord(b->ev[0], b->stream));
  HSB_CUDA(cudaGraphLaunch(exec, b->stream));
  HSB_CUDA(cudaEventRecord(b->ev[3], b->stream));
  HSB_CUDA(cudaStreamSynchronize(b->stream));
  float ms = 0.f, kms = 0.f;
  cudaEventElapsedTime(&kms, b->ev[1], b->ev[2]);
  cudaEventElapsedTime(&ms, b->ev[0], b->ev[3]);
  st->launches += 1;
  st->kernel_ms += kms;
  st->device_ms += ms;
  // per chip: results, the model's view of its state buffer, fallbacks
  double cs = 0.0;
  for (int c = 0; c < b->n && !rc; c++) {
    hsb_dev_model *m = b->models[c];
    FastWork *w = (FastWork *)m->fast;
    const long long *o = b->h_out + (size_t)c * TB_OUT;
    st->rk4_steps += o[0];
    st->rk4_attempts += o[1];
    st->slope_evals += o[3];
    cs += (double)o[0] * m->ncell;
    const int cur = (int)o[6];
    m->y = b->h_chips[c].y[cur];
    w->ytemp = b->h_chips[c].y[cur ^ 1];
    if (o[2] == 2) rc = set_error(HSB_E_CUDA, "batched transient: a chip barrier did not complete in time");
    else if (o[2] == 1) rc = set_error(HSB_E_NOCONV, "batched transient: RK4 attempt cap reached");
    else if (o[2] == 3) {
      // the retries of a step outgrew the kernel: the stage form finishes that
      // interval of this chip, and the chip's later intervals run one by one
      double tt[2];
      memcpy(tt, &o[4], sizeof(tt));
      const int iv = (int)o[7];
      st->fallbacks += 1;
      for (int k = iv; k < K && !rc; k++) {
        if (power && (rc = b2g(m, b->d_bpow + (long long)k * b->nbtotal + b->boff[c], m->pgrid, HSB_V_POWER)))
          break;
        if (k == iv) {
          rc = rk4_stage_run(m, w, time_elapsed - tt[0], tt[1], st);
        } else {
          void *work = nullptr;
          int fell = 0;
          rc = rk4_fast_interval_begin(m, time_elapsed, st, &work, nullptr);
          if (!rc) rc = cuda_ok(cudaStreamSynchronize(m->stream), "fallback interval");
          if (!rc) rc = rk4_fast_interval_end(m, work, time_elapsed, st, &fell);
        }
      }
      if (!rc) rc = cuda_ok(cudaStreamSynchronize(m->stream), "fallback intervals");
      // the single-model path may have swapped the buffers
      long long now = m->y == b->h_chips[c].y[0] ? 0 : 1;
      b->h_out[(size_t)c * TB_OUT + 6] = now;
      if (!rc && h2d_on(b->d_out + (size_t)c * TB_OUT + 6, &now, sizeof(now), b->stream) !=
                     cudaSuccess)
        rc = set_error(HSB_E_CUDA, "batch state index");
    }
  }
  st->sim_time += time_elapsed * K;
  if (tuning >= 0 && rc == HSB_OK) {
    b->cands[tuning].ms_per_gcs = cs > 0 ? kms / (cs / 1e9) : 1e300;
    b->tune_next = tuning + 1;
    if (b->tune_next >= (int)b->cands.size()) {
      int best = 0;
      for (int k = 1; k < (int)b->cands.size(); k++)
        if (b->cands[k].ms_per_gcs < b->cands[best].ms_per_gcs) best = k;
      const hsb_batch::Cand c = b->cands[best];
      b->policy = c.policy;
      b->split = c.split;
      b->tune_next = -1;
      {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_tuned.push_back({b->signature, c});
      }
      rc = batch_schedule(b);
    }
  }
  return rc;
}

int hsb_batch_transient(hsb_batch *b, const double *block_power, double time_elapsed, hsb_stats *st) {
  return hsb_batch_transient_trace(b, block_power, 1, time_elapsed, st);
}

int hsb_batch_set_ctas(hsb_batch *b, int ctas) {
  if (!b || ctas < 0) return set_error(HSB_E_ARG, "bad CTA cap");
  b->cta_cap = ctas;
  return batch_schedule(b);
}

int hsb_batch_run_subset(hsb_batch *b, const int *chips, int n, const double *block_powers, int K,
                         double time_elapsed, hsb_stats *st) {
  if (!b || !chips || n < 1 || !block_powers || K < 1) return set_error(HSB_E_ARG, "bad subset launch");
  hsb_stats local;
  if (!st) st = &local;
  cudaSetDevice(b->device);
  int rc, G;
  std::vector<char> seen(b->n, 0);
  for (int k = 0; k < n; k++) {
    if (chips[k] < 0 || chips[k] >= b->n) return set_error(HSB_E_ARG, "chip index out of range");
    if (seen[chips[k]]++) return set_error(HSB_E_ARG, "a chip is listed twice");
  }
  if ((rc = batch_bpow(b, K))) return rc;
  if ((rc = batch_ctas(b, &G))) return rc;
  std::vector<int> sub(chips, chips + n);
  std::vector<long long> off(n + 1, 0);   // packed rows: the listed chips' vectors in list order
  for (int k = 0; k < n; k++) off[k + 1] = off[k] + (b->boff[sub[k] + 1] - b->boff[sub[k]]);
  const long long nbt = off[n];
  std::vector<int4> work;
  std::vector<int> wptr;
  batch_lists(b, sub, off, G, work, wptr);
  const int need = (int)std::max(work.size(), wptr.size()) + 1;
  if (need > b->scap) {
    void *p[] = {b->d_swork, b->d_swptr};
    for (void *q : p)
      if (q) cudaFree(q);
    if (b->h_swork) cudaFreeHost(b->h_swork);
    if (b->h_swptr) cudaFreeHost(b->h_swptr);
    b->d_swork = nullptr;
    b->d_swptr = nullptr;
    b->h_swork = nullptr;
    b->h_swptr = nullptr;
    b->scap = 0;
    const int cap = need * 2;
    HSB_CUDA(cudaMalloc(&b->d_swork, sizeof(int4) * cap));
    HSB_CUDA(cudaMalloc(&b->d_swptr, sizeof(int) * cap));
    HSB_CUDA(cudaMallocHost(&b->h_swork, sizeof(int4) * cap));
    HSB_CUDA(cudaMallocHost(&b->h_swptr, sizeof(int) * cap));
    b->scap = cap;
  }
  memcpy(b->h_swork, work.data(), sizeof(int4) * work.size());
  memcpy(b->h_swptr, wptr.data(), sizeof(int) * wptr.size());
  memcpy(b->h_bpow, block_powers, sizeof(double) * nbt * K);
  for (int c : sub) {
    hsb_dev_model *m = b->models[c];
    const long long cur = m->y == b->h_chips[c].y[0] ? 0 : 1;
    if (m->y != b->h_chips[c].y[cur] || ((FastWork *)m->fast)->ytemp != b->h_chips[c].y[cur ^ 1])
      return set_error(HSB_E_ARG, "a batch model's state buffers were reallocated");
    b->h_out[(size_t)c * TB_OUT + 6] = cur;
  }
  HSB_CUDA(cudaMemcpyAsync(b->d_out, b->h_out, sizeof(long long) * TB_OUT * b->n, cudaMemcpyHostToDevice,
                           b->stream));
  HSB_CUDA(cudaMemcpyAsync(b->d_bpow, b->h_bpow, sizeof(double) * nbt * K, cudaMemcpyHostToDevice, b->stream));
  HSB_CUDA(cudaMemcpyAsync(b->d_swork, b->h_swork, sizeof(int4) * work.size(), cudaMemcpyHostToDevice,
                           b->stream));
  HSB_CUDA(cudaMemcpyAsync(b->d_swptr, b->h_swptr, sizeof(int) * wptr.size(), cudaMemcpyHostToDevice,
                           b->stream));
  HSB_CUDA(cudaMemsetAsync(b->d_bar, 0, sizeof(unsigned) * 2 * b->n, b->stream));
  HSB_CUDA(cudaEventRecord(b->ev[1], b->stream));
  const TChip *chips_d = b->d_chips;
  const int4 *work_d = b->d_swork;
  const int *wptr_d = b->d_swptr;
  long long *out = b->d_out;
  const double *bpow = b->d_bpow;
  long long nbtot = nbt;
  long long max_attempts = 10000000;
  int Kk = K;
  double T = time_elapsed;
  void *args[] = {&chips_d, &work_d, &wptr_d, &out, &T, &Kk, &bpow, &nbtot, &max_attempts};
  cudaLaunchConfig_t cfg;
  memset(&cfg, 0, sizeof(cfg));
  cfg.gridDim = dim3((unsigned)(wptr.size() - 1));
  cfg.blockDim = dim3(TB_THREADS);
  cfg.dynamicSmemBytes = b->dyn;
  cfg.stream = b->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  HSB_CUDA(cudaLaunchKernelExC(&cfg, tb_kernel(), args));
  HSB_CUDA(cudaEventRecord(b->ev[2], b->stream));
  HSB_CUDA(cudaMemcpyAsync(b->h_out, b->d_out, sizeof(long long) * TB_OUT * b->n, cudaMemcpyDeviceToHost,
                           b->stream));
  HSB_CUDA(cudaStreamSynchronize(b->stream));
  float kms = 0.f;
  cudaEventElapsedTime(&kms, b->ev[1], b->ev[2]);
  st->launches += 1;
  st->kernel_ms += kms;
  for (int q = 0; q < n; q++) {
    const int c = sub[q];
    hsb_dev_model *m = b->models[c];
    FastWork *w = (FastWork *)m->fast;
    const long long *o = b->h_out + (size_t)c * TB_OUT;
    st->rk4_steps += o[0];
    st->rk4_attempts += o[1];
    const int cur = (int)o[6];
    m->y = b->h_chips[c].y[cur];
    w->ytemp = b->h_chips[c].y[cur ^ 1];
    if (o[2] == 2) return set_error(HSB_E_CUDA, "batched transient: a chip barrier did not complete in time");
    if (o[2] == 1) return set_error(HSB_E_NOCONV, "batched transient: RK4 attempt cap reached");
    if (o[2] == 3) {   // the retries of a step outgrew the kernel: as in hsb_batch_transient_trace
      double tt[2];
      memcpy(tt, &o[4], sizeof(tt));
      const int iv = (int)o[7];
      st->fallbacks += 1;
      for (int k = iv; k < K; k++) {
        if ((rc = b2g(m, b->d_bpow + (long long)k * nbt + off[q], m->pgrid, HSB_V_POWER))) return rc;
        if (k == iv) {
          if ((rc = rk4_stage_run(m, w, time_elapsed - tt[0], tt[1], st))) return rc;
        } else {
          void *wk = nullptr;
          int fell = 0;
          if ((rc = rk4_fast_interval_begin(m, time_elapsed, st, &wk, nullptr))) return rc;
          if ((rc = cuda_ok(cudaStreamSynchronize(m->stream), "fallback interval"))) return rc;
          if ((rc = rk4_fast_interval_end(m, wk, time_elapsed, st, &fell))) return rc;
        }
      }
      if ((rc = cuda_ok(cudaStreamSynchronize(m->stream), "fallback intervals"))) return rc;
    }
  }
  st->sim_time += time_elapsed * K;
  return HSB_OK;
}

// boundaries of the chips' block-power vectors: chip c's row segment is
// [off[c], off[c + 1]) of a row of hsb_batch_transient_trace's layout
int hsb_batch_offsets(hsb_batch *b, long long *off) {
  if (!b || !off) return set_error(HSB_E_ARG, "null argument");
  for (int c = 0; c <= b->n; c++) off[c] = b->boff[c];
  return HSB_OK;
}

// the autotuner's measurements: up to n candidates as (tile policy, split,
// 0, ms per 10^9 cell-steps); returns how many were measured
int hsb_batch_tuning(hsb_batch *b, double *out, int n) {
  if (!b) return set_error(HSB_E_ARG, "null batch");
  int k = 0;
  for (; k < (int)b->cands.size() && k < n; k++) {
    out[4 * k] = b->cands[k].policy;
    out[4 * k + 1] = b->cands[k].split;
    out[4 * k + 2] = 0;
    out[4 * k + 3] = b->cands[k].ms_per_gcs;
  }
  return k;
}

// per-chip accepted steps of the last call (n entries)
int hsb_batch_chip_steps(hsb_batch *b, long long *steps) {
  if (!b || !steps) return set_error(HSB_E_ARG, "null argument");
  for (int c = 0; c < b->n; c++) steps[c] = b->h_out[(size_t)c * TB_OUT];
  return HSB_OK;
}

// own-tile shape of chip c under the current schedule
int hsb_batch_chip_tile(hsb_batch *b, int c, int *rows, int *cols) {
  if (!b || c < 0 || c >= b->n) return set_error(HSB_E_ARG, "bad chip index");
  if (rows) *rows = b->h_chips[c].oi;
  if (cols) *cols = b->h_chips[c].oj;
  return HSB_OK;
}

}  // extern "C"
