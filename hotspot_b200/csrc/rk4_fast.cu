// rk4_fast.cu -- the fast transient form (HSB_FORM_FAST).
//
// The same adaptive step-doubling RK4 as the reference (RCutil.c:544-640,
// including the reuse of k1 = f(t1) on a retry) and the same interval loop
// (temperature_grid.c:3676-3692), run as ONE cooperative persistent kernel
// per sampling interval:
//   * every RK4 stage is a grid-stride pass over (i, j) columns, each thread
//     walking the layers so vertical neighbours stay in registers; stage
//     inputs t = y + a*k are formed on the fly (no axpy passes);
//   * stencil arithmetic in FP32: neighbour differences are taken in FP64
//     (y is FP64) and rounded once to FP32, slopes k are stored in FP32;
//   * state y, the RK4 combination y + h(k1+2k2+2k3+k4)/6 and the error
//     norm |ytemp - t2| stay in FP64;
//   * the package nodes' edge sums are reduced by dedicated warps in a fixed
//     order (deterministic); every CTA then evaluates the package nodes
//     redundantly in shared memory, so one grid barrier per stage suffices;
//   * step-size control runs on the device: each CTA reads the global
//     max-norm after the barrier and takes the identical decision.
#include <cooperative_groups.h>

#include <cmath>

#include "stencil_exact.cuh"

namespace cg = cooperative_groups;

namespace hsb {

#define FT_THREADS 256
#define FT_WARPS (FT_THREADS / 32)
#define NXMAX (HSB_EXTRA + HSB_EXTRA_SEC)

struct LayerF {
  float gNS, gEW;       // lateral conductances
  float gDown;          // conductance to layer n+1 (1/rz[n])
  float invC;           // 1 / capacitance
  float gEdgeNS, gEdgeEW, gAmb;
  int kind;
};

struct FastWork {
  long long ncell;
  int grid, coef_version;
  float *k1, *k2, *k3, *pf;
  double *ytemp, *t1, *t2;
  float *gN, *gS, *gW, *gE, *gA, *gB, *invC;
  float *aN, *aS, *aW, *aE, *aO;
  LayerF *Lf;
  double *es;                     // [2][20] edge sums
  unsigned long long *err;        // [2] max-norm bits
  long long *cnt;                 // [0]=steps [1]=attempts [2]=final buffer [3]=status
  long long *h_cnt;               // pinned mirror
};

struct FastArgs {
  StencilArgs S;                  // FP64 layer table and package (for the package nodes)
  int spidx, hsidx, subidx, solderidx, pcbidx;
  const LayerF *Lf;
  const float *gN, *gS, *gW, *gE, *gA, *gB, *invC;
  const float *aN, *aS, *aW, *aE, *aO;
  const double *qin;
  const double *pgrid;
  float *pf;
  double *y, *ytemp, *t1, *t2;
  float *k1, *k2, *k3;
  double *es;
  unsigned long long *err;
  long long *cnt;
  double T;
  long long max_attempts;
};

enum { M_K = 0, M_COMBINE = 1, M_COMBINE_ERR = 2 };

struct StageIO {
  const double *yb;     // base state of the stage (grid part)
  const double *ypb;    // base state, package part (shared memory)
  const float *kin;     // slope the input is formed with (null: t = y)
  const double *kinp;
  double a;             // t = y + a * kin
  float *kout;          // output slope (M_K)
  double *koutp;
  // combine
  const float *k1, *k2;
  const double *k1p, *k2p;
  double h;
  double *yout, *youtp;
  const double *ycmp, *ycmpp;
};

__device__ __forceinline__ float tdiff(double ynb, double yc, float a, float knb, float kc) {
  // (y_nb + a k_nb) - (y_c + a k_c), the FP64 part first
  return (float)(ynb - yc) + a * (knb - kc);
}

template <bool FIELD, bool ADV, int MODE>
__device__ __forceinline__ double stage(const FastArgs &A, cg::grid_group &grid, const StageIO &io,
                                        int &ep, int &sp, double *xs, double *es_s, double *dv,
                                        double *wred) {
  const StencilArgs &S = A.S;
  const int nl = S.nl, nr = S.nr, nc = S.nc, nx = S.nx;
  const long long plane = S.plane, ncell = S.ncell;
  const float af = (float)io.a;
  const bool hasK = io.kin != nullptr;
  double errl = 0.0;

  // package-node temperatures of this stage's input
  if (threadIdx.x < nx) xs[threadIdx.x] = hasK ? io.ypb[threadIdx.x] + io.a * io.kinp[threadIdx.x]
                                               : io.ypb[threadIdx.x];
  __syncthreads();

  // edge sums sum_k (t_k - x_node), one warp per edge, fixed order
  {
    const int ne = S.secondary ? 20 : 8;
    const int gw = blockIdx.x * FT_WARPS + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (gw < ne) {
      int layer, which, node;
      edge_desc(gw, A.spidx, A.hsidx, A.subidx, A.solderidx, A.pcbidx, &layer, &which, &node);
      const double x = xs[node];
      const int len = which < 2 ? nc : nr;
      const long long base = (long long)layer * plane +
                             (which == 0 ? 0 : which == 1 ? (long long)(nr - 1) * nc : which == 2 ? 0 : nc - 1);
      const long long stride = which < 2 ? 1 : nc;
      double s = 0.0;
      for (int q = lane; q < len; q += 32) {
        const long long c = base + q * stride;
        const double t = hasK ? io.yb[c] + io.a * (double)io.kin[c] : io.yb[c];
        s += t - x;
      }
      for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
      if (lane == 0) A.es[sp * 20 + gw] = s;
    }
  }

  // grid cells, one (i, j) column per thread iteration
  const long long ncol = plane;
  for (long long col = (long long)blockIdx.x * blockDim.x + threadIdx.x; col < ncol;
       col += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(col / nc), j = (int)(col - (long long)i * nc);
    double yUp = 0.0, yC = io.yb[col];
    float kUp = 0.f, kC = hasK ? io.kin[col] : 0.f;
    for (int n = 0; n < nl; n++) {
      const long long c = (long long)n * plane + col;
      double yDn = 0.0;
      float kDn = 0.f;
      if (n < nl - 1) {
        yDn = io.yb[c + plane];
        kDn = hasK ? io.kin[c + plane] : 0.f;
      }
      const LayerF &L = A.Lf[n];
      float psum = 0.f;
      if (i > 0) {
        const float g = FIELD ? A.gN[c] : L.gNS;
        psum += g * tdiff(io.yb[c - nc], yC, af, hasK ? io.kin[c - nc] : 0.f, kC);
      }
      if (i < nr - 1) {
        const float g = FIELD ? A.gS[c] : L.gNS;
        psum += g * tdiff(io.yb[c + nc], yC, af, hasK ? io.kin[c + nc] : 0.f, kC);
      }
      if (j < nc - 1) {
        const float g = FIELD ? A.gE[c] : L.gEW;
        psum += g * tdiff(io.yb[c + 1], yC, af, hasK ? io.kin[c + 1] : 0.f, kC);
      }
      if (j > 0) {
        const float g = FIELD ? A.gW[c] : L.gEW;
        psum += g * tdiff(io.yb[c - 1], yC, af, hasK ? io.kin[c - 1] : 0.f, kC);
      }
      if (n > 0) {
        const float g = FIELD ? A.gA[c] : A.Lf[n - 1].gDown;
        psum += g * tdiff(yUp, yC, af, kUp, kC);
      }
      if (n < nl - 1) {
        const float g = FIELD ? A.gB[c] : L.gDown;
        psum += g * tdiff(yDn, yC, af, kDn, kC);
      }
      if (L.kind != LK_PLAIN) {
        int eN, eS, eE, eW;
        switch (L.kind) {
          case LK_SPREADER: eN = HSB_SP_N; eS = HSB_SP_S; eE = HSB_SP_E; eW = HSB_SP_W; break;
          case LK_SINK:
            psum += L.gAmb * ((float)(S.ambient - yC) - af * kC);
            eN = HSB_SINK_C_N; eS = HSB_SINK_C_S; eE = HSB_SINK_C_E; eW = HSB_SINK_C_W; break;
          case LK_PCB:
            psum += L.gAmb * ((float)(S.ambient - yC) - af * kC);
            eN = HSB_PCB_C_N; eS = HSB_PCB_C_S; eE = HSB_PCB_C_E; eW = HSB_PCB_C_W; break;
          case LK_SUB: eN = HSB_SUB_N; eS = HSB_SUB_S; eE = HSB_SUB_E; eW = HSB_SUB_W; break;
          default: eN = HSB_SOLDER_N; eS = HSB_SOLDER_S; eE = HSB_SOLDER_E; eW = HSB_SOLDER_W; break;
        }
        if (i == 0) psum += L.gEdgeNS * ((float)(xs[eN] - yC) - af * kC);
        if (i == nr - 1) psum += L.gEdgeNS * ((float)(xs[eS] - yC) - af * kC);
        if (j == nc - 1) psum += L.gEdgeEW * ((float)(xs[eE] - yC) - af * kC);
        if (j == 0) psum += L.gEdgeEW * ((float)(xs[eW] - yC) - af * kC);
      }
      if (ADV && ((S.uchan_mask >> n) & 1ull)) {
        // advection carries absolute temperatures: FP64
        const double tc = yC + io.a * (double)kC;
        double adv = 0.0;
        if (i > 0) adv += (double)A.aN[c] * ((io.yb[c - nc] + io.a * (double)(hasK ? io.kin[c - nc] : 0.f) + tc) / 2.0);
        if (i < nr - 1) adv += (double)A.aS[c] * ((io.yb[c + nc] + io.a * (double)(hasK ? io.kin[c + nc] : 0.f) + tc) / 2.0);
        if (j > 0) adv += (double)A.aW[c] * ((io.yb[c - 1] + io.a * (double)(hasK ? io.kin[c - 1] : 0.f) + tc) / 2.0);
        if (j < nc - 1) adv += (double)A.aE[c] * ((io.yb[c + 1] + io.a * (double)(hasK ? io.kin[c + 1] : 0.f) + tc) / 2.0);
        adv += A.qin[c] + (double)A.aO[c] * tc;
        psum += (float)adv;
      }
      const float k = (A.pf[c] + psum) * (FIELD ? A.invC[c] : L.invC);
      if (MODE == M_K) {
        io.kout[c] = k;
      } else {
        const double yo = io.yb[c] + io.h * ((double)io.k1[c] + 2.0 * (double)io.k2[c] +
                                             2.0 * (double)kC + (double)k) / 6.0;
        io.yout[c] = yo;
        if (MODE == M_COMBINE_ERR) errl = fmax(errl, fabs(io.ycmp[c] - yo));
      }
      yUp = yC; kUp = kC;
      yC = yDn; kC = kDn;
    }
  }
  if (MODE == M_COMBINE_ERR) {
    for (int o = 16; o > 0; o >>= 1) errl = fmax(errl, __shfl_down_sync(0xffffffffu, errl, o));
    if ((threadIdx.x & 31) == 0) wred[threadIdx.x >> 5] = errl;
    __syncthreads();
    if (threadIdx.x == 0) {
      double mx = wred[0];
      for (int w = 1; w < FT_WARPS; w++) mx = fmax(mx, wred[w]);
      atomicMax(A.err + ep, (unsigned long long)__double_as_longlong(mx));
    }
  }
  grid.sync();

  // package nodes, evaluated identically by every CTA
  const int ne = S.secondary ? 20 : 8;
  if (threadIdx.x < ne) es_s[threadIdx.x] = A.es[sp * 20 + threadIdx.x];
  __syncthreads();
  if (threadIdx.x == 0) pack_slope_exact(S, xs, es_s, dv, A.spidx, A.hsidx, A.subidx, A.solderidx, A.pcbidx);
  __syncthreads();
  double perr = 0.0;
  if (threadIdx.x < nx) {
    const int q = threadIdx.x;
    if (MODE == M_K) {
      io.koutp[q] = dv[q];
    } else {
      const double yo = io.ypb[q] + io.h * (io.k1p[q] + 2.0 * io.k2p[q] + 2.0 * io.kinp[q] + dv[q]) / 6.0;
      io.youtp[q] = yo;
      if (MODE == M_COMBINE_ERR) perr = fabs(io.ycmpp[q] - yo);
    }
  }
  sp ^= 1;
  if (MODE == M_COMBINE_ERR) {
    // global max of the grid cells (visible after the barrier) and of the package nodes
    for (int o = 16; o > 0; o >>= 1) perr = fmax(perr, __shfl_down_sync(0xffffffffu, perr, o));
    __shared__ double pmax;
    if (threadIdx.x == 0) pmax = perr;
    __syncthreads();
    const double gmax = __longlong_as_double((long long)(*(volatile unsigned long long *)(A.err + ep)));
    const double mx = fmax(gmax, pmax);
    __syncthreads();
    if (blockIdx.x == 0 && threadIdx.x == 0) A.err[ep ^ 1] = 0ull;
    ep ^= 1;
    return mx;
  }
  __syncthreads();
  return 0.0;
}

template <bool FIELD, bool ADV>
__device__ __forceinline__ void core(const FastArgs &A, cg::grid_group &grid, const double *yb,
                                     const double *ypb, const float *k1, const double *k1p, double h,
                                     double *yout, double *youtp, const double *ycmp,
                                     const double *ycmpp, double *kp2, double *kp3, int &ep, int &sp,
                                     double *xs, double *es_s, double *dv, double *wred, double *errp) {
  StageIO io{};
  io.yb = yb; io.ypb = ypb;
  io.kin = k1; io.kinp = k1p; io.a = h / 2.0; io.kout = A.k2; io.koutp = kp2;
  stage<FIELD, ADV, M_K>(A, grid, io, ep, sp, xs, es_s, dv, wred);
  io.kin = A.k2; io.kinp = kp2; io.a = h / 2.0; io.kout = A.k3; io.koutp = kp3;
  stage<FIELD, ADV, M_K>(A, grid, io, ep, sp, xs, es_s, dv, wred);
  io.kin = A.k3; io.kinp = kp3; io.a = h;
  io.k1 = k1; io.k2 = A.k2; io.k1p = k1p; io.k2p = kp2; io.h = h;
  io.yout = yout; io.youtp = youtp; io.ycmp = ycmp; io.ycmpp = ycmpp;
  if (ycmp) *errp = stage<FIELD, ADV, M_COMBINE_ERR>(A, grid, io, ep, sp, xs, es_s, dv, wred);
  else stage<FIELD, ADV, M_COMBINE>(A, grid, io, ep, sp, xs, es_s, dv, wred);
}

template <bool FIELD, bool ADV>
__global__ void __launch_bounds__(FT_THREADS) rk4_fast_kernel(FastArgs A) {
  cg::grid_group grid = cg::this_grid();
  __shared__ double yp[NXMAX], kp1[NXMAX], kp2[NXMAX], kp3[NXMAX], ytp[NXMAX], t1p[NXMAX], t2p[NXMAX];
  __shared__ double xs[NXMAX], dv[NXMAX], es_s[20], wred[FT_WARPS];
  const StencilArgs &S = A.S;
  const int nx = S.nx;
  // FP32 power for this interval
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < S.ncell;
       c += (long long)gridDim.x * blockDim.x)
    A.pf[c] = (float)A.pgrid[c];
  if (threadIdx.x < nx) yp[threadIdx.x] = A.y[S.ncell + threadIdx.x];
  if (blockIdx.x == 0 && threadIdx.x == 0) { A.err[0] = 0ull; A.err[1] = 0ull; }
  grid.sync();
  double *y = A.y, *ytemp = A.ytemp;
  int ep = 0, sp = 0;
  long long steps = 0, attempts = 0;
  double t, h = 0.0, new_h, mx = 0.0;
  StageIO io{};
  for (t = 0, new_h = 1e-7; t < A.T && new_h >= 1e-7 * 1.0e-6; t += h) {
    h = new_h;
    io.yb = y; io.ypb = yp; io.kin = nullptr; io.kinp = nullptr; io.a = 0.0;
    io.kout = A.k1; io.koutp = kp1;
    stage<FIELD, ADV, M_K>(A, grid, io, ep, sp, xs, es_s, dv, wred);     // k1 = f(y)
    do {
      h = new_h;
      core<FIELD, ADV>(A, grid, y, yp, A.k1, kp1, h, ytemp, ytp, nullptr, nullptr, kp2, kp3, ep, sp,
                       xs, es_s, dv, wred, &mx);
      core<FIELD, ADV>(A, grid, y, yp, A.k1, kp1, h / 2.0, A.t1, t1p, nullptr, nullptr, kp2, kp3, ep,
                       sp, xs, es_s, dv, wred, &mx);
      io.yb = A.t1; io.ypb = t1p; io.kin = nullptr; io.kinp = nullptr; io.a = 0.0;
      io.kout = A.k1; io.koutp = kp1;
      stage<FIELD, ADV, M_K>(A, grid, io, ep, sp, xs, es_s, dv, wred);   // k1 = f(t1)
      core<FIELD, ADV>(A, grid, A.t1, t1p, A.k1, kp1, h / 2.0, A.t2, t2p, ytemp, ytp, kp2, kp3, ep,
                       sp, xs, es_s, dv, wred, &mx);
      attempts++;
      if (mx <= 0.01) {
        new_h = 0.95 * h * pow(fabs(0.01 / mx), 0.2);
        if (new_h > 5.0 * h) new_h = 5.0 * h;
      } else {
        new_h = 0.95 * h * pow(fabs(0.01 / mx), 0.25);
        if (new_h < h / 10.0) new_h = h / 10.0;
      }
      if (attempts >= A.max_attempts) break;
    } while (new_h < h);
    if (attempts >= A.max_attempts) break;
    // commit: the full-step result becomes the state
    double *tmp = y; y = ytemp; ytemp = tmp;
    if (threadIdx.x < nx) yp[threadIdx.x] = ytp[threadIdx.x];
    __syncthreads();
    steps++;
    new_h = new_h < A.T - t - h ? new_h : A.T - t - h;
  }
  if (blockIdx.x == 0) {
    if (threadIdx.x < nx) y[S.ncell + threadIdx.x] = yp[threadIdx.x];
    if (threadIdx.x == 0) {
      A.cnt[0] = steps;
      A.cnt[1] = attempts;
      A.cnt[2] = (y == A.y) ? 0 : 1;
      A.cnt[3] = attempts >= A.max_attempts ? 1 : 0;
    }
  }
}

static void free_fast(void *p) {
  FastWork *w = (FastWork *)p;
  if (!w) return;
  void *bufs[] = {w->k1, w->k2, w->k3, w->pf, w->ytemp, w->t1, w->t2, w->gN, w->gS, w->gW, w->gE,
                  w->gA, w->gB, w->invC, w->aN, w->aS, w->aW, w->aE, w->aO, w->Lf, w->es, w->err, w->cnt};
  for (void *b : bufs)
    if (b) cudaFree(b);
  if (w->h_cnt) cudaFreeHost(w->h_cnt);
  delete w;
}

__global__ void to_float_recip(const double *__restrict__ r, float *__restrict__ g, long long n) {
  long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) g[k] = r[k] != 0.0 ? (float)(1.0 / r[k]) : 0.f;
}
__global__ void to_float(const double *__restrict__ r, float *__restrict__ g, long long n) {
  long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) g[k] = (float)r[k];
}

// (re)build the FP32 coefficient tables from the device model's FP64 ones
static int fast_prepare(hsb_dev_model *m, FastWork **out) {
  FastWork *w = (FastWork *)m->fast;
  const long long n = m->ncell;
  if (!w) {
    w = new FastWork();
    memset(w, 0, sizeof(*w));
    w->ncell = n;
    w->coef_version = -1;
    m->fast = w;
    m->fast_free = free_fast;
    HSB_CUDA(cudaMalloc(&w->k1, sizeof(float) * n));
    HSB_CUDA(cudaMalloc(&w->k2, sizeof(float) * n));
    HSB_CUDA(cudaMalloc(&w->k3, sizeof(float) * n));
    HSB_CUDA(cudaMalloc(&w->pf, sizeof(float) * n));
    HSB_CUDA(cudaMalloc(&w->ytemp, sizeof(double) * m->vlen));
    HSB_CUDA(cudaMalloc(&w->t1, sizeof(double) * m->vlen));
    HSB_CUDA(cudaMalloc(&w->t2, sizeof(double) * m->vlen));
    HSB_CUDA(cudaMalloc(&w->Lf, sizeof(LayerF) * HSB_MAX_LAYERS));
    HSB_CUDA(cudaMalloc(&w->es, sizeof(double) * 40));
    HSB_CUDA(cudaMalloc(&w->err, sizeof(unsigned long long) * 2));
    HSB_CUDA(cudaMalloc(&w->cnt, sizeof(long long) * 4));
    HSB_CUDA(cudaMallocHost(&w->h_cnt, sizeof(long long) * 4));
    int per_sm = 0, nsm = 0, dev = m->device;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const bool adv = m->uchan_mask != 0;
    const void *fn = m->field ? (adv ? (const void *)rk4_fast_kernel<true, true> : (const void *)rk4_fast_kernel<true, false>)
                              : (adv ? (const void *)rk4_fast_kernel<false, true> : (const void *)rk4_fast_kernel<false, false>);
    HSB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, FT_THREADS, 0));
    const long long need = (m->plane + FT_THREADS - 1) / FT_THREADS;
    long long g = (long long)per_sm * nsm;
    if (g > need) g = need < 1 ? 1 : need;
    w->grid = (int)g;
  }
  if (w->coef_version == m->coef_version) {
    *out = w;
    return HSB_OK;
  }
  w->coef_version = m->coef_version;
  // per-layer FP32 coefficients from the FP64 table
  LayerF Lf[HSB_MAX_LAYERS];
  for (int l = 0; l < m->nl; l++) {
    const LayerCoef &c = m->hostL0[l];
    Lf[l].gNS = (float)(1.0 / c.rNS);
    Lf[l].gEW = (float)(1.0 / c.rEW);
    Lf[l].gDown = (float)(1.0 / c.rz);
    Lf[l].invC = c.cap != 0.0 ? (float)(1.0 / c.cap) : 0.f;
    Lf[l].gEdgeNS = c.edgeNS != 0.0 ? (float)(1.0 / c.edgeNS) : 0.f;
    Lf[l].gEdgeEW = c.edgeEW != 0.0 ? (float)(1.0 / c.edgeEW) : 0.f;
    Lf[l].gAmb = c.ramb != 0.0 ? (float)(1.0 / c.ramb) : 0.f;
    Lf[l].kind = c.kind;
  }
  HSB_CUDA(cudaMemcpyAsync(w->Lf, Lf, sizeof(LayerF) * m->nl, cudaMemcpyHostToDevice, m->stream));
  const int T = 256;
  const unsigned B = (unsigned)((n + T - 1) / T);
  if (m->field) {
    float **g[] = {&w->gN, &w->gS, &w->gW, &w->gE, &w->gA, &w->gB};
    const double *r[] = {m->rN, m->rS, m->rW, m->rE, m->rA, m->rB};
    for (int q = 0; q < 6; q++) {
      if (!*g[q]) HSB_CUDA(cudaMalloc(g[q], sizeof(float) * n));
      to_float_recip<<<B, T, 0, m->stream>>>(r[q], *g[q], n);
    }
    if (!w->invC) HSB_CUDA(cudaMalloc(&w->invC, sizeof(float) * n));
    to_float_recip<<<B, T, 0, m->stream>>>(m->cap, w->invC, n);
  }
  if (m->uchan_mask) {
    float **a[] = {&w->aN, &w->aS, &w->aW, &w->aE, &w->aO};
    const double *s[] = {m->aN, m->aS, m->aW, m->aE, m->aO};
    for (int q = 0; q < 5; q++) {
      if (!*a[q]) HSB_CUDA(cudaMalloc(a[q], sizeof(float) * n));
      to_float<<<B, T, 0, m->stream>>>(s[q], *a[q], n);
    }
  }
  HSB_CUDA(cudaGetLastError());
  *out = w;
  return HSB_OK;
}

int rk4_fast_interval(hsb_dev_model *m, double time_elapsed, hsb_stats *st) {
  FastWork *w;
  int rc;
  if ((rc = fast_prepare(m, &w))) return rc;
  FastArgs A;
  memset(&A, 0, sizeof(A));
  A.S = make_args(m, m->L0, m->nr, m->nc);
  A.spidx = m->spidx; A.hsidx = m->hsidx;
  A.subidx = m->subidx; A.solderidx = m->solderidx; A.pcbidx = m->pcbidx;
  A.Lf = w->Lf;
  A.gN = w->gN; A.gS = w->gS; A.gW = w->gW; A.gE = w->gE; A.gA = w->gA; A.gB = w->gB;
  A.invC = w->invC;
  A.aN = w->aN; A.aS = w->aS; A.aW = w->aW; A.aE = w->aE; A.aO = w->aO; A.qin = m->qin;
  A.pgrid = m->pgrid; A.pf = w->pf;
  A.y = m->y; A.ytemp = w->ytemp; A.t1 = w->t1; A.t2 = w->t2;
  A.k1 = w->k1; A.k2 = w->k2; A.k3 = w->k3;
  A.es = w->es; A.err = w->err; A.cnt = w->cnt;
  A.T = time_elapsed;
  A.max_attempts = 10000000;
  void *args[] = {&A};
  const bool adv = m->uchan_mask != 0;
  const void *fn = m->field ? (adv ? (const void *)rk4_fast_kernel<true, true> : (const void *)rk4_fast_kernel<true, false>)
                            : (adv ? (const void *)rk4_fast_kernel<false, true> : (const void *)rk4_fast_kernel<false, false>);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, m->stream);
  HSB_CUDA(cudaLaunchCooperativeKernel(fn, dim3(w->grid), dim3(FT_THREADS), args, 0, m->stream));
  cudaEventRecord(e1, m->stream);
  HSB_CUDA(cudaMemcpyAsync(w->h_cnt, w->cnt, sizeof(long long) * 4, cudaMemcpyDeviceToHost, m->stream));
  HSB_CUDA(cudaStreamSynchronize(m->stream));
  {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    st->kernel_ms += ms;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
  }
  st->launches += 1;
  if (w->h_cnt[2]) {   // the state ended in the other buffer
    double *tmp = m->y;
    m->y = w->ytemp;
    w->ytemp = tmp;
  }
  st->rk4_steps += w->h_cnt[0];
  st->rk4_attempts += w->h_cnt[1];
  st->slope_evals += w->h_cnt[0] + 10 * w->h_cnt[1];
  st->sim_time += time_elapsed;
  if (w->h_cnt[3]) return set_error(HSB_E_NOCONV, "fast transient: RK4 attempt cap reached");
  return HSB_OK;
}

// ---------------------------------------------------------------------------
// The same kernel on buffers the caller provides (state, power, and every
// scratch array), for the allocation-free entry point.  Nothing here
// allocates device memory; the per-layer FP32 table is copied into the
// caller's buffer.
// ---------------------------------------------------------------------------
size_t rk4_fast_layer_table_bytes() { return sizeof(LayerF) * HSB_MAX_LAYERS; }

// the state can finish in the scratch buffer: copy it back when it did
__global__ void fast_finish(const long long *__restrict__ cnt, const double *__restrict__ ytemp,
                            double *__restrict__ y, long long n) {
  if (cnt[2] == 0) return;
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n;
       k += (long long)gridDim.x * blockDim.x)
    y[k] = ytemp[k];
}

int rk4_fast_on_buffers(hsb_dev_model *m, const FastBuffers &b, double time_elapsed, hsb_stats *st) {
  if (m->field || m->uchan_mask)
    return set_error(HSB_E_ARG, "this entry point takes models with per-layer conductances only");
  LayerF Lf[HSB_MAX_LAYERS];
  for (int l = 0; l < m->nl; l++) {
    const LayerCoef &c = m->hostL0[l];
    Lf[l].gNS = (float)(1.0 / c.rNS);
    Lf[l].gEW = (float)(1.0 / c.rEW);
    Lf[l].gDown = (float)(1.0 / c.rz);
    Lf[l].invC = c.cap != 0.0 ? (float)(1.0 / c.cap) : 0.f;
    Lf[l].gEdgeNS = c.edgeNS != 0.0 ? (float)(1.0 / c.edgeNS) : 0.f;
    Lf[l].gEdgeEW = c.edgeEW != 0.0 ? (float)(1.0 / c.edgeEW) : 0.f;
    Lf[l].gAmb = c.ramb != 0.0 ? (float)(1.0 / c.ramb) : 0.f;
    Lf[l].kind = c.kind;
  }
  HSB_CUDA(cudaMemcpyAsync(b.layer_table, Lf, sizeof(LayerF) * m->nl, cudaMemcpyHostToDevice, m->stream));
  FastArgs A;
  memset(&A, 0, sizeof(A));
  A.S = make_args(m, m->L0, m->nr, m->nc);
  A.spidx = m->spidx; A.hsidx = m->hsidx;
  A.subidx = m->subidx; A.solderidx = m->solderidx; A.pcbidx = m->pcbidx;
  A.Lf = (const LayerF *)b.layer_table;
  A.pgrid = b.pgrid; A.pf = b.pf;
  A.y = b.y; A.ytemp = b.ytemp; A.t1 = b.t1; A.t2 = b.t2;
  A.k1 = b.k1; A.k2 = b.k2; A.k3 = b.k3;
  A.es = b.es; A.err = b.err; A.cnt = b.cnt;
  A.T = time_elapsed;
  A.max_attempts = 10000000;
  int per_sm = 0, nsm = 0;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, m->device);
  HSB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, rk4_fast_kernel<false, false>, FT_THREADS, 0));
  const long long need = (m->plane + FT_THREADS - 1) / FT_THREADS;
  long long g = (long long)per_sm * nsm;
  if (g > need) g = need < 1 ? 1 : need;
  void *args[] = {&A};
  HSB_CUDA(cudaLaunchCooperativeKernel((const void *)rk4_fast_kernel<false, false>, dim3((unsigned)g),
                                       dim3(FT_THREADS), args, 0, m->stream));
  fast_finish<<<64, 256, 0, m->stream>>>(b.cnt, b.ytemp, b.y, m->vlen);
  HSB_CUDA(cudaGetLastError());
  long long cnt[4];
  HSB_CUDA(cudaMemcpyAsync(cnt, b.cnt, sizeof(cnt), cudaMemcpyDeviceToHost, m->stream));
  HSB_CUDA(cudaStreamSynchronize(m->stream));
  if (st) {
    st->rk4_steps += cnt[0];
    st->rk4_attempts += cnt[1];
    st->slope_evals += cnt[0] + 10 * cnt[1];
    st->sim_time += time_elapsed;
    st->launches += 2;
  }
  if (cnt[3]) return set_error(HSB_E_NOCONV, "fast transient: RK4 attempt cap reached");
  return HSB_OK;
}

}  // namespace hsb
