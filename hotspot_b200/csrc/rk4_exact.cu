// rk4_exact.cu -- FP64 transient in the reference's exact operation order
// (compiled with -fmad=false).
//
// Replays compute_temp_grid's loop (temperature_grid.c:3676-3692) and the
// step-doubling RK4 of RCutil.c:440-640 on the device.  Each RK4 stage is
// one fused kernel: the stage input t = y + a*k_prev is formed on the fly
// from y and k_prev (no separate axpy pass), the slope is evaluated, and the
// final stage of each rk4_core also forms yout = y + h*(k1+2k2+2k3+k4)/6.0
// and, for the last half step, the max-norm |ytemp - t2| with a block
// reduction plus one atomicMax.  The package nodes are handled by one extra
// block per launch, whose lanes form the edge sums in the reference's
// sequential order.  The host keeps the step-size control, with the C
// library's pow(), so the accepted-step sequence is the reference's.
#include <cmath>

#include "stencil_exact.cuh"

namespace hsb {

enum { EPI_STORE = 0, EPI_COMBINE = 1, EPI_COMBINE_ERR = 2 };

struct Epi {
  const double *k1, *k2, *k3;   // slopes of the current rk4_core
  double h;                     // step of the current rk4_core
  double *yout;                 // y + h*(k1+2k2+2k3+k4)/6.0
  const double *ycmp;           // full-step result compared against
  unsigned long long *errbits;  // max |ycmp - yout| as ordered bits
  int spidx, hsidx, subidx, solderidx, pcbidx;
};

template <bool HAS_K>
struct TVal {
  const double *__restrict__ y;
  const double *__restrict__ k;
  double a;
  __device__ __forceinline__ double operator()(long long c) const {
    // t[i] = y[i] + h/2.0 * k1[i]  (RCutil.c:469, 486, 503)
    return HAS_K ? y[c] + a * k[c] : y[c];
  }
};

template <int EPI>
__device__ __forceinline__ double epilogue(const Epi &E, const double *__restrict__ y,
                                           double *__restrict__ kout, long long c, double kv) {
  if (EPI == EPI_STORE) {
    kout[c] = kv;
    return 0.0;
  }
  // yout[i] = y[i] + h * (k1[i] + 2*k2[i] + 2*k3[i] + k4[i])/6.0  (RCutil.c:527)
  const double yo = y[c] + E.h * (E.k1[c] + 2 * E.k2[c] + 2 * E.k3[c] + kv) / 6.0;
  E.yout[c] = yo;
  if (EPI == EPI_COMBINE_ERR) return fabs(E.ycmp[c] - yo);   // RCutil.c:592
  return 0.0;
}

template <bool FIELD, bool ADV, bool HAS_K, int EPI>
__global__ void __launch_bounds__(256)
stage_exact(StencilArgs A, const double *__restrict__ y, const double *__restrict__ kin, double a,
            double *__restrict__ kout, const double *__restrict__ p, Epi E) {
  TVal<HAS_K> tv{y, kin, a};
  double err = 0.0;
  if (blockIdx.x < gridDim.x - 1) {
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c < A.ncell) {
      const int n = (int)(c / A.plane);
      const long long rem = c - (long long)n * A.plane;
      const int i = (int)(rem / A.nc), j = (int)(rem - (long long)i * A.nc);
      const double kv = slope_cell_exact<FIELD, ADV>(A, tv, p, n, i, j, c);
      err = epilogue<EPI>(E, y, kout, c, kv);
    }
  } else {
    // package nodes (slope_fn_pack)
    __shared__ double xs[HSB_EXTRA + HSB_EXTRA_SEC], dvs[HSB_EXTRA + HSB_EXTRA_SEC], es[20];
    const int t = threadIdx.x;
    if (t < A.nx) xs[t] = tv(A.ncell + t);
    __syncthreads();
    const int ne = A.secondary ? 20 : 8;
    if (t < ne) {
      int layer, which, node;
      edge_desc(t, E.spidx, E.hsidx, E.subidx, E.solderidx, E.pcbidx, &layer, &which, &node);
      es[t] = edge_sum_exact(A, tv, layer, which, xs[node]);
    }
    __syncthreads();
    if (t == 0) pack_slope_exact(A, xs, es, dvs, E.spidx, E.hsidx, E.subidx, E.solderidx, E.pcbidx);
    __syncthreads();
    if (t < A.nx) err = epilogue<EPI>(E, y, kout, A.ncell + t, dvs[t]);
  }
  if (EPI == EPI_COMBINE_ERR) {
    // block max of |ytemp - t2|, then one atomicMax on the ordered bit pattern
    __shared__ double wmax[8];
    for (int o = 16; o > 0; o >>= 1) err = fmax(err, __shfl_down_sync(0xffffffffu, err, o));
    if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = err;
    __syncthreads();
    if (threadIdx.x == 0) {
      double mx = wmax[0];
      for (int w = 1; w < (int)(blockDim.x >> 5); w++) mx = fmax(mx, wmax[w]);
      atomicMax(E.errbits, (unsigned long long)__double_as_longlong(mx));
    }
  }
}

template <bool FIELD, bool ADV>
static void launch_stage(hsb_dev_model *m, const StencilArgs &A, const double *y, const double *kin,
                         double a, double *kout, const Epi &E, int epi) {
  const int T = 256;
  const unsigned nb = (unsigned)((A.ncell + T - 1) / T) + 1;
  cudaStream_t s = m->stream;
  if (kin) {
    if (epi == EPI_STORE) stage_exact<FIELD, ADV, true, EPI_STORE><<<nb, T, 0, s>>>(A, y, kin, a, kout, m->pgrid, E);
    else if (epi == EPI_COMBINE) stage_exact<FIELD, ADV, true, EPI_COMBINE><<<nb, T, 0, s>>>(A, y, kin, a, kout, m->pgrid, E);
    else stage_exact<FIELD, ADV, true, EPI_COMBINE_ERR><<<nb, T, 0, s>>>(A, y, kin, a, kout, m->pgrid, E);
  } else {
    stage_exact<FIELD, ADV, false, EPI_STORE><<<nb, T, 0, s>>>(A, y, nullptr, 0.0, kout, m->pgrid, E);
  }
}

static void stage(hsb_dev_model *m, const StencilArgs &A, const double *y, const double *kin,
                  double a, double *kout, const Epi &E, int epi) {
  const bool adv = m->uchan_mask != 0;
  if (m->field) {
    if (adv) launch_stage<true, true>(m, A, y, kin, a, kout, E, epi);
    else launch_stage<true, false>(m, A, y, kin, a, kout, E, epi);
  } else {
    if (adv) launch_stage<false, true>(m, A, y, kin, a, kout, E, epi);
    else launch_stage<false, false>(m, A, y, kin, a, kout, E, epi);
  }
}

// rk4_core (RCutil.c:440-531): yout = RK4(y, k1, h)
static void rk4_core(hsb_dev_model *m, const StencilArgs &A, Epi E, const double *y,
                     const double *k1, double h, double *yout, const double *ycmp) {
  E.k1 = k1; E.k2 = m->k2; E.k3 = m->k3; E.h = h; E.yout = yout; E.ycmp = ycmp;
  stage(m, A, y, k1, h / 2.0, m->k2, E, EPI_STORE);
  stage(m, A, y, m->k2, h / 2.0, m->k3, E, EPI_STORE);
  stage(m, A, y, m->k3, h, nullptr, E, ycmp ? EPI_COMBINE_ERR : EPI_COMBINE);
}

#define RK4_SAFETY 0.95
#define RK4_MAXUP 5.0
#define RK4_MAXDOWN 10.0
#define RK4_PRECISION 0.01

// rk4 (RCutil.c:544-640) on the device state m->y; returns the next step
static int rk4_step(hsb_dev_model *m, const StencilArgs &A, double *h, double *next_h,
                    hsb_stats *st) {
  Epi E{};
  E.errbits = m->errbits;
  E.spidx = m->spidx; E.hsidx = m->hsidx;
  E.subidx = m->subidx; E.solderidx = m->solderidx; E.pcbidx = m->pcbidx;
  double max, new_h = *h;
  stage(m, A, m->y, nullptr, 0.0, m->k1, E, EPI_STORE);   // k1 = f(y)
  st->slope_evals += 1;
  st->launches += 1;
  do {
    *h = new_h;
    rk4_core(m, A, E, m->y, m->k1, *h, m->ytemp, nullptr);
    rk4_core(m, A, E, m->y, m->k1, (*h) / 2.0, m->t1, nullptr);
    stage(m, A, m->t1, nullptr, 0.0, m->k1, E, EPI_STORE);      // k1 = f(t1)
    HSB_CUDA(cudaMemsetAsync(m->errbits, 0, sizeof(unsigned long long), m->stream));
    rk4_core(m, A, E, m->t1, m->k1, (*h) / 2.0, m->t2, m->ytemp);
    HSB_CUDA(cudaGetLastError());
    HSB_CUDA(cudaMemcpyAsync(m->h_err, m->errbits, sizeof(double), cudaMemcpyDeviceToHost,
                             m->stream));
    HSB_CUDA(cudaStreamSynchronize(m->stream));
    max = m->h_err[0];
    st->slope_evals += 10;
    st->launches += 10;
    st->rk4_attempts += 1;
    if (max <= RK4_PRECISION) {
      new_h = RK4_SAFETY * (*h) * pow(fabs(RK4_PRECISION / max), 0.2);
      if (new_h > RK4_MAXUP * (*h)) new_h = RK4_MAXUP * (*h);
    } else {
      new_h = RK4_SAFETY * (*h) * pow(fabs(RK4_PRECISION / max), 0.25);
      if (new_h < (*h) / RK4_MAXDOWN) new_h = (*h) / RK4_MAXDOWN;
    }
  } while (new_h < (*h));
  // commit ytemp as the new state (copy_dvector(yout, ytemp) becomes a swap)
  double *tmp = m->y;
  m->y = m->ytemp;
  m->ytemp = tmp;
  st->rk4_steps += 1;
  *next_h = new_h;
  return HSB_OK;
}

#define MIN_STEP 1e-7
#define DELTA 1.0e-6
#define HMIN(x, y) (((x) < (y)) ? (x) : (y))

int rk4_exact_run(hsb_dev_model *m, double time_elapsed, double h0, hsb_stats *st) {
  const StencilArgs A = make_args(m, m->L0, m->nr, m->nc);
  double t, h = 0.0, new_h;
  int rc;
  // temperature_grid.c:3676-3692
  for (t = 0, new_h = h0; t < time_elapsed && new_h >= MIN_STEP * DELTA; t += h) {
    h = new_h;
    if ((rc = rk4_step(m, A, &h, &new_h, st))) return rc;
    new_h = HMIN(new_h, time_elapsed - t - h);
  }
  st->sim_time += t;
  return HSB_OK;
}

int rk4_exact_interval(hsb_dev_model *m, double time_elapsed, hsb_stats *st) {
  return rk4_exact_run(m, time_elapsed, MIN_STEP, st);
}

}  // namespace hsb
