// rk4_batch.cu -- many grid models in ONE persistent launch (the batched
// fast transient form).
//
// A batch is a set of independent models (chips) of uneven size: grid
// sides, layer counts and floorplans differ.  One cooperative launch advances
// every chip by one sampling interval with the Krylov-form fast transient
// (step-doubling RK4 of RCutil.c:440-640 evaluated through Krylov vectors of
// the affine slope operator, FP32 vectors, FP64 state/coefficients/error;
// see rk4_krylov.cu), chip by chip exactly the arithmetic of the single-model
// kernel, so each chip keeps its own adaptive step sequence.
//
// Schedule: the co-resident CTAs are divided among the chips.  A chip large
// enough to deserve several CTAs gets a dedicated group of them that meets
// at a chip-local barrier (a counter and a generation word in global memory,
// bounded spin) after every stencil pass; smaller chips are packed several
// to a CTA and run one after another.  Every CTA belongs to at most one
// multi-CTA group, which it serves first, so groups never wait on each other.
// The schedule (CTAs per SM, how finely chips are split) is chosen by the
// batch autotuner (hsb_batch_autotune).
//
// Per pass a CTA streams its share of the chip's 32x8 column tiles: thread 0
// issues the TMA copy of the NEXT tile's input box (halo included, all
// layers) into the second of two shared-memory buffers before the CTA
// computes the current one, so HBM latency overlaps the stencil arithmetic.
// Vectors the error pass combines are read with coalesced plain loads.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "fast_common.cuh"
#include "krylov_coef.cuh"

namespace hsb {

// one chip as the batch kernel sees it (device array, 128-byte aligned so the
// tensor maps inside are 64-byte aligned)
struct alignas(128) BChip {
  CUtensorMap m_y[2];        // FP64 halo boxes of the two state buffers
  CUtensorMap m_pf;          // FP32 interior boxes of the power
  CUtensorMap m_N;           // FP32 halo boxes of the Krylov vectors (4-D)
  const LayerF *Lf;
  const PackF *pk;
  const double *pgrid;
  float *pf;
  double *y[2];              // the two state buffers
  float *N;
  long long ns, plane, ncell;
  double *part;              // [2][NEDGE][segmax]
  unsigned long long *err;   // [2]
  unsigned *bar;             // [0] arrivals, [1] generation
  double ambient;
  int nl, nr, nc, nx, segmax, spidx, hsidx, ntiles, ntj, pad;
};

// per-chip results (long long words): [0] steps [1] attempts [2] status
// [3] passes [4] time reached (double bits) [5] next step size (double bits)
// [6] state buffer index (in and out)
#define BOUT 8

#define BNB 4
#define BCH 2   // layers per chunk of the error pass's loads

struct BShared {
  double yp[NXMAX];
  double Np[KRY_DMAX + 1][NXMAX];
  double es[NEDGE], wred[FT_WARPS];
  double gmax, pmax;
  float xsf[NXMAX];
  Coef E, D, F1, K, E1, D1, F11;
  double ps[PMAX];
  unsigned long long bar[BNB];
  int lost;
  alignas(16) LayerF L[FT_MAX_LAYERS];
};

// tile-buffer geometry of a launch (sized for the batch's largest layer count)
struct BBufs {
  size_t full, kry;   // bytes of one buffer
  int nfull, nkry;    // full-slope buffers (1 or 2), Krylov-pass ring length
};

struct BCtl {
  int pkind, pm;     // pending package evaluation: kind (-1 none), output index
  double ps;
  int psp, sp, ep;   // edge-partial slots, error slot
  unsigned phase;    // bit b: parity of tile buffer b's next completion
  unsigned gen;      // chip barrier generation
  long long passes;
};

enum { BK_FULL = 0, BK_KRY = 1 };
#define BAR_LIMIT (1 << 25)

// tile buffers: the full-slope pass double-buffers FP64 state boxes (plus the
// power box); the Krylov passes use the same bytes as a deeper ring of the
// smaller FP32 boxes (up to BNB buffers), so more copies are in flight
__host__ __device__ inline size_t bfull_bytes(int nl) { return al128(al128(8 * (size_t)nl * DP) + 4 * (size_t)nl * NI); }
__host__ __device__ inline size_t bkry_bytes(int nl) { return al128(4 * (size_t)nl * KP); }
__host__ __device__ inline int bkry_count(int nl, int nfull) {
  const int k = (int)(nfull * bfull_bytes(nl) / bkry_bytes(nl));
  return k < 2 ? 2 : k > BNB ? BNB : k;
}

// chip-local barrier over `size` CTAs (bounded wait)
__device__ __forceinline__ void bsync(const BChip &C, int size, BCtl &c, BShared &sh) {
  __syncthreads();
  if (size > 1 && threadIdx.x == 0) {
    __threadfence();
    const unsigned g = c.gen;
    if (atomicAdd(&C.bar[0], 1u) == (unsigned)size - 1) {
      atomicExch(&C.bar[0], 0u);
      __threadfence();
      atomicAdd(&C.bar[1], 1u);
    } else {
      int it = 0;
      while (*(volatile unsigned *)&C.bar[1] == g) {
        if (++it >= BAR_LIMIT) {
          sh.lost = 1;
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
  }
  c.gen++;
  __syncthreads();
}

// package nodes of the pending pass (as rk4_krylov.cu's kfinish)
__device__ __forceinline__ void bfinish(const BChip &C, BCtl &c, BShared &sh) {
  if (c.pkind < 0) return;
  const int nx = C.nx, ne = 8;
  const int tid = threadIdx.x, tx = tid & 31, ty = tid >> 5;
  const int ntj = C.ntj, nti = (C.nr + TI - 1) / TI;
  for (int e = ty; e < ne; e += FT_WARPS) {
    const int nseg = (e & 3) < 2 ? ntj : nti;
    const double *pp = C.part + ((long long)c.psp * NEDGE + e) * C.segmax;
    double s = 0.0;
    for (int q = tx; q < nseg; q += 32) s += __ldcg(pp + q);
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (tx == 0) sh.es[e] = s;
  }
  __syncthreads();
  if (ty == 0 && tx < nx) {
    const PackF &P = *C.pk;
    const bool full = c.pkind == BK_FULL;
    const double *x = full ? sh.yp : sh.Np[c.pm - 1];
    const double xq = x[tx];
    double s = full ? P.gamb[tx] * (C.ambient - xq) : -P.gamb[tx] * xq;
    if (P.eidx[tx] >= 0) s += P.ge[tx] * sh.es[P.eidx[tx]];
#pragma unroll
    for (int l = 0; l < PK_LINKS; l++)
      if (P.nb[tx][l] >= 0) s += P.g[tx][l] * (x[P.nb[tx][l]] - xq);
    sh.Np[c.pm][tx] = full ? s * P.invC[tx] : s * P.invC[tx] * c.ps;
  }
  c.pkind = -1;
}

// thread 0: the input box of `tile` into buffer b
template <bool FULL>
__device__ __forceinline__ void bissue(const BChip &C, unsigned char *buf, BShared &sh, int b, int tile, int m,
                                       int cur) {
  const unsigned nl = (unsigned)C.nl;
  const int i0 = (tile / C.ntj) * TI, j0 = (tile % C.ntj) * TJ;
  asm volatile("fence.proxy.async.global;\n" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
  if (FULL) {
    mbar_expect_tx(&sh.bar[b], nl * (DP * 8 + NI * 4));
    tma3(buf, &C.m_y[cur], j0 - 2, i0 - 1, &sh.bar[b]);
    tma3(buf + al128(8 * (size_t)nl * DP), &C.m_pf, j0, i0, &sh.bar[b]);
  } else {
    mbar_expect_tx(&sh.bar[b], nl * KP * 4);
    tma4(buf, &C.m_N, j0 - 4, i0 - 1, m - 1, &sh.bar[b]);
  }
}

// one warp polls the tile copy's mbarrier; the others wait at the CTA
// barrier, issuing nothing (the barrier also makes the copied tile visible
// to them)
__device__ __forceinline__ void bwait(BShared &sh, BCtl &c, int b) {
  if (threadIdx.x < 32) {
    int it = 0;
    while (!mbar_try_wait(&sh.bar[b], (c.phase >> b) & 1u)) {
      if (++it >= WAIT_LIMIT) {
        sh.lost = 1;
        break;
      }
    }
  }
  __syncthreads();
  c.phase ^= 1u << b;
}

// One stencil pass of this CTA's share of the chip: N_m = s L N_{m-1} (KRY)
// or N_0 = f(y) (FULL); ERR also combines the error and the candidate state.
template <bool FULL, bool ERR>
__device__ __forceinline__ void bpass(const BChip &C, int rank, int size, BCtl &c, BShared &sh, unsigned char *dyn,
                                      const BBufs &bb, int m, double s, int cur) {
  const int nl = C.nl, nr = C.nr, nc = C.nc, nx = C.nx;
  const long long plane = C.plane, ns = C.ns;
  const int ne = 8;
  const int tid = threadIdx.x, tx = tid & 31, ty = tid >> 5;
  const double amb = C.ambient;
  const float sf = (float)s;
  const int ntj = C.ntj, ntiles = C.ntiles;
  const float *Nv = C.N;
  float *Nout = C.N + (long long)m * ns;
  const double *yb = C.y[cur];
  double *ynew = C.y[cur ^ 1];
  double *part = C.part;
  const int segmax = C.segmax, spidx = C.spidx, hsidx = C.hsidx;
  double errl = 0.0;
  constexpr int W = FULL ? DW : KW, P = FULL ? DP : KP, X0 = FULL ? 2 : 4;
  const int p_i = (ty + 1) * W + tx + X0;
  const size_t pw_off = al128(8 * (size_t)nl * DP);
  const size_t bsz = FULL ? bb.full : bb.kry;
  const int nbuf = FULL ? bb.nfull : bb.nkry;
  // the vectors the error pass combines (nonzero coefficient), as a bitmask
  unsigned use = 0u;
  if (ERR)
    for (int jj = 0; jj < m && jj < 32; jj++)
      if (sh.E.c[jj] != 0.0 || (jj < sh.D.n && sh.D.c[jj] != 0.0)) use |= 1u << jj;

  // prefetch: tile k of this CTA goes to buffer k % nbuf, nbuf-1 tiles ahead
  if (tid == 0)
    for (int k = 0; k < nbuf - 1 && rank + k * size < ntiles; k++)
      bissue<FULL>(C, dyn + k * bsz, sh, k, rank + k * size, m, cur);
  bfinish(C, c, sh);
  if (tid < nx) sh.xsf[tid] = FULL ? (float)(sh.yp[tid] - amb) : (float)sh.Np[m - 1][tid];
  const double *xin = FULL ? sh.yp : sh.Np[m > 0 ? m - 1 : 0];
  __syncthreads();

  int k = 0;
  for (int tile = rank; tile < ntiles && !sh.lost; tile += size, k++) {
    const int b = k % nbuf;
    const int ti = tile / ntj, tj = tile - ti * ntj;
    const int i0 = ti * TI, j0 = tj * TJ;
    const int i = i0 + ty, j = j0 + tx;
    {
      const int kn = k + nbuf - 1, tn = rank + kn * size;
      if (tid == 0 && tn < ntiles) bissue<FULL>(C, dyn + (kn % nbuf) * bsz, sh, kn % nbuf, tn, m, cur);
    }
    bwait(sh, c, b);
    unsigned char *buf = dyn + b * bsz;
    const double *th = (const double *)buf;
    const float *pw = (const float *)(buf + pw_off);
    const float *vh = (const float *)buf;
    if (i < nr && j < nc) {
      const long long coff = (long long)i * nc + j;
      const bool hN = i > 0, hS = i < nr - 1, hE = j < nc - 1, hW = j > 0;
      // input value at smem index q: FP32 deviation from ambient (FULL) or the vector
      auto val = [&](int q) -> float { return FULL ? (float)(th[q] - amb) : vh[q]; };
      // the column is walked top-down; the vertical neighbours come from registers
      float t_prev = 0.f, t_cur = val(p_i), g_up = 0.f;
      for (int n0 = 0; n0 < nl; n0 += BCH) {
        // error pass: every load of this chunk of layers is issued before the math
        float w[BCH][8];
        double yv[BCH];
        if (ERR) {
#pragma unroll
          for (int u = 0; u < BCH; u++) {
            const long long cc = (long long)(n0 + u) * plane + coff;
            yv[u] = n0 + u < nl ? __ldcg(yb + cc) : 0.0;
#pragma unroll
            for (int jj = 0; jj < 8; jj++)
              w[u][jj] = (n0 + u < nl && ((use >> jj) & 1u)) ? __ldcg(Nv + (long long)jj * ns + cc) : 0.f;
          }
        }
#pragma unroll
        for (int u = 0; u < BCH; u++) {
          const int n = n0 + u;
          if (n >= nl) break;
          const long long cc = (long long)n * plane + coff;
          const int q = n * P + p_i;
          const float4 La = *reinterpret_cast<const float4 *>(&sh.L[n]);   // gNS, gEW, gDown, invC
          const float tc = t_cur;
          const float t_next = n < nl - 1 ? val(q + P) : 0.f;
          float psum = 0.f;
          if (hN) psum += La.x * (val(q - W) - tc);
          if (hS) psum += La.x * (val(q + W) - tc);
          if (hE) psum += La.y * (val(q + 1) - tc);
          if (hW) psum += La.y * (val(q - 1) - tc);
          if (n > 0) psum += g_up * (t_prev - tc);
          if (n < nl - 1) psum += La.z * (t_next - tc);
          const LayerF &L = sh.L[n];
          if (L.kind != LK_PLAIN) {
            int eN, eS, eE, eW;
            if (L.kind == LK_SPREADER) {
              eN = HSB_SP_N; eS = HSB_SP_S; eE = HSB_SP_E; eW = HSB_SP_W;
            } else {
              psum -= L.gAmb * tc;
              eN = HSB_SINK_C_N; eS = HSB_SINK_C_S; eE = HSB_SINK_C_E; eW = HSB_SINK_C_W;
            }
            if (i == 0) psum += L.gEdgeNS * (sh.xsf[eN] - tc);
            if (i == nr - 1) psum += L.gEdgeNS * (sh.xsf[eS] - tc);
            if (j == nc - 1) psum += L.gEdgeEW * (sh.xsf[eE] - tc);
            if (j == 0) psum += L.gEdgeEW * (sh.xsf[eW] - tc);
          }
          t_prev = tc;
          t_cur = t_next;
          g_up = La.z;
          const float kv = FULL ? (pw[n * NI + tid] + psum) * La.w : psum * (La.w * sf);
          Nout[cc] = kv;
          if (ERR) {
            // same order as the single-model kernel: E_m N_m, then j ascending
            const int nD = sh.D.n;
            double e = sh.E.c[m] * (double)kv, dy = 0.0;
#pragma unroll
            for (int jj = 0; jj < 8; jj++) {
              if (jj < m && ((use >> jj) & 1u)) {
                const double wv = (double)w[u][jj];
                e += sh.E.c[jj] * wv;
                if (jj < nD) dy += sh.D.c[jj] * wv;
              }
            }
            for (int jj = 8; jj < m; jj++) {   // after rejections only
              const double ce = sh.E.c[jj], cd = jj < nD ? sh.D.c[jj] : 0.0;
              if (ce != 0.0 || cd != 0.0) {
                const double wv = (double)__ldcg(Nv + (long long)jj * ns + cc);
                e += ce * wv;
                dy += cd * wv;
              }
            }
            errl = fmax(errl, fabs(e));
            ynew[cc] = yv[u] + dy;
          }
        }
      }
    }
    // partial edge sums of (v - x_node) of this pass's input over the tile
    const bool onN = i0 == 0, onS = i0 + TI >= nr, onW = j0 == 0, onE = j0 + TJ >= nc;
    for (int e = ty; e < ne; e += FT_WARPS) {
      const int side = e & 3;
      if (!((side == 0 && onN) || (side == 1 && onS) || (side == 2 && onW) || (side == 3 && onE))) continue;
      int layer, which, node;
      edge_desc(e, spidx, hsidx, -1, -1, -1, &layer, &which, &node);
      int pos = -1;
      if (side < 2) {
        const int r = side == 0 ? 1 : (nr - 1 - i0) + 1;
        if (j0 + tx < nc) pos = r * W + tx + X0;
      } else {
        const int col = side == 2 ? 0 : nc - 1 - j0;
        if (tx < TI && i0 + tx < nr) pos = (tx + 1) * W + col + X0;
      }
      double v = 0.0;
      if (pos >= 0) v = (FULL ? th[layer * DP + pos] : (double)vh[layer * KP + pos]) - xin[node];
      for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
      if (tx == 0) part[((long long)c.sp * NEDGE + e) * segmax + (side < 2 ? tj : ti)] = v;
    }
    __syncthreads();
  }
  if (ERR) {
    for (int o = 16; o > 0; o >>= 1) errl = fmax(errl, __shfl_down_sync(0xffffffffu, errl, o));
    if (tx == 0) sh.wred[ty] = errl;
    __syncthreads();
    if (tid == 0) {
      double mx = sh.wred[0];
      for (int w = 1; w < FT_WARPS; w++) mx = fmax(mx, sh.wred[w]);
      atomicMax(C.err + c.ep, (unsigned long long)__double_as_longlong(mx));
    }
  }
  bsync(C, size, c, sh);
  c.pkind = FULL ? BK_FULL : BK_KRY;
  c.pm = m;
  c.ps = s;
  c.psp = c.sp;
  c.sp ^= 1;
  c.passes++;
}

__device__ __forceinline__ double berr_finish(const BChip &C, int rank, BCtl &c, BShared &sh) {
  const int tid = threadIdx.x, tx = tid & 31, ty = tid >> 5;
  bfinish(C, c, sh);
  if (tid == FT_THREADS - 1) sh.gmax = __longlong_as_double((long long)(*(volatile unsigned long long *)(C.err + c.ep)));
  if (ty == 0) {
    double perr = 0.0;
    if (tx < C.nx) {
      double e = 0.0;
      for (int jj = 0; jj < sh.E.n; jj++) e += sh.E.c[jj] * sh.Np[jj][tx];
      perr = fabs(e);
    }
    for (int o = 16; o > 0; o >>= 1) perr = fmax(perr, __shfl_down_sync(0xffffffffu, perr, o));
    if (tx == 0) sh.pmax = perr;
  }
  __syncthreads();
  const double mx = fmax(sh.gmax, sh.pmax);
  if (rank == 0 && tid == 0) C.err[c.ep ^ 1] = 0ull;
  c.ep ^= 1;
  __syncthreads();
  return mx;
}

// one sampling interval of one chip by a group of `size` CTAs (this is `rank`)
__device__ void bchip(const BChip &C, int rank, int size, long long *out, BShared &sh, unsigned char *dyn,
                      const BBufs &bsz, unsigned &phase, double T) {
  const int tid = threadIdx.x;
  const int nx = C.nx, nl = C.nl;
  if (tid < nl) sh.L[tid] = C.Lf[tid];
  int cur = (int)out[6];
  for (long long q = (long long)rank * blockDim.x + tid; q < C.ncell; q += (long long)size * blockDim.x)
    C.pf[q] = (float)C.pgrid[q];
  if (tid < nx) sh.yp[tid] = __ldcg(C.y[cur] + C.ncell + tid);
  if (rank == 0 && tid == 0) {
    C.err[0] = 0ull;
    C.err[1] = 0ull;
  }
  BCtl c;
  c.pkind = -1;
  c.sp = 0;
  c.ep = 0;
  c.phase = phase;
  c.gen = 0;
  c.passes = 0;
  bsync(C, size, c, sh);
  long long steps = 0, attempts = 0;
  int status = 0;
  double t = 0.0, h = 0.0, new_h = 1e-7;
  while (t < T && new_h >= 1e-7 * 1.0e-6 && !sh.lost) {
    h = new_h;
    bpass<true, false>(C, rank, size, c, sh, dyn, bsz, 0, 1.0, cur);   // N_0 = f(y)
    int dcomp = 0;
    if (tid == 0) c_one(sh.K);
    double mx = 0.0;
    bool first = true;
    for (;;) {
      h = new_h;
      if (first) {
        if (tid < PMAX) {
          const int q = tid;
          sh.ps[q] = h;
          if (q < sh.E1.n) sh.E.c[q] = h * sh.E1.c[q];
          if (q < sh.D1.n) sh.D.c[q] = h * sh.D1.c[q];
          if (q < sh.F11.n) sh.F1.c[q] = sh.F11.c[q];
          if (q == 0) {
            sh.E.n = sh.E1.n;
            sh.D.n = sh.D1.n;
            sh.F1.n = sh.F11.n;
          }
        }
        first = false;
      } else if (tid == 0) {
        kry_plan(sh.E, sh.D, sh.F1, sh.K, sh.ps, h, dcomp);
      }
      __syncthreads();
      const int dE = sh.E.n - 1;
      if (dE > KRY_DMAX || dE <= dcomp) {
        status = 3;
        break;
      }
      for (int q = dcomp + 1; q < dE && !sh.lost; q++)
        bpass<false, false>(C, rank, size, c, sh, dyn, bsz, q, sh.ps[q], cur);
      bpass<false, true>(C, rank, size, c, sh, dyn, bsz, dE, sh.ps[dE], cur);
      if (sh.lost) break;
      dcomp = dE;
      mx = berr_finish(C, rank, c, sh);
      attempts++;
      if (mx <= 0.01) {
        new_h = 0.95 * h * pow(fabs(0.01 / mx), 0.2);
        if (new_h > 5.0 * h) new_h = 5.0 * h;
      } else {
        new_h = 0.95 * h * pow(fabs(0.01 / mx), 0.25);
        if (new_h < h / 10.0) new_h = h / 10.0;
      }
      if (new_h >= h) break;
      if (tid == 0) c_copy(sh.K, sh.F1);
      __syncthreads();
    }
    if (status || sh.lost) break;
    if (tid < nx) {
      double dy = 0.0;
      for (int q = 0; q < sh.D.n; q++) dy += sh.D.c[q] * sh.Np[q][tid];
      sh.yp[tid] += dy;
    }
    cur ^= 1;
    steps++;
    new_h = new_h < T - t - h ? new_h : T - t - h;
    t += h;
  }
  __syncthreads();
  phase = c.phase;
  if (rank == 0) {
    if (tid < nx) C.y[cur][C.ncell + tid] = sh.yp[tid];
    if (tid == 0) {
      out[0] = steps;
      out[1] = attempts;
      out[2] = sh.lost ? 2 : status;
      out[3] = c.passes;
      double tt[2] = {t, new_h};
      memcpy(&out[4], tt, sizeof(tt));
      out[6] = cur;
    }
  }
}

__global__ void __launch_bounds__(FT_THREADS, 2)
    rk4_batch_kernel(const BChip *__restrict__ chips, const int4 *__restrict__ work, const int *__restrict__ wptr,
                     long long *__restrict__ out, BBufs bsz, double T) {
  extern __shared__ __align__(128) unsigned char bdyn_raw[];
  __shared__ BShared sh;
  unsigned char *dyn = bdyn_raw + ((128u - (smem_u32(bdyn_raw) & 127u)) & 127u);
  if (threadIdx.x == 0) {
    sh.lost = 0;
    for (int b = 0; b < BNB; b++) mbar_init(&sh.bar[b], 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    // first-attempt coefficients for h = 1 (they scale with h; chip-independent)
    for (int q = 0; q < PMAX; q++) sh.ps[q] = 1.0;
    c_one(sh.K);
    kry_plan(sh.E, sh.D, sh.F1, sh.K, sh.ps, 1.0, 0);
    c_copy(sh.E1, sh.E);
    c_copy(sh.D1, sh.D);
    c_copy(sh.F11, sh.F1);
  }
  __syncthreads();
  unsigned phase = 0;
  for (int w = wptr[blockIdx.x]; w < wptr[blockIdx.x + 1]; w++) {
    const int4 a = work[w];
    bchip(chips[a.x], a.y, a.z, out + (long long)a.x * BOUT, sh, dyn, bsz, phase, T);
    if (sh.lost) break;
  }
  if (sh.lost && threadIdx.x == 0) {
    // let a tile copy still in flight land before the CTA exits
    for (int b = 0; b < BNB; b++)
      for (int it = 0; it < WAIT_LIMIT && !mbar_try_wait(&sh.bar[b], (phase >> b) & 1u); it++) {
      }
  }
}

// batched block -> grid power: one CTA range per chip
__global__ void batch_b2g(const int *__restrict__ cta_off, int nchips, const int *const *__restrict__ ptr,
                          const int *const *__restrict__ blk, const double *const *__restrict__ occ,
                          const double *const *__restrict__ area, const double *__restrict__ bpow,
                          const long long *__restrict__ boff, double *const *__restrict__ grid,
                          const long long *__restrict__ ncell, const int *__restrict__ nblk,
                          const double *__restrict__ cell_area, int nx) {
  int lo = 0, hi = nchips - 1;
  while (lo < hi) {   // chip of this CTA: last chip whose first CTA <= blockIdx.x
    const int mid = (lo + hi + 1) / 2;
    if (cta_off[mid] <= (int)blockIdx.x) lo = mid;
    else hi = mid - 1;
  }
  const int ch = lo;
  const long long c = (long long)(blockIdx.x - cta_off[ch]) * blockDim.x + threadIdx.x;
  const long long N = ncell[ch];
  const double *b = bpow + boff[ch];
  double *g = grid[ch];
  if (c < N) {
    double val = 0.0;
    const int e0 = ptr[ch][c], e1 = ptr[ch][c + 1];
    for (int e = e0; e < e1; e++) val += occ[ch][e] * b[blk[ch][e]] / area[ch][e];   // blist_avg :331
    g[c] = val * cell_area[ch];
  } else if (c < N + nx) {
    g[c] = b[nblk[ch] + (c - N)];
  }
}

}  // namespace hsb

// ---------------------------------------------------------------------------
// host side: the batch object and its C-ABI
// ---------------------------------------------------------------------------
using namespace hsb;

struct hsb_batch {
  int n, device, nlmax;
  std::vector<hsb_dev_model *> models;
  std::vector<BChip> h_chips;
  BChip *d_chips = nullptr;
  int4 *d_work = nullptr;
  int *d_wptr = nullptr;
  long long *d_out = nullptr, *h_out = nullptr;
  unsigned *d_bar = nullptr;
  int grid = 0;
  BBufs bsz{};
  size_t smem = 0;
  cudaStream_t stream = nullptr;
  // schedule
  int ctas_per_sm = 2;
  double split = 1.0;        // a chip gets about split * (its share of the work) CTAs
  int ring = 0;              // Krylov-pass ring length (0: as many as fit)
  // online autotuning: candidate k runs on call k; the fastest per cell-step wins
  struct Cand { int cps; double split; int ring; double ms_per_gcs; };
  std::vector<Cand> cands;
  int tune_next = -1;        // index of the candidate of the next call, -1: not tuning
  unsigned long long signature = 0;
  // batched b2g tables
  int *d_cta_off = nullptr;
  int b2g_ctas = 0;
  const int **d_ptr = nullptr, **d_blk = nullptr;
  const double **d_occ = nullptr, **d_area = nullptr;
  double **d_grid = nullptr;
  long long *d_boff = nullptr, *d_ncell = nullptr;
  int *d_nblk = nullptr;
  double *d_cell_area = nullptr;
  double *d_bpow = nullptr;
  std::vector<long long> boff;   // offsets of the chips' block vectors
  long long nbtotal = 0;
  double *h_bpow = nullptr;      // pinned staging of the block powers
  bool started = false;
};

static void batch_free(hsb_batch *b) {
  if (!b) return;
  void *d[] = {b->d_chips, b->d_work, b->d_wptr, b->d_out, b->d_bar, b->d_cta_off, b->d_ptr, b->d_blk,
               b->d_occ, b->d_area, b->d_grid, b->d_boff, b->d_ncell, b->d_nblk, b->d_cell_area, b->d_bpow};
  for (void *p : d)
    if (p) cudaFree(p);
  if (b->h_out) cudaFreeHost(b->h_out);
  if (b->h_bpow) cudaFreeHost(b->h_bpow);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
}

// CTA work lists for the current schedule; returns the grid size
static int batch_schedule(hsb_batch *b) {
  int nsm = 0;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, b->device);
  // three or more CTAs per SM: one FP64 box buffer (no prefetch in the
  // full-slope pass) so that the shared memory of three CTAs fits an SM
  b->bsz.nfull = b->ctas_per_sm >= 3 ? 1 : 2;
  b->bsz.full = bfull_bytes(b->nlmax);
  b->bsz.kry = bkry_bytes(b->nlmax);
  b->bsz.nkry = bkry_count(b->nlmax, b->bsz.nfull);
  if (b->ring > 0 && b->ring < b->bsz.nkry) b->bsz.nkry = b->ring;
  size_t ring = b->bsz.kry * b->bsz.nkry;
  size_t dyn = b->bsz.nfull * b->bsz.full;
  b->smem = (ring > dyn ? ring : dyn) + 128;
  {
    const int rc0 = raise_smem_limit((const void *)rk4_batch_kernel, b->smem);
    if (rc0) return rc0;
  }
  int per_sm = 0;
  HSB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void *)rk4_batch_kernel, FT_THREADS,
                                                         b->smem));
  if (per_sm < 1) return set_error(HSB_E_ARG, "batch kernel does not fit an SM");
  if (b->ctas_per_sm < per_sm) per_sm = b->ctas_per_sm;
  const int G = per_sm * nsm;
  // work of a chip ~ its tiles x layers.  A chip worth `split` x (or more)
  // two CTAs' fair share gets a group of CTAs; the rest are packed onto
  // single CTAs (longest first onto the least loaded), and the packed part
  // always keeps the CTAs its work needs at the fair share.
  std::vector<double> wk(b->n);
  double W = 0;
  for (int c = 0; c < b->n; c++) {
    wk[c] = (double)b->h_chips[c].ntiles * b->h_chips[c].nl;
    W += wk[c];
  }
  std::vector<int> order(b->n);
  for (int c = 0; c < b->n; c++) order[c] = c;
  std::sort(order.begin(), order.end(), [&](int a, int c) { return wk[a] > wk[c]; });
  const double share = W / G;
  std::vector<int> g(b->n, 1);
  double w_small = 0.0, sum_g = 0.0;
  for (int c = 0; c < b->n; c++) {
    // a chip worth more than one fair share gets enough CTAs that none of
    // them carries more than a share (rounded up, not down)
    const double ratio = wk[c] / share * b->split;
    int q = ratio > 1.0 ? (int)ceil(ratio) : 1;
    if (q > b->h_chips[c].ntiles) q = b->h_chips[c].ntiles;
    if (q >= 2) {
      g[c] = q;
      sum_g += q;
    } else {
      g[c] = 1;
      w_small += wk[c];
    }
  }
  int g_small = (int)ceil(w_small / share);
  if (w_small > 0 && g_small < 1) g_small = 1;
  if (g_small > G - 1) g_small = G - 1;
  const double avail = G - g_small;
  if (sum_g > avail) {   // scale the groups down to the CTAs left
    const double f = avail / sum_g;
    for (int c = 0; c < b->n; c++)
      if (g[c] >= 2) {
        int q = (int)(g[c] * f);
        if (q < 2) {
          q = 1;
          w_small += wk[c];
        }
        g[c] = q;
      }
  }
  std::vector<std::vector<int4>> lists;
  std::vector<double> load;
  for (int c : order)
    if (g[c] >= 2)
      for (int r = 0; r < g[c]; r++) {
        lists.push_back({make_int4(c, r, g[c], 0)});
        load.push_back(wk[c] / g[c]);
      }
  const int base = (int)lists.size();
  const int remaining = G - base > 0 ? G - base : 1;
  for (int k = 0; k < remaining; k++) {
    lists.push_back({});
    load.push_back(0.0);
  }
  for (int c : order) {
    if (g[c] >= 2) continue;
    int best = base;
    for (int k = base; k < (int)lists.size(); k++)
      if (load[k] < load[best]) best = k;
    lists[best].push_back(make_int4(c, 0, 1, 0));
    load[best] += wk[c];
  }
  // drop CTAs left without work
  {
    std::vector<std::vector<int4>> keep;
    for (auto &l : lists)
      if (!l.empty()) keep.push_back(l);
    lists.swap(keep);
  }
  std::vector<int> wptr(lists.size() + 1, 0);
  std::vector<int4> work;
  for (size_t k = 0; k < lists.size(); k++) {
    for (auto &a : lists[k]) work.push_back(a);
    wptr[k + 1] = (int)work.size();
  }
  if (b->d_work) cudaFree(b->d_work);
  if (b->d_wptr) cudaFree(b->d_wptr);
  b->d_work = nullptr;
  b->d_wptr = nullptr;
  HSB_CUDA(cudaMalloc(&b->d_work, sizeof(int4) * (work.size() + 1)));
  HSB_CUDA(cudaMalloc(&b->d_wptr, sizeof(int) * wptr.size()));
  HSB_CUDA(cudaMemcpy(b->d_work, work.data(), sizeof(int4) * work.size(), cudaMemcpyHostToDevice));
  HSB_CUDA(cudaMemcpy(b->d_wptr, wptr.data(), sizeof(int) * wptr.size(), cudaMemcpyHostToDevice));
  b->grid = (int)lists.size();
  return HSB_OK;
}

extern "C" {

int hsb_batch_create(hsb_batch **out, hsb_dev_model *const *models, int n) {
  if (!out || !models || n < 1) return set_error(HSB_E_ARG, "null argument");
  hsb_batch *b = new hsb_batch();
  b->n = n;
  b->models.assign(models, models + n);
  b->device = models[0]->device;
  b->nlmax = 0;
  int rc;
  auto fail = [&](int code) {
    batch_free(b);
    return code;
  };
  if (cudaSetDevice(b->device) != cudaSuccess) return fail(set_error(HSB_E_CUDA, "cudaSetDevice"));
  if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess)
    return fail(set_error(HSB_E_CUDA, "batch stream"));
  if (cudaMalloc(&b->d_bar, sizeof(unsigned) * 2 * n) != cudaSuccess ||
      cudaMalloc(&b->d_out, sizeof(long long) * BOUT * n) != cudaSuccess ||
      cudaMallocHost(&b->h_out, sizeof(long long) * BOUT * n) != cudaSuccess)
    return fail(set_error(HSB_E_NOMEM, "batch control arrays"));
  b->h_chips.resize(n);
  b->boff.resize(n + 1, 0);
  for (int c = 0; c < n; c++) {
    hsb_dev_model *m = models[c];
    if (!m) return fail(set_error(HSB_E_ARG, "null model in batch"));
    if (m->device != b->device) return fail(set_error(HSB_E_ARG, "batch models must share one device"));
    if (m->field || m->uchan_mask || m->nx != HSB_EXTRA)
      return fail(set_error(HSB_E_ARG, "batched transient takes per-layer-conductance models of the primary heat path"));
    if (!m->b2g_ptr) return fail(set_error(HSB_E_ARG, "batch model without block-grid maps"));
    FastWork *w;
    if ((rc = fast_prepare(m, &w))) return fail(rc);
    if ((rc = kry_prepare(m, w))) return fail(rc);
    BChip &C = b->h_chips[c];
    memset(&C, 0, sizeof(C));
    if ((rc = make_map(&C.m_y[0], m->y, true, m, DW, HR))) return fail(rc);
    if ((rc = make_map(&C.m_y[1], w->ytemp, true, m, DW, HR))) return fail(rc);
    C.m_pf = w->kmap_pf;
    C.m_N = w->kmap_N;
    C.Lf = w->Lf;
    C.pk = w->pk;
    C.pgrid = m->pgrid;
    C.pf = w->pf;
    C.y[0] = m->y;
    C.y[1] = w->ytemp;
    C.N = w->N;
    C.ns = w->nstride;
    C.plane = m->plane;
    C.ncell = m->ncell;
    C.part = w->part;
    C.err = w->err;
    C.bar = b->d_bar + 2 * c;
    C.ambient = m->ambient;
    C.nl = m->nl;
    C.nr = m->nr;
    C.nc = m->nc;
    C.nx = m->nx;
    C.segmax = w->segmax;
    C.spidx = m->spidx;
    C.hsidx = m->hsidx;
    C.ntj = (m->nc + TJ - 1) / TJ;
    C.ntiles = C.ntj * ((m->nr + TI - 1) / TI);
    if (m->nl > b->nlmax) b->nlmax = m->nl;
    b->boff[c + 1] = b->boff[c] + m->total_n_blocks + m->nx;
  }
  b->nbtotal = b->boff[n];
  if (cudaMalloc(&b->d_chips, sizeof(BChip) * n) != cudaSuccess) return fail(set_error(HSB_E_NOMEM, "batch chips"));
  if (cudaMemcpy(b->d_chips, b->h_chips.data(), sizeof(BChip) * n, cudaMemcpyHostToDevice) != cudaSuccess)
    return fail(set_error(HSB_E_CUDA, "batch chips upload"));
  std::vector<long long> init(BOUT * (size_t)n, 0);
  if (cudaMemcpy(b->d_out, init.data(), sizeof(long long) * BOUT * n, cudaMemcpyHostToDevice) != cudaSuccess)
    return fail(set_error(HSB_E_CUDA, "batch outputs"));
  if ((rc = batch_schedule(b))) return fail(rc);
  // batched b2g tables
  {
    std::vector<int> cta_off(n);
    std::vector<const int *> ptr(n), blk(n);
    std::vector<const double *> occ(n), area(n);
    std::vector<double *> grid(n);
    std::vector<long long> ncell(n);
    std::vector<int> nblk(n);
    std::vector<double> carea(n);
    int ctas = 0;
    for (int c = 0; c < n; c++) {
      hsb_dev_model *m = models[c];
      cta_off[c] = ctas;
      ctas += (int)((m->vlen + 255) / 256);
      ptr[c] = m->b2g_ptr;
      blk[c] = m->b2g_blk;
      occ[c] = m->b2g_occ;
      area[c] = m->b2g_area;
      grid[c] = m->pgrid;
      ncell[c] = m->ncell;
      nblk[c] = m->total_n_blocks;
      carea[c] = m->cell_area;
    }
    b->b2g_ctas = ctas;
    bool ok = cudaMalloc(&b->d_cta_off, sizeof(int) * n) == cudaSuccess &&
              cudaMalloc(&b->d_ptr, sizeof(void *) * n) == cudaSuccess &&
              cudaMalloc(&b->d_blk, sizeof(void *) * n) == cudaSuccess &&
              cudaMalloc(&b->d_occ, sizeof(void *) * n) == cudaSuccess &&
              cudaMalloc(&b->d_area, sizeof(void *) * n) == cudaSuccess &&
              cudaMalloc(&b->d_grid, sizeof(void *) * n) == cudaSuccess &&
              cudaMalloc(&b->d_boff, sizeof(long long) * (n + 1)) == cudaSuccess &&
              cudaMalloc(&b->d_ncell, sizeof(long long) * n) == cudaSuccess &&
              cudaMalloc(&b->d_nblk, sizeof(int) * n) == cudaSuccess &&
              cudaMalloc(&b->d_cell_area, sizeof(double) * n) == cudaSuccess &&
              cudaMalloc(&b->d_bpow, sizeof(double) * (b->nbtotal + 1)) == cudaSuccess &&
              cudaMallocHost(&b->h_bpow, sizeof(double) * (b->nbtotal + 1)) == cudaSuccess;
    if (!ok) return fail(set_error(HSB_E_NOMEM, "batch b2g tables"));
    cudaMemcpy(b->d_cta_off, cta_off.data(), sizeof(int) * n, cudaMemcpyHostToDevice);
    cudaMemcpy(b->d_ptr, ptr.data(), sizeof(void *) * n, cudaMemcpyHostToDevice);
    cudaMemcpy(b->d_blk, blk.data(), sizeof(void *) * n, cudaMemcpyHostToDevice);
    cudaMemcpy(b->d_occ, occ.data(), sizeof(void *) * n, cudaMemcpyHostToDevice);
    cudaMemcpy(b->d_area, area.data(), sizeof(void *) * n, cudaMemcpyHostToDevice);
    cudaMemcpy(b->d_grid, grid.data(), sizeof(void *) * n, cudaMemcpyHostToDevice);
    cudaMemcpy(b->d_boff, b->boff.data(), sizeof(long long) * (n + 1), cudaMemcpyHostToDevice);
    cudaMemcpy(b->d_ncell, ncell.data(), sizeof(long long) * n, cudaMemcpyHostToDevice);
    cudaMemcpy(b->d_nblk, nblk.data(), sizeof(int) * n, cudaMemcpyHostToDevice);
    if (cudaMemcpy(b->d_cell_area, carea.data(), sizeof(double) * n, cudaMemcpyHostToDevice) != cudaSuccess)
      return fail(set_error(HSB_E_CUDA, "batch b2g tables upload"));
  }
  *out = b;
  return HSB_OK;
}

void hsb_batch_destroy(hsb_batch *b) { batch_free(b); }

int hsb_batch_set_schedule(hsb_batch *b, int ctas_per_sm, double split) {
  if (!b || ctas_per_sm < 1 || !(split > 0)) return set_error(HSB_E_ARG, "bad batch schedule");
  b->ctas_per_sm = ctas_per_sm;
  b->split = split;
  return batch_schedule(b);
}

// schedules chosen by the autotuner, by batch shape (process-wide)
static std::mutex g_tune_mu;
static std::vector<std::pair<unsigned long long, hsb_batch::Cand>> g_tuned;

static unsigned long long batch_signature(const hsb_batch *b) {
  std::vector<unsigned long long> keys;
  for (auto &C : b->h_chips) keys.push_back(((unsigned long long)C.nl << 40) | ((unsigned long long)C.nr << 20) | C.nc);
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
        b->ctas_per_sm = e.second.cps;
        b->split = e.second.split;
        b->ring = e.second.ring;
        b->tune_next = -1;
        return batch_schedule(b);
      }
  }
  b->cands.clear();
  const int cps[2] = {2, 1};
  const double split[3] = {1.0, 1.5, 2.0};
  const int ring[2] = {0, 2};
  for (int a : cps)
    for (double sp : split)
      for (int r : ring) b->cands.push_back({a, sp, r, 0.0});
  b->tune_next = 0;
  return HSB_OK;
}

int hsb_batch_info(hsb_batch *b, int *grid, long long *cells, int *ctas_per_sm, double *split) {
  if (!b) return set_error(HSB_E_ARG, "null batch");
  long long n = 0;
  for (auto *m : b->models) n += m->ncell;
  if (grid) *grid = b->grid;
  if (cells) *cells = n;
  if (ctas_per_sm) *ctas_per_sm = b->ctas_per_sm;
  if (split) *split = b->split;
  return HSB_OK;
}

int hsb_batch_transient(hsb_batch *b, const double *block_power, double time_elapsed, hsb_stats *st) {
  if (!b) return set_error(HSB_E_ARG, "null batch");
  hsb_stats local;
  if (!st) st = &local;
  cudaSetDevice(b->device);
  const int tuning = b->tune_next;
  if (tuning >= 0) {
    const hsb_batch::Cand &c = b->cands[tuning];
    b->ctas_per_sm = c.cps;
    b->split = c.split;
    b->ring = c.ring;
    int rc0;
    if ((rc0 = batch_schedule(b))) return rc0;
  }
  const long long steps0 = st->rk4_steps;
  const double kms0 = st->kernel_ms;
  cudaEvent_t e0, e1, k0, k1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventCreate(&k0);
  cudaEventCreate(&k1);
  cudaEventRecord(e0, b->stream);
  if (block_power) {
    memcpy(b->h_bpow, block_power, sizeof(double) * b->nbtotal);
    HSB_CUDA(cudaMemcpyAsync(b->d_bpow, b->h_bpow, sizeof(double) * b->nbtotal, cudaMemcpyHostToDevice, b->stream));
    batch_b2g<<<b->b2g_ctas, 256, 0, b->stream>>>(b->d_cta_off, b->n, b->d_ptr, b->d_blk, b->d_occ, b->d_area,
                                                  b->d_bpow, b->d_boff, b->d_grid, b->d_ncell, b->d_nblk,
                                                  b->d_cell_area, HSB_EXTRA);
    HSB_CUDA(cudaGetLastError());
    st->launches += 1;
  }
  // which buffer holds each model's state (single-model calls may have swapped them)
  {
    bool changed = false;
    for (int c = 0; c < b->n; c++) {
      const long long cur = b->models[c]->y == b->h_chips[c].y[0] ? 0 : 1;
      if (b->models[c]->y != b->h_chips[c].y[cur])
        return set_error(HSB_E_ARG, "a batch model's state buffers were reallocated");
      if (b->h_out[(size_t)c * BOUT + 6] != cur) changed = true;
      b->h_out[(size_t)c * BOUT + 6] = cur;
    }
    if (changed || !b->started)
      HSB_CUDA(cudaMemcpyAsync(b->d_out, b->h_out, sizeof(long long) * BOUT * b->n, cudaMemcpyHostToDevice, b->stream));
    b->started = true;
  }
  HSB_CUDA(cudaMemsetAsync(b->d_bar, 0, sizeof(unsigned) * 2 * b->n, b->stream));
  cudaEventRecord(k0, b->stream);
  void *args[] = {&b->d_chips, &b->d_work, &b->d_wptr, &b->d_out, &b->bsz, &time_elapsed};
  HSB_CUDA(cudaLaunchCooperativeKernel((const void *)rk4_batch_kernel, dim3(b->grid), dim3(FT_THREADS), args,
                                       b->smem, b->stream));
  cudaEventRecord(k1, b->stream);
  HSB_CUDA(cudaMemcpyAsync(b->h_out, b->d_out, sizeof(long long) * BOUT * b->n, cudaMemcpyDeviceToHost, b->stream));
  HSB_CUDA(cudaStreamSynchronize(b->stream));
  float ms = 0.f, kms = 0.f;
  cudaEventElapsedTime(&kms, k0, k1);
  st->launches += 1;
  int rc = HSB_OK;
  // per chip: results, the model's view of its state buffer, fallbacks
  for (int c = 0; c < b->n && !rc; c++) {
    hsb_dev_model *m = b->models[c];
    FastWork *w = (FastWork *)m->fast;
    const long long *o = b->h_out + (size_t)c * BOUT;
    st->rk4_steps += o[0];
    st->rk4_attempts += o[1];
    st->slope_evals += o[3];
    const int cur = (int)o[6];
    m->y = b->h_chips[c].y[cur];
    w->ytemp = b->h_chips[c].y[cur ^ 1];
    if (o[2] == 2) rc = set_error(HSB_E_CUDA, "batched transient: a tile copy or chip barrier did not complete in time");
    else if (o[2] == 3) {
      // rejection budget exhausted: the stage form finishes this chip's interval
      double tt[2];
      memcpy(tt, &o[4], sizeof(tt));
      st->fallbacks += 1;
      rc = rk4_stage_run(m, w, time_elapsed - tt[0], tt[1], st);
      // the stage form may have swapped the model's buffers
      const int now = m->y == b->h_chips[c].y[0] ? 0 : 1;
      if (now != cur) {
        long long v = now;
        if (cudaMemcpy(b->d_out + (size_t)c * BOUT + 6, &v, sizeof(v), cudaMemcpyHostToDevice) != cudaSuccess)
          rc = set_error(HSB_E_CUDA, "batch state index");
      }
    }
  }
  cudaEventRecord(e1, b->stream);
  cudaEventSynchronize(e1);
  cudaEventElapsedTime(&ms, e0, e1);
  st->device_ms += ms;
  st->kernel_ms += kms;
  st->sim_time += time_elapsed;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaEventDestroy(k0);
  cudaEventDestroy(k1);
  if (tuning >= 0 && rc == HSB_OK) {
    // kernel time per 10^9 cell-steps of this call
    double cs = 0.0;
    for (int c = 0; c < b->n; c++) cs += (double)b->h_out[(size_t)c * BOUT] * b->models[c]->ncell;
    (void)steps0;
    b->cands[tuning].ms_per_gcs = cs > 0 ? (st->kernel_ms - kms0) / (cs / 1e9) : 1e300;
    b->tune_next = tuning + 1;
    if (b->tune_next >= (int)b->cands.size()) {
      int best = 0;
      for (int k = 1; k < (int)b->cands.size(); k++)
        if (b->cands[k].ms_per_gcs < b->cands[best].ms_per_gcs) best = k;
      const hsb_batch::Cand c = b->cands[best];
      b->ctas_per_sm = c.cps;
      b->split = c.split;
      b->ring = c.ring;
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

// the autotuner's measurements: up to n candidates as (ctas_per_sm, split,
// ring, ms per 10^9 cell-steps); returns how many were measured
int hsb_batch_tuning(hsb_batch *b, double *out, int n) {
  if (!b) return set_error(HSB_E_ARG, "null batch");
  int k = 0;
  for (; k < (int)b->cands.size() && k < n; k++) {
    out[4 * k] = b->cands[k].cps;
    out[4 * k + 1] = b->cands[k].split;
    out[4 * k + 2] = b->cands[k].ring;
    out[4 * k + 3] = b->cands[k].ms_per_gcs;
  }
  return k;
}

// per-chip accepted steps of the last call (n entries)
int hsb_batch_chip_steps(hsb_batch *b, long long *steps) {
  if (!b || !steps) return set_error(HSB_E_ARG, "null argument");
  for (int c = 0; c < b->n; c++) steps[c] = b->h_out[(size_t)c * BOUT];
  return HSB_OK;
}

}  // extern "C"
