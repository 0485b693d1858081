// rk4_fast.cu -- the fast transient form (HSB_FORM_FAST).
//
// The same adaptive step-doubling RK4 as the reference (RCutil.c:544-640,
// including the reuse of k1 = f(t1) on a retry) and the same interval loop
// (temperature_grid.c:3676-3692), run as ONE cooperative persistent kernel
// per sampling interval, one grid barrier per RK4 stage:
//   * a stage works on 32x8 (j x i) tiles through all layers: one thread of
//     the CTA issues TMA tensor copies (cp.async.bulk.tensor, completion on
//     an mbarrier) of the tile with its one-cell halo and of every per-cell
//     operand of the stage, all layers at once, into shared memory; each
//     thread then evaluates its (i, j) column from shared memory (vertical
//     neighbours included), so a stage waits on one round trip to L2/HBM;
//   * stencil arithmetic in FP32: the stage input t = y + a*k is formed in
//     FP64 (y is FP64) once per cell and kept as the FP32 deviation t - T_amb,
//     slopes k are FP32;
//   * state y, the combination y + h(k1+2k2+2k3+k4)/6 and the error norm
//     |ytemp - t2| stay in FP64;
//   * the package nodes' edge sums come from per-tile partials reduced in a
//     fixed order (deterministic); every CTA evaluates the package nodes from
//     a precomputed sparse FP64 conductance table, one lane per node, at the
//     start of the next stage while that stage's tile copies are in flight;
//   * step-size control runs on the device: every CTA reads the global
//     max-norm after the barrier and takes the identical decision.
#include "fast_common.cuh"
#include "rk4_tb.cuh"

namespace cg = cooperative_groups;

namespace hsb {

struct FastArgs {
  Maps M;
  const double *bufP, *bufQ;
  StencilArgs S;
  int spidx, hsidx, subidx, solderidx, pcbidx;
  int segmax;
  const LayerF *Lf;
  const PackF *pk;
  const float *gN, *gS, *gW, *gE, *gA, *gB, *invC;
  const float *aN, *aS, *aW, *aE, *aO;
  const double *qin;
  const double *pgrid;
  float *pf;
  double *y, *ytemp, *t1, *t2;
  float *k1, *k2, *k3;
  double *part;
  unsigned long long *err;
  long long *cnt;
  double T, h0;
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
  const double *k1p, *k2p;  // combine
  double h;
  double *yout, *youtp;
  const double *ycmpp;
  const CUtensorMap *m_yb, *m_kin, *m_k1, *m_k2, *m_yc;
};

// Running control state, identical in every thread: the package-node part
// of a stage is evaluated at the start of the NEXT stage, while that stage's
// tile copies are in flight, and `mode` .. `ycmpp` record what is pending.
struct Ctl {
  int mode;             // -1: nothing pending
  int psp;              // edge-partial slot of the pending stage
  double h;
  double *koutp, *youtp;
  const double *ypb, *k1p, *k2p, *kinp, *ycmpp;
  int ep;               // error-accumulator slot
  int sp;               // edge-partial slot of the next stage
  unsigned phase;       // completed tile-copy phases
};

// per-CTA shared state of the kernel (static part)
struct Shared {
  double yp[NXMAX], kp1[NXMAX], kp2[NXMAX], kp3[NXMAX], ytp[NXMAX], t1p[NXMAX], t2p[NXMAX];
  double xs[2][NXMAX];  // package-node stage inputs, by partial slot
  double es[NEDGE], wred[FT_WARPS];
  double gmax, pmax;
  float xsf[NXMAX];     // xs - T_amb in FP32, for the cells' edge terms
  unsigned long long bar;
  int lost;
  LayerF L[FT_MAX_LAYERS];
};

// dynamic shared memory, per layer: FP64 halo box of the base state (turned
// into the stage input t in place), FP32 halo box of k, the interior cells'
// power and, for the combination stages, k1, k2, comparison state and base
// state; FP32 deviations t - T_amb; then the package table
struct DynSmem {
  double *th;           // [nl][HR][DW]
  float *kh;            // [nl][HR][KW]
  float *pw, *k1, *k2;  // [nl][NI]
  double *yc, *yb;      // [nl][NI]
  float *d;             // [nl][HR][DW]
  PackF *pk;
};


// byte offsets of the DynSmem arrays; returns the bytes to request (with
// slack for aligning the base to 128 bytes, as TMA destinations need)
__host__ __device__ inline size_t dyn_layout(int nl, size_t off[9]) {
  size_t o = 0;
  off[0] = o; o = al128(o + 8 * (size_t)nl * DP);
  off[1] = o; o = al128(o + 4 * (size_t)nl * KP);
  off[2] = o; o = al128(o + 4 * (size_t)nl * NI);
  off[3] = o; o = al128(o + 4 * (size_t)nl * NI);
  off[4] = o; o = al128(o + 4 * (size_t)nl * NI);
  off[5] = o; o = al128(o + 8 * (size_t)nl * NI);
  off[6] = o; o = al128(o + 8 * (size_t)nl * NI);
  off[7] = o; o = al128(o + 4 * (size_t)nl * DP);
  off[8] = o; o = al128(o + sizeof(PackF));
  return o + 128;
}


// wait for the current tile-copy phase, bounded; a lost copy is recorded
// and the kernel runs on to its end (the host reports the error)
__device__ __forceinline__ void tile_wait(Shared &sh, Ctl &c) {
  int it = 0;
  while (!mbar_try_wait(&sh.bar, c.phase & 1u)) {
    if (++it >= WAIT_LIMIT) {
      sh.lost = 1;
      break;
    }
  }
  c.phase++;
}

__device__ __forceinline__ const CUtensorMap *halo_map(const FastArgs &A, const double *p) {
  return p == A.bufP ? &A.M.yP_h : p == A.bufQ ? &A.M.yQ_h : &A.M.t1_h;
}
__device__ __forceinline__ const CUtensorMap *int_map(const FastArgs &A, const double *p) {
  return p == A.bufP ? &A.M.yP_i : &A.M.yQ_i;
}

template <int MODE>
__device__ __forceinline__ void issue_tile(const FastArgs &A, const StageIO &io, const DynSmem &ds,
                                           Shared &sh, int i0, int j0) {
  if (threadIdx.x != 0) return;
  const unsigned nl = (unsigned)A.S.nl;
  unsigned bytes = nl * (DP * 8 + NI * 4);
  if (io.kin) bytes += nl * KP * 4;
  if (MODE != M_K) bytes += nl * NI * 8;
  if (MODE == M_COMBINE_ERR) bytes += nl * NI * 8;
  // order the generic-proxy writes seen through the grid barrier (global)
  // and the reads of the previous tile (shared) before the async copies
  asm volatile("fence.proxy.async.global;\n" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
  mbar_expect_tx(&sh.bar, bytes);
  tma3(ds.th, io.m_yb, j0 - 2, i0 - 1, &sh.bar);
  if (io.kin) tma3(ds.kh, io.m_kin, j0 - 4, i0 - 1, &sh.bar);
  tma3(ds.pw, &A.M.pf_i, j0, i0, &sh.bar);
  if (MODE != M_K) {
    tma3(ds.k1, io.m_k1, j0, i0, &sh.bar);
    tma3(ds.k2, io.m_k2, j0, i0, &sh.bar);
  }
  if (MODE == M_COMBINE_ERR) tma3(ds.yc, io.m_yc, j0, i0, &sh.bar);
}

// Package nodes of the pending stage: edge partial sums reduced in a fixed
// order, then one lane of warp 0 per node.  Each package vector entry is
// read and written by the same lane throughout the kernel, so no barrier is
// needed after it.  Returns the package part of the error norm folded with
// the cells' part (combination-with-error stages), else 0.
__device__ __forceinline__ double finish_pending(const FastArgs &A, Ctl &c, Shared &sh, const DynSmem &ds) {
  if (c.mode < 0) return 0.0;
  const StencilArgs &S = A.S;
  const int nx = S.nx, ne = S.secondary ? NEDGE : 8;
  const int tid = threadIdx.x, tx = tid & 31, ty = tid >> 5;
  const int ntj = (S.nc + TJ - 1) / TJ, nti = (S.nr + TI - 1) / TI;
  if (c.mode == M_COMBINE_ERR && tid == FT_THREADS - 1)
    sh.gmax = __longlong_as_double((long long)(*(volatile unsigned long long *)(A.err + c.ep)));
  for (int e = ty; e < ne; e += FT_WARPS) {
    const int nseg = (e & 3) < 2 ? ntj : nti;
    const double *pp = A.part + ((long long)c.psp * NEDGE + e) * A.segmax;
    double s = 0.0;
    for (int q = tx; q < nseg; q += 32) s += pp[q];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (tx == 0) sh.es[e] = s;
  }
  __syncthreads();
  if (ty == 0) {
    double perr = 0.0;
    if (tx < nx) {
      const double *xs = sh.xs[c.psp];
      const PackF &P = *ds.pk;
      const double xq = xs[tx];
      double s = P.gamb[tx] * (S.ambient - xq);
      if (P.eidx[tx] >= 0) s += P.ge[tx] * sh.es[P.eidx[tx]];
#pragma unroll
      for (int l = 0; l < PK_LINKS; l++)
        if (P.nb[tx][l] >= 0) s += P.g[tx][l] * (xs[P.nb[tx][l]] - xq);
      const double d = s * P.invC[tx];
      if (c.mode == M_K) {
        c.koutp[tx] = d;
      } else {
        const double yo = c.ypb[tx] + c.h * (c.k1p[tx] + 2.0 * c.k2p[tx] + 2.0 * c.kinp[tx] + d) / 6.0;
        c.youtp[tx] = yo;
        if (c.mode == M_COMBINE_ERR) perr = fabs(c.ycmpp[tx] - yo);
      }
    }
    if (c.mode == M_COMBINE_ERR) {
      for (int o = 16; o > 0; o >>= 1) perr = fmax(perr, __shfl_down_sync(0xffffffffu, perr, o));
      if (tx == 0) sh.pmax = perr;
    }
  }
  if (c.mode == M_COMBINE_ERR) {
    __syncthreads();
    const double mx = fmax(sh.gmax, sh.pmax);
    if (blockIdx.x == 0 && tid == 0) A.err[c.ep ^ 1] = 0ull;
    c.ep ^= 1;
    __syncthreads();
    return mx;
  }
  return 0.0;
}

template <bool FIELD, bool ADV, int MODE>
__device__ __forceinline__ void stage(const FastArgs &A, cg::grid_group &grid, const StageIO &io, Ctl &c,
                                      Shared &sh, const DynSmem &ds) {
  constexpr int CH = Chunk<FIELD, ADV>::n;
  const StencilArgs &S = A.S;
  const int nl = S.nl, nr = S.nr, nc = S.nc, nx = S.nx;
  const long long plane = S.plane;
  const bool hasK = io.kin != nullptr;
  const int ne = S.secondary ? NEDGE : 8;
  const int tid = threadIdx.x, tx = tid & 31, ty = tid >> 5;
  const double a = io.a, amb = S.ambient;
  const int ntj = (nc + TJ - 1) / TJ, nti = (nr + TI - 1) / TI, ntiles = ntj * nti;
  double errl = 0.0;

  // positions of this thread's interior cell and halo cell (84 of the
  // threads own one of the halo ring's cells) in the FP64 / FP32 boxes
  const int pd_i = (ty + 1) * DW + tx + 2, pk_i = (ty + 1) * KW + tx + 4;
  int hr = -1, hc = 0;
  if (tid < TJ + 2) { hr = 0; hc = tid; }
  else if (tid < 2 * (TJ + 2)) { hr = HR - 1; hc = tid - (TJ + 2); }
  else if (tid < 2 * (TJ + 2) + TI) { hr = tid - 2 * (TJ + 2) + 1; hc = 0; }
  else if (tid < 2 * (TJ + 2) + 2 * TI) { hr = tid - 2 * (TJ + 2) - TI + 1; hc = TJ + 1; }
  const int pd_h = hr * DW + hc + 1, pk_h = hr * KW + hc + 3;

  // first tile's copies go out before the pending package work
  if ((int)blockIdx.x < ntiles)
    issue_tile<MODE>(A, io, ds, sh, (blockIdx.x / ntj) * TI, (blockIdx.x % ntj) * TJ);
  finish_pending(A, c, sh, ds);
  // package-node temperatures of this stage's input (each lane uses the
  // package slopes it wrote itself; published by the barrier below)
  if (tid < nx) {
    const double x = hasK ? io.ypb[tid] + a * io.kinp[tid] : io.ypb[tid];
    sh.xs[c.sp][tid] = x;
    sh.xsf[tid] = (float)(x - amb);
  }
  const double *xs = sh.xs[c.sp];

  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int ti = tile / ntj, tj = tile - ti * ntj;
    const int i0 = ti * TI, j0 = tj * TJ;
    const int i = i0 + ty, j = j0 + tx;
    if (tile != (int)blockIdx.x) issue_tile<MODE>(A, io, ds, sh, i0, j0);
    tile_wait(sh, c);
    // stage input t = y + a*k (FP64, in place) and t - T_amb (FP32); each
    // thread its own positions
    for (int n = 0; n < nl; n++) {
      double *th = ds.th + n * DP;
      float *dn = ds.d + n * DP;
      const float *kh = ds.kh + n * KP;
      double v = th[pd_i];
      if (MODE != M_K) ds.yb[n * NI + tid] = v;
      if (hasK) {
        v = v + a * (double)kh[pk_i];
        th[pd_i] = v;
      }
      dn[pd_i] = (float)(v - amb);
      if (hr >= 0) {
        double w = th[pd_h];
        if (hasK) {
          w = w + a * (double)kh[pk_h];
          th[pd_h] = w;
        }
        dn[pd_h] = (float)(w - amb);
      }
    }
    __syncthreads();
    if (i < nr && j < nc) {
      const long long coff = (long long)i * nc + j;
      for (int n0 = 0; n0 < nl; n0 += CH) {
        float gN[CH], gS[CH], gE[CH], gW[CH], gA[CH], gB[CH], iC[CH];
        float aN[CH], aS[CH], aW[CH], aE[CH], aO[CH];
        double qn[CH];
        if (FIELD || ADV) {
#pragma unroll
          for (int u = 0; u < CH; u++) {
            const long long cc = (long long)(n0 + u) * plane + coff;
            if (n0 + u < nl) {
              if (FIELD) {
                gN[u] = A.gN[cc]; gS[u] = A.gS[cc]; gE[u] = A.gE[cc]; gW[u] = A.gW[cc];
                gA[u] = A.gA[cc]; gB[u] = A.gB[cc]; iC[u] = A.invC[cc];
              }
              if (ADV && ((S.uchan_mask >> (n0 + u)) & 1ull)) {
                aN[u] = A.aN[cc]; aS[u] = A.aS[cc]; aW[u] = A.aW[cc]; aE[u] = A.aE[cc]; aO[u] = A.aO[cc];
                qn[u] = A.qin[cc];
              }
            }
          }
        }
#pragma unroll
        for (int u = 0; u < CH; u++) {
          const int n = n0 + u;
          if (n >= nl) break;
          const long long cc = (long long)n * plane + coff;
          const float *dn = ds.d + n * DP;
          const float tc = dn[pd_i];
          const LayerF &L = sh.L[n];
          float psum = 0.f;
          if (i > 0) psum += (FIELD ? gN[u] : L.gNS) * (dn[pd_i - DW] - tc);
          if (i < nr - 1) psum += (FIELD ? gS[u] : L.gNS) * (dn[pd_i + DW] - tc);
          if (j < nc - 1) psum += (FIELD ? gE[u] : L.gEW) * (dn[pd_i + 1] - tc);
          if (j > 0) psum += (FIELD ? gW[u] : L.gEW) * (dn[pd_i - 1] - tc);
          if (n > 0) psum += (FIELD ? gA[u] : sh.L[n - 1].gDown) * (dn[pd_i - DP] - tc);
          if (n < nl - 1) psum += (FIELD ? gB[u] : L.gDown) * (dn[pd_i + DP] - tc);
          if (L.kind != LK_PLAIN) {
            int eN, eS, eE, eW;
            switch (L.kind) {
              case LK_SPREADER: eN = HSB_SP_N; eS = HSB_SP_S; eE = HSB_SP_E; eW = HSB_SP_W; break;
              case LK_SINK:
                psum -= L.gAmb * tc;
                eN = HSB_SINK_C_N; eS = HSB_SINK_C_S; eE = HSB_SINK_C_E; eW = HSB_SINK_C_W; break;
              case LK_PCB:
                psum -= L.gAmb * tc;
                eN = HSB_PCB_C_N; eS = HSB_PCB_C_S; eE = HSB_PCB_C_E; eW = HSB_PCB_C_W; break;
              case LK_SUB: eN = HSB_SUB_N; eS = HSB_SUB_S; eE = HSB_SUB_E; eW = HSB_SUB_W; break;
              default: eN = HSB_SOLDER_N; eS = HSB_SOLDER_S; eE = HSB_SOLDER_E; eW = HSB_SOLDER_W; break;
            }
            if (i == 0) psum += L.gEdgeNS * (sh.xsf[eN] - tc);
            if (i == nr - 1) psum += L.gEdgeNS * (sh.xsf[eS] - tc);
            if (j == nc - 1) psum += L.gEdgeEW * (sh.xsf[eE] - tc);
            if (j == 0) psum += L.gEdgeEW * (sh.xsf[eW] - tc);
          }
          if (ADV && ((S.uchan_mask >> n) & 1ull)) {
            // advection carries absolute temperatures: FP64
            const double *th = ds.th + n * DP;
            const double T = th[pd_i];
            double adv = qn[u] + (double)aO[u] * T;
            if (i > 0) adv += (double)aN[u] * ((th[pd_i - DW] + T) / 2.0);
            if (i < nr - 1) adv += (double)aS[u] * ((th[pd_i + DW] + T) / 2.0);
            if (j > 0) adv += (double)aW[u] * ((th[pd_i - 1] + T) / 2.0);
            if (j < nc - 1) adv += (double)aE[u] * ((th[pd_i + 1] + T) / 2.0);
            psum += (float)adv;
          }
          const int q = n * NI + tid;
          const float k = (ds.pw[q] + psum) * (FIELD ? iC[u] : L.invC);
          if (MODE == M_K) {
            io.kout[cc] = k;
          } else {
            const double yo = ds.yb[q] + io.h * ((double)ds.k1[q] + 2.0 * (double)ds.k2[q] +
                                                 2.0 * (double)ds.kh[n * KP + pk_i] + (double)k) / 6.0;
            io.yout[cc] = yo;
            if (MODE == M_COMBINE_ERR) errl = fmax(errl, fabs(ds.yc[q] - yo));
          }
        }
      }
    }
    // partial edge sums of (t - x_node) over this tile's share of each edge
    const bool onN = i0 == 0, onS = i0 + TI >= nr, onW = j0 == 0, onE = j0 + TJ >= nc;
    for (int e = ty; e < ne; e += FT_WARPS) {
      const int side = e & 3;
      if (!((side == 0 && onN) || (side == 1 && onS) || (side == 2 && onW) || (side == 3 && onE))) continue;
      int layer, which, node;
      edge_desc(e, A.spidx, A.hsidx, A.subidx, A.solderidx, A.pcbidx, &layer, &which, &node);
      const double *th = ds.th + layer * DP;
      double v = 0.0;
      if (side < 2) {
        const int r = side == 0 ? 1 : (nr - 1 - i0) + 1;
        if (j0 + tx < nc) v = th[r * DW + tx + 2] - xs[node];
      } else {
        const int col = side == 2 ? 0 : nc - 1 - j0;
        if (tx < TI && i0 + tx < nr) v = th[(tx + 1) * DW + col + 2] - xs[node];
      }
      for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
      if (tx == 0) A.part[((long long)c.sp * NEDGE + e) * A.segmax + (side < 2 ? tj : ti)] = v;
    }
    __syncthreads();
  }
  if (MODE == M_COMBINE_ERR) {
    for (int o = 16; o > 0; o >>= 1) errl = fmax(errl, __shfl_down_sync(0xffffffffu, errl, o));
    if (tx == 0) sh.wred[ty] = errl;
    __syncthreads();
    if (tid == 0) {
      double mx = sh.wred[0];
      for (int w = 1; w < FT_WARPS; w++) mx = fmax(mx, sh.wred[w]);
      atomicMax(A.err + c.ep, (unsigned long long)__double_as_longlong(mx));
    }
  }
  grid.sync();
  c.mode = MODE;
  c.psp = c.sp;
  c.h = io.h;
  c.koutp = io.koutp;
  c.youtp = io.youtp;
  c.ypb = io.ypb;
  c.k1p = io.k1p;
  c.k2p = io.k2p;
  c.kinp = io.kinp;
  c.ycmpp = io.ycmpp;
  c.sp ^= 1;
}

// one RK4 step of size h from (yb, ypb) with k1 given (RCutil.c:544-574)
template <bool FIELD, bool ADV>
__device__ __forceinline__ void core(const FastArgs &A, cg::grid_group &grid, const double *yb,
                                     const double *ypb, const double *k1p, double h, double *yout,
                                     double *youtp, const double *ycmp, const double *ycmpp, Ctl &c,
                                     Shared &sh, const DynSmem &ds) {
  StageIO io{};
  io.yb = yb; io.ypb = ypb; io.m_yb = halo_map(A, yb);
  io.kin = A.k1; io.kinp = k1p; io.m_kin = &A.M.k1_h; io.a = h / 2.0;
  io.kout = A.k2; io.koutp = sh.kp2;
  stage<FIELD, ADV, M_K>(A, grid, io, c, sh, ds);
  io.kin = A.k2; io.kinp = sh.kp2; io.m_kin = &A.M.k2_h; io.a = h / 2.0;
  io.kout = A.k3; io.koutp = sh.kp3;
  stage<FIELD, ADV, M_K>(A, grid, io, c, sh, ds);
  io.kin = A.k3; io.kinp = sh.kp3; io.m_kin = &A.M.k3_h; io.a = h;
  io.k1p = k1p; io.k2p = sh.kp2; io.h = h;
  io.m_k1 = &A.M.k1_i; io.m_k2 = &A.M.k2_i;
  io.yout = yout; io.youtp = youtp; io.ycmpp = ycmpp;
  if (ycmp) {
    io.m_yc = int_map(A, ycmp);
    stage<FIELD, ADV, M_COMBINE_ERR>(A, grid, io, c, sh, ds);
  } else {
    stage<FIELD, ADV, M_COMBINE>(A, grid, io, c, sh, ds);
  }
}

template <bool FIELD, bool ADV>
__global__ void __launch_bounds__(FT_THREADS, 2) rk4_fast_kernel(const __grid_constant__ FastArgs A) {
  cg::grid_group grid = cg::this_grid();
  extern __shared__ __align__(128) unsigned char dyn_raw[];
  __shared__ Shared sh;
  const StencilArgs &S = A.S;
  const int nx = S.nx, nl = S.nl;
  DynSmem ds;
  {
    size_t off[9];
    dyn_layout(nl, off);
    unsigned char *base = dyn_raw + ((128u - (smem_u32(dyn_raw) & 127u)) & 127u);
    ds.th = (double *)(base + off[0]);
    ds.kh = (float *)(base + off[1]);
    ds.pw = (float *)(base + off[2]);
    ds.k1 = (float *)(base + off[3]);
    ds.k2 = (float *)(base + off[4]);
    ds.yc = (double *)(base + off[5]);
    ds.yb = (double *)(base + off[6]);
    ds.d = (float *)(base + off[7]);
    ds.pk = (PackF *)(base + off[8]);
  }
  {
    const double *src = (const double *)A.pk;
    double *dst = (double *)ds.pk;
    for (int q = threadIdx.x; q < (int)(sizeof(PackF) / 8); q += blockDim.x) dst[q] = src[q];
    if (threadIdx.x < nl) sh.L[threadIdx.x] = A.Lf[threadIdx.x];
    if (threadIdx.x == 0) {
      sh.lost = 0;
      mbar_init(&sh.bar, 1);
      asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
  }
  // FP32 power for this interval
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < S.ncell;
       c += (long long)gridDim.x * blockDim.x)
    A.pf[c] = (float)A.pgrid[c];
  if (threadIdx.x < nx) sh.yp[threadIdx.x] = A.y[S.ncell + threadIdx.x];
  if (blockIdx.x == 0 && threadIdx.x == 0) { A.err[0] = 0ull; A.err[1] = 0ull; }
  grid.sync();
  double *y = A.y, *ytemp = A.ytemp;
  Ctl c;
  c.mode = -1;
  c.ep = 0;
  c.sp = 0;
  c.phase = 0;
  long long steps = 0, attempts = 0;
  double t, h = 0.0, new_h, mx = 0.0;
  StageIO io{};
  for (t = 0, new_h = A.h0; t < A.T && new_h >= 1e-7 * 1.0e-6; t += h) {
    h = new_h;
    io.yb = y; io.ypb = sh.yp; io.m_yb = halo_map(A, y);
    io.kin = nullptr; io.kinp = nullptr; io.a = 0.0;
    io.kout = A.k1; io.koutp = sh.kp1;
    stage<FIELD, ADV, M_K>(A, grid, io, c, sh, ds);     // k1 = f(y)
    do {
      h = new_h;
      core<FIELD, ADV>(A, grid, y, sh.yp, sh.kp1, h, ytemp, sh.ytp, nullptr, nullptr, c, sh, ds);
      core<FIELD, ADV>(A, grid, y, sh.yp, sh.kp1, h / 2.0, A.t1, sh.t1p, nullptr, nullptr, c, sh, ds);
      io.yb = A.t1; io.ypb = sh.t1p; io.m_yb = &A.M.t1_h;
      io.kin = nullptr; io.kinp = nullptr; io.a = 0.0;
      io.kout = A.k1; io.koutp = sh.kp1;
      stage<FIELD, ADV, M_K>(A, grid, io, c, sh, ds);   // k1 = f(t1)
      core<FIELD, ADV>(A, grid, A.t1, sh.t1p, sh.kp1, h / 2.0, A.t2, sh.t2p, ytemp, sh.ytp, c, sh, ds);
      mx = finish_pending(A, c, sh, ds);
      c.mode = -1;
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
    if (threadIdx.x < nx) sh.yp[threadIdx.x] = sh.ytp[threadIdx.x];
    steps++;
    new_h = new_h < A.T - t - h ? new_h : A.T - t - h;
  }
  __syncthreads();
  if (sh.lost && threadIdx.x == 0) {
    // let any copy still in flight land before the CTA exits (bounded)
    for (int it = 0; it < WAIT_LIMIT && !mbar_try_wait(&sh.bar, c.phase & 1u); it++) {
    }
    A.cnt[3] = 2;
  }
  if (blockIdx.x == 0) {
    if (threadIdx.x < nx) y[S.ncell + threadIdx.x] = sh.yp[threadIdx.x];
    if (threadIdx.x == 0) {
      A.cnt[0] = steps;
      A.cnt[1] = attempts;
      A.cnt[2] = (y == A.y) ? 0 : 1;
      if (attempts >= A.max_attempts) A.cnt[3] = 1;
    }
  }
}

static const void *kernel_for(bool field, bool adv) {
  return field ? (adv ? (const void *)rk4_fast_kernel<true, true> : (const void *)rk4_fast_kernel<true, false>)
               : (adv ? (const void *)rk4_fast_kernel<false, true> : (const void *)rk4_fast_kernel<false, false>);
}

static size_t tile_smem(int nl) {
  size_t off[9];
  return dyn_layout(nl, off);
}

static int fast_grid(hsb_dev_model *m, const void *fn, int *grid) {
  return coop_grid(m, fn, tile_smem(m->nl), grid);
}


static int build_maps(Maps *M, const hsb_dev_model *m, const double *P, const double *Q, const double *t1,
                      const float *k1, const float *k2, const float *k3, const float *pf) {
  int rc;
  if ((rc = make_map(&M->yP_h, P, true, m, DW, HR))) return rc;
  if ((rc = make_map(&M->yP_i, P, true, m, TJ, TI))) return rc;
  if ((rc = make_map(&M->yQ_h, Q, true, m, DW, HR))) return rc;
  if ((rc = make_map(&M->yQ_i, Q, true, m, TJ, TI))) return rc;
  if ((rc = make_map(&M->t1_h, t1, true, m, DW, HR))) return rc;
  if ((rc = make_map(&M->k1_h, k1, false, m, KW, HR))) return rc;
  if ((rc = make_map(&M->k1_i, k1, false, m, TJ, TI))) return rc;
  if ((rc = make_map(&M->k2_h, k2, false, m, KW, HR))) return rc;
  if ((rc = make_map(&M->k2_i, k2, false, m, TJ, TI))) return rc;
  if ((rc = make_map(&M->k3_h, k3, false, m, KW, HR))) return rc;
  if ((rc = make_map(&M->pf_i, pf, false, m, TJ, TI))) return rc;
  return HSB_OK;
}



static void free_fast(void *p) {
  FastWork *w = (FastWork *)p;
  if (!w) return;
  void *bufs[] = {w->k1, w->k2, w->k3, w->pf, w->ytemp, w->t1, w->t2, w->gN, w->gS, w->gW, w->gE,
                  w->gA, w->gB, w->invC, w->aN, w->aS, w->aW, w->aE, w->aO, w->Lf, w->pk, w->part,
                  w->err, w->cnt, w->N};
  for (void *b : bufs)
    if (b) cudaFree(b);
  if (w->h_cnt) cudaFreeHost(w->h_cnt);
  if (w->kev[0]) cudaEventDestroy(w->kev[0]);
  if (w->kev[1]) cudaEventDestroy(w->kev[1]);
  tb_res_free((TbRes *)w->tb);
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
int fast_prepare(hsb_dev_model *m, FastWork **out) {
  FastWork *w = (FastWork *)m->fast;
  const long long n = m->ncell;
  int rc;
  if ((rc = check_shape(m))) return rc;
  if (!w) {
    w = new FastWork();
    memset(w, 0, sizeof(*w));
    w->ncell = n;
    w->coef_version = -1;
    m->fast = w;
    m->fast_free = free_fast;
    w->segmax = segmax_of(m);
    HSB_CUDA(cudaMalloc(&w->k1, sizeof(float) * n));
    HSB_CUDA(cudaMalloc(&w->k2, sizeof(float) * n));
    HSB_CUDA(cudaMalloc(&w->k3, sizeof(float) * n));
    HSB_CUDA(cudaMalloc(&w->pf, sizeof(float) * n));
    HSB_CUDA(cudaMalloc(&w->ytemp, sizeof(double) * m->vlen));
    HSB_CUDA(cudaMalloc(&w->t1, sizeof(double) * m->vlen));
    HSB_CUDA(cudaMalloc(&w->t2, sizeof(double) * m->vlen));
    HSB_CUDA(cudaMalloc(&w->Lf, sizeof(LayerF) * HSB_MAX_LAYERS));
    HSB_CUDA(cudaMalloc(&w->pk, sizeof(PackF)));
    HSB_CUDA(cudaMalloc(&w->part, sizeof(double) * 2 * NEDGE * w->segmax));
    HSB_CUDA(cudaMalloc(&w->err, sizeof(unsigned long long) * 2));
    HSB_CUDA(cudaMalloc(&w->cnt, sizeof(long long) * 8));
    HSB_CUDA(cudaMallocHost(&w->h_cnt, sizeof(long long) * 8));
  }
  // the maps describe the two state buffers whichever role each has now
  const bool same = (w->mapP == m->y && w->mapQ == w->ytemp) || (w->mapP == w->ytemp && w->mapQ == m->y);
  if (!same) {
    if ((rc = build_maps(&w->maps, m, m->y, w->ytemp, w->t1, w->k1, w->k2, w->k3, w->pf))) return rc;
    w->mapP = m->y;
    w->mapQ = w->ytemp;
  }
  if (w->coef_version == m->coef_version) {
    *out = w;
    return HSB_OK;
  }
  w->coef_version = m->coef_version;
  LayerF Lf[HSB_MAX_LAYERS];
  PackF P;
  host_tables(m, Lf, &P);
  HSB_CUDA(cudaMemcpyAsync(w->Lf, Lf, sizeof(LayerF) * m->nl, cudaMemcpyHostToDevice, m->stream));
  HSB_CUDA(cudaMemcpyAsync(w->pk, &P, sizeof(PackF), cudaMemcpyHostToDevice, m->stream));
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
  // a re-uploaded model may have switched between per-layer and per-cell values
  if ((rc = fast_grid(m, kernel_for(m->field, m->uchan_mask != 0), &w->grid))) return rc;
  *out = w;
  return HSB_OK;
}

static void fill_common(FastArgs &A, const hsb_dev_model *m) {
  A.S = make_args(m, m->L0, m->nr, m->nc);
  A.spidx = m->spidx; A.hsidx = m->hsidx;
  A.subidx = m->subidx; A.solderidx = m->solderidx; A.pcbidx = m->pcbidx;
  A.segmax = segmax_of(m);
  A.max_attempts = 10000000;
  A.h0 = 1e-7;
}

static int status_error(long long status) {
  if (status == 1) return set_error(HSB_E_NOCONV, "fast transient: RK4 attempt cap reached");
  if (status == 2) return set_error(HSB_E_CUDA, "fast transient: a tile copy did not complete in time");
  return HSB_OK;
}

int rk4_stage_run(hsb_dev_model *m, FastWork *w, double T, double h0, hsb_stats *st) {
  FastArgs A;
  memset(&A, 0, sizeof(A));
  fill_common(A, m);
  A.M = w->maps;
  A.bufP = w->mapP;
  A.bufQ = w->mapQ;
  A.Lf = w->Lf;
  A.pk = w->pk;
  A.gN = w->gN; A.gS = w->gS; A.gW = w->gW; A.gE = w->gE; A.gA = w->gA; A.gB = w->gB;
  A.invC = w->invC;
  A.aN = w->aN; A.aS = w->aS; A.aW = w->aW; A.aE = w->aE; A.aO = w->aO; A.qin = m->qin;
  A.pgrid = m->pgrid; A.pf = w->pf;
  A.y = m->y; A.ytemp = w->ytemp; A.t1 = w->t1; A.t2 = w->t2;
  A.k1 = w->k1; A.k2 = w->k2; A.k3 = w->k3;
  A.part = w->part; A.err = w->err; A.cnt = w->cnt;
  A.T = T;
  A.h0 = h0;
  HSB_CUDA(cudaMemsetAsync(w->cnt, 0, sizeof(long long) * 4, m->stream));
  void *args[] = {&A};
  const void *fn = kernel_for(m->field, m->uchan_mask != 0);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, m->stream);
  HSB_CUDA(cudaLaunchCooperativeKernel(fn, dim3(w->grid), dim3(FT_THREADS), args, tile_smem(m->nl), m->stream));
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
  return status_error(w->h_cnt[3]);
}

int rk4_fast_stages_interval(hsb_dev_model *m, double time_elapsed, hsb_stats *st) {
  FastWork *w;
  int rc;
  if ((rc = fast_prepare(m, &w))) return rc;
  rc = rk4_stage_run(m, w, time_elapsed, 1e-7, st);
  st->sim_time += time_elapsed;
  return rc;
}

// one interval in two halves, so the caller can queue work that reads the
// result (g2b with the state buffer chosen on the device) before waiting;
// bpow_dev: the block powers, mapped to the grid in the kernel (null: the
// grid power is in pgrid already)
int rk4_fast_interval_begin(hsb_dev_model *m, double time_elapsed, hsb_stats *st, void **work,
                            const double *bpow_dev) {
  FastWork *w;
  int rc;
  if ((rc = fast_prepare(m, &w))) return rc;
  *work = w;
  return rk4_krylov_enqueue(m, w, time_elapsed, st, bpow_dev, bpow_dev ? 1 : 0);
}

int rk4_fast_interval_end(hsb_dev_model *m, void *work, double time_elapsed, hsb_stats *st, int *fell_back) {
  FastWork *w = (FastWork *)work;
  int rc, done = 0;
  double t_done = time_elapsed, h_next = 0.0;
  *fell_back = 0;
  if ((rc = rk4_krylov_complete(m, w, time_elapsed, st, &t_done, &h_next, &done))) return rc;
  if (t_done < time_elapsed) {   // the rest of the interval: the stage form (all-FP64 variant: the replay)
    st->fallbacks += 1;
    *fell_back = 1;
    rc = m->fast_passes == 2 ? rk4_exact_run(m, time_elapsed - t_done, h_next, st)
                             : rk4_stage_run(m, w, time_elapsed - t_done, h_next, st);
    if (rc) return rc;
  }
  st->sim_time += time_elapsed;
  return HSB_OK;
}

// the host-side preparation of the Krylov form (workspace, tensor maps,
// co-resident grid) without launching anything
int rk4_fast_ready(hsb_dev_model *m, void **work, const void **kernel) {
  FastWork *w;
  int rc;
  if ((rc = fast_prepare(m, &w))) return rc;
  if ((rc = kry_prepare(m, w))) return rc;
  *work = w;
  *kernel = w->kfn;
  return HSB_OK;
}

// the second state buffer of the fast forms and the device word saying
// which of the two buffers holds the state after the last launch
void fast_state_buffers(hsb_dev_model *m, void *work, double **second, const long long **which) {
  (void)m;
  FastWork *w = (FastWork *)work;
  *second = w->ytemp;
  *which = w->cnt + 6;
}

// K intervals in as few launches as possible: one Krylov-form launch runs
// them back to back; an interval whose rejection budget runs out is finished
// by the stage form (from its own grid power) and the launches resume after it
int rk4_fast_trace(hsb_dev_model *m, const double *bpow_dev, int K, double time_elapsed, hsb_stats *st) {
  FastWork *w;
  int rc;
  if ((rc = fast_prepare(m, &w))) return rc;
  const long long nb = (long long)m->total_n_blocks + m->nx;
  int i0 = 0;
  while (i0 < K) {
    int done = 0;
    double t_done = time_elapsed, h_next = 0.0;
    if ((rc = rk4_krylov_trace(m, w, bpow_dev + i0 * nb, K - i0, time_elapsed, st, &done, &t_done, &h_next)))
      return rc;
    if (done >= K - i0) break;
    const int k = i0 + done;
    if ((rc = b2g(m, bpow_dev + (long long)k * nb, m->pgrid, HSB_V_POWER))) return rc;
    st->launches += 1;
    st->fallbacks += 1;
    rc = m->fast_passes == 2 ? rk4_exact_run(m, time_elapsed - t_done, h_next, st)
                             : rk4_stage_run(m, w, time_elapsed - t_done, h_next, st);
    if (rc) return rc;
    i0 = k + 1;
  }
  // the last interval's grid power is in pgrid: the kernel wrote it, or the
  // b2g before the stage form did
  st->sim_time += time_elapsed * K;
  return HSB_OK;
}

// ---------------------------------------------------------------------------
// The same kernel on buffers the caller provides (state, power, and every
// scratch array), for the allocation-free entry point.  Nothing here
// allocates device memory; the layer and package tables are copied into the
// caller's buffers and the tensor maps are encoded on the host per call.
// ---------------------------------------------------------------------------
size_t rk4_fast_layer_table_bytes() { return sizeof(LayerF) * HSB_MAX_LAYERS; }
size_t rk4_fast_pack_table_bytes() { return sizeof(PackF); }
size_t rk4_fast_part_bytes(const hsb_dev_model *m) { return sizeof(double) * 2 * NEDGE * segmax_of(m); }

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
  int rc;
  if ((rc = check_shape(m))) return rc;
  FastArgs A;
  memset(&A, 0, sizeof(A));
  if ((rc = build_maps(&A.M, m, b.y, b.ytemp, b.t1, b.k1, b.k2, b.k3, b.pf))) return rc;
  LayerF Lf[HSB_MAX_LAYERS];
  PackF P;
  host_tables(m, Lf, &P);
  HSB_CUDA(cudaMemcpyAsync(b.layer_table, Lf, sizeof(LayerF) * m->nl, cudaMemcpyHostToDevice, m->stream));
  HSB_CUDA(cudaMemcpyAsync(b.pack_table, &P, sizeof(PackF), cudaMemcpyHostToDevice, m->stream));
  fill_common(A, m);
  A.bufP = b.y;
  A.bufQ = b.ytemp;
  A.Lf = (const LayerF *)b.layer_table;
  A.pk = (const PackF *)b.pack_table;
  A.pgrid = b.pgrid; A.pf = b.pf;
  A.y = b.y; A.ytemp = b.ytemp; A.t1 = b.t1; A.t2 = b.t2;
  A.k1 = b.k1; A.k2 = b.k2; A.k3 = b.k3;
  A.part = b.part; A.err = b.err; A.cnt = b.cnt;
  A.T = time_elapsed;
  int g = 0;
  const void *fn = kernel_for(false, false);
  if ((rc = fast_grid(m, fn, &g))) return rc;
  void *args[] = {&A};
  HSB_CUDA(cudaLaunchCooperativeKernel(fn, dim3((unsigned)g), dim3(FT_THREADS), args, tile_smem(m->nl), m->stream));
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
  return status_error(cnt[3]);
}

}  // namespace hsb
