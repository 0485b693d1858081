// rk4_krylov.cu -- the fast transient form (HSB_FORM_FAST), Krylov evaluation.
//
// Within a sampling interval the grid model's slope is affine,
//   f(T) = L T + c   (temperature_grid.c:3130-3601 cells, 2857-3093 package),
// with L the fixed conductance/capacitance operator (advection included) and
// c the power and ambient terms.  Then every stage of the reference's
// step-doubling RK4 (RCutil.c:440-640) is a polynomial in L applied to
// F = f(y):  with K the reference's k1 (K = F, or f(t1) of the previous
// attempt after a rejection, RCutil.c:568),
//   rk4_core:  k2 = F + (h/2) L K,  k3 = F + (h/2) L k2,  k4 = F + h L k3,
//              y_out - y = h (K + 2 k2 + 2 k3 + k4) / 6,
//   f(t1) = F + L (t1 - y),  t2 - t1 = rk4_core from t1 with k1 = f(t1),
//   error = max |ytemp - t2|,  accepted: y = ytemp.
// The kernel keeps Krylov vectors N_m = s_m L N_{m-1}, N_0 = F (FP32 cells,
// FP64 package nodes; s_m = the h of the attempt that first needed N_m, so
// the vectors stay of the order of F) and represents every stage vector by
// its coefficients over them (FP64, a few dozen per attempt).  A step is one
// pass that evaluates F = f(y) from the FP64 state, then the stencil passes
// that extend the sequence to the error polynomial's degree (7, +4 per
// rejection); each of those reads one FP32 vector (TMA halo box) and writes
// one, and the last one also forms the error norm and the candidate state
// ytemp in the second state buffer, which becomes the state when the step
// is accepted.
//
// Arithmetic: stencil passes in FP32 from FP32 vectors (F from the FP64
// state as FP32 deviations from ambient); state y, coefficient algebra,
// error norm, package nodes in FP64.  The step-size control is the
// reference's (SAFETY 0.95, growth <= 5, shrink >= 1/10, PRECISION 0.01) on
// the error norm computed as a combination of the Krylov vectors; every CTA
// reads the same global norm and takes the same decision.  When a step needs
// more than KRY_DMAX vectors (seven rejections in a row) the kernel stops at
// the last accepted step and the stage form finishes the interval.
#include <algorithm>

#include "fast_common.cuh"
#include "krylov_coef.cuh"
#include "rk4_tb.cuh"

namespace cg = cooperative_groups;

namespace hsb {

struct KryArgs {
  CUtensorMap m_y, m_y2;           // FP64 halo boxes of the two state buffers
  CUtensorMap m_pf;                // FP32 interior boxes of the power
  CUtensorMap m_N;                 // FP32 halo boxes of the Krylov vectors (4-D: vector index last)
  CUtensorMap m_Ni;                // FP32 interior boxes of the Krylov vectors
  CUtensorMap m_yi, m_y2i;         // FP64 interior boxes of the two state buffers
  StencilArgs S;
  int spidx, hsidx, subidx, solderidx, pcbidx;
  int segmax;
  const LayerF *Lf;
  const PackF *pk;
  const float *gN, *gS, *gW, *gE, *gA, *gB, *invC;
  const float *aN, *aS, *aW, *aE, *aO;
  double *pgrid;                   // FP64 grid power (read when K = 0, written for the last interval when K > 0)
  float *pf;
  double *y, *y2;                  // the two state buffers (which holds the state alternates)
  float *N;
  long long ns;                    // stride between Krylov vectors
  double *part;
  unsigned long long *err;
  long long *cnt;                  // [0] steps [1] attempts [2] status [3] passes [4..5] tout [6] final buffer
  double *tout;                    // [0] time reached [1] next step size
  double T;
  long long max_attempts;
  // trace mode (K > 0): K intervals in one launch, the power of interval k
  // from block powers bpow + k*nbv mapped to the grid in the kernel (the
  // arithmetic of xlate_vector_b2g, temperature_grid.c:1888-1929)
  int K;
  long long nbv;
  const double *bpow;
  const int *b2g_ptr, *b2g_blk;
  const double *b2g_occ, *b2g_area;
  double cell_area;
};

enum { K_FULL = 0, K_KRY = 1 };

struct KShared {
  double yp[NXMAX];                    // package part of the state
  double Np[KRY_DMAX + 1][NXMAX];      // package parts of the Krylov vectors
  double es[NEDGE], wred[FT_WARPS];
  double gmax, pmax;
  float xsf[NXMAX];                    // package inputs of the pass in FP32 (cells' edge terms)
  Coef E, D, F1, K;                    // error, full-step increment, f(t1), k1
  Coef E1, D1, F11;                    // E / h, D / h, F1 of a first attempt (k1 = F, uniform scale h)
  double ps[PMAX];                     // ps[m]: scale of N_m over L N_{m-1}
  unsigned long long bar;
  int lost;
  LayerF L[FT_MAX_LAYERS];
};

#define ERR_STAGED 8   // Krylov vectors the error pass stages in shared memory

// dynamic shared memory; the full-slope pass and the Krylov passes use the
// same bytes
struct KDyn {
  double *th;   // [nl][HR][DW]  FP64 state box (full slope pass)
  float *pw;    // [nl][NI]      power
  float *d;     // [nl][HR][DW]  state - T_amb in FP32
  float *vh;    // [nl][HR][KW]  input Krylov vector box
  float *vi;    // [ERR_STAGED][nl][NI] interior boxes of the vectors the error combines
  double *yi;   // [nl][NI]      interior box of the state (error pass)
};

__host__ __device__ inline size_t kdyn_layout(int nl, size_t off[6]) {
  size_t o = 0;
  off[0] = o; o = al128(o + 8 * (size_t)nl * DP);
  off[1] = o; o = al128(o + 4 * (size_t)nl * NI);
  off[2] = o; o = al128(o + 4 * (size_t)nl * DP);
  const size_t full = o;
  o = 0;
  off[3] = o; o = al128(o + 4 * (size_t)nl * KP);
  off[4] = o; o = al128(o + 4 * (size_t)ERR_STAGED * nl * NI);
  off[5] = o; o = al128(o + 8 * (size_t)nl * NI);
  return (o > full ? o : full) + 128;
}

// control state, identical in every thread
struct KCtl {
  int pkind, pm;        // pending package evaluation: kind (-1 none) and output index
  double ps;            // its scale
  int psp, sp, ep;      // edge-partial slots, error slot
  unsigned phase;       // completed tile-copy phases
  long long passes;
};

// the attempt's polynomials (one thread): D = ytemp - y, F1 = f(t1), E = ytemp - t2
// the h = 1 first-attempt coefficients (E1, D1, F11), once computed
__device__ Coef g_first[3];
__device__ int g_first_ready;

__device__ __forceinline__ void plan_attempt(KShared &sh, double h, int dcomp) {
  kry_plan(sh.E, sh.D, sh.F1, sh.K, sh.ps, h, dcomp);
}

// ---------------------------------------------------------------------------
// package nodes of the pending pass (one lane of warp 0 per node)
// ---------------------------------------------------------------------------
__device__ __forceinline__ void kfinish(const KryArgs &A, KCtl &c, KShared &sh) {
  if (c.pkind < 0) return;
  const StencilArgs &S = A.S;
  const int nx = S.nx, ne = S.secondary ? NEDGE : 8;
  const int tid = threadIdx.x, tx = tid & 31, ty = tid >> 5;
  const int ntj = (S.nc + TJ - 1) / TJ, nti = (S.nr + TI - 1) / TI;
  for (int e = ty; e < ne; e += FT_WARPS) {
    const int nseg = (e & 3) < 2 ? ntj : nti;
    const double *pp = A.part + ((long long)c.psp * NEDGE + e) * A.segmax;
    double s = 0.0;
    for (int q = tx; q < nseg; q += 32) s += pp[q];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (tx == 0) sh.es[e] = s;
  }
  __syncthreads();
  if (ty == 0 && tx < nx) {
    // full slope (with ambient) of the state, or s * L applied to N_{m-1}
    const PackF &P = *A.pk;
    const bool full = c.pkind == K_FULL;
    const double *x = full ? sh.yp : sh.Np[c.pm - 1];
    const double xq = x[tx];
    double s = full ? P.gamb[tx] * (S.ambient - xq) : -P.gamb[tx] * xq;
    if (P.eidx[tx] >= 0) s += P.ge[tx] * sh.es[P.eidx[tx]];
#pragma unroll
    for (int l = 0; l < PK_LINKS; l++)
      if (P.nb[tx][l] >= 0) s += P.g[tx][l] * (x[P.nb[tx][l]] - xq);
    sh.Np[c.pm][tx] = full ? s * P.invC[tx] : s * P.invC[tx] * c.ps;
  }
  c.pkind = -1;
}

// one warp polls the tile copy's mbarrier; the others wait at the CTA
// barrier, issuing nothing (the barrier also makes the copied tile visible
// to them)
__device__ __forceinline__ void kwait(KShared &sh, KCtl &c) {
  if (threadIdx.x < 32) {
    int it = 0;
    while (!mbar_try_wait(&sh.bar, c.phase & 1u)) {
      if (++it >= WAIT_LIMIT) {
        sh.lost = 1;
        break;
      }
    }
  }
  __syncthreads();
  c.phase++;
}

// the error pass stages N_j (j < min(m, ERR_STAGED), nonzero coefficient)
// and the state's interior box along with the halo box
__device__ __forceinline__ bool err_uses(const KShared &sh, int j) {
  return sh.E.c[j] != 0.0 || (j < sh.D.n && sh.D.c[j] != 0.0);
}

template <bool FULL, bool ERR>
__device__ __forceinline__ void kissue(const KryArgs &A, const KDyn &ds, KShared &sh, int m, int i0, int j0,
                                       const CUtensorMap *my) {
  if (threadIdx.x != 0) return;
  const unsigned nl = (unsigned)A.S.nl;
  asm volatile("fence.proxy.async.global;\n" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
  if (FULL) {
    mbar_expect_tx(&sh.bar, nl * (DP * 8 + NI * 4));
    tma3(ds.th, my, j0 - 2, i0 - 1, &sh.bar);
    tma3(ds.pw, &A.m_pf, j0, i0, &sh.bar);
  } else {
    unsigned bytes = nl * KP * 4;
    if (ERR) {
      bytes += nl * NI * 8;
      for (int j = 0; j < m && j < ERR_STAGED; j++)
        if (err_uses(sh, j)) bytes += nl * NI * 4;
    }
    mbar_expect_tx(&sh.bar, bytes);
    tma4(ds.vh, &A.m_N, j0 - 4, i0 - 1, m - 1, &sh.bar);
    if (ERR) {
      tma3(ds.yi, my, j0, i0, &sh.bar);
      for (int j = 0; j < m && j < ERR_STAGED; j++)
        if (err_uses(sh, j)) tma4(ds.vi + (size_t)j * nl * NI, &A.m_Ni, j0, i0, j, &sh.bar);
    }
  }
}

// One stencil pass: N_m = s L N_{m-1} (KRY) or N_0 = f(y) (FULL).  With ERR,
// the cells' part of the error combination sum_j E_j N_j is folded in.
// ERR: also the candidate state ynew = yb + sum_j D_j N_j of the own cells.
template <bool FIELD, bool ADV, bool FULL, bool ERR>
__device__ __forceinline__ void kpass(const KryArgs &A, cg::grid_group &grid, KCtl &c, KShared &sh,
                                      const KDyn &ds, int m, double s, const CUtensorMap *my = nullptr,
                                      const double *yb = nullptr, double *ynew = nullptr) {
  constexpr int CH = Chunk<FIELD, ADV>::n;
  const StencilArgs &S = A.S;
  const int nl = S.nl, nr = S.nr, nc = S.nc, nx = S.nx;
  const long long plane = S.plane;
  const int ne = S.secondary ? NEDGE : 8;
  const int tid = threadIdx.x, tx = tid & 31, ty = tid >> 5;
  const double amb = S.ambient;
  const float sf = (float)s;
  const int ntj = (nc + TJ - 1) / TJ, nti = (nr + TI - 1) / TI, ntiles = ntj * nti;
  float *Nout = A.N + (long long)m * A.ns;
  double errl = 0.0;
  // positions in the boxes: FULL reads the FP64 state box (row DW), KRY the
  // FP32 vector box (row KW)
  constexpr int W = FULL ? DW : KW, P = FULL ? DP : KP, X0 = FULL ? 2 : 4;
  const int p_i = (ty + 1) * W + tx + X0;
  int hr, hc;
  halo_cell(tid, &hr, &hc);
  const int p_h = hr * W + hc + X0 - 1;

  if ((int)blockIdx.x < ntiles)
    kissue<FULL, ERR>(A, ds, sh, m, (blockIdx.x / ntj) * TI, (blockIdx.x % ntj) * TJ, my);
  kfinish(A, c, sh);
  if (tid < nx) sh.xsf[tid] = FULL ? (float)(sh.yp[tid] - amb) : (float)sh.Np[m - 1][tid];
  const double *xin = FULL ? sh.yp : sh.Np[m > 0 ? m - 1 : 0];

  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int ti = tile / ntj, tj = tile - ti * ntj;
    const int i0 = ti * TI, j0 = tj * TJ;
    const int i = i0 + ty, j = j0 + tx;
    if (tile != (int)blockIdx.x) kissue<FULL, ERR>(A, ds, sh, m, i0, j0, my);
    kwait(sh, c);
    if (FULL) {
      for (int n = 0; n < nl; n++) {
        ds.d[n * DP + p_i] = (float)(ds.th[n * DP + p_i] - amb);
        if (hr >= 0) ds.d[n * DP + p_h] = (float)(ds.th[n * DP + p_h] - amb);
      }
    }
    __syncthreads();
    if (i < nr && j < nc) {
      const long long coff = (long long)i * nc + j;
      for (int n0 = 0; n0 < nl; n0 += CH) {
        float gN[CH], gS[CH], gE[CH], gW[CH], gA[CH], gB[CH], iC[CH];
        float aN[CH], aS[CH], aW[CH], aE[CH], aO[CH];
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
              }
            }
          }
        }
#pragma unroll
        for (int u = 0; u < CH; u++) {
          const int n = n0 + u;
          if (n >= nl) break;
          const long long cc = (long long)n * plane + coff;
          const float *vn = FULL ? ds.d + n * DP : ds.vh + n * KP;
          const float tc = vn[p_i];
          const LayerF &L = sh.L[n];
          float psum = 0.f;
          if (i > 0) psum += (FIELD ? gN[u] : L.gNS) * (vn[p_i - W] - tc);
          if (i < nr - 1) psum += (FIELD ? gS[u] : L.gNS) * (vn[p_i + W] - tc);
          if (j < nc - 1) psum += (FIELD ? gE[u] : L.gEW) * (vn[p_i + 1] - tc);
          if (j > 0) psum += (FIELD ? gW[u] : L.gEW) * (vn[p_i - 1] - tc);
          if (n > 0) psum += (FIELD ? gA[u] : sh.L[n - 1].gDown) * (vn[p_i - P] - tc);
          if (n < nl - 1) psum += (FIELD ? gB[u] : L.gDown) * (vn[p_i + P] - tc);
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
            // advection: FP64 on absolute temperatures (full slope) or on the vector
            double adv;
            if (FULL) {
              const double *th = ds.th + n * DP;
              const double T = th[p_i];
              adv = A.S.qin[cc] + (double)aO[u] * T;
              if (i > 0) adv += (double)aN[u] * ((th[p_i - DW] + T) / 2.0);
              if (i < nr - 1) adv += (double)aS[u] * ((th[p_i + DW] + T) / 2.0);
              if (j > 0) adv += (double)aW[u] * ((th[p_i - 1] + T) / 2.0);
              if (j < nc - 1) adv += (double)aE[u] * ((th[p_i + 1] + T) / 2.0);
            } else {
              const double T = tc;
              adv = (double)aO[u] * T;
              if (i > 0) adv += (double)aN[u] * (((double)vn[p_i - W] + T) / 2.0);
              if (i < nr - 1) adv += (double)aS[u] * (((double)vn[p_i + W] + T) / 2.0);
              if (j > 0) adv += (double)aW[u] * (((double)vn[p_i - 1] + T) / 2.0);
              if (j < nc - 1) adv += (double)aE[u] * (((double)vn[p_i + 1] + T) / 2.0);
            }
            psum += (float)adv;
          }
          const float ic = FIELD ? iC[u] : L.invC;
          const float k = FULL ? (ds.pw[n * NI + tid] + psum) * ic : psum * (ic * sf);
          Nout[cc] = k;
          if (ERR) {
            // the vectors the error and the candidate state combine: the
            // first ERR_STAGED from shared memory, the rest (after rejections) from global
            const int nD = sh.D.n, q = n * NI + tid;
            double e = sh.E.c[m] * (double)k, dy = 0.0;
            for (int jj = 0; jj < m && jj < ERR_STAGED; jj++) {
              if (!err_uses(sh, jj)) continue;
              const double w = (double)ds.vi[(size_t)jj * nl * NI + q];
              e += sh.E.c[jj] * w;
              if (jj < nD) dy += sh.D.c[jj] * w;
            }
            const double ybv = ds.yi[q];
            for (int jj = ERR_STAGED; jj < m; jj++) {
              const double ce = sh.E.c[jj], cd = jj < nD ? sh.D.c[jj] : 0.0;
              if (ce != 0.0 || cd != 0.0) {
                const double w = (double)A.N[(long long)jj * A.ns + cc];
                e += ce * w;
                dy += cd * w;
              }
            }
            errl = fmax(errl, fabs(e));
            ynew[cc] = ybv + dy;
          }
        }
      }
    }
    // partial edge sums of (v - x_node) of this pass's input over this tile's
    // share of each package edge
    const bool onN = i0 == 0, onS = i0 + TI >= nr, onW = j0 == 0, onE = j0 + TJ >= nc;
    for (int e = ty; e < ne; e += FT_WARPS) {
      const int side = e & 3;
      if (!((side == 0 && onN) || (side == 1 && onS) || (side == 2 && onW) || (side == 3 && onE))) continue;
      int layer, which, node;
      edge_desc(e, A.spidx, A.hsidx, A.subidx, A.solderidx, A.pcbidx, &layer, &which, &node);
      int pos = -1;
      if (side < 2) {
        const int r = side == 0 ? 1 : (nr - 1 - i0) + 1;
        if (j0 + tx < nc) pos = r * W + tx + X0;
      } else {
        const int col = side == 2 ? 0 : nc - 1 - j0;
        if (tx < TI && i0 + tx < nr) pos = (tx + 1) * W + col + X0;
      }
      double v = 0.0;
      if (pos >= 0) v = (FULL ? ds.th[layer * DP + pos] : (double)ds.vh[layer * KP + pos]) - xin[node];
      for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
      if (tx == 0) A.part[((long long)c.sp * NEDGE + e) * A.segmax + (side < 2 ? tj : ti)] = v;
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
      atomicMax(A.err + c.ep, (unsigned long long)__double_as_longlong(mx));
    }
  }
  grid.sync();
  c.pkind = FULL ? K_FULL : K_KRY;
  c.pm = m;
  c.ps = s;
  c.psp = c.sp;
  c.sp ^= 1;
  c.passes++;
}

// global error norm of the attempt: cells (already reduced) and package nodes
__device__ __forceinline__ double kerr_finish(const KryArgs &A, KCtl &c, KShared &sh) {
  const int tid = threadIdx.x, tx = tid & 31, ty = tid >> 5;
  kfinish(A, c, sh);
  if (tid == FT_THREADS - 1)
    sh.gmax = __longlong_as_double((long long)(*(volatile unsigned long long *)(A.err + c.ep)));
  if (ty == 0) {
    double perr = 0.0;
    if (tx < A.S.nx) {
      double e = 0.0;
      for (int jj = 0; jj < sh.E.n; jj++) e += sh.E.c[jj] * sh.Np[jj][tx];
      perr = fabs(e);
    }
    for (int o = 16; o > 0; o >>= 1) perr = fmax(perr, __shfl_down_sync(0xffffffffu, perr, o));
    if (tx == 0) sh.pmax = perr;
  }
  __syncthreads();
  const double mx = fmax(sh.gmax, sh.pmax);
  if (blockIdx.x == 0 && tid == 0) A.err[c.ep ^ 1] = 0ull;
  c.ep ^= 1;
  __syncthreads();
  return mx;
}

// FP32 grid power of interval iv: from A.pgrid (single interval), or mapped
// from the interval's block powers exactly as b2g_kernel does in FP64
__device__ __forceinline__ void kpower(const KryArgs &A, int iv) {
  const long long n = A.S.ncell, stride = (long long)gridDim.x * blockDim.x;
  if (A.K == 0) {
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += stride)
      A.pf[q] = (float)A.pgrid[q];
    return;
  }
  const double *b = A.bpow + (long long)iv * A.nbv;
  const bool last = iv == A.K - 1;   // later calls (and a stage-form fallback) find this power in pgrid
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += stride) {
    double val = 0.0;
    for (int e = A.b2g_ptr[q]; e < A.b2g_ptr[q + 1]; e++) val += A.b2g_occ[e] * b[A.b2g_blk[e]] / A.b2g_area[e];
    val *= A.cell_area;
    A.pf[q] = (float)val;
    if (last) A.pgrid[q] = val;
  }
}

template <bool FIELD, bool ADV>
__global__ void __launch_bounds__(FT_THREADS, 2) rk4_krylov_kernel(const __grid_constant__ KryArgs A) {
  cg::grid_group grid = cg::this_grid();
  extern __shared__ __align__(128) unsigned char dyn_raw[];
  __shared__ KShared sh;
  const StencilArgs &S = A.S;
  const int nx = S.nx, nl = S.nl;
  KDyn ds;
  {
    size_t off[6];
    kdyn_layout(nl, off);
    unsigned char *base = dyn_raw + ((128u - (smem_u32(dyn_raw) & 127u)) & 127u);
    ds.th = (double *)(base + off[0]);
    ds.pw = (float *)(base + off[1]);
    ds.d = (float *)(base + off[2]);
    ds.vh = (float *)(base + off[3]);
    ds.vi = (float *)(base + off[4]);
    ds.yi = (double *)(base + off[5]);
  }
  if (threadIdx.x < nl) sh.L[threadIdx.x] = A.Lf[threadIdx.x];
  if (threadIdx.x == 0) {
    sh.lost = 0;
    mbar_init(&sh.bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  kpower(A, 0);
  if (threadIdx.x < nx) sh.yp[threadIdx.x] = A.y[S.ncell + threadIdx.x];
  if (blockIdx.x == 0 && threadIdx.x == 0) { A.err[0] = 0ull; A.err[1] = 0ull; }
  // first-attempt coefficients for h = 1 (they scale with h); they depend on
  // nothing but the method, so the first launch in the process computes them
  // (one thread, tens of microseconds of FP64 scalar work) and later
  // launches read them back
  if (threadIdx.x == 0) {
    for (int q = 0; q < PMAX; q++) sh.ps[q] = 1.0;
    c_one(sh.K);
    if (*(volatile int *)&g_first_ready) {
      __threadfence();
      c_copy(sh.E1, g_first[0]);
      c_copy(sh.D1, g_first[1]);
      c_copy(sh.F11, g_first[2]);
    } else {
      plan_attempt(sh, 1.0, 0);
      c_copy(sh.E1, sh.E);
      c_copy(sh.D1, sh.D);
      c_copy(sh.F11, sh.F1);
      if (blockIdx.x == 0) {
        c_copy(g_first[0], sh.E1);
        c_copy(g_first[1], sh.D1);
        c_copy(g_first[2], sh.F11);
        __threadfence();
        atomicExch(&g_first_ready, 1);
      }
    }
  }
  grid.sync();
  KCtl c;
  c.pkind = -1;
  c.sp = 0;
  c.ep = 0;
  c.phase = 0;
  c.passes = 0;
  long long steps = 0, attempts = 0;
  int status = 0;
  double t = 0.0, h = 0.0, new_h = 1e-7;
  double *yb = A.y, *yn = A.y2;
  const int nint = A.K > 0 ? A.K : 1;
  int iv = 0;
  for (iv = 0; iv < nint; iv++) {
    if (iv > 0) {
      // the next interval: its power, and h restarts as in compute_temp_grid
      kpower(A, iv);
      grid.sync();
      t = 0.0;
      new_h = 1e-7;
    }
    while (t < A.T && new_h >= 1e-7 * 1.0e-6) {
      h = new_h;
      const CUtensorMap *myb = yb == A.y ? &A.m_y : &A.m_y2;
      kpass<FIELD, ADV, true, false>(A, grid, c, sh, ds, 0, 1.0, myb);   // N_0 = f(y)
      int dcomp = 0;
      if (threadIdx.x == 0) c_one(sh.K);
      double mx = 0.0;
      bool first = true;
      for (;;) {
        h = new_h;
        if (first) {
          // k1 = F and every vector made with scale h: the h = 1 coefficients scaled
          if (threadIdx.x < PMAX) {
            const int q = threadIdx.x;
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
        } else if (threadIdx.x == 0) {
          plan_attempt(sh, h, dcomp);
        }
        __syncthreads();
        const int dE = sh.E.n - 1;
        if (dE > KRY_DMAX || dE <= dcomp) {
          status = 3;
          break;
        }
        for (int q = dcomp + 1; q < dE; q++) kpass<FIELD, ADV, false, false>(A, grid, c, sh, ds, q, sh.ps[q]);
        kpass<FIELD, ADV, false, true>(A, grid, c, sh, ds, dE, sh.ps[dE], yb == A.y ? &A.m_yi : &A.m_y2i, yb, yn);
        dcomp = dE;
        mx = kerr_finish(A, c, sh);
        attempts++;
        if (mx <= 0.01) {
          new_h = 0.95 * h * pow(fabs(0.01 / mx), 0.2);
          if (new_h > 5.0 * h) new_h = 5.0 * h;
        } else {
          new_h = 0.95 * h * pow(fabs(0.01 / mx), 0.25);
          if (new_h < h / 10.0) new_h = h / 10.0;
        }
        if (attempts >= A.max_attempts) break;
        if (new_h >= h) break;
        // rejected: the retry's k1 is f(t1) of this attempt
        if (threadIdx.x == 0) c_copy(sh.K, sh.F1);
        __syncthreads();
      }
      if (status || attempts >= A.max_attempts) break;
      // accepted: the candidate buffer becomes the state
      if (threadIdx.x < nx) {
        double dy = 0.0;
        for (int q = 0; q < sh.D.n; q++) dy += sh.D.c[q] * sh.Np[q][threadIdx.x];
        sh.yp[threadIdx.x] += dy;
      }
      double *tmp = yb;
      yb = yn;
      yn = tmp;
      steps++;
      new_h = new_h < A.T - t - h ? new_h : A.T - t - h;
      t += h;
    }
    if (status || attempts >= A.max_attempts || sh.lost) break;
  }
  __syncthreads();
  if (sh.lost && threadIdx.x == 0) {
    for (int it = 0; it < WAIT_LIMIT && !mbar_try_wait(&sh.bar, c.phase & 1u); it++) {
    }
    status = 2;
  }
  if (status == 2) A.cnt[2] = 2;
  if (blockIdx.x == 0) {
    if (threadIdx.x < nx) yb[S.ncell + threadIdx.x] = sh.yp[threadIdx.x];
    if (threadIdx.x == 0) {
      A.cnt[6] = yb == A.y ? 0 : 1;
      A.cnt[0] = steps;
      A.cnt[1] = attempts;
      if (status == 3) A.cnt[2] = 3;
      if (attempts >= A.max_attempts) A.cnt[2] = 1;
      A.cnt[3] = c.passes;
      A.tout[0] = t;
      A.tout[1] = new_h;
      A.cnt[7] = iv;   // intervals completed
    }
  }
}

static const void *kry_kernel_for(bool field, bool adv) {
  return field ? (adv ? (const void *)rk4_krylov_kernel<true, true> : (const void *)rk4_krylov_kernel<true, false>)
               : (adv ? (const void *)rk4_krylov_kernel<false, true> : (const void *)rk4_krylov_kernel<false, false>);
}

static size_t kry_smem(int nl) {
  size_t off[6];
  return kdyn_layout(nl, off);
}

int kry_prepare_vectors(hsb_dev_model *m, FastWork *w);

// the temporally blocked kernel for this model: its resources, tile shape,
// co-resident grid and the chip descriptors for both roles of the state buffers
static int tb_prepare_single(hsb_dev_model *m, FastWork *w) {
  int rc;
  TbRes *r = (TbRes *)w->tb;
  rc = tb_res_prepare(m, &r, w->pk);
  w->tb = r;
  if (rc) return rc;
  const int v = m->fast_passes == 2 ? 1 : 0;   // kernel variant: FP32 or FP64 passes
  const bool fp64 = v == 1;
  if (m->tile_oi > 0 && (r->chip_oi[v] != m->tile_oi || r->chip_oj[v] != m->tile_oj)) r->chip_oi[v] = 0;
  if (r->chip_oi[v] == 0) {
    int nsm = 0, cap = 0;
    HSB_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, m->device));
    HSB_CUDA(cudaDeviceGetAttribute(&cap, cudaDevAttrMaxSharedMemoryPerBlockOptin, m->device));
    int oi = m->tile_oi, oj = m->tile_oj;
    if (oi <= 0 && (rc = tb_tile_for(m->nl, m->nr, m->nc, nsm, (size_t)cap, &oi, &oj, fp64))) return rc;
    if (oi * oj > TB_THREADS * tb_slots_rt(fp64, m->nl) ||
        2 * (size_t)tb_rcap(m->nl, oi, oj, fp64, (size_t)cap) * m->nl * (fp64 ? 8 : 4) + tb_static_smem(fp64) >
            (size_t)cap)
      return set_error(HSB_E_ARG, "requested tile of the blocked transient kernel does not fit");
    const size_t dyn = tb_dyn_smem(m->nl, oi, oj, fp64, (size_t)cap);
    if ((rc = raise_smem_limit(tb_kernel(fp64), dyn))) return rc;
    int per_sm = 0;
    HSB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, tb_kernel(fp64), TB_THREADS, dyn));
    if (per_sm < 1) return set_error(HSB_E_ARG, "temporally blocked transient kernel does not fit an SM");
    const long long tiles = (long long)((m->nr + oi - 1) / oi) * ((m->nc + oj - 1) / oj);
    r->grid[v] = (int)std::min<long long>((long long)per_sm * nsm, tiles);
    r->dyn[v] = dyn;
    r->chip_oi[v] = oi;
    r->chip_oj[v] = oj;
    r->cap = (size_t)cap;
    r->chip_y0 = r->chip_y1 = nullptr;
  }
  const bool same = (r->chip_y0 == m->y && r->chip_y1 == w->ytemp) || (r->chip_y0 == w->ytemp && r->chip_y1 == m->y);
  if (!same) {
    // descriptors of both variants (those not configured yet are placeholders)
    TChip C[4];
    memset(C, 0, sizeof(C));
    for (int q = 0; q < 2; q++) {
      if (!r->chip_oi[q]) continue;
      if ((rc = tb_fill_chip(m, r, m->y, w->ytemp, w->pf, w->t1, r->chip_oi[q], r->chip_oj[q], q == 1, r->cap,
                             &C[2 * q])))
        return rc;
      if ((rc = tb_fill_chip(m, r, w->ytemp, m->y, w->pf, w->t1, r->chip_oi[q], r->chip_oj[q], q == 1, r->cap,
                             &C[2 * q + 1])))
        return rc;
    }
    HSB_CUDA(h2d_on(r->d_chip, C, sizeof(C), m->stream));
    r->chip_y0 = m->y;
    r->chip_y1 = w->ytemp;
  }
  w->kfn = tb_kernel(fp64);
  w->kgrid = r->grid[v];
  if (!w->kev[0]) {
    HSB_CUDA(cudaEventCreate(&w->kev[0]));
    HSB_CUDA(cudaEventCreate(&w->kev[1]));
  }
  return HSB_OK;
}

// The fast form's kernel for a model.  From TB_MIN_CELLS cells up the
// temporally blocked kernel: its working set (two FP64 states, the Krylov
// vectors of the pass-by-pass form) no longer fits L2, and it reads the state
// once per attempt instead of streaming a vector per pass.  Below, the
// pass-by-pass kernel: its passes run from L2 and an attempt recomputes no
// halo (on a B200 it is 1.5x faster on a 256x256x6 stack, 1.2x on a 64x64x3
// chip).  The choice depends on the model's shape only, so a model's results
// do not depend on when or beside what it runs.
#define TB_MIN_CELLS (1LL << 21)
int kry_prepare(hsb_dev_model *m, FastWork *w) {
  const bool tb = tb_eligible(m);
  if (m->fast_passes >= 2) {
    if (!tb) return set_error(HSB_E_ARG, "the blocked forms take models with per-layer conductances and 3..12 layers");
    return tb_prepare_single(m, w);
  }
  if (m->fast_passes == 0 && tb && m->ncell >= TB_MIN_CELLS) return tb_prepare_single(m, w);
  return kry_prepare_vectors(m, w);
}

// the pass-by-pass kernel's Krylov vectors, tensor maps and grid
int kry_prepare_vectors(hsb_dev_model *m, FastWork *w) {
  int rc;
  if (!w->N) {
    w->nstride = (m->ncell + 63) / 64 * 64;
    HSB_CUDA(cudaMalloc(&w->N, sizeof(float) * w->nstride * (KRY_DMAX + 1)));
    if ((rc = make_map(&w->kmap_pf, w->pf, false, m, TJ, TI))) return rc;
    if ((rc = make_map4(&w->kmap_N, w->N, m, KW, HR, KRY_DMAX + 1, w->nstride))) return rc;
    if ((rc = make_map4(&w->kmap_Ni, w->N, m, TJ, TI, KRY_DMAX + 1, w->nstride))) return rc;
  }
  if (w->kmap_ybuf == w->ytemp && w->kmap_y2buf == m->y) {   // the buffers swapped roles: swap their maps
    CUtensorMap t = w->kmap_y;
    w->kmap_y = w->kmap_y2;
    w->kmap_y2 = t;
    t = w->kmap_yi;
    w->kmap_yi = w->kmap_y2i;
    w->kmap_y2i = t;
    w->kmap_ybuf = m->y;
    w->kmap_y2buf = w->ytemp;
  }
  if (w->kmap_ybuf != m->y) {
    if ((rc = make_map(&w->kmap_y, m->y, true, m, DW, HR))) return rc;
    if ((rc = make_map(&w->kmap_yi, m->y, true, m, TJ, TI))) return rc;
    w->kmap_ybuf = m->y;
  }
  if (w->kmap_y2buf != w->ytemp) {
    if ((rc = make_map(&w->kmap_y2, w->ytemp, true, m, DW, HR))) return rc;
    if ((rc = make_map(&w->kmap_y2i, w->ytemp, true, m, TJ, TI))) return rc;
    w->kmap_y2buf = w->ytemp;
  }
  const void *fn = kry_kernel_for(m->field, m->uchan_mask != 0);
  if (w->kfn != fn) {   // co-resident grid of this kernel variant, once
    if ((rc = coop_grid(m, fn, kry_smem(m->nl), &w->kgrid))) return rc;
    w->kfn = fn;
  }
  if (!w->kev[0]) {
    HSB_CUDA(cudaEventCreate(&w->kev[0]));
    HSB_CUDA(cudaEventCreate(&w->kev[1]));
  }
  return HSB_OK;
}

static int krylov_launch(hsb_dev_model *m, FastWork *w, double T, hsb_stats *st, double *t_done, double *h_next,
                         const double *bpow, int K, int *done);

int rk4_krylov_trace(hsb_dev_model *m, FastWork *w, const double *bpow, int K, double T, hsb_stats *st, int *done,
                     double *t_done, double *h_next) {
  return krylov_launch(m, w, T, st, t_done, h_next, bpow, K, done);
}

// the launch and the copy of its counters to the host, without waiting
// the temporally blocked kernel's launch (one chip, every co-resident CTA)
static int tb_enqueue(hsb_dev_model *m, FastWork *w, double T, hsb_stats *st, const double *bpow, int K) {
  TbRes *r = (TbRes *)w->tb;
  const int v = w->kfn == tb_kernel(true) ? 1 : 0;
  const TChip *chips = r->d_chip + 2 * v + (m->y == r->chip_y0 ? 0 : 1);
  const int4 *work = nullptr;
  const int *wptr = nullptr;
  long long *out = w->cnt;
  long long nbtot = (long long)m->total_n_blocks + m->nx;
  long long max_attempts = 10000000;
  HSB_CUDA(cudaMemsetAsync(w->cnt, 0, sizeof(long long) * 8, m->stream));
  HSB_CUDA(cudaMemsetAsync(r->bar, 0, sizeof(unsigned) * 2, m->stream));
  void *args[] = {&chips, &work, &wptr, &out, &T, &K, &bpow, &nbtot, &max_attempts};
  cudaLaunchConfig_t cfg;
  memset(&cfg, 0, sizeof(cfg));
  cfg.gridDim = dim3(r->grid[v]);
  cfg.blockDim = dim3(TB_THREADS);
  cfg.dynamicSmemBytes = r->dyn[v];
  cfg.stream = m->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  HSB_CUDA(cudaStreamIsCapturing(m->stream, &cap));
  const unsigned rec = cap == cudaStreamCaptureStatusActive ? cudaEventRecordExternal : cudaEventRecordDefault;
  HSB_CUDA(cudaEventRecordWithFlags(w->kev[0], m->stream, rec));
  HSB_CUDA(cudaLaunchKernelExC(&cfg, w->kfn, args));
  HSB_CUDA(cudaEventRecordWithFlags(w->kev[1], m->stream, rec));
  HSB_CUDA(cudaMemcpyAsync(w->h_cnt, w->cnt, sizeof(long long) * 8, cudaMemcpyDeviceToHost, m->stream));
  st->launches += 1;
  return HSB_OK;
}

int rk4_krylov_enqueue(hsb_dev_model *m, FastWork *w, double T, hsb_stats *st, const double *bpow, int K) {
  int rc;
  if ((rc = kry_prepare(m, w))) return rc;
  if (w->kfn == tb_kernel(false) || w->kfn == tb_kernel(true)) return tb_enqueue(m, w, T, st, bpow, K);
  KryArgs A;
  memset(&A, 0, sizeof(A));
  A.m_y = w->kmap_y;
  A.m_y2 = w->kmap_y2;
  A.m_yi = w->kmap_yi;
  A.m_y2i = w->kmap_y2i;
  A.m_Ni = w->kmap_Ni;
  A.m_pf = w->kmap_pf;
  A.m_N = w->kmap_N;
  A.S = make_args(m, m->L0, m->nr, m->nc);
  A.spidx = m->spidx; A.hsidx = m->hsidx;
  A.subidx = m->subidx; A.solderidx = m->solderidx; A.pcbidx = m->pcbidx;
  A.segmax = w->segmax;
  A.Lf = w->Lf;
  A.pk = w->pk;
  A.gN = w->gN; A.gS = w->gS; A.gW = w->gW; A.gE = w->gE; A.gA = w->gA; A.gB = w->gB;
  A.invC = w->invC;
  A.aN = w->aN; A.aS = w->aS; A.aW = w->aW; A.aE = w->aE; A.aO = w->aO;
  A.pgrid = m->pgrid;
  A.pf = w->pf;
  A.y = m->y;
  A.y2 = w->ytemp;
  A.N = w->N;
  A.ns = w->nstride;
  A.part = w->part;
  A.err = w->err;
  A.cnt = w->cnt;
  A.tout = (double *)(w->cnt + 4);
  A.T = T;
  A.max_attempts = 10000000;
  A.K = K;
  A.bpow = bpow;
  A.nbv = (long long)m->total_n_blocks + m->nx;
  A.b2g_ptr = m->b2g_ptr;
  A.b2g_blk = m->b2g_blk;
  A.b2g_occ = m->b2g_occ;
  A.b2g_area = m->b2g_area;
  A.cell_area = m->cell_area;
  const void *fn = w->kfn;
  HSB_CUDA(cudaMemsetAsync(w->cnt, 0, sizeof(long long) * 8, m->stream));
  void *args[] = {&A};
  // a cooperative launch through the attribute form, which stream capture
  // records as a cooperative kernel node
  cudaLaunchConfig_t cfg;
  memset(&cfg, 0, sizeof(cfg));
  cfg.gridDim = dim3(w->kgrid);
  cfg.blockDim = dim3(FT_THREADS);
  cfg.dynamicSmemBytes = kry_smem(m->nl);
  cfg.stream = m->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  // under stream capture the records are external ones, which become
  // event-record nodes, so a replayed graph still times the kernel (the
  // external flag is refused outside a capture)
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  HSB_CUDA(cudaStreamIsCapturing(m->stream, &cap));
  const unsigned rec = cap == cudaStreamCaptureStatusActive ? cudaEventRecordExternal : cudaEventRecordDefault;
  HSB_CUDA(cudaEventRecordWithFlags(w->kev[0], m->stream, rec));
  HSB_CUDA(cudaLaunchKernelExC(&cfg, fn, args));
  HSB_CUDA(cudaEventRecordWithFlags(w->kev[1], m->stream, rec));
  HSB_CUDA(cudaMemcpyAsync(w->h_cnt, w->cnt, sizeof(long long) * 8, cudaMemcpyDeviceToHost, m->stream));
  st->launches += 1;
  return HSB_OK;
}

// after the stream has reached the launch's counters: statistics, the swap of
// the state buffers, and the outcome (*t_done < T: rejection budget ran out)
int rk4_krylov_complete(hsb_dev_model *m, FastWork *w, double T, hsb_stats *st, double *t_done, double *h_next,
                        int *done) {
  {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, w->kev[0], w->kev[1]) == cudaSuccess) st->kernel_ms += ms;
    else cudaGetLastError();
  }
  if (w->h_cnt[6]) {   // the state ended in the second buffer
    double *tmp = m->y;
    m->y = w->ytemp;
    w->ytemp = tmp;
  }
  st->rk4_steps += w->h_cnt[0];
  st->rk4_attempts += w->h_cnt[1];
  st->slope_evals += w->h_cnt[3];
  double tout[2];
  memcpy(tout, w->h_cnt + 4, sizeof(tout));
  *t_done = T;
  *h_next = 0.0;
  *done = (int)w->h_cnt[7];
  if (w->h_cnt[2] == 1) return set_error(HSB_E_NOCONV, "fast transient: RK4 attempt cap reached");
  if (w->h_cnt[2] == 2) return set_error(HSB_E_CUDA, "fast transient: a tile copy did not complete in time");
  if (w->h_cnt[2] == 3) {
    *t_done = tout[0];
    *h_next = tout[1];
  }
  return HSB_OK;
}

static int krylov_launch(hsb_dev_model *m, FastWork *w, double T, hsb_stats *st, double *t_done, double *h_next,
                         const double *bpow, int K, int *done) {
  int rc;
  if ((rc = rk4_krylov_enqueue(m, w, T, st, bpow, K))) return rc;
  HSB_CUDA(cudaStreamSynchronize(m->stream));
  return rk4_krylov_complete(m, w, T, st, t_done, h_next, done);
}

}  // namespace hsb

extern "C" int hsb_dev_transient_kernel(const hsb_dev_model *m, int *kind) {
  if (!m || !kind) return hsb::set_error(HSB_E_ARG, "null argument");
  const hsb::FastWork *w = (const hsb::FastWork *)m->fast;
  *kind = 0;
  if (w && w->kfn) {
    if (w->kfn == hsb::tb_kernel(false)) *kind = HSB_TK_BLOCKED;
    else if (w->kfn == hsb::tb_kernel(true)) *kind = HSB_TK_BLOCKED_FP64;
    else *kind = HSB_TK_PASSES;
  }
  return HSB_OK;
}
