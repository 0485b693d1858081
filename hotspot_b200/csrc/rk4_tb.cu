// rk4_tb.cu -- the fast transient form with temporally blocked Krylov passes.
//
// The arithmetic is the Krylov form of rk4_krylov.cu: within a sampling
// interval the slope of the grid model (temperature_grid.c:3130-3601 cells,
// :2857-3093 package) is affine, f(T) = L T + c, so every stage of the
// reference's step-doubling RK4 (RCutil.c:440-640) is a polynomial in L
// applied to F = f(y).  An attempt with step h needs the vectors
//   V_0 = F,  V_m = h L V_{m-1}   (m = 1 .. dE; dE = 7 for a first attempt,
//                                  +4 for every rejection in a row)
// and forms, per cell, the increment d = sum_j D_j V_j (candidate state
// y + d) and the error e = sum_j E_j V_j (max-norm, step control).
//
// rk4_krylov.cu evaluates V_1 .. V_dE one grid-wide pass at a time: every
// pass streams one FP32 vector in and one out and ends in a grid barrier
// (the package nodes need edge sums of the whole grid).  Here a CTA loads
// the FP64 state of its tile plus a halo of dE + 1 cells ONCE and runs all
// dE + 1 passes in shared memory, the valid region shrinking by one cell per
// pass, so the own cells end with every V_m and nothing but the state, the
// power and the candidate state crosses HBM.
//
// The package nodes couple to the cells only through the edge rows and
// columns of the spreader/sink (and secondary-path) layers.  Split the cell
// part of V_m as A_m + B_m:
//   A_m = h L_cc A_{m-1},  A_0 = V_0            (no package input after F)
//   B_m = h (L_cc B_{m-1} + L_cp V^p_{m-1}),  B_0 = 0
// A is local (temporal blocking from y); B is linear in the package vectors
// and nonzero only within m - 1 cells of the grid boundary.  Its edge sums,
// which the package recursion needs, are sum_k h^{m-k} ER[m-1-k] V^p_k with
// ER[j][e'][e] = sum over edge e of L_cc^j L_cp u_{e'} -- a small FP64 table
// computed once per model.  An attempt therefore takes two chip barriers:
//   phase 1  every tile: A by temporal blocking.  Cells at least dE cells
//            from the grid's edge (where every B_m is 0) finish (candidate
//            state, error); the others keep the A part of their increment in
//            the candidate state and of their error sum in an FP64 buffer;
//            boundary tiles record the edge sums of A_0 .. A_{dE-1}
//   barrier; every CTA runs the package recursion (scalars, FP64)
//   phase 2  B on the band of width dE along the grid's edge, in boxes
//            (about one per CTA) whose grid-edge sides are fixed and whose
//            other sides carry a dE + 1 halo; the band cells finish
//            (increment += sum D_m B_m, error |E.A + E.B|)
//   barrier; every CTA reads the error norm and takes the step decision.
// Edge sums are reduced in a fixed order (per-tile partials), so results do
// not depend on timing.
//
// Precision: stencil passes in FP32 from the FP64 state as FP32 deviations
// from ambient (as rk4_krylov.cu); increment and error sums, package nodes,
// coefficient algebra and step control in FP64.  Step control is the
// reference's (SAFETY 0.95, growth <= 5, shrink >= 1/10, PRECISION 0.01).
// A rejection's retry uses k1 = f(t1) of the rejected attempt (RCutil.c:568)
// and recomputes its vectors from the state with a larger halo, splitting
// the tile into sub-tiles that fit shared memory.
//
// One kernel serves single models (one chip, every CTA) and batches (chips
// of uneven size and layer count, CTA groups and packed CTAs as the batch
// scheduler lays them out); chip-local barriers are counters in global
// memory with bounded waits.
#include <mutex>
#include <vector>

#include "fast_common.cuh"
#include "krylov_coef.cuh"
#include "rk4_tb.cuh"

namespace hsb {

// own cells per thread (accumulator slots): two for the FP32 kernel on up to
// six layers, else one, so that the FP64 sums of every layer stay in registers
template <typename V, int NL>
__host__ __device__ constexpr int tb_slots() {
  return (sizeof(V) == 4 && NL <= 6) ? 2 : 1;
}

__device__ Coef g_tb_first[3];
__device__ int g_tb_first_ready;

// layer table and package inputs in the vector type of the kernel variant
template <typename V> struct TLay;
template <> struct TLay<float> { typedef TLayer T; };
template <> struct TLay<double> { typedef TLayerD T; };

template <typename V>
struct TSh {
  typename TLay<V>::T L[TB_NLMAX];
  double Vp[TB_DMAX + 1][NXMAX];       // package parts of V_0 .. V_dE
  double yp[NXMAX];                    // package part of the state
  double es[TB_DMAX + 1][NEDGE];       // this tile's edge sums: [0] of y - y_node, [m + 1] of A_m
  double SA[TB_DMAX + 1][NEDGE];       // the chip's edge sums, same slots
  double wred[TB_WARPS];
  Coef E, D, F1, K, E1, D1, F11;
  double ps[PMAX];
  V xs[2][NXMAX];                      // package inputs of pass m in xs[m & 1] (in the cells' arithmetic)
  double gmax, pmax, hprev;
  int lost;
  int dE, dD, eLo, sep, SI, SJ;        // the attempt's plan
  int SEG;                             // phase 2: band segment length (0: on the sub-tiles)
};

// ---------------------------------------------------------------------------
// chip barrier over `size` CTAs (bounded wait; size 1: a CTA barrier)
// ---------------------------------------------------------------------------
template <typename V>
__device__ __forceinline__ void tsync(const TChip &C, int size, unsigned &gen, TSh<V> &sh) {
  __syncthreads();
  if (size > 1 && threadIdx.x == 0) {
    __threadfence();
    const unsigned g = gen;
    if (atomicAdd(&C.bar[0], 1u) == (unsigned)size - 1) {
      atomicExch(&C.bar[0], 0u);
      __threadfence();
      atomicAdd(&C.bar[1], 1u);
    } else {
      int it = 0;
      while (*(volatile unsigned *)&C.bar[1] == g) {
        if (++it >= TB_BAR_LIMIT) {
          sh.lost = 1;
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
  }
  gen++;
  __syncthreads();
}

// the grid power in the kernel variant's type
template <typename V> __device__ __forceinline__ const V *tb_power_of(const TChip &C);
template <> __device__ __forceinline__ const float *tb_power_of<float>(const TChip &C) { return C.pf; }
template <> __device__ __forceinline__ const double *tb_power_of<double>(const TChip &C) { return C.pd; }

// ---------------------------------------------------------------------------
// one stencil pass over the region rectangle [ra, rb) x [ca, cb) of an
// RI x RJ box whose cell (0, 0) is grid cell (gi0, gj0):
// P0: dst = V_0 = (p + L y) / C from the state deviations in src, with the
// grid power p already in dst (staged with the state box);
// else dst = h L src.  Package inputs from xs (BND: grid-boundary cells
// present in the region).  The operation order per cell is rk4_krylov.cu's.
// The rectangle's columns are dealt to the CTA's threads in row-major order
// (consecutive threads take consecutive columns of a row), so every thread
// gets the same number of columns to within one whatever the rectangle's
// shape.
// ---------------------------------------------------------------------------
template <typename V, int NL, bool BND, bool P0>
__device__ __forceinline__ void tb_pass(const TChip &C, const TSh<V> &sh, const V *__restrict__ xs,
                                        const V *__restrict__ src, V *__restrict__ dst, int RI, int RJ, int ra,
                                        int rb, int ca, int cb, int gi0, int gj0, V hf) {
  const int LP = RI * RJ;
  const int nrow = rb - ra, ncol = cb - ca;
  if (nrow <= 0 || ncol <= 0) return;
  const int tot = nrow * ncol;
  const int nr = C.nr, nc = C.nc;
  int rr = (int)threadIdx.x / ncol, cc = (int)threadIdx.x - rr * ncol;
  const int dr = TB_THREADS / ncol, dc = TB_THREADS - dr * ncol;
  for (int k = threadIdx.x; k < tot; k += TB_THREADS) {
    const int r = ra + rr, c = ca + cc;
    cc += dc;
    rr += dr;
    if (cc >= ncol) {
      cc -= ncol;
      rr++;
    }
    const int gi = gi0 + r, gj = gj0 + c;
    if (BND && ((unsigned)gi >= (unsigned)nr || (unsigned)gj >= (unsigned)nc)) continue;
    const V *p = src + r * RJ + c;
    V *o = dst + r * RJ + c;
    const bool hN = !BND || gi > 0, hS = !BND || gi < nr - 1, hW = !BND || gj > 0, hE = !BND || gj < nc - 1;
    V up = 0, cur = p[0], gup = 0;
#pragma unroll
    for (int n = 0; n < NL; n++) {
      const V *pn = p + n * LP;
      V gNS, gEW, gDn, invC, gEdgeNS, gEdgeEW, gAmb;
      int nb;
      if constexpr (sizeof(V) == 4) {   // two vector loads of the FP32 table
        const float4 L4 = *reinterpret_cast<const float4 *>(&sh.L[n]);          // gNS, gEW, gDn, invC
        const float4 E4 = *reinterpret_cast<const float4 *>(&sh.L[n].gEdgeNS);  // gEdgeNS, gEdgeEW, gAmb, nbase
        gNS = L4.x; gEW = L4.y; gDn = L4.z; invC = L4.w;
        gEdgeNS = E4.x; gEdgeEW = E4.y; gAmb = E4.z;
        nb = __float_as_int(E4.w);
      } else {
        gNS = sh.L[n].gNS; gEW = sh.L[n].gEW; gDn = sh.L[n].gDn; invC = sh.L[n].invC;
        gEdgeNS = sh.L[n].gEdgeNS; gEdgeEW = sh.L[n].gEdgeEW; gAmb = sh.L[n].gAmb;
        nb = sh.L[n].nbase;
      }
      const V dn = n < NL - 1 ? pn[LP] : V(0);
      V s = 0;
      if (hN) s += gNS * (pn[-RJ] - cur);
      if (hS) s += gNS * (pn[RJ] - cur);
      if (hE) s += gEW * (pn[1] - cur);
      if (hW) s += gEW * (pn[-1] - cur);
      if (n > 0) s += gup * (up - cur);
      if (n < NL - 1) s += gDn * (dn - cur);
      s -= gAmb * cur;                         // sink / PCB to ambient (0 elsewhere)
      if (BND) {
        if (nb >= 0) {
          if (gi == 0) s += gEdgeNS * (xs[nb + 2] - cur);
          if (gi == nr - 1) s += gEdgeNS * (xs[nb + 3] - cur);
          if (gj == nc - 1) s += gEdgeEW * (xs[nb + 1] - cur);
          if (gj == 0) s += gEdgeEW * (xs[nb + 0] - cur);
        }
      }
      if constexpr (P0) o[n * LP] = (o[n * LP] + s) * invC;   // the grid power, staged with the state box
      else o[n * LP] = s * (invC * hf);
      gup = gDn;
      up = cur;
      cur = dn;
    }
  }
}

template <typename V, int NL, bool P0>
__device__ __forceinline__ void tb_pass_any(bool bnd, const TChip &C, const TSh<V> &sh, const V *xs, const V *src,
                                            V *dst, int RI, int RJ, int ra, int rb, int ca, int cb, int gi0, int gj0,
                                            V hf) {
  if (bnd) tb_pass<V, NL, true, P0>(C, sh, xs, src, dst, RI, RJ, ra, rb, ca, cb, gi0, gj0, hf);
  else tb_pass<V, NL, false, P0>(C, sh, xs, src, dst, RI, RJ, ra, rb, ca, cb, gi0, gj0, hf);
}

// the sides of the grid a sub-tile's own cells lie on: bit 0 N, 1 S, 2 W, 3 E
__device__ __forceinline__ int tb_sides(const TChip &C, int i0, int j0, int SI, int SJ) {
  return (i0 == 0 ? 1 : 0) | (i0 + SI >= C.nr ? 2 : 0) | (j0 == 0 ? 4 : 0) | (j0 + SJ >= C.nc ? 8 : 0);
}

// edge sums over the sub-tile's own cells on the boundary: slot 0 from the
// FP64 state (minus the node temperature), slot m + 1 from A_m in smem
template <typename V>
__device__ __forceinline__ void tb_edge_sums(const TChip &C, TSh<V> &sh, const V *v, const double *yb, int slot,
                                             int RI, int RJ, int H, int i0, int j0, int SI, int SJ, int sides) {
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int LP = RI * RJ;
  const int ni = min(SI, C.nr - i0), nj = min(SJ, C.nc - j0);
  for (int e = w; e < C.ne; e += TB_WARPS) {
    const int side = e & 3;
    if (!((sides >> side) & 1)) continue;
    const int layer = C.eg_layer[e >> 2];
    const int node = C.eg_node[e >> 2] + ((side + 2) & 3);
    const int cnt = side < 2 ? nj : ni;
    double s = 0.0;
    for (int k = lane; k < cnt; k += 32) {
      const int oi = side == 0 ? 0 : side == 1 ? ni - 1 : k;
      const int oj = side < 2 ? k : side == 2 ? 0 : nj - 1;
      if (slot == 0)
        s += yb[(long long)layer * C.plane + (long long)(i0 + oi) * C.nc + (j0 + oj)] - sh.yp[node];
      else
        s += (double)v[layer * LP + (oi + H) * RJ + (oj + H)];
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) sh.es[slot][e] += s;
  }
}

// a cell the package reaches within an attempt: B_m (below) is zero more
// than m - 1 cells from the grid's edge, so every B_m of an attempt of degree
// dE is zero at in-plane distance dE and beyond
__device__ __forceinline__ bool tb_band(const TChip &C, int gi, int gj, int dE) {
  return min(min(gi, C.nr - 1 - gi), min(gj, C.nc - 1 - gj)) < dE;
}

// One sub-tile, phase 1: load the state box, run passes 0 .. dE of the A
// part (package input through V_0 only: A_0 = V_0, A_m = h L_cc A_{m-1});
// SUMS: edge sums into sh.es.  Own cells out of the package's reach finish
// (candidate state, error); the others get the A part of their increment in
// the candidate state and of their error sum in C.ea, finished by tb_bbox.
template <typename V, int NL>
__device__ void tb_subtile(const TChip &C, TSh<V> &sh, V *buf0, V *buf1, const double *__restrict__ yb,
                           double *__restrict__ yn, int i0, int j0, bool sums, double h, double &errl) {
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int dE = sh.dE, dD = sh.dD, eLo = sh.eLo, H = dE + 1;
  const int SI = sh.SI, SJ = sh.SJ;
  const int RI = SI + 2 * H, RJ = SJ + 2 * H, LP = RI * RJ;
  const int gi0 = i0 - H, gj0 = j0 - H;
  const int nr = C.nr, nc = C.nc;
  const bool bnd = gi0 < 1 || gj0 < 1 || gi0 + RI > nr - 1 || gj0 + RJ > nc - 1;
  const int sides = tb_sides(C, i0, j0, SI, SJ);
  const double amb = C.ambient;
  const bool sep = sh.sep != 0;
  constexpr int S = tb_slots<V, NL>();
  // own cells of this thread: slot s -> own index tid + s * TB_THREADS
  int q[S];
  long long g[S];
  bool ok[S], bd[S];
#pragma unroll
  for (int s = 0; s < S; s++) {
    const int idx = tid + s * TB_THREADS;
    const int oi = idx / SJ, oj = idx - (idx / SJ) * SJ;
    ok[s] = idx < SI * SJ && i0 + oi < nr && j0 + oj < nc;
    bd[s] = tb_band(C, i0 + oi, j0 + oj, dE);
    q[s] = (oi + H) * RJ + (oj + H);
    g[s] = (long long)(i0 + oi) * nc + (j0 + oj);
  }
  // per own cell and layer: the increment sum, then the error sum (sep); or
  // the error sum only, the increment going straight to the candidate state
  double acc[S][NL];
#pragma unroll
  for (int s = 0; s < S; s++)
#pragma unroll
    for (int n = 0; n < NL; n++) acc[s][n] = 0.0;

  // the state box as deviations from ambient in the kernel's type
  for (int r = w; r < RI; r += TB_WARPS) {
    const int gi = gi0 + r;
    if ((unsigned)gi >= (unsigned)nr) continue;
    for (int c = lane; c < RJ; c += 32) {
      const int gj = gj0 + c;
      if ((unsigned)gj >= (unsigned)nc) continue;
      const double *py = yb + (long long)gi * nc + gj;
      const V *pw = tb_power_of<V>(C) + (long long)gi * nc + gj;
#pragma unroll
      for (int n = 0; n < NL; n++) {
        buf0[n * LP + r * RJ + c] = (V)(__ldcg(py + (long long)n * C.plane) - amb);
        buf1[n * LP + r * RJ + c] = __ldcg(pw + (long long)n * C.plane);   // pass 0 adds it in place
      }
    }
  }
  if (tid < C.nx) sh.xs[0][tid] = (V)(sh.yp[tid] - amb);
  __syncthreads();
  if (sums) tb_edge_sums<V>(C, sh, nullptr, yb, 0, RI, RJ, H, i0, j0, SI, SJ, sides);

  // One CTA barrier per pass.  After the barrier that ends pass m, a thread
  // reads pass m's output (own cells, edge sums) and goes on to pass m + 1,
  // which writes the buffer pass m read: every thread finished reading it
  // before that barrier.  Package inputs are double-buffered for the same
  // reason: pass m + 1's are written before the barrier that ends pass m.
  V *src = buf0, *dst = buf1;
  const V hf = (V)h;
  for (int m = 0; m <= dE; m++) {
    if (m == 0) tb_pass_any<V, NL, true>(bnd, C, sh, sh.xs[0], src, dst, RI, RJ, 1, RI - 1, 1, RJ - 1, gi0, gj0, V(1));
    else
      tb_pass_any<V, NL, false>(bnd, C, sh, sh.xs[m & 1], src, dst, RI, RJ, m + 1, RI - m - 1, m + 1, RJ - m - 1, gi0,
                                gj0, hf);
    // the next pass's package input: none after V_0
    if (tid < C.nx) sh.xs[(m + 1) & 1][tid] = V(0);
    __syncthreads();
    const double cd = m <= dD ? sh.D.c[m] : 0.0, ce = m >= eLo ? sh.E.c[m] : 0.0;
    if (sep) {
      const double cf = m <= dD ? cd : ce;
      if (cf != 0.0) {
#pragma unroll
        for (int s = 0; s < S; s++)
          if (ok[s])
#pragma unroll
            for (int n = 0; n < NL; n++) acc[s][n] += cf * (double)dst[n * LP + q[s]];
      }
      if (m == dD) {   // the increment is complete: the candidate state, then the error sums
#pragma unroll
        for (int s = 0; s < S; s++)
          if (ok[s])
#pragma unroll
            for (int n = 0; n < NL; n++) {
              const long long cc = (long long)n * C.plane + g[s];
              yn[cc] = __ldcg(yb + cc) + acc[s][n];
              acc[s][n] = 0.0;
            }
      }
    } else {   // overlapping increment and error terms (a retry): the increment in the candidate state
#pragma unroll
      for (int s = 0; s < S; s++)
        if (ok[s])
#pragma unroll
          for (int n = 0; n < NL; n++) {
            const double v = (double)dst[n * LP + q[s]];
            if (m <= dD) {
              const long long cc = (long long)n * C.plane + g[s];
              yn[cc] = (m == 0 ? __ldcg(yb + cc) : yn[cc]) + cd * v;
            }
            acc[s][n] += ce * v;
          }
    }
    if (sums && m < dE) tb_edge_sums<V>(C, sh, dst, yb, m + 1, RI, RJ, H, i0, j0, SI, SJ, sides);
    V *t = src;
    src = dst;
    dst = t;
  }
  __syncthreads();   // the last pass's output is read; the buffers are free for the next sub-tile
#pragma unroll
  for (int s = 0; s < S; s++)
    if (ok[s])
#pragma unroll
      for (int n = 0; n < NL; n++) {
        if (bd[s]) C.ea[(long long)n * C.plane + g[s]] = acc[s][n];
        else errl = fmax(errl, fabs(acc[s][n]));
      }
}

// Phase 2 on one box: the package part B of V_1 .. V_dE, B_0 = 0 and
// B_m = h (L_cc B_{m-1} + L_cp V^p_{m-1}), over the box [gi0, gi0 + RI) x
// [gj0, gj0 + RJ) holding the own rectangle [i0, i0 + SI) x [j0, j0 + SJ).
// Box sides on the grid's edge (fN, fS, fW, fE) are fixed; the others shrink
// by one cell per pass, and lie dE + 1 cells beyond the own rectangle.  Own
// cells the package reaches finish: the increment gets sum D_m B_m on top of
// its A part, the error |E.A + E.B| enters the norm.
template <typename V, int NL>
__device__ void tb_bbox(const TChip &C, TSh<V> &sh, V *buf0, V *buf1, double *__restrict__ yn, int i0, int j0,
                        int SI, int SJ, int gi0, int gj0, int RI, int RJ, bool fN, bool fS, bool fW, bool fE,
                        double h, double &errl) {
  const int tid = threadIdx.x;
  const int dE = sh.dE, dD = sh.dD, eLo = sh.eLo;
  const int LP = RI * RJ;
  const int nr = C.nr, nc = C.nc;
  const bool bnd = gi0 < 1 || gj0 < 1 || gi0 + RI > nr - 1 || gj0 + RJ > nc - 1;
  const bool sep = sh.sep != 0;
  constexpr int S = tb_slots<V, NL>();
  int q[S];
  long long g[S];
  bool ok[S];
#pragma unroll
  for (int s = 0; s < S; s++) {
    const int idx = tid + s * TB_THREADS;
    const int oi = idx / SJ, oj = idx - (idx / SJ) * SJ;
    const int gi = i0 + oi, gj = j0 + oj;
    ok[s] = idx < SI * SJ && gi < nr && gj < nc && tb_band(C, gi, gj, dE);
    q[s] = (gi - gi0) * RJ + (gj - gj0);
    g[s] = (long long)gi * nc + gj;
  }
  double acc[S][NL];
#pragma unroll
  for (int s = 0; s < S; s++)
#pragma unroll
    for (int n = 0; n < NL; n++) acc[s][n] = 0.0;
  for (int k = tid; k < NL * LP; k += TB_THREADS) buf0[k] = V(0);   // B_0
  if (tid < C.nx) sh.xs[1][tid] = (V)sh.Vp[0][tid];                 // pass 1's package input
  __syncthreads();
  V *src = buf0, *dst = buf1;
  const V hf = (V)h;
  for (int m = 1; m <= dE; m++) {
    tb_pass_any<V, NL, false>(bnd, C, sh, sh.xs[m & 1], src, dst, RI, RJ, fN ? 0 : m + 1, fS ? RI : RI - m - 1,
                              fW ? 0 : m + 1, fE ? RJ : RJ - m - 1, gi0, gj0, hf);
    if (tid < C.nx && m < dE) sh.xs[(m + 1) & 1][tid] = (V)sh.Vp[m][tid];
    __syncthreads();
    const double cd = m <= dD ? sh.D.c[m] : 0.0, ce = m >= eLo ? sh.E.c[m] : 0.0;
    if (sep) {
      const double cf = m <= dD ? cd : ce;
      if (cf != 0.0) {
#pragma unroll
        for (int s = 0; s < S; s++)
          if (ok[s])
#pragma unroll
            for (int n = 0; n < NL; n++) acc[s][n] += cf * (double)dst[n * LP + q[s]];
      }
      if (m == dD) {
#pragma unroll
        for (int s = 0; s < S; s++)
          if (ok[s])
#pragma unroll
            for (int n = 0; n < NL; n++) {
              const long long cc = (long long)n * C.plane + g[s];
              yn[cc] = __ldcg(yn + cc) + acc[s][n];   // written by another CTA in phase 1: read from L2
              acc[s][n] = 0.0;
            }
      }
    } else {
#pragma unroll
      for (int s = 0; s < S; s++)
        if (ok[s])
#pragma unroll
          for (int n = 0; n < NL; n++) {
            const double v = (double)dst[n * LP + q[s]];
            if (m <= dD) {
              const long long cc = (long long)n * C.plane + g[s];
              yn[cc] = __ldcg(yn + cc) + cd * v;
            }
            acc[s][n] += ce * v;
          }
    }
    V *t = src;
    src = dst;
    dst = t;
  }
  __syncthreads();
#pragma unroll
  for (int s = 0; s < S; s++)
    if (ok[s])
#pragma unroll
      for (int n = 0; n < NL; n++) {
        const long long cc = (long long)n * C.plane + g[s];
        errl = fmax(errl, fabs(__ldcg(C.ea + cc) + acc[s][n]));
      }
}

// a box for phase 2: the own rectangle [i0, i0 + SI) x [j0, j0 + SJ) with
// dE + 1 cells of halo, clipped to the grid (clipped sides fixed)
template <typename V, int NL>
__device__ __forceinline__ void tb_bbox_own(const TChip &C, TSh<V> &sh, V *buf0, V *buf1, double *yn, int i0, int j0,
                                            int SI, int SJ, double h, double &errl) {
  const int H = sh.dE + 1;
  int lo_i = i0 - H, hi_i = i0 + SI + H, lo_j = j0 - H, hi_j = j0 + SJ + H;
  const bool fN = lo_i <= 0, fS = hi_i >= C.nr, fW = lo_j <= 0, fE = hi_j >= C.nc;
  if (fN) lo_i = 0;
  if (fS) hi_i = C.nr;
  if (fW) lo_j = 0;
  if (fE) hi_j = C.nc;
  tb_bbox<V, NL>(C, sh, buf0, buf1, yn, i0, j0, SI, SJ, lo_i, lo_j, hi_i - lo_i, hi_j - lo_j, fN, fS, fW, fE, h, errl);
}

// the package recursion: V^p_0 .. V^p_dE from the chip's edge sums of y and
// of A_0 .. A_{dE-1} (sh.SA) and the edge-response table (one warp; lanes
// are edges, then nodes)
template <typename V>
__device__ __noinline__ void tb_package(const TChip &C, TSh<V> &sh, double h) {
  const int lane = threadIdx.x & 31;
  const int nx = C.nx, ne = C.ne, dE = sh.dE;
  const PackF &P = *C.pk;
  __shared__ double es_m[NEDGE];
  // V^p_0: the full package slope of the state (ambient, edge sums, links)
  if (lane < nx) {
    const double xq = sh.yp[lane];
    double s = P.gamb[lane] * (C.ambient - xq);
    if (P.eidx[lane] >= 0) s += P.ge[lane] * sh.SA[0][P.eidx[lane]];
#pragma unroll
    for (int l = 0; l < PK_LINKS; l++)
      if (P.nb[lane][l] >= 0) s += P.g[lane][l] * (sh.yp[P.nb[lane][l]] - xq);
    sh.Vp[0][lane] = s * P.invC[lane];
  }
  __syncwarp();
  for (int m = 1; m <= dE; m++) {
    // edge sums of V_{m-1} - x_node: A part from the tiles, B part from the table
    if (lane < ne) {
      const int e = lane;
      double sb = 0.0;
      double hk = h;   // h^{m-1-k}, k = m-2 down to 0
      for (int k = m - 2; k >= 0; k--) {
        const double *er = C.er + ((long long)(m - 2 - k) * ne) * ne;
        double t = 0.0;
        for (int e2 = 0; e2 < ne; e2++) t += er[e2 * ne + e] * sh.Vp[k][C.eg_node[e2 >> 2] + (((e2 & 3) + 2) & 3)];
        sb += hk * t;
        hk *= h;
      }
      const int node = C.eg_node[e >> 2] + (((e & 3) + 2) & 3);
      const double n_e = (e & 3) < 2 ? (double)C.nc : (double)C.nr;
      es_m[e] = sh.SA[m][e] + sb - n_e * sh.Vp[m - 1][node];
    }
    __syncwarp();
    if (lane < nx) {
      const double *x = sh.Vp[m - 1];
      const double xq = x[lane];
      double s = -P.gamb[lane] * xq;
      if (P.eidx[lane] >= 0) s += P.ge[lane] * es_m[P.eidx[lane]];
#pragma unroll
      for (int l = 0; l < PK_LINKS; l++)
        if (P.nb[lane][l] >= 0) s += P.g[lane][l] * (x[P.nb[lane][l]] - xq);
      sh.Vp[m][lane] = s * P.invC[lane] * h;
    }
    __syncwarp();
  }
}

// the attempt's coefficients (thread 0); returns 0, or 3 when the degree is
// beyond what a sub-tile of this chip can hold
template <typename V>
__device__ __noinline__ int tb_plan(const TChip &C, TSh<V> &sh, double h, bool first, int size) {
  if (first) {
    for (int q = 0; q < PMAX; q++) sh.ps[q] = h;
    sh.E.n = sh.E1.n;
    sh.D.n = sh.D1.n;
    sh.F1.n = sh.F11.n;
    for (int q = 0; q < sh.E1.n; q++) sh.E.c[q] = h * sh.E1.c[q];
    for (int q = 0; q < sh.D1.n; q++) sh.D.c[q] = h * sh.D1.c[q];
    for (int q = 0; q < sh.F11.n; q++) sh.F1.c[q] = sh.F11.c[q];
  } else {
    // k1 = f(t1) of the rejected attempt, re-expressed over the basis of the
    // new step (V_j scales with h^j)
    const double r = sh.hprev / h;
    double rj = 1.0;
    c_copy(sh.K, sh.F1);
    for (int j = 0; j < sh.K.n; j++) {
      sh.K.c[j] *= rj;
      rj *= r;
    }
    kry_plan(sh.E, sh.D, sh.F1, sh.K, sh.ps, h, 0);
  }
  const int dE = sh.E.n - 1, dD = sh.D.n - 1;
  int eLo = 0;
  while (eLo < dE && sh.E.c[eLo] == 0.0) eLo++;
  const int sep = dD < eLo ? 1 : 0;
  sh.dE = dE;
  sh.dD = dD;
  sh.eLo = eLo;
  sh.sep = sep;
  if (dE > TB_DMAX) return 3;
  // sub-tile: the own tile, halved until its box fits the buffers and its
  // own cells fit the threads' accumulator slots
  const int H = dE + 1, slots = tb_slots_rt(sizeof(V) == 8, C.nl);
  // phase 2's band segments: a box of 2 dE + 1 cells across the band and
  // SEG + 2 H along it; about one segment per CTA of the chip, at least 8 long
  {
    int fit = C.rcap / (2 * dE + 1) - 2 * H;
    if (dE > 0 && fit > TB_THREADS * slots / dE) fit = TB_THREADS * slots / dE;
    const int perim = 2 * C.nc + 2 * max(0, C.nr - 2 * dE);
    int seg = max(8, (perim + size - 1) / size);
    if (seg > fit) seg = fit;
    sh.SEG = seg >= 4 ? seg : 0;
  }
  for (int SJ = C.oj; SJ >= 8; SJ >>= 1)
    for (int SI = C.oi; SI >= 1; SI >>= 1)
      if ((SI + 2 * H) * (SJ + 2 * H) <= C.rcap && SI * SJ <= TB_THREADS * slots) {
        sh.SI = SI;
        sh.SJ = SJ;
        return 0;
      }
  return 3;
}

// grid power of interval iv for this CTA's tiles, in the kernel's type
template <typename V>
__device__ void tb_power(const TChip &C, int rank, int size, int K, int iv, const double *bpow, long long nbtot,
                         long long boff) {
  const double *b = K > 0 ? bpow + (long long)iv * nbtot + boff : nullptr;
  const bool last = K > 0 && iv == K - 1;
  for (int t = rank; t < C.ntiles; t += size) {
    const int i0 = (t / C.ntj) * C.oi, j0 = (t % C.ntj) * C.oj;
    const int ni = min(C.oi, C.nr - i0), nj = min(C.oj, C.nc - j0);
    for (int k = threadIdx.x; k < C.nl * ni * nj; k += blockDim.x) {
      const int n = k / (ni * nj), rem = k - n * (ni * nj), oi = rem / nj, oj = rem - (rem / nj) * nj;
      const long long qq = (long long)n * C.plane + (long long)(i0 + oi) * C.nc + (j0 + oj);
      if (K == 0) {
        if constexpr (sizeof(V) == 4) C.pf[qq] = (float)C.pgrid[qq];
        else C.pd[qq] = C.pgrid[qq];
      } else {
        double val = 0.0;
        for (int e = C.b2g_ptr[qq]; e < C.b2g_ptr[qq + 1]; e++)
          val += C.b2g_occ[e] * b[C.b2g_blk[e]] / C.b2g_area[e];   // blist_avg, temperature_grid.c:331
        val *= C.cell_area;
        if constexpr (sizeof(V) == 4) C.pf[qq] = (float)val;
        else C.pd[qq] = val;
        if (last) C.pgrid[qq] = val;
      }
    }
  }
}

// K sampling intervals (K = 0: one, power from C.pgrid) of one chip by a
// group of `size` CTAs of which this is `rank`
template <typename V, int NL>
__device__ void tb_chip(const TChip &C, int rank, int size, long long *out, TSh<V> &sh, V *dyn, double T, int K,
                        const double *bpow, long long nbtot, long long boff, long long max_attempts) {
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int nx = C.nx;
  V *buf0 = dyn, *buf1 = dyn + (size_t)C.rcap * NL;
  if constexpr (sizeof(V) == 4) {
    if (tid < NL) sh.L[tid] = C.L[tid];
  } else {
    if (tid < NL) sh.L[tid] = C.Ld[tid];
  }
  int cur = (int)out[6];
  if (tid < nx) sh.yp[tid] = __ldcg(C.y[cur] + C.ncell + tid);
  unsigned gen = 0;
  long long steps = 0, attempts = 0, passes = 0, a = 0;
  int status = 0;
  double t = 0.0, h = 0.0, new_h = 1e-7;
  const int nint = K > 0 ? K : 1;
  int iv = 0;
  if (rank == 0 && tid < 3) C.err[tid] = 0ull;
  for (iv = 0; iv < nint && !status && !sh.lost; iv++) {
    tb_power<V>(C, rank, size, K, iv, bpow, nbtot, boff);
    tsync(C, size, gen, sh);
    t = 0.0;
    new_h = 1e-7;
    while (t < T && new_h >= 1e-7 * 1.0e-6 && !sh.lost) {
      h = new_h;
      bool first = true;
      double mx = 0.0;
      for (;;) {
        h = new_h;
        if (tid == 0) status = tb_plan(C, sh, h, first, size);
        if (tid == 0) sh.wred[0] = (double)status;
        __syncthreads();
        status = (int)sh.wred[0];
        __syncthreads();
        if (status) break;
        first = false;
        const int dE = sh.dE, SI = sh.SI, SJ = sh.SJ;
        const double *yb = C.y[cur];
        double *yn = C.y[cur ^ 1];
        double errl = 0.0;
        // ---- phase 1: A by temporal blocking on every tile
        for (int tt = rank; tt < C.ntiles && !sh.lost; tt += size) {
          const int ti0 = (tt / C.ntj) * C.oi, tj0 = (tt % C.ntj) * C.oj;
          const bool tsides = ti0 == 0 || tj0 == 0 || ti0 + C.oi >= C.nr || tj0 + C.oj >= C.nc;
          if (tsides) {
            for (int k = tid; k < (dE + 1) * NEDGE; k += blockDim.x) (&sh.es[0][0])[k] = 0.0;
            __syncthreads();
          }
          for (int si = 0; si < C.oi; si += SI)
            for (int sj = 0; sj < C.oj; sj += SJ) {
              const int i0 = ti0 + si, j0 = tj0 + sj;
              if (i0 >= C.nr || j0 >= C.nc) continue;
              const bool sums = tb_sides(C, i0, j0, SI, SJ) != 0;
              tb_subtile<V, NL>(C, sh, buf0, buf1, yb, yn, i0, j0, sums, h, errl);
            }
          if (tsides) {   // this tile's partial edge sums
            const int ti = tt / C.ntj, tj = tt % C.ntj;
            const int ts = (ti0 == 0 ? 1 : 0) | (ti0 + C.oi >= C.nr ? 2 : 0) | (tj0 == 0 ? 4 : 0) |
                           (tj0 + C.oj >= C.nc ? 8 : 0);
            for (int k = tid; k < (dE + 1) * C.ne; k += blockDim.x) {
              const int slot = k / C.ne, e = k - slot * C.ne, side = e & 3;
              if ((ts >> side) & 1)
                C.part[((long long)slot * NEDGE + e) * C.segmax + (side < 2 ? tj : ti)] = sh.es[slot][e];
            }
            __syncthreads();
          }
        }
        tsync(C, size, gen, sh);
        if (sh.lost) break;
        // ---- the chip's edge sums, then the package recursion (every CTA)
        for (int k = w; k < (dE + 1) * C.ne; k += TB_WARPS) {
          const int slot = k / C.ne, e = k - slot * C.ne;
          const int nseg = (e & 3) < 2 ? C.ntj : C.nti;
          const double *pp = C.part + ((long long)slot * NEDGE + e) * C.segmax;
          double s = 0.0;
          for (int qq = lane; qq < nseg; qq += 32) s += __ldcg(pp + qq);
          for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
          if (lane == 0) sh.SA[slot][e] = s;
        }
        __syncthreads();
        if (w == 0) tb_package<V>(C, sh, h);
        if (rank == 0 && tid == 0) C.err[(a + 1) % 3] = 0ull;
        __syncthreads();
        // ---- phase 2: the package part B on the band within dE cells of
        // the grid's edge, in segments dealt over the chip's CTAs (the four
        // strips: N and S full width, W and E between them); or, when no
        // segment box fits the buffers, on the sub-tiles that reach the band
        if (sh.SEG > 0) {
          const int SEG = sh.SEG, nr = C.nr, nc = C.nc;
          const int b = min(dE, nr), sS = max(b, nr - dE), wc = min(dE, nc), eC = max(wc, nc - dE);
          const int nN = (nc + SEG - 1) / SEG, nS = sS < nr ? nN : 0;
          const int nW = sS > b ? (sS - b + SEG - 1) / SEG : 0, nE = eC < nc ? nW : 0;
          for (int sg = rank; sg < nN + nS + nW + nE && !sh.lost; sg += size) {
            int i0, j0, si, sj;
            if (sg < nN + nS) {
              const int k = sg < nN ? sg : sg - nN;
              j0 = k * SEG;
              sj = min(SEG, nc - j0);
              i0 = sg < nN ? 0 : sS;
              si = sg < nN ? b : nr - sS;
            } else {
              const int k = sg - nN - nS, kk = k < nW ? k : k - nW;
              i0 = b + kk * SEG;
              si = min(SEG, sS - i0);
              j0 = k < nW ? 0 : eC;
              sj = k < nW ? wc : nc - eC;
            }
            tb_bbox_own<V, NL>(C, sh, buf0, buf1, yn, i0, j0, si, sj, h, errl);
          }
        } else {
          for (int tt = rank; tt < C.ntiles && !sh.lost; tt += size) {
            const int ti0 = (tt / C.ntj) * C.oi, tj0 = (tt % C.ntj) * C.oj;
            for (int si = 0; si < C.oi; si += SI)
              for (int sj = 0; sj < C.oj; sj += SJ) {
                const int i0 = ti0 + si, j0 = tj0 + sj;
                if (i0 >= C.nr || j0 >= C.nc) continue;
                const bool reach = i0 < dE || j0 < dE || i0 + SI > C.nr - dE || j0 + SJ > C.nc - dE;
                if (reach) tb_bbox_own<V, NL>(C, sh, buf0, buf1, yn, i0, j0, SI, SJ, h, errl);
              }
          }
        }
        // ---- the error norm: cells (all CTAs of the chip) and package nodes
        for (int o = 16; o > 0; o >>= 1) errl = fmax(errl, __shfl_down_sync(0xffffffffu, errl, o));
        if (lane == 0) sh.wred[w] = errl;
        __syncthreads();
        if (tid == 0) {
          double mxl = sh.wred[0];
          for (int q = 1; q < TB_WARPS; q++) mxl = fmax(mxl, sh.wred[q]);
          atomicMax(C.err + a % 3, (unsigned long long)__double_as_longlong(mxl));
        }
        tsync(C, size, gen, sh);
        if (sh.lost) break;
        if (tid == 0) sh.gmax = __longlong_as_double((long long)(*(volatile unsigned long long *)(C.err + a % 3)));
        if (w == 0) {
          double perr = 0.0;
          if (lane < nx) {
            double e = 0.0;
            for (int jj = 0; jj < sh.E.n; jj++) e += sh.E.c[jj] * sh.Vp[jj][lane];
            perr = fabs(e);
          }
          for (int o = 16; o > 0; o >>= 1) perr = fmax(perr, __shfl_down_sync(0xffffffffu, perr, o));
          if (lane == 0) sh.pmax = perr;
        }
        __syncthreads();
        mx = fmax(sh.gmax, sh.pmax);
        a++;
        attempts++;
        passes += dE + 1;
        if (mx <= 0.01) {
          new_h = 0.95 * h * pow(fabs(0.01 / mx), 0.2);
          if (new_h > 5.0 * h) new_h = 5.0 * h;
        } else {
          new_h = 0.95 * h * pow(fabs(0.01 / mx), 0.25);
          if (new_h < h / 10.0) new_h = h / 10.0;
        }
        if (attempts >= max_attempts) break;
        if (new_h >= h) break;
        if (tid == 0) sh.hprev = h;   // rejected: the retry's k1 is f(t1) of this attempt
        __syncthreads();
      }
      if (status || sh.lost || attempts >= max_attempts) break;
      // accepted: the candidate buffer becomes the state
      if (tid < nx) {
        double dy = 0.0;
        for (int qd = 0; qd < sh.D.n; qd++) dy += sh.D.c[qd] * sh.Vp[qd][tid];
        sh.yp[tid] += dy;
      }
      __syncthreads();
      cur ^= 1;
      steps++;
      new_h = new_h < T - t - h ? new_h : T - t - h;
      t += h;
    }
    if (status || sh.lost || attempts >= max_attempts) break;
  }
  __syncthreads();
  if (rank == 0) {
    if (tid < nx) C.y[cur][C.ncell + tid] = sh.yp[tid];
    if (tid == 0) {
      out[0] = steps;
      out[1] = attempts;
      out[2] = sh.lost ? 2 : status == 3 ? 3 : attempts >= max_attempts ? 1 : 0;
      out[3] = passes;
      double tt[2] = {t, new_h};
      memcpy(&out[4], tt, sizeof(tt));
      out[6] = cur;
      out[7] = iv;
    }
  }
}

template <typename V>
__global__ void __launch_bounds__(TB_THREADS, 1)
    rk4_tb_kernel(const TChip *__restrict__ chips, const int4 *__restrict__ work, const int *__restrict__ wptr,
                  long long *__restrict__ out, double T, int K, const double *__restrict__ bpow, long long nbtot,
                  long long max_attempts) {
  extern __shared__ __align__(16) unsigned char tdyn_raw[];
  V *tdyn = reinterpret_cast<V *>(tdyn_raw);
  __shared__ TSh<V> sh;
  if (threadIdx.x == 0) {
    sh.lost = 0;
    // first-attempt coefficients for h = 1 (they scale with h), computed once
    // per process by the first launch and read back by later ones
    for (int q = 0; q < PMAX; q++) sh.ps[q] = 1.0;
    c_one(sh.K);
    if (*(volatile int *)&g_tb_first_ready) {
      __threadfence();
      c_copy(sh.E1, g_tb_first[0]);
      c_copy(sh.D1, g_tb_first[1]);
      c_copy(sh.F11, g_tb_first[2]);
    } else {
      kry_plan(sh.E, sh.D, sh.F1, sh.K, sh.ps, 1.0, 0);
      c_copy(sh.E1, sh.E);
      c_copy(sh.D1, sh.D);
      c_copy(sh.F11, sh.F1);
      if (blockIdx.x == 0) {
        c_copy(g_tb_first[0], sh.E1);
        c_copy(g_tb_first[1], sh.D1);
        c_copy(g_tb_first[2], sh.F11);
        __threadfence();
        atomicExch(&g_tb_first_ready, 1);
      }
    }
  }
  __syncthreads();
  const int w0 = work ? wptr[blockIdx.x] : 0, w1 = work ? wptr[blockIdx.x + 1] : 1;
  for (int wi = w0; wi < w1 && !sh.lost; wi++) {
    const int4 it = work ? work[wi] : make_int4(0, (int)blockIdx.x, (int)gridDim.x, 0);
    const TChip &C = chips[it.x];
    long long *o = out + (long long)it.x * TB_OUT;
    switch (C.nl) {
#define TB_CASE(n) \
  case n: tb_chip<V, n>(C, it.y, it.z, o, sh, tdyn, T, K, bpow, nbtot, it.w, max_attempts); break;
      TB_CASE(3) TB_CASE(4) TB_CASE(5) TB_CASE(6) TB_CASE(7) TB_CASE(8) TB_CASE(9) TB_CASE(10) TB_CASE(11)
      TB_CASE(12)
#undef TB_CASE
      default: break;
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// the edge-response table ER[j][e'][e] = sum over edge e of (L_cc^j L_cp
// u_{e'}), FP64, from the model's FP64 layer coefficients
// ---------------------------------------------------------------------------
__global__ void tb_er_seed(const TLayerD *__restrict__ L, int nl, int nr, int nc, int layer, int side,
                           double *__restrict__ u) {
  const long long n = (long long)nl * nr * nc;
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    const int l = (int)(k / ((long long)nr * nc));
    const long long rem = k - (long long)l * nr * nc;
    const int i = (int)(rem / nc), j = (int)(rem - (long long)i * nc);
    double v = 0.0;
    if (l == layer) {
      const bool on = side == 0 ? i == 0 : side == 1 ? i == nr - 1 : side == 2 ? j == 0 : j == nc - 1;
      if (on) v = (side < 2 ? L[l].gEdgeNS : L[l].gEdgeEW) * L[l].invC;
    }
    u[k] = v;
  }
}

__global__ void tb_er_apply(const TLayerD *__restrict__ L, int nl, int nr, int nc, const double *__restrict__ u,
                            double *__restrict__ v) {
  const long long plane = (long long)nr * nc, n = (long long)nl * plane;
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    const int l = (int)(k / plane);
    const long long rem = k - (long long)l * plane;
    const int i = (int)(rem / nc), j = (int)(rem - (long long)i * nc);
    const double x = u[k];
    const TLayerD &Q = L[l];
    double s = 0.0;
    if (i > 0) s += Q.gNS * (u[k - nc] - x);
    if (i < nr - 1) s += Q.gNS * (u[k + nc] - x);
    if (j < nc - 1) s += Q.gEW * (u[k + 1] - x);
    if (j > 0) s += Q.gEW * (u[k - 1] - x);
    if (l > 0) s += L[l - 1].gDn * (u[k - plane] - x);
    if (l < nl - 1) s += Q.gDn * (u[k + plane] - x);
    s -= Q.gAmb * x;
    if (Q.nbase >= 0) {
      if (i == 0) s -= Q.gEdgeNS * x;
      if (i == nr - 1) s -= Q.gEdgeNS * x;
      if (j == nc - 1) s -= Q.gEdgeEW * x;
      if (j == 0) s -= Q.gEdgeEW * x;
    }
    v[k] = s * Q.invC;
  }
}

// block e: the sum over edge e (fixed-order tree)
__global__ void tb_er_sums(const double *__restrict__ u, int nr, int nc, const int *__restrict__ eg_layer, int ne,
                           double *__restrict__ row) {
  __shared__ double red[256];
  const int e = blockIdx.x;
  if (e >= ne) return;
  const int side = e & 3, layer = eg_layer[e >> 2];
  const long long plane = (long long)nr * nc;
  const int cnt = side < 2 ? nc : nr;
  double s = 0.0;
  for (int k = threadIdx.x; k < cnt; k += blockDim.x) {
    const int i = side == 0 ? 0 : side == 1 ? nr - 1 : k;
    const int j = side < 2 ? k : side == 2 ? 0 : nc - 1;
    s += u[(long long)layer * plane + (long long)i * nc + j];
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) row[e] = red[0];
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------

static int edge_group(int kind) {
  switch (kind) {
    case LK_SINK: return 0;
    case LK_SPREADER: return 1;
    case LK_PCB: return 2;
    case LK_SOLDER: return 3;
    case LK_SUB: return 4;
    default: return -1;
  }
}
static int group_node_base(int g) {
  return g == 0 ? HSB_SINK_C_W : g == 1 ? HSB_SP_W : g == 2 ? HSB_PCB_C_W : g == 3 ? HSB_SOLDER_W : HSB_SUB_W;
}

// per-layer conductances, a layer count the kernel is compiled for, and a
// layer for every package group whose edges couple to cells
bool tb_eligible(const hsb_dev_model *m) {
  if (m->field || m->uchan_mask || m->nl < TB_NLMIN || m->nl > TB_NLMAX) return false;
  int have[5] = {0, 0, 0, 0, 0};
  for (int l = 0; l < m->nl; l++) {
    const int g = edge_group(m->hostL0[l].kind);
    if (g >= 0) have[g]++;
  }
  const int groups = m->nx > HSB_EXTRA ? 5 : 2;
  for (int g = 0; g < groups; g++)
    if (have[g] != 1) return false;
  return true;
}

// static shared memory of the kernel variant as compiled (the shared state
// plus the shared arrays of its device functions)
size_t tb_static_smem(bool fp64) {
  static size_t have[2] = {0, 0};
  static std::once_flag once[2];
  const int v = fp64 ? 1 : 0;
  std::call_once(once[v], [v] {
    cudaFuncAttributes a;
    const void *fn = v ? (const void *)rk4_tb_kernel<double> : (const void *)rk4_tb_kernel<float>;
    if (cudaFuncGetAttributes(&a, fn) == cudaSuccess) have[v] = a.sharedSizeBytes;
    else {
      cudaGetLastError();
      have[v] = v ? sizeof(TSh<double>) + 1024 : sizeof(TSh<float>) + 1024;
    }
  });
  return have[v];
}

const void *tb_kernel(bool fp64) {
  return fp64 ? (const void *)rk4_tb_kernel<double> : (const void *)rk4_tb_kernel<float>;
}

// layer tables (FP32 for the kernel, FP64 for the edge-response table)
static void tb_tables(const hsb_dev_model *m, TLayer *Lf, TLayerD *Ld, int eg_layer[5], int eg_node[5], int *ne) {
  for (int g = 0; g < 5; g++) {
    eg_layer[g] = -1;
    eg_node[g] = group_node_base(g);
  }
  for (int l = 0; l < m->nl; l++) {
    const LayerCoef &c = m->hostL0[l];
    const int g = edge_group(c.kind);
    const bool amb = c.kind == LK_SINK || c.kind == LK_PCB;
    Ld[l].gNS = 1.0 / c.rNS;
    Ld[l].gEW = 1.0 / c.rEW;
    Ld[l].gDn = 1.0 / c.rz;
    Ld[l].invC = c.cap != 0.0 ? 1.0 / c.cap : 0.0;
    Ld[l].gEdgeNS = g >= 0 && c.edgeNS != 0.0 ? 1.0 / c.edgeNS : 0.0;
    Ld[l].gEdgeEW = g >= 0 && c.edgeEW != 0.0 ? 1.0 / c.edgeEW : 0.0;
    Ld[l].gAmb = amb && c.ramb != 0.0 ? 1.0 / c.ramb : 0.0;
    Ld[l].nbase = g >= 0 ? group_node_base(g) : -1;
    Lf[l].gNS = (float)(1.0 / c.rNS);
    Lf[l].gEW = (float)(1.0 / c.rEW);
    Lf[l].gDn = (float)(1.0 / c.rz);
    Lf[l].invC = c.cap != 0.0 ? (float)(1.0 / c.cap) : 0.f;
    Lf[l].gEdgeNS = g >= 0 && c.edgeNS != 0.0 ? (float)(1.0 / c.edgeNS) : 0.f;
    Lf[l].gEdgeEW = g >= 0 && c.edgeEW != 0.0 ? (float)(1.0 / c.edgeEW) : 0.f;
    Lf[l].gAmb = amb && c.ramb != 0.0 ? (float)(1.0 / c.ramb) : 0.f;
    Lf[l].nbase = g >= 0 ? group_node_base(g) : -1;
    if (g >= 0) eg_layer[g] = l;
  }
  *ne = m->nx > HSB_EXTRA ? NEDGE : 8;
}

// the edge-response table of a model (FP64, on the model's stream)
static int tb_edge_response(hsb_dev_model *m, const TLayerD *Ld_host, const int eg_layer[5], int ne, double *d_er) {
  const long long n = m->ncell;
  double *u = nullptr, *v = nullptr, *row = nullptr;
  TLayerD *dL = nullptr;
  int *deg = nullptr;
  int rc = HSB_OK;
  auto fail = [&](int code) {
    if (u) cudaFree(u);
    if (v) cudaFree(v);
    if (row) cudaFree(row);
    if (dL) cudaFree(dL);
    if (deg) cudaFree(deg);
    return code;
  };
  if (cudaMalloc(&u, sizeof(double) * n) != cudaSuccess || cudaMalloc(&v, sizeof(double) * n) != cudaSuccess ||
      cudaMalloc(&dL, sizeof(TLayerD) * m->nl) != cudaSuccess || cudaMalloc(&deg, sizeof(int) * 5) != cudaSuccess)
    return fail(set_error(HSB_E_NOMEM, "edge-response workspace"));
  if (cudaMemcpyAsync(dL, Ld_host, sizeof(TLayerD) * m->nl, cudaMemcpyHostToDevice, m->stream) != cudaSuccess ||
      cudaMemcpyAsync(deg, eg_layer, sizeof(int) * 5, cudaMemcpyHostToDevice, m->stream) != cudaSuccess)
    return fail(set_error(HSB_E_CUDA, "edge-response tables"));
  const int T = 256;
  const unsigned B = (unsigned)std::min<long long>((n + T - 1) / T, 148 * 16);
  for (int ep = 0; ep < ne; ep++) {
    const int layer = eg_layer[ep >> 2];
    tb_er_seed<<<B, T, 0, m->stream>>>(dL, m->nl, m->nr, m->nc, layer, ep & 3, u);
    for (int j = 0; j < TB_JMAX; j++) {
      tb_er_sums<<<ne, 256, 0, m->stream>>>(u, m->nr, m->nc, deg, ne, d_er + ((long long)j * ne + ep) * ne);
      if (j + 1 < TB_JMAX) {
        tb_er_apply<<<B, T, 0, m->stream>>>(dL, m->nl, m->nr, m->nc, u, v);
        std::swap(u, v);
      }
    }
  }
  if (cudaGetLastError() != cudaSuccess) rc = set_error(HSB_E_CUDA, "edge-response kernels");
  if (cudaStreamSynchronize(m->stream) != cudaSuccess) rc = set_error(HSB_E_CUDA, "edge-response kernels");
  fail(0);
  return rc;
}

// work of one own tile in a first attempt (halo 8, eight passes), in cells
// per layer: the state box it loads plus the shrinking rectangle of each pass
double tb_tile_work(int oi, int oj) {
  double w = (double)(oi + 16) * (oj + 16);
  for (int m = 0; m < 8; m++) w += (double)(oi + 14 - 2 * m) * (oj + 14 - 2 * m);
  return w;
}

// region cells per layer of one buffer for an own tile: every cell the
// shared memory of a CTA holds (at least the first attempt's box, halo 8),
// so that a retry's larger halo (12, 16, ... after one, two, ... rejections)
// still finds a sub-tile
int tb_rcap(int nl, int oi, int oj, bool fp64, size_t smem_cap) {
  const int base = (oi + 16) * (oj + 16);
  const long long fit =
      ((long long)smem_cap - (long long)tb_static_smem(fp64)) / (2LL * nl * (fp64 ? 8 : 4));
  return (int)(fit > base ? fit : base);
}

// own-tile shape for a model with `ctas` co-resident CTAs: among the
// candidates whose two region buffers fit next to the static shared memory,
// the one with the least work for the busiest CTA (tiles dealt round-robin)
int tb_tile_for(int nl, int nr, int nc, int ctas, size_t smem_cap, int *oi, int *oj, bool fp64) {
  static const int cand[][2] = {{16, 64}, {32, 32}, {16, 32}, {8, 64}, {8, 32}, {8, 16}};
  int best = -1;
  double best_cost = 0.0;
  for (int k = 0; k < 6; k++) {
    const size_t rc = (size_t)tb_rcap(nl, cand[k][0], cand[k][1], fp64, smem_cap);
    if (2 * rc * nl * (fp64 ? 8 : 4) + tb_static_smem(fp64) > smem_cap) continue;
    if (cand[k][0] * cand[k][1] > TB_THREADS * tb_slots_rt(fp64, nl)) continue;
    const long long tiles = (long long)((nr + cand[k][0] - 1) / cand[k][0]) * ((nc + cand[k][1] - 1) / cand[k][1]);
    const double cost = (double)((tiles + ctas - 1) / ctas) * tb_tile_work(cand[k][0], cand[k][1]);
    if (best < 0 || cost < best_cost) {
      best = k;
      best_cost = cost;
    }
  }
  if (best < 0) return set_error(HSB_E_ARG, "no tile of the temporally blocked transient fits shared memory");
  *oi = cand[best][0];
  *oj = cand[best][1];
  return HSB_OK;
}

size_t tb_dyn_smem(int nl, int oi, int oj, bool fp64, size_t smem_cap) {
  return (size_t)2 * tb_rcap(nl, oi, oj, fp64, smem_cap) * nl * (fp64 ? 8 : 4);
}

int tb_fill_chip(hsb_dev_model *m, TbRes *r, const double *y0, const double *y1, float *pf, double *pd, int oi,
                 int oj, bool fp64, size_t smem_cap, TChip *C) {
  memset(C, 0, sizeof(*C));
  C->y[0] = const_cast<double *>(y0);
  C->y[1] = const_cast<double *>(y1);
  C->pf = pf;
  C->pd = pd;
  C->pgrid = m->pgrid;
  C->b2g_ptr = m->b2g_ptr;
  C->b2g_blk = m->b2g_blk;
  C->b2g_occ = m->b2g_occ;
  C->b2g_area = m->b2g_area;
  C->cell_area = m->cell_area;
  C->L = r->L;
  C->Ld = r->Ld;
  C->pk = r->pk;
  C->er = r->er;
  C->part = r->part;
  C->ea = r->ea;
  C->err = r->err;
  C->bar = r->bar;
  C->ncell = m->ncell;
  C->plane = m->plane;
  C->ambient = m->ambient;
  C->nl = m->nl;
  C->nr = m->nr;
  C->nc = m->nc;
  C->nx = m->nx;
  C->ne = r->ne;
  for (int g = 0; g < 5; g++) {
    C->eg_layer[g] = r->eg_layer[g];
    C->eg_node[g] = r->eg_node[g];
  }
  C->oi = oi;
  C->oj = oj;
  C->nti = (m->nr + oi - 1) / oi;
  C->ntj = (m->nc + oj - 1) / oj;
  C->ntiles = C->nti * C->ntj;
  C->segmax = r->segmax;
  C->rcap = tb_rcap(m->nl, oi, oj, fp64, smem_cap);
  if (C->nti > r->segmax || C->ntj > r->segmax) return set_error(HSB_E_ARG, "tile grid exceeds the edge partials");
  return HSB_OK;
}

void tb_res_free(TbRes *r) {
  if (!r) return;
  void *d[] = {r->L, r->Ld, r->part, r->ea, r->err, r->bar, r->d_chip};   // pk is the fast workspace's; er the cache's
  for (void *p : d)
    if (p) cudaFree(p);
  delete r;
}

// Edge-response tables depend only on the grid's shape and its FP64 layer
// coefficients, so models of the same stack and grid share one table.  The
// cache keeps every table it computed until the process exits (about 58 KB
// each at most).
namespace {
struct ErEntry {
  int device, nl, nr, nc, ne;
  std::vector<double> coef;
  double *er;
};
std::mutex g_er_mu;
std::vector<ErEntry> g_er_cache;
}  // namespace

// per-model resources of the kernel: tables, edge-response table, partials
int tb_res_prepare(hsb_dev_model *m, TbRes **out, const PackF *pk_dev) {
  TbRes *r = *out;
  if (!r) {
    r = new TbRes();
    memset(r, 0, sizeof(*r));
    r->version = -1;
    *out = r;
    // partial edge sums per own tile along each edge: the smallest tile is 8 wide
    r->segmax = (std::max(m->nr, m->nc) + 7) / 8;
    HSB_CUDA(cudaMalloc(&r->L, sizeof(TLayer) * TB_NLMAX));
    HSB_CUDA(cudaMalloc(&r->Ld, sizeof(TLayerD) * TB_NLMAX));
    HSB_CUDA(cudaMalloc(&r->part, sizeof(double) * (TB_DMAX + 1) * NEDGE * r->segmax));
    HSB_CUDA(cudaMalloc(&r->ea, sizeof(double) * m->ncell));
    HSB_CUDA(cudaMalloc(&r->err, sizeof(unsigned long long) * 4));
    HSB_CUDA(cudaMalloc(&r->bar, sizeof(unsigned) * 2));
    HSB_CUDA(cudaMemsetAsync(r->bar, 0, sizeof(unsigned) * 2, m->stream));
    HSB_CUDA(cudaMalloc(&r->d_chip, sizeof(TChip) * 4));
  }
  r->pk = const_cast<PackF *>(pk_dev);
  if (r->version == m->coef_version) return HSB_OK;
  TLayer Lf[TB_NLMAX];
  TLayerD Ld[TB_NLMAX];
  memset(Lf, 0, sizeof(Lf));
  memset(Ld, 0, sizeof(Ld));
  tb_tables(m, Lf, Ld, r->eg_layer, r->eg_node, &r->ne);
  HSB_CUDA(cudaMemcpyAsync(r->L, Lf, sizeof(TLayer) * m->nl, cudaMemcpyHostToDevice, m->stream));
  HSB_CUDA(cudaMemcpyAsync(r->Ld, Ld, sizeof(TLayerD) * m->nl, cudaMemcpyHostToDevice, m->stream));
  // the edge-response table: from the cache, or computed and added to it
  std::vector<double> coef;
  for (int l = 0; l < m->nl; l++) {
    const double v[8] = {Ld[l].gNS, Ld[l].gEW, Ld[l].gDn, Ld[l].invC, Ld[l].gEdgeNS, Ld[l].gEdgeEW, Ld[l].gAmb,
                         (double)Ld[l].nbase};
    coef.insert(coef.end(), v, v + 8);
  }
  for (int g = 0; g < 5; g++) coef.push_back((double)r->eg_layer[g]);
  std::lock_guard<std::mutex> lk(g_er_mu);
  for (const ErEntry &e : g_er_cache)
    if (e.device == m->device && e.nl == m->nl && e.nr == m->nr && e.nc == m->nc && e.ne == r->ne &&
        e.coef == coef) {
      r->er = e.er;
      r->version = m->coef_version;
      return HSB_OK;
    }
  double *er = nullptr;
  HSB_CUDA(cudaMalloc(&er, sizeof(double) * TB_JMAX * NEDGE * NEDGE));
  int rc;
  if ((rc = tb_edge_response(m, Ld, r->eg_layer, r->ne, er))) {
    cudaFree(er);
    return rc;
  }
  g_er_cache.push_back({m->device, m->nl, m->nr, m->nc, r->ne, coef, er});
  r->er = er;
  r->version = m->coef_version;
  return HSB_OK;
}

}  // namespace hsb
