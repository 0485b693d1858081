// solvers_fast.cu -- steady state of non-symmetric models (HSB_STEADY_BICGSTAB).
//
// Microchannel layers make the steady system G T = P non-symmetric: the
// reference assembles the advection between fluid cells as +-Cv*flow/2
// off-diagonal terms (build_transient_grid_matrix, temperature_grid.c:
// 5347-5387, the same terms slope_fn_grid uses, :3256-3309) and can only
// solve that system with SuperLU (direct_SLU, :5130-5194).  Here it is
// solved to FP64 accuracy by iterative refinement:
//
//   outer loop (FP64):  r = P - G T;  solve G e = r approximately;  T += e
//   inner solver (FP32): BiCGStab, right-preconditioned by one V-cycle
//
// The flow in the channels dominates conduction by two to three orders of
// magnitude (cell Peclet numbers 10^2..10^3 at 1-10 mL/min), so point or
// z-line smoothers and 2x2 coarsening do not converge on it.  The V-cycle is
// therefore built around the flow direction:
//   * smoother: red-black PLANE Gauss-Seidel over the j index -- every plane
//     of fixed j (all rows i and all layers n, i.e. whole channels together
//     with the silicon above and the spreader/sink below them) is solved
//     exactly with a banded LU factorised once per model (bandwidth = the
//     number of layers), then the 12 package nodes are solved exactly;
//   * coarsening in j only (semi-coarsening): coarse operators are the
//     Galerkin sums over pairs of planes, with the coupling between planes
//     halved (and the diagonal adjusted so rows keep their sums), which is
//     the conductance of a cell twice as wide.
// The plane matrices are positive real (their symmetric part is the
// conduction operator plus the non-negative inlet/outlet diagonal), so the
// LU exists without pivoting; it is computed in FP64 and stored in FP32.
#include <cmath>
#include <cstring>
#include <vector>

#include "dev_model.cuh"

namespace hsb {

#define BCT 256
#define BNX 12          // package nodes of the primary heat path
#define BC_MAX_NL 12    // layers supported by the plane solver

struct BcPack {                 // the package nodes' equations (level 0, FP64)
  double link[BNX][BNX];        // conductance between package nodes
  double gamb[BNX];             // conductance to ambient
  double ge0[BNX];              // per-cell conductance to the attached edge cells
  int elayer[BNX], eside[BNX];  // attached edge: layer, side (0 N, 1 S, 2 W, 3 E); -1 none
};

struct BcLevelDev {
  const float *pinv;                               // 12 x 12 inverse of the package block
  int nl, nr, nc;
  long long plane, ncell;
  const float *cN, *cS, *cW, *cE, *cA, *cB, *dg;   // A[c, neighbour] and A[c, c]
  const float *rs;                                 // row sums without the package edges
  const float *LF, *UB;                            // plane LU factors (plane storage)
  float geNS[BC_MAX_NL], geEW[BC_MAX_NL];          // cell <-> package edge conductance per layer
  float escNS;                                     // N/S package rows: edge conductance scale 2^k
  int spidx, hsidx;
};

struct BcLevel {
  int nc;
  long long plane, ncell, n;
  float *cN, *cS, *cW, *cE, *cA, *cB, *dg, *rs;
  float *LF, *UB;              // plane LU factors (plane storage)
  float *x, *f, *r;
  float *pr, *py;              // plane right-hand sides and forward-pass values (plane storage)
  float *pinv;                 // 12 x 12 inverse of the package block at this level
};

struct BcWork {
  int nlev, coef_version;
  std::vector<BcLevel> lv;
  BcPack pk;
  BcPack *d_pk;
  double geNS0[BC_MAX_NL], geEW0[BC_MAX_NL];
  double *c64;                 // 8 x ncell: cN cS cW cE cA cB dg rs (FP64, level 0)
  double *b64, *r64;           // right-hand side, residual (vlen)
  double *band;                // FP64 band scratch of the factorisation
  // BiCGStab vectors (level 0, FP32, n = ncell + 12)
  float *r, *rh, *p, *v, *s, *t, *ph, *sh, *e;
  double *red;                 // reductions and scalars
  double *h_red;
  // one refinement pass (FP64 residual, inner BiCGStab, correction) as a graph
  int R, tpb;                  // rows per streamed chunk, planes (threads) per CTA of the plane solve
  int *status;                 // raised by a plane solve whose chunk copy did not arrive
  cudaGraphExec_t pass_exec;
  const double *pass_T;        // the state buffer the graph was captured for
  long long pass_launches;
};

__device__ __forceinline__ int bc_edge_node(int layer, int side, int spidx, int hsidx) {
  if (layer == hsidx) return side == 0 ? HSB_SINK_C_N : side == 1 ? HSB_SINK_C_S : side == 2 ? HSB_SINK_C_W : HSB_SINK_C_E;
  if (layer == spidx) return side == 0 ? HSB_SP_N : side == 1 ? HSB_SP_S : side == 2 ? HSB_SP_W : HSB_SP_E;
  return -1;
}

// ---------------------------------------------------------------------------
// level-0 operator in FP64 (the reference's steady system with advection)
// ---------------------------------------------------------------------------
// A[c, nbr] = -1/R(nbr, c) - a(nbr->c)/2 for the four lateral neighbours,
// -1/R for the vertical ones; A[c, c] = sum 1/R - (aN+aS+aW+aE)/2 - aO + edge
// and ambient conductances; b = P + qin + ambient terms
// (temperature_grid.c:5347-5387 and 6524-6694).
__global__ void bc_build64(const StencilArgs S, const double *__restrict__ pgrid, const double *__restrict__ geNS,
                           const double *__restrict__ geEW, double *__restrict__ c64, double *__restrict__ b64,
                           const double *__restrict__ gamb_pk) {
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= S.ncell) {
    if (c < S.ncell + S.nx) b64[c] = gamb_pk[c - S.ncell] * S.ambient;
    return;
  }
  const long long N = S.ncell;
  const int n = (int)(c / S.plane);
  const long long q = c - n * S.plane;
  const int i = (int)(q / S.nc), j = (int)(q - (long long)i * S.nc);
  const LayerCoef &L = S.L[n];
  double gN = 0, gS = 0, gW = 0, gE = 0, gA = 0, gB = 0;
  if (S.field) {
    if (i > 0) gN = 1.0 / S.rN[c];
    if (i < S.nr - 1) gS = 1.0 / S.rS[c];
    if (j > 0) gW = 1.0 / S.rW[c];
    if (j < S.nc - 1) gE = 1.0 / S.rE[c];
    if (n > 0) gA = 1.0 / S.rA[c];
    if (n < S.nl - 1) gB = 1.0 / S.rB[c];
  } else {
    if (i > 0) gN = 1.0 / L.rNS;
    if (i < S.nr - 1) gS = 1.0 / L.rNS;
    if (j > 0) gW = 1.0 / L.rEW;
    if (j < S.nc - 1) gE = 1.0 / L.rEW;
    if (n > 0) gA = 1.0 / S.L[n - 1].rz;
    if (n < S.nl - 1) gB = 1.0 / L.rz;
  }
  double aN = 0, aS = 0, aW = 0, aE = 0, aO = 0, qin = 0;
  if ((S.uchan_mask >> n) & 1ull) {
    aN = S.aN[c]; aS = S.aS[c]; aW = S.aW[c]; aE = S.aE[c]; aO = S.aO[c]; qin = S.qin[c];
  }
  double dg = gN + gS + gW + gE + gA + gB - (aN + aS + aW + aE) / 2.0 - aO;
  double b = pgrid[c] + qin;
  if (L.kind == LK_SPREADER || L.kind == LK_SINK) {
    if (i == 0) dg += geNS[n];
    if (i == S.nr - 1) dg += geNS[n];
    if (j == 0) dg += geEW[n];
    if (j == S.nc - 1) dg += geEW[n];
  }
  if (L.kind == LK_SINK) {
    dg += 1.0 / L.ramb;
    b += S.ambient / L.ramb;
  }
  c64[0 * N + c] = i > 0 ? -gN - aN / 2.0 : 0.0;
  c64[1 * N + c] = i < S.nr - 1 ? -gS - aS / 2.0 : 0.0;
  c64[2 * N + c] = j > 0 ? -gW - aW / 2.0 : 0.0;
  c64[3 * N + c] = j < S.nc - 1 ? -gE - aE / 2.0 : 0.0;
  c64[4 * N + c] = n > 0 ? -gA : 0.0;
  c64[5 * N + c] = n < S.nl - 1 ? -gB : 0.0;
  c64[6 * N + c] = dg;
  // row sum without the package edges: the coefficient of x itself in the
  // difference form rs x + sum(-c)(x - x_nbr) + ge (x - x_pk)
  double edges = 0.0;
  if (L.kind == LK_SPREADER || L.kind == LK_SINK)
    edges = (i == 0 ? geNS[n] : 0.0) + (i == S.nr - 1 ? geNS[n] : 0.0) + (j == 0 ? geEW[n] : 0.0) +
            (j == S.nc - 1 ? geEW[n] : 0.0);
  c64[7 * N + c] = dg + c64[0 * N + c] + c64[1 * N + c] + c64[2 * N + c] + c64[3 * N + c] + c64[4 * N + c] +
                   c64[5 * N + c] - edges;
  b64[c] = b;
}

__global__ void bc_to32(const double *__restrict__ a, float *__restrict__ b, long long n) {
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) b[k] = (float)a[k];
}

// FP64 residual of the cells: r = b - A T; max |r| into maxbits; FP32 copy
__global__ void bc_residual64(const StencilArgs S, const double *__restrict__ c64, const double *__restrict__ geNS,
                              const double *__restrict__ geEW, const double *__restrict__ T,
                              const double *__restrict__ b, double *__restrict__ r, float *__restrict__ r32,
                              unsigned long long *maxbits) {
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  double res = 0.0;
  if (c < S.ncell) {
    const long long N = S.ncell;
    const int n = (int)(c / S.plane);
    const long long q = c - n * S.plane;
    const int i = (int)(q / S.nc), j = (int)(q - (long long)i * S.nc);
    double s = c64[6 * N + c] * T[c];
    if (i > 0) s += c64[0 * N + c] * T[c - S.nc];
    if (i < S.nr - 1) s += c64[1 * N + c] * T[c + S.nc];
    if (j > 0) s += c64[2 * N + c] * T[c - 1];
    if (j < S.nc - 1) s += c64[3 * N + c] * T[c + 1];
    if (n > 0) s += c64[4 * N + c] * T[c - S.plane];
    if (n < S.nl - 1) s += c64[5 * N + c] * T[c + S.plane];
    const LayerCoef &L = S.L[n];
    if (L.kind == LK_SPREADER || L.kind == LK_SINK) {
      const double *x = T + N;
      const bool sp = L.kind == LK_SPREADER;
      if (i == 0) s -= geNS[n] * x[sp ? HSB_SP_N : HSB_SINK_C_N];
      if (i == S.nr - 1) s -= geNS[n] * x[sp ? HSB_SP_S : HSB_SINK_C_S];
      if (j == 0) s -= geEW[n] * x[sp ? HSB_SP_W : HSB_SINK_C_W];
      if (j == S.nc - 1) s -= geEW[n] * x[sp ? HSB_SP_E : HSB_SINK_C_E];
    }
    res = b[c] - s;
    r[c] = res;
    r32[c] = (float)res;
  }
  res = fabs(res);
  for (int o = 16; o > 0; o >>= 1) res = fmax(res, __shfl_down_sync(0xffffffffu, res, o));
  if ((threadIdx.x & 31) == 0) atomicMax(maxbits, (unsigned long long)__double_as_longlong(res));
}

// FP64 residual of the package rows (one CTA)
__global__ void bc_pack_residual64(const StencilArgs S, const BcPack *__restrict__ pk, const double *__restrict__ T,
                                   const double *__restrict__ b, double *__restrict__ r, float *__restrict__ r32,
                                   unsigned long long *maxbits) {
  __shared__ double esum[BNX];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int k = w; k < BNX; k += blockDim.x >> 5) {
    double s = 0.0;
    const int layer = pk->elayer[k], side = pk->eside[k];
    if (layer >= 0) {
      const int len = side < 2 ? S.nc : S.nr;
      const long long base = (long long)layer * S.plane +
                             (side == 0 ? 0 : side == 1 ? (long long)(S.nr - 1) * S.nc : side == 2 ? 0 : S.nc - 1);
      const long long st = side < 2 ? 1 : S.nc;
      for (int q = lane; q < len; q += 32) s += T[S.ncell + k] - T[base + q * st];
      for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    }
    if (lane == 0) esum[k] = s;
  }
  __syncthreads();
  if (threadIdx.x < BNX) {
    const int k = threadIdx.x;
    const double *x = T + S.ncell;
    double s = pk->ge0[k] * esum[k] + pk->gamb[k] * x[k];
    for (int o = 0; o < BNX; o++) s += pk->link[k][o] * (x[k] - x[o]);
    const double res = b[S.ncell + k] - s;
    r[S.ncell + k] = res;
    r32[S.ncell + k] = (float)res;
    atomicMax(maxbits, (unsigned long long)__double_as_longlong(fabs(res)));
  }
}

// ---------------------------------------------------------------------------
// FP32 levels: coarsening in j, plane factorisation, smoother, transfers
// ---------------------------------------------------------------------------
// coarse cell (n, i, J) from the fine cells (n, i, 2J) and (n, i, 2J+1)
__global__ void bc_coarsen(BcLevelDev F, float *cN, float *cS, float *cW, float *cE, float *cA, float *cB,
                           float *dg, float *rs, int cnc) {
  const long long cpl = (long long)F.nr * cnc;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= cpl * F.nl) return;
  const int n = (int)(t / cpl);
  const long long r = t - n * cpl;
  const int i = (int)(r / cnc), J = (int)(r - (long long)i * cnc);
  const long long a = (long long)n * F.plane + (long long)i * F.nc + 2 * J, b = a + 1;
  cN[t] = F.cN[a] + F.cN[b];
  cS[t] = F.cS[a] + F.cS[b];
  cA[t] = F.cA[a] + F.cA[b];
  cB[t] = F.cB[a] + F.cB[b];
  const float wg = F.cW[a], eg = F.cE[b];
  cW[t] = 0.5f * wg;
  cE[t] = 0.5f * eg;
  dg[t] = F.dg[a] + F.dg[b] + F.cE[a] + F.cW[b] + 0.5f * wg + 0.5f * eg;
  rs[t] = F.rs[a] + F.rs[b];   // the pair's row sums (the halving keeps them)
}

// Plane storage: plane j sits in slot (j & 1) * half + (j >> 1), half =
// (nc + 1) / 2, so the planes of one colour are consecutive; every plane's
// data is contiguous and its records are padded to 16 bytes, so one thread
// can stream its plane through shared memory with bulk copies and read it
// back with 128-bit loads.  With VP = LFP = round4(nl), UBP = round4(nl+1):
//   LF[(slot*nq + q)*LFP + m-1]      = L(q, q-m)                 m = 1..nl
//   UB[(slot*nq + q)*UBP + m-1]      = U(q, q+m),  UB[.. + nl] = 1 / U(q, q)
//   right-hand sides, forward values: [(slot*nr + i)*VP + n]
__host__ __device__ __forceinline__ int bc_r4(int v) { return (v + 3) & ~3; }
__device__ __forceinline__ int bc_slot(int j, int nc) { return (j & 1) * ((nc + 1) / 2) + (j >> 1); }

// banded LU (no pivoting) of every plane j: band entry (q, q+d) at
// band[(q*(2nl+1) + d+nl) * nc + slot], FP64 in place; factors out in FP32
__global__ void bc_factor(BcLevelDev L, double *__restrict__ band, float *__restrict__ LF, float *__restrict__ UB) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= L.nc) return;
  const int nl = L.nl, W = 2 * nl + 1;
  const int nq = L.nr * nl;
  const long long np = L.nc;
  const int slot = bc_slot(j, L.nc);
  const int LFP = bc_r4(nl), UBP = bc_r4(nl + 1);
  auto B = [&](int q, int d) -> double & { return band[((long long)q * W + d + nl) * np + slot]; };
  for (int q = 0; q < nq; q++) {
    for (int d = -nl; d <= nl; d++) B(q, d) = 0.0;
    const int i = q / nl, n = q - i * nl;
    const long long c = (long long)n * L.plane + (long long)i * L.nc + j;
    B(q, 0) = L.dg[c];
    if (n > 0) B(q, -1) = L.cA[c];
    if (n < nl - 1) B(q, 1) = L.cB[c];
    if (i > 0) B(q, -nl) = L.cN[c];
    if (i < L.nr - 1) B(q, nl) = L.cS[c];
  }
  for (int p = 0; p < nq; p++) {
    const double piv = B(p, 0);
    const int last = p + nl < nq - 1 ? p + nl : nq - 1;
    for (int r = p + 1; r <= last; r++) {
      const double l = B(r, p - r) / piv;
      B(r, p - r) = l;
      if (l != 0.0)
        for (int c = p + 1; c <= last; c++) B(r, c - r) -= l * B(p, c - p);
    }
  }
  const long long base = (long long)slot * nq;
  for (int q = 0; q < nq; q++) {
    for (int m = 1; m <= LFP; m++) LF[(base + q) * LFP + m - 1] = (m <= nl && q - m >= 0) ? (float)B(q, -m) : 0.f;
    for (int m = 1; m <= UBP; m++) UB[(base + q) * UBP + m - 1] = (m <= nl && q + m < nq) ? (float)B(q, m) : 0.f;
    UB[(base + q) * UBP + nl] = (float)(1.0 / B(q, 0));
  }
}

// right-hand sides of the planes of one colour: prhs = f - (couplings to
// the neighbouring planes and to the package nodes) x, written in plane
// storage through a shared-memory transpose (32 planes x 32 q per CTA)
__global__ void __launch_bounds__(256) bc_plane_rhs(BcLevelDev L, const float *__restrict__ x,
                                                    const float *__restrict__ f, float *__restrict__ prhs, int color) {
  __shared__ float tile[32][33];
  const int half = (L.nc + 1) / 2;
  const int ncol = color ? L.nc / 2 : half;   // planes of this colour
  const int nq = L.nr * L.nl;
  const int k0 = blockIdx.x * 32, q0 = blockIdx.y * 32;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  for (int qq = ty; qq < 32; qq += 8) {
    const int q = q0 + qq, k = k0 + tx;
    if (q < nq && k < ncol) {
      const int j = 2 * k + color;
      const int i = q / L.nl, n = q - i * L.nl;
      const long long c = (long long)n * L.plane + (long long)i * L.nc + j;
      float rhs = f[c];
      if (j > 0) rhs -= L.cW[c] * x[c - 1];
      if (j < L.nc - 1) rhs -= L.cE[c] * x[c + 1];
      if (n == L.spidx || n == L.hsidx) {
        const float *xp = x + L.ncell;
        if (i == 0) rhs += L.geNS[n] * xp[bc_edge_node(n, 0, L.spidx, L.hsidx)];
        if (i == L.nr - 1) rhs += L.geNS[n] * xp[bc_edge_node(n, 1, L.spidx, L.hsidx)];
        if (j == 0) rhs += L.geEW[n] * xp[bc_edge_node(n, 2, L.spidx, L.hsidx)];
        if (j == L.nc - 1) rhs += L.geEW[n] * xp[bc_edge_node(n, 3, L.spidx, L.hsidx)];
      }
      tile[qq][tx] = rhs;
    }
  }
  __syncthreads();
  for (int kk = ty; kk < 32; kk += 8) {
    const int k = k0 + kk, q = q0 + tx;
    if (q < nq && k < ncol) {
      const int i = q / L.nl, n = q - i * L.nl;
      prhs[((long long)(color * half + k) * L.nr + i) * bc_r4(L.nl) + n] = tile[tx][kk];
    }
  }
}

// ---- bulk-copy primitives (one thread, its own mbarriers) -----------------
__device__ __forceinline__ unsigned bc_smem(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void bc_bar_init(unsigned long long *bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(bc_smem(bar)) : "memory");
}
__device__ __forceinline__ void bc_bulk_load(void *dst, const void *src, unsigned bytes, unsigned long long *bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                   bc_smem(dst)),
               "l"(src), "r"(bytes), "r"(bc_smem(bar))
               : "memory");
}
__device__ __forceinline__ void bc_expect(unsigned long long *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bc_smem(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool bc_try_wait(unsigned long long *bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(bc_smem(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ void bc_bulk_store(void *dst, const void *src, unsigned bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;\n" ::"l"(dst), "r"(bc_smem(src)),
               "r"(bytes)
               : "memory");
  asm volatile("cp.async.bulk.commit_group;\n" ::: "memory");
}
__device__ __forceinline__ void bc_store_read_done() { asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory"); }
__device__ __forceinline__ void bc_store_done() { asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory"); }
__device__ __forceinline__ void bc_fence_smem() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

#define BC_WAIT_LIMIT (1 << 22)

#define BC_NB 4   // chunk buffers per plane: three copies in flight while one is computed

// per-thread shared-memory stride (floats): the ring, rounded so that it is
// 4 (mod 32): the 128-bit loads of 8 consecutive threads then hit distinct banks
__host__ __device__ __forceinline__ int bc_thread_stride(int nl, int R) {
  const int mx = bc_r4(nl) > bc_r4(nl + 1) ? bc_r4(nl) : bc_r4(nl + 1);
  const int ring = BC_NB * (R * bc_r4(nl) + R * nl * mx);
  return ring + (((4 - ring) % 32) + 32) % 32;
}

// One half sweep of plane Gauss-Seidel: planes j = 2k + color solve
// A_jj x_j = prhs_j exactly by forward/back substitution with the band
// factors.  Each thread owns one plane and streams it through shared memory
// in chunks of R rows with a ring of BC_NB buffers: the bulk copies of the
// next BC_NB-1 chunks are in flight while one chunk is computed, so the
// recurrence does not wait on global memory.  The forward pass writes y in
// place of the chunk's right-hand sides and stores it with a bulk copy (the
// buffer is refilled one iteration later, once that store has read it); the
// backward pass streams y back the same way.  A chunk that does not arrive
// within BC_WAIT_LIMIT polls raises *status and ends the sweep.
template <int NL>
__global__ void __launch_bounds__(32)
    bc_plane_solve(const float *__restrict__ LF, const float *__restrict__ UB, const float *__restrict__ prhs,
                   float *__restrict__ yb, float *__restrict__ x, int nr, int nc, long long pl, int color, int R,
                   int *status) {
  constexpr int VP = (NL + 3) & ~3, LFP = VP, UBP = (NL + 4) & ~3, MX = LFP > UBP ? LFP : UBP;
  extern __shared__ __align__(128) float bc_dyn[];
  __shared__ __align__(8) unsigned long long bars[32][BC_NB];
  const int half = (nc + 1) / 2;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 2 * k + color;
  const int t = threadIdx.x;
  for (int b = 0; b < BC_NB; b++) bc_bar_init(&bars[t][b]);
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  __syncthreads();
  if (j >= nc) return;
  const int nq = nr * NL, nch = nr / R;
  const long long slot = color * half + k;
  const float *rp = prhs + slot * nr * VP;
  float *yp = yb + slot * nr * VP;
  const float *lp = LF + slot * nq * LFP;
  const float *up = UB + slot * nq * UBP;
  // per-thread ring of BC_NB x [R*VP values][R*NL*MX factors]
  const int BUF = R * VP + R * NL * MX;
  float *const buf0 = bc_dyn + (size_t)t * bc_thread_stride(NL, R);
  auto buf = [&](int b) { return buf0 + b * BUF; };
  unsigned phase = 0u;   // bit b: parity of buffer b's next completion
  bool lost = false;
  auto wait = [&](int b) {
    int it = 0;
    while (!bc_try_wait(&bars[t][b], (phase >> b) & 1u)) {
      if (++it >= BC_WAIT_LIMIT) {
        lost = true;
        return;
      }
    }
    phase ^= 1u << b;
  };
  auto issue_fwd = [&](int c, int b) {
    const unsigned bv = R * VP * 4, bf = R * NL * LFP * 4;
    bc_fence_smem();
    bc_expect(&bars[t][b], bv + bf);
    bc_bulk_load(buf(b), rp + (long long)c * R * VP, bv, &bars[t][b]);
    bc_bulk_load(buf(b) + R * VP, lp + (long long)c * R * NL * LFP, bf, &bars[t][b]);
  };
  auto issue_bwd = [&](int c, int b) {
    const unsigned bv = R * VP * 4, bf = R * NL * UBP * 4;
    bc_fence_smem();
    bc_expect(&bars[t][b], bv + bf);
    bc_bulk_load(buf(b), yp + (long long)c * R * VP, bv, &bars[t][b]);
    bc_bulk_load(buf(b) + R * VP, up + (long long)c * R * NL * UBP, bf, &bars[t][b]);
  };
  // ---- forward: y = L^-1 prhs; chunk c in buffer c % BC_NB ----
  float yprev[NL], ycur[NL];
#pragma unroll
  for (int n = 0; n < NL; n++) yprev[n] = 0.f;
  for (int c = 0; c < BC_NB - 1 && c < nch; c++) issue_fwd(c, c);
  for (int c = 0; c < nch; c++) {
    const int b = c % BC_NB;
    wait(b);
    if (lost) break;
    float *v = buf(b);
    const float *lf = buf(b) + R * VP;
    for (int r = 0; r < R; r++) {
      float rv[VP];
#pragma unroll
      for (int u = 0; u < VP; u += 4) *reinterpret_cast<float4 *>(rv + u) = *reinterpret_cast<const float4 *>(v + r * VP + u);
#pragma unroll
      for (int n = 0; n < NL; n++) {
        float lr[LFP];
#pragma unroll
        for (int u = 0; u < LFP; u += 4)
          *reinterpret_cast<float4 *>(lr + u) = *reinterpret_cast<const float4 *>(lf + (r * NL + n) * LFP + u);
        // oldest values first: the value just computed (m = 1) enters last,
        // so the recurrence waits on one multiply-add per unknown, not NL
        float a = rv[n];
#pragma unroll
        for (int m = NL; m >= 1; m--) a -= lr[m - 1] * (m <= n ? ycur[n - m] : yprev[NL + n - m]);
        ycur[n] = a;
        rv[n] = a;
      }
#pragma unroll
      for (int u = 0; u < VP; u += 4) *reinterpret_cast<float4 *>(v + r * VP + u) = *reinterpret_cast<const float4 *>(rv + u);
#pragma unroll
      for (int n = 0; n < NL; n++) yprev[n] = ycur[n];
    }
    bc_fence_smem();
    bc_bulk_store(yp + (long long)c * R * VP, v, R * VP * 4);
    // refill the previous chunk's buffer: its store (one group back) has read it
    const int cn = c + BC_NB - 1;
    if (cn < nch) {
      asm volatile("cp.async.bulk.wait_group.read 1;\n" ::: "memory");
      issue_fwd(cn, cn % BC_NB);
    }
  }
  bc_store_done();
  // ---- backward: x = U^-1 y; the s-th chunk from the end in buffer s % BC_NB ----
  float xnext[NL], xcur[NL];
#pragma unroll
  for (int n = 0; n < NL; n++) xnext[n] = 0.f;
  if (!lost)
    for (int s = 0; s < BC_NB - 1 && s < nch; s++) issue_bwd(nch - 1 - s, s);
  for (int s = 0; s < nch && !lost; s++) {
    const int c = nch - 1 - s, b = s % BC_NB;
    wait(b);
    if (lost) break;
    const float *v = buf(b);
    const float *ub = buf(b) + R * VP;
    for (int r = R - 1; r >= 0; r--) {
      const int i = c * R + r;
      float yv[VP];
#pragma unroll
      for (int u = 0; u < VP; u += 4) *reinterpret_cast<float4 *>(yv + u) = *reinterpret_cast<const float4 *>(v + r * VP + u);
#pragma unroll
      for (int n = NL - 1; n >= 0; n--) {
        float ur[UBP];
#pragma unroll
        for (int u = 0; u < UBP; u += 4)
          *reinterpret_cast<float4 *>(ur + u) = *reinterpret_cast<const float4 *>(ub + (r * NL + n) * UBP + u);
        float a = yv[n];
#pragma unroll
        for (int m = NL; m >= 1; m--) a -= ur[m - 1] * (n + m < NL ? xcur[n + m] : xnext[n + m - NL]);
        xcur[n] = a * ur[NL];
      }
#pragma unroll
      for (int n = 0; n < NL; n++) {
        x[(long long)n * pl + (long long)i * nc + j] = xcur[n];
        xnext[n] = xcur[n];
      }
    }
    const int sn = s + BC_NB - 1;
    if (sn < nch) issue_bwd(nch - 1 - sn, sn % BC_NB);
  }
  if (lost) {
    // let the copies still in flight land before the CTA exits
    for (int b = 0; b < BC_NB; b++)
      for (int it = 0; it < BC_WAIT_LIMIT && !bc_try_wait(&bars[t][b], (phase >> b) & 1u); it++) {
      }
    bc_store_done();
    atomicAdd(status, 1);
  }
}

static size_t bc_solve_smem(int nl, int R, int tpb) { return (size_t)tpb * bc_thread_stride(nl, R) * sizeof(float); }

// the package rows at level L: sums over the attached edges
__device__ void bc_edge_sums(const BcLevelDev &L, const BcPack *pk, const float *x, float *esum) {
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int k = w; k < BNX; k += blockDim.x >> 5) {
    float s = 0.f;
    const int layer = pk->elayer[k], side = pk->eside[k];
    if (layer >= 0) {
      const int len = side < 2 ? L.nc : L.nr;
      const long long base = (long long)layer * L.plane +
                             (side == 0 ? 0 : side == 1 ? (long long)(L.nr - 1) * L.nc : side == 2 ? 0 : L.nc - 1);
      const long long st = side < 2 ? 1 : L.nc;
      for (int q = lane; q < len; q += 32) s += x[base + q * st];
      for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    }
    if (lane == 0) esum[k] = s;
  }
}

__device__ __forceinline__ float bc_pack_ge(const BcLevelDev &L, const BcPack *pk, int k) {
  return (float)pk->ge0[k] * (pk->eside[k] < 2 ? L.escNS : 1.f);
}

// exact solve of the package nodes with the cells fixed: x_pk = M^-1 (f_pk +
// ge * edge sums), M^-1 precomputed per level
__global__ void bc_pack_solve(BcLevelDev L, const BcPack *__restrict__ pk, float *__restrict__ x,
                              const float *__restrict__ f) {
  __shared__ float esum[BNX], rhs[BNX];
  bc_edge_sums(L, pk, x, esum);
  __syncthreads();
  if (threadIdx.x < BNX) {
    const int k = threadIdx.x;
    rhs[k] = f[L.ncell + k] + bc_pack_ge(L, pk, k) * esum[k];
  }
  __syncthreads();
  if (threadIdx.x < BNX) {
    const int k = threadIdx.x;
    float s = 0.f;
#pragma unroll
    for (int o = 0; o < BNX; o++) s += L.pinv[k * BNX + o] * rhs[o];
    x[L.ncell + k] = s;
  }
}

// y = A x (mode 0) or y = f - A x (mode 1), cells, in difference form
// rs x + sum(-c)(x - x_nbr) + ge (x - x_pk): the system is nearly singular
// and the plain form diag*x + sum c*x_nbr would cancel the FP32 digits of
// smooth vectors
__global__ void bc_apply_cells(BcLevelDev L, const float *__restrict__ x, float *__restrict__ y,
                               const float *__restrict__ f, int mode) {
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= L.ncell) return;
  const int n = (int)(c / L.plane);
  const long long r = c - n * L.plane;
  const int i = (int)(r / L.nc), j = (int)(r - (long long)i * L.nc);
  const float xc = x[c];
  float s = L.rs[c] * xc;
  if (i > 0) s -= L.cN[c] * (xc - x[c - L.nc]);
  if (i < L.nr - 1) s -= L.cS[c] * (xc - x[c + L.nc]);
  if (j > 0) s -= L.cW[c] * (xc - x[c - 1]);
  if (j < L.nc - 1) s -= L.cE[c] * (xc - x[c + 1]);
  if (n > 0) s -= L.cA[c] * (xc - x[c - L.plane]);
  if (n < L.nl - 1) s -= L.cB[c] * (xc - x[c + L.plane]);
  if (n == L.spidx || n == L.hsidx) {
    const float *xp = x + L.ncell;
    if (i == 0) s += L.geNS[n] * (xc - xp[bc_edge_node(n, 0, L.spidx, L.hsidx)]);
    if (i == L.nr - 1) s += L.geNS[n] * (xc - xp[bc_edge_node(n, 1, L.spidx, L.hsidx)]);
    if (j == 0) s += L.geEW[n] * (xc - xp[bc_edge_node(n, 2, L.spidx, L.hsidx)]);
    if (j == L.nc - 1) s += L.geEW[n] * (xc - xp[bc_edge_node(n, 3, L.spidx, L.hsidx)]);
  }
  y[c] = mode ? f[c] - s : s;
}

// same, package rows (one CTA), difference form
__global__ void bc_apply_pack(BcLevelDev L, const BcPack *__restrict__ pk, const float *__restrict__ x,
                              float *__restrict__ y, const float *__restrict__ f, int mode) {
  __shared__ float esum[BNX];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const float *xp = x + L.ncell;
  for (int k = w; k < BNX; k += blockDim.x >> 5) {
    float s = 0.f;
    const int layer = pk->elayer[k], side = pk->eside[k];
    if (layer >= 0) {
      const int len = side < 2 ? L.nc : L.nr;
      const long long base = (long long)layer * L.plane +
                             (side == 0 ? 0 : side == 1 ? (long long)(L.nr - 1) * L.nc : side == 2 ? 0 : L.nc - 1);
      const long long st = side < 2 ? 1 : L.nc;
      const float xk = xp[k];
      for (int q = lane; q < len; q += 32) s += xk - x[base + q * st];
      for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    }
    if (lane == 0) esum[k] = s;
  }
  __syncthreads();
  if (threadIdx.x < BNX) {
    const int k = threadIdx.x;
    float s = bc_pack_ge(L, pk, k) * esum[k] + (float)pk->gamb[k] * xp[k];
    for (int o = 0; o < BNX; o++) s += (float)pk->link[k][o] * (xp[k] - xp[o]);
    y[L.ncell + k] = mode ? f[L.ncell + k] - s : s;
  }
}

// coarse f = sum of the two fine residuals of each pair of planes
__global__ void bc_restrict(const float *__restrict__ rf, float *__restrict__ fc, int nl, int nr, int cnc) {
  const long long cpl = (long long)nr * cnc, ncell = cpl * nl;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < ncell) {
    const long long row = t / cnc;
    const int J = (int)(t - row * cnc);
    const float *s = rf + row * (2 * cnc) + 2 * J;
    fc[t] = s[0] + s[1];
  } else if (t < ncell + BNX) {
    fc[t] = rf[2 * ncell + (t - ncell)];
  }
}

// fine x += coarse correction, constant over each pair of planes
__global__ void bc_prolong_add(const float *__restrict__ xc, float *__restrict__ xf, int nl, int nr, int cnc) {
  const long long fcell = (long long)nr * 2 * cnc * nl;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < fcell) {
    const long long row = t / (2 * cnc);
    const int j = (int)(t - row * 2 * cnc);
    xf[t] += xc[row * cnc + j / 2];
  } else if (t < fcell + BNX) {
    xf[t] += xc[fcell / 2 + (t - fcell)];
  }
}

__global__ void bc_zero(float *x, long long n) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) x[t] = 0.f;
}

// ---------------------------------------------------------------------------
// BiCGStab vector kernels: FP32 data, FP64 reductions in a fixed order
// ---------------------------------------------------------------------------
// scalars: sc[0] rho, [1] rho_old, [2] alpha, [3] omega, [4..9] dot results
enum { SC_RHO = 0, SC_RHO_OLD, SC_ALPHA, SC_OMEGA, SC_D0, SC_D1, SC_D2, SC_D3, SC_NE, SC_MAX };
#define BC_DOT_BLOCKS 296
// layout of BcWork::red: scalars, max-norm bits, dot partials, edge conductances
#define RED_MAXBITS SC_MAX
#define RED_PART 64
#define RED_GE (RED_PART + 2 * BC_DOT_BLOCKS)
#define RED_STATUS (RED_GE + 2 * BC_MAX_NL)   // one int: plane-solve copy failures
#define RED_TOTAL (RED_STATUS + 1)

__global__ void bc_dot_partial(const float *__restrict__ a, const float *__restrict__ b,
                               const float *__restrict__ c, const float *__restrict__ d, long long n,
                               double *__restrict__ part) {
  // part[blk] = (a, b); part[BC_DOT_BLOCKS + blk] = (c, d) when c != nullptr
  __shared__ double sm[2][BCT / 32];
  double s0 = 0.0, s1 = 0.0;
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    s0 += (double)a[k] * (double)b[k];
    if (c) s1 += (double)c[k] * (double)d[k];
  }
  for (int o = 16; o > 0; o >>= 1) {
    s0 += __shfl_down_sync(0xffffffffu, s0, o);
    s1 += __shfl_down_sync(0xffffffffu, s1, o);
  }
  if ((threadIdx.x & 31) == 0) {
    sm[0][threadIdx.x >> 5] = s0;
    sm[1][threadIdx.x >> 5] = s1;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double t0 = 0.0, t1 = 0.0;
    for (int w = 0; w < BCT / 32; w++) {
      t0 += sm[0][w];
      t1 += sm[1][w];
    }
    part[blockIdx.x] = t0;
    part[BC_DOT_BLOCKS + blockIdx.x] = t1;
  }
}

__global__ void bc_dot_final(const double *__restrict__ part, double *__restrict__ out0, double *__restrict__ out1) {
  __shared__ double sm[2][32];
  double s0 = 0.0, s1 = 0.0;
  for (int k = threadIdx.x; k < BC_DOT_BLOCKS; k += blockDim.x) {
    s0 += part[k];
    s1 += part[BC_DOT_BLOCKS + k];
  }
  for (int o = 16; o > 0; o >>= 1) {
    s0 += __shfl_down_sync(0xffffffffu, s0, o);
    s1 += __shfl_down_sync(0xffffffffu, s1, o);
  }
  if ((threadIdx.x & 31) == 0) {
    sm[0][threadIdx.x >> 5] = s0;
    sm[1][threadIdx.x >> 5] = s1;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double t0 = 0.0, t1 = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) {
      t0 += sm[0][w];
      t1 += sm[1][w];
    }
    *out0 = t0;
    if (out1) *out1 = t1;
  }
}

__device__ __forceinline__ double bc_div(double a, double b) { return b != 0.0 && isfinite(a / b) ? a / b : 0.0; }

// start of an inner solve: r = rh = r0, e = p = v = 0, rho_old = alpha = omega = 1
__global__ void bc_start(const float *__restrict__ r0, float *__restrict__ r, float *__restrict__ rh,
                         float *__restrict__ e, float *__restrict__ p, float *__restrict__ v, double *__restrict__ sc,
                         long long n) {
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) {
    r[k] = r0[k];
    rh[k] = r0[k];
    e[k] = 0.f;
    p[k] = 0.f;
    v[k] = 0.f;
  }
  if (k == 0) {
    sc[SC_RHO_OLD] = 1.0;
    sc[SC_ALPHA] = 1.0;
    sc[SC_OMEGA] = 1.0;
  }
}

// p = r + beta (p - omega v), beta = (rho / rho_old)(alpha / omega); sc[SC_RHO] holds rho
__global__ void bc_update_p(float *__restrict__ p, const float *__restrict__ r, const float *__restrict__ v,
                            const double *__restrict__ sc, long long n) {
  const double beta = bc_div(sc[SC_RHO], sc[SC_RHO_OLD]) * bc_div(sc[SC_ALPHA], sc[SC_OMEGA]);
  const float b = (float)beta, om = (float)sc[SC_OMEGA];
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) p[k] = r[k] + b * (p[k] - om * v[k]);
}

// alpha = rho / (rh, v); s = r - alpha v
__global__ void bc_update_s(float *__restrict__ s, const float *__restrict__ r, const float *__restrict__ v,
                            double *__restrict__ sc, long long n) {
  const double alpha = bc_div(sc[SC_RHO], sc[SC_D0]);
  const float a = (float)alpha;
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) s[k] = r[k] - a * v[k];
  if (k == 0) sc[SC_ALPHA] = alpha;   // no thread of this kernel reads SC_ALPHA
}

// omega = (t, s) / (t, t); e += alpha ph + omega sh; r = s - omega t; rho_old = rho
__global__ void bc_update_er(float *__restrict__ e, float *__restrict__ r, const float *__restrict__ ph,
                             const float *__restrict__ sh, const float *__restrict__ s, const float *__restrict__ t,
                             const double *__restrict__ sc, long long n) {
  const double omega = bc_div(sc[SC_D1], sc[SC_D2]);
  const float a = (float)sc[SC_ALPHA], om = (float)omega;
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) {
    e[k] += a * ph[k] + om * sh[k];
    r[k] = s[k] - om * t[k];
  }
}

__global__ void bc_shift_scalars(double *sc) {
  sc[SC_OMEGA] = bc_div(sc[SC_D1], sc[SC_D2]);
  sc[SC_RHO_OLD] = sc[SC_RHO];
}

// T += e; the max |e| (K) into *emax_bits (zeroed by the caller)
__global__ void bc_add_correction(double *__restrict__ T, const float *__restrict__ e, long long n,
                                  unsigned long long *emax_bits) {
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  double a = 0.0;
  if (k < n) {
    T[k] += (double)e[k];
    a = fabs((double)e[k]);
  }
  for (int o = 16; o > 0; o >>= 1) a = fmax(a, __shfl_down_sync(0xffffffffu, a, o));
  if ((threadIdx.x & 31) == 0 && a > 0.0) atomicMax(emax_bits, (unsigned long long)__double_as_longlong(a));
}

// heuristic start: the ambient temperature everywhere
__global__ void bc_fill(double *__restrict__ T, double v, long long n) {
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) T[k] = v;
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
static inline unsigned bnb(long long n) { return (unsigned)((n + BCT - 1) / BCT); }

static BcLevelDev bc_dev(const hsb_dev_model *m, const BcWork *w, int k) {
  const BcLevel &L = w->lv[k];
  BcLevelDev d;
  memset(&d, 0, sizeof(d));
  d.nl = m->nl; d.nr = m->nr; d.nc = L.nc;
  d.plane = L.plane; d.ncell = L.ncell;
  d.cN = L.cN; d.cS = L.cS; d.cW = L.cW; d.cE = L.cE; d.cA = L.cA; d.cB = L.cB; d.dg = L.dg;
  d.rs = L.rs;
  d.LF = L.LF; d.UB = L.UB;
  d.pinv = L.pinv;
  const double sc = (double)(1ll << k);
  for (int n = 0; n < m->nl && n < BC_MAX_NL; n++) {
    d.geNS[n] = (float)(w->geNS0[n] * sc);
    d.geEW[n] = (float)w->geEW0[n];
  }
  d.escNS = (float)sc;
  d.spidx = m->spidx; d.hsidx = m->hsidx;
  return d;
}

typedef void (*SolveFn)(const float *, const float *, const float *, float *, float *, int, int, long long, int,
                        int, int *);
static SolveFn solve_for(int nl);

static void free_bc(void *p) {
  BcWork *w = (BcWork *)p;
  if (!w) return;
  for (auto &L : w->lv) {
    float *b[] = {L.cN, L.cS, L.cW, L.cE, L.cA, L.cB, L.dg, L.rs, L.LF, L.UB, L.x, L.f, L.r, L.pr, L.py, L.pinv};
    for (float *q : b)
      if (q) cudaFree(q);
  }
  void *b2[] = {w->d_pk, w->c64, w->b64, w->r64, w->band, w->r, w->rh, w->p, w->v,
                w->s, w->t, w->ph, w->sh, w->e, w->red};
  for (void *q : b2)
    if (q) cudaFree(q);
  if (w->h_red) cudaFreeHost(w->h_red);
  if (w->pass_exec) cudaGraphExecDestroy(w->pass_exec);
  delete w;
}

static int bc_setup(hsb_dev_model *m, BcWork **out) {
  BcWork *w = new BcWork();
  w->coef_version = -1;
  const int nl = m->nl;
  int nc = m->nc;
  for (;;) {
    BcLevel L{};
    L.nc = nc;
    L.plane = (long long)m->nr * nc;
    L.ncell = L.plane * nl;
    L.n = L.ncell + BNX;
    w->lv.push_back(L);
    if (nc < 4 || (nc & 1)) break;
    nc /= 2;
  }
  w->nlev = (int)w->lv.size();
  auto fail = [&](int rc) {
    free_bc(w);
    return rc;
  };
  size_t band_max = 0;
  for (auto &L : w->lv) {
    float **arr[] = {&L.cN, &L.cS, &L.cW, &L.cE, &L.cA, &L.cB, &L.dg, &L.rs};
    for (float **a : arr)
      if (cudaMalloc(a, sizeof(float) * L.ncell) != cudaSuccess) return fail(set_error(HSB_E_NOMEM, "BiCGStab levels"));
    const size_t nqa = (size_t)L.ncell;   // planes x nq
    const size_t nva = (size_t)L.nc * m->nr * bc_r4(nl);
    if (cudaMalloc(&L.LF, sizeof(float) * nqa * bc_r4(nl)) != cudaSuccess ||
        cudaMalloc(&L.UB, sizeof(float) * nqa * bc_r4(nl + 1)) != cudaSuccess || cudaMalloc(&L.x, sizeof(float) * L.n) != cudaSuccess ||
        cudaMalloc(&L.f, sizeof(float) * L.n) != cudaSuccess || cudaMalloc(&L.r, sizeof(float) * L.n) != cudaSuccess ||
        cudaMalloc(&L.pr, sizeof(float) * nva) != cudaSuccess || cudaMalloc(&L.py, sizeof(float) * nva) != cudaSuccess ||
        cudaMalloc(&L.pinv, sizeof(float) * BNX * BNX) != cudaSuccess)
      return fail(set_error(HSB_E_NOMEM, "BiCGStab levels"));
    const size_t bm = (size_t)L.ncell * (2 * nl + 1);
    if (bm > band_max) band_max = bm;
  }
  const long long n0 = m->vlen;
  if (cudaMalloc(&w->d_pk, sizeof(BcPack)) != cudaSuccess || cudaMalloc(&w->c64, sizeof(double) * 8 * m->ncell) != cudaSuccess ||
      cudaMalloc(&w->b64, sizeof(double) * n0) != cudaSuccess || cudaMalloc(&w->r64, sizeof(double) * n0) != cudaSuccess ||
      cudaMalloc(&w->band, sizeof(double) * band_max) != cudaSuccess)
    return fail(set_error(HSB_E_NOMEM, "BiCGStab operator"));
  float **vec[] = {&w->r, &w->rh, &w->p, &w->v, &w->s, &w->t, &w->ph, &w->sh, &w->e};
  for (float **a : vec)
    if (cudaMalloc(a, sizeof(float) * n0) != cudaSuccess) return fail(set_error(HSB_E_NOMEM, "BiCGStab vectors"));
  if (cudaMalloc(&w->red, sizeof(double) * RED_TOTAL) != cudaSuccess ||
      cudaMallocHost(&w->h_red, sizeof(double) * 16) != cudaSuccess)
    return fail(set_error(HSB_E_NOMEM, "BiCGStab reductions"));
  w->status = (int *)(w->red + RED_STATUS);
  if (cudaMemsetAsync(w->status, 0, sizeof(int), m->stream) != cudaSuccess)
    return fail(set_error(HSB_E_CUDA, "BiCGStab status"));
  // plane solve: chunks of R rows, as many planes per CTA as fit ~200 KB
  w->R = m->nr % 16 == 0 ? 16 : m->nr % 8 == 0 ? 8 : m->nr % 4 == 0 ? 4 : m->nr % 2 == 0 ? 2 : 1;
  const size_t per = bc_solve_smem(nl, w->R, 1);
  w->tpb = (int)(200 * 1024 / per);
  if (w->tpb > 32) w->tpb = 32;
  if (w->tpb < 1) w->tpb = 1;
  if (raise_smem_limit((const void *)solve_for(nl), bc_solve_smem(nl, w->R, w->tpb)) != HSB_OK)
    return fail(set_error(HSB_E_CUDA, "BiCGStab plane solver shared memory"));
  *out = w;
  return HSB_OK;
}

static int bc_build(hsb_dev_model *m, BcWork *w) {
  const int nl = m->nl;
  const package_RC_t &pk = m->h_pk;
  // per-layer edge conductances (spreader and sink), package system
  for (int n = 0; n < BC_MAX_NL; n++) w->geNS0[n] = w->geEW0[n] = 0.0;
  for (int n = 0; n < nl; n++) {
    const LayerCoef &c = m->hostL0[n];
    if (c.kind == LK_SINK || c.kind == LK_SPREADER) {
      w->geNS0[n] = 1.0 / c.edgeNS;
      w->geEW0[n] = 1.0 / c.edgeEW;
    }
  }
  BcPack &P = w->pk;
  memset(&P, 0, sizeof(P));
  for (int k = 0; k < BNX; k++) P.elayer[k] = P.eside[k] = -1;
  auto link = [&](int a, int b, double r) {
    P.link[a][b] += 1.0 / r;
    P.link[b][a] += 1.0 / r;
  };
  const int nodesC[4] = {HSB_SINK_C_N, HSB_SINK_C_S, HSB_SINK_C_W, HSB_SINK_C_E};
  const int nodesO[4] = {HSB_SINK_N, HSB_SINK_S, HSB_SINK_W, HSB_SINK_E};
  const int nodesS[4] = {HSB_SP_N, HSB_SP_S, HSB_SP_W, HSB_SP_E};
  for (int s = 0; s < 4; s++) {
    const bool y = s < 2;
    P.gamb[nodesO[s]] = 1.0 / (pk.r_hs_per + pk.r_amb_per);
    link(nodesO[s], nodesC[s], (y ? pk.r_hs2_y : pk.r_hs2_x) + pk.r_hs);
    P.gamb[nodesC[s]] = 1.0 / (y ? pk.r_hs_c_per_y + pk.r_amb_c_per_y : pk.r_hs_c_per_x + pk.r_amb_c_per_x);
    link(nodesC[s], nodesS[s], y ? pk.r_sp_per_y : pk.r_sp_per_x);
    P.elayer[nodesC[s]] = m->hsidx;
    P.eside[nodesC[s]] = s;
    P.ge0[nodesC[s]] = y ? w->geNS0[m->hsidx] : w->geEW0[m->hsidx];
    P.elayer[nodesS[s]] = m->spidx;
    P.eside[nodesS[s]] = s;
    P.ge0[nodesS[s]] = y ? w->geNS0[m->spidx] : w->geEW0[m->spidx];
  }
  HSB_CUDA(cudaMemcpyAsync(w->d_pk, &P, sizeof(P), cudaMemcpyHostToDevice, m->stream));
  // package block of every level (its edge conductance totals do not change
  // with the level: nc_k cells of 2^k times the level-0 conductance), inverted
  // in FP64 by Gauss-Jordan with partial pivoting
  for (int k = 0; k < w->nlev; k++) {
    double M[BNX][2 * BNX];
    for (int a = 0; a < BNX; a++) {
      const int cnt = P.elayer[a] < 0 ? 0 : (P.eside[a] < 2 ? w->lv[k].nc : m->nr);
      const double ge = P.ge0[a] * (P.eside[a] >= 0 && P.eside[a] < 2 ? (double)(1ll << k) : 1.0);
      double D = cnt * ge + P.gamb[a];
      for (int b = 0; b < BNX; b++) {
        D += P.link[a][b];
        M[a][b] = -P.link[a][b];
        M[a][BNX + b] = a == b ? 1.0 : 0.0;
      }
      M[a][a] = D;
    }
    for (int c = 0; c < BNX; c++) {
      int piv = c;
      for (int r = c + 1; r < BNX; r++)
        if (fabs(M[r][c]) > fabs(M[piv][c])) piv = r;
      if (piv != c)
        for (int q = 0; q < 2 * BNX; q++) {
          const double t = M[c][q];
          M[c][q] = M[piv][q];
          M[piv][q] = t;
        }
      const double inv = 1.0 / M[c][c];
      for (int q = 0; q < 2 * BNX; q++) M[c][q] *= inv;
      for (int r = 0; r < BNX; r++)
        if (r != c && M[r][c] != 0.0) {
          const double fct = M[r][c];
          for (int q = 0; q < 2 * BNX; q++) M[r][q] -= fct * M[c][q];
        }
    }
    float inv32[BNX * BNX];
    for (int a = 0; a < BNX; a++)
      for (int b = 0; b < BNX; b++) inv32[a * BNX + b] = (float)M[a][BNX + b];
    HSB_CUDA(h2d_on(w->lv[k].pinv, inv32, sizeof(inv32), m->stream));
  }
  // the edge conductances go to the device with the FP64 build (scratch in r64)
  double ge[2 * BC_MAX_NL];
  memcpy(ge, w->geNS0, sizeof(double) * BC_MAX_NL);
  memcpy(ge + BC_MAX_NL, w->geEW0, sizeof(double) * BC_MAX_NL);
  double *d_ge = w->red + RED_GE;
  HSB_CUDA(cudaMemcpyAsync(d_ge, ge, sizeof(ge), cudaMemcpyHostToDevice, m->stream));
  double *d_gamb = w->r64;                          // temporary: package ambient conductances
  HSB_CUDA(cudaMemcpyAsync(d_gamb, P.gamb, sizeof(P.gamb), cudaMemcpyHostToDevice, m->stream));
  const StencilArgs S = make_args(m, m->L0, m->nr, m->nc);
  bc_build64<<<bnb(m->vlen), BCT, 0, m->stream>>>(S, m->pgrid, d_ge, d_ge + BC_MAX_NL, w->c64, w->b64, d_gamb);
  // FP32 level 0 and the coarse levels
  BcLevel &L0 = w->lv[0];
  float *dst[8] = {L0.cN, L0.cS, L0.cW, L0.cE, L0.cA, L0.cB, L0.dg, L0.rs};
  for (int a = 0; a < 8; a++) bc_to32<<<bnb(m->ncell), BCT, 0, m->stream>>>(w->c64 + (size_t)a * m->ncell, dst[a], m->ncell);
  for (int k = 1; k < w->nlev; k++) {
    BcLevel &C = w->lv[k];
    bc_coarsen<<<bnb(C.ncell), BCT, 0, m->stream>>>(bc_dev(m, w, k - 1), C.cN, C.cS, C.cW, C.cE, C.cA, C.cB, C.dg,
                                                    C.rs, C.nc);
  }
  for (int k = 0; k < w->nlev; k++) {
    BcLevel &L = w->lv[k];
    bc_factor<<<(L.nc + 63) / 64, 64, 0, m->stream>>>(bc_dev(m, w, k), w->band, L.LF, L.UB);
  }
  HSB_CUDA(cudaGetLastError());
  return HSB_OK;
}

// the right-hand side depends on the power: rebuilt every solve (cheap)
static int bc_rhs(hsb_dev_model *m, BcWork *w) {
  double *d_ge = w->red + RED_GE;
  double *d_gamb = w->r64;
  HSB_CUDA(cudaMemcpyAsync(d_gamb, w->pk.gamb, sizeof(w->pk.gamb), cudaMemcpyHostToDevice, m->stream));
  const StencilArgs S = make_args(m, m->L0, m->nr, m->nc);
  bc_build64<<<bnb(m->vlen), BCT, 0, m->stream>>>(S, m->pgrid, d_ge, d_ge + BC_MAX_NL, w->c64, w->b64, d_gamb);
  HSB_CUDA(cudaGetLastError());
  return HSB_OK;
}

static SolveFn solve_for(int nl) {
  switch (nl) {
    case 1: return bc_plane_solve<1>;
    case 2: return bc_plane_solve<2>;
    case 3: return bc_plane_solve<3>;
    case 4: return bc_plane_solve<4>;
    case 5: return bc_plane_solve<5>;
    case 6: return bc_plane_solve<6>;
    case 7: return bc_plane_solve<7>;
    case 8: return bc_plane_solve<8>;
    case 9: return bc_plane_solve<9>;
    case 10: return bc_plane_solve<10>;
    case 11: return bc_plane_solve<11>;
    case 12: return bc_plane_solve<12>;
  }
  return nullptr;
}

static void bc_half_sweep(hsb_dev_model *m, BcWork *w, const BcLevelDev &d, int k, float *x, const float *f,
                          int color) {
  BcLevel &L = w->lv[k];
  const int ncol = color ? d.nc / 2 : (d.nc + 1) / 2;
  const int nq = d.nr * d.nl;
  dim3 g((unsigned)((ncol + 31) / 32), (unsigned)((nq + 31) / 32));
  bc_plane_rhs<<<g, 256, 0, m->stream>>>(d, x, f, L.pr, color);
  solve_for(m->nl)<<<(unsigned)((ncol + w->tpb - 1) / w->tpb), w->tpb, bc_solve_smem(m->nl, w->R, w->tpb),
                     m->stream>>>(L.LF, L.UB, L.pr, L.py, x, d.nr, d.nc, d.plane, color, w->R, w->status);
}

static void bc_smooth(hsb_dev_model *m, BcWork *w, int k, float *x, const float *f, bool pre) {
  const BcLevelDev d = bc_dev(m, w, k);
  if (pre) {
    bc_half_sweep(m, w, d, k, x, f, 0);
    bc_half_sweep(m, w, d, k, x, f, 1);
    bc_pack_solve<<<1, 384, 0, m->stream>>>(d, w->d_pk, x, f);
  } else {
    bc_pack_solve<<<1, 384, 0, m->stream>>>(d, w->d_pk, x, f);
    bc_half_sweep(m, w, d, k, x, f, 1);
    bc_half_sweep(m, w, d, k, x, f, 0);
  }
}

// x = V-cycle applied to f on level k (from x = 0)
static void bc_vcycle(hsb_dev_model *m, BcWork *w, int k, float *x, const float *f, long long *launches) {
  const BcLevel &L = w->lv[k];
  bc_zero<<<bnb(L.n), BCT, 0, m->stream>>>(x, L.n);
  *launches += 1;
  if (k == w->nlev - 1) {
    for (int s = 0; s < 4; s++) bc_smooth(m, w, k, x, f, true);
    *launches += 20;
    return;
  }
  const BcLevelDev d = bc_dev(m, w, k);
  bc_smooth(m, w, k, x, f, true);
  bc_apply_cells<<<bnb(L.ncell), BCT, 0, m->stream>>>(d, x, L.r, f, 1);
  bc_apply_pack<<<1, 384, 0, m->stream>>>(d, w->d_pk, x, L.r, f, 1);
  BcLevel &C = w->lv[k + 1];
  bc_restrict<<<bnb(C.n), BCT, 0, m->stream>>>(L.r, C.f, m->nl, m->nr, C.nc);
  bc_vcycle(m, w, k + 1, C.x, C.f, launches);
  bc_prolong_add<<<bnb(L.n), BCT, 0, m->stream>>>(C.x, x, m->nl, m->nr, C.nc);
  bc_smooth(m, w, k, x, f, false);
  *launches += 15;
}

static void bc_matvec(hsb_dev_model *m, BcWork *w, const float *x, float *y) {
  const BcLevelDev d = bc_dev(m, w, 0);
  bc_apply_cells<<<bnb(w->lv[0].ncell), BCT, 0, m->stream>>>(d, x, y, nullptr, 0);
  bc_apply_pack<<<1, 384, 0, m->stream>>>(d, w->d_pk, x, y, nullptr, 0);
}

static void bc_dot2(hsb_dev_model *m, BcWork *w, const float *a, const float *b, const float *c, const float *d,
                    long long n, double *out0, double *out1) {
  double *part = w->red + RED_PART;
  bc_dot_partial<<<BC_DOT_BLOCKS, BCT, 0, m->stream>>>(a, b, c, d, n, part);
  bc_dot_final<<<1, 256, 0, m->stream>>>(part, out0, out1);
}

// one refinement pass on the model's stream: r = b - G T (FP64), BiCGStab
// on G e = r (FP32, `inner` iterations), T += e, |e|_2^2 and max |r| to the host
static void bc_pass(hsb_dev_model *m, BcWork *w, double *T, int inner, long long *launches) {
  const StencilArgs S = make_args(m, m->L0, m->nr, m->nc);
  const long long n0 = m->vlen;
  double *sc = w->red;
  unsigned long long *maxbits = (unsigned long long *)(w->red + RED_MAXBITS);
  double *d_ge = w->red + RED_GE;
  cudaMemsetAsync(maxbits, 0, sizeof(unsigned long long), m->stream);
  bc_residual64<<<bnb(m->ncell), BCT, 0, m->stream>>>(S, w->c64, d_ge, d_ge + BC_MAX_NL, T, w->b64, w->r64, w->s,
                                                      maxbits);
  bc_pack_residual64<<<1, 384, 0, m->stream>>>(S, w->d_pk, T, w->b64, w->r64, w->s, maxbits);
  bc_start<<<bnb(n0), BCT, 0, m->stream>>>(w->s, w->r, w->rh, w->e, w->p, w->v, sc, n0);
  *launches += 3;
  for (int it = 0; it < inner; it++) {
    bc_dot2(m, w, w->rh, w->r, nullptr, nullptr, n0, sc + SC_RHO, nullptr);
    bc_update_p<<<bnb(n0), BCT, 0, m->stream>>>(w->p, w->r, w->v, sc, n0);
    bc_vcycle(m, w, 0, w->ph, w->p, launches);
    bc_matvec(m, w, w->ph, w->v);
    bc_dot2(m, w, w->rh, w->v, nullptr, nullptr, n0, sc + SC_D0, nullptr);
    bc_update_s<<<bnb(n0), BCT, 0, m->stream>>>(w->s, w->r, w->v, sc, n0);
    bc_vcycle(m, w, 0, w->sh, w->s, launches);
    bc_matvec(m, w, w->sh, w->t);
    bc_dot2(m, w, w->t, w->s, w->t, w->t, n0, sc + SC_D1, sc + SC_D2);
    bc_update_er<<<bnb(n0), BCT, 0, m->stream>>>(w->e, w->r, w->ph, w->sh, w->s, w->t, sc, n0);
    bc_shift_scalars<<<1, 1, 0, m->stream>>>(sc);
    *launches += 16;
  }
  // the max norm of this correction (K) decides convergence
  cudaMemsetAsync(sc + SC_NE, 0, sizeof(double), m->stream);
  bc_add_correction<<<bnb(n0), BCT, 0, m->stream>>>(T, w->e, n0, (unsigned long long *)(sc + SC_NE));
  *launches += 3;
  cudaMemcpyAsync(w->h_red, sc, sizeof(double) * (SC_MAX + 1), cudaMemcpyDeviceToHost, m->stream);
  cudaMemcpyAsync(w->h_red + 12, w->status, sizeof(int), cudaMemcpyDeviceToHost, m->stream);
}

#ifndef BC_INNER
#define BC_INNER 10   // BiCGStab iterations per FP64 refinement pass
#endif

int bicgstab_steady(hsb_dev_model *m, const hsb_solver_opts *o, hsb_stats *st) {
  if (m->nx != HSB_EXTRA) return set_error(HSB_E_ARG, "the BiCGStab steady solver models the primary heat path only");
  if (m->nl > BC_MAX_NL) return set_error(HSB_E_ARG, "the BiCGStab steady solver supports up to 12 layers");
  BcWork *w = (BcWork *)m->krylov;
  int rc;
  if (!w) {
    if ((rc = bc_setup(m, &w))) return rc;
    m->krylov = w;
    m->krylov_free = free_bc;
  }
  if (w->coef_version != m->coef_version) {
    if ((rc = bc_build(m, w))) return rc;
    w->coef_version = m->coef_version;
  }
  if ((rc = bc_rhs(m, w))) return rc;
  const StencilArgs S = make_args(m, m->L0, m->nr, m->nc);
  const long long n0 = m->vlen;
  const double tol = (o && o->steady_tol > 0) ? o->steady_tol : 1e-7;
  const int max_ref = (o && o->max_iters > 0) ? o->max_iters : 40;
  double *T = m->ys;
  double *sc = w->red;
  unsigned long long *maxbits = (unsigned long long *)(w->red + RED_MAXBITS);
  double *d_ge = w->red + RED_GE;
  long long launches = 0;
  bc_fill<<<bnb(n0), BCT, 0, m->stream>>>(T, m->ambient, n0);
  HSB_CUDA(cudaGetLastError());
  // the refinement pass is the same kernel sequence every time: capture it once
  if (!w->pass_exec || w->pass_T != T) {
    if (w->pass_exec) {
      cudaGraphExecDestroy(w->pass_exec);
      w->pass_exec = nullptr;
    }
    cudaGraph_t g;
    long long cnt = 0;
    HSB_CUDA(cudaStreamBeginCapture(m->stream, cudaStreamCaptureModeThreadLocal));
    bc_pass(m, w, T, BC_INNER, &cnt);
    const cudaError_t ce = cudaStreamEndCapture(m->stream, &g);
    if (ce != cudaSuccess) return cuda_check(ce, "capturing the BiCGStab refinement pass");
    const cudaError_t ie = cudaGraphInstantiate(&w->pass_exec, g, 0);
    cudaGraphDestroy(g);
    if (ie != cudaSuccess) {
      w->pass_exec = nullptr;
      return cuda_check(ie, "instantiating the BiCGStab refinement pass");
    }
    w->pass_T = T;
    w->pass_launches = cnt;
  }
  // stopping as in the multigrid solver: the last correction below tol, or
  // passes contracting so fast (rho = |e_k| / |e_k-1| < 0.1) that the next
  // correction, rho |e_k|, is below tol / 10
  double emax = 1e300, rmax = 0.0, eprev = 0.0;
  bool converged = false;
  for (int ref = 0; ref < max_ref; ref++) {
    HSB_CUDA(cudaGraphLaunch(w->pass_exec, m->stream));
    HSB_CUDA(cudaStreamSynchronize(m->stream));
    launches += w->pass_launches;
    {
      unsigned long long bits;
      memcpy(&bits, w->h_red + SC_NE, sizeof(bits));
      memcpy(&emax, &bits, sizeof(emax));
    }
    int lost = 0;
    memcpy(&lost, w->h_red + 12, sizeof(int));
    if (lost) return set_error(HSB_E_CUDA, "BiCGStab plane solve: a chunk copy did not complete in time");
    st->refinements += 1;
    st->cycles += BC_INNER;
    if (!(emax == emax)) return set_error(HSB_E_NOCONV, "BiCGStab steady solve broke down (NaN correction)");
    if (emax < tol) {
      converged = true;
      break;
    }
    if (ref > 0 && eprev > 0.0) {
      const double rho = emax / eprev;
      if (rho < 0.1 && 10.0 * rho * emax < tol) {
        converged = true;
        break;
      }
    }
    eprev = emax;
    if (m->yield_fn) m->yield_fn(m->yield_ctx);
  }
  // final FP64 residual for the record
  HSB_CUDA(cudaMemsetAsync(maxbits, 0, sizeof(unsigned long long), m->stream));
  bc_residual64<<<bnb(m->ncell), BCT, 0, m->stream>>>(S, w->c64, d_ge, d_ge + BC_MAX_NL, T, w->b64, w->r64, w->s,
                                                      maxbits);
  bc_pack_residual64<<<1, 384, 0, m->stream>>>(S, w->d_pk, T, w->b64, w->r64, w->s, maxbits);
  launches += 3;
  HSB_CUDA(cudaMemcpyAsync(w->h_red, sc, sizeof(double) * (SC_MAX + 1), cudaMemcpyDeviceToHost, m->stream));
  HSB_CUDA(cudaStreamSynchronize(m->stream));
  {
    unsigned long long bits;
    memcpy(&bits, w->h_red + SC_MAX, sizeof(bits));
    memcpy(&rmax, &bits, sizeof(rmax));
  }
  st->residual = rmax;
  st->launches += launches;
  if (!converged) return set_error(HSB_E_NOCONV, "BiCGStab steady solve did not converge");
  return HSB_OK;
}

}  // namespace hsb
