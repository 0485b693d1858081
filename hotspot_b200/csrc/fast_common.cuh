// fast_common.cuh -- pieces shared by the fast transient kernels
// (rk4_fast.cu: stage-by-stage step-doubling RK4; rk4_krylov.cu: the same
// steps evaluated through Krylov vectors of the affine slope operator).
//
// Tiles are 32 x 8 (j x i) cells through all layers, one thread per (i, j)
// column.  Stage inputs are staged in shared memory by TMA tensor copies of
// the tile plus a one-cell halo; the halo boxes start 2 doubles / 4 floats
// left of the tile so every copy's x coordinate is 16-byte aligned.
#pragma once
#include <cooperative_groups.h>
#include <cuda.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <mutex>

#include "stencil_exact.cuh"

namespace hsb {

#define FT_THREADS 256
#define FT_WARPS (FT_THREADS / 32)
#define TJ 32                 // tile columns (j)
#define TI 8                  // tile rows (i)
#define NI (TI * TJ)          // cells of a tile layer, one per thread
#define HR (TI + 2)           // halo box rows
#define DW 36                 // FP64 halo box row: columns j0-2 .. j0+33 (x start 16-byte aligned)
#define KW 40                 // FP32 halo box row: columns j0-4 .. j0+35
#define DP (HR * DW)          // FP64 halo box layer
#define KP (HR * KW)          // FP32 halo box layer
#define NXMAX (HSB_EXTRA + HSB_EXTRA_SEC)
#define NEDGE 20
#define FT_MAX_LAYERS 16
#define PK_LINKS 4
#define WAIT_LIMIT (1 << 22)  // mbarrier polls before a tile copy is declared lost
#define KRY_DMAX 31           // highest Krylov vector index (six step rejections in a row)

struct LayerF {
  float gNS, gEW;       // lateral conductances
  float gDown;          // conductance to layer n+1 (1/rz[n])
  float invC;           // 1 / capacitance
  float gEdgeNS, gEdgeEW, gAmb;
  int kind;
};

// package nodes as conductances (FP64): dv_k = (ge_k * es[eidx_k] +
// gamb_k (amb - x_k) + sum_l g[k][l] (x_nb[k][l] - x_k)) * invC_k, the
// couplings of slope_fn_pack (temperature_grid.c:2857-3093), including its
// one-sided solder/substrate links; every node has at most two links
struct PackF {
  double invC[NXMAX], gamb[NXMAX], ge[NXMAX];
  double g[NXMAX][PK_LINKS];
  int eidx[NXMAX];
  int nb[NXMAX][PK_LINKS];
};

// TMA descriptors of the arrays a stage reads: halo boxes (_h) for stage
// inputs, interior boxes (_i) for per-cell operands.  P and Q are the two
// state buffers that swap roles (y / ytemp) as steps are accepted.
struct Maps {
  CUtensorMap yP_h, yP_i, yQ_h, yQ_i, t1_h, k1_h, k1_i, k2_h, k2_i, k3_h, pf_i;
};

struct FastWork {
  long long ncell;
  int grid, coef_version, segmax;
  float *k1, *k2, *k3, *pf;
  double *ytemp, *t1, *t2;
  float *gN, *gS, *gW, *gE, *gA, *gB, *invC;
  float *aN, *aS, *aW, *aE, *aO;
  LayerF *Lf;
  PackF *pk;
  double *part;                   // [2][NEDGE][segmax] edge partial sums
  unsigned long long *err;        // [2] max-norm bits
  long long *cnt;                 // [0]=steps [1]=attempts [2]=final buffer [3]=status
  long long *h_cnt;               // pinned mirror
  Maps maps;
  const double *mapP, *mapQ;      // the state buffers the maps describe
  // Krylov form (rk4_krylov.cu)
  float *N;                       // [KRY_DMAX + 1][nstride] Krylov vectors
  long long nstride;
  CUtensorMap kmap_y, kmap_y2, kmap_yi, kmap_y2i, kmap_pf, kmap_N, kmap_Ni;   // kmap_N(i): all vectors, 4-D
  const double *kmap_ybuf, *kmap_y2buf;           // the state buffers kmap_y / kmap_y2 describe
  const void *kfn;                // Krylov kernel variant kgrid was computed for
  int kgrid;                      // its co-resident grid
  cudaEvent_t kev[2];             // kernel timing events
  void *tb;                       // temporally blocked kernel's resources (rk4_tb.cu), or null
};

// Layers are processed in fixed-size chunks, so that a chunk's per-cell
// coefficient loads (detailed 3-D and microchannel models) are all issued
// before their first use.
template <bool FIELD, bool ADV>
struct Chunk {
  static constexpr int n = (FIELD || ADV) ? 1 : 4;
};

__host__ __device__ inline size_t al128(size_t x) { return (x + 127) & ~(size_t)127; }

// ---------------------------------------------------------------------------
// TMA and mbarrier primitives
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// 3-D tiled load of box (x, y, z=0) into shared memory; x is 16-byte aligned
// by construction (halo boxes start 2 doubles / 4 floats left of the tile)
__device__ __forceinline__ void tma3(void *dst, const CUtensorMap *map, int x, int y, unsigned long long *bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];\n" ::"r"(
          smem_u32(dst)),
      "l"(map), "r"(x), "r"(y), "r"(0), "r"(smem_u32(bar))
      : "memory");
}
// 4-D tiled load of box (x, y, z=0, w) into shared memory
__device__ __forceinline__ void tma4(void *dst, const CUtensorMap *map, int x, int y, int w, unsigned long long *bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];\n" ::"r"(
          smem_u32(dst)),
      "l"(map), "r"(x), "r"(y), "r"(0), "r"(w), "r"(smem_u32(bar))
      : "memory");
}

static_assert(sizeof(PackF) % 8 == 0, "package table is copied as 8-byte words");
static_assert(NI == FT_THREADS, "one thread per cell of a tile");
static_assert(2 * (TJ + 2) + 2 * TI <= FT_THREADS, "one thread per halo cell");

// thread -> halo-ring cell of a 32x8 tile: row hr in [0, HR), column hc in
// [0, TJ+2) counted from j0-1; hr = -1 for threads without one
__device__ __forceinline__ void halo_cell(int tid, int *hr, int *hc) {
  *hr = -1;
  *hc = 0;
  if (tid < TJ + 2) { *hr = 0; *hc = tid; }
  else if (tid < 2 * (TJ + 2)) { *hr = HR - 1; *hc = tid - (TJ + 2); }
  else if (tid < 2 * (TJ + 2) + TI) { *hr = tid - 2 * (TJ + 2) + 1; *hc = 0; }
  else if (tid < 2 * (TJ + 2) + 2 * TI) { *hr = tid - 2 * (TJ + 2) - TI + 1; *hc = TJ + 1; }
}

// ---------------------------------------------------------------------------
// tensor maps
// ---------------------------------------------------------------------------
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *,
                                  CUtensorMapInterleave, CUtensorMapSwizzle, CUtensorMapL2promotion,
                                  CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_tiled() {
  static EncodeTiledFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (EncodeTiledFn)p;
  });
  return fn;
}

// [nl][nr][nc] array of doubles (f64) or floats seen as a 3-D tensor with
// box (bx, by, nl); out-of-range box elements read as zero
static int make_map(CUtensorMap *map, const void *base, bool f64, const hsb_dev_model *m, unsigned bx,
                    unsigned by) {
  EncodeTiledFn enc = encode_tiled();
  if (!enc) return set_error(HSB_E_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
  if (((uintptr_t)base & 15u) != 0) return set_error(HSB_E_ARG, "fast transient buffers must be 16-byte aligned");
  const cuuint64_t es = f64 ? 8 : 4;
  const cuuint64_t dims[3] = {(cuuint64_t)m->nc, (cuuint64_t)m->nr, (cuuint64_t)m->nl};
  const cuuint64_t strides[2] = {(cuuint64_t)m->nc * es, (cuuint64_t)m->nr * m->nc * es};
  const cuuint32_t box[3] = {bx, by, (cuuint32_t)m->nl};
  const cuuint32_t estr[3] = {1, 1, 1};
  const CUresult r = enc(map, f64 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3,
                         const_cast<void *>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                         CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return set_error(HSB_E_ARG, "tensor map encoding failed for the fast transient form");
  return HSB_OK;
}

// `count` [nl][nr][nc] FP32 arrays `stride` floats apart, seen as one 4-D
// tensor with box (bx, by, nl, 1)
static int make_map4(CUtensorMap *map, const float *base, const hsb_dev_model *m, unsigned bx, unsigned by,
                     int count, long long stride) {
  EncodeTiledFn enc = encode_tiled();
  if (!enc) return set_error(HSB_E_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
  if (((uintptr_t)base & 15u) != 0 || (stride * 4) % 16 != 0)
    return set_error(HSB_E_ARG, "fast transient buffers must be 16-byte aligned");
  const cuuint64_t dims[4] = {(cuuint64_t)m->nc, (cuuint64_t)m->nr, (cuuint64_t)m->nl, (cuuint64_t)count};
  const cuuint64_t strides[3] = {(cuuint64_t)m->nc * 4, (cuuint64_t)m->nr * m->nc * 4, (cuuint64_t)stride * 4};
  const cuuint32_t box[4] = {bx, by, (cuuint32_t)m->nl, 1};
  const cuuint32_t estr[4] = {1, 1, 1, 1};
  const CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, const_cast<float *>(base), dims, strides, box,
                         estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                         CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return set_error(HSB_E_ARG, "tensor map encoding failed for the fast transient form");
  return HSB_OK;
}

static int check_shape(const hsb_dev_model *m) {
  if (m->nl > FT_MAX_LAYERS) return set_error(HSB_E_ARG, "the fast transient form supports up to 16 layers");
  if (m->nc % 4 != 0) return set_error(HSB_E_ARG, "the fast transient form needs a multiple of 4 grid columns");
  return HSB_OK;
}

// FP32 layer table and FP64 package table from the model's FP64 values
static void host_tables(const hsb_dev_model *m, LayerF *Lf, PackF *P) {
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
  memset(P, 0, sizeof(PackF));
  for (int k = 0; k < NXMAX; k++) {
    P->eidx[k] = -1;
    for (int l = 0; l < PK_LINKS; l++) P->nb[k][l] = -1;
  }
  const package_RC_t &pk = m->h_pk;
  const LayerCoef *L = m->hostL0;
  auto edge = [&](int node, int e, double R) {
    P->eidx[node] = e;
    P->ge[node] = 1.0 / R;
  };
  auto lnk = [&](int a, int b, double R) {
    for (int l = 0; l < PK_LINKS; l++) {
      if (P->nb[a][l] == b || P->nb[a][l] < 0) {
        P->nb[a][l] = b;
        P->g[a][l] += 1.0 / R;
        return;
      }
    }
  };
  const int cN[4] = {HSB_SINK_C_N, HSB_SINK_C_S, HSB_SINK_C_W, HSB_SINK_C_E};
  const int oN[4] = {HSB_SINK_N, HSB_SINK_S, HSB_SINK_W, HSB_SINK_E};
  const int sN[4] = {HSB_SP_N, HSB_SP_S, HSB_SP_W, HSB_SP_E};
  for (int s = 0; s < 4; s++) {
    const bool y = s < 2;
    const double r_hs2 = (y ? pk.r_hs2_y : pk.r_hs2_x) + pk.r_hs;
    P->gamb[oN[s]] = 1.0 / (pk.r_hs_per + pk.r_amb_per);
    lnk(oN[s], cN[s], r_hs2);
    P->invC[oN[s]] = 1.0 / (pk.c_hs_per + pk.c_amb_per);
    edge(cN[s], s, y ? L[m->hsidx].edgeNS : L[m->hsidx].edgeEW);
    P->gamb[cN[s]] = 1.0 / (y ? pk.r_hs_c_per_y + pk.r_amb_c_per_y : pk.r_hs_c_per_x + pk.r_amb_c_per_x);
    lnk(cN[s], sN[s], y ? pk.r_sp_per_y : pk.r_sp_per_x);
    lnk(cN[s], oN[s], r_hs2);
    P->invC[cN[s]] = 1.0 / (y ? pk.c_hs_c_per_y + pk.c_amb_c_per_y : pk.c_hs_c_per_x + pk.c_amb_c_per_x);
    edge(sN[s], 4 + s, y ? L[m->spidx].edgeNS : L[m->spidx].edgeEW);
    lnk(sN[s], cN[s], y ? pk.r_sp_per_y : pk.r_sp_per_x);
    P->invC[sN[s]] = 1.0 / (y ? pk.c_sp_per_y : pk.c_sp_per_x);
  }
  if (m->nx > HSB_EXTRA) {
    const int pO[4] = {HSB_PCB_N, HSB_PCB_S, HSB_PCB_W, HSB_PCB_E};
    const int pC[4] = {HSB_PCB_C_N, HSB_PCB_C_S, HSB_PCB_C_W, HSB_PCB_C_E};
    const int sO[4] = {HSB_SOLDER_N, HSB_SOLDER_S, HSB_SOLDER_W, HSB_SOLDER_E};
    const int bO[4] = {HSB_SUB_N, HSB_SUB_S, HSB_SUB_W, HSB_SUB_E};
    for (int s = 0; s < 4; s++) {
      const bool y = s < 2;
      const double r_p2 = (y ? pk.r_pcb2_y : pk.r_pcb2_x) + pk.r_pcb;
      P->gamb[pO[s]] = 1.0 / pk.r_amb_sec_per;
      lnk(pO[s], pC[s], r_p2);
      P->invC[pO[s]] = 1.0 / (pk.c_pcb_per + pk.c_amb_sec_per);
      edge(pC[s], 8 + s, y ? L[m->pcbidx].edgeNS : L[m->pcbidx].edgeEW);
      P->gamb[pC[s]] = 1.0 / (y ? pk.r_amb_sec_c_per_y : pk.r_amb_sec_c_per_x);
      lnk(pC[s], sO[s], y ? pk.r_pcb_c_per_y : pk.r_pcb_c_per_x);
      lnk(pC[s], pO[s], r_p2);
      P->invC[pC[s]] = 1.0 / (y ? pk.c_pcb_c_per_y + pk.c_amb_sec_c_per_y : pk.c_pcb_c_per_x + pk.c_amb_sec_c_per_x);
      edge(sO[s], 12 + s, y ? L[m->solderidx].edgeNS : L[m->solderidx].edgeEW);
      lnk(sO[s], pC[s], y ? pk.r_pcb_c_per_y : pk.r_pcb_c_per_x);
      P->invC[sO[s]] = 1.0 / (y ? pk.c_solder_per_y : pk.c_solder_per_x);
      edge(bO[s], 16 + s, y ? L[m->subidx].edgeNS : L[m->subidx].edgeEW);
      lnk(bO[s], sO[s], y ? pk.r_solder_per_y : pk.r_solder_per_x);
      P->invC[bO[s]] = 1.0 / (y ? pk.c_sub_per_y : pk.c_sub_per_x);
    }
  }
}

static int segmax_of(const hsb_dev_model *m) {
  const int ntj = (m->nc + TJ - 1) / TJ, nti = (m->nr + TI - 1) / TI;
  return ntj > nti ? ntj : nti;
}

// co-resident grid of a cooperative launch over the model's tiles
static int coop_grid(const hsb_dev_model *m, const void *fn, size_t smem, int *grid) {
  { const int rc0 = raise_smem_limit(fn, smem); if (rc0) return rc0; }
  int per_sm = 0, nsm = 0;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, m->device);
  HSB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, FT_THREADS, smem));
  if (per_sm < 1) return set_error(HSB_E_ARG, "fast transient kernel does not fit an SM");
  const long long tiles = (long long)((m->nc + TJ - 1) / TJ) * ((m->nr + TI - 1) / TI);
  long long g = (long long)per_sm * nsm;
  if (g > tiles) g = tiles;
  *grid = (int)g;
  return HSB_OK;
}

int fast_prepare(hsb_dev_model *m, FastWork **out);
// stage-by-stage fast RK4 over [0, T) starting from step size h0
int rk4_stage_run(hsb_dev_model *m, FastWork *w, double T, double h0, hsb_stats *st);
// the fast transient's kernel for the model (temporally blocked where it
// applies, else the Krylov vectors and their tensor maps, allocated once)
int kry_prepare(hsb_dev_model *m, FastWork *w);
// the pass-by-pass kernel's Krylov vectors and tensor maps, whatever the model
int kry_prepare_vectors(hsb_dev_model *m, FastWork *w);
// K intervals in one launch from K device block-power vectors; *done = the
// intervals completed (< K: the rejection budget ran out in interval *done at
// *t_done, continue with step size *h_next)
int rk4_krylov_trace(hsb_dev_model *m, FastWork *w, const double *bpow, int K, double T, hsb_stats *st, int *done,
                     double *t_done, double *h_next);
// the two halves of a launch: enqueue (kernel + counters to the host, no
// wait) and complete (after the stream reached the counters)
int rk4_krylov_enqueue(hsb_dev_model *m, FastWork *w, double T, hsb_stats *st, const double *bpow, int K);
int rk4_krylov_complete(hsb_dev_model *m, FastWork *w, double T, hsb_stats *st, double *t_done, double *h_next,
                        int *done);

}  // namespace hsb
