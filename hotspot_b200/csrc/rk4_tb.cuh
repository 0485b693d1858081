// rk4_tb.cuh -- descriptors of the temporally blocked fast transient kernel
// (rk4_tb.cu), shared with the single-model launcher (rk4_krylov.cu) and the
// batch (rk4_batch.cu).
#pragma once
#include "fast_common.cuh"

namespace hsb {

#define TB_THREADS 512
#define TB_WARPS (TB_THREADS / 32)
#define TB_NLMIN 3
#define TB_NLMAX 12
#define TB_DMAX 27            // highest Krylov degree in the kernel (first attempt 7, +4 per rejection)
#define TB_JMAX (TB_DMAX - 1) // edge-response table depth: L_cc^j, j < TB_JMAX
#define TB_OUT 8              // per-chip result words (layout of FastWork::cnt)
#define TB_BAR_LIMIT (1 << 25)

// own cells per thread (the kernel's FP64 accumulator slots): two for the
// FP32 kernel on up to six layers, else one; a tile or sub-tile holds at most
// TB_THREADS x that many own cells
__host__ __device__ inline int tb_slots_rt(bool fp64, int nl) { return (!fp64 && nl <= 6) ? 2 : 1; }

// FP32 layer coefficients as the kernel reads them: two float4 loads
struct alignas(16) TLayer {
  float gNS, gEW, gDn, invC;        // lateral, to the layer below, 1/C
  float gEdgeNS, gEdgeEW, gAmb;     // to the package node at the boundary, to ambient (sink, PCB)
  int nbase;                        // W node of this layer's package group (W, E, N, S), -1: none
};

// the same in FP64, for the all-FP64 variant of the kernel
struct alignas(16) TLayerD {
  double gNS, gEW, gDn, invC, gEdgeNS, gEdgeEW, gAmb;
  int nbase, pad;
};

// one chip (model) as the kernel sees it
struct TChip {
  double *y[2];                     // state buffers: y[out[6]] holds the state at launch
  float *pf;                        // FP32 grid power (FP32 kernel)
  double *pd;                       // FP64 grid power (FP64 kernel; a scratch vector of ncell doubles)
  double *pgrid;                    // FP64 grid power (K = 0: source; K > 0: the last interval's, written)
  const int *b2g_ptr, *b2g_blk;
  const double *b2g_occ, *b2g_area;
  double cell_area;
  const TLayer *L;
  const TLayerD *Ld;
  const PackF *pk;
  const double *er;                 // [TB_JMAX][ne][ne] edge responses
  double *part;                     // [TB_DMAX + 1][NEDGE][segmax] per-tile edge sums
  double *ea;                       // [ncell] error sums of the A part at cells the package reaches
  unsigned long long *err;          // [3] rotating error-norm slots
  unsigned *bar;                    // [2] chip barrier: arrivals, generation
  long long ncell, plane;
  double ambient;
  int nl, nr, nc, nx, ne;
  int eg_layer[5], eg_node[5];      // per package group: its layer (-1: absent), its W node
  int oi, oj, nti, ntj, ntiles;     // own tiles
  int segmax;
  int rcap;                         // region cells per layer of one buffer
};

// per-model resources
struct TbRes {
  TLayer *L;
  TLayerD *Ld;
  PackF *pk;
  double *er;
  double *part;
  double *ea;
  unsigned long long *err;
  unsigned *bar;
  TChip *d_chip;                    // [variant * 2 + role]: FP32 / FP64 kernel; state in the first buffer / second
  const double *chip_y0, *chip_y1;  // the buffers d_chip[v * 2] describes (y, ytemp)
  int chip_oi[2], chip_oj[2];       // per variant: own tile (0: not chosen yet)
  int version, ne, segmax;
  int eg_layer[5], eg_node[5];
  size_t cap;                       // the device's shared memory per CTA (opt-in)
  int grid[2];                      // per variant: co-resident CTAs of a single-model launch
  size_t dyn[2];                    // per variant: dynamic shared memory of that launch
};

// fp64: the all-FP64 variant (stencil passes in FP64 too)
bool tb_eligible(const hsb_dev_model *m);
const void *tb_kernel(bool fp64 = false);
size_t tb_static_smem(bool fp64 = false);
int tb_rcap(int nl, int oi, int oj, bool fp64, size_t smem_cap);
size_t tb_dyn_smem(int nl, int oi, int oj, bool fp64, size_t smem_cap);
int tb_tile_for(int nl, int nr, int nc, int ctas, size_t smem_cap, int *oi, int *oj, bool fp64 = false);
double tb_tile_work(int oi, int oj);
int tb_res_prepare(hsb_dev_model *m, TbRes **r, const PackF *pk_dev);
void tb_res_free(TbRes *r);
int tb_fill_chip(hsb_dev_model *m, TbRes *r, const double *y0, const double *y1, float *pf, double *pd, int oi,
                 int oj, bool fp64, size_t smem_cap, TChip *C);

}  // namespace hsb
