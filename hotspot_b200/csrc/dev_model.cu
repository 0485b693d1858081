// dev_model.cu -- the device model object, block<->grid translation and the
// hsb_dev_* C-ABI entry points (declared in include/hsb_device.h).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>

#include "dev_model.cuh"

namespace hsb {

static thread_local std::string g_err;

int set_error(int code, const std::string &msg) {
  g_err = msg;
  return code;
}

int cuda_check(cudaError_t e, const char *what) {
  return set_error(e == cudaErrorMemoryAllocation ? HSB_E_NOMEM : HSB_E_CUDA,
                   std::string(what) + ": " + cudaGetErrorString(e));
}

// The dynamic shared memory limit is a per-function (per-device) setting
// shared by every thread and model: it is only ever raised, under a lock, so
// a model needing less can never lower it below what another model in
// flight launched with.
int raise_smem_limit(const void *fn, size_t bytes) {
  static std::mutex mu;
  static std::map<std::pair<int, const void *>, size_t> cur;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(mu);
  size_t &have = cur[{dev, fn}];
  if (bytes <= have) return HSB_OK;
  const cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();   // a refused attribute must not surface again in a later check
    return cuda_check(e, "cudaFuncSetAttribute(MaxDynamicSharedMemorySize)");
  }
  have = bytes;
  return HSB_OK;
}

StencilArgs make_args(const hsb_dev_model *m, const LayerCoef *L, int nr, int nc) {
  StencilArgs A;
  A.nl = m->nl;
  A.nr = nr;
  A.nc = nc;
  A.nx = m->nx;
  A.plane = (long long)nr * nc;
  A.ncell = A.plane * m->nl;
  A.field = m->field;
  A.secondary = m->nx > HSB_EXTRA;
  A.uchan_mask = m->uchan_mask;
  A.ambient = m->ambient;
  A.L = L;
  A.pk = m->pk;
  A.rN = m->rN; A.rS = m->rS; A.rW = m->rW; A.rE = m->rE; A.rA = m->rA; A.rB = m->rB;
  A.cap = m->cap;
  A.aN = m->aN; A.aS = m->aS; A.aW = m->aW; A.aE = m->aE; A.aO = m->aO; A.qin = m->qin;
  return A;
}

// ---------------------------------------------------------------------------
// block -> grid (xlate_vector_b2g, temperature_grid.c:1888-1929)
// ---------------------------------------------------------------------------
__global__ void b2g_kernel(const int *__restrict__ ptr, const int *__restrict__ blk,
                           const double *__restrict__ occ, const double *__restrict__ area,
                           const double *__restrict__ b, double *__restrict__ g,
                           long long ncell, int nx, int nblk, double cell_area, int type) {
  long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c < ncell) {
    double val = 0.0;
    const int e0 = ptr[c], e1 = ptr[c + 1];
    if (type == HSB_V_POWER) {
      for (int e = e0; e < e1; e++) val += occ[e] * b[blk[e]] / area[e];   // blist_avg :331
      g[c] = val * cell_area;
    } else {
      for (int e = e0; e < e1; e++) val += occ[e] * b[blk[e]];             // :334
      g[c] = val;
    }
  } else if (c < ncell + nx) {
    g[c] = b[nblk + (c - ncell)];
  }
}

// grid -> block (xlate_temp_g2b, temperature_grid.c:1932-2015)
__device__ __forceinline__ void g2b_one(const int *__restrict__ map, const double *__restrict__ g,
                                        double *__restrict__ b, int nblk, int nx, int nr, int nc, long long ncell,
                                        int mode, int u) {
  if (u < nblk) {
    const int n = map[5 * u], i1 = map[5 * u + 1], i2 = map[5 * u + 2];
    const int j1 = map[5 * u + 3], j2 = map[5 * u + 4];
    const double *G = g + (long long)n * nr * nc;
    if (mode == HSB_GRID_CENTER) {
      const int ci1 = (i1 + i2) / 2, cj1 = (j1 + j2) / 2;
      const int ci2 = ci1 - !((i2 - i1) % 2), cj2 = cj1 - !((j2 - j1) % 2);
      b[u] = (G[ci1 * nc + cj1] + G[ci2 * nc + cj1] + G[ci1 * nc + cj2] + G[ci2 * nc + cj2]) / 4;
      return;
    }
    double avg = 0.0, mn, mx;
    int count = 0;
    mn = mx = G[i1 * nc + j1];
    for (int i = i1; i < i2; i++)
      for (int j = j1; j < j2; j++) {
        const double v = G[i * nc + j];
        avg += v;
        if (v < mn) mn = v;
        if (v > mx) mx = v;
        count++;
      }
    b[u] = mode == HSB_GRID_AVG ? avg / count : mode == HSB_GRID_MIN ? mn : mx;
  } else if (u < nblk + nx) {
    b[u] = g[ncell + (u - nblk)];
  }
}

__global__ void g2b_kernel(const int *__restrict__ map, const double *__restrict__ g,
                           double *__restrict__ b, int nblk, int nx, int nr, int nc,
                           long long ncell, int mode) {
  g2b_one(map, g, b, nblk, nx, nr, nc, ncell, mode, blockIdx.x * blockDim.x + threadIdx.x);
}

// the same on whichever of g0 / g1 the device word *which selects
__global__ void g2b_select_kernel(const int *__restrict__ map, const double *__restrict__ g0,
                                  const double *__restrict__ g1, const long long *__restrict__ which,
                                  double *__restrict__ b, int nblk, int nx, int nr, int nc, long long ncell,
                                  int mode) {
  g2b_one(map, *which ? g1 : g0, b, nblk, nx, nr, nc, ncell, mode, blockIdx.x * blockDim.x + threadIdx.x);
}

int b2g(hsb_dev_model *m, const double *blk_dev, double *grid_dev, int type) {
  return b2g_on(m, blk_dev, grid_dev, type, m->stream);
}

int b2g_on(hsb_dev_model *m, const double *blk_dev, double *grid_dev, int type, cudaStream_t s) {
  const long long n = m->vlen;
  const int T = 256;
  b2g_kernel<<<(unsigned)((n + T - 1) / T), T, 0, s>>>(
      m->b2g_ptr, m->b2g_blk, m->b2g_occ, m->b2g_area, blk_dev, grid_dev, m->ncell, m->nx,
      m->total_n_blocks, m->cell_area, type);
  HSB_CUDA(cudaGetLastError());
  return HSB_OK;
}

int g2b(hsb_dev_model *m, const double *grid_dev, double *blk_dev) {
  return g2b_on(m, grid_dev, blk_dev, m->stream);
}

int g2b_select(hsb_dev_model *m, const double *g0, const double *g1, const long long *which, double *blk_dev) {
  const int n = m->total_n_blocks + m->nx, T = 128;
  g2b_select_kernel<<<(n + T - 1) / T, T, 0, m->stream>>>(m->g2b, g0, g1, which, blk_dev, m->total_n_blocks,
                                                          m->nx, m->nr, m->nc, m->ncell, m->map_mode);
  HSB_CUDA(cudaGetLastError());
  return HSB_OK;
}

int g2b_on(hsb_dev_model *m, const double *grid_dev, double *blk_dev, cudaStream_t s) {
  const int n = m->total_n_blocks + m->nx, T = 128;
  g2b_kernel<<<(n + T - 1) / T, T, 0, s>>>(m->g2b, grid_dev, blk_dev, m->total_n_blocks,
                                                   m->nx, m->nr, m->nc, m->ncell, m->map_mode);
  HSB_CUDA(cudaGetLastError());
  return HSB_OK;
}

static void fill_layer_table(const hsb_dev_model *m, LayerCoef *L, int nr, int nc, double rz_div,
                             double c_mul) {
  const package_RC_t &pk = m->h_pk;
  for (int n = 0; n < m->nl; n++) {
    LayerCoef &l = L[n];
    memset(&l, 0, sizeof(l));
    const double rx = m->h_rx[n], ry = m->h_ry[n];
    // multigrid coarsening divides rz by 4 and multiplies c by 4 per level
    // (temperature_grid.c:2753-2757); both are exact power-of-two scalings
    l.rz = m->h_rz[n] / rz_div;
    l.cap = m->h_c[n] * c_mul;
    l.ramb = l.rz;
    l.rNS = rx / 2.0 + rx / 2.0;   // find_res, temperature_grid.c:123-125
    l.rEW = ry / 2.0 + ry / 2.0;   // :126-128
    l.kind = LK_PLAIN;
    if (n == m->spidx) {
      l.kind = LK_SPREADER;
      l.edgeNS = ry / 2.0 + nc * pk.r_sp1_y;
      l.edgeEW = rx / 2.0 + nr * pk.r_sp1_x;
    } else if (n == m->hsidx) {
      l.kind = LK_SINK;
      l.edgeNS = ry / 2.0 + nc * pk.r_hs1_y;
      l.edgeEW = rx / 2.0 + nr * pk.r_hs1_x;
    } else if (m->nx > HSB_EXTRA && n == m->pcbidx) {
      l.kind = LK_PCB;
      l.edgeNS = ry / 2.0 + nc * pk.r_pcb1_y;
      l.edgeEW = rx / 2.0 + nr * pk.r_pcb1_x;
      // r_convec_sec * (s_pcb * s_pcb) / (cw * ch) at this level's cell size
      // (temperature_grid.c:2562-2565, 3212-3214)
      const double cw = m->width / nc, ch = m->height / nr;
      l.ramb = m->pcb_amb_num / (cw * ch);
    } else if (m->nx > HSB_EXTRA && n == m->subidx) {
      l.kind = LK_SUB;
      l.edgeNS = ry / 2.0 + nc * pk.r_sub1_y;
      l.edgeEW = rx / 2.0 + nr * pk.r_sub1_x;
    } else if (m->nx > HSB_EXTRA && n == m->solderidx) {
      l.kind = LK_SOLDER;
      l.edgeNS = ry / 2.0 + nc * pk.r_solder1_y;
      l.edgeEW = rx / 2.0 + nr * pk.r_solder1_x;
    }
  }
}

int upload_layers(hsb_dev_model *m) {
  m->coef_version++;
  fill_layer_table(m, m->hostL0, m->nr, m->nc, 1.0, 1.0);
  HSB_CUDA(cudaMemcpyAsync(m->L0, m->hostL0, sizeof(LayerCoef) * m->nl, cudaMemcpyHostToDevice,
                           m->stream));
  HSB_CUDA(cudaMemcpyAsync(m->pk, &m->h_pk, sizeof(package_RC_t), cudaMemcpyHostToDevice,
                           m->stream));
  // coarse levels of the nested-iteration multigrid
  for (int l = 0; l < m->n_levels; l++) {
    LevelBuf &lv = m->levels[l];
    fill_layer_table(m, lv.hostL, lv.nr, lv.nc, 1.0, 1.0);
    // apply the repeated in-place /4 and *4 exactly as the recursion does
    for (int n = 0; n < m->nl; n++) {
      double rz = m->h_rz[n], c = m->h_c[n];
      for (int k = 0; k < l; k++) { rz /= 4; c *= 4; }
      lv.hostL[n].rz = rz;
      lv.hostL[n].cap = c;
      if (lv.hostL[n].kind == LK_SINK) lv.hostL[n].ramb = rz;
    }
    HSB_CUDA(cudaMemcpyAsync(lv.L, lv.hostL, sizeof(LayerCoef) * m->nl, cudaMemcpyHostToDevice,
                             m->stream));
  }
  HSB_CUDA(cudaStreamSynchronize(m->stream));
  return HSB_OK;
}

static void free_model(hsb_dev_model *m) {
  if (!m) return;
  if (m->fast && m->fast_free) m->fast_free(m->fast);
  if (m->mg && m->mg_free) m->mg_free(m->mg);
  if (m->krylov && m->krylov_free) m->krylov_free(m->krylov);
  double **bufs[] = {&m->y, &m->ys, &m->pgrid, &m->k1, &m->k2, &m->k3, &m->ytemp, &m->t1, &m->t2,
                     &m->rN, &m->rS, &m->rW, &m->rE, &m->rA, &m->rB, &m->cap, &m->aN, &m->aS,
                     &m->aW, &m->aE, &m->aO, &m->qin, &m->b2g_occ, &m->b2g_area, &m->blk_in,
                     &m->blk_out, &m->gs_delta, &m->trace_buf};
  for (double **b : bufs)
    if (*b) cudaFree(*b);
  if (m->errbits) cudaFree(m->errbits);
  if (m->pk) cudaFree(m->pk);
  if (m->L0) cudaFree(m->L0);
  if (m->b2g_ptr) cudaFree(m->b2g_ptr);
  if (m->b2g_blk) cudaFree(m->b2g_blk);
  if (m->g2b) cudaFree(m->g2b);
  if (m->gs_status) cudaFree(m->gs_status);
  if (m->h_err) cudaFreeHost(m->h_err);
  if (m->h_blk) cudaFreeHost(m->h_blk);
  for (auto &g : m->ivg)
    if (g.exec) cudaGraphExecDestroy(g.exec);
  if (m->ev[0]) cudaEventDestroy(m->ev[0]);
  if (m->ev[1]) cudaEventDestroy(m->ev[1]);
  if (m->h_gs) cudaFreeHost(m->h_gs);
  if (m->h_gsd) cudaFreeHost(m->h_gsd);
  if (m->levels) {
    for (int l = 1; l < m->n_levels; l++) {
      if (m->levels[l].p) cudaFree(m->levels[l].p);
      if (m->levels[l].v) cudaFree(m->levels[l].v);
    }
    for (int l = 0; l < m->n_levels; l++)
      if (m->levels[l].L) cudaFree(m->levels[l].L);
    delete[] m->levels;
  }
  if (m->stream) cudaStreamDestroy(m->stream);
  delete m;
}

}  // namespace hsb

using namespace hsb;

extern "C" {

const char *hsb_dev_last_error(void) { return g_err.c_str(); }

int hsb_dev_create(hsb_dev_model **out, const hsb_grid_desc *d) {
  if (!out || !d) return set_error(HSB_E_ARG, "null argument");
  *out = nullptr;
  if (d->nl < 1 || d->nl > HSB_MAX_LAYERS || d->nr < 1 || d->nc < 1)
    return set_error(HSB_E_ARG, "invalid grid dimensions");
  if (d->n_extra != HSB_EXTRA && d->n_extra != HSB_EXTRA + HSB_EXTRA_SEC)
    return set_error(HSB_E_ARG, "n_extra must be 12 or 28");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1)
    return set_error(HSB_E_NODEV, "no CUDA device visible to libhotspot_b200");
  hsb_dev_model *m = new hsb_dev_model();
  memset(m, 0, sizeof(*m));
  m->nl = d->nl; m->nr = d->nr; m->nc = d->nc; m->nx = d->n_extra;
  m->plane = (long long)d->nr * d->nc;
  m->ncell = m->plane * d->nl;
  m->vlen = m->ncell + m->nx;
  m->spidx = d->spidx; m->hsidx = d->hsidx;
  m->subidx = d->subidx; m->solderidx = d->solderidx; m->pcbidx = d->pcbidx;
  m->field = d->field; m->map_mode = d->map_mode; m->total_n_blocks = d->total_n_blocks;
  cudaGetDevice(&m->device);
  int rc;
#define ALLOC(p, bytes)                                                       \
  do {                                                                        \
    cudaError_t e_ = cudaMalloc((void **)&(p), (bytes));                      \
    if (e_ != cudaSuccess) { rc = cuda_check(e_, "cudaMalloc " #p); goto fail; } \
  } while (0)
  {
    cudaError_t e = cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) { rc = cuda_check(e, "cudaStreamCreate"); goto fail; }
    if ((e = cudaEventCreate(&m->ev[0])) != cudaSuccess || (e = cudaEventCreate(&m->ev[1])) != cudaSuccess) {
      rc = cuda_check(e, "cudaEventCreate");
      goto fail;
    }
  }
  {
    const size_t vb = sizeof(double) * (size_t)m->vlen;
    ALLOC(m->y, vb); ALLOC(m->ys, vb); ALLOC(m->pgrid, vb);
    ALLOC(m->k1, vb); ALLOC(m->k2, vb); ALLOC(m->k3, vb);
    ALLOC(m->ytemp, vb); ALLOC(m->t1, vb); ALLOC(m->t2, vb);
    cudaMemsetAsync(m->y, 0, vb, m->stream);
    cudaMemsetAsync(m->ys, 0, vb, m->stream);
    ALLOC(m->errbits, sizeof(unsigned long long));
    ALLOC(m->pk, sizeof(package_RC_t));
    ALLOC(m->L0, sizeof(LayerCoef) * HSB_MAX_LAYERS);
    const size_t bb = sizeof(double) * (size_t)(d->total_n_blocks + d->n_extra);
    ALLOC(m->blk_in, 2 * bb);
    ALLOC(m->blk_out, bb);
    ALLOC(m->gs_status, 4 * sizeof(int));
    ALLOC(m->gs_delta, 4 * sizeof(double));
    if (cudaMallocHost((void **)&m->h_err, sizeof(double) * 4) != cudaSuccess ||
        cudaMallocHost((void **)&m->h_gs, 4 * sizeof(int)) != cudaSuccess ||
        cudaMallocHost((void **)&m->h_gsd, 4 * sizeof(double)) != cudaSuccess ||
        cudaMallocHost((void **)&m->h_blk, 3 * bb) != cudaSuccess) {
      rc = set_error(HSB_E_NOMEM, "cudaMallocHost failed");
      goto fail;
    }
  }
  // nested-iteration levels: halve rows and cols until either reaches 1
  // (recursive_multigrid, temperature_grid.c:2733-2797)
  {
    int nr = d->nr, nc = d->nc, n = 1;
    while (nr > 1 && nc > 1) { nr /= 2; nc /= 2; n++; }
    m->n_levels = n;
    m->levels = new LevelBuf[n];
    memset(m->levels, 0, sizeof(LevelBuf) * n);
    nr = d->nr; nc = d->nc;
    for (int l = 0; l < n; l++) {
      LevelBuf &lv = m->levels[l];
      lv.nr = nr; lv.nc = nc;
      ALLOC(lv.L, sizeof(LayerCoef) * HSB_MAX_LAYERS);
      if (l == 0) {
        lv.p = m->pgrid;
        lv.v = m->ys;
      } else {
        const size_t b = sizeof(double) * ((size_t)nr * nc * d->nl + d->n_extra);
        ALLOC(lv.p, b);
        ALLOC(lv.v, b);
      }
      nr /= 2; nc /= 2;
    }
  }
#undef ALLOC
  *out = m;
  if (d->layer_rx) {
    rc = hsb_dev_set_layers(m, d->layer_rx, d->layer_ry, d->layer_rz, d->layer_c, d->pack,
                            d->ambient, d->width, d->height, d->pcb_amb_num);
    if (rc) { *out = nullptr; free_model(m); return rc; }
  }
  return HSB_OK;
fail:
  free_model(m);
  return rc;
}

void hsb_dev_destroy(hsb_dev_model *m) {
  if (m) {
    cudaStreamSynchronize(m->stream);
    free_model(m);
  }
}

int hsb_dev_set_layers(hsb_dev_model *m, const double *rx, const double *ry, const double *rz,
                       const double *c, const double *pack52, double ambient, double width,
                       double height, double pcb_amb_num) {
  if (!m || !rx || !ry || !rz || !pack52) return set_error(HSB_E_ARG, "null argument");
  for (int n = 0; n < m->nl; n++) {
    m->h_rx[n] = rx[n];
    m->h_ry[n] = ry[n];
    m->h_rz[n] = rz[n];
    m->h_c[n] = c ? c[n] : 0.0;
  }
  memcpy(&m->h_pk, pack52, sizeof(package_RC_t));
  m->ambient = ambient;
  m->width = width;
  m->height = height;
  m->pcb_amb_num = pcb_amb_num;
  return upload_layers(m);
}

static int upload_array(hsb_dev_model *m, double **dst, const double *src, size_t n) {
  if (!src) return HSB_OK;
  if (!*dst) HSB_CUDA(cudaMalloc((void **)dst, sizeof(double) * n));
  HSB_CUDA(cudaMemcpyAsync(*dst, src, sizeof(double) * n, cudaMemcpyHostToDevice, m->stream));
  return HSB_OK;
}

int hsb_dev_set_cells(hsb_dev_model *m, const double *rN, const double *rS, const double *rW,
                      const double *rE, const double *rA, const double *rB, const double *cap) {
  if (!m) return set_error(HSB_E_ARG, "null model");
  const size_t n = (size_t)m->ncell;
  int rc;
  if ((rc = upload_array(m, &m->rN, rN, n)) || (rc = upload_array(m, &m->rS, rS, n)) ||
      (rc = upload_array(m, &m->rW, rW, n)) || (rc = upload_array(m, &m->rE, rE, n)) ||
      (rc = upload_array(m, &m->rA, rA, n)) || (rc = upload_array(m, &m->rB, rB, n)) ||
      (rc = upload_array(m, &m->cap, cap, n)))
    return rc;
  m->field = 1;
  m->coef_version++;
  HSB_CUDA(cudaStreamSynchronize(m->stream));
  return HSB_OK;
}

int hsb_dev_set_advection(hsb_dev_model *m, const double *aN, const double *aS, const double *aW,
                          const double *aE, const double *aO, const double *qin) {
  if (!m || !aN || !aS || !aW || !aE || !aO || !qin) return set_error(HSB_E_ARG, "null argument");
  const size_t n = (size_t)m->ncell;
  int rc;
  if ((rc = upload_array(m, &m->aN, aN, n)) || (rc = upload_array(m, &m->aS, aS, n)) ||
      (rc = upload_array(m, &m->aW, aW, n)) || (rc = upload_array(m, &m->aE, aE, n)) ||
      (rc = upload_array(m, &m->aO, aO, n)) || (rc = upload_array(m, &m->qin, qin, n)))
    return rc;
  // a layer takes the advection path when any of its coefficients is non-zero
  unsigned long long mask = 0;
  for (int l = 0; l < m->nl; l++) {
    const size_t o = (size_t)l * m->plane;
    for (size_t k = 0; k < (size_t)m->plane; k++)
      if (aN[o + k] != 0 || aS[o + k] != 0 || aW[o + k] != 0 || aE[o + k] != 0 ||
          aO[o + k] != 0 || qin[o + k] != 0) {
        mask |= 1ull << l;
        break;
      }
  }
  m->uchan_mask = mask;
  m->coef_version++;
  HSB_CUDA(cudaStreamSynchronize(m->stream));
  return HSB_OK;
}

int hsb_dev_set_maps(hsb_dev_model *m, const int *b2g_ptr, const int *b2g_blk,
                     const double *b2g_occ, const double *b2g_area, double cell_area,
                     const int *g2b) {
  if (!m || !b2g_ptr || !g2b) return set_error(HSB_E_ARG, "null argument");
  const int nnz = b2g_ptr[m->ncell];
  if (m->b2g_ptr) { cudaFree(m->b2g_ptr); m->b2g_ptr = nullptr; }
  if (m->b2g_blk) { cudaFree(m->b2g_blk); m->b2g_blk = nullptr; }
  if (m->b2g_occ) { cudaFree(m->b2g_occ); m->b2g_occ = nullptr; }
  if (m->b2g_area) { cudaFree(m->b2g_area); m->b2g_area = nullptr; }
  if (!m->g2b) HSB_CUDA(cudaMalloc((void **)&m->g2b, sizeof(int) * 5 * (m->total_n_blocks + 1)));
  HSB_CUDA(cudaMalloc((void **)&m->b2g_ptr, sizeof(int) * (m->ncell + 1)));
  HSB_CUDA(cudaMalloc((void **)&m->b2g_blk, sizeof(int) * (nnz + 1)));
  HSB_CUDA(cudaMalloc((void **)&m->b2g_occ, sizeof(double) * (nnz + 1)));
  HSB_CUDA(cudaMalloc((void **)&m->b2g_area, sizeof(double) * (nnz + 1)));
  HSB_CUDA(cudaMemcpyAsync(m->b2g_ptr, b2g_ptr, sizeof(int) * (m->ncell + 1),
                           cudaMemcpyHostToDevice, m->stream));
  if (nnz) {
    HSB_CUDA(cudaMemcpyAsync(m->b2g_blk, b2g_blk, sizeof(int) * nnz, cudaMemcpyHostToDevice, m->stream));
    HSB_CUDA(cudaMemcpyAsync(m->b2g_occ, b2g_occ, sizeof(double) * nnz, cudaMemcpyHostToDevice, m->stream));
    HSB_CUDA(cudaMemcpyAsync(m->b2g_area, b2g_area, sizeof(double) * nnz, cudaMemcpyHostToDevice, m->stream));
  }
  HSB_CUDA(cudaMemcpyAsync(m->g2b, g2b, sizeof(int) * 5 * m->total_n_blocks, cudaMemcpyHostToDevice,
                           m->stream));
  m->cell_area = cell_area;
  // new map arrays: whatever captured the old pointers (interval graphs,
  // derived tables) is rebuilt on next use
  m->coef_version++;
  HSB_CUDA(cudaStreamSynchronize(m->stream));
  return HSB_OK;
}

// The fast form's interval replayed from a CUDA graph: the block powers
// from pinned staging, the Krylov kernel (which maps them to the grid
// itself), its counters to the host, g2b of the state buffer the kernel
// ended in and the block temperatures back to staging -- one launch and one
// wait per interval.  Returns 1, having done nothing, when the sequence
// cannot be captured; the caller then launches step by step.
static int fast_interval_graphed(hsb_dev_model *m, const double *block_power, double T, double *block_temp_out,
                                 hsb_stats *st) {
  const size_t nb = (size_t)m->total_n_blocks + m->nx;
  void *work = nullptr;
  const void *fn = nullptr;
  int rc;
  if ((rc = rk4_fast_ready(m, &work, &fn))) return rc;
  const int want = block_temp_out != nullptr;
  double *second = nullptr;
  const long long *which = nullptr;
  fast_state_buffers(m, work, &second, &which);
  hsb_dev_model::IvGraph *g = nullptr;
  for (auto &e : m->ivg)
    if (e.exec && e.y == m->y && e.y2 == second && e.T == T && e.out == want && e.version == m->coef_version &&
        e.fn == fn && e.mode == m->map_mode)
      g = &e;
  if (!g) {
    g = &m->ivg[m->ivg_next];
    m->ivg_next = (m->ivg_next + 1) % 4;
    if (g->exec) cudaGraphExecDestroy(g->exec);
    g->exec = nullptr;
    hsb_stats scratch;
    memset(&scratch, 0, sizeof(scratch));
    if (cudaStreamBeginCapture(m->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
      cudaGetLastError();
      m->ivg_off = 1;
      return 1;
    }
    bool ok = cudaMemcpyAsync(m->blk_in, m->h_blk, sizeof(double) * nb, cudaMemcpyHostToDevice, m->stream) ==
              cudaSuccess;
    void *w2 = nullptr;
    ok = ok && rk4_fast_interval_begin(m, T, &scratch, &w2, m->blk_in) == HSB_OK;
    if (ok && want) {
      ok = g2b_select(m, m->y, second, which, m->blk_out) == HSB_OK &&
           cudaMemcpyAsync(m->h_blk + nb, m->blk_out, sizeof(double) * nb, cudaMemcpyDeviceToHost, m->stream) ==
               cudaSuccess;
    }
    cudaGraph_t graph = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(m->stream, &graph);
    if (!ok || ce != cudaSuccess || !graph || cudaGraphInstantiate(&g->exec, graph, 0) != cudaSuccess) {
      if (graph) cudaGraphDestroy(graph);
      g->exec = nullptr;
      cudaGetLastError();
      m->ivg_off = 1;
      return 1;
    }
    cudaGraphDestroy(graph);
    g->y = m->y;
    g->y2 = second;
    g->T = T;
    g->out = want;
    g->version = m->coef_version;
    g->fn = fn;
    g->mode = m->map_mode;
  }
  memcpy(m->h_blk, block_power, sizeof(double) * nb);
  HSB_CUDA(cudaEventRecord(m->ev[0], m->stream));
  HSB_CUDA(cudaGraphLaunch(g->exec, m->stream));
  HSB_CUDA(cudaEventRecord(m->ev[1], m->stream));
  HSB_CUDA(cudaStreamSynchronize(m->stream));
  st->launches += 1 + want;
  int fell_back = 0;
  if ((rc = rk4_fast_interval_end(m, work, T, st, &fell_back))) return rc;
  if (fell_back) {   // the stage form finished the interval in place of the kernel
    if (want) {
      if ((rc = g2b(m, m->y, m->blk_out))) return rc;
      st->launches += 1;
      HSB_CUDA(cudaMemcpyAsync(block_temp_out, m->blk_out, sizeof(double) * nb, cudaMemcpyDeviceToHost,
                               m->stream));
    }
    HSB_CUDA(cudaEventRecord(m->ev[1], m->stream));
    HSB_CUDA(cudaStreamSynchronize(m->stream));
  } else if (want) {
    memcpy(block_temp_out, m->h_blk + nb, sizeof(double) * nb);
  }
  float ms = 0;
  if (cudaEventElapsedTime(&ms, m->ev[0], m->ev[1]) == cudaSuccess) st->device_ms += ms;
  else cudaGetLastError();
  return HSB_OK;
}

// HSB_FORM_FAST_PASSES, HSB_FORM_FP64_BLOCKED and HSB_FORM_FAST_BLOCKED are
// the fast form's interval run by a named kernel (pass by pass; all-FP64
// blocked; blocked): record the kernel choice on the model and return the form
static int fast_form(hsb_dev_model *m, int form) {
  if (form == HSB_FORM_FAST_PASSES || form == HSB_FORM_FP64_BLOCKED || form == HSB_FORM_FAST_BLOCKED) {
    m->fast_passes = form == HSB_FORM_FAST_PASSES ? 1 : form == HSB_FORM_FP64_BLOCKED ? 2 : 3;
    return HSB_FORM_FAST;
  }
  if (form == HSB_FORM_FAST) m->fast_passes = 0;
  return form;
}

int hsb_dev_transient(hsb_dev_model *m, const double *block_power, const double *block_temp_in,
                      double time_elapsed, double *block_temp_out, const hsb_solver_opts *o,
                      hsb_stats *st) {
  if (!m || !block_power) return set_error(HSB_E_ARG, "null argument");
  if (!m->b2g_ptr) return set_error(HSB_E_ARG, "block-grid maps not set");
  const size_t nb = (size_t)m->total_n_blocks + m->nx;
  hsb_stats local;
  if (!st) st = &local;
  int rc;
  const int form = fast_form(m, o ? o->form : HSB_FORM_PARITY);
  // after the first interval (which sets up the workspace) the fast form
  // replays its interval from a graph
  if (form == HSB_FORM_FAST && !block_temp_in && m->fast && !m->ivg_off) {
    rc = fast_interval_graphed(m, block_power, time_elapsed, block_temp_out, st);
    if (rc != 1) return rc;
  }
  cudaEventRecord(m->ev[0], m->stream);
  HSB_CUDA(cudaMemcpyAsync(m->blk_in, block_power, sizeof(double) * nb, cudaMemcpyHostToDevice,
                           m->stream));
  if ((rc = b2g(m, m->blk_in, m->pgrid, HSB_V_POWER))) return rc;
  st->launches += 1;
  if (block_temp_in) {
    HSB_CUDA(cudaMemcpyAsync(m->blk_in + nb, block_temp_in, sizeof(double) * nb,
                             cudaMemcpyHostToDevice, m->stream));
    if ((rc = b2g(m, m->blk_in + nb, m->y, HSB_V_TEMP))) return rc;
    st->launches += 1;
  }
  if (form == HSB_FORM_FAST) {
    // the Krylov launch, then the block temperatures read from whichever
    // state buffer the kernel ended in (chosen on the device), one wait
    void *work = nullptr;
    if ((rc = rk4_fast_interval_begin(m, time_elapsed, st, &work, nullptr))) return rc;
    if (block_temp_out) {
      double *second;
      const long long *which;
      fast_state_buffers(m, work, &second, &which);
      if ((rc = g2b_select(m, m->y, second, which, m->blk_out))) return rc;
      st->launches += 1;
      HSB_CUDA(cudaMemcpyAsync(block_temp_out, m->blk_out, sizeof(double) * nb, cudaMemcpyDeviceToHost,
                               m->stream));
    }
    cudaEventRecord(m->ev[1], m->stream);
    HSB_CUDA(cudaStreamSynchronize(m->stream));
    int fell_back = 0;
    if ((rc = rk4_fast_interval_end(m, work, time_elapsed, st, &fell_back))) return rc;
    if (fell_back) {   // the stage form finished the interval: its state
      if (block_temp_out) {
        if ((rc = g2b(m, m->y, m->blk_out))) return rc;
        st->launches += 1;
        HSB_CUDA(cudaMemcpyAsync(block_temp_out, m->blk_out, sizeof(double) * nb, cudaMemcpyDeviceToHost,
                                 m->stream));
      }
      cudaEventRecord(m->ev[1], m->stream);
      HSB_CUDA(cudaStreamSynchronize(m->stream));
    }
  } else {
    rc = form == HSB_FORM_FAST_STAGES ? rk4_fast_stages_interval(m, time_elapsed, st)
                                      : rk4_exact_interval(m, time_elapsed, st);
    if (rc) return rc;
    if (block_temp_out) {
      if ((rc = g2b(m, m->y, m->blk_out))) return rc;
      st->launches += 1;
      HSB_CUDA(cudaMemcpyAsync(block_temp_out, m->blk_out, sizeof(double) * nb,
                               cudaMemcpyDeviceToHost, m->stream));
    }
    cudaEventRecord(m->ev[1], m->stream);
    HSB_CUDA(cudaStreamSynchronize(m->stream));
  }
  float ms = 0;
  if (cudaEventElapsedTime(&ms, m->ev[0], m->ev[1]) == cudaSuccess) st->device_ms += ms;
  else cudaGetLastError();
  return HSB_OK;
}

int hsb_dev_transient_trace(hsb_dev_model *m, const double *block_powers, int K, const double *block_temp_in,
                            double time_elapsed, double *block_temp_out, const hsb_solver_opts *o, hsb_stats *st) {
  if (!m || !block_powers || K < 1) return set_error(HSB_E_ARG, "null argument or no intervals");
  if (!m->b2g_ptr) return set_error(HSB_E_ARG, "block-grid maps not set");
  const int form = fast_form(m, o ? o->form : HSB_FORM_PARITY);
  const size_t nb = (size_t)m->total_n_blocks + m->nx;
  hsb_stats local;
  if (!st) st = &local;
  if (form != HSB_FORM_FAST) {   // the other forms: one interval per call
    for (int k = 0; k < K; k++) {
      const int rc = hsb_dev_transient(m, block_powers + k * nb, k == 0 ? block_temp_in : nullptr, time_elapsed,
                                       k == K - 1 ? block_temp_out : nullptr, o, st);
      if (rc) return rc;
    }
    return HSB_OK;
  }
  cudaEventRecord(m->ev[0], m->stream);
  int rc;
  // the block powers of all intervals, in a device buffer kept with the model
  if (m->trace_cap < (long long)(K * nb)) {
    if (m->trace_buf) cudaFree(m->trace_buf);
    m->trace_buf = nullptr;
    m->trace_cap = 0;
    HSB_CUDA(cudaMalloc(&m->trace_buf, sizeof(double) * K * nb));
    m->trace_cap = (long long)K * nb;
  }
  HSB_CUDA(cudaMemcpyAsync(m->trace_buf, block_powers, sizeof(double) * K * nb, cudaMemcpyHostToDevice, m->stream));
  if (block_temp_in) {
    HSB_CUDA(cudaMemcpyAsync(m->blk_in + nb, block_temp_in, sizeof(double) * nb, cudaMemcpyHostToDevice, m->stream));
    if ((rc = b2g(m, m->blk_in + nb, m->y, HSB_V_TEMP))) return rc;
    st->launches += 1;
  }
  if ((rc = rk4_fast_trace(m, m->trace_buf, K, time_elapsed, st))) return rc;
  if (block_temp_out) {
    if ((rc = g2b(m, m->y, m->blk_out))) return rc;
    st->launches += 1;
    HSB_CUDA(cudaMemcpyAsync(block_temp_out, m->blk_out, sizeof(double) * nb, cudaMemcpyDeviceToHost, m->stream));
  }
  cudaEventRecord(m->ev[1], m->stream);
  HSB_CUDA(cudaStreamSynchronize(m->stream));
  float ms = 0;
  if (cudaEventElapsedTime(&ms, m->ev[0], m->ev[1]) == cudaSuccess) st->device_ms += ms;
  else cudaGetLastError();
  return HSB_OK;
}

}  // extern "C"

// the steady solve from the block powers in m->blk_in (device) to the grid
// state m->ys and the block temperatures in m->blk_out (device)
int hsb::steady_core(hsb_dev_model *m, const hsb_solver_opts *o, hsb_stats *st) {
  int rc;
  if ((rc = b2g(m, m->blk_in, m->pgrid, HSB_V_POWER))) return rc;
  st->launches += 1;
  int method = o->steady_method;
  if (method == HSB_STEADY_AUTO) {
    if (m->uchan_mask) method = HSB_STEADY_BICGSTAB;
    else if (o->form != HSB_FORM_PARITY && o->form != HSB_FORM_FP64_BLOCKED)
      method = HSB_STEADY_MG;
    else method = HSB_STEADY_GS_REPLAY;
  }
  if (method == HSB_STEADY_GS_REPLAY && m->uchan_mask)
    return set_error(HSB_E_ARG,
                     "Steady-state computations with microfluidic cooling need the BiCGStab solver");
  switch (method) {
    case HSB_STEADY_GS_REPLAY: rc = gs_exact_steady(m, o, st); break;
    case HSB_STEADY_MG: rc = mg_steady(m, o, st); break;
    case HSB_STEADY_BICGSTAB: rc = bicgstab_steady(m, o, st); break;
    default: rc = set_error(HSB_E_ARG, "unknown steady method");
  }
  if (rc) return rc;
  if ((rc = g2b(m, m->ys, m->blk_out))) return rc;
  st->launches += 1;
  return HSB_OK;
}

extern "C" {

int hsb_dev_steady(hsb_dev_model *m, const double *block_power, double *block_temp_out,
                   const hsb_solver_opts *o, hsb_stats *st) {
  if (!m || !block_power) return set_error(HSB_E_ARG, "null argument");
  if (!m->b2g_ptr) return set_error(HSB_E_ARG, "block-grid maps not set");
  const size_t nb = (size_t)m->total_n_blocks + m->nx;
  hsb_stats local;
  if (!st) st = &local;
  hsb_solver_opts def = {HSB_FORM_PARITY, HSB_STEADY_AUTO, 0.0, 0};
  if (!o) o = &def;
  cudaEventRecord(m->ev[0], m->stream);
  int rc;
  HSB_CUDA(cudaMemcpyAsync(m->blk_in, block_power, sizeof(double) * nb, cudaMemcpyHostToDevice,
                           m->stream));
  if ((rc = steady_core(m, o, st))) return rc;
  if (block_temp_out)
    HSB_CUDA(cudaMemcpyAsync(block_temp_out, m->blk_out, sizeof(double) * nb,
                             cudaMemcpyDeviceToHost, m->stream));
  cudaEventRecord(m->ev[1], m->stream);
  HSB_CUDA(cudaStreamSynchronize(m->stream));
  float ms = 0;
  if (cudaEventElapsedTime(&ms, m->ev[0], m->ev[1]) == cudaSuccess) st->device_ms += ms;
  else cudaGetLastError();
  return HSB_OK;
}

int hsb_dev_set_priority(hsb_dev_model *m, int high) {
  if (!m) return set_error(HSB_E_ARG, "null model");
  int least = 0, greatest = 0;
  HSB_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
  cudaStream_t s;
  HSB_CUDA(cudaStreamCreateWithPriority(&s, cudaStreamNonBlocking, high ? greatest : least));
  HSB_CUDA(cudaStreamSynchronize(m->stream));   // nothing of the model is left in flight
  cudaStreamDestroy(m->stream);
  m->stream = s;
  return HSB_OK;
}

int hsb_dev_get_state(hsb_dev_model *m, int which, double *out) {
  if (!m || !out) return set_error(HSB_E_ARG, "null argument");
  HSB_CUDA(cudaMemcpyAsync(out, which ? m->ys : m->y, sizeof(double) * m->vlen,
                           cudaMemcpyDeviceToHost, m->stream));
  HSB_CUDA(cudaStreamSynchronize(m->stream));
  return HSB_OK;
}

int hsb_dev_set_tile(hsb_dev_model *m, int rows, int cols) {
  if (!m || rows < 0 || cols < 0 || (rows == 0) != (cols == 0)) return set_error(HSB_E_ARG, "bad tile");
  m->tile_oi = rows;
  m->tile_oj = cols;
  return HSB_OK;
}

int hsb_dev_workspaces(const hsb_dev_model *m, int *mask) {
  if (!m || !mask) return set_error(HSB_E_ARG, "null argument");
  *mask = (m->fast ? HSB_WS_FAST_TRANSIENT : 0) | (m->mg ? HSB_WS_MG : 0) | (m->krylov ? HSB_WS_BICGSTAB : 0);
  return HSB_OK;
}

int hsb_dev_set_state(hsb_dev_model *m, int which, const double *in) {
  if (!m || !in) return set_error(HSB_E_ARG, "null argument");
  HSB_CUDA(cudaMemcpyAsync(which ? m->ys : m->y, in, sizeof(double) * m->vlen,
                           cudaMemcpyHostToDevice, m->stream));
  HSB_CUDA(cudaStreamSynchronize(m->stream));
  return HSB_OK;
}

}  // extern "C"
