// noalloc.cu -- a transient entry point that allocates nothing.
//
// Some callers of this library may not allocate device memory while they
// run: a host simulator that reserves all of its GPU memory at start-up and
// forbids later allocations, a real-time co-simulation loop that must not
// take cudaMalloc's implicit device synchronisation, or code that only runs
// between set-up phases.  hsb_dev_transient_noalloc() serves them: it runs
// the fast transient form on a state and a power vector the caller already
// owns in device memory, and takes all of its temporaries from one
// file-scope static device array instead of calling cudaMalloc.
//
// The array is hsb_noalloc_scratch below, about 2.8 MB; every GPU that
// loads this library holds it until the process exits.  It fits models of
// up to HSB_NOALLOC_MAX_CELLS grid cells of at most 4096 rows and 16384
// columns.  Every call shares it and it keeps
// the previous call's contents, so calls whose work overlaps on the GPU
// (different streams, or different host threads on one device) race; the
// error accumulators that must start at zero are cleared by each call.
#include <mutex>

#include "dev_model.cuh"

namespace {

constexpr long long kMaxCells = HSB_NOALLOC_MAX_CELLS;
constexpr long long kMaxVec = kMaxCells + HSB_EXTRA + HSB_EXTRA_SEC;
constexpr size_t a256(size_t x) { return (x + 255) & ~size_t(255); }
constexpr size_t kOffPf = 0;
constexpr size_t kOffK1 = a256(kOffPf + sizeof(float) * kMaxCells);
constexpr size_t kOffK2 = a256(kOffK1 + sizeof(float) * kMaxCells);
constexpr size_t kOffK3 = a256(kOffK2 + sizeof(float) * kMaxCells);
constexpr size_t kOffYt = a256(kOffK3 + sizeof(float) * kMaxCells);
constexpr size_t kOffT1 = a256(kOffYt + sizeof(double) * kMaxVec);
constexpr size_t kOffT2 = a256(kOffT1 + sizeof(double) * kMaxVec);
constexpr size_t kLayerBytes = 64 * 32;
constexpr size_t kPackBytes = 8192;
constexpr size_t kPartBytes = sizeof(double) * 2 * 20 * 512;   // 512 tile rows or columns
constexpr size_t kOffLt = a256(kOffT2 + sizeof(double) * kMaxVec);
constexpr size_t kOffPk = a256(kOffLt + kLayerBytes);
constexpr size_t kOffPt = a256(kOffPk + kPackBytes);
constexpr size_t kOffErr = a256(kOffPt + kPartBytes);
constexpr size_t kOffCnt = a256(kOffErr + sizeof(unsigned long long) * 2);
constexpr size_t kTotal = a256(kOffCnt + sizeof(long long) * 4);

}  // namespace

// The scratch.  In host code this name is only a host-side stand-in for the
// symbol, not a device address: the device address is looked up per device
// with cudaGetSymbolAddress and handed to the kernels.
static __device__ __align__(256) unsigned char hsb_noalloc_scratch[kTotal];

namespace {

std::mutex g_mu;
// device address of the scratch, per device ordinal, kept for the life of the
// process: a cudaDeviceReset (which may reload the module elsewhere) is not
// supported while the library is loaded
void *g_addr[256];

// once per device, with that device current
int scratch_address(int dev, unsigned char **out) {
  if (dev < 0 || dev >= 256) return hsb::set_error(HSB_E_ARG, "device ordinal out of range");
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_addr[dev]) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, hsb_noalloc_scratch);
    if (e != cudaSuccess) return hsb::cuda_check(e, "cudaGetSymbolAddress(hsb_noalloc_scratch)");
    g_addr[dev] = p;
  }
  *out = (unsigned char *)g_addr[dev];
  return HSB_OK;
}

}  // namespace

extern "C" int hsb_dev_transient_noalloc(hsb_dev_model *m, double *y, const double *pgrid,
                                         double time_elapsed, hsb_stats *st) {
  using namespace hsb;
  if (!m || !y || !pgrid) return set_error(HSB_E_ARG, "null argument");
  if (m->ncell > kMaxCells)
    return set_error(HSB_E_ARG, "model has more grid cells than the allocation-free entry point's "
                                "static scratch holds (HSB_NOALLOC_MAX_CELLS)");
  if (m->field || m->uchan_mask)
    return set_error(HSB_E_ARG, "the allocation-free entry point takes models with per-layer "
                                "conductances only (no detailed 3-D or microchannel layers)");
  if (rk4_fast_layer_table_bytes() > kLayerBytes || rk4_fast_pack_table_bytes() > kPackBytes)
    return set_error(HSB_E_ARG, "coefficient tables do not fit the static scratch");
  if (rk4_fast_part_bytes(m) > kPartBytes)
    return set_error(HSB_E_ARG, "grid too elongated for the allocation-free entry point's static "
                                "scratch (at most 4096 rows and 16384 columns)");
  int dev = -1;
  HSB_CUDA(cudaGetDevice(&dev));
  if (dev != m->device) return set_error(HSB_E_ARG, "call with the model's device current");
  unsigned char *s = nullptr;
  int rc = scratch_address(dev, &s);
  if (rc) return rc;
  FastBuffers b;
  b.y = y;
  b.pgrid = pgrid;
  b.pf = (float *)(s + kOffPf);
  b.k1 = (float *)(s + kOffK1);
  b.k2 = (float *)(s + kOffK2);
  b.k3 = (float *)(s + kOffK3);
  b.ytemp = (double *)(s + kOffYt);
  b.t1 = (double *)(s + kOffT1);
  b.t2 = (double *)(s + kOffT2);
  b.layer_table = (void *)(s + kOffLt);
  b.pack_table = (void *)(s + kOffPk);
  b.part = (double *)(s + kOffPt);
  b.err = (unsigned long long *)(s + kOffErr);
  b.cnt = (long long *)(s + kOffCnt);
  // what the kernel reads before writing starts from zero on every call
  HSB_CUDA(cudaMemsetAsync(b.err, 0, sizeof(unsigned long long) * 2, m->stream));
  HSB_CUDA(cudaMemsetAsync(b.cnt, 0, sizeof(long long) * 4, m->stream));
  return rk4_fast_on_buffers(m, b, time_elapsed, st);
}
