// leakage.cu -- the temperature-leakage fixed point of the steady solve
// (steady_state_temp with leakage_used, temperature.c:706-746) with every
// block vector on the device between iterations.
//
// Each iteration: the power blocks' leakage at their current temperature
// (calc_leakage, temperature.c:910-927) is added to their dynamic power, the
// steady solve runs from that power (the model's steady solver of the chosen
// form, on the device), and the largest temperature rise over the power
// blocks decides convergence.  As in the reference, the blocks of layers
// without power get zero power in the iteration's power vector, and the loop
// stops below LEAK_TOL, fails above TEMP_HIGH (thermal runaway) or after
// LEAKAGE_MAX_ITER + 1 iterations.  One 8-byte read per iteration reaches the
// host.
#include <cmath>

#include "dev_model.cuh"

// temperature.h:10, 29, 30
#define LEAK_TEMP_HIGH 500.0
#define LEAK_MAX_ITER 100
#define LEAK_TOL 0.01
// calc_leakage's model, temperature.c:916-918
#define LEAK_ALPHA 1.5e+4
#define LEAK_BETA 0.036
#define LEAK_TBASE 383.15

namespace hsb {

// power_new = power + alpha h w exp(beta (T - Tbase)) on the power blocks
// (area > 0), 0 elsewhere; temp_old = temp on the power blocks
__global__ void leak_power(const double *__restrict__ power, const double *__restrict__ height,
                           const double *__restrict__ width, const double *__restrict__ temp,
                           double *__restrict__ power_new, double *__restrict__ temp_old, int nblk, int nb) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nb) return;
  if (b < nblk && height[b] > 0.0) {
    const double h = height[b], w = width[b];
    power_new[b] = power[b] + LEAK_ALPHA * h * w * exp(LEAK_BETA * (temp[b] - LEAK_TBASE));
    temp_old[b] = temp[b];
  } else {
    power_new[b] = 0.0;
  }
}

// the largest rise temp - temp_old over the power blocks (at least 0), as the
// bits of a non-negative double, into *out (zeroed by the caller)
__global__ void leak_rise(const double *__restrict__ height, const double *__restrict__ temp,
                          const double *__restrict__ temp_old, int nblk, unsigned long long *out) {
  double d = 0.0;
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nblk; b += gridDim.x * blockDim.x)
    if (height[b] > 0.0) d = fmax(d, temp[b] - temp_old[b]);
  for (int o = 16; o > 0; o >>= 1) d = fmax(d, __shfl_down_sync(0xffffffffu, d, o));
  if ((threadIdx.x & 31) == 0 && d > 0.0) atomicMax(out, (unsigned long long)__double_as_longlong(d));
}

}  // namespace hsb

using namespace hsb;

extern "C" int hsb_dev_steady_leakage(hsb_dev_model *m, const double *block_power, const double *height,
                                      const double *width, double *block_temp, const hsb_solver_opts *o,
                                      int *iterations, hsb_stats *st) {
  if (!m || !block_power || !height || !width || !block_temp) return set_error(HSB_E_ARG, "null argument");
  if (!m->b2g_ptr) return set_error(HSB_E_ARG, "block-grid maps not set");
  hsb_stats local;
  if (!st) st = &local;
  hsb_solver_opts def = {HSB_FORM_PARITY, HSB_STEADY_AUTO, 0.0, 0};
  if (!o) o = &def;
  if (cudaSetDevice(m->device) != cudaSuccess) return set_error(HSB_E_CUDA, "cudaSetDevice");
  const int nblk = m->total_n_blocks, nb = nblk + m->nx;
  // power, height, width, temperature, previous temperature; the rise
  double *buf = nullptr;
  unsigned long long *rise = nullptr, *h_rise = nullptr;
  int rc = HSB_OK;
  auto done = [&](int code) {
    if (buf) cudaFree(buf);
    if (rise) cudaFree(rise);
    if (h_rise) cudaFreeHost(h_rise);
    return code;
  };
  if (cudaMalloc(&buf, sizeof(double) * (size_t)nb * 5) != cudaSuccess ||
      cudaMalloc(&rise, sizeof(unsigned long long)) != cudaSuccess ||
      cudaMallocHost(&h_rise, sizeof(unsigned long long)) != cudaSuccess)
    return done(set_error(HSB_E_NOMEM, "leakage loop buffers"));
  double *d_pow = buf, *d_h = buf + nb, *d_w = buf + 2 * (size_t)nb, *d_t = buf + 3 * (size_t)nb,
         *d_old = buf + 4 * (size_t)nb;
  cudaEventRecord(m->ev[0], m->stream);
  const cudaError_t e0 = cudaMemcpyAsync(d_pow, block_power, sizeof(double) * nb, cudaMemcpyHostToDevice, m->stream);
  const cudaError_t e1 = cudaMemcpyAsync(d_h, height, sizeof(double) * nblk, cudaMemcpyHostToDevice, m->stream);
  const cudaError_t e2 = cudaMemcpyAsync(d_w, width, sizeof(double) * nblk, cudaMemcpyHostToDevice, m->stream);
  const cudaError_t e3 = cudaMemcpyAsync(d_t, block_temp, sizeof(double) * nb, cudaMemcpyHostToDevice, m->stream);
  if (e0 != cudaSuccess || e1 != cudaSuccess || e2 != cudaSuccess || e3 != cudaSuccess)
    return done(cuda_check(cudaGetLastError(), "leakage loop inputs"));
  bool converged = false;
  int it;
  for (it = 0; !converged && it <= LEAK_MAX_ITER; it++) {
    leak_power<<<(nb + 255) / 256, 256, 0, m->stream>>>(d_pow, d_h, d_w, d_t, m->blk_in, d_old, nblk, nb);
    st->launches += 1;
    if ((rc = steady_core(m, o, st))) return done(rc);
    if ((rc = cuda_ok(cudaMemcpyAsync(d_t, m->blk_out, sizeof(double) * nb, cudaMemcpyDeviceToDevice, m->stream),
                      "leakage loop temperatures")))
      return done(rc);
    if ((rc = cuda_ok(cudaMemsetAsync(rise, 0, sizeof(unsigned long long), m->stream), "leakage loop rise")))
      return done(rc);
    leak_rise<<<(nblk + 255) / 256 > 0 ? (nblk + 255) / 256 : 1, 256, 0, m->stream>>>(d_h, d_t, d_old, nblk, rise);
    st->launches += 1;
    if ((rc = cuda_ok(cudaMemcpyAsync(h_rise, rise, sizeof(unsigned long long), cudaMemcpyDeviceToHost, m->stream),
                      "leakage loop rise")) ||
        (rc = cuda_ok(cudaStreamSynchronize(m->stream), "leakage loop")))
      return done(rc);
    double dmax;
    memcpy(&dmax, h_rise, sizeof(dmax));
    if (dmax < LEAK_TOL) converged = true;
    if (dmax > LEAK_TEMP_HIGH && it > 0)
      return done(set_error(HSB_E_NOCONV, "temperature is too high, possible thermal runaway"));
  }
  if (iterations) *iterations = it;
  if (!converged)
    return done(set_error(HSB_E_NOCONV, "too many iterations before temperature-leakage convergence"));
  if ((rc = cuda_ok(cudaMemcpyAsync(block_temp, d_t, sizeof(double) * nb, cudaMemcpyDeviceToHost, m->stream),
                    "leakage loop result")))
    return done(rc);
  cudaEventRecord(m->ev[1], m->stream);
  if ((rc = cuda_ok(cudaStreamSynchronize(m->stream), "leakage loop"))) return done(rc);
  float ms = 0;
  if (cudaEventElapsedTime(&ms, m->ev[0], m->ev[1]) == cudaSuccess) st->device_ms += ms;
  else cudaGetLastError();
  return done(HSB_OK);
}
