// The GCM step's conversions either side of a call (maxichem/coupling/composition.py:102-183 of the reference): mass
// mixing ratios q [B][ns] to mole fractions x = (q / mw) / sum(q / mw), and back, q = x mw (mass / sum(x mw)). One
// warp per cell streams its row (consecutive lanes, consecutive addresses), so each conversion reads and writes
// [B][ns] once: HBM bound. Row sums are formed in the warp's order (lane l adds entries l, l + 32, ..., then a
// butterfly). Problems are reported as bits or-ed into one word for the host to explain.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>

#include "../../include/maxichem_b200.h"

namespace {

constexpr unsigned FULL = 0xffffffffu;
constexpr int WARPS = 8;  // warps (cells in flight) per block

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
  return v;
}

// q -> x. bad bits: 1 a non-finite q, 2 a negative q (unless signed_ok), 4 a cell whose sum of q / mw is not above 0
__global__ void __launch_bounds__(32 * WARPS) mass_to_mole_kernel(const double* __restrict__ q,
                                                                  const double* __restrict__ mw, int64_t B, int ns,
                                                                  int signed_ok, double* __restrict__ x,
                                                                  int* __restrict__ bad) {
  const int lane = threadIdx.x & 31;
  int flags = 0;
  for (int64_t cell = (int64_t)blockIdx.x * WARPS + (threadIdx.x >> 5); cell < B; cell += (int64_t)gridDim.x * WARPS) {
    const double* qc = q + cell * ns;
    double* xc = x + cell * ns;
    double part = 0.0;
    for (int i = lane; i < ns; i += 32) {
      const double v = qc[i];
      flags |= isfinite(v) ? 0 : 1;
      flags |= (!signed_ok && v < 0.0) ? 2 : 0;
      part += v / __ldg(mw + i);
    }
    const double total = warp_sum(part);
    flags |= (!signed_ok && !(total > 0.0)) ? 4 : 0;
    for (int i = lane; i < ns; i += 32) xc[i] = (qc[i] / __ldg(mw + i)) / total;
  }
  flags = __reduce_or_sync(FULL, flags);
  if (lane == 0 && flags) atomicOr(bad, flags);
}

// x, mass -> q. bad bits: 1 a non-finite x, 2 a negative x, 4 a cell whose sum of x mw is not above 0, 8 a mass that
// is negative or not finite
__global__ void __launch_bounds__(32 * WARPS) mole_to_mass_kernel(const double* __restrict__ x,
                                                                  const double* __restrict__ mw,
                                                                  const double* __restrict__ mass, int64_t B, int ns,
                                                                  double* __restrict__ q, int* __restrict__ bad) {
  const int lane = threadIdx.x & 31;
  int flags = 0;
  for (int64_t cell = (int64_t)blockIdx.x * WARPS + (threadIdx.x >> 5); cell < B; cell += (int64_t)gridDim.x * WARPS) {
    const double* xc = x + cell * ns;
    double* qc = q + cell * ns;
    double part = 0.0;
    for (int i = lane; i < ns; i += 32) {
      const double v = xc[i];
      flags |= isfinite(v) ? 0 : 1;
      flags |= v < 0.0 ? 2 : 0;
      part += v * __ldg(mw + i);
    }
    const double weight = warp_sum(part);
    const double m = mass[cell];
    flags |= weight > 0.0 ? 0 : 4;
    flags |= (isfinite(m) && m >= 0.0) ? 0 : 8;
    const double f = m / weight;
    for (int i = lane; i < ns; i += 32) qc[i] = (xc[i] * __ldg(mw + i)) * f;
  }
  flags = __reduce_or_sync(FULL, flags);
  if (lane == 0 && flags) atomicOr(bad, flags);
}

int grid_for(int64_t B) {
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int64_t blocks = (B + WARPS - 1) / WARPS;
  const int64_t most = (int64_t)sms * 8;  // 8 blocks of 256 threads per SM
  return (int)(blocks < most ? (blocks > 0 ? blocks : 1) : most);
}

}  // namespace

extern "C" int mx_mass_to_mole(const double* q, const double* mw, int64_t B, int32_t ns, int32_t signed_ok,
                               double* x, int32_t* bad, void* stream) {
  if (B < 0 || ns < 1 || ns > MX_MAX_SPECIES || !mw || !bad || (B > 0 && (!q || !x))) return MX_ERR_ARGUMENT;
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e = cudaMemsetAsync(bad, 0, sizeof(int32_t), st);
  if (e == cudaSuccess && B > 0) {
    mass_to_mole_kernel<<<grid_for(B), 32 * WARPS, 0, st>>>(q, mw, B, ns, signed_ok, x, bad);
    e = cudaGetLastError();
  }
  return e == cudaSuccess ? MX_OK : MX_ERR_CUDA;
}

extern "C" int mx_mole_to_mass(const double* x, const double* mw, const double* mass, int64_t B, int32_t ns,
                               double* q, int32_t* bad, void* stream) {
  if (B < 0 || ns < 1 || ns > MX_MAX_SPECIES || !mw || !bad || (B > 0 && (!x || !mass || !q))) return MX_ERR_ARGUMENT;
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e = cudaMemsetAsync(bad, 0, sizeof(int32_t), st);
  if (e == cudaSuccess && B > 0) {
    mole_to_mass_kernel<<<grid_for(B), 32 * WARPS, 0, st>>>(x, mw, mass, B, ns, q, bad);
    e = cudaGetLastError();
  }
  return e == cudaSuccess ? MX_OK : MX_ERR_CUDA;
}
