// Host-side pieces that the library's translation units share: the solver handle, error messages, the device scope,
// uploads and the recompute list. Internal to the library: not part of the C-ABI.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <vector>

#include "device.cuh"

constexpr int WARPS = 4;  // warps per cell by default (the derivative kernels' only mapping); the call takes 2 or 4

typedef void (*CallFn)(const mx::Net, const mx::CallArgs, long long*);
typedef void (*DebugFn)(const mx::Net, const double*, double, double, double, const double*, double, double, double*);
typedef void (*RecoverFn)(const mx::Net, const mx::CallArgs, int);
typedef void (*TimeFn)(const mx::Net, const double*, double, double, double, const double*, int, long long*);
typedef void (*MixedFn)(const mx::Net, const mx::CallArgs, int, double, long long*);
typedef void (*MixedDebugFn)(const mx::Net, const double*, double, double, double, const double*, double, double, int,
                             double*);

struct mx_derivatives;  // the tangent and adjoint kernels' state (derivatives.cu)

struct mx_solver {
  int device = 0;
  int warps = WARPS;  // warps per cell of the call, recovery and mixed kernels (2 or 4)
  mx::Net net{};
  std::vector<void*> buffers;
  CallFn call = nullptr;
  CallFn call_prof = nullptr;
  CallFn call_list = nullptr;  // the plain kernel over the cells the mixed kernel listed (a.sel)
  RecoverFn recover = nullptr;
  DebugFn debug = nullptr;
  TimeFn timer = nullptr;
  int rows_per_lane = 0;
  size_t smem = 0;
  int sms = 0, call_ctas = 0, recover_ctas = 0;
  int grid_ctas = -1;  // call-kernel CTAs per SM: 1..call_ctas persistent, 0 one CTA per cell; -1 call_ctas
  int* list = nullptr;
  int64_t list_capacity = 0;
  unsigned long long* tries = nullptr;
  long long* phases = nullptr;
  std::vector<uint64_t> rx8_host;  // the reactions' slots, for the adjoint's species gather table
  std::vector<uint64_t> st8_host;  // S's columns: per reaction up to 6 (species byte, coefficient code) pairs
  mx_derivatives* deriv = nullptr;  // the tangent and adjoint kernels' state, at their first call
  // the mixed-precision path (mixed.cu): its layout, kernels and settings, and the list of cells it hands back
  mx::Net net32{};
  MixedFn mixed = nullptr, mixed_prof = nullptr, mixed_list = nullptr;
  MixedDebugFn mixed_debug = nullptr;
  size_t mixed_smem = 0;
  int mixed_ctas = 0;
  int precision = MX_PRECISION_FP64, sweeps = 1;
  double mixed_tol = MX_MIXED_TOL;
  int* sel = nullptr;        // cells the mixed kernel listed for the plain kernel [B]
  int64_t sel_capacity = 0;
  int* sel_count = nullptr;  // device int[2]: listed cells, the plain kernel's queue over them
  long long* escalated = nullptr;  // a caller's device int64 that later mixed calls add their listed cells to
};

// The mixed-precision path (mixed.cu): its layout and kernels at mx_create; its launch within mx_call.
int mx_mixed_prepare(mx_solver* s, int n_pieces, char* err, size_t errlen);
cudaError_t mx_mixed_launch(mx_solver* s, const mx::CallArgs& a, int64_t B, bool list, cudaStream_t st);

// The call's grid of the plain kernel: persistent CTAs per SM as set by mx_set_grid, or one per cell.
inline int call_grid(const mx_solver* s, int64_t B) {
  if (s->grid_ctas == 0) return (int)B;
  const int per_sm = s->grid_ctas < 0 ? s->call_ctas : std::min(s->grid_ctas, s->call_ctas);
  return (int)std::min<int64_t>(B, (int64_t)per_sm * s->sms);
}

// Frees a solver's derivative state and scratch (derivatives.cu); nothing when it has none.
void mx_release_derivatives(mx_solver* s);

namespace {  // each translation unit keeps its own copies

void set_error(char* err, size_t len, const char* fmt, ...) __attribute__((format(printf, 3, 4)));
void set_error(char* err, size_t len, const char* fmt, ...) {
  if (!err || !len) return;
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(err, len, fmt, ap);
  va_end(ap);
}

// Restores the caller's current device on scope exit.
struct DeviceScope {
  int old = -1;
  cudaError_t status;
  explicit DeviceScope(int dev) {
    cudaGetDevice(&old);
    status = cudaSetDevice(dev);
  }
  ~DeviceScope() {
    if (old >= 0) cudaSetDevice(old);
  }
};

template <typename T>
cudaError_t upload(mx_solver* s, const T* host, size_t count, const T** dev) {
  void* p = nullptr;
  const size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
  cudaError_t e = cudaMalloc(&p, bytes);
  if (e != cudaSuccess) return e;
  s->buffers.push_back(p);
  if (count) e = cudaMemcpy(p, host, count * sizeof(T), cudaMemcpyHostToDevice);
  *dev = (const T*)p;
  return e;
}

int grow_list(mx_solver* s, int64_t B, char* err, size_t errlen) {
  if (B <= s->list_capacity) return MX_OK;
  if (s->list) cudaFree(s->list);
  s->list = nullptr;
  s->list_capacity = 0;
  const cudaError_t e = cudaMalloc(&s->list, (size_t)B * sizeof(int));
  if (e != cudaSuccess) {
    set_error(err, errlen, "mx_call: the recompute list of %lld cells: %s", (long long)B, cudaGetErrorString(e));
    return MX_ERR_CUDA;
  }
  s->list_capacity = B;
  return MX_OK;
}

__global__ void add_counts_kernel(const int* count, long long* total) {
  const int i = (int)threadIdx.x;
  if (i < MX_COUNT_SLOTS) total[i] += count[i];
}

}  // namespace
