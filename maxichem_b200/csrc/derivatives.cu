// The derivative entry points mx_jvp and mx_vjp and their kernels (jvp.cuh, vjp.cuh). A translation unit of their
// own: the call kernel's module (maxichem_b200.cu) is compiled without them, so its code does not depend on theirs.
#include <new>

#include "solver.cuh"
#include "vjp.cuh"

using namespace mx;

namespace {

typedef void (*VjpFn)(const Net, const CallArgs, const AdjArgs, const AdjLayout);
typedef void (*VjpRecoverFn)(const Net, const CallArgs, const AdjArgs, const AdjLayout, int);

// the adjoint kernels for rows_per_lane R of the warp solves
bool pick_vjp_kernels(int r, VjpFn* vjp, VjpRecoverFn* rec) {
  switch (r) {
    case 1: *vjp = vjp_kernel<WARPS, 1>; *rec = vjp_recover_kernel<WARPS, 1>; return true;
    case 2: *vjp = vjp_kernel<WARPS, 2>; *rec = vjp_recover_kernel<WARPS, 2>; return true;
    case 3: *vjp = vjp_kernel<WARPS, 3>; *rec = vjp_recover_kernel<WARPS, 3>; return true;
    case 4: *vjp = vjp_kernel<WARPS, 4>; *rec = vjp_recover_kernel<WARPS, 4>; return true;
    case 8: *vjp = vjp_kernel<WARPS, 8>; *rec = vjp_recover_kernel<WARPS, 8>; return true;
    default: return false;
  }
}  // fmt: skip

typedef void (*JvpFn)(const Net, const CallArgs, const TanArgs, const TanLayout);
typedef void (*JvpRecoverFn)(const Net, const CallArgs, const TanArgs, const TanLayout, int);

// the tangent kernels for rows_per_lane R of the warp solves
bool pick_jvp_kernels(int r, JvpFn* jvp, JvpRecoverFn* rec) {
  switch (r) {
    case 1: *jvp = jvp_kernel<WARPS, 1>; *rec = jvp_recover_kernel<WARPS, 1>; return true;
    case 2: *jvp = jvp_kernel<WARPS, 2>; *rec = jvp_recover_kernel<WARPS, 2>; return true;
    case 3: *jvp = jvp_kernel<WARPS, 3>; *rec = jvp_recover_kernel<WARPS, 3>; return true;
    case 4: *jvp = jvp_kernel<WARPS, 4>; *rec = jvp_recover_kernel<WARPS, 4>; return true;
    case 8: *jvp = jvp_kernel<WARPS, 8>; *rec = jvp_recover_kernel<WARPS, 8>; return true;
    default: return false;
  }
}  // fmt: skip

}  // namespace

// The tangent and adjoint kernels of one solver: functions, layouts, launch limits, tables and scratch, set up at
// their first call.
struct mx_derivatives {
  JvpFn jvp = nullptr;
  JvpRecoverFn jvp_recover = nullptr;
  TanLayout tan_layout{};
  size_t jvp_smem = 0;
  int jvp_ctas = 0, jvp_recover_ctas = 0;
  double* jvp_scratch = nullptr;
  size_t jvp_scratch_doubles = 0;
  VjpFn vjp = nullptr;
  VjpRecoverFn vjp_recover = nullptr;
  AdjLayout adj_layout{};
  size_t vjp_smem = 0;
  int vjp_ctas = 0, vjp_recover_ctas = 0;
  const int *sp_ptr = nullptr, *sp_ent = nullptr;  // species gather table (in the solver's buffers)
  const uint64_t* st8 = nullptr;                  // S's columns (in the solver's buffers)
  double* vjp_scratch = nullptr;
  size_t vjp_scratch_doubles = 0;
  double* vjp_glc = nullptr;  // the rate table's chunk partial sums [nr][chunks][9]
  size_t vjp_glc_doubles = 0;
  double* vjp_glq = nullptr;  // recovered cells' rate-table cotangents [listed][nr][3]
  size_t vjp_glq_doubles = 0;
  int* vjp_ints = nullptr;    // chunk flags [chunks], the chunk queue [1], list slots [B]
  size_t vjp_ints_count = 0;
};

namespace {

// the solver's derivative state, made at the first derivative call
mx_derivatives* derivatives_of(mx_solver* s) {
  if (!s->deriv) s->deriv = new (std::nothrow) mx_derivatives();
  return s->deriv;
}

}  // namespace

void mx_release_derivatives(mx_solver* s) {
  mx_derivatives* d = s->deriv;
  if (!d) return;
  if (d->jvp_scratch) cudaFree(d->jvp_scratch);
  if (d->vjp_scratch) cudaFree(d->vjp_scratch);
  if (d->vjp_glc) cudaFree(d->vjp_glc);
  if (d->vjp_glq) cudaFree(d->vjp_glq);
  if (d->vjp_ints) cudaFree(d->vjp_ints);
  delete d;
  s->deriv = nullptr;
}

// ---- mx_jvp: the call and its tangent ----

namespace {

// The tangent kernels' shared-memory layout and launch limits, once per solver.
int setup_jvp(mx_solver* s, char* err, size_t errlen) {
  mx_derivatives* d = derivatives_of(s);
  if (!d) {
    set_error(err, errlen, "mx_jvp: out of host memory");
    return MX_ERR_CUDA;
  }
  if (d->jvp) return MX_OK;
  const Net& net = s->net;
  const int ns = net.ns, nr = net.nr;
  TanLayout& l = d->tan_layout;
  int off = net.doubles;
  auto take = [&](int doubles) {
    const int o = off;
    off += (doubles + 1) & ~1;
    return o;
  };
  l.stride = (ns + 2) & ~1;
  l.oTN = take(ns + 1);
  l.oTn = take(ns + 1);
  l.oTF = take(ns + 1);
  l.oTu = take(ns + 1);
  l.oTY = take(ns + 1);
  l.oJK = take(4 * l.stride);
  l.oTK = take(4 * l.stride);
  l.oZ = take(std::max(nr, ns) + 1);
  l.doubles = off;
  const size_t smem = (size_t)off * sizeof(double);
  JvpFn jvp = nullptr;
  JvpRecoverFn rec = nullptr;
  if (!pick_jvp_kernels(s->rows_per_lane, &jvp, &rec)) {
    set_error(err, errlen, "mx_jvp: no tangent kernels for %d rows per lane", s->rows_per_lane);
    return MX_ERR_NETWORK;
  }
  int optin = 0;
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, s->device);
  if ((size_t)optin < smem) {
    set_error(err, errlen, "the tangent kernels need %zu B of shared memory per cell; the device has %d per block",
              smem, optin);
    return MX_ERR_NETWORK;
  }
  cudaError_t e = cudaFuncSetAttribute((const void*)jvp, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute((const void*)rec, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  int a = 0, b = 0;
  if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, (const void*)jvp, 32 * WARPS, smem);
  if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, (const void*)rec, 32 * WARPS, smem);
  if (e == cudaSuccess && (a < 1 || b < 1)) e = cudaErrorInvalidConfiguration;
  if (e != cudaSuccess) {
    set_error(err, errlen, "mx_jvp: %s", cudaGetErrorString(e));
    return MX_ERR_CUDA;
  }
  d->jvp_smem = smem;
  d->jvp_ctas = a;
  d->jvp_recover_ctas = b;
  d->jvp = jvp;
  d->jvp_recover = rec;
  return MX_OK;
}

}  // namespace

extern "C" int mx_jvp(mx_solver* s, const double* x, const double* T, const double* P, const double* dt,
                      const double* h_in, const double* J, const double* lm, const double* rc, int64_t B, double rtol,
                      double atol, int32_t max_steps, int32_t adapt, int32_t D, const double* dx, const double* dT,
                      const double* dP, const double* ddt, const double* dh, const double* dlm, const double* drc,
                      const double* dJ, double* x_out, double* h_out, int32_t* done, double* steps, int32_t* flag,
                      int32_t* status, double* dx_out, double* dh_out, int32_t* count, int64_t* total, void* stream,
                      char* err, size_t errlen) {
  if (!s) {
    set_error(err, errlen, "this solver was closed; build a new one");
    return MX_ERR_CLOSED;
  }
  if (s->warps != WARPS) {
    set_error(err, errlen, "mx_jvp: the derivative kernels take %d warps per cell; this solver's tables are for %d",
              WARPS, s->warps);
    return MX_ERR_NETWORK;
  }
  if (B < 0 || B > 0x7fffffff) {
    set_error(err, errlen, "mx_jvp: B out of range: %lld", (long long)B);
    return MX_ERR_ARGUMENT;
  }
  if (!(rtol > 0.0 && rtol < 1e300 && atol > 0.0 && atol < 1e300)) {
    set_error(err, errlen, "rtol and atol finite and positive expected, got %g, %g", rtol, atol);
    return MX_ERR_ARGUMENT;
  }
  if (max_steps < 1 || (int64_t)MX_REC_STEPS * max_steps > 0x7fffffff) {
    set_error(err, errlen, "max_steps from 1 to %d expected, got %d", 0x7fffffff / MX_REC_STEPS, max_steps);
    return MX_ERR_ARGUMENT;
  }
  if (D < 1 || D > MX_JVP_MAX_DIRECTIONS || (adapt != 0 && adapt != 1)) {
    set_error(err, errlen, "mx_jvp: from 1 to %d directions and adapt 0 or 1 expected, got %d and %d",
              MX_JVP_MAX_DIRECTIONS, D, adapt);
    return MX_ERR_ARGUMENT;
  }
  if (!count || !total || (B > 0 && (!x || !T || !P || !dt || !h_in || !x_out || !h_out || !done || !steps ||
                                     !flag || !status || (s->net.nj > 0 && !J) || !dx || !dT || !dP || !ddt ||
                                     !dh || !dx_out || !dh_out))) {
    set_error(err, errlen, "mx_jvp: a required array is null");
    return MX_ERR_ARGUMENT;
  }
  DeviceScope scope(s->device);
  if (scope.status != cudaSuccess) {
    set_error(err, errlen, "mx_jvp: device %d: %s", s->device, cudaGetErrorString(scope.status));
    return MX_ERR_CUDA;
  }
  int rcode = setup_jvp(s, err, errlen);
  if (rcode) return rcode;
  mx_derivatives* d = s->deriv;
  rcode = grow_list(s, std::max<int64_t>(B, 1), err, errlen);
  if (rcode) return rcode;
  const Net& n0 = s->net;
  const long long slot = ((long long)D * (2 * n0.nr + 2 + n0.ns + 1 + 4) + 1) & ~1ll;
  const int grid = (int)std::min<int64_t>(std::max<int64_t>(B, 1), (int64_t)d->jvp_ctas * s->sms);
  const int rgrid = (int)std::min<int64_t>(std::max<int64_t>(B, 1), (int64_t)d->jvp_recover_ctas * s->sms);
  const size_t need = (size_t)std::max(grid, rgrid) * (size_t)slot;
  if (need > d->jvp_scratch_doubles) {
    if (d->jvp_scratch) cudaFree(d->jvp_scratch);
    d->jvp_scratch = nullptr;
    d->jvp_scratch_doubles = 0;
    const cudaError_t e = cudaMalloc(&d->jvp_scratch, need * sizeof(double));
    if (e != cudaSuccess) {
      set_error(err, errlen, "mx_jvp: the tangent scratch of %zu doubles: %s", need, cudaGetErrorString(e));
      return MX_ERR_CUDA;
    }
    d->jvp_scratch_doubles = need;
  }
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e = cudaMemsetAsync(count, 0, MX_COUNT_SLOTS * sizeof(int32_t), st);
  if (e == cudaSuccess && B > 0) {
    Net net = s->net;
    if (rc) net.rc = rc;  // the caller's rate table
    const CallArgs a{x, T, P, dt, h_in, J, (int)B, rtol, atol, max_steps, x_out, h_out, done, steps, flag, status,
                     count, s->list, nullptr};
    const TanArgs ta{lm, dx, dT, dP, ddt, dh, dlm, drc, s->net.nj > 0 ? dJ : nullptr, D, adapt, dx_out, dh_out,
                     d->jvp_scratch, slot};
    d->jvp<<<grid, 32 * WARPS, d->jvp_smem, st>>>(net, a, ta, d->tan_layout);
    d->jvp_recover<<<rgrid, 32 * WARPS, d->jvp_smem, st>>>(net, a, ta, d->tan_layout, MX_REC_STEPS * max_steps);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) {
    add_counts_kernel<<<1, 32, 0, st>>>(count, (long long*)total);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) {
    set_error(err, errlen, "mx_jvp: %s", cudaGetErrorString(e));
    return MX_ERR_CUDA;
  }
  return MX_OK;
}

// ---- mx_vjp: the call and its adjoint ----

namespace {

// grow a solver-owned device buffer of doubles to at least `need`
int grow_doubles(double** p, size_t* have, size_t need, const char* what, char* err, size_t errlen) {
  if (need <= *have) return MX_OK;
  if (*p) cudaFree(*p);
  *p = nullptr;
  *have = 0;
  const cudaError_t e = cudaMalloc(p, need * sizeof(double));
  if (e != cudaSuccess) {
    set_error(err, errlen, "mx_vjp: the %s of %zu doubles: %s", what, need, cudaGetErrorString(e));
    return MX_ERR_CUDA;
  }
  *have = need;
  return MX_OK;
}

// The adjoint kernels' shared-memory layout, launch limits and species gather table, once per solver.
int setup_vjp(mx_solver* s, char* err, size_t errlen) {
  mx_derivatives* d = derivatives_of(s);
  if (!d) {
    set_error(err, errlen, "mx_vjp: out of host memory");
    return MX_ERR_CUDA;
  }
  if (d->vjp) return MX_OK;
  const Net& net = s->net;
  const int ns = net.ns, nr = net.nr;
  AdjLayout& l = d->adj_layout;
  int off = net.doubles;
  auto take = [&](int doubles) {
    const int o = off;
    off += (doubles + 1) & ~1;
    return o;
  };
  l.stride = (ns + 2) & ~1;
  l.oNb = take(ns + 1);
  l.oYb = take(ns + 1);
  l.oFb = take(ns + 1);
  l.oUb = take(ns + 1);
  l.oNn = take(ns + 1);
  l.oNx = take(ns + 1);
  l.oKb = take(4 * l.stride);
  l.oBb = take(4 * l.stride);
  l.oRed = take(32 * WARPS + 2);
  l.doubles = off;
  const size_t smem = (size_t)off * sizeof(double);
  VjpFn vjp = nullptr;
  VjpRecoverFn rec = nullptr;
  if (!pick_vjp_kernels(s->rows_per_lane, &vjp, &rec)) {
    set_error(err, errlen, "mx_vjp: no adjoint kernels for %d rows per lane", s->rows_per_lane);
    return MX_ERR_NETWORK;
  }
  int optin = 0;
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, s->device);
  if ((size_t)optin < smem) {
    set_error(err, errlen, "the adjoint kernels need %zu B of shared memory per cell; the device has %d per block",
              smem, optin);
    return MX_ERR_NETWORK;
  }
  // species j's reaction slots (r * 8 + m), in ascending reaction and slot order
  std::vector<int> ptr(ns + 1, 0), ent;
  for (int j = 0; j < ns; j++) {
    for (int r = 0; r < nr; r++)
      for (int m = 0; m < 6; m++)
        if ((int)((s->rx8_host[r] >> (8 * m)) & 255) == j) ent.push_back(r * 8 + m);
    ptr[j + 1] = (int)ent.size();
  }
  cudaError_t e = upload(s, ptr.data(), ptr.size(), &d->sp_ptr);
  if (e == cudaSuccess) e = upload(s, ent.data(), ent.size(), &d->sp_ent);
  if (e == cudaSuccess) e = upload(s, s->st8_host.data(), s->st8_host.size(), &d->st8);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute((const void*)vjp, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute((const void*)rec, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  int a = 0, b = 0;
  if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, (const void*)vjp, 32 * WARPS, smem);
  if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, (const void*)rec, 32 * WARPS, smem);
  if (e == cudaSuccess && (a < 1 || b < 1)) e = cudaErrorInvalidConfiguration;
  if (e != cudaSuccess) {
    set_error(err, errlen, "mx_vjp: %s", cudaGetErrorString(e));
    return MX_ERR_CUDA;
  }
  d->vjp_smem = smem;
  d->vjp_ctas = a;
  d->vjp_recover_ctas = b;
  d->vjp = vjp;
  d->vjp_recover = rec;
  return MX_OK;
}

}  // namespace

extern "C" int mx_vjp(mx_solver* s, const double* x, const double* T, const double* P, const double* dt,
                      const double* h_in, const double* J, const double* lm, const double* rc, int64_t B, double rtol,
                      double atol, int32_t max_steps, int32_t adapt, int32_t cap, const double* gx, const double* gh,
                      double* x_out, double* h_out, int32_t* done, double* steps, int32_t* flag, int32_t* status,
                      double* gx0, double* gT, double* gP, double* gdt, double* gh0, double* glm, double* grc,
                      double* gJ, int32_t* count, int64_t* total, void* stream, char* err, size_t errlen) {
  if (!s) {
    set_error(err, errlen, "this solver was closed; build a new one");
    return MX_ERR_CLOSED;
  }
  if (s->warps != WARPS) {
    set_error(err, errlen, "mx_vjp: the derivative kernels take %d warps per cell; this solver's tables are for %d",
              WARPS, s->warps);
    return MX_ERR_NETWORK;
  }
  if (B < 0 || B > 0x7fffffff) {
    set_error(err, errlen, "mx_vjp: B out of range: %lld", (long long)B);
    return MX_ERR_ARGUMENT;
  }
  if (!(rtol > 0.0 && rtol < 1e300 && atol > 0.0 && atol < 1e300)) {
    set_error(err, errlen, "rtol and atol finite and positive expected, got %g, %g", rtol, atol);
    return MX_ERR_ARGUMENT;
  }
  if (cap < 1 || cap > 100000 || (adapt != 0 && adapt != 1)) {
    set_error(err, errlen, "mx_vjp: cap from 1 to 100000 and adapt 0 or 1 expected, got %d and %d", cap, adapt);
    return MX_ERR_ARGUMENT;
  }
  const int64_t reach = (int64_t)(2 * cap) * (2 * cap) / MX_REC_STEPS;  // what the recovery's checkpoints reach
  if (max_steps < 1 || max_steps > reach) {
    set_error(err, errlen, "max_steps: at most %lld at cap %d expected, got %d", (long long)reach, cap, max_steps);
    return MX_ERR_ARGUMENT;
  }
  if (!count || !total || (B > 0 && (!x || !T || !P || !dt || !h_in || !x_out || !h_out || !done || !steps ||
                                     !flag || !status || (s->net.nj > 0 && (!J || !gJ)) || !gx || !gx0 || !gT ||
                                     !gP || !gdt || !gh0 || !glm || !grc))) {
    set_error(err, errlen, "mx_vjp: a required array is null");
    return MX_ERR_ARGUMENT;
  }
  DeviceScope scope(s->device);
  if (scope.status != cudaSuccess) {
    set_error(err, errlen, "mx_vjp: device %d: %s", s->device, cudaGetErrorString(scope.status));
    return MX_ERR_CUDA;
  }
  int rcode = setup_vjp(s, err, errlen);
  if (rcode) return rcode;
  mx_derivatives* d = s->deriv;
  rcode = grow_list(s, std::max<int64_t>(B, 1), err, errlen);
  if (rcode) return rcode;
  const Net& n0 = s->net;
  const int stored = 2 * cap;
  // per CTA: k_bar, c1, c2, the try states, the cell's rate-table cotangents (3 nr)
  const long long slot = ((long long)17 * n0.nr + 2LL * stored * (n0.ns + REC_EXTRA) + 1) & ~1ll;
  const int nchunks = (int)((std::max<int64_t>(B, 1) + ADJ_CHUNK - 1) / ADJ_CHUNK);
  const int grid = (int)std::min<int64_t>(nchunks, (int64_t)d->vjp_ctas * s->sms);
  const int rgrid = (int)std::min<int64_t>(std::max<int64_t>(B, 1), (int64_t)d->vjp_recover_ctas * s->sms);
  rcode = grow_doubles(&d->vjp_scratch, &d->vjp_scratch_doubles, (size_t)std::max(grid, rgrid) * (size_t)slot,
                       "adjoint scratch", err, errlen);
  if (rcode) return rcode;
  rcode = grow_doubles(&d->vjp_glc, &d->vjp_glc_doubles, (size_t)n0.nr * nchunks * 9,
                       "the rate table's chunk sums", err, errlen);
  if (rcode) return rcode;
  const size_t ints = (size_t)nchunks + 1 + (size_t)std::max<int64_t>(B, 1);
  if (ints > d->vjp_ints_count) {
    if (d->vjp_ints) cudaFree(d->vjp_ints);
    d->vjp_ints = nullptr;
    d->vjp_ints_count = 0;
    if (cudaMalloc(&d->vjp_ints, ints * sizeof(int)) != cudaSuccess) {
      set_error(err, errlen, "mx_vjp: the chunk flags and list slots of %lld cells", (long long)B);
      return MX_ERR_CUDA;
    }
    d->vjp_ints_count = ints;
  }
  int* chunk_listed = d->vjp_ints;
  int* chunk_queue = d->vjp_ints + nchunks;
  int* pos = chunk_queue + 1;
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e = cudaMemsetAsync(count, 0, MX_COUNT_SLOTS * sizeof(int32_t), st);
  if (e == cudaSuccess) e = cudaMemsetAsync(chunk_queue, 0, sizeof(int), st);
  if (e == cudaSuccess && B > 0) {
    Net net = s->net;
    if (rc) net.rc = rc;  // the caller's rate table
    const CallArgs a{x, T, P, dt, h_in, J, (int)B, rtol, atol, max_steps, x_out, h_out, done, steps, flag, status,
                     count, s->list, nullptr};
    AdjArgs aa{lm, gx, gh, adapt, stored, gx0, gT, gP, gdt, gh0, glm, s->net.nj > 0 ? gJ : nullptr, d->vjp_glc,
               nchunks, chunk_listed, chunk_queue, nullptr, pos, d->vjp_scratch, slot, d->sp_ptr, d->sp_ent, d->st8};
    d->vjp<<<grid, 32 * WARPS, d->vjp_smem, st>>>(net, a, aa, d->adj_layout);
    // the recovered cells' cotangents get a slot each: size them from the count of listed cells (one small read)
    int listed = 0;
    e = cudaMemcpyAsync(&listed, count + MX_COUNT_RECOMPUTED, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e == cudaSuccess) {
      rcode = grow_doubles(&d->vjp_glq, &d->vjp_glq_doubles, (size_t)std::max(listed, 1) * n0.nr * 3,
                           "the recovered cells' rate-table cotangents", err, errlen);
      if (rcode) return rcode;
      aa.gLq = d->vjp_glq;
      d->vjp_recover<<<rgrid, 32 * WARPS, d->vjp_smem, st>>>(net, a, aa, d->adj_layout, MX_REC_STEPS * max_steps);
      arrh_kernel<<<n0.nr, 32, 0, st>>>(net, a, aa, grc);
      e = cudaGetLastError();
    }
  } else if (e == cudaSuccess && grc) {  // an empty batch: the rate table's cotangent is zero (if asked for)
    e = cudaMemsetAsync(grc, 0, (size_t)n0.nr * 9 * sizeof(double), st);
  }
  if (e == cudaSuccess) {
    add_counts_kernel<<<1, 32, 0, st>>>(count, (long long*)total);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) {
    set_error(err, errlen, "mx_vjp: %s", cudaGetErrorString(e));
    return MX_ERR_CUDA;
  }
  return MX_OK;
}

