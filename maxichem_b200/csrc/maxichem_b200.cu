// The C-ABI library: the call, recovery and guard kernels for sm_100a, and the entry points of
// include/maxichem_b200.h.
//
// Layout: one CTA of W warps steps one cell at a time, persistent over an atomic cell queue (call.cuh:174-176 of the
// reference keeps the same queue), with the cell's dense matrix, rates and vectors in shared memory. The guard's
// test runs in the call kernel's epilogue on the cell's result while it is still in shared memory, so a result is
// written to HBM once; the recovery kernel recomputes only the cells the guard listed.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

#include "solver.cuh"

using namespace mx;

namespace {

// Phases of a try that the profiling variant of the call kernel times (clock64 on thread 0, summed over cells).
enum { PH_RATES, PH_RHS_JAC, PH_LU, PH_STAGE12, PH_STAGE3, PH_STAGE4, PH_CONTROL, PH_OUTPUT, PH_COUNT };

// The call kernel: screening, rates, Rodas3 steps, output and the guard, per cell (call.cuh:5-177, guard.cuh:114-140).
// PROF: also sum clock64 cycles per phase into prof[PH_COUNT]. LIST: step only the cells a.in_list lists
// (a.in_count[0] of them: the mixed kernel's hand-backs, or the surrogate's fallbacks), with a.in_count[1] as the queue.
template <int W, int R, bool PROF, bool LIST = false>
__global__ void __launch_bounds__(32 * W, 16 / W) call_kernel(const Net net, const CallArgs a, long long* prof) {
  extern __shared__ double smem[];
  const Cell c = cell_arrays(net, smem);
  const int tid = (int)threadIdx.x, nt = 32 * W, lane = tid & 31, warp = tid >> 5, ns = net.ns, ld = net.ld;
  long long ph[PH_COUNT], t0 = 0;
  if (PROF) {
#pragma unroll
    for (int q = 0; q < PH_COUNT; q++) ph[q] = 0;
    t0 = clock64();
  }
  auto mark = [&](int q) {
    if (PROF && tid == 0) {
      const long long t = clock64();
      ph[q] += t - t0;
      t0 = t;
    }
  };
  const int nb = LIST ? a.in_count[0] : a.B;
  int q = (int)blockIdx.x;
  while (q < nb) {
    const int cell = LIST ? a.in_list[q] : q;
    const double Tc = a.T[cell], dt = a.dt[cell], hin = a.h_in[cell];
    const double nd = a.P[cell] / (MX_KB * Tc);
    const double* x0 = a.x + (size_t)cell * ns;
    const double* Jc = a.J + (size_t)cell * net.nj;
    for (int i = tid; i < ns; i += nt) c.N[i] = x0[__ldg(net.perm + i)];
    __syncthreads();
    if (warp == 0) {  // screening on one warp, in the warp's own summation order (common.cuh:246-279)
      const double nan = __longlong_as_double(0x7ff8000000000000ll);
      double p = 0.0, pm = 0.0;
      for (int i = lane; i < ns; i += 32) {
        const double xi = c.N[i];
        p += xi >= 0.0 ? xi : nan;
        pm = fmax(pm, xi);
      }
      for (int b = lane; b < net.nj; b += 32) {
        const double q = Jc[b];
        p += q >= 0.0 ? 0.0 * q : nan;
      }
      const double ps = warp_sum(p), mxv = warp_max(pm);
      const bool forcing = isfinite(Tc) && isfinite(nd) && nd > 0.0 && isfinite(dt) && dt >= 0.0;
      const bool fine = fabs(ps - 1.0) <= MX_X_SUM_TOL && mxv > 0.0 && forcing;
      const int st =
          Tc < MX_T_MIN ? MX_REFUSED_COLD : (Tc > MX_T_MAX ? MX_REFUSED_HOT : (fine ? 0 : MX_REFUSED_BAD_INPUT));
      if (lane == 0) {
        c.ints[0] = st;
        a.status[cell] = st;
        if (!isfinite(hin)) atomicAdd(a.count + MX_COUNT_NONFINITE_H, 1);
      }
    }
    __syncthreads();
    const int st = c.ints[0];
    if (st == 0) cell_rates(net, c, Tc, nd, Jc, tid, nt);
    mark(PH_RATES);
    const double h0 = isfinite(hin) ? hin : dt;  // a non-finite h acts as dt
    StepState s = {fmax(fmin(h0, dt), MX_H_MIN), 0.0, 0.0, 0.0, 0.0, false};
    int it = (dt > 0.0 && st == 0) ? 0 : a.max_steps;  // a refused cell takes no step
    double c0 = 0.0;
    int tries = 0, retries = 0;
    while (it < a.max_steps && s.t < dt * MX_CALL_END) {
      const double ha = fmin(s.h, dt - s.t), igh = 1.0 / (GAMMA * ha), ih = 1.0 / ha;
      tries++;
      retries += s.prej ? 1 : 0;
      // F, u and -Jn at N: a retry after a rejection recomputes those of the rejected try, bit for bit
      const double ntot = rhs(net, c, c.N, true, nd, tid, nt);
      jacobian_w(net, c, ntot, tid, nt);
      for (int i = tid; i < ns; i += nt) c.A[i * ld + i] += igh;  // M0 = I / (gamma h) - Jn
      __syncthreads();
      mark(PH_RHS_JAC);
      lu_factor<32 * W>(net, c.A, c.dinv, tid);
      mark(PH_LU);
      if (warp == 0) {  // stage 1: K1 on warp 0 and M0^-1 w on warp 1 (msolve, call.cuh:122-131), then Sherman-Morrison
        for (int i = lane; i < ns; i += 32) c.K1[i] = c.F[i];
        __syncwarp();
        lu_solve<R, 1>(net, c.A, c.dinv, c.K1, nullptr, lane);
      } else if (warp == 1) {
        lu_solve<R, 1>(net, c.A, c.dinv, c.U, nullptr, lane);
      }
      __syncthreads();
      if (warp == 0) {
        c0 = 1.0 / (1.0 - lane_sum(c.U, ns, lane));
        sherman(net, c.K1, c.U, c0, lane);
      }
      __syncthreads();
      for (int i = tid; i < ns; i += nt) {
        c.K2[i] = fma(RODAS_C21 * ih, c.K1[i], c.F[i]);
        c.Y[i] = c.N[i] + 2.0 * c.K1[i];
      }
      __syncthreads();
      if (warp == 0) {  // stage 2 on warp 0 while the other warps evaluate F(Y3), Y3 = N + 2 K1
        lu_solve<R, 1>(net, c.A, c.dinv, c.K2, nullptr, lane);
        sherman(net, c.K2, c.U, c0, lane);
      } else {
        rhs(net, c, c.Y, false, nd, tid - 32, nt - 32, 1);
      }
      __syncthreads();
      mark(PH_STAGE12);
      if (warp == 0) {  // stage 3
        for (int i = lane; i < ns; i += 32) c.K3[i] = fma(ih, c.K1[i] - c.K2[i], c.F[i]);
        __syncwarp();
        lu_solve<R, 1>(net, c.A, c.dinv, c.K3, nullptr, lane);
        sherman(net, c.K3, c.U, c0, lane);
        for (int i = lane; i < ns; i += 32) c.Y[i] = c.N[i] + 2.0 * c.K1[i] + c.K3[i];
      }
      __syncthreads();
      rhs(net, c, c.Y, false, nd, tid, nt);
      mark(PH_STAGE3);
      if (warp == 0) {  // stage 4 and the error
        for (int i = lane; i < ns; i += 32)
          c.K4[i] = fma(ih, fma(-RODAS_C43, c.K3[i], c.K1[i] - c.K2[i]), c.F[i]);
        __syncwarp();
        lu_solve<R, 1>(net, c.A, c.dinv, c.K4, nullptr, lane);
        sherman(net, c.K4, c.U, c0, lane);
        try_error(net, c, s.t == 0.0, a.rtol, a.atol, lane);
      }
      __syncthreads();
      mark(PH_STAGE4);
      const double en = c.red[0];
      const bool ok = c.red[1] != 0.0;
      if (ok) {
        for (int i = tid; i < ns; i += nt) c.N[i] = fmax(c.Y[i], 0.0);
        s.t += ha;
        s.nok += 1.0;
      }
      const double fac = step_factor(en, ok, s.prej, s.pen, s.pha, ha);
      s.h = ha * fac;
      s.prej = !ok;
      s.pen = en;
      s.pha = ha;
      it++;
      __syncthreads();
      mark(PH_CONTROL);
    }
    // x = N / sum N in the network's order (write_state), then the guard on it (check_cell)
    if (warp == 0) {
      const double sum = lane_sum(c.N, ns, lane);
      if (lane == 0) c.red[3] = sum;
    }
    __syncthreads();
    const double sum = c.red[3];
    for (int i = tid; i < ns; i += nt) c.Y[__ldg(net.perm + i)] = c.N[i] / sum;
    const double *at = net.atoms, *xin = x0;
    stage_guard_inputs(net, c, x0, tid, nt, &at, &xin);
    __syncthreads();
    if (warp == 0) {
      const int done = (st == 0 && s.t >= dt * MX_CALL_END) ? 1 : 0;
      const int g = st == 0 ? check_cell(net, xin, c.Y, done, s.nok, a.atol, lane, at, c.G) : 0;
      if (lane == 0) {
        a.h_out[cell] = s.h;
        a.done[cell] = done;
        a.steps[cell] = s.nok;
        int r = 0;
        if (st == MX_REFUSED_COLD)
          atomicAdd(a.count + MX_COUNT_COLD, 1);
        else if (st == MX_REFUSED_HOT)
          atomicAdd(a.count + MX_COUNT_HOT, 1);
        else if (st == MX_REFUSED_BAD_INPUT)
          atomicAdd(a.count + MX_COUNT_BAD_INPUT, 1);
        else {
          if (g & GUARD_NONFINITE) atomicAdd(a.count + MX_COUNT_NONFINITE, 1);
          if (g & GUARD_UNFINISHED) atomicAdd(a.count + MX_COUNT_UNFINISHED, 1);
          if (g & GUARD_DRIFT) atomicAdd(a.count + MX_COUNT_DRIFT, 1);
          if (g) {
            r = 1;
            a.list[atomicAdd(a.count + MX_COUNT_RECOMPUTED, 1)] = cell;
          }
        }
        a.flag[cell] = r;
        if (a.tries) {
          atomicAdd(a.tries, (unsigned long long)tries);
          atomicAdd(a.tries + 1, (unsigned long long)retries);
        }
        c.ints[1] = (int)(gridDim.x + atomicAdd(LIST ? a.in_count + 1 : a.count + MX_COUNT_QUEUE, 1));
      }
    }
    __syncthreads();
    double* xo = a.x_out + (size_t)cell * ns;
    for (int i = tid; i < ns; i += nt) xo[i] = c.Y[i];
    q = c.ints[1];
    __syncthreads();
    mark(PH_OUTPUT);
  }
  if (PROF && tid == 0) {
#pragma unroll
    for (int p = 0; p < PH_COUNT; p++) atomicAdd((unsigned long long*)prof + p, (unsigned long long)ph[p]);
  }
}

// The recovery: listed cells recomputed from their inputs with the dense W = I / (gamma h) - Jn - w 1^T factored with
// threshold pivoting, REC_STEPS times the tries, and up to REC_RETRIES retries with a smaller first try when only the
// element test failed (recover.cuh:231-310).
template <int W, int R>
__global__ void __launch_bounds__(32 * W, 16 / W) recover_kernel(const Net net, const CallArgs a, int max_steps) {
  const int nfl = a.count[MX_COUNT_RECOMPUTED];
  if ((int)blockIdx.x >= nfl) return;
  extern __shared__ double smem[];
  const Cell c = cell_arrays(net, smem);
  const int tid = (int)threadIdx.x, nt = 32 * W, lane = tid & 31, warp = tid >> 5, ns = net.ns, ld = net.ld;
  int* pr = c.ints + 4;
  int q = (int)blockIdx.x;
  while (q < nfl) {
    const int cell = a.list[q];
    const double Tc = a.T[cell], dt = a.dt[cell], hin = a.h_in[cell];
    const double nd = a.P[cell] / (MX_KB * Tc);
    const double* x0 = a.x + (size_t)cell * ns;
    const double* Jc = a.J + (size_t)cell * net.nj;
    cell_rates(net, c, Tc, nd, Jc, tid, nt);  // a listed cell passed the screening (status 0)
    const double h0 = isfinite(hin) ? hin : dt, m = fmin(h0, dt);
    for (int k = 0;; k++) {
      for (int i = tid; i < ns; i += nt) c.N[i] = x0[__ldg(net.perm + i)];
      __syncthreads();
      const double start = k == 0 ? m : fmin(m, dt * pow(MX_REC_RETRY_SPLIT, (double)k));
      StepState s = {fmax(start, MX_H_MIN), 0.0, 0.0, 0.0, 0.0, false};
      int it = dt > 0.0 ? 0 : max_steps;
      while (it < max_steps && s.t < dt * MX_CALL_END) {
        const double ha = fmin(s.h, dt - s.t), igh = 1.0 / (GAMMA * ha), ih = 1.0 / ha;
        if (tid == 0 && a.tries) atomicAdd(a.tries + 2, 1ull);
        const double ntot = rhs(net, c, c.N, true, nd, tid, nt);
        jacobian_w(net, c, ntot, tid, nt);
        for (int e = tid; e < ns * ns; e += nt) {  // form_dense_w
          const int i = e / ns, j = e - i * ns;
          double* p = c.A + i * ld + j;
          *p = (i == j ? *p + igh : *p) - c.U[i];
        }
        __syncthreads();
        if (warp == 0) {
          for (int i = lane; i < ns; i += 32) c.K1[i] = c.F[i];
          __syncwarp();
          dense_lu_pivot(net, c.A, c.dinv, pr, lane);
          dense_solve<R>(net, c.A, c.dinv, pr, c.K1, lane);
          for (int i = lane; i < ns; i += 32) c.K2[i] = fma(RODAS_C21 * ih, c.K1[i], c.F[i]);
          __syncwarp();
          dense_solve<R>(net, c.A, c.dinv, pr, c.K2, lane);
          for (int i = lane; i < ns; i += 32) c.Y[i] = c.N[i] + 2.0 * c.K1[i];
        }
        __syncthreads();
        rhs(net, c, c.Y, false, nd, tid, nt);
        if (warp == 0) {
          for (int i = lane; i < ns; i += 32) c.K3[i] = fma(ih, c.K1[i] - c.K2[i], c.F[i]);
          __syncwarp();
          dense_solve<R>(net, c.A, c.dinv, pr, c.K3, lane);
          for (int i = lane; i < ns; i += 32) c.Y[i] = c.N[i] + 2.0 * c.K1[i] + c.K3[i];
        }
        __syncthreads();
        rhs(net, c, c.Y, false, nd, tid, nt);
        if (warp == 0) {
          for (int i = lane; i < ns; i += 32)
            c.K4[i] = fma(ih, fma(-RODAS_C43, c.K3[i], c.K1[i] - c.K2[i]), c.F[i]);
          __syncwarp();
          dense_solve<R>(net, c.A, c.dinv, pr, c.K4, lane);
          try_error(net, c, s.t == 0.0, a.rtol, a.atol, lane);
        }
        __syncthreads();
        const double en = c.red[0];
        const bool ok = c.red[1] != 0.0;
        if (ok) {
          for (int i = tid; i < ns; i += nt) c.N[i] = fmax(c.Y[i], 0.0);
          s.t += ha;
          s.nok += 1.0;
        }
        const double fac = step_factor(en, ok, s.prej, s.pen, s.pha, ha);
        s.h = ha * fac;
        s.prej = !ok;
        s.pen = en;
        s.pha = ha;
        it++;
        __syncthreads();
      }
      if (warp == 0) {
        const double sum = lane_sum(c.N, ns, lane);
        if (lane == 0) c.red[3] = sum;
      }
      __syncthreads();
      const double sum = c.red[3];
      for (int i = tid; i < ns; i += nt) c.Y[__ldg(net.perm + i)] = c.N[i] / sum;
      const double *at = net.atoms, *xin = x0;
      stage_guard_inputs(net, c, x0, tid, nt, &at, &xin);
      __syncthreads();
      if (warp == 0) {
        const int dn = s.t >= dt * MX_CALL_END ? 1 : 0;
        const int g = check_cell(net, xin, c.Y, dn, s.nok, a.atol, lane, at, c.G);
        if (lane != 0) {
        } else if (g == GUARD_DRIFT && k < MX_REC_RETRIES) {
          c.ints[1] = -1;  // only the element test failed: again from the inputs with a smaller first try
        } else {
          a.h_out[cell] = s.h;
          a.done[cell] = g ? 0 : dn;
          a.steps[cell] = s.nok;
          a.flag[cell] = g ? 2 : 1;
          atomicAdd(a.count + (g ? MX_COUNT_STILL_FAILED : MX_COUNT_RECOVERED), 1);
          c.ints[1] = (int)(gridDim.x + atomicAdd(a.count + MX_COUNT_RECOVERY_QUEUE, 1));
        }
      }
      __syncthreads();
      double* xo = a.x_out + (size_t)cell * ns;
      for (int i = tid; i < ns; i += nt) xo[i] = c.Y[i];
      const int nq = c.ints[1];
      __syncthreads();
      if (nq >= 0) {
        q = nq;
        break;
      }
    }
  }
}

// One fresh try of one cell with every stage written out (a test hook that runs the call kernel's device functions):
// out = kf, kr [nr each], F, u0 [ns each], -Jn [ns][ns], w [ns], LU factors [ns][ns], dinv, K1, K2, K3, K4, Y [ns each],
// err, ok.
template <int W, int R>
__global__ void __launch_bounds__(32 * W) debug_try_kernel(const Net net, const double* x0, double Tc, double P,
                                                           double ha, const double* Jc, double rtol, double atol,
                                                           double* out) {
  extern __shared__ double smem[];
  const Cell c = cell_arrays(net, smem);
  const int tid = (int)threadIdx.x, nt = 32 * W, lane = tid & 31, warp = tid >> 5, ns = net.ns, ld = net.ld;
  const double nd = P / (MX_KB * Tc);
  double* o = out;
  for (int i = tid; i < ns; i += nt) c.N[i] = x0[__ldg(net.perm + i)];
  __syncthreads();
  cell_rates(net, c, Tc, nd, Jc, tid, nt);
  for (int r = tid; r < net.nr; r += nt) {
    o[r] = c.kf[r];
    o[net.nr + r] = c.kr[r];
  }
  o += 2 * net.nr;
  const double igh = 1.0 / (GAMMA * ha), ih = 1.0 / ha;
  const double ntot = rhs(net, c, c.N, true, nd, tid, nt);
  for (int i = tid; i < ns; i += nt) {
    o[i] = c.F[i];
    o[ns + i] = c.U[i];
  }
  o += 2 * ns;
  __syncthreads();
  jacobian_w(net, c, ntot, tid, nt);
  // -Jn is in A before the diagonal; w in U
  for (int e = tid; e < ns * ns; e += nt) o[e] = c.A[(e / ns) * ld + e % ns];
  o += ns * ns;
  for (int i = tid; i < ns; i += nt) o[i] = c.U[i];
  o += ns;
  __syncthreads();
  for (int i = tid; i < ns; i += nt) c.A[i * ld + i] += igh;
  __syncthreads();
  lu_factor<32 * W>(net, c.A, c.dinv, tid);
  for (int e = tid; e < ns * ns; e += nt) o[e] = c.A[(e / ns) * ld + e % ns];
  o += ns * ns;
  for (int i = tid; i < ns; i += nt) o[i] = c.dinv[i];
  o += ns;
  double c0 = 0.0;
  if (warp == 0) {
    for (int i = lane; i < ns; i += 32) c.K1[i] = c.F[i];
    __syncwarp();
    lu_solve<R, 2>(net, c.A, c.dinv, c.K1, c.U, lane);
    c0 = 1.0 / (1.0 - lane_sum(c.U, ns, lane));
    sherman(net, c.K1, c.U, c0, lane);
    for (int i = lane; i < ns; i += 32) c.K2[i] = fma(RODAS_C21 * ih, c.K1[i], c.F[i]);
    __syncwarp();
    lu_solve<R, 1>(net, c.A, c.dinv, c.K2, nullptr, lane);
    sherman(net, c.K2, c.U, c0, lane);
    for (int i = lane; i < ns; i += 32) c.Y[i] = c.N[i] + 2.0 * c.K1[i];
  }
  __syncthreads();
  rhs(net, c, c.Y, false, nd, tid, nt);
  if (warp == 0) {
    for (int i = lane; i < ns; i += 32) c.K3[i] = fma(ih, c.K1[i] - c.K2[i], c.F[i]);
    __syncwarp();
    lu_solve<R, 1>(net, c.A, c.dinv, c.K3, nullptr, lane);
    sherman(net, c.K3, c.U, c0, lane);
    for (int i = lane; i < ns; i += 32) c.Y[i] = c.N[i] + 2.0 * c.K1[i] + c.K3[i];
  }
  __syncthreads();
  rhs(net, c, c.Y, false, nd, tid, nt);
  if (warp == 0) {
    for (int i = lane; i < ns; i += 32) c.K4[i] = fma(ih, fma(-RODAS_C43, c.K3[i], c.K1[i] - c.K2[i]), c.F[i]);
    __syncwarp();
    lu_solve<R, 1>(net, c.A, c.dinv, c.K4, nullptr, lane);
    sherman(net, c.K4, c.U, c0, lane);
    try_error(net, c, true, rtol, atol, lane);
  }
  __syncthreads();
  for (int i = tid; i < ns; i += nt) {
    o[i] = c.K1[i];
    o[ns + i] = c.K2[i];
    o[2 * ns + i] = c.K3[i];
    o[3 * ns + i] = c.K4[i];
    o[4 * ns + i] = c.Y[i];
  }
  o += 5 * ns;
  if (tid == 0) {
    o[0] = c.red[0];
    o[1] = c.red[1];
  }
}

// Cycles of each device function of a try, repeated reps times on one cell in every CTA (a tuning hook): rates,
// F, Jacobian and w, LU, two-vector solve, one-vector solve, Sherman-Morrison, error, guard test. cycles[9] receives
// the CTA-0 averages.
template <int W, int R>
__global__ void __launch_bounds__(32 * W, 16 / W) time_phases_kernel(const Net net, const double* x0, double Tc, double P,
                                                             double ha, const double* Jc, int reps,
                                                             long long* cycles) {
  extern __shared__ double smem[];
  const Cell c = cell_arrays(net, smem);
  const int tid = (int)threadIdx.x, nt = 32 * W, lane = tid & 31, warp = tid >> 5, ns = net.ns, ld = net.ld;
  const double nd = P / (MX_KB * Tc), igh = 1.0 / (GAMMA * ha);
  long long acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int i = tid; i < ns; i += nt) c.N[i] = x0[__ldg(net.perm + i)];
  __syncthreads();
  for (int r = 0; r < reps; r++) {
    long long t = clock64();
    cell_rates(net, c, Tc, nd, Jc, tid, nt);
    long long u = clock64();
    acc[0] += u - t;
    const double ntot = rhs(net, c, c.N, true, nd, tid, nt);
    t = clock64();
    acc[1] += t - u;
    jacobian_w(net, c, ntot, tid, nt);
    for (int i = tid; i < ns; i += nt) c.A[i * ld + i] += igh;
    __syncthreads();
    u = clock64();
    acc[2] += u - t;
    lu_factor<32 * W>(net, c.A, c.dinv, tid);
    t = clock64();
    acc[3] += t - u;
    if (warp == 0) {
      for (int i = lane; i < ns; i += 32) c.K1[i] = c.F[i];
      __syncwarp();
      u = clock64();
      lu_solve<R, 2>(net, c.A, c.dinv, c.K1, c.U, lane);
      t = clock64();
      acc[4] += t - u;
      lu_solve<R, 1>(net, c.A, c.dinv, c.K2, nullptr, lane);
      u = clock64();
      acc[5] += u - t;
      sherman(net, c.K2, c.U, 0.5, lane);
      t = clock64();
      acc[6] += t - u;
      try_error(net, c, true, 1e-3, 1e-25, lane);
      u = clock64();
      acc[7] += u - t;
    }
    __syncthreads();
    if (warp == 0) {
      for (int i = lane; i < ns; i += 32) c.Y[__ldg(net.perm + i)] = c.N[i];
      __syncwarp();
      t = clock64();
      check_cell(net, x0, c.Y, 1, 1.0, 1e-25, lane, net.atoms, c.G);
      u = clock64();
      acc[8] += u - t;
    }
    __syncthreads();
  }
  if (blockIdx.x == 0 && tid == 0)
    for (int q = 0; q < 9; q++) cycles[q] = acc[q] / reps;
}

// The guard alone, one warp per cell (guard.cuh:114-140), on results in global memory; 4 warps per block.
__global__ void __launch_bounds__(128) guard_kernel(const Net net, const double* x0, double* xout, const int* done,
                                                    const double* nok, const int* status, int B, double atol,
                                                    int* flag, int* count, int* list) {
  extern __shared__ double gsm[];  // guard_scratch(ns) doubles per warp
  const int cell = (int)(blockIdx.x * 4 + (threadIdx.x >> 5)), lane = (int)(threadIdx.x & 31);
  if (cell >= B) return;
  const int s = status[cell];
  double* scr = gsm + (threadIdx.x >> 5) * guard_scratch(net.ns);
  const int g = s == 0 ? check_cell(net, x0 + (size_t)cell * net.ns, xout + (size_t)cell * net.ns, done[cell],
                                    nok[cell], atol, lane, net.atoms, scr)
                       : 0;
  if (lane != 0) return;
  int r = 0;
  if (s == MX_REFUSED_COLD)
    atomicAdd(count + MX_COUNT_COLD, 1);
  else if (s == MX_REFUSED_HOT)
    atomicAdd(count + MX_COUNT_HOT, 1);
  else if (s == MX_REFUSED_BAD_INPUT)
    atomicAdd(count + MX_COUNT_BAD_INPUT, 1);
  else {
    if (g & GUARD_NONFINITE) atomicAdd(count + MX_COUNT_NONFINITE, 1);
    if (g & GUARD_UNFINISHED) atomicAdd(count + MX_COUNT_UNFINISHED, 1);
    if (g & GUARD_DRIFT) atomicAdd(count + MX_COUNT_DRIFT, 1);
    if (g) {
      r = 1;
      list[atomicAdd(count + MX_COUNT_RECOMPUTED, 1)] = cell;
    }
  }
  flag[cell] = r;
}

template <int W, int R>
void kernels_for(mx_solver* s) {
  s->timer = time_phases_kernel<W, R>;
  s->call = call_kernel<W, R, false>;
  s->call_prof = call_kernel<W, R, true>;
  s->call_list = call_kernel<W, R, false, true>;
  s->recover = recover_kernel<W, R>;
  s->debug = debug_try_kernel<W, R>;
  s->rows_per_lane = R;
}

template <int W>
bool kernels_of(int ns, mx_solver* s) {  // rows per lane of the warp solves: species up to 32, 64, 96, 128, 256
  const int need = (ns + 31) / 32;
  if (need <= 1) { kernels_for<W, 1>(s); return true; }
  if (need <= 2) { kernels_for<W, 2>(s); return true; }
  if (need <= 3) { kernels_for<W, 3>(s); return true; }
  if (need <= 4) { kernels_for<W, 4>(s); return true; }
  if (need <= 8) { kernels_for<W, 8>(s); return true; }
  return false;
}

// the kernels for the solver's warps per cell (2 or 4: the tables' thread streams were built for one of them)
bool pick_kernels(int ns, mx_solver* s) {
  if (s->warps == 4) return kernels_of<4>(ns, s);
  if (s->warps == 2) return kernels_of<2>(ns, s);
  return false;
}

}  // namespace

namespace {

// The shared-memory layout of one cell (doubles): A [ns][ld], kf kr, v (or G/RT), n, N Y F U K1-K4 dinv, red, ints,
// the S.v pieces' partial sums, and the guard's scratch; sets net's offsets and net.doubles.
void cell_layout(const mx_network* n, Net& net) {
  const int ns = n->ns, nr = n->nr;
  net.ld = ns | 1;  // odd: a column of A is read without bank conflicts
  int off = 0;
  auto take = [&](int doubles) {
    const int o = off;
    off += (doubles + 1) & ~1;
    return o;
  };
  net.oA = take(ns * net.ld);
  net.a_doubles = ns * net.ld;
  net.oK = take(2 * nr + 2);
  net.oV = take(std::max(nr + 1, ns + 1));
  net.on = take(ns + 1);
  net.oN = take(ns);
  net.oY = take(ns);
  net.oF = take(ns);
  net.oU = take(ns);
  net.oK1 = take(ns);
  net.oK2 = take(ns);
  net.oK3 = take(ns);
  net.oK4 = take(ns);
  net.oD = take(ns);
  net.oRed = take(8);
  net.oInts = take((ns + 8) / 2 + 1);
  net.oPart = take(n->n_pieces);
  {  // the guard's scratch: in the matrix's space past the staged atoms and input row when it fits there
    const int staged = (ns * n->nel + ns + 1) & ~1;
    if (staged + guard_scratch(ns) <= ns * net.ld)
      net.oG = net.oA + staged;
    else
      net.oG = take(guard_scratch(ns));
  }
  net.doubles = off;
}

void release(mx_solver* s) {
  for (void* p : s->buffers) cudaFree(p);
  s->buffers.clear();
  if (s->list) cudaFree(s->list);
  s->list = nullptr;
  if (s->sel) cudaFree(s->sel);
  s->sel = nullptr;
  if (s->sel_count) cudaFree(s->sel_count);
  s->sel_count = nullptr;
  mx_release_derivatives(s);
}

// The mixed path's list of cells for the plain kernel, grown to B cells, and its two counters.
int grow_sel(mx_solver* s, int64_t B, char* err, size_t errlen) {
  cudaError_t e = cudaSuccess;
  if (!s->sel_count) e = cudaMalloc(&s->sel_count, 2 * sizeof(int));
  if (e == cudaSuccess && B > s->sel_capacity) {
    if (s->sel) cudaFree(s->sel);
    s->sel = nullptr;
    s->sel_capacity = 0;
    e = cudaMalloc(&s->sel, (size_t)B * sizeof(int));
    if (e == cudaSuccess) s->sel_capacity = B;
  }
  if (e != cudaSuccess) {
    set_error(err, errlen, "mx_call: the mixed path's list of %lld cells: %s", (long long)B, cudaGetErrorString(e));
    return MX_ERR_CUDA;
  }
  return MX_OK;
}

__global__ void add_escalated_kernel(const int* sel_count, long long* escalated) {
  if (threadIdx.x == 0) escalated[0] += sel_count[0];
}

}  // namespace

extern "C" int mx_create(const mx_network* n, double drift, int device, mx_solver** out, char* err, size_t errlen) {
  if (!n || !out) {
    set_error(err, errlen, "mx_create: null network or output");
    return MX_ERR_ARGUMENT;
  }
  *out = nullptr;
  if (n->ns < 1 || n->ns > MX_MAX_SPECIES || n->nr < 0 || n->nr >= 2048 || n->nel < 1 || n->nel > MX_MAX_ELEMENTS ||
      n->nj != n->nr - n->nrt || n->n_entries < 0) {
    set_error(err, errlen, "mx_create: network sizes out of range (ns %d, nr %d, nel %d)", n->ns, n->nr, n->nel);
    return MX_ERR_NETWORK;
  }
  if (!(drift >= 0.0 && drift <= 1e300)) {
    set_error(err, errlen, "drift: a finite allowance of at least 0 expected, got %g", drift);
    return MX_ERR_ARGUMENT;
  }
  DeviceScope scope(device);
  if (scope.status != cudaSuccess) {
    set_error(err, errlen, "mx_create: device %d: %s", device, cudaGetErrorString(scope.status));
    return MX_ERR_CUDA;
  }
  mx_solver* s = new (std::nothrow) mx_solver();
  if (!s) return MX_ERR_CUDA;
  s->device = device;
  Net& net = s->net;
  const int ns = n->ns, nr = n->nr;
  net.ns = ns;
  net.nr = nr;
  net.nrt = n->nrt;
  net.nj = n->nj;
  net.nel = n->nel;
  net.n_entries = n->n_entries;
  net.drift = drift;
  double etot = 0.0;
  for (int i = 0; i < ns * n->nel; i++) etot += n->atoms[i];
  net.etot = etot;
  s->warps = n->stream_threads[0] / 32;
  if (n->stream_threads[0] % 32 || (s->warps != 2 && s->warps != 4) || n->stream_threads[1] != 32 * (s->warps - 1)) {
    set_error(err, errlen, "mx_create: thread streams for %d and %d threads; the kernels take 2 or 4 warps per cell "
              "(64 and 32, or 128 and 96 threads)", n->stream_threads[0], n->stream_threads[1]);
    delete s;
    return MX_ERR_NETWORK;
  }
  if (!pick_kernels(ns, s)) {
    delete s;
    return MX_ERR_NETWORK;
  }
  cell_layout(n, net);
  s->smem = (size_t)net.doubles * sizeof(double);

  int optin = 0;
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
  cudaDeviceGetAttribute(&s->sms, cudaDevAttrMultiProcessorCount, device);
  if ((size_t)optin < s->smem) {
    set_error(err, errlen, "one cell needs %zu B of shared memory; the device has %d per block", s->smem, optin);
    delete s;
    return MX_ERR_NETWORK;
  }
  cudaError_t e = cudaFuncSetAttribute((const void*)s->call, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s->smem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute((const void*)s->recover, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s->smem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute((const void*)s->debug, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s->smem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute((const void*)s->timer, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s->smem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute((const void*)s->call_prof, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s->smem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute((const void*)s->call_list, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s->smem);
  if (e == cudaSuccess)
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&s->call_ctas, (const void*)s->call, 32 * s->warps, s->smem);
  if (e == cudaSuccess)
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&s->recover_ctas, (const void*)s->recover, 32 * s->warps, s->smem);
  if (e == cudaSuccess && (s->call_ctas < 1 || s->recover_ctas < 1)) e = cudaErrorInvalidConfiguration;
  // the tables
  std::vector<uint64_t> rx8(nr);
  for (int r = 0; r < nr; r++) {
    uint64_t w = 0;
    for (int q = 0; q < 6; q++) w |= (uint64_t)n->rx[6 * r + q] << (8 * q);
    rx8[r] = w;
  }
  s->rx8_host = rx8;
  {  // S's columns from its rows' terms: species bytes 0-5 (padding ns), coefficient codes 2 bits each from bit 48
    std::vector<int> used(nr, 0);
    s->st8_host.assign(nr, 0);
    for (int r = 0; r < nr; r++)
      for (int m = 0; m < 6; m++) s->st8_host[r] |= (uint64_t)ns << (8 * m);
    for (int i = 0; i < ns; i++)
      for (int t = n->sv_ptr[i]; t < n->sv_ptr[i + 1]; t++) {
        const uint32_t w = n->sv_term[t];
        const int r = (int)(w & 0xffff), m = used[r]++;
        if (r >= nr || m >= 6) {
          set_error(err, errlen, "mx_create: reaction %d has more than 6 stoichiometry entries", r);
          delete s;
          return MX_ERR_NETWORK;
        }
        s->st8_host[r] &= ~((uint64_t)255 << (8 * m));
        s->st8_host[r] |= (uint64_t)i << (8 * m) | (uint64_t)((w >> 16) & 3) << (48 + 2 * m);
      }
  }
  const int nsv = n->sv_ptr[ns], njt = n->jac_ptr[n->n_entries];
  if (e == cudaSuccess) e = upload(s, n->perm, ns, &net.perm);
  if (e == cudaSuccess) e = upload(s, rx8.data(), nr, &net.rx8);
  if (e == cudaSuccess) e = upload(s, n->rc, (size_t)nr * 14, &net.rc);
  if (e == cudaSuccess) e = upload(s, n->rf, nr, &net.rf);
  if (e == cudaSuccess) e = upload(s, n->nasa, (size_t)2 * ns * 9, &net.nasa);
  if (e == cudaSuccess) e = upload(s, n->atoms, (size_t)ns * n->nel, &net.atoms);
  if (e == cudaSuccess) e = upload(s, n->sv_ptr, ns + 1, &net.sv_ptr);
  if (e == cudaSuccess) e = upload(s, n->sv_term, nsv, &net.sv_term);
  if (e == cudaSuccess) e = upload(s, n->jac_ptr, n->n_entries + 1, &net.jac_ptr);
  if (e == cudaSuccess) e = upload(s, n->jac_entry, n->n_entries, &net.jac_entry);
  if (e == cudaSuccess) e = upload(s, n->jac_term, njt, &net.jac_term);
  net.n_pieces = n->n_pieces;
  if (e == cudaSuccess) e = upload(s, n->sv_row_ptr, ns + 1, &net.sv_row_ptr);
  for (int g = 0; g < 2 && e == cudaSuccess; g++) {
    const int t = n->stream_threads[g];
    net.st_threads[g] = t;
    net.sv_rounds[g] = n->sv_rounds[g];
    net.sv_nrows[g] = n->sv_nrows[g];
    net.jac_rounds[g] = n->jac_rounds[g];
    net.jac_nents[g] = n->jac_nents[g];
    e = upload(s, n->sv_stream[g], (size_t)n->sv_rounds[g] * t, &net.sv[g]);
    if (e == cudaSuccess) e = upload(s, n->sv_rows[g], (size_t)n->sv_nrows[g] * t, &net.sv_rows[g]);
    if (e == cudaSuccess) e = upload(s, n->jac_stream[g], (size_t)n->jac_rounds[g] * t, &net.jt[g]);
    if (e == cudaSuccess) e = upload(s, n->jac_dst[g], (size_t)n->jac_nents[g] * t, &net.jd[g]);
  }
  if (e != cudaSuccess) {
    set_error(err, errlen, "mx_create: %s", cudaGetErrorString(e));
    release(s);
    delete s;
    return MX_ERR_CUDA;
  }
  const int mrc = mx_mixed_prepare(s, n->n_pieces, err, errlen);
  if (mrc) {
    release(s);
    delete s;
    return mrc;
  }
  *out = s;
  return MX_OK;
}

extern "C" int mx_call(mx_solver* s, const double* x, const double* T, const double* P, const double* dt,
                       const double* h_in, const double* J, int64_t B, double rtol, double atol, int32_t max_steps,
                       double* x_out, double* h_out, int32_t* done, double* steps, int32_t* flag, int32_t* status,
                       int32_t* count, int64_t* total, void* stream, char* err, size_t errlen) {
  if (!s) {
    set_error(err, errlen, "this solver was closed; build a new one");
    return MX_ERR_CLOSED;
  }
  if (B < 0 || B > 0x7fffffff) {
    set_error(err, errlen, "mx_call: B out of range: %lld", (long long)B);
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
  if (!count || !total || (B > 0 && (!x || !T || !P || !dt || !h_in || !x_out || !h_out || !done || !steps ||
                                     !flag || !status || (s->net.nj > 0 && !J)))) {
    set_error(err, errlen, "mx_call: a required array is null");
    return MX_ERR_ARGUMENT;
  }
  DeviceScope scope(s->device);
  if (scope.status != cudaSuccess) {
    set_error(err, errlen, "mx_call: device %d: %s", s->device, cudaGetErrorString(scope.status));
    return MX_ERR_CUDA;
  }
  cudaStream_t st = (cudaStream_t)stream;
  int rc = grow_list(s, std::max<int64_t>(B, 1), err, errlen);
  if (rc) return rc;
  const bool mixed = s->precision == MX_PRECISION_MIXED && B > 0;
  if (mixed) {
    rc = grow_sel(s, B, err, errlen);
    if (rc) return rc;
  }
  cudaError_t e = cudaMemsetAsync(count, 0, MX_COUNT_SLOTS * sizeof(int32_t), st);
  if (e == cudaSuccess && mixed) e = cudaMemsetAsync(s->sel_count, 0, 2 * sizeof(int), st);
  if (e == cudaSuccess && B > 0) {
    CallArgs a{x, T, P, dt, h_in, J, (int)B, rtol, atol, max_steps, x_out, h_out, done, steps, flag, status, count,
               s->list, s->tries, nullptr, nullptr, s->sel, s->sel_count};
    const int grid = call_grid(s, B);
    if (mixed) {
      // the mixed kernel, then the plain kernel on the cells it handed back (it returns at once when none)
      e = mx_mixed_launch(s, a, B, false, st);
      CallArgs back = a;
      back.in_list = s->sel;
      back.in_count = s->sel_count;
      if (e == cudaSuccess) s->call_list<<<grid, 32 * s->warps, s->smem, st>>>(s->net, back, nullptr);
    } else if (s->phases) {
      s->call_prof<<<grid, 32 * s->warps, s->smem, st>>>(s->net, a, s->phases);
    } else {
      s->call<<<grid, 32 * s->warps, s->smem, st>>>(s->net, a, nullptr);
    }
    const int rgrid = (int)std::min<int64_t>(B, (int64_t)s->recover_ctas * s->sms);
    if (e == cudaSuccess) s->recover<<<rgrid, 32 * s->warps, s->smem, st>>>(s->net, a, MX_REC_STEPS * max_steps);
    if (e == cudaSuccess) e = cudaGetLastError();
  }
  if (e == cudaSuccess) {
    add_counts_kernel<<<1, 32, 0, st>>>(count, (long long*)total);
    if (mixed && s->escalated) add_escalated_kernel<<<1, 32, 0, st>>>(s->sel_count, s->escalated);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) {
    set_error(err, errlen, "mx_call: %s", cudaGetErrorString(e));
    return MX_ERR_CUDA;
  }
  return MX_OK;
}

extern "C" int mx_set_precision(mx_solver* s, int32_t precision, int32_t sweeps, double tol) {
  if (!s) return MX_ERR_CLOSED;
  if ((precision != MX_PRECISION_FP64 && precision != MX_PRECISION_MIXED) || sweeps < 1 ||
      sweeps > MX_MIXED_MAX_SWEEPS || !(tol > 0.0 && tol < 1e300))
    return MX_ERR_ARGUMENT;
  s->precision = precision;
  s->sweeps = sweeps;
  s->mixed_tol = tol;
  return MX_OK;
}

extern "C" int mx_set_escalation_counter(mx_solver* s, int64_t* counter) {
  if (!s) return MX_ERR_CLOSED;
  s->escalated = (long long*)counter;
  return MX_OK;
}

extern "C" int mx_guard(mx_solver* s, const double* x, double* x_out, const int32_t* done, const double* steps,
                        const int32_t* status, int64_t B, double atol, int32_t* flag, int32_t* count, void* stream,
                        char* err, size_t errlen) {
  if (!s) {
    set_error(err, errlen, "this solver was closed; build a new one");
    return MX_ERR_CLOSED;
  }
  if (B < 0 || B > 0x7fffffff || !count || (B > 0 && (!x || !x_out || !done || !steps || !status || !flag))) {
    set_error(err, errlen, "mx_guard: bad arguments");
    return MX_ERR_ARGUMENT;
  }
  DeviceScope scope(s->device);
  cudaStream_t st = (cudaStream_t)stream;
  int rc = grow_list(s, std::max<int64_t>(B, 1), err, errlen);
  if (rc) return rc;
  cudaError_t e = cudaMemsetAsync(count, 0, MX_COUNT_SLOTS * sizeof(int32_t), st);
  if (e == cudaSuccess && B > 0) {
    const size_t gsmem = 4 * sizeof(double) * guard_scratch(s->net.ns);
    guard_kernel<<<(int)((B + 3) / 4), 128, gsmem, st>>>(s->net, x, x_out, done, steps, status, (int)B, atol, flag,
                                                              count, s->list);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) {
    set_error(err, errlen, "mx_guard: %s", cudaGetErrorString(e));
    return MX_ERR_CUDA;
  }
  return MX_OK;
}

extern "C" int mx_info(const mx_solver* s, int32_t* values, int32_t n) {
  if (!s || !values) return MX_ERR_ARGUMENT;
  const int32_t v[] = {s->warps, s->rows_per_lane, (int32_t)s->smem, s->call_ctas, s->recover_ctas, s->sms, s->net.ld,
                       s->grid_ctas < 0 ? s->call_ctas : s->grid_ctas, (int32_t)s->list_capacity,
                       (int32_t)s->mixed_smem, s->mixed_ctas, s->precision, s->sweeps};
  for (int i = 0; i < n && i < (int)(sizeof v / sizeof v[0]); i++) values[i] = v[i];
  return MX_OK;
}

extern "C" int mx_set_grid(mx_solver* s, int32_t ctas_per_sm) {
  if (!s) return MX_ERR_CLOSED;
  if (ctas_per_sm < -1 || ctas_per_sm > std::max(s->call_ctas, s->mixed_ctas)) return MX_ERR_ARGUMENT;
  s->grid_ctas = ctas_per_sm;
  return MX_OK;
}

extern "C" int mx_destroy(mx_solver* s) {
  if (!s) return MX_OK;
  {
    DeviceScope scope(s->device);
    release(s);
  }
  delete s;
  return MX_OK;
}

extern "C" int mx_debug_try(mx_solver* s, const double* x, double T, double P, double h, const double* J, double rtol,
                            double atol, double* out, void* stream) {
  if (!s || !x || !out || (s->net.nj > 0 && !J)) return MX_ERR_ARGUMENT;
  DeviceScope scope(s->device);
  s->debug<<<1, 32 * s->warps, s->smem, (cudaStream_t)stream>>>(s->net, x, T, P, h, J, rtol, atol, out);
  return cudaGetLastError() == cudaSuccess ? MX_OK : MX_ERR_CUDA;
}

extern "C" int mx_time_phases(mx_solver* s, const double* x, double T, double P, double h, const double* J,
                              int32_t reps, int32_t ctas, int64_t* cycles, void* stream) {
  if (!s || !x || !cycles || reps < 1 || ctas < 1 || (s->net.nj > 0 && !J)) return MX_ERR_ARGUMENT;
  DeviceScope scope(s->device);
  s->timer<<<ctas, 32 * s->warps, s->smem, (cudaStream_t)stream>>>(s->net, x, T, P, h, J, reps, (long long*)cycles);
  return cudaGetLastError() == cudaSuccess ? MX_OK : MX_ERR_CUDA;
}

extern "C" int mx_set_phase_counter(mx_solver* s, int64_t* cycles) {
  if (!s) return MX_ERR_CLOSED;
  s->phases = (long long*)cycles;
  return MX_OK;
}

extern "C" int mx_set_try_counter(mx_solver* s, int64_t* tries) {
  if (!s) return MX_ERR_CLOSED;
  s->tries = (unsigned long long*)tries;
  return MX_OK;
}

namespace {
// Independent fma chains, for the FP64 issue peak of the device (a measurement of the roofline's denominator).
__global__ void probe_fp64_kernel(double* out, long long iters, double a, double b) {
  double x[8];
#pragma unroll
  for (int q = 0; q < 8; q++) x[q] = threadIdx.x * 1e-7 + q;
  for (long long i = 0; i < iters; i++) {
#pragma unroll
    for (int q = 0; q < 8; q++) x[q] = fma(x[q], a, b);
  }
  double s = 0.0;
#pragma unroll
  for (int q = 0; q < 8; q++) s += x[q];
  if (s == 12345.678) out[0] = s;  // keeps the chains alive
}
}  // namespace

extern "C" int mx_probe_fp64(int device, int64_t iters, double* gflops) {
  if (!gflops || iters < 1) return MX_ERR_ARGUMENT;
  DeviceScope scope(device);
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  double* out = nullptr;
  if (cudaMalloc(&out, sizeof(double)) != cudaSuccess) return MX_ERR_CUDA;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int blocks = sms * 8, threads = 256;
  probe_fp64_kernel<<<blocks, threads>>>(out, iters / 10 + 1, 0.999999, 1e-9);  // warm-up
  cudaEventRecord(e0);
  probe_fp64_kernel<<<blocks, threads>>>(out, iters, 0.999999, 1e-9);
  cudaEventRecord(e1);
  cudaError_t e = cudaEventSynchronize(e1);
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  if (e != cudaSuccess || ms <= 0.0f) return MX_ERR_CUDA;
  *gflops = 2.0 * 8.0 * (double)iters * blocks * threads / (ms * 1e-3) / 1e9;
  return MX_OK;
}

// ---- mx_call_static: the call for callers that cannot allocate device memory ----
// For a GCM whose framework holds the GPU's memory in its own pool, or whose time loop must not pay the device-wide
// synchronisation of cudaMalloc and cudaFree. The only scratch a call owns is the recompute list (one int per cell).
// Here it is a file-scope device array of MX_STATIC_MAX_CELLS entries that every mx_call_static call shares. In host
// code its name stands for a host-side shadow, not a device address, so each call looks up its address on the
// solver's device (cudaGetSymbolAddress, with that device current) and passes that to the kernels. Looking it up on
// every call, rather than caching it per device, keeps it right after a cudaDeviceReset or under another context.

static __device__ __align__(256) int g_static_list[MX_STATIC_MAX_CELLS];

namespace {

int static_list(int device, int** out, char* err, size_t errlen) {
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_static_list);
  if (e != cudaSuccess || !p) {
    set_error(err, errlen, "mx_call_static: the static scratch's address on device %d: %s", device,
              cudaGetErrorString(e));
    return MX_ERR_CUDA;
  }
  *out = static_cast<int*>(p);
  return MX_OK;
}

}  // namespace

extern "C" int mx_call_static(mx_solver* s, const double* x, const double* T, const double* P, const double* dt,
                              const double* h_in, const double* J, int64_t B, double rtol, double atol,
                              int32_t max_steps, double* x_out, double* h_out, int32_t* done, double* steps,
                              int32_t* flag, int32_t* status, int32_t* count, int64_t* total, void* stream, char* err,
                              size_t errlen) {
  if (!s) {
    set_error(err, errlen, "this solver was closed; build a new one");
    return MX_ERR_CLOSED;
  }
  if (B < 0 || B > MX_STATIC_MAX_CELLS) {
    set_error(err, errlen, "mx_call_static: B = %lld cells; from 0 to MX_STATIC_MAX_CELLS = %d expected (use mx_call "
              "for larger batches)", (long long)B, MX_STATIC_MAX_CELLS);
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
  if (!count || !total || (B > 0 && (!x || !T || !P || !dt || !h_in || !x_out || !h_out || !done || !steps ||
                                     !flag || !status || (s->net.nj > 0 && !J)))) {
    set_error(err, errlen, "mx_call_static: a required array is null");
    return MX_ERR_ARGUMENT;
  }
  DeviceScope scope(s->device);
  if (scope.status != cudaSuccess) {
    set_error(err, errlen, "mx_call_static: device %d: %s", s->device, cudaGetErrorString(scope.status));
    return MX_ERR_CUDA;
  }
  int* list = nullptr;
  const int rc = static_list(s->device, &list, err, errlen);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  // count holds the cell queue and the list's length: both must start at zero. The list itself needs no clearing:
  // a call writes each entry before its recovery kernel reads it.
  cudaError_t e = cudaMemsetAsync(count, 0, MX_COUNT_SLOTS * sizeof(int32_t), st);
  if (e == cudaSuccess && B > 0) {
    CallArgs a{x, T, P, dt, h_in, J, (int)B, rtol, atol, max_steps, x_out, h_out, done, steps, flag, status, count,
               list, s->tries};
    const int grid = call_grid(s, B);
    s->call<<<grid, 32 * s->warps, s->smem, st>>>(s->net, a, nullptr);
    const int rgrid = (int)std::min<int64_t>(B, (int64_t)s->recover_ctas * s->sms);
    s->recover<<<rgrid, 32 * s->warps, s->smem, st>>>(s->net, a, MX_REC_STEPS * max_steps);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) {
    add_counts_kernel<<<1, 32, 0, st>>>(count, (long long*)total);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) {
    set_error(err, errlen, "mx_call_static: %s", cudaGetErrorString(e));
    return MX_ERR_CUDA;
  }
  return MX_OK;
}

extern "C" const char* mx_version(void) { return "maxichem_b200 0.1 sm_100a"; }

extern "C" int mx_warps_per_cell(void) { return WARPS; }

extern "C" int mx_cells_per_sm(const mx_network* n, int32_t device) {
  if (!n || n->ns < 1 || n->ns > MX_MAX_SPECIES || n->nr < 0 || n->nr >= 2048 || n->nel < 1 ||
      n->nel > MX_MAX_ELEMENTS)
    return -MX_ERR_NETWORK;
  Net net{};
  cell_layout(n, net);
  int per_sm = 0, reserved = 0;
  if (cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, device) != cudaSuccess ||
      cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, device) != cudaSuccess)
    return -MX_ERR_CUDA;
  return (int)((size_t)per_sm / ((size_t)net.doubles * sizeof(double) + (size_t)reserved));
}

extern "C" int mx_warps_supported(int32_t warps) { return warps == 2 || warps == 4 ? 1 : 0; }
