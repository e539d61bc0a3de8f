// The mixed-precision call: the linear algebra of each Rodas3 try in FP32, everything whose stability needs it in FP64.
//
// Per try the matrix M0 = I / (gamma h) - Jn is formed with each row scaled by a power of two (its largest magnitude
// brought into [0.5, 1), so the scaling is exact and atol-sized entries keep FP32's relative precision), factored
// in FP32 in the plain path's elimination order and blocked schedule, and every stage solve W K = b (W = M0 - w 1^T,
// the constant-pressure rank-one term) is refined in FP64: K <- K + W~^-1 (b - W K), where W~^-1 is the FP32 factors
// with the Sherman-Morrison correction, and the residual is formed in FP64 from the rate tables and the number
// densities already in shared memory, W K = K / (gamma h) - Jn K - w sum(K), with Jn K = S dv(K) (dv the directional
// derivative of each reaction's rate of progress along K). No FP64 matrix is stored: the cell's shared memory is
// 39.5 KB instead of 55.9 KB at 69 species, so 5 cells share an SM instead of 4.
//
// FP64 stays where the method needs it: rate coefficients and NASA-9 equilibrium constants, the right-hand sides,
// the residuals, the stage vectors, the error estimate and step-size control, and the guard's element bookkeeping.
// An accepted try whose last refinement still moved a stage vector by more than `tol` of the error-control scale
// (rtol |N| + atol) is not trusted: its cell is listed and redone from its inputs by the plain FP64 call kernel, which
// mx_call launches on the listed cells right after this kernel.
//
// The stage structure, rates, step control and guard follow imalsky/maxichem maxichem/kernels/call.cuh:34-177 and
// common.cuh (cited in device.cuh); the precision split is this library's own design.
#include <cuda_runtime.h>

#include <cmath>

#include "solver.cuh"

using namespace mx;

// Shared memory the mixed kernel's cells may take on one SM (bytes); the rest of the unified 256 KB stays L1.
constexpr int MIXED_SMEM_BUDGET = 164 * 1024;

namespace {

enum { PH_RATES, PH_RHS_JAC, PH_LU, PH_STAGE12, PH_STAGE3, PH_STAGE4, PH_CONTROL, PH_OUTPUT, PH_COUNT };

// The mixed layout's extra arrays.
struct Extra {
  float *A, *dinv;
  double *S, *Dg, *nN, *w, *R, *B;
};

__device__ __forceinline__ Extra extra_arrays(const Net& net, double* smem) {
  Extra e;
  e.A = (float*)(smem + net.oA);
  e.dinv = (float*)(smem + net.oD);
  e.S = smem + net.oS;
  e.Dg = smem + net.oDg;
  e.nN = smem + net.onN;
  e.w = smem + net.oW;
  e.R = smem + net.oR;
  e.B = smem + net.oB;
  return e;
}

__device__ __forceinline__ double padded(const double* y, int q, int ns) { return q < ns ? y[q] : 0.0; }

// dv_r = sum_q (d v_r / d n_q) y_q at n = nN for each reaction into c.v (c.v[nr] = 0), the product rule over each
// side's (at most three) species: d(n0 n1 n2) = y0 n1 n2 + n0 (y1 n2 + n1 y2); the padding species ns has n = 1, y = 0.
// S dv is then Jn y (jacobian_times_x, common.cuh:395-402, as a product of the rate tables instead of a matrix).
__device__ __forceinline__ void directional_rates(const Net& net, const Cell& c, const double* nN, const double* y,
                                                  int gtid, int gnt) {
  const int ns = net.ns;
  for (int r = gtid; r < net.nr; r += gnt) {
    const uint64_t wd = __ldg(net.rx8 + r);
    const int a0 = wd & 255, a1 = (wd >> 8) & 255, a2 = (wd >> 16) & 255;
    const int b0 = (wd >> 24) & 255, b1 = (wd >> 32) & 255, b2 = (wd >> 40) & 255;
    const double df = fma(padded(y, a0, ns), nN[a1] * nN[a2],
                          nN[a0] * fma(padded(y, a1, ns), nN[a2], nN[a1] * padded(y, a2, ns)));
    const double db = fma(padded(y, b0, ns), nN[b1] * nN[b2],
                          nN[b0] * fma(padded(y, b1, ns), nN[b2], nN[b1] * padded(y, b2, ns)));
    c.v[r] = fma(c.kf[r], df, -(c.kr[r] * db));
  }
  if (gtid == 0) c.v[net.nr] = 0.0;
}

// A (FP32, row stride ld) = -Jn off the diagonal, Dg = -Jn's diagonal (FP64), from the plain path's entry streams.
// Two barriers.
__device__ __forceinline__ void jacobian_mixed(const Net& net, const Cell& c, const Extra& e, int tid, int nt) {
  const int ns = net.ns, ld = net.ld;
  for (int i = tid; i < ns * ld; i += nt) e.A[i] = 0.0f;
  for (int i = tid; i < ns; i += nt) e.Dg[i] = 0.0;
  __syncthreads();
  const uint32_t* __restrict__ jw = net.jt[0] + tid;
  const uint16_t* __restrict__ jd = net.jd[0] + tid;
  const int rounds = net.jac_rounds[0];
  double acc = 0.0;
  int k = 0;
#pragma unroll 4
  for (int q = 0; q < rounds; q++) {
    const unsigned w = __ldg(jw + q * nt);
    const double pr = c.kf[w & 0xfffu] * c.n[(w >> 16) & 255u] * c.n[w >> 24];
    acc = fma(code_coefficient(w >> 12), pr, acc);
    if (w & 0x4000u) {
      const int dst = __ldg(jd + k * nt);
      if (dst % (ld + 1) == 0)  // p == q: the diagonal, kept in FP64 until gamma h is added
        e.Dg[dst / (ld + 1)] = -acc;
      else
        e.A[dst] = (float)(-acc);
      acc = 0.0;
      k++;
    }
  }
  __syncthreads();
}

// Row i of M0 scaled by S_i = 2^-e_i, its largest magnitude (the diagonal igh + Dg_i in FP64, the rest as stored)
// brought into [0.5, 1): exact in FP32 down to its subnormal range. One thread per row; one barrier.
__device__ __forceinline__ void scale_rows(const Net& net, const Extra& e, double igh, int tid, int nt) {
  const int ns = net.ns, ld = net.ld;
  for (int i = tid; i < ns; i += nt) {
    float* ai = e.A + i * ld;
    const double di = igh + e.Dg[i];
    float m = 0.0f;
    for (int j = 0; j < ns; j++) m = fmaxf(m, fabsf(ai[j]));
    const double mm = fmax((double)m, fabs(di));
    int ex = 0;
    if (mm > 0.0 && isfinite(mm)) frexp(mm, &ex);
    ex = min(max(ex, -120), 120);
    const double sc = ldexp(1.0, -ex);
    const float fs = (float)sc;
    for (int j = 0; j < ns; j++) ai[j] *= fs;
    ai[i] = (float)(di * sc);
    e.S[i] = sc;
  }
  __syncthreads();
}

// y <- M0^-1 y on one warp with the FP32 factors: the right side row-scaled (S) and brought by one power of two g to
// a largest magnitude in [0.5, 1), the FP32 sweeps of the plain path, the solution back in FP64 (divided by g).
template <int R>
__device__ __noinline__ void solve32(const Net& net, const Extra& e, double* y, int lane) {
  const int ns = net.ns;
  double b[R];
  double m = 0.0;
#pragma unroll
  for (int p = 0; p < R; p++) {
    const int i = lane + 32 * p;
    b[p] = i < ns ? y[i] * e.S[i] : 0.0;
    m = fmax(m, fabs(b[p]));
  }
  m = warp_max(m);
  int ex = 0;
  if (m > 0.0 && isfinite(m)) frexp(m, &ex);
  ex = min(max(ex, -1000), 1000);
  const double g = ldexp(1.0, -ex), ig = ldexp(1.0, ex);
  float a[1][R], d[R];
#pragma unroll
  for (int p = 0; p < R; p++) {
    const int i = lane + 32 * p;
    a[0][p] = (float)(b[p] * g);
    d[p] = i < ns ? e.dinv[i] : 0.0f;
  }
  lu_sweep<R, 1, float>(net, e.A, a, d, lane);
  __syncwarp();
#pragma unroll
  for (int p = 0; p < R; p++) {
    const int i = lane + 32 * p;
    if (i < ns) y[i] = (double)(a[0][p] * d[p]) * ig;
  }
  __syncwarp();
}

// R <- b - W x in FP64 by the group (gtid of gnt threads, named barrier bar): W x = igh x - Jn x - w sum(x). Three
// barriers.
__device__ __forceinline__ void residual(const Net& net, const Cell& c, const Extra& e, const double* x, const double* b,
                                         double igh, int gtid, int gnt, int bar) {
  directional_rates(net, c, e.nN, x, gtid, gnt);
  if (gtid < 32) {
    const double sx = lane_sum(x, net.ns, gtid);
    if (gtid == 0) c.red[4] = sx;
  }
  group_sync(bar, gnt);
  sv_pieces_of(net, c, c.v, gtid, gnt);
  group_sync(bar, gnt);
  const double sx = c.red[4];
  for (int i = gtid; i < net.ns; i += gnt) {
    const double jx = sv_row(net, c, i);
    e.R[i] = fma(e.w[i], sx, fma(-igh, x[i], b[i]) + jx);
  }
  group_sync(bar, gnt);
}

// F (and u0) at Y: the plain path's rhs, kept out of line here so that the kernel's three evaluations share one copy
// of its code (the mixed kernel's code is larger than the plain kernel's, and instruction fetch, not arithmetic,
// stalled it). Two forms with fixed barriers (a barrier id known only at run time would make the kernel reserve all
// sixteen named barriers and cost it a CTA per SM): the whole CTA (barrier 0), and warps 1 .. W - 1 (barrier 1).
__device__ __noinline__ double rhs_cta(const Net& net, const Cell& c, const double* Y, bool u0, double nd, int tid,
                                       int nt) {
  return rhs(net, c, Y, u0, nd, tid, nt, 0);
}
__device__ __noinline__ void rhs_tail(const Net& net, const Cell& c, const double* Y, double nd, int gtid, int gnt) {
  rhs(net, c, Y, false, nd, gtid, gnt, 1);
}

// The refinement of one stage vector x (right side b): `sweeps` times the FP64 residual (all threads) and its FP32
// correction with the Sherman-Morrison term (warp 0). Returns on warp 0 the last correction's largest size on the
// error-control scale rtol |N| + atol.
template <int R>
__device__ __noinline__ double refine(const Net& net, const Cell& c, const Extra& e, double* x, const double* b,
                                         double igh, double c0, double rtol, double atol, int sweeps, int tid, int nt) {
  const int lane = tid & 31, warp = tid >> 5;
  double worst = 0.0;
  for (int s = 0; s < sweeps; s++) {
    residual(net, c, e, x, b, igh, tid, nt, 0);
    if (warp == 0) {
      solve32<R>(net, e, e.R, lane);
      sherman(net, e.R, c.U, c0, lane);
      double q = 0.0;
      for (int i = lane; i < net.ns; i += 32) {
        const double d = e.R[i];
        x[i] += d;
        q = fmax(q, fabs(d) / fma(rtol, fabs(c.N[i]), atol));
      }
      worst = warp_max(q);
      __syncwarp();
    }
    __syncthreads();
  }
  return worst;
}

// The mixed-precision call kernel: the plain call kernel's screening, rates, steps, output and guard, with each try's
// linear algebra as above. A cell whose refinement does not settle is listed in a.sel (counted in a.sel_count[0])
// for the plain kernel and left otherwise untouched (no output, counts or flag). LIST: step only the cells of
// a.in_list (a.in_count[0] of them, queue a.in_count[1]), as the plain kernel's list mode.
template <int W, int R, bool PROF, bool LIST = false>
__global__ void __launch_bounds__(32 * W, 20 / W)
    mixed_kernel(const Net net, const CallArgs a, int sweeps, double tol, long long* prof) {
  extern __shared__ double smem[];
  const Cell c = cell_arrays(net, smem);
  const Extra e = extra_arrays(net, smem);
  const int tid = (int)threadIdx.x, nt = 32 * W, lane = tid & 31, warp = tid >> 5, ns = net.ns;
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
    if (warp == 0) {  // screening on one warp, as the plain kernel's (common.cuh:246-279)
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
      if (lane == 0) c.ints[0] = st;
    }
    __syncthreads();
    const int st = c.ints[0];
    if (st == 0) cell_rates(net, c, Tc, nd, Jc, tid, nt);
    mark(PH_RATES);
    const double h0 = isfinite(hin) ? hin : dt;
    StepState s = {fmax(fmin(h0, dt), MX_H_MIN), 0.0, 0.0, 0.0, 0.0, false};
    int it = (dt > 0.0 && st == 0) ? 0 : a.max_steps;
    double c0 = 0.0;
    int tries = 0, retries = 0;
    bool escalate = false;
    while (it < a.max_steps && s.t < dt * MX_CALL_END) {
      const double ha = fmin(s.h, dt - s.t), igh = 1.0 / (GAMMA * ha), ih = 1.0 / ha;
      tries++;
      retries += s.prej ? 1 : 0;
      const double ntot = rhs_cta(net, c, c.N, true, nd, tid, nt);  // F, u0 in U, n at N
      for (int i = tid; i <= ns; i += nt) e.nN[i] = c.n[i];
      jacobian_mixed(net, c, e, tid, nt);
      // w = u0 - Jn N / ntot (jacobian_times_x, call.cuh:61-79), in FP64 from the rate tables
      directional_rates(net, c, e.nN, c.N, tid, nt);
      __syncthreads();
      sv_pieces_of(net, c, c.v, tid, nt);
      __syncthreads();
      for (int i = tid; i < ns; i += nt) {
        const double wi = c.U[i] - sv_row(net, c, i) / ntot;
        e.w[i] = wi;
        c.U[i] = wi;
      }
      scale_rows(net, e, igh, tid, nt);  // ends with a barrier
      mark(PH_RHS_JAC);
      lu_factor<32 * W, float>(net, e.A, e.dinv, tid);
      mark(PH_LU);
      double worst = 0.0;
      if (warp == 0) {  // stage 1: K1 on warp 0, M0^-1 w on warp 1, then Sherman-Morrison
        for (int i = lane; i < ns; i += 32) c.K1[i] = c.F[i];
        __syncwarp();
        solve32<R>(net, e, c.K1, lane);
      } else if (warp == 1) {
        solve32<R>(net, e, c.U, lane);
      }
      __syncthreads();
      if (warp == 0) {
        c0 = 1.0 / (1.0 - lane_sum(c.U, ns, lane));
        sherman(net, c.K1, c.U, c0, lane);
        if (lane == 0) c.red[2] = c0;
      }
      __syncthreads();
      c0 = c.red[2];
      worst = fmax(worst, refine<R>(net, c, e, c.K1, c.F, igh, c0, a.rtol, a.atol, sweeps, tid, nt));
      for (int i = tid; i < ns; i += nt) {
        const double b2 = fma(RODAS_C21 * ih, c.K1[i], c.F[i]);
        e.B[i] = b2;
        c.K2[i] = b2;
        c.Y[i] = c.N[i] + 2.0 * c.K1[i];
      }
      __syncthreads();
      if (warp == 0) {  // stage 2 on warp 0 while the other warps evaluate F(Y3), Y3 = N + 2 K1
        solve32<R>(net, e, c.K2, lane);
        sherman(net, c.K2, c.U, c0, lane);
      } else {
        rhs_tail(net, c, c.Y, nd, tid - 32, nt - 32);
      }
      __syncthreads();
      worst = fmax(worst, refine<R>(net, c, e, c.K2, e.B, igh, c0, a.rtol, a.atol, sweeps, tid, nt));
      mark(PH_STAGE12);
      if (warp == 0) {  // stage 3
        for (int i = lane; i < ns; i += 32) {
          const double b3 = fma(ih, c.K1[i] - c.K2[i], c.F[i]);
          e.B[i] = b3;
          c.K3[i] = b3;
        }
        __syncwarp();
        solve32<R>(net, e, c.K3, lane);
        sherman(net, c.K3, c.U, c0, lane);
      }
      __syncthreads();
      worst = fmax(worst, refine<R>(net, c, e, c.K3, e.B, igh, c0, a.rtol, a.atol, sweeps, tid, nt));
      for (int i = tid; i < ns; i += nt) c.Y[i] = c.N[i] + 2.0 * c.K1[i] + c.K3[i];
      __syncthreads();
      rhs_cta(net, c, c.Y, false, nd, tid, nt);
      mark(PH_STAGE3);
      if (warp == 0) {  // stage 4
        for (int i = lane; i < ns; i += 32) {
          const double b4 = fma(ih, fma(-RODAS_C43, c.K3[i], c.K1[i] - c.K2[i]), c.F[i]);
          e.B[i] = b4;
          c.K4[i] = b4;
        }
        __syncwarp();
        solve32<R>(net, e, c.K4, lane);
        sherman(net, c.K4, c.U, c0, lane);
      }
      __syncthreads();
      worst = fmax(worst, refine<R>(net, c, e, c.K4, e.B, igh, c0, a.rtol, a.atol, sweeps, tid, nt));
      if (warp == 0) {
        try_error(net, c, s.t == 0.0, a.rtol, a.atol, lane);
        // an accepted try must be trusted; a rejected one only sets the next try's size
        if (lane == 0) c.red[6] = (sweeps > 0 && c.red[1] != 0.0 && !(worst <= tol)) ? 1.0 : 0.0;
      }
      __syncthreads();
      mark(PH_STAGE4);
      if (c.red[6] != 0.0) {  // the refinement did not settle: the plain kernel redoes the cell
        escalate = true;
        break;
      }
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
    if (escalate) {
      if (tid == 0) {
        a.sel[atomicAdd(a.sel_count, 1)] = cell;
        if (a.tries) {
          atomicAdd(a.tries, (unsigned long long)tries);
          atomicAdd(a.tries + 1, (unsigned long long)retries);
        }
        c.ints[1] = (int)(gridDim.x + atomicAdd(LIST ? a.in_count + 1 : a.count + MX_COUNT_QUEUE, 1));
      }
      __syncthreads();
      q = c.ints[1];
      __syncthreads();
      continue;
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
      const int done = (st == 0 && s.t >= dt * MX_CALL_END) ? 1 : 0;
      const int g = st == 0 ? check_cell(net, xin, c.Y, done, s.nok, a.atol, lane, at, c.G) : 0;
      if (lane == 0) {
        a.status[cell] = st;
        if (!isfinite(hin)) atomicAdd(a.count + MX_COUNT_NONFINITE_H, 1);
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

// One fresh try of one cell through the mixed path (a test hook): out = K1, K2, K3, K4, Y [ns each, elimination
// order], err, ok, the refinement's largest last correction on the error-control scale, and the FP32 solve's
// largest first correction (the correction of the first sweep) on that scale.
template <int W, int R>
__global__ void __launch_bounds__(32 * W) mixed_debug_kernel(const Net net, const double* x0, double Tc, double P,
                                                             double ha, const double* Jc, double rtol, double atol,
                                                             int sweeps, double* out) {
  extern __shared__ double smem[];
  const Cell c = cell_arrays(net, smem);
  const Extra e = extra_arrays(net, smem);
  const int tid = (int)threadIdx.x, nt = 32 * W, lane = tid & 31, warp = tid >> 5, ns = net.ns;
  const double nd = P / (MX_KB * Tc), igh = 1.0 / (GAMMA * ha), ih = 1.0 / ha;
  for (int i = tid; i < ns; i += nt) c.N[i] = x0[__ldg(net.perm + i)];
  __syncthreads();
  cell_rates(net, c, Tc, nd, Jc, tid, nt);
  const double ntot = rhs(net, c, c.N, true, nd, tid, nt);
  for (int i = tid; i <= ns; i += nt) e.nN[i] = c.n[i];
  jacobian_mixed(net, c, e, tid, nt);
  directional_rates(net, c, e.nN, c.N, tid, nt);
  __syncthreads();
  sv_pieces_of(net, c, c.v, tid, nt);
  __syncthreads();
  for (int i = tid; i < ns; i += nt) {
    const double wi = c.U[i] - sv_row(net, c, i) / ntot;
    e.w[i] = wi;
    c.U[i] = wi;
  }
  scale_rows(net, e, igh, tid, nt);
  lu_factor<32 * W, float>(net, e.A, e.dinv, tid);
  if (warp == 0) {
    for (int i = lane; i < ns; i += 32) c.K1[i] = c.F[i];
    __syncwarp();
    solve32<R>(net, e, c.K1, lane);
  } else if (warp == 1) {
    solve32<R>(net, e, c.U, lane);
  }
  __syncthreads();
  double c0 = 0.0;
  if (warp == 0) {
    c0 = 1.0 / (1.0 - lane_sum(c.U, ns, lane));
    sherman(net, c.K1, c.U, c0, lane);
    if (lane == 0) c.red[2] = c0;
  }
  __syncthreads();
  c0 = c.red[2];
  const double first = refine<R>(net, c, e, c.K1, c.F, igh, c0, rtol, atol, sweeps > 0 ? 1 : 0, tid, nt);
  double worst = sweeps > 1 ? refine<R>(net, c, e, c.K1, c.F, igh, c0, rtol, atol, sweeps - 1, tid, nt) : first;
  for (int i = tid; i < ns; i += nt) {
    const double b2 = fma(RODAS_C21 * ih, c.K1[i], c.F[i]);
    e.B[i] = b2;
    c.K2[i] = b2;
    c.Y[i] = c.N[i] + 2.0 * c.K1[i];
  }
  __syncthreads();
  if (warp == 0) {
    solve32<R>(net, e, c.K2, lane);
    sherman(net, c.K2, c.U, c0, lane);
  }
  __syncthreads();
  worst = fmax(worst, refine<R>(net, c, e, c.K2, e.B, igh, c0, rtol, atol, sweeps, tid, nt));
  rhs(net, c, c.Y, false, nd, tid, nt);
  if (warp == 0) {
    for (int i = lane; i < ns; i += 32) {
      const double b3 = fma(ih, c.K1[i] - c.K2[i], c.F[i]);
      e.B[i] = b3;
      c.K3[i] = b3;
    }
    __syncwarp();
    solve32<R>(net, e, c.K3, lane);
    sherman(net, c.K3, c.U, c0, lane);
  }
  __syncthreads();
  worst = fmax(worst, refine<R>(net, c, e, c.K3, e.B, igh, c0, rtol, atol, sweeps, tid, nt));
  for (int i = tid; i < ns; i += nt) c.Y[i] = c.N[i] + 2.0 * c.K1[i] + c.K3[i];
  __syncthreads();
  rhs(net, c, c.Y, false, nd, tid, nt);
  if (warp == 0) {
    for (int i = lane; i < ns; i += 32) {
      const double b4 = fma(ih, fma(-RODAS_C43, c.K3[i], c.K1[i] - c.K2[i]), c.F[i]);
      e.B[i] = b4;
      c.K4[i] = b4;
    }
    __syncwarp();
    solve32<R>(net, e, c.K4, lane);
    sherman(net, c.K4, c.U, c0, lane);
  }
  __syncthreads();
  worst = fmax(worst, refine<R>(net, c, e, c.K4, e.B, igh, c0, rtol, atol, sweeps, tid, nt));
  if (warp == 0) try_error(net, c, true, rtol, atol, lane);
  __syncthreads();
  for (int i = tid; i < ns; i += nt) {
    out[i] = c.K1[i];
    out[ns + i] = c.K2[i];
    out[2 * ns + i] = c.K3[i];
    out[3 * ns + i] = c.K4[i];
    out[4 * ns + i] = c.Y[i];
  }
  if (tid == 0) {
    out[5 * ns] = c.red[0];
    out[5 * ns + 1] = c.red[1];
    out[5 * ns + 2] = worst;
    out[5 * ns + 3] = first;
  }
}

template <int W, int R>
void mixed_kernels_for(mx_solver* s) {
  s->mixed = mixed_kernel<W, R, false>;
  s->mixed_prof = mixed_kernel<W, R, true>;
  s->mixed_list = mixed_kernel<W, R, false, true>;
  s->mixed_debug = mixed_debug_kernel<W, R>;
}

template <int W>
bool mixed_kernels_of(mx_solver* s) {
  switch (s->rows_per_lane) {
    case 1: mixed_kernels_for<W, 1>(s); return true;
    case 2: mixed_kernels_for<W, 2>(s); return true;
    case 3: mixed_kernels_for<W, 3>(s); return true;
    case 4: mixed_kernels_for<W, 4>(s); return true;
    case 8: mixed_kernels_for<W, 8>(s); return true;
    default: return false;
  }
}

}  // namespace

int mx_mixed_prepare(mx_solver* s, int n_pieces, char* err, size_t errlen) {
  const int ns = s->net.ns, nr = s->net.nr, nel = s->net.nel;
  if (!(s->warps == 4 ? mixed_kernels_of<4>(s) : mixed_kernels_of<2>(s))) {
    set_error(err, errlen, "mx_create: no mixed-precision kernel for %d rows per lane", s->rows_per_lane);
    return MX_ERR_NETWORK;
  }
  Net& m = s->net32;
  m = s->net;  // the tables; the layout below replaces the plain one's offsets
  int off = 0;
  auto take = [&](int doubles) {
    const int o = off;
    off += (doubles + 1) & ~1;
    return o;
  };
  m.oA = take((ns * m.ld + 1) / 2);  // FP32 matrix
  m.a_doubles = ns * m.ld / 2;
  m.oK = take(2 * nr + 2);
  m.oV = take(std::max(nr + 1, ns + 1));
  m.on = take(ns + 1);
  m.onN = take(ns + 1);
  m.oN = take(ns);
  m.oY = take(ns);
  m.oF = take(ns);
  m.oU = take(ns);
  m.oK1 = take(ns);
  m.oK2 = take(ns);
  m.oK3 = take(ns);
  m.oK4 = take(ns);
  m.oD = take((ns + 1) / 2);  // FP32 reciprocal pivots
  m.oS = take(ns);
  m.oW = take(ns);
  m.oR = take(ns);
  m.oDg = m.oR;  // the Jacobian's diagonal is dead once the rows are scaled, before any residual
  m.oB = take(ns);
  m.oRed = take(8);
  m.oInts = take((ns + 8) / 2 + 1);
  m.oPart = take(n_pieces);
  {
    const int staged = (ns * nel + ns + 1) & ~1;
    if (staged + guard_scratch(ns) <= m.a_doubles)
      m.oG = m.oA + staged;
    else
      m.oG = take(guard_scratch(ns));
  }
  m.doubles = off;
  s->mixed_smem = (size_t)off * sizeof(double);
  cudaError_t e = cudaFuncSetAttribute((const void*)s->mixed, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)s->mixed_smem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute((const void*)s->mixed_prof, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)s->mixed_smem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute((const void*)s->mixed_debug, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)s->mixed_smem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute((const void*)s->mixed_list, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)s->mixed_smem);
  // Shared memory for at most the cells that fit 164 KB, the rest of the SM's 256 KB left to L1 for the rate tables and
  // term streams every try reads (measured at 69 species: 4 cells a SM with 92 KB of L1 ran the call 6 % faster than
  // 5 cells with 28 KB); the carveout is a percentage of the SM's shared-memory maximum.
  int per_sm_max = 0, reserved = 0;
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&per_sm_max, cudaDevAttrMaxSharedMemoryPerMultiprocessor, s->device);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, s->device);
  int cells = 1;
  if (e == cudaSuccess) {
    const size_t per_cell = s->mixed_smem + (size_t)reserved;
    cells = std::max(1, (int)((size_t)MIXED_SMEM_BUDGET / per_cell));
    const int percent = std::min(100, (int)((100 * (size_t)cells * per_cell + per_sm_max - 1) / per_sm_max));
    for (const void* f : {(const void*)s->mixed, (const void*)s->mixed_prof, (const void*)s->mixed_debug,
                          (const void*)s->mixed_list})
      if (e == cudaSuccess) e = cudaFuncSetAttribute(f, cudaFuncAttributePreferredSharedMemoryCarveout, percent);
  }
  if (e == cudaSuccess)
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&s->mixed_ctas, (const void*)s->mixed, 32 * s->warps,
                                                      s->mixed_smem);
  if (e == cudaSuccess) s->mixed_ctas = std::min(s->mixed_ctas, cells);
  if (e == cudaSuccess && s->mixed_ctas < 1) e = cudaErrorInvalidConfiguration;
  if (e != cudaSuccess) {
    set_error(err, errlen, "mx_create: the mixed-precision kernel: %s", cudaGetErrorString(e));
    return MX_ERR_CUDA;
  }
  return MX_OK;
}

cudaError_t mx_mixed_launch(mx_solver* s, const CallArgs& a, int64_t B, bool list, cudaStream_t st) {
  const int per_sm = s->grid_ctas < 0 ? s->mixed_ctas : std::min(s->grid_ctas, s->mixed_ctas);
  const int grid = s->grid_ctas == 0 ? (int)B : (int)std::min<int64_t>(B, (int64_t)per_sm * s->sms);
  if (list)
    s->mixed_list<<<grid, 32 * s->warps, s->mixed_smem, st>>>(s->net32, a, s->sweeps, s->mixed_tol, nullptr);
  else if (s->phases)
    s->mixed_prof<<<grid, 32 * s->warps, s->mixed_smem, st>>>(s->net32, a, s->sweeps, s->mixed_tol, s->phases);
  else
    s->mixed<<<grid, 32 * s->warps, s->mixed_smem, st>>>(s->net32, a, s->sweeps, s->mixed_tol, nullptr);
  return cudaGetLastError();
}

extern "C" int mx_debug_try_mixed(mx_solver* s, const double* x, double T, double P, double h, const double* J,
                                  double rtol, double atol, int32_t sweeps, double* out, void* stream) {
  if (!s || !x || !out || (s->net.nj > 0 && !J) || sweeps < 0 || sweeps > MX_MIXED_MAX_SWEEPS) return MX_ERR_ARGUMENT;
  DeviceScope scope(s->device);
  if (scope.status != cudaSuccess) return MX_ERR_CUDA;
  s->mixed_debug<<<1, 32 * s->warps, s->mixed_smem, (cudaStream_t)stream>>>(s->net32, x, T, P, h, J, rtol, atol, sweeps,
                                                                         out);
  return cudaGetLastError() == cudaSuccess ? MX_OK : MX_ERR_CUDA;
}
