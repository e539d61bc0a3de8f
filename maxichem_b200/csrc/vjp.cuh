// The adjoint of one call (the reference's ADSolver.vjp, maxichem/kincuda_ad.py:455-556; its kernels
// maxichem/kernels/vjp.cuh, ad_common.cuh), on the B200.
//
// Each cell runs the call forward once (the call kernel's device functions in the same order, so the primal is the
// call's bit for bit), storing the state before each try; beyond CAP tries it keeps a checkpoint every
// ceil(n / CAP) tries and recomputes each segment (docs/method.md:219-224 of the reference). The reverse pass
// recomputes each try from its stored state and takes its adjoint: the step control's partials, err's adjoint, the
// stage cotangents through transposed solves on the try's own factors, W^-T y = M0^-T (y + c0 (u_hat . y) 1) (the
// recovery's dense pivoted W^-T for recovered cells), F's adjoint at Y4, Y3 and N, and the derivative of W itself:
// sum_k b_k^T J_N K_k, whose Jacobian part comes reaction by reaction from second products of the concentrations.
// Species sums gather each species' reaction slots from a table in a fixed order: no atomics enter the arithmetic,
// so the same inputs give the same bits. The rate cotangents reduce to T, P, the log multipliers and J per cell, and
// to the rate table's Arrhenius columns: the forward kernel takes cells in fixed chunks of ADJ_CHUNK consecutive
// cells from its queue and adds each passing cell's contribution to its chunk's partial sum in cell order; a cell the
// recovery redoes leaves its contribution in a slot of its own; a last kernel adds the chunks and those slots in a
// fixed order.
#pragma once
#include "jvp.cuh"

namespace mx {

// The adjoint's inputs and outputs of one mx_vjp call (device pointers; lm, gh may be null).
struct AdjArgs {
  const double *lm, *gx, *gh;
  int adapt, cap;  // cap: stored try states per cell (2 cap of checkpoints and of segment states)
  double *gx0, *gT, *gP, *gdt, *gh0, *glm, *gJ;
  double* gLc;        // [nr][nchunks][9]: per chunk the rate-table cotangent of its cells that passed the guard
  int nchunks;
  int* chunk_listed;  // [nchunks]: 1 when a cell of the chunk went to the recovery
  int* chunk_queue;   // the forward kernel's chunk queue
  double* gLq;        // [listed][nr][3]: a recovered cell's cotangents of ln k0's terms and ln k_inf, by list slot
  int* pos;           // [B]: a listed cell's slot in the recovery's list
  double* scratch;
  long long slot;
  const int *sp_ptr, *sp_ent;  // species gather: species j's reaction slots sp_ent[sp_ptr[j] .. sp_ptr[j + 1]) = r*8 + m
  const uint64_t* st8;         // S's columns: species bytes 0-5 (padding ns), coefficient codes 2 bits each from bit 48
};

// Shared-memory offsets of the adjoint's vectors past the call's layout.
struct AdjLayout {
  int oNb, oYb, oFb, oUb, oNn, oNx, oKb, oBb, oRed, doubles, stride;
};

struct AdjCell {
  double *Nb, *Yb, *Fb, *Ub, *Nn, *Nx, *red;
  double* Kb[4];
  double* Bb[4];
};

__device__ __forceinline__ AdjCell adj_arrays(const AdjLayout& l, double* smem) {
  AdjCell a;
  a.Nb = smem + l.oNb;
  a.Yb = smem + l.oYb;
  a.Fb = smem + l.oFb;
  a.Ub = smem + l.oUb;
  a.Nn = smem + l.oNn;
  a.Nx = smem + l.oNx;
  a.red = smem + l.oRed;
#pragma unroll
  for (int k = 0; k < 4; k++) {
    a.Kb[k] = smem + l.oKb + k * l.stride;
    a.Bb[k] = smem + l.oBb + k * l.stride;
  }
  return a;
}

// per-CTA scratch: k_bar [2 nr], slot contributions c1 [nr][6], c2 [nr][6], try states [2][cap][ns + 8], the cell's
// cotangents of ln k0's terms and ln k_inf [nr][3]
constexpr int REC_EXTRA = 8;  // h, t, pen, pha, prej, nok and two spare
constexpr int ADJ_CHUNK = 64;  // cells per chunk of the rate table's partial sums
__device__ __forceinline__ double* adj_kbar(const Net& net, double* sl) { return sl; }
__device__ __forceinline__ double* adj_c1(const Net& net, double* sl) { return sl + 2 * net.nr; }
__device__ __forceinline__ double* adj_c2(const Net& net, double* sl) { return sl + 8 * net.nr; }
__device__ __forceinline__ double* adj_state(const Net& net, const AdjArgs& aa, double* sl, int bank, int i) {
  return sl + 14 * net.nr + ((size_t)bank * aa.cap + i) * (net.ns + REC_EXTRA);
}
__device__ __forceinline__ double* adj_gl(const Net& net, const AdjArgs& aa, double* sl) {
  return sl + 14 * net.nr + (size_t)2 * aa.cap * (net.ns + REC_EXTRA);
}

// a block-wide sum in a fixed order: every thread's value, then thread 0 adds them in thread order; every thread
// returns it. Two barriers.
__device__ __forceinline__ double block_sum(double v, double* red, int tid, int nt) {
  red[tid] = v;
  __syncthreads();
  if (tid < 32) {
    double s = 0.0;
    for (int q = tid; q < nt; q += 32) s += red[q];
    s = warp_sum(s);
    if (tid == 0) red[nt] = s;
  }
  __syncthreads();
  const double r = red[nt];
  __syncthreads();
  return r;
}

// ---- the primal try and its storage ----

__device__ __forceinline__ void store_state(const Net& net, const Cell& c, double* rec, const StepState& s, int tid,
                                            int nt) {
  const int ns = net.ns;
  for (int i = tid; i < ns; i += nt) rec[i] = c.N[i];
  if (tid == 0) {
    rec[ns] = s.h;
    rec[ns + 1] = s.t;
    rec[ns + 2] = s.pen;
    rec[ns + 3] = s.pha;
    rec[ns + 4] = s.prej ? 1.0 : 0.0;
    rec[ns + 5] = s.nok;
  }
}

__device__ __forceinline__ StepState load_state(const Net& net, const Cell& c, const double* rec, int tid, int nt) {
  const int ns = net.ns;
  for (int i = tid; i < ns; i += nt) c.N[i] = rec[i];
  StepState s;
  s.h = rec[ns];
  s.t = rec[ns + 1];
  s.pen = rec[ns + 2];
  s.pha = rec[ns + 3];
  s.prej = rec[ns + 4] != 0.0;
  s.nok = rec[ns + 5];
  __syncthreads();
  return s;
}

// One try of the call (call_kernel's, or recover_kernel's dense one), through the error: K1-K4, Y = N', the factors,
// en and ok in c.red[0..1]. c0 is warp 0's.
template <int W, int R, bool DENSE>
__device__ __noinline__ void primal_try(const Net& net, const Cell& c, const StepState& s, double dt, double nd, double rtol,
                           double atol, const int* pr, double& c0, int tid) {
  constexpr int nt = 32 * W;
  const int ns = net.ns, ld = net.ld, lane = tid & 31, warp = tid >> 5;
  const double ha = fmin(s.h, dt - s.t), igh = 1.0 / (GAMMA * ha), ih = 1.0 / ha;
  const double ntot = rhs(net, c, c.N, true, nd, tid, nt);
  jacobian_w(net, c, ntot, tid, nt);
  if (DENSE) {
    for (int e = tid; e < ns * ns; e += nt) {
      const int i = e / ns, j = e - i * ns;
      double* p = c.A + i * ld + j;
      *p = (i == j ? *p + igh : *p) - c.U[i];
    }
    __syncthreads();
    if (warp == 0) {
      for (int i = lane; i < ns; i += 32) c.K1[i] = c.F[i];
      __syncwarp();
      dense_lu_pivot(net, c.A, c.dinv, (int*)pr, lane);
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
      for (int i = lane; i < ns; i += 32) c.K4[i] = fma(ih, fma(-RODAS_C43, c.K3[i], c.K1[i] - c.K2[i]), c.F[i]);
      __syncwarp();
      dense_solve<R>(net, c.A, c.dinv, pr, c.K4, lane);
      try_error(net, c, s.t == 0.0, rtol, atol, lane);
    }
    __syncthreads();
    return;
  }
  for (int i = tid; i < ns; i += nt) c.A[i * ld + i] += igh;
  __syncthreads();
  lu_factor<nt>(net, c.A, c.dinv, tid);
  if (warp == 0) {
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
  if (warp == 0) {
    lu_solve<R, 1>(net, c.A, c.dinv, c.K2, nullptr, lane);
    sherman(net, c.K2, c.U, c0, lane);
  } else {
    rhs(net, c, c.Y, false, nd, tid - 32, nt - 32, 1);
  }
  __syncthreads();
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
    try_error(net, c, s.t == 0.0, rtol, atol, lane);
  }
  __syncthreads();
}

// the step update after a try (the call kernel's)
__device__ __forceinline__ void primal_update(const Net& net, const Cell& c, StepState& s, double dt, int tid,
                                              int nt) {
  const double ha = fmin(s.h, dt - s.t), en = c.red[0];
  const bool ok = c.red[1] != 0.0;
  if (ok) {
    for (int i = tid; i < net.ns; i += nt) c.N[i] = fmax(c.Y[i], 0.0);
    s.t += ha;
    s.nok += 1.0;
  }
  const double fac = step_factor(en, ok, s.prej, s.pen, s.pha, ha);
  s.h = ha * fac;
  s.prej = !ok;
  s.pen = en;
  s.pha = ha;
  __syncthreads();
}

// ---- transposed solves (one warp) ----

// y <- M0^-T y with the factors of lu_factor (unit L below the diagonal, U on and above it), on one warp: U^T z = y in
// ascending pivots (z_k = a_k / U_kk, then a_i -= U_ki z_k for i > k), then L^T x = z in descending pivots
// (a_i -= L_ki x_k for i < k). Lane l holds rows l + 32 p; row k of the factors is read across the lanes
// (consecutive addresses). As lu_solve: pivots 32 at a time, the pivot's value from a register chosen at compile
// time and one shuffle, and the next row loaded while the current pivot is applied; a lane whose row takes no update
// from pivot k uses the multiplier 0 (fma(-0, z, a) = a for finite z). Each entry takes the one-pivot sweep's fma's in
// its order.
template <int R>
__device__ __noinline__ void lu_solve_t(const Net& net, const double* A, const double* dinv, double* y, int lane) {
  const int ns = net.ns, ld = net.ld, last = ns - 1;
  double a[R], d[R];
#pragma unroll
  for (int p = 0; p < R; p++) {
    const int i = lane + 32 * p;
    a[p] = i < ns ? y[i] : 0.0;
    d[p] = i < ns ? dinv[i] : 0.0;
  }
#pragma unroll
  for (int c = 0; c < R; c++) {  // U^T: pivots 32c .. 32c + 31
    const int k0 = 32 * c, k1 = min(k0 + 32, ns);
    if (k0 >= k1) break;
    double m[R];
#pragma unroll
    for (int p = c; p < R; p++) m[p] = A[k0 * ld + min(lane + 32 * p, last)];
#pragma unroll 2
    for (int k = k0; k < k1; k++) {
      const double zk = __shfl_sync(FULL, a[c] * d[c], k & 31);
      if (lane == (k & 31)) a[c] = zk;
      double mn[R];
#pragma unroll
      for (int p = c; p < R; p++) mn[p] = A[min(k + 1, last) * ld + min(lane + 32 * p, last)];
#pragma unroll
      for (int p = c; p < R; p++) {
        const bool act = (p > c ? true : lane > k - k0) && lane + 32 * p < ns;
        a[p] = fma(-(act ? m[p] : 0.0), zk, a[p]);
        m[p] = mn[p];
      }
    }
  }
#pragma unroll
  for (int c = R - 1; c >= 0; c--) {  // L^T: pivots 32c + 31 .. 32c (down to 1)
    const int k0 = 32 * c, khi = min(k0 + 31, last), klo = max(k0, 1);
    if (khi < klo) continue;
    double m[R];
#pragma unroll
    for (int p = 0; p <= c; p++) m[p] = A[khi * ld + min(lane + 32 * p, last)];
#pragma unroll 2
    for (int k = khi; k >= klo; k--) {
      const double xk = __shfl_sync(FULL, a[c], k & 31);
      double mn[R];
#pragma unroll
      for (int p = 0; p <= c; p++) mn[p] = A[max(k - 1, 0) * ld + min(lane + 32 * p, last)];
#pragma unroll
      for (int p = 0; p <= c; p++) {
        const bool act = p < c ? true : lane < k - k0;
        a[p] = fma(-(act ? m[p] : 0.0), xk, a[p]);
        m[p] = mn[p];
      }
    }
  }
  __syncwarp();
#pragma unroll
  for (int p = 0; p < R; p++) {
    const int i = lane + 32 * p;
    if (i < ns) y[i] = a[p];
  }
  __syncwarp();
}

// y <- W^-T y on warp 0: the call's W = M0 - u 1^T, W^-T y = M0^-T (y + c0 (u_hat . y) 1), u_hat = M0^-1 u (in U after
// the try); or the recovery's dense pivoted W = P^T L U, W^-T y = P^T L^-T U^-T y.
template <int R, bool DENSE>
__device__ __forceinline__ void stage_solve_t(const Net& net, const Cell& c, double* y, double c0, const int* pr,
                                              double* tmp, int lane) {
  const int ns = net.ns;
  if (DENSE) {
    lu_solve_t<R>(net, c.A, c.dinv, y, lane);
    for (int i = lane; i < ns; i += 32) tmp[i] = y[i];
    __syncwarp();
    for (int i = lane; i < ns; i += 32) y[pr[i]] = tmp[i];
    __syncwarp();
  } else {
    double p = 0.0;
    for (int i = lane; i < ns; i += 32) p = fma(c.U[i], y[i], p);
    const double s = c0 * warp_sum(p);
    for (int i = lane; i < ns; i += 32) y[i] += s;
    __syncwarp();
    lu_solve_t<R>(net, c.A, c.dinv, y, lane);
  }
}

// ---- adjoints of F and of the Jacobian terms ----

// the concentrations of a reaction's six slots (c.n) and its slot indices
struct Slots {
  double a[6];
  int s[6];
};

__device__ __forceinline__ Slots slots_of(const Net& net, const Cell& c, int r) {
  const uint64_t w = __ldg(net.rx8 + r);
  Slots q;
#pragma unroll
  for (int m = 0; m < 6; m++) {
    q.s[m] = (int)((w >> (8 * m)) & 255);
    q.a[m] = c.n[q.s[m]];
  }
  return q;
}

// (S^T y)_r from S's column r (a photolysis branch's products are in S, not in the reaction's slots)
__device__ __forceinline__ double st_entry(const AdjArgs& aa, int r, const double* y, int ns) {
  const uint64_t w = __ldg(aa.st8 + r);
  double z = 0.0;
#pragma unroll
  for (int m = 0; m < 6; m++) {
    const int s = (int)((w >> (8 * m)) & 255);
    if (s < ns) z = fma(code_coefficient((unsigned)(w >> (48 + 2 * m)) & 3u), y[s], z);
  }
  return z;
}

// prod_{l != m} a_l of one side (slots b .. b + 2)
__device__ __forceinline__ double others(const Slots& q, int m) {
  const int b = m < 3 ? 0 : 3, i = m - b;
  return (i == 0 ? 1.0 : q.a[b]) * (i == 1 ? 1.0 : q.a[b + 1]) * (i == 2 ? 1.0 : q.a[b + 2]);
}

// species gather: out_j = sum of c[r][m] over species j's slots, in table order
__device__ __forceinline__ void gather(const Net& net, const AdjArgs& aa, const double* cr, double* out, int tid,
                                       int nt) {
  for (int j = tid; j < net.ns; j += nt) {
    double s = 0.0;
    const int e1 = __ldg(aa.sp_ptr + j + 1);
    for (int e = __ldg(aa.sp_ptr + j); e < e1; e++) {
      const int w = __ldg(aa.sp_ent + e);
      s += cr[(w >> 3) * 6 + (w & 7)];
    }
    out[j] = s;
  }
}

// n = nd Y / ntot at the state Y = N + a K1 + b K3 (which 0, 1, 2); returns ntot. One barrier.
__device__ __forceinline__ double state_n(const Net& net, const Cell& c, int which, double nd, int tid, int nt) {
  const int ns = net.ns, lane = tid & 31;
  double p = 0.0;
  for (int i = lane; i < ns; i += 32)
    p += which == 0 ? c.N[i] : (which == 1 ? c.N[i] + 2.0 * c.K1[i] : c.N[i] + 2.0 * c.K1[i] + c.K3[i]);
  const double ntot = warp_sum(p), xf = nd / ntot;
  for (int i = tid; i < ns; i += nt) {
    const double y = which == 0 ? c.N[i] : (which == 1 ? c.N[i] + 2.0 * c.K1[i] : c.N[i] + 2.0 * c.K1[i] + c.K3[i]);
    c.n[i] = y * xf;
  }
  if (tid == 0) c.n[ns] = 1.0;
  __syncthreads();
  return ntot;
}

// F's adjoint at the state Y (which 1: Y3, 2: Y4) for the cotangent fb: adds to Yb (N's, K1's and K3's shares
// follow from Y's form), to k_bar and to ndb (thread 0's).
__device__ __noinline__ void f_adjoint(const Net& net, const Cell& c, const AdjCell& b, const AdjArgs& aa, double* sl, int which,
                          const double* fb, double nd, double& ndb, int tid, int nt) {
  const int ns = net.ns, nr = net.nr;
  const double ntot = state_n(net, c, which, nd, tid, nt), xf = nd / ntot, ixf = ntot / nd;
  double* kb = adj_kbar(net, sl);
  double* cr = adj_c1(net, sl);
  double sv = 0.0;
  for (int r = tid; r < nr; r += nt) {
    const Slots q = slots_of(net, c, r);
    const double kf = c.kf[r], kr = c.kr[r];
    const double pf = q.a[0] * q.a[1] * q.a[2], pb = q.a[3] * q.a[4] * q.a[5];
    const double z = st_entry(aa, r, fb, ns), ab = ixf * z;
    sv = fma(z, kf * pf - kr * pb, sv);
#pragma unroll
    for (int m = 0; m < 6; m++) cr[r * 6 + m] = m < 3 ? ab * kf * others(q, m) : -ab * kr * others(q, m);
    kb[r] = fma(ab, pf, kb[r]);
    kb[nr + r] = fma(-ab, pb, kb[nr + r]);
  }
  const double ixfb = block_sum(sv, b.red, tid, nt);  // F . fb / ixf = s . fb
  gather(net, aa, cr, b.Nn, tid, nt);
  __syncthreads();
  double px = 0.0;
  for (int i = tid; i < ns; i += nt) {
    const double y = which == 1 ? c.N[i] + 2.0 * c.K1[i] : c.N[i] + 2.0 * c.K1[i] + c.K3[i];
    px = fma(b.Nn[i], y, px);
  }
  const double xfb = block_sum(px, b.red, tid, nt);
  const double ntb = ixfb / nd - xfb * nd / (ntot * ntot);
  if (tid == 0) ndb += -ixfb * ntot / (nd * nd) + xfb / ntot;
  for (int i = tid; i < ns; i += nt) {
    const double yb = fma(b.Nn[i], xf, ntb);
    b.Nb[i] += yb;
    b.Kb[0][i] = fma(2.0, yb, b.Kb[0][i]);
    if (which == 2) b.Kb[2][i] += yb;
  }
  __syncthreads();
}

// The adjoint at N of F (cotangent Fb), of u = S v / nd - (Jn N) / ntot (cotangent Ub) and of sum_k Bb_k^T Jn K_k:
// adds to Nb, k_bar and ndb.
__device__ void n_adjoint(const Net& net, const Cell& c, const AdjCell& b, const AdjArgs& aa, double* sl, double nd,
                          double& ndb, int tid, int nt) {
  const int ns = net.ns, nr = net.nr;
  const double ntot = state_n(net, c, 0, nd, tid, nt), xf = nd / ntot, ixf = ntot / nd;
  double* kb = adj_kbar(net, sl);
  double* c1 = adj_c1(net, sl);
  double* c2 = adj_c2(net, sl);
  double sF = 0.0, sU = 0.0, sW = 0.0;
  for (int r = tid; r < nr; r += nt) {
    const Slots q = slots_of(net, c, r);
    const double kf = c.kf[r], kr = c.kr[r];
    const double pf = q.a[0] * q.a[1] * q.a[2], pb = q.a[3] * q.a[4] * q.a[5];
    const double v = kf * pf - kr * pb;
    const double zF = st_entry(aa, r, b.Fb, ns), zU = st_entry(aa, r, b.Ub, ns);
    const double zw = -zU / ntot;  // (S^T w_bar)_r, w = Jn N, w_bar = -u_bar / ntot
    double zk[4];
#pragma unroll
    for (int k = 0; k < 4; k++) zk[k] = st_entry(aa, r, b.Bb[k], ns);
    // Q_l: the second products' weights per slot, sum_k zk K_k + zw N at the slot's species
    double Q[6], Nv[6];
#pragma unroll
    for (int m = 0; m < 6; m++) {
      const int s = q.s[m];
      Nv[m] = s < ns ? c.N[s] : 0.0;
      double acc = zw * Nv[m];
      if (s < ns) {
        acc = fma(zk[0], c.K1[s], acc);
        acc = fma(zk[1], c.K2[s], acc);
        acc = fma(zk[2], c.K3[s], acc);
        acc = fma(zk[3], c.K4[s], acc);
      }
      Q[m] = acc;
    }
    const double ab = ixf * zF + zU / nd;  // first-order weight on dv / dn
    const double nf1 = Nv[0] * q.a[1] * q.a[2] + q.a[0] * Nv[1] * q.a[2] + q.a[0] * q.a[1] * Nv[2];
    const double nb1 = Nv[3] * q.a[4] * q.a[5] + q.a[3] * Nv[4] * q.a[5] + q.a[3] * q.a[4] * Nv[5];
    sF = fma(zF, v, sF);
    sU = fma(zU, v, sU);
    sW = fma(zU, kf * nf1 - kr * nb1, sW);
#pragma unroll
    for (int m = 0; m < 6; m++) {
      const int base = m < 3 ? 0 : 3, i = m - base;
      const double sign = m < 3 ? kf : -kr;
      // sum_{l != m} Q_l prod of the third slot
      const int l1 = base + (i == 0 ? 1 : 0), l2 = base + (i == 2 ? 1 : 2);
      const double second = Q[l1] * q.a[l2] + Q[l2] * q.a[l1];
      const double o = others(q, m);
      c1[r * 6 + m] = sign * fma(ab, o, second);
      c2[r * 6 + m] = sign * zw * o;
    }
    double kfb = ab * pf, krb = -ab * pb;
#pragma unroll
    for (int m = 0; m < 3; m++) kfb = fma(Q[m], others(q, m), kfb);
#pragma unroll
    for (int m = 3; m < 6; m++) krb = fma(-Q[m], others(q, m), krb);
    kb[r] += kfb;
    kb[nr + r] += krb;
  }
  const double ixfb = block_sum(sF, b.red, tid, nt);   // Fb . s
  const double us = block_sum(sU, b.red, tid, nt);     // Ub . s
  const double uw = block_sum(sW, b.red, tid, nt);     // Ub . w
  gather(net, aa, c1, b.Nn, tid, nt);
  gather(net, aa, c2, b.Nx, tid, nt);
  __syncthreads();
  double px = 0.0;
  for (int i = tid; i < ns; i += nt) px = fma(b.Nn[i], c.N[i], px);
  const double xfb = block_sum(px, b.red, tid, nt);
  const double ntb = ixfb / nd - xfb * nd / (ntot * ntot) + uw / (ntot * ntot);
  if (tid == 0) ndb += -ixfb * ntot / (nd * nd) + xfb / ntot - us / (nd * nd);
  for (int i = tid; i < ns; i += nt) b.Nb[i] += fma(b.Nn[i], xf, b.Nx[i] + ntb);
  __syncthreads();
}

// ---- the step control's partials ----

// fac and its partials in en, pen, pha and ha (step_factor's derivative, ties and clamps as step_factor_tangent)
struct FacParts {
  double f, e, pen, pha, ha;
};

__device__ __forceinline__ FacParts step_factor_parts(double en, bool ok, bool prej, double pen, double pha,
                                                      double ha) {
  FacParts p = {MX_FAC_NONFINITE, 0.0, 0.0, 0.0, 0.0};
  const bool efin = isfinite(en);
  double f = MX_FAC_NONFINITE;
  if (efin) {
    const double e = fmax(en, MX_ERR_FLOOR);
    f = MX_STEP_SAFETY / cbrt(e);
    p.e = en >= MX_ERR_FLOOR ? -f / (3.0 * e) : 0.0;
  }
  const double lo = ok ? MX_FACACC : MX_FACREJ;
  if (f < lo) p.e = 0.0;
  f = fmax(f, lo);
  if (f > MX_FACMAX) p.e = 0.0;
  f = fmin(f, MX_FACMAX);
  if (!ok && efin && prej && en > 1.0 && pen > 1.0 && pha > ha) {
    const double lph = log(pha / ha), pe = log(pen / en) / lph;
    p.e = 0.0;
    if (pe > MX_SECANT_MIN_ORDER) {
      const double pp = fmin(pe, MX_SECANT_MAX_ORDER), act = pe <= MX_SECANT_MAX_ORDER ? 1.0 : 0.0;
      const double g = pow(MX_SECANT_TARGET / en, 1.0 / pp), L = log(MX_SECANT_TARGET / en);
      f = fmax(g, MX_SECMIN);
      if (g >= MX_SECMIN) {
        const double dlp = -L / (pp * pp) * act;  // d ln g / d pe
        p.e = g * (-1.0 / (en * pp) + dlp * (-1.0 / (en * lph)));
        p.pen = g * dlp / (pen * lph);
        p.pha = g * dlp * (-pe / (pha * lph));
        p.ha = g * dlp * (pe / (ha * lph));
      }
    } else {
      f = MX_SECMIN;
    }
  }
  if (!ok && f > MX_FAC_AFTER_REJECT) p.e = p.pen = p.pha = p.ha = 0.0;
  p.f = ok ? f : fmin(f, MX_FAC_AFTER_REJECT);
  return p;
}

// Step-state cotangents carried backwards between tries (thread-uniform): of h, t, pen and pha after the try, and
// the accumulated dt_bar and nd_bar.
struct StepBar {
  double h, t, pen, pha, dt, nd;
};

// The adjoint of one try (after primal_try recomputed it from its stored state s). Nb holds N's cotangent after the
// try on entry and before it on exit; sb the step cotangents likewise.
template <int W, int R, bool DENSE>
__device__ __noinline__ void adjoint_try(const Net& net, const Cell& c, const AdjCell& b, const AdjArgs& aa, double* sl,
                            const StepState& s, double dt, double nd, double c0, const int* pr, double rtol,
                            double atol, StepBar& sb, int tid) {
  constexpr int nt = 32 * W;
  const int ns = net.ns, lane = tid & 31, warp = tid >> 5;
  const double ha = fmin(s.h, dt - s.t), ih = 1.0 / ha, en = c.red[0];
  const bool ok = c.red[1] != 0.0, first = s.t == 0.0;
  if (!ok && !aa.adapt) return;  // frozen: a rejected try drops out (it changes neither N nor a fixed size)
  double hab = 0.0, enb = 0.0, penb = 0.0, phab = 0.0;
  if (aa.adapt) {
    const FacParts fp = step_factor_parts(en, ok, s.prej, s.pen, s.pha, ha);
    hab = sb.h * fma(ha, fp.ha, fp.f) + sb.pha;
    enb = fma(sb.h * ha, fp.e, sb.pen);
    penb = sb.h * ha * fp.pen;
    phab = sb.h * ha * fp.pha;
    if (ok) hab += sb.t;
  }
  // N' = N + 2 K1 + K3 + K4 and the accepted state max(N', 0): N' takes N's cotangent where N' >= 0
  for (int i = tid; i < ns; i += nt) {
    const double nb = b.Nb[i];
    b.Yb[i] = ok ? (c.Y[i] >= 0.0 ? nb : 0.0) : 0.0;
    if (ok) b.Nb[i] = 0.0;
  }
  __syncthreads();
  if (warp == 0 && aa.adapt && isfinite(en) && enb != 0.0) {  // err's adjoint (try_error's)
    double e2 = 0.0, em = 0.0;
    for (int i = lane; i < ns; i += 32) {
      const double sc = fma(rtol, fmax(fabs(c.N[i]), fabs(c.Y[i])), atol), q = c.K4[i] / sc;
      e2 = fma(q, q, e2);
      em = fmax(em, fabs(q));
    }
    const double er = sqrt(warp_sum(e2) / ns), emx = warp_max(em);
    double erb = enb, emb = 0.0;
    if (first && isfinite(er)) {
      erb = er > emx ? enb : (emx > er ? 0.0 : 0.5 * enb);
      emb = enb - erb;
    }
    double cnt = 0.0;
    for (int i = lane; i < ns; i += 32) {
      const double sc = fma(rtol, fmax(fabs(c.N[i]), fabs(c.Y[i])), atol), q = c.K4[i] / sc;
      cnt += fabs(q) == emx ? 1.0 : 0.0;
    }
    cnt = warp_sum(cnt);
    for (int i = lane; i < ns; i += 32) {
      const double an = fabs(c.N[i]), ay = fabs(c.Y[i]);
      const double sc = fma(rtol, fmax(an, ay), atol), q = c.K4[i] / sc;
      double qb = er > 0.0 ? erb * q / (ns * er) : 0.0;
      if (emb != 0.0 && fabs(q) == emx && cnt > 0.0) qb += emb * (q > 0.0 ? 1.0 : (q < 0.0 ? -1.0 : 0.0)) / cnt;
      const double scb = -qb * q / sc, mb = rtol * scb;
      const double wa = an > ay ? 1.0 : (ay > an ? 0.0 : 0.5);
      const double sn = c.N[i] > 0.0 ? 1.0 : (c.N[i] < 0.0 ? -1.0 : 0.0);
      const double sy = c.Y[i] > 0.0 ? 1.0 : (c.Y[i] < 0.0 ? -1.0 : 0.0);
      b.Nb[i] += wa * mb * sn;
      b.Yb[i] += (1.0 - wa) * mb * sy;
      b.Kb[3][i] = qb / sc;  // K4's own share; N''s follows below
    }
  } else if (warp == 0) {
    for (int i = lane; i < ns; i += 32) b.Kb[3][i] = 0.0;
  }
  __syncthreads();
  for (int i = tid; i < ns; i += nt) {
    const double yb = b.Yb[i];
    b.Nb[i] += yb;
    b.Kb[0][i] = 2.0 * yb;
    b.Kb[1][i] = 0.0;
    b.Kb[2][i] = yb;
    b.Kb[3][i] += yb;
  }
  __syncthreads();
  // stage 4: K4 = W^-1 (F(Y4) + (K1 - K2 - C43 K3) / h)
  if (warp == 0) {
    for (int i = lane; i < ns; i += 32) b.Bb[3][i] = b.Kb[3][i];
    __syncwarp();
    stage_solve_t<R, DENSE>(net, c, b.Bb[3], c0, pr, b.Nn, lane);
    double p = 0.0;
    for (int i = lane; i < ns; i += 32) {
      const double bb = b.Bb[3][i];
      b.Kb[0][i] = fma(ih, bb, b.Kb[0][i]);
      b.Kb[1][i] = fma(-ih, bb, b.Kb[1][i]);
      b.Kb[2][i] = fma(-RODAS_C43 * ih, bb, b.Kb[2][i]);
      p = fma(fma(-RODAS_C43, c.K3[i], c.K1[i] - c.K2[i]), bb, p);
    }
    p = warp_sum(p);
    if (lane == 0) b.red[nt + 1] = -ih * ih * p;
  }
  __syncthreads();
  hab += b.red[nt + 1];
  __syncthreads();
  f_adjoint(net, c, b, aa, sl, 2, b.Bb[3], nd, sb.nd, tid, nt);
  // stage 3: K3 = W^-1 (F(Y3) + (K1 - K2) / h)
  if (warp == 0) {
    for (int i = lane; i < ns; i += 32) b.Bb[2][i] = b.Kb[2][i];
    __syncwarp();
    stage_solve_t<R, DENSE>(net, c, b.Bb[2], c0, pr, b.Nn, lane);
    double p = 0.0;
    for (int i = lane; i < ns; i += 32) {
      const double bb = b.Bb[2][i];
      b.Kb[0][i] = fma(ih, bb, b.Kb[0][i]);
      b.Kb[1][i] = fma(-ih, bb, b.Kb[1][i]);
      p = fma(c.K1[i] - c.K2[i], bb, p);
    }
    p = warp_sum(p);
    if (lane == 0) b.red[nt + 1] = -ih * ih * p;
  }
  __syncthreads();
  hab += b.red[nt + 1];
  __syncthreads();
  f_adjoint(net, c, b, aa, sl, 1, b.Bb[2], nd, sb.nd, tid, nt);
  // stages 2 and 1: K2 = W^-1 (F(N) + C21 K1 / h), K1 = W^-1 F(N)
  if (warp == 0) {
    for (int i = lane; i < ns; i += 32) b.Bb[1][i] = b.Kb[1][i];
    __syncwarp();
    stage_solve_t<R, DENSE>(net, c, b.Bb[1], c0, pr, b.Nn, lane);
    double p = 0.0;
    for (int i = lane; i < ns; i += 32) {
      const double bb = b.Bb[1][i];
      b.Kb[0][i] = fma(RODAS_C21 * ih, bb, b.Kb[0][i]);
      p = fma(c.K1[i], bb, p);
    }
    p = warp_sum(p);
    __syncwarp();
    for (int i = lane; i < ns; i += 32) b.Bb[0][i] = b.Kb[0][i];
    __syncwarp();
    stage_solve_t<R, DENSE>(net, c, b.Bb[0], c0, pr, b.Nn, lane);
    // W's own derivative: dW = -dh / (gamma h^2) I - dJ_N, so h gains sum_k Bb_k . K_k / (gamma h^2), and J_N's
    // cotangent is sum_k Bb_k K_k^T: u's share is sum_k (sum K_k) Bb_k
    double w = 0.0, sk[4] = {0.0, 0.0, 0.0, 0.0};
    const double* K[4] = {c.K1, c.K2, c.K3, c.K4};
#pragma unroll
    for (int k = 0; k < 4; k++) {
      double a = 0.0;
      for (int i = lane; i < ns; i += 32) {
        w = fma(b.Bb[k][i], K[k][i], w);
        a += K[k][i];
      }
      sk[k] = warp_sum(a);
    }
    w = warp_sum(w);
    for (int i = lane; i < ns; i += 32) {
      b.Fb[i] = b.Bb[0][i] + b.Bb[1][i];
      b.Ub[i] = sk[0] * b.Bb[0][i] + sk[1] * b.Bb[1][i] + sk[2] * b.Bb[2][i] + sk[3] * b.Bb[3][i];
    }
    if (lane == 0) b.red[nt + 1] = -RODAS_C21 * ih * ih * p + w / (GAMMA * ha * ha);
  }
  __syncthreads();
  hab += b.red[nt + 1];
  __syncthreads();
  n_adjoint(net, c, b, aa, sl, nd, sb.nd, tid, nt);
  // ha = min(h, dt - t): a tie splits
  if (aa.adapt) {
    const double rem = dt - s.t, w = s.h < rem ? 1.0 : (rem < s.h ? 0.0 : 0.5);
    sb.h = w * hab;
    sb.dt += (1.0 - w) * hab;
    sb.t -= (1.0 - w) * hab;
    sb.pen = penb;
    sb.pha = phab;
  }
}

// The rates' adjoint and the cell's cotangents: k_bar -> T, P (with nd_bar), lm, J and the Arrhenius exponents.
// Writes gT, gP, glm, gJ, gL of the cell. Two block sums.
__device__ void rates_adjoint(const Net& net, const Cell& c, const AdjCell& b, const AdjArgs& aa, double* sl,
                              int cell, double Tc, double P, double nd, double ndb, double* g, double* dg, int tid,
                              int nt) {
  const int ns = net.ns, nr = net.nr;
  const double lT = log(Tc), iT = 1.0 / Tc, lKT = log(MX_KB * Tc / MX_P0);
  const double* cf = net.nasa + (Tc < MX_NASA_SPLIT_T ? 0 : ns * 9);
  for (int i = tid; i < ns; i += nt) {
    g[i] = gibbs_rt(cf + 9 * i, Tc, lT, iT);
    dg[i] = gibbs_rt_dT(cf + 9 * i, Tc, lT, iT);
  }
  if (tid == 0) g[ns] = dg[ns] = 0.0;
  __syncthreads();
  const double* kb = adj_kbar(net, sl);
  double Tb = 0.0, rb = 0.0;  // cotangents of T (at fixed n_tot) and of ln n_tot
  for (int r = tid; r < nr; r += nt) {
    const double kf = c.kf[r], kr = c.kr[r];
    const double gf = kb[r] * kf, gr = kb[nr + r] * kr;  // cotangents of ln kf, ln kr
    if (aa.glm) aa.glm[(size_t)cell * nr + r] = gf + gr;
    double* gl = adj_gl(net, aa, sl) + (size_t)r * 3;
    if (r >= net.nrt) {  // kf = J e^lm
      const int b = r - net.nrt;
      const double em = aa.lm ? exp(aa.lm[(size_t)cell * nr + r]) : 1.0;
      if (aa.gJ) aa.gJ[(size_t)cell * net.nj + b] = kb[r] * em;
      gl[0] = gl[1] = gl[2] = 0.0;
      continue;
    }
    const int fl = __ldg(net.rf + r);
    const uint64_t w = __ldg(net.rx8 + r);
    const int x0 = w & 255, x1 = (w >> 8) & 255, x2 = (w >> 16) & 255;
    const int x3 = (w >> 24) & 255, x4 = (w >> 32) & 255, x5 = (w >> 40) & 255;
    const double* q = net.rc + 14 * r;
    const LawParts lp = law_parts(q, fl, Tc, lT, iT, nd);
    const double k = law(q, fl, Tc, lT, iT, nd);
    const double dgv = g[x3] + g[x4] + g[x5] - g[x0] - g[x1] - g[x2];
    const bool tb = (fl & FL_THREE_BODY) != 0;
    const double c3 = tb ? nd : 1.0;
    const double dmu = (double)(((fl >> 3) & 7) - 4);
    const double kfp = k * c3, krp = (k * exp(dgv + dmu * lKT)) * c3;
    const int mf = (fl >> 10) & 3, mr = (fl >> 12) & 3;
    const double bf = bimolecular_rate(mf, tb, kfp, nd), br = bimolecular_rate(mr, tb, krp, nd);
    const double qm = fmax(bf, br);
    const double lim = qm > MX_K_COLL ? 1.0 : (qm == MX_K_COLL ? 0.5 : 0.0);
    const double wf = bf > br ? 1.0 : (br > bf ? 0.0 : 0.5);
    const double sf = (mf == 3 ? 1.0 : 0.0) - (mf < 2 && tb ? 1.0 : 0.0);
    const double sr = (mr == 3 ? 1.0 : 0.0) - (mr < 2 && tb ? 1.0 : 0.0);
    const double gT = dg[x3] + dg[x4] + dg[x5] - dg[x0] - dg[x1] - dg[x2] + dmu * iT;
    // d ln kf = dA + dlnc + dlm, d ln kr = dA + dG + dlnc + dlm, dlnc = -lim (wf (dA + sf rho) + (1 - wf)(dA + dG + sr rho))
    const double G = (kf == 0.0 ? 0.0 : gf) + (kr == 0.0 ? 0.0 : gr), Gc = -lim * G;
    const double Ab = G + Gc, Gb = (kr == 0.0 ? 0.0 : gr) + Gc * (1.0 - wf);
    Tb += Ab * lp.aT + Gb * gT;
    rb += Ab * (lp.aN + (tb ? 1.0 : 0.0)) + Gc * (wf * sf + (1.0 - wf) * sr);
    gl[0] = Ab * lp.a1;
    gl[1] = Ab * lp.a2;
    gl[2] = Ab * lp.ainf;
  }
  Tb = block_sum(Tb, b.red, tid, nt);
  rb = block_sum(rb, b.red, tid, nt) + ndb * nd;
  if (tid == 0) {
    aa.gT[cell] = Tb - rb / Tc;  // ln n_tot = ln P - ln T - ln k_B
    aa.gP[cell] = rb / P;
  }
}

// the cell's x cotangent into N's: x = N / sum N (before the guard's correction)
__device__ __forceinline__ void x_adjoint(const Net& net, const Cell& c, const AdjCell& b, const AdjArgs& aa, int cell,
                                          double sum, int tid, int nt) {
  const int ns = net.ns;
  const double* gx = aa.gx + (size_t)cell * ns;
  double p = 0.0;
  for (int i = tid; i < ns; i += nt) {
    const double xb = gx[__ldg(net.perm + i)];
    b.Nb[i] = xb;
    p = fma(xb, c.N[i] / sum, p);
  }
  const double dot = block_sum(p, b.red, tid, nt);
  for (int i = tid; i < ns; i += nt) b.Nb[i] = (b.Nb[i] - dot) / sum;
  __syncthreads();
}

// The reverse pass over a pass of n tries from the initial state (N0 in c.N on entry is overwritten): states from the
// store, or checkpoints and recomputed segments. Leaves N0's cotangent in Nb and the step cotangents in sb.
template <int W, int R, bool DENSE>
__device__ void reverse_pass(const Net& net, const Cell& c, const AdjCell& b, const AdjArgs& aa, double* sl,
                             const StepState& s0, int n, double dt, double nd, const int* pr, double rtol,
                             double atol, StepBar& sb, int tid) {
  constexpr int nt = 32 * W;
  const int cap = aa.cap;
  if (n <= cap) {  // every try's state is in bank 0
    for (int i = n - 1; i >= 0; i--) {
      const StepState s = load_state(net, c, adj_state(net, aa, sl, 0, i), tid, nt);
      double c0 = 0.0;
      primal_try<W, R, DENSE>(net, c, s, dt, nd, rtol, atol, pr, c0, tid);
      adjoint_try<W, R, DENSE>(net, c, b, aa, sl, s, dt, nd, c0, pr, rtol, atol, sb, tid);
    }
    return;
  }
  // checkpoints every `stride` tries into bank 1, then each segment recomputed into bank 0 and reversed
  const int stride = (n + cap - 1) / cap, segs = (n + stride - 1) / stride;
  StepState s = load_state(net, c, adj_state(net, aa, sl, 0, 0), tid, nt);  // the first try's state (N0)
  for (int i = 0; i < n; i++) {
    if (i % stride == 0) store_state(net, c, adj_state(net, aa, sl, 1, i / stride), s, tid, nt);
    __syncthreads();
    double c0 = 0.0;
    primal_try<W, R, DENSE>(net, c, s, dt, nd, rtol, atol, pr, c0, tid);
    primal_update(net, c, s, dt, tid, nt);
  }
  for (int g = segs - 1; g >= 0; g--) {
    const int i0 = g * stride, i1 = min(n, i0 + stride);
    s = load_state(net, c, adj_state(net, aa, sl, 1, g), tid, nt);
    for (int i = i0; i < i1; i++) {
      store_state(net, c, adj_state(net, aa, sl, 0, i - i0), s, tid, nt);
      __syncthreads();
      if (i + 1 < i1) {
        double c0 = 0.0;
        primal_try<W, R, DENSE>(net, c, s, dt, nd, rtol, atol, pr, c0, tid);
        primal_update(net, c, s, dt, tid, nt);
      }
    }
    for (int i = i1 - 1; i >= i0; i--) {
      const StepState si = load_state(net, c, adj_state(net, aa, sl, 0, i - i0), tid, nt);
      double c0 = 0.0;
      primal_try<W, R, DENSE>(net, c, si, dt, nd, rtol, atol, pr, c0, tid);
      adjoint_try<W, R, DENSE>(net, c, b, aa, sl, si, dt, nd, c0, pr, rtol, atol, sb, tid);
    }
  }
}

// The cotangents of the cell's inputs after the reverse pass: x0 (from Nb), h and dt (from the first try's size
// max(min(h0, dt), H_MIN), or min(h0, dt, dt split^k) on retry k), then the rates'.
__device__ void finish_cell(const Net& net, const Cell& c, const AdjCell& b, const AdjArgs& aa, double* sl, int cell,
                            double Tc, double P, double nd, double hin, double dt, int retry, StepBar& sb, bool nan,
                            double* g, double* dg, int tid, int nt) {
  const int ns = net.ns;
  if (nan) {
    const double q = __longlong_as_double(0x7ff8000000000000ll);
    for (int i = tid; i < ns; i += nt) aa.gx0[(size_t)cell * ns + __ldg(net.perm + i)] = q;
    for (int r = tid; r < net.nr; r += nt) {
      if (aa.glm) aa.glm[(size_t)cell * net.nr + r] = q;
      double* gl = adj_gl(net, aa, sl) + (size_t)r * 3;
      gl[0] = gl[1] = gl[2] = q;
    }
    for (int j = tid; j < net.nj; j += nt) aa.gJ[(size_t)cell * net.nj + j] = q;
    if (tid == 0) aa.gT[cell] = aa.gP[cell] = aa.gdt[cell] = aa.gh0[cell] = q;
    __syncthreads();
    return;
  }
  for (int i = tid; i < ns; i += nt) aa.gx0[(size_t)cell * ns + __ldg(net.perm + i)] = b.Nb[i];
  if (tid == 0) {
    double hb = 0.0, dtb = sb.dt;
    if (aa.adapt) {
      const bool fin = isfinite(hin);
      const double h0 = fin ? hin : dt, m = fmin(h0, dt);
      double start = m, wm = 1.0;  // start's share that goes to m
      if (retry > 0) {
        const double cap = dt * pow(MX_REC_RETRY_SPLIT, (double)retry);
        start = fmin(m, cap);
        wm = m < cap ? 1.0 : (cap < m ? 0.0 : 0.5);
        dtb += (1.0 - wm) * (start >= MX_H_MIN ? sb.h : 0.0) * pow(MX_REC_RETRY_SPLIT, (double)retry);
      }
      const double mb = start >= MX_H_MIN ? wm * sb.h : 0.0;
      const double w0 = h0 < dt ? 1.0 : (dt < h0 ? 0.0 : 0.5);
      if (fin) {
        hb = w0 * mb;
        dtb += (1.0 - w0) * mb;
      } else {
        dtb += mb;  // a non-finite h acts as dt, with no cotangent of its own
      }
    }
    aa.gh0[cell] = hb;
    aa.gdt[cell] = dtb;
  }
  rates_adjoint(net, c, b, aa, sl, cell, Tc, P, nd, sb.nd, g, dg, tid, nt);
  __syncthreads();
}

// ---- the kernels ----

// A passing cell's rate-table cotangent (adj_gl) into its chunk's partial sum: per reaction (one thread) and
// exponent e, the sum over the chunk's passing cells in cell order of g, g ln T and -g / T; the chunk's first
// passing cell writes, the others add.
__device__ __forceinline__ void add_to_chunk(const Net& net, const AdjArgs& aa, double* sl, int chunk, double Tc,
                                             bool first, int tid, int nt) {
  const double lT = log(Tc), iT = 1.0 / Tc;
  const double* gl = adj_gl(net, aa, sl);
  for (int r = tid; r < net.nr; r += nt) {
    double* dst = aa.gLc + ((size_t)r * aa.nchunks + chunk) * 9;
#pragma unroll
    for (int e = 0; e < 3; e++) {
      const double g = gl[3 * r + e];
      if (first) {
        dst[3 * e] = g;
        dst[3 * e + 1] = g * lT;
        dst[3 * e + 2] = -g * iT;
      } else {
        dst[3 * e] += g;
        dst[3 * e + 1] = fma(g, lT, dst[3 * e + 1]);
        dst[3 * e + 2] = fma(-g, iT, dst[3 * e + 2]);
      }
    }
  }
}

// The adjoint kernel: the call kernel's screening, rates, tries (each try's state stored), output and guard, then,
// for a cell that passed the guard, the reverse pass and its cotangents. A listed cell is left to the recovery's.
// Cells come in chunks of ADJ_CHUNK consecutive cells from the queue, each chunk's cells in order, so each chunk's
// partial sum of the rate table's cotangent is formed by one CTA in a fixed order.
template <int W, int R>
__global__ void __launch_bounds__(32 * W, 3) vjp_kernel(const Net net, const CallArgs a, const AdjArgs aa,
                                                        const AdjLayout al) {
  extern __shared__ double smem[];
  const Cell c = cell_arrays(net, smem);
  const AdjCell b = adj_arrays(al, smem);
  const int tid = (int)threadIdx.x, nt = 32 * W, lane = tid & 31, warp = tid >> 5, ns = net.ns;
  double* sl = aa.scratch + (size_t)blockIdx.x * aa.slot;
  int chunk = (int)blockIdx.x;
  while (chunk < aa.nchunks) {
    const int first_cell = chunk * ADJ_CHUNK, end_cell = min(a.B, first_cell + ADJ_CHUNK);
    bool started = false, any_listed = false;
    for (int cell = first_cell; cell < end_cell; cell++) {
      const double Tc = a.T[cell], dt = a.dt[cell], hin = a.h_in[cell], P = a.P[cell];
      const double nd = P / (MX_KB * Tc);
      const double* x0 = a.x + (size_t)cell * ns;
      const double* Jc = a.J + (size_t)cell * net.nj;
      const double* lmc = aa.lm ? aa.lm + (size_t)cell * net.nr : nullptr;
      for (int i = tid; i < ns; i += nt) c.N[i] = x0[__ldg(net.perm + i)];
      __syncthreads();
      if (warp == 0) {  // screening, as the call kernel's
        const double nan = __longlong_as_double(0x7ff8000000000000ll);
        double p = 0.0, pm = 0.0;
        for (int i = lane; i < ns; i += 32) {
          const double xi = c.N[i];
          p += xi >= 0.0 ? xi : nan;
          pm = fmax(pm, xi);
        }
        for (int j = lane; j < net.nj; j += 32) {
          const double q = Jc[j];
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
      const bool lm_fine = multipliers_finite(net, lmc, tid);
      if (st == 0) {
        cell_rates(net, c, Tc, nd, Jc, tid, nt);
        if (lmc) apply_multipliers(net, c, lmc, tid, nt);
      }
      const double h0 = isfinite(hin) ? hin : dt;
      StepState s = {fmax(fmin(h0, dt), MX_H_MIN), 0.0, 0.0, 0.0, 0.0, false};
      const StepState s0 = s;
      int it = (dt > 0.0 && st == 0 && lm_fine) ? 0 : a.max_steps, n = 0;
      while (it < a.max_steps && s.t < dt * MX_CALL_END) {
        if (n < aa.cap) store_state(net, c, adj_state(net, aa, sl, 0, n), s, tid, nt);
        double c0 = 0.0;
        primal_try<W, R, false>(net, c, s, dt, nd, a.rtol, a.atol, nullptr, c0, tid);
        primal_update(net, c, s, dt, tid, nt);
        it++;
        n++;
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
          c.ints[2] = r;
        }
      }
      __syncthreads();
      double* xo = a.x_out + (size_t)cell * ns;
      for (int i = tid; i < ns; i += nt) xo[i] = c.Y[i];
      const int listed = c.ints[2];
      if (!listed) {  // a listed cell's cotangents come from the recovery
        double* kb = adj_kbar(net, sl);
        for (int r = tid; r < 2 * net.nr; r += nt) kb[r] = 0.0;
        StepBar sb = {aa.adapt && aa.gh ? aa.gh[cell] : 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        __syncthreads();
        if (st == 0) {
          x_adjoint(net, c, b, aa, cell, sum, tid, nt);
          reverse_pass<W, R, false>(net, c, b, aa, sl, s0, n, dt, nd, nullptr, a.rtol, a.atol, sb, tid);
        }
        finish_cell(net, c, b, aa, sl, cell, Tc, P, nd, hin, dt, 0, sb, st != 0, c.v, b.Nn, tid, nt);
        if (st == 0) {  // a refused cell stays out of the rate table's sum
          add_to_chunk(net, aa, sl, chunk, Tc, !started, tid, nt);
          started = true;
        }
      } else {
        any_listed = true;
      }
      __syncthreads();
    }
    if (!started)  // no passing cell: the chunk's partial sum is zero
      for (int r = tid; r < net.nr; r += nt)
        for (int k = 0; k < 9; k++) aa.gLc[((size_t)r * aa.nchunks + chunk) * 9 + k] = 0.0;
    if (tid == 0) {
      aa.chunk_listed[chunk] = any_listed ? 1 : 0;
      atomicAdd(a.count + MX_COUNT_QUEUE, end_cell - first_cell);
      c.ints[1] = (int)(gridDim.x + atomicAdd(aa.chunk_queue, 1));
    }
    __syncthreads();
    chunk = c.ints[1];
    __syncthreads();
  }
}

// The adjoint of the recovery (recover_kernel's path): each listed cell redone on the dense pivoted W, retries
// included, and the pass whose result is the cell's reversed. A cell that still fails has NaN cotangents.
template <int W, int R>
__global__ void __launch_bounds__(32 * W, 3) vjp_recover_kernel(const Net net, const CallArgs a, const AdjArgs aa,
                                                                const AdjLayout al, int max_steps) {
  const int nfl = a.count[MX_COUNT_RECOMPUTED];
  if ((int)blockIdx.x >= nfl) return;
  extern __shared__ double smem[];
  const Cell c = cell_arrays(net, smem);
  const AdjCell b = adj_arrays(al, smem);
  const int tid = (int)threadIdx.x, nt = 32 * W, lane = tid & 31, warp = tid >> 5, ns = net.ns;
  int* pr = c.ints + 4;
  double* sl = aa.scratch + (size_t)blockIdx.x * aa.slot;
  int q = (int)blockIdx.x;
  while (q < nfl) {
    const int cell = a.list[q];
    const double Tc = a.T[cell], dt = a.dt[cell], hin = a.h_in[cell], P = a.P[cell];
    const double nd = P / (MX_KB * Tc);
    const double* x0 = a.x + (size_t)cell * ns;
    const double* Jc = a.J + (size_t)cell * net.nj;
    const double* lmc = aa.lm ? aa.lm + (size_t)cell * net.nr : nullptr;
    const bool lm_fine = multipliers_finite(net, lmc, tid);
    cell_rates(net, c, Tc, nd, Jc, tid, nt);
    if (lmc) apply_multipliers(net, c, lmc, tid, nt);
    const double h0 = isfinite(hin) ? hin : dt, m = fmin(h0, dt);
    for (int k = 0;; k++) {
      for (int i = tid; i < ns; i += nt) c.N[i] = x0[__ldg(net.perm + i)];
      __syncthreads();
      const double start = k == 0 ? m : fmin(m, dt * pow(MX_REC_RETRY_SPLIT, (double)k));
      StepState s = {fmax(start, MX_H_MIN), 0.0, 0.0, 0.0, 0.0, false};
      const StepState s0 = s;
      int it = (dt > 0.0 && lm_fine) ? 0 : max_steps, n = 0;
      while (it < max_steps && s.t < dt * MX_CALL_END) {
        if (n < aa.cap) store_state(net, c, adj_state(net, aa, sl, 0, n), s, tid, nt);
        double c0 = 0.0;
        primal_try<W, R, true>(net, c, s, dt, nd, a.rtol, a.atol, pr, c0, tid);
        primal_update(net, c, s, dt, tid, nt);
        it++;
        n++;
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
          c.ints[1] = -1;
        } else {
          a.h_out[cell] = s.h;
          a.done[cell] = g ? 0 : dn;
          a.steps[cell] = s.nok;
          a.flag[cell] = g ? 2 : 1;
          c.ints[2] = g;
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
        const bool failed = c.ints[2] != 0;
        double* kb = adj_kbar(net, sl);
        for (int r = tid; r < 2 * net.nr; r += nt) kb[r] = 0.0;
        StepBar sb = {aa.adapt && aa.gh ? aa.gh[cell] : 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        __syncthreads();
        if (!failed) {
          x_adjoint(net, c, b, aa, cell, sum, tid, nt);
          reverse_pass<W, R, true>(net, c, b, aa, sl, s0, n, dt, nd, pr, a.rtol, a.atol, sb, tid);
        }
        finish_cell(net, c, b, aa, sl, cell, Tc, P, nd, hin, dt, k, sb, failed, c.v, b.Nn, tid, nt);
        // the cell's rate-table cotangent into its list slot, for the fixed-order sum
        const double* gl = adj_gl(net, aa, sl);
        for (int e = tid; e < 3 * net.nr; e += nt) aa.gLq[(size_t)q * 3 * net.nr + e] = gl[e];
        if (tid == 0) aa.pos[cell] = q;
        __syncthreads();
        q = nq;
        break;
      }
    }
  }
}

// The rate table's cotangent: per reaction (one block of 9 threads, one per column), the chunks' partial sums in
// chunk order, each chunk followed by its recovered cells in cell order (their list slots' cotangents times 1, ln T,
// -1 / T); cells that still fail (flag 2) or were refused are left out. Photolysis rows are 0. A fixed order: the
// same inputs give the same bits, whatever the queues did.
__global__ void arrh_kernel(const Net net, const CallArgs a, const AdjArgs aa, double* grc) {
  const int r = (int)blockIdx.x, j = (int)threadIdx.x;
  if (j >= 9) return;
  double acc = 0.0;
  if (r < net.nrt) {
    const int e = j / 3, kind = j % 3;
    for (int k = 0; k < aa.nchunks; k++) {
      acc += aa.gLc[((size_t)r * aa.nchunks + k) * 9 + j];
      if (!aa.chunk_listed[k]) continue;
      const int c1 = min(a.B, (k + 1) * ADJ_CHUNK);
      for (int cell = k * ADJ_CHUNK; cell < c1; cell++) {
        if (a.flag[cell] != 1) continue;  // passed (in the chunk's sum), still failed or refused
        const double g = aa.gLq[((size_t)aa.pos[cell] * net.nr + r) * 3 + e], Tc = a.T[cell];
        acc = kind == 0 ? acc + g : (kind == 1 ? fma(g, log(Tc), acc) : fma(-g, 1.0 / Tc, acc));
      }
    }
  }
  grc[(size_t)r * 9 + j] = acc;
}

}  // namespace mx
