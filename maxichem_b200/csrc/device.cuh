// Device arithmetic of the per-call chemistry solve: rates, right-hand side, Jacobian, dense LU and solves,
// Rodas3 stages, step control and the guard. One CTA steps one cell at a time; its W warps share the cell's arrays in
// shared memory. Every sum that reaches the state has a fixed order (ascending index, or the 32-lane butterfly), so
// a cell's result does not depend on the batch, its order, or the launch shape.
//
// Arithmetic follows imalsky/maxichem maxichem/kernels/common.cuh, call.cuh, guard.cuh and recover.cuh (cited per
// function). The library is built with -fmad=false: every fused multiply-add is an explicit fma().
#pragma once
#include <cstdint>

#include "../../include/maxichem_b200.h"

namespace mx {

constexpr unsigned FULL = 0xffffffffu;
constexpr double GAMMA = 0.5;            // Rodas3's diagonal coefficient (Sandu et al. 1997)
constexpr double RODAS_C21 = 4.0;        // stage coupling C_21
constexpr double RODAS_C43 = 8.0 / 3.0;  // stage coupling, -C_43
constexpr double TROE_C0 = 0.4, TROE_C1 = 0.67, TROE_N0 = 0.75, TROE_N1 = 1.27, TROE_D = 0.14;  // Venot et al. 2012
constexpr int FL_FALLOFF = 1, FL_SECOND_K0 = 2, FL_THREE_BODY = 4, FL_TROE = 64, FL_EFF = 128, FL_VM11 = 512;
constexpr int GUARD_NONFINITE = 4, GUARD_UNFINISHED = 8, GUARD_DRIFT = 16;
constexpr int PANEL = 8;  // pivots per block of the blocked LU

// A network's tables on the device, and the per-CTA shared-memory layout (offsets in doubles).
struct Net {
  int ns, nr, nrt, nj, nel, n_entries;
  const int* perm;
  const uint64_t* rx8;  // 8 bytes per reaction: reactants 0-2, products 3-5, padding
  const double* rc;
  const int* rf;
  const double* nasa;
  const double* atoms;
  const int* sv_ptr;
  const uint32_t* sv_term;
  const int* jac_ptr;
  const uint32_t* jac_entry;
  const uint32_t* jac_term;
  double etot, drift;
  // per-thread streams of the S v and Jacobian sums for the CTA (group 0) and its last 96 threads (group 1)
  int st_threads[2], sv_rounds[2], sv_nrows[2], jac_rounds[2], jac_nents[2], n_pieces;
  const int* sv_row_ptr;
  const uint16_t* sv[2];
  const uint16_t* sv_rows[2];
  const uint32_t* jt[2];
  const uint16_t* jd[2];
  // shared-memory layout (offsets in doubles); a_doubles: the matrix region's size in doubles. The mixed-precision
  // layout adds the row scales (oS), the Jacobian's diagonal (oDg), n at the try's state (onN), w (oW), the
  // residual (oR) and a stage's right side (oB); the plain layout leaves them 0.
  int ld, oA, oK, oV, on, oN, oY, oF, oU, oK1, oK2, oK3, oK4, oD, oRed, oInts, oPart, oG, doubles, a_doubles;
  int oS, oDg, onN, oW, oR, oB;
};

struct CallArgs {
  const double *x, *T, *P, *dt, *h_in, *J;
  int B;
  double rtol, atol;
  int max_steps;
  double *x_out, *h_out;
  int* done;
  double* steps;
  int *flag, *status, *count, *list;
  unsigned long long* tries;  // nullable: [0] tries, [1] tries after a rejection, [2] recovery tries
  const int* in_list;  // list-mode kernels: the cells to step, in_count[0] of them (in_count[1]: their queue)
  int* in_count;
  int* sel;        // the mixed kernel's hand-backs for the plain kernel, sel_count[0] of them
  int* sel_count;
};

// Pointers into one CTA's shared memory.
struct Cell {
  double *A, *kf, *kr, *v, *n, *N, *Y, *F, *U, *K1, *K2, *K3, *K4, *dinv, *red, *part, *G;
  int* ints;
};

__device__ __forceinline__ Cell cell_arrays(const Net& net, double* smem) {
  Cell c;
  c.A = smem + net.oA;
  c.kf = smem + net.oK;
  c.kr = c.kf + net.nr;
  c.v = smem + net.oV;
  c.n = smem + net.on;
  c.N = smem + net.oN;
  c.Y = smem + net.oY;
  c.F = smem + net.oF;
  c.U = smem + net.oU;
  c.K1 = smem + net.oK1;
  c.K2 = smem + net.oK2;
  c.K3 = smem + net.oK3;
  c.K4 = smem + net.oK4;
  c.dinv = smem + net.oD;
  c.red = smem + net.oRed;
  c.ints = (int*)(smem + net.oInts);
  c.part = smem + net.oPart;
  c.G = smem + net.oG;
  return c;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
  return v;
}

__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(FULL, v, o));
  return v;
}

// sum of y[0..n) as a warp forms it: lane l adds y[l], y[l + 32], ... then the butterfly (every lane returns it).
__device__ __forceinline__ double lane_sum(const double* y, int n, int lane) {
  double p = 0.0;
  for (int i = lane; i < n; i += 32) p += y[i];
  return warp_sum(p);
}

__device__ __forceinline__ double code_coefficient(unsigned c) {
  return (c & 2u) ? ((c & 1u) ? -2.0 : 2.0) : ((c & 1u) ? -1.0 : 1.0);
}

// ---- rates (common.cuh:136-242) ----

__device__ __forceinline__ double law(const double* __restrict__ q, int fl, double Tc, double lT, double iT,
                                      double nd) {
  double k = exp(q[0] + q[1] * lT - q[2] * iT);
  if (fl & FL_SECOND_K0) k += exp(q[3] + q[4] * lT - q[5] * iT);
  if (fl & FL_FALLOFF) {
    const double pr = k * nd / exp(q[6] + q[7] * lT - q[8] * iT);
    k = k > 0.0 ? k / (1.0 + pr) : 0.0;
    if ((fl & FL_TROE) && k > 0.0) {
      const double fc = log10((1.0 - q[9]) * exp(-Tc / q[10]) + q[9] * exp(-Tc / q[11]) + exp(-q[12] / Tc));
      const double x = (fl & FL_VM11) ? log10(pr) : log10(pr) - TROE_C0 - TROE_C1 * fc;
      // at Pr = 0 the standard ratio tends to -1 / d, so F to Fc^(d^2 / (1 + d^2)); the VM11 one to -inf, F to 1
      const double y = (fl & FL_VM11) ? x / (TROE_N0 - TROE_N1 * fc)
                                      : (isfinite(x) ? x / (TROE_N0 - TROE_N1 * fc - TROE_D * x) : -1.0 / TROE_D);
      k *= exp10(fc / (1.0 + y * y));
    }
  }
  if (fl & FL_EFF) k *= q[13];
  return k;
}

__device__ __forceinline__ double bimolecular_rate(int molecules, bool three_body, double k, double nd) {
  return molecules >= 2 ? k * (molecules == 3 ? nd : 1.0) : (three_body ? k / nd : 0.0);
}

__device__ __forceinline__ double gibbs_rt(const double* __restrict__ a, double Tc, double lT, double iT) {
  const double T2 = Tc * Tc, T3 = T2 * Tc, T4 = T3 * Tc;
  const double h = -a[0] * iT * iT + a[1] * lT * iT + a[2] + a[3] * Tc / 2 + a[4] * T2 / 3 + a[5] * T3 / 4 +
                   a[6] * T4 / 5 + a[7] * iT;
  const double s = -a[0] * iT * iT / 2 - a[1] * iT + a[2] * lT + a[3] * Tc + a[4] * T2 / 2 + a[5] * T3 / 3 +
                   a[6] * T4 / 4 + a[8];
  return h - s;
}

// kf, kr of one cell (cell_rates, common.cuh:222-242); g (ns + 1 doubles) is scratch. Two barriers.
__device__ __forceinline__ void cell_rates(const Net& net, const Cell& c, double Tc, double nd, const double* __restrict__ Jc,
                           int tid, int nt) {
  const double lT = log(Tc), iT = 1.0 / Tc, lKT = log(MX_KB * Tc / MX_P0);
  double* g = c.v;
  const double* cf = net.nasa + (Tc < MX_NASA_SPLIT_T ? 0 : net.ns * 9);
  for (int i = tid; i < net.ns; i += nt) g[i] = gibbs_rt(cf + 9 * i, Tc, lT, iT);
  if (tid == 0) g[net.ns] = 0.0;
  __syncthreads();
  for (int r = tid; r < net.nr; r += nt) {
    if (r >= net.nrt) {
      c.kf[r] = Jc[r - net.nrt];
      c.kr[r] = 0.0;
      continue;
    }
    const int fl = __ldg(net.rf + r);
    const uint64_t w = __ldg(net.rx8 + r);
    const int x0 = w & 255, x1 = (w >> 8) & 255, x2 = (w >> 16) & 255;
    const int x3 = (w >> 24) & 255, x4 = (w >> 32) & 255, x5 = (w >> 40) & 255;
    const double k = law(net.rc + 14 * r, fl, Tc, lT, iT, nd);
    const double dg = g[x3] + g[x4] + g[x5] - g[x0] - g[x1] - g[x2];
    const double c3 = (fl & FL_THREE_BODY) ? nd : 1.0;
    const double dmu = (double)(((fl >> 3) & 7) - 4);
    double kf = k * c3, kr = (k * exp(dg + dmu * lKT)) * c3;
    const int mf = (fl >> 10) & 3, mr = (fl >> 12) & 3;
    const bool tb = (fl & FL_THREE_BODY) != 0;
    const double q = fmax(bimolecular_rate(mf, tb, kf, nd), bimolecular_rate(mr, tb, kr, nd));
    if (q > MX_K_COLL) {
      const double cc = MX_K_COLL / q;
      kf *= cc;
      kr *= cc;
    }
    c.kf[r] = kf;
    c.kr[r] = kr;
  }
  if (tid == 0) c.kf[2 * net.nr] = 0.0;  // the zero rate of the Jacobian stream's padding
  __syncthreads();
}

// ---- right-hand side (rhs, common.cuh:282-353) ----

// A barrier over the threads of a group: named barrier id (0 is __syncthreads' own) over n threads.
__device__ __forceinline__ void group_sync(int id, int n) { asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(n) : "memory"); }

// S v's pieces into part: each thread of the group its pieces (ascending reactions) from its coalesced word stream;
// v[nr] = 0 pads. Row i of S v is then part[sv_row_ptr[i]] + ... in order (sv_row of the caller).
__device__ __forceinline__ void sv_pieces_of(const Net& net, const Cell& c, const double* v, int gtid, int gnt) {
  const int g = gnt == net.st_threads[0] ? 0 : 1;
  const uint16_t* __restrict__ sw = net.sv[g] + gtid;
  const uint16_t* __restrict__ sr = net.sv_rows[g] + gtid;
  double s = 0.0;
  int piece = 0;
  const int rounds = net.sv_rounds[g];
#pragma unroll 4
  for (int q = 0; q < rounds; q++) {
    const unsigned w = __ldg(sw + q * gnt);
    s = fma(code_coefficient(w >> 11), v[w & 0x7ffu], s);
    if (w & 0x2000u) {
      c.part[__ldg(sr + piece * gnt)] = s;
      s = 0.0;
      piece++;
    }
  }
}

// Row i of S v from its pieces, added in order.
__device__ __forceinline__ double sv_row(const Net& net, const Cell& c, int i) {
  const int p0 = __ldg(net.sv_row_ptr + i), p1 = __ldg(net.sv_row_ptr + i + 1);
  double r = c.part[p0];
  for (int p = p0 + 1; p < p1; p++) r += c.part[p];
  return r;
}

// F = (ntot / nd) S v(n) at Y, u0 = S v / nd into U when u0; n = nd Y / ntot. Returns ntot. Run by a group of whole
// warps (gtid its thread index, gnt its size, synchronised by named barrier bar); three barriers.
__device__ __forceinline__ double rhs(const Net& net, const Cell& c, const double* Y, bool u0, double nd, int gtid, int gnt, int bar) {
  const int lane = gtid & 31, ns = net.ns;
  const double ntot = lane_sum(Y, ns, lane), xf = nd / ntot, ixf = ntot / nd;
  for (int i = gtid; i < ns; i += gnt) c.n[i] = Y[i] * xf;
  if (gtid == 0) {
    c.n[ns] = 1.0;
    c.v[net.nr] = 0.0;
  }
  group_sync(bar, gnt);
  const double* n = c.n;
  for (int r = gtid; r < net.nr; r += gnt) {
    const uint64_t w = __ldg(net.rx8 + r);
    const double a = c.kf[r] * n[w & 255] * n[(w >> 8) & 255] * n[(w >> 16) & 255];
    const double b = c.kr[r] * n[(w >> 24) & 255] * n[(w >> 32) & 255] * n[(w >> 40) & 255];
    c.v[r] = a - b;
  }
  group_sync(bar, gnt);
  sv_pieces_of(net, c, c.v, gtid, gnt);
  group_sync(bar, gnt);
  // each row: its pieces added in order
  for (int i = gtid; i < ns; i += gnt) {
    const double r = sv_row(net, c, i);
    c.F[i] = r * ixf;
    if (u0) c.U[i] = r / nd;
  }
  group_sync(bar, gnt);
  return ntot;
}

__device__ __forceinline__ double rhs(const Net& net, const Cell& c, const double* Y, bool u0, double nd, int tid,
                                      int nt) {
  return rhs(net, c, Y, u0, nd, tid, nt, 0);
}

// A = -Jn (dense, row stride ld), then U = u0 + (-Jn N) / ntot (call.cuh:61-79, jacobian_times_x). Three barriers.
__device__ __forceinline__ void jacobian_w(const Net& net, const Cell& c, double ntot, int tid, int nt) {
  const int ns = net.ns, ld = net.ld;
  for (int i = tid; i < ns * ld; i += nt) c.A[i] = 0.0;
  __syncthreads();
  {  // each thread its entries from its coalesced word stream; the padding words use the zero rate kf[2 nr]
    const uint32_t* __restrict__ jw = net.jt[0] + tid;
    const uint16_t* __restrict__ jd = net.jd[0] + tid;
    const int rounds = net.jac_rounds[0];
    double acc = 0.0;
    int e = 0;
#pragma unroll 4
    for (int q = 0; q < rounds; q++) {
      const unsigned w = __ldg(jw + q * nt);
      const double pr = c.kf[w & 0xfffu] * c.n[(w >> 16) & 255u] * c.n[w >> 24];
      acc = fma(code_coefficient(w >> 12), pr, acc);
      if (w & 0x4000u) {
        c.A[__ldg(jd + e * nt)] = -acc;
        acc = 0.0;
        e++;
      }
    }
  }
  __syncthreads();
  for (int i = tid; i < ns; i += nt) {
    const double* a = c.A + i * ld;
    double acc = 0.0;
    for (int j = 0; j < ns; j++) acc = fma(a[j], c.N[j], acc);
    c.U[i] = c.U[i] + acc / ntot;
  }
  __syncthreads();
}

// ---- dense LU without exchanges, blocked (PANEL pivots at a time), with a lookahead of one panel ----
// Every entry receives its updates A_ij <- fma(-l_ik, A_kj, A_ij) in ascending k, l_ik = A_ik / A_kk taken as
// A_ik * (1 / A_kk): the order and the operations of the right-looking LU, so the bits of the sparse factorisation
// on the fill pattern (call.cuh:81-112) for finite data. Per block: the block's pivot rows beyond the panel (one
// thread per column); then warp 0 applies the block to the next panel's columns and factors that panel (one lane per
// row, warp syncs only) while warps 1-3 apply it to the columns past the next panel, as a rank-PANEL update in 4 x 4
// register tiles (rows and columns cyclic, so a warp's loads are broadcast or consecutive).

// the element type's correctly rounded reciprocal (FP64 for the plain path, FP32 for the mixed path's factors)
__device__ __forceinline__ double rcp_rn(double a) { return __drcp_rn(a); }
__device__ __forceinline__ float rcp_rn(float a) { return __frcp_rn(a); }

// the trailing update of rows ke.. and columns cs.. (cs >= ke) by NT threads
template <int NT, typename T>
__device__ __forceinline__ void trailing_update_from(T* A, int ld, int kb, int nb, int ke, int cs, int ns, int tid) {
  constexpr int CG = 16, RG = NT / CG;
  const int cg = tid % CG, rg = tid / CG, m = ns - ke, mc = ns - cs;
  for (int rb = rg; rb < m; rb += 4 * RG) {
    for (int cb = cg; cb < mc; cb += 4 * CG) {
      int row[4], col[4];
      bool rok[4], cok[4];
#pragma unroll
      for (int a = 0; a < 4; a++) {
        rok[a] = rb + RG * a < m;
        row[a] = ke + (rok[a] ? rb + RG * a : 0);
        cok[a] = cb + CG * a < mc;
        col[a] = cs + (cok[a] ? cb + CG * a : 0);
      }
      T acc[4][4];
#pragma unroll
      for (int a = 0; a < 4; a++)
#pragma unroll
        for (int b = 0; b < 4; b++) acc[a][b] = A[row[a] * ld + col[b]];
#pragma unroll 2
      for (int t = 0; t < PANEL; t++) {
        if (t < nb) {
          T l[4], u[4];
#pragma unroll
          for (int a = 0; a < 4; a++) {
            l[a] = A[row[a] * ld + kb + t];
            u[a] = A[(kb + t) * ld + col[a]];
          }
#pragma unroll
          for (int a = 0; a < 4; a++)
#pragma unroll
            for (int b = 0; b < 4; b++) acc[a][b] = fma(-l[a], u[b], acc[a][b]);
        }
      }
#pragma unroll
      for (int a = 0; a < 4; a++)
#pragma unroll
        for (int b = 0; b < 4; b++)
          if (rok[a] && cok[b]) A[row[a] * ld + col[b]] = acc[a][b];
    }
  }
}

// the panel kb .. kb + nb - 1 on one warp (lane), warp-level syncs only
template <typename T>
__device__ __forceinline__ void panel_warp(T* A, int ld, T* dinv, int kb, int nb, int ns, int lane) {
  const int ke = kb + nb;
  if (lane == 0) dinv[kb] = rcp_rn(A[kb * ld + kb]);
  __syncwarp();
  for (int k = kb; k < ke; k++) {
    const T d = dinv[k];
    T piv[PANEL];
#pragma unroll
    for (int jj = 1; jj < PANEL; jj++) piv[jj] = k + jj < ke ? A[k * ld + k + jj] : T(0);
    for (int i = k + 1 + lane; i < ns; i += 32) {
      T* ai = A + i * ld;
      const T l = ai[k] * d;
      ai[k] = l;
#pragma unroll
      for (int jj = 1; jj < PANEL; jj++)
        if (k + jj < ke) ai[k + jj] = fma(-l, piv[jj], ai[k + jj]);
    }
    // the next pivot is final now and its row is lane 0's (its first row), so lane 0 takes the reciprocal of its own
    // write, after the row loop
    if (lane == 0 && k + 1 < ke) dinv[k + 1] = rcp_rn(A[(k + 1) * ld + k + 1]);
    __syncwarp();
  }
}

// the blocked LU with a lookahead of one panel: while warps 1-3 apply panel p to the columns past panel p + 1, warp 0
// applies it to panel p + 1's columns and factors panel p + 1. Each entry takes its updates in ascending pivot order.
template <int NT, typename T>
__device__ __forceinline__ void lu_factor(const Net& net, T* A, T* dinv, int tid) {
  const int ns = net.ns, ld = net.ld, warp = tid >> 5, lane = tid & 31;
  if (warp == 0) panel_warp(A, ld, dinv, 0, min(PANEL, ns), ns, lane);
  __syncthreads();
  for (int kb = 0; kb < ns; kb += PANEL) {
    const int ke = min(kb + PANEL, ns), nb = ke - kb;
    if (ke == ns) break;
    for (int j = ke + tid; j < ns; j += NT) {  // the block's pivot rows beyond the panel
      T row[PANEL];
#pragma unroll
      for (int s = 0; s < PANEL; s++) row[s] = s < nb ? A[(kb + s) * ld + j] : T(0);
#pragma unroll
      for (int s = 1; s < PANEL; s++) {
        if (s < nb) {
          T a = row[s];
#pragma unroll
          for (int t = 0; t < PANEL; t++)
            if (t < s) a = fma(-A[(kb + s) * ld + kb + t], row[t], a);
          row[s] = a;
          A[(kb + s) * ld + j] = a;
        }
      }
    }
    __syncthreads();
    const int ken = min(ke + PANEL, ns);
    if (warp == 0) {
      for (int i = ke + lane; i < ns; i += 32) {  // panel p + 1's columns, rows ke..
        T* ai = A + i * ld;
        T l[PANEL];
#pragma unroll
        for (int t = 0; t < PANEL; t++) l[t] = t < nb ? ai[kb + t] : T(0);
        for (int j = ke; j < ken; j++) {
          T acc = ai[j];
#pragma unroll
          for (int t = 0; t < PANEL; t++)
            if (t < nb) acc = fma(-l[t], A[(kb + t) * ld + j], acc);
          ai[j] = acc;
        }
      }
      __syncwarp();
      panel_warp(A, ld, dinv, ke, ken - ke, ns, lane);
    } else {
      trailing_update_from<NT - 32, T>(A, ld, kb, nb, ke, ken, ns, tid - 32);
    }
    __syncthreads();
  }
}

// value a[p] for p = idx (R known at compile time: no local memory)
template <int R>
__device__ __forceinline__ double pick(const double (&a)[R], int idx) {
  double v = a[0];
#pragma unroll
  for (int p = 1; p < R; p++)
    if (idx == p) v = a[p];
  return v;
}

// y <- M0^-1 y on one warp for NV vectors (1 or 2) with the factors of lu_factor: lane l holds rows l + 32 p.
// Forward unit L in ascending k, U in descending k with x_k = a_k / U_kk (msolve, common.cuh:504-522). Pivots are
// taken 32 at a time, so the pivot's value comes from a register chosen at compile time (c) and one shuffle; the next
// column of L or U is loaded while the current pivot is applied. A lane whose row takes no update from pivot k uses
// the multiplier 0, and fma(-0, y, a) = a for finite y. Each entry receives the one-pivot sweep's fma's in its order.
// Not inlined: the call kernel solves at four places, and one copy of the code keeps the instruction cache warm.
// The forward and backward sweeps of M0^-1 on NV register-held vectors (a: lane l holds rows l + 32 p; d: 1 / U_kk),
// the body of lu_solve (double) and of the mixed path's solve (float). On return a[v][p] * d[p] is the solution.
template <int R, int NV, typename T>
__device__ __forceinline__ void lu_sweep(const Net& net, const T* A, T (&a)[NV][R], const T (&d)[R], int lane) {
  const int ns = net.ns, ld = net.ld, last = ns - 1;
#pragma unroll
  for (int c = 0; c < R; c++) {  // forward: pivots 32c .. 32c + 31
    const int k0 = 32 * c, k1 = min(k0 + 32, last);
    if (k0 >= k1) break;
    T m[R];
#pragma unroll
    for (int p = c; p < R; p++) m[p] = A[min(lane + 32 * p, last) * ld + k0];
#pragma unroll 2
    for (int k = k0; k < k1; k++) {
      T yk[NV];
#pragma unroll
      for (int v = 0; v < NV; v++) yk[v] = __shfl_sync(FULL, a[v][c], k & 31);
      T mn[R];
#pragma unroll
      for (int p = c; p < R; p++) mn[p] = A[min(lane + 32 * p, last) * ld + min(k + 1, last)];
#pragma unroll
      for (int p = c; p < R; p++) {
        const bool act = (p > c ? true : lane > k - k0) && lane + 32 * p < ns;
        const T mm = act ? m[p] : T(0);
#pragma unroll
        for (int v = 0; v < NV; v++) a[v][p] = fma(-mm, yk[v], a[v][p]);
        m[p] = mn[p];
      }
    }
  }
#pragma unroll
  for (int c = R - 1; c >= 0; c--) {  // backward: pivots 32c + 31 .. 32c (down to 1)
    const int k0 = 32 * c, khi = min(k0 + 31, last), klo = max(k0, 1);
    if (khi < klo) continue;
    T m[R];
#pragma unroll
    for (int p = 0; p <= c; p++) m[p] = A[min(lane + 32 * p, last) * ld + khi];
#pragma unroll 2
    for (int k = khi; k >= klo; k--) {
      T z[NV];
#pragma unroll
      for (int v = 0; v < NV; v++) z[v] = __shfl_sync(FULL, a[v][c] * d[c], k & 31);
      T mn[R];
#pragma unroll
      for (int p = 0; p <= c; p++) mn[p] = A[min(lane + 32 * p, last) * ld + max(k - 1, 0)];
#pragma unroll
      for (int p = 0; p <= c; p++) {
        const bool act = p < c ? true : lane < k - k0;
        const T mm = act ? m[p] : T(0);
#pragma unroll
        for (int v = 0; v < NV; v++) a[v][p] = fma(-mm, z[v], a[v][p]);
        m[p] = mn[p];
      }
    }
  }
}

// y <- M0^-1 y on one warp for NV vectors (1 or 2) with the factors of lu_factor: lane l holds rows l + 32 p.
// Forward unit L in ascending k, U in descending k with x_k = a_k / U_kk (msolve, common.cuh:504-522). Pivots are
// taken 32 at a time, so the pivot's value comes from a register chosen at compile time (c) and one shuffle; the next
// column of L or U is loaded while the current pivot is applied. A lane whose row takes no update from pivot k uses
// the multiplier 0, and fma(-0, y, a) = a for finite y. Each entry receives the one-pivot sweep's fma's in its order.
// Not inlined: the call kernel solves at four places, and one copy of the code keeps the instruction cache warm.
template <int R, int NV>
__device__ __noinline__ void lu_solve(const Net& net, const double* A, const double* dinv, double* y0, double* y1,
                                         int lane) {
  const int ns = net.ns;
  double a[NV][R], d[R];
#pragma unroll
  for (int p = 0; p < R; p++) {
    const int i = lane + 32 * p;
    d[p] = i < ns ? dinv[i] : 0.0;
    a[0][p] = i < ns ? y0[i] : 0.0;
    if (NV == 2) a[NV - 1][p] = i < ns ? y1[i] : 0.0;
  }
  lu_sweep<R, NV, double>(net, A, a, d, lane);
  __syncwarp();
#pragma unroll
  for (int p = 0; p < R; p++) {
    const int i = lane + 32 * p;
    if (i < ns) {
      y0[i] = a[0][p] * d[p];
      if (NV == 2) y1[i] = a[NV - 1][p] * d[p];
    }
  }
  __syncwarp();
}

// y <- y + c0 (sum y) u on one warp (sherman_morrison_update, common.cuh:542-557)
__device__ __forceinline__ void sherman(const Net& net, double* y, const double* u, double c0, int lane) {
  const double s = lane_sum(y, net.ns, lane) * c0;
  for (int i = lane; i < net.ns; i += 32) y[i] = fma(s, u[i], y[i]);
  __syncwarp();
}

// ---- the recovery's dense LU with threshold partial pivoting (recover.cuh:7-82), on one warp ----

__device__ __forceinline__ void dense_lu_pivot(const Net& net, double* A, double* dinv, int* pr, int lane) {
  const int ns = net.ns, ld = net.ld;
  for (int i = lane; i < ns; i += 32) pr[i] = i;
  __syncwarp();
  for (int k = 0; k < ns; k++) {
    double best = -1.0;
    int bi = ns;
    for (int i = k + lane; i < ns; i += 32) {
      const double a = fabs(A[i * ld + k]);
      if (a > best) {
        best = a;
        bi = i;
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double ob = __shfl_xor_sync(FULL, best, o);
      const int oi = __shfl_xor_sync(FULL, bi, o);
      if (ob > best || (ob == best && oi < bi)) {
        best = ob;
        bi = oi;
      }
    }
    const bool exchange = bi != ns && bi != k && !(fabs(A[k * ld + k]) >= MX_PIVTAU * best);
    __syncwarp();
    if (exchange) {
      for (int j = lane; j < ns; j += 32) {
        const double a = A[k * ld + j];
        A[k * ld + j] = A[bi * ld + j];
        A[bi * ld + j] = a;
      }
      if (lane == 0) {
        const int t = pr[k];
        pr[k] = pr[bi];
        pr[bi] = t;
      }
    }
    __syncwarp();
    const double dk = 1.0 / A[k * ld + k];
    if (lane == 0) dinv[k] = dk;
    for (int i = k + 1 + lane; i < ns; i += 32) {
      const double l = A[i * ld + k] * dk;
      A[i * ld + k] = l;
      for (int j = k + 1; j < ns; j++) A[i * ld + j] = fma(-l, A[k * ld + j], A[i * ld + j]);
    }
    __syncwarp();
  }
}

template <int R>
__device__ __forceinline__ void dense_solve(const Net& net, const double* A, const double* dinv, const int* pr, double* y, int lane) {
  const int ns = net.ns, ld = net.ld;
  double a[R], d[R];
#pragma unroll
  for (int p = 0; p < R; p++) {
    const int i = lane + 32 * p;
    a[p] = i < ns ? y[pr[i]] : 0.0;
    d[p] = i < ns ? dinv[i] : 0.0;
  }
  for (int k = 0; k < ns - 1; k++) {
    const double yk = __shfl_sync(FULL, pick<R>(a, k >> 5), k & 31);
#pragma unroll
    for (int p = 0; p < R; p++) {
      const int i = lane + 32 * p;
      if (i > k && i < ns) a[p] = fma(-A[i * ld + k], yk, a[p]);
    }
  }
  for (int k = ns - 1; k > 0; k--) {
    const double z = __shfl_sync(FULL, pick<R>(a, k >> 5) * pick<R>(d, k >> 5), k & 31);
#pragma unroll
    for (int p = 0; p < R; p++) {
      const int i = lane + 32 * p;
      if (i < k) a[p] = fma(-A[i * ld + k], z, a[p]);
    }
  }
  __syncwarp();
#pragma unroll
  for (int p = 0; p < R; p++) {
    const int i = lane + 32 * p;
    if (i < ns) y[i] = a[p] * d[p];
  }
  __syncwarp();
}

// ---- step control (common.cuh:90-133) ----

struct StepState {
  double h, t, nok, pen, pha;
  bool prej;
};

__device__ __forceinline__ double step_factor(double en, bool ok, bool prej, double pen, double pha, double ha) {
  const bool efin = isfinite(en);
  double fac = efin ? MX_STEP_SAFETY / cbrt(fmax(en, MX_ERR_FLOOR)) : MX_FAC_NONFINITE;
  fac = fmin(fmax(fac, ok ? MX_FACACC : MX_FACREJ), MX_FACMAX);
  if (!ok && efin && prej && en > 1.0 && pen > 1.0 && pha > ha) {
    const double pe = log(pen / en) / log(pha / ha);
    fac = pe > MX_SECANT_MIN_ORDER
              ? fmax(pow(MX_SECANT_TARGET / en, 1.0 / fmin(pe, MX_SECANT_MAX_ORDER)), MX_SECMIN)
              : MX_SECMIN;
  }
  if (!ok) fac = fmin(fac, MX_FAC_AFTER_REJECT);
  return fac;
}

// err of a try on warp 0 (try_error, common.cuh:570-590): Y = N + 2 K1 + K3 + K4; writes en and ok to red[0..1].
static __device__ void try_error(const Net& net, const Cell& c, bool first, double rtol, double atol, int lane) {
  double e2 = 0.0, em = 0.0;
  bool nn = true;
  for (int i = lane; i < net.ns; i += 32) {
    const double y = c.N[i] + 2.0 * c.K1[i] + c.K3[i] + c.K4[i];
    c.Y[i] = y;
    const double sc = fma(rtol, fmax(fabs(c.N[i]), fabs(y)), atol);
    const double q = c.K4[i] / sc;
    e2 = fma(q, q, e2);
    em = fmax(em, fabs(q));
    nn = nn && (y >= -atol);
  }
  const double er = sqrt(warp_sum(e2) / net.ns), emx = warp_max(em);
  const double en = (first && isfinite(er)) ? fmax(er, emx) : er;
  const bool ok = (en <= 1.0) && __all_sync(FULL, nn) && isfinite(en);
  if (lane == 0) {
    c.red[0] = en;
    c.red[1] = ok ? 1.0 : 0.0;
  }
}

// ---- the guard's test (guard.cuh:13-108), on one warp ----
// Sums over species are formed as a warp forms them: lane l adds species l, l + 32, ... in order, then the butterfly.
// The small element system (at most MX_MAX_ELEMENTS) is factored by every lane alike from the butterflied sums.

// Doubles of shared scratch the guard needs (guard_scratch): e0 and e1, the element matrix, its first diagonal, the
// right side, lambda, the sum, and g per species.
__host__ __device__ constexpr int guard_scratch(int ns) {
  return 2 * MX_MAX_ELEMENTS + MX_MAX_ELEMENTS * MX_MAX_ELEMENTS + 3 * MX_MAX_ELEMENTS + 2 + ns;
}

// The guard's test of a stepped cell's result xo (network species order) against its input x0, on one warp: the bits
// GUARD_NONFINITE, GUARD_UNFINISHED, GUARD_DRIFT, 0 when it passed (guard.cuh:63-108). A passing result has its element
// shares put back in place (element_multipliers, guard.cuh:24-57): x' = x (1 + sum_e lambda_e a_ie), clamped,
// renormalised. Every sum runs over the species in network order, one lane per sum, as the reference's one thread
// per cell adds them, so each sum has the reference's bits. at: atoms [ns][nel]; scr: guard_scratch(ns) doubles of
// shared memory, free during the guard.
static __device__ __noinline__ int check_cell(const Net& net, const double* x0, double* xo, int done, double nok,
                                       double atol, int lane, const double* at, double* scr) {
  constexpr int ME = MX_MAX_ELEMENTS;
  const int ns = net.ns, nel = net.nel;
  double* se = scr;            // [2 ME]: e0, then e1 at ME
  double* m = se + 2 * ME;     // [ME][ME], upper triangle
  double* m0 = m + ME * ME;    // [ME]
  double* y = m0 + ME;         // [ME]
  double* lam = y + ME;        // [ME]
  double* sum_at = lam + ME;   // [2]
  double* g = sum_at + 2;      // [ns]
  if (lane < 2 * nel) {        // e0[e] on lanes 0..nel-1, e1[e] on lanes nel..2 nel-1 (guard.cuh:70-77)
    const int e = lane < nel ? lane : lane - nel;
    const double* xs = lane < nel ? x0 : xo;
    double acc = 0.0;
    for (int i = 0; i < ns; i++) acc = fma(at[i * nel + e], xs[i], acc);
    se[lane < nel ? e : ME + e] = acc;
  }
  bool fin = true;
  for (int i = lane; i < ns; i += 32) fin = fin && isfinite(xo[i]);
  const bool xfin = __all_sync(FULL, fin);
  __syncwarp();
  double s0 = 0.0, s1 = 0.0;
  for (int e = 0; e < nel; e++) {
    s0 += se[e];
    s1 += se[ME + e];
  }
  bool drift = false;  // shares_drifted (guard.cuh:13-21)
  for (int e = 0; e < nel; e++)
    drift = drift || fabs(se[ME + e] / s1 - se[e] / s0) > net.drift * se[e] / s0 + 2.0 * atol * nok * net.etot / s0;
  const int c = (xfin ? 0 : GUARD_NONFINITE) | (done ? 0 : GUARD_UNFINISHED) | (drift ? GUARD_DRIFT : 0);
  if (c) return c;
  // (A X A^T)[e][f], f >= e: over species with a_ie and a_if both nonzero (guard.cuh:29-37)
  for (int q = lane; q < nel * nel; q += 32) {
    const int e = q / nel, f = q - e * nel;
    if (f >= e) {
      double acc = 0.0;
      for (int i = 0; i < ns; i++) {
        const double ae = at[i * nel + e], af = at[i * nel + f];
        if (ae != 0.0 && af != 0.0) acc = fma(ae * af, xo[i], acc);
      }
      m[e * ME + f] = acc;
    }
  }
  __syncwarp();
  if (lane == 0) {  // LDL^T and the back substitution; an element whose pivot vanishes is left out (guard.cuh:38-56)
    const double r = s1 / s0;
    for (int e = 0; e < nel; e++) {
      m0[e] = m[e * ME + e];
      y[e] = fma(se[e], r, -se[ME + e]);
    }
    for (int k = 0; k < nel; k++) {
      if (!(m[k * ME + k] > MX_ELEMENT_PIVOT_MIN * m0[k])) continue;
      for (int j = k + 1; j < nel; j++) {
        const double l = m[k * ME + j] / m[k * ME + k];
        for (int f = j; f < nel; f++) m[j * ME + f] = fma(-l, m[k * ME + f], m[j * ME + f]);
        y[j] = fma(-l, y[k], y[j]);
      }
    }
    for (int k = nel - 1; k >= 0; k--) {
      lam[k] = 0.0;
      if (!(m[k * ME + k] > MX_ELEMENT_PIVOT_MIN * m0[k])) continue;
      double b = y[k];
      for (int f = k + 1; f < nel; f++) b = fma(-m[k * ME + f], lam[f], b);
      lam[k] = b / m[k * ME + k];
    }
  }
  __syncwarp();
  for (int i = lane; i < ns; i += 32) {  // g per species (guard.cuh:94-99)
    double gi = 1.0;
    for (int e = 0; e < nel; e++) {
      const double a = at[i * nel + e];
      if (a != 0.0) gi = fma(lam[e], a, gi);
    }
    g[i] = fmin(fmax(gi, 1.0 - MX_GMAX), 1.0 + MX_GMAX);
  }
  __syncwarp();
  if (lane == 0) {  // the sum of x g in network order (guard.cuh:100)
    double sum = 0.0;
    for (int i = 0; i < ns; i++) sum = fma(xo[i], g[i], sum);
    sum_at[0] = sum;
  }
  __syncwarp();
  const double sum = sum_at[0];
  for (int i = lane; i < ns; i += 32) xo[i] *= g[i];
  __syncwarp();
  if (!(isfinite(sum) && sum > 0.0)) return GUARD_NONFINITE;
  const double is = 1.0 / sum;
  for (int i = lane; i < ns; i += 32) xo[i] *= is;
  __syncwarp();
  return 0;
}

// The guard's inputs into the matrix's space, free once the steps are done: atoms [ns][nel] and the cell's input row,
// so the guard's species sums read shared memory. Falls back to global memory when they do not fit.
__device__ __forceinline__ void stage_guard_inputs(const Net& net, const Cell& c, const double* x0, int tid, int nt,
                                                   const double** at, const double** xin) {
  const int ns = net.ns, na = ns * net.nel;
  if (na + ns > net.a_doubles) return;
  for (int e = tid; e < na; e += nt) c.A[e] = __ldg(net.atoms + e);
  for (int i = tid; i < ns; i += nt) c.A[na + i] = x0[i];
  *at = c.A;
  *xin = c.A + na;
}

}  // namespace mx
