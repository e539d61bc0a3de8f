/*
 * TEST INFRASTRUCTURE ONLY: the CPU oracle of the per-call chemistry solve. Only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg may load it, and only as the oracle or the timed CPU baseline; the product never does.
 *
 * A scalar, one-cell-at-a-time restatement of the reference solver's arithmetic (imalsky/maxichem):
 *   rates            maxichem/kernels/common.cuh:136-242 (law, collision_limit, gibbs_rt, rate_pair, cell_rates)
 *   screening        common.cuh:246-279 (screen_x, screen_J, cell_status, cell_fine)
 *   right-hand side  common.cuh:282-353 (reaction_rate, sv_lane, gather_row, rhs)
 *   Jacobian and w   common.cuh:357-402 (jacobian_lane, jacobian_times_x), call.cuh:61-79
 *   LU and solves    common.cuh:405-522 (scale_column, lu_update, factor_trailing, msolve), call.cuh:81-112
 *   Sherman-Morrison common.cuh:526-557
 *   stages, error    common.cuh:560-590, call.cuh:119-158
 *   step control     common.cuh:90-133, call.cuh:47-177
 *   output           common.cuh:592-599
 *   guard            maxichem/kernels/guard.cuh:13-140 (shares_drifted, element_multipliers, check_cell, guard)
 *   recovery         maxichem/kernels/recover.cuh:7-82 (dense_lu, dense_solve), 125-130 (form_dense_w), 197-308
 * Transcendentals are libm's (exp, log, log10, exp10, pow, cbrt); built with -ffp-contract=off, so every fused
 * multiply-add is an explicit fma(). Sums that the CUDA kernel forms across the 32 lanes of a warp (the state's sum,
 * the error norms, the Sherman-Morrison sums, the screening sum) are formed here in the same lane order and butterfly,
 * so the oracle and the kernel differ only by the last bits of the transcendentals.
 */
#define _GNU_SOURCE
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/maxichem_b200.h"

#define FL_FALLOFF 1
#define FL_SECOND_K0 2
#define FL_THREE_BODY 4
#define FL_TROE 64
#define FL_EFF 128
#define FL_VM11 512
#define GUARD_NONFINITE 4
#define GUARD_UNFINISHED 8
#define GUARD_DRIFT 16

static const double GAMMA = 0.5, C21 = 4.0, C43 = 8.0 / 3.0;
static const double TROE_C0 = 0.4, TROE_C1 = 0.67, TROE_N0 = 0.75, TROE_N1 = 1.27, TROE_D = 0.14;

/* The sum a warp forms: lane l adds v[l], v[l + 32], ... in order, then a butterfly over xor 16, 8, 4, 2, 1. */
static double lane_sum(const double* v, int n) {
  double p[32];
  for (int l = 0; l < 32; l++) p[l] = 0.0;
  for (int i = 0; i < n; i++) p[i & 31] += v[i];
  for (int o = 16; o > 0; o >>= 1) {
    double q[32];
    for (int l = 0; l < 32; l++) q[l] = p[l] + p[l ^ o];
    memcpy(p, q, sizeof p);
  }
  return p[0];
}

static double butterfly_sum(double* p) {
  for (int o = 16; o > 0; o >>= 1) {
    double q[32];
    for (int l = 0; l < 32; l++) q[l] = p[l] + p[l ^ o];
    memcpy(p, q, 32 * sizeof(double));
  }
  return p[0];
}

static double butterfly_max(double* p) {
  for (int o = 16; o > 0; o >>= 1) {
    double q[32];
    for (int l = 0; l < 32; l++) q[l] = fmax(p[l], p[l ^ o]);
    memcpy(p, q, 32 * sizeof(double));
  }
  return p[0];
}

/* ---- rates (common.cuh:136-242) ---- */

static double law(const double* q, int fl, double Tc, double lT, double iT, double nd) {
  double k = exp(q[0] + q[1] * lT - q[2] * iT);
  if (fl & FL_SECOND_K0) k += exp(q[3] + q[4] * lT - q[5] * iT);
  if (fl & FL_FALLOFF) {
    const double pr = k * nd / exp(q[6] + q[7] * lT - q[8] * iT);
    k = k > 0.0 ? k / (1.0 + pr) : 0.0;
    if ((fl & FL_TROE) && k > 0.0) {
      const double fc = log10((1.0 - q[9]) * exp(-Tc / q[10]) + q[9] * exp(-Tc / q[11]) + exp(-q[12] / Tc));
      const double x = (fl & FL_VM11) ? log10(pr) : log10(pr) - TROE_C0 - TROE_C1 * fc;
      const double y = (fl & FL_VM11) ? x / (TROE_N0 - TROE_N1 * fc)
                                      : (isfinite(x) ? x / (TROE_N0 - TROE_N1 * fc - TROE_D * x) : -1.0 / TROE_D);
      k *= exp10(fc / (1.0 + y * y));
    }
  }
  if (fl & FL_EFF) k *= q[13];
  return k;
}

static double bimolecular_rate(int molecules, int three_body, double k, double nd) {
  return molecules >= 2 ? k * (molecules == 3 ? nd : 1.0) : (three_body ? k / nd : 0.0);
}

static void collision_limit(int fl, double* kf, double* kr, double nd) {
  const int mf = (fl >> 10) & 3, mr = (fl >> 12) & 3, tb = (fl & FL_THREE_BODY) != 0;
  const double q = fmax(bimolecular_rate(mf, tb, *kf, nd), bimolecular_rate(mr, tb, *kr, nd));
  if (q > MX_K_COLL) {
    const double c = MX_K_COLL / q;
    *kf *= c;
    *kr *= c;
  }
}

static double gibbs(const double* a, double Tc, double lT, double iT) {
  const double T2 = Tc * Tc, T3 = T2 * Tc, T4 = T3 * Tc;
  const double h = -a[0] * iT * iT + a[1] * lT * iT + a[2] + a[3] * Tc / 2 + a[4] * T2 / 3 + a[5] * T3 / 4 +
                   a[6] * T4 / 5 + a[7] * iT;
  const double s = -a[0] * iT * iT / 2 - a[1] * iT + a[2] * lT + a[3] * Tc + a[4] * T2 / 2 + a[5] * T3 / 3 +
                   a[6] * T4 / 4 + a[8];
  return h - s;
}

/* kf, kr [nr] of one cell (common.cuh:222-242); g: [ns + 1] work. */
void mxo_rates(const mx_network* net, double Tc, double nd, const double* Jc, double* kf, double* kr, double* g) {
  const int ns = net->ns;
  const double lT = log(Tc), iT = 1.0 / Tc, lKT = log(MX_KB * Tc / MX_P0);
  const double* cf = net->nasa + (Tc < MX_NASA_SPLIT_T ? 0 : ns * 9);
  for (int i = 0; i < ns; i++) g[i] = gibbs(cf + 9 * i, Tc, lT, iT);
  g[ns] = 0.0;
  for (int r = 0; r < net->nr; r++) {
    if (r >= net->nrt) {
      kf[r] = Jc[r - net->nrt];
      kr[r] = 0.0;
      continue;
    }
    const int fl = net->rf[r];
    const uint8_t* x = net->rx + 6 * r;
    const double k = law(net->rc + 14 * r, fl, Tc, lT, iT, nd);
    const double dg = g[x[3]] + g[x[4]] + g[x[5]] - g[x[0]] - g[x[1]] - g[x[2]];
    const double c3 = (fl & FL_THREE_BODY) ? nd : 1.0;
    const double dmu = (double)(((fl >> 3) & 7) - 4);
    kf[r] = k * c3;
    kr[r] = (k * exp(dg + dmu * lKT)) * c3;
    collision_limit(fl, &kf[r], &kr[r], nd);
  }
}

/* ---- right-hand side, Jacobian (common.cuh:282-402) ---- */

typedef struct {
  const mx_network* net;
  int ns, nr;
  double *k, *n, *v; /* k: kf [nr] then kr [nr] */
} cellctx;

/* F = (ntot / nd) S v(n), u0 = S v / nd (if u0), n = nd Y / ntot; returns ntot. */
static double rhs(const cellctx* c, const double* Y, double* F, double* u0, double nd) {
  const mx_network* net = c->net;
  const int ns = c->ns, nr = c->nr;
  const double ntot = lane_sum(Y, ns), xf = nd / ntot, ixf = ntot / nd;
  double* n = c->n;
  for (int i = 0; i < ns; i++) n[i] = Y[i] * xf;
  n[ns] = 1.0;
  const double *kf = c->k, *kr = c->k + nr;
  for (int r = 0; r < nr; r++) {
    const uint8_t* q = net->rx + 6 * r;
    const double a = kf[r] * n[q[0]] * n[q[1]] * n[q[2]];
    const double b = kr[r] * n[q[3]] * n[q[4]] * n[q[5]];
    c->v[r] = a - b;
  }
  static const double code[4] = {1.0, -1.0, 2.0, -2.0};
  /* row i: its terms in pieces of sv_piece, each summed from 0 in ascending reaction order, the pieces added in order */
  const int P = net->sv_piece;
  for (int i = 0; i < ns; i++) {
    double s = 0.0;
    const int t0 = net->sv_ptr[i], t1 = net->sv_ptr[i + 1];
    for (int c0 = t0; c0 < t1 || c0 == t0; c0 += P) {
      double part = 0.0;
      for (int t = c0; t < t1 && t < c0 + P; t++) {
        const uint32_t w = net->sv_term[t];
        part = fma(code[(w >> 16) & 3], c->v[w & 0xffff], part);
      }
      s = c0 == t0 ? part : s + part;
      if (t1 == t0) break;
    }
    F[i] = s * ixf;
    if (u0) u0[i] = s / nd;
  }
  return ntot;
}

/* A = -Jn, dense [ns][ns] (entries outside the Jacobian's pattern 0). */
static void jacobian(const cellctx* c, double* A) {
  const mx_network* net = c->net;
  const int ns = c->ns;
  static const double code[4] = {1.0, -1.0, 2.0, -2.0};
  memset(A, 0, sizeof(double) * ns * ns);
  for (int e = 0; e < net->n_entries; e++) {
    double acc = 0.0;
    for (int t = net->jac_ptr[e]; t < net->jac_ptr[e + 1]; t++) {
      const uint32_t w = net->jac_term[t];
      const double pr = c->k[w & 0xfff] * c->n[(w >> 16) & 0xff] * c->n[(w >> 24) & 0xff];
      acc = fma(code[(w >> 12) & 3], pr, acc);
    }
    const uint32_t pq = net->jac_entry[e];
    A[(pq >> 16) * ns + (pq & 0xffff)] = -acc;
  }
}

/* u = u0 + (-Jn N) / ntot, row by row in column order (jacobian_times_x). */
static void add_w(int ns, const double* A, const double* N, double ntot, double* u) {
  for (int i = 0; i < ns; i++) {
    double acc = 0.0;
    for (int j = 0; j < ns; j++) acc = fma(A[i * ns + j], N[j], acc);
    u[i] = u[i] + acc / ntot;
  }
}

/* LU without exchanges in place (unit L below the diagonal); dinv = 1 / U_kk. */
static void lu_factor(int ns, double* A, double* dinv) {
  for (int k = 0; k < ns; k++) {
    const double d = 1.0 / A[k * ns + k];
    dinv[k] = d;
    for (int i = k + 1; i < ns; i++) {
      const double a = A[i * ns + k];
      if (a == 0.0) continue; /* l = 0 leaves the row unchanged bit for bit (finite data) */
      const double l = a * d;
      A[i * ns + k] = l;
      double* ai = A + i * ns;
      const double* ak = A + k * ns;
      for (int j = k + 1; j < ns; j++) ai[j] = fma(-l, ak[j], ai[j]);
    }
  }
}

static void lu_solve(int ns, const double* A, const double* dinv, double* y) {
  for (int k = 0; k < ns - 1; k++) {
    const double yk = y[k];
    for (int i = k + 1; i < ns; i++) y[i] = fma(-A[i * ns + k], yk, y[i]);
  }
  for (int k = ns - 1; k > 0; k--) {
    const double z = y[k] * dinv[k];
    for (int i = 0; i < k; i++) y[i] = fma(-A[i * ns + k], z, y[i]);
  }
  for (int i = 0; i < ns; i++) y[i] = y[i] * dinv[i];
}

/* ---- step control (common.cuh:90-133) ---- */

typedef struct {
  double h, t, nok, pen, pha;
  int prej;
} stepstate;

static double step_factor(double en, int ok, int prej, double pen, double pha, double ha) {
  const int efin = isfinite(en);
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

/* err of a try (try_error): RMS of K4 / (atol + rtol max(|N|, |N'|)), and the max-norm while first; Y = N'. */
static double try_error(int ns, const double* N, const double* K1, const double* K3, const double* K4, double* Y,
                        int first, double rtol, double atol, int* ok) {
  double e2[32], em[32];
  int nn = 1;
  for (int l = 0; l < 32; l++) e2[l] = em[l] = 0.0;
  for (int i = 0; i < ns; i++) {
    const double y = N[i] + 2.0 * K1[i] + K3[i] + K4[i];
    Y[i] = y;
    const double sc = fma(rtol, fmax(fabs(N[i]), fabs(y)), atol);
    const double q = K4[i] / sc;
    e2[i & 31] = fma(q, q, e2[i & 31]);
    em[i & 31] = fmax(em[i & 31], fabs(q));
    nn = nn && (y >= -atol);
  }
  const double er = sqrt(butterfly_sum(e2) / ns), emx = butterfly_max(em);
  const double en = (first && isfinite(er)) ? fmax(er, emx) : er;
  *ok = (en <= 1.0) && nn && isfinite(en);
  return en;
}

/* The Sherman-Morrison update of a solved stage: y += c0 (sum y) u. */
static void sherman(int ns, double* y, const double* u, double c0) {
  const double s = lane_sum(y, ns) * c0;
  for (int i = 0; i < ns; i++) y[i] = fma(s, u[i], y[i]);
}

/* ---- guard (guard.cuh:13-108) ----
 * Every sum runs over the species in network order, as the reference's one thread per cell adds them. */

/* check_cell: guard bits of a stepped cell's result; a passing result has its element shares put back in xo. */
int mxo_check_cell(const mx_network* net, const double* x0, double* xo, int done, double nok, double atol,
                   double drift) {
  const int ns = net->ns, nel = net->nel;
  const double* at = net->atoms;
  double e0[MX_MAX_ELEMENTS], e1[MX_MAX_ELEMENTS], lam[MX_MAX_ELEMENTS];
  double etot = 0.0, s0 = 0.0, s1 = 0.0;
  for (int i = 0; i < ns * nel; i++) etot += at[i];
  int xfin = 1;
  for (int e = 0; e < nel; e++) e0[e] = e1[e] = 0.0;
  for (int i = 0; i < ns; i++) { /* guard.cuh:70-77 */
    xfin = xfin && isfinite(xo[i]);
    for (int e = 0; e < nel; e++) {
      e0[e] = fma(at[i * nel + e], x0[i], e0[e]);
      e1[e] = fma(at[i * nel + e], xo[i], e1[e]);
    }
  }
  for (int e = 0; e < nel; e++) {
    s0 += e0[e];
    s1 += e1[e];
  }
  int drifted = 0; /* shares_drifted, guard.cuh:13-21 */
  for (int e = 0; e < nel; e++)
    drifted = drifted || fabs(e1[e] / s1 - e0[e] / s0) > drift * e0[e] / s0 + 2.0 * atol * nok * etot / s0;
  const int c = (xfin ? 0 : GUARD_NONFINITE) | (done ? 0 : GUARD_UNFINISHED) | (drifted ? GUARD_DRIFT : 0);
  if (c) return c;
  /* element_multipliers, guard.cuh:24-57 */
  double m[MX_MAX_ELEMENTS * MX_MAX_ELEMENTS], m0[MX_MAX_ELEMENTS], y[MX_MAX_ELEMENTS];
  for (int e = 0; e < nel * nel; e++) m[e] = 0.0;
  for (int i = 0; i < ns; i++) {
    const double* ai = at + i * nel;
    for (int e = 0; e < nel; e++) {
      if (ai[e] == 0.0) continue;
      for (int f = e; f < nel; f++)
        if (ai[f] != 0.0) m[e * nel + f] = fma(ai[e] * ai[f], xo[i], m[e * nel + f]);
    }
  }
  const double r = s1 / s0;
  for (int e = 0; e < nel; e++) {
    m0[e] = m[e * nel + e];
    y[e] = fma(e0[e], r, -e1[e]);
  }
  for (int k = 0; k < nel; k++) {
    if (!(m[k * nel + k] > MX_ELEMENT_PIVOT_MIN * m0[k])) continue;
    for (int j = k + 1; j < nel; j++) {
      const double l = m[k * nel + j] / m[k * nel + k];
      for (int f = j; f < nel; f++) m[j * nel + f] = fma(-l, m[k * nel + f], m[j * nel + f]);
      y[j] = fma(-l, y[k], y[j]);
    }
  }
  for (int k = nel - 1; k >= 0; k--) {
    lam[k] = 0.0;
    if (!(m[k * nel + k] > MX_ELEMENT_PIVOT_MIN * m0[k])) continue;
    double b = y[k];
    for (int f = k + 1; f < nel; f++) b = fma(-m[k * nel + f], lam[f], b);
    lam[k] = b / m[k * nel + k];
  }
  double sum = 0.0; /* guard.cuh:93-101 */
  for (int i = 0; i < ns; i++) {
    const double* ai = at + i * nel;
    double g = 1.0;
    for (int e = 0; e < nel; e++)
      if (ai[e] != 0.0) g = fma(lam[e], ai[e], g);
    g = fmin(fmax(g, 1.0 - MX_GMAX), 1.0 + MX_GMAX);
    sum = fma(xo[i], g, sum);
    xo[i] *= g;
  }
  if (!(isfinite(sum) && sum > 0.0)) return GUARD_NONFINITE;
  const double is = 1.0 / sum;
  for (int i = 0; i < ns; i++) xo[i] *= is;
  return 0;
}

/* ---- the recovery's dense pivoted factorisation (recover.cuh:7-82) ---- */

void mxo_dense_lu(int ns, double* A, double* dinv, int* pr) {
  for (int i = 0; i < ns; i++) pr[i] = i;
  for (int k = 0; k < ns; k++) {
    double best[32];
    int bi[32];
    for (int l = 0; l < 32; l++) {
      best[l] = -1.0;
      bi[l] = ns;
      for (int i = k + l; i < ns; i += 32) {
        const double a = fabs(A[i * ns + k]);
        if (a > best[l]) {
          best[l] = a;
          bi[l] = i;
        }
      }
    }
    for (int o = 16; o > 0; o >>= 1) {
      double nb[32];
      int ni[32];
      for (int l = 0; l < 32; l++) {
        const double ob = best[l ^ o];
        const int oi = bi[l ^ o];
        nb[l] = best[l];
        ni[l] = bi[l];
        if (ob > best[l] || (ob == best[l] && oi < bi[l])) {
          nb[l] = ob;
          ni[l] = oi;
        }
      }
      memcpy(best, nb, sizeof best);
      memcpy(bi, ni, sizeof bi);
    }
    const int b = bi[0];
    if (b != ns && b != k && !(fabs(A[k * ns + k]) >= MX_PIVTAU * best[0])) {
      for (int j = 0; j < ns; j++) {
        const double a = A[k * ns + j];
        A[k * ns + j] = A[b * ns + j];
        A[b * ns + j] = a;
      }
      const int t = pr[k];
      pr[k] = pr[b];
      pr[b] = t;
    }
    const double dk = 1.0 / A[k * ns + k];
    dinv[k] = dk;
    for (int i = k + 1; i < ns; i++) {
      const double l = A[i * ns + k] * dk;
      A[i * ns + k] = l;
      for (int j = k + 1; j < ns; j++) A[i * ns + j] = fma(-l, A[k * ns + j], A[i * ns + j]);
    }
  }
}

void mxo_dense_solve(int ns, const double* A, const double* dinv, const int* pr, double* y, double* work) {
  for (int i = 0; i < ns; i++) work[i] = y[pr[i]];
  for (int k = 0; k < ns - 1; k++) {
    const double yk = work[k];
    for (int i = k + 1; i < ns; i++) work[i] = fma(-A[i * ns + k], yk, work[i]);
  }
  for (int k = ns - 1; k > 0; k--) {
    const double z = work[k] * dinv[k];
    for (int i = 0; i < k; i++) work[i] = fma(-A[i * ns + k], z, work[i]);
  }
  for (int i = 0; i < ns; i++) y[i] = work[i] * dinv[i];
}

/* ---- one cell ---- */

typedef struct {
  double *A, *dinv, *N, *Y, *F, *u, *K1, *K2, *K3, *K4, *k, *n, *v, *g, *w;
  int* pr;
} workspace;

static void ws_alloc(workspace* w, int ns, int nr) {
  w->A = malloc(sizeof(double) * ns * ns);
  double* b = malloc(sizeof(double) * (size_t)(12 * (ns + 1) + 3 * nr + 4));
  w->dinv = b;
  w->N = b + (ns + 1);
  w->Y = b + 2 * (ns + 1);
  w->F = b + 3 * (ns + 1);
  w->u = b + 4 * (ns + 1);
  w->K1 = b + 5 * (ns + 1);
  w->K2 = b + 6 * (ns + 1);
  w->K3 = b + 7 * (ns + 1);
  w->K4 = b + 8 * (ns + 1);
  w->n = b + 9 * (ns + 1);
  w->g = b + 10 * (ns + 1);
  w->w = b + 11 * (ns + 1);
  w->k = b + 12 * (ns + 1);
  w->v = w->k + 2 * nr;
  w->pr = malloc(sizeof(int) * (ns + 1));
}

static void ws_free(workspace* w) {
  free(w->A);
  free(w->dinv);
  free(w->pr);
}

/* Rodas3 over one call; dense: the recovery's form (W dense and pivoted), else the call kernel's. */
static void integrate(const mx_network* net, workspace* w, double nd, double dt, stepstate* s, int max_steps,
                      double rtol, double atol, int dense) {
  const int ns = net->ns;
  cellctx c = {net, ns, net->nr, w->k, w->n, w->v};
  int it = dt > 0.0 ? 0 : max_steps;
  while (it < max_steps && s->t < dt * MX_CALL_END) {
    const double ha = fmin(s->h, dt - s->t), igh = 1.0 / (GAMMA * ha), ih = 1.0 / ha;
    /* a retry after a rejection starts from the same state, so F, u and -Jn recomputed here are those of the
       rejected try bit for bit (the reference restores a saved copy) */
    const double ntot = rhs(&c, w->N, w->F, w->u, nd);
    jacobian(&c, w->A);
    add_w(ns, w->A, w->N, ntot, w->u);
    if (dense) {
      for (int i = 0; i < ns; i++)
        for (int j = 0; j < ns; j++) {
          double* a = w->A + i * ns + j;
          *a = (i == j ? *a + igh : *a) - w->u[i];
        }
      for (int i = 0; i < ns; i++) w->K1[i] = w->F[i];
      mxo_dense_lu(ns, w->A, w->dinv, w->pr);
      mxo_dense_solve(ns, w->A, w->dinv, w->pr, w->K1, w->w);
      for (int i = 0; i < ns; i++) w->K2[i] = fma(C21 * ih, w->K1[i], w->F[i]);
      mxo_dense_solve(ns, w->A, w->dinv, w->pr, w->K2, w->w);
      for (int i = 0; i < ns; i++) w->Y[i] = w->N[i] + 2.0 * w->K1[i];
      rhs(&c, w->Y, w->F, NULL, nd);
      for (int i = 0; i < ns; i++) w->K3[i] = fma(ih, w->K1[i] - w->K2[i], w->F[i]);
      mxo_dense_solve(ns, w->A, w->dinv, w->pr, w->K3, w->w);
      for (int i = 0; i < ns; i++) w->Y[i] = w->N[i] + 2.0 * w->K1[i] + w->K3[i];
      rhs(&c, w->Y, w->F, NULL, nd);
      for (int i = 0; i < ns; i++) w->K4[i] = fma(ih, fma(-C43, w->K3[i], w->K1[i] - w->K2[i]), w->F[i]);
      mxo_dense_solve(ns, w->A, w->dinv, w->pr, w->K4, w->w);
    } else {
      for (int i = 0; i < ns; i++) w->A[i * ns + i] += igh;
      lu_factor(ns, w->A, w->dinv);
      for (int i = 0; i < ns; i++) w->K1[i] = w->F[i];
      lu_solve(ns, w->A, w->dinv, w->K1);
      lu_solve(ns, w->A, w->dinv, w->u);
      const double c0 = 1.0 / (1.0 - lane_sum(w->u, ns));
      sherman(ns, w->K1, w->u, c0);
      for (int i = 0; i < ns; i++) w->K2[i] = fma(C21 * ih, w->K1[i], w->F[i]);
      lu_solve(ns, w->A, w->dinv, w->K2);
      sherman(ns, w->K2, w->u, c0);
      for (int i = 0; i < ns; i++) w->Y[i] = w->N[i] + 2.0 * w->K1[i];
      rhs(&c, w->Y, w->F, NULL, nd);
      for (int i = 0; i < ns; i++) w->K3[i] = fma(ih, w->K1[i] - w->K2[i], w->F[i]);
      lu_solve(ns, w->A, w->dinv, w->K3);
      sherman(ns, w->K3, w->u, c0);
      for (int i = 0; i < ns; i++) w->Y[i] = w->N[i] + 2.0 * w->K1[i] + w->K3[i];
      rhs(&c, w->Y, w->F, NULL, nd);
      for (int i = 0; i < ns; i++) w->K4[i] = fma(ih, fma(-C43, w->K3[i], w->K1[i] - w->K2[i]), w->F[i]);
      lu_solve(ns, w->A, w->dinv, w->K4);
      sherman(ns, w->K4, w->u, c0);
    }
    int ok = 0;
    const double en = try_error(ns, w->N, w->K1, w->K3, w->K4, w->Y, s->t == 0.0, rtol, atol, &ok);
    if (ok) {
      for (int i = 0; i < ns; i++) w->N[i] = fmax(w->Y[i], 0.0);
      s->t += ha;
      s->nok += 1.0;
    }
    const double fac = step_factor(en, ok, s->prej, s->pen, s->pha, ha);
    s->h = ha * fac;
    s->prej = !ok;
    s->pen = en;
    s->pha = ha;
    it++;
  }
}

static void write_state(int ns, const double* N, const int32_t* perm, double* out) {
  const double s = lane_sum(N, ns);
  for (int i = 0; i < ns; i++) out[perm[i]] = N[i] / s;
}

/* Screening of one cell (common.cuh:246-279, call.cuh:36-43): its status, and N = x0 in elimination order. */
int mxo_screen(const mx_network* net, const double* x0, double Tc, double P, double dt, const double* Jc, double* N) {
  const int ns = net->ns;
  double p[32], pm[32];
  for (int l = 0; l < 32; l++) p[l] = pm[l] = 0.0;
  for (int i = 0; i < ns; i++) {
    N[i] = x0[net->perm[i]];
    p[i & 31] += N[i] >= 0.0 ? N[i] : NAN;
    pm[i & 31] = fmax(pm[i & 31], N[i]);
  }
  for (int b = 0; b < net->nj; b++) p[b & 31] += Jc[b] >= 0.0 ? 0.0 * Jc[b] : NAN;
  const double ps = butterfly_sum(p), mx = butterfly_max(pm);
  const double nd = P / (MX_KB * Tc);
  const int forcing = isfinite(Tc) && isfinite(nd) && nd > 0.0 && isfinite(dt) && dt >= 0.0;
  const int fine = fabs(ps - 1.0) <= MX_X_SUM_TOL && mx > 0.0 && forcing;
  return Tc < MX_T_MIN ? MX_REFUSED_COLD : (Tc > MX_T_MAX ? MX_REFUSED_HOT : (fine ? 0 : MX_REFUSED_BAD_INPUT));
}

/*
 * One whole call on the CPU (CudaSolver.launch's call, guard and recovery). Host arrays; count [MX_COUNT_SLOTS] is
 * zeroed here. threads <= 0: all OpenMP threads. Returns 0.
 */
int mxo_call(const mx_network* net, double drift, const double* x, const double* T, const double* P,
             const double* dt, const double* h_in, const double* J, int64_t B, double rtol, double atol,
             int32_t max_steps, double* x_out, double* h_out, int32_t* done, double* steps, int32_t* flag,
             int32_t* status, int32_t* count, int threads) {
  const int ns = net->ns;
  memset(count, 0, sizeof(int32_t) * MX_COUNT_SLOTS);
#ifdef _OPENMP
  if (threads > 0) omp_set_num_threads(threads);
#else
  (void)threads;
#endif
  int32_t cnt[MX_COUNT_SLOTS] = {0};
#pragma omp parallel
  {
    workspace w;
    ws_alloc(&w, ns, net->nr);
    int32_t local[MX_COUNT_SLOTS] = {0};
#pragma omp for schedule(dynamic, 4)
    for (int64_t cell = 0; cell < B; cell++) {
      const double Tc = T[cell], d = dt[cell], nd = P[cell] / (MX_KB * Tc);
      const double* Jc = net->nj ? J + cell * net->nj : NULL;
      const int st = mxo_screen(net, x + cell * ns, Tc, P[cell], d, Jc, w.N);
      status[cell] = st;
      if (st == 0) mxo_rates(net, Tc, nd, Jc, w.k, w.k + net->nr, w.g);
      const double h0 = isfinite(h_in[cell]) ? h_in[cell] : d;
      if (!isfinite(h_in[cell])) local[MX_COUNT_NONFINITE_H]++;
      stepstate s = {fmax(fmin(h0, d), MX_H_MIN), 0.0, 0.0, 0.0, 0.0, 0};
      if (st == 0) integrate(net, &w, nd, d, &s, max_steps, rtol, atol, 0);
      double* xo = x_out + cell * ns;
      write_state(ns, w.N, net->perm, xo);
      h_out[cell] = s.h;
      done[cell] = (st == 0 && s.t >= d * MX_CALL_END) ? 1 : 0;
      steps[cell] = s.nok;
      /* guard (guard.cuh:114-140) */
      int r = 0;
      if (st == MX_REFUSED_COLD)
        local[MX_COUNT_COLD]++;
      else if (st == MX_REFUSED_HOT)
        local[MX_COUNT_HOT]++;
      else if (st == MX_REFUSED_BAD_INPUT)
        local[MX_COUNT_BAD_INPUT]++;
      else {
        const int c = mxo_check_cell(net, x + cell * ns, xo, done[cell], steps[cell], atol, drift);
        if (c & GUARD_NONFINITE) local[MX_COUNT_NONFINITE]++;
        if (c & GUARD_UNFINISHED) local[MX_COUNT_UNFINISHED]++;
        if (c & GUARD_DRIFT) local[MX_COUNT_DRIFT]++;
        if (c) {
          r = 1;
          local[MX_COUNT_RECOMPUTED]++;
          /* recovery (recover.cuh:261-308): from the inputs, dense pivoted W, REC_STEPS times the tries */
          mxo_rates(net, Tc, nd, Jc, w.k, w.k + net->nr, w.g);
          const double m = fmin(h0, d);
          for (int k = 0;; k++) {
            for (int i = 0; i < ns; i++) w.N[i] = x[cell * ns + net->perm[i]];
            const double start = k == 0 ? m : fmin(m, d * pow(MX_REC_RETRY_SPLIT, (double)k));
            stepstate q = {fmax(start, MX_H_MIN), 0.0, 0.0, 0.0, 0.0, 0};
            integrate(net, &w, nd, d, &q, MX_REC_STEPS * max_steps, rtol, atol, 1);
            write_state(ns, w.N, net->perm, xo);
            const int dn = q.t >= d * MX_CALL_END ? 1 : 0;
            const int cc = mxo_check_cell(net, x + cell * ns, xo, dn, q.nok, atol, drift);
            if (cc == GUARD_DRIFT && k < MX_REC_RETRIES) continue;
            h_out[cell] = q.h;
            done[cell] = cc ? 0 : dn;
            steps[cell] = q.nok;
            r = cc ? 2 : 1;
            local[cc ? MX_COUNT_STILL_FAILED : MX_COUNT_RECOVERED]++;
            break;
          }
        }
      }
      flag[cell] = r;
    }
#pragma omp critical
    for (int i = 0; i < MX_COUNT_SLOTS; i++) cnt[i] += local[i];
    ws_free(&w);
  }
  memcpy(count, cnt, sizeof cnt);
  return 0;
}

/* Building blocks for the tests: one cell's F and u0 at Y, and its -Jn (dense [ns][ns]). */
double mxo_rhs_jacobian(const mx_network* net, const double* kf_kr, const double* Y, double nd, double* F, double* u0,
                        double* A) {
  const int ns = net->ns;
  double* n = malloc(sizeof(double) * (ns + 1));
  double* v = malloc(sizeof(double) * net->nr);
  cellctx c = {net, ns, net->nr, (double*)kf_kr, n, v};
  const double ntot = rhs(&c, Y, F, u0, nd);
  if (A) jacobian(&c, A);
  free(n);
  free(v);
  return ntot;
}

/* One fresh try of one cell with every stage written out, in the layout of the library's mx_debug_try. */
void mxo_debug_try(const mx_network* net, const double* x0, double Tc, double P, double ha, const double* Jc,
                   double rtol, double atol, double* out) {
  const int ns = net->ns, nr = net->nr;
  workspace w;
  ws_alloc(&w, ns, nr);
  cellctx c = {net, ns, nr, w.k, w.n, w.v};
  const double nd = P / (MX_KB * Tc);
  for (int i = 0; i < ns; i++) w.N[i] = x0[net->perm[i]];
  mxo_rates(net, Tc, nd, Jc, w.k, w.k + nr, w.g);
  double* o = out;
  memcpy(o, w.k, sizeof(double) * 2 * nr);
  o += 2 * nr;
  const double igh = 1.0 / (GAMMA * ha), ih = 1.0 / ha;
  const double ntot = rhs(&c, w.N, w.F, w.u, nd);
  memcpy(o, w.F, sizeof(double) * ns);
  memcpy(o + ns, w.u, sizeof(double) * ns);
  o += 2 * ns;
  jacobian(&c, w.A);
  memcpy(o, w.A, sizeof(double) * ns * ns);
  o += ns * ns;
  add_w(ns, w.A, w.N, ntot, w.u);
  memcpy(o, w.u, sizeof(double) * ns);
  o += ns;
  for (int i = 0; i < ns; i++) w.A[i * ns + i] += igh;
  lu_factor(ns, w.A, w.dinv);
  memcpy(o, w.A, sizeof(double) * ns * ns);
  o += ns * ns;
  memcpy(o, w.dinv, sizeof(double) * ns);
  o += ns;
  for (int i = 0; i < ns; i++) w.K1[i] = w.F[i];
  lu_solve(ns, w.A, w.dinv, w.K1);
  lu_solve(ns, w.A, w.dinv, w.u);
  const double c0 = 1.0 / (1.0 - lane_sum(w.u, ns));
  sherman(ns, w.K1, w.u, c0);
  for (int i = 0; i < ns; i++) w.K2[i] = fma(C21 * ih, w.K1[i], w.F[i]);
  lu_solve(ns, w.A, w.dinv, w.K2);
  sherman(ns, w.K2, w.u, c0);
  for (int i = 0; i < ns; i++) w.Y[i] = w.N[i] + 2.0 * w.K1[i];
  rhs(&c, w.Y, w.F, NULL, nd);
  for (int i = 0; i < ns; i++) w.K3[i] = fma(ih, w.K1[i] - w.K2[i], w.F[i]);
  lu_solve(ns, w.A, w.dinv, w.K3);
  sherman(ns, w.K3, w.u, c0);
  for (int i = 0; i < ns; i++) w.Y[i] = w.N[i] + 2.0 * w.K1[i] + w.K3[i];
  rhs(&c, w.Y, w.F, NULL, nd);
  for (int i = 0; i < ns; i++) w.K4[i] = fma(ih, fma(-C43, w.K3[i], w.K1[i] - w.K2[i]), w.F[i]);
  lu_solve(ns, w.A, w.dinv, w.K4);
  sherman(ns, w.K4, w.u, c0);
  int ok = 0;
  const double en = try_error(ns, w.N, w.K1, w.K3, w.K4, w.Y, 1, rtol, atol, &ok);
  memcpy(o, w.K1, sizeof(double) * ns);
  memcpy(o + ns, w.K2, sizeof(double) * ns);
  memcpy(o + 2 * ns, w.K3, sizeof(double) * ns);
  memcpy(o + 3 * ns, w.K4, sizeof(double) * ns);
  memcpy(o + 4 * ns, w.Y, sizeof(double) * ns);
  o += 5 * ns;
  o[0] = en;
  o[1] = ok;
  ws_free(&w);
}

int mxo_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
