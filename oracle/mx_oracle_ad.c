/*
 * TEST INFRASTRUCTURE ONLY: the CPU oracle of the call's tangent (the forward-mode derivative of one call, the
 * reference's ADSolver.jvp, maxichem/kincuda_ad.py:325-453, contracts in docs/method.md:185-236). Only tests/ load it,
 * as the oracle of the CUDA tangent; the product never does.
 *
 * Dual numbers (value, tangent) carried through the oracle's own call (mx_oracle.c): every operation of its primal
 * arithmetic, in its order, on the value parts, so the values are the primal oracle's bits, and each operation's
 * derivative rule on the tangent parts. So the tangent is the exact derivative of the computed call, found by a route
 * independent of the CUDA kernel's (which solves the stage tangents with the try's own factors and forms the
 * Jacobian's derivative reaction by reaction).
 *
 * Differentiated inputs (docs/method.md:187-192): x, T, P, dt, the starting step h, per-cell log rate multipliers lm
 * [B][nr] (a multiplier scales both directions of a reaction after the collision limit; a photolysis branch has
 * kf = J e^lm), the nine Arrhenius columns of the rate table and J. Ties follow torch's conventions
 * (docs/method.md:205-207): a tie of min or max of two variables splits the tangent evenly, a maximum over species is
 * shared evenly among those attaining it, d|a| = 0 at 0, and a clamp at a constant bound passes at the bound.
 * Contracts: frozen (adapt 0) holds every try's size fixed (no tangent through dt, h or the error; h_out's tangent 0);
 * adaptive (adapt 1) differentiates the step control too, rejected tries included. A cell that the guard recomputes is
 * differentiated along the recovery's path (dense W, pivoted), retries included; one that still fails has NaN tangents.
 * The guard's element-share correction does not enter the tangent (docs/method.md:169-171).
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
#define GUARD_DRIFT 16

static const double GAMMA = 0.5, C21 = 4.0, C43 = 8.0 / 3.0;
static const double TROE_C0 = 0.4, TROE_C1 = 0.67, TROE_N0 = 0.75, TROE_N1 = 1.27, TROE_D = 0.14;

/* the primal oracle's exported pieces (mx_oracle.c) */
int mxo_screen(const mx_network* net, const double* x0, double Tc, double P, double dt, const double* Jc, double* N);
int mxo_check_cell(const mx_network* net, const double* x0, double* xo, int done, double nok, double atol,
                   double drift);

/* ---- dual numbers ---- */

typedef struct {
  double v, d;
} dn;

static inline dn mk(double v, double d) {
  dn r;
  r.v = v;
  r.d = d;
  return r;
}
static inline dn cst(double v) { return mk(v, 0.0); }
static inline dn add(dn a, dn b) { return mk(a.v + b.v, a.d + b.d); }
static inline dn sub(dn a, dn b) { return mk(a.v - b.v, a.d - b.d); }
static inline dn neg(dn a) { return mk(-a.v, -a.d); }
static inline dn mul(dn a, dn b) { return mk(a.v * b.v, a.d * b.v + a.v * b.d); }
static inline dn dvd(dn a, dn b) {
  const double q = a.v / b.v;
  return mk(q, (a.d - q * b.d) / b.v);
}
static inline dn fmad(dn a, dn b, dn c) { return mk(fma(a.v, b.v, c.v), a.d * b.v + a.v * b.d + c.d); }
static inline dn dexp(dn a) {
  const double e = exp(a.v);
  return mk(e, e * a.d);
}
static inline dn dlog(dn a) { return mk(log(a.v), a.d / a.v); }
static inline dn dlog10(dn a) { return mk(log10(a.v), a.d / (a.v * M_LN10)); }
static inline dn dexp10(dn a) {
  const double e = exp10(a.v);
  return mk(e, e * M_LN10 * a.d);
}
static inline dn dcbrt(dn a) {
  const double c = cbrt(a.v);
  return mk(c, a.d / (3.0 * c * c));
}
static inline dn dpow(dn a, dn b) {
  const double p = pow(a.v, b.v);
  return mk(p, p * (b.d * log(a.v) + b.v * a.d / a.v));
}
static inline dn dabs(dn a) { return mk(fabs(a.v), a.v > 0.0 ? a.d : (a.v < 0.0 ? -a.d : 0.0)); }
/* max and min of two variables: a tie splits the tangent evenly (a NaN side gives way, as fmax's value does) */
static inline dn dmax(dn a, dn b) {
  const double d = isnan(a.v) ? b.d : isnan(b.v) ? a.d : a.v > b.v ? a.d : b.v > a.v ? b.d : 0.5 * (a.d + b.d);
  return mk(fmax(a.v, b.v), d);
}
static inline dn dmin(dn a, dn b) {
  const double d = isnan(a.v) ? b.d : isnan(b.v) ? a.d : a.v < b.v ? a.d : b.v < a.v ? b.d : 0.5 * (a.d + b.d);
  return mk(fmin(a.v, b.v), d);
}
/* a clamp at a constant bound: the tangent passes at the bound */
static inline dn clamp_lo(dn a, double c) { return mk(fmax(a.v, c), a.v >= c ? a.d : 0.0); }
static inline dn clamp_hi(dn a, double c) { return mk(fmin(a.v, c), a.v <= c ? a.d : 0.0); }

/* the warp's sum order (mx_oracle.c lane_sum): lane l adds v[l], v[l + 32], ... then the butterfly */
static dn d_butterfly_sum(dn* p) {
  for (int o = 16; o > 0; o >>= 1) {
    dn q[32];
    for (int l = 0; l < 32; l++) q[l] = add(p[l], p[l ^ o]);
    memcpy(p, q, sizeof q);
  }
  return p[0];
}

static dn d_lane_sum(const dn* v, int n) {
  dn p[32];
  for (int l = 0; l < 32; l++) p[l] = cst(0.0);
  for (int i = 0; i < n; i++) p[i & 31] = add(p[i & 31], v[i]);
  return d_butterfly_sum(p);
}

/* ---- rates (mx_oracle.c law, gibbs, mxo_rates) ---- */

static dn d_arrhenius(const dn* q, dn lT, dn iT) { return dexp(sub(add(q[0], mul(q[1], lT)), mul(q[2], iT))); }

static dn d_law(const dn* q, int fl, dn Tc, dn lT, dn iT, dn nd) {
  dn k = d_arrhenius(q, lT, iT);
  if (fl & FL_SECOND_K0) k = add(k, d_arrhenius(q + 3, lT, iT));
  if (fl & FL_FALLOFF) {
    const dn pr = dvd(mul(k, nd), d_arrhenius(q + 6, lT, iT));
    k = k.v > 0.0 ? dvd(k, add(cst(1.0), pr)) : cst(0.0);
    if ((fl & FL_TROE) && k.v > 0.0) {
      const dn a = mul(sub(cst(1.0), q[9]), dexp(dvd(neg(Tc), q[10])));
      const dn b = mul(q[9], dexp(dvd(neg(Tc), q[11])));
      const dn fc = dlog10(add(add(a, b), dexp(dvd(neg(q[12]), Tc))));
      const dn x = (fl & FL_VM11) ? dlog10(pr) : sub(sub(dlog10(pr), cst(TROE_C0)), mul(cst(TROE_C1), fc));
      dn y;
      if (fl & FL_VM11)
        y = dvd(x, sub(cst(TROE_N0), mul(cst(TROE_N1), fc)));
      else
        y = isfinite(x.v) ? dvd(x, sub(sub(cst(TROE_N0), mul(cst(TROE_N1), fc)), mul(cst(TROE_D), x)))
                          : cst(-1.0 / TROE_D);
      k = mul(k, dexp10(dvd(fc, add(cst(1.0), mul(y, y)))));
    }
  }
  if (fl & FL_EFF) k = mul(k, q[13]);
  return k;
}

static dn d_gibbs(const double* a, dn Tc, dn lT, dn iT) {
  const dn T2 = mul(Tc, Tc), T3 = mul(T2, Tc), T4 = mul(T3, Tc);
  dn h = mul(mul(cst(-a[0]), iT), iT);
  h = add(h, mul(mul(cst(a[1]), lT), iT));
  h = add(h, cst(a[2]));
  h = add(h, dvd(mul(cst(a[3]), Tc), cst(2.0)));
  h = add(h, dvd(mul(cst(a[4]), T2), cst(3.0)));
  h = add(h, dvd(mul(cst(a[5]), T3), cst(4.0)));
  h = add(h, dvd(mul(cst(a[6]), T4), cst(5.0)));
  h = add(h, mul(cst(a[7]), iT));
  dn s = dvd(mul(mul(cst(-a[0]), iT), iT), cst(2.0));
  s = sub(s, mul(cst(a[1]), iT));
  s = add(s, mul(cst(a[2]), lT));
  s = add(s, mul(cst(a[3]), Tc));
  s = add(s, dvd(mul(cst(a[4]), T2), cst(2.0)));
  s = add(s, dvd(mul(cst(a[5]), T3), cst(3.0)));
  s = add(s, dvd(mul(cst(a[6]), T4), cst(4.0)));
  s = add(s, cst(a[8]));
  return sub(h, s);
}

static dn d_bimolecular(int molecules, int three_body, dn k, dn nd) {
  return molecules >= 2 ? mul(k, molecules == 3 ? nd : cst(1.0)) : (three_body ? dvd(k, nd) : cst(0.0));
}

/* kf, kr [nr] of one cell with their tangents; drc: this direction's [nr][9] or NULL; lm, dlm: [nr] or NULL */
static void d_rates(const mx_network* net, dn Tc, dn nd, const double* Jc, const double* dJc, const double* lm,
                    const double* dlm, const double* drc, dn* kf, dn* kr, dn* g) {
  const int ns = net->ns;
  const dn lT = dlog(Tc), iT = dvd(cst(1.0), Tc), lKT = dlog(dvd(mul(cst(MX_KB), Tc), cst(MX_P0)));
  const double* cf = net->nasa + (Tc.v < MX_NASA_SPLIT_T ? 0 : ns * 9);
  for (int i = 0; i < ns; i++) g[i] = d_gibbs(cf + 9 * i, Tc, lT, iT);
  g[ns] = cst(0.0);
  for (int r = 0; r < net->nr; r++) {
    if (r >= net->nrt) {
      const int b = r - net->nrt;
      kf[r] = mk(Jc[b], dJc ? dJc[b] : 0.0);
      kr[r] = cst(0.0);
    } else {
      const int fl = net->rf[r];
      const uint8_t* x = net->rx + 6 * r;
      dn q[14];
      for (int c = 0; c < 14; c++) q[c] = mk(net->rc[14 * r + c], (drc && c < 9) ? drc[9 * r + c] : 0.0);
      const dn k = d_law(q, fl, Tc, lT, iT, nd);
      const dn dg = sub(sub(sub(add(add(g[x[3]], g[x[4]]), g[x[5]]), g[x[0]]), g[x[1]]), g[x[2]]);
      const dn c3 = (fl & FL_THREE_BODY) ? nd : cst(1.0);
      const double dmu = (double)(((fl >> 3) & 7) - 4);
      kf[r] = mul(k, c3);
      kr[r] = mul(mul(k, dexp(add(dg, mul(cst(dmu), lKT)))), c3);
      /* the collision limit (mx_oracle.c collision_limit): both directions times K_COLL / q above it; at q equal to
         K_COLL the limit is a tie and takes half the tangent */
      const int mf = (fl >> 10) & 3, mr = (fl >> 12) & 3, tb = (fl & FL_THREE_BODY) != 0;
      const dn qm = dmax(d_bimolecular(mf, tb, kf[r], nd), d_bimolecular(mr, tb, kr[r], nd));
      if (qm.v > MX_K_COLL) {
        const dn c = dvd(cst(MX_K_COLL), qm);
        kf[r] = mul(kf[r], c);
        kr[r] = mul(kr[r], c);
      } else if (qm.v == MX_K_COLL) {
        const double dlc = -0.5 * qm.d / qm.v;
        kf[r].d += kf[r].v * dlc;
        kr[r].d += kr[r].v * dlc;
      }
    }
    if (lm) {
      const dn e = dexp(mk(lm[r], dlm ? dlm[r] : 0.0));
      kf[r] = mul(kf[r], e);
      kr[r] = mul(kr[r], e);
    } else if (dlm) { /* no multipliers: lm = 0, whose tangent still scales both directions */
      kf[r].d += kf[r].v * dlm[r];
      kr[r].d += kr[r].v * dlm[r];
    }
  }
}

/* ---- right-hand side, Jacobian, LU (mx_oracle.c rhs, jacobian, add_w, lu_factor, lu_solve, sherman) ---- */

typedef struct {
  const mx_network* net;
  int ns, nr;
  dn *k, *n, *v;
} dctx;

static dn d_rhs(const dctx* c, const dn* Y, dn* F, dn* u0, dn nd) {
  const mx_network* net = c->net;
  const int ns = c->ns, nr = c->nr;
  const dn ntot = d_lane_sum(Y, ns), xf = dvd(nd, ntot), ixf = dvd(ntot, nd);
  dn* n = c->n;
  for (int i = 0; i < ns; i++) n[i] = mul(Y[i], xf);
  n[ns] = cst(1.0);
  const dn *kf = c->k, *kr = c->k + nr;
  for (int r = 0; r < nr; r++) {
    const uint8_t* q = net->rx + 6 * r;
    const dn a = mul(mul(mul(kf[r], n[q[0]]), n[q[1]]), n[q[2]]);
    const dn b = mul(mul(mul(kr[r], n[q[3]]), n[q[4]]), n[q[5]]);
    c->v[r] = sub(a, b);
  }
  static const double code[4] = {1.0, -1.0, 2.0, -2.0};
  const int P = net->sv_piece;
  for (int i = 0; i < ns; i++) {
    dn s = cst(0.0);
    const int t0 = net->sv_ptr[i], t1 = net->sv_ptr[i + 1];
    for (int c0 = t0; c0 < t1 || c0 == t0; c0 += P) {
      dn part = cst(0.0);
      for (int t = c0; t < t1 && t < c0 + P; t++) {
        const uint32_t w = net->sv_term[t];
        part = fmad(cst(code[(w >> 16) & 3]), c->v[w & 0xffff], part);
      }
      s = c0 == t0 ? part : add(s, part);
      if (t1 == t0) break;
    }
    F[i] = mul(s, ixf);
    if (u0) u0[i] = dvd(s, nd);
  }
  return ntot;
}

static void d_jacobian(const dctx* c, dn* A) {
  const mx_network* net = c->net;
  const int ns = c->ns;
  static const double code[4] = {1.0, -1.0, 2.0, -2.0};
  for (int i = 0; i < ns * ns; i++) A[i] = cst(0.0);
  for (int e = 0; e < net->n_entries; e++) {
    dn acc = cst(0.0);
    for (int t = net->jac_ptr[e]; t < net->jac_ptr[e + 1]; t++) {
      const uint32_t w = net->jac_term[t];
      const dn pr = mul(mul(c->k[w & 0xfff], c->n[(w >> 16) & 0xff]), c->n[(w >> 24) & 0xff]);
      acc = fmad(cst(code[(w >> 12) & 3]), pr, acc);
    }
    const uint32_t pq = net->jac_entry[e];
    A[(pq >> 16) * ns + (pq & 0xffff)] = neg(acc);
  }
}

static void d_add_w(int ns, const dn* A, const dn* N, dn ntot, dn* u) {
  for (int i = 0; i < ns; i++) {
    dn acc = cst(0.0);
    for (int j = 0; j < ns; j++) acc = fmad(A[i * ns + j], N[j], acc);
    u[i] = add(u[i], dvd(acc, ntot));
  }
}

static void d_lu_factor(int ns, dn* A, dn* dinv) {
  for (int k = 0; k < ns; k++) {
    const dn d = dvd(cst(1.0), A[k * ns + k]);
    dinv[k] = d;
    for (int i = k + 1; i < ns; i++) {
      const dn a = A[i * ns + k];
      if (a.v == 0.0 && a.d == 0.0) continue; /* as the primal's skip, which changes no value bit */
      const dn l = mul(a, d);
      A[i * ns + k] = l;
      dn* ai = A + i * ns;
      const dn* ak = A + k * ns;
      for (int j = k + 1; j < ns; j++) ai[j] = fmad(neg(l), ak[j], ai[j]);
    }
  }
}

static void d_lu_solve(int ns, const dn* A, const dn* dinv, dn* y) {
  for (int k = 0; k < ns - 1; k++) {
    const dn yk = y[k];
    for (int i = k + 1; i < ns; i++) y[i] = fmad(neg(A[i * ns + k]), yk, y[i]);
  }
  for (int k = ns - 1; k > 0; k--) {
    const dn z = mul(y[k], dinv[k]);
    for (int i = 0; i < k; i++) y[i] = fmad(neg(A[i * ns + k]), z, y[i]);
  }
  for (int i = 0; i < ns; i++) y[i] = mul(y[i], dinv[i]);
}

static void d_sherman(int ns, dn* y, const dn* u, dn c0) {
  const dn s = mul(d_lane_sum(y, ns), c0);
  for (int i = 0; i < ns; i++) y[i] = fmad(s, u[i], y[i]);
}

/* the recovery's pivoted LU and solve (mx_oracle.c mxo_dense_lu, mxo_dense_solve): pivots chosen on the values */
static void d_dense_lu(int ns, dn* A, dn* dinv, int* pr) {
  for (int i = 0; i < ns; i++) pr[i] = i;
  for (int k = 0; k < ns; k++) {
    double best = -1.0;
    int b = ns;
    for (int i = k; i < ns; i++) {
      const double a = fabs(A[i * ns + k].v);
      if (a > best) {
        best = a;
        b = i;
      }
    }
    if (b != ns && b != k && !(fabs(A[k * ns + k].v) >= MX_PIVTAU * best)) {
      for (int j = 0; j < ns; j++) {
        const dn a = A[k * ns + j];
        A[k * ns + j] = A[b * ns + j];
        A[b * ns + j] = a;
      }
      const int t = pr[k];
      pr[k] = pr[b];
      pr[b] = t;
    }
    const dn dk = dvd(cst(1.0), A[k * ns + k]);
    dinv[k] = dk;
    for (int i = k + 1; i < ns; i++) {
      const dn l = mul(A[i * ns + k], dk);
      A[i * ns + k] = l;
      for (int j = k + 1; j < ns; j++) A[i * ns + j] = fmad(neg(l), A[k * ns + j], A[i * ns + j]);
    }
  }
}

static void d_dense_solve(int ns, const dn* A, const dn* dinv, const int* pr, dn* y, dn* work) {
  for (int i = 0; i < ns; i++) work[i] = y[pr[i]];
  for (int k = 0; k < ns - 1; k++) {
    const dn yk = work[k];
    for (int i = k + 1; i < ns; i++) work[i] = fmad(neg(A[i * ns + k]), yk, work[i]);
  }
  for (int k = ns - 1; k > 0; k--) {
    const dn z = mul(work[k], dinv[k]);
    for (int i = 0; i < k; i++) work[i] = fmad(neg(A[i * ns + k]), z, work[i]);
  }
  for (int i = 0; i < ns; i++) y[i] = mul(work[i], dinv[i]);
}

/* ---- step control (mx_oracle.c step_factor, try_error) ---- */

typedef struct {
  dn h, t, pen, pha;
  double nok;
  int prej;
} dstep;

static dn d_step_factor(dn en, int ok, int prej, dn pen, dn pha, dn ha) {
  const int efin = isfinite(en.v);
  dn fac = efin ? dvd(cst(MX_STEP_SAFETY), dcbrt(clamp_lo(en, MX_ERR_FLOOR))) : cst(MX_FAC_NONFINITE);
  fac = clamp_hi(clamp_lo(fac, ok ? MX_FACACC : MX_FACREJ), MX_FACMAX);
  if (!ok && efin && prej && en.v > 1.0 && pen.v > 1.0 && pha.v > ha.v) {
    const dn pe = dvd(dlog(dvd(pen, en)), dlog(dvd(pha, ha)));
    fac = pe.v > MX_SECANT_MIN_ORDER
              ? clamp_lo(dpow(dvd(cst(MX_SECANT_TARGET), en), dvd(cst(1.0), clamp_hi(pe, MX_SECANT_MAX_ORDER))),
                         MX_SECMIN)
              : cst(MX_SECMIN);
  }
  if (!ok) fac = clamp_hi(fac, MX_FAC_AFTER_REJECT);
  return fac;
}

static dn d_try_error(int ns, const dn* N, const dn* K1, const dn* K3, const dn* K4, dn* Y, int first, double rtol,
                      double atol, int* ok, dn* q) {
  dn e2[32];
  double em[32];
  int nn = 1;
  for (int l = 0; l < 32; l++) {
    e2[l] = cst(0.0);
    em[l] = 0.0;
  }
  for (int i = 0; i < ns; i++) {
    const dn y = add(add(add(N[i], mul(cst(2.0), K1[i])), K3[i]), K4[i]);
    Y[i] = y;
    const dn sc = fmad(cst(rtol), dmax(dabs(N[i]), dabs(y)), cst(atol));
    q[i] = dvd(K4[i], sc);
    e2[i & 31] = fmad(q[i], q[i], e2[i & 31]);
    em[i & 31] = fmax(em[i & 31], fabs(q[i].v));
    nn = nn && (y.v >= -atol);
  }
  const dn s2 = d_butterfly_sum(e2);
  for (int o = 16; o > 0; o >>= 1) {
    double t[32];
    for (int l = 0; l < 32; l++) t[l] = fmax(em[l], em[l ^ o]);
    memcpy(em, t, sizeof t);
  }
  const double rv = sqrt(s2.v / ns);
  const dn er = mk(rv, rv > 0.0 ? s2.d / (2.0 * ns * rv) : 0.0);
  dn en = er;
  if (first && isfinite(er.v)) {
    /* the maximum over species, its tangent shared evenly among those attaining it */
    const double mv = em[0];
    double sd = 0.0;
    int cnt = 0;
    for (int i = 0; i < ns; i++) {
      const dn a = dabs(q[i]);
      if (a.v == mv) {
        sd += a.d;
        cnt++;
      }
    }
    en = dmax(er, mk(mv, cnt ? sd / cnt : 0.0));
  }
  *ok = (en.v <= 1.0) && nn && isfinite(en.v);
  return en;
}

/* ---- one cell ---- */

typedef struct {
  dn *A, *dinv, *N, *Y, *F, *u, *K1, *K2, *K3, *K4, *k, *n, *v, *g, *w, *q;
  int* pr;
} dws;

static void dws_alloc(dws* w, int ns, int nr) {
  w->A = malloc(sizeof(dn) * ns * ns);
  dn* b = malloc(sizeof(dn) * (size_t)(14 * (ns + 1) + 3 * nr + 4));
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
  w->q = b + 12 * (ns + 1);
  w->k = b + 14 * (ns + 1);
  w->v = w->k + 2 * nr + 2;
  w->pr = malloc(sizeof(int) * (ns + 1));
}

static void dws_free(dws* w) {
  free(w->A);
  free(w->dinv);
  free(w->pr);
}

/* Rodas3 over one call on dual numbers (mx_oracle.c integrate); adapt 0 holds every try's size fixed */
static void d_integrate(const mx_network* net, dws* w, dn nd, dn dt, dstep* s, int max_steps, double rtol, double atol,
                        int dense, int adapt) {
  const int ns = net->ns;
  dctx c = {net, ns, net->nr, w->k, w->n, w->v};
  int it = dt.v > 0.0 ? 0 : max_steps;
  while (it < max_steps && s->t.v < dt.v * MX_CALL_END) {
    dn ha = dmin(s->h, sub(dt, s->t));
    if (!adapt) ha.d = 0.0;
    const dn igh = dvd(cst(1.0), mul(cst(GAMMA), ha)), ih = dvd(cst(1.0), ha);
    const dn ntot = d_rhs(&c, w->N, w->F, w->u, nd);
    d_jacobian(&c, w->A);
    d_add_w(ns, w->A, w->N, ntot, w->u);
    const dn c21h = mul(cst(C21), ih);
    if (dense) {
      for (int i = 0; i < ns; i++)
        for (int j = 0; j < ns; j++) {
          dn* a = w->A + i * ns + j;
          *a = sub(i == j ? add(*a, igh) : *a, w->u[i]);
        }
      for (int i = 0; i < ns; i++) w->K1[i] = w->F[i];
      d_dense_lu(ns, w->A, w->dinv, w->pr);
      d_dense_solve(ns, w->A, w->dinv, w->pr, w->K1, w->w);
      for (int i = 0; i < ns; i++) w->K2[i] = fmad(c21h, w->K1[i], w->F[i]);
      d_dense_solve(ns, w->A, w->dinv, w->pr, w->K2, w->w);
      for (int i = 0; i < ns; i++) w->Y[i] = add(w->N[i], mul(cst(2.0), w->K1[i]));
      d_rhs(&c, w->Y, w->F, NULL, nd);
      for (int i = 0; i < ns; i++) w->K3[i] = fmad(ih, sub(w->K1[i], w->K2[i]), w->F[i]);
      d_dense_solve(ns, w->A, w->dinv, w->pr, w->K3, w->w);
      for (int i = 0; i < ns; i++) w->Y[i] = add(add(w->N[i], mul(cst(2.0), w->K1[i])), w->K3[i]);
      d_rhs(&c, w->Y, w->F, NULL, nd);
      for (int i = 0; i < ns; i++)
        w->K4[i] = fmad(ih, fmad(cst(-C43), w->K3[i], sub(w->K1[i], w->K2[i])), w->F[i]);
      d_dense_solve(ns, w->A, w->dinv, w->pr, w->K4, w->w);
    } else {
      for (int i = 0; i < ns; i++) w->A[i * ns + i] = add(w->A[i * ns + i], igh);
      d_lu_factor(ns, w->A, w->dinv);
      for (int i = 0; i < ns; i++) w->K1[i] = w->F[i];
      d_lu_solve(ns, w->A, w->dinv, w->K1);
      d_lu_solve(ns, w->A, w->dinv, w->u);
      const dn c0 = dvd(cst(1.0), sub(cst(1.0), d_lane_sum(w->u, ns)));
      d_sherman(ns, w->K1, w->u, c0);
      for (int i = 0; i < ns; i++) w->K2[i] = fmad(c21h, w->K1[i], w->F[i]);
      d_lu_solve(ns, w->A, w->dinv, w->K2);
      d_sherman(ns, w->K2, w->u, c0);
      for (int i = 0; i < ns; i++) w->Y[i] = add(w->N[i], mul(cst(2.0), w->K1[i]));
      d_rhs(&c, w->Y, w->F, NULL, nd);
      for (int i = 0; i < ns; i++) w->K3[i] = fmad(ih, sub(w->K1[i], w->K2[i]), w->F[i]);
      d_lu_solve(ns, w->A, w->dinv, w->K3);
      d_sherman(ns, w->K3, w->u, c0);
      for (int i = 0; i < ns; i++) w->Y[i] = add(add(w->N[i], mul(cst(2.0), w->K1[i])), w->K3[i]);
      d_rhs(&c, w->Y, w->F, NULL, nd);
      for (int i = 0; i < ns; i++)
        w->K4[i] = fmad(ih, fmad(cst(-C43), w->K3[i], sub(w->K1[i], w->K2[i])), w->F[i]);
      d_lu_solve(ns, w->A, w->dinv, w->K4);
      d_sherman(ns, w->K4, w->u, c0);
    }
    int ok = 0;
    const dn en = d_try_error(ns, w->N, w->K1, w->K3, w->K4, w->Y, s->t.v == 0.0, rtol, atol, &ok, w->q);
    if (ok) {
      for (int i = 0; i < ns; i++) w->N[i] = clamp_lo(w->Y[i], 0.0);
      s->t = add(s->t, ha);
      s->nok += 1.0;
    }
    const dn fac = d_step_factor(en, ok, s->prej, s->pen, s->pha, ha);
    s->h = mul(ha, fac);
    s->prej = !ok;
    s->pen = en;
    s->pha = ha;
    it++;
  }
}

/* x = N / sum N in network order, with its tangent */
static void d_write_state(int ns, const dn* N, const int32_t* perm, double* out, double* dout) {
  const dn s = d_lane_sum(N, ns);
  for (int i = 0; i < ns; i++) {
    const dn x = dvd(N[i], s);
    out[perm[i]] = x.v;
    if (dout) dout[perm[i]] = x.d;
  }
}

typedef struct {
  const mx_network* net;
  double drift, rtol, atol;
  int max_steps, adapt;
  const double *x, *T, *P, *dt, *h, *J, *lm;
  int64_t B;
  int D;
  const double *dx, *dT, *dP, *ddt, *dh, *dlm, *drc, *dJ;
} jvp_job;

/* One cell along direction d (d < 0: no tangent): the call, guard and recovery of mxo_call on dual numbers. Writes the
   primal results, and the tangents of x and h when d >= 0. Returns the guard's count slot bits in *slots. */
static void d_cell(const jvp_job* j, dws* w, int64_t cell, int d, double* xo, double* ho, int32_t* done,
                   double* steps, int32_t* flag, int32_t* status, double* dxo, double* dho, int32_t* counts) {
  const mx_network* net = j->net;
  const int ns = net->ns, nr = net->nr, nj = net->nj;
  const int64_t B = j->B;
  const int tan = d >= 0;
  const size_t dc = tan ? (size_t)d * (size_t)B + (size_t)cell : 0;
  const double* x0 = j->x + cell * ns;
  const double* Jc = nj ? j->J + cell * nj : NULL;
  const double* lmc = j->lm ? j->lm + cell * nr : NULL;
  const double* dJc = (tan && nj && j->dJ) ? j->dJ + dc * nj : NULL;
  const double* dlmc = (tan && j->dlm) ? j->dlm + dc * nr : NULL;
  const double* drc = (tan && j->drc) ? j->drc + (size_t)d * nr * 9 : NULL;
  const double* dxc = tan ? j->dx + dc * ns : NULL;
  double* nv = malloc(sizeof(double) * (ns + 1));
  const double Tv = j->T[cell], dv = j->dt[cell], hv = j->h[cell];
  const int st = mxo_screen(net, x0, Tv, j->P[cell], dv, Jc, nv);
  free(nv);
  *status = st;
  const dn Tc = mk(Tv, tan ? j->dT[dc] : 0.0), P = mk(j->P[cell], tan ? j->dP[dc] : 0.0);
  const dn dtd = mk(dv, tan ? j->ddt[dc] : 0.0);
  const dn nd = dvd(P, mul(cst(MX_KB), Tc));
  int lm_fine = 1;
  if (lmc)
    for (int r = 0; r < nr; r++) lm_fine = lm_fine && isfinite(lmc[r]);
  if (st == 0) d_rates(net, Tc, nd, Jc, dJc, lmc, dlmc, drc, w->k, w->k + nr, w->g);
  /* a non-finite h acts as dt, with no tangent of its own: the tie min(dt, dt) then passes dt's whole */
  const dn h0 = isfinite(hv) ? mk(hv, tan ? j->dh[dc] : 0.0) : dtd;
  if (!isfinite(hv)) counts[MX_COUNT_NONFINITE_H]++;
  for (int i = 0; i < ns; i++) w->N[i] = mk(x0[net->perm[i]], tan ? dxc[net->perm[i]] : 0.0);
  dstep s = {clamp_lo(dmin(h0, dtd), MX_H_MIN), cst(0.0), cst(0.0), cst(0.0), 0.0, 0};
  if (st == 0 && lm_fine) d_integrate(net, w, nd, dtd, &s, j->max_steps, j->rtol, j->atol, 0, j->adapt);
  d_write_state(ns, w->N, net->perm, xo, dxo);
  *ho = s.h.v;
  if (dho) *dho = j->adapt ? s.h.d : 0.0;
  *done = (st == 0 && s.t.v >= dv * MX_CALL_END) ? 1 : 0;
  *steps = s.nok;
  int r = 0;
  if (st == MX_REFUSED_COLD)
    counts[MX_COUNT_COLD]++;
  else if (st == MX_REFUSED_HOT)
    counts[MX_COUNT_HOT]++;
  else if (st == MX_REFUSED_BAD_INPUT)
    counts[MX_COUNT_BAD_INPUT]++;
  else {
    const int c = mxo_check_cell(net, x0, xo, *done, *steps, j->atol, j->drift);
    if (c & 4) counts[MX_COUNT_NONFINITE]++;
    if (c & 8) counts[MX_COUNT_UNFINISHED]++;
    if (c & 16) counts[MX_COUNT_DRIFT]++;
    if (c) {
      r = 1;
      counts[MX_COUNT_RECOMPUTED]++;
      const dn m = dmin(h0, dtd);
      for (int k = 0;; k++) {
        for (int i = 0; i < ns; i++) w->N[i] = mk(x0[net->perm[i]], tan ? dxc[net->perm[i]] : 0.0);
        const dn start = k == 0 ? m : dmin(m, mul(dtd, cst(pow(MX_REC_RETRY_SPLIT, (double)k))));
        dstep q = {clamp_lo(start, MX_H_MIN), cst(0.0), cst(0.0), cst(0.0), 0.0, 0};
        if (lm_fine)
          d_integrate(net, w, nd, dtd, &q, MX_REC_STEPS * j->max_steps, j->rtol, j->atol, 1, j->adapt);
        d_write_state(ns, w->N, net->perm, xo, dxo);
        const int dn_ = q.t.v >= dv * MX_CALL_END ? 1 : 0;
        const int cc = mxo_check_cell(net, x0, xo, dn_, q.nok, j->atol, j->drift);
        if (cc == GUARD_DRIFT && k < MX_REC_RETRIES) continue;
        *ho = q.h.v;
        if (dho) *dho = j->adapt ? q.h.d : 0.0;
        *done = cc ? 0 : dn_;
        *steps = q.nok;
        r = cc ? 2 : 1;
        counts[cc ? MX_COUNT_STILL_FAILED : MX_COUNT_RECOVERED]++;
        break;
      }
    }
  }
  *flag = r;
  if (r == 2 && dxo) {
    for (int i = 0; i < ns; i++) dxo[i] = NAN;
    *dho = NAN;
  }
}

/*
 * One call with its tangent along D directions, on the CPU (ADSolver.jvp, kincuda_ad.py:325-453). Host arrays:
 * x [B][ns], T, P, dt, h [B], J [B][nj] (NULL when nj == 0), lm [B][nr] or NULL (no multipliers), rc [nr][14] or NULL
 * (the network's table); tangents dx [D][B][ns], dT, dP, ddt, dh [D][B], dlm [D][B][nr], drc [D][nr][9], dJ
 * [D][B][nj] (the last three NULL for zero). Outputs as mxo_call's, and dx_out [D][B][ns], dh_out [D][B]. D may be 0
 * (the primal alone). count [MX_COUNT_SLOTS] is zeroed here. threads <= 0: all OpenMP threads. Returns 0.
 */
int mxo_jvp(const mx_network* net0, double drift, const double* x, const double* T, const double* P, const double* dt,
            const double* h, const double* J, const double* lm, const double* rc, int64_t B, double rtol, double atol,
            int32_t max_steps, int32_t adapt, int32_t D, const double* dx, const double* dT, const double* dP,
            const double* ddt, const double* dh, const double* dlm, const double* drc, const double* dJ,
            double* x_out, double* h_out, int32_t* done, double* steps, int32_t* flag, int32_t* status,
            int32_t* count, double* dx_out, double* dh_out, int threads) {
  mx_network net = *net0;
  if (rc) net.rc = rc;
  const int ns = net.ns;
  memset(count, 0, sizeof(int32_t) * MX_COUNT_SLOTS);
#ifdef _OPENMP
  if (threads > 0) omp_set_num_threads(threads);
#else
  (void)threads;
#endif
  const jvp_job j = {&net, drift, rtol, atol, max_steps, adapt, x, T, P, dt, h, J, lm, B, D,
                     dx, dT, dP, ddt, dh, dlm, drc, dJ};
  int32_t cnt[MX_COUNT_SLOTS] = {0};
#pragma omp parallel
  {
    dws w;
    dws_alloc(&w, ns, net.nr);
    int32_t local[MX_COUNT_SLOTS] = {0};
    double* xs = malloc(sizeof(double) * ns);
#pragma omp for schedule(dynamic, 1)
    for (int64_t cell = 0; cell < B; cell++) {
      /* the primal from the first pass; every pass repeats its values bit for bit */
      int32_t* ct = local;
      int32_t scratch[MX_COUNT_SLOTS];
      for (int d = 0; d < (D > 0 ? D : 1); d++) {
        double hd = 0.0;
        int32_t dn_, fl, stt;
        double sp;
        const int tan = D > 0;
        double* xo = d == 0 ? x_out + cell * ns : xs;
        d_cell(&j, &w, cell, tan ? d : -1, xo, d == 0 ? h_out + cell : &hd, d == 0 ? done + cell : &dn_,
               d == 0 ? steps + cell : &sp, d == 0 ? flag + cell : &fl, d == 0 ? status + cell : &stt,
               tan ? dx_out + ((size_t)d * B + cell) * ns : NULL, tan ? dh_out + (size_t)d * B + cell : NULL, ct);
        memset(scratch, 0, sizeof scratch);
        ct = scratch; /* count the cell once */
      }
    }
    free(xs);
#pragma omp critical
    for (int i = 0; i < MX_COUNT_SLOTS; i++) cnt[i] += local[i];
    dws_free(&w);
  }
  memcpy(count, cnt, sizeof cnt);
  return 0;
}
