// The tangent of one call (the reference's ADSolver.jvp, maxichem/kincuda_ad.py:325-453; its kernels
// maxichem/kernels/jvp.cuh, ad_common.cuh), on the B200: the call kernel's own device functions step each cell, so the
// primal is the call's bit for bit, and after each try the stage tangents of every direction are solved with the
// try's own factors.
//
// For a direction with tangents of N, the rates (k_dot) and n_tot, each try's stage tangents solve
//   W K_i' = b_i' + (h' / (gamma h^2)) K_i + J_N' K_i,   J_N' K = Jn' K + u' (sum K)
// with W^-1 in the call's form (M0^-1 and Sherman-Morrison; the recovery's dense pivoted W^-1 for recovered cells).
// Jn' K, the Jacobian's derivative along the direction applied to K, comes reaction by reaction from hyper-dual
// products of the reaction's concentrations: for one side with values a_m, the first product sum_m e_m prod_{l!=m} a_l
// and the second sum_{m!=l} e_m f_l prod_{others} a. The rate tangents (Arrhenius, falloff with its Troe factor,
// three-body, NASA-9 reverse, the collision limit's weights, docs/method.md:195-202 of the reference) are formed once
// per cell and direction. Contracts (docs/method.md:209-217): frozen holds every accepted try's size fixed and skips
// rejected tries; adaptive differentiates the step size through the step control, rejected tries included. Ties of
// min and max split the tangent evenly; a clamp at a constant bound passes it; d|a| = 0 at 0.
#pragma once
#include "device.cuh"

namespace mx {

constexpr double LN10 = 2.302585092994045684;

// The tangent inputs and outputs of one mx_jvp call (device pointers; lm, dlm, drc, dJ may be null).
struct TanArgs {
  const double *lm, *dx, *dT, *dP, *ddt, *dh, *dlm, *drc, *dJ;
  int D, adapt;
  double *dx_out, *dh_out;
  double* scratch;  // per CTA: [D][2 nr + 2] rate tangents, [D][ns + 1] state tangents, [D][4] step tangents
  long long slot;   // doubles per CTA
};

// Shared-memory offsets (doubles) of the tangent's vectors, past the call's own layout.
struct TanLayout {
  int oTN, oTn, oTF, oTu, oJK, oTK, oTY, oZ, doubles, stride;  // oJK, oTK: 4 vectors each, `stride` apart
};

struct TanCell {
  double *tN, *tn, *tF, *tu, *tY, *z;
  double* JK[4];
  double* tK[4];
};

__device__ __forceinline__ TanCell tan_arrays(const TanLayout& l, double* smem) {
  TanCell t;
  t.tN = smem + l.oTN;
  t.tn = smem + l.oTn;
  t.tF = smem + l.oTF;
  t.tu = smem + l.oTu;
  t.tY = smem + l.oTY;
  t.z = smem + l.oZ;
#pragma unroll
  for (int k = 0; k < 4; k++) {
    t.JK[k] = smem + l.oJK + k * l.stride;
    t.tK[k] = smem + l.oTK + k * l.stride;
  }
  return t;
}

// per-CTA scratch regions of direction d
__device__ __forceinline__ double* rate_tangent(const Net& net, const TanArgs& ta, double* sl, int d) {
  return sl + (size_t)d * (2 * net.nr + 2);
}
__device__ __forceinline__ double* state_tangent(const Net& net, const TanArgs& ta, double* sl, int d) {
  return sl + (size_t)ta.D * (2 * net.nr + 2) + (size_t)d * (net.ns + 1);
}
__device__ __forceinline__ double* step_tangent(const Net& net, const TanArgs& ta, double* sl, int d) {
  return sl + (size_t)ta.D * (2 * net.nr + 2 + net.ns + 1) + 4 * d;
}

// ---- the rate tangents ----

// d ln k of the law (law in device.cuh) by parts: per unit dT at fixed n_tot (aT), per unit d ln n_tot (aN), and per
// unit change of the exponents ln A + B ln T - C / T of k0's two terms and of k_inf (a1, a2, ainf).
struct LawParts {
  double aT, aN, a1, a2, ainf;
};

__device__ __forceinline__ LawParts law_parts(const double* __restrict__ q, int fl, double Tc, double lT, double iT,
                                              double nd) {
  LawParts p = {0.0, 0.0, 0.0, 0.0, 0.0};
  const double k1 = exp(q[0] + q[1] * lT - q[2] * iT);
  const double k2 = (fl & FL_SECOND_K0) ? exp(q[3] + q[4] * lT - q[5] * iT) : 0.0;
  const double k0 = k1 + k2;
  if (!(k0 > 0.0) || !isfinite(k0)) return p;
  const double iT2 = iT * iT, w1 = k1 / k0, w2 = k2 / k0;
  const double g0 = w1 * (q[1] * iT + q[2] * iT2) + w2 * ((fl & FL_SECOND_K0) ? q[4] * iT + q[5] * iT2 : 0.0);
  // d ln k = ak0 d ln k0 + aN d ln nd + ainf d ln k_inf + fT dT; ak0 = 1 / (1 + pr) + dFl, aN = -pr / (1 + pr) + dFl,
  // ainf = -aN, with dFl the Troe factor's d ln F / d ln pr: 1 / (1 + pr) is formed directly, not as
  // 1 - pr / (1 + pr), which would cancel deep in the high-pressure limit
  double ak0 = 1.0, aN = 0.0, ginf = 0.0, fT = 0.0;
  if (fl & FL_FALLOFF) {
    const double pr = k0 * nd / exp(q[6] + q[7] * lT - q[8] * iT);
    ginf = q[7] * iT + q[8] * iT2;
    if (!(pr < INFINITY)) return p;  // k_inf = 0: k is the high-pressure rate 0
    ak0 = 1.0 / (1.0 + pr);
    aN = -pr / (1.0 + pr);
    if (fl & FL_TROE) {
      const double al = q[9], e3 = exp(-Tc / q[10]), e1 = exp(-Tc / q[11]), e2 = exp(-q[12] / Tc);
      const double Fc = (1.0 - al) * e3 + al * e1 + e2;
      const double fc = log10(Fc);
      const double dfc = (-(1.0 - al) / q[10] * e3 - al / q[11] * e1 + q[12] * iT2 * e2) / (Fc * LN10);
      const double lp = log10(pr);
      double y, dy_lp = 0.0, dy_fc = 0.0;
      if (fl & FL_VM11) {
        const double den = TROE_N0 - TROE_N1 * fc;
        y = lp / den;
        dy_lp = 1.0 / den;
        dy_fc = lp * TROE_N1 / (den * den);
      } else {
        const double x = lp - TROE_C0 - TROE_C1 * fc;
        if (isfinite(x)) {
          const double den = TROE_N0 - TROE_N1 * fc - TROE_D * x;
          y = x / den;
          dy_lp = (TROE_N0 - TROE_N1 * fc) / (den * den);
          dy_fc = (-TROE_C1 * den - x * (TROE_D * TROE_C1 - TROE_N1)) / (den * den);
        } else {
          y = -1.0 / TROE_D;
        }
      }
      if (isfinite(y)) {
        const double u = 1.0 + y * y, dF_dy = -2.0 * fc * y / (u * u);  // d log10 F / dy
        const double dFl = dF_dy * dy_lp;
        ak0 += dFl;
        aN += dFl;
        fT = LN10 * (1.0 / u + dF_dy * dy_fc) * dfc;
      }  // else log10 F = fc / (1 + y^2) is 0, flat in pr and T
    }
  }
  p.aT = ak0 * g0 - aN * ginf + fT;
  p.aN = aN;
  p.a1 = ak0 * w1;
  p.a2 = ak0 * w2;
  p.ainf = -aN;
  return p;
}

// d (G / RT) / dT of one species (gibbs_rt's derivative)
__device__ __forceinline__ double gibbs_rt_dT(const double* __restrict__ a, double Tc, double lT, double iT) {
  const double iT2 = iT * iT, iT3 = iT2 * iT, T2 = Tc * Tc, T3 = T2 * Tc;
  const double dh = 2.0 * a[0] * iT3 + a[1] * (1.0 - lT) * iT2 + a[3] / 2 + 2.0 * a[4] * Tc / 3 + 3.0 * a[5] * T2 / 4 +
                    4.0 * a[6] * T3 / 5 - a[7] * iT2;
  const double ds = a[0] * iT3 + a[1] * iT2 + a[2] * iT + a[3] + a[4] * Tc + a[5] * T2 + a[6] * T3;
  return dh - ds;
}

// k_dot of every reaction and direction of one cell into the CTA's scratch. c.kf, c.kr hold the cell's rates (after
// the log multipliers); g and dg (ns + 1 doubles each) are shared scratch. Two barriers.
__device__ void rate_tangents(const Net& net, const Cell& c, const TanArgs& ta, double* sl, int cell, int B, double Tc,
                              double P, double nd, const double* __restrict__ Jc, double* g, double* dg, int tid,
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
  for (int r = tid; r < nr; r += nt) {
    const double kf = c.kf[r], kr = c.kr[r];
    if (r >= net.nrt) {  // photolysis: kf = J e^lm, its tangent J_dot e^lm + kf lm_dot
      const int b = r - net.nrt;
      const double em = ta.lm ? exp(ta.lm[(size_t)cell * nr + r]) : 1.0;
      for (int d = 0; d < ta.D; d++) {
        const size_t dc = (size_t)d * B + cell;
        double dk = ta.dJ ? ta.dJ[dc * net.nj + b] * em : 0.0;
        if (ta.dlm) dk = fma(kf, ta.dlm[dc * nr + r], dk);
        double* kd = rate_tangent(net, ta, sl, d);
        kd[r] = dk;
        kd[nr + r] = 0.0;
      }
      continue;
    }
    const int fl = __ldg(net.rf + r);
    const uint64_t w = __ldg(net.rx8 + r);
    const int x0 = w & 255, x1 = (w >> 8) & 255, x2 = (w >> 16) & 255;
    const int x3 = (w >> 24) & 255, x4 = (w >> 32) & 255, x5 = (w >> 40) & 255;
    const double* q = net.rc + 14 * r;
    const LawParts lp = law_parts(q, fl, Tc, lT, iT, nd);
    // the primal's limit decision, from the same arithmetic as cell_rates
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
    const double gT = dg[x3] + dg[x4] + dg[x5] - dg[x0] - dg[x1] - dg[x2] + dmu * iT;  // d (ln kr - ln kf) / dT
    for (int d = 0; d < ta.D; d++) {
      const size_t dc = (size_t)d * B + cell;
      const double dT = ta.dT[dc], rho = ta.dP[dc] / P - dT / Tc;  // d ln n_tot
      double dA = fma(lp.aT, dT, (lp.aN + (tb ? 1.0 : 0.0)) * rho);
      if (ta.drc) {
        const double* e = ta.drc + ((size_t)d * nr + r) * 9;
        dA += lp.a1 * (e[0] + e[1] * lT - e[2] * iT) + lp.a2 * (e[3] + e[4] * lT - e[5] * iT) +
              lp.ainf * (e[6] + e[7] * lT - e[8] * iT);
      }
      const double dG = gT * dT;
      const double dlq = wf * (dA + sf * rho) + (1.0 - wf) * (dA + dG + sr * rho);
      const double dlm = ta.dlm ? ta.dlm[dc * nr + r] : 0.0;
      const double dlf = dA - lim * dlq + dlm, dlr = dlf + dG;
      double* kd = rate_tangent(net, ta, sl, d);
      kd[r] = kf == 0.0 ? 0.0 : kf * dlf;
      kd[nr + r] = kr == 0.0 ? 0.0 : kr * dlr;
    }
  }
  __syncthreads();
}

// ---- the try's tangent ----

// the first and second products of one side of a reaction: sum_m e_m prod_{l != m} a_l, and
// sum_{m != l} e_m f_l prod_{others} a
__device__ __forceinline__ double side1(double a0, double a1, double a2, double e0, double e1, double e2) {
  return e0 * a1 * a2 + a0 * e1 * a2 + a0 * a1 * e2;
}
__device__ __forceinline__ double side2(double a0, double a1, double a2, double e0, double e1, double e2, double f0,
                                        double f1, double f2) {
  return e0 * (f1 * a2 + a1 * f2) + e1 * (f0 * a2 + a0 * f2) + e2 * (f0 * a1 + a0 * f1);
}

// y = S z on the CTA (z [nr + 1] with z[nr] = 0), through the call's per-thread S v streams. Two barriers.
__device__ __forceinline__ void s_apply(const Net& net, const Cell& c, const double* z, double* y, int tid, int nt) {
  const uint16_t* __restrict__ sw = net.sv[0] + tid;
  const uint16_t* __restrict__ sr = net.sv_rows[0] + tid;
  double s = 0.0;
  int piece = 0;
  const int rounds = net.sv_rounds[0];
#pragma unroll 4
  for (int q = 0; q < rounds; q++) {
    const unsigned w = __ldg(sw + q * nt);
    s = fma(code_coefficient(w >> 11), z[w & 0x7ffu], s);
    if (w & 0x2000u) {
      c.part[__ldg(sr + piece * nt)] = s;
      s = 0.0;
      piece++;
    }
  }
  __syncthreads();
  for (int i = tid; i < net.ns; i += nt) {
    const int p0 = __ldg(net.sv_row_ptr + i), p1 = __ldg(net.sv_row_ptr + i + 1);
    double r = c.part[p0];
    for (int p = p0 + 1; p < p1; p++) r += c.part[p];
    y[i] = r;
  }
  __syncthreads();
}

// n = nd Y / ntot and its tangent at the state Y (given as N + a K1 + b K3) with tangent Yd; returns the factors
// (ixf, its tangent) of F = S v ixf. Y is formed as the primal forms it. One barrier.
struct StateFactors {
  double ntot, ntd, ixf, ixfd;
};

__device__ __forceinline__ StateFactors state_at(const Net& net, const Cell& c, const TanCell& t, int which,
                                                 const double* Yd, double nd, double rho, int tid, int nt) {
  const int ns = net.ns, lane = tid & 31;
  double p = 0.0, pd = 0.0;
  for (int i = lane; i < ns; i += 32) {
    const double y = which == 0 ? c.N[i] : (which == 1 ? c.N[i] + 2.0 * c.K1[i] : c.N[i] + 2.0 * c.K1[i] + c.K3[i]);
    p += y;
    pd += Yd[i];
  }
  StateFactors f;
  f.ntot = warp_sum(p);
  f.ntd = warp_sum(pd);
  const double xf = nd / f.ntot, xfd = xf * (rho - f.ntd / f.ntot);
  f.ixf = f.ntot / nd;
  f.ixfd = f.ixf * (f.ntd / f.ntot - rho);
  for (int i = tid; i < ns; i += nt) {
    const double y = which == 0 ? c.N[i] : (which == 1 ? c.N[i] + 2.0 * c.K1[i] : c.N[i] + 2.0 * c.K1[i] + c.K3[i]);
    c.n[i] = y * xf;
    t.tn[i] = fma(Yd[i], xf, y * xfd);
  }
  if (tid == 0) {
    c.n[ns] = 1.0;
    t.tn[ns] = 0.0;
    c.v[net.nr] = 0.0;
    t.z[net.nr] = 0.0;
  }
  __syncthreads();
  return f;
}

// the reaction's sides: concentrations a (n), their tangents e (tn), and a vector y's entries (0 at the padding)
struct Sides {
  double a[6], e[6];
  int s[6];
};

__device__ __forceinline__ Sides sides_of(const Net& net, const Cell& c, const TanCell& t, int r) {
  const uint64_t w = __ldg(net.rx8 + r);
  Sides q;
#pragma unroll
  for (int m = 0; m < 6; m++) {
    q.s[m] = (int)((w >> (8 * m)) & 255);
    q.a[m] = c.n[q.s[m]];
    q.e[m] = t.tn[q.s[m]];
  }
  return q;
}

__device__ __forceinline__ double entry(const double* y, int i, int ns) { return i < ns ? y[i] : 0.0; }

// F's tangent at the state of c.n, t.tn into y: S (v_dot ixf + v ixf_dot). Three barriers.
__device__ __forceinline__ void f_tangent(const Net& net, const Cell& c, const TanCell& t, const double* kd,
                                          const StateFactors& f, double* y, int tid, int nt) {
  const int nr = net.nr;
  for (int r = tid; r < nr; r += nt) {
    const Sides q = sides_of(net, c, t, r);
    const double kf = c.kf[r], kr = c.kr[r];
    const double pf = q.a[0] * q.a[1] * q.a[2], pr = q.a[3] * q.a[4] * q.a[5];
    const double v = kf * pf - kr * pr;
    const double vd = kd[r] * pf + kf * side1(q.a[0], q.a[1], q.a[2], q.e[0], q.e[1], q.e[2]) - kd[nr + r] * pr -
                      kr * side1(q.a[3], q.a[4], q.a[5], q.e[3], q.e[4], q.e[5]);
    c.v[r] = fma(vd, f.ixf, v * f.ixfd);
  }
  __syncthreads();
  s_apply(net, c, c.v, y, tid, nt);
}

// Jn' y for two vectors ya, yb (ns entries each) into S-applied outputs oa, ob. Five barriers.
__device__ __forceinline__ void jacobian_tangent2(const Net& net, const Cell& c, const TanCell& t, const double* kd,
                                                  const double* ya, const double* yb, double* oa, double* ob, int tid,
                                                  int nt) {
  const int nr = net.nr, ns = net.ns;
  for (int r = tid; r < nr; r += nt) {
    const Sides q = sides_of(net, c, t, r);
    const double kf = c.kf[r], kr = c.kr[r], dkf = kd[r], dkr = kd[nr + r];
    double out[2];
#pragma unroll
    for (int v = 0; v < 2; v++) {
      const double* y = v ? yb : ya;
      double f[6];
#pragma unroll
      for (int m = 0; m < 6; m++) f[m] = entry(y, q.s[m], ns);
      out[v] = dkf * side1(q.a[0], q.a[1], q.a[2], f[0], f[1], f[2]) +
               kf * side2(q.a[0], q.a[1], q.a[2], q.e[0], q.e[1], q.e[2], f[0], f[1], f[2]) -
               dkr * side1(q.a[3], q.a[4], q.a[5], f[3], f[4], f[5]) -
               kr * side2(q.a[3], q.a[4], q.a[5], q.e[3], q.e[4], q.e[5], f[3], f[4], f[5]);
    }
    c.v[r] = out[0];
    t.z[r] = out[1];
  }
  __syncthreads();
  s_apply(net, c, c.v, oa, tid, nt);
  s_apply(net, c, t.z, ob, tid, nt);
}

// one stage's solve on warp 0: y <- W^-1 y (the call's M0^-1 and Sherman-Morrison, or the recovery's dense W^-1)
template <int R, bool DENSE>
__device__ __forceinline__ void stage_solve(const Net& net, const Cell& c, double* y, double c0, const int* pr,
                                            int lane) {
  if (DENSE) {
    dense_solve<R>(net, c.A, c.dinv, pr, y, lane);
  } else {
    lu_solve<R, 1>(net, c.A, c.dinv, y, nullptr, lane);
    sherman(net, y, c.U, c0, lane);
  }
}

// The step factor's tangent (step_factor's derivative), given the primal's arguments and their tangents.
__device__ __forceinline__ double step_factor_tangent(double en, double den, bool ok, bool prej, double pen,
                                                      double dpen, double pha, double dpha, double ha, double dha) {
  const bool efin = isfinite(en);
  double f = MX_FAC_NONFINITE, df = 0.0;
  if (efin) {
    const double e = fmax(en, MX_ERR_FLOOR);
    f = MX_STEP_SAFETY / cbrt(e);
    df = en >= MX_ERR_FLOOR ? -f * den / (3.0 * e) : 0.0;
  }
  const double lo = ok ? MX_FACACC : MX_FACREJ;
  if (f < lo) df = 0.0;
  f = fmax(f, lo);
  if (f > MX_FACMAX) df = 0.0;
  f = fmin(f, MX_FACMAX);
  if (!ok && efin && prej && en > 1.0 && pen > 1.0 && pha > ha) {
    const double lpe = log(pen / en), lph = log(pha / ha), pe = lpe / lph;
    if (pe > MX_SECANT_MIN_ORDER) {
      const double dpe = ((dpen / pen - den / en) - pe * (dpha / pha - dha / ha)) / lph;
      const double p = fmin(pe, MX_SECANT_MAX_ORDER), dp = pe <= MX_SECANT_MAX_ORDER ? dpe : 0.0;
      const double gv = pow(MX_SECANT_TARGET / en, 1.0 / p);
      const double dg = gv * (-den / (en * p) - log(MX_SECANT_TARGET / en) * dp / (p * p));
      f = fmax(gv, MX_SECMIN);
      df = gv >= MX_SECMIN ? dg : 0.0;
    } else {
      f = MX_SECMIN;
      df = 0.0;
    }
  }
  if (!ok && f > MX_FAC_AFTER_REJECT) df = 0.0;
  return df;
}

// err's tangent on warp 0 (try_error's derivative): q_i = K4_i / sc_i, sc_i = atol + rtol max(|N_i|, |N'_i|); the RMS,
// or while first the larger of it and max |q| (shared evenly among the species attaining it).
__device__ double error_tangent(const Net& net, const Cell& c, const double* tK4, const double* tN, const double* tY,
                                bool first, double rtol, double atol, int lane) {
  const int ns = net.ns;
  double e2 = 0.0, em = 0.0, de = 0.0;
  for (int i = lane; i < ns; i += 32) {
    const double y = c.Y[i], ni = c.N[i];
    const double an = fabs(ni), ay = fabs(y);
    const double dan = ni > 0.0 ? tN[i] : (ni < 0.0 ? -tN[i] : 0.0);
    const double day = y > 0.0 ? tY[i] : (y < 0.0 ? -tY[i] : 0.0);
    const double dmx = an > ay ? dan : (ay > an ? day : 0.5 * (dan + day));
    const double sc = fma(rtol, fmax(an, ay), atol);
    const double q = c.K4[i] / sc;
    e2 = fma(q, q, e2);
    em = fmax(em, fabs(q));
    de = fma(q, (tK4[i] - q * rtol * dmx) / sc, de);
  }
  const double er = sqrt(warp_sum(e2) / ns), emx = warp_max(em), s = warp_sum(de);
  const double der = er > 0.0 ? s / (ns * er) : 0.0;
  if (!(first && isfinite(er))) return der;
  double sd = 0.0, cnt = 0.0;
  for (int i = lane; i < ns; i += 32) {
    const double y = c.Y[i], ni = c.N[i];
    const double an = fabs(ni), ay = fabs(y);
    const double dan = ni > 0.0 ? tN[i] : (ni < 0.0 ? -tN[i] : 0.0);
    const double day = y > 0.0 ? tY[i] : (y < 0.0 ? -tY[i] : 0.0);
    const double dmx = an > ay ? dan : (ay > an ? day : 0.5 * (dan + day));
    const double sc = fma(rtol, fmax(an, ay), atol);
    const double q = c.K4[i] / sc, dq = (tK4[i] - q * rtol * dmx) / sc;
    if (fabs(q) == emx) {
      sd += q > 0.0 ? dq : (q < 0.0 ? -dq : 0.0);
      cnt += 1.0;
    }
  }
  sd = warp_sum(sd);
  cnt = warp_sum(cnt);
  const double demx = cnt > 0.0 ? sd / cnt : 0.0;
  return er > emx ? der : (emx > er ? demx : 0.5 * (der + demx));
}

// The primal's try, as far as the step state goes: what the tangent of a try needs of it.
struct TryState {
  double ha, c0, en, h, t, pen, pha;
  bool ok, prej, first;
};

// The tangent of one try along direction d, after the primal's error and before its update. Reads K1-K4, N, Y (= N'),
// the factors (A, dinv, U or pr) and the rates; uses n, v, F and part as scratch. Updates the direction's state
// tangent (if accepted) and step tangents in the CTA's scratch.
template <int W, int R, bool DENSE>
__device__ void tangent_try(const Net& net, const Cell& c, const TanCell& t, const TanArgs& ta, double* sl, int d,
                            int cell, int B, const TryState& ts, double dt, double Tc, double P, double nd,
                            const int* pr, double rtol, double atol, int tid) {
  constexpr int nt = 32 * W;
  const int ns = net.ns, lane = tid & 31, warp = tid >> 5;
  const size_t dc = (size_t)d * B + cell;
  const double rho = ta.dP[dc] / P - ta.dT[dc] / Tc;
  const double* kd = rate_tangent(net, ta, sl, d);
  double* Nd = state_tangent(net, ta, sl, d);
  double* sc = step_tangent(net, ta, sl, d);
  const double hd = sc[0], td = sc[1], pend = sc[2], phad = sc[3];
  double had = 0.0;  // the try's size min(h, dt - t): a tie splits
  if (ta.adapt) {
    const double rem = dt - ts.t, rd = ta.ddt[dc] - td;
    had = ts.h < rem ? hd : (rem < ts.h ? rd : 0.5 * (hd + rd));
  }
  for (int i = tid; i < ns; i += nt) t.tN[i] = Nd[i];
  __syncthreads();
  // at N: F's tangent, u's tangent and Jn' K for the four stages
  const StateFactors f0 = state_at(net, c, t, 0, t.tN, nd, rho, tid, nt);
  {
    const int nr = net.nr;
    const double i2 = 1.0 / (f0.ntot * f0.ntot);
    for (int r = tid; r < nr; r += nt) {
      const Sides q = sides_of(net, c, t, r);
      const double kf = c.kf[r], kr = c.kr[r], dkf = kd[r], dkr = kd[nr + r];
      double Nv[6], Ndv[6];
#pragma unroll
      for (int m = 0; m < 6; m++) {
        Nv[m] = entry(c.N, q.s[m], ns);
        Ndv[m] = entry(t.tN, q.s[m], ns);
      }
      const double pf = q.a[0] * q.a[1] * q.a[2], pb = q.a[3] * q.a[4] * q.a[5];
      const double v = kf * pf - kr * pb;
      const double vd = dkf * pf + kf * side1(q.a[0], q.a[1], q.a[2], q.e[0], q.e[1], q.e[2]) - dkr * pb -
                        kr * side1(q.a[3], q.a[4], q.a[5], q.e[3], q.e[4], q.e[5]);
      const double nf1 = side1(q.a[0], q.a[1], q.a[2], Nv[0], Nv[1], Nv[2]);
      const double nb1 = side1(q.a[3], q.a[4], q.a[5], Nv[3], Nv[4], Nv[5]);
      const double jn = kf * nf1 - kr * nb1;  // (Jn N)'s reaction term
      const double jdn = dkf * nf1 + kf * side2(q.a[0], q.a[1], q.a[2], q.e[0], q.e[1], q.e[2], Nv[0], Nv[1], Nv[2]) -
                         dkr * nb1 - kr * side2(q.a[3], q.a[4], q.a[5], q.e[3], q.e[4], q.e[5], Nv[3], Nv[4], Nv[5]);
      const double jnd = kf * side1(q.a[0], q.a[1], q.a[2], Ndv[0], Ndv[1], Ndv[2]) -
                         kr * side1(q.a[3], q.a[4], q.a[5], Ndv[3], Ndv[4], Ndv[5]);
      c.v[r] = fma(vd, f0.ixf, v * f0.ixfd);
      // u = S v / nd - (Jn N) / ntot
      t.z[r] = (vd - v * rho) / nd - (jdn + jnd) / f0.ntot + jn * f0.ntd * i2;
    }
  }
  __syncthreads();
  s_apply(net, c, c.v, t.tF, tid, nt);
  s_apply(net, c, t.z, t.tu, tid, nt);
  jacobian_tangent2(net, c, t, kd, c.K1, c.K2, t.JK[0], t.JK[1], tid, nt);
  jacobian_tangent2(net, c, t, kd, c.K3, c.K4, t.JK[2], t.JK[3], tid, nt);
  const double ha = ts.ha, ih = 1.0 / ha, ihd = -had / (ha * ha), gh2 = had / (GAMMA * ha * ha);
  if (warp == 0) {  // stages 1 and 2
    const double s1 = lane_sum(c.K1, ns, lane), s2 = lane_sum(c.K2, ns, lane);
    for (int i = lane; i < ns; i += 32)
      t.tK[0][i] = t.tF[i] + gh2 * c.K1[i] + t.JK[0][i] + t.tu[i] * s1;
    __syncwarp();
    stage_solve<R, DENSE>(net, c, t.tK[0], ts.c0, pr, lane);
    for (int i = lane; i < ns; i += 32)
      t.tK[1][i] = t.tF[i] + RODAS_C21 * (ih * t.tK[0][i] + ihd * c.K1[i]) + gh2 * c.K2[i] + t.JK[1][i] +
                   t.tu[i] * s2;
    __syncwarp();
    stage_solve<R, DENSE>(net, c, t.tK[1], ts.c0, pr, lane);
    for (int i = lane; i < ns; i += 32) t.tY[i] = t.tN[i] + 2.0 * t.tK[0][i];
  }
  __syncthreads();
  {  // stage 3 at Y3 = N + 2 K1
    const StateFactors f3 = state_at(net, c, t, 1, t.tY, nd, rho, tid, nt);
    f_tangent(net, c, t, kd, f3, c.F, tid, nt);
  }
  if (warp == 0) {
    const double s3 = lane_sum(c.K3, ns, lane);
    for (int i = lane; i < ns; i += 32)
      t.tK[2][i] = c.F[i] + ih * (t.tK[0][i] - t.tK[1][i]) + ihd * (c.K1[i] - c.K2[i]) + gh2 * c.K3[i] +
                   t.JK[2][i] + t.tu[i] * s3;
    __syncwarp();
    stage_solve<R, DENSE>(net, c, t.tK[2], ts.c0, pr, lane);
    for (int i = lane; i < ns; i += 32) t.tY[i] = t.tN[i] + 2.0 * t.tK[0][i] + t.tK[2][i];
  }
  __syncthreads();
  {  // stage 4 at Y4 = N + 2 K1 + K3
    const StateFactors f4 = state_at(net, c, t, 2, t.tY, nd, rho, tid, nt);
    f_tangent(net, c, t, kd, f4, c.F, tid, nt);
  }
  if (warp == 0) {
    const double s4 = lane_sum(c.K4, ns, lane);
    for (int i = lane; i < ns; i += 32)
      t.tK[3][i] = c.F[i] + ih * fma(-RODAS_C43, t.tK[2][i], t.tK[0][i] - t.tK[1][i]) +
                   ihd * fma(-RODAS_C43, c.K3[i], c.K1[i] - c.K2[i]) + gh2 * c.K4[i] + t.JK[3][i] + t.tu[i] * s4;
    __syncwarp();
    stage_solve<R, DENSE>(net, c, t.tK[3], ts.c0, pr, lane);
    for (int i = lane; i < ns; i += 32) t.tY[i] += t.tK[3][i];  // N'
    __syncwarp();
    const double den = ta.adapt ? error_tangent(net, c, t.tK[3], t.tN, t.tY, ts.first, rtol, atol, lane) : 0.0;
    if (ts.ok)
      for (int i = lane; i < ns; i += 32) Nd[i] = c.Y[i] >= 0.0 ? t.tY[i] : 0.0;  // the clamp at 0 passes at 0
    if (lane == 0 && ta.adapt) {
      const double fac = step_factor(ts.en, ts.ok, ts.prej, ts.pen, ts.pha, ha);
      const double dfac = step_factor_tangent(ts.en, den, ts.ok, ts.prej, ts.pen, pend, ts.pha, phad, ha, had);
      sc[0] = fma(had, fac, ha * dfac);
      if (ts.ok) sc[1] = td + had;
      sc[2] = den;
      sc[3] = had;
    }
  }
  __syncthreads();
}

// The direction states at the start of a pass: N's tangent from dx (elimination order) and the first try's tangent
// max(start, H_MIN) with start = min(h0, dt), or min(h0, dt, dt split^k) on retry k. A non-finite h acts as dt with no
// tangent of its own.
__device__ __forceinline__ void start_tangents(const Net& net, const TanArgs& ta, double* sl, int cell, int B,
                                               double hin, double dt, int retry, int tid, int nt) {
  const int ns = net.ns;
  for (int d = 0; d < ta.D; d++) {
    const size_t dc = (size_t)d * B + cell;
    double* Nd = state_tangent(net, ta, sl, d);
    const double* dx = ta.dx + dc * ns;
    for (int i = tid; i < ns; i += nt) Nd[i] = dx[__ldg(net.perm + i)];
    if (tid == 0) {
      const bool fin = isfinite(hin);
      const double h0 = fin ? hin : dt, dh0 = fin ? ta.dh[dc] : ta.ddt[dc], ddt = ta.ddt[dc];
      const double m = fmin(h0, dt), dm = h0 < dt ? dh0 : (dt < h0 ? ddt : 0.5 * (dh0 + ddt));
      double start = m, ds = dm;
      if (retry > 0) {
        const double sp = pow(MX_REC_RETRY_SPLIT, (double)retry), cap = dt * sp, dcap = ddt * sp;
        start = fmin(m, cap);
        ds = m < cap ? dm : (cap < m ? dcap : 0.5 * (dm + dcap));
      }
      double* sc = step_tangent(net, ta, sl, d);
      sc[0] = start >= MX_H_MIN ? ds : 0.0;
      sc[1] = sc[2] = sc[3] = 0.0;
    }
  }
  __syncthreads();
}

// dx = (N_dot - x sum N_dot) / sum N in network order, dh = h's tangent (0 frozen); NaN when nan.
__device__ __forceinline__ void write_tangents(const Net& net, const Cell& c, const TanArgs& ta, double* sl, int cell,
                                               int B, double sum, bool nan, int tid, int nt) {
  const int ns = net.ns, lane = tid & 31;
  for (int d = 0; d < ta.D; d++) {
    const size_t dc = (size_t)d * B + cell;
    const double* Nd = state_tangent(net, ta, sl, d);
    const double sd = lane_sum(Nd, ns, lane);
    double* out = ta.dx_out + dc * ns;
    for (int i = tid; i < ns; i += nt) {
      const double x = c.N[i] / sum;
      out[__ldg(net.perm + i)] = nan ? __longlong_as_double(0x7ff8000000000000ll) : (Nd[i] - x * sd) / sum;
    }
    if (tid == 0)
      ta.dh_out[dc] = nan ? __longlong_as_double(0x7ff8000000000000ll) : (ta.adapt ? step_tangent(net, ta, sl, d)[0] : 0.0);
  }
}

// the cell's log multipliers: applied to both directions (after the collision limit), and all finite?
__device__ __forceinline__ void apply_multipliers(const Net& net, const Cell& c, const double* lm, int tid, int nt) {
  for (int r = tid; r < net.nr; r += nt) {
    const double e = exp(lm[r]);
    c.kf[r] = c.kf[r] * e;
    c.kr[r] = c.kr[r] * e;
  }
  __syncthreads();
}

__device__ __forceinline__ bool multipliers_finite(const Net& net, const double* lm, int tid) {
  bool fin = true;
  if (lm)
    for (int r = tid; r < net.nr; r += blockDim.x) fin = fin && isfinite(lm[r]);
  return __syncthreads_and(fin) != 0;
}

// ---- the kernels ----

// The tangent kernel: the call kernel's screening, rates, Rodas3 tries, output and guard (call_kernel, same device
// functions, same order, so the same bits), with the tangent of every try that the contract differentiates, and the
// tangents of the uncorrected result written out. A non-finite log multiplier takes no step (the guard then lists the
// cell, and the recovery fails it).
template <int W, int R>
__global__ void __launch_bounds__(32 * W, 3) jvp_kernel(const Net net, const CallArgs a, const TanArgs ta,
                                                        const TanLayout tl) {
  extern __shared__ double smem[];
  const Cell c = cell_arrays(net, smem);
  const TanCell t = tan_arrays(tl, smem);
  const int tid = (int)threadIdx.x, nt = 32 * W, lane = tid & 31, warp = tid >> 5, ns = net.ns, ld = net.ld;
  double* sl = ta.scratch + (size_t)blockIdx.x * ta.slot;
  int cell = (int)blockIdx.x;
  while (cell < a.B) {
    const double Tc = a.T[cell], dt = a.dt[cell], hin = a.h_in[cell], P = a.P[cell];
    const double nd = P / (MX_KB * Tc);
    const double* x0 = a.x + (size_t)cell * ns;
    const double* Jc = a.J + (size_t)cell * net.nj;
    const double* lmc = ta.lm ? ta.lm + (size_t)cell * net.nr : nullptr;
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
    const bool lm_fine = multipliers_finite(net, lmc, tid);
    if (st == 0) {
      cell_rates(net, c, Tc, nd, Jc, tid, nt);
      if (lmc) apply_multipliers(net, c, lmc, tid, nt);
      rate_tangents(net, c, ta, sl, cell, a.B, Tc, P, nd, Jc, c.v, t.z, tid, nt);
    }
    start_tangents(net, ta, sl, cell, a.B, hin, dt, 0, tid, nt);
    const double h0 = isfinite(hin) ? hin : dt;
    StepState s = {fmax(fmin(h0, dt), MX_H_MIN), 0.0, 0.0, 0.0, 0.0, false};
    int it = (dt > 0.0 && st == 0 && lm_fine) ? 0 : a.max_steps;
    double c0 = 0.0;
    while (it < a.max_steps && s.t < dt * MX_CALL_END) {
      const double ha = fmin(s.h, dt - s.t), igh = 1.0 / (GAMMA * ha), ih = 1.0 / ha;
      const double ntot = rhs(net, c, c.N, true, nd, tid, nt);
      jacobian_w(net, c, ntot, tid, nt);
      for (int i = tid; i < ns; i += nt) c.A[i * ld + i] += igh;
      __syncthreads();
      lu_factor<32 * W>(net, c.A, c.dinv, tid);
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
        for (int i = lane; i < ns; i += 32)
          c.K4[i] = fma(ih, fma(-RODAS_C43, c.K3[i], c.K1[i] - c.K2[i]), c.F[i]);
        __syncwarp();
        lu_solve<R, 1>(net, c.A, c.dinv, c.K4, nullptr, lane);
        sherman(net, c.K4, c.U, c0, lane);
        try_error(net, c, s.t == 0.0, a.rtol, a.atol, lane);
      }
      __syncthreads();
      const double en = c.red[0];
      const bool ok = c.red[1] != 0.0;
      if (ta.adapt || ok) {
        const TryState ts = {ha, c0, en, s.h, s.t, s.pen, s.pha, ok, s.prej, s.t == 0.0};
        for (int d = 0; d < ta.D; d++)
          tangent_try<W, R, false>(net, c, t, ta, sl, d, cell, a.B, ts, dt, Tc, P, nd, nullptr, a.rtol, a.atol, tid);
      }
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
    write_tangents(net, c, ta, sl, cell, a.B, sum, false, tid, nt);
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
        c.ints[1] = (int)(gridDim.x + atomicAdd(a.count + MX_COUNT_QUEUE, 1));
      }
    }
    __syncthreads();
    double* xo = a.x_out + (size_t)cell * ns;
    for (int i = tid; i < ns; i += nt) xo[i] = c.Y[i];
    cell = c.ints[1];
    __syncthreads();
  }
}

// The tangent of the recovery (recover_kernel's path, dense pivoted W, retries included): the listed cells redone
// with their tangents. A cell that still fails has NaN tangents.
template <int W, int R>
__global__ void __launch_bounds__(32 * W, 3) jvp_recover_kernel(const Net net, const CallArgs a, const TanArgs ta,
                                                                const TanLayout tl, int max_steps) {
  const int nfl = a.count[MX_COUNT_RECOMPUTED];
  if ((int)blockIdx.x >= nfl) return;
  extern __shared__ double smem[];
  const Cell c = cell_arrays(net, smem);
  const TanCell t = tan_arrays(tl, smem);
  const int tid = (int)threadIdx.x, nt = 32 * W, lane = tid & 31, warp = tid >> 5, ns = net.ns, ld = net.ld;
  int* pr = c.ints + 4;
  double* sl = ta.scratch + (size_t)blockIdx.x * ta.slot;
  int q = (int)blockIdx.x;
  while (q < nfl) {
    const int cell = a.list[q];
    const double Tc = a.T[cell], dt = a.dt[cell], hin = a.h_in[cell], P = a.P[cell];
    const double nd = P / (MX_KB * Tc);
    const double* x0 = a.x + (size_t)cell * ns;
    const double* Jc = a.J + (size_t)cell * net.nj;
    const double* lmc = ta.lm ? ta.lm + (size_t)cell * net.nr : nullptr;
    const bool lm_fine = multipliers_finite(net, lmc, tid);
    cell_rates(net, c, Tc, nd, Jc, tid, nt);  // a listed cell passed the screening (status 0)
    if (lmc) apply_multipliers(net, c, lmc, tid, nt);
    rate_tangents(net, c, ta, sl, cell, a.B, Tc, P, nd, Jc, c.v, t.z, tid, nt);
    const double h0 = isfinite(hin) ? hin : dt, m = fmin(h0, dt);
    for (int k = 0;; k++) {
      for (int i = tid; i < ns; i += nt) c.N[i] = x0[__ldg(net.perm + i)];
      __syncthreads();
      start_tangents(net, ta, sl, cell, a.B, hin, dt, k, tid, nt);
      const double start = k == 0 ? m : fmin(m, dt * pow(MX_REC_RETRY_SPLIT, (double)k));
      StepState s = {fmax(start, MX_H_MIN), 0.0, 0.0, 0.0, 0.0, false};
      int it = (dt > 0.0 && lm_fine) ? 0 : max_steps;
      while (it < max_steps && s.t < dt * MX_CALL_END) {
        const double ha = fmin(s.h, dt - s.t), igh = 1.0 / (GAMMA * ha), ih = 1.0 / ha;
        const double ntot = rhs(net, c, c.N, true, nd, tid, nt);
        jacobian_w(net, c, ntot, tid, nt);
        for (int e = tid; e < ns * ns; e += nt) {
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
        if (ta.adapt || ok) {
          const TryState ts = {ha, 0.0, en, s.h, s.t, s.pen, s.pha, ok, s.prej, s.t == 0.0};
          for (int d = 0; d < ta.D; d++)
            tangent_try<W, R, true>(net, c, t, ta, sl, d, cell, a.B, ts, dt, Tc, P, nd, pr, a.rtol, a.atol, tid);
        }
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
          c.ints[2] = g;
          atomicAdd(a.count + (g ? MX_COUNT_STILL_FAILED : MX_COUNT_RECOVERED), 1);
          c.ints[1] = (int)(gridDim.x + atomicAdd(a.count + MX_COUNT_RECOVERY_QUEUE, 1));
        }
      }
      __syncthreads();
      double* xo = a.x_out + (size_t)cell * ns;
      for (int i = tid; i < ns; i += nt) xo[i] = c.Y[i];
      const int nq = c.ints[1];
      if (nq >= 0) write_tangents(net, c, ta, sl, cell, a.B, sum, c.ints[2] != 0, tid, nt);
      __syncthreads();
      if (nq >= 0) {
        q = nq;
        break;
      }
    }
  }
}

}  // namespace mx
