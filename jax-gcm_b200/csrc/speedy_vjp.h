// speedy_vjp.h -- hand-written reverse pass of one SPEEDY column (the adjoint of
// SpeedyPhysics.compute_tendencies, jcm/physics/speedy/speedy_physics.py:88-127).
//
// column_vjp<KX, F> runs the column forward once, keeping the per-level state (T, q, phi, qsat
// and its two partials, RH, dry static energy) and the scalars one term hands to the next
// (convective top and base flux, precipitation, cloud cover, the shortwave and longwave fluxes
// the surface and the upward pass read), then walks the terms backwards.  Each term recomputes
// its own internals from those kept values (its level loops, transmissivities and flux
// recurrences) and applies its derivative by hand.  Nothing is taped: per column the storage is
// a few per-level arrays, so the adjoint costs a small multiple of the forward.
//
// The derivative conventions are those of jax's JVP rules, so that the result is jax.vjp's:
// max/min/clip ties split the derivative evenly between the two arguments; where() passes it to
// the chosen branch only; integer level indices (convective top, cloud top, the cloud-top level
// set) carry none.  The forward arithmetic follows speedy_generic.h operation for operation, so
// every branch is taken as in the forward kernel that records a tape.
//
// The same source builds for the host (F = double or float) and the device (F = float).
#pragma once

#include <math.h>
#include <stdint.h>

#include "speedy_b200.h"
#include "speedy_generic.h"

// Loop unrolling on the device: every loop of the reverse pass is unrolled fully (the level
// count is a template parameter).  Indexed by constants, the small arrays (band fluxes,
// transmissivities, blackbody fractions and their adjoints) become registers and the per-level
// arrays are placed by the register allocator, spilled where they must be, instead of all
// living in local memory behind a dynamic index.  Measured on T170 with 16 levels: 0.916 ms
// with every loop rolled, 0.777 with the band loops unrolled, level loops unrolled by 2 / 4 / 8
// 0.748 / 0.728 / 0.701, fully 0.619.
#if defined(__CUDA_ARCH__)
#define SPD_BANDS _Pragma("unroll")
#define SPD_LEVELS _Pragma("unroll")
#else
#define SPD_BANDS
#define SPD_LEVELS
#endif

namespace spdvjp {

using spdgen::ColumnIn;
using spdgen::DiffParams;

SPD_HD float fexp(float x) { return expf(x); }
SPD_HD double fexp(double x) { return exp(x); }
SPD_HD float fpow(float x, float y) { return powf(x, y); }
SPD_HD double fpow(double x, double y) { return pow(x, y); }
SPD_HD float fsqrt(float x) { return sqrtf(x); }
SPD_HD double fsqrt(double x) { return sqrt(x); }
SPD_HD bool fnan(float x) { return x != x; }
SPD_HD bool fnan(double x) { return x != x; }

// max/min with the value convention of the tape (a tie, NaN included, returns the first).
template <class F> SPD_HD F vmax(F a, F b) { return a > b ? a : (b > a ? b : a); }
template <class F> SPD_HD F vmin(F a, F b) { return a < b ? a : (b < a ? b : a); }
// Derivative of max(a, b) / min(a, b) with respect to a; ties (and NaN) give one half.
template <class F> SPD_HD F wmax(F a, F b) { return a > b ? F(1) : (b > a ? F(0) : F(0.5)); }
template <class F> SPD_HD F wmin(F a, F b) { return a < b ? F(1) : (b < a ? F(0) : F(0.5)); }

enum { P_PSMIN, P_TRCNV, P_RHIL, P_RHBL, P_ENTMAX, P_SMF, P_TRLSC, P_RHLSC, P_DRHLSC,
       P_RHBLSC, P_ALBCL, P_ALBCLS, P_N };

// get_qsat (humidity.py:73-104) and its partials with respect to ta and ps.
template <class F>
SPD_HD F qsat_d(F ta, F ps, F sig, F& d_t, F& d_p) {
  const F e0 = F(6.108e-3), t0 = F(273.16);
  const bool warm = ta >= t0;
  const F c = warm ? F(17.269) : F(21.875);
  const F tt = warm ? F(35.86) : F(7.66);
  const F num = c * (ta - t0), den = ta - tt;
  const F r = num / den;
  const F e = e0 * fexp(r);
  const F de = e * (c / den - r / den);
  const F D = sig * ps - F(0.378) * e;
  const F q = F(622.0) * e / D;
  d_t = (F(622.0) / D + (q / D) * F(0.378)) * de;
  d_p = -(q / D) * sig;
  return q;
}

// qcorh of the orographic correction (orographic_correction.py:117-174; see the forward's
// orographic_horizontal).  Needed by the adjoint only to select the levels verify_tendencies
// limits: the correction depends on no differentiated input.
template <class F>
SPD_HD F orographic_qcorh(F phis0, F fmask, F stl, F sst, F gamlat, F pexp) {
  const F tcorh = gamlat * phis0;
  const F tsfc = fmask * stl + (F(1) - fmask) * sst;
  const F tref = tsfc + tcorh;
  const F psfc = fpow(tsfc / tref, pexp);
  F d1, d2;
  const F qref = qsat_d(tref, F(1), F(1), d1, d2);
  const F qsfc = qsat_d(tsfc, psfc, F(1), d1, d2);
  return F(0.7) * (qref - qsfc);
}

// radset (longwave_radiation.py): band fractions of the blackbody flux and their derivative
// with respect to the temperature.
template <class F>
SPD_HD void radset_d(F temp, F epslw, F fb[4], F dfb[4]) {
  const F lo = vmax(temp, F(200));
  const F j = vmin(lo, F(320));
  const F wj = wmax(temp, F(200)) * wmin(lo, F(320));
  const F a1 = j - F(247), a2 = j - F(282), a3 = j - F(315);
  const F f1 = F(0.148) - F(3.0e-6) * (a1 * a1);
  const F f2 = F(0.356) - F(5.2e-6) * (a2 * a2);
  const F f3 = F(0.314) + F(1.0e-5) * (a3 * a3);
  const F f0 = F(1) - (((F(0) + f1) + f2) + f3);
  const F w = F(1) - epslw;
  fb[0] = w * f0;
  fb[1] = w * f1;
  fb[2] = w * f2;
  fb[3] = w * f3;
  const F d1 = -F(3.0e-6) * F(2) * a1, d2 = -F(5.2e-6) * F(2) * a2, d3 = F(1.0e-5) * F(2) * a3;
  dfb[0] = w * (-(d1 + d2 + d3)) * wj;
  dfb[1] = w * d1 * wj;
  dfb[2] = w * d2 * wj;
  dfb[3] = w * d3 * wj;
}

// What the reverse pass keeps from the forward pass.
template <int KX, class F>
struct Col {
  F t[KX], q[KX], phi[KX];
  F qsat[KX];
  F dfl[KX];  // longwave flux divergence per level, all contributions
  // relative humidity and dry static energy (humidity.py:44, convection.py:123), recomputed at
  // each use rather than kept
  SPD_HD F RH(int k) const { return q[k] / qsat[k]; }
  SPD_HD F SE(int k) const { return F(1004.0) * t[k] + phi[k]; }
  F psa, u, v;
  F qdif;
  int ktop2, iptop_cv;
  bool case1, case2;
  F precnv, precls;
  int iptop;
  F cloudc, clstr, qcloud;
  int icltop;
  bool cloud_nan;
  F rsds, fsw0, fsw1, rlds, rlus2, tsfc;
  F alb_l, albsfc, snowc;
};

// Adjoints.  Those of RH = q / qsat and SE = 1004 T + phi are applied where they arise.
template <int KX, class F>
struct Bar {
  F t[KX], q[KX], phi[KX], qsat[KX];
  F psa, u, v;
  F par[P_N];
  SPD_HD void add_rh(const Col<KX, F>& c, int k, F v) {
    q[k] += v / c.qsat[k];
    qsat[k] -= v * (c.RH(k) / c.qsat[k]);
  }
  SPD_HD void add_se(int k, F v) {
    t[k] += F(1004.0) * v;
    phi[k] += v;
  }
};

struct Ctx {
  const spd_vgrid_t* vg;
  const spd_params_t* p;
  uint32_t flags;
  int model_step;
  uint32_t S;
};

// ---------------------------------------------------------------------------------------------
// spec_hum_to_rel_hum (humidity.py:16-51) and the dry static energy (convection.py:123)
// ---------------------------------------------------------------------------------------------
template <int KX, class F>
SPD_HD void humidity(const Ctx& x, Col<KX, F>& c) {
  SPD_LEVELS
  for (int k = 0; k < KX; ++k) {
    F d_t, d_p;
    c.qsat[k] = qsat_d(c.t[k], c.psa, F(x.vg->fsg[k]), d_t, d_p);
  }
}

template <int KX, class F>
SPD_HD void humidity_rev(const Ctx& x, const Col<KX, F>& c, Bar<KX, F>& b) {
  SPD_LEVELS
  for (int k = 0; k < KX; ++k) {
    F d_t, d_p;
    qsat_d(c.t[k], c.psa, F(x.vg->fsg[k]), d_t, d_p);
    b.t[k] += b.qsat[k] * d_t;
    b.psa += b.qsat[k] * d_p;
  }
}

// ---------------------------------------------------------------------------------------------
// diagnose_convection (convection.py:15-97)
// ---------------------------------------------------------------------------------------------
template <int KX, class F>
SPD_HD F mss2_at(const Ctx& x, const Col<KX, F>& c, int k) {
  if (k >= KX - 1) return F(0);
  const F m0 = c.SE(k) + F(2501.0) * c.qsat[k];
  const F m1 = c.SE(k + 1) + F(2501.0) * c.qsat[k + 1];
  return m0 + F(x.vg->wvi[k][1]) * (m1 - m0);
}

template <int KX, class F>
SPD_HD void dconv(const Ctx& x, const DiffParams<F>& g, Col<KX, F>& c) {
  const F mse0 = c.SE(KX - 1) + F(2501.0) * c.q[KX - 1];
  const F mse1 = vmin(mse0, c.SE(KX - 2) + F(2501.0) * c.q[KX - 2]);
  const F mss0 = vmax(mse0, c.SE(KX - 1) + F(2501.0) * c.qsat[KX - 1]);
  int ktop1 = KX, ktop2 = KX;
  SPD_LEVELS
  for (int k = KX - 4; k >= 2; --k) {
    const F m2 = mss2_at(x, c, k);
    if (mss0 > m2) ktop1 = k + 1;
    if (mse1 > m2) ktop2 = k + 1;
  }
  const F msthr = mss2_at(x, c, ktop2 - 1);
  const F qthr0 = g.rhbl * c.qsat[KX - 1];
  const F qthr1 = g.rhbl * c.qsat[KX - 2];
  const bool lqthr = c.q[KX - 1] > qthr0 && c.q[KX - 2] > qthr1;
  const bool mask_psa = c.psa > g.psmin;
  c.case1 = mask_psa && ktop1 < KX && ktop2 < KX;
  c.case2 = mask_psa && ktop1 < KX && !(ktop2 < KX) && lqthr;
  c.ktop2 = ktop2;
  c.iptop_cv = (c.case1 || c.case2) ? ktop1 : KX + 1;
  c.qdif = F(0);
  if (c.case1) c.qdif = vmax(c.q[KX - 1] - qthr0, (mse0 - msthr) * F(1.0 / 2501.0));
  if (c.case2) c.qdif = c.q[KX - 1] - qthr0;
}

template <int KX, class F>
SPD_HD void dconv_rev(const Ctx& x, const DiffParams<F>& g, const Col<KX, F>& c, F qdif_b,
                      Bar<KX, F>& b) {
  F qthr0_b = F(0);
  const F qthr0 = g.rhbl * c.qsat[KX - 1];
  if (c.case1) {
    const F mse0 = c.SE(KX - 1) + F(2501.0) * c.q[KX - 1];
    // the threshold level j = ktop2 - 1, matched in a loop so that the per-level arrays are
    // addressed by constants
    const int jt = c.ktop2 - 1;
    F msthr = F(0);
    SPD_LEVELS
    for (int j = 0; j < KX; ++j)
      if (j == jt) msthr = mss2_at(x, c, j);
    const F A = c.q[KX - 1] - qthr0;
    const F B = (mse0 - msthr) * F(1.0 / 2501.0);
    const F Ab = qdif_b * wmax(A, B);
    const F Bb = qdif_b * wmax(B, A);
    b.q[KX - 1] += Ab;
    qthr0_b -= Ab;
    const F mse0_b = Bb * F(1.0 / 2501.0);
    const F msthr_b = -mse0_b;
    b.add_se(KX - 1, mse0_b);
    b.q[KX - 1] += F(2501.0) * mse0_b;
    SPD_LEVELS
    for (int j = 0; j < KX - 1; ++j) {
      if (j != jt) continue;
      const F w = F(x.vg->wvi[j][1]);
      const F m0b = msthr_b - w * msthr_b, m1b = w * msthr_b;
      b.add_se(j, m0b);
      b.qsat[j] += F(2501.0) * m0b;
      b.add_se(j + 1, m1b);
      b.qsat[j + 1] += F(2501.0) * m1b;
    }
  } else if (c.case2) {
    b.q[KX - 1] += qdif_b;
    qthr0_b -= qdif_b;
  }
  b.par[P_RHBL] += qthr0_b * c.qsat[KX - 1];
  b.qsat[KX - 1] += qthr0_b * g.rhbl;
}

// ---------------------------------------------------------------------------------------------
// get_convection_tendencies (convection.py:99-237)
// ---------------------------------------------------------------------------------------------
template <int KX, class F>
struct Cv {
  F entr[KX], sb3[KX], qb3[KX], fm3[KX], fus3[KX], fuq3[KX], fds3[KX], fdq3[KX];
  F dfse[KX], dfqa[KX];
  F sentr, escale, fm0, rdps, qmax, sb, qb, fpsa, mn2, fmass, ratio, mn, cbmf;
  F fus, fuq, fds, fdq, qsatb, X, precnv, rps;
};

template <int KX, class F>
SPD_HD void conv(const Ctx& x, const DiffParams<F>& g, const Col<KX, F>& c, Cv<KX, F>& w) {
  const spd_vgrid_t& vg = *x.vg;
  const int iptop = c.iptop_cv;
  w.sentr = F(0);
  SPD_LEVELS
  for (int k = 1; k < KX - 1; ++k) {
    const F e = vmax(F(0), F(vg.fsg[k]) - F(0.5));
    w.entr[k] = e * e;
    w.sentr = w.sentr + w.entr[k];
  }
  w.escale = g.entmax / w.sentr;
  SPD_LEVELS
  for (int k = 1; k < KX - 1; ++k) w.entr[k] = w.entr[k] * w.escale;
  w.fm0 = F(1e5) * F(vg.dhs[KX - 1]) / (F(9.81) * g.trcnv * F(3600.0));
  w.rdps = F(2.0) / (F(1.0) - g.psmin);
  const bool mask = iptop < KX;
  w.qmax = vmax(F(1.01) * c.q[KX - 1], c.qsat[KX - 1]);
  w.sb3[0] = w.qb3[0] = F(0);
  SPD_LEVELS
  for (int k = 1; k < KX; ++k) {
    w.sb3[k] = c.SE(k - 1) + F(vg.wvi[k - 1][1]) * (c.SE(k) - c.SE(k - 1));
    w.qb3[k] = c.q[k - 1] + F(vg.wvi[k - 1][1]) * (c.q[k] - c.q[k - 1]);
  }
  w.sb = w.sb3[KX - 1];
  w.qb = vmin(w.qb3[KX - 1], c.q[KX - 1]);
  w.mn2 = vmin(F(1.0), (c.psa - g.psmin) * w.rdps);
  w.fpsa = c.psa * w.mn2;
  w.ratio = c.qdif / (w.qmax - w.qb);
  w.mn = vmin(F(5.0), w.ratio);
  w.fmass = w.fm0 * w.fpsa * w.mn;
  w.cbmf = mask ? w.fmass : F(0) * w.fmass;
  w.fus = w.fmass * c.SE(KX - 1);
  w.fuq = w.fmass * w.qmax;
  w.fds = w.fmass * w.sb;
  w.fdq = w.fmass * w.qb;
  F cm = F(0), cs = F(0), cq = F(0);
  SPD_LEVELS
  for (int k = KX - 1; k >= 0; --k) {
    const bool lm = (k <= KX - 2) && (k >= iptop);
    F en = (k >= 1 && k <= KX - 2) ? w.entr[k] * c.psa * w.cbmf : F(0);
    en = lm ? en : F(0) * en;
    cm = cm + en * F(1.0);
    cs = cs + en * c.SE(k);
    cq = cq + en * c.q[k];
    w.fm3[k] = w.fmass + cm;
    w.fus3[k] = w.fus + cs;
    w.fuq3[k] = w.fuq + cq;
    w.fds3[k] = (k == KX - 1) ? w.fds : w.fm3[k] * w.sb3[k];
    w.fdq3[k] = (k == KX - 1) ? w.fdq : w.fm3[k] * w.qb3[k];
  }
  w.dfse[KX - 1] = w.fds - w.fus;
  w.dfqa[KX - 1] = w.fdq - w.fuq;
  SPD_LEVELS
  for (int k = 0; k < KX - 1; ++k) {
    const bool lm = (k >= iptop);
    const F a = (w.fus3[k + 1] - w.fds3[k + 1]) - (w.fus3[k] - w.fds3[k]);
    const F bq = (w.fuq3[k + 1] - w.fdq3[k + 1]) - (w.fuq3[k] - w.fdq3[k]);
    w.dfse[k] = lm ? a : F(0) * a;
    w.dfqa[k] = lm ? bq : F(0) * bq;
  }
  F fsq_sum = F(0);
  SPD_LEVELS
  for (int k = 0; k < KX; ++k) {
    const bool lm = (k <= KX - 2) && (k >= iptop);
    const F d0 = g.rhil * c.qsat[k] - c.q[k];
    const F delq = lm ? d0 : F(0) * d0;
    const F fsq = (delq > F(0) ? g.smf : F(0) * g.smf) * w.cbmf * delq;
    w.dfqa[k] = w.dfqa[k] + fsq;
    fsq_sum = fsq_sum + fsq;
  }
  w.dfqa[KX - 1] = w.dfqa[KX - 1] + (-fsq_sum);
  w.precnv = F(0);
  w.qsatb = w.X = F(0);
  // the top layer k = iptop (1 <= iptop <= kx - 1): a loop over the levels with one match
  // instead of an index, so that the per-level arrays are addressed by constants
  SPD_LEVELS
  for (int k = 1; k < KX; ++k) {
    if (k != iptop) continue;
    const int kt = k - 1;
    w.qsatb = c.qsat[kt] + F(vg.wvi[kt][1]) * (c.qsat[kt + 1] - c.qsat[kt]);
    w.X = w.fuq3[k] - w.fm3[k] * w.qsatb;
    w.precnv = vmax(w.X, F(0));
    w.dfse[kt] = w.fus3[k] - w.fds3[k] + F(2501.0) * w.precnv;
    w.dfqa[kt] = w.fuq3[k] - w.fdq3[k] - w.precnv;
  }
  w.rps = F(1) / c.psa;
}

template <int KX, class F>
SPD_HD void conv_tend(const Ctx& x, const Cv<KX, F>& w, F dt[KX], F dq[KX]) {
  dt[0] = dt[0] + w.dfse[0];
  dq[0] = dq[0] + w.dfqa[0];
  SPD_LEVELS
  for (int k = 1; k < KX; ++k) {
    dt[k] = dt[k] + w.dfse[k] * w.rps * F(x.vg->grdscp[k]);
    dq[k] = dq[k] + w.dfqa[k] * w.rps * F(x.vg->grdsig[k]);
  }
}

template <int KX, class F>
SPD_HD F conv_rev(const Ctx& x, const DiffParams<F>& g, const Col<KX, F>& c, Cv<KX, F>& w,
                  const F* dt_b, const F* dq_b, F precnv_b, Bar<KX, F>& b) {
  const spd_vgrid_t& vg = *x.vg;
  const int iptop = c.iptop_cv;
  F dfse_b[KX], dfqa_b[KX];
  F rps_b = F(0);
  dfse_b[0] = dt_b[0];
  dfqa_b[0] = dq_b[0];
  SPD_LEVELS
  for (int k = 1; k < KX; ++k) {
    dfse_b[k] = dt_b[k] * F(vg.grdscp[k]) * w.rps;
    dfqa_b[k] = dq_b[k] * F(vg.grdsig[k]) * w.rps;
    rps_b += dt_b[k] * F(vg.grdscp[k]) * w.dfse[k] + dq_b[k] * F(vg.grdsig[k]) * w.dfqa[k];
  }
  b.psa += -rps_b * (w.rps / c.psa);
  F fus3_b[KX], fuq3_b[KX], fds3_b[KX], fdq3_b[KX], fm3_b[KX], sb3_b[KX], qb3_b[KX];
  SPD_LEVELS
  for (int k = 0; k < KX; ++k)
    fus3_b[k] = fuq3_b[k] = fds3_b[k] = fdq3_b[k] = fm3_b[k] = sb3_b[k] = qb3_b[k] = F(0);
  SPD_LEVELS
  for (int k = 1; k < KX; ++k) {  // the top layer k = iptop, addressed by constants
    if (k != iptop) continue;
    const int kt = k - 1;
    const F se_b = dfse_b[kt], qa_b = dfqa_b[kt];
    fus3_b[k] += se_b;
    fds3_b[k] -= se_b;
    fuq3_b[k] += qa_b;
    fdq3_b[k] -= qa_b;
    const F pb = precnv_b + F(2501.0) * se_b - qa_b;
    dfse_b[kt] = dfqa_b[kt] = F(0);
    const F Xb = pb * wmax(w.X, F(0));
    fuq3_b[k] += Xb;
    fm3_b[k] -= Xb * w.qsatb;
    const F qsatb_b = -Xb * w.fm3[k];
    const F ww = F(vg.wvi[kt][1]);
    b.qsat[kt] += qsatb_b - ww * qsatb_b;
    b.qsat[kt + 1] += ww * qsatb_b;
  }
  // dfqa[KX-1] -= sum(fsq); dfqa[k] += fsq[k]
  const F fsq_sum_b = -dfqa_b[KX - 1];
  F cbmf_b = F(0);
  SPD_LEVELS
  for (int k = 0; k < KX; ++k) {
    const bool lm = (k <= KX - 2) && (k >= iptop);
    if (!lm) continue;
    const F d0 = g.rhil * c.qsat[k] - c.q[k];
    const F fsq_b = dfqa_b[k] + fsq_sum_b;
    const F sm = d0 > F(0) ? g.smf : F(0);
    cbmf_b += fsq_b * d0 * sm;
    if (d0 > F(0)) b.par[P_SMF] += fsq_b * d0 * w.cbmf;
    const F d0_b = fsq_b * (sm * w.cbmf);
    b.par[P_RHIL] += d0_b * c.qsat[k];
    b.qsat[k] += d0_b * g.rhil;
    b.q[k] -= d0_b;
  }
  F fds_b = dfse_b[KX - 1], fus_b = -dfse_b[KX - 1];
  F fdq_b = dfqa_b[KX - 1], fuq_b = -dfqa_b[KX - 1];
  SPD_LEVELS
  for (int k = 0; k < KX - 1; ++k) {
    if (k < iptop) continue;
    const F a = dfse_b[k], q = dfqa_b[k];
    fus3_b[k + 1] += a;
    fds3_b[k + 1] -= a;
    fus3_b[k] -= a;
    fds3_b[k] += a;
    fuq3_b[k + 1] += q;
    fdq3_b[k + 1] -= q;
    fuq3_b[k] -= q;
    fdq3_b[k] += q;
  }
  // the downward accumulation of entrainment
  F fmass_b = F(0), CMB = F(0), CSB = F(0), CQB = F(0);
  SPD_LEVELS
  for (int k = 0; k < KX; ++k) {
    if (k == KX - 1) {
      fds_b += fds3_b[k];
      fdq_b += fdq3_b[k];
    } else {
      fm3_b[k] += fds3_b[k] * w.sb3[k] + fdq3_b[k] * w.qb3[k];
      sb3_b[k] += fds3_b[k] * w.fm3[k];
      qb3_b[k] += fdq3_b[k] * w.fm3[k];
    }
    fmass_b += fm3_b[k];
    CMB += fm3_b[k];
    fus_b += fus3_b[k];
    CSB += fus3_b[k];
    fuq_b += fuq3_b[k];
    CQB += fuq3_b[k];
    const bool lm = (k <= KX - 2) && (k >= iptop);
    if (lm && k >= 1) {
      const F en = w.entr[k] * c.psa * w.cbmf;
      const F en_b = CMB + CSB * c.SE(k) + CQB * c.q[k];
      b.add_se(k, CSB * en);
      b.q[k] += CQB * en;
      const F ep = w.entr[k] * c.psa;
      cbmf_b += en_b * ep;
      const F ep_b = en_b * w.cbmf;
      b.psa += ep_b * w.entr[k];
      // entr[k] = e^2 * escale, escale = entmax / sentr
      const F e = vmax(F(0), F(vg.fsg[k]) - F(0.5));
      b.par[P_ENTMAX] += ep_b * c.psa * (e * e) / w.sentr;
    }
  }
  fmass_b += fus_b * c.SE(KX - 1) + fuq_b * w.qmax + fds_b * w.sb + fdq_b * w.qb;
  b.add_se(KX - 1, fus_b * w.fmass);
  F qmax_b = fuq_b * w.fmass;
  F sb_b = fds_b * w.fmass;
  F qb_b = fdq_b * w.fmass;
  if (iptop < KX) fmass_b += cbmf_b;
  // fmass = fm0 * fpsa * min(5, qdif / (qmax - qb))
  const F A = w.fm0 * w.fpsa;
  const F A_b = fmass_b * w.mn;
  const F mn_b = fmass_b * A;
  const F fm0_b = A_b * w.fpsa;
  const F fpsa_b = A_b * w.fm0;
  const F ratio_b = mn_b * wmin(w.ratio, F(5.0));
  const F den = w.qmax - w.qb;
  const F qdif_b = ratio_b / den;
  const F den_b = -ratio_b * (w.ratio / den);
  qmax_b += den_b;
  qb_b -= den_b;
  // fpsa = psa * min(1, (psa - psmin) * rdps)
  b.psa += fpsa_b * w.mn2;
  const F y_b = fpsa_b * c.psa * wmin((c.psa - g.psmin) * w.rdps, F(1.0));
  b.psa += y_b * w.rdps;
  b.par[P_PSMIN] -= y_b * w.rdps;
  const F rdps_b = y_b * (c.psa - g.psmin);
  // qb = min(qb3[KX-1], q[KX-1]); sb = sb3[KX-1]
  qb3_b[KX - 1] += qb_b * wmin(w.qb3[KX - 1], c.q[KX - 1]);
  b.q[KX - 1] += qb_b * wmin(c.q[KX - 1], w.qb3[KX - 1]);
  sb3_b[KX - 1] += sb_b;
  SPD_LEVELS
  for (int k = 1; k < KX; ++k) {
    const F ww = F(vg.wvi[k - 1][1]);
    b.add_se(k - 1, sb3_b[k] - ww * sb3_b[k]);
    b.add_se(k, ww * sb3_b[k]);
    b.q[k - 1] += qb3_b[k] - ww * qb3_b[k];
    b.q[k] += ww * qb3_b[k];
  }
  // qmax = max(1.01 q[KX-1], qsat[KX-1])
  const F q101 = F(1.01) * c.q[KX - 1];
  b.q[KX - 1] += qmax_b * wmax(q101, c.qsat[KX - 1]) * F(1.01);
  b.qsat[KX - 1] += qmax_b * wmax(c.qsat[KX - 1], q101);
  // rdps = 2 / (1 - psmin); fm0 = c / (9.81 trcnv 3600)
  b.par[P_PSMIN] += rdps_b * (w.rdps / (F(1.0) - g.psmin));
  b.par[P_TRCNV] += -fm0_b * (w.fm0 / g.trcnv);
  return qdif_b;
}

// ---------------------------------------------------------------------------------------------
// get_large_scale_condensation_tendencies (large_scale_condensation.py:14-86)
// ---------------------------------------------------------------------------------------------
template <int KX, class F>
SPD_HD void lsc(const Ctx& x, const DiffParams<F>& g, Col<KX, F>& c, F* dt, F* dq) {
  const spd_vgrid_t& vg = *x.vg;
  const F rtlsc = F(1.0) / (g.trlsc * F(3600.0));
  const F tfact = F(2501.0 / 1004.0);
  const F prg = F(1e5 / 9.81);
  const F psa2 = c.psa * c.psa;
  F psum = F(0);
  int first = 0;
  SPD_LEVELS
  for (int k = 1; k < KX; ++k) {
    const F sig2 = F(vg.fsg[k]) * F(vg.fsg[k]);
    const F rhref = vmax(g.rhlsc + g.drhlsc * (sig2 - F(1.0)), g.rhblsc);
    const F dqmax = F(10.0) * sig2 * rtlsc;
    const F dqa = rhref * c.qsat[k] - c.q[k];
    F dql = F(0), dtl = F(0);
    if (dqa < F(0)) {
      dql = dqa * rtlsc;
      dtl = tfact * vmin(-dql, dqmax * psa2);
      if (first == 0) first = k;
    }
    dt[k] = dt[k] + dtl;
    dq[k] = dq[k] + dql;
    psum = psum + (F(vg.dhs[k]) * prg) * dql;
  }
  c.precls = (F(0) - psum) * c.psa;
  const int f1 = first == 0 ? 1 : first;
  c.iptop = f1 < c.iptop_cv ? f1 : c.iptop_cv;
}

template <int KX, class F>
SPD_HD void lsc_rev(const Ctx& x, const DiffParams<F>& g, const Col<KX, F>& c, const F* dt_b,
                    const F* dq_b, F precls_b, Bar<KX, F>& b) {
  const spd_vgrid_t& vg = *x.vg;
  const F rtlsc = F(1.0) / (g.trlsc * F(3600.0));
  const F tfact = F(2501.0 / 1004.0);
  const F prg = F(1e5 / 9.81);
  const F psa2 = c.psa * c.psa;
  F psum = F(0);
  F rtlsc_b = F(0), psa2_b = F(0);
  // precls = (0 - psum) * psa: psum is needed first
  SPD_LEVELS
  for (int k = 1; k < KX; ++k) {
    const F sig2 = F(vg.fsg[k]) * F(vg.fsg[k]);
    const F rhref = vmax(g.rhlsc + g.drhlsc * (sig2 - F(1.0)), g.rhblsc);
    const F dqa = rhref * c.qsat[k] - c.q[k];
    if (dqa < F(0)) psum = psum + (F(vg.dhs[k]) * prg) * (dqa * rtlsc);
  }
  b.psa += precls_b * (F(0) - psum);
  const F psum_b = -precls_b * c.psa;
  SPD_LEVELS
  for (int k = 1; k < KX; ++k) {
    const F sig2 = F(vg.fsg[k]) * F(vg.fsg[k]);
    const F X = g.rhlsc + g.drhlsc * (sig2 - F(1.0));
    const F rhref = vmax(X, g.rhblsc);
    const F dqmax = F(10.0) * sig2 * rtlsc;
    const F dqa = rhref * c.qsat[k] - c.q[k];
    if (!(dqa < F(0))) continue;
    const F dql = dqa * rtlsc;
    F dql_b = dq_b[k] + psum_b * (F(vg.dhs[k]) * prg);
    const F m_b = dt_b[k] * tfact;
    const F P = dqmax * psa2;
    dql_b += -m_b * wmin(-dql, P);
    const F P_b = m_b * wmin(P, -dql);
    const F dqmax_b = P_b * psa2;
    psa2_b += P_b * dqmax;
    const F dqa_b = dql_b * rtlsc;
    rtlsc_b += dql_b * dqa + dqmax_b * (F(10.0) * sig2);
    const F rhref_b = dqa_b * c.qsat[k];
    b.qsat[k] += dqa_b * rhref;
    b.q[k] -= dqa_b;
    const F X_b = rhref_b * wmax(X, g.rhblsc);
    b.par[P_RHBLSC] += rhref_b * wmax(g.rhblsc, X);
    b.par[P_RHLSC] += X_b;
    b.par[P_DRHLSC] += X_b * (sig2 - F(1.0));
  }
  b.psa += psa2_b * F(2) * c.psa;
  b.par[P_TRLSC] += -rtlsc_b * (rtlsc / g.trlsc);
}

// ---------------------------------------------------------------------------------------------
// clouds (shortwave_radiation.py:313-404)
// ---------------------------------------------------------------------------------------------
template <int KX, class F>
struct Cl {
  F upd[KX], pm[KX];
  uint32_t mk;
  F cloudc0, cmax, gse, pr1v, pr1, cc, Z, fstab_y, fstab_m, N, clstr1, clstrl_m;
  bool m0;
};

template <int KX, class F>
SPD_HD void clouds(const Ctx& x, Col<KX, F>& c, Cl<KX, F>& w, F fmask) {
  const spd_params_t& p = *x.p;
  const int nl1 = KX - 2;
  w.m0 = c.RH(nl1) > F(p.rhcl1);
  w.cloudc0 = w.m0 ? c.RH(nl1) - F(p.rhcl1) : F(0);
  const int icl0 = w.m0 ? nl1 : KX;
  w.mk = 0u;
  w.cmax = F(0);
  SPD_LEVELS
  for (int k = 2; k < KX - 2; ++k) {
    const F drh = c.RH(k) - F(p.rhcl1);
    const bool m = drh > w.cloudc0 && c.q[k] > F(p.qacl);
    if (m) w.mk |= 1u << k;
    w.upd[k] = m ? drh : w.cloudc0;
    w.cmax = (k == 2) ? w.upd[k] : vmax(w.cmax, w.upd[k]);
    w.pm[k] = w.cmax;
  }
  int icl = -1;
  SPD_LEVELS
  for (int k = 2; k < KX - 2; ++k) {
    const int cand = (w.cmax == w.upd[k]) ? (((w.mk >> k) & 1u) ? k : icl0) : icl0;
    icl = cand > icl ? cand : icl;
  }
  w.gse = (c.SE(KX - 2) - c.SE(KX - 1)) / (c.phi[KX - 2] - c.phi[KX - 1]);
  const F rrcl = F(1.0) / (F(p.rhcl2) - F(p.rhcl1));
  w.pr1v = F(86.4) * (c.precnv + c.precls);
  w.pr1 = vmin(F(p.pmaxcl), w.pr1v);
  w.cc = vmin(F(1.0), w.cmax * rrcl);
  w.Z = F(p.wpcl) * fsqrt(vmax(F(1e-9), w.pr1)) + w.cc * w.cc;
  F cloudc = vmin(F(1.0), w.Z);
  c.cloud_nan = fnan(cloudc);
  if (c.cloud_nan) cloudc = F(1.0);
  c.cloudc = cloudc;
  c.icltop = c.iptop < icl ? c.iptop : icl;
  c.qcloud = c.q[nl1];
  const F rgse = F(1.0) / (F(p.gse_s1) - F(p.gse_s0));
  w.fstab_y = rgse * (w.gse - F(p.gse_s0));
  w.fstab_m = vmax(w.fstab_y, F(0.0));
  const F fstab = vmin(w.fstab_m, F(1.0));
  w.N = vmax(F(p.clsmax) - F(1.2) * cloudc, F(0.0));
  w.clstr1 = fstab * w.N;
  w.clstrl_m = vmax(w.clstr1, F(p.clsminl));
  const F clstrl = w.clstrl_m * c.RH(KX - 1);
  c.clstr = w.clstr1 + fmask * (clstrl - w.clstr1);
}

template <int KX, class F>
SPD_HD void clouds_rev(const Ctx& x, const Col<KX, F>& c, const Cl<KX, F>& w, F fmask,
                       F cloudc_b, F clstr_b, F qcloud_b, F& precnv_b, F& precls_b,
                       Bar<KX, F>& b) {
  const spd_params_t& p = *x.p;
  const int nl1 = KX - 2;
  // clstr = clstr1 + fmask (clstrl - clstr1); clstrl = max(clstr1, clsminl) rh[KX-1]
  F clstr1_b = clstr_b - fmask * clstr_b;
  const F clstrl_b = fmask * clstr_b;
  b.add_rh(c, KX - 1, clstrl_b * w.clstrl_m);
  clstr1_b += clstrl_b * c.RH(KX - 1) * wmax(w.clstr1, F(p.clsminl));
  // clstr1 = fstab * max(clsmax - 1.2 cloudc, 0)
  const F fstab = vmin(w.fstab_m, F(1.0));
  const F fstab_b = clstr1_b * w.N;
  const F N_b = clstr1_b * fstab;
  cloudc_b += -F(1.2) * N_b * wmax(F(p.clsmax) - F(1.2) * c.cloudc, F(0.0));
  // fstab = min(max(rgse (gse - gse_s0), 0), 1)
  const F rgse = F(1.0) / (F(p.gse_s1) - F(p.gse_s0));
  const F y_b = fstab_b * wmin(w.fstab_m, F(1.0)) * wmax(w.fstab_y, F(0.0));
  const F gse_b = y_b * rgse;
  const F den = c.phi[KX - 2] - c.phi[KX - 1];
  const F a_b = gse_b / den;
  const F d_b = -gse_b * (w.gse / den);
  b.add_se(KX - 2, a_b);
  b.add_se(KX - 1, -(a_b));
  b.phi[KX - 2] += d_b;
  b.phi[KX - 1] -= d_b;
  b.q[nl1] += qcloud_b;
  if (c.cloud_nan) return;
  // cloudc = min(1, wpcl sqrt(max(1e-9, pr1)) + cc^2)
  const F Z_b = cloudc_b * wmin(w.Z, F(1.0));
  const F cc_b = Z_b * F(2) * w.cc;
  const F mx = vmax(F(1e-9), w.pr1);
  const F mx_b = Z_b * F(p.wpcl) * (F(0.5) / fsqrt(mx));
  const F pr1_b = mx_b * wmax(w.pr1, F(1e-9));
  const F v_b = pr1_b * wmin(w.pr1v, F(p.pmaxcl));
  precnv_b += v_b * F(86.4);
  precls_b += v_b * F(86.4);
  const F rrcl = F(1.0) / (F(p.rhcl2) - F(p.rhcl1));
  F cmax_b = cc_b * wmin(w.cmax * rrcl, F(1.0)) * rrcl;
  F cloudc0_b = F(0);
  SPD_LEVELS
  for (int k = KX - 3; k >= 2; --k) {
    F ub;
    if (k > 2) {
      ub = cmax_b * wmax(w.upd[k], w.pm[k - 1]);
      cmax_b = cmax_b * wmax(w.pm[k - 1], w.upd[k]);
    } else {
      ub = cmax_b;
    }
    if ((w.mk >> k) & 1u)
      b.add_rh(c, k, ub);
    else
      cloudc0_b += ub;
  }
  if (w.m0) b.add_rh(c, nl1, cloudc0_b);
}

// ---------------------------------------------------------------------------------------------
// shortwave_rad_fluxes (shortwave_radiation.py:27-217)
// ---------------------------------------------------------------------------------------------
template <int KX, class F>
struct Sw {
  F tau0[KX], tau1[KX], r[KX], f1v[KX], f2v[KX], upv[KX + 1], dfabs[KX];
  F psaz, acloud, mnq, f1a, f1b, f1;
};

struct SurfaceRow {
  float fsol, ozupp, ozone, zenit, stratz, sqrt_coa;
};

template <int KX, class F>
SPD_HD void shortwave(const Ctx& x, const DiffParams<F>& g, Col<KX, F>& c, const SurfaceRow& z,
                      Sw<KX, F>& w) {
  const spd_vgrid_t& vg = *x.vg;
  const spd_params_t& p = *x.p;
  const bool cmask = c.icltop < KX;
  SPD_LEVELS
  for (int k = 0; k < KX; ++k) w.r[k] = (((x.S >> k) & 1u) && cmask) ? g.albcl * c.cloudc : F(0);
  w.r[KX - 1] = g.albcls * c.clstr;
  w.psaz = c.psa * F(z.zenit);
  w.mnq = vmin(F(p.abscl1) * c.qcloud, F(p.abscl2));
  w.acloud = c.cloudc * w.mnq;
  w.tau0[0] = fexp(-w.psaz * F(vg.dhs[0]) * F(p.absdry));
  SPD_LEVELS
  for (int k = 1; k < KX - 1; ++k) {
    const F abs1 = F(p.absdry) + F(p.absaer) * (F(vg.fsg[k]) * F(vg.fsg[k]));
    const F cl = (k >= c.icltop) ? w.acloud : F(0) * w.acloud;
    w.tau0[k] = fexp(-w.psaz * F(vg.dhs[k]) * (abs1 + F(p.abswv1) * c.q[k] + cl));
  }
  {
    const F abs1 = F(p.absdry) + F(p.absaer) * (F(vg.fsg[KX - 1]) * F(vg.fsg[KX - 1]));
    w.tau0[KX - 1] = fexp(-w.psaz * F(vg.dhs[KX - 1]) * (abs1 + F(p.abswv1) * c.q[KX - 1]));
  }
  w.tau1[0] = F(1);
  SPD_LEVELS
  for (int k = 1; k < KX; ++k)
    w.tau1[k] = fexp(-w.psaz * F(vg.dhs[k]) * F(p.abswv2) * c.q[k]);
  F f1 = F(z.fsol) * F(0.95);
  w.dfabs[0] = f1;
  f1 = w.tau0[0] * (f1 - F(z.ozupp) * c.psa);
  w.f1a = f1;
  w.dfabs[0] = w.dfabs[0] + (-f1);
  w.dfabs[1] = f1;
  f1 = w.tau0[1] * (f1 - F(z.ozone) * c.psa);
  w.f1b = f1;
  w.dfabs[1] = w.dfabs[1] + (-f1);
  F rs[KX];
  rs[0] = w.r[0];
  rs[1] = w.r[1];
  SPD_LEVELS
  for (int k = 2; k < KX; ++k) {
    const F prev = f1;
    w.f1v[k] = prev;
    f1 = prev * w.tau0[k] * (F(1) - w.r[k]);
    w.dfabs[k] = prev * (F(1) - w.r[k]) * (F(1) - w.tau0[k]);
    rs[k] = w.r[k] * prev;
  }
  w.f1 = f1;
  F f2 = F(z.fsol) * F(0.05);
  SPD_LEVELS
  for (int k = 1; k < KX; ++k) {
    const F prev = f2;
    w.f2v[k] = prev;
    f2 = prev * w.tau1[k];
    w.dfabs[k] = w.dfabs[k] + prev * (F(1) - w.tau1[k]);
  }
  c.rsds = f1 + f2;
  F up = f1 * c.albsfc;
  w.upv[KX] = up;
  w.dfabs[KX - 1] = w.dfabs[KX - 1] + up * (F(1) - w.tau0[KX - 1]);
  SPD_LEVELS
  for (int k = KX - 1; k >= 1; --k) {
    up = up * w.tau0[k] + rs[k];
    w.upv[k] = up;
    w.dfabs[k - 1] = w.dfabs[k - 1] + up * (F(1) - w.tau0[k - 1]);
  }
  c.fsw0 = w.tau0[0] * up + w.r[0];
  c.fsw1 = f2;
}

template <int KX, class F>
SPD_HD void shortwave_rev(const Ctx& x, const DiffParams<F>& g, const Col<KX, F>& c,
                          const SurfaceRow& z, Sw<KX, F>& w, const F* dt_b, F rsds_b,
                          F fsw0_b, F fsw1_b, F& cloudc_b, F& clstr_b, F& qcloud_b,
                          Bar<KX, F>& b) {
  const spd_vgrid_t& vg = *x.vg;
  const spd_params_t& p = *x.p;
  const bool swon = (x.model_step % 3) == 0;
  F dfabs_b[KX], tau0_b[KX], tau1_b[KX], r_b[KX], rs_b[KX];
  SPD_LEVELS
  for (int k = 0; k < KX; ++k) {
    dfabs_b[k] = F(0);
    if (swon) {
      dfabs_b[k] = dt_b[k] * F(vg.grdscp[k]) / c.psa;
      b.psa += -dt_b[k] * ((w.dfabs[k] * F(vg.grdscp[k])) / c.psa) / c.psa;
    }
    tau0_b[k] = tau1_b[k] = r_b[k] = rs_b[k] = F(0);
  }
  F f2_b = fsw1_b + rsds_b;
  F f1_b = rsds_b;
  // flux_sw0 = tau0[0] up + r[0]
  tau0_b[0] += fsw0_b * w.upv[1];
  F up_b = fsw0_b * w.tau0[0];
  r_b[0] += fsw0_b;
  SPD_LEVELS
  for (int k = 1; k < KX; ++k) {
    up_b += dfabs_b[k - 1] * (F(1) - w.tau0[k - 1]);
    tau0_b[k - 1] -= dfabs_b[k - 1] * w.upv[k];
    tau0_b[k] += up_b * w.upv[k + 1];
    rs_b[k] += up_b;
    up_b = up_b * w.tau0[k];
  }
  up_b += dfabs_b[KX - 1] * (F(1) - w.tau0[KX - 1]);
  tau0_b[KX - 1] -= dfabs_b[KX - 1] * w.upv[KX];
  f1_b += up_b * c.albsfc;
  SPD_LEVELS
  for (int k = KX - 1; k >= 1; --k) {
    tau1_b[k] += f2_b * w.f2v[k] - dfabs_b[k] * w.f2v[k];
    f2_b = f2_b * w.tau1[k] + dfabs_b[k] * (F(1) - w.tau1[k]);
  }
  r_b[1] += rs_b[1];
  r_b[0] += rs_b[0];
  SPD_LEVELS
  for (int k = KX - 1; k >= 2; --k) {
    const F prev = w.f1v[k];
    const F om = F(1) - w.r[k];
    const F t0 = w.tau0[k];
    const F prev_b = rs_b[k] * w.r[k] + dfabs_b[k] * om * (F(1) - t0) + f1_b * t0 * om;
    r_b[k] += rs_b[k] * prev - dfabs_b[k] * prev * (F(1) - t0) - f1_b * prev * t0;
    tau0_b[k] += -dfabs_b[k] * prev * om + f1_b * prev * om;
    f1_b = prev_b;
  }
  {  // level 1: dfabs[1] = f1a; f1b = tau0[1] (f1a - ozone psa); dfabs[1] -= f1b
    const F fb_b = f1_b - dfabs_b[1];
    tau0_b[1] += fb_b * (w.f1a - F(z.ozone) * c.psa);
    const F gg = fb_b * w.tau0[1];
    b.psa -= gg * F(z.ozone);
    f1_b = gg + dfabs_b[1];
  }
  {  // level 0: f1a = tau0[0] (fsol 0.95 - ozupp psa); dfabs[0] = fsol 0.95 - f1a
    const F fa_b = f1_b - dfabs_b[0];
    const F f10 = F(z.fsol) * F(0.95);
    tau0_b[0] += fa_b * (f10 - F(z.ozupp) * c.psa);
    b.psa -= fa_b * w.tau0[0] * F(z.ozupp);
  }
  F psaz_b = F(0), acloud_b = F(0);
  SPD_LEVELS
  for (int k = 1; k < KX; ++k) {
    const F Eb = tau1_b[k] * w.tau1[k];
    const F c0 = F(vg.dhs[k]) * F(p.abswv2);
    b.q[k] += Eb * (-w.psaz * c0);
    psaz_b += -Eb * c0 * c.q[k];
  }
  psaz_b += -tau0_b[0] * w.tau0[0] * F(vg.dhs[0]) * F(p.absdry);
  SPD_LEVELS
  for (int k = 1; k < KX; ++k) {
    const F Eb = tau0_b[k] * w.tau0[k];
    const F abs1 = F(p.absdry) + F(p.absaer) * (F(vg.fsg[k]) * F(vg.fsg[k]));
    const bool cl = (k < KX - 1) && (k >= c.icltop);
    const F inner = abs1 + F(p.abswv1) * c.q[k] + (cl ? w.acloud : F(0));
    psaz_b += -Eb * F(vg.dhs[k]) * inner;
    const F ib = Eb * (-w.psaz * F(vg.dhs[k]));
    b.q[k] += ib * F(p.abswv1);
    if (cl) acloud_b += ib;
  }
  cloudc_b += acloud_b * w.mnq;
  qcloud_b += acloud_b * c.cloudc * wmin(F(p.abscl1) * c.qcloud, F(p.abscl2)) * F(p.abscl1);
  b.psa += psaz_b * F(z.zenit);
  b.par[P_ALBCLS] += r_b[KX - 1] * c.clstr;
  clstr_b += r_b[KX - 1] * g.albcls;
  const bool cmask = c.icltop < KX;
  SPD_LEVELS
  for (int k = 0; k < KX - 1; ++k) {
    if (((x.S >> k) & 1u) && cmask) {
      b.par[P_ALBCL] += r_b[k] * c.cloudc;
      cloudc_b += r_b[k] * g.albcl;
    }
  }
}

// ---------------------------------------------------------------------------------------------
// longwave: transmissivities (shortwave_radiation.py:174-206), blackbody fluxes, the downward
// pass (longwave_radiation.py:16-117) and the upward pass (:119-202)
// ---------------------------------------------------------------------------------------------
template <int KX, class F>
struct Lw {
  F fld[KX][4];      // downward pass: fluxes after level k
  F flu[KX + 1][4];  // upward pass: fluxes entering level k from below (flu[KX]: surface)
};

// One level's transmissivities and blackbody terms, recomputed wherever they are needed.
template <class F>
struct LwLevel {
  F tau[4], st0, st1;
};

template <int KX, class F>
SPD_HD void lw_absorb(const Ctx& x, const Col<KX, F>& c, int k, F ablco2, F a[4]) {
  const spd_params_t& p = *x.p;
  const F acl1 = c.cloudc * F(p.ablcl1), acl2 = c.cloudc * F(p.ablcl2);
  F a0 = F(p.ablwin), a2 = F(p.ablwv1) * c.q[k], a3 = F(p.ablwv2) * c.q[k];
  if (k == 0) a2 = a3 = F(0);
  if (k >= 2 && k <= KX - 2) {
    a0 = a0 + ((k > c.icltop) ? acl1 : acl2);
    a2 = vmax(a2, acl2);
    a3 = vmax(a3, acl2);
  }
  a[0] = a0;
  a[1] = ablco2;
  a[2] = a2;
  a[3] = a3;
}

// half-level temperature (longwave_radiation.py: interpolation to the layer interfaces)
template <int KX, class F>
SPD_HD F lw_th(const Ctx& x, const Col<KX, F>& c, int k) {
  return c.t[k] + F(x.vg->wvi[k][1]) * (c.t[k + 1] - c.t[k]);
}

template <int KX, class F>
SPD_HD void lw_level(const Ctx& x, const Col<KX, F>& c, int k, F ablco2, LwLevel<F>& L) {
  F a[4];
  lw_absorb(x, c, k, ablco2, a);
  const F dh = F(x.vg->dhs[k]);
  SPD_BANDS
  for (int b = 0; b < 4; ++b) L.tau[b] = fexp(-a[b] * c.psa * dh);
  const F sbc = F(5.67e-8);
  if (k == 0) {
    const F s10 = F(0.75) * c.t[0] + F(0.25) * lw_th(x, c, 0);
    L.st0 = sbc * ((s10 * s10) * (s10 * s10));
    L.st1 = F(0);
  } else if (k == 1) {
    const F s11 = F(0.50) * c.t[1] + F(0.25) * (lw_th(x, c, 0) + lw_th(x, c, 1));
    L.st0 = sbc * ((s11 * s11) * (s11 * s11));
    L.st1 = F(0);
  } else {
    const F grad = (k < KX - 1) ? F(0.5) * vmax(lw_th(x, c, k) - lw_th(x, c, k - 1), F(0.0))
                                : vmax(c.t[KX - 1] - lw_th(x, c, KX - 2), F(0.0));
    const F st3 = sbc * (c.t[k] * c.t[k] * c.t[k]);
    L.st0 = st3 * c.t[k];
    L.st1 = F(4.0) * st3 * grad;
  }
}

template <int KX, class F>
SPD_HD void longwave_down(const Ctx& x, Col<KX, F>& c, F ablco2, Lw<KX, F>& w) {
  const spd_params_t& p = *x.p;
  F fb[4], dfb[4];
  LwLevel<F> L;
  lw_level(x, c, 0, ablco2, L);
  radset_d(c.t[0], F(p.epslw), fb, dfb);
  SPD_BANDS
  for (int b = 0; b < 4; ++b) {
    const F emis = F(1) - L.tau[b];
    w.fld[0][b] = emis * (fb[b] * (L.st0 + emis * L.st1));
  }
  w.fld[0][2] = w.fld[0][3] = F(0);
  F sprev = ((w.fld[0][0] + w.fld[0][1]) + w.fld[0][2]) + w.fld[0][3];
  c.dfl[0] = F(0) + (-sprev);
  F st0_last = L.st0;
  SPD_LEVELS
  for (int k = 1; k < KX; ++k) {
    lw_level(x, c, k, ablco2, L);
    radset_d(c.t[k], F(p.epslw), fb, dfb);
    SPD_BANDS
    for (int b = 0; b < 4; ++b) {
      const F emis = F(1) - L.tau[b];
      w.fld[k][b] = L.tau[b] * w.fld[k - 1][b] + emis * (fb[b] * (L.st0 + emis * L.st1));
    }
    const F sk = ((w.fld[k][0] + w.fld[k][1]) + w.fld[k][2]) + w.fld[k][3];
    c.dfl[k] = F(0) + (-(sk - sprev));
    sprev = sk;
    st0_last = L.st0;
  }
  const F e = F(p.emisfc);
  const F* fl = w.fld[KX - 1];
  F rlds = ((e * fl[0] + e * fl[1]) + e * fl[2]) + e * fl[3];
  const F corlw = F(p.epslw) * F(p.emisfc) * st0_last;
  c.dfl[KX - 1] = c.dfl[KX - 1] + (-corlw);
  c.rlds = rlds + corlw;
}

template <int KX, class F>
SPD_HD void longwave_up(const Ctx& x, Col<KX, F>& c, const SurfaceRow& z, F ablco2,
                        Lw<KX, F>& w) {
  const spd_vgrid_t& vg = *x.vg;
  const spd_params_t& p = *x.p;
  const F refsfc = F(1) - F(p.emisfc);
  F fb[4], dfb[4];
  LwLevel<F> L;
  radset_d(c.tsfc, F(p.epslw), fb, dfb);
  const F fsw[4] = {c.fsw0, c.fsw1, F(0), F(0)};
  SPD_BANDS
  for (int b = 0; b < 4; ++b) w.flu[KX][b] = fb[b] * c.rlus2 + refsfc * fsw[b];
  c.dfl[KX - 1] = c.dfl[KX - 1] + F(p.epslw) * c.rlus2;
  F sk = ((w.flu[KX][0] + w.flu[KX][1]) + w.flu[KX][2]) + w.flu[KX][3];
  SPD_LEVELS
  for (int k = KX - 1; k >= 1; --k) {
    lw_level(x, c, k, ablco2, L);
    radset_d(c.t[k], F(p.epslw), fb, dfb);
    SPD_BANDS
    for (int b = 0; b < 4; ++b) {
      const F emis = F(1) - L.tau[b];
      w.flu[k][b] = L.tau[b] * w.flu[k + 1][b] + emis * (fb[b] * (L.st0 - emis * L.st1));
    }
    const F skm1 = ((w.flu[k][0] + w.flu[k][1]) + w.flu[k][2]) + w.flu[k][3];
    c.dfl[k] = c.dfl[k] + (sk - skm1);
    sk = skm1;
  }
  lw_level(x, c, 0, ablco2, L);
  radset_d(c.t[0], F(p.epslw), fb, dfb);
  F top[2];
  SPD_BANDS
  for (int b = 0; b < 2; ++b) {
    const F emis = F(1) - L.tau[b];
    top[b] = L.tau[b] * w.flu[1][b] + emis * (fb[b] * (L.st0 - emis * L.st1));
  }
  c.dfl[0] = c.dfl[0] + ((w.flu[1][0] - top[0]) + (w.flu[1][1] - top[1]));
  LwLevel<F> L1;
  lw_level(x, c, 1, ablco2, L1);
  const F eps1 = F(p.epslw) / (F(vg.dhs[0]) + F(vg.dhs[1]));
  const F stratc0 = F(z.stratz) * c.psa, stratc1 = eps1 * c.psa;
  const F corlw1 = F(vg.dhs[0]) * stratc1 * L.st0 + stratc0;
  const F corlw2 = F(vg.dhs[1]) * stratc1 * L1.st0;
  c.dfl[0] = c.dfl[0] + (-corlw1);
  c.dfl[1] = c.dfl[1] + (-corlw2);
}

// One radiative step of the reverse: U = tau Uprev + emis (fb (st0 + sgn emis st1)).
template <class F>
SPD_HD void lw_step_rev(F Ub, F tau, F uprev, F fb, F dfb, F st0, F st1, F sgn, F& tau_b,
                        F& uprev_b, F& t_b, F& st0_b, F& st1_b) {
  const F emis = F(1) - tau;
  const F H = st0 + sgn * emis * st1;
  const F G = fb * H;
  tau_b += Ub * uprev;
  uprev_b = Ub * tau;
  F e_b = Ub * G;
  const F G_b = Ub * emis;
  t_b += G_b * H * dfb;
  const F H_b = G_b * fb;
  st0_b += H_b;
  e_b += sgn * H_b * st1;
  st1_b += sgn * H_b * emis;
  tau_b -= e_b;
}

// Applies the adjoints of level k's transmissivities and blackbody terms at once (they enter
// linearly): to psa, q[k], T around level k and the two cloud absorption factors.
template <int KX, class F>
SPD_HD void lw_level_rev(const Ctx& x, const Col<KX, F>& c, int k, F ablco2,
                         const LwLevel<F>& L, const F tau_b[4], F st0_b, F st1_b, F& acl1_b,
                         F& acl2_b, Bar<KX, F>& b) {
  const spd_params_t& p = *x.p;
  F a[4];
  lw_absorb(x, c, k, ablco2, a);
  const F dh = F(x.vg->dhs[k]);
  F ab[4];
  SPD_BANDS
  for (int bb = 0; bb < 4; ++bb) {
    const F Eb = tau_b[bb] * L.tau[bb];
    ab[bb] = -Eb * c.psa * dh;
    b.psa += -Eb * a[bb] * dh;
  }
  if (k >= 2 && k <= KX - 2) {
    if (k > c.icltop)
      acl1_b += ab[0];
    else
      acl2_b += ab[0];
    const F acl2 = c.cloudc * F(p.ablcl2);
    const F q1 = F(p.ablwv1) * c.q[k], q2 = F(p.ablwv2) * c.q[k];
    b.q[k] += ab[2] * wmax(q1, acl2) * F(p.ablwv1) + ab[3] * wmax(q2, acl2) * F(p.ablwv2);
    acl2_b += ab[2] * wmax(acl2, q1) + ab[3] * wmax(acl2, q2);
  } else if (k > 0) {
    b.q[k] += ab[2] * F(p.ablwv1) + ab[3] * F(p.ablwv2);
  }
  // blackbody terms; th_j = t_j + w_j (t_{j+1} - t_j)
  const F sbc = F(5.67e-8);
  auto add_th = [&](int j, F v) {
    const F ww = F(x.vg->wvi[j][1]);
    b.t[j] += v - ww * v;
    b.t[j + 1] += ww * v;
  };
  if (k == 0) {
    const F s10 = F(0.75) * c.t[0] + F(0.25) * lw_th(x, c, 0);
    const F s10_b = st0_b * sbc * F(4) * (s10 * s10 * s10);
    b.t[0] += F(0.75) * s10_b;
    add_th(0, F(0.25) * s10_b);
  } else if (k == 1) {
    const F s11 = F(0.50) * c.t[1] + F(0.25) * (lw_th(x, c, 0) + lw_th(x, c, 1));
    const F s11_b = st0_b * sbc * F(4) * (s11 * s11 * s11);
    b.t[1] += F(0.50) * s11_b;
    add_th(0, F(0.25) * s11_b);
    add_th(1, F(0.25) * s11_b);
  } else {
    const F t = c.t[k];
    const F st3 = sbc * (t * t * t);
    const F dd = (k < KX - 1) ? lw_th(x, c, k) - lw_th(x, c, k - 1)
                              : c.t[KX - 1] - lw_th(x, c, KX - 2);
    const F grad = (k < KX - 1) ? F(0.5) * vmax(dd, F(0.0)) : vmax(dd, F(0.0));
    const F st3_b = st0_b * t + st1_b * F(4.0) * grad;
    b.t[k] += st0_b * st3 + st3_b * F(3) * sbc * t * t;
    const F grad_b = st1_b * F(4.0) * st3;
    const F d_b = grad_b * ((k < KX - 1) ? F(0.5) : F(1)) * wmax(dd, F(0.0));
    if (k < KX - 1) {
      add_th(k, d_b);
      add_th(k - 1, -d_b);
    } else {
      b.t[KX - 1] += d_b;
      add_th(KX - 2, -d_b);
    }
  }
}

// First half of the longwave reverse: the flux divergence's psa factor and the upward pass.
// Gives the adjoints of the surface's upward flux rlus2 and of the two shortwave fluxes the
// pass starts from; adds the cloud factors' adjoints to acl1_b, acl2_b.
template <int KX, class F>
SPD_HD void longwave_rev_up(const Ctx& x, const Col<KX, F>& c, const SurfaceRow& z,
                            const Lw<KX, F>& w, F ablco2, const F* dt_b, F& rlus2_b, F& fsw0_b,
                            F& fsw1_b, F& acl1_b, F& acl2_b, Bar<KX, F>& b) {
  const spd_vgrid_t& vg = *x.vg;
  const spd_params_t& p = *x.p;
  auto dflb = [&](int k) { return dt_b[k] * F(vg.grdscp[k]) / c.psa; };
  SPD_LEVELS
  for (int k = 0; k < KX; ++k) b.psa += -dt_b[k] * ((c.dfl[k] * F(vg.grdscp[k])) / c.psa) / c.psa;
  F st0b_0, st0b_1;
  {
    const F corlw1_b = -dflb(0), corlw2_b = -dflb(1);
    LwLevel<F> L0, L1;
    lw_level(x, c, 0, ablco2, L0);
    lw_level(x, c, 1, ablco2, L1);
    const F eps1 = F(p.epslw) / (F(vg.dhs[0]) + F(vg.dhs[1]));
    const F stratc1 = eps1 * c.psa;
    const F stratc1_b = corlw1_b * F(vg.dhs[0]) * L0.st0 + corlw2_b * F(vg.dhs[1]) * L1.st0;
    st0b_0 = corlw1_b * (F(vg.dhs[0]) * stratc1);
    st0b_1 = corlw2_b * (F(vg.dhs[1]) * stratc1);
    b.psa += corlw1_b * F(z.stratz) + stratc1_b * eps1;
  }
  F Ub[4] = {dflb(0), dflb(0), F(0), F(0)};
  F fb[4], dfb[4];
  LwLevel<F> L;
  {
    lw_level(x, c, 0, ablco2, L);
    radset_d(c.t[0], F(p.epslw), fb, dfb);
    F tb[4] = {F(0), F(0), F(0), F(0)};
    F s0b = st0b_0, s1b = F(0);
    SPD_BANDS
    for (int bb = 0; bb < 2; ++bb) {
      F ub_prev;
      lw_step_rev(-dflb(0), L.tau[bb], w.flu[1][bb], fb[bb], dfb[bb], L.st0, L.st1, F(-1),
                  tb[bb], ub_prev, b.t[0], s0b, s1b);
      Ub[bb] += ub_prev;
    }
    lw_level_rev(x, c, 0, ablco2, L, tb, s0b, s1b, acl1_b, acl2_b, b);
  }
  SPD_LEVELS
  for (int k = 1; k < KX; ++k) {
    const F Sb = (k >= 2 ? dflb(k - 1) : F(0)) - dflb(k);
    lw_level(x, c, k, ablco2, L);
    radset_d(c.t[k], F(p.epslw), fb, dfb);
    F tb[4] = {F(0), F(0), F(0), F(0)};
    F s0b = (k == 1) ? st0b_1 : F(0), s1b = F(0);
    SPD_BANDS
    for (int bb = 0; bb < 4; ++bb) {
      F nb;
      lw_step_rev(Ub[bb] + Sb, L.tau[bb], w.flu[k + 1][bb], fb[bb], dfb[bb], L.st0, L.st1,
                  F(-1), tb[bb], nb, b.t[k], s0b, s1b);
      Ub[bb] = nb;
    }
    lw_level_rev(x, c, k, ablco2, L, tb, s0b, s1b, acl1_b, acl2_b, b);
  }
  const F refsfc = F(1) - F(p.emisfc);
  F fbs[4], dfbs[4];
  radset_d(c.tsfc, F(p.epslw), fbs, dfbs);
  rlus2_b = dflb(KX - 1) * F(p.epslw);
  SPD_BANDS
  for (int bb = 0; bb < 4; ++bb) {
    const F u = Ub[bb] + dflb(KX - 1);
    rlus2_b += u * fbs[bb];
    if (bb == 0) fsw0_b = u * refsfc;
    if (bb == 1) fsw1_b = u * refsfc;
  }
}

// Second half: the downward pass (given the adjoint of the surface's downward flux rlds) with
// each level's transmissivities and blackbody terms.
template <int KX, class F>
SPD_HD void longwave_rev_down(const Ctx& x, const Col<KX, F>& c, const Lw<KX, F>& w, F ablco2,
                              const F* dt_b, F rlds_b, F& acl1_b, F& acl2_b, Bar<KX, F>& b) {
  const spd_vgrid_t& vg = *x.vg;
  const spd_params_t& p = *x.p;
  auto dflb = [&](int k) { return dt_b[k] * F(vg.grdscp[k]) / c.psa; };
  const F corlw_b = rlds_b - dflb(KX - 1);
  F Db[4];
  SPD_BANDS
  for (int bb = 0; bb < 4; ++bb) Db[bb] = rlds_b * F(p.emisfc);
  F fb[4], dfb[4];
  LwLevel<F> L;
  SPD_LEVELS
  for (int k = KX - 1; k >= 0; --k) {
    const F Sb = -dflb(k) + (k < KX - 1 ? dflb(k + 1) : F(0));
    lw_level(x, c, k, ablco2, L);
    radset_d(c.t[k], F(p.epslw), fb, dfb);
    F tb[4] = {F(0), F(0), F(0), F(0)};
    F s0b = (k == KX - 1) ? corlw_b * (F(p.epslw) * F(p.emisfc)) : F(0), s1b = F(0);
    const int nb_ = (k == 0) ? 2 : 4;
    SPD_BANDS
    for (int bb = 0; bb < 4; ++bb) {
      if (bb >= nb_) continue;
      F nb;
      const F prev = (k == 0) ? F(0) : w.fld[k - 1][bb];
      lw_step_rev(Db[bb] + Sb, L.tau[bb], prev, fb[bb], dfb[bb], L.st0, L.st1, F(1), tb[bb],
                  nb, b.t[k], s0b, s1b);
      Db[bb] = nb;
    }
    lw_level_rev(x, c, k, ablco2, L, tb, s0b, s1b, acl1_b, acl2_b, b);
  }
}

// ---------------------------------------------------------------------------------------------
// get_surface_fluxes (surface_flux.py:15-300)
// ---------------------------------------------------------------------------------------------
template <class F>
struct Sf {
  bool warm, tsk_gt, sst_gt, evap_pos;
  F u0, v0, dt1, t1_0p, t1_1p, t2_1, t2_0, t1_0, t1_1, t0, A, B, denv0;
  F tskin, dthl_v, denv1, cdldv, forog, qs10, qs10_t, qs10_p, q1_0, qs00, qs00_t, qs00_p;
  F Mv, evap0a, tsk3, drls, rlus0a, qs01r, qs01r_t, qs01r_p, qs01, den, dtskin, hfl0;
  F dths_v, denv2, qs11, qs11_t, qs11_p, q1_1, cdsdv, qss, qss_t, qss_p;
  F ustr0, vstr0, shf0, evap0, rlus0, ustr1, vstr1, shf1, evap1;
  F ustr2, vstr2, shf2, evap2, rps;
};

struct SurfaceIn {
  float sst, stl, soilw, snowc, sice, alb0, fmask, orog, phis0;
};

template <int KX, class F>
SPD_HD void surface(const Ctx& x, Col<KX, F>& c, const SurfaceIn& s, const SurfaceRow& z,
                    Sf<F>& w) {
  const spd_vgrid_t& vg = *x.vg;
  const spd_params_t& p = *x.p;
  const F esbc = F(p.emisfc) * F(5.67e-8);
  const F ta1 = c.t[KX - 1], ta2 = c.t[KX - 2];
  const F phi0 = F(s.orog) * F(9.81);
  w.u0 = F(p.fwind0) * c.u;
  w.v0 = F(p.fwind0) * c.v;
  const F astab = (x.flags & SPD_LSCASYM) ? F(0.5) : F(1.0);
  const F rdth = F(p.fstab) / F(p.dtheta);
  const bool land = (x.flags & SPD_LFLUXLAND) != 0;
  w.ustr0 = w.ustr1 = w.vstr0 = w.vstr1 = w.shf0 = w.evap0 = w.rlus0 = F(0);
  w.t1_1 = w.q1_1 = w.denv2 = F(0);
  c.rlus2 = F(0);
  c.tsfc = F(0);
  w.ustr2 = w.vstr2 = w.shf2 = w.evap2 = F(0);
  w.rps = F(1) / c.psa;
  if (!land) return;
  const F rcp = F(1.0 / 1004.0);
  w.dt1 = F(vg.wvi[KX - 1][1]) * (ta1 - ta2);
  w.t1_0p = F(0) + (ta1 + w.dt1);
  w.t1_1p = w.t1_0p - phi0 * w.dt1 / (F(2.0 / 7.0 * 1004.0 * 288.0) * F(vg.sigl[KX - 1]));
  w.t2_1 = ta1 + rcp * c.phi[KX - 1];
  w.t2_0 = w.t2_1 - rcp * phi0;
  w.warm = ta1 > ta2;
  if (w.warm) {
    w.t1_0 = F(p.ftemp0) * w.t1_0p + (F(1) - F(p.ftemp0)) * w.t2_0;
    w.t1_1 = F(p.ftemp0) * w.t1_1p + (F(1) - F(p.ftemp0)) * w.t2_1;
  } else {
    w.t1_0 = ta1;
    w.t1_1 = ta1;
  }
  w.t0 = w.t1_1 + F(s.fmask) * (w.t1_0 - w.t1_1);
  w.A = F(1e5) * c.psa / (F(2.0 / 7.0 * 1004.0) * w.t0);
  w.B = fsqrt(w.u0 * w.u0 + w.v0 * w.v0 + F(p.vgust) * F(p.vgust));
  w.denv0 = w.A * w.B;
  const F kts = F(p.ctday) * F(z.sqrt_coa);
  w.tskin = F(s.stl) + kts * c.rsds * (F(1) - c.alb_l) * c.psa;
  w.tsk_gt = w.tskin > w.t2_0;
  w.dthl_v = w.tsk_gt ? vmin(F(p.dtheta), w.tskin - w.t2_0)
                      : vmax(-F(p.dtheta), astab * (w.tskin - w.t2_0));
  w.denv1 = w.denv0 * (F(1) + w.dthl_v * rdth);
  const F rhdrag = F(1) / (F(9.81) * F(p.hdrag));
  const F ph = F(s.phis0) > F(0) ? F(s.phis0) : F(0);
  w.forog = F(1) + rhdrag * (F(1) - fexp(-ph * rhdrag));
  w.cdldv = F(p.cdl) * w.denv0 * w.forog;
  w.ustr0 = -w.cdldv * c.u;
  w.vstr0 = -w.cdldv * c.v;
  const F chlcp = F(p.chl) * F(1004.0);
  w.shf0 = chlcp * w.denv1 * (w.tskin - w.t1_0);
  const bool fh = F(p.fhum0) > F(0);
  w.qs10 = qsat_d(w.t1_0, c.psa, F(1), w.qs10_t, w.qs10_p);
  w.q1_0 = fh ? F(p.fhum0) * (c.RH(KX - 1) * w.qs10) + (F(1) - F(p.fhum0)) * c.q[KX - 1]
              : c.q[KX - 1];
  w.qs00 = qsat_d(w.tskin, c.psa, F(1), w.qs00_t, w.qs00_p);
  w.Mv = F(s.soilw) * w.qs00 - w.q1_0;
  w.evap0 = F(p.chl) * w.denv1 * vmax(F(0), w.Mv);
  w.evap0a = w.evap0;
  w.tsk3 = w.tskin * w.tskin * w.tskin;
  w.drls = F(4.0) * esbc * w.tsk3;
  w.rlus0 = esbc * w.tsk3 * w.tskin;
  w.rlus0a = w.rlus0;
  w.hfl0 = c.rsds * (F(1) - c.alb_l) + c.rlds - (w.rlus0 + w.shf0 + (F(2501.0) * w.evap0));
  if (x.flags & SPD_LSKINEB) {
    const F clamb = F(p.clambda) + (c.snowc * (F(p.clambsn) - F(p.clambda)));
    w.hfl0 = w.hfl0 - (clamb * (w.tskin - F(s.stl)));
    w.qs01r = qsat_d(w.tskin + F(1), c.psa, F(1), w.qs01r_t, w.qs01r_p);
    w.evap_pos = w.evap0 > F(0);
    w.qs01 = w.evap_pos ? F(s.soilw) * (w.qs01r - w.qs00) : F(0);
    w.den = clamb + w.drls + (F(p.chl) * w.denv1 * (F(1004.0) + (F(2501.0) * w.qs01)));
    w.dtskin = w.hfl0 / w.den;
    w.shf0 = w.shf0 + chlcp * w.denv1 * w.dtskin;
    w.evap0 = w.evap0 + F(p.chl) * w.denv1 * w.qs01 * w.dtskin;
    w.rlus0 = w.rlus0 + w.drls * w.dtskin;
  }
  w.sst_gt = F(s.sst) > w.t2_1;
  w.dths_v = w.sst_gt ? vmin(F(p.dtheta), F(s.sst) - w.t2_1)
                      : vmax(-F(p.dtheta), astab * (F(s.sst) - w.t2_1));
  w.denv2 = w.denv0 * (F(1) + w.dths_v * rdth);
  w.qs11 = qsat_d(w.t1_1, c.psa, F(1), w.qs11_t, w.qs11_p);
  w.q1_1 = fh ? F(p.fhum0) * (c.RH(KX - 1) * w.qs11) + (F(1) - F(p.fhum0)) * c.q[KX - 1]
              : c.q[KX - 1];
  w.cdsdv = F(p.cds) * w.denv2;
  w.ustr1 = -w.cdsdv * c.u;
  w.vstr1 = -w.cdsdv * c.v;
  w.shf1 = F(p.chs) * F(1004.0) * w.denv2 * (F(s.sst) - w.t1_1);
  w.qss = qsat_d(F(s.sst), c.psa, F(1), w.qss_t, w.qss_p);
  w.evap1 = F(p.chs) * w.denv2 * (w.qss - w.q1_1);
  const F rlus1 = esbc * ((F(s.sst) * F(s.sst)) * (F(s.sst) * F(s.sst)));
  const F fm = F(s.fmask);
  w.ustr2 = w.ustr1 + fm * (w.ustr0 - w.ustr1);
  w.vstr2 = w.vstr1 + fm * (w.vstr0 - w.vstr1);
  w.shf2 = w.shf1 + fm * (w.shf0 - w.shf1);
  w.evap2 = w.evap1 + fm * (w.evap0 - w.evap1);
  c.rlus2 = rlus1 + fm * (w.rlus0 - rlus1);
  c.tsfc = F(s.sst) + fm * (F(s.stl) - F(s.sst));
}

template <int KX, class F>
SPD_HD void surface_tend(const Ctx& x, const Sf<F>& w, F* dt, F* dq, F& du, F& dv) {
  const spd_vgrid_t& vg = *x.vg;
  du = F(0) + w.ustr2 * w.rps * F(vg.grdsig[KX - 1]);
  dv = F(0) + w.vstr2 * w.rps * F(vg.grdsig[KX - 1]);
  dt[KX - 1] = dt[KX - 1] + (F(0) + w.shf2 * w.rps * F(vg.grdscp[KX - 1]));
  dq[KX - 1] = dq[KX - 1] + (F(0) + w.evap2 * w.rps * F(vg.grdsig[KX - 1]));
}

template <int KX, class F>
SPD_HD void surface_rev(const Ctx& x, const Col<KX, F>& c, const SurfaceIn& s,
                        const SurfaceRow& z, const Sf<F>& w, F du_b, F dv_b, F dtK_b, F dqK_b,
                        F rlus2_b, F& rsds_b, F& rlds_b, Bar<KX, F>& b) {
  const spd_vgrid_t& vg = *x.vg;
  const spd_params_t& p = *x.p;
  if (!(x.flags & SPD_LFLUXLAND)) return;  // every flux is a constant zero
  const F esbc = F(p.emisfc) * F(5.67e-8);
  const F astab = (x.flags & SPD_LSCASYM) ? F(0.5) : F(1.0);
  const F rdth = F(p.fstab) / F(p.dtheta);
  const F chlcp = F(p.chl) * F(1004.0);
  const F gs = F(vg.grdsig[KX - 1]), gc = F(vg.grdscp[KX - 1]);
  const F rps_b = du_b * w.ustr2 * gs + dv_b * w.vstr2 * gs + dtK_b * w.shf2 * gc +
                  dqK_b * w.evap2 * gs;
  b.psa += -rps_b * (w.rps / c.psa);
  const F ustr2_b = du_b * gs * w.rps, vstr2_b = dv_b * gs * w.rps;
  const F shf2_b = dtK_b * gc * w.rps, evap2_b = dqK_b * gs * w.rps;
  const F fm = F(s.fmask);
  F ustr0_b = ustr2_b * fm, ustr1_b = ustr2_b - fm * ustr2_b;
  F vstr0_b = vstr2_b * fm, vstr1_b = vstr2_b - fm * vstr2_b;
  F shf0_b = shf2_b * fm, shf1_b = shf2_b - fm * shf2_b;
  F evap0_b = evap2_b * fm, evap1_b = evap2_b - fm * evap2_b;
  F rlus0_b = rlus2_b * fm;
  F denv2_b = F(0), denv1_b = F(0), denv0_b = F(0), t1_1_b = F(0), t1_0_b = F(0);
  F tskin_b = F(0), q1_1_b = F(0), q1_0_b = F(0), ua_b = F(0), va_b = F(0);
  F t2_1_b = F(0), t2_0_b = F(0), ta1_b = F(0), ta2_b = F(0);
  // evap1 = chs denv2 (qsat(sst) - q1_1); shf1 = chs 1004 denv2 (sst - t1_1)
  denv2_b += evap1_b * F(p.chs) * (w.qss - w.q1_1);
  {
    const F D = evap1_b * F(p.chs) * w.denv2;
    b.psa += D * w.qss_p;
    q1_1_b -= D;
  }
  denv2_b += shf1_b * F(p.chs) * F(1004.0) * (F(s.sst) - w.t1_1);
  t1_1_b -= shf1_b * F(p.chs) * F(1004.0) * w.denv2;
  // ustr1 = -cds denv2 u
  {
    const F cd_b = -ustr1_b * c.u - vstr1_b * c.v;
    ua_b += -ustr1_b * w.cdsdv;
    va_b += -vstr1_b * w.cdsdv;
    denv2_b += cd_b * F(p.cds);
  }
  const bool fh = F(p.fhum0) > F(0);
  if (fh) {
    b.add_rh(c, KX - 1, q1_1_b * F(p.fhum0) * w.qs11);
    const F qs_b = q1_1_b * F(p.fhum0) * c.RH(KX - 1);
    b.q[KX - 1] += q1_1_b * (F(1) - F(p.fhum0));
    t1_1_b += qs_b * w.qs11_t;
    b.psa += qs_b * w.qs11_p;
  } else {
    b.q[KX - 1] += q1_1_b;
  }
  // denv2 = denv0 (1 + dths rdth)
  denv0_b += denv2_b * (F(1) + w.dths_v * rdth);
  {
    const F dths_b = denv2_b * w.denv0 * rdth;
    if (w.sst_gt)
      t2_1_b -= dths_b * wmin(F(s.sst) - w.t2_1, F(p.dtheta));
    else
      t2_1_b -= dths_b * wmax(astab * (F(s.sst) - w.t2_1), -F(p.dtheta)) * astab;
  }
  F qs00_b = F(0), evap0a_b = evap0_b, rlus0a_b = rlus0_b, shf0a_b = shf0_b, drls_b = F(0);
  if (x.flags & SPD_LSKINEB) {
    const F clamb = F(p.clambda) + (c.snowc * (F(p.clambsn) - F(p.clambda)));
    const F dtskin_b = shf0_b * chlcp * w.denv1 + evap0_b * F(p.chl) * w.denv1 * w.qs01 +
                       rlus0_b * w.drls;
    denv1_b += shf0_b * chlcp * w.dtskin + evap0_b * F(p.chl) * w.qs01 * w.dtskin;
    F qs01_b = evap0_b * F(p.chl) * w.denv1 * w.dtskin;
    drls_b += rlus0_b * w.dtskin;
    const F hfl0_b = dtskin_b / w.den;
    const F den_b = -dtskin_b * (w.dtskin / w.den);
    drls_b += den_b;
    denv1_b += den_b * F(p.chl) * (F(1004.0) + F(2501.0) * w.qs01);
    qs01_b += den_b * F(p.chl) * w.denv1 * F(2501.0);
    if (w.evap_pos) {
      const F r_b = qs01_b * F(s.soilw);
      qs00_b -= r_b;
      tskin_b += r_b * w.qs01r_t;
      b.psa += r_b * w.qs01r_p;
    }
    tskin_b -= hfl0_b * clamb;
    rsds_b += hfl0_b * (F(1) - c.alb_l);
    rlds_b += hfl0_b;
    rlus0a_b -= hfl0_b;
    shf0a_b -= hfl0_b;
    evap0a_b -= F(2501.0) * hfl0_b;
  }
  // rlus0 = esbc tsk3 tskin; drls = 4 esbc tsk3; tsk3 = tskin^3
  {
    const F tsk3_b = rlus0a_b * esbc * w.tskin + drls_b * F(4.0) * esbc;
    tskin_b += rlus0a_b * esbc * w.tsk3 + tsk3_b * F(3) * w.tskin * w.tskin;
  }
  // evap0 = chl denv1 max(0, soilw qs00 - q1_0)
  {
    const F mx = vmax(F(0), w.Mv);
    denv1_b += evap0a_b * F(p.chl) * mx;
    const F v_b = evap0a_b * F(p.chl) * w.denv1 * wmax(w.Mv, F(0));
    qs00_b += v_b * F(s.soilw);
    q1_0_b -= v_b;
  }
  tskin_b += qs00_b * w.qs00_t;
  b.psa += qs00_b * w.qs00_p;
  if (fh) {
    b.add_rh(c, KX - 1, q1_0_b * F(p.fhum0) * w.qs10);
    const F qs_b = q1_0_b * F(p.fhum0) * c.RH(KX - 1);
    b.q[KX - 1] += q1_0_b * (F(1) - F(p.fhum0));
    t1_0_b += qs_b * w.qs10_t;
    b.psa += qs_b * w.qs10_p;
  } else {
    b.q[KX - 1] += q1_0_b;
  }
  // shf0 = chl 1004 denv1 (tskin - t1_0)
  denv1_b += shf0a_b * chlcp * (w.tskin - w.t1_0);
  tskin_b += shf0a_b * chlcp * w.denv1;
  t1_0_b -= shf0a_b * chlcp * w.denv1;
  // ustr0 = -cdl denv0 forog u
  {
    const F cd_b = -ustr0_b * c.u - vstr0_b * c.v;
    ua_b += -ustr0_b * w.cdldv;
    va_b += -vstr0_b * w.cdldv;
    denv0_b += cd_b * F(p.cdl) * w.forog;
  }
  // denv1 = denv0 (1 + dthl rdth)
  denv0_b += denv1_b * (F(1) + w.dthl_v * rdth);
  {
    const F dthl_b = denv1_b * w.denv0 * rdth;
    F d_b;
    if (w.tsk_gt)
      d_b = dthl_b * wmin(w.tskin - w.t2_0, F(p.dtheta));
    else
      d_b = dthl_b * wmax(astab * (w.tskin - w.t2_0), -F(p.dtheta)) * astab;
    tskin_b += d_b;
    t2_0_b -= d_b;
  }
  // tskin = stl + ctday sqrt_coa rsds (1 - alb_l) psa
  {
    const F kts = F(p.ctday) * F(z.sqrt_coa);
    rsds_b += tskin_b * kts * (F(1) - c.alb_l) * c.psa;
    b.psa += tskin_b * kts * c.rsds * (F(1) - c.alb_l);
  }
  // denv0 = A B
  {
    const F A_b = denv0_b * w.B, B_b = denv0_b * w.A;
    const F Bs_b = B_b * (F(0.5) / w.B);
    ua_b += Bs_b * F(2) * w.u0 * F(p.fwind0);
    va_b += Bs_b * F(2) * w.v0 * F(p.fwind0);
    const F K2 = F(2.0 / 7.0 * 1004.0);
    b.psa += A_b * F(1e5) / (K2 * w.t0);
    const F t0_b = -A_b * (w.A / w.t0);
    t1_1_b += t0_b - F(s.fmask) * t0_b;
    t1_0_b += t0_b * F(s.fmask);
  }
  F t1_0p_b = F(0), t1_1p_b = F(0);
  if (w.warm) {
    t1_0p_b = t1_0_b * F(p.ftemp0);
    t2_0_b += t1_0_b * (F(1) - F(p.ftemp0));
    t1_1p_b = t1_1_b * F(p.ftemp0);
    t2_1_b += t1_1_b * (F(1) - F(p.ftemp0));
  } else {
    ta1_b += t1_0_b + t1_1_b;
  }
  const F rcp = F(1.0 / 1004.0);
  t2_1_b += t2_0_b;
  ta1_b += t2_1_b;
  b.phi[KX - 1] += t2_1_b * rcp;
  const F phi0 = F(s.orog) * F(9.81);
  t1_0p_b += t1_1p_b;
  F dt1_b = -t1_1p_b * phi0 / (F(2.0 / 7.0 * 1004.0 * 288.0) * F(vg.sigl[KX - 1]));
  ta1_b += t1_0p_b;
  dt1_b += t1_0p_b;
  const F ww = F(vg.wvi[KX - 1][1]);
  ta1_b += dt1_b * ww;
  ta2_b -= dt1_b * ww;
  b.t[KX - 1] += ta1_b;
  b.t[KX - 2] += ta2_b;
  b.u += ua_b;
  b.v += va_b;
}

// ---------------------------------------------------------------------------------------------
// get_vertical_diffusion_tend (vertical_diffusion.py:10-136)
// ---------------------------------------------------------------------------------------------
template <int KX, class F>
struct VdConst {
  F fshcq, fshcse, fvdiq, fvdise, drh0, fvdiq2;
};

template <int KX, class F>
SPD_HD VdConst<KX, F> vd_const(const Ctx& x) {
  const spd_vgrid_t& vg = *x.vg;
  const spd_params_t& p = *x.p;
  const int nl1 = KX - 1;
  VdConst<KX, F> v;
  const F cshc = F(vg.dhs[KX - 1]) / F(3600.0);
  const F cvdi = (F(vg.hsg[nl1]) - F(vg.hsg[1])) / (F(nl1 - 1) * F(3600.0));
  v.fshcq = cshc / F(p.trshc);
  v.fshcse = cshc / (F(p.trshc) * F(1004.0));
  v.fvdiq = cvdi / F(p.trvdi);
  v.fvdise = cvdi / (F(p.trvds) * F(1004.0));
  v.drh0 = F(p.rhgrad) * (F(vg.fsg[KX - 1]) - F(vg.fsg[nl1 - 1]));
  v.fvdiq2 = v.fvdiq * F(vg.hsg[nl1]);
  return v;
}

template <int KX, class F>
SPD_HD void vdiff(const Ctx& x, const Col<KX, F>& c, F* dt, F* dq) {
  const spd_vgrid_t& vg = *x.vg;
  const spd_params_t& p = *x.p;
  const VdConst<KX, F> v = vd_const<KX, F>(x);
  const int nl1 = KX - 1;
  const int icnv = KX - c.iptop - 1;
  F tt[KX], qt[KX];
  SPD_LEVELS
  for (int k = 0; k < KX; ++k) tt[k] = qt[k] = F(0);
  const F dmse = c.SE(KX - 1) - c.SE(nl1 - 1) + F(2501.0) * (c.q[KX - 1] - c.qsat[nl1 - 1]);
  const F drh = c.RH(KX - 1) - c.RH(nl1 - 1);
  const F fcnv = (icnv > 0 && dmse >= F(0)) ? F(p.redshc) : F(1);
  if (dmse >= F(0)) {
    const F fluxse = fcnv * v.fshcse * dmse;
    tt[nl1 - 1] = fluxse * (F(1) / F(vg.dhs[nl1 - 1]));
    tt[KX - 1] = -fluxse * (F(1) / F(vg.dhs[KX - 1]));
    if (drh >= F(0)) {
      const F fq = fcnv * v.fshcq * c.qsat[KX - 1] * drh;
      qt[nl1 - 1] = fq * (F(1) / F(vg.dhs[nl1 - 1]));
      qt[KX - 1] = -fq * (F(1) / F(vg.dhs[KX - 1]));
    }
  } else if (dmse < F(0) && drh > v.drh0) {
    const F fq = v.fvdiq2 * c.qsat[nl1 - 1] * drh;
    qt[nl1 - 1] = fq * (F(1) / F(vg.dhs[nl1 - 1]));
    qt[KX - 1] = -fq * (F(1) / F(vg.dhs[KX - 1]));
  }
  F fluxq[KX];
  SPD_LEVELS
  for (int k = 2; k < KX - 2; ++k) {
    const bool cond = F(vg.hsg[k + 1]) > F(0.5);
    const F d0 = F(p.rhgrad) * (F(vg.fsg[k + 1]) - F(vg.fsg[k]));
    const F f2 = v.fvdiq * F(vg.hsg[k + 1]);
    const F dr = c.RH(k + 1) - c.RH(k);
    fluxq[k] = (dr >= d0 && cond) ? f2 * c.qsat[k] * dr : F(0);
    qt[k] = qt[k] + fluxq[k] * (F(1) / F(vg.dhs[k]));
  }
  SPD_LEVELS
  for (int k = 2; k < KX - 2; ++k) qt[k + 1] = qt[k + 1] + (-fluxq[k] * (F(1) / F(vg.dhs[k + 1])));
  F fse[KX];
  SPD_LEVELS
  for (int k = 0; k < nl1; ++k) {
    const F se0 = c.SE(k + 1) - F(p.segrad) * (c.phi[k + 1] - c.phi[k]);
    fse[k] = (c.SE(k) < se0) ? v.fvdise * (se0 - c.SE(k)) : F(0);
    tt[k] = tt[k] + fse[k] * (F(1) / F(vg.dhs[k]));
  }
  F cum = F(0);
  SPD_LEVELS
  for (int k = 0; k < nl1; ++k) {
    cum = cum + fse[k] * (F(1) / (F(1) - F(vg.hsg[k + 1])));
    tt[k + 1] = tt[k + 1] + (-cum);
  }
  SPD_LEVELS
  for (int k = 0; k < KX; ++k) {
    dt[k] = dt[k] + tt[k];
    dq[k] = dq[k] + qt[k];
  }
}

template <int KX, class F>
SPD_HD void vdiff_rev(const Ctx& x, const Col<KX, F>& c, const F* dt_b, const F* dq_b,
                      Bar<KX, F>& b) {
  const spd_vgrid_t& vg = *x.vg;
  const spd_params_t& p = *x.p;
  const VdConst<KX, F> v = vd_const<KX, F>(x);
  const int nl1 = KX - 1;
  const int icnv = KX - c.iptop - 1;
  // the cumulative flux: tt[k+1] -= sum_{j<=k} fse[j] / (1 - hsg[j+1])
  F acc = F(0);
  SPD_LEVELS
  for (int k = nl1 - 1; k >= 0; --k) {
    acc += -dt_b[k + 1];
    const F fse_b = acc * (F(1) / (F(1) - F(vg.hsg[k + 1]))) + dt_b[k] * (F(1) / F(vg.dhs[k]));
    const F se0 = c.SE(k + 1) - F(p.segrad) * (c.phi[k + 1] - c.phi[k]);
    if (c.SE(k) < se0) {
      const F s_b = fse_b * v.fvdise;
      b.add_se(k, -(s_b));
      b.add_se(k + 1, s_b);
      b.phi[k + 1] -= s_b * F(p.segrad);
      b.phi[k] += s_b * F(p.segrad);
    }
  }
  SPD_LEVELS
  for (int k = 2; k < KX - 2; ++k) {
    const bool cond = F(vg.hsg[k + 1]) > F(0.5);
    const F d0 = F(p.rhgrad) * (F(vg.fsg[k + 1]) - F(vg.fsg[k]));
    const F dr = c.RH(k + 1) - c.RH(k);
    if (!(dr >= d0 && cond)) continue;
    const F f2 = v.fvdiq * F(vg.hsg[k + 1]);
    const F fl_b = dq_b[k] * (F(1) / F(vg.dhs[k])) - dq_b[k + 1] * (F(1) / F(vg.dhs[k + 1]));
    b.qsat[k] += fl_b * f2 * dr;
    const F dr_b = fl_b * f2 * c.qsat[k];
    b.add_rh(c, k + 1, dr_b);
    b.add_rh(c, k, -(dr_b));
  }
  const F dmse = c.SE(KX - 1) - c.SE(nl1 - 1) + F(2501.0) * (c.q[KX - 1] - c.qsat[nl1 - 1]);
  const F drh = c.RH(KX - 1) - c.RH(nl1 - 1);
  const F fcnv = (icnv > 0 && dmse >= F(0)) ? F(p.redshc) : F(1);
  const F fq_b = dq_b[nl1 - 1] * (F(1) / F(vg.dhs[nl1 - 1])) -
                 dq_b[KX - 1] * (F(1) / F(vg.dhs[KX - 1]));
  F dmse_b = F(0), drh_b = F(0);
  if (dmse >= F(0)) {
    const F fx_b = dt_b[nl1 - 1] * (F(1) / F(vg.dhs[nl1 - 1])) -
                   dt_b[KX - 1] * (F(1) / F(vg.dhs[KX - 1]));
    dmse_b = fx_b * fcnv * v.fshcse;
    if (drh >= F(0)) {
      b.qsat[KX - 1] += fq_b * fcnv * v.fshcq * drh;
      drh_b = fq_b * fcnv * v.fshcq * c.qsat[KX - 1];
    }
  } else if (dmse < F(0) && drh > v.drh0) {
    b.qsat[nl1 - 1] += fq_b * v.fvdiq2 * drh;
    drh_b = fq_b * v.fvdiq2 * c.qsat[nl1 - 1];
  }
  b.add_se(KX - 1, dmse_b);
  b.add_se(nl1 - 1, -(dmse_b));
  b.q[KX - 1] += F(2501.0) * dmse_b;
  b.qsat[nl1 - 1] -= F(2501.0) * dmse_b;
  b.add_rh(c, KX - 1, drh_b);
  b.add_rh(c, nl1 - 1, -(drh_b));
}

// ---------------------------------------------------------------------------------------------
// The column: forward, then every term in reverse order.
//
// in.q holds the humidity as given (before verify_state).  ct_* are the cotangents of the four
// tendency outputs (after verify_tendencies and the humidity scale, when those are fused);
// ct_u/ct_v are the cotangents of the lowest-level wind tendencies.  On return b holds the
// gradients: b.q with respect to the humidity as given.  With SPD_OROGRAPHIC and the fused
// verify, qcorv (the orographic humidity profile) and gamlat, pexp give the correction's
// humidity tendency, which takes part in verify_tendencies' choice of limited levels.
// ---------------------------------------------------------------------------------------------
template <int KX, class F>
SPD_HD void column_vjp(const Ctx& x, const DiffParams<F>& g, F ablco2, F dt_seconds,
                       F q_tend_scale, const ColumnIn<F, F>& in, const F* ct_t, const F* ct_q,
                       F ct_u, F ct_v, Bar<KX, F>& b, const float* qcorv = nullptr,
                       float gamlat = 0.0f, float pexp = 0.0f) {
  const spd_params_t& p = *x.p;
  const bool verify = (x.flags & SPD_FUSE_VERIFY) != 0;
  Col<KX, F> c;
  SPD_LEVELS
  for (int k = 0; k < KX; ++k) {
    c.t[k] = in.t[k];
    c.q[k] = (verify && in.q[k] < F(0)) ? F(0) : in.q[k];
    c.phi[k] = in.phi[k];
  }
  c.psa = in.psa;
  c.u = in.u_low;
  c.v = in.v_low;
  const SurfaceIn s{(float)in.sst, (float)in.stl,   (float)in.soilw,
                    (float)in.snowc, (float)in.sice, (float)in.alb0,
                    (float)in.fmask, (float)in.orog, (float)in.phis0};
  const SurfaceRow z{(float)in.fsol,  (float)in.ozupp,  (float)in.ozone,
                     (float)in.zenit, (float)in.stratz, (float)in.sqrt_coa};
  // set_forcing (physics/speedy/forcing.py:11-39)
  c.snowc = in.snowc < F(1) ? in.snowc : F(1);
  c.alb_l = in.alb0 + c.snowc * (F(p.albsn) - in.alb0);
  {
    const F alb_s = F(p.albsea) + in.sice * (F(p.albice) - F(p.albsea));
    c.albsfc = alb_s + in.fmask * (c.alb_l - alb_s);
  }
  // ---- forward ----
  F dq[KX], dt[KX];
  SPD_LEVELS
  for (int k = 0; k < KX; ++k) dq[k] = dt[k] = F(0);
  humidity(x, c);
  dconv(x, g, c);
  // The term internals share one scratch: convection and shortwave run (and are recomputed)
  // outside the span in which the longwave fluxes are kept.  (The reverse passes keep their
  // own work arrays as locals: addressed through pointers into this scratch, the device build
  // corrupted one of them.)
  union Scratch {
    Cv<KX, F> cv;
    Sw<KX, F> sw;
    Lw<KX, F> lw;
  } sc;
  conv(x, g, c, sc.cv);
  c.precnv = sc.cv.precnv;
  if (verify) conv_tend(x, sc.cv, dt, dq);
  lsc(x, g, c, dt, dq);
  Cl<KX, F> cl;
  clouds(x, c, cl, F(in.fmask));
  shortwave(x, g, c, z, sc.sw);
  Lw<KX, F>& lw = sc.lw;
  longwave_down(x, c, ablco2, lw);
  Sf<F> sf;
  surface(x, c, s, z, sf);
  longwave_up(x, c, z, ablco2, lw);
  // ---- cotangents of the physics tendencies ----
  const F* dt_b = ct_t;
  F dq_b[KX];
  uint32_t limited = 0u;  // levels where verify_tendencies replaced dq by -q / dt
  if (verify) {
    F du, dv;
    surface_tend<KX, F>(x, sf, dt, dq, du, dv);
    vdiff(x, c, dt, dq);
    if (qcorv && (x.flags & SPD_OROGRAPHIC)) {  // the last term's humidity tendency
      const F qcorh = orographic_qcorh(in.phis0, in.fmask, in.stl, in.sst, F(gamlat), F(pexp));
      SPD_LEVELS
      for (int k = 0; k < KX; ++k) dq[k] = dq[k] + (qcorh * F(qcorv[k])) / dt_seconds;
    }
  }
  SPD_LEVELS
  for (int k = 0; k < KX; ++k) {
    F qb = ct_q[k] * q_tend_scale;
    if (verify && !(in.q[k] + dt_seconds * dq[k] >= F(0))) {
      limited |= 1u << k;
      qb = F(0);
    }
    dq_b[k] = qb;
  }
  SPD_LEVELS
  for (int k = 0; k < KX; ++k)
    b.t[k] = b.q[k] = b.phi[k] = b.qsat[k] = F(0);
  b.psa = b.u = b.v = F(0);
  SPD_BANDS
  for (int j = 0; j < P_N; ++j) b.par[j] = F(0);
  // ---- reverse ----
  vdiff_rev(x, c, dt_b, dq_b, b);
  // the longwave reverse is split around the surface term: the upward pass gives the adjoint
  // of the surface's upward flux, the surface gives that of the downward flux at the surface
  F rlus2_b = F(0), fsw0_b = F(0), fsw1_b = F(0), cloudc_b = F(0), rsds_b = F(0), rlds_b = F(0);
  {
    F acl1_b = F(0), acl2_b = F(0);
    longwave_rev_up(x, c, z, lw, ablco2, dt_b, rlus2_b, fsw0_b, fsw1_b, acl1_b, acl2_b, b);
    surface_rev(x, c, s, z, sf, ct_u, ct_v, dt_b[KX - 1], dq_b[KX - 1], rlus2_b, rsds_b,
                rlds_b, b);
    longwave_rev_down(x, c, lw, ablco2, dt_b, rlds_b, acl1_b, acl2_b, b);
    cloudc_b += acl1_b * F(p.ablcl1) + acl2_b * F(p.ablcl2);
  }
  F clstr_b = F(0), qcloud_b = F(0);
  shortwave(x, g, c, z, sc.sw);
  shortwave_rev(x, g, c, z, sc.sw, dt_b, rsds_b, fsw0_b, fsw1_b, cloudc_b, clstr_b, qcloud_b, b);
  F precnv_b = F(0), precls_b = F(0);
  clouds_rev(x, c, cl, F(in.fmask), cloudc_b, clstr_b, qcloud_b, precnv_b, precls_b, b);
  lsc_rev(x, g, c, dt_b, dq_b, precls_b, b);
  conv(x, g, c, sc.cv);
  const F qdif_b = conv_rev(x, g, c, sc.cv, dt_b, dq_b, precnv_b, b);
  dconv_rev(x, g, c, qdif_b, b);
  humidity_rev(x, c, b);
  SPD_LEVELS
  for (int k = 0; k < KX; ++k) {
    const F qb = (verify && in.q[k] < F(0)) ? F(0) : b.q[k];
    b.q[k] = qb + (((limited >> k) & 1u) ? -(ct_q[k] * q_tend_scale) / dt_seconds : F(0));
  }
}

}  // namespace spdvjp
