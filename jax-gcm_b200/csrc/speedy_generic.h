// speedy_generic.h -- the SPEEDY column physics of one column, generic in the value type.
//
// column_generic<KX, R, F> evaluates SpeedyPhysics.compute_tendencies
// (jcm/physics/speedy/speedy_physics.py:88-127) for one column, term by term in the reference's
// order, with the differentiable quantities (state, the 12 tuning parameters and everything
// derived from them) of type R and the non-differentiated constants of type F.  With
// R = spdad::Adj<F> it records the reverse-mode tape of the column (speedy_ad.h).  Its users are
// host builds: the tests' float32/float64 forward, the taped float64 VJP that checks the
// device's hand-written reverse pass (speedy_vjp.h), and the compiled CPU restatement of the
// reference (oracle/cpu_port.cpp, R = F = float) that the benchmark times as its CPU baseline.
//
// Each block cites the reference lines it restates (paths relative to the JAX-GCM root).  The
// shortwave cloud-top level set S of the instance (shortwave_radiation.py:62-68) is an input.
#pragma once

#include "speedy_ad.h"
#include "speedy_b200.h"

// The column loops stay rolled on the device: with Adj values the per-level arrays live in
// local memory anyway, and unrolling only multiplies code size and compile time.
#if defined(__CUDA_ARCH__)
#define SPD_ROLL _Pragma("unroll 1")
#else
#define SPD_ROLL
#endif

namespace spdgen {

using spdad::gexp;
using spdad::gisnan;
using spdad::gmax;
using spdad::gmin;
using spdad::gsqrt;
using spdad::val;

// The 12 differentiated parameters (params.py:11-16, :51-54, :72-73).
template <class R>
struct DiffParams {
  R psmin, trcnv, rhil, rhbl, entmax, smf, trlsc, rhlsc, drhlsc, rhblsc, albcl, albcls;
};

template <class R, class F>
struct ColumnIn {
  R t[SPD_MAX_KX], q[SPD_MAX_KX], phi[SPD_MAX_KX];
  R psa, u_low, v_low;
  F sst, stl, soilw, snowc, sice, alb0, fmask, orog, phis0;
  F fsol, ozupp, ozone, zenit, stratz, sqrt_coa;  // per-latitude solar row (not differentiated)
};

template <class R>
struct ColumnOut {
  R dt[SPD_MAX_KX], dq[SPD_MAX_KX];
  R du_low, dv_low, precnv, precls, cloudc, rsds, rlds;
  int iptop, icltop;
};

template <class R, class F>
SPD_HD R qsat_g(const R& ta, const R& ps, F sig) {
  // get_qsat (humidity.py:73-104), sig > 0
  const F e0 = F(6.108e-3), c1 = F(17.269), c2 = F(21.875), t0 = F(273.16), t1 = F(35.86),
          t2 = F(7.66);
  const R e = (val(ta) >= val(F(t0))) ? e0 * gexp(c1 * (ta - t0) / (ta - t1))
                                      : e0 * gexp(c2 * (ta - t0) / (ta - t2));
  return F(622.0) * e / (sig * ps - F(0.378) * e);
}

template <class R, class F>
SPD_HD void radset_r(const R& temp, F epslw, R fb[4]) {
  const R j = gmin(gmax(temp, F(200)), F(320));
  const R f1 = F(0.148) - F(3.0e-6) * ((j - F(247)) * (j - F(247)));
  const R f2 = F(0.356) - F(5.2e-6) * ((j - F(282)) * (j - F(282)));
  const R f3 = F(0.314) + F(1.0e-5) * ((j - F(315)) * (j - F(315)));
  const R f0 = F(1) - (((F(0) + f1) + f2) + f3);
  const F w = F(1) - epslw;
  fb[0] = w * f0;
  fb[1] = w * f1;
  fb[2] = w * f2;
  fb[3] = w * f3;
}

template <int KX, class R, class F>
SPD_HD void column_generic(const spd_vgrid_t& vg, const spd_params_t& p, const DiffParams<R>& g,
                           uint32_t flags, int model_step, F ablco2, uint32_t S,
                           const ColumnIn<R, F>& in, ColumnOut<R>& o,
                           bool through_clouds_only = false) {
  const R psa = in.psa;
  const R* t = in.t;
  const R* q = in.q;
  const R* phi = in.phi;
  R qsat[KX], rh[KX], se[KX];
  SPD_ROLL
  for (int k = 0; k < KX; ++k) o.dt[k] = o.dq[k] = R(F(0));

  // ---- spec_hum_to_rel_hum (humidity.py:16-51) ----
  SPD_ROLL
  for (int k = 0; k < KX; ++k) {
    qsat[k] = qsat_g<R, F>(t[k], psa, F(vg.fsg[k]));
    rh[k] = q[k] / qsat[k];
    se[k] = F(1004.0) * t[k] + phi[k];  // convection.py:123
  }

  // ---- set_forcing (physics/speedy/forcing.py:11-39) ----
  const F snowc = in.snowc < F(1) ? in.snowc : F(1);
  const F alb_l = in.alb0 + snowc * (F(p.albsn) - in.alb0);
  const F alb_s = F(p.albsea) + in.sice * (F(p.albice) - F(p.albsea));
  const F albsfc = alb_s + in.fmask * (alb_l - alb_s);

  // ---- diagnose_convection (convection.py:15-97) ----
  int iptop = KX + 1;
  R qdif = R(F(0));
  {
    R mss[KX], mss2[KX];
    SPD_ROLL
    for (int k = 0; k < KX; ++k) mss[k] = se[k] + F(2501.0) * qsat[k];
    const R mse0 = se[KX - 1] + F(2501.0) * q[KX - 1];
    const R mse1 = gmin(mse0, se[KX - 2] + F(2501.0) * q[KX - 2]);
    const R mss0 = gmax(mse0, mss[KX - 1]);
    SPD_ROLL
    for (int k = 0; k < KX - 1; ++k) mss2[k] = mss[k] + F(vg.wvi[k][1]) * (mss[k + 1] - mss[k]);
    mss2[KX - 1] = R(F(0));
    int ktop1 = KX, ktop2 = KX;
    SPD_ROLL
    for (int k = KX - 4; k >= 2; --k) {
      if (val(mss0) > val(mss2[k])) ktop1 = k + 1;
      if (val(mse1) > val(mss2[k])) ktop2 = k + 1;
    }
    const R msthr = mss2[ktop2 - 1];
    const R qthr0 = g.rhbl * qsat[KX - 1];
    const R qthr1 = g.rhbl * qsat[KX - 2];
    const bool lqthr = val(q[KX - 1]) > val(qthr0) && val(q[KX - 2]) > val(qthr1);
    const bool mask_psa = val(psa) > val(g.psmin);
    const bool case1 = mask_psa && ktop1 < KX && ktop2 < KX;
    const bool case2 = mask_psa && ktop1 < KX && !(ktop2 < KX) && lqthr;
    if (case1 || case2) iptop = ktop1;
    if (case1) qdif = gmax(q[KX - 1] - qthr0, (mse0 - msthr) * F(1.0 / 2501.0));
    if (case2) qdif = q[KX - 1] - qthr0;
  }

  // ---- get_convection_tendencies (convection.py:99-237) ----
  R precnv = R(F(0)), cbmf;
  {
    R entr[KX];
    R sentr = R(F(0));
    SPD_ROLL
    for (int k = 1; k < KX - 1; ++k) {
      const R e = gmax(F(0), R(F(vg.fsg[k]) - F(0.5)));
      entr[k] = e * e;
      sentr = sentr + entr[k];
    }
    const R escale = g.entmax / sentr;
    SPD_ROLL
    for (int k = 1; k < KX - 1; ++k) entr[k] = entr[k] * escale;
    const R fm0 = F(1e5) * F(vg.dhs[KX - 1]) / (F(9.81) * g.trcnv * F(3600.0));
    const R rdps = F(2.0) / (F(1.0) - g.psmin);
    const bool mask = iptop < KX;
    const R qmax = gmax(F(1.01) * q[KX - 1], qsat[KX - 1]);
    R sb3[KX], qb3[KX];
    sb3[0] = qb3[0] = R(F(0));
    SPD_ROLL
    for (int k = 1; k < KX; ++k) {
      sb3[k] = se[k - 1] + F(vg.wvi[k - 1][1]) * (se[k] - se[k - 1]);
      qb3[k] = q[k - 1] + F(vg.wvi[k - 1][1]) * (q[k] - q[k - 1]);
    }
    const R sb = sb3[KX - 1];
    const R qb = gmin(qb3[KX - 1], q[KX - 1]);
    const R fpsa = psa * gmin(F(1.0), (psa - g.psmin) * rdps);
    const R fmass = fm0 * fpsa * gmin(F(5.0), qdif / (qmax - qb));
    cbmf = mask ? fmass : F(0) * fmass;
    const R fus = fmass * se[KX - 1], fuq = fmass * qmax;
    const R fds = fmass * sb, fdq = fmass * qb;
    R dfse[KX], dfqa[KX], fm3[KX], fus3[KX], fuq3[KX], fds3[KX], fdq3[KX];
    R cm = R(F(0)), cs = R(F(0)), cq = R(F(0));
    SPD_ROLL
    for (int k = KX - 1; k >= 0; --k) {
      const bool lm = (k <= KX - 2) && (k >= iptop);
      R en = (k >= 1 && k <= KX - 2) ? entr[k] * psa * cbmf : R(F(0));
      en = lm ? en : F(0) * en;
      cm = cm + en * F(1.0);
      cs = cs + en * se[k];
      cq = cq + en * q[k];
      fm3[k] = fmass + cm;
      fus3[k] = fus + cs;
      fuq3[k] = fuq + cq;
      fds3[k] = (k == KX - 1) ? fds : fm3[k] * sb3[k];
      fdq3[k] = (k == KX - 1) ? fdq : fm3[k] * qb3[k];
    }
    dfse[KX - 1] = fds - fus;
    dfqa[KX - 1] = fdq - fuq;
    SPD_ROLL
    for (int k = 0; k < KX - 1; ++k) {
      const bool lm = (k >= iptop);
      const R a = (fus3[k + 1] - fds3[k + 1]) - (fus3[k] - fds3[k]);
      const R b = (fuq3[k + 1] - fdq3[k + 1]) - (fuq3[k] - fdq3[k]);
      dfse[k] = lm ? a : F(0) * a;
      dfqa[k] = lm ? b : F(0) * b;
    }
    R fsq_sum = R(F(0));
    SPD_ROLL
    for (int k = 0; k < KX; ++k) {
      const bool lm = (k <= KX - 2) && (k >= iptop);
      const R d0 = g.rhil * qsat[k] - q[k];
      const R delq = lm ? d0 : F(0) * d0;
      const R fsq = (val(delq) > F(0) ? g.smf : F(0) * g.smf) * cbmf * delq;
      dfqa[k] = dfqa[k] + fsq;
      fsq_sum = fsq_sum + fsq;
    }
    dfqa[KX - 1] = dfqa[KX - 1] + (-fsq_sum);
    if (iptop <= KX - 1) {
      const int kt = iptop - 1;
      const R qsatb = qsat[kt] + F(vg.wvi[kt][1]) * (qsat[kt + 1] - qsat[kt]);
      precnv = gmax(fuq3[iptop] - fm3[iptop] * qsatb, F(0));
      dfse[kt] = fus3[iptop] - fds3[iptop] + F(2501.0) * precnv;
      dfqa[kt] = fuq3[iptop] - fdq3[iptop] - precnv;
    }
    const R rps = F(1) / psa;
    o.dt[0] = o.dt[0] + dfse[0];
    o.dq[0] = o.dq[0] + dfqa[0];
    SPD_ROLL
    for (int k = 1; k < KX; ++k) {
      o.dt[k] = o.dt[k] + dfse[k] * rps * F(vg.grdscp[k]);
      o.dq[k] = o.dq[k] + dfqa[k] * rps * F(vg.grdsig[k]);
    }
  }
  o.precnv = precnv;

  // ---- get_large_scale_condensation_tendencies (large_scale_condensation.py:14-86) ----
  R precls;
  {
    const R rtlsc = F(1.0) / (g.trlsc * F(3600.0));
    const F tfact = F(2501.0 / 1004.0);
    const F prg = F(1e5 / 9.81);
    const R psa2 = psa * psa;
    R psum = R(F(0));
    int first = 0;
    SPD_ROLL
    for (int k = 1; k < KX; ++k) {
      const F sig2 = F(vg.fsg[k]) * F(vg.fsg[k]);
      const R rhref = gmax(g.rhlsc + g.drhlsc * (sig2 - F(1.0)), g.rhblsc);
      const R dqmax = F(10.0) * sig2 * rtlsc;
      const R dqa = rhref * qsat[k] - q[k];
      R dql = R(F(0)), dtl = R(F(0));
      if (val(dqa) < F(0)) {
        dql = dqa * rtlsc;
        dtl = tfact * gmin(-dql, dqmax * psa2);
        if (first == 0) first = k;
      }
      o.dt[k] = o.dt[k] + dtl;
      o.dq[k] = o.dq[k] + dql;
      psum = psum + (F(vg.dhs[k]) * prg) * dql;
    }
    precls = (F(0) - psum) * psa;
    iptop = (first == 0 ? 1 : first) < iptop ? (first == 0 ? 1 : first) : iptop;
  }
  o.precls = precls;
  o.iptop = iptop;

  // ---- clouds (shortwave_radiation.py:313-404) ----
  R cloudc, clstr, qcloud;
  int icltop;
  {
    const int nl1 = KX - 2;
    const bool m0 = val(rh[nl1]) > F(p.rhcl1);
    const R cloudc0 = m0 ? rh[nl1] - F(p.rhcl1) : R(F(0));
    const int icl0 = m0 ? nl1 : KX;
    R upd[KX];
    bool mk[KX];
    R cmax = R(F(0));
    bool first = true;
    SPD_ROLL
    for (int k = 2; k < KX - 2; ++k) {
      const R drh = rh[k] - F(p.rhcl1);
      mk[k] = val(drh) > val(cloudc0) && val(q[k]) > F(p.qacl);
      upd[k] = mk[k] ? drh : cloudc0;
      cmax = first ? upd[k] : gmax(cmax, upd[k]);
      first = false;
    }
    int icl = -1;
    SPD_ROLL
    for (int k = 2; k < KX - 2; ++k) {
      const int cand = (val(cmax) == val(upd[k])) ? (mk[k] ? k : icl0) : icl0;
      icl = cand > icl ? cand : icl;
    }
    const R gse = (se[KX - 2] - se[KX - 1]) / (phi[KX - 2] - phi[KX - 1]);
    const F rrcl = F(1.0) / (F(p.rhcl2) - F(p.rhcl1));
    const R pr1 = gmin(F(p.pmaxcl), F(86.4) * (precnv + precls));
    const R cc = gmin(F(1.0), cmax * rrcl);
    cloudc = gmin(F(1.0), F(p.wpcl) * gsqrt(gmax(F(1e-9), pr1)) + cc * cc);
    if (gisnan(cloudc)) cloudc = R(F(1.0));
    icltop = iptop < icl ? iptop : icl;
    qcloud = q[nl1];
    const F rgse = F(1.0) / (F(p.gse_s1) - F(p.gse_s0));
    const R fstab = gmin(gmax(rgse * (gse - F(p.gse_s0)), F(0.0)), F(1.0));
    clstr = fstab * gmax(F(p.clsmax) - F(1.2) * cloudc, F(0.0));
    const R clstrl = gmax(clstr, F(p.clsminl)) * rh[KX - 1];
    clstr = clstr + in.fmask * (clstrl - clstr);
  }
  o.cloudc = cloudc;
  o.icltop = icltop;
  // The cloud-top level set S of the instance needs every column's icltop: a caller that
  // forms S itself runs the terms up to here first (through_clouds_only), then the column.
  if (through_clouds_only) return;

  // ---- shortwave_rad_fluxes (shortwave_radiation.py:27-217) ----
  R flux_sw0, flux_sw1, rsds;
  {
    const bool cmask = icltop < KX;
    R tau0[KX], tau1[KX], r[KX], dfabs[KX];
    SPD_ROLL
    for (int k = 0; k < KX; ++k) r[k] = ((S >> k) & 1u) && cmask ? g.albcl * cloudc : R(F(0));
    r[KX - 1] = g.albcls * clstr;
    const R psaz = psa * in.zenit;
    const R acloud = cloudc * gmin(F(p.abscl1) * qcloud, F(p.abscl2));
    tau0[0] = gexp(-psaz * F(vg.dhs[0]) * F(p.absdry));
    SPD_ROLL
    for (int k = 1; k < KX - 1; ++k) {
      const F abs1 = F(p.absdry) + F(p.absaer) * (F(vg.fsg[k]) * F(vg.fsg[k]));
      const R cl = (k >= icltop) ? acloud : F(0) * acloud;
      tau0[k] = gexp(-psaz * F(vg.dhs[k]) * (abs1 + F(p.abswv1) * q[k] + cl));
    }
    {
      const F abs1 = F(p.absdry) + F(p.absaer) * (F(vg.fsg[KX - 1]) * F(vg.fsg[KX - 1]));
      tau0[KX - 1] = gexp(-psaz * F(vg.dhs[KX - 1]) * (abs1 + F(p.abswv1) * q[KX - 1]));
    }
    SPD_ROLL
    for (int k = 1; k < KX; ++k) tau1[k] = gexp(-psaz * F(vg.dhs[k]) * F(p.abswv2) * q[k]);
    R f1 = in.fsol * F(0.95);
    dfabs[0] = f1;
    f1 = tau0[0] * (f1 - in.ozupp * psa);
    dfabs[0] = dfabs[0] + (-f1);
    dfabs[1] = f1;
    f1 = tau0[1] * (f1 - in.ozone * psa);
    dfabs[1] = dfabs[1] + (-f1);
    SPD_ROLL
    for (int k = 2; k < KX; ++k) {
      const R prev = f1;
      f1 = prev * tau0[k] * (F(1) - r[k]);
      dfabs[k] = prev * (F(1) - r[k]) * (F(1) - tau0[k]);
      r[k] = r[k] * prev;
    }
    R f2 = R(in.fsol * F(0.05));
    SPD_ROLL
    for (int k = 1; k < KX; ++k) {
      const R prev = f2;
      f2 = prev * tau1[k];
      dfabs[k] = dfabs[k] + prev * (F(1) - tau1[k]);
    }
    rsds = f1 + f2;
    R up = f1 * albsfc;
    dfabs[KX - 1] = dfabs[KX - 1] + up * (F(1) - tau0[KX - 1]);
    SPD_ROLL
    for (int k = KX - 1; k >= 1; --k) {
      up = up * tau0[k] + r[k];
      dfabs[k - 1] = dfabs[k - 1] + up * (F(1) - tau0[k - 1]);
    }
    flux_sw0 = tau0[0] * up + r[0];
    flux_sw1 = f2;
    if ((model_step % 3) == 0) {
      SPD_ROLL
      for (int k = 0; k < KX; ++k) o.dt[k] = o.dt[k] + dfabs[k] * F(vg.grdscp[k]) / psa;
    }
  }
  o.rsds = rsds;

  // ---- longwave: transmissivities (shortwave_radiation.py:174-206), st4a, down pass ----
  R tau[KX][4], st0[KX], st1[KX], dfl[KX];
  {
    const R acl1 = cloudc * F(p.ablcl1), acl2 = cloudc * F(p.ablcl2);
    SPD_ROLL
    for (int k = 0; k < KX; ++k) {
      R a0 = R(F(p.ablwin)), a2 = F(p.ablwv1) * q[k], a3 = F(p.ablwv2) * q[k];
      if (k == 0) a2 = a3 = R(F(0));
      if (k >= 2 && k <= KX - 2) {
        a0 = a0 + ((k > icltop) ? acl1 : acl2);
        a2 = gmax(a2, acl2);
        a3 = gmax(a3, acl2);
      }
      tau[k][0] = gexp(-a0 * psa * F(vg.dhs[k]));
      tau[k][1] = gexp(-ablco2 * psa * F(vg.dhs[k]));
      tau[k][2] = gexp(-a2 * psa * F(vg.dhs[k]));
      tau[k][3] = gexp(-a3 * psa * F(vg.dhs[k]));
    }
    R th[KX];
    SPD_ROLL
    for (int k = 0; k < KX - 1; ++k) th[k] = t[k] + F(vg.wvi[k][1]) * (t[k + 1] - t[k]);
    const R s10 = F(0.75) * t[0] + F(0.25) * th[0];
    const R s11 = F(0.50) * t[1] + F(0.25) * (th[0] + th[1]);
    const F sbc = F(5.67e-8);
    st0[0] = sbc * ((s10 * s10) * (s10 * s10));
    st1[0] = R(F(0));
    st0[1] = sbc * ((s11 * s11) * (s11 * s11));
    st1[1] = R(F(0));
    SPD_ROLL
    for (int k = 2; k < KX; ++k) {
      const R grad = (k < KX - 1) ? F(0.5) * gmax(th[k] - th[k - 1], F(0.0))
                                  : gmax(t[KX - 1] - th[KX - 2], F(0.0));
      const R st3 = sbc * (t[k] * t[k] * t[k]);
      st0[k] = st3 * t[k];
      st1[k] = F(4.0) * st3 * grad;
    }
  }
  R rlds;
  {
    R fl[4], fb[4];
    radset_r(t[0], F(p.epslw), fb);
    SPD_ROLL
    for (int b = 0; b < 4; ++b) {
      const R emis = F(1) - tau[0][b];
      fl[b] = emis * (fb[b] * (st0[0] + emis * st1[0]));
    }
    fl[2] = fl[3] = R(F(0));
    R sprev = ((fl[0] + fl[1]) + fl[2]) + fl[3];
    dfl[0] = F(0) + (-sprev);
    SPD_ROLL
    for (int k = 1; k < KX; ++k) {
      radset_r(t[k], F(p.epslw), fb);
      SPD_ROLL
      for (int b = 0; b < 4; ++b) {
        const R emis = F(1) - tau[k][b];
        fl[b] = tau[k][b] * fl[b] + emis * (fb[b] * (st0[k] + emis * st1[k]));
      }
      const R sk = ((fl[0] + fl[1]) + fl[2]) + fl[3];
      dfl[k] = F(0) + (-(sk - sprev));
      sprev = sk;
    }
    const F e = F(p.emisfc);
    rlds = ((e * fl[0] + e * fl[1]) + e * fl[2]) + e * fl[3];
    const R corlw = F(p.epslw) * F(p.emisfc) * st0[KX - 1];
    dfl[KX - 1] = dfl[KX - 1] + (-corlw);
    rlds = rlds + corlw;
  }
  o.rlds = rlds;

  // ---- get_surface_fluxes (surface_flux.py:15-300) ----
  R rlus2 = R(F(0));
  F tsfc = F(0);
  {
    const F esbc = F(p.emisfc) * F(5.67e-8);
    const R ta1 = t[KX - 1], ta2 = t[KX - 2];
    const R ua = in.u_low, va = in.v_low;
    const F phi0 = in.orog * F(9.81);
    const R u0 = F(p.fwind0) * ua, v0 = F(p.fwind0) * va;
    R ustr0 = R(F(0)), ustr1 = R(F(0)), vstr0 = R(F(0)), vstr1 = R(F(0)), shf0 = R(F(0));
    R evap0 = R(F(0)), rlus0 = R(F(0)), t1_1 = R(F(0)), q1_1 = R(F(0)), denv2 = R(F(0));
    R tskin = R(F(0));
    const F astab = (flags & SPD_LSCASYM) ? F(0.5) : F(1.0);
    const F rdth = F(p.fstab) / F(p.dtheta);
    const bool land = (flags & SPD_LFLUXLAND) != 0;
    if (land) {
      const F rcp = F(1.0 / 1004.0);
      const R dt1 = F(vg.wvi[KX - 1][1]) * (ta1 - ta2);
      R t1_0 = F(0) + (ta1 + dt1);
      t1_1 = t1_0 - phi0 * dt1 / (F(2.0 / 7.0 * 1004.0 * 288.0) * F(vg.sigl[KX - 1]));
      const R t2_1 = ta1 + rcp * phi[KX - 1];
      const R t2_0 = t2_1 - rcp * phi0;
      if (val(ta1) > val(ta2)) {
        t1_0 = F(p.ftemp0) * t1_0 + (F(1) - F(p.ftemp0)) * t2_0;
        t1_1 = F(p.ftemp0) * t1_1 + (F(1) - F(p.ftemp0)) * t2_1;
      } else {
        t1_0 = ta1;
        t1_1 = ta1;
      }
      const R t0 = t1_1 + in.fmask * (t1_0 - t1_1);
      const R denv0 = (F(1e5) * psa / (F(2.0 / 7.0 * 1004.0) * t0)) *
                      gsqrt(u0 * u0 + v0 * v0 + F(p.vgust) * F(p.vgust));
      tskin = in.stl + F(p.ctday) * in.sqrt_coa * rsds * (F(1) - alb_l) * psa;
      const R dthl = (val(tskin) > val(t2_0)) ? gmin(F(p.dtheta), tskin - t2_0)
                                              : gmax(-F(p.dtheta), astab * (tskin - t2_0));
      const R denv1 = denv0 * (F(1) + dthl * rdth);
      const F rhdrag = F(1) / (F(9.81) * F(p.hdrag));
      const F ph = in.phis0 > F(0) ? in.phis0 : F(0);
      const F forog = F(1) + rhdrag * (F(1) - (F)exp(-ph * rhdrag));
      const R cdldv = F(p.cdl) * denv0 * forog;
      ustr0 = -cdldv * ua;
      vstr0 = -cdldv * va;
      const F chlcp = F(p.chl) * F(1004.0);
      shf0 = chlcp * denv1 * (tskin - t1_0);
      const R q1_0 = (F(p.fhum0) > F(0))
                         ? F(p.fhum0) * (rh[KX - 1] * qsat_g<R, F>(t1_0, psa, F(1))) +
                               (F(1) - F(p.fhum0)) * q[KX - 1]
                         : q[KX - 1];
      const R qs00 = qsat_g<R, F>(tskin, psa, F(1));
      evap0 = F(p.chl) * denv1 * gmax(F(0), in.soilw * qs00 - q1_0);
      const R tsk3 = tskin * tskin * tskin;
      const R drls = F(4.0) * esbc * tsk3;
      rlus0 = esbc * tsk3 * tskin;
      R hfl0 = rsds * (F(1) - alb_l) + rlds - (rlus0 + shf0 + (F(2501.0) * evap0));
      if (flags & SPD_LSKINEB) {
        const F clamb = F(p.clambda) + (snowc * (F(p.clambsn) - F(p.clambda)));
        hfl0 = hfl0 - (clamb * (tskin - in.stl));
        R qs01 = qsat_g<R, F>(tskin + F(1), psa, F(1));
        qs01 = (val(evap0) > F(0)) ? in.soilw * (qs01 - qs00) : R(F(0));
        const R dtskin = hfl0 / (clamb + drls + (F(p.chl) * denv1 * (F(1004.0) + (F(2501.0) * qs01))));
        tskin = tskin + dtskin;
        shf0 = shf0 + chlcp * denv1 * dtskin;
        evap0 = evap0 + F(p.chl) * denv1 * qs01 * dtskin;
        rlus0 = rlus0 + drls * dtskin;
      }
      const R dths = (in.sst > val(t2_1)) ? gmin(F(p.dtheta), in.sst - t2_1)
                                          : gmax(-F(p.dtheta), astab * (in.sst - t2_1));
      denv2 = denv0 * (F(1) + dths * rdth);
      q1_1 = (F(p.fhum0) > F(0))
                 ? F(p.fhum0) * (rh[KX - 1] * qsat_g<R, F>(t1_1, psa, F(1))) +
                       (F(1) - F(p.fhum0)) * q[KX - 1]
                 : q[KX - 1];
      const R cdsdv = F(p.cds) * denv2;
      ustr1 = -cdsdv * ua;
      vstr1 = -cdsdv * va;
    }
    const R shf1 = F(p.chs) * F(1004.0) * denv2 * (in.sst - t1_1);
    const R evap1 = F(p.chs) * denv2 * (qsat_g<R, F>(R(in.sst), psa, F(1)) - q1_1);
    const F rlus1 = esbc * ((in.sst * in.sst) * (in.sst * in.sst));
    R ustr2 = R(F(0)), vstr2 = R(F(0)), shf2 = R(F(0)), evap2 = R(F(0));
    if (land) {
      const F fm = in.fmask;
      ustr2 = ustr1 + fm * (ustr0 - ustr1);
      vstr2 = vstr1 + fm * (vstr0 - vstr1);
      shf2 = shf1 + fm * (shf0 - shf1);
      evap2 = evap1 + fm * (evap0 - evap1);
      rlus2 = rlus1 + fm * (rlus0 - rlus1);
      tsfc = in.sst + fm * (in.stl - in.sst);
    }
    const R rps = F(1) / psa;
    o.du_low = F(0) + ustr2 * rps * F(vg.grdsig[KX - 1]);
    o.dv_low = F(0) + vstr2 * rps * F(vg.grdsig[KX - 1]);
    o.dt[KX - 1] = o.dt[KX - 1] + (F(0) + shf2 * rps * F(vg.grdscp[KX - 1]));
    o.dq[KX - 1] = o.dq[KX - 1] + (F(0) + evap2 * rps * F(vg.grdsig[KX - 1]));
  }

  // ---- get_upward_longwave_rad_fluxes (longwave_radiation.py:119-202) ----
  {
    const F refsfc = F(1) - F(p.emisfc);
    R fb[4], fl[4];
    radset_r(R(tsfc), F(p.epslw), fb);
    const R fsw[4] = {flux_sw0, flux_sw1, R(F(0)), R(F(0))};
    SPD_ROLL
    for (int b = 0; b < 4; ++b) fl[b] = fb[b] * rlus2 + refsfc * fsw[b];
    dfl[KX - 1] = dfl[KX - 1] + F(p.epslw) * rlus2;
    R sk = ((fl[0] + fl[1]) + fl[2]) + fl[3];
    SPD_ROLL
    for (int k = KX - 1; k >= 1; --k) {
      radset_r(t[k], F(p.epslw), fb);
      SPD_ROLL
      for (int b = 0; b < 4; ++b) {
        const R emis = F(1) - tau[k][b];
        fl[b] = tau[k][b] * fl[b] + emis * (fb[b] * (st0[k] - emis * st1[k]));
      }
      const R skm1 = ((fl[0] + fl[1]) + fl[2]) + fl[3];
      dfl[k] = dfl[k] + (sk - skm1);
      sk = skm1;
    }
    radset_r(t[0], F(p.epslw), fb);
    R top[4];
    SPD_ROLL
    for (int b = 0; b < 4; ++b) {
      const R emis = F(1) - tau[0][b];
      top[b] = (b < 2) ? tau[0][b] * fl[b] + emis * (fb[b] * (st0[0] - emis * st1[0])) : fl[b];
    }
    dfl[0] = dfl[0] + ((fl[0] - top[0]) + (fl[1] - top[1]));
    const F eps1 = F(p.epslw) / (F(vg.dhs[0]) + F(vg.dhs[1]));
    const R stratc0 = in.stratz * psa, stratc1 = eps1 * psa;
    const R corlw1 = F(vg.dhs[0]) * stratc1 * st0[0] + stratc0;
    const R corlw2 = F(vg.dhs[1]) * stratc1 * st0[1];
    dfl[0] = dfl[0] + (-corlw1);
    dfl[1] = dfl[1] + (-corlw2);
    SPD_ROLL
    for (int k = 0; k < KX; ++k) o.dt[k] = o.dt[k] + dfl[k] * F(vg.grdscp[k]) / psa;
  }

  // ---- get_vertical_diffusion_tend (vertical_diffusion.py:10-136) ----
  {
    const int nl1 = KX - 1;
    const int icnv = KX - iptop - 1;
    R tt[KX], qt[KX];
    SPD_ROLL
    for (int k = 0; k < KX; ++k) tt[k] = qt[k] = R(F(0));
    const F cshc = F(vg.dhs[KX - 1]) / F(3600.0);
    const F cvdi = (F(vg.hsg[nl1]) - F(vg.hsg[1])) / (F(nl1 - 1) * F(3600.0));
    const F fshcq = cshc / F(p.trshc), fshcse = cshc / (F(p.trshc) * F(1004.0));
    const F fvdiq = cvdi / F(p.trvdi), fvdise = cvdi / (F(p.trvds) * F(1004.0));
    const F drh0 = F(p.rhgrad) * (F(vg.fsg[KX - 1]) - F(vg.fsg[nl1 - 1]));
    const F fvdiq2 = fvdiq * F(vg.hsg[nl1]);
    const R dmse = se[KX - 1] - se[nl1 - 1] + F(2501.0) * (q[KX - 1] - qsat[nl1 - 1]);
    const R drh = rh[KX - 1] - rh[nl1 - 1];
    const F fcnv = (icnv > 0 && val(dmse) >= F(0)) ? F(p.redshc) : F(1);
    if (val(dmse) >= F(0)) {
      const R fluxse = fcnv * fshcse * dmse;
      tt[nl1 - 1] = fluxse * (F(1) / F(vg.dhs[nl1 - 1]));
      tt[KX - 1] = -fluxse * (F(1) / F(vg.dhs[KX - 1]));
      if (val(drh) >= F(0)) {
        const R fq = fcnv * fshcq * qsat[KX - 1] * drh;
        qt[nl1 - 1] = fq * (F(1) / F(vg.dhs[nl1 - 1]));
        qt[KX - 1] = -fq * (F(1) / F(vg.dhs[KX - 1]));
      }
    } else if (val(dmse) < F(0) && val(drh) > drh0) {
      const R fq = fvdiq2 * qsat[nl1 - 1] * drh;
      qt[nl1 - 1] = fq * (F(1) / F(vg.dhs[nl1 - 1]));
      qt[KX - 1] = -fq * (F(1) / F(vg.dhs[KX - 1]));
    }
    R fluxq[KX];
    SPD_ROLL
    for (int k = 2; k < KX - 2; ++k) {
      const bool cond = F(vg.hsg[k + 1]) > F(0.5);
      const F d0 = F(p.rhgrad) * (F(vg.fsg[k + 1]) - F(vg.fsg[k]));
      const F f2 = fvdiq * F(vg.hsg[k + 1]);
      const R dr = rh[k + 1] - rh[k];
      fluxq[k] = (val(dr) >= d0 && cond) ? f2 * qsat[k] * dr : R(F(0));
      qt[k] = qt[k] + fluxq[k] * (F(1) / F(vg.dhs[k]));
    }
    SPD_ROLL
    for (int k = 2; k < KX - 2; ++k) qt[k + 1] = qt[k + 1] + (-fluxq[k] * (F(1) / F(vg.dhs[k + 1])));
    R fse[KX];
    SPD_ROLL
    for (int k = 0; k < nl1; ++k) {
      const R se0 = se[k + 1] - F(p.segrad) * (phi[k + 1] - phi[k]);
      fse[k] = (val(se[k]) < val(se0)) ? fvdise * (se0 - se[k]) : R(F(0));
      tt[k] = tt[k] + fse[k] * (F(1) / F(vg.dhs[k]));
    }
    R cum = R(F(0));
    SPD_ROLL
    for (int k = 0; k < nl1; ++k) {
      cum = cum + fse[k] * (F(1) / (F(1) - F(vg.hsg[k + 1])));
      tt[k + 1] = tt[k + 1] + (-cum);
    }
    SPD_ROLL
    for (int k = 0; k < KX; ++k) {
      o.dt[k] = o.dt[k] + tt[k];
      o.dq[k] = o.dq[k] + qt[k];
    }
  }
}

}  // namespace spdgen
