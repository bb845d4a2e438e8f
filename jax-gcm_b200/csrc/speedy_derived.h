// speedy_derived.h -- launch-uniform constants of the SPEEDY column physics.
//
// Everything here depends only on the parameters, the vertical grid and the date, so it is
// evaluated once per launch on the host, in float32 and in the reference's expression order,
// and reaches the kernel through the constant bank.  Each entry cites the reference line it
// restates (paths relative to the JAX-GCM root).
#pragma once

#include <math.h>
#include <stdint.h>

#include "speedy_b200.h"

namespace spd {

struct Derived {
  float rsig[SPD_MAX_KX];     // 1/dhs                                (vertical_diffusion.py:54)
  float rsig1[SPD_MAX_KX];    // 1/(1-hsg[k+1]), 0 at kx-1            (vertical_diffusion.py:55-56)
  float entr[SPD_MAX_KX];     // scaled entrainment, k = 1..kx-2      (convection.py:135-137)
  float rhref[SPD_MAX_KX];    // LSC RH threshold                     (large_scale_condensation.py:298-299)
  float dqmax[SPD_MAX_KX];    // LSC max tendency                     (large_scale_condensation.py:300)
  float pfact[SPD_MAX_KX];    // dhs * p0/g                           (large_scale_condensation.py:314)
  float abs1[SPD_MAX_KX];     // SW dry + aerosol absorptivity        (shortwave_radiation.py:82,93)
  float drh0v[SPD_MAX_KX];    // vdiff RH-gradient thresholds         (vertical_diffusion.py:103)
  float fvdiq2v[SPD_MAX_KX];  // vdiff moisture coefficients          (vertical_diffusion.py:104)
  uint32_t vdcond;            // bit k: hsg[k+1] > 0.5                (vertical_diffusion.py:100)
  float fm0, rdps;            // convection.py:140-141
  float rtlsc;                // large_scale_condensation.py:285
  float fshcq, fshcse, fvdise, drh0, fvdiq2;  // vertical_diffusion.py:45-60
  float eps1;                 // shortwave_radiation.py:203
  float rhdrag;               // surface_flux.py:311
  float chlcp, esbc, rdth, astab, ghum0, gtemp0;  // surface_flux.py:75-76,135-137,102,153
  float w_lw, refsfc, corlw_f;  // longwave_radiation.py:226, :156, :100
  float ablco2;               // physics/speedy/forcing.py:136
  float rgas288_sigl;         // rgas*288*sigl[kx-1]                   (surface_flux.py:111)
  float rrcl, rgse;           // shortwave_radiation.py:348, :387
  float tcorv[SPD_MAX_KX];    // orographic temperature profile        (orographic_correction.py:18-55)
  float qcorv[SPD_MAX_KX];    // orographic humidity profile           (orographic_correction.py:58-93)
  float gamlat, pexp;         // orographic_correction.py:110, :151
  // date-only parts of the per-latitude solar row (get_zonal_average_fields,
  // shortwave_radiation.py:220-296; solar, :406-452); the kernels finish each column's row
  // from its latitude's sia and coa
  float sol_tdecl, sol_sdecl, sol_cdecl, sol_scale;  // tan/sin/cos(decl), csolp * fdis
  float coz1, cos_rzen, sin_rzen;
};

// Host evaluation (plain IEEE float32 arithmetic, no contraction on the host target).
inline Derived derive_constants(const spd_desc_t* d, const spd_vgrid_t* vg,
                                const spd_params_t* p) {
  Derived D = {};
  const int kx = d->kx;
  for (int k = 0; k < kx; ++k) {
    D.rsig[k] = 1.0f / vg->dhs[k];
    D.rsig1[k] = (k < kx - 1) ? 1.0f / (1.0f - vg->hsg[k + 1]) : 0.0f;
  }
  float sentr = 0.0f;
  for (int k = 1; k < kx - 1; ++k) {
    const float e = fmaxf(0.0f, vg->fsg[k] - 0.5f);
    D.entr[k] = e * e;
    sentr = sentr + D.entr[k];
  }
  const float escale = p->entmax / sentr;
  for (int k = 1; k < kx - 1; ++k) D.entr[k] = D.entr[k] * escale;
  D.fm0 = 1e5f * vg->dhs[kx - 1] / (9.81f * p->trcnv * 3600.0f);
  D.rdps = 2.0f / (1.0f - p->psmin);
  D.rtlsc = 1.0f / (p->trlsc * 3600.0f);
  const float prg = (float)(1e5 / 9.81);
  for (int k = 0; k < kx; ++k) {
    const float sig2 = vg->fsg[k] * vg->fsg[k];
    D.rhref[k] = fmaxf(p->rhlsc + p->drhlsc * (sig2 - 1.0f), p->rhblsc);
    D.dqmax[k] = 10.0f * sig2 * D.rtlsc;
    D.pfact[k] = vg->dhs[k] * prg;
    D.abs1[k] = p->absdry + p->absaer * sig2;
  }
  const int nl1 = kx - 1;
  const float cshc = vg->dhs[kx - 1] / 3600.0f;
  const float cvdi = (vg->hsg[nl1] - vg->hsg[1]) / ((float)(nl1 - 1) * 3600.0f);
  D.fshcq = cshc / p->trshc;
  D.fshcse = cshc / (p->trshc * 1004.0f);
  const float fvdiq = cvdi / p->trvdi;
  D.fvdise = cvdi / (p->trvds * 1004.0f);
  D.drh0 = p->rhgrad * (vg->fsg[kx - 1] - vg->fsg[nl1 - 1]);
  D.fvdiq2 = fvdiq * vg->hsg[nl1];
  D.vdcond = 0;
  for (int k = 2; k < kx - 2; ++k) {
    D.drh0v[k] = p->rhgrad * (vg->fsg[k + 1] - vg->fsg[k]);
    D.fvdiq2v[k] = fvdiq * vg->hsg[k + 1];
    if (vg->hsg[k + 1] > 0.5f) D.vdcond |= 1u << k;
  }
  D.eps1 = p->epslw / (vg->dhs[0] + vg->dhs[1]);
  D.rhdrag = 1.0f / (9.81f * p->hdrag);
  D.chlcp = p->chl * 1004.0f;
  D.esbc = p->emisfc * (float)5.67e-8;
  D.rdth = p->fstab / p->dtheta;
  D.astab = (d->flags & SPD_LSCASYM) ? 0.5f : 1.0f;
  D.ghum0 = 1.0f - p->fhum0;
  D.gtemp0 = 1.0f - p->ftemp0;
  D.w_lw = 1.0f - p->epslw;
  D.refsfc = 1.0f - p->emisfc;
  D.corlw_f = p->epslw * p->emisfc;
  D.ablco2 = 6.0f;
  if (d->flags & SPD_INCREASE_CO2)
    D.ablco2 = 6.0f * expf(0.005f * ((float)d->model_year + d->tyear - (float)d->co2_year_ref));
  D.rgas288_sigl = (float)(2.0 / 7.0 * 1004.0 * 288.0) * vg->sigl[kx - 1];
  D.rrcl = 1.0f / (p->rhcl2 - p->rhcl1);
  D.rgse = 1.0f / (p->gse_s1 - p->gse_s0);
  // orographic correction (orographic_correction.py): the reference evaluates these in float32
  // from double constants (rgas = 2/7 * 1004, gamma = 6, g = 9.81, hscale / hshum = 3)
  {
    const double rgas = 2.0 / 7.0 * 1004.0, gamma = 6.0, grav = 9.81;
    const float rgam = (float)(rgas * gamma / (1000.0 * grav));
    const float qexp = (float)(7.5 / 2.5);
    for (int k = 0; k < kx; ++k) {
      D.tcorv[k] = (k == 0) ? 0.0f : powf(vg->fsg[k], rgam);
      D.qcorv[k] = (k < 2) ? 0.0f : powf(vg->fsg[k], qexp);
    }
    D.gamlat = (float)(gamma / (1000.0 * grav));
    D.pexp = (float)(1000.0 * grav / (rgas * gamma));
  }
  {  // solar (shortwave_radiation.py:406-452), csol = 4 solc, the parts without latitude
    const float tyear = d->tyear;
    const float pigr = 2.0f * asinf(1.0f);
    const float alpha = 2.0f * pigr * tyear;
    const float ca1 = cosf(alpha), sa1 = sinf(alpha);
    const float ca2 = ca1 * ca1 - sa1 * sa1;
    const float sa2 = 2.0f * sa1 * ca1;
    const float ca3 = ca1 * ca2 - sa1 * sa2;
    const float sa3 = sa1 * ca2 + sa2 * ca1;
    const float decl = 0.006918f - 0.399912f * ca1 + 0.070257f * sa1 - 0.006758f * ca2 +
                       0.000907f * sa2 - 0.002697f * ca3 + 0.001480f * sa3;
    const float fdis =
        1.000110f + 0.034221f * ca1 + 0.001280f * sa1 + 0.000719f * ca2 + 0.000077f * sa2;
    D.sol_cdecl = cosf(decl);
    D.sol_sdecl = sinf(decl);
    D.sol_tdecl = D.sol_sdecl / D.sol_cdecl;
    D.sol_scale = (1368.0f / pigr) * fdis;
    // get_zonal_average_fields (shortwave_radiation.py:242-262)
    const float asin1 = asinf(1.0f);
    const float a2 = 4.0f * asin1 * (tyear + (float)(10.0 / 365.0));
    D.coz1 = fmaxf(0.0f, cosf(a2 - 0.0f));
    const float rzen = -cosf(a2) * 23.45f * asin1 / 90.0f;
    D.cos_rzen = cosf(rzen);
    D.sin_rzen = sinf(rzen);
  }
  return D;
}

}  // namespace spd
