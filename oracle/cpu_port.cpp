// cpu_port.cpp -- compiled CPU restatement of JAX-GCM's SPEEDY physics
// (SpeedyPhysics.compute_tendencies, jcm/physics/speedy/speedy_physics.py:88-127) for the
// benchmark's timed CPU baseline.
//
// BENCHMARK AND TEST INFRASTRUCTURE ONLY.  The reference itself is JAX and cannot be installed
// in this image; this is the CPU arm it is compared with: float32 arithmetic, -O3 without
// fast-math, OpenMP over columns on the host's cores.  Per column it runs the generic column
// (jax-gcm_b200/csrc/speedy_generic.h, R = F = float), which restates the reference term by term.
// Only the benchmark's cpu_baseline and reference arms and the tests load it (through
// oracle/cpu_port.py); the CUDA product path never does.
//
// One instance takes two passes over its columns: the terms up to the clouds, to form the
// instance's cloud-top level set S (shortwave_radiation.py:62-68, an OR over every column's
// clipped icltop), then every term with S.  The reference forms S between its cloud and
// shortwave terms, with all columns' clouds done; a column-at-a-time loop needs the first pass
// for it (it costs the humidity, convection, condensation and cloud terms a second time).
#include <math.h>
#include <omp.h>
#include <stdint.h>

#include <algorithm>
#include <vector>

#include "speedy_generic.h"

namespace {

// Per-latitude solar row (get_zonal_average_fields, shortwave_radiation.py:220-296; solar,
// :406-452), float32, and sqrt(coa) for the skin temperature (surface_flux.py:132).
struct SolarRow {
  float fsol, ozupp, ozone, zenit, stratz, sqrt_coa;
};

SolarRow solar_row(float tyear, float sia, float coa) {
  const float pigr = 2.0f * asinf(1.0f);
  const float a1 = 2.0f * pigr * tyear;
  const float ca1 = cosf(a1), sa1 = sinf(a1);
  const float ca2 = ca1 * ca1 - sa1 * sa1, sa2 = 2.0f * sa1 * ca1;
  const float ca3 = ca1 * ca2 - sa1 * sa2, sa3 = sa1 * ca2 + sa2 * ca1;
  const float decl = 0.006918f - 0.399912f * ca1 + 0.070257f * sa1 - 0.006758f * ca2 +
                     0.000907f * sa2 - 0.002697f * ca3 + 0.001480f * sa3;
  const float fdis =
      1.000110f + 0.034221f * ca1 + 0.001280f * sa1 + 0.000719f * ca2 + 0.000077f * sa2;
  const float cdecl = cosf(decl), sdecl = sinf(decl);
  const float tdecl = sdecl / cdecl;
  const float csolp = 1368.0f / pigr;
  float ch0 = -tdecl * sia / coa;
  ch0 = fminf(fmaxf(ch0, (float)(-1.0 + 1e-9)), (float)(1.0 - 1e-9));
  const float h0 = acosf(ch0);
  const float fsol = csolp * fdis * (h0 * sia * sdecl + sinf(h0) * coa * cdecl);
  const float asin1 = asinf(1.0f);
  const float alpha = 4.0f * asin1 * (tyear + (float)(10.0 / 365.0));
  const float coz1 = fmaxf(0.0f, cosf(alpha - 0.0f));
  const float rzen = -cosf(alpha) * 23.45f * asin1 / 90.0f;
  const float flat2 = 1.5f * (sia * sia) - 0.5f;
  const float ozone = (float)(0.4 * 0.02) * (1.0f + coz1 * sia + 1.8f * flat2);
  const float base = 1.0f - (coa * cosf(rzen) + sia * sinf(rzen));
  const float zenit = 1.0f + base * base;
  SolarRow r;
  r.fsol = fsol;
  r.ozupp = fsol * 0.01f * zenit;
  r.ozone = fsol * ozone * zenit;
  r.zenit = zenit;
  r.stratz = fmaxf(6.0f - fsol, 0.0f);
  r.sqrt_coa = sqrtf(coa);
  return r;
}

}  // namespace

extern "C" {

// One grid instance in the reference layout: level fields [kx][ix][il], surface fields
// [ix][il], latitude tables [il]; column c = i * il + j.  Outputs: the four tendency planes
// (u and v non-zero at the lowest level only, as the reference returns them), precnv, precls,
// cloudc, rsds, rlds, iptop, icltop (any of the last seven may be NULL).
typedef struct {
  int kx, ix, il;
  uint32_t flags;
  int model_step;
  float tyear, ablco2;
  const float *u, *v, *t, *q, *phi, *psa, *sst, *stl, *soilw, *snowc, *sice, *alb0, *fmask,
      *orog, *phis0, *sia, *coa;
  float *du, *dv, *dt, *dq, *precnv, *precls, *cloudc, *rsds, *rlds;
  int32_t *iptop, *icltop;
} cpu_port_instance_t;

}  // extern "C"

namespace {

template <int KX>
void gather(const cpu_port_instance_t& I, const SolarRow* rows, int c,
            spdgen::ColumnIn<float, float>& in) {
  const size_t C = (size_t)I.ix * I.il;
  for (int k = 0; k < KX; ++k) {
    in.t[k] = I.t[k * C + c];
    in.q[k] = I.q[k * C + c];
    in.phi[k] = I.phi[k * C + c];
  }
  in.psa = I.psa[c];
  in.u_low = I.u[(KX - 1) * C + c];
  in.v_low = I.v[(KX - 1) * C + c];
  in.sst = I.sst[c];
  in.stl = I.stl[c];
  in.soilw = I.soilw[c];
  in.snowc = I.snowc[c];
  in.sice = I.sice[c];
  in.alb0 = I.alb0[c];
  in.fmask = I.fmask[c];
  in.orog = I.orog[c];
  in.phis0 = I.phis0[c];
  const SolarRow& z = rows[c % I.il];
  in.fsol = z.fsol;
  in.ozupp = z.ozupp;
  in.ozone = z.ozone;
  in.zenit = z.zenit;
  in.stratz = z.stratz;
  in.sqrt_coa = z.sqrt_coa;
}

spdgen::DiffParams<float> diff_params(const spd_params_t& p) {
  spdgen::DiffParams<float> g;
  g.psmin = p.psmin; g.trcnv = p.trcnv; g.rhil = p.rhil; g.rhbl = p.rhbl; g.entmax = p.entmax;
  g.smf = p.smf; g.trlsc = p.trlsc; g.rhlsc = p.rhlsc; g.drhlsc = p.drhlsc;
  g.rhblsc = p.rhblsc; g.albcl = p.albcl; g.albcls = p.albcls;
  return g;
}

// Pass 1 over columns [c0, c1): the OR of their clipped cloud-top levels.
template <int KX>
uint32_t level_bits(const spd_vgrid_t& vg, const spd_params_t& p,
                    const spdgen::DiffParams<float>& g, const cpu_port_instance_t& I,
                    const SolarRow* rows, int c0, int c1) {
  uint32_t S = 0;
  for (int c = c0; c < c1; ++c) {
    spdgen::ColumnIn<float, float> in;
    spdgen::ColumnOut<float> o;
    gather<KX>(I, rows, c, in);
    spdgen::column_generic<KX, float, float>(vg, p, g, I.flags, I.model_step, I.ablco2, 0u, in,
                                             o, true);
    const int l = o.icltop < 0 ? 0 : (o.icltop > KX - 1 ? KX - 1 : o.icltop);
    S |= 1u << l;
  }
  return S;
}

// Pass 2 over columns [c0, c1): every term with the instance's level set S, and the outputs.
template <int KX>
void columns(const spd_vgrid_t& vg, const spd_params_t& p, const spdgen::DiffParams<float>& g,
             const cpu_port_instance_t& I, const SolarRow* rows, uint32_t S, int c0, int c1) {
  const size_t Cs = (size_t)I.ix * I.il;
  for (int c = c0; c < c1; ++c) {
    spdgen::ColumnIn<float, float> in;
    spdgen::ColumnOut<float> o;
    gather<KX>(I, rows, c, in);
    spdgen::column_generic<KX, float, float>(vg, p, g, I.flags, I.model_step, I.ablco2, S, in,
                                             o);
    for (int k = 0; k < KX; ++k) {
      I.dt[k * Cs + c] = o.dt[k];
      I.dq[k * Cs + c] = o.dq[k];
      I.du[k * Cs + c] = k == KX - 1 ? o.du_low : 0.0f;
      I.dv[k * Cs + c] = k == KX - 1 ? o.dv_low : 0.0f;
    }
    if (I.precnv) I.precnv[c] = o.precnv;
    if (I.precls) I.precls[c] = o.precls;
    if (I.cloudc) I.cloudc[c] = o.cloudc;
    if (I.rsds) I.rsds[c] = o.rsds;
    if (I.rlds) I.rlds[c] = o.rlds;
    if (I.iptop) I.iptop[c] = o.iptop;
    if (I.icltop) I.icltop[c] = o.icltop;
  }
}

uint32_t level_bits_any(const spd_vgrid_t& vg, const spd_params_t& p,
                        const spdgen::DiffParams<float>& g, const cpu_port_instance_t& I,
                        const SolarRow* rows, int c0, int c1) {
  switch (I.kx) {
    case 7: return level_bits<7>(vg, p, g, I, rows, c0, c1);
    case 8: return level_bits<8>(vg, p, g, I, rows, c0, c1);
    default: return level_bits<16>(vg, p, g, I, rows, c0, c1);
  }
}

void columns_any(const spd_vgrid_t& vg, const spd_params_t& p, const spdgen::DiffParams<float>& g,
                 const cpu_port_instance_t& I, const SolarRow* rows, uint32_t S, int c0, int c1) {
  switch (I.kx) {
    case 7: columns<7>(vg, p, g, I, rows, S, c0, c1); break;
    case 8: columns<8>(vg, p, g, I, rows, S, c0, c1); break;
    default: columns<16>(vg, p, g, I, rows, S, c0, c1); break;
  }
}

constexpr int kChunk = 256;  // columns per work item

struct Chunk {
  int inst, c0, c1;
};

}  // namespace

extern "C" {

// Runs n instances (each with its own vertical grid and parameters) on `nthreads` OpenMP
// threads (0: OpenMP's default) in one parallel region: the per-latitude solar tables, then
// pass 1 over every instance's columns in chunks of kChunk (forming each level set), then
// pass 2.  `rows` is caller scratch of 6 floats per latitude of every instance, in order.
// Returns 0, or -1 - i for an instance i with an unsupported level count.
int cpu_port_forward_many(const spd_vgrid_t* vgs, const spd_params_t* ps,
                          const cpu_port_instance_t* insts, int n, float* rows, int nthreads) {
  for (int i = 0; i < n; ++i)
    if (insts[i].kx != 7 && insts[i].kx != 8 && insts[i].kx != 16) return -1 - i;
  std::vector<Chunk> chunks;
  std::vector<size_t> row0(n);
  std::vector<spdgen::DiffParams<float>> gs(n);
  size_t r = 0;
  for (int i = 0; i < n; ++i) {
    row0[i] = r;
    r += (size_t)insts[i].il;
    gs[i] = diff_params(ps[i]);
    const int C = insts[i].ix * insts[i].il;
    for (int c0 = 0; c0 < C; c0 += kChunk) chunks.push_back(Chunk{i, c0, std::min(C, c0 + kChunk)});
  }
  SolarRow* R = reinterpret_cast<SolarRow*>(rows);
  std::vector<uint32_t> S(n, 0u);
  const int nch = (int)chunks.size();
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel
  {
#pragma omp for schedule(static)
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < insts[i].il; ++j)
        R[row0[i] + j] = solar_row(insts[i].tyear, insts[i].sia[j], insts[i].coa[j]);
#pragma omp for schedule(dynamic, 1)
    for (int w = 0; w < nch; ++w) {
      const Chunk& ch = chunks[w];
      const uint32_t b =
          level_bits_any(vgs[ch.inst], ps[ch.inst], gs[ch.inst], insts[ch.inst],
                         R + row0[ch.inst], ch.c0, ch.c1);
#pragma omp atomic
      S[ch.inst] |= b;
    }
#pragma omp for schedule(dynamic, 1)
    for (int w = 0; w < nch; ++w) {
      const Chunk& ch = chunks[w];
      columns_any(vgs[ch.inst], ps[ch.inst], gs[ch.inst], insts[ch.inst], R + row0[ch.inst],
                  S[ch.inst], ch.c0, ch.c1);
    }
  }
  return 0;
}

// One instance (cpu_port_forward_many with n = 1).
int cpu_port_forward(const spd_vgrid_t* vg, const spd_params_t* p,
                     const cpu_port_instance_t* inst, float* rows, int nthreads) {
  return cpu_port_forward_many(vg, p, inst, 1, rows, nthreads);
}

int cpu_port_max_threads(void) { return omp_get_max_threads(); }

}  // extern "C"
