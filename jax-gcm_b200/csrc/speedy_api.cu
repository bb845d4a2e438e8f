// speedy_api.cu -- C-ABI entry points of the plain per-instance drop-in.
//
// spd_fwd runs the physics of every column (speedy_physics.py:88-127) on the caller's stream
// with the batched kernels of speedy_ensemble.cu over a one-member plan passed by value.  The
// one cross-column dependency is the instance's cloud-top level set S (an OR over the columns'
// clip(icltop, 0, kx-1), shortwave_radiation.py:62-68), which the shortwave of every column
// reads.  By default the call predicts S from the previous call on the same scratch:
//   1. ensemble_fused: every column whole, in one pass, its shortwave using the predicted S
//      while the columns OR their own cloud tops into the true S; the last block to finish
//      compares the two and keeps the true one as the next prediction;
//   2. ensemble_fixup: returns at once when the prediction held, else computes every column
//      again with the true S.
// With SPD_NO_SPECULATION (or SPD_ACCUMULATE_DIAGNOSTICS) a light launch forms S first
// (ensemble_levelset) and ensemble_fused reads it.  One thread owns one column
// (speedy_kernels.cuh, speedy_column_smem.cuh).
#include <cuda_runtime.h>
#include <stdint.h>

#include "speedy_ensemble.cuh"

namespace spd {

constexpr size_t kHeaderBytes = 256;  // launch words and level-set state, padding

static bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

namespace {
struct Span {
  uintptr_t lo, hi;  // [lo, hi)
};
Span span(const void* p, size_t n) {
  const uintptr_t a = reinterpret_cast<uintptr_t>(p);
  return Span{a, a + n * sizeof(float)};
}
bool overlap(const Span& a, const Span& b) { return a.lo < b.hi && b.lo < a.hi; }
}  // namespace

// True when an output field overlaps an input field or another output field.
static bool outputs_alias(const spd_desc_t* d, const spd_inputs_t* in, const spd_outputs_t* out) {
  const size_t C = (size_t)d->ix * d->il, L = (size_t)d->kx * C;
  const size_t W = (d->flags & SPD_LOW_LEVEL_WINDS) ? C : L;  // wind planes
  const Span ins[] = {span(in->u_wind, W), span(in->v_wind, W), span(in->temperature, L),
                      span(in->specific_humidity, L), span(in->geopotential, L),
                      span(in->normalized_surface_pressure, C), span(in->alb0, C),
                      span(in->sice_am, C), span(in->snowc_am, C), span(in->soilw_am, C),
                      span(in->stl_am, C), span(in->sea_surface_temperature, C),
                      span(in->fmask, C), span(in->orog, C), span(in->phis0, C),
                      span(in->sia, d->il), span(in->coa, d->il)};
  float* const diag[] = {out->cbmf, out->cloudc, out->cloudstr, out->rsds, out->rsns,
                         out->ftop_sw, out->rlds, out->rlns, out->ftop_lw, out->tsfc,
                         out->tskin, out->shf, out->evap};
  Span outs[6 + 13 + 2];
  int n = 0;
  outs[n++] = span(out->u_wind, W);
  outs[n++] = span(out->v_wind, W);
  outs[n++] = span(out->temperature, L);
  outs[n++] = span(out->specific_humidity, L);
  outs[n++] = span(out->precnv, C);
  outs[n++] = span(out->precls, C);
  for (float* p : diag)
    if (p) outs[n++] = span(p, C);
  if (out->iptop) outs[n++] = span(out->iptop, C);
  if (out->icltop) outs[n++] = span(out->icltop, C);
  for (int i = 0; i < n; ++i) {
    for (const Span& a : ins)
      if (overlap(outs[i], a)) return true;
    for (int j = 0; j < i; ++j)
      if (overlap(outs[i], outs[j])) return true;
  }
  return false;
}

int check_instance(const spd_desc_t* d, const spd_inputs_t* in, const spd_outputs_t* out) {
  if (!d || !in || !out) return SPD_ERR_NULL;
  if (d->kx != 7 && d->kx != 8 && d->kx != 16) return SPD_ERR_KX;
  if (d->ix <= 0 || d->il <= 0 || (int64_t)d->ix * d->il > (1 << 30)) return SPD_ERR_SHAPE;
  const void* req[] = {in->u_wind, in->v_wind, in->temperature, in->specific_humidity,
                       in->geopotential, in->normalized_surface_pressure, in->alb0, in->sice_am,
                       in->snowc_am, in->soilw_am, in->stl_am, in->sea_surface_temperature,
                       in->fmask, in->orog, in->phis0, in->sia, in->coa, out->u_wind,
                       out->v_wind, out->temperature, out->specific_humidity, out->precnv,
                       out->precls};
  for (const void* p : req)
    if (!p) return SPD_ERR_NULL;
  for (const void* p : req)
    if (!aligned16(p)) return SPD_ERR_ALIGN;
  return SPD_OK;
}

// check_instance plus the forward's own rule: its outputs overlap neither its inputs nor one
// another (a column's outputs are written while other columns still read their inputs).
int check_forward_instance(const spd_desc_t* d, const spd_inputs_t* in,
                           const spd_outputs_t* out) {
  const int rc = check_instance(d, in, out);
  if (rc != SPD_OK) return rc;
  return outputs_alias(d, in, out) ? SPD_ERR_ALIAS : SPD_OK;
}

Consts make_consts(const spd_desc_t* d, const spd_vgrid_t* vg, const spd_params_t* p) {
  Consts K;
  K.vg = *vg;
  K.p = *p;
  K.C = d->ix * d->il;
  K.il = d->il;
  K.flags = d->flags;
  K.tyear = d->tyear;
  K.model_year = d->model_year;
  K.model_step = d->model_step;
  K.co2_year_ref = d->co2_year_ref;
  K.dt_seconds = d->dt_seconds;
  K.q_tend_scale = d->q_tend_scale;
  return K;
}

// The forward of one instance: the batched kernels over an implicit one-member plan passed
// by value (tile t = columns t*kNT ..), one block per tile.  The plain and the batched path
// therefore run the same code and agree bitwise.  `header` is the instance's 256-byte scratch
// header: words 0-1 the launch words, 4-6 the level-set state T, R, P (stride 1), 7 the
// cumulative count of redone calls; words 0-5 are cleared by every call, P and the count kept.
int dispatch_fwd(const ConstsD& CD, int kx, const spd_inputs_t& in, const spd_outputs_t& out,
                 uint32_t* header, cudaStream_t st, cudaEvent_t marker) {
  if (kx != 7 && kx != 8 && kx != 16) return SPD_ERR_KX;
  ClassArgs A;
  A.cls[0] = CD;
  TileSource T{};
  T.single.in = in;
  T.single.out = out;
  T.single.C = CD.K.C;
  T.single.il = CD.K.il;
  T.single.kx = kx;
  T.single.cls = 0;
  T.single.S = header + 4;
  T.single.ls_stride = 1;
  T.nmembers = 1;
  T.launch = header;
  T.redone = header + 7;
  const bool speculate =
      (CD.K.flags & (SPD_ACCUMULATE_DIAGNOSTICS | SPD_NO_SPECULATION)) == 0;
  const int ntiles = (CD.K.C + kNT - 1) / kNT;
  return launch_forward(A, T, ntiles, kx, SPD_GRID_PER_TILE, speculate, 6 * sizeof(uint32_t),
                        st, marker);
}

int preload_ensemble();
int preload_adjoint();
int preload_held_suarez();

}  // namespace spd

extern "C" {

int spd_preload(void) {
  const int b = spd::preload_ensemble();
  const int c = spd::preload_adjoint();
  const int h = spd::preload_held_suarez();
  return (b == SPD_OK && c == SPD_OK && h == SPD_OK) ? SPD_OK : SPD_ERR_CUDA;
}


size_t spd_fwd_scratch_bytes(const spd_desc_t* desc) {
  if (!desc || desc->il <= 0) return 0;
  return spd::kHeaderBytes;
}

int spd_fwd(const spd_desc_t* desc, const spd_vgrid_t* vgrid, const spd_params_t* params,
            const spd_inputs_t* in, const spd_outputs_t* out, void* scratch,
            size_t scratch_bytes, void* stream) {
  return spd_fwd_marked(desc, vgrid, params, in, out, scratch, scratch_bytes, stream, nullptr);
}

int spd_fwd_marked(const spd_desc_t* desc, const spd_vgrid_t* vgrid, const spd_params_t* params,
                   const spd_inputs_t* in, const spd_outputs_t* out, void* scratch,
                   size_t scratch_bytes, void* stream, void* event) {
  int rc = spd::check_forward_instance(desc, in, out);
  if (rc != SPD_OK) return rc;
  if (!vgrid || !params) return SPD_ERR_NULL;
  if (!scratch || (reinterpret_cast<uintptr_t>(scratch) & 255u) ||
      scratch_bytes < spd_fwd_scratch_bytes(desc))
    return SPD_ERR_SCRATCH;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  spd::ConstsD CD;
  CD.K = spd::make_consts(desc, vgrid, params);
  CD.D = spd::derive_constants(desc, vgrid, params);
  return spd::dispatch_fwd(CD, desc->kx, *in, *out, static_cast<uint32_t*>(scratch), st,
                           static_cast<cudaEvent_t>(event));
}

const char* spd_status_string(int status) {
  switch (status) {
    case SPD_OK: return "ok";
    case SPD_ERR_NULL: return "a required pointer is NULL";
    case SPD_ERR_SHAPE: return "shape out of range";
    case SPD_ERR_KX: return "unsupported level count (supported: 7, 8, 16)";
    case SPD_ERR_SCRATCH: return "scratch buffer NULL, too small or not 256-byte aligned";
    case SPD_ERR_CUDA: return "CUDA launch or runtime call failed";
    case SPD_ERR_ALIGN: return "a field pointer is not 16-byte aligned";
    case SPD_ERR_NOALLOC_LIMIT:
      return "instance has more latitudes than spd_fwd_noalloc's fixed scratch holds "
             "(SPD_NOALLOC_MAX_IL)";
    case SPD_ERR_ALIAS: return "an output field overlaps an input field or another output";
    case SPD_ERR_STREAM_DEVICE:
      return "the stream belongs to another device than the current one (spd_fwd_noalloc)";
    default: return "unknown status";
  }
}

int spd_abi_version(void) { return SPD_ABI_VERSION; }

void spd_default_params(spd_params_t* p) {
  if (!p) return;
  *p = spd_params_t{};
  p->psmin = 0.8f; p->trcnv = 6.0f; p->rhil = 0.7f; p->rhbl = 0.9f; p->entmax = 0.5f;
  p->smf = 0.8f;
  p->trlsc = 4.0f; p->rhlsc = 0.9f; p->drhlsc = 0.1f; p->rhblsc = 0.95f;
  p->albcl = 0.43f; p->albcls = 0.50f; p->absdry = 0.033f; p->absaer = 0.033f;
  p->abswv1 = 0.022f; p->abswv2 = 15.0f; p->abscl1 = 0.015f; p->abscl2 = 0.15f;
  p->ablwin = 0.3f; p->ablwv1 = 0.7f; p->ablwv2 = 50.0f; p->ablcl1 = 12.0f; p->ablcl2 = 0.6f;
  p->rhcl1 = 0.30f; p->rhcl2 = 1.0f; p->qacl = 0.20f; p->wpcl = 0.2f; p->pmaxcl = 10.0f;
  p->clsmax = 0.60f; p->clsminl = 0.15f; p->gse_s0 = 0.25f; p->gse_s1 = 0.40f;
  p->albsea = 0.07f; p->albice = 0.60f; p->albsn = 0.60f; p->epslw = 0.05f; p->emisfc = 0.98f;
  p->fwind0 = 0.95f; p->ftemp0 = 1.0f; p->fhum0 = 0.0f; p->cdl = 2.4e-3f; p->cds = 1.0e-3f;
  p->chl = 1.2e-3f; p->chs = 0.9e-3f; p->vgust = 5.0f; p->ctday = 1.0e-2f; p->dtheta = 3.0f;
  p->fstab = 0.67f; p->clambda = 7.0f; p->clambsn = 7.0f; p->hdrag = 2000.0f;
  p->trshc = 6.0f; p->trvdi = 24.0f; p->trvds = 6.0f; p->redshc = 0.5f; p->rhgrad = 0.5f;
  p->segrad = 0.1f;
}

}  // extern "C"
