// spd_ffi.cc -- XLA FFI handlers around spd_fwd and spd_vjp: the jax.ffi side of the drop-in
// for SpeedyPhysics.compute_tendencies (jcm/physics/speedy/speedy_physics.py:88-127), called
// from jcm/physics_interface.py:137-152 through a Physics subclass (jax_physics.py).
//
// Built only where jaxlib's FFI headers exist (jax.ffi.include_dir()), by jax_physics.build_ffi;
// it links against libspeedy_b200.so.
//
// Static per model (attributes): the descriptor without its date fields, the vertical grid and
// the parameters, as byte images of spd_desc_t / spd_vgrid_t / spd_params_t.  Traced per step
// (operands): the date, as a 3-element int32 buffer {float32 bits of tyear, model_year,
// model_step} -- the library takes the date by value on the host, so the handler reads these 12
// bytes back on the call's stream and waits for them (one small device-to-host copy per call).
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include "speedy_b200.h"
#include "xla/ffi/api/ffi.h"

namespace ffi = xla::ffi;

namespace {

template <class T>
bool image(ffi::Span<const uint8_t> bytes, T* out) {
  if (bytes.size() != sizeof(T)) return false;
  memcpy(out, bytes.begin(), sizeof(T));
  return true;
}

ffi::Error status_error(int rc) {
  return ffi::Error(ffi::ErrorCode::kInternal, spd_status_string(rc));
}

// The traced date into the descriptor.
ffi::Error read_date(cudaStream_t st, ffi::Buffer<ffi::S32> date, spd_desc_t* d) {
  if (date.element_count() != 3)
    return ffi::Error(ffi::ErrorCode::kInvalidArgument, "date must hold 3 int32 words");
  int32_t h[3];
  if (cudaMemcpyAsync(h, date.typed_data(), sizeof(h), cudaMemcpyDeviceToHost, st) !=
          cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return status_error(SPD_ERR_CUDA);
  memcpy(&d->tyear, &h[0], sizeof(float));
  d->model_year = h[1];
  d->model_step = h[2];
  return ffi::Error::Success();
}

using F32 = ffi::Buffer<ffi::F32>;
using R32 = ffi::ResultBuffer<ffi::F32>;

spd_inputs_t inputs(F32 u, F32 v, F32 t, F32 q, F32 phi, F32 psa, F32 alb0, F32 sice,
                    F32 snowc, F32 soilw, F32 stl, F32 sst, F32 fmask, F32 orog, F32 phis0,
                    F32 sia, F32 coa) {
  spd_inputs_t in;
  in.u_wind = u.typed_data();
  in.v_wind = v.typed_data();
  in.temperature = t.typed_data();
  in.specific_humidity = q.typed_data();
  in.geopotential = phi.typed_data();
  in.normalized_surface_pressure = psa.typed_data();
  in.alb0 = alb0.typed_data();
  in.sice_am = sice.typed_data();
  in.snowc_am = snowc.typed_data();
  in.soilw_am = soilw.typed_data();
  in.stl_am = stl.typed_data();
  in.sea_surface_temperature = sst.typed_data();
  in.fmask = fmask.typed_data();
  in.orog = orog.typed_data();
  in.phis0 = phis0.typed_data();
  in.sia = sia.typed_data();
  in.coa = coa.typed_data();
  return in;
}

ffi::Error SpdFwd(cudaStream_t st, F32 u, F32 v, F32 t, F32 q, F32 phi, F32 psa, F32 alb0,
                  F32 sice, F32 snowc, F32 soilw, F32 stl, F32 sst, F32 fmask, F32 orog,
                  F32 phis0, F32 sia, F32 coa, ffi::Buffer<ffi::S32> date,
                  ffi::Span<const uint8_t> desc_b, ffi::Span<const uint8_t> vgrid_b,
                  ffi::Span<const uint8_t> params_b, R32 du, R32 dv, R32 dt, R32 dq,
                  R32 precnv, R32 precls, ffi::ResultBuffer<ffi::U8> scratch) {
  spd_desc_t d;
  spd_vgrid_t vg;
  spd_params_t p;
  if (!image(desc_b, &d) || !image(vgrid_b, &vg) || !image(params_b, &p))
    return ffi::Error(ffi::ErrorCode::kInvalidArgument, "struct image of the wrong size");
  ffi::Error e = read_date(st, date, &d);
  if (e.failure()) return e;
  const spd_inputs_t in = inputs(u, v, t, q, phi, psa, alb0, sice, snowc, soilw, stl, sst,
                                 fmask, orog, phis0, sia, coa);
  spd_outputs_t out;
  memset(&out, 0, sizeof(out));
  out.u_wind = du->typed_data();
  out.v_wind = dv->typed_data();
  out.temperature = dt->typed_data();
  out.specific_humidity = dq->typed_data();
  out.precnv = precnv->typed_data();
  out.precls = precls->typed_data();
  const int rc = spd_fwd(&d, &vg, &p, &in, &out, scratch->typed_data(), scratch->size_bytes(),
                         st);
  return rc ? status_error(rc) : ffi::Error::Success();
}

ffi::Error SpdVjp(cudaStream_t st, F32 u, F32 v, F32 t, F32 q, F32 phi, F32 psa, F32 alb0,
                  F32 sice, F32 snowc, F32 soilw, F32 stl, F32 sst, F32 fmask, F32 orog,
                  F32 phis0, F32 sia, F32 coa, ffi::Buffer<ffi::S32> date, F32 ct_u, F32 ct_v,
                  F32 ct_t, F32 ct_q, ffi::Span<const uint8_t> desc_b,
                  ffi::Span<const uint8_t> vgrid_b, ffi::Span<const uint8_t> params_b, R32 gu,
                  R32 gv, R32 gt, R32 gq, R32 gphi, R32 gpsa, R32 gparams,
                  ffi::ResultBuffer<ffi::U8> scratch) {
  spd_desc_t d;
  spd_vgrid_t vg;
  spd_params_t p;
  if (!image(desc_b, &d) || !image(vgrid_b, &vg) || !image(params_b, &p))
    return ffi::Error(ffi::ErrorCode::kInvalidArgument, "struct image of the wrong size");
  ffi::Error e = read_date(st, date, &d);
  if (e.failure()) return e;
  const spd_inputs_t in = inputs(u, v, t, q, phi, psa, alb0, sice, snowc, soilw, stl, sst,
                                 fmask, orog, phis0, sia, coa);
  spd_cotangents_t ct;
  ct.u_wind = ct_u.typed_data();
  ct.v_wind = ct_v.typed_data();
  ct.temperature = ct_t.typed_data();
  ct.specific_humidity = ct_q.typed_data();
  spd_grads_t g;
  g.u_wind = gu->typed_data();
  g.v_wind = gv->typed_data();
  g.temperature = gt->typed_data();
  g.specific_humidity = gq->typed_data();
  g.geopotential = gphi->typed_data();
  g.normalized_surface_pressure = gpsa->typed_data();
  g.params = gparams->typed_data();
  const int rc = spd_vjp(&d, &vg, &p, &in, &ct, &g, scratch->typed_data(),
                         scratch->size_bytes(), st);
  return rc ? status_error(rc) : ffi::Error::Success();
}

}  // namespace

#define SPD_FFI_INPUTS                                                                   \
  .Arg<F32>().Arg<F32>().Arg<F32>().Arg<F32>().Arg<F32>().Arg<F32>().Arg<F32>().Arg<F32>() \
      .Arg<F32>().Arg<F32>().Arg<F32>().Arg<F32>().Arg<F32>().Arg<F32>().Arg<F32>()        \
      .Arg<F32>().Arg<F32>().Arg<ffi::Buffer<ffi::S32>>()

XLA_FFI_DEFINE_HANDLER_SYMBOL(SpdFwdHandler, SpdFwd,
                              ffi::Ffi::Bind()
                                  .Ctx<ffi::PlatformStream<cudaStream_t>>()
                                  SPD_FFI_INPUTS
                                  .Attr<ffi::Span<const uint8_t>>("desc")
                                  .Attr<ffi::Span<const uint8_t>>("vgrid")
                                  .Attr<ffi::Span<const uint8_t>>("params")
                                  .Ret<F32>().Ret<F32>().Ret<F32>().Ret<F32>().Ret<F32>()
                                  .Ret<F32>().Ret<ffi::Buffer<ffi::U8>>());

XLA_FFI_DEFINE_HANDLER_SYMBOL(SpdVjpHandler, SpdVjp,
                              ffi::Ffi::Bind()
                                  .Ctx<ffi::PlatformStream<cudaStream_t>>()
                                  SPD_FFI_INPUTS
                                  .Arg<F32>().Arg<F32>().Arg<F32>().Arg<F32>()
                                  .Attr<ffi::Span<const uint8_t>>("desc")
                                  .Attr<ffi::Span<const uint8_t>>("vgrid")
                                  .Attr<ffi::Span<const uint8_t>>("params")
                                  .Ret<F32>().Ret<F32>().Ret<F32>().Ret<F32>().Ret<F32>()
                                  .Ret<F32>().Ret<F32>().Ret<ffi::Buffer<ffi::U8>>());
