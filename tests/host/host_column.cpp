// Host build of the generic column physics (jax-gcm_b200/csrc/speedy_generic.h) for the CPU
// tests: forward in float32 and float64, the reverse-mode VJP with the tape in host memory, and
// the hand-written reverse pass (jax-gcm_b200/csrc/speedy_vjp.h).  Test infrastructure only.
#include <cmath>
#include <cstdint>
#include <vector>

#include "speedy_derived.h"
#include "speedy_generic.h"
#include "speedy_vjp.h"

using spdad::Adj;
using spdad::TapeT;

struct HostColumn {
  int kx;
  uint32_t flags;
  int model_step;
  float ablco2;
  uint32_t S;
  float t[16], q[16], phi[16];
  float psa, u_low, v_low;
  float sst, stl, soilw, snowc, sice, alb0, fmask, orog, phis0;
  float fsol, ozupp, ozone, zenit, stratz, sqrt_coa;
};

struct HostOut {
  double dt[16], dq[16], du_low, dv_low, precnv, precls, cloudc, rsds, rlds;
  int iptop, icltop;
};

template <class R, class F>
static void fill_in(const HostColumn& h, spdgen::ColumnIn<R, F>& in) {
  for (int k = 0; k < h.kx; ++k) {
    in.t[k] = R(F(h.t[k]));
    in.q[k] = R(F(h.q[k]));
    in.phi[k] = R(F(h.phi[k]));
  }
  in.psa = R(F(h.psa));
  in.u_low = R(F(h.u_low));
  in.v_low = R(F(h.v_low));
  in.sst = h.sst; in.stl = h.stl; in.soilw = h.soilw; in.snowc = h.snowc; in.sice = h.sice;
  in.alb0 = h.alb0; in.fmask = h.fmask; in.orog = h.orog; in.phis0 = h.phis0;
  in.fsol = h.fsol; in.ozupp = h.ozupp; in.ozone = h.ozone; in.zenit = h.zenit;
  in.stratz = h.stratz; in.sqrt_coa = h.sqrt_coa;
}

template <class R>
static void fill_params(const spd_params_t& p, spdgen::DiffParams<R>& g) {
  g.psmin = R(p.psmin); g.trcnv = R(p.trcnv); g.rhil = R(p.rhil); g.rhbl = R(p.rhbl);
  g.entmax = R(p.entmax); g.smf = R(p.smf); g.trlsc = R(p.trlsc); g.rhlsc = R(p.rhlsc);
  g.drhlsc = R(p.drhlsc); g.rhblsc = R(p.rhblsc); g.albcl = R(p.albcl); g.albcls = R(p.albcls);
}

template <int KX, class F>
static void fwd(const spd_vgrid_t& vg, const spd_params_t& p, const HostColumn& h, HostOut& out) {
  spdgen::ColumnIn<F, F> in;
  fill_in(h, in);
  spdgen::DiffParams<F> g;
  fill_params(p, g);
  spdgen::ColumnOut<F> o;
  spdgen::column_generic<KX, F, F>(vg, p, g, h.flags, h.model_step, F(h.ablco2), h.S, in, o);
  for (int k = 0; k < KX; ++k) {
    out.dt[k] = o.dt[k];
    out.dq[k] = o.dq[k];
  }
  out.du_low = o.du_low; out.dv_low = o.dv_low; out.precnv = o.precnv; out.precls = o.precls;
  out.cloudc = o.cloudc; out.rsds = o.rsds; out.rlds = o.rlds;
  out.iptop = o.iptop; out.icltop = o.icltop;
}

// VJP in float64: ct_dt/ct_dq [kx], ct_du/ct_dv (lowest level).  Gradients: g_t, g_q, g_phi
// [kx], g_psa, g_u, g_v (lowest level), g_params[12].  Returns the tape length.
template <int KX, class T = double>
static int vjp(const spd_vgrid_t& vg, const spd_params_t& p, const HostColumn& h,
               const double* ct_dt, const double* ct_dq, double ct_du, double ct_dv,
               double* g_t, double* g_q, double* g_phi, double* g_psa, double* g_u,
               double* g_v, double* g_params, double dt_seconds = 1800.0,
               double q_tend_scale = 1.0) {
  typedef Adj<T> A;
  const int cap = 1 << 20;
  std::vector<int32_t> ia(cap), ib(cap);
  std::vector<T> pa(cap), pb(cap), adj(cap);
  TapeT<T> tp{ia.data(), ib.data(), pa.data(), pb.data(), adj.data(), 1, 0, cap, 0};
  auto leaf = [&](T v) { return A(v, tp.leaf(), &tp); };
  spdgen::DiffParams<A> g;
  g.psmin = leaf(p.psmin); g.trcnv = leaf(p.trcnv); g.rhil = leaf(p.rhil); g.rhbl = leaf(p.rhbl);
  g.entmax = leaf(p.entmax); g.smf = leaf(p.smf); g.trlsc = leaf(p.trlsc);
  g.rhlsc = leaf(p.rhlsc); g.drhlsc = leaf(p.drhlsc); g.rhblsc = leaf(p.rhblsc);
  g.albcl = leaf(p.albcl); g.albcls = leaf(p.albcls);
  spdgen::ColumnIn<A, T> in;
  fill_in(h, in);
  const bool verify = (h.flags & SPD_FUSE_VERIFY) != 0;
  A qraw[KX];
  for (int k = 0; k < KX; ++k) {
    in.t[k] = leaf(h.t[k]);
    qraw[k] = leaf(h.q[k]);
    // verify_state (physics_interface.py:316): where(q < 0, 0, q)
    in.q[k] = (verify && qraw[k].v < T(0)) ? A(T(0)) : qraw[k];
    in.phi[k] = leaf(h.phi[k]);
  }
  in.psa = leaf(h.psa);
  in.u_low = leaf(h.u_low);
  in.v_low = leaf(h.v_low);
  spdgen::ColumnOut<A> o;
  spdgen::column_generic<KX, A, T>(vg, p, g, h.flags, h.model_step, T(h.ablco2), h.S, in, o);
  for (int k = 0; k < KX; ++k) {
    A dq = o.dq[k];
    if (verify)  // verify_tendencies (physics_interface.py:334-340)
      dq = (qraw[k].v + T(dt_seconds) * dq.v >= T(0)) ? dq : -qraw[k] / T(dt_seconds);
    if (q_tend_scale != 1.0) dq = dq * T(q_tend_scale);
    tp.seed(o.dt[k].i, T(ct_dt[k]));
    tp.seed(dq.i, T(ct_dq[k]));
  }
  tp.seed(o.du_low.i, T(ct_du));
  tp.seed(o.dv_low.i, T(ct_dv));
  tp.reverse();
  for (int k = 0; k < KX; ++k) {
    g_t[k] = tp.grad(in.t[k].i);
    g_q[k] = tp.grad(qraw[k].i);
    g_phi[k] = tp.grad(in.phi[k].i);
  }
  *g_psa = tp.grad(in.psa.i);
  *g_u = tp.grad(in.u_low.i);
  *g_v = tp.grad(in.v_low.i);
  const A* ps[12] = {&g.psmin, &g.trcnv, &g.rhil, &g.rhbl, &g.entmax, &g.smf,
                     &g.trlsc, &g.rhlsc, &g.drhlsc, &g.rhblsc, &g.albcl, &g.albcls};
  for (int j = 0; j < 12; ++j) g_params[j] = tp.grad(ps[j]->i);
  return tp.overflow ? -1 : tp.n;
}

// The hand-written reverse pass, same arguments as vjp.
template <int KX, class T = double>
static int vjp_hand(const spd_vgrid_t& vg, const spd_params_t& p, const HostColumn& h,
                    const double* ct_dt, const double* ct_dq, double ct_du, double ct_dv,
                    double* g_t, double* g_q, double* g_phi, double* g_psa, double* g_u,
                    double* g_v, double* g_params, double dt_seconds = 1800.0,
                    double q_tend_scale = 1.0) {
  spdgen::DiffParams<T> g;
  fill_params(p, g);
  spdgen::ColumnIn<T, T> in;
  fill_in(h, in);
  spdvjp::Ctx x{&vg, &p, h.flags, h.model_step, h.S};
  T ct[2][KX];
  for (int k = 0; k < KX; ++k) {
    ct[0][k] = T(ct_dt[k]);
    ct[1][k] = T(ct_dq[k]);
  }
  spdvjp::Bar<KX, T> b;
  spd_desc_t d{};  // the orographic profile depends on the level count only
  d.kx = KX;
  const spd::Derived D = spd::derive_constants(&d, &vg, &p);
  spdvjp::column_vjp<KX, T>(x, g, T(h.ablco2), T(dt_seconds), T(q_tend_scale), in, ct[0], ct[1],
                            T(ct_du), T(ct_dv), b, D.qcorv, D.gamlat, D.pexp);
  for (int k = 0; k < KX; ++k) {
    g_t[k] = b.t[k];
    g_q[k] = b.q[k];
    g_phi[k] = b.phi[k];
  }
  *g_psa = b.psa;
  *g_u = b.u;
  *g_v = b.v;
  for (int j = 0; j < 12; ++j) g_params[j] = b.par[j];
  return 1;
}

// Float64 rollout of one column as a single-column instance (its own cloud-top level set at
// every step): the fused step (verify_state, physics, verify_tendencies) and the explicit
// update x += dt * tendency for T, q and the lowest-level winds.  x0: t[16], q[16], phi[16],
// psa, u, v.  ct: t[16], q[16], u, v.  Returns <ct, x_N>; with grad non-null, also the
// gradient of that with respect to x0 (same layout as x0) and the 12 parameters, by storing
// every state and applying the hand-written reverse pass from the last step to the first.
template <int KX>
static double rollout(const spd_vgrid_t& vg, const spd_params_t& p, const HostColumn& h,
                      const double* x0, int nsteps, double dt, const double* ct, double* grad,
                      double* gpar) {
  typedef spdgen::ColumnIn<double, double> In;
  std::vector<In> xs(nsteps + 1);
  fill_in(h, xs[0]);
  for (int k = 0; k < KX; ++k) {
    xs[0].t[k] = x0[k];
    xs[0].q[k] = x0[16 + k];
    xs[0].phi[k] = x0[32 + k];
  }
  xs[0].psa = x0[48];
  xs[0].u_low = x0[49];
  xs[0].v_low = x0[50];
  std::vector<uint32_t> S(nsteps);
  spdgen::DiffParams<double> g;
  fill_params(p, g);
  const uint32_t fl = h.flags & ~(uint32_t)SPD_FUSE_VERIFY;
  for (int n = 0; n < nsteps; ++n) {
    In xu = xs[n];
    for (int k = 0; k < KX; ++k) xu.q[k] = xs[n].q[k] < 0.0 ? 0.0 : xs[n].q[k];
    spdgen::ColumnOut<double> o;
    spdgen::column_generic<KX, double, double>(vg, p, g, fl, h.model_step + n, h.ablco2, 0u,
                                               xu, o);
    const int ic = o.icltop < 0 ? 0 : (o.icltop > KX - 1 ? KX - 1 : o.icltop);
    S[n] = 1u << ic;
    spdgen::column_generic<KX, double, double>(vg, p, g, fl, h.model_step + n, h.ablco2, S[n],
                                               xu, o);
    xs[n + 1] = xs[n];
    for (int k = 0; k < KX; ++k) {
      double dq = o.dq[k];
      if (!(xs[n].q[k] + dt * dq >= 0.0)) dq = -xs[n].q[k] / dt;
      xs[n + 1].t[k] += dt * o.dt[k];
      xs[n + 1].q[k] += dt * dq;
    }
    xs[n + 1].u_low += dt * o.du_low;
    xs[n + 1].v_low += dt * o.dv_low;
  }
  const In& xN = xs[nsteps];
  double loss = ct[32] * xN.u_low + ct[33] * xN.v_low;
  for (int k = 0; k < KX; ++k) loss += ct[k] * xN.t[k] + ct[16 + k] * xN.q[k];
  if (!grad) return loss;
  double xt[KX], xq[KX], phib[KX] = {}, xu_ = ct[32], xv_ = ct[33], psab = 0.0, par[12] = {};
  for (int k = 0; k < KX; ++k) {
    xt[k] = ct[k];
    xq[k] = ct[16 + k];
  }
  for (int n = nsteps - 1; n >= 0; --n) {
    spdvjp::Ctx x{&vg, &p, h.flags | (uint32_t)SPD_FUSE_VERIFY, h.model_step + n, S[n]};
    double ctt[KX], ctq[KX];
    for (int k = 0; k < KX; ++k) {
      ctt[k] = dt * xt[k];
      ctq[k] = dt * xq[k];
    }
    spdvjp::Bar<KX, double> b;
    spdvjp::column_vjp<KX, double>(x, g, h.ablco2, dt, 1.0, xs[n], ctt, ctq, dt * xu_, dt * xv_,
                                   b);
    for (int k = 0; k < KX; ++k) {
      xt[k] += b.t[k];
      xq[k] += b.q[k];
      phib[k] += b.phi[k];
    }
    xu_ += b.u;
    xv_ += b.v;
    psab += b.psa;
    for (int j = 0; j < 12; ++j) par[j] += b.par[j];
  }
  for (int k = 0; k < KX; ++k) {
    grad[k] = xt[k];
    grad[16 + k] = xq[k];
    grad[32 + k] = phib[k];
  }
  grad[48] = psab;
  grad[49] = xu_;
  grad[50] = xv_;
  for (int j = 0; j < 12; ++j) gpar[j] = par[j];
  return loss;
}

extern "C" {

double hc_rollout(const spd_vgrid_t* vg, const spd_params_t* p, const HostColumn* h,
                  const double* x0, int nsteps, double dt, const double* ct, double* grad,
                  double* gpar) {
  switch (h->kx) {
    case 8: return rollout<8>(*vg, *p, *h, x0, nsteps, dt, ct, grad, gpar);
    case 16: return rollout<16>(*vg, *p, *h, x0, nsteps, dt, ct, grad, gpar);
  }
  return 0.0;
}

#define HC_VJP_ARGS                                                                        \
  const spd_vgrid_t *vg, const spd_params_t *p, const HostColumn *h, const double *ct_dt, \
      const double *ct_dq, double ct_du, double ct_dv, double *g_t, double *g_q,          \
      double *g_phi, double *g_psa, double *g_u, double *g_v, double *g_params,           \
      double dt_seconds, double q_tend_scale
#define HC_VJP_PASS                                                                      \
  *vg, *p, *h, ct_dt, ct_dq, ct_du, ct_dv, g_t, g_q, g_phi, g_psa, g_u, g_v, g_params, \
      dt_seconds, q_tend_scale

// mode: 0 tape float64, 1 tape float32, 2 hand float64, 3 hand float32
int hc_vjp_any(int mode, HC_VJP_ARGS) {
  switch (h->kx * 4 + mode) {
    case 7 * 4 + 0: return vjp<7, double>(HC_VJP_PASS);
    case 7 * 4 + 1: return vjp<7, float>(HC_VJP_PASS);
    case 7 * 4 + 2: return vjp_hand<7, double>(HC_VJP_PASS);
    case 7 * 4 + 3: return vjp_hand<7, float>(HC_VJP_PASS);
    case 8 * 4 + 0: return vjp<8, double>(HC_VJP_PASS);
    case 8 * 4 + 1: return vjp<8, float>(HC_VJP_PASS);
    case 8 * 4 + 2: return vjp_hand<8, double>(HC_VJP_PASS);
    case 8 * 4 + 3: return vjp_hand<8, float>(HC_VJP_PASS);
    case 16 * 4 + 0: return vjp<16, double>(HC_VJP_PASS);
    case 16 * 4 + 1: return vjp<16, float>(HC_VJP_PASS);
    case 16 * 4 + 2: return vjp_hand<16, double>(HC_VJP_PASS);
    case 16 * 4 + 3: return vjp_hand<16, float>(HC_VJP_PASS);
  }
  return -2;
}

// hc_vjp_any over n columns: ct[n][34] holds each column's 16 temperature and 16 humidity
// cotangents and the lowest-level wind cotangents; out[n][63] receives the temperature,
// humidity and geopotential gradients (16 each), psa, u, v and the 12 parameter gradients.
// Returns n, or -1 - i for the first column i whose VJP failed.
int hc_vjp_batch(int mode, const spd_vgrid_t* vg, const spd_params_t* p, const HostColumn* hs,
                 int n, const double* ct, double* out, double dt_seconds,
                 double q_tend_scale) {
  for (int i = 0; i < n; ++i) {
    const double* c = ct + (size_t)i * 34;
    double* o = out + (size_t)i * 63;
    const int rc = hc_vjp_any(mode, vg, p, hs + i, c, c + 16, c[32], c[33], o, o + 16, o + 32,
                              o + 48, o + 49, o + 50, o + 51, dt_seconds, q_tend_scale);
    if (rc <= 0) return -1 - i;
  }
  return n;
}

int hc_vjp32(const spd_vgrid_t* vg, const spd_params_t* p, const HostColumn* h,
             const double* ct_dt, const double* ct_dq, double ct_du, double ct_dv, double* g_t,
             double* g_q, double* g_phi, double* g_psa, double* g_u, double* g_v,
             double* g_params) {
  switch (h->kx) {
    case 7: return vjp<7, float>(*vg, *p, *h, ct_dt, ct_dq, ct_du, ct_dv, g_t, g_q, g_phi, g_psa, g_u, g_v, g_params);
    case 8: return vjp<8, float>(*vg, *p, *h, ct_dt, ct_dq, ct_du, ct_dv, g_t, g_q, g_phi, g_psa, g_u, g_v, g_params);
    case 16: return vjp<16, float>(*vg, *p, *h, ct_dt, ct_dq, ct_du, ct_dv, g_t, g_q, g_phi, g_psa, g_u, g_v, g_params);
  }
  return -2;
}

int hc_fwd(const spd_vgrid_t* vg, const spd_params_t* p, const HostColumn* h, int f64,
           HostOut* out) {
  switch (h->kx) {
    case 7: f64 ? fwd<7, double>(*vg, *p, *h, *out) : fwd<7, float>(*vg, *p, *h, *out); return 0;
    case 8: f64 ? fwd<8, double>(*vg, *p, *h, *out) : fwd<8, float>(*vg, *p, *h, *out); return 0;
    case 16: f64 ? fwd<16, double>(*vg, *p, *h, *out) : fwd<16, float>(*vg, *p, *h, *out); return 0;
  }
  return -1;
}

int hc_vjp(const spd_vgrid_t* vg, const spd_params_t* p, const HostColumn* h,
           const double* ct_dt, const double* ct_dq, double ct_du, double ct_dv, double* g_t,
           double* g_q, double* g_phi, double* g_psa, double* g_u, double* g_v,
           double* g_params) {
  switch (h->kx) {
    case 7: return vjp<7>(*vg, *p, *h, ct_dt, ct_dq, ct_du, ct_dv, g_t, g_q, g_phi, g_psa, g_u, g_v, g_params);
    case 8: return vjp<8>(*vg, *p, *h, ct_dt, ct_dq, ct_du, ct_dv, g_t, g_q, g_phi, g_psa, g_u, g_v, g_params);
    case 16: return vjp<16>(*vg, *p, *h, ct_dt, ct_dq, ct_du, ct_dv, g_t, g_q, g_phi, g_psa, g_u, g_v, g_params);
  }
  return -2;
}

}  // extern "C"
